"""MCC_jw collision tables: the product's builder (pic_b200/mcc_tables.py)
against the oracle's own restatement (oracle/oracle_tables.c) of
SigmaNormalizedUpdate (mc/MCCSigma.f90:123-172), ProbilityNonReactive
(mc/MCCInit.F90:107-152) and the null-collision ratio (MCCInit.F90:54), and
the cross-section data the product ships (pic_b200/data/ar_pegasus.json)
against a digest of the reference's raw Pegasus files
(tests/golden/pegasus_ar_digest.json, written by tests/golden/make_golden.py
with a parser of its own).  CPU only."""
import json
import os

import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import deck, mcc_tables

HERE = os.path.dirname(os.path.abspath(__file__))


def _data():
    return json.load(open(mcc_tables.DATA))


def test_shipped_cross_sections_match_the_raw_pegasus_files():
    dig = json.load(open(os.path.join(HERE, "golden", "pegasus_ar_digest.json")))
    data = _data()
    for key, bundle in (("ElectronAr.txt", data["electron"]), ("Ar(+)Ar.txt", data["ion"])):
        g = dig[key]
        assert bundle["model"] == g["model"]
        assert len(bundle["reactions"]) == len(g["reactions"])
        for r, gr in zip(bundle["reactions"], g["reactions"]):
            t = np.array(r["table"])
            assert r["index"] == gr["index"] and r["threshold"] == gr["threshold"]
            assert r["pegasus_type"] == gr["type"] and len(t) == gr["n"]
            assert sum(t[:, 0].tolist()) == gr["sum_e"] and sum(t[:, 1].tolist()) == gr["sum_sigma_cm2"]
            assert t[0].tolist() == gr["first"] and t[-1].tolist() == gr["last"]


@pytest.mark.parametrize("species", ["electron", "ion"])
@pytest.mark.parametrize("cfg_name", ["cfg1", "cfg5"])
def test_tables_match_the_oracle(species, cfg_name):
    """sigma(E) on the grid, the cumulative probabilities and P_null,
    bit for bit (the same FP64 operations in the same order)."""
    cfg = deck.config(cfg_name)
    dt_s = cfg.dt * cfg.scales["time_ref"]
    n_gas = cfg.gas_p_Pa / (deck.KB * cfg.gas_T_K)
    data = _data()[species]
    mass = deck.ME if species == "electron" else deck.AR_MASS
    t, prob, pmax = mcc_tables.build_table(data, 0 if species == "electron" else 1, mass, deck.AR_MASS,
                                           n_gas, dt_s, 1 if species == "electron" else -1,
                                           species == "ion")
    sig_o, prob_o, pmax_o, ratio_o, emax_o = ob.mcc_table(data, mass, deck.AR_MASS, n_gas, dt_s)
    emin, _ = (-3.0, 3.0) if data["model"] == 1 else (-1.0, 3.0)
    eint = t.energy_interval
    for j, r in enumerate(data["reactions"]):
        sig_p = mcc_tables.sigma_table(r, emin, eint, 10001)
        assert np.array_equal(sig_p, sig_o[j]), j
    assert np.array_equal(prob, prob_o)
    assert pmax == pmax_o and t.collision_ratio == ratio_o and t.energy_max == emax_o
    # cumulative, normalised: the last reaction's column reaches 1 somewhere
    assert np.all(np.diff(prob_o, axis=1) >= 0) and prob_o.max() == 1.0


def test_sigma_interpolation_known_answers():
    """Closed-form checks of the restated interpolation on a one-segment
    table: 0 at and below threshold; between the raw points linear in
    grid-index space with the reference's index shift (its S1 uses the
    1-based grid index i against 0-based raw positions); Alfa/E at and above
    the last raw energy; cm^2 -> m^2."""
    bundle = {"model": 1, "reactions": [{"threshold": 1.0, "table": [[1.0, 0.0], [100.0, 4e-16]]}]}
    sig, _, _, _, _ = ob.mcc_table(bundle, deck.ME, deck.AR_MASS, 1e20, 1e-12)
    emin, eint = -3.0, 6.0 / 10000
    m = np.arange(10001)
    E = np.array([10.0 ** (emin + k * eint) for k in m])
    s = sig[0]
    assert np.all(s[E <= 1.0] == 0.0)
    hi = E >= 100.0
    assert np.allclose(s[hi], 4e-20 * 100.0 / E[hi], rtol=1e-15, atol=0)
    le, ue = (0.0 - emin) / eint, (2.0 - emin) / eint
    mid = (E > 1.0) & (E < 100.0)
    want = ((m[mid] + 1) - le) / (ue - le) * 4e-20
    assert np.allclose(s[mid], want, rtol=1e-12, atol=0)
