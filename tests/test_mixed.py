"""Mixed precision (PIC_PREC_MIXED): particles as element + FP32 offsets and
FP32 velocities, FP32 field records, int64 fixed-point deposit.  Checked
against the FP64 path -- which is bit-exact with the oracle
(test_gpu_parity.py) -- on the same seeded inputs.

Bars: positions to 1e-6 of a cell after upload/download and 1e-5 of a cell
after one push; velocities to 1e-6 relative; node charge to 1e-6 of the
largest node value after one step; total charge exact to the fixed-point
rounding of each weight; after 20 steps with MCC, phi and E within 1e-3 of
their largest magnitude (FP32 rounding grows with the plasma's own
sensitivity to initial conditions) and the same particle counts to 1%.
"""
import numpy as np
import pytest

from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _pair(name="cfg1", **over):
    sims = []
    for prec in (api.PIC_PREC_FP64, api.PIC_PREC_MIXED):
        cfg = deck.config(name, precision=prec, **over)
        sims.append(Simulation(cfg))
    return sims


def _by_id(p):
    o = np.argsort(p["id"])
    return {k: v[o] for k, v in p.items()}


def test_mixed_upload_download_round_trip():
    d, m = _pair()
    try:
        hx = m.mesh.hx
        for s in range(2):
            a, b = _by_id(d.download(s)), _by_id(m.download(s))
            assert np.array_equal(a["id"], b["id"]) and np.array_equal(a["loc"], b["loc"])
            assert np.abs(a["x"] - b["x"]).max() <= 1e-6 * hx
            assert np.abs(a["y"] - b["y"]).max() <= 1e-6 * hx
            for v in ("vx", "vy", "vz"):
                assert np.allclose(a[v], b[v], rtol=1e-6, atol=1e-6 * np.abs(a[v]).max())
    finally:
        d.close()
        m.close()


def test_mixed_push_and_deposit_match_fp64():
    d, m = _pair()
    try:
        for sim in (d, m):
            sim.initial_fields()
        rho_d, rho_m = d.field("rho"), m.field("rho")
        assert np.abs(rho_d - rho_m).max() <= 1e-6 * np.abs(rho_d).max()
        for sim in (d, m):
            for s in range(2):
                sim.move_all(s)
            sim.get_par_chg()
        hx = d.mesh.hx
        for s in range(2):
            a, b = _by_id(d.download(s)), _by_id(m.download(s))
            common, ia, ib = np.intersect1d(a["id"], b["id"], return_indices=True)
            assert common.size >= 0.999 * max(a["id"].size, b["id"].size)
            assert np.abs(a["x"][ia] - b["x"][ib]).max() <= 1e-5 * hx
            assert np.abs(a["y"][ia] - b["y"][ib]).max() <= 1e-5 * hx
            assert np.allclose(a["vx"][ia], b["vx"][ib], rtol=1e-5, atol=1e-5 * np.abs(a["vx"]).max())
        rho_d, rho_m = d.field("rho"), m.field("rho")
        assert np.abs(rho_d - rho_m).max() <= 1e-4 * np.abs(rho_d).max()
    finally:
        d.close()
        m.close()


def test_mixed_charge_is_conserved():
    """Each particle deposits four fixed-point weights that sum to 2^40 within
    2 units in either precision, so the total charge of the mixed path equals
    the FP64 path's to that rounding (relative 1e-10)."""
    d, m = _pair()
    try:
        vol = d.mesh.array("cell_volume")
        for sim in (d, m):
            sim.get_par_chg()
        for f in ("rho_e", "rho_i"):
            td, tm = (d.field(f) * vol).sum(), (m.field(f) * vol).sum()
            assert abs(td - tm) <= 1e-10 * abs(td)
    finally:
        d.close()
        m.close()


def test_mixed_steps_track_fp64():
    d, m = _pair("cfg1", ppc=20)
    try:
        for sim in (d, m):
            sim.initial_fields()
        for _ in range(20):
            d.step()
            m.step()
        for f in ("phi", "efx", "efy"):
            a, b = d.field(f), m.field(f)
            err = np.abs(a - b).max() / np.abs(a).max()
            print(f"\n20 steps: {f} max |mixed - fp64| / max|fp64| = {err:.2e}")
            assert err <= 1e-3
        for s in range(2):
            na, nb = d.count(s), m.count(s)
            assert abs(na - nb) <= 0.01 * na
    finally:
        d.close()
        m.close()
