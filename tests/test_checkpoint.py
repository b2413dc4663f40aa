"""Checkpoint and restart (pic_b200.checkpoint): a run restored from a
checkpoint continues bit for bit like the uninterrupted run (particles by
id, counts, rho, phi), in FP64 and mixed precision, across a counting sort
and MCC steps; restore refuses a checkpoint of another deck."""
import numpy as np
import pytest

from pic_b200 import api, checkpoint, deck


def _by_id(p):
    o = np.argsort(p["id"])
    return {k: v[o] for k, v in p.items()}


def _state(sim):
    return ([_by_id(sim.download(s)) for s in range(2)], sim.field("rho"), sim.field("phi"),
            [sim.count(s) for s in range(2)])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [api.PIC_PREC_FP64, api.PIC_PREC_MIXED])
def test_restart_continues_bit_for_bit(prec, tmp_path):
    from pic_b200.simulation import Simulation
    cfg = deck.config("cfg1", precision=prec)
    path = str(tmp_path / "run.npz")
    sim = Simulation(cfg)
    try:
        sim.initial_fields()
        for _ in range(7):
            sim.step()
        checkpoint.save(sim, path)
        for _ in range(7):  # the counting sort runs at step 10
            sim.step()
        want = _state(sim)
    finally:
        sim.close()
    sim = checkpoint.restore(cfg, path)
    try:
        assert sim.step_index == 7
        for _ in range(7):
            sim.step()
        got = _state(sim)
        # a next id below the one in use is refused (ids would repeat)
        assert sim.lib.pic_set_next_id(0, 0) == api.PIC_ERR_ARG
    finally:
        sim.close()
    (pa, ra, fa, na), (pb, rb, fb, nb) = want, got
    assert na == nb
    for a, b in zip(pa, pb):
        for k in ("id", "loc", "x", "y", "vx", "vy", "vz"):
            assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(ra, rb) and np.array_equal(fa, fb)


def test_restore_rejects_another_deck(tmp_path):
    """Checked before anything touches the device."""
    cfg = deck.config("cfg1")
    path = str(tmp_path / "other.npz")
    np.savez(path, version=np.int64(checkpoint._VERSION), step=np.int64(3), nnx=np.int64(cfg.ncx + 2),
             nny=np.int64(cfg.ncy + 1), seed=np.uint64(cfg.seed), precision=np.int64(cfg.precision),
             n_species=np.int64(2), phi=np.zeros(4), physics=checkpoint._physics(cfg))
    with pytest.raises(ValueError, match="nnx"):
        checkpoint.restore(cfg, path)
    np.savez(path, version=np.int64(1))
    with pytest.raises(ValueError, match="version"):
        checkpoint.restore(cfg, path)


def _fake(path, cfg, physics):
    np.savez(path, version=np.int64(checkpoint._VERSION), step=np.int64(3), nnx=np.int64(cfg.ncx + 1),
             nny=np.int64(cfg.ncy + 1), seed=np.uint64(cfg.seed), precision=np.int64(cfg.precision),
             n_species=np.int64(2), phi=np.zeros(4), physics=physics)


@pytest.mark.parametrize("change,field", [
    ({"delta": 1}, "delta"), ({"dt": 0.04}, "dt"), ({"n0": 2e15}, "n0"),
    ({"ppc": 40}, "species0_weight"), ({"gas_p_Pa": 2.0}, "gas_p_Pa"),
    ({"rf": (0, 100.0, 13.56e6)}, "rf_wall"),
])
def test_restore_rejects_other_physics_on_the_same_mesh(tmp_path, change, field):
    """A checkpoint of a deck with the same mesh size and seed but other
    physics is refused, naming the first parameter that differs."""
    cfg = deck.config("cfg1")
    path = str(tmp_path / "phys.npz")
    _fake(path, deck.config("cfg1", **change), checkpoint._physics(deck.config("cfg1", **change)))
    with pytest.raises(ValueError, match=field):
        checkpoint.restore(cfg, path)
