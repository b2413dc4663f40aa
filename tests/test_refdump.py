"""A simulation written as the reference's restart files (Dump_2D +
ParticleBundle%Dump) and read back into a fresh one (Restart_2D +
LoadParticleBundle): phi and E bit for bit, y (kept in L_ref units as the
reference's PosRes keeps it) bit for bit, x and the velocities to the
rounding of the SI round trip (x * L_ref / L_ref), and the next steps agree
(MCC off: restored particles get new ids, which key the collision draws)."""
import numpy as np
import pytest

from pic_b200 import deck, refdump
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _by_pos(p):
    o = np.lexsort((p["vx"], p["y"], p["x"]))
    return {k: v[o] for k, v in p.items()}


@pytest.mark.parametrize("name", ["tiny", "tiny_axi"])
def test_dump_restore_round_trip(tmp_path, name):
    cfg = deck.config(name)
    a = Simulation(cfg, mcc=False)
    try:
        a.initial_fields()
        for _ in range(3):
            a.step()
        refdump.dump(a, str(tmp_path), 3)
        phi_a, efx_a = a.field("phi"), a.field("efx")
        parts_a = [_by_pos(a.download(s)) for s in range(2)]
        counts = [a.count(s) for s in range(2)]
        a.step()
        after_a = a.field("phi")
    finally:
        a.close()
    b = Simulation(cfg, load=False, mcc=False, capacity=[2 * max(c, 1) + 1024 for c in counts])
    try:
        var = refdump.restore(b, str(tmp_path), 3)
        assert var["lap"] == 3 and var["ns"] == counts
        assert np.array_equal(b.field("phi"), phi_a) and np.array_equal(b.field("efx"), efx_a)
        for s in range(2):
            assert b.count(s) == counts[s]
            pb = _by_pos(b.download(s))
            assert np.array_equal(pb["y"], parts_a[s]["y"])
            for k in ("x", "vx", "vy", "vz"):
                assert np.allclose(pb[k], parts_a[s][k], rtol=4e-16, atol=0), (s, k)
            assert np.array_equal(pb["loc"], parts_a[s]["loc"])
        b.step()
        after_b = b.field("phi")
        assert np.abs(after_b - after_a).max() <= 1e-10 * np.abs(after_a).max()
    finally:
        b.close()
