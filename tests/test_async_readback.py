"""pic_get_fields_async and pic_set_field_async: the fields a step leaves
are copied to host, and the next phi copied in, on the library's copy stream
while the caller's next step pushes its particles; every reader or writer of
a field on the device waits for its copies.  Two identical runs, one with
synchronous pic_set_field / pic_get_field calls and one with the
asynchronous ones (each step's phi goes back in from the array the previous
step's readback filled, as a Fortran caller passes Phi in), give identical
fields and an identical final state."""
import ctypes as C

import numpy as np
import pytest
import torch

from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

FIELDS = (("rho", 0), ("phi", 1), ("efx", 2), ("efy", 3))


def _pinned(n):
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()


@pytest.mark.parametrize("precision", [api.PIC_PREC_FP64, api.PIC_PREC_MIXED])
def test_async_readback_matches_synchronous(precision):
    cfg = deck.config("cfg1", precision=precision)
    steps = 4
    runs = []
    for overlap in (False, True):
        sim = Simulation(cfg)
        try:
            sim.initial_fields()
            nn = sim.mesh.nn
            lib = sim.lib
            bufs = [{k: _pinned(nn) for k, _ in FIELDS} for _ in range(steps)]
            phi_in = _pinned(nn)
            phi_in[:] = sim.field("phi")
            for t in range(steps):
                src = phi_in if t == 0 else bufs[t - 1]["phi"]
                if overlap:
                    api.check(lib.pic_set_field_async(1, api.dptr(src)), "async set phi")
                else:
                    api.check(lib.pic_set_field(1, api.dptr(src)), "set phi")
                sim.step()
                if overlap:
                    b = bufs[t]
                    api.check(lib.pic_get_fields_async(api.dptr(b["rho"]), api.dptr(b["phi"]),
                                                       api.dptr(b["efx"]), api.dptr(b["efy"])), "async")
                else:
                    for k, w in FIELDS:
                        api.check(lib.pic_get_field(w, api.dptr(bufs[t][k])), "get")
            api.check(lib.pic_wait_fields(), "wait")
            final = (sim.field("rho"), sim.field("phi"), [sim.count(s) for s in range(2)])
            runs.append(([{k: v.copy() for k, v in b.items()} for b in bufs], final))
        finally:
            sim.close()
    (ba, fa), (bb, fb) = runs
    for t in range(steps):
        for k, _ in FIELDS:
            assert np.array_equal(ba[t][k], bb[t][k]), (t, k)
    assert np.array_equal(fa[0], fb[0]) and np.array_equal(fa[1], fb[1]) and fa[2] == fb[2]
