"""pic_deposit_noalloc: the allocation-free charge deposit, for callers that
cannot allocate device memory (their device memory comes from an arena owned
by another framework, or their loop must not pay cudaMalloc's implicit
synchronisation).  Called through the C-ABI and compared with the density
that the allocating path (pic_get_par_chg) produces for the same particles,
twice in a row so a stale accumulator from the first call would show.

This file is collected last so that a run stopping at the first failure has
run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def test_noalloc_deposit_matches_get_par_chg():
    import torch

    lib = api.load()
    sim = Simulation(deck.config("cfg1"))
    try:
        sim.get_par_chg()
        m = sim.mesh
        dev_vol = torch.tensor(m.array("cell_volume"), dtype=torch.float64, device="cuda")
        for s, name in ((0, "rho_e"), (1, "rho_i")):
            want = sim.field(name)
            ptrs = (C.c_void_p * 7)()
            nslots = C.c_int64()
            api.check(lib.pic_particle_device_ptrs(s, ptrs, C.byref(nslots)), "ptrs")
            wq = sim.species[s][2] * sim.species[s][0]
            for call in range(2):
                out = torch.full((m.nn,), float("nan"), dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                rc = lib.pic_deposit_noalloc(m.nnx, m.nny, m.desc.xmin, m.desc.xmax, m.desc.ymin,
                                             m.desc.ymax, nslots.value, ptrs[0], ptrs[1], ptrs[5],
                                             dev_vol.data_ptr(), wq, sim.scales["L_ref"], sim.cfg.n0,
                                             out.data_ptr(), None)
                assert rc == 0, lib.pic_last_error()
                torch.cuda.synchronize()
                got = out.cpu().numpy()
                # same fixed-point algorithm: identical bits (tolerance 0)
                assert np.array_equal(got, want), (s, call, np.abs(got - want).max())
        # meshes above the static scratch are refused before any launch
        big = int(np.ceil(np.sqrt(api_max_nodes() + 1))) + 1
        rc = lib.pic_deposit_noalloc(big, big, 0.0, 1.0, 0.0, 1.0, 0, None, None, None,
                                     dev_vol.data_ptr(), 1.0, 1.0, 1.0, dev_vol.data_ptr(), None)
        assert rc == -1 and b"static scratch" in lib.pic_last_error()
    finally:
        sim.close()


def test_noalloc_inputs_refused_in_mixed_precision():
    """A mixed-precision context stores FP32 element offsets where the FP64
    layout keeps positions: its particle buffers are not valid input for the
    allocation-free deposit, and the zero-copy pointer query refuses them
    rather than hand out buffers that would be misread as doubles."""
    lib = api.load()
    sim = Simulation(deck.config("tiny", precision=api.PIC_PREC_MIXED))
    try:
        ptrs = (C.c_void_p * 7)()
        nslots = C.c_int64()
        rc = lib.pic_particle_device_ptrs(0, ptrs, C.byref(nslots))
        assert rc == api.PIC_ERR_STATE, rc
        assert b"mixed-precision layout" in lib.pic_last_error()
        assert ptrs[0] is None  # nothing handed out
    finally:
        sim.close()


def api_max_nodes():
    import os
    import re
    h = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                          "include", "picgpu.h")).read()
    return int(re.search(r"#define PIC_NOALLOC_MAX_NODES (\d+)", h).group(1))
