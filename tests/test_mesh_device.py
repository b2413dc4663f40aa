"""pic_mesh_build_device: the interface elements' Q1 IFE basis, element
stiffness and load matrices built in FP64 on the GPU (one thread per
interface element, the host builder's own code compiled for the device)
give the descriptor of the host builder bit for bit, Cartesian and r-z."""
import ctypes as C

import numpy as np
import pytest

from pic_b200 import api, deck

pytestmark = pytest.mark.gpu

ARRAYS = ("node_type", "node_index", "element_index", "phi_dirichlet", "cell_volume", "a_srow", "a_jcol", "a_k",
          "xt_srow", "xt_jcol", "xt_k", "a_diag", "mass_q1", "ife_mass", "patch_ptr", "patch_nodes")


@pytest.mark.parametrize("name,over", [("tiny", {}), ("tiny_axi", {}), ("cfg1", {}),
                                       ("cfg4", dict(ncx=256, ncy=256)), ("cfg5", dict(ncx=256, ncy=128))])
def test_device_interface_elements_match_host(name, over):
    cfg = deck.config(name, **over)
    host = deck.Mesh(cfg, device=False)
    dev = deck.Mesh(cfg, device=True)
    try:
        assert host.desc.n_interface == dev.desc.n_interface > 0
        for a in ARRAYS + (("mass_rows",) if cfg.delta == 1 else ()):
            assert np.array_equal(host.array(a), dev.array(a)), a
        # the basis itself, through the builder's query, at each element's centre
        lib = api.load()
        for k in range(1, host.desc.n_interface + 1, max(1, host.desc.n_interface // 50)):
            el = C.c_int32()
            api.check(lib.pic_mesh_interface_info(host.ptr, k, C.byref(el), None, None, None, None, None), "info")
            e = el.value - 1
            i, j = e // (host.nny - 1), e % (host.nny - 1)
            x = host.desc.xmin + (i + 0.37) * host.hx
            y = host.desc.ymin + (j + 0.61) * host.hy
            for b in range(4):
                vh, vd = C.c_double(), C.c_double()
                api.check(lib.pic_mesh_ife_basis(host.ptr, k, b, x, y, C.byref(vh), None, None), "basis")
                api.check(lib.pic_mesh_ife_basis(dev.ptr, k, b, x, y, C.byref(vd), None, None), "basis")
                assert vh.value == vd.value, (k, b)
    finally:
        host.close()
        dev.close()
