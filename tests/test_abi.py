"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/picgpu.h; CPU-side error paths need no device."""
import ctypes as C
import os
import re

from pic_b200 import api, deck

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "picgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pic_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    lib = api.load()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(api.EXPORTS) == names


def test_calls_before_init_fail_cleanly():
    lib = api.load()
    lib.pic_finalize()
    rc = lib.pic_step(1, None)
    assert rc == -6
    assert b"pic_init" in lib.pic_last_error()
    import numpy as np
    out = np.zeros(64)
    cnt = np.zeros(8, np.int64)
    assert lib.pic_average_x(api.dptr(out)) == -6
    assert lib.pic_energy_spectrum(0, 8, 5.0, 1.0, api.lptr(cnt), api.lptr(cnt)) == -6
    assert b"pic_init" in lib.pic_last_error()
    assert lib.pic_velocity_moments(0, 8, api.lptr(cnt), api.dptr(out), api.dptr(out)) == -6
    assert lib.pic_set_wall_rf(0, 1.0, 13.56e6, 0.0) == -6


def test_mesh_builder_rejects_bad_decks():
    lib = api.load()
    d = deck.make_deck(deck.config("tiny"))
    d.nnx = 2
    ptr = C.POINTER(api.MeshDesc)()
    assert lib.pic_mesh_build(C.byref(d), C.byref(ptr)) == -1
    d = deck.make_deck(deck.config("tiny"))
    d.delta = 2  # neither Cartesian (0) nor axisymmetric (1)
    assert lib.pic_mesh_build(C.byref(d), C.byref(ptr)) == -1
    # two overlapping objects
    d = deck.make_deck(deck.config("tiny"))
    d.n_objects = 2
    d.objects[1] = d.objects[0]
    assert lib.pic_mesh_build(C.byref(d), C.byref(ptr)) == -8
