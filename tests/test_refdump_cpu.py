"""The reference's restart files (Dump_2D.f90, Restart_2D.f90,
ParticleBundle.f90:286-375) as pic_b200.refdump writes and reads them:
the byte layout of Fortran unformatted sequential records (payload between
two int32 byte counts), the 84-byte ParticleOne record, the list-directed
var file, round trips, the compiler-dependent particle file name, the r-z
velocity frame, and refusal of damaged files.  CPU only."""
import math
import os

import numpy as np
import pytest

from pic_b200 import refdump as rd


def test_phi_file_is_one_record(tmp_path):
    p = str(tmp_path / "phi0000012dump")
    rd.write_phi(p, np.array([1.5, -2.0, 3.25]))
    b = open(p, "rb").read()
    assert len(b) == 4 + 24 + 4
    assert np.frombuffer(b[:4], "<i4")[0] == 24 and np.frombuffer(b[-4:], "<i4")[0] == 24
    assert np.array_equal(np.frombuffer(b[4:28], "<f8"), [1.5, -2.0, 3.25])
    assert np.array_equal(rd.read_phi(p), [1.5, -2.0, 3.25])


def _cols(n, seed=0):
    rng = np.random.default_rng(seed)
    c = {k: rng.standard_normal(n) for k in ("X", "Y", "Z", "Vx", "Vy", "Vz", "Ax", "Ay", "Az", "Wq")}
    c["Location"] = rng.integers(1, 1000, n)
    return c


def test_particle_file_layout(tmp_path):
    p = str(tmp_path / "10000Electron.dat")
    c = _cols(2)
    rd.write_particles(p, -1.6022e-19, 9.1095e-31, 123.0, c, 7)
    b = open(p, "rb").read()
    # [NPar, NParNormal] int32, [Charge, Mass, Weight] float64, 2 x (84-byte record)
    assert len(b) == (4 + 8 + 4) + (4 + 24 + 4) + 2 * (4 + 84 + 4)
    assert list(np.frombuffer(b[0:16], "<i4")) == [8, 2, 7, 8]
    assert np.frombuffer(b[16:20], "<i4")[0] == 24
    assert list(np.frombuffer(b[20:44], "<f8")) == [-1.6022e-19, 9.1095e-31, 123.0]
    r0 = 48  # first particle record
    assert np.frombuffer(b[r0:r0 + 4], "<i4")[0] == 84
    vals = np.frombuffer(b[r0 + 4:r0 + 84], "<f8")
    assert np.array_equal(vals, [c[k][0] for k in ("X", "Y", "Z", "Vx", "Vy", "Vz", "Ax", "Ay", "Az", "Wq")])
    assert np.frombuffer(b[r0 + 84:r0 + 88], "<i4")[0] == c["Location"][0]
    assert np.frombuffer(b[r0 + 88:r0 + 92], "<i4")[0] == 84
    r = rd.read_particles(p)
    assert r["npar"] == 2 and r["npar_normal"] == 7 and r["weight"] == 123.0
    for k in c:
        assert np.array_equal(r[k], c[k]), k


def test_var_file_round_trip_and_fortran_forms(tmp_path):
    p = str(tmp_path / "var0001000dump")
    rd.write_var(p, 1000, [120, 95], 65, 33, 8300.5, 7, 2)
    v = rd.read_var(p, 2)
    assert v == {"lap": 1000, "ntot": 215, "ns": [120, 95], "nx": 65, "ny": 33, "period_res": 8300.5,
                 "istep_previous": 7, "nperiod": 2}
    # what a Fortran list-directed WRITE gives (padding, D exponent, comma) reads the same
    with open(p, "w") as f:
        f.write("        1000\n         215\n         120          95\n          65,33\n"
                "   8300.5000000000000D+00\n           7\n           2\n")
    assert rd.read_var(p, 2)["period_res"] == 8300.5 and rd.read_var(p, 2)["nx"] == 65


def test_particle_file_name_with_blanks(tmp_path):
    rd.write_particles(str(tmp_path / "       10000 Ar(+).dat"), 1.6022e-19, 6.63e-26, 1.0, _cols(3), 3)
    f = rd.find_particle_file(str(tmp_path), "Ar(+)")
    assert rd.read_particles(f)["npar"] == 3
    with pytest.raises(FileNotFoundError):
        rd.find_particle_file(str(tmp_path), "Electron")


def test_damaged_files_are_refused(tmp_path):
    p = str(tmp_path / "phi")
    rd.write_phi(p, np.arange(10.0))
    b = open(p, "rb").read()
    open(p, "wb").write(b[:-6])
    with pytest.raises(ValueError):
        rd.read_phi(p)
    q = str(tmp_path / "10000Electron.dat")
    rd.write_particles(q, -1.0, 1.0, 1.0, _cols(4), 4)
    b = open(q, "rb").read()
    open(q, "wb").write(b[:-92])  # one particle record short of its header
    with pytest.raises(ValueError):
        rd.read_particles(q)


def test_rz_frame_of_reference_velocities():
    """A particle at angle Z with Cartesian transverse velocity (Vy, Vz):
    radial and azimuthal components in its own frame."""
    z = np.array([0.0, math.pi / 2, math.pi, 0.3])
    vy = np.array([1.0, 1.0, 2.0, math.cos(0.3)])
    vz = np.array([0.5, 0.0, 0.0, math.sin(0.3)])
    vr, vt = rd.transverse_to_frame(z, vy, vz)
    assert np.allclose(vr, [1.0, 0.0, -2.0, 1.0], atol=1e-15)
    assert np.allclose(vt, [0.5, -1.0, 0.0, 0.0], atol=1e-15)
    # at angle 0 the frames coincide: what dump writes reads back unchanged
    a, b = rd.transverse_to_frame(np.zeros(3), np.array([1.0, 2.0, 3.0]), np.array([4.0, 5.0, 6.0]))
    assert np.array_equal(a, [1.0, 2.0, 3.0]) and np.array_equal(b, [4.0, 5.0, 6.0])
