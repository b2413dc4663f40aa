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


class _FakeSim:
    """The parts of Simulation that dump/restore use, on host arrays."""

    def __init__(self, nnx=5, nny=4, delta=0, n=(6, 3), seed=1):
        from types import SimpleNamespace
        rng = np.random.default_rng(seed)
        self.cfg = SimpleNamespace(delta=delta)
        self.mesh = SimpleNamespace(nnx=nnx, nny=nny, nn=nnx * nny)
        self.scales = {"L_ref": 2.5e-4, "v_ref": 5.9e5}
        self.species = [(-1.0, 9.1095e-31, 3.0e3, 0.0), (1.0, 6.63e-26, 3.0e3, 0.0)]
        self.parts = [{"x": rng.random(k), "y": rng.random(k), "vx": rng.standard_normal(k),
                       "vy": rng.standard_normal(k), "vz": rng.standard_normal(k),
                       "loc": rng.integers(0, (nnx - 1) * (nny - 1), k).astype(np.int32)} for k in n]
        self.phi = rng.standard_normal(nnx * nny)
        self.uploaded, self.step_index, self.ppr_calls = {}, 0, 0

    def download(self, s):
        return {k: v.copy() for k, v in self.parts[s].items()}

    def field(self, name):
        assert name == "phi"
        return self.phi.copy()

    def upload(self, s, x, y, vx, vy, vz):
        self.uploaded[s] = (x, y, vx, vy, vz)

    def set_field(self, name, v):
        assert name == "phi"
        self.phi = np.asarray(v).copy()

    def get_efield_ppr(self):
        self.ppr_calls += 1


def test_dump_writes_reference_units_and_restore_inverts_them(tmp_path):
    a = _FakeSim()
    rd.dump(a, str(tmp_path), 40, period_res=12.5, istep_previous=3, nperiod=1)
    var = rd.read_var(rd.var_path(str(tmp_path), 40), 2)
    assert var == {"lap": 40, "ntot": 9, "ns": [6, 3], "nx": 5, "ny": 4, "period_res": 12.5,
                   "istep_previous": 3, "nperiod": 1}
    r = rd.read_particles(str(tmp_path / "10000Electron.dat"))
    p = a.parts[0]
    L, V = a.scales["L_ref"], a.scales["v_ref"]
    assert np.array_equal(r["X"], p["x"] * L) and np.array_equal(r["Y"], p["y"])  # PosRes scales X alone
    assert np.array_equal(r["Vz"], p["vz"] * V) and np.all(r["Z"] == 0.0)
    assert np.array_equal(r["Location"], p["loc"] + 1)
    assert r["charge"] == -1.6022e-19 and r["weight"] == 3.0e3
    b = _FakeSim(seed=2)
    got = rd.restore(b, str(tmp_path), 40)
    assert got["lap"] == 40 and b.step_index == 40 and b.ppr_calls == 1
    assert np.array_equal(b.phi, a.phi)
    x, y, vx, vy, vz = b.uploaded[1]
    q = a.parts[1]
    assert np.array_equal(y, q["y"])
    assert np.allclose(x, q["x"], rtol=4e-16, atol=0) and np.allclose(vz, q["vz"], rtol=4e-16, atol=0)


def test_restore_refuses_another_mesh_or_inconsistent_counts(tmp_path):
    rd.dump(_FakeSim(), str(tmp_path), 7)
    with pytest.raises(ValueError, match="node mesh"):
        rd.restore(_FakeSim(nnx=6), str(tmp_path), 7)
    # the var file says 6 electrons; a particle file holding 5 is refused
    rd.write_particles(str(tmp_path / "10000Electron.dat"), -1.6022e-19, 9.1095e-31, 1.0, _cols(5), 5)
    with pytest.raises(ValueError, match="particles in its file"):
        rd.restore(_FakeSim(), str(tmp_path), 7)


def test_restore_rotates_rz_velocities_into_the_particle_frame(tmp_path):
    a = _FakeSim(delta=1)
    rd.dump(a, str(tmp_path), 1)
    # a reference-written file: the same particles at angle pi/2, velocities Cartesian
    f = str(tmp_path / "10000Ar(+).dat")
    r = rd.read_particles(f)
    ang = np.full(r["npar"], math.pi / 2)
    cols = {k: r[k] for k in ("X", "Y", "Vx", "Ax", "Ay", "Az", "Wq", "Location")}
    cols["Z"] = ang
    cols["Vy"] = -r["Vz"]  # (v_r, v_theta) at angle pi/2 in Cartesian components
    cols["Vz"] = r["Vy"]
    rd.write_particles(f, r["charge"], r["mass"], r["weight"], cols, r["npar_normal"])
    b = _FakeSim(delta=1)
    rd.restore(b, str(tmp_path), 1)
    x, y, vx, vy, vz = b.uploaded[1]
    q = a.parts[1]
    assert np.allclose(vy, q["vy"], rtol=1e-14, atol=1e-14) and np.allclose(vz, q["vz"], rtol=1e-14, atol=1e-14)
