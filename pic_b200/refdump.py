"""The reference's restart files, written from and read into a Simulation.

Dump_2D(lap) (code/PIC/Dump_2D.f90:30-72) and, per species,
ParticleBundle%Dump(0) (MCC_jw/code/base/ParticleBundle.f90:286-331);
read back as Restart_2D (code/PIC/Restart_2D.f90:37-79) and LoadParticleBundle
(ParticleBundle.f90:333-375) do:

    DUMP/var%07ddump   list-directed text, one value group a line: lap; ntot;
                       ns(1..n_species); nx, ny; Period_res; iStep_previous;
                       nPeriod (the last three are the RF bookkeeping of the
                       main loop)
    DUMP/phi%07ddump   Fortran unformatted sequential, one record:
                       phi(1:Field_Size), float64, in node order
    10000<Name>.dat    Fortran unformatted sequential, per species:
                       [NPar, NParNormal] int32; [Charge, Mass, Weight]
                       float64; then one record a particle: X, Y, Z, Vx, Vy,
                       Vz, Ax, Ay, Az, Wq float64 and Location int32 (84
                       bytes); the bundle is rescaled before the write by
                       PosRes, which scales X alone (ParticleOne.f90,
                       PositionRescaleParticleOne), and VelRes: X in metres,
                       Y in L_ref units, velocities in m/s

A Fortran unformatted sequential record is its payload between two int32
byte counts (little-endian, as gfortran and ifort write records below 2 GiB),
a derived type's components one after another without padding.
The name 10000<Name>.dat is DefaultNameIndex (MCC_jw/code/base/ControlFlow.f90:12)
and the species' name; the reference builds it with a list-directed internal
write, whose blanks depend on the compiler, so the reader also accepts a
name with blanks around the index.

On an r-z mesh (delta = 1) the reference keeps the angle in Z and Cartesian
transverse velocities (Vy, Vz) (code/IMPIC/MoveOne.f90:246-260); the
simulation holds (v_z, v_r, v_theta) in the particle's own frame, which is the
Cartesian frame at angle 0: the dump writes Z = 0, (Vy, Vz) = (v_r, v_theta),
and the restore rotates (Vy, Vz) by -Z.
"""
from __future__ import annotations

import glob
import os

import numpy as np

from .deck import QE

NAME_INDEX = 10000
SPECIES_NAMES = ("Electron", "Ar(+)")  # the cross-section files ElectronAr.txt, Ar(+)Ar.txt

PARTICLE_RECORD = np.dtype([("head", "<i4"), ("X", "<f8"), ("Y", "<f8"), ("Z", "<f8"), ("Vx", "<f8"),
                            ("Vy", "<f8"), ("Vz", "<f8"), ("Ax", "<f8"), ("Ay", "<f8"), ("Az", "<f8"),
                            ("Wq", "<f8"), ("Location", "<i4"), ("tail", "<i4")])
_PAYLOAD = PARTICLE_RECORD.itemsize - 8  # 84


# ---- Fortran unformatted sequential records --------------------------------
def write_record(f, payload: bytes) -> None:
    n = np.array([len(payload)], "<i4").tobytes()
    f.write(n)
    f.write(payload)
    f.write(n)


def read_record(f) -> bytes:
    head = f.read(4)
    if len(head) != 4:
        raise EOFError("no record")
    n = int(np.frombuffer(head, "<i4")[0])
    if n < 0:
        raise ValueError("record split into subrecords (over 2 GiB): not a file of this layout")
    payload = f.read(n)
    tail = f.read(4)
    if len(payload) != n or len(tail) != 4 or int(np.frombuffer(tail, "<i4")[0]) != n:
        raise ValueError("truncated or corrupt record")
    return payload


# ---- the three kinds of file ---------------------------------------------
def var_path(directory: str, lap: int) -> str:
    return os.path.join(directory, "DUMP", "var%07ddump" % lap)


def phi_path(directory: str, lap: int) -> str:
    return os.path.join(directory, "DUMP", "phi%07ddump" % lap)


def particle_path(directory: str, name: str) -> str:
    return os.path.join(directory, "%d%s.dat" % (NAME_INDEX, name))


def write_var(path: str, lap: int, ns, nx: int, ny: int, period_res: float = 0.0, istep_previous: int = 0,
              nperiod: int = 0) -> None:
    ns = [int(v) for v in ns]
    lines = [str(int(lap)), str(sum(ns)), " ".join(str(v) for v in ns), "%d %d" % (nx, ny),
             repr(float(period_res)), str(int(istep_previous)), str(int(nperiod))]
    with open(path, "w") as f:
        f.write("".join(" " + s + "\n" for s in lines))


def read_var(path: str, n_species: int) -> dict:
    with open(path) as f:
        tok = f.read().replace(",", " ").split()
    # list-directed input: the values in order, whatever the line breaks
    v = iter(tok)
    lap, ntot = int(next(v)), int(next(v))
    ns = [int(next(v)) for _ in range(n_species)]
    nx, ny = int(next(v)), int(next(v))
    period_res = float(next(v).replace("D", "E").replace("d", "e"))
    istep_previous, nperiod = int(next(v)), int(next(v))
    return {"lap": lap, "ntot": ntot, "ns": ns, "nx": nx, "ny": ny, "period_res": period_res,
            "istep_previous": istep_previous, "nperiod": nperiod}


def write_phi(path: str, phi: np.ndarray) -> None:
    with open(path, "wb") as f:
        write_record(f, np.ascontiguousarray(phi, "<f8").tobytes())


def read_phi(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        return np.frombuffer(read_record(f), "<f8").copy()


def write_particles(path: str, charge: float, mass: float, weight: float, cols: dict, npar_normal: int) -> None:
    """cols: X, Y, Z, Vx, Vy, Vz, Ax, Ay, Az, Wq (float64) and Location (int32), all of one length."""
    n = len(cols["X"])
    rec = np.zeros(n, PARTICLE_RECORD)
    rec["head"] = _PAYLOAD
    rec["tail"] = _PAYLOAD
    for k in ("X", "Y", "Z", "Vx", "Vy", "Vz", "Ax", "Ay", "Az", "Wq", "Location"):
        rec[k] = cols[k]
    with open(path, "wb") as f:
        write_record(f, np.array([n, npar_normal], "<i4").tobytes())
        write_record(f, np.array([charge, mass, weight], "<f8").tobytes())
        rec.tofile(f)


def read_particles(path: str) -> dict:
    with open(path, "rb") as f:
        npar, npar_normal = (int(a) for a in np.frombuffer(read_record(f), "<i4"))
        charge, mass, weight = (float(a) for a in np.frombuffer(read_record(f), "<f8"))
        rec = np.fromfile(f, PARTICLE_RECORD, count=npar)
        extra = f.read(1)
    if rec.size != npar or extra:
        raise ValueError("particle file holds %d records, its header says %d" % (rec.size, npar))
    if np.any(rec["head"] != _PAYLOAD) or np.any(rec["tail"] != _PAYLOAD):
        raise ValueError("particle records are not 84-byte ParticleOne records")
    out = {k: rec[k].copy() for k in ("X", "Y", "Z", "Vx", "Vy", "Vz", "Ax", "Ay", "Az", "Wq", "Location")}
    out.update(npar=npar, npar_normal=npar_normal, charge=charge, mass=mass, weight=weight)
    return out


def find_particle_file(directory: str, name: str) -> str:
    p = particle_path(directory, name)
    if os.path.exists(p):
        return p
    # the reference's list-directed file name may carry blanks around the index
    cands = [c for c in glob.glob(os.path.join(directory, "*%d*%s.dat" % (NAME_INDEX, glob.escape(name))))
             if os.path.basename(c).replace(" ", "") == os.path.basename(p)]
    if not cands:
        raise FileNotFoundError(p)
    return cands[0]


def transverse_to_frame(angle, vy, vz):
    """r-z: the reference's Cartesian transverse velocity (Vy, Vz) of a
    particle at angle Z (X = r cos Z, Y = r sin Z, MoveOne.f90:246-260) as
    (v_r, v_theta) in the particle's own frame."""
    c, s = np.cos(angle), np.sin(angle)
    return c * vy + s * vz, c * vz - s * vy


# ---- a Simulation to and from the files -----------------------------------
def dump(sim, directory: str, lap: int, period_res: float = 0.0, istep_previous: int = 0, nperiod: int = 0) -> None:
    """Dump_2D(lap) and ParticleGlobal(isp)%Dump(0) of every species."""
    os.makedirs(os.path.join(directory, "DUMP"), exist_ok=True)
    L, V = sim.scales["L_ref"], sim.scales["v_ref"]
    counts = []
    for s, (charge, mass, weight, _) in enumerate(sim.species):
        p = sim.download(s)
        n = p["x"].size
        counts.append(n)
        zero = np.zeros(n)
        # an r-z particle's own frame is the Cartesian one at angle 0: Z = 0
        cols = {"X": p["x"] * L, "Y": p["y"], "Z": zero, "Vx": p["vx"] * V, "Vy": p["vy"] * V,
                "Vz": p["vz"] * V, "Ax": zero, "Ay": zero, "Az": zero, "Wq": np.full(n, weight),
                "Location": p["loc"].astype(np.int64) + 1}
        # SpecyOne.f90:159-160: charge in coulomb, mass in kg
        write_particles(particle_path(directory, SPECIES_NAMES[s]), charge * QE, mass, weight, cols, max(n, 1))
    write_phi(phi_path(directory, lap), sim.field("phi"))
    write_var(var_path(directory, lap), lap, counts, sim.mesh.nnx, sim.mesh.nny, period_res, istep_previous,
              nperiod)


def restore(sim, directory: str, lap: int) -> dict:
    """Restart_2D at `lap` and LoadParticleBundle of every species into a
    Simulation built from the same deck: phi, then the particles (ids 0..n-1
    in file order, the next id n), then E recovered from phi; the step
    counter continues from lap.  Returns the var file's values."""
    ns = len(sim.species)
    var = read_var(var_path(directory, lap), ns)
    if (var["nx"], var["ny"]) != (sim.mesh.nnx, sim.mesh.nny):
        raise ValueError("dump is for a %dx%d node mesh, the simulation has %dx%d"
                         % (var["nx"], var["ny"], sim.mesh.nnx, sim.mesh.nny))
    phi = read_phi(phi_path(directory, lap))
    if phi.size != sim.mesh.nn:
        raise ValueError("phi record holds %d values for %d nodes" % (phi.size, sim.mesh.nn))
    L, V = sim.scales["L_ref"], sim.scales["v_ref"]
    axi = getattr(sim.cfg, "delta", 0) == 1
    for s in range(ns):
        r = read_particles(find_particle_file(directory, SPECIES_NAMES[s]))
        if r["npar"] != var["ns"][s]:
            raise ValueError("species %d: %d particles in its file, %d in the var file" % (s, r["npar"], var["ns"][s]))
        vy, vz = transverse_to_frame(r["Z"], r["Vy"], r["Vz"]) if axi else (r["Vy"], r["Vz"])
        x = np.ascontiguousarray(r["X"] / L)
        y = np.ascontiguousarray(r["Y"])  # PosRes leaves Y in L_ref units
        vx = np.ascontiguousarray(r["Vx"] / V)
        vy = np.ascontiguousarray(vy / V)
        vz = np.ascontiguousarray(vz / V)
        sim.upload(s, x, y, vx, vy, vz)
    sim.set_field("phi", phi)
    sim.get_efield_ppr()
    sim.step_index = int(var["lap"])
    return var


__all__ = ["dump", "restore", "transverse_to_frame", "read_var", "write_var", "read_phi", "write_phi", "read_particles",
           "write_particles", "read_record", "write_record", "PARTICLE_RECORD", "SPECIES_NAMES", "NAME_INDEX"]
