"""Time-dependent (RF) wall potential, pic_set_wall_rf: the reference's
bc_value(1) = V/Phi_ref*SIN(2*Pi*Frequency*time*time_ref) on the left
Dirichlet boundary (IFE_Solve_2D.f90:104-121).  The wall's nodes carry
static value + A sin(omega t + phase) into the RHS and into phi; the solve
is bit-exact against the oracle given the same Dirichlet values, and the
step drives it with t = step * dt.

The tiny deck's left wall has a static value of 5 V, so these tests pin the
additive form (static + sine).  The reference's commented-out line replaces
the wall value by the sine; the two coincide when the static value is 0."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle_bind as ob
from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

VOLTS, FREQ, PHASE = 3.0, 13.56e6, 0.3


def _expected(sim, t):
    amp = VOLTS / sim.scales["Phi_ref"]
    return amp * math.sin(2.0 * math.pi * FREQ * sim.scales["time_ref"] * t + PHASE)


def _left(sim):
    return np.arange(sim.mesh.nny)  # nodes i = 0


def test_rf_wall_solve_matches_oracle():
    sim = Simulation(deck.config("tiny"))
    try:
        sim.set_wall_rf(0, VOLTS, FREQ, PHASE)
        nn = sim.mesh.nn
        rho = np.random.default_rng(8).standard_normal(nn) * 0.05
        sim.set_field("rho", rho)
        # a view onto the descriptor's own table, which the oracle reads
        pd = np.ctypeslib.as_array(sim.mesh.desc.phi_dirichlet, shape=(nn,))
        static = pd.copy()
        phi = static.copy()
        t = 2000.0
        st = sim.ife_solve(phi, time=t)
        left = _left(sim)
        v = phi[left] - static[left]
        assert np.all(v == v[0])
        assert abs(v[0] - _expected(sim, t)) <= 1e-12 * max(1.0, abs(v[0]))
        assert abs(v[0]) > 0.1 * VOLTS / sim.scales["Phi_ref"]
        # the oracle with the wall values the device used
        try:
            pd[left] = phi[left]
            b = ob.rhs(sim.mesh.ptr, rho, nn)
            assert np.array_equal(sim.field("b"), b)
            po, so = ob.pcg(sim.mesh.ptr, b, pd.copy(), sim.cfg.pcg_tol, sim.cfg.pcg_maxit)
        finally:
            pd[:] = static
        assert st.ierr == 0 and st.iterations == so["iterations"]
        assert np.array_equal(phi, po)
    finally:
        sim.close()


def test_rf_wall_follows_the_step_time():
    sim = Simulation(deck.config("tiny", rf=(0, VOLTS, FREQ, PHASE)))
    try:
        sim.initial_fields()
        static = sim.mesh.array("phi_dirichlet").copy()
        left = _left(sim)
        phi = sim.field("phi")
        assert np.allclose(phi[left] - static[left], _expected(sim, 0.0), rtol=0, atol=1e-12)
        for k in range(1, 4):
            sim.step()
            phi = sim.field("phi")
            got = phi[left] - static[left]
            assert np.allclose(got, _expected(sim, k * sim.cfg.dt), rtol=0, atol=1e-12), k
    finally:
        sim.close()


def test_rf_off_restores_the_static_wall_and_bad_walls_are_refused():
    sim = Simulation(deck.config("tiny"))
    try:
        lib = api.load()
        assert lib.pic_set_wall_rf(2, 1.0, FREQ, 0.0) == api.PIC_ERR_ARG
        assert lib.pic_set_wall_rf(0, float("nan"), FREQ, 0.0) == api.PIC_ERR_ARG
        sim.set_wall_rf(0, VOLTS, FREQ, PHASE)
        sim.set_wall_rf(0, 0.0, FREQ, PHASE)
        static = sim.mesh.array("phi_dirichlet").copy()
        phi = static.copy()
        sim.ife_solve(phi, time=1234.0)
        assert np.array_equal(phi[_left(sim)], static[_left(sim)])
    finally:
        sim.close()
    sim = Simulation(deck.config("tiny", wall_dirichlet=(0, 1, 1, 1)))
    try:
        lib = api.load()
        assert lib.pic_set_wall_rf(0, 1.0, FREQ, 0.0) == api.PIC_ERR_ARG
        assert b"not a Dirichlet wall" in lib.pic_last_error()
        assert lib.pic_set_wall_rf(1, 1.0, FREQ, 0.0) == 0
    finally:
        sim.close()
