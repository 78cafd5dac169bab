"""The reference-shaped API on the GPU.

The 4-particle tests restate the reference's own SPH function tests
(S/sph/tests/function_test_template.py with test_density_funcs.py,
test_eos_funcs.py, test_pressure_funcs.py): SPHCalc.sph() against the tests'
O(N^2) reference loops, to the same decimal places.  The solver tests run the
elliptical drop and the dam break through Solver / PredictorCorrectorIntegrator
(the fused engine path) against the oracle, and the integrator's building
blocks (calc-by-calc) against the fused path.
"""
import math

import numpy as np
import pytest
import torch

import pysph_b200.base.api as base
import pysph_b200.sph.api as sph
import pysph_b200.solver.api as solver
from pysph_b200 import workloads as W

from helpers import oracle_from
from pysph_b200.engine import fluid_scheme

pytestmark = pytest.mark.gpu
Fluid, Solid = base.Fluid, base.Solid


def square():
    x = np.array([0, 0, 1, 1], np.float64)
    y = np.array([0, 1, 1, 0], np.float64)
    pa = base.get_particle_array(name="test", x=x, y=y, z=np.zeros(4), m=np.ones(4),
                                 u=np.array([1, 0, 0, -1], np.float64),
                                 p=np.array([0, 0, 1, 1], np.float64))
    return pa, base.Particles([pa]), base.CubicSplineKernel(dim=2)


def ref_grad(k, ri, rj, h):
    g = base.Point()
    k.py_gradient(ri, rj, h, g)
    return g


def test_square_sph_rho():
    pa, particles, k = square()
    func = sph.SPHRho.withargs().get_func(pa, pa)
    calc = sph.SPHCalc(particles, [pa], pa, k, [func], ["rho"])
    calc.sph()
    tmpx = pa.get("_tmpx").cpu().numpy()
    x, y, m, h = (pa.get(n).cpu().numpy() for n in ("x", "y", "m", "h"))
    for i in range(4):
        ri = base.Point(x[i], y[i], 0)
        rho = sum(m[j] * k.py_function(ri, base.Point(x[j], y[j], 0), 0.5 * (h[i] + h[j]))
                  for j in range(4))
        assert round(tmpx[i] - rho, 6) == 0


def test_square_tait():
    pa, particles, k = square()
    pa.set(rho=np.array([1000.0, 1001.5, 998.0, 1010.0]))
    func = sph.TaitEquation.withargs(gamma=7.0).get_func(pa, pa)
    calc = sph.SPHCalc(particles, [pa], pa, k, [func], ["p", "cs"])
    calc.sph()
    B = 1.0 * 1.0 * 1000 / 7.0
    rho = pa.get("rho").cpu().numpy()
    for i in range(4):
        ratio = rho[i] / 1000
        assert round(pa._tmpx[i].item() - (np.power(ratio, 7.0) - 1.0) * B, 10) == 0
        assert round(pa._tmpy[i].item() - np.power(ratio, 3.0), 10) == 0


@pytest.mark.parametrize("which", ["pgrad", "momentum"])
def test_square_pressure_and_momentum(which):
    pa, particles, k = square()
    pa.set(cs=np.array([1.0, 2.0, 0.5, 1.5]))
    if which == "pgrad":
        func = sph.SPHPressureGradient.withargs().get_func(pa, pa)
    else:
        func = sph.MomentumEquation.withargs(alpha=1.0, beta=1.0, gamma=1.4,
                                             eta=0.1).get_func(pa, pa)
    calc = sph.SPHCalc(particles, [pa], pa, k, [func], ["rho"])
    calc.sph()
    out = [pa.get(n).cpu().numpy() for n in ("_tmpx", "_tmpy", "_tmpz")]
    x, y, p, rho, h, m, u, v, cs = (pa.get(n).cpu().numpy()
                                    for n in ("x", "y", "p", "rho", "h", "m", "u", "v", "cs"))
    for i in range(4):
        ri = base.Point(x[i], y[i], 0)
        f = np.zeros(3)
        for j in range(4):
            rj = base.Point(x[j], y[j], 0)
            havg = 0.5 * (h[i] + h[j])
            g = ref_grad(k, ri, rj, havg)
            tmp = p[i] / rho[i] ** 2 + p[j] / rho[j] ** 2
            if which == "momentum":
                rab = ri - rj
                dot = (u[i] - u[j]) * rab.x + (v[i] - v[j]) * rab.y
                if dot < 0:
                    cab = 0.5 * (cs[i] + cs[j])
                    rhoab = 0.5 * (rho[i] + rho[j])
                    mu = havg * dot / (rab.norm() + 0.01 * havg * havg)
                    tmp += (-1.0 * cab * mu + 1.0 * mu * mu) / rhoab
            tmp *= -m[j]
            f += tmp * np.array([g.x, g.y, g.z])
        for d in range(3):
            assert round(out[d][i] - f[d], 6) == 0


def test_locator_lists_self_last():
    arrays, _, params = W.elliptical_drop(dx=0.1)
    a = arrays[0]
    pa = base.get_particle_array(name="fluid", **{n: a[n] for n in ("x", "y", "h", "m")})
    particles = base.Particles([pa])
    particles.kernel = base.CubicSplineKernel(dim=2)
    loc = particles.nnps_manager.get_neighbor_particle_locator(pa, pa, 2.0)
    osys = oracle_from(arrays, params, fluid_scheme(1), 2)
    osys.update_pairs([(0, 0)])
    off, idx = osys.neighbors(0, 0)
    for i in range(pa.get_number_of_particles()):
        got = loc.py_get_nearest_particles(i)
        ref = idx[off[i]:off[i + 1]]
        assert got[-1] == i and ref[-1] == i
        assert sorted(got.tolist()) == sorted(ref.tolist())


def drop_solver(dx=0.025, precision=None):
    arrays, _, params = W.elliptical_drop(dx=dx)
    a = arrays[0]
    pa = base.get_particle_array(name="fluid", **a)
    particles = base.Particles([pa], precision=precision)
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                        from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    s.set_time_step(1e-5)
    s.set_final_time(1e-4 - 1e-12)
    s.setup(particles)
    return s, pa, arrays, params


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_solver_drop_matches_oracle(precision):
    s, pa, arrays, params = drop_solver(precision=precision)
    assert s.integrator.plan is not None
    s.solve()
    assert s.count == 10
    osys = oracle_from(arrays, params, fluid_scheme(1), 2)
    for _ in range(10):
        osys.pc_step(1e-5)
    O = osys.arrays[0]
    dx = 0.025
    tol = 1e-10 if precision == "fp64" else 2e-6
    assert np.max(np.abs(pa.x.cpu().numpy() - O.x)) / dx <= tol
    assert np.max(np.abs(pa.y.cpu().numpy() - O.y)) / dx <= tol
    rtol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(pa.rho.cpu().numpy() - O.rho) / O.rho) <= rtol
    # the properties the reference's integrator exposes are filled in
    assert np.max(np.abs(pa.get("_x0").cpu().numpy() - O.x0)) / dx <= tol


def test_integrator_building_blocks_match_fused():
    """The calc-by-calc path (SPHCalc.sph + elementwise steps) gives the
    fused engine step's result."""
    s1, pa1, _, _ = drop_solver(dx=0.05)
    s2, pa2, _, _ = drop_solver(dx=0.05)
    s2.integrator.plan = None
    for _ in range(3):
        s1.integrator.integrate(1e-5)
        s2.integrator.integrate(1e-5)
    for n in ("x", "y", "u", "v", "rho"):
        a = pa1.get(n).cpu().numpy()
        b = pa2.get(n).cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(a))), n


def test_solver_dam_break_cfl_on_device():
    arrays, types, params = W.dam_break(dx=0.02)
    f = base.get_particle_array(name="fluid", type=Fluid, **arrays[0])
    w = base.get_particle_array(name="wall", type=Solid, **arrays[1])
    particles = base.Particles([f, w])
    co = params["c0"]
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid, Solid],
                                        from_types=[Fluid, Solid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=co, ro=1000.0),
                                        on_types=[Fluid, Solid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0), on_types=[Fluid],
        from_types=[Fluid, Solid], updates=["u", "v"], id="mom"))
    s.add_operation(solver.SPHIntegration(sph.GravityForce.withargs(gy=-9.81),
                                          on_types=[Fluid], updates=["u", "v"], id="grav"))
    s.add_operation_step([Fluid])
    s.set_time_step(1e-4)
    s.set_final_time(6.5e-4)
    s.setup(particles)
    s.time_step_function = solver.ViscousAndForceBasedTimeStep(co=co, cfl=0.3,
                                                               particles=particles)
    s.solve()
    osys = oracle_from(arrays, params, fluid_scheme(2), 2)
    dts = []
    for _ in range(s.count):
        dt = osys.cfl_time_step(0.3, co, 1e-4)
        osys.pc_step(dt)
        dts.append(dt)
    np.testing.assert_allclose(s.dt_history, dts, rtol=1e-12)
    O = osys.arrays[0]
    assert np.max(np.abs(f.x.cpu().numpy() - O.x)) / 0.02 <= 1e-10
    assert np.max(np.abs(f.y.cpu().numpy() - O.y)) / 0.02 <= 1e-10
    rho = w.rho.cpu().numpy()
    assert np.max(np.abs(rho - osys.arrays[1].rho) / osys.arrays[1].rho) <= 1e-12


def test_host_edits_reach_the_engine():
    """Velocities set on the host between two steps are the ones the next
    step uses (compared with the oracle started from the edited state)."""
    s, pa, arrays, params = drop_solver(dx=0.05)
    s.integrator.integrate(1e-5)
    state = {n: pa.get(n).cpu().numpy().copy() for n in ("x", "y", "m", "h", "rho", "p", "cs")}
    rng = np.random.default_rng(2)
    n = pa.get_number_of_particles()
    u = rng.uniform(-50, 50, n)
    v = rng.uniform(-50, 50, n)
    pa.set(u=u, v=v)
    s.integrator.integrate(1e-5)
    osys = oracle_from([dict(state, z=np.zeros(n), u=u, v=v, w=np.zeros(n))], params,
                       fluid_scheme(1), 2)
    osys.pc_step(1e-5)
    assert np.max(np.abs(pa.x.cpu().numpy() - osys.arrays[0].x)) / 0.05 <= 1e-10
    assert np.max(np.abs(pa.u.cpu().numpy() - osys.arrays[0].u)) <= 1e-8 * 50


def drop_continuity_solver(dx=0.025, precision=None):
    """The drop with the continuity scheme: Tait, SPHDensityRate, momentum,
    position stepping with XSPH (eps 0.5)."""
    arrays, _, params = W.elliptical_drop(dx=dx)
    pa = base.get_particle_array(name="fluid", **arrays[0])
    particles = base.Particles([pa], precision=precision)
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(sph.SPHDensityRate.withargs(hks=False),
                                          on_types=[Fluid], from_types=[Fluid],
                                          updates=["rho"], id="density"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid], xsph=True, eps=0.5)
    s.set_time_step(1e-5)
    s.set_final_time(1e-4 - 1e-12)
    s.setup(particles)
    return s, pa, arrays, params


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_solver_drop_continuity_matches_oracle(precision):
    """Solver.solve on the continuity scheme runs fused on the engine and
    tracks the oracle (itself pinned to the reference's fixtures)."""
    from oracle import OracleArray, OracleSystem
    from pysph_b200.engine import continuity_scheme
    s, pa, arrays, params = drop_continuity_solver(precision=precision)
    assert s.integrator.plan is not None and s.integrator.plan.scheme.continuity
    s.solve()
    assert s.count == 10
    sch = continuity_scheme(1, 0.5)
    o = OracleSystem([OracleArray("a0", **{k: np.array(v, np.float64)
                                          for k, v in arrays[0].items()})],
                     dim=2, tait_on=sch.tait_on, mom_src=sch.mom_src, step_on=sch.step_on,
                     rate_src=sch.rate_src, xsph_src=sch.xsph_src, xsph_eps=0.5,
                     c0=1400.0, rho0=1.0, alpha=0.1, beta=0.0, eta=0.1)
    for _ in range(10):
        o.pc_step(1e-5)
    O = o.arrays[0]
    dx = 0.025
    tol = 1e-10 if precision == "fp64" else 2e-6
    assert np.max(np.abs(pa.x.cpu().numpy() - O.x)) / dx <= tol
    assert np.max(np.abs(pa.y.cpu().numpy() - O.y)) / dx <= tol
    rtol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(pa.rho.cpu().numpy() - O.rho) / O.rho) <= rtol
    assert np.max(np.abs(pa.get("_rho0").cpu().numpy() - O.rho0) / O.rho0) <= rtol


def test_continuity_building_blocks_match_fused():
    """SPHDensityRate and XSPHCorrection calc by calc (SPHCalc.sph on the
    engine + elementwise steps) give the fused engine step's result."""
    s1, pa1, _, _ = drop_continuity_solver(dx=0.05)
    s2, pa2, _, _ = drop_continuity_solver(dx=0.05)
    s2.integrator.plan = None
    for _ in range(3):
        s1.integrator.integrate(1e-5)
        s2.integrator.integrate(1e-5)
    for n in ("x", "y", "u", "v", "rho"):
        a = pa1.get(n).cpu().numpy()
        b = pa2.get(n).cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(a))), n


@pytest.mark.parametrize("integ", ["euler", "rk2", "rk4"])
def test_solver_other_integrators_match_oracle(integ):
    """Solver with the reference's Euler / RK2 / RK4 integrators (fused on
    the engine) against the oracle's restatement of each (pinned to
    reference fixtures)."""
    cls = {"euler": solver.EulerIntegrator, "rk2": solver.RK2Integrator,
           "rk4": solver.RK4Integrator}[integ]
    arrays, _, params = W.elliptical_drop(dx=0.05)
    pa = base.get_particle_array(name="fluid", **arrays[0])
    particles = base.Particles([pa])
    s = solver.Solver(dim=2, integrator_type=cls)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                        from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    s.set_time_step(1e-5)
    s.set_final_time(5e-5 - 1e-12)
    s.setup(particles)
    assert s.integrator.plan is not None
    s.solve()
    assert s.count == 5
    osys = oracle_from(arrays, params, fluid_scheme(1), 2)
    for _ in range(5):
        osys.step(1e-5, integ)
    O = osys.arrays[0]
    dx = 0.05
    for n in ("x", "y"):
        assert np.max(np.abs(pa.get(n).cpu().numpy() - getattr(O, n))) / dx <= 1e-10, n
    assert np.max(np.abs(pa.rho.cpu().numpy() - O.rho) / O.rho) <= 1e-12


# -- variable smoothing length: Particles(variable_h=True), hks functions -----
def varh_arrays():
    """The drop (dx = 0.05) with h growing from 1.0 to 1.4 times 1.3 dx
    across x."""
    arrays, _, params = W.elliptical_drop(dx=0.05)
    a = arrays[0]
    a["h"] = 1.3 * 0.05 * (1.0 + 0.2 * (a["x"] + 1.0))
    return arrays, params


def varh_oracle(arrays, cont):
    from oracle import OracleArray, OracleSystem
    sch = {"rate_src": {0: [0]}, "xsph_src": {0: [0]}} if cont else {"rho_src": {0: [0]}}
    return OracleSystem([OracleArray("a0", **{k: np.array(v, np.float64)
                                             for k, v in arrays[0].items()})],
                        dim=2, tait_on=(0,), mom_src={0: [0]}, step_on=(0,), xsph_eps=0.5,
                        c0=1400.0, rho0=1.0, alpha=0.1, beta=0.0, eta=0.1,
                        variable_h=True, hks=True, **sch)


def varh_solver(cont, precision=None):
    arrays, params = varh_arrays()
    pa = base.get_particle_array(name="fluid", **arrays[0])
    particles = base.Particles([pa], variable_h=True, precision=precision)
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    if not cont:
        s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(hks=True), on_types=[Fluid],
                                            from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    if cont:
        s.add_operation(solver.SPHIntegration(sph.SPHDensityRate.withargs(hks=True),
                                              on_types=[Fluid], from_types=[Fluid],
                                              updates=["rho"], id="density"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1, hks=True),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    if cont:
        s.add_operation_xsph(eps=0.5, hks=True)
    s.set_time_step(1e-5)
    s.set_final_time(5e-5 - 1e-12)
    s.setup(particles)
    return s, pa, arrays


def test_varh_locator_symmetric_sets():
    """Particles(variable_h=True): the locator hands out the symmetric sets
    of VarHNbrParticleLocator, self last."""
    arrays, _ = varh_arrays()
    pa = base.get_particle_array(name="fluid", **{n: arrays[0][n] for n in ("x", "y", "h", "m")})
    particles = base.Particles([pa], variable_h=True)
    particles.kernel = base.CubicSplineKernel(dim=2)
    loc = particles.nnps_manager.get_neighbor_particle_locator(pa, pa, 2.0)
    osys = varh_oracle(arrays, False)
    osys.update_pairs([(0, 0)])
    off, idx = osys.neighbors(0, 0)
    for i in range(pa.get_number_of_particles()):
        got = loc.py_get_nearest_particles(i)
        ref = idx[off[i]:off[i + 1]]
        assert got[-1] == i
        assert sorted(got.tolist()) == sorted(ref.tolist())


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("cont", [False, True])
def test_solver_varh_hks_matches_oracle(precision, cont):
    """Variable h with hks kernels through Solver.solve (fused on the engine)
    against the oracle, itself pinned to the reference's fixtures."""
    s, pa, arrays = varh_solver(cont, precision)
    plan = s.integrator.plan
    assert plan is not None and plan.scheme.hks and plan.scheme.continuity == cont
    s.solve()
    assert s.count == 5
    o = varh_oracle(arrays, cont)
    for _ in range(5):
        o.pc_step(1e-5)
    O = o.arrays[0]
    dx = 0.05
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        assert np.max(np.abs(pa.get(n).cpu().numpy() - getattr(O, n))) / dx <= tol, n
    rtol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(pa.rho.cpu().numpy() - O.rho) / O.rho) <= rtol


@pytest.mark.parametrize("cont", [False, True])
def test_varh_building_blocks_match_fused(cont):
    """The hks functions calc by calc give the fused step's result."""
    s1, pa1, _ = varh_solver(cont)
    s2, pa2, _ = varh_solver(cont)
    s2.integrator.plan = None
    for _ in range(3):
        s1.integrator.integrate(1e-5)
        s2.integrator.integrate(1e-5)
    for n in ("x", "y", "u", "v", "rho"):
        a = pa1.get(n).cpu().numpy()
        b = pa2.get(n).cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(a))), n


# -- the quintic spline and Wendland quintic kernels --------------------------
def kernel_solver(kernel, rho0=1.0, cont=False):
    arrays, _, params = W.elliptical_drop(dx=0.05)
    pa = base.get_particle_array(name="fluid", **arrays[0])
    particles = base.Particles([pa])
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator,
                      kernel=kernel(dim=2))
    if not cont:
        s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                            from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=rho0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    if cont:
        s.add_operation(solver.SPHIntegration(sph.SPHDensityRate.withargs(),
                                              on_types=[Fluid], from_types=[Fluid],
                                              updates=["rho"], id="density"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    if cont:
        s.add_operation_xsph(eps=0.5)
    s.set_time_step(1e-5)
    s.set_final_time(5e-5 - 1e-12)
    s.setup(particles)
    return s, pa, arrays


@pytest.mark.parametrize("cont", [False, True])
@pytest.mark.parametrize("kname", ["QuinticSplineKernel", "WendlandQuinticSplineKernel"])
def test_solver_other_kernels_match_oracle(kname, cont):
    """Solver(kernel=QuinticSplineKernel / WendlandQuinticSplineKernel) runs
    fused on the engine and tracks the oracle (pinned to the reference)."""
    from oracle import KERNEL_RADIUS, OracleArray, OracleSystem
    kernel = getattr(base, kname)
    rho0 = float(np.pi ** 2) if kname.startswith("Wendland") and not cont else 1.0
    s, pa, arrays = kernel_solver(kernel, rho0, cont)
    plan = s.integrator.plan
    kt = kernel(dim=2).get_type()
    assert plan is not None and plan.kernel == kt
    s.solve()
    assert s.count == 5
    sch = ({"rate_src": {0: [0]}, "xsph_src": {0: [0]}} if cont else {"rho_src": {0: [0]}})
    o = OracleSystem([OracleArray("a0", **{k: np.array(v, np.float64)
                                          for k, v in arrays[0].items()})],
                     dim=2, tait_on=(0,), mom_src={0: [0]}, step_on=(0,), xsph_eps=0.5,
                     c0=1400.0, rho0=rho0, alpha=0.1, beta=0.0, eta=0.1, kernel=kt,
                     radius_scale=KERNEL_RADIUS[kt], **sch)
    for _ in range(5):
        o.pc_step(1e-5)
    O = o.arrays[0]
    dx = 0.05
    for n in ("x", "y"):
        assert np.max(np.abs(pa.get(n).cpu().numpy() - getattr(O, n))) / dx <= 1e-10, n
    assert np.max(np.abs(pa.rho.cpu().numpy() - O.rho) / O.rho) <= 1e-12
    # calc by calc gives the fused result
    s2, pa2, _ = kernel_solver(kernel, rho0, cont)
    s2.integrator.plan = None
    for _ in range(5):
        s2.integrator.integrate(1e-5)
    for n in ("x", "y", "rho"):
        a = pa.get(n).cpu().numpy()
        b = pa2.get(n).cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-10 * max(1.0, np.max(np.abs(a))), n


def _drop_for(cls, precision):
    arrays, _, _ = W.elliptical_drop(dx=0.05)
    pa = base.get_particle_array(name="fluid", cl_precision=precision, **arrays[0])
    particles = base.Particles([pa])
    s = solver.Solver(dim=2, integrator_type=cls)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                        from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, eta=0.1),
        on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    s.set_time_step(1e-5)
    s.setup(particles)
    assert s.integrator.plan is not None
    return s, pa


@pytest.mark.parametrize("precision", ["single", "double"])
@pytest.mark.parametrize("integ", ["pc", "euler", "rk2", "rk4"])
def test_graphed_steps_match_eager_steps(integ, precision):
    """The fused integrators replay one captured CUDA graph per step once
    the step repeats (Engine.step_graphed): bit for bit the eager launches,
    over steps that run alone, steps after host writes of the state (which
    refresh the records and re-measure the displacements), and a change of
    dt, for every integrator (Euler's one stage runs unfused in a graph)."""
    cls = {"pc": solver.PredictorCorrectorIntegrator, "euler": solver.EulerIntegrator,
           "rk2": solver.RK2Integrator, "rk4": solver.RK4Integrator}[integ]
    runs = []
    for graphs in (True, False):
        s, pa = _drop_for(cls, precision)
        eng = s.integrator._fused_session().engine
        eng.graphs = graphs
        for i in range(12):
            if 4 <= i < 8:
                # the host rewrites the state it has just read
                pa.set(x=pa.get("x").cpu().numpy(), u=pa.get("u").cpu().numpy() * 1.001)
            s.integrator.integrate(1e-5 if i < 10 else 2e-5)
        if graphs:
            assert eng._graphs, "no step was replayed from a graph"
        runs.append({n: pa.get(n).cpu().numpy().copy() for n in ("x", "y", "u", "v", "rho", "p")})
        eng.check_status()
    for n in runs[0]:
        assert np.array_equal(runs[0][n], runs[1][n]), n


def test_get_of_several_properties_matches_single_gets():
    """ParticleArray.get of several properties the engine has newer values
    of copies them back in one launch (sphb_exchange_many): the same values
    as one get per property."""
    vals = []
    for batched in (True, False):
        s, pa = _drop_for(solver.PredictorCorrectorIntegrator, "single")
        for _ in range(3):
            s.integrator.integrate(1e-5)
        names = ("x", "y", "u", "v", "rho", "p", "_a_u_1", "dt_fac")
        got = pa.get(*names) if batched else [pa.get(n) for n in names]
        vals.append([t.cpu().numpy().copy() for t in got])
    for n, a, b in zip(("x", "y", "u", "v", "rho", "p", "_a_u_1", "dt_fac"), *vals):
        assert np.array_equal(a, b), n
