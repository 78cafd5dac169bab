"""The split-form MonaghanArtificialViscosity on the GPU, against the
fixture the reference itself wrote (tests/golden/avisc.npz, by
tests/golden/make_golden.py): the function alone through SPHCalc on the
4-particle unit square (its eta left at the reference's unset 0, and
assigned 0.1 by hand), and a drop scheme that pairs it with
SPHPressureGradient, through Solver / PredictorCorrectorIntegrator (one
calc at a time: the fused plan does not take this scheme).

FP64 to round-off (the sums run in another order than the reference's);
FP32C to the FP32 path's bars: 1e-5 relative density, 1e-4 of the largest
acceleration.
"""
import os

import numpy as np
import pytest
import torch

import pysph_b200.base.api as base
import pysph_b200.sph.api as sph
import pysph_b200.solver.api as solver

pytestmark = pytest.mark.gpu
Fluid = base.Fluid
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "avisc.npz")
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")
TOL = {"double": 1e-12, "single": 1e-4}


def gold():
    return dict(np.load(GOLD))


def rel(got, ref):
    scale = max(float(np.max(np.abs(ref))), 1e-300)
    return float(np.max(np.abs(np.asarray(got) - ref))) / scale


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("name,eta", [("square", None), ("square_eta", 0.1)])
def test_square_viscosity_against_reference(precision, name, eta):
    g = gold()
    pa = base.get_particle_array(
        name="test", cl_precision=precision, x=np.array([0, 0, 1, 1.0]),
        y=np.array([0, 1, 1, 0.0]), z=np.zeros(4), m=np.ones(4), h=np.ones(4),
        u=np.array([1, 0, 0, -1.0]), v=np.array([0, 0.5, 0, 0.25]),
        p=np.array([0, 0, 1, 1.0]), cs=np.array([1.0, 2.0, 0.5, 1.5]),
        rho=np.array([1.0, 1.5, 0.98, 1.1]))
    particles = base.Particles([pa])
    k = base.CubicSplineKernel(dim=2)
    f = sph.MonaghanArtificialViscosity.withargs(alpha=1.0, beta=1.0, gamma=1.4,
                                                 eta=0.1).get_func(pa, pa)
    assert f.eta == 0.0          # the constructor's eta is not stored
    if eta is not None:
        f.eta = eta
    calc = sph.SPHCalc(particles, [pa], pa, k, [f], ["u", "v"], integrates=True)
    pa.set_to_zero(["_tmpx", "_tmpy", "_tmpz"])
    calc.sph("_tmpx", "_tmpy", "_tmpz")
    for i, n in enumerate(("_tmpx", "_tmpy")):
        assert rel(pa.get(n).cpu().numpy(), g[f"{name}_{i}"]) <= TOL[precision], n
    assert rel(pa.get("dt_fac").cpu().numpy(), g[f"{name}_dt_fac"]) <= TOL[precision]


def drop_split_solver(g, precision):
    pa = base.get_particle_array(name="fluid", type=Fluid, cl_precision=precision,
                                 **{k: g[f"in_{k}"].copy() for k in PROPS})
    particles = base.Particles([pa])
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                        from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=1400.0, ro=1.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(sph.SPHPressureGradient.withargs(),
                                          on_types=[Fluid], from_types=[Fluid],
                                          updates=["u", "v"], id="pgrad"))
    s.add_operation(solver.SPHIntegration(
        sph.MonaghanArtificialViscosity.withargs(alpha=0.1, beta=0.0), on_types=[Fluid],
        from_types=[Fluid], updates=["u", "v"], id="avisc"))
    s.add_operation_step([Fluid])
    s.set_time_step(1e-5)
    s.setup(particles)
    assert s.integrator.plan is None   # evaluated calc by calc
    return s, pa


@pytest.mark.parametrize("precision", ["double", "single"])
def test_split_scheme_first_stage_against_reference(precision):
    g = gold()
    s, pa = drop_split_solver(g, precision)
    it = s.integrator
    it.save_initial_arrays()
    it.reset_accelerations(step=1)
    it.eval()
    rho_tol = 1e-12 if precision == "double" else 1e-5
    rho = pa.get("rho").cpu().numpy()
    assert float(np.max(np.abs(rho - g["stage0_rho"]) / g["stage0_rho"])) <= rho_tol
    for n in ("_a_u_1", "_a_v_1", "dt_fac"):
        tol = 1e-10 if precision == "double" else 1e-4
        assert rel(pa.get(n).cpu().numpy(), g[f"stage0_{n}"]) <= tol, n


@pytest.mark.parametrize("precision", ["double", "single"])
def test_split_scheme_five_steps_against_reference(precision):
    g = gold()
    s, pa = drop_split_solver(g, precision)
    for _ in range(5):
        s.integrator.integrate(1e-5)
    dx = 0.05
    for n in ("x", "y"):
        err = float(np.max(np.abs(pa.get(n).cpu().numpy() - g[f"step5_{n}_0"]))) / dx
        assert err <= (1e-10 if precision == "double" else 2e-6), n
    for n in ("u", "v"):
        assert rel(pa.get(n).cpu().numpy(), g[f"step5_{n}_0"]) <= (
            1e-10 if precision == "double" else 2e-5), n
    rho = pa.get("rho").cpu().numpy()
    assert float(np.max(np.abs(rho - g["step5_rho_0"]) / g["step5_rho_0"])) <= (
        1e-12 if precision == "double" else 1e-5)
