"""The reference's own FP64 Cython particle path, driven through its own
API -- TEST INFRASTRUCTURE ONLY.

oracle/build_reference.py builds the reference (PySPH 0.9beta) from its
sources, patched mechanically for Python 3 / Cython 3 and with no change to
its arithmetic, into oracle/_ref/refbuild (git-ignored).  This module imports
that build and drives it the way the reference's own solver loop does
(S/solver/solver.py:546-566): get_particle_array, Particles (CellManager +
NNPSManager), SPHOperation / SPHIntegration calcs, PredictorCorrectorIntegrator
and ViscousAndForceBasedTimeStep.  Its users are the golden-fixture script
(tests/golden/make_golden.py) and bench.py's CPU legs, which time the
reference itself beside the CUDA path; the product never imports it.
"""
from __future__ import annotations

import glob
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(_HERE, "_ref", "refbuild")
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")


def available(build_dir: str = BUILD_DIR) -> bool:
    """Whether the reference's extension modules are built in build_dir."""
    need = ("carray", "particle_array", "cell", "nnps", "kernels")
    base = os.path.join(build_dir, "pysph", "base")
    return all(glob.glob(os.path.join(base, f"{m}.*.so")) for m in need)


def modules(build_dir: str = BUILD_DIR):
    """The reference's modules of the particle path, imported from the build."""
    if build_dir not in sys.path:
        sys.path.insert(0, build_dir)
    import pysph.base.particle_array as PA
    import pysph.base.particles as P
    import pysph.base.kernels as K
    import pysph.sph.sph_calc as C
    import pysph.sph.funcs.density_funcs as D
    import pysph.sph.funcs.eos_funcs as E
    import pysph.sph.funcs.pressure_funcs as PF
    import pysph.sph.funcs.position_funcs as POS
    import pysph.sph.funcs.external_force as EF
    import pysph.sph.funcs.xsph_funcs as X
    import pysph.sph.funcs.viscosity_funcs as V
    import pysph.solver.sph_equation as EQ
    import pysph.solver.integrator as I
    import pysph.solver.time_step_functions as T
    from pysph.base.point import Point
    return dict(PA=PA, P=P, K=K, C=C, D=D, E=E, PF=PF, POS=POS, EF=EF, EQ=EQ, I=I, T=T, X=X,
                V=V, Point=Point)


def make_array(R, props, name, ptype):
    """A reference ParticleArray from a dict of numpy properties."""
    d = {k: np.asarray(props[k], np.float64).copy() for k in PROPS if k in props}
    return R["PA"].get_particle_array(name=name, type=ptype, **d)


def scheme_ops(R, ntypes, c0, rho0, alpha, beta, eta, gy, dim, xsph_eps=None, hks=False):
    """The summation-density scheme, or with xsph_eps the continuity scheme
    of the reference's dam-break example (examples/dam-break/dam_break.py:
    184-241): Tait, SPHDensityRate (integrated rho on every array), momentum,
    gravity, position stepping and XSPHCorrection on the fluid."""
    EQ, D, E, PF, POS, EF = R["EQ"], R["D"], R["E"], R["PF"], R["POS"], R["EF"]
    types = list(range(ntypes))
    vel = ["u", "v", "w"][:dim]
    pos = ["x", "y", "z"][:dim]
    if xsph_eps is None:
        ops = [EQ.SPHOperation(D.SPHRho.withargs(hks=hks), on_types=types, from_types=types,
                               updates=["rho"], id="sd"),
               EQ.SPHOperation(E.TaitEquation.withargs(co=c0, ro=rho0), on_types=types,
                               updates=["p", "cs"], id="eos")]
    else:
        ops = [EQ.SPHOperation(E.TaitEquation.withargs(co=c0, ro=rho0), on_types=types,
                               updates=["p", "cs"], id="eos"),
               EQ.SPHIntegration(D.SPHDensityRate.withargs(hks=hks), on_types=types,
                                 from_types=types, updates=["rho"], id="density")]
    ops.append(EQ.SPHIntegration(PF.MomentumEquation.withargs(alpha=alpha, beta=beta, eta=eta,
                                                              hks=hks),
                                 on_types=[0], from_types=types, updates=vel, id="mom"))
    if gy:
        ops.append(EQ.SPHIntegration(EF.GravityForce.withargs(gy=gy), on_types=[0],
                                     updates=vel, id="grav"))
    ops.append(EQ.SPHIntegration(POS.PositionStepping.withargs(), on_types=[0],
                                 updates=pos, id="step"))
    if xsph_eps is not None:
        ops.append(EQ.SPHIntegration(R["X"].XSPHCorrection.withargs(eps=xsph_eps, hks=hks),
                                     on_types=[0], from_types=[0], updates=pos, id="xsph"))
    return ops


def build_sim(R, arrays, types, params, dim, xsph_eps=None, integrator=None,
              variable_h=False, hks=False, kernel="CubicSplineKernel"):
    pas = [make_array(R, a, f"a{i}", t) for i, (a, t) in enumerate(zip(arrays, types))]
    particles = R["P"].Particles(pas, variable_h=variable_h)
    kernel = getattr(R["K"], kernel)(dim=dim)
    ops = scheme_ops(R, len(pas), params["c0"], params["rho0"], params["alpha"],
                     params["beta"], params["eta"], params["gravity"][1], dim, xsph_eps, hks)
    calcs = []
    for op in ops:
        calcs.extend(op.get_calcs(particles, kernel))
    integ = (integrator or R["I"].PredictorCorrectorIntegrator)(particles, calcs)
    integ.setup_integrator()
    return pas, particles, integ


class SolverView:
    """What the time-step functions read from a Solver."""

    def __init__(self, integrator, dt, dim):
        self.integrator = integrator
        self.dt = dt
        self.dim = dim
        self.count = 0


def stepper(arrays, types, params, dim, build_dir=BUILD_DIR):
    """The reference's particle arrays and a function that advances them one
    predictor-corrector step of the summation-density scheme.  With
    params["cfl"] > 0 a step is the solver loop's with the CFL rule (count,
    Particles.update, ViscousAndForceBasedTimeStep.compute_time_step,
    integrate(dt)); otherwise Particles.update and integrate(params["dt"])."""
    R = modules(build_dir)
    pas, particles, integ = build_sim(R, arrays, types, params, dim)
    cfl = params.get("cfl", 0.0) > 0.0
    if cfl:
        tsf = R["T"].ViscousAndForceBasedTimeStep(cfl=params["cfl"], co=params["c0"],
                                                  particles=particles)
        sv = SolverView(integ, params["dt_initial"], dim)

    def step():
        particles.update()
        if cfl:
            sv.count += 1
            integ.integrate(tsf.compute_time_step(sv))
        else:
            integ.integrate(params.get("dt", 1e-5))

    return pas, step


def time_steps(arrays, types, params, dim, steps, warmup=1, build_dir=BUILD_DIR):
    """Wall time of `steps` steps of `stepper` after `warmup` untimed ones,
    on one host thread (the reference's particle path has no threads)."""
    pas, step = stepper(arrays, types, params, dim, build_dir)
    for _ in range(warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = time.perf_counter() - t0
    n = sum(pa.get_number_of_particles() for pa in pas)
    return {"seconds": dt, "steps": steps, "steps_per_s": steps / dt, "particles": n}
