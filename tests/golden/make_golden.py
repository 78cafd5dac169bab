"""Write the golden fixtures of tests/golden from the reference itself.

    python oracle/build_reference.py --ref <reference checkout>
                                                # patched build in oracle/_ref/refbuild
    python tests/golden/make_golden.py          # writes tests/golden/*.npz

Every fixture is computed by the reference's own FP64 Cython path, through
its own API: get_particle_array, Particles (CellManager + NNPSManager),
SPHCalc / SPHOperation / SPHIntegration, PredictorCorrectorIntegrator and
ViscousAndForceBasedTimeStep, with the solver loop's order of calls
(S/solver/solver.py:546-566).  Inputs come from pysph_b200.workloads
(seeded, synthetic).  Fixtures:

  square.npz      the 4-particle unit square of the reference's function
                  tests: SPHRho, TaitEquation, SPHPressureGradient and
                  MomentumEquation outputs
  drop.npz        elliptical drop, dx = 0.025 (5,025 particles): neighbour
                  lists in the reference's order, the first stage's rho, p,
                  cs, accelerations and dt_fac, and the state after 1 and 10
                  predictor-corrector steps of dt = 1e-5
  lattice3d.npz   3D jittered 16^3 lattice (h = 1.2 dx): neighbour lists,
                  SPHRho and SPHPressureGradient
  dam.npz         dam break at dx = 0.05 with walls: 5 steps with the CFL
                  time step (the dt sequence and the final state)
  npz_ref_read.npz  output format v1 across both implementations: what the
                  reference's load reads from npz_repo_written.npz (written
                  here by Solver.dump_output); npz_ref_written.npz is a file
                  the reference's own savez wrote
  avisc.npz       the split-form MonaghanArtificialViscosity: the unit square,
                  and a drop scheme with SPHPressureGradient + the viscosity
                  (first stage and 5 steps)
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.reference import (SolverView as _SolverView, build_sim,  # noqa: E402
                              make_array, modules as ref_modules, scheme_ops)
from pysph_b200 import workloads as W  # noqa: E402

PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")


def lists_of(R, particles, src, dst, radius_scale=2.0):
    loc = particles.nnps_manager.get_neighbor_particle_locator(src, dst, radius_scale)
    n = dst.get_number_of_particles()
    out = [np.asarray(loc.py_get_nearest_particles(i).get_npy_array(), np.int32).copy()
           for i in range(n)]
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum([len(a) for a in out])
    return off, np.concatenate(out) if out else np.zeros(0, np.int32)


def state(pas, names=("x", "y", "u", "v", "rho", "p", "cs")):
    return {f"{n}_{i}": np.asarray(pa.get(n), np.float64).copy()
            for i, pa in enumerate(pas) for n in names}


def square(R):
    x = np.array([0, 0, 1, 1], np.float64)
    y = np.array([0, 1, 1, 0], np.float64)
    out = {}
    kernel = R["K"].CubicSplineKernel(dim=2)
    for fname, fac, outs in (
            ("rho", lambda pa: R["D"].SPHRho.withargs().get_func(pa, pa), 1),
            ("tait", lambda pa: R["E"].TaitEquation.withargs(gamma=7.0).get_func(pa, pa), 2),
            ("pgrad", lambda pa: R["PF"].SPHPressureGradient.withargs().get_func(pa, pa), 3),
            ("mom", lambda pa: R["PF"].MomentumEquation.withargs(
                alpha=1.0, beta=1.0, gamma=1.4, eta=0.1).get_func(pa, pa), 3)):
        pa = R["PA"].get_particle_array(name="test", x=x.copy(), y=y.copy(), z=np.zeros(4),
                                        m=np.ones(4), u=np.array([1, 0, 0, -1.0]),
                                        p=np.array([0, 0, 1, 1.0]),
                                        cs=np.array([1.0, 2.0, 0.5, 1.5]),
                                        rho=np.array([1000.0, 1001.5, 998.0, 1010.0])
                                        if fname == "tait" else np.ones(4))
        particles = R["P"].Particles([pa])
        calc = R["C"].SPHCalc(particles, [pa], pa, kernel, [fac(pa)], ["rho"])
        calc.sph()
        for k, n in enumerate(("_tmpx", "_tmpy", "_tmpz")[:outs]):
            out[f"{fname}_{k}"] = np.asarray(pa.get(n), np.float64).copy()
    return out


def drop(R):
    arrays, types, params = W.elliptical_drop(dx=0.025)
    pas, particles, integ = build_sim(R, arrays, types, params, 2)
    out = {f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS}
    off, idx = lists_of(R, particles, pas[0], pas[0])
    out["nbr_off"], out["nbr_idx"] = off, idx
    out["cell_size"] = particles.cell_manager.cell_size
    # the first stage: Integrator.eval at t = 0
    integ.save_initial_arrays()
    integ.reset_accelerations(step=1)
    integ.eval()
    out.update({f"stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                for n in ("rho", "p", "cs", "_a_u_1", "_a_v_1", "dt_fac")})
    pas, particles, integ = build_sim(R, arrays, types, params, 2)
    for step in range(10):
        particles.update()
        integ.integrate(1e-5)
        if step == 0:
            out.update({f"step1_{k}": v for k, v in state(pas).items()})
    out.update({f"step10_{k}": v for k, v in state(pas).items()})
    return out


def lattice(R):
    arrays, types, params = W.lattice3d(n=16)
    a = arrays[0]
    pa = make_array(R, a, "lat", 0)
    particles = R["P"].Particles([pa])
    kernel = R["K"].CubicSplineKernel(dim=3)
    out = {f"in_{k}": np.asarray(a[k]) for k in PROPS}
    off, idx = lists_of(R, particles, pa, pa)
    out["nbr_off"], out["nbr_idx"] = off, idx
    out["cell_size"] = particles.cell_manager.cell_size
    calc = R["C"].SPHCalc(particles, [pa], pa, kernel,
                          [R["D"].SPHRho.withargs().get_func(pa, pa)], ["rho"])
    calc.sph("_tmpx")
    out["rho_sum"] = np.asarray(pa.get("_tmpx"), np.float64).copy()
    calc = R["C"].SPHCalc(particles, [pa], pa, kernel,
                          [R["PF"].SPHPressureGradient.withargs().get_func(pa, pa)],
                          ["u", "v", "w"], integrates=True)
    for n in ("_tmpx", "_tmpy", "_tmpz"):
        pa.get(n)[:] = 0
    calc.sph("_tmpx", "_tmpy", "_tmpz")
    for k, n in enumerate(("_tmpx", "_tmpy", "_tmpz")):
        out[f"pgrad_{k}"] = np.asarray(pa.get(n), np.float64).copy()
    return out


def dam(R):
    arrays, types, params = W.dam_break(dx=0.05)
    pas, particles, integ = build_sim(R, arrays, types, params, 2)
    out = {f"in{i}_{k}": np.asarray(arrays[i][k]) for i in range(2) for k in PROPS}
    tsf = R["T"].ViscousAndForceBasedTimeStep(cfl=params["cfl"], co=params["c0"],
                                              particles=particles)
    sv = _SolverView(integ, params["dt_initial"], 2)
    dts = []
    for _ in range(5):
        sv.count += 1
        particles.update()
        dt = tsf.compute_time_step(sv)
        integ.integrate(dt)
        dts.append(dt)
    out["dts"] = np.asarray(dts)
    out.update({f"step5_{k}": v for k, v in state(pas).items()})
    return out


XSPH_EPS = 0.5   # XSPHCorrection's default eps


def integrators(R):
    """The elliptical drop (dx = 0.05) stepped by the reference's Euler, RK2
    and RK4 integrators, 5 steps of dt = 1e-5, summation density and, for
    RK2, the continuity scheme too."""
    arrays, types, params = W.elliptical_drop(dx=0.05)
    out = {f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS}
    I = R["I"]
    for name, cls, eps in (("euler", I.EulerIntegrator, None), ("rk2", I.RK2Integrator, None),
                           ("rk4", I.RK4Integrator, None), ("rk2cont", I.RK2Integrator, XSPH_EPS)):
        pas, particles, integ = build_sim(R, arrays, types, params, 2, eps, integrator=cls)
        for step in range(5):
            particles.update()
            integ.integrate(1e-5)
            if step == 0:
                out.update({f"{name}_step1_{k}": v for k, v in state(pas).items()})
        out.update({f"{name}_step5_{k}": v for k, v in state(pas).items()})
    return out


def drop_cont(R):
    """Elliptical drop with the continuity scheme: first-stage rates, then 10
    steps of dt = 1e-5."""
    arrays, types, params = W.elliptical_drop(dx=0.025)
    pas, particles, integ = build_sim(R, arrays, types, params, 2, XSPH_EPS)
    out = {f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS}
    integ.save_initial_arrays()
    integ.reset_accelerations(step=1)
    integ.eval()
    out.update({f"stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                for n in ("p", "cs", "_a_rho_1", "_a_u_1", "_a_v_1", "_a_x_1", "_a_y_1",
                          "dt_fac")})
    pas, particles, integ = build_sim(R, arrays, types, params, 2, XSPH_EPS)
    for step in range(10):
        particles.update()
        integ.integrate(1e-5)
        if step == 0:
            out.update({f"step1_{k}": v for k, v in state(pas).items()})
    out.update({f"step10_{k}": v for k, v in state(pas).items()})
    return out


def dam_cont(R):
    """The dam break (dx = 0.05) with the continuity scheme of the
    reference's dam-break example: first-stage rates of both arrays, then 5
    CFL steps."""
    arrays, types, params = W.dam_break(dx=0.05)
    pas, particles, integ = build_sim(R, arrays, types, params, 2, XSPH_EPS)
    out = {f"in{i}_{k}": np.asarray(arrays[i][k]) for i in range(2) for k in PROPS}
    integ.save_initial_arrays()
    integ.reset_accelerations(step=1)
    integ.eval()
    for i in range(2):
        names = ("p", "cs", "_a_rho_1") + (("_a_u_1", "_a_v_1", "_a_x_1", "_a_y_1", "dt_fac")
                                           if i == 0 else ())
        out.update({f"stage0_{n}_{i}": np.asarray(pas[i].get(n), np.float64).copy()
                    for n in names})
    pas, particles, integ = build_sim(R, arrays, types, params, 2, XSPH_EPS)
    tsf = R["T"].ViscousAndForceBasedTimeStep(cfl=params["cfl"], co=params["c0"],
                                              particles=particles)
    sv = _SolverView(integ, params["dt_initial"], 2)
    dts = []
    for _ in range(5):
        sv.count += 1
        particles.update()
        dt = tsf.compute_time_step(sv)
        integ.integrate(dt)
        dts.append(dt)
    out["dts"] = np.asarray(dts)
    out.update({f"step5_{k}": v for k, v in state(pas).items()})
    return out


def varh_drop():
    """The drop (dx = 0.05) with smoothing lengths growing from 1.0 to 1.4
    times 1.3 dx across x."""
    arrays, types, params = W.elliptical_drop(dx=0.05)
    a = arrays[0]
    a["h"] = 1.3 * 0.05 * (1.0 + 0.2 * (a["x"] + 1.0))
    return arrays, types, params


def varh(R):
    """Variable smoothing length: the reference's symmetric neighbour lists
    (VarHNbrParticleLocator) with hks kernels, summation and continuity
    schemes: lists, the first stage and 5 PC steps."""
    arrays, types, params = varh_drop()
    out = {f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS}
    for name, eps in (("sum", None), ("cont", XSPH_EPS)):
        pas, particles, integ = build_sim(R, arrays, types, params, 2, eps,
                                          variable_h=True, hks=True)
        if name == "sum":
            off, idx = lists_of(R, particles, pas[0], pas[0])
            out["nbr_off"], out["nbr_idx"] = off, idx
        integ.save_initial_arrays()
        integ.reset_accelerations(step=1)
        integ.eval()
        names = ("rho", "p", "cs", "_a_u_1", "_a_v_1", "dt_fac") + (
            ("_a_rho_1", "_a_x_1", "_a_y_1") if eps else ())
        out.update({f"{name}_stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                    for n in names})
        pas, particles, integ = build_sim(R, arrays, types, params, 2, eps,
                                          variable_h=True, hks=True)
        for _ in range(5):
            particles.update()
            integ.integrate(1e-5)
        out.update({f"{name}_step5_{k}": v for k, v in state(pas).items()})
    return out


def varh3d_case():
    """A jittered 10^3 lattice with h growing from 1.2 to 1.56 dx along z
    and random velocities (so the viscosity acts)."""
    arrays, types, params = W.lattice3d(n=10)
    a = arrays[0]
    dx = 0.1
    a["h"] = 1.2 * dx * (1.0 + 0.3 * a["z"])
    rng = np.random.default_rng(3)
    for c in ("u", "v", "w"):
        a[c] = rng.normal(0.0, 0.5, len(a["x"]))
    params = dict(c0=10.0, rho0=1.0, alpha=0.1, beta=0.0, eta=0.1, gravity=(0.0, 0.0, 0.0))
    return arrays, types, params


def varh3d(R):
    """Variable h with hks kernels in 3D (summation scheme): the symmetric
    lists, the first stage and 3 PC steps."""
    arrays, types, params = varh3d_case()
    out = {f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS}
    pas, particles, integ = build_sim(R, arrays, types, params, 3, variable_h=True, hks=True)
    off, idx = lists_of(R, particles, pas[0], pas[0])
    out["nbr_off"], out["nbr_idx"] = off, idx
    integ.save_initial_arrays()
    integ.reset_accelerations(step=1)
    integ.eval()
    out.update({f"stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                for n in ("rho", "p", "cs", "_a_u_1", "_a_v_1", "_a_w_1", "dt_fac")})
    pas, particles, integ = build_sim(R, arrays, types, params, 3, variable_h=True, hks=True)
    for _ in range(3):
        particles.update()
        integ.integrate(1e-4)
    out.update({f"step3_{k}": v for k, v in state(pas, ("x", "y", "z", "u", "v", "w", "rho",
                                                         "p")).items()})
    return out


def kernels(R):
    """The quintic spline and Wendland quintic kernels (2D): W and grad W on
    a line of distances, and the drop (dx = 0.05) with each kernel under both
    schemes: neighbour lists (radius 3h for the quintic), the first stage and
    5 PC steps.  Wendland's normalisation (7 pi / 4 where 7 / (4 pi) is
    meant) makes the summed density pi^2 times the rest density, so its
    summation case takes TaitEquation ro = pi^2 to keep the drop intact."""
    out = {}
    arrays, types, params = W.elliptical_drop(dx=0.05)
    out.update({f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS})
    rs = np.linspace(0.0, 3.2, 65)
    for kname in ("QuinticSplineKernel", "WendlandQuinticSplineKernel"):
        k = getattr(R["K"], kname)(dim=2)
        pb = R["Point"](0.0, 0.0, 0.0)
        w, g = [], []
        for r in rs:
            pa = R["Point"](0.6 * r, 0.8 * r, 0.0)
            w.append(k.py_function(pa, pb, 1.1))
            gr = R["Point"]()
            k.py_gradient(pa, pb, 1.1, gr)
            g.append((gr.x, gr.y, gr.z))
        out[f"{kname}_w"] = np.array(w)
        out[f"{kname}_grad"] = np.array(g)
        for name, eps in (("sum", None), ("cont", XSPH_EPS)):
            p = dict(params)
            if kname.startswith("Wendland") and name == "sum":
                p["rho0"] = float(np.pi ** 2)
            out[f"{kname}_{name}_rho0"] = np.float64(p["rho0"])
            pas, particles, integ = build_sim(R, arrays, types, p, 2, eps, kernel=kname)
            if name == "sum":
                off, idx = lists_of(R, particles, pas[0], pas[0], k.radius())
                out[f"{kname}_nbr_off"], out[f"{kname}_nbr_idx"] = off, idx
            integ.save_initial_arrays()
            integ.reset_accelerations(step=1)
            integ.eval()
            names = ("rho", "p", "cs", "_a_u_1", "_a_v_1", "dt_fac") + (
                ("_a_rho_1", "_a_x_1", "_a_y_1") if eps else ())
            out.update({f"{kname}_{name}_stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                        for n in names})
            pas, particles, integ = build_sim(R, arrays, types, p, 2, eps, kernel=kname)
            for _ in range(5):
                particles.update()
                integ.integrate(1e-5)
            out.update({f"{kname}_{name}_step5_{k_}": v for k_, v in state(pas).items()})
    return out


def avisc(R):
    """The split-form MonaghanArtificialViscosity (S/sph/funcs/
    viscosity_funcs.pyx:19-157): on the 4-particle unit square (alpha =
    beta = 1, with the constructor's eta = 0.1 ignored and, once, the
    attribute set to 0.1 by hand), and in a scheme of its own on the
    elliptical drop at dx = 0.05 -- SPHRho, TaitEquation, then
    SPHPressureGradient and MonaghanArtificialViscosity (alpha 0.1, beta 0)
    both integrating u, v, and PositionStepping: the first stage's
    accelerations and dt_fac, and 5 predictor-corrector steps of dt = 1e-5."""
    out = {}
    x = np.array([0, 0, 1, 1], np.float64)
    y = np.array([0, 1, 1, 0], np.float64)
    kernel = R["K"].CubicSplineKernel(dim=2)
    for name, eta_attr in (("square", None), ("square_eta", 0.1)):
        pa = R["PA"].get_particle_array(name="test", x=x.copy(), y=y.copy(), z=np.zeros(4),
                                        m=np.ones(4), u=np.array([1, 0, 0, -1.0]),
                                        v=np.array([0, 0.5, 0, 0.25]), h=np.ones(4),
                                        p=np.array([0, 0, 1, 1.0]),
                                        cs=np.array([1.0, 2.0, 0.5, 1.5]),
                                        rho=np.array([1.0, 1.5, 0.98, 1.1]))
        particles = R["P"].Particles([pa])
        f = R["V"].MonaghanArtificialViscosity.withargs(alpha=1.0, beta=1.0, gamma=1.4,
                                                        eta=0.1).get_func(pa, pa)
        if eta_attr is not None:
            f.eta = eta_attr
        calc = R["C"].SPHCalc(particles, [pa], pa, kernel, [f], ["u", "v"], integrates=True)
        for n in ("_tmpx", "_tmpy", "_tmpz"):
            pa.get(n)[:] = 0
        calc.sph("_tmpx", "_tmpy", "_tmpz")
        for k, n in enumerate(("_tmpx", "_tmpy", "_tmpz")):
            out[f"{name}_{k}"] = np.asarray(pa.get(n), np.float64).copy()
        out[f"{name}_dt_fac"] = np.asarray(pa.get("dt_fac"), np.float64).copy()
    arrays, types, params = W.elliptical_drop(dx=0.05)
    EQ, D, E, PF, POS, V = R["EQ"], R["D"], R["E"], R["PF"], R["POS"], R["V"]

    def sim():
        pas = [make_array(R, arrays[0], "fluid", types[0])]
        particles = R["P"].Particles(pas)
        ops = [EQ.SPHOperation(D.SPHRho.withargs(), on_types=[0], from_types=[0],
                               updates=["rho"], id="sd"),
               EQ.SPHOperation(E.TaitEquation.withargs(co=params["c0"], ro=params["rho0"]),
                               on_types=[0], updates=["p", "cs"], id="eos"),
               EQ.SPHIntegration(PF.SPHPressureGradient.withargs(), on_types=[0],
                                 from_types=[0], updates=["u", "v"], id="pgrad"),
               EQ.SPHIntegration(V.MonaghanArtificialViscosity.withargs(
                   alpha=params["alpha"], beta=params["beta"]), on_types=[0],
                   from_types=[0], updates=["u", "v"], id="avisc"),
               EQ.SPHIntegration(POS.PositionStepping.withargs(), on_types=[0],
                                 updates=["x", "y"], id="step")]
        calcs = []
        for op in ops:
            calcs.extend(op.get_calcs(particles, R["K"].CubicSplineKernel(dim=2)))
        integ = R["I"].PredictorCorrectorIntegrator(particles, calcs)
        integ.setup_integrator()
        return pas, particles, integ

    out.update({f"in_{k}": np.asarray(arrays[0][k]) for k in PROPS})
    pas, particles, integ = sim()
    integ.save_initial_arrays()
    integ.reset_accelerations(step=1)
    integ.eval()
    out.update({f"stage0_{n}": np.asarray(pas[0].get(n), np.float64).copy()
                for n in ("rho", "p", "cs", "_a_u_1", "_a_v_1", "dt_fac")})
    pas, particles, integ = sim()
    for _ in range(5):
        particles.update()
        integ.integrate(1e-5)
    out.update({f"step5_{k}": v for k, v in state(pas).items()})
    return out


def npz_interop(R):
    """The output format v1 (S/solver/utils.py:34-186, 294-340;
    S/solver/solver.py:605-695) across the two implementations, on the
    dam break at dx = 0.1 (fluid and wall arrays) with solver data dt =
    1e-4, t = 0.25, count = 7:

    * the reference writes npz_ref_written.npz with its own savez, from the
      dicts its Solver.dump_output assembles (ParticleArray.
      get_property_arrays);
    * this build writes npz_repo_written.npz through its Solver.dump_output,
      and the reference's own load reads it back: what it read is this
      function's fixture (npz_ref_read.npz)."""
    import shutil
    import tempfile
    sys.path.insert(0, ROOT)
    import pysph.solver.utils as RU
    from pysph_b200.base import api as base
    from pysph_b200.solver.solver import Solver
    arrays, types, params = W.dam_break(dx=0.1)
    names = ("fluid", "wall")
    pas = [make_array(R, a, n, t) for a, n, t in zip(arrays, names, types)]
    props = {"arrays": {pa.name: pa.get_property_arrays(all=False) for pa in pas},
             "solver_data": {"dt": 1e-4, "t": 0.25, "count": 7}}
    RU.savez(os.path.join(HERE, "npz_ref_written.npz"), version=1, **props)
    rpas = [base.get_particle_array(name=n, type=t, device="cpu",
                                    **{k: np.asarray(a[k], np.float64) for k in PROPS
                                       if k in a})
            for a, n, t in zip(arrays, names, types)]
    s = Solver(dim=2)
    s.particles = base.Particles(rpas)
    s.t, s.count = 0.25, 7
    tmp = tempfile.mkdtemp()
    try:
        s.output_directory = tmp
        s.fname = "npz_repo_written"
        path = s.dump_output(1e-4)
        shutil.copy(path, os.path.join(HERE, "npz_repo_written.npz"))
    finally:
        shutil.rmtree(tmp)
    d = RU.load(os.path.join(HERE, "npz_repo_written.npz"))
    out = {f"solver_{k}": np.float64(v) for k, v in d["solver_data"].items()}
    for name, pa in d["arrays"].items():
        pnames = sorted(pa.properties.keys())
        out[f"{name}__names"] = np.array(pnames)
        for p in pnames:
            out[f"{name}_{p}"] = np.asarray(pa.get(p)).copy()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--build", default=os.path.join(ROOT, "oracle", "_ref", "refbuild"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", nargs="*", default=None, help="fixture names to write")
    a = ap.parse_args()
    R = ref_modules(a.build)
    for name, fn in (("square", square), ("drop", drop), ("lattice3d", lattice), ("dam", dam),
                     ("drop_cont", drop_cont), ("dam_cont", dam_cont),
                     ("integrators", integrators), ("varh", varh), ("kernels", kernels),
                     ("varh3d", varh3d), ("avisc", avisc), ("npz_ref_read", npz_interop)):
        if a.only and name not in a.only:
            continue
        data = fn(R)
        path = os.path.join(a.out, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
