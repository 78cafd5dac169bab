"""Host-side logic of the reference-shaped API (no device work): particle
array defaults and properties, operation -> calc grouping, and recognition
of the fused particle-update scheme."""
import os

import numpy as np
import pytest
import torch

import pysph_b200.base.api as base
import pysph_b200.sph.api as sph
import pysph_b200.solver.api as solver

Fluid, Solid = base.Fluid, base.Solid


def arrays(device="cpu"):
    x = np.linspace(0, 1, 11)
    f = base.get_particle_array(name="fluid", type=Fluid, x=x, y=x * 0, h=np.full(11, 0.2),
                                device=device)
    w = base.get_particle_array(name="wall", type=Solid, x=x, y=x * 0 - 0.1,
                                h=np.full(11, 0.2), device=device)
    return f, w


def test_get_particle_array_defaults():
    # S/base/particle_array.pyx:1428-1470
    pa = base.get_particle_array(x=[0.0, 1.0, 2.0], name="a", device="cpu", cl_precision="double")
    assert pa.name == "a" and pa.particle_type == Fluid
    assert pa.get_number_of_particles() == 3
    for name, v in {"m": 1.0, "h": 1.0, "rho": 1.0, "p": 0.0, "cs": 0.0, "u": 0.0}.items():
        assert torch.all(pa.get(name) == v)
    assert pa.get("idx").tolist() == [0, 1, 2]
    assert pa.get("tag").dtype == torch.int64 and int(pa.get("tag").sum()) == 0
    assert pa.num_real_particles == 3
    pa.set(u=np.array([1.0, 2.0, 3.0]))
    assert pa.u.tolist() == [1.0, 2.0, 3.0]
    x, u = pa.get("x", "u")
    assert x.tolist() == [0.0, 1.0, 2.0]
    pa.add_property({"name": "dt_fac"})
    assert pa.has_array("dt_fac")
    pa.copy_over_properties({"u": "_tmpx"})
    assert pa._tmpx.tolist() == [1.0, 2.0, 3.0]
    pa.set_to_zero(["_tmpx"])
    assert float(pa._tmpx.abs().sum()) == 0
    pa.remove_particles([1])
    assert pa.get_number_of_particles() == 2 and pa.u.tolist() == [1.0, 3.0]
    with pytest.raises(AssertionError):
        base.get_particle_array(x=[0.0], type=99)


def test_operation_grouping():
    # S/solver/sph_equation.py:101-228: one calc per dest, one func per source
    f, w = arrays()
    particles = base.Particles([f, w])
    k = base.CubicSplineKernel(dim=2)
    op = solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid, Solid],
                             from_types=[Fluid, Solid], updates=["rho"], id="sd")
    calcs = op.get_calcs(particles, k)
    assert [c.dest.name for c in calcs] == ["fluid", "wall"]
    assert [[s.name for s in c.sources] for c in calcs] == [["fluid", "wall"]] * 2
    assert calcs[0].id == "sd_fluid"
    mom = solver.SPHIntegration(sph.MomentumEquation.withargs(alpha=0.1, beta=0.0),
                                on_types=[Fluid], from_types=[Fluid, Solid],
                                updates=["u", "v"], id="mom")
    mc = mom.get_calcs(particles, k)
    assert len(mc) == 1 and mc[0].integrates and mc[0].to_reset == ["dt_fac"]
    assert f.has_array("dt_fac")
    with pytest.raises(ValueError):
        solver.SPHOperation(sph.TaitEquation.withargs(), on_types=[Fluid],
                            from_types=[Fluid], updates=["p", "cs"], id="eos").get_calcs(particles, k)


def dam_solver(order=("sd", "eos", "mom", "grav", "step"), gravity=True):
    f, w = arrays()
    particles = base.Particles([f, w])
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    ops = {
        "sd": solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid, Solid],
                                  from_types=[Fluid, Solid], updates=["rho"], id="sd"),
        "eos": solver.SPHOperation(sph.TaitEquation.withargs(co=62.6, ro=1000.0),
                                   on_types=[Fluid, Solid], updates=["p", "cs"], id="eos"),
        "mom": solver.SPHIntegration(sph.MomentumEquation.withargs(alpha=0.1, beta=0.0),
                                     on_types=[Fluid], from_types=[Fluid, Solid],
                                     updates=["u", "v"], id="mom"),
        "grav": solver.SPHIntegration(sph.GravityForce.withargs(gy=-9.81),
                                      on_types=[Fluid], updates=["u", "v"], id="grav"),
    }
    for oid in order:
        if oid == "step":
            s.add_operation_step([Fluid])
        elif oid != "grav" or gravity:
            s.add_operation(ops[oid])
    s.setup(particles)
    return s


def test_fused_plan_recognised():
    s = dam_solver()
    plan = s.integrator.plan
    assert plan is not None
    assert plan.scheme.rho_src == {0: [0, 1], 1: [0, 1]}
    assert plan.scheme.mom_src == {0: [0, 1]}
    assert plan.scheme.tait_on == (0, 1) and plan.scheme.step_on == (0,)
    assert plan.params.c0 == 62.6 and plan.params.rho0 == 1000.0
    assert plan.params.alpha == 0.1 and plan.params.beta == 0.0
    assert plan.params.gravity == (0.0, -9.81, 0.0)
    # initial-value and acceleration properties (S/solver/integrator.py:212-260)
    f = s.particles.arrays[0]
    for name in ("_u0", "_v0", "_x0", "_y0", "_a_u_1", "_a_v_1", "_a_x_1", "_a_y_1"):
        assert f.has_array(name)


def test_fused_plan_rejects_other_orders():
    # Tait before SPHRho reads the old density: not the fused scheme
    assert dam_solver(order=("eos", "sd", "mom", "grav", "step")).integrator.plan is None
    assert dam_solver(gravity=False).integrator.plan.params.gravity == (0.0, 0.0, 0.0)


def test_unsupported_features_fail_loudly():
    f, w = arrays()
    with pytest.raises(NotImplementedError):
        base.Particles([f], periodic_domain=object())
    with pytest.raises(NotImplementedError):
        sph.MomentumEquation(f, f, deltap=0.1)
    # as the reference: XSPH needs the position stepping it corrects
    with pytest.raises(AssertionError):
        solver.Solver(dim=2).add_operation_xsph(eps=0.5)


def test_kernel_host_formulas():
    k = base.CubicSplineKernel(dim=2)
    assert k.radius() == 2.0
    assert k.py_fac(0.01) == pytest.approx(10 / (7 * np.pi) / 1e-4)
    g = base.Point()
    k.py_gradient(base.Point(0.5, 0, 0), base.Point(0, 0, 0), 1.0, g)
    assert g.x < 0 and g.y == 0


def continuity_solver(xsph=True):
    """The reference dam-break example's scheme (examples/dam-break/
    dam_break.py:184-241)."""
    f, w = arrays()
    particles = base.Particles([f, w])
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=62.6, ro=1000.0),
                                        on_types=[Fluid, Solid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(sph.SPHDensityRate.withargs(hks=False),
                                          on_types=[Fluid, Solid], from_types=[Fluid, Solid],
                                          updates=["rho"], id="density"))
    s.add_operation(solver.SPHIntegration(sph.MomentumEquation.withargs(alpha=0.1, beta=0.0),
                                          on_types=[Fluid], from_types=[Fluid, Solid],
                                          updates=["u", "v"], id="mom"))
    s.add_operation(solver.SPHIntegration(sph.GravityForce.withargs(gy=-9.81),
                                          on_types=[Fluid], updates=["u", "v"], id="grav"))
    s.add_operation_step([Fluid])
    if xsph:
        s.add_operation_xsph(eps=0.5)
    s.setup(particles)
    return s


def test_fused_plan_continuity_scheme():
    plan = continuity_solver().integrator.plan
    assert plan is not None
    sc = plan.scheme
    assert sc.continuity and sc.rho_src == {}
    assert sc.rate_src == {0: [0, 1], 1: [0, 1]} and sc.mom_src == {0: [0, 1]}
    assert sc.xsph_src == {0: [0]} and sc.xsph_eps == 0.5
    assert sc.tait_on == (0, 1) and sc.step_on == (0,)
    assert plan.tait_only == ()
    # rho is integrated on both arrays (S/solver/integrator.py:212-260)
    for pa in continuity_solver().particles.arrays:
        assert pa.has_array("_rho0") and pa.has_array("_a_rho_1")
    assert continuity_solver(xsph=False).integrator.plan.scheme.xsph_src == {}


def test_output_format_v1_round_trip(tmp_path):
    """Solver.dump_output writes the reference's format version 1 (an .npz
    with version, solver_data and arrays as object arrays);
    solver.utils.load reads it back into ParticleArrays, and
    Solver.load_output resumes from it."""
    from pysph_b200.solver import utils
    s = dam_solver()
    s.set_output_directory(str(tmp_path))
    f = s.particles.arrays[0]
    f.set(u=np.linspace(0.0, 1.0, 11))
    s.count, s.t = 7, 0.25
    path = s.dump_output(1e-4, *s.print_properties)
    assert os.path.basename(path) == "Solver_7.npz"
    raw = np.load(path, allow_pickle=True)
    assert int(raw["version"]) == 1 and raw["arrays"].dtype == object
    data = utils.load(path)
    assert data["solver_data"] == {"dt": 1e-4, "t": 0.25, "count": 7}
    g = data["arrays"]["fluid"]
    assert np.allclose(g.get("u").cpu().numpy(), np.linspace(0.0, 1.0, 11))
    assert "_u0" not in g.get_property_names() and "_tmpx" in g.get_property_names()
    s.set_output_printing_level(True)
    assert "_u0" in utils.load(s.dump_output(1e-4))["arrays"]["fluid"].get_property_names()
    # resume
    f.set(u=np.zeros(11))
    s.count, s.t = 0, 0.0
    assert s.load_output("?") == [7]
    s.load_output(7)
    assert s.count == 7 and s.t == 0.25
    assert np.allclose(f.get("u").cpu().numpy(), np.linspace(0.0, 1.0, 11))
    with pytest.raises(IOError):
        s.load_output(3)


def test_variable_h_and_hks_options():
    """Particles(variable_h=True) selects the symmetric neighbour sets; the
    functions' hks option reaches the fused scheme when every pair function
    agrees on it, and calc by calc otherwise."""
    f, w = arrays()
    assert base.Particles([f], variable_h=True).variable_h
    assert sph.XSPHCorrection(f, f, hks=True).hks
    sc = continuity_solver().integrator.plan.scheme
    assert not sc.hks

    def solver_hks(rho_hks, mom_hks):
        f, _ = arrays()
        particles = base.Particles([f], variable_h=True)
        s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator)
        s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(hks=rho_hks), on_types=[Fluid],
                                            from_types=[Fluid], updates=["rho"], id="sd"))
        s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=62.6, ro=1000.0),
                                            on_types=[Fluid], updates=["p", "cs"], id="eos"))
        s.add_operation(solver.SPHIntegration(
            sph.MomentumEquation.withargs(alpha=0.1, beta=0.0, hks=mom_hks),
            on_types=[Fluid], from_types=[Fluid], updates=["u", "v"], id="mom"))
        s.add_operation_step([Fluid])
        s.setup(particles)
        return s.integrator.plan

    assert solver_hks(True, True).scheme.hks
    assert not solver_hks(False, False).scheme.hks
    assert solver_hks(True, False) is None


def test_other_kernels_host_formulas():
    """QuinticSplineKernel / WendlandQuinticSplineKernel host formulas
    against the values the reference's own kernels gave (fixture), quirks
    included; 2D only, as in the reference."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "kernels.npz"))
    rs = np.linspace(0.0, 3.2, 65)
    for kname, radius in (("QuinticSplineKernel", 3.0), ("WendlandQuinticSplineKernel", 2.0)):
        k = getattr(base, kname)(dim=2)
        assert k.radius() == radius
        w, gr = [], []
        for r in rs:
            pa, pb = base.Point(0.6 * r, 0.8 * r, 0.0), base.Point(0.0, 0.0, 0.0)
            w.append(k.py_function(pa, pb, 1.1))
            q = base.Point()
            k.py_gradient(pa, pb, 1.1, q)
            gr.append((q.x, q.y, q.z))
        np.testing.assert_allclose(w, g[f"{kname}_w"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(gr, g[f"{kname}_grad"], rtol=1e-12, atol=1e-14)
        with pytest.raises(NotImplementedError):
            getattr(base, kname)(dim=3)


def test_fused_plan_kernel_type():
    f, _ = arrays()
    particles = base.Particles([f])
    s = solver.Solver(dim=2, integrator_type=solver.PredictorCorrectorIntegrator,
                      kernel=base.QuinticSplineKernel(dim=2))
    s.add_operation(solver.SPHOperation(sph.SPHRho.withargs(), on_types=[Fluid],
                                        from_types=[Fluid], updates=["rho"], id="sd"))
    s.add_operation(solver.SPHOperation(sph.TaitEquation.withargs(co=62.6, ro=1000.0),
                                        on_types=[Fluid], updates=["p", "cs"], id="eos"))
    s.add_operation(solver.SPHIntegration(
        sph.MomentumEquation.withargs(alpha=0.1, beta=0.0), on_types=[Fluid],
        from_types=[Fluid], updates=["u", "v"], id="mom"))
    s.add_operation_step([Fluid])
    s.setup(particles)
    assert s.integrator.plan.kernel == 3
    assert dam_solver().integrator.plan.kernel == 1
