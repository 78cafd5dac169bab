"""The oracle against fixtures written by the reference itself
(tests/golden/make_golden.py runs the reference's own FP64 Cython path).

Neighbour lists are compared in the reference's own order (cells x-major,
ascending index, self swapped last); floating-point results must agree to
the last bit wherever the reference's arithmetic is restated operation by
operation (summation density, Tait, momentum, the integrator), which is the
claim of oracle/sph_oracle.c.
"""
import os

import numpy as np
import pytest

from oracle import OracleArray, OracleSystem
from pysph_b200.engine import continuity_scheme, fluid_scheme

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def oracle_for(g, prefixes, scheme, params, dim):
    arrs = [OracleArray(f"a{i}", **{k: g[f"{p}{k}"].copy() for k in PROPS})
            for i, p in enumerate(prefixes)]
    return OracleSystem(arrs, dim=dim, rho_src=scheme.rho_src, tait_on=scheme.tait_on,
                        mom_src=scheme.mom_src, step_on=scheme.step_on,
                        rate_src=scheme.rate_src, xsph_src=scheme.xsph_src,
                        xsph_eps=scheme.xsph_eps, **params)


DROP = dict(c0=1400.0, rho0=1.0, gamma=7.0, alpha=0.1, beta=0.0, eta=0.1)


def test_drop_neighbour_lists_in_reference_order():
    g = load("drop")
    o = oracle_for(g, ["in_"], fluid_scheme(1), DROP, 2)
    o.update()
    assert o.cell_size == g["cell_size"]
    off, idx = o.neighbors(0, 0)
    np.testing.assert_array_equal(off, g["nbr_off"])
    np.testing.assert_array_equal(idx, g["nbr_idx"])


def test_drop_first_stage_bit_exact():
    g = load("drop")
    o = oracle_for(g, ["in_"], fluid_scheme(1), DROP, 2)
    o.update()
    o.eval()
    A = o.arrays[0]
    for name, got in (("rho", A.rho), ("p", A.p), ("cs", A.cs), ("_a_u_1", A.au),
                      ("_a_v_1", A.av), ("dt_fac", A.dt_fac)):
        np.testing.assert_array_equal(got, g[f"stage0_{name}"], err_msg=name)


@pytest.mark.parametrize("steps", [1, 10])
def test_drop_trajectory_bit_exact(steps):
    g = load("drop")
    o = oracle_for(g, ["in_"], fluid_scheme(1), DROP, 2)
    for _ in range(steps):
        o.pc_step(1e-5)
    A = o.arrays[0]
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(A, n), g[f"step{steps}_{n}_0"], err_msg=n)


def test_lattice3d_lists_density_pgrad():
    g = load("lattice3d")
    o = oracle_for(g, ["in_"], fluid_scheme(1), dict(c0=10.0, rho0=1.0), 3)
    o.update_pairs([(0, 0)])
    assert o.cell_size == g["cell_size"]
    off, idx = o.neighbors(0, 0)
    np.testing.assert_array_equal(off, g["nbr_off"])
    np.testing.assert_array_equal(idx, g["nbr_idx"])
    out = np.zeros(len(g["in_x"]))
    o.sph_rho(0, 0, out)
    np.testing.assert_array_equal(out, g["rho_sum"])
    o3 = [np.zeros(len(out)) for _ in range(3)]
    o.pgrad(0, 0, *o3)
    for k in range(3):
        np.testing.assert_array_equal(o3[k], g[f"pgrad_{k}"])


def test_dam_break_cfl_steps_bit_exact():
    g = load("dam")
    params = dict(c0=10.0 * np.sqrt(2 * 9.81 * 2.0), rho0=1000.0, gamma=7.0, alpha=0.1,
                  beta=0.0, eta=0.1, gravity=(0.0, -9.81, 0.0))
    o = oracle_for(g, ["in0_", "in1_"], fluid_scheme(2), params, 2)
    dts = []
    for _ in range(5):
        dt = o.cfl_time_step(0.3, params["c0"], 1e-4)
        o.pc_step(dt)
        dts.append(dt)
    np.testing.assert_array_equal(np.asarray(dts), g["dts"])
    for i in range(2):
        for n in ("x", "y", "u", "v", "rho", "p", "cs"):
            np.testing.assert_array_equal(getattr(o.arrays[i], n), g[f"step5_{n}_{i}"],
                                          err_msg=f"{n}_{i}")


def test_square_functions():
    g = load("square")
    x = np.array([0, 0, 1, 1], np.float64)
    y = np.array([0, 1, 1, 0], np.float64)
    base = dict(x=x, y=y, z=np.zeros(4), m=np.ones(4), u=np.array([1, 0, 0, -1.0]),
                p=np.array([0, 0, 1, 1.0]), cs=np.array([1.0, 2.0, 0.5, 1.5]), h=np.ones(4))
    pa = OracleArray("t", rho=np.ones(4), **base)
    o = OracleSystem([pa], dim=2)
    o.update_pairs([(0, 0)])
    out = np.zeros(4)
    o.sph_rho(0, 0, out)
    np.testing.assert_array_equal(out, g["rho_0"])
    o3 = [np.zeros(4) for _ in range(3)]
    o.pgrad(0, 0, *o3)
    for k in range(3):
        np.testing.assert_array_equal(o3[k], g[f"pgrad_{k}"])
    o3 = [np.zeros(4) for _ in range(3)]
    o.momentum(0, 0, 1.0, 1.0, 0.1, *o3, np.zeros(4))
    for k in range(3):
        np.testing.assert_array_equal(o3[k], g[f"mom_{k}"])
    pt = OracleArray("t", rho=np.array([1000.0, 1001.5, 998.0, 1010.0]), **base)
    o = OracleSystem([pt], dim=2)
    p, cs = np.zeros(4), np.zeros(4)
    o.tait(0, 1.0, 1000.0, 7.0, p, cs)
    np.testing.assert_array_equal(p, g["tait_0"])
    np.testing.assert_array_equal(cs, g["tait_1"])


# -- the continuity scheme (SPHDensityRate + XSPHCorrection) -------------------
DAM = dict(c0=10.0 * np.sqrt(2 * 9.81 * 2.0), rho0=1000.0, gamma=7.0, alpha=0.1,
           beta=0.0, eta=0.1, gravity=(0.0, -9.81, 0.0))


def test_drop_continuity_first_stage_bit_exact():
    g = load("drop_cont")
    o = oracle_for(g, ["in_"], continuity_scheme(1, 0.5), DROP, 2)
    o.update()
    o.eval()
    A = o.arrays[0]
    for name, got in (("p", A.p), ("cs", A.cs), ("_a_rho_1", A.arho), ("_a_u_1", A.au),
                      ("_a_v_1", A.av), ("_a_x_1", A.ax), ("_a_y_1", A.ay),
                      ("dt_fac", A.dt_fac)):
        np.testing.assert_array_equal(got, g[f"stage0_{name}"], err_msg=name)


@pytest.mark.parametrize("steps", [1, 10])
def test_drop_continuity_trajectory_bit_exact(steps):
    g = load("drop_cont")
    o = oracle_for(g, ["in_"], continuity_scheme(1, 0.5), DROP, 2)
    for _ in range(steps):
        o.pc_step(1e-5)
    A = o.arrays[0]
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(A, n), g[f"step{steps}_{n}_0"], err_msg=n)


def test_dam_break_continuity_bit_exact():
    """Walls integrate their density too (SPHDensityRate on every array);
    XSPH from the fluid only; 5 CFL steps."""
    g = load("dam_cont")
    o = oracle_for(g, ["in0_", "in1_"], continuity_scheme(2, 0.5), DAM, 2)
    o.update()
    o.eval()
    for i in range(2):
        A = o.arrays[i]
        names = (("p", A.p), ("cs", A.cs), ("_a_rho_1", A.arho))
        if i == 0:
            names += (("_a_u_1", A.au), ("_a_v_1", A.av), ("_a_x_1", A.ax),
                      ("_a_y_1", A.ay), ("dt_fac", A.dt_fac))
        for name, got in names:
            np.testing.assert_array_equal(got, g[f"stage0_{name}_{i}"], err_msg=f"{name}_{i}")
    o = oracle_for(g, ["in0_", "in1_"], continuity_scheme(2, 0.5), DAM, 2)
    dts = []
    for _ in range(5):
        dt = o.cfl_time_step(0.3, DAM["c0"], 1e-4)
        o.pc_step(dt)
        dts.append(dt)
    np.testing.assert_array_equal(np.asarray(dts), g["dts"])
    for i in range(2):
        for n in ("x", "y", "u", "v", "rho", "p", "cs"):
            np.testing.assert_array_equal(getattr(o.arrays[i], n), g[f"step5_{n}_{i}"],
                                          err_msg=f"{n}_{i}")


# -- the other integrators (Euler, RK2, RK4) -----------------------------------
@pytest.mark.parametrize("name,integ,cont", [("euler", "euler", False), ("rk2", "rk2", False),
                                             ("rk4", "rk4", False), ("rk2cont", "rk2", True)])
@pytest.mark.parametrize("steps", [1, 5])
def test_integrators_bit_exact(name, integ, cont, steps):
    g = load("integrators")
    sch = continuity_scheme(1, 0.5) if cont else fluid_scheme(1)
    o = oracle_for(g, ["in_"], sch, DROP, 2)
    for _ in range(steps):
        o.step(1e-5, integ)
    A = o.arrays[0]
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(A, n), g[f"{name}_step{steps}_{n}_0"],
                                      err_msg=f"{name} {n}")


# -- variable smoothing length: symmetric lists and hks kernels ---------------
def oracle_varh(g, scheme):
    arrs = [OracleArray("a0", **{k: g[f"in_{k}"].copy() for k in PROPS})]
    return OracleSystem(arrs, dim=2, rho_src=scheme.rho_src, tait_on=scheme.tait_on,
                        mom_src=scheme.mom_src, step_on=scheme.step_on,
                        rate_src=scheme.rate_src, xsph_src=scheme.xsph_src,
                        xsph_eps=scheme.xsph_eps, variable_h=True, hks=True, **DROP)


def test_varh_lists_in_reference_order():
    """VarHNbrParticleLocator: each dest's own radius-h_a list, then every
    source whose radius-h_b list holds it, in source order."""
    g = load("varh")
    o = oracle_varh(g, fluid_scheme(1))
    o.update()
    off, idx = o.neighbors(0, 0)
    np.testing.assert_array_equal(off, g["nbr_off"])
    np.testing.assert_array_equal(idx, g["nbr_idx"])


@pytest.mark.parametrize("name", ["sum", "cont"])
def test_varh_hks_first_stage_and_steps_bit_exact(name):
    g = load("varh")
    sch = fluid_scheme(1) if name == "sum" else continuity_scheme(1, 0.5)
    o = oracle_varh(g, sch)
    o.update()
    o.eval()
    A = o.arrays[0]
    got = {"rho": A.rho, "p": A.p, "cs": A.cs, "_a_u_1": A.au, "_a_v_1": A.av,
           "dt_fac": A.dt_fac, "_a_rho_1": A.arho, "_a_x_1": A.ax, "_a_y_1": A.ay}
    for key in g:
        if key.startswith(f"{name}_stage0_"):
            n = key[len(f"{name}_stage0_"):]
            np.testing.assert_array_equal(got[n], g[key], err_msg=n)
    o = oracle_varh(g, sch)
    for _ in range(5):
        o.pc_step(1e-5)
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(o.arrays[0], n), g[f"{name}_step5_{n}_0"],
                                      err_msg=n)


# -- the quintic spline and Wendland quintic kernels (2D) ---------------------
KERNELS = {"QuinticSplineKernel": 3, "WendlandQuinticSplineKernel": 4}


@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_values_bit_exact(kname):
    """W and grad W on a line of distances through q = 0..2.9 (h = 1.1),
    with the reference's own quirks (the quintic's W weight and gradient
    sign, Wendland's 7 pi / 4 normalisation)."""
    from oracle import kernel_grad, kernel_w
    g = load("kernels")
    kt = KERNELS[kname]
    rs = np.linspace(0.0, 3.2, 65)
    w = [kernel_w(0.6 * r, 0.8 * r, 0.0, 1.1, 2, kt) for r in rs]
    gr = [kernel_grad(0.6 * r, 0.8 * r, 0.0, 1.1, 2, kt) for r in rs]
    np.testing.assert_array_equal(np.array(w), g[f"{kname}_w"])
    np.testing.assert_array_equal(np.array(gr), g[f"{kname}_grad"])


def oracle_kernel(g, scheme, kname, name="sum"):
    from oracle import KERNEL_RADIUS
    kt = KERNELS[kname]
    arrs = [OracleArray("a0", **{k: g[f"in_{k}"].copy() for k in PROPS})]
    par = dict(DROP, rho0=float(g[f"{kname}_{name}_rho0"]))
    return OracleSystem(arrs, dim=2, rho_src=scheme.rho_src, tait_on=scheme.tait_on,
                        mom_src=scheme.mom_src, step_on=scheme.step_on,
                        rate_src=scheme.rate_src, xsph_src=scheme.xsph_src,
                        xsph_eps=scheme.xsph_eps, kernel=kt, radius_scale=KERNEL_RADIUS[kt],
                        **par)


@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_lists_in_reference_order(kname):
    """The locator radius is the kernel's support (3h for the quintic)."""
    g = load("kernels")
    o = oracle_kernel(g, fluid_scheme(1), kname)
    o.update()
    off, idx = o.neighbors(0, 0)
    np.testing.assert_array_equal(off, g[f"{kname}_nbr_off"])
    np.testing.assert_array_equal(idx, g[f"{kname}_nbr_idx"])


@pytest.mark.parametrize("name", ["sum", "cont"])
@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_first_stage_and_steps_bit_exact(kname, name):
    g = load("kernels")
    sch = fluid_scheme(1) if name == "sum" else continuity_scheme(1, 0.5)
    o = oracle_kernel(g, sch, kname, name)
    o.update()
    o.eval()
    A = o.arrays[0]
    got = {"rho": A.rho, "p": A.p, "cs": A.cs, "_a_u_1": A.au, "_a_v_1": A.av,
           "dt_fac": A.dt_fac, "_a_rho_1": A.arho, "_a_x_1": A.ax, "_a_y_1": A.ay}
    pre = f"{kname}_{name}_stage0_"
    keys = [k for k in g if k.startswith(pre)]
    assert keys
    for key in keys:
        n = key[len(pre):]
        np.testing.assert_array_equal(got[n], g[key], err_msg=n)
    o = oracle_kernel(g, sch, kname, name)
    for _ in range(5):
        o.pc_step(1e-5)
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(o.arrays[0], n),
                                      g[f"{kname}_{name}_step5_{n}_0"], err_msg=n)


# -- variable h with hks in 3D --------------------------------------------------
VARH3D = dict(c0=10.0, rho0=1.0, gamma=7.0, alpha=0.1, beta=0.0, eta=0.1)


def oracle_varh3d(g):
    arrs = [OracleArray("a0", **{k: g[f"in_{k}"].copy() for k in PROPS})]
    sch = fluid_scheme(1)
    return OracleSystem(arrs, dim=3, rho_src=sch.rho_src, tait_on=sch.tait_on,
                        mom_src=sch.mom_src, step_on=sch.step_on, variable_h=True, hks=True,
                        **VARH3D)


def test_varh3d_lists_stage_and_steps_bit_exact():
    g = load("varh3d")
    o = oracle_varh3d(g)
    o.update()
    off, idx = o.neighbors(0, 0)
    np.testing.assert_array_equal(off, g["nbr_off"])
    np.testing.assert_array_equal(idx, g["nbr_idx"])
    o.eval()
    A = o.arrays[0]
    got = {"rho": A.rho, "p": A.p, "cs": A.cs, "_a_u_1": A.au, "_a_v_1": A.av,
           "_a_w_1": A.aw, "dt_fac": A.dt_fac}
    for n, v in got.items():
        np.testing.assert_array_equal(v, g[f"stage0_{n}"], err_msg=n)
    o = oracle_varh3d(g)
    for _ in range(3):
        o.pc_step(1e-4)
    for n in ("x", "y", "z", "u", "v", "w", "rho", "p"):
        np.testing.assert_array_equal(getattr(o.arrays[0], n), g[f"step3_{n}_0"], err_msg=n)


# -- the split-form MonaghanArtificialViscosity ---------------------------------
def test_monaghan_av_square_bit_exact():
    """The viscosity alone on the unit square, with its eta left unset (0:
    the constructor ignores its eta argument) and set by hand to 0.1; its
    dt_fac always uses 0.01 h_ab^2."""
    g = load("avisc")
    base = dict(x=np.array([0, 0, 1, 1.0]), y=np.array([0, 1, 1, 0.0]), z=np.zeros(4),
                m=np.ones(4), u=np.array([1, 0, 0, -1.0]), v=np.array([0, 0.5, 0, 0.25]),
                h=np.ones(4), p=np.array([0, 0, 1, 1.0]), cs=np.array([1.0, 2.0, 0.5, 1.5]),
                rho=np.array([1.0, 1.5, 0.98, 1.1]))
    for name, eta in (("square", 0.0), ("square_eta", 0.1)):
        o = OracleSystem([OracleArray("t", **base)], dim=2)
        o.update_pairs([(0, 0)])
        o3 = [np.zeros(4) for _ in range(3)]
        dtf = np.zeros(4)
        o.monaghan_av(0, 0, 1.0, 1.0, eta, *o3, dtf)
        for k in range(3):
            np.testing.assert_array_equal(o3[k], g[f"{name}_{k}"], err_msg=(name, k))
        np.testing.assert_array_equal(dtf, g[f"{name}_dt_fac"], err_msg=name)


def _split_drop(g):
    pa = OracleArray("fluid", **{k: g[f"in_{k}"].copy() for k in PROPS})
    return OracleSystem([pa], dim=2, rho_src={0: [0]}, tait_on=(0,), mom_src={0: [0]},
                        step_on=(0,), split_av=True, av_eta=0.0, **DROP)


def test_monaghan_av_split_scheme_bit_exact():
    """SPHRho, Tait, SPHPressureGradient + MonaghanArtificialViscosity (both
    into _a_u_1, _a_v_1) on the drop: the first stage, then 5 PC steps."""
    g = load("avisc")
    o = _split_drop(g)
    o.update()
    o.eval()
    A = o.arrays[0]
    for name, got in (("rho", A.rho), ("p", A.p), ("cs", A.cs), ("_a_u_1", A.au),
                      ("_a_v_1", A.av), ("dt_fac", A.dt_fac)):
        np.testing.assert_array_equal(got, g[f"stage0_{name}"], err_msg=name)
    o = _split_drop(g)
    for _ in range(5):
        o.pc_step(1e-5)
    A = o.arrays[0]
    for n in ("x", "y", "u", "v", "rho", "p", "cs"):
        np.testing.assert_array_equal(getattr(A, n), g[f"step5_{n}_0"], err_msg=n)
