"""The CUDA engine against fixtures written by the reference itself.

Neighbour sets (sorted index lists) and cell coordinates bit-exact; FP64
results within 1e-12 relative (the engine sums neighbours in its own cell
order, so the last bits differ from the reference's order); FP32C
(FP32 pair sums with Kahan compensation) within 1e-5 relative density
error, positions within 2e-6 particle spacings after 10 steps.
"""
import os

import numpy as np
import pytest

from pysph_b200.engine import Engine, fluid_scheme

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")
DROP = dict(c0=1400.0, rho0=1.0, gamma=7.0, alpha=0.1, beta=0.0, eta=0.1, dt=1e-5)


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def arrays(g, prefixes):
    return [{k: g[f"{p}{k}"].copy() for k in PROPS} for p in prefixes]


def sorted_pairs(off, idx):
    n = len(off) - 1
    di = np.repeat(np.arange(n), np.diff(off))
    order = np.lexsort((idx, di))
    return di[order], idx[order].astype(np.int64)


@pytest.mark.parametrize("name,dim", [("drop", 2), ("lattice3d", 3)])
def test_neighbour_sets_and_cells(name, dim):
    g = load(name)
    arr = arrays(g, ["in_"])
    eng = Engine([(arr, DROP)], fluid_scheme(1), dim=dim, precision="fp64",
                 step_lists=False)
    assert eng.cell_size() == float(g["cell_size"])
    di, _, sj = eng.neighbors(0, 1)
    rdi, rsj = sorted_pairs(g["nbr_off"], g["nbr_idx"])
    np.testing.assert_array_equal(di, rdi)
    np.testing.assert_array_equal(sj, rsj)
    cc = eng.cell_coords(0, 0)
    a = arr[0]
    cs = float(g["cell_size"])
    ref = np.stack([np.floor(a["x"] / cs), np.floor(a["y"] / cs),
                    np.floor(a["z"] / cs) if dim == 3 else 0 * a["z"]], 1).astype(np.int32)
    np.testing.assert_array_equal(cc, ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_drop_first_stage(precision):
    g = load("drop")
    eng = Engine([(arrays(g, ["in_"]), DROP)], fluid_scheme(1), dim=2, precision=precision)
    eng.density()
    eng.momentum()
    eng.check_status()
    rho = eng.get(0, "rho").cpu().numpy()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(rho - g["stage0_rho"]) / g["stage0_rho"]) <= tol
    scale = max(np.abs(g["stage0__a_u_1"]).max(), np.abs(g["stage0__a_v_1"]).max())
    atol = 1e-10 if precision == "fp64" else 1e-4
    for n in ("_a_u_1", "_a_v_1"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"stage0_{n}"])) / scale <= atol, n


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_drop_ten_steps(precision):
    g = load("drop")
    eng = Engine([(arrays(g, ["in_"]), DROP)], fluid_scheme(1), dim=2, precision=precision)
    for _ in range(10):
        eng.pc_step()
    eng.check_status()
    dx = 0.025
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"step10_{n}_0"])) / dx <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(rho - g["step10_rho_0"]) / g["step10_rho_0"]) <= rtol


def test_lattice3d_density_and_pgrad():
    g = load("lattice3d")
    arr = arrays(g, ["in_"])
    for precision, tol in (("fp64", 1e-12), ("fp32c", 1e-5)):
        eng = Engine([(arr, dict(c0=10.0, rho0=1.0))], fluid_scheme(1), dim=3,
                     precision=precision, lanes=4)
        eng.momentum(gravity=False, mode=1)   # pgrad from the input rho, p
        scale = max(np.abs(g[f"pgrad_{k}"]).max() for k in range(3))
        for k, n in enumerate(("_a_u_1", "_a_v_1", "_a_w_1")):
            got = eng.get(0, n).cpu().numpy()
            assert np.max(np.abs(got - g[f"pgrad_{k}"])) / scale <= 10 * tol, (precision, n)
        eng.density(eos=False)
        rho = eng.get(0, "rho").cpu().numpy()
        assert np.max(np.abs(rho - g["rho_sum"]) / g["rho_sum"]) <= tol, precision


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_dam_break_cfl(precision):
    g = load("dam")
    params = dict(c0=10.0 * np.sqrt(2 * 9.81 * 2.0), rho0=1000.0, gamma=7.0, alpha=0.1,
                  beta=0.0, eta=0.1, gravity=(0.0, -9.81, 0.0), cfl=0.3, dt_initial=1e-4)
    eng = Engine([(arrays(g, ["in0_", "in1_"]), params)], fluid_scheme(2), dim=2,
                 precision=precision)
    dts = []
    for _ in range(5):
        eng.pc_step()
        dts.append(eng.scene_state()[0].dt)
    eng.check_status()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(dts, g["dts"], rtol=rtol)
    dx = 0.05
    ptol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"step5_{n}_0"])) / dx <= ptol, n
    for i in range(2):
        rho = eng.get(i, "rho").cpu().numpy()
        ref = g[f"step5_rho_{i}"]
        assert np.max(np.abs(rho - ref) / ref) <= rtol


# -- the continuity scheme (SPHDensityRate + XSPHCorrection) -------------------
from pysph_b200.engine import continuity_scheme  # noqa: E402

DAM = dict(c0=10.0 * np.sqrt(2 * 9.81 * 2.0), rho0=1000.0, gamma=7.0, alpha=0.1,
           beta=0.0, eta=0.1, gravity=(0.0, -9.81, 0.0), cfl=0.3, dt_initial=1e-4)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_drop_continuity_first_stage(precision):
    """One evaluation of the continuity scheme: Tait on the given density,
    then SPHDensityRate + MomentumEquation + XSPH in one pair pass."""
    g = load("drop_cont")
    eng = Engine([(arrays(g, ["in_"]), DROP)], continuity_scheme(1, 0.5), dim=2,
                 precision=precision)
    eng.eval_stage()
    eng.check_status()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    for n in ("p", "cs"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"stage0_{n}"]
        assert np.max(np.abs(got - ref)) <= rtol * np.max(np.abs(ref)) + 1e-300, n
    atol = 1e-10 if precision == "fp64" else 1e-4
    for n in ("_a_rho_1", "_a_u_1", "_a_v_1"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"stage0_{n}"]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, n


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_drop_continuity_ten_steps(precision):
    """Integrated density and XSPH-corrected positions over 10 steps."""
    g = load("drop_cont")
    eng = Engine([(arrays(g, ["in_"]), DROP)], continuity_scheme(1, 0.5), dim=2,
                 precision=precision)
    for _ in range(10):
        eng.pc_step()
    eng.check_status()
    dx = 0.025
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"step10_{n}_0"])) / dx <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    assert np.max(np.abs(rho - g["step10_rho_0"]) / g["step10_rho_0"]) <= rtol


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_dam_break_continuity_cfl(precision):
    """The reference's dam-break scheme: walls integrate their density too;
    5 CFL steps (dt sequence, positions, both arrays' densities)."""
    g = load("dam_cont")
    eng = Engine([(arrays(g, ["in0_", "in1_"]), DAM)], continuity_scheme(2, 0.5), dim=2,
                 precision=precision)
    dts = []
    for _ in range(5):
        eng.pc_step()
        dts.append(eng.scene_state()[0].dt)
    eng.check_status()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(dts, g["dts"], rtol=rtol)
    dx = 0.05
    ptol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"step5_{n}_0"])) / dx <= ptol, n
    for i in range(2):
        rho = eng.get(i, "rho").cpu().numpy()
        ref = g[f"step5_rho_{i}"]
        assert np.max(np.abs(rho - ref) / ref) <= rtol, i


# -- Euler, RK2 and RK4 fused on the engine -----------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("name,kind,cont", [("euler", "euler", False), ("rk2", "rk2", False),
                                            ("rk4", "rk4", False), ("rk2cont", "rk2", True)])
def test_integrators_five_steps(precision, name, kind, cont):
    g = load("integrators")
    sch = continuity_scheme(1, 0.5) if cont else fluid_scheme(1)
    eng = Engine([(arrays(g, ["in_"]), DROP)], sch, dim=2, precision=precision)
    for _ in range(5):
        eng.step(kind)
    eng.check_status()
    dx = 0.05
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"{name}_step5_{n}_0"])) / dx <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    ref = g[f"{name}_step5_rho_0"]
    assert np.max(np.abs(rho - ref) / ref) <= rtol


# -- variable smoothing length: symmetric lists and hks kernels ---------------
def varh_scheme(cont):
    sch = continuity_scheme(1, 0.5) if cont else fluid_scheme(1)
    sch.hks = True
    return sch


def test_varh_neighbour_sets():
    """Symmetric neighbour sets (VarHNbrParticleLocator): r < 2 max(h_a, h_b),
    more pairs than the dest's own support gives."""
    g = load("varh")
    arr = arrays(g, ["in_"])
    eng = Engine([(arr, DROP)], varh_scheme(False), dim=2, precision="fp64",
                 step_lists=False, variable_h=True)
    di, _, sj = eng.neighbors(0, 1)
    rdi, rsj = sorted_pairs(g["nbr_off"], g["nbr_idx"])
    np.testing.assert_array_equal(di, rdi)
    np.testing.assert_array_equal(sj, rsj)
    fixed = Engine([(arr, DROP)], fluid_scheme(1), dim=2, precision="fp64", step_lists=False)
    assert len(fixed.neighbors(0, 1)[0]) < len(rdi)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("name", ["sum", "cont"])
def test_varh_hks_first_stage(precision, name):
    """One evaluation with variable h and hks kernels: summation density +
    Tait + momentum, or Tait + SPHDensityRate + momentum + XSPH."""
    g = load("varh")
    cont = name == "cont"
    eng = Engine([(arrays(g, ["in_"]), DROP)], varh_scheme(cont), dim=2,
                 precision=precision, variable_h=True)
    eng.eval_stage()
    eng.check_status()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    for n in ("rho", "p", "cs"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"{name}_stage0_{n}"]
        assert np.max(np.abs(got - ref)) <= rtol * np.max(np.abs(ref)) + 1e-300, n
    atol = 1e-10 if precision == "fp64" else 1e-4
    names = ["_a_u_1", "_a_v_1", "dt_fac"] + (["_a_rho_1"] if cont else [])
    for n in names:
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"{name}_stage0_{n}"]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, n
    if cont:
        # position rate: u + the XSPH correction
        for c, v in (("x", "u"), ("y", "v")):
            got = (eng.get(0, v) + eng.get(0, f"_xsph_{v}")).cpu().numpy()
            ref = g[f"cont_stage0__a_{c}_1"]
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, c


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("name", ["sum", "cont"])
def test_varh_hks_five_steps(precision, name):
    g = load("varh")
    eng = Engine([(arrays(g, ["in_"]), DROP)], varh_scheme(name == "cont"), dim=2,
                 precision=precision, variable_h=True)
    for _ in range(5):
        eng.pc_step()
    eng.check_status()
    dx = 0.05
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"{name}_step5_{n}_0"])) / dx <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    ref = g[f"{name}_step5_rho_0"]
    assert np.max(np.abs(rho - ref) / ref) <= rtol


# -- the quintic spline and Wendland quintic kernels (2D) ---------------------
KERNELS = {"QuinticSplineKernel": 3, "WendlandQuinticSplineKernel": 4}


def kernel_engine(g, kname, name, precision, **kw):
    sch = continuity_scheme(1, 0.5) if name == "cont" else fluid_scheme(1)
    par = dict(DROP, rho0=float(g[f"{kname}_{name}_rho0"]))
    return Engine([(arrays(g, ["in_"]), par)], sch, dim=2, precision=precision,
                  kernel=KERNELS[kname], **kw)


@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_neighbour_sets(kname):
    """The neighbour radius is the kernel's support (3h for the quintic)."""
    g = load("kernels")
    eng = kernel_engine(g, kname, "sum", "fp64", step_lists=False)
    di, _, sj = eng.neighbors(0, 1)
    rdi, rsj = sorted_pairs(g[f"{kname}_nbr_off"], g[f"{kname}_nbr_idx"])
    np.testing.assert_array_equal(di, rdi)
    np.testing.assert_array_equal(sj, rsj)


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("name", ["sum", "cont"])
@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_first_stage(kname, name, precision):
    g = load("kernels")
    cont = name == "cont"
    eng = kernel_engine(g, kname, name, precision)
    eng.eval_stage()
    eng.check_status()
    pre = f"{kname}_{name}_stage0_"
    rtol = 1e-12 if precision == "fp64" else 1e-5
    for n in ("rho", "p", "cs"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[pre + n]
        assert np.max(np.abs(got - ref)) <= rtol * np.max(np.abs(ref)) + 1e-300, n
    atol = 1e-10 if precision == "fp64" else 1e-4
    for n in ["_a_u_1", "_a_v_1", "dt_fac"] + (["_a_rho_1"] if cont else []):
        got = eng.get(0, n).cpu().numpy()
        ref = g[pre + n]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, n
    if cont:
        for c, v in (("x", "u"), ("y", "v")):
            got = (eng.get(0, v) + eng.get(0, f"_xsph_{v}")).cpu().numpy()
            ref = g[f"{pre}_a_{c}_1"]
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, c


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("name", ["sum", "cont"])
@pytest.mark.parametrize("kname", sorted(KERNELS))
def test_other_kernels_five_steps(kname, name, precision):
    g = load("kernels")
    eng = kernel_engine(g, kname, name, precision)
    for _ in range(5):
        eng.pc_step()
    eng.check_status()
    dx = 0.05
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"{kname}_{name}_step5_{n}_0"])) / dx <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    ref = g[f"{kname}_{name}_step5_rho_0"]
    assert np.max(np.abs(rho - ref) / ref) <= rtol


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_varh3d_hks(precision):
    """3D, variable h with hks kernels: symmetric neighbour sets, the first
    stage and 3 PC steps against the reference's fixture."""
    g = load("varh3d")
    par = dict(c0=10.0, rho0=1.0, gamma=7.0, alpha=0.1, beta=0.0, eta=0.1, dt=1e-4)
    eng = Engine([(arrays(g, ["in_"]), par)], varh_scheme(False), dim=3, precision=precision,
                 variable_h=True, lanes=4)
    if precision == "fp64":
        di, _, sj = eng.neighbors(0, 1)
        rdi, rsj = sorted_pairs(g["nbr_off"], g["nbr_idx"])
        np.testing.assert_array_equal(di, rdi)
        np.testing.assert_array_equal(sj, rsj)
    eng.eval_stage()
    eng.check_status()
    rtol = 1e-12 if precision == "fp64" else 1e-5
    for n in ("rho", "p", "cs"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"stage0_{n}"]
        assert np.max(np.abs(got - ref)) <= rtol * np.max(np.abs(ref)), n
    atol = 1e-10 if precision == "fp64" else 1e-4
    for n in ("_a_u_1", "_a_v_1", "_a_w_1", "dt_fac"):
        got = eng.get(0, n).cpu().numpy()
        ref = g[f"stage0_{n}"]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) <= atol, n
    eng = Engine([(arrays(g, ["in_"]), par)], varh_scheme(False), dim=3, precision=precision,
                 variable_h=True, lanes=4)
    for _ in range(3):
        eng.pc_step()
    eng.check_status()
    tol = 1e-10 if precision == "fp64" else 2e-6
    for n in ("x", "y", "z"):
        got = eng.get(0, n).cpu().numpy()
        assert np.max(np.abs(got - g[f"step3_{n}_0"])) / 0.1 <= tol, n
    rho = eng.get(0, "rho").cpu().numpy()
    assert np.max(np.abs(rho - g["step3_rho_0"]) / g["step3_rho_0"]) <= rtol
