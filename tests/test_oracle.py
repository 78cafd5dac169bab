"""The oracle against the reference's own known-answer tests.

Each check restates a test of the reference project (cited) and runs it on
the C oracle: kernel normalisation / moments (S/base/tests/test_kernels.py),
the 4-particle unit square of the SPH function tests
(S/sph/tests/function_test_template.py:41-59 with test_density_funcs.py,
test_eos_funcs.py, test_pressure_funcs.py), neighbour lists against brute
force on the reference's NNPS datasets (S/base/tests/common_data.py), and
the predictor-corrector integrator on a motion with a closed-form answer.
"""
import math

import numpy as np
import pytest

import oracle
from oracle import OracleArray, OracleSystem

PI = np.pi


def kernel_w_py(ri, rj, h, dim=2):
    """CubicSplineKernel.function as a Python loop would evaluate it."""
    rab = math.sqrt(sum((a - b) ** 2 for a, b in zip(ri, rj)))
    q = rab / h
    fac = (10 / (7 * PI) if dim == 2 else 1 / PI) / h ** dim
    if q > 2:
        return 0.0
    if q > 1:
        return 0.25 * (2 - q) ** 3 * fac
    return (1 - 1.5 * q * q * (1 - 0.5 * q)) * fac


def kernel_grad_py(ri, rj, h, dim=2):
    rab = math.sqrt(sum((a - b) ** 2 for a, b in zip(ri, rj)))
    q = rab / h
    fac = (10 / (7 * PI) if dim == 2 else 1 / PI) / h ** dim
    val = 0.0
    if q > 2:
        pass
    elif q >= 1:
        val = -0.75 * (2 - q) ** 2 / (h * rab)
    elif q > 1e-14:
        val = 3.0 * (0.75 * q - 1) / (h * h)
    return np.array([(a - b) * val * fac for a, b in zip(ri, rj)])


# ---------------------------------------------------------------- kernels
def test_kernel_fac():
    # S/base/tests/test_kernels.py:224-231
    h = 0.01
    fac = 10 / (7 * np.pi) / (h * h)
    assert oracle.kernel_w(0, 0, 0, h, 2) == pytest.approx(fac, rel=1e-12)


def _grid21():
    x = np.linspace(-1, 1, 21)
    dx = x[1] - x[0]
    xg, yg = np.meshgrid(x, x)
    return xg.ravel(), yg.ravel(), dx


def test_kernel_normalisation_2d():
    # S/base/tests/test_kernels.py:233-252: sum W dx^2 == 1 (4 places)
    xg, yg, dx = _grid21()
    hs = 2 * dx
    val = sum(oracle.kernel_w(-px, -py, 0.0, hs, 2) * dx * dx
              for px, py in zip(xg, yg))
    assert round(val - 1.0, 4) == 0


def test_kernel_gradient_and_moment_2d():
    # S/base/tests/test_kernels.py:254-300: sum grad W dx^2 == 0 and the
    # first moment sum (x0 - x) W dx^2 == 0 (10 places)
    xg, yg, dx = _grid21()
    hs = 2 * dx
    g = np.zeros(3)
    mom = np.zeros(2)
    for px, py in zip(xg, yg):
        gr = oracle.kernel_grad(-px, -py, 0.0, hs, 2)
        assert gr[2] == 0
        g += gr * dx * dx
        w = oracle.kernel_w(-px, -py, 0.0, hs, 2) * dx * dx
        mom += np.array([-px, -py]) * w
    assert abs(g[0]) < 1e-10 and abs(g[1]) < 1e-10
    assert abs(mom[0]) < 1e-10 and abs(mom[1]) < 1e-10


def test_kernel_matches_python_restatement():
    rng = np.random.default_rng(3)
    for dim in (2, 3):
        for _ in range(200):
            d = rng.uniform(-2.5, 2.5, 3)
            if dim == 2:
                d[2] = 0
            h = rng.uniform(0.5, 1.5)
            w = oracle.kernel_w(d[0], d[1], d[2], h, dim)
            assert w == pytest.approx(kernel_w_py(d, (0, 0, 0), h, dim), rel=1e-13, abs=1e-15)
            g = oracle.kernel_grad(d[0], d[1], d[2], h, dim)
            np.testing.assert_allclose(g, kernel_grad_py(d, (0, 0, 0), h, dim),
                                       rtol=1e-12, atol=1e-15)


# -------------------------------------------------- 4-particle unit square
def square(**extra):
    # S/sph/tests/function_test_template.py:41-59
    x = np.array([0, 0, 1, 1], np.float64)
    y = np.array([0, 1, 1, 0], np.float64)
    props = dict(x=x, y=y, z=np.zeros(4), m=np.ones(4),
                 u=np.array([1, 0, 0, -1], np.float64),
                 p=np.array([0, 0, 1, 1], np.float64))
    props.update(extra)
    return OracleArray("test", **props)


def test_square_sph_rho():
    # test_density_funcs.py:37-80 (6 places); m = h = 1 so the reference
    # loop's swapped (m, h) pair is harmless
    pa = square()
    sys_ = OracleSystem([pa], dim=2)
    sys_.update_pairs([(0, 0)])
    out = np.zeros(4)
    sys_.sph_rho(0, 0, out)
    for i in range(4):
        ri = (pa.x[i], pa.y[i], 0.0)
        rho = sum(pa.m[j] * kernel_w_py(ri, (pa.x[j], pa.y[j], 0.0),
                                        0.5 * (pa.h[i] + pa.h[j]))
                  for j in range(4))
        assert round(out[i] - rho, 6) == 0


def test_square_tait():
    # test_eos_funcs.py:67-122 (10 places, double)
    pa = square(rho=np.array([1000.0, 1001.5, 998.0, 1010.0]))
    sys_ = OracleSystem([pa], dim=2)
    p = np.zeros(4)
    cs = np.zeros(4)
    sys_.tait(0, 1.0, 1000.0, 7.0, p, cs)
    B = 1.0 * 1.0 * 1000 / 7.0
    for i in range(4):
        ratio = pa.rho[i] / 1000
        assert round(p[i] - (np.power(ratio, 7.0) - 1.0) * B, 10) == 0
        assert round(cs[i] - np.power(ratio, 3.0) * 1.0, 10) == 0


def test_square_pressure_gradient():
    # test_pressure_funcs.py:17-102 (6 places)
    pa = square()
    sys_ = OracleSystem([pa], dim=2)
    sys_.update_pairs([(0, 0)])
    o = [np.zeros(4) for _ in range(3)]
    sys_.pgrad(0, 0, *o)
    for i in range(4):
        ri = (pa.x[i], pa.y[i], 0.0)
        f = np.zeros(3)
        for j in range(4):
            rj = (pa.x[j], pa.y[j], 0.0)
            tmp = -pa.m[j] * (pa.p[i] / pa.rho[i] ** 2 + pa.p[j] / pa.rho[j] ** 2)
            f += tmp * kernel_grad_py(ri, rj, 0.5 * (pa.h[i] + pa.h[j]))
        for d in range(3):
            assert round(o[d][i] - f[d], 6) == 0


def test_square_momentum_equation():
    # test_pressure_funcs.py:105-187 (alpha = beta = 1, eta = 0.1; 6 places)
    pa = square(cs=np.array([1.0, 2.0, 0.5, 1.5]))
    sys_ = OracleSystem([pa], dim=2)
    sys_.update_pairs([(0, 0)])
    o = [np.zeros(4) for _ in range(3)]
    dtf = np.zeros(4)
    sys_.momentum(0, 0, 1.0, 1.0, 0.1, *o, dtf)
    for i in range(4):
        ri = np.array([pa.x[i], pa.y[i], 0.0])
        va = np.array([pa.u[i], pa.v[i], 0.0])
        f = np.zeros(3)
        for j in range(4):
            rj = np.array([pa.x[j], pa.y[j], 0.0])
            vb = np.array([pa.u[j], pa.v[j], 0.0])
            havg = 0.5 * (pa.h[i] + pa.h[j])
            tmp = pa.p[i] / pa.rho[i] ** 2 + pa.p[j] / pa.rho[j] ** 2
            rab = ri - rj
            dot = np.dot(va - vb, rab)
            piab = 0.0
            if dot < 0:
                cab = 0.5 * (pa.cs[i] + pa.cs[j])
                rhoab = 0.5 * (pa.rho[i] + pa.rho[j])
                mu = havg * dot / (np.dot(rab, rab) + 0.01 * havg * havg)
                piab = (-1.0 * cab * mu + 1.0 * mu * mu) / rhoab
            tmp = -pa.m[j] * (tmp + piab)
            f += tmp * kernel_grad_py(tuple(ri), tuple(rj), havg)
        for d in range(3):
            assert round(o[d][i] - f[d], 6) == 0
    assert np.all(dtf >= 0) and dtf.max() > 0


# ----------------------------------------------------------- neighbours
def brute_pairs(D, S, same, scale=2.0):
    out = []
    for i in range(len(D["x"])):
        r = D["h"][i] * scale
        r2 = r * r
        for j in range(len(S["x"])):
            dx = S["x"][j] - D["x"][i]
            dy = S["y"][j] - D["y"][i]
            dz = S["z"][j] - D["z"][i]
            if dx * dx + dy * dy + dz * dz < r2:
                out.append((i, j))
    return sorted(out)


def _dataset1():
    # S/base/tests/common_data.py:8-26
    a = dict(x=np.array([0.25, 0.8, 0.5, 0.8, 0.2, 0.5, 1.5, 1.5]),
             y=np.array([0.25, 0.1, 0.5, 0.8, 0.9, 1.5, 0.5, 1.5]),
             z=np.zeros(8), h=np.ones(8))
    b = dict(x=np.array([0.2, 1.2, 1.5, 0.4]), y=np.zeros(4),
             z=np.array([1.6, 1.5, -0.5, 0.4]), h=np.ones(4))
    return a, b


def _dataset2():
    # S/base/tests/common_data.py:28-43
    return dict(x=np.array([-0.5, -0.5, 0.5, 0.5, 1.5, 2.5, 2.5]),
                y=np.array([2.5, -0.5, 1.5, 0.5, 0.5, 0.5, -0.5]),
                z=np.zeros(7), h=np.ones(7))


@pytest.mark.parametrize("scale", [0.5, 1.0, 2.0])
def test_neighbors_common_data(scale):
    a, b = _dataset1()
    for h in (0.3, 0.6, 1.0):
        A = dict(a, h=np.full(8, h * scale))
        B = dict(b, h=np.full(4, h * scale))
        sys_ = OracleSystem([OracleArray("a", **A), OracleArray("b", **B)], dim=3)
        sys_.update_pairs([(0, 0), (0, 1), (1, 0), (1, 1)])
        for d, s, DD, SS in ((0, 0, A, A), (0, 1, A, B), (1, 0, B, A), (1, 1, B, B)):
            off, idx = sys_.neighbors(d, s)
            got = sorted((i, int(j)) for i in range(len(DD["x"]))
                         for j in idx[off[i]:off[i + 1]])
            assert got == brute_pairs(DD, SS, d == s)
    c = _dataset2()
    sys_ = OracleSystem([OracleArray("c", **c)], dim=2)
    sys_.update_pairs([(0, 0)])
    off, idx = sys_.neighbors(0, 0)
    got = sorted((i, int(j)) for i in range(7) for j in idx[off[i]:off[i + 1]])
    assert got == brute_pairs(c, c, True)


@pytest.mark.parametrize("dim", [2, 3])
def test_neighbors_random_and_self_last(dim):
    rng = np.random.default_rng(11)
    n = 400
    A = dict(x=rng.uniform(-1, 1, n), y=rng.uniform(-1, 1, n),
             z=rng.uniform(-1, 1, n) if dim == 3 else np.zeros(n),
             h=rng.uniform(0.05, 0.12, n))
    sys_ = OracleSystem([OracleArray("a", **A)], dim=dim)
    sys_.update_pairs([(0, 0)])
    off, idx = sys_.neighbors(0, 0)
    got = sorted((i, int(j)) for i in range(n) for j in idx[off[i]:off[i + 1]])
    assert got == brute_pairs(A, A, True)
    # self is always a neighbour and sits last (S/base/nnps.pyx:612-619)
    for i in range(n):
        assert idx[off[i + 1] - 1] == i


def test_cell_ids_floor():
    rng = np.random.default_rng(5)
    x = rng.uniform(-3, 3, 1000)
    y = rng.uniform(-3, 3, 1000)
    z = rng.uniform(-3, 3, 1000)
    cs = 0.37
    ids = oracle.cell_ids(x, y, z, cs)
    np.testing.assert_array_equal(ids[:, 0], np.floor(x / cs).astype(np.int32))
    np.testing.assert_array_equal(ids[:, 1], np.floor(y / cs).astype(np.int32))
    np.testing.assert_array_equal(ids[:, 2], np.floor(z / cs).astype(np.int32))


# ------------------------------------------------------------ integrator
def test_pc_free_fall_exact():
    """Isolated particles under gravity: the predictor-corrector is exact for
    constant acceleration, x(t) = x0 + u0 t + g t^2 / 2
    (S/solver/integrator.py:614-683)."""
    n = 5
    x0 = np.arange(n) * 10.0
    u0 = np.linspace(-1, 1, n)
    pa = OracleArray("fluid", x=x0.copy(), y=np.zeros(n), u=u0.copy(),
                     v=np.zeros(n), h=np.full(n, 0.1), m=np.ones(n),
                     rho=np.ones(n))
    g = -9.81
    sys_ = OracleSystem([pa], dim=2, rho_src={0: [0]}, tait_on=[0],
                        mom_src={0: [0]}, step_on=[0], c0=1.0, rho0=1.0,
                        alpha=0.1, beta=0.0, gravity=(0.0, g, 0.0))
    dt = 1e-3
    for _ in range(100):
        sys_.pc_step(dt)
    t = 100 * dt
    np.testing.assert_allclose(pa.x, x0 + u0 * t, rtol=0, atol=1e-12)
    np.testing.assert_allclose(pa.y, 0.5 * g * t * t, rtol=1e-10)
    np.testing.assert_allclose(pa.v, g * t, rtol=1e-10)
