"""The hand-written adjoint of the rollout (pysph_b200.adjoint) against
(1) torch autograd through a dense O(N^2) FP64 restatement of the same
predictor-corrector rollout at N ~ 500, and (2) central finite differences
in FP64 along 16 random directions of the initial velocities, on the
differentiable-rollout workload: elliptical drop with 50k particles
(dx = 0.0079), 200 steps of dt = 2e-6, checkpoints every 20 steps, loss =
mean squared distance of the final positions to those of a run with
velocity scale 110.  Bars: 1e-6 relative to the autograd gradient (both
FP64), 1e-4 median relative error against finite differences.
"""
import math

import numpy as np
import pytest
import torch

from pysph_b200 import workloads as W
from pysph_b200.adjoint import Rollout, RolloutFunction
from pysph_b200.engine import fluid_scheme

pytestmark = pytest.mark.gpu

KFAC2 = 10.0 / (7.0 * math.pi)


def dense_rollout(X, V, m, h, p, steps, dt):
    """Dense FP64 torch restatement: SPHRho -> Tait -> MomentumEquation ->
    PositionStepping with the predictor-corrector integrator."""
    c0, rho0, gamma, alpha, beta, eta = p["c0"], p["rho0"], 7.0, p["alpha"], p["beta"], p["eta"]
    B = c0 * c0 * rho0 / gamma

    def F(X, V):
        d = X[:, None, :] - X[None, :, :]
        r2 = (d * d).sum(-1)
        hi = h[:, None]
        hab = 0.5 * (h[:, None] + h[None, :])
        mask = r2 < (2.0 * hi) ** 2
        nz = r2 > 0
        r = torch.sqrt(torch.where(nz, r2, torch.ones_like(r2)))
        q = r / hab
        fac = KFAC2 / (hab * hab)
        w_in = 1 - 1.5 * q * q * (1 - 0.5 * q)
        w_out = 0.25 * (2 - q) ** 3
        W_ = torch.where(q > 2, torch.zeros_like(q), torch.where(q > 1, w_out, w_in)) * fac
        W_ = torch.where(nz, W_, fac)       # self: W(0)
        rho = (mask * W_ * m[None, :]).sum(1)
        ratio = rho / rho0
        pr = (ratio ** gamma - 1.0) * B
        cs = ratio ** (0.5 * (gamma - 1.0)) * c0
        g_in = 3.0 * (0.75 * q - 1) / (hab * hab)
        g_out = -0.75 * (2 - q) ** 2 / (hab * r)
        g = torch.where(q > 2, torch.zeros_like(q), torch.where(q >= 1, g_out, g_in)) * fac
        g = torch.where(nz, g, torch.zeros_like(g))
        dv = V[:, None, :] - V[None, :, :]
        dot = (dv * d).sum(-1)
        mu = hab * dot / (r2 + eta * eta * hab * hab)
        cab = 0.5 * (cs[:, None] + cs[None, :])
        rhoab = 0.5 * (rho[:, None] + rho[None, :])
        Pi = torch.where(dot < 0, (-alpha * cab * mu + beta * mu * mu) / rhoab, torch.zeros_like(mu))
        tmp = pr[:, None] / rho[:, None] ** 2 + pr[None, :] / rho[None, :] ** 2 + Pi
        coef = mask * (-m[None, :]) * tmp * g
        return (coef[..., None] * d).sum(1)

    for _ in range(steps):
        Fa = F(X, V)
        Xh = X + dt / 2 * V
        Vh = V + dt / 2 * Fa
        Fb = F(Xh, Vh)
        X, V = X + dt * Vh, V + dt * Fb
    return X


def drop(dx, scale=100.0):
    arrays, _, params = W.elliptical_drop(dx=dx, vel_scale=scale)
    return arrays, params


def final_positions(arrays, params, steps, dt, v0, precision="fp64"):
    r = Rollout(arrays, params, fluid_scheme(1), dim=2, dt=dt, steps=steps,
                checkpoint_every=10, precision=precision)
    return r.forward({0: v0})[0][0], r


def test_adjoint_matches_dense_autograd():
    dx = math.sqrt(math.pi / 500)
    arrays, params = drop(dx)
    a = arrays[0]
    n = len(a["x"])
    steps, dt = 20, 1e-5
    dev = torch.device("cuda")
    v0 = torch.tensor(np.stack([a["u"], a["v"]]), dtype=torch.float64, device=dev)
    target_arrays, _ = drop(dx, scale=110.0)
    r = Rollout(arrays, params, fluid_scheme(1), dim=2, dt=dt, steps=steps,
                checkpoint_every=10, precision="fp64")
    tgt = Rollout(target_arrays, params, fluid_scheme(1), dim=2, dt=dt, steps=steps,
                  precision="fp64")
    xt = tgt.forward({0: torch.tensor(np.stack([target_arrays[0]["u"], target_arrays[0]["v"]]),
                                      dtype=torch.float64, device=dev)})[0][0]
    v = v0.clone().requires_grad_(True)
    xf = RolloutFunction.apply(v, r)
    loss = ((xf - xt) ** 2).sum() / n
    loss.backward()
    g_ours = v.grad.clone()
    # dense reference (particle order = input order)
    X = torch.tensor(np.stack([a["x"], a["y"]], 1), dtype=torch.float64, device=dev)
    V = v0.T.clone().requires_grad_(True)
    m = torch.tensor(a["m"], dtype=torch.float64, device=dev)
    h = torch.tensor(a["h"], dtype=torch.float64, device=dev)
    Xf = dense_rollout(X, V, m, h, params, steps, dt)
    assert torch.max(torch.abs(Xf.T - xf.detach())) < 1e-12
    ld = ((Xf.T - xt) ** 2).sum() / n
    ld.backward()
    g_ref = V.grad.T
    err = float((g_ours - g_ref).abs().max() / g_ref.abs().max())
    # both FP64; they differ only by summation order, amplified through 20
    # steps of a stiff (c0 = 1400) system
    assert err <= 1e-6, err


CONFIG4 = dict(dx=0.0079, steps=200, dt=2e-6)   # c0 dt / h = 0.27


def config4_gradient(precision):
    """Gradient of the config-4 loss w.r.t. the initial velocities (50k
    particles, 200 steps, checkpoints every 20)."""
    dx, steps, dt = CONFIG4["dx"], CONFIG4["steps"], CONFIG4["dt"]
    arrays, params = drop(dx)
    a = arrays[0]
    n = len(a["x"])
    dev = torch.device("cuda")
    v0 = torch.tensor(np.stack([a["u"], a["v"]]), dtype=torch.float64, device=dev)
    tarr, _ = drop(dx, scale=110.0)
    xt = Rollout(tarr, params, fluid_scheme(1), 2, dt, steps, precision="fp64").forward(
        {0: torch.tensor(np.stack([tarr[0]["u"], tarr[0]["v"]]), dtype=torch.float64,
                         device=dev)})[0][0]
    r = Rollout(arrays, params, fluid_scheme(1), 2, dt, steps, checkpoint_every=20,
                precision=precision)
    v = v0.clone().requires_grad_(True)
    loss = ((RolloutFunction.apply(v, r) - xt) ** 2).sum() / n
    loss.backward()
    return v.grad, v0, xt, arrays, params, n


def test_adjoint_central_fd_full_rollout():
    """FD in FP64 on 16 random unit directions (seed 0) of the initial
    velocities, eps = 1e-4 (velocity units, |v| ~ 100).  Bars: median over
    the directions of |FD - adjoint| / |FD| <= 1e-4, and every direction's
    |FD - adjoint| <= 1e-5 |grad|.  The second form is the meaningful one
    per direction: a random direction in 100k dimensions sees ~|grad| / 300
    of the gradient, some far less, and there the FD's own noise (round-off
    amplified over 200 stiff steps, pairs crossing the artificial-viscosity
    switch v.r = 0 between the two evaluations) dominates |FD - adjoint| /
    |FD|.  Measured on B200: median 8e-5, max 5e-7 |grad|; eps from 1e-3
    to 1e-5 gives the same floor, 1e-6 and below is round-off bound."""
    g, v0, xt, arrays, params, n = config4_gradient("fp64")
    dev = v0.device
    fd = Rollout(arrays, params, fluid_scheme(1), 2, CONFIG4["dt"], CONFIG4["steps"],
                 checkpoint_every=CONFIG4["steps"], precision="fp64")

    def L(vv):
        xf = fd.forward({0: vv})[0][0]
        return float(((xf - xt) ** 2).sum() / n)

    rng = np.random.default_rng(0)
    eps = 1e-4
    gnorm = float(torch.linalg.norm(g))
    errs, errs_g = [], []
    for _ in range(16):
        d = torch.tensor(rng.standard_normal((2, n)), dtype=torch.float64, device=dev)
        d /= torch.linalg.norm(d)
        fdv = (L(v0 + eps * d) - L(v0 - eps * d)) / (2 * eps)
        adv = float((g * d).sum())
        errs.append(abs(fdv - adv) / max(abs(fdv), 1e-30))
        errs_g.append(abs(fdv - adv) / gnorm)
    print("FD relative errors:", errs)
    print("FD errors / |grad|:", errs_g)
    assert np.median(errs) <= 1e-4, errs
    assert np.max(errs_g) <= 1e-5, errs_g


def test_adjoint_fp32c_forward_gradient():
    """The production setting -- FP32C forward, FP64 adjoint -- against the
    FP64 forward's gradient: relative error of the whole gradient vector."""
    g32 = config4_gradient("fp32c")[0]
    g64 = config4_gradient("fp64")[0]
    err = float(torch.linalg.norm(g32 - g64) / torch.linalg.norm(g64))
    print("fp32c vs fp64 gradient:", err)
    assert err <= 1e-2, err
