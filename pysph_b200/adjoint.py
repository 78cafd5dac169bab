"""Differentiable predictor-corrector rollout with a hand-written adjoint.

Rollout advances one scene for `steps` steps of fixed dt on a forward
engine (FP32C by default: FP32 pair sums with Kahan compensation, FP64
state) and keeps a checkpoint of the state every `checkpoint_every` steps.
backward() walks the segments in reverse: it recomputes a segment from its
checkpoint on the same forward engine (deterministic, so the states are the
forward's own), exporting both stage states of every step, then applies the
adjoint of each step in reverse order.  The adjoint of the acceleration
function F(X, V) -- summation density -> Tait -> MomentumEquation -- is
evaluated at each stage state by the FP64 kernels sphb_force_vjp,
sphb_eos_vjp and sphb_density_vjp (FP64 adjoint reductions).

With X0, V0 the state at the start of a step and F = F(X0, V0):
  Xh = X0 + dt/2 V0,   Vh = V0 + dt/2 F,   F' = F(Xh, Vh),
  X1 = X0 + dt Vh,     V1 = V0 + dt F'
(PredictorCorrectorIntegrator, S/solver/integrator.py:614-683: X1 =
2 (X0 + dt/2 Vh) - X0).  Reverse, given lX1, lV1:
  lVh = dt lX1;  lF' = dt lV1;  (lXh, lVh') = VJP_F(Xh, Vh; lF');  lVh += lVh'
  lX0 = lX1 + lXh;  lV0 = lV1 + dt/2 lXh + lVh;  lF = dt/2 lVh
  (lX0', lV0') = VJP_F(X0, V0; lF);  lX0 += lX0';  lV0 += lV0'

RolloutFunction wraps it as a torch.autograd.Function of the initial
velocities.

With graphs=True (CUDA devices) the forward step, a segment's recompute
(with every step's two stage states exported) and the segment's adjoint
are each captured once in a CUDA graph and replayed: one launch per step
forward and two per segment backward instead of thousands, with the
results of the eager calls.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as nat
from .engine import Engine, Scheme, SceneParams


class Rollout:
    def __init__(self, arrays, params, scheme: Scheme, dim: int = 2, dt: float = 1e-5,
                 steps: int = 200, checkpoint_every: int = 20, precision: str = "fp32c",
                 device=None, lanes: int = 1, pair_block: int = 128, graphs: bool = True,
                 adj_lanes: int = 2, adj_pair_block: int = 128):
        if scheme.continuity:
            raise NotImplementedError("the adjoint covers the summation-density scheme")
        if scheme.hks:
            raise NotImplementedError("the adjoint covers kernels at h_ab only (hks off)")
        if scheme.mom_src and set(scheme.step_on) != set(scheme.mom_src):
            raise ValueError("the integrated arrays must be the MomentumEquation dests")
        self.arrays = arrays
        self.params = dict(params)
        self.params["dt"] = dt
        self.params["cfl"] = 0.0
        self.scheme = scheme
        self.dim = dim
        self.dt = dt
        self.steps = steps
        self.k = checkpoint_every
        self.fwd = Engine([(arrays, self.params)], scheme, dim=dim, precision=precision,
                          device=device, lanes=lanes, pair_block=pair_block)
        # the FP64 adjoint engine: two lanes per particle (the VJP kernels
        # carry far more work per pair than the forward passes; on the 50k
        # drop the backward took 92.8 ms with one lane, 80.9 with two, 89.3
        # with four and 101.8 with eight)
        self.adj = Engine([(arrays, self.params)], scheme, dim=dim, precision="fp64",
                          device=device, lanes=adj_lanes, pair_block=adj_pair_block)
        self.device = self.fwd.device
        self.moving = list(scheme.step_on)
        self.checkpoints = []
        self._scratch = None
        self.graphs = bool(graphs)
        self._g = {}   # captured graphs and their fixed buffers

    # ---------------------------------------------------------------- state
    def _comps(self):
        return ("x", "y", "z")[:self.dim], ("u", "v", "w")[:self.dim]

    def get_state(self, eng=None):
        eng = eng or self.fwd
        px, pv = self._comps()
        return {a: (torch.stack([eng.get(a, c) for c in px]),
                    torch.stack([eng.get(a, c) for c in pv])) for a in self.moving}

    def set_state(self, state, eng=None, rebin=True):
        """The state into an engine, rebinned there: every restart from the
        same state (the forward's checkpoints, the backward's recomputes)
        then starts from the same order and lists.  rebin=False leaves the
        rebin to the engine's next decision (the VJPs' stage states, which
        lie within the list skin of each other)."""
        eng = eng or self.fwd
        px, pv = self._comps()
        for a, (X, V) in state.items():
            for d, c in enumerate(px):
                eng.exchange_in(a, c, X[d])
            for d, c in enumerate(pv):
                eng.exchange_in(a, c, V[d])
        eng.invalidate_box()
        if rebin:
            eng.rebin_now()

    # -------------------------------------------------------------- forward
    def forward(self, velocities):
        """velocities: {array: tensor [dim, n]} initial velocities (user
        order).  Returns the final state {array: (X, V)}."""
        state0 = {a: (self._initial_positions(a), velocities[a].to(self.device, torch.float64))
                  for a in self.moving}
        self.set_state(state0)
        self.checkpoints = [self._clone(state0)]
        eng = self.fwd
        eng.set_dt_async(self.dt)
        for n in range(self.steps):
            self._fwd_step()
            if (n + 1) % self.k == 0 and n + 1 < self.steps:
                ck = self._clone(self.get_state())
                self.checkpoints.append(ck)
                # restart from the checkpoint exactly as backward() will, so
                # the recomputed segment is bit-identical to this one
                self.set_state(ck)
        eng.check_status()
        return self.get_state()

    def _initial_positions(self, a):
        px, _ = self._comps()
        return torch.stack([torch.as_tensor(self.arrays[a][c], dtype=torch.float64)
                            for c in px]).to(self.device)

    @staticmethod
    def _clone(state):
        return {a: (X.clone(), V.clone()) for a, (X, V) in state.items()}

    # ------------------------------------------------------------- graphs
    def _fwd_step(self):
        """One forward step: eager the first time, captured the second,
        replayed after that."""
        g = self._g.get("fwd")
        if not self.graphs or g is None:
            if self.graphs:
                self._g["fwd"] = "warm"
            self.fwd.pc_step()
            return
        if g == "warm":
            torch.cuda.synchronize(self.device)
            g = self._g["fwd"] = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.fwd.pc_step()
        g.replay()

    # ---------------------------------------------------------------- VJP
    def vjp_F(self, state, lam_F):
        """(d F / d(X, V))^T lam_F at state: {array: (lX, lV)}."""
        eng = self.adj
        # the stage states of a segment lie close together: the lists of the
        # last rebin (with their skin) hold every pair while the decision
        # keeps them, and the VJP kernels test each pair themselves
        self.set_state(state, eng, rebin=False)
        eng.density(reuse=True)
        N = eng.N
        dim = self.dim
        dev = self.device
        if self._scratch is None:
            # one buffer, cleared by one launch per VJP
            self._scratch_buf = torch.zeros((3 * dim + 3) * N, dtype=torch.float64, device=dev)
            parts = self._scratch_buf.split([dim * N] * 3 + [N] * 3)
            self._scratch = dict(lam_a=parts[0].view(dim, N), lam_x=parts[1].view(dim, N),
                                 lam_v=parts[2].view(dim, N), lam_rho=parts[3],
                                 lam_p=parts[4], lam_c=parts[5])
        S = self._scratch
        self._scratch_buf.zero_()
        for a, L in lam_F.items():
            for d in range(dim):
                eng.call("sphb_permute", eng.cur, a, 0, L[d].contiguous().data_ptr(),
                         S["lam_a"][d].data_ptr(), eng.user_offset[a].data_ptr())
        mom = self.scheme.mom_dests
        eng.call("sphb_force_vjp", eng.cur, mom, S["lam_a"].data_ptr(), S["lam_x"].data_ptr(),
                 S["lam_v"].data_ptr(), S["lam_rho"].data_ptr(), S["lam_p"].data_ptr(),
                 S["lam_c"].data_ptr())
        eng.call("sphb_eos_vjp", eng.cur, S["lam_rho"].data_ptr(), S["lam_p"].data_ptr(),
                 S["lam_c"].data_ptr())
        eng.call("sphb_density_vjp", eng.cur, self.scheme.rho_dests, S["lam_rho"].data_ptr(),
                 S["lam_x"].data_ptr())
        out = {}
        for a in self.moving:
            n = eng.user_n[a]
            lX = torch.empty(dim, n, dtype=torch.float64, device=dev)
            lV = torch.empty(dim, n, dtype=torch.float64, device=dev)
            for d in range(dim):
                eng.call("sphb_permute", eng.cur, a, 1, lX[d].data_ptr(),
                         S["lam_x"][d].data_ptr(), eng.user_offset[a].data_ptr())
                eng.call("sphb_permute", eng.cur, a, 1, lV[d].data_ptr(),
                         S["lam_v"][d].data_ptr(), eng.user_offset[a].data_ptr())
            out[a] = (lX, lV)
        return out

    def step_adjoint(self, s0, sh, lam):
        dt = self.dt
        lVh = {a: dt * lX1 for a, (lX1, lV1) in lam.items()}
        lFp = {a: dt * lV1 for a, (lX1, lV1) in lam.items()}
        g = self.vjp_F(sh, lFp)
        lX0, lV0, lF = {}, {}, {}
        for a, (lX1, lV1) in lam.items():
            lXh, lVh_add = g[a]
            lVh[a] = lVh[a] + lVh_add
            lX0[a] = lX1 + lXh
            lV0[a] = lV1 + 0.5 * dt * lXh + lVh[a]
            lF[a] = 0.5 * dt * lVh[a]
        g0 = self.vjp_F(s0, lF)
        return {a: (lX0[a] + g0[a][0], lV0[a] + g0[a][1]) for a in lam}

    def backward(self, lam_final):
        """lam_final: {array: (dL/dX_final, dL/dV_final)}.  Returns
        {array: (dL/dX_0, dL/dV_0)}."""
        lam = {a: (lX.to(self.device, torch.float64), lV.to(self.device, torch.float64))
               for a, (lX, lV) in lam_final.items()}
        nseg = len(self.checkpoints)
        for si in reversed(range(nseg)):
            start = si * self.k
            n = min(self.k, self.steps - start)
            # the segment's states, recomputed from its checkpoint, then its
            # steps' adjoints in reverse: one graph replay each
            self.set_state(self.checkpoints[si])
            self.fwd.set_dt_async(self.dt)
            states = self._segment_rec(n)
            lam = self._clone(self._segment_adj(n, states, lam))
        self.adj.check_status()
        self.fwd.check_status()
        return lam

    def _recompute(self, n):
        """n forward steps from the engine's state; per step the states
        (X0, V0) and (Xh, Vh) of its two stages."""
        out = []
        for _ in range(n):
            s0 = self.get_state()
            half = {}
            self.fwd.pc_step(on_half=lambda: half.__setitem__("sh", self.get_state()))
            out.append((s0, half["sh"]))
        return out

    def _adjoint(self, states, lam):
        for s0, sh in reversed(states):
            lam = self.step_adjoint(s0, sh, lam)
        return lam

    # A segment's recompute and its adjoint each run eagerly the first time
    # (warming every kernel and allocation), are captured the second time
    # and replayed after that.  The captured adjoint reads the recompute
    # graph's own output tensors and a fixed copy of the incoming lam.
    def _segment_rec(self, n):
        key = ("rec", n)
        g = self._g.get(key)
        if not self.graphs or g is None:
            if self.graphs:
                self._g[key] = "warm"
            return self._recompute(n)
        if g == "warm":
            torch.cuda.synchronize(self.device)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                out = self._recompute(n)
            g = self._g[key] = (graph, out)
        graph, out = g
        graph.replay()
        return out

    def _segment_adj(self, n, states, lam):
        key = ("adj", n)
        g = self._g.get(key)
        if not self.graphs or g is None:
            if self.graphs:
                self._g[key] = "warm"
            return self._adjoint(states, lam)
        if g == "warm":
            buf = self._clone(lam)
            torch.cuda.synchronize(self.device)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                out = self._adjoint(states, buf)
            g = self._g[key] = (graph, states, buf, out)
            lam = None   # the buffer holds it already
        graph, cap_states, buf, out = g
        if states is not cap_states:
            raise RuntimeError("the adjoint graph reads the recompute graph's outputs")
        for a, (X, V) in (lam or {}).items():
            buf[a][0].copy_(X)
            buf[a][1].copy_(V)
        graph.replay()
        return out


class RolloutFunction(torch.autograd.Function):
    """Final positions of a Rollout as a differentiable function of the
    initial velocities of array 0 (shape [dim, n])."""

    @staticmethod
    def forward(ctx, v0, rollout: Rollout):
        a = rollout.moving[0]
        final = rollout.forward({a: v0.detach()})
        ctx.rollout = rollout
        return final[a][0]

    @staticmethod
    def backward(ctx, grad_x):
        r = ctx.rollout
        a = r.moving[0]
        lam = {a: (grad_x.contiguous(), torch.zeros_like(grad_x))}
        g = r.backward(lam)
        return g[a][1], None
