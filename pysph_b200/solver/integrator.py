"""Integrators (S/solver/integrator.py:140-683).

PredictorCorrectorIntegrator.integrate(dt) is the hot path.  When its calcs
are the particle-update scheme -- SPHRho, then TaitEquation, then
MomentumEquation (or SPHPressureGradient), then GravityForce, then
PositionStepping, on any arrays -- or its continuity-equation form --
TaitEquation, SPHDensityRate, MomentumEquation, GravityForce,
PositionStepping, XSPHCorrection -- the whole step runs in the CUDA engine as
one fused pipeline per stage (rebin, density + EOS or Tait, one pair pass,
integrator stage); see fused_plan.  Any other calc list goes through the
building blocks below (eval: every calc's SPHCalc.sph on the engine; step:
elementwise updates of the FP64 properties), as the reference does.
"""
from __future__ import annotations

import torch

from .. import _native as nat
from ..engine import Scheme, SceneParams
from ..sph.sph_func import (SPHRho, TaitEquation, MomentumEquation,
                            SPHPressureGradient, GravityForce, PositionStepping,
                            SPHDensityRate, XSPHCorrection)


class FusedPlan:
    def __init__(self, scheme, params, mode, dim, tait_only, kernel=1):
        self.scheme = scheme
        self.params = params
        self.mode = mode
        self.dim = dim
        self.tait_only = tait_only
        self.kernel = kernel    # smoothing kernel type (KernelBase.get_type)


def fused_plan(particles, calcs):
    """The engine scheme of a calc list, or None when the list is not the
    particle-update scheme in its canonical order."""
    arrays = particles.arrays

    def idx(pa):
        for i, q in enumerate(arrays):
            if q is pa:
                return i
        raise ValueError("calc array not in particles")

    order = {SPHRho: 0, TaitEquation: 1, SPHDensityRate: 2, MomentumEquation: 3,
             SPHPressureGradient: 3, GravityForce: 4, PositionStepping: 5, XSPHCorrection: 6}
    rho_src, mom_src, tait_on, step_on, grav_on = {}, {}, set(), set(), set()
    rate_src, xsph_src = {}, {}
    params = {}
    mode = None
    last = -1
    dim = None
    ktype = None

    def agree(key, val):
        if key in params and params[key] != val:
            raise _NoPlan()
        params[key] = val

    try:
        for calc in calcs:
            cls = type(calc.funcs[0])
            if cls not in order:
                return None
            stage = order[cls]
            if stage < last:
                return None
            last = stage
            dim = dim or calc.kernel.dim
            ktype = ktype or calc.kernel.get_type()
            # one kernel for every calc, one the pair passes evaluate
            if calc.kernel.dim != dim or calc.kernel.get_type() != ktype:
                return None
            if ktype not in (1, 3, 4) or (ktype != 1 and dim != 2):
                return None
            d = idx(calc.dest)
            srcs = sum(1 << idx(s) for s in calc.sources)
            ups = list(calc.updates)
            # one hks option for every pair function of the fused passes
            for f in calc.funcs:
                if f.kind == "pair":
                    agree("hks", bool(f.hks))
            vel = ["u", "v", "w"][:dim]
            pos = ["x", "y", "z"][:dim]
            if cls is SPHRho:
                if calc.integrates or ups[:1] != ["rho"] or d in rho_src:
                    return None
                rho_src[d] = [b for b in range(len(arrays)) if srcs >> b & 1]
            elif cls is TaitEquation:
                if calc.integrates or ups[:2] != ["p", "cs"]:
                    return None
                f = calc.funcs[0]
                agree("c0", f.co)
                agree("rho0", f.ro)
                agree("gamma", f.gamma)
                tait_on.add(d)
            elif cls in (MomentumEquation, SPHPressureGradient):
                if not calc.integrates or ups[:dim] != vel or d in mom_src:
                    return None
                m = 0 if cls is MomentumEquation else 1
                if mode is not None and mode != m:
                    return None
                mode = m
                if m == 0:
                    f = calc.funcs[0]
                    agree("alpha", f.alpha)
                    agree("beta", f.beta)
                    agree("eta", f.eta)
                mom_src[d] = [b for b in range(len(arrays)) if srcs >> b & 1]
            elif cls is GravityForce:
                if not calc.integrates or ups[:dim] != vel:
                    return None
                f = calc.funcs[0]
                agree("gravity", (f.gx, f.gy, f.gz))
                grav_on.add(d)
            elif cls is PositionStepping:
                if not calc.integrates or ups[:dim] != pos:
                    return None
                step_on.add(d)
            elif cls is SPHDensityRate:
                if not calc.integrates or ups[:1] != ["rho"] or d in rate_src:
                    return None
                rate_src[d] = [b for b in range(len(arrays)) if srcs >> b & 1]
            elif cls is XSPHCorrection:
                # added to the position rate of an array already stepped
                if not calc.integrates or ups[:dim] != pos or d not in step_on or d in xsph_src:
                    return None
                agree("xsph_eps", calc.funcs[0].eps)
                xsph_src[d] = [b for b in range(len(arrays)) if srcs >> b & 1]
    except _NoPlan:
        return None
    if rho_src and rate_src:
        return None   # summation density and the continuity equation at once
    if not step_on or set(mom_src) != step_on:
        return None
    if grav_on and grav_on != step_on:
        return None
    if not grav_on:
        params["gravity"] = (0.0, 0.0, 0.0)
    tait_only = tait_on - set(rho_src) if not rate_src else set()
    scheme = Scheme(rho_src=rho_src, mom_src=mom_src, tait_on=tuple(sorted(tait_on)),
                    step_on=tuple(sorted(step_on)), rate_src=rate_src, xsph_src=xsph_src,
                    xsph_eps=params.get("xsph_eps", 0.5), hks=params.get("hks", False))
    p = SceneParams(**{k: v for k, v in params.items()
                       if k in SceneParams.__dataclass_fields__})
    return FusedPlan(scheme, p, mode or 0, dim, tuple(sorted(tait_only)), ktype or 1)


class _NoPlan(Exception):
    pass


class Integrator:
    """Base integrator: properties, accelerations, eval, step."""

    def __init__(self, particles=None, calcs=(), pcalcs=()):
        self.particles = particles
        self.calcs = list(calcs)
        self.nsteps = 1
        self.cstep = 1
        self.time = 0.0
        self.local_time = 0.0
        self.rupdate_list = []
        self.step_props = {}
        self.initial_properties = {}
        self.velocity_accelerations = {}
        self.plan = None
        self.check_every = 0

    def set_rupdate_list(self):
        self.rupdate_list = [[] for _ in self.particles.arrays]

    def setup_integrator(self):
        """Create the _<p>0 initial and _a_<p>_<k> acceleration properties of
        every integrating calc (S/solver/integrator.py:180-260)."""
        self.arrays = self.particles.arrays
        for array in self.arrays:
            self.step_props[array.name] = {k + 1: {} for k in range(self.nsteps)}
            self.initial_properties[array.name] = {}
            self.velocity_accelerations[array.name] = {k + 1: {} for k in range(self.nsteps)}
        for calc in self.calcs:
            dest = calc.dest
            if not calc.integrates:
                continue
            for update_prop in calc.updates:
                initial_prop = "_" + update_prop + "0"
                dest.add_property({"name": initial_prop})
                self.initial_properties[dest.name][update_prop] = initial_prop
                for k in range(self.nsteps):
                    k_num = k + 1
                    step_prop = "_a_" + update_prop + "_" + str(k_num)
                    dest.add_property({"name": step_prop})
                    self.step_props[dest.name][k_num][update_prop] = [initial_prop, step_prop]
                    calc.dst_writes.setdefault(k_num, []).append(step_prop)
        self.set_rupdate_list()
        self.plan = fused_plan(self.particles, self.calcs)

    # -------------------------------------------------------- building blocks
    def reset_accelerations(self, step):
        for array in self.arrays:
            for prop, (init, acc) in self.step_props[array.name][step].items():
                array.set_to_zero([acc])

    def save_initial_arrays(self):
        for array in self.arrays:
            array.copy_over_properties(self.initial_properties[array.name])

    def eval(self):
        k_num = self.cstep
        for calc in self.calcs:
            calc.dest.set_time(self.local_time)
            if calc.integrates:
                calc.sph(*calc.dst_writes[k_num])
            else:
                calc.sph(*calc.updates)

    def step(self, dt):
        k_num = self.cstep
        for array in self.arrays:
            to_step = self.step_props[array.name][k_num]
            for prop, (initial_prop, step_prop) in to_step.items():
                init = array.get(initial_prop)
                acc = array.get(step_prop)
                array.set(**{prop: init + acc * dt})
                if prop in ("u", "v", "w"):
                    self.velocity_accelerations[array.name][k_num][step_prop] = acc
        self.cstep += 1

    def get_max_acceleration(self, array, solver):
        if solver.count == 1:
            return solver.dt
        acc = -float("inf")
        if array.has_array("_a_u_1"):
            comps = [array.get("_a_u_1"), array.get("_a_v_1"), array.get("_a_w_1")][:solver.dim]
            a2 = sum(c * c for c in comps)
            acc = max(acc, float(torch.sqrt(a2).max().item()))
        return acc

    def integrate(self, dt):
        raise NotImplementedError

    # --------------------------------------------------------------- fused
    def _fused_session(self):
        s = self.particles.session(dim=self.plan.dim, scheme=self.plan.scheme,
                                   params=self.plan.params, kernel=self.plan.kernel)
        s.engine.force_mode = self.plan.mode
        s.engine.tait_only_mask = sum(1 << a for a in self.plan.tait_only)
        return s

    def _fused_reads(self, s):
        reads = set()
        for a, pa in enumerate(self.particles.arrays):
            for n in ("x", "y", "z", "u", "v", "w", "m", "h"):
                reads.add((a, n))
            if a not in self.plan.scheme.rho_src:
                reads |= {(a, "rho")}
            if a not in self.plan.scheme.tait_on:
                reads |= {(a, "p"), (a, "cs")}
        return reads

    def _fused_outputs(self, s, last_stage=1):
        """Mark what the fused step wrote as newer on the engine; the
        rates of the step's last stage go to _a_<p>_<last_stage> (1 for the
        predictor-corrector, Euler and RK2, whose stages all write k = 1;
        4 for RK4, whose K1 .. K3 stay on the device as a running sum)."""
        sc = self.plan.scheme
        dim = self.plan.dim
        acc = [f"_a_u_{last_stage}", f"_a_v_{last_stage}"] + (
            [f"_a_w_{last_stage}"] if dim == 3 else [])
        for a in range(len(self.particles.arrays)):
            names = []
            if a in sc.rho_src:
                names.append("rho")
            if a in sc.rate_src:
                names += ["rho", "_rho0", f"_a_rho_{last_stage}"]
            if a in sc.tait_on:
                names += ["p", "cs"]
            if a in sc.step_on:
                names += (["x", "y", "u", "v"] if dim == 2
                          else ["x", "y", "z", "u", "v", "w"])
                names += ["_x0", "_y0", "_u0", "_v0"] if dim == 2 else \
                    ["_x0", "_y0", "_z0", "_u0", "_v0", "_w0"]
                names += acc
            if a in sc.mom_src and self.plan.mode == 0:
                names.append("dt_fac")
            s.mark_engine_newer(a, names)


    def _fused_integrate(self, dt, device_dt, kind):
        """The whole step on the engine (fused plan)."""
        s = self._fused_session()
        imports = []   # host-written positions / velocities, imported by the step
        s.ensure(self._fused_reads(s), step_decides=True, defer=imports)
        eng = s.engine
        if not device_dt:
            eng.set_dt_async(dt)
        # one CUDA graph per step once the step repeats (Engine.step_graphed)
        eng.step_graphed(kind, imports)
        self._fused_outputs(s, 4 if kind == "rk4" else 1)
        self.time += dt if not device_dt else 0.0
        self._steps = getattr(self, "_steps", 0) + 1
        if self.check_every and self._steps % self.check_every == 0:
            s.check()


class PredictorCorrectorIntegrator(Integrator):
    """X(t+h/2) = X0 + h/2 F(X); X(t+h/2) = X0 + h/2 F(X(t+h/2));
    X(t+h) = 2 X(t+h/2) - X0 (S/solver/integrator.py:614-683)."""

    def __init__(self, particles, calcs):
        Integrator.__init__(self, particles, calcs)
        self.nsteps = 1

    def final_step(self):
        for array in self.arrays:
            for prop, (initial_prop, _) in self.step_props[array.name][1].items():
                cur = array.get(prop)
                init = array.get(initial_prop)
                array.set(**{prop: 2 * cur - init})

    def integrate(self, dt, device_dt=False):
        """One step.  device_dt: the engine's CFL rule chooses dt (the Solver
        uses it for the viscous / force time-step functions)."""
        if self.plan is not None:
            return self._fused_integrate(dt, device_dt, "pc")
        self.save_initial_arrays()
        self.reset_accelerations(step=1)
        self.local_time = self.time
        self.eval()
        self.step(dt / 2)
        self.particles.update()
        self.cstep = 1
        self.reset_accelerations(step=1)
        self.local_time = self.time + dt / 2
        self.eval()
        self.step(dt / 2)
        self.particles.update()
        self.final_step()
        self.particles.update()
        self.cstep = 1


class EulerIntegrator(Integrator):
    """Forward Euler: X(t+h) = X0 + h F(X) (S/solver/integrator.py:420-447)."""

    def integrate(self, dt, device_dt=False):
        if self.plan is not None:
            return self._fused_integrate(dt, device_dt, "euler")
        self.save_initial_arrays()
        self.reset_accelerations(step=1)
        self.local_time = self.time
        self.eval()
        self.step(dt)
        self.particles.update()
        self.cstep = 1


class RK2Integrator(Integrator):
    """X(t+h/2) = X0 + h/2 F(X); X(t+h) = X0 + h F(X(t+h/2))
    (S/solver/integrator.py:452-499)."""

    def integrate(self, dt, device_dt=False):
        if self.plan is not None:
            return self._fused_integrate(dt, device_dt, "rk2")
        self.save_initial_arrays()
        self.reset_accelerations(step=1)
        self.local_time = self.time
        self.eval()
        self.step(dt / 2)
        self.particles.update()
        self.cstep = 1
        self.reset_accelerations(step=1)
        self.local_time = self.time + dt / 2
        self.eval()
        self.step(dt)
        self.particles.update()
        self.cstep = 1


class RK4Integrator(Integrator):
    """Classical RK4 with four evaluations and X(t+h) = X0 + h/6 (K1 + 2 K2
    + 2 K3 + K4) (S/solver/integrator.py:504-609).  With a fused plan the
    whole step runs on the engine (stage kinds 4-7, K1 + 2 K2 + 2 K3 kept as
    a running sum on the device, K4 in _a_<p>_4); otherwise calc by calc,
    the four stage rates in the particle arrays as the reference keeps
    them."""

    def __init__(self, particles, calcs):
        Integrator.__init__(self, particles, calcs)
        self.nsteps = 4

    def final_step(self, dt):
        fac = 1.0 / 6.0
        for array in self.arrays:
            to_step = [self.step_props[array.name][k] for k in (1, 2, 3, 4)]
            for prop in to_step[0]:
                init = array.get(to_step[0][prop][0])
                k1, k2, k3, k4 = (array.get(t[prop][1]) for t in to_step)
                array.set(**{prop: init + fac * dt * (k1 + 2 * k2 + 2 * k3 + k4)})

    def integrate(self, dt, device_dt=False):
        if self.plan is not None:
            return self._fused_integrate(dt, device_dt, "rk4")
        self.save_initial_arrays()
        self.reset_accelerations(step=1)
        self.local_time = self.time
        self.eval()
        self.step(dt / 2)
        self.particles.update()
        self.reset_accelerations(step=2)
        self.local_time = self.time + dt / 2
        self.eval()
        self.step(dt / 2)
        self.particles.update()
        self.reset_accelerations(step=3)
        self.local_time = self.time + dt / 2
        self.eval()
        self.step(dt)
        self.particles.update()
        self.reset_accelerations(step=4)
        self.local_time = self.time + dt
        self.eval()
        self.final_step(dt)
        self.particles.update()
        self.cstep = 1
