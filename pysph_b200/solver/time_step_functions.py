"""Time-step functions (S/solver/time_step_functions.py:1-71).

compute_time_step(solver) keeps the reference's rules.  When the solver's
integrator runs the fused engine path, the viscous / force criteria are
evaluated on the GPU from the max dt_fac and |a| the force kernel keeps
(sphb_step_begin), so no per-particle array crosses to the host; the host
versions below are used otherwise.
"""
from __future__ import annotations

import torch


class TimeStep:
    device_rule = None

    def compute_time_step(self, solver):
        return solver.dt


class ViscousTimeStep(TimeStep):
    """dt = min over arrays with dt_fac of cfl h / (co + max dt_fac)."""

    device_rule = "viscous"

    def __init__(self, cfl, co, particles):
        self.cfl = cfl
        self.co = co
        self.particles = particles

    def compute_time_step(self, solver):
        dt = 1.0
        for array in self.particles.arrays:
            if array.has_array("dt_fac"):
                h, dt_fac = array.get("h", "dt_fac")
                _dt = float(torch.min(self.cfl * h / (self.co + torch.max(dt_fac))).item())
                dt = min(_dt, dt)
        return dt


class ViscousAndForceBasedTimeStep(ViscousTimeStep):
    """Also dt <= cfl sqrt(h / max |a|) (solver.dt stands in for max |a| at
    the first step, as Integrator.get_max_acceleration does)."""

    device_rule = "viscous+force"

    def compute_time_step(self, solver):
        dt = ViscousTimeStep.compute_time_step(self, solver)
        integrator = solver.integrator
        for array in self.particles.arrays:
            if array.has_array("_a_u_1"):
                fmax = integrator.get_max_acceleration(array, solver)
                h = array.get("h")
                _dt = self.cfl * float(torch.min(torch.sqrt(h / fmax)).item())
                dt = min(dt, _dt)
        return dt


class VelocityBasedTimeStep:
    def __init__(self, particles, cfl=0.3):
        self.cfl = cfl
        self.particles = particles

    def compute_time_step(self, solver):
        v = float("inf")
        for pa in solver.particles.arrays:
            val = float(torch.min(pa.get("h") / (pa.get("cs") + (
                pa.get("u") ** 2 + pa.get("v") ** 2 + pa.get("w") ** 2) ** 0.5)).item())
            v = min(v, val)
        return self.cfl * v
