"""Solver: operations -> calcs -> integrator, and the time loop
(S/solver/solver.py:60-590).

solve() runs the reference's loop: t += dt, count += 1, update the
particles, choose dt, integrate.  With the fused engine path and a
viscous / force-based time-step function, dt is chosen on the GPU by the
same rule (sphb_step_begin) and read back once per step together with the
simulated time, which the loop needs to know when to stop.
"""
from __future__ import annotations

import logging
import os

from ..base.kernels import CubicSplineKernel
from ..base.particle_types import ParticleType
from ..sph.sph_func import PositionStepping, XSPHCorrection
from .integrator import PredictorCorrectorIntegrator
from .sph_equation import SPHIntegration, SPHOperation
from .time_step_functions import TimeStep
from .utils import load, savez

logger = logging.getLogger(__name__)

Fluids = ParticleType.Fluid


class Solver:
    def __init__(self, dim, integrator_type=PredictorCorrectorIntegrator,
                 kernel=None, **kwargs):
        self.dim = dim
        self.integrator_type = integrator_type
        self.kernel = kernel or CubicSplineKernel(dim=dim)
        self.operation_dict = {}
        self.order = []
        self.t = 0.0
        self.tf = 1.0
        self.dt = 1e-3
        self.count = 0
        self.pfreq = 100
        self.time_step_function = TimeStep()
        self.pre_step_functions = []
        self.post_step_functions = []
        self.execute_commands = None
        self.command_interval = 1
        self.print_properties = ["x", "u", "m", "h", "p", "e", "rho"]
        if dim > 1:
            self.print_properties.extend(["y", "v"])
        if dim > 2:
            self.print_properties.extend(["z", "w"])
        self.particles = None
        self.integrator = None
        self.with_cl = False
        self.rank = 0
        # output files (S/solver/solver.py:142-148): <fname>_<count>.npz in
        # <fname>_output, written at the start of solve() and every pfreq
        # steps; dump_output=False turns them off
        self.fname = type(self).__name__
        self.output_directory = self.fname + "_output"
        self.dump = True
        self.detailed_output = False
        self.dt_history = []

    # ------------------------------------------------------------ set-up
    def add_operation(self, operation, before=False, id=None):
        if operation.id in self.operation_dict:
            raise RuntimeError(f"operation {operation.id!r} exists")
        self.operation_dict[operation.id] = operation
        if id is None:
            self.order.append(operation.id)
        else:
            i = self.order.index(id)
            self.order.insert(i if before else i + 1, operation.id)

    def replace_operation(self, id, new_operation):
        i = self.order.index(id)
        self.operation_dict.pop(id)
        self.order[i] = new_operation.id
        self.operation_dict[new_operation.id] = new_operation

    def remove_operation(self, id):
        self.order.remove(id)
        self.operation_dict.pop(id)

    def add_operation_step(self, types, xsph=False, eps=0.5):
        """Position stepping dx/dt = v on `types` (S/solver/solver.py:168-183),
        followed by the XSPH correction when xsph."""
        updates = ["x", "y", "z"][:self.dim]
        self.add_operation(SPHIntegration(PositionStepping.withargs(), on_types=types,
                                          updates=updates, id="step"))
        if xsph:
            self.add_operation_xsph(eps)

    def add_operation_xsph(self, eps, hks=False):
        """XSPHCorrection on the arrays the position stepping moves, from
        those same arrays, added to their position rate
        (S/solver/solver.py:185-220)."""
        assert eps > 0, "Invalid value for XSPH epsilon: %f" % eps
        self.eps = eps
        assert "step" in self.operation_dict, "position stepping function does not exist!"
        step = self.operation_dict["step"]
        self.add_operation(SPHIntegration(
            XSPHCorrection.withargs(eps=eps, hks=hks), from_types=step.on_types,
            on_types=step.on_types, updates=step.updates, id="xsph"))

    def set_final_time(self, tf):
        self.tf = tf

    def set_time_step(self, dt):
        self.dt = dt

    def set_print_freq(self, n):
        self.pfreq = n

    def set_output_fname(self, fname):
        self.fname = fname

    def set_output_printing_level(self, detailed_output):
        self.detailed_output = detailed_output

    def set_output_directory(self, path):
        self.output_directory = path

    # ------------------------------------------------------------ output
    def dump_output(self, dt, *print_properties):
        """Write <output_directory>/<fname>_<count>.npz in format version 1
        (S/solver/solver.py:605-695): solver_data (dt, t, count) and, per
        particle array, its properties -- all of them with detailed output,
        else those not starting with '_' plus _tmpx/_tmpy/_tmpz."""
        if not self.dump:
            return None
        os.makedirs(self.output_directory, exist_ok=True)
        path = os.path.join(self.output_directory, f"{self.fname}_{self.count}.npz")
        props = {"arrays": {}, "solver_data": {"dt": dt, "t": self.t, "count": self.count}}
        for array in self.particles.arrays:
            props["arrays"][array.name] = array.get_property_arrays(all=self.detailed_output)
        savez(path, version=1, **props)
        return path

    def load_output(self, count):
        """Resume from <fname>_<count>.npz (S/solver/solver.py:697-739):
        the arrays' properties, t and count; '?' lists the counts on disk."""
        counts = sorted({int(f.rsplit("_", 1)[1][:-4]) for f in os.listdir(self.output_directory)
                         if f.startswith(self.fname) and f.endswith(".npz")})
        if count == "?":
            return counts
        if int(count) not in counts:
            raise IOError(f"File with iteration count `{count}` does not exist\n"
                          f"Valid iteration counts are {counts}")
        data = load(os.path.join(self.output_directory, f"{self.fname}_{count}.npz"))
        for pa in self.particles.arrays:
            src = data["arrays"][pa.name]
            vals = {n: src.get(n) for n in src.get_property_names()
                    if pa.has_array(n) and n not in ("group", "local", "pid", "idx")}
            pa.set(**vals)
            pa.constants.update(src.constants)
        self.t = float(data["solver_data"]["t"])
        self.count = int(data["solver_data"]["count"])

    def set_command_handler(self, callable, command_interval=1):
        self.execute_commands = callable
        self.command_interval = command_interval

    def setup(self, particles=None):
        """Build the calcs of every operation, in order, and the integrator."""
        self.particles = particles
        particles.kernel = self.kernel
        calcs = []
        for oid in self.order:
            op = self.operation_dict[oid]
            calcs.extend(op.get_calcs(particles, self.kernel))
        self.integrator = self.integrator_type(particles, calcs)
        self.integrator.setup_integrator()

    # -------------------------------------------------------------- loop
    def _device_rule(self):
        rule = getattr(self.time_step_function, "device_rule", None)
        return rule if (rule and self.integrator.plan is not None) else None

    def solve(self, show_progress=False):
        dt = self.dt
        self.dump_output(dt, *self.print_properties)
        self.integrator.time = self.t
        rule = self._device_rule()
        if rule:
            f = self.time_step_function
            s = self.integrator._fused_session()
            s.engine.update_params(cfl=float(f.cfl), c0=s.engine.params[0].c0,
                                   dt_initial=float(self.dt),
                                   cfl_force=(rule == "viscous+force"))
            self.integrator.plan.params = s.engine.params[0]
        while self.t < self.tf:
            self.t += dt
            self.count += 1
            self.particles.update()
            for func in self.pre_step_functions:
                func.eval(self)
            if rule:
                self.integrator.integrate(0.0, device_dt=True)
                st = self.integrator.particles.session().engine.scene_state()[0]
                dt = st.dt
                self.integrator.time += dt
            else:
                dt = self.time_step_function.compute_time_step(self)
                self.integrator.integrate(dt)
                self.integrator.time += dt
            self.dt_history.append(dt)
            for array in self.particles.arrays:
                array.set_time(self.t)
            for func in self.post_step_functions:
                func.eval(self)
            if self.count % self.pfreq == 0:
                self.dump_output(dt, *self.print_properties)
            if self.execute_commands is not None and self.count % self.command_interval == 0:
                self.execute_commands(self)
        if rule:
            self.particles.session().check()

    def get_options(self, opt_parser):
        pass
