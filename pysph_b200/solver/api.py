"""`import pysph_b200.solver.api as solver` -- operations, integrators,
time-step functions and the Solver of the particle-update path."""
from .integrator import (Integrator, PredictorCorrectorIntegrator, EulerIntegrator,
                         RK2Integrator, RK4Integrator, fused_plan)
from .solver import Solver
from .sph_equation import SPHOperation, SPHIntegration
from .time_step_functions import (TimeStep, ViscousTimeStep,
                                  ViscousAndForceBasedTimeStep, VelocityBasedTimeStep)

HAS_CL = False

__all__ = ["Integrator", "PredictorCorrectorIntegrator", "EulerIntegrator",
           "RK2Integrator", "RK4Integrator", "Solver",
           "SPHOperation", "SPHIntegration", "TimeStep", "ViscousTimeStep",
           "ViscousAndForceBasedTimeStep", "VelocityBasedTimeStep", "fused_plan"]
