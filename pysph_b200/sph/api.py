"""`import pysph_b200.sph.api as sph` -- the functions of the particle-update
path and SPHCalc."""
from .sph_calc import SPHCalc
from .sph_func import (Function, SPHFunction, SPHFunctionParticle,
                       CSPHFunctionParticle, SPHRho, TaitEquation,
                       MomentumEquation, SPHPressureGradient,
                       MonaghanArtificialViscosity, GravityForce,
                       PositionStepping, SPHDensityRate, XSPHCorrection)

__all__ = ["SPHCalc", "Function", "SPHFunction", "SPHFunctionParticle",
           "CSPHFunctionParticle", "SPHRho", "TaitEquation", "MomentumEquation",
           "SPHPressureGradient", "MonaghanArtificialViscosity", "GravityForce", "PositionStepping",
           "SPHDensityRate", "XSPHCorrection"]
