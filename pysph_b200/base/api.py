"""`import pysph_b200.base.api as base` -- the names of pysph.base.api that
this build provides."""
from .kernels import (CubicSplineKernel, KernelBase, QuinticSplineKernel,
                      WendlandQuinticSplineKernel)
from .particle_array import ParticleArray, get_particle_array
from .particle_types import (ParticleType, LocalReal, Dummy, LocalDummy,
                             RemoteReal, RemoteDummy, get_local_real_tag,
                             get_dummy_tag, get_local_dummy_tag,
                             get_remote_real_tag, get_remote_dummy_tag)
from .particles import Particles, NeighborLocatorType, NNPSManager, Locator
from .point import Point

Fluid = ParticleType.Fluid
Solid = ParticleType.Solid

__all__ = ["CubicSplineKernel", "QuinticSplineKernel", "WendlandQuinticSplineKernel",
           "KernelBase", "ParticleArray", "get_particle_array",
           "ParticleType", "Particles", "NeighborLocatorType", "NNPSManager",
           "Locator", "Point", "Fluid", "Solid", "LocalReal"]
