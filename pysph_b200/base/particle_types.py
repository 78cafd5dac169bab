"""Particle types and tags (S/base/particle_types.py:1-38,
S/base/particle_array.pxd:20-26)."""


class ParticleType:
    """Enum of particle types.  Fluid, Solid, DummyFluid, Probe, Boundary."""
    Fluid = 0
    Solid = 1
    DummyFluid = 2
    Probe = 3
    Boundary = 4

    def __init__(self):
        raise SystemError("Do not instantiate the ParticleType class")


# particle tags
LocalReal = 0
Dummy = 1
LocalDummy = 2
RemoteReal = 3
RemoteDummy = 4
GhostParticle = 5


def get_local_real_tag():
    return LocalReal


def get_dummy_tag():
    return Dummy


def get_local_dummy_tag():
    return LocalDummy


def get_remote_real_tag():
    return RemoteReal


def get_remote_dummy_tag():
    return RemoteDummy


def is_local_real(tag):
    return tag == LocalReal
