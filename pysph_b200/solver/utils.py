"""Output files of the solver (S/solver/utils.py:34-186, 294-340).

Format version 1, as the reference writes it: one uncompressed ``.npz`` per
dump with three entries -- ``version`` (1), ``solver_data`` (a dict with dt,
t and count) and ``arrays`` (a dict of particle-array name -> dict of
property name -> numpy array, plus the array's constants), the two dicts
stored as numpy object arrays.  Files written here load in the reference and
the other way round.
"""
from __future__ import annotations

import os

import numpy as np


def savez(file, *args, **kwds):
    """Several arrays into one uncompressed .npz (numpy.savez)."""
    np.savez(file, *args, **kwds)


def savez_compressed(file, *args, **kwds):
    """Several arrays into one compressed .npz (numpy.savez_compressed)."""
    np.savez_compressed(file, *args, **kwds)


def _unwrap(obj):
    """A dict stored by savez as a 0-d object array."""
    a = np.asarray(obj)
    if a.dtype == object:
        a = a.reshape(1)[0]
    return a


def load(fname, device=None):
    """Data of an output file: {"arrays": {name: ParticleArray},
    "solver_data": {"dt", "t", "count"}} (S/solver/utils.py:294-340)."""
    from ..base.particle_array import get_particle_array
    data = np.load(fname, allow_pickle=True)
    if "version" not in data.files:
        raise RuntimeError("Wrong file type! No version number recorded.")
    version = int(data["version"])
    if version != 1:
        raise RuntimeError("Version not understood!")
    arrays = _unwrap(data["arrays"])
    solver_data = _unwrap(data["solver_data"])
    ret = {"arrays": {}, "solver_data": solver_data}
    for name, props in arrays.items():
        ret["arrays"][name] = get_particle_array(name=name, device=device, **props)
    return ret


def load_and_concatenate(prefix, nprocs=1, directory=".", count=None):
    """The arrays of the per-rank files <prefix>_<rank>_<count>.npz of one
    dump, concatenated per array name (S/solver/utils.py:342-380)."""
    if count is None:
        counts = sorted({int(f.rsplit("_", 1)[1][:-4]) for f in os.listdir(directory)
                         if f.startswith(prefix) and f.endswith(".npz")})
        count = counts[-1]
    parts = []
    for rank in range(nprocs):
        name = f"{prefix}_{rank}_{count}.npz" if nprocs > 1 else f"{prefix}_{count}.npz"
        parts.append(np.load(os.path.join(directory, name), allow_pickle=True))
    arrays = [_unwrap(p["arrays"]) for p in parts]
    out = {"arrays": {}, "solver_data": _unwrap(parts[0]["solver_data"])}
    for name in arrays[0]:
        props = {}
        for k in arrays[0][name]:
            vals = [a[name][k] for a in arrays]
            props[k] = (np.concatenate(vals) if isinstance(vals[0], np.ndarray)
                        and vals[0].ndim else vals[0])
        out["arrays"][name] = props
    return out
