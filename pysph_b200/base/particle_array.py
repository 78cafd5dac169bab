"""ParticleArray: the reference's SoA particle container, backed by torch
tensors (S/base/particle_array.pyx:96-1400, get_particle_array :1400-1490).

Properties are 1-D tensors on one device (FP64 for 'double', int64 for
'long'/'int').  The values a user sees are always in the array's own index
order: when the engine has computed a property more recently than the
tensor, reading it (get, attribute access, get_carray) first copies it back
from the engine; set() marks the property as changed for the engine.  Edits
made in place on a tensor obtained from the array are not tracked -- call
set_dirty(True) (or Particles.update()) afterwards, as the reference requires
for moved particles.
"""
from __future__ import annotations

import numpy as np
import torch

from .particle_types import ParticleType, LocalReal

POSITION_PROPS = ("x", "y", "z")
DEFAULT_PROPS = {"x": 0.0, "y": 0.0, "z": 0.0, "u": 0.0, "v": 0.0, "w": 0.0,
                 "m": 1.0, "h": 1.0, "p": 0.0, "e": 0.0, "rho": 1.0, "cs": 0.0,
                 "_tmpx": 0.0, "_tmpy": 0.0, "_tmpz": 0.0}


def default_device():
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


def _dtype(kind):
    if kind in ("int", "long"):
        return torch.int64
    if kind in ("double", None):
        return torch.float64
    if kind == "float":
        return torch.float32
    raise ValueError(f"unknown property type {kind!r}")


class ParticleArray:
    """Particle properties of one particle type (fluid, solid, ...)."""

    def __init__(self, name: str = "", particle_type: int = ParticleType.Fluid,
                 cl_precision: str = "double", device=None, **props):
        self.name = name
        self.particle_type = particle_type
        self.cl_precision = cl_precision
        self.device = torch.device(device) if device is not None else default_device()
        self.properties: dict[str, torch.Tensor] = {}
        self.property_types: dict[str, str] = {}
        self.default_values: dict[str, float] = {}
        self.constants: dict = {}
        self.is_dirty = True
        self.time = 0.0
        self._n = 0
        # engine link (set by Particles): property -> True when the engine
        # holds a newer value than the tensor
        self._engine_newer: set[str] = set()
        self._session = None
        self._versions: dict[str, int] = {}
        for spec in props.values():
            if isinstance(spec, dict) and spec.get("data") is not None:
                self._n = len(spec["data"])
                break
        for pname, spec in props.items():
            if not isinstance(spec, dict):
                spec = {"data": spec}
            info = dict(spec)
            info.setdefault("name", pname)
            self.add_property(info)
        for pname, kind, default in (("tag", "long", LocalReal), ("group", "long", 0),
                                     ("local", "long", 1), ("pid", "long", 0)):
            if pname not in self.properties:
                self.add_property({"name": pname, "type": kind, "default": default})

    # ------------------------------------------------------------------ info
    def get_number_of_particles(self) -> int:
        return self._n

    @property
    def num_real_particles(self) -> int:
        return int((self.properties["tag"] == LocalReal).sum().item()) if self._n else 0

    def has_array(self, name: str) -> bool:
        return name in self.properties

    def get_property_names(self):
        return list(self.properties)

    def __len__(self):
        return self._n

    def __repr__(self):
        return f"ParticleArray(name={self.name!r}, n={self._n})"

    # ------------------------------------------------------------ properties
    def add_property(self, prop_info: dict):
        """Add a property: {'name', 'type' ('double'|'long'|'int'), 'default',
        'data'} (ParticleArray.add_property)."""
        name = prop_info["name"]
        kind = prop_info.get("type", "double")
        default = prop_info.get("default", DEFAULT_PROPS.get(name, 0.0))
        data = prop_info.get("data")
        dt = _dtype(kind)
        if data is not None:
            t = torch.as_tensor(np.asarray(data) if not isinstance(data, torch.Tensor) else data,
                                dtype=dt).to(self.device).clone()
            if t.dim() != 1:
                raise ValueError(f"property {name} must be 1-D")
            if self._n and t.numel() != self._n:
                raise ValueError(f"property {name} has {t.numel()} values, "
                                 f"the array has {self._n} particles")
            self._n = t.numel()
        else:
            if name in self.properties:
                return
            t = torch.full((self._n,), default, dtype=dt, device=self.device)
        self.properties[name] = t
        self.property_types[name] = "long" if dt == torch.int64 else "double"
        self.default_values[name] = default
        self._touch(name)

    def _touch(self, name):
        self._versions[name] = self._versions.get(name, 0) + 1
        self._engine_newer.discard(name)
        if name in POSITION_PROPS:
            self.is_dirty = True
        if self._session is not None:
            self._session.user_changed(self, name)

    def version(self, name) -> int:
        return self._versions.get(name, 0)

    def _sync(self, name):
        if name in self._engine_newer and self._session is not None:
            self._session.export_to_array(self, name)

    def _check_property(self, name):
        if name not in self.properties:
            raise AttributeError(f"property {name!r} not present in {self.name!r}")

    def get(self, *names, only_real_particles=True):
        """The tensor(s) of the named properties (one tensor for one name)."""
        if not names:
            return None
        for name in names:
            self._check_property(name)
        stale = [n for n in dict.fromkeys(names) if n in self._engine_newer]
        if len(stale) > 1 and self._session is not None:
            # the engine's newer values of several properties: one launch
            self._session.export_many(self, stale)
        out = []
        for name in names:
            self._sync(name)
            out.append(self.properties[name])
        return out[0] if len(out) == 1 else out

    def get_carray(self, name):
        return self.get(name)

    def set(self, **props):
        """Copy values into properties (ParticleArray.set).  The values are
        copied when it returns: host-to-device copies of several properties
        are queued together and waited for once."""
        held = []   # host sources of queued copies, alive until the wait
        for name, value in props.items():
            self._check_property(name)
            t = self.properties[name]
            v = torch.as_tensor(np.asarray(value) if not isinstance(value, torch.Tensor)
                                else value, dtype=t.dtype)
            if v.dim() == 0:
                t.fill_(v.item())
            elif v.device.type == "cpu" and t.device.type == "cuda":
                # one copy, host memory straight into the property
                t.copy_(v, non_blocking=True)
                held.append(v)
            else:
                t.copy_(v)
            self._touch(name)
        if held:
            torch.cuda.current_stream(self.device).synchronize()

    def __getattr__(self, name):
        props = self.__dict__.get("properties")
        if props is not None and name in props:
            return self.get(name)
        raise AttributeError(name)

    def set_to_zero(self, names):
        for name in names:
            self._check_property(name)
            self.properties[name].zero_()
            self._touch(name)

    def copy_over_properties(self, props: dict):
        """props maps a property to the one receiving its values
        (e.g. {'x': '_x0'})."""
        for src, dst in props.items():
            self._sync(src)
            self.properties[dst].copy_(self.properties[src])
            self._touch(dst)

    def set_dirty(self, value: bool):
        self.is_dirty = bool(value)
        if value and self._session is not None:
            self._session.invalidate(self)

    def set_time(self, t):
        self.time = t

    def get_time(self):
        return self.time

    def remove_particles(self, indices):
        """Remove the particles at `indices` (host-side resize)."""
        idx = torch.as_tensor(np.asarray(indices), dtype=torch.int64)
        keep = torch.ones(self._n, dtype=torch.bool)
        keep[idx] = False
        keep = keep.to(self.device)
        for name in list(self.properties):
            self._sync(name)
            self.properties[name] = self.properties[name][keep].clone()
            self._touch(name)
        self._n = int(keep.sum().item())
        if self._session is not None:
            self._session.detach()

    def numpy(self, name):
        return self.get(name).detach().cpu().numpy()

    def get_property_arrays(self, all=False):
        """Numpy copies of the properties (all=False: the ones not starting
        with '_', plus _tmpx/_tmpy/_tmpz), and the constants
        (S/base/particle_array.pyx:634-650)."""
        if all:
            props = list(self.properties)
        else:
            props = [p for p in self.properties if not p.startswith("_")]
            props += [p for p in ("_tmpx", "_tmpy", "_tmpz") if p in self.properties]
        ret = {p: self.get(p, only_real_particles=False).detach().cpu().numpy().copy()
               for p in props}
        ret.update(self.constants)
        return ret


def get_particle_array(cl_precision="double", device=None, **props):
    """ParticleArray with the reference's default properties
    (S/base/particle_array.pyx:1400-1490): x y z u v w m h p e rho cs _tmpx
    _tmpy _tmpz, plus idx; name= and type= set the name and particle type;
    non-array keyword values become constants."""
    name = props.pop("name", "")
    ptype = props.pop("type", ParticleType.Fluid)
    if ptype not in (ParticleType.Fluid, ParticleType.Solid, ParticleType.Probe,
                     ParticleType.Boundary, ParticleType.DummyFluid):
        raise AssertionError("Type not understood!")
    prop_dict = {}
    constants = {}
    n = 0
    for pname, value in props.items():
        if isinstance(value, (np.ndarray, torch.Tensor, list, tuple)):
            n = len(value)
            kind = "long" if pname in ("idx", "tag") else "double"
            prop_dict[pname] = {"data": value, "type": kind}
        else:
            constants[pname] = value
    for pname, default in DEFAULT_PROPS.items():
        if pname not in prop_dict:
            prop_dict[pname] = {"name": pname, "type": "double", "default": default}
    if "idx" not in prop_dict and n:
        prop_dict["idx"] = {"data": np.arange(n), "type": "long"}
    # data-bearing properties first, so the array length is known
    ordered = dict(sorted(prop_dict.items(), key=lambda kv: kv[1].get("data") is None))
    pa = ParticleArray(name=name, particle_type=ptype, cl_precision=cl_precision,
                       device=device, **ordered)
    pa.constants.update(constants)
    return pa
