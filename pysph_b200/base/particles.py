"""Particles: the collection of particle arrays of a simulation and its
binding to the CUDA engine (S/base/particles.py:35-227).

The reference keeps a CellManager and an NNPSManager and rebuilds them in
update().  Here the cell binning and the neighbour search run inside the
engine (pysph_b200.engine), so update() only records that positions may have
changed; the next calc or integrator stage re-imports what changed and
rebins on the GPU.  The engine lives in a Session, created on first use by
SPHCalc / the integrators with the kernel's dimension.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _native as nat
from ..engine import Engine, Scheme, SceneParams
from .particle_array import ParticleArray
from .particle_types import ParticleType

SPHNeighborLocator = 0   # NeighborLocatorType (S/base/nnps.pyx:40-45)

# properties the engine holds
MASTER = ("x", "y", "z", "u", "v", "w", "m", "h", "_x0", "_y0", "_z0", "_u0",
          "_v0", "_w0")
DERIVED = ("rho", "p", "cs", "_a_u_1", "_a_v_1", "_a_w_1", "dt_fac")
IMPORTABLE = MASTER + ("rho", "p", "cs")


class NeighborLocatorType:
    SPHNeighborLocator = 0
    NSquareNeighborLocator = 1


class Session:
    """One engine scene holding the arrays of a Particles collection."""

    def __init__(self, particles: "Particles", dim: int, precision: str,
                 scheme: Scheme | None = None, params: SceneParams | None = None,
                 lanes: int = 1, pair_block: int = 128, kernel: int = nat.KERNEL_CUBIC):
        self.particles = particles
        self.dim = dim
        self.precision = precision
        self.kernel = kernel
        arrays = particles.arrays
        A = len(arrays)
        if scheme is None:
            allv = list(range(A))
            scheme = Scheme(rho_src={a: allv for a in allv}, mom_src={a: allv for a in allv},
                            tait_on=tuple(allv), step_on=())
        self.scheme = scheme
        self.params = params or SceneParams()
        specs = []
        for pa in arrays:
            d = {}
            for name in ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs"):
                if pa.has_array(name):
                    pa._sync(name)
                    d[name] = pa.properties[name]
            d["tag"] = pa.properties["tag"]
            specs.append(d)
        opts = dict(lanes=lanes, pair_block=pair_block)
        opts.update(particles.engine_options)
        self.engine = Engine([(specs, self.params)], scheme, dim=dim,
                             precision=precision, device=arrays[0].device,
                             variable_h=particles.variable_h, kernel=kernel, **opts)
        self.valid = {}
        for a, pa in enumerate(arrays):
            for name in IMPORTABLE:
                self.valid[(a, name)] = pa.has_array(name) or name in ("x", "y", "z", "u", "v", "w", "m", "h")
            self.valid[(a, "tag")] = True
            pa._session = self
        self.need_bin = False
        self.positions_version = self._pos_versions()

    # ------------------------------------------------------------- state
    def index(self, pa: ParticleArray) -> int:
        for a, q in enumerate(self.particles.arrays):
            if q is pa:
                return a
        raise ValueError(f"array {pa.name!r} is not part of this Particles")

    def _pos_versions(self):
        return [tuple(pa.version(c) for c in ("x", "y", "z", "h", "m", "tag"))
                for pa in self.particles.arrays]

    def user_changed(self, pa, name):
        a = self.index(pa)
        if (a, name) in self.valid:
            self.valid[(a, name)] = False
        if name in ("x", "y", "z"):
            self.need_bin = True

    def invalidate(self, pa=None):
        """Positions were edited in place: re-import them and rebin."""
        arrays = [pa] if pa is not None else self.particles.arrays
        for q in arrays:
            a = self.index(q)
            for name in ("x", "y", "z", "u", "v", "w", "m", "tag"):
                self.valid[(a, name)] = False
        self.need_bin = True

    def detach(self):
        """Drop the engine (e.g. after particles were removed)."""
        for pa in self.particles.arrays:
            for name in list(pa._engine_newer):
                self.export_to_array(pa, name)
            pa._session = None
        self.particles._session = None

    # ------------------------------------------------------------ moving data
    def export_to_array(self, pa, name):
        a = self.index(pa)
        if name not in pa.properties:
            pa.add_property({"name": name})
        self.engine.exchange_out(a, name, out=pa.properties[name])
        pa._engine_newer.discard(name)

    def export_many(self, pa, names):
        """export_to_array of several properties in one launch (FP64,
        contiguous properties; the others one by one)."""
        a = self.index(pa)
        batch = []
        for name in names:
            if name not in pa.properties:
                pa.add_property({"name": name})
            t = pa.properties[name]
            if t.dtype == torch.float64 and t.is_contiguous():
                batch.append(name)
            else:
                self.export_to_array(pa, name)
        self.engine.exchange_out_many(a, batch, [pa.properties[n] for n in batch])
        for name in batch:
            pa._engine_newer.discard(name)

    def mark_engine_newer(self, a, names):
        pa = self.particles.arrays[a]
        for n in names:
            if n not in pa.properties:
                pa.add_property({"name": n})
            self.valid[(a, n)] = True
            pa._engine_newer.add(n)

    def ensure(self, reads, step_decides=False, defer=None):
        """Import every (array, property) in reads the engine does not hold,
        then rebin if any position changed.  step_decides: an engine step
        with its own rebin decision follows at once (the fused integrators),
        so with list reuse and nothing else to import after a rebin the
        decision is left to that step, which measures the host-written
        positions first.  defer: a list that receives the (array, name,
        tensor) imports of positions and velocities that the step is to
        launch itself (Engine.step_graphed), when nothing here needs them
        first; the rest are imported at once."""
        eng = self.engine
        if self._pos_versions() != self.positions_version:
            self.need_bin = True
        for a, pa in enumerate(self.particles.arrays):
            for name in ("x", "y", "z", "m", "h"):
                if (a, name) in self.valid and not self.valid[(a, name)]:
                    reads = set(reads) | {(a, name)}
            if self.valid.get((a, "tag"), True) is False:
                eng.exchange_tag(a, pa.properties["tag"], 0)
                self.valid[(a, "tag")] = True
        masters = [(a, n) for a, n in reads if n in MASTER]
        derived = [(a, n) for a, n in reads if n not in MASTER]
        if derived:
            defer = None
        for a, name in masters:
            self._import(a, name, defer)
        if self.need_bin and step_decides and eng.step_lists and not derived:
            # the step's first bin refreshes the records and decides; every
            # derived field the step reads it computes itself
            eng.invalidate_box()
            self.need_bin = False
            self.positions_version = self._pos_versions()
            for pa in self.particles.arrays:
                pa.is_dirty = False
        if self.need_bin:
            if defer:
                # the rebin reads them
                for a, name, t in defer:
                    eng.exchange_in(a, name, t)
                defer.clear()
            self.bin()
        for a, name in derived:
            self._import(a, name)

    def _import(self, a, name, defer=None):
        if self.dim == 2 and name in ("z", "w", "_z0", "_w0"):
            return
        if self.valid.get((a, name), False):
            return
        pa = self.particles.arrays[a]
        if not pa.has_array(name):
            pa.add_property({"name": name})
        if defer is not None and name in ("x", "y", "z", "u", "v", "w"):
            defer.append((a, name, pa.properties[name]))
        else:
            self.engine.exchange_in(a, name, pa.properties[name])
        self.valid[(a, name)] = True
        if name in ("x", "y", "z"):
            self.need_bin = True

    def bin(self):
        """Rebin after positions changed on the host; derived fields the
        user has not read yet are copied out first because a rebin reorders
        the particles under them.  With neighbour lists kept across steps the
        device decides: it measures every particle's displacement from its
        position at the last rebin and rebins only when some particle moved
        half the list skin (or the lists were withdrawn, e.g. by new masses),
        so host-driven steps that move the particles a little keep the lists
        and cells, which still cover every pair."""
        for a, pa in enumerate(self.particles.arrays):
            for name in DERIVED:
                if name in pa._engine_newer:
                    self.export_to_array(pa, name)
        self.engine.invalidate_box()
        if self.engine.step_lists:
            self.engine.bin(nat.BIN_IF_NEEDED | nat.BIN_MOVE_INITIAL)
        else:
            self.engine.bin(nat.BIN_MOVE_INITIAL)
        for a in range(len(self.particles.arrays)):
            for name in DERIVED:
                self.valid[(a, name)] = False
        self.need_bin = False
        self.positions_version = self._pos_versions()
        for pa in self.particles.arrays:
            pa.is_dirty = False

    def check(self):
        self.engine.check_status()


class Locator:
    """Neighbour lists of a (source, dest) pair: FixedDestNbrParticleLocator
    (S/base/nnps.pyx:385-686), computed by the engine with the reference's
    predicate r^2 < (radius_scale h_dest)^2; self last when source is dest.
    With Particles(variable_h=True) the lists are VarHNbrParticleLocator's
    symmetric sets (S/base/nnps.pyx:691-786), r^2 < (radius_scale h_dest)^2
    or r^2 < (radius_scale h_source)^2, in ascending source index with self
    last (the reference lists the same particles in its cell order)."""

    def __init__(self, particles, source, dest, radius_scale):
        self.particles = particles
        self.source = source
        self.dest = dest
        self.radius_scale = radius_scale
        self._cache = None
        self._version = None

    def _lists(self):
        p = self.particles
        s = p.session(dim=p._default_dim())
        s.ensure([])
        key = (id(s), tuple(s.positions_version))
        if self._cache is None or self._version != key:
            if self.radius_scale != s.engine.params[0].radius_scale:
                raise NotImplementedError("radius_scale other than the kernel's support")
            d = s.index(self.dest)
            a = s.index(self.source)
            di, _, sj = s.engine.neighbors(d, 1 << a)
            n = self.dest.get_number_of_particles()
            off = np.zeros(n + 1, np.int64)
            np.add.at(off, di + 1, 1)
            off = np.cumsum(off)
            self._cache = (off, sj)
            self._version = key
        return self._cache

    def py_get_nearest_particles(self, i, exclude_self=False):
        off, idx = self._lists()
        nb = list(idx[off[i]:off[i + 1]])
        if self.source is self.dest and i in nb:
            nb.remove(i)
            if not exclude_self:
                nb.append(i)
        return np.asarray(nb, dtype=np.int64)


class NNPSManager:
    """Hands out neighbour locators (S/base/nnps.pyx:791-932)."""

    def __init__(self, particles):
        self.particles = particles
        self._locators = {}

    def get_neighbor_particle_locator(self, src, dst, radius_scale=2.0):
        key = (id(src), id(dst), radius_scale)
        if key not in self._locators:
            self._locators[key] = Locator(self.particles, src, dst, radius_scale)
        return self._locators[key]

    def py_update(self):
        return 0


class Particles:
    """A collection of particle arrays (S/base/particles.py:35-227).

    precision: 'fp64' (default: the reference's arithmetic) or 'fp32c' (FP32
    pair sums with Kahan compensation, FP64 state); arrays created with
    cl_precision='single' select 'fp32c' by default."""

    def __init__(self, arrays=(), in_parallel=False, variable_h=False,
                 load_balancing=True, locator_type=SPHNeighborLocator,
                 periodic_domain=None, min_cell_size=-1, max_cell_size=0,
                 max_radius_scale=2, update_particles=True, precision=None):
        arrays = list(arrays)
        assert len(arrays) > 0, "Particles must be given some arrays!"
        prec = arrays[0].cl_precision
        for arr in arrays[1:]:
            assert arr.cl_precision == prec, "All arrays must have the same cl_precision"
        if in_parallel:
            raise NotImplementedError("MPI-distributed particles are not part of this build")
        if periodic_domain is not None:
            raise NotImplementedError("periodic domains are not part of this build")
        devs = {str(a.device) for a in arrays}
        if len(devs) != 1:
            raise ValueError("all arrays must live on one device")
        self.arrays = arrays
        self.in_parallel = False
        # symmetric neighbour sets for varying smoothing lengths
        # (VarHNbrParticleLocator, S/base/nnps.pyx:691-786)
        self.variable_h = bool(variable_h)
        self.max_radius_scale = max_radius_scale
        self.precision = precision or ("fp32c" if prec == "single" else "fp64")
        self.kernel = None
        # launch shape of the engine behind these arrays (this build's own
        # option, no reference counterpart): Engine keyword arguments such
        # as pairs, stencil, lanes, pair_block, skin_margin, e.g. from
        # pysph_b200.autotune.autotune
        self.engine_options: dict = {}
        self.correction_manager = None
        self.misc_prop_update_functions = []
        self.nnps_manager = NNPSManager(self)
        self._session: Session | None = None
        self._dim = None
        self.update()

    def _default_dim(self):
        if self._dim is not None:
            return self._dim
        if self.kernel is not None:
            return self.kernel.dim
        return 3 if any(bool(torch.any(a.properties["z"] != 0)) for a in self.arrays
                        if a.get_number_of_particles()) else 2

    def session(self, dim=None, scheme=None, params=None, lanes=1, pair_block=128,
                kernel=None):
        """The engine session; (re)built when the dimension, the kernel type
        or, when given, the scheme / parameters change."""
        dim = dim or self._default_dim()
        s = self._session
        if kernel is None:
            kernel = (s.kernel if s is not None else
                      self.kernel.get_type() if self.kernel is not None else nat.KERNEL_CUBIC)
        rebuild = (s is None or s.dim != dim or s.precision != self.precision
                   or s.kernel != kernel
                   or (scheme is not None and s.scheme != scheme)
                   or (params is not None and s.params != params)
                   or any(s.engine.sizes[0, a] != pa.get_number_of_particles()
                          for a, pa in enumerate(self.arrays)))
        if not rebuild:
            h_changed = any(not s.valid.get((a, "h"), True) for a in range(len(self.arrays)))
            rebuild = h_changed
        if rebuild:
            if s is not None:
                s.detach()
            self._session = Session(self, dim, self.precision, scheme, params, lanes,
                                    pair_block, kernel)
            self._dim = dim
        return self._session

    def update(self, cache_neighbors=False):
        """Particles.update (S/base/particles.py:184-215).  Positions the
        engine moved are rebinned by the engine itself at the start of every
        stage, and positions set through ParticleArray.set are tracked; only
        in-place tensor edits need ParticleArray.set_dirty(True)."""
        for f in self.misc_prop_update_functions:
            f.eval()

    def get_named_particle_array(self, name):
        for a in self.arrays:
            if a.name == name:
                return a
        return None

    def barrier(self):
        pass

    def update_remote_particle_properties(self, update_list):
        pass
