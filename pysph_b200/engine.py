"""Engine: the device state of a batch of independent scenes and the calls
that advance it through libsphb.so.

A scene is a list of particle arrays (e.g. [fluid, wall]) with its own
physical parameters; every scene of an engine has the same array roles, and
the scheme (which arrays are SPHRho / Tait / MomentumEquation destinations,
which are their sources, which are integrated) is shared.  All scenes live
in one SoA set ("engine order"), sorted by cell inside each (scene, array)
segment, and every stage is one launch over all scenes.

torch provides the device memory and the stream; all arithmetic runs in
the sm_100a kernels of libsphb.so.
"""
from __future__ import annotations

import contextlib
import ctypes
import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as nat

ELEM_TILE = 256
SKIN_MARGIN = 0.15
MASTER = ("x", "y", "z", "u", "v", "w", "x0", "y0", "z0", "u0", "v0", "w0",
          "m", "h")
USER_PROPS = ("x", "y", "z", "u", "v", "w", "m", "h")


@dataclass
class SceneParams:
    """Per-scene constants of the pinned scheme (defaults: the reference's
    own defaults for TaitEquation and MomentumEquation)."""
    c0: float = 1.0
    rho0: float = 1000.0
    gamma: float = 7.0
    alpha: float = 1.0
    beta: float = 1.0
    eta: float = 0.1
    gravity: tuple = (0.0, 0.0, 0.0)
    dt: float = 1e-4
    cfl: float = 0.0            # > 0: ViscousAndForceBasedTimeStep
    dt_initial: float = 1e-4     # solver.dt, used by the CFL rule at step 1
    radius_scale: float = 2.0    # kernel support / h (set from the engine's kernel)
    cfl_force: bool = True       # CFL rule with the force criterion too

    @staticmethod
    def from_dict(d: dict) -> "SceneParams":
        keys = SceneParams.__dataclass_fields__.keys()
        return SceneParams(**{k: v for k, v in d.items() if k in keys})


@dataclass
class Scheme:
    """Which array indices take part in which operation.

    Summation density: rho_src (SPHRho).  Continuity equation: rate_src
    (SPHDensityRate, rho integrated on its dests), optionally with
    XSPHCorrection (xsph_src, xsph_eps) added to the position rate.  hks:
    every pair function averages its kernel over h_a and h_b (the
    functions' hks option) instead of evaluating it at (h_a + h_b) / 2."""
    rho_src: dict = field(default_factory=dict)   # dest -> [sources]
    mom_src: dict = field(default_factory=dict)   # dest -> [sources]
    tait_on: tuple = ()
    step_on: tuple = ()
    rate_src: dict = field(default_factory=dict)  # dest -> [sources]
    xsph_src: dict = field(default_factory=dict)  # dest -> [sources]
    xsph_eps: float = 0.5
    hks: bool = False

    @property
    def continuity(self) -> bool:
        return any(self.rate_src.values())

    def masks2(self):
        """Continuity and XSPH source masks per dest array."""
        rate = [0] * nat.MAX_ARRAYS
        xs = [0] * nat.MAX_ARRAYS
        for d, s in self.rate_src.items():
            rate[d] = sum(1 << a for a in s)
        for d, s in self.xsph_src.items():
            xs[d] = sum(1 << a for a in s)
        return rate, xs

    def masks(self):
        rho = [0] * nat.MAX_ARRAYS
        mom = [0] * nat.MAX_ARRAYS
        for d, s in self.rho_src.items():
            rho[d] = sum(1 << a for a in s)
        for d, s in self.mom_src.items():
            mom[d] = sum(1 << a for a in s)
        tait = sum(1 << a for a in self.tait_on)
        step = sum(1 << a for a in self.step_on)
        return rho, mom, tait, step

    @property
    def rho_dests(self) -> int:
        return sum(1 << d for d, s in self.rho_src.items() if s)

    @property
    def mom_dests(self) -> int:
        return sum(1 << d for d, s in self.mom_src.items() if s)

    @property
    def pair_dests(self) -> int:
        """Arrays that are the dest of any pair function."""
        m = 0
        for srcs in (self.rho_src, self.mom_src, self.rate_src, self.xsph_src):
            m |= sum(1 << d for d, s in srcs.items() if s)
        return m


def fluid_scheme(num_arrays: int = 1) -> Scheme:
    """Array 0 is the fluid; arrays 1.. are fixed walls.  SPHRho and Tait on
    every array from every array; MomentumEquation on the fluid from every
    array; only the fluid is integrated."""
    all_ = list(range(num_arrays))
    return Scheme(rho_src={a: all_ for a in all_}, mom_src={0: all_},
                  tait_on=tuple(all_), step_on=(0,))


def continuity_scheme(num_arrays: int = 1, xsph_eps: float = 0.5) -> Scheme:
    """The reference's dam-break scheme (examples/dam-break/dam_break.py:
    184-241, FluidSolver S/solver/fluid_solver.py:55-87): Tait on every
    array; SPHDensityRate on every array from every array (rho integrated
    on all of them, walls included); MomentumEquation on the fluid (array
    0) from every array; the fluid's positions stepped with XSPHCorrection
    from the fluid (eps = xsph_eps; 0 leaves XSPH out)."""
    all_ = list(range(num_arrays))
    return Scheme(mom_src={0: all_}, tait_on=tuple(all_), step_on=(0,),
                  rate_src={a: all_ for a in all_},
                  xsph_src={0: [0]} if xsph_eps else {}, xsph_eps=xsph_eps)


class Engine:
    """Batch of scenes on one GPU.

    scenes: list of (arrays, params) where arrays is a list of dicts of
    numpy/torch FP64 properties (x, y, z, u, v, w, m, h, rho, p, cs, tag)
    and params a SceneParams or dict."""

    def __init__(self, scenes, scheme: Scheme, dim: int = 2,
                 precision: str = "fp32c", stencil: int = 1, lanes: int = 1,
                 pair_block: int = 128, cell_capacity: int | None = None,
                 grid_growth: float = 2.0, device=None, use_lists: bool = True,
                 step_lists: bool = True, skin_margin: float | None = None,
                 list_batch: int = 4, variable_h: bool = False,
                 kernel: int = nat.KERNEL_CUBIC, fuse_stage: bool = True,
                 pairs: str = "lists"):
        if dim not in (2, 3):
            raise ValueError("dim must be 2 or 3")
        if precision not in ("fp64", "fp32c"):
            raise ValueError("precision must be 'fp64' or 'fp32c'")
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise RuntimeError("the engine runs on CUDA devices only")
        if self.device.index is None:
            # an explicit index: every launch looks up the device's current
            # stream, which for a bare "cuda" device costs a query of the
            # current device each time
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.L = nat.lib()
        self.dim = dim
        self.precision = precision
        self.f32 = precision == "fp32c"
        self.scheme = scheme
        self.S = len(scenes)
        self.A = len(scenes[0][0])
        if self.S < 1 or not 1 <= self.A <= nat.MAX_ARRAYS:
            raise ValueError("need >= 1 scene and 1..4 arrays per scene")
        # smoothing kernel (KernelBase.get_type ids); the quintic spline and
        # the Wendland quintic are 2D only, as in the reference
        if kernel not in nat.KERNEL_RADIUS:
            raise ValueError("kernel must be 1 (cubic), 3 (quintic) or 4 (Wendland quintic)")
        if kernel != nat.KERNEL_CUBIC and dim != 2:
            raise NotImplementedError("the quintic and Wendland kernels are 2D only")
        self.kernel = kernel
        # how the pair passes find neighbours: "lists" (recorded by the
        # density pass after a rebin, read back while the skin holds) or
        # "tiled" (every pass searches the cells from shared memory, where
        # each block stages its dests' stencil rows; 2D FP32C summation
        # density with one h per pair, one thread per dest)
        if pairs not in ("lists", "tiled"):
            raise ValueError("pairs must be 'lists' or 'tiled'")
        if pairs == "tiled":
            if dim != 2 or precision != "fp32c":
                raise NotImplementedError("tiled pair passes are 2D FP32C")
            if scheme.continuity or scheme.hks or variable_h:
                raise NotImplementedError("tiled pair passes: summation density, one h per pair")
            if lanes != 1:
                raise ValueError("tiled pair passes run one thread per dest (lanes=1)")
        self.pairs = pairs
        params = [p if isinstance(p, SceneParams) else SceneParams.from_dict(p)
                  for _, p in scenes]
        # the neighbour radius is the kernel's support
        self.params = [dataclasses.replace(p, radius_scale=nat.KERNEL_RADIUS[kernel])
                       for p in params]
        sizes = np.zeros((self.S, self.A), np.int64)
        for s, (arrays, _) in enumerate(scenes):
            if len(arrays) != self.A:
                raise ValueError("every scene needs the same number of arrays")
            for a, arr in enumerate(arrays):
                sizes[s, a] = len(arr["x"])
        self.sizes = sizes
        seg = np.zeros(self.S * self.A + 1, np.int64)
        seg[1:] = np.cumsum(sizes.ravel())
        if seg[-1] >= 2 ** 31 - 1:
            raise ValueError("too many particles for int32 indexing")
        self.N = int(seg[-1])
        self.seg_offset_host = seg.astype(np.int32)
        # user-side layout: per array, scenes concatenated
        self.user_offset_host = [np.concatenate([[0], np.cumsum(sizes[:, a])[:-1]]).astype(np.int32)
                                 for a in range(self.A)]
        self.user_n = [int(sizes[:, a].sum()) for a in range(self.A)]
        self._stencil = stencil
        self.use_lists = use_lists
        # list reuse across stages and steps: cells larger than the support
        # by skin_margin leave room for a skin, and the device rebins only
        # once some particle has moved half the skin; off, every stage
        # rebins and the cell size is exactly the reference's
        self.step_lists = bool(use_lists and step_lists)
        if skin_margin is None:
            skin_margin = SKIN_MARGIN
        if self.step_lists and not 0.0 < skin_margin <= 1.0:
            raise ValueError("skin_margin must be in (0, 1]")
        self.skin_margin = float(skin_margin) if self.step_lists else 0.0
        # symmetric neighbour sets r < radius_scale max(h_a, h_b)
        # (VarHNbrParticleLocator) instead of r < radius_scale h_a
        self.variable_h = bool(variable_h)
        # run the integrator stage in the force pass's epilogue (FP32C)
        self.fuse_stage = bool(fuse_stage)
        self.force_mode = 0       # 0 MomentumEquation, 1 SPHPressureGradient
        self.tait_only_mask = 0    # Tait dests that are not SPHRho dests
        # step_graphed: on/off, launch states seen once, their captured steps
        self.graphs = True
        self._graph_seen: set = set()
        self._graphs: dict = {}
        self._host_scene_tables(scenes)
        if cell_capacity is None:
            cell_capacity = self._estimate_capacity(grid_growth)
        self.cell_capacity = int(cell_capacity)
        if list_batch not in (2, 4):
            raise ValueError("list_batch must be 2 or 4")
        self.list_batch = list_batch
        self._alloc(lanes, pair_block)
        self._upload(scenes)

    # ------------------------------------------------------------------ setup
    def _host_scene_tables(self, scenes):
        dim = self.dim
        step = set(self.scheme.step_on)
        sc = (nat.Scene * self.S)()
        self._extent = []
        self._h_cap = []     # largest h the cells of each scene cover
        for s, (arrays, _) in enumerate(scenes):
            p = self.params[s]
            hs = [np.asarray(_np(arr["h"]), np.float64) for arr in arrays]
            max_h = max(float(h.max()) if len(h) else 0.0 for h in hs)
            if max_h <= 0:
                max_h = 0.5  # the reference's "cell size 0 -> 1"
            cs = p.radius_scale * max_h * (1.0 + self.skin_margin) / self._stencil
            step_h = [h for a, h in enumerate(hs) if a in step and len(h)]
            h_min = min(float(h.min()) for h in step_h) if step_h else max_h
            lo = np.full(3, np.inf)
            hi = np.full(3, -np.inf)
            alo = np.full(3, np.inf)
            ahi = np.full(3, -np.inf)
            for a, arr in enumerate(arrays):
                if len(arr["x"]) == 0:
                    continue
                pts = [np.asarray(_np(arr[c]), np.float64) for c in "xyz"[:dim]]
                for d in range(dim):
                    alo[d] = min(alo[d], pts[d].min())
                    ahi[d] = max(ahi[d], pts[d].max())
                    if a not in step:
                        lo[d] = min(lo[d], pts[d].min())
                        hi[d] = max(hi[d], pts[d].max())
            self._extent.append((alo, ahi, cs))
            self._h_cap.append(max_h)
            t = sc[s]
            t.cell_size = cs
            # list radius (support + skin)(1 + 1e-5) must stay within R cells
            t.skin_max = (p.radius_scale * max_h * (self.skin_margin - 1e-4)
                          if self.skin_margin else 0.0)
            t.xsph_eps = self.scheme.xsph_eps
            t.variable_h = int(self.variable_h)
            t.hks = int(bool(self.scheme.hks))
            t.radius_scale = p.radius_scale
            t.h_min = h_min
            t.c0, t.rho0, t.gamma = p.c0, p.rho0, p.gamma
            t.B = p.c0 * p.c0 * p.rho0 / p.gamma
            t.alpha, t.beta, t.eta = p.alpha, p.beta, p.eta
            for d in range(3):
                t.g[d] = float(p.gravity[d]) if d < len(p.gravity) else 0.0
                t.static_lo[d] = lo[d]
                t.static_hi[d] = hi[d]
            t.cfl = p.cfl
            t.dt_initial = p.dt_initial
            t.use_cfl = (1 if p.cfl_force else 2) if p.cfl > 0 else 0
            nonempty = [h for h in hs if len(h)]
            t.uniform_h = int(bool(nonempty) and
                              min(float(h.min()) for h in nonempty) ==
                              max(float(h.max()) for h in nonempty))
        self._scene_host = sc

    def _estimate_capacity(self, growth: float) -> int:
        R = self._stencil
        total = 0
        for alo, ahi, cs in self._extent:
            n = 1
            for d in range(self.dim):
                span = (ahi[d] - alo[d]) if np.isfinite(ahi[d]) else 0.0
                cells = math.floor(span / cs) + 2
                n *= int(math.ceil(cells * growth)) + 2 * R + 2
            total += self.A * n
        return max(total, 1024)

    def _alloc(self, lanes, pair_block):
        dev, N, dim = self.device, self.N, self.dim
        f64 = dict(dtype=torch.float64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.seg_offset = torch.from_numpy(self.seg_offset_host).to(dev)
        self.user_offset = [torch.from_numpy(u).to(dev) for u in self.user_offset_host]
        self.scene_dev = _struct_to_device(self._scene_host, dev)
        st = (nat.SceneState * self.S)()
        for s in range(self.S):
            st[s].dt = self.params[s].dt
        self.sstate_dev = _struct_to_device(st, dev)
        # buffers
        self.bufs = []
        for _ in range(2):
            b = {}
            for name in MASTER:
                if dim == 2 and name in ("z", "w", "z0", "w0"):
                    b[name] = None
                else:
                    b[name] = torch.zeros(N, **f64)
            b["idx"] = torch.zeros(N, **i32)
            b["tag"] = torch.zeros(N, **i32)
            # the continuity equation integrates the density
            cont = self.scheme.continuity
            b["rho"] = torch.zeros(N, **f64) if cont else None
            b["rho0"] = torch.zeros(N, **f64) if cont else None
            # RK4's running sums, allocated by the first RK4 step
            for name in ("kx", "ky", "kz", "ku", "kv", "kw", "krho"):
                b[name] = None
            self.bufs.append(b)
        f = {}
        if self.f32:
            f32 = dict(dtype=torch.float32, device=dev)
            f["rho"] = f["p"] = f["cs"] = None
            f["au"] = torch.zeros(N, **f32)
            f["av"] = torch.zeros(N, **f32)
            f["aw"] = torch.zeros(N, **f32) if dim == 3 else None
            f["dt_fac"] = torch.zeros(N, **f32)
            f["geo"] = torch.zeros(N, 4, **f32)
            f["mass"] = torch.zeros(N, **f32) if dim == 3 else None
            f["vel"] = torch.zeros(N, 2 if dim == 2 else 4, **f32)
            f["thermo"] = torch.zeros(N, 4, **f32)
            # the second copy of the records: the force pass that runs the
            # integrator stage writes the moved particles' records there
            f["geo_next"] = torch.zeros_like(f["geo"])
            f["vel_next"] = torch.zeros_like(f["vel"])
        else:
            for n in ("rho", "p", "cs", "au", "av", "dt_fac"):
                f[n] = torch.zeros(N, **f64)
            f["aw"] = torch.zeros(N, **f64) if dim == 3 else None
            f["geo"] = f["mass"] = f["vel"] = f["thermo"] = None
            f["geo_next"] = f["vel_next"] = None
        f["cell"] = torch.zeros(N, **i32)
        # outputs of SPHDensityRate (_a_rho_1) and XSPHCorrection (velocity):
        # the continuity scheme's, and any single calc's on this engine
        ft = dict(dtype=torch.float32 if self.f32 else torch.float64, device=dev)
        f["drho"] = torch.zeros(N, **ft)
        for c in ("xu", "xv", "xw"):
            f[c] = torch.zeros(N, **ft) if (c != "xw" or dim == 3) else None
        # per-stage neighbour lists (density pass writes, force pass reads)
        idx_bits = 26 if dim == 2 else 23
        self.list_cap = (64 if dim == 2 else 160) if (self.use_lists and N < 2 ** idx_bits) else 0
        if self.list_cap and self.pairs == "tiled":
            # per-stage lists: the entries the density pass accepted (within
            # the support, no skin), for the force pass of the same stage
            self.list_cap = 48
        elif self.list_cap:
            # capacity for the skin and the kernel's support (3h for the
            # quintic): entries grow as (radius (1 + margin))^dim; a lane
            # whose list overflows searches its cells instead
            grow = ((1.0 + self.skin_margin) * nat.KERNEL_RADIUS[self.kernel] / 2.0) ** dim
            self.list_cap = int(math.ceil(self.list_cap * grow / 8.0)) * 8
        if self.list_cap:
            f["nbr"] = torch.zeros(self.list_cap * N, **i32)
            f["nbr_cnt"] = torch.zeros(8 * N, **i32)
        else:
            f["nbr"] = f["nbr_cnt"] = None
        # binned positions, for the rebin decision of the list reuse
        f["anchor"] = (torch.zeros(N, 2 if dim == 2 else 4, dtype=torch.float32, device=dev)
                       if self.step_lists else None)
        self.fields = f
        # scratch
        cfg = self._config(lanes, pair_block)
        offs = (ctypes.c_size_t * 9)()
        total = ctypes.c_size_t()
        nat.check(self.L.sphb_workspace_layout(ctypes.byref(cfg), offs,
                                               ctypes.byref(total)),
                  "sphb_workspace_layout")
        self.work_buf = torch.zeros(total.value, dtype=torch.uint8, device=dev)
        self.work_offsets = list(offs)
        self.tiles = self._make_tiles(ELEM_TILE)
        self.set_launch(lanes, pair_block)

    def _config(self, lanes, pair_block):
        cfg = nat.Config()
        cfg.dim = self.dim
        cfg.precision = nat.FP32C if self.f32 else nat.FP64
        cfg.num_scenes = self.S
        cfg.num_arrays = self.A
        cfg.stencil = self._stencil
        cfg.lanes = lanes
        cfg.pair_block = pair_block
        cfg.list_batch = getattr(self, "list_batch", 4)
        cfg.kernel = self.kernel
        cfg.pair_mode = nat.PAIRS_TILED if getattr(self, "pairs", "lists") == "tiled" else 0
        cfg.num_particles = self.N
        cfg.cell_capacity = self.cell_capacity
        rho, mom, tait, step = self.scheme.masks()
        for a in range(nat.MAX_ARRAYS):
            cfg.rho_src[a] = rho[a]
            cfg.mom_src[a] = mom[a]
        cfg.tait_on = tait
        cfg.step_on = step
        rate, xs = self.scheme.masks2()
        for a in range(nat.MAX_ARRAYS):
            cfg.rate_src[a] = rate[a]
            cfg.xsph_src[a] = xs[a]
        return cfg

    def _make_tiles(self, tile_size):
        n = ctypes.c_int32()
        seg = self.seg_offset_host
        nseg = len(seg) - 1
        nat.check(self.L.sphb_make_tiles(seg.ctypes.data, nseg, tile_size, None,
                                         ctypes.byref(n)), "sphb_make_tiles")
        arr = (nat.Tile * max(n.value, 1))()
        nat.check(self.L.sphb_make_tiles(seg.ctypes.data, nseg, tile_size,
                                         ctypes.addressof(arr), ctypes.byref(n)),
                  "sphb_make_tiles")
        return _struct_to_device(arr, self.device), n.value

    def set_launch(self, lanes: int, pair_block: int, list_batch: int | None = None):
        """Pair-kernel launch shape: lanes per dest particle, block size and
        how many list entries the FP32C force pass loads ahead (2 or 4)."""
        if lanes not in (1, 2, 4, 8) or pair_block % 32 or not 32 <= pair_block <= 256:
            raise ValueError("bad pair-kernel launch shape")
        if self.pairs == "tiled" and lanes != 1:
            raise ValueError("tiled pair passes run one thread per dest (lanes=1)")
        if list_batch is not None:
            if list_batch not in (2, 4):
                raise ValueError("list_batch must be 2 or 4")
            self.list_batch = list_batch
        self.lanes, self.pair_block = lanes, pair_block
        self.pair_tiles = self._make_tiles(pair_block // lanes)
        self._build_desc()
        # the lists are laid out per lane: record them again
        self.invalidate_lists()

    def _build_desc(self):
        d = nat.EngineDesc()
        d.cfg = self._config(self.lanes, self.pair_block)
        d.seg_offset = self.seg_offset.data_ptr()
        d.scene = self.scene_dev.data_ptr()
        d.sstate = self.sstate_dev.data_ptr()
        d.tiles = self.tiles[0].data_ptr()
        d.num_tiles = self.tiles[1]
        d.pair_tiles = self.pair_tiles[0].data_ptr()
        d.num_pair_tiles = self.pair_tiles[1]
        for i in range(2):
            for name in nat.BUFFER_FIELDS:
                t = self.bufs[i][name]
                setattr(d.buf[i], name, t.data_ptr() if t is not None else None)
        for name in nat.FIELD_NAMES:
            t = self.fields[name]
            setattr(d.f, name, t.data_ptr() if t is not None else None)
        d.f.list_cap = self.list_cap
        base = self.work_buf.data_ptr()
        for name, off in zip(nat.WORK_NAMES, self.work_offsets):
            setattr(d.work, name, base + off)
        self.desc = d
        self._pdesc = ctypes.byref(d)
        self.cur = getattr(self, "cur", 0)

    def _upload(self, scenes):
        """Copy the user arrays in, set identity indices, then bin."""
        self.cur = 0
        self._box_valid = False
        self.call("sphb_init_index", 0)
        user = self._user_tensors(scenes)
        for a in range(self.A):
            for name in USER_PROPS:
                if self.dim == 2 and name in ("z", "w"):
                    continue
                self._exchange_in(a, name, user[a][name])
            self.exchange_tag(a, user[a]["tag"], 0)
        self.bin(0)
        for a in range(self.A):
            for name in ("rho", "p", "cs"):
                self.exchange_in(a, name, user[a][name])

    def _user_tensors(self, scenes):
        out = []
        for a in range(self.A):
            d = {}
            for name in USER_PROPS + ("rho", "p", "cs"):
                parts = []
                for arrays, _ in scenes:
                    arr = arrays[a]
                    n = len(arr["x"])
                    v = arr.get(name)
                    if v is None:
                        v = {"m": 1.0, "h": 1.0, "rho": 1.0}.get(name, 0.0)
                    parts.append(torch.as_tensor(_np_b(v, n), dtype=torch.float64))
                d[name] = torch.cat(parts).to(self.device)
            tags = []
            for arrays, _ in scenes:
                arr = arrays[a]
                n = len(arr["x"])
                v = arr.get("tag", 0)
                tags.append(torch.as_tensor(_np_b(v, n), dtype=torch.int32))
            d["tag"] = torch.cat(tags).to(self.device)
            out.append(d)
        return out

    # ------------------------------------------------------------ low level
    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def call(self, name, *args):
        fn = getattr(self.L, name)
        if name == "sphb_step_begin":
            rc = fn(self._pdesc, self.stream)
        else:
            rc = fn(self._pdesc, *args, self.stream)
        nat.check(rc, name)

    def bin(self, flags: int = 0):
        """Rebin into the other buffer; with BIN_IF_NEEDED the device decides
        and the state stays in the current buffer either way.  After
        positions or velocities written from the host the records are
        refreshed and every displacement measured first, so the decision
        may keep the lists."""
        if not self._box_valid:
            flags |= nat.BIN_BOX
        if (flags & nat.BIN_IF_NEEDED) and getattr(self, "_host_state", False):
            self.call("sphb_refresh", self.cur)
        self._host_state = False
        self.call("sphb_bin", self.cur, flags)
        if flags & nat.BIN_IF_NEEDED:
            # the box is rebuilt only by a rebin that happens; keep asking
            # for it until a pc_stage has accumulated it again
            return
        self.cur ^= 1
        self._box_valid = False   # until a pc_stage accumulates it again

    @contextlib.contextmanager
    def masks(self, rho_src=None, mom_src=None, tait_on=None, step_on=None,
              rate_src=None, xsph_src=None):
        """Temporarily replace the scheme masks the kernels see (dest array
        -> source bitmask), for evaluating one calc at a time."""
        cfg = self.desc.cfg
        saved = (list(cfg.rho_src), list(cfg.mom_src), cfg.tait_on, cfg.step_on,
                 list(cfg.rate_src), list(cfg.xsph_src))
        try:
            for a, m in (rho_src or {}).items():
                cfg.rho_src[a] = m
            for a, m in (mom_src or {}).items():
                cfg.mom_src[a] = m
            for a, m in (rate_src or {}).items():
                cfg.rate_src[a] = m
            for a, m in (xsph_src or {}).items():
                cfg.xsph_src[a] = m
            if tait_on is not None:
                cfg.tait_on = tait_on
            if step_on is not None:
                cfg.step_on = step_on
            yield
        finally:
            for a in range(nat.MAX_ARRAYS):
                cfg.rho_src[a] = saved[0][a]
                cfg.mom_src[a] = saved[1][a]
                cfg.rate_src[a] = saved[4][a]
                cfg.xsph_src[a] = saved[5][a]
            cfg.tait_on, cfg.step_on = saved[2], saved[3]

    def update_params(self, scene=None, **kw):
        """Change scene constants (c0, rho0, gamma, alpha, beta, eta, gravity,
        cfl, dt_initial) and re-upload the scene table when they differ."""
        scenes = range(self.S) if scene is None else [scene]
        changed = False
        for s in scenes:
            p = self.params[s]
            for k, v in kw.items():
                if getattr(p, k) != v:
                    setattr(p, k, v)
                    changed = True
        if not changed:
            return
        for s in scenes:
            p = self.params[s]
            t = self._scene_host[s]
            t.c0, t.rho0, t.gamma = p.c0, p.rho0, p.gamma
            t.B = p.c0 * p.c0 * p.rho0 / p.gamma
            t.alpha, t.beta, t.eta = p.alpha, p.beta, p.eta
            for d in range(3):
                t.g[d] = float(p.gravity[d]) if d < len(p.gravity) else 0.0
            t.cfl, t.dt_initial = p.cfl, p.dt_initial
            t.use_cfl = (1 if p.cfl_force else 2) if p.cfl > 0 else 0
        self.scene_dev.copy_(_struct_to_device(self._scene_host, self.device))

    def set_hks(self, hks: bool):
        """The pair functions' hks option for the next passes (scene table
        re-uploaded when it changes)."""
        if all(t.hks == int(bool(hks)) for t in self._scene_host):
            return
        for t in self._scene_host:
            t.hks = int(bool(hks))
        self.scene_dev.copy_(_struct_to_device(self._scene_host, self.device))

    def set_xsph_eps(self, eps: float):
        """XSPHCorrection eps of every scene (scene table re-uploaded when it
        changes)."""
        if all(t.xsph_eps == eps for t in self._scene_host):
            return
        for t in self._scene_host:
            t.xsph_eps = float(eps)
        self.scene_dev.copy_(_struct_to_device(self._scene_host, self.device))

    def set_dt_async(self, dt: float):
        """dt of the next stages for every scene without the CFL rule, set by
        a kernel (no host round trip)."""
        nat.check(self.L.sphb_set_dt(self._pdesc, float(dt), self.stream), "sphb_set_dt")

    def invalidate_lists(self):
        """The neighbour lists may no longer match the state or the launch
        shape: the next device rebin decision rebins and they are recorded
        again (work.meta[2..4] cleared, in stream order)."""
        if not hasattr(self, "work_buf"):
            return
        off = self.work_offsets[nat.WORK_NAMES.index("meta")]
        self.work_buf[off + 8:off + 20].zero_()

    def rebin_now(self):
        """Rebin at once, the state staying in its buffer (a device-decided
        rebin with the lists withdrawn; a plain rebin without list reuse),
        e.g. after the host rewrote the state: every later launch sees the
        same buffers, so graphs captured around it replay."""
        if not self.step_lists:
            return self.bin(nat.BIN_MOVE_INITIAL)
        self.invalidate_lists()
        self._host_state = False
        self.bin(nat.BIN_IF_NEEDED | nat.BIN_MOVE_INITIAL)

    def invalidate_box(self):
        """Positions were changed outside the integrator: the next bin
        recomputes every scene box from all particles."""
        self._box_valid = False

    def _sync_cells(self):
        """With list reuse the cell tables are those of the last rebin; a
        device decision first rebins if any particle has since moved half
        the skin, so a cell search still finds every pair."""
        if self.step_lists:
            self.bin(nat.BIN_IF_NEEDED | nat.BIN_MOVE_INITIAL)

    def density(self, dest_mask=None, eos=True, reuse=False):
        """SPHRho (+ Tait) on the dest arrays.  reuse: with list reuse, read
        the neighbour lists when the rebin decision that just ran kept them
        (else record them with the skin), as an integrator stage does; the
        lists then hold every pair within the support plus the skin."""
        if dest_mask is None:
            dest_mask = self.scheme.rho_dests
        self._sync_cells()
        flags = nat.DENSITY_EOS if eos else 0
        if reuse and self.step_lists:
            flags |= nat.DENSITY_LIST_IF_VALID
        self.call("sphb_density", self.cur, dest_mask, flags)

    def tait(self, dest_mask=None):
        if dest_mask is None:
            dest_mask = sum(1 << a for a in self.scheme.tait_on)
        self.call("sphb_tait", self.cur, dest_mask)

    def momentum(self, dest_mask=None, gravity=True, mode=0, synced=False):
        """The force pass; synced: the cells are known to cover every pair
        (the stage's rebin decision has just run), so no decision first."""
        if dest_mask is None:
            dest_mask = (self.scheme.pair_dests if self.scheme.continuity
                         else self.scheme.mom_dests)
        if not mode & nat.FORCE_USE_LIST and not synced:
            self._sync_cells()
        self.call("sphb_momentum", self.cur, dest_mask, 1 if gravity else 0, mode)

    def pc_stage(self, stage: int):
        self.call("sphb_pc_stage", self.cur, stage)
        self._box_valid = True

    @property
    def fuses_stage(self) -> bool:
        """Whether the integrator stage runs in the force pass's epilogue
        (FP32C, with every stepped and density-rate array a force dest)."""
        if not (self.f32 and self.fuse_stage):
            return False
        dests = self.scheme.pair_dests if self.scheme.continuity else self.scheme.mom_dests
        need = sum(1 << a for a in self.scheme.step_on)
        need |= sum(1 << d for d, s in self.scheme.rate_src.items() if s)
        return need & ~dests == 0

    def _swap_records(self):
        f = self.fields
        f["geo"], f["geo_next"] = f["geo_next"], f["geo"]
        f["vel"], f["vel_next"] = f["vel_next"], f["vel"]
        for name in ("geo", "geo_next", "vel", "vel_next"):
            setattr(self.desc.f, name, f[name].data_ptr())

    def _stage(self, kind: int):
        """Integrator.eval at the current positions, then stage `kind` of
        sphb_pc_stage: fused into the force pass when the engine allows it
        (the predictor's pass then leaves the CFL maxima alone), else as its
        own pass.  A fused stage swaps the two record copies, so a captured
        graph must hold an even number of them: a PC or RK2 step does, and
        an Euler step (one stage) being captured runs its stage on its own."""
        capturing = self.device.type == "cuda" and torch.cuda.is_current_stream_capturing()
        if self.fuses_stage and not (kind == 2 and capturing):
            self.eval_stage(stage=kind)
            self._box_valid = True
        else:
            self.eval_stage()
            self.pc_stage(kind)

    def step_begin(self):
        self.call("sphb_step_begin")

    def eval_stage(self, stage: int | None = None):
        """Integrator.eval of the pinned scheme at the current positions:
        SPHRho + Tait (fused), Tait on arrays without SPHRho, then
        MomentumEquation (or SPHPressureGradient) + GravityForce.  The
        density pass records the neighbour lists the force pass reads; with
        list reuse it reads the lists the last rebin decision kept.  With
        `stage` (engines where fuses_stage) the force pass also runs that
        integrator stage and the record copies swap."""
        reuse = nat.DENSITY_LIST_IF_VALID if self.step_lists else 0
        mode = self.force_mode | (nat.FORCE_USE_LIST if self.list_cap else 0)
        if stage is not None:
            if not self.fuses_stage:
                raise ValueError("this engine runs the integrator stage on its own")
            # the CFL rule reads the step's last force pass: the earlier
            # stages' passes leave the maxima alone
            mode |= nat.FORCE_STAGE(stage) | (nat.FORCE_NO_MAXIMA if stage in (0, 4, 5, 6)
                                              else 0)
        if self.scheme.continuity:
            # TaitEquation on the integrated density, then one pair pass:
            # SPHDensityRate + MomentumEquation + XSPHCorrection; the density
            # kernel only records the lists (after a rebin)
            self.call("sphb_density", self.cur, self.scheme.pair_dests,
                      nat.DENSITY_LISTS_ONLY | reuse)
            self.tait()
            self.call("sphb_momentum", self.cur, self.scheme.pair_dests, 1, mode)
        else:
            self.call("sphb_density", self.cur, self.scheme.rho_dests, nat.DENSITY_EOS | reuse)
            if self.tait_only_mask:
                self.tait(self.tait_only_mask)
            # the density pass above searched the same cells
            self.momentum(mode=mode, synced=True)
        if stage is not None:
            self._swap_records()

    def pc_step(self, on_half=None):
        """One PredictorCorrectorIntegrator.integrate(dt) of every scene,
        preceded by the Solver's per-step prologue (count, dt).  on_half,
        when given, is called after the predictor stage.  With list reuse
        both stages rebin only when the device finds it necessary, and the
        state never changes buffers, so one captured graph replays every
        step."""
        reuse = nat.BIN_IF_NEEDED if self.step_lists else 0
        self._begin_and_bin(reuse)
        self._stage(0)
        if on_half is not None:
            on_half()
        self.bin(nat.BIN_MOVE_INITIAL | reuse)
        self._stage(1)

    def _begin_and_bin(self, reuse):
        """The step prologue and the first bin: one launch (the rebin
        decision runs the prologue) when the device decides the rebin."""
        if reuse:
            self.bin(reuse | nat.BIN_STEP_BEGIN)
        else:
            self.step_begin()
            self.bin(reuse)

    def step(self, integrator: str = "pc", on_half=None):
        """One step of the named integrator: "pc" (pc_step), "euler"
        (EulerIntegrator: X = X0 + dt F), "rk2" (RK2Integrator:
        X_half = X0 + dt/2 F(X0), X = X0 + dt F(X_half)) or "rk4"
        (RK4Integrator: K1 .. K4 at X0, X0 + dt/2 K1, X0 + dt/2 K2,
        X0 + dt K3; X = X0 + dt/6 (K1 + 2 K2 + 2 K3 + K4))."""
        if integrator == "pc":
            return self.pc_step(on_half)
        if integrator not in ("euler", "rk2", "rk4"):
            raise NotImplementedError(f"{integrator} is not fused on the engine")
        reuse = nat.BIN_IF_NEEDED if self.step_lists else 0
        if integrator == "rk4":
            self._rk4_sums()
            self._begin_and_bin(reuse)
            for kind in (4, 5, 6, 7):
                if kind > 4:
                    self.bin(nat.BIN_MOVE_INITIAL | reuse)
                self._stage(kind)
            return
        self._begin_and_bin(reuse)
        if integrator == "euler":
            self._stage(2)
            return
        self._stage(0)
        if on_half is not None:
            on_half()
        self.bin(nat.BIN_MOVE_INITIAL | reuse)
        self._stage(3)

    def _launch_state(self):
        """Everything a step's launches depend on besides device memory:
        the descriptor the kernels receive by value, and the host-side flags
        and masks that choose the calls and their arguments."""
        sc = self.scheme
        return (ctypes.string_at(ctypes.addressof(self.desc), ctypes.sizeof(self.desc)),
                self.cur, bool(getattr(self, "_host_state", False)), self._box_valid,
                self.step_lists, self.fuses_stage, self.force_mode, self.list_cap,
                self.tait_only_mask, sc.continuity, sc.rho_dests, sc.mom_dests,
                sc.pair_dests)

    def _import_inline(self, imports):
        by_array: dict = {}
        for a, name, t in imports:
            if t.numel():
                by_array.setdefault(a, []).append((name, t))
        for a, items in by_array.items():
            self._exchange_many(a, 0, items)

    def _exchange_many(self, array: int, direction: int, items):
        """sphb_exchange of several (name, FP64 user-order tensor) of one
        array, SPHB_EXCHANGE_MAX per launch."""
        for i in range(0, len(items), nat.EXCHANGE_MAX):
            part = items[i:i + nat.EXCHANGE_MAX]
            fields = (ctypes.c_int32 * len(part))(*[self._field_id(array, n) for n, _ in part])
            users = (ctypes.c_void_p * len(part))(*[t.data_ptr() for _, t in part])
            self.call("sphb_exchange_many", self.cur, array, direction, len(part), fields,
                      users, self.user_offset[array].data_ptr())

    def exchange_out_many(self, array: int, names, outs):
        """exchange_out of several properties into the given FP64 tensors in
        one launch."""
        if self.user_n[array] and names:
            self._exchange_many(array, 1, list(zip(names, outs)))

    def step_graphed(self, integrator: str = "pc", imports=()):
        """step(integrator) through a CUDA graph: the first step from a given
        launch state runs as it is (loading every kernel), the second is
        captured, and later ones replay it -- one launch instead of one per
        pass, so the host no longer paces the device.  Steps whose launches
        would differ (another descriptor, flags or masks) get their own
        graph.  imports: (array, name, tensor) positions or velocities that
        the host wrote, imported as the step's first launches (the graph
        reads the tensors' memory, so a replay imports their values of the
        moment).  With graphs off, off CUDA, or inside another capture, it
        is the imports and step()."""
        inline = []
        for a, name, t in imports:
            if (name in ("x", "y", "z", "u", "v", "w") and t.dtype == torch.float64
                    and t.device == self.device and t.is_contiguous()
                    and t.numel() == self.user_n[a]):
                inline.append((a, name, t))
            else:
                self.exchange_in(a, name, t)
        if inline:
            # the host flags such an import sets (_exchange_in)
            self._box_valid = False
            self._host_state = True
        if (not self.graphs or self.device.type != "cuda"
                or torch.cuda.is_current_stream_capturing()):
            self._import_inline(inline)
            return self.step(integrator)
        if integrator == "rk4":
            self._rk4_sums()   # buffers made outside any capture
        key = (integrator, tuple((a, n, t.data_ptr()) for a, n, t in inline),
               self._launch_state())
        hit = self._graphs.get(key)
        if hit is None:
            if key not in self._graph_seen:
                if len(self._graph_seen) >= 64:
                    # states that never repeat (e.g. new tensors every step)
                    # must not grow the record without bound
                    self._graph_seen.clear()
                self._graph_seen.add(key)
                self._import_inline(inline)
                return self.step(integrator)
            if len(self._graphs) >= 8:
                self._graphs.clear()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._import_inline(inline)
                self.step(integrator)
            hit = (g, (self.cur, self._host_state, self._box_valid))
            # kept for replays only when the step leaves the descriptor as
            # it found it (an even number of record swaps, as every fused
            # integrator's step has); replayed this once either way
            if self._launch_state()[0] == key[2][0]:
                self._graphs[key] = hit
            self._graph_last = hit
        g, after = hit
        g.replay()
        self.cur, self._host_state, self._box_valid = after

    def _rk4_sums(self):
        """RK4's running sums (K1 + 2 K2 + 2 K3 of every integrated
        property), in both state buffers so that rebins carry them; made
        once, before the first RK4 step (and before any graph of one)."""
        if self.bufs[0]["kx"] is not None:
            return
        f64 = dict(dtype=torch.float64, device=self.device)
        names = ["kx", "ky", "ku", "kv"] + (["kz", "kw"] if self.dim == 3 else [])
        if self.scheme.continuity:
            names.append("krho")
        for b in self.bufs:
            for name in names:
                b[name] = torch.zeros(self.N, **f64)
        self._build_desc()

    def rebin_count(self) -> int:
        """1 when the last device-decided rebin happened (host sync)."""
        off = self.work_offsets[nat.WORK_NAMES.index("meta")]
        return int(self.work_buf[off + 4:off + 8].view(torch.int32).item())

    # ---------------------------------------------------------- host sync
    def status(self) -> int:
        off = self.work_offsets[nat.WORK_NAMES.index("status")]
        return int(self.work_buf[off:off + 4].view(torch.int32).item())

    def clear_status(self):
        off = self.work_offsets[nat.WORK_NAMES.index("status")]
        self.work_buf[off:off + 4].zero_()

    def check_status(self):
        st = self.status()
        if st:
            raise RuntimeError("engine status: " + nat.status_message(st))

    def pair_counts(self):
        off = self.work_offsets[nat.WORK_NAMES.index("pairs")]
        v = self.work_buf[off:off + 32].view(torch.int64).tolist()
        return v[0], v[1]

    def fallback_blocks(self) -> int:
        """Blocks of the tiled pair passes (since the last
        reset_pair_counts) whose stencil rows did not fit shared memory and
        that read their records from global memory instead."""
        off = self.work_offsets[nat.WORK_NAMES.index("pairs")]
        return int(self.work_buf[off + 16:off + 24].view(torch.int64).item())

    def device_rebins(self) -> int:
        """Rebins the device's decisions ran since the last
        reset_pair_counts (each captured or eager SPHB_BIN_IF_NEEDED bin that
        did not keep the cells)."""
        off = self.work_offsets[nat.WORK_NAMES.index("pairs")]
        return int(self.work_buf[off + 24:off + 32].view(torch.int64).item())

    def reset_pair_counts(self):
        off = self.work_offsets[nat.WORK_NAMES.index("pairs")]
        self.work_buf[off:off + 32].zero_()

    def scene_state(self):
        raw = self.sstate_dev.cpu().numpy().tobytes()
        arr = (nat.SceneState * self.S).from_buffer_copy(raw)
        return [arr[s] for s in range(self.S)]

    def set_dt(self, dt):
        st = (nat.SceneState * self.S).from_buffer_copy(self.sstate_dev.cpu().numpy().tobytes())
        dts = dt if isinstance(dt, (list, tuple, np.ndarray)) else [dt] * self.S
        for s in range(self.S):
            st[s].dt = float(dts[s])
        self.sstate_dev.copy_(_struct_to_device(st, self.device))

    # --------------------------------------------------------- exchange
    def exchange_in(self, array: int, name: str, values: torch.Tensor):
        """User-order FP64 values (scenes concatenated) -> engine."""
        self._exchange_in(array, name, values)
        if name == "h" and any(t.uniform_h for t in self._scene_host):
            # smoothing lengths may now differ within a scene
            for t in self._scene_host:
                t.uniform_h = 0
            self.scene_dev.copy_(_struct_to_device(self._scene_host, self.device))

    def _exchange_in(self, array: int, name: str, values: torch.Tensor):
        v = values.to(device=self.device, dtype=torch.float64).contiguous()
        if v.numel() != self.user_n[array]:
            raise ValueError("size mismatch")
        if name == "h" and v.numel():
            # the cells were sized for the largest h at construction
            off = self.user_offset_host[array]
            hm = v.cpu().numpy()
            for s in range(self.S):
                n = int(self.sizes[s, array])
                if n and float(hm[off[s]:off[s] + n].max()) > self._h_cap[s]:
                    raise ValueError("smoothing length above the largest one the cells were "
                                     "sized for: build a new engine")
        if v.numel():   # (an array without particles has nothing to copy)
            self.call("sphb_exchange", self.cur, array, self._field_id(array, name), 0,
                      v.data_ptr(), self.user_offset[array].data_ptr())
        self._keep = v  # keep alive until the stream passes it
        if name in ("x", "y", "z", "u", "v", "w", "m", "h"):
            # the next bin recomputes the boxes; new m or h withdraw the
            # lists, new positions or velocities need the records refreshed
            # and the displacements measured before the lists are trusted
            self._box_valid = False
            if name not in ("m", "h"):
                self._host_state = True

    def exchange_out(self, array: int, name: str, out: torch.Tensor | None = None):
        """Engine -> user-order FP64 tensor (scenes concatenated)."""
        if out is None:
            out = torch.empty(self.user_n[array], dtype=torch.float64, device=self.device)
        if self.user_n[array]:
            self.call("sphb_exchange", self.cur, array, self._field_id(array, name), 1,
                      out.data_ptr(), self.user_offset[array].data_ptr())
        return out

    def _field_id(self, array: int, name: str) -> int:
        """Exchange id of a property.  With the continuity equation the
        density of an SPHDensityRate dest is the integrated state."""
        name = _canon(name)
        if name == "rho" and self.scheme.rate_src.get(array):
            return nat.FIELDS["rho_state"]
        return nat.FIELDS[name]

    def exchange_tag(self, array: int, values: torch.Tensor, direction: int):
        v = values.to(device=self.device, dtype=torch.int32).contiguous()
        if v.numel():
            self.call("sphb_exchange_tag", self.cur, array, direction, v.data_ptr(),
                      self.user_offset[array].data_ptr())
        return v

    def get(self, array: int, name: str, scene: int | None = None):
        out = self.exchange_out(array, name)
        if scene is None:
            return out
        o = int(self.user_offset_host[array][scene])
        return out[o:o + int(self.sizes[scene, array])]

    # ------------------------------------------------------- inspection
    def neighbors(self, dest_array: int, src_mask: int, scene: int = 0):
        """Neighbour pairs of scene `scene`, dest array `dest_array`, with the
        FP64 reference predicate: numpy arrays (dest user index, source array,
        source user index), lexicographically sorted."""
        dev = self.device
        self._sync_cells()
        counts = torch.zeros(self.N, dtype=torch.int32, device=dev)
        dm = 1 << dest_array
        self.call("sphb_neighbors", self.cur, dm, src_mask, counts.data_ptr(),
                  None, None, 0)
        c64 = counts.to(torch.int64)
        offs = torch.cumsum(c64, 0) - c64
        total = int(c64.sum().item())
        out = torch.zeros(max(total, 1), dtype=torch.int32, device=dev)
        self.call("sphb_neighbors", self.cur, dm, src_mask, counts.data_ptr(),
                  offs.data_ptr(), out.data_ptr(), total)
        self.check_status()
        idx = self.bufs[self.cur]["idx"].cpu().numpy()
        counts = counts.cpu().numpy()
        out = out[:total].cpu().numpy()
        seg = self.seg_offset_host
        k = np.repeat(np.arange(self.N), counts)
        seg_of = np.searchsorted(seg, np.arange(self.N), side="right") - 1
        keep = seg_of[k] == scene * self.A + dest_array
        k = k[keep]
        j = out[keep]
        sj = seg_of[j]
        d_user = idx[k]
        s_arr = sj % self.A
        j_user = idx[j]
        order = np.lexsort((j_user, s_arr, d_user))
        return d_user[order], s_arr[order], j_user[order]

    def neighbor_csr(self, dest_array: int, src_array: int, scene: int = 0):
        """The neighbour lists of (scene, dest_array) in src_array with the
        FP64 reference predicate, as CSR in user order: (offsets int64
        [n_dest + 1], source user indices int32), each dest's list
        ascending.  The sort runs on the device, so lists of millions of
        particles come back in a fraction of a second."""
        dev = self.device
        self._sync_cells()
        counts = torch.zeros(self.N, dtype=torch.int32, device=dev)
        dm, sm = 1 << dest_array, 1 << src_array
        self.call("sphb_neighbors", self.cur, dm, sm, counts.data_ptr(), None, None, 0)
        c64 = counts.to(torch.int64)
        offs = torch.cumsum(c64, 0) - c64
        total = int(c64.sum().item())
        out = torch.zeros(max(total, 1), dtype=torch.int32, device=dev)
        self.call("sphb_neighbors", self.cur, dm, sm, counts.data_ptr(), offs.data_ptr(),
                  out.data_ptr(), total)
        self.check_status()
        g = scene * self.A + dest_array
        b, e = int(self.seg_offset_host[g]), int(self.seg_offset_host[g + 1])
        ns = int(self.sizes[scene, src_array])
        lo = int(offs[b].item()) if e > b else 0
        hi = lo + int(c64[b:e].sum().item())
        idx = self.bufs[self.cur]["idx"]
        k = torch.repeat_interleave(torch.arange(b, e, device=dev), c64[b:e])
        j = out[lo:hi].to(torch.int64)
        key = idx[k].to(torch.int64) * max(ns, 1) + idx[j].to(torch.int64)
        del k, j
        key = torch.sort(key).values
        n_dest = e - b
        per = torch.bincount((key // max(ns, 1)), minlength=n_dest)
        off = torch.zeros(n_dest + 1, dtype=torch.int64, device=dev)
        off[1:] = torch.cumsum(per, 0)
        lst = (key % max(ns, 1)).to(torch.int32)
        return off.cpu().numpy(), lst.cpu().numpy()

    def cell_coords(self, scene: int = 0, array: int = 0):
        """Global integer cell coordinates floor(x / cell_size) per user
        particle of (scene, array)."""
        if self.step_lists:
            # cells of the current positions, not of the last rebin
            self.bin(nat.BIN_MOVE_INITIAL)
        out = torch.zeros(self.N * 3, dtype=torch.int32, device=self.device)
        self.call("sphb_cell_coords", self.cur, out.data_ptr())
        out = out.view(self.N, 3).cpu().numpy()
        g = scene * self.A + array
        b, e = self.seg_offset_host[g], self.seg_offset_host[g + 1]
        idx = self.bufs[self.cur]["idx"][b:e].cpu().numpy()
        res = np.empty((e - b, 3), np.int32)
        res[idx] = out[b:e]
        return res

    def cell_size(self, scene: int = 0) -> float:
        return self._scene_host[scene].cell_size


def _canon(name: str) -> str:
    return {"x0": "_x0", "y0": "_y0", "z0": "_z0", "u0": "_u0", "v0": "_v0",
            "w0": "_w0", "au": "_a_u_1", "av": "_a_v_1", "aw": "_a_w_1"}.get(name, name)


def _np(v):
    if isinstance(v, torch.Tensor):
        return v.detach().cpu().numpy()
    return v


def _np_b(v, n):
    v = _np(v)
    return np.array(np.broadcast_to(np.asarray(v), (n,)))


def _struct_to_device(cstruct, device):
    raw = ctypes.string_at(ctypes.addressof(cstruct), ctypes.sizeof(cstruct))
    t = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
    return t.to(device)
