"""CPU oracle for the PySPH particle-update path -- TEST INFRASTRUCTURE ONLY.

This package is the checker for the CUDA path (``pysph_b200``) and the timed
CPU baseline of ``bench.py``.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU legs may import it; the product never does.

``sph_oracle.c`` restates the reference's FP64 Cython algorithm (file:line
citations in its header) in the reference's own operand order and neighbour
order, so that its results reproduce the reference bit for bit.  The pin is
``tests/golden/*.npz``: fixtures written by the reference itself (the script
``tests/golden/make_golden.py`` builds and runs it) and by the reference's own
known-answer tests (``tests/test_oracle.py``).

The time-step function (``cfl_time_step``) restates
``ViscousAndForceBasedTimeStep.compute_time_step`` (S/solver/
time_step_functions.py:36-57) and ``Integrator.get_max_acceleration``
(S/solver/integrator.py:369-412) in numpy.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_LIB_PATH = os.path.join(_BUILD, "liboracle.so")
_SRC = os.path.join(_HERE, "sph_oracle.c")

MAX_ARRAYS = 4
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs",
         "au", "av", "aw", "ax", "ay", "az", "dt_fac",
         "x0", "y0", "z0", "u0", "v0", "w0", "arho", "rho0")


def build(force: bool = False) -> str:
    """Compile sph_oracle.c into _build/liboracle.so (gcc, OpenMP, no FMA)."""
    os.makedirs(_BUILD, exist_ok=True)
    if (not force and os.path.exists(_LIB_PATH)
            and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(_SRC)):
        return _LIB_PATH
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-fPIC", "-shared", _SRC, "-o", _LIB_PATH + ".tmp", "-lm"]
    subprocess.check_call(cmd)
    os.replace(_LIB_PATH + ".tmp", _LIB_PATH)
    return _LIB_PATH


class _Array(ctypes.Structure):
    _fields_ = ([("n", ctypes.c_int64)]
                + [(p, ctypes.POINTER(ctypes.c_double)) for p in PROPS]
                + [("tag", ctypes.POINTER(ctypes.c_int64))])


class _System(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("narrays", ctypes.c_int32),
        ("radius_scale", ctypes.c_double), ("cell_scale", ctypes.c_double),
        ("rho_src", ctypes.c_uint32 * MAX_ARRAYS), ("tait_on", ctypes.c_uint32),
        ("mom_src", ctypes.c_uint32 * MAX_ARRAYS), ("step_on", ctypes.c_uint32),
        ("c0", ctypes.c_double), ("rho0", ctypes.c_double),
        ("gamma_eos", ctypes.c_double),
        ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("gamma_av", ctypes.c_double), ("eta", ctypes.c_double),
        ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
        ("nthreads", ctypes.c_int32), ("pad_", ctypes.c_int32),
        ("a", _Array * MAX_ARRAYS),
        ("pairs", ctypes.c_int64),
        ("rate_src", ctypes.c_uint32 * MAX_ARRAYS),
        ("xsph_src", ctypes.c_uint32 * MAX_ARRAYS),
        ("xsph_eps", ctypes.c_double),
        ("variable_h", ctypes.c_int32), ("hks", ctypes.c_int32),
        ("kernel", ctypes.c_int32), ("pad2_", ctypes.c_int32),
        ("split_av", ctypes.c_int32), ("pad3_", ctypes.c_int32),
        ("av_eta", ctypes.c_double),
    ]

# kernel type ids (KernelBase.get_type, S/base/kernels.pyx:31-40) and the
# support radius of each (radius())
CUBIC_SPLINE, QUINTIC_SPLINE, WENDLAND_QUINTIC_SPLINE = 1, 3, 4
KERNEL_RADIUS = {CUBIC_SPLINE: 2.0, QUINTIC_SPLINE: 3.0, WENDLAND_QUINTIC_SPLINE: 2.0}


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()   # no-op unless sph_oracle.c is newer than the library
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        L.orc_nnps_new.restype = ctypes.c_void_p
        L.orc_nnps_free.argtypes = [ctypes.c_void_p]
        L.orc_cell_size.restype = ctypes.c_double
        L.orc_cell_size.argtypes = [ctypes.c_void_p]
        L.orc_grid.argtypes = [ctypes.c_void_p, P(ctypes.c_int32), P(ctypes.c_int32)]
        L.orc_update.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_uint32]
        L.orc_nbr_total.restype = ctypes.c_int64
        L.orc_nbr_total.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_nbr_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                   P(ctypes.c_int64), P(ctypes.c_int32)]
        L.orc_nbr_copy_sorted.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          P(ctypes.c_int64), P(ctypes.c_int32),
                                          ctypes.c_int]
        L.orc_scheme_pairs.restype = ctypes.c_uint32
        L.orc_scheme_pairs.argtypes = [P(_System)]
        L.orc_eval.argtypes = [P(_System), ctypes.c_void_p]
        L.orc_pc_step.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_double]
        L.orc_integrate.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_double,
                                    ctypes.c_int]
        dp = P(ctypes.c_double)
        L.orc_sph_rho.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int,
                                  ctypes.c_int, dp]
        L.orc_tait.argtypes = [P(_System), ctypes.c_int, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_momentum.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, dp, dp, dp, dp]
        L.orc_monaghan_av.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, dp, dp, dp, dp]
        L.orc_pgrad.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int,
                                ctypes.c_int, dp, dp, dp]
        L.orc_density_rate.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_int, dp]
        L.orc_xsph.argtypes = [P(_System), ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                               ctypes.c_double, dp, dp, dp]
        L.orc_kernel_w.restype = ctypes.c_double
        L.orc_kernel_w.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int]
        L.orc_kernel_grad.argtypes = [ctypes.c_double] * 4 + [ctypes.c_int, dp]
        L.orc_kernel_w2.restype = ctypes.c_double
        L.orc_kernel_w2.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_int]
        L.orc_kernel_grad2.argtypes = ([ctypes.c_int] + [ctypes.c_double] * 4
                                       + [ctypes.c_int, dp])
        L.orc_cell_ids.argtypes = [ctypes.c_int64, dp, dp, dp, ctypes.c_double,
                                   P(ctypes.c_int32)]
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleArray:
    """One particle array (FP64 SoA, like a reference ParticleArray)."""

    def __init__(self, name: str = "", **props):
        n = None
        for k, v in props.items():
            if isinstance(v, np.ndarray) or isinstance(v, (list, tuple)):
                n = len(v)
                break
        if n is None:
            raise ValueError("at least one array-valued property is required")
        self.name = name
        self.n = n
        defaults = {"m": 1.0, "h": 1.0, "rho": 1.0}
        self.props = {}
        for p in PROPS:
            v = props.get(p, defaults.get(p, 0.0))
            self.props[p] = np.ascontiguousarray(np.broadcast_to(
                np.asarray(v, dtype=np.float64), (n,))).copy()
        self.tag = np.ascontiguousarray(
            np.asarray(props.get("tag", np.zeros(n)), dtype=np.int64)).copy()

    def __getattr__(self, k):
        props = self.__dict__.get("props")
        if props is not None and k in props:
            return props[k]
        raise AttributeError(k)

    def fill(self, A: _Array):
        A.n = self.n
        for p in PROPS:
            setattr(A, p, _dptr(self.props[p]))
        A.tag = self.tag.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


class OracleSystem:
    """A Particles-like collection plus the scheme, evaluated in the order
    SPHRho -> TaitEquation -> SPHDensityRate -> MomentumEquation ->
    GravityForce -> PositionStepping -> XSPHCorrection (summation density:
    rho_src; continuity equation: rate_src, with xsph_src / xsph_eps).

    rho_src / rate_src / mom_src / xsph_src map a dest array index to the
    list of its source array indices; tait_on / step_on list array
    indices.  split_av: the momentum is SPHPressureGradient then
    MonaghanArtificialViscosity (eta = av_eta) on the mom_src pairs."""

    def __init__(self, arrays, dim=2, rho_src=None, tait_on=(), mom_src=None,
                 step_on=(), c0=1.0, rho0=1000.0, gamma=7.0, alpha=1.0,
                 beta=1.0, eta=0.1, gravity=(0.0, 0.0, 0.0), nthreads=0,
                 radius_scale=2.0, cell_scale=2.0, rate_src=None, xsph_src=None,
                 xsph_eps=0.5, variable_h=False, hks=False, kernel=CUBIC_SPLINE,
                 split_av=False, av_eta=0.0):
        self.arrays = list(arrays)
        assert 1 <= len(self.arrays) <= MAX_ARRAYS
        self.dim = dim
        s = _System()
        s.dim = dim
        s.narrays = len(self.arrays)
        s.radius_scale = radius_scale
        s.cell_scale = cell_scale
        for d, srcs in (rho_src or {}).items():
            s.rho_src[d] = sum(1 << a for a in srcs)
        s.tait_on = sum(1 << a for a in tait_on)
        for d, srcs in (mom_src or {}).items():
            s.mom_src[d] = sum(1 << a for a in srcs)
        s.step_on = sum(1 << a for a in step_on)
        for d, srcs in (rate_src or {}).items():
            s.rate_src[d] = sum(1 << a for a in srcs)
        for d, srcs in (xsph_src or {}).items():
            s.xsph_src[d] = sum(1 << a for a in srcs)
        s.xsph_eps = xsph_eps
        s.variable_h = int(bool(variable_h))
        s.hks = int(bool(hks))
        # split momentum: SPHPressureGradient + MonaghanArtificialViscosity
        # (its eta is 0 unless assigned, as in the reference)
        s.split_av = int(bool(split_av))
        s.av_eta = float(av_eta)
        if kernel not in KERNEL_RADIUS:
            raise ValueError("kernel must be 1 (cubic), 3 (quintic) or 4 (Wendland)")
        if kernel != CUBIC_SPLINE and dim != 2:
            raise NotImplementedError("the quintic and Wendland kernels are 2D only")
        s.kernel = kernel
        s.c0, s.rho0, s.gamma_eos = c0, rho0, gamma
        s.alpha, s.beta, s.gamma_av, s.eta = alpha, beta, 1.4, eta
        s.gx, s.gy, s.gz = gravity
        s.nthreads = nthreads
        for i, arr in enumerate(self.arrays):
            arr.fill(s.a[i])
        self._s = s
        self._c = lib().orc_nnps_new()
        self.count = 0

    def __del__(self):
        c = getattr(self, "_c", None)
        if c:
            lib().orc_nnps_free(c)
            self._c = None

    def refill(self):
        for i, arr in enumerate(self.arrays):
            arr.fill(self._s.a[i])

    # -- Particles.update -------------------------------------------------
    def update(self, pair_mask=None):
        if pair_mask is None:
            pair_mask = lib().orc_scheme_pairs(ctypes.byref(self._s))
        rc = lib().orc_update(ctypes.byref(self._s), self._c, pair_mask)
        if rc:
            raise RuntimeError(f"oracle update failed ({rc})")

    def update_pairs(self, pairs):
        self.update(sum(1 << (d * 4 + s) for d, s in pairs))

    @property
    def cell_size(self):
        return lib().orc_cell_size(self._c)

    def grid(self):
        g0 = (ctypes.c_int32 * 3)()
        gn = (ctypes.c_int32 * 3)()
        lib().orc_grid(self._c, g0, gn)
        return tuple(g0), tuple(gn)

    def neighbors(self, d, s):
        """CSR neighbour lists of dest array d in source array s, in the
        reference's own order (self last)."""
        tot = lib().orc_nbr_total(self._c, d, s)
        if tot < 0:
            raise RuntimeError("neighbour lists not built for this pair")
        off = np.empty(self.arrays[d].n + 1, np.int64)
        idx = np.empty(max(tot, 1), np.int32)
        lib().orc_nbr_copy(self._c, d, s,
                           off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return off, idx[:tot]

    def neighbors_sorted(self, d, s):
        """neighbors(d, s) with every dest's list in ascending order (the
        canonical form sets are compared in)."""
        tot = lib().orc_nbr_total(self._c, d, s)
        if tot < 0:
            raise RuntimeError("neighbour lists not built for this pair")
        off = np.empty(self.arrays[d].n + 1, np.int64)
        idx = np.empty(max(tot, 1), np.int32)
        lib().orc_nbr_copy_sorted(self._c, d, s,
                                  off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                  idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                  int(self._s.nthreads))
        return off, idx[:tot]

    # -- functions --------------------------------------------------------
    def sph_rho(self, d, s, out):
        rc = lib().orc_sph_rho(ctypes.byref(self._s), self._c, d, s, _dptr(out))
        assert rc == 0

    def tait(self, d, co, ro, gamma, out1, out2):
        lib().orc_tait(ctypes.byref(self._s), d, co, ro, gamma, _dptr(out1),
                       _dptr(out2))

    def momentum(self, d, s, alpha, beta, eta, o1, o2, o3, dt_fac):
        rc = lib().orc_momentum(ctypes.byref(self._s), self._c, d, s, alpha,
                                beta, eta, _dptr(o1), _dptr(o2), _dptr(o3),
                                _dptr(dt_fac))
        assert rc == 0

    def monaghan_av(self, d, s, alpha, beta, eta, o1, o2, o3, dt_fac):
        """MonaghanArtificialViscosity (split form) of dest d from source s,
        added into o1..o3; dt_fac takes the max."""
        rc = lib().orc_monaghan_av(ctypes.byref(self._s), self._c, d, s, alpha, beta, eta,
                                   _dptr(o1), _dptr(o2), _dptr(o3), _dptr(dt_fac))
        assert rc == 0

    def pgrad(self, d, s, o1, o2, o3):
        rc = lib().orc_pgrad(ctypes.byref(self._s), self._c, d, s, _dptr(o1),
                             _dptr(o2), _dptr(o3))
        assert rc == 0

    def eval(self):
        rc = lib().orc_eval(ctypes.byref(self._s), self._c)
        if rc:
            raise RuntimeError(f"oracle eval failed ({rc})")

    def pc_step(self, dt):
        rc = lib().orc_pc_step(ctypes.byref(self._s), self._c, float(dt))
        if rc:
            raise RuntimeError(f"oracle step failed ({rc})")
        self.count += 1

    INTEGRATORS = {"euler": 0, "rk2": 1, "rk4": 2}

    def step(self, dt, integrator="pc"):
        """One step of the named integrator (pc, euler, rk2, rk4)."""
        if integrator == "pc":
            return self.pc_step(dt)
        rc = lib().orc_integrate(ctypes.byref(self._s), self._c, float(dt),
                                 self.INTEGRATORS[integrator])
        if rc:
            raise RuntimeError(f"oracle step failed ({rc})")
        self.count += 1

    @property
    def pairs(self):
        """Pair interactions evaluated by eval / pc_step so far."""
        return int(self._s.pairs)

    def cfl_time_step(self, cfl, co, dt_initial):
        """ViscousAndForceBasedTimeStep for the arrays stepped by the
        scheme; `self.count` is the number of steps taken so far."""
        s = self._s
        dt = 1
        for d, arr in enumerate(self.arrays):
            if s.mom_src[d]:
                _dt = np.min(cfl * arr.h / (co + np.max(arr.dt_fac)))
                dt = min(_dt, dt)
        for d, arr in enumerate(self.arrays):
            if s.step_on & (1 << d):
                if self.count + 1 == 1:
                    fmax = dt_initial
                elif self.dim == 2:
                    fmax = np.max(np.sqrt(arr.au * arr.au + arr.av * arr.av))
                else:
                    fmax = np.max(np.sqrt(arr.au * arr.au + arr.av * arr.av
                                          + arr.aw * arr.aw))
                _dt = cfl * np.min(np.sqrt(arr.h / fmax))
                dt = min(dt, _dt)
        return dt


def kernel_w(dx, dy, dz, h, dim, kernel=CUBIC_SPLINE):
    if kernel == CUBIC_SPLINE:
        return lib().orc_kernel_w(dx, dy, dz, h, dim)
    return lib().orc_kernel_w2(kernel, dx, dy, dz, h, dim)


def kernel_grad(dx, dy, dz, h, dim, kernel=CUBIC_SPLINE):
    g = (ctypes.c_double * 3)()
    if kernel == CUBIC_SPLINE:
        lib().orc_kernel_grad(dx, dy, dz, h, dim, g)
    else:
        lib().orc_kernel_grad2(kernel, dx, dy, dz, h, dim, g)
    return np.array(g[:])


def cell_ids(x, y, z, cell_size):
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    z = np.ascontiguousarray(z, np.float64)
    out = np.empty((len(x), 3), np.int32)
    lib().orc_cell_ids(len(x), _dptr(x), _dptr(y), _dptr(z), cell_size,
                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return out
