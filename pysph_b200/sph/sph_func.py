"""SPH functions of the particle-update path (S/sph/sph_func.pyx,
S/sph/funcs/{density,eos,pressure,external_force,position}_funcs.pyx).

The classes keep the reference's names, constructor arguments, withargs()
factory, ids and tags.  They carry no arithmetic of their own: an SPHCalc (or
the predictor-corrector integrator) hands them to the CUDA engine, which
evaluates the pair sums.  Each class declares what the engine runs for it:

  SPHRho               summation density            sphb_density
  TaitEquation         p, cs from rho               sphb_tait
  MomentumEquation     pressure gradient + Monaghan  sphb_momentum (mode 0)
  SPHPressureGradient  pressure gradient            sphb_momentum (mode 1)
  MonaghanArtificialViscosity  split-form viscosity  sphb_momentum (mode 2)
  GravityForce         += g                         integrator / SPHCalc
  PositionStepping     dx/dt = v                    integrator / SPHCalc
"""
from __future__ import annotations


class Function:
    """A function class plus its arguments; get_func(source, dest) builds
    the SPHFunction for one source/dest pair (S/sph/sph_func.pyx:26-80)."""

    def __init__(self, cls, *args, **kwargs):
        self.cls = cls
        self.args = args
        self.kwargs = kwargs

    def get_func(self, source, dest):
        return self.cls(source, dest, *self.args, **self.kwargs)

    def get_func_class(self):
        return self.cls


class SPHFunction:
    """Base of every function: one dest array, evaluated per dest particle
    (S/sph/sph_func.pyx:107-227)."""

    kind = "single"          # single | pair
    engine_op = None
    num_outputs = 3

    def __init__(self, source, dest=None, setup_arrays=True, *args, **kwargs):
        self.name = ""
        self.id = ""
        self.tag = ""
        self.source = source
        self.dest = source
        self.kernel = None
        self.nbr_locator = None
        self.to_reset = []
        self.src_reads = []
        self.dst_reads = []
        self.set_src_dst_reads()

    def set_src_dst_reads(self):
        pass

    @classmethod
    def withargs(cls, *args, **kwargs):
        return Function(cls, *args, **kwargs)

    @classmethod
    def get_func(cls, source, dest):
        return Function(cls).get_func(source, dest)

    @classmethod
    def get_func_class(cls):
        return cls

    def setup_calc_updates(self, calc):
        return list(calc.updates)

    def params(self) -> dict:
        return {}


class SPHFunctionParticle(SPHFunction):
    """A function with a neighbour sum over the source array
    (S/sph/sph_func.pyx:400-441)."""

    kind = "pair"

    def __init__(self, source, dest, setup_arrays=True, hks=False, exclude_self=False,
                 nbr_locator=None, *args, **kwargs):
        SPHFunction.__init__(self, source, dest, setup_arrays)
        self.dest = dest
        # hks: W and grad W averaged over h_a and h_b instead of taken at
        # (h_a + h_b) / 2 (e.g. S/sph/funcs/density_funcs.pyx:56-63)
        self.hks = bool(hks)
        self.exclude_self = exclude_self
        if exclude_self:
            raise NotImplementedError("exclude_self is not part of this build")


class CSPHFunctionParticle(SPHFunctionParticle):
    pass


class SPHRho(CSPHFunctionParticle):
    """Summation density rho_a = sum_b m_b W_ab
    (S/sph/funcs/density_funcs.pyx:14-83)."""

    engine_op = "density"
    num_outputs = 1

    def __init__(self, source, dest, setup_arrays=True, **kwargs):
        CSPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        self.id = "sphrho"
        self.tag = "density"

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m"]
        self.dst_reads = ["x", "y", "z", "h", "tag"]


class TaitEquation(SPHFunction):
    """p = B ((rho/ro)^gamma - 1), B = co^2 ro / gamma;
    cs = co (rho/ro)^((gamma-1)/2) (S/sph/funcs/eos_funcs.pyx:57-129)."""

    engine_op = "tait"
    num_outputs = 2

    def __init__(self, source, dest, setup_arrays=True, co=1.0, ro=1000.0,
                 gamma=7.0, **kwargs):
        SPHFunction.__init__(self, source, dest, setup_arrays)
        self.co = float(co)
        self.ro = float(ro)
        self.gamma = float(gamma)
        self.B = self.co * self.co * self.ro / self.gamma
        self.id = "tait"
        self.tag = "state"

    def set_src_dst_reads(self):
        self.dst_reads = ["rho"]

    def params(self):
        return {"c0": self.co, "rho0": self.ro, "gamma": self.gamma}


class MomentumEquation(SPHFunctionParticle):
    """Pressure gradient + Monaghan artificial viscosity, with the viscous
    time-step factor dt_fac (S/sph/funcs/pressure_funcs.pyx:174-398)."""

    engine_op = "momentum"

    def __init__(self, source, dest, setup_arrays=True, alpha=1, beta=1, gamma=1.4,
                 eta=0.1, deltap=None, n=1, eps=0.2, **kwargs):
        SPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        self.alpha = float(alpha)
        self.beta = float(beta)
        self.gamma = float(gamma)
        self.eta = float(eta)
        if deltap is not None:
            if deltap < 0:
                raise RuntimeError("deltap cannot be negative!")
            raise NotImplementedError("the artificial-pressure term (deltap) is not "
                                      "part of this build")
        self.n = n
        self.eps = eps
        self.id = "momentumequation"
        self.tag = "velocity"
        self.to_reset = ["dt_fac"]
        if dest is not None and not dest.has_array("dt_fac"):
            dest.add_property({"name": "dt_fac"})

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m", "rho", "p", "u", "v", "w", "cs"]
        self.dst_reads = ["x", "y", "z", "h", "rho", "p", "u", "v", "w", "cs", "tag"]

    def params(self):
        return {"alpha": self.alpha, "beta": self.beta, "eta": self.eta}


class MonaghanArtificialViscosity(SPHFunctionParticle):
    """The split form of Monaghan's artificial viscosity, for schemes that
    pair it with SPHPressureGradient: a_a += -m_b Pi_ab grad W_ab when
    v_ab . r_ab < 0, and dt_fac (S/sph/funcs/viscosity_funcs.pyx:19-157).

    Kept as the reference has it: the constructor takes eta but never
    stores it, so the viscosity's eta is 0 until the attribute is assigned,
    and its dt_fac uses 0.01 h_ab^2 whatever eta is.  gamma is accepted and
    unused."""

    engine_op = "avisc"

    def __init__(self, source, dest, setup_arrays=True, alpha=1, beta=1, gamma=1.4,
                 eta=0.1, **kwargs):
        SPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        self.alpha = float(alpha)
        self.beta = float(beta)
        self.gamma = float(gamma)
        self.eta = 0.0          # the eta argument is not stored (see above)
        self.id = "momavisc"
        self.tag = "velocity"
        self.to_reset = ["dt_fac"]
        if dest is not None and not dest.has_array("dt_fac"):
            dest.add_property({"name": "dt_fac"})

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m", "rho", "u", "v", "w", "cs"]
        self.dst_reads = ["x", "y", "z", "h", "p", "u", "v", "w", "cs", "rho", "tag"]

    def params(self):
        return {"alpha": self.alpha, "beta": self.beta, "eta": float(self.eta)}


class SPHPressureGradient(SPHFunctionParticle):
    """-sum_b m_b (P_a/rho_a^2 + P_b/rho_b^2) grad W_ab
    (S/sph/funcs/pressure_funcs.pyx:19-168)."""

    engine_op = "pgrad"

    def __init__(self, source, dest, setup_arrays=True, deltap=None, n=1, eps=0.2,
                 **kwargs):
        SPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        if deltap is not None:
            raise NotImplementedError("the artificial-pressure term (deltap) is not "
                                      "part of this build")
        self.id = "pgrad"
        self.tag = "velocity"

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m", "rho", "p"]
        self.dst_reads = ["x", "y", "z", "h", "rho", "p", "tag"]


class GravityForce(SPHFunction):
    """Constant body force (S/sph/funcs/external_force.pyx:13-62)."""

    engine_op = "gravity"

    def __init__(self, source, dest, setup_arrays=True, gx=0.0, gy=0.0, gz=0.0,
                 hks=False):
        SPHFunction.__init__(self, source, dest, setup_arrays)
        self.gx, self.gy, self.gz = float(gx), float(gy), float(gz)
        self.id = "gravityforce"
        self.tag = "velocity"

    def params(self):
        return {"gravity": (self.gx, self.gy, self.gz)}


class PositionStepping(SPHFunction):
    """dx/dt = u (S/sph/funcs/position_funcs.pyx:10-56)."""

    engine_op = "position"

    def __init__(self, source, dest, setup_arrays=True):
        SPHFunction.__init__(self, source, dest, setup_arrays)
        self.id = "positionstepper"
        self.tag = "position"

    def set_src_dst_reads(self):
        self.dst_reads = ["u", "v", "w", "tag"]


class SPHDensityRate(SPHFunctionParticle):
    """Continuity equation drho_a/dt = sum_b m_b (v_a - v_b) . grad_a W_ab
    (S/sph/funcs/density_funcs.pyx:88-171); integrates rho."""

    engine_op = "density_rate"
    num_outputs = 1

    def __init__(self, source, dest, setup_arrays=True, **kwargs):
        SPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        self.id = "densityrate"
        self.tag = "density"

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m", "u", "v", "w"]
        self.dst_reads = ["x", "y", "z", "h", "tag", "u", "v", "w"]


class XSPHCorrection(CSPHFunctionParticle):
    """XSPH velocity added to the position rate:
    eps sum_b m_b W_ab (v_b - v_a) / rho_ab, rho_ab = (rho_a + rho_b) / 2
    (S/sph/funcs/xsph_funcs.pyx:9-90)."""

    engine_op = "xsph"

    def __init__(self, source, dest, setup_arrays=True, eps=0.5, **kwargs):
        CSPHFunctionParticle.__init__(self, source, dest, setup_arrays, **kwargs)
        self.eps = float(eps)
        self.id = "xsph"
        self.tag = "position"

    def set_src_dst_reads(self):
        self.src_reads = ["x", "y", "z", "h", "m", "rho", "u", "v", "w"]
        self.dst_reads = ["x", "y", "z", "h", "rho", "u", "v", "w"]
