"""SPHCalc: evaluate one function family for one dest array over its
sources (S/sph/sph_calc.pyx:79-440).

sph(out1, out2, out3) keeps the reference's output semantics: a
non-integrating calc first zeroes its outputs, every calc zeroes `to_reset`
(dt_fac for MomentumEquation), results are added to the named outputs of
LocalReal dest particles, and other particles' outputs are set to 0
(SPHFunction.eval, S/sph/sph_func.pyx:208-227).  The neighbour sums run in
the CUDA engine of the Particles collection, one launch for all sources of
the calc; the result is copied into the named output property.
"""
from __future__ import annotations

import torch

from ..base.particle_types import LocalReal
from .sph_func import SPHFunction

DEFAULT_OUTPUTS = ("_tmpx", "_tmpy", "_tmpz")


class SPHCalc:
    def __init__(self, particles, sources, dest, kernel, funcs, updates=(),
                 integrates=False, dnum=0, nbr_info=True, id="",
                 kernel_gradient_correction=False, kernel_correction=-1, dim=1,
                 snum="", reset_arrays=True):
        self.particles = particles
        self.sources = list(sources)
        self.nsrcs = len(self.sources)
        self.dest = dest
        self.kernel = kernel
        self.funcs = list(funcs)
        self.integrates = integrates
        self.dnum = dnum
        self.nbr_info = nbr_info
        self.id = id
        self.dim = dim
        self.snum = snum
        self.reset_arrays = reset_arrays
        self.updates = list(updates)
        if kernel_correction != -1 or kernel_gradient_correction:
            raise NotImplementedError("kernel correction is not part of this build")
        self.kernel_correction = kernel_correction
        self.dst_writes = {}
        self.tensor_eval = False
        self.check_internals()
        self.updates = self.funcs[0].setup_calc_updates(self)
        self.nupdates = len(self.updates)
        self.tag = self.funcs[0].tag
        self.to_reset = list(self.funcs[0].to_reset)
        self.src_reads = self.funcs[0].src_reads
        self.dst_reads = self.funcs[0].dst_reads
        if particles.kernel is None:
            particles.kernel = kernel
        self.nnps_manager = particles.nnps_manager
        self.nbr_locators = [self.nnps_manager.get_neighbor_particle_locator(
            s, dest, kernel.radius()) for s in self.sources]
        for f, loc in zip(self.funcs, self.nbr_locators):
            f.kernel = kernel
            f.nbr_locator = loc

    def check_internals(self):
        if len(self.funcs) == 0 or len(self.funcs) != len(self.sources):
            raise ValueError("One sph function is needed per source")
        for i in range(len(self.funcs) - 1):
            if type(self.funcs[i]) is not type(self.funcs[i + 1]):
                raise ValueError("All sph_funcs should be of same type")
            if self.funcs[i].tag != self.funcs[i + 1].tag:
                raise ValueError("All functions should have the same tag")
        for i, f in enumerate(self.funcs):
            if f.source is not self.sources[i]:
                raise ValueError(f"SPHFunction.source not same as SPHCalc.sources[{i}]")

    # ------------------------------------------------------------------
    def sph(self, output_array1=None, output_array2=None, output_array3=None,
            exclude_self=False):
        outs = [output_array1 or DEFAULT_OUTPUTS[0], output_array2 or DEFAULT_OUTPUTS[1],
                output_array3 or DEFAULT_OUTPUTS[2]]
        dest = self.dest
        for name in outs:
            if not dest.has_array(name):
                dest.add_property({"name": name})
        if not self.integrates and self.reset_arrays:
            dest.set_to_zero(outs)
        dest.set_to_zero([n for n in self.to_reset if dest.has_array(n)])
        self.sph_array(outs, exclude_self)

    def sph_array(self, outs, exclude_self=False):
        if exclude_self:
            raise NotImplementedError("exclude_self is not part of this build")
        evaluate(self, outs)


def _apply(dest, out_name, value, tag):
    """out += value for LocalReal particles, out = 0 for the others."""
    t = dest.get(out_name)
    t.add_(value)
    t.masked_fill_(tag != LocalReal, 0.0)
    dest._touch(out_name)


def evaluate(calc: SPHCalc, outs):
    f0: SPHFunction = calc.funcs[0]
    op = f0.engine_op
    dest = calc.dest
    tag = dest.get("tag")
    if op == "gravity":
        g = (f0.gx, f0.gy, f0.gz)
        for k in range(3):
            _apply(dest, outs[k], torch.full_like(dest.get(outs[k]), g[k]), tag)
        return
    if op == "position":
        # PositionStepping sets (not adds) its outputs
        for k, v in enumerate(("u", "v", "w")):
            t = dest.get(outs[k])
            t.copy_(dest.get(v))
            t.masked_fill_(tag != LocalReal, 0.0)
            dest._touch(outs[k])
        return
    if op is None:
        raise NotImplementedError(f"{type(f0).__name__} is not part of this build")

    P = calc.particles
    s = P.session(dim=calc.kernel.dim, kernel=calc.kernel.get_type())
    eng = s.engine
    a = s.index(dest)
    src_mask = 0
    reads = set()
    for f in calc.funcs:
        b = s.index(f.source)
        src_mask |= 1 << b
        reads |= {(b, n) for n in f.src_reads}
    reads |= {(a, n) for n in f0.dst_reads}
    reads = {(b, n) for b, n in reads if n not in ("tag",)}
    params = f0.params()
    if params:
        eng.update_params(**params)
    if f0.kind == "pair":
        eng.set_hks(f0.hks)
    s.ensure(reads)
    dim = calc.kernel.dim
    if op == "density":
        with eng.masks(rho_src={a: src_mask}):
            eng.density(dest_mask=1 << a, eos=False)
        fields = ["rho"]
    elif op == "tait":
        eng.tait(dest_mask=1 << a)
        fields = ["p", "cs"]
    elif op in ("momentum", "pgrad", "avisc"):
        with eng.masks(mom_src={a: src_mask}):
            eng.momentum(dest_mask=1 << a, gravity=False,
                         mode={"momentum": 0, "pgrad": 1, "avisc": 2}[op])
        fields = ["_a_u_1", "_a_v_1", "_a_w_1"][:dim]
    elif op == "density_rate":
        # the force pass with only its SPHDensityRate term on
        with eng.masks(mom_src={a: 0}, rate_src={a: src_mask}):
            eng.momentum(dest_mask=1 << a, gravity=False, mode=0)
        fields = ["_a_rho_1"]
    elif op == "xsph":
        eng.set_xsph_eps(f0.eps)
        with eng.masks(mom_src={a: 0}, xsph_src={a: src_mask}):
            eng.momentum(dest_mask=1 << a, gravity=False, mode=0)
        fields = ["_xsph_u", "_xsph_v", "_xsph_w"][:dim]
    else:
        raise NotImplementedError(op)
    s.check()
    for k, field in enumerate(fields):
        res = eng.exchange_out(a, field)
        _apply(dest, outs[k], res, tag)
        s.valid[(a, field)] = (outs[k] == field and not calc.integrates
                               and calc.reset_arrays)
    if op in ("momentum", "avisc"):
        res = eng.exchange_out(a, "dt_fac")
        if not dest.has_array("dt_fac"):
            dest.add_property({"name": "dt_fac"})
        t = dest.get("dt_fac")
        torch.maximum(t, res, out=t)
        dest._touch("dt_fac")
        s.valid[(a, "dt_fac")] = False
