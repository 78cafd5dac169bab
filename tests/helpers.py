"""Shared helpers of the parity tests: build the same inputs for the CUDA
engine and the oracle, and compare them."""
import numpy as np

from oracle import OracleArray, OracleSystem


def oracle_from(arrays, params, scheme, dim, nthreads=0):
    """OracleSystem over copies of the numpy property dicts."""
    oarrs = [OracleArray(f"a{i}", **{k: np.array(v, np.float64, copy=True)
                                     for k, v in a.items() if k != "tag"})
             for i, a in enumerate(arrays)]
    g = tuple(params.get("gravity", (0.0, 0.0, 0.0)))
    return OracleSystem(
        oarrs, dim=dim, rho_src=scheme.rho_src, tait_on=scheme.tait_on,
        mom_src=scheme.mom_src, step_on=scheme.step_on,
        rate_src=scheme.rate_src, xsph_src=scheme.xsph_src, xsph_eps=scheme.xsph_eps,
        c0=params.get("c0", 1.0), rho0=params.get("rho0", 1000.0),
        gamma=params.get("gamma", 7.0), alpha=params.get("alpha", 1.0),
        beta=params.get("beta", 1.0), eta=params.get("eta", 0.1), gravity=g,
        nthreads=nthreads)


def oracle_density_eos(osys, scheme):
    """SPHRho then Tait as the calcs of Integrator.eval do them."""
    for d, srcs in scheme.rho_src.items():
        A = osys.arrays[d]
        A.rho[:] = 0
        for s in srcs:
            osys.sph_rho(d, s, A.rho)
    p = osys._s
    for d in scheme.tait_on:
        A = osys.arrays[d]
        A.p[:] = 0
        A.cs[:] = 0
        osys.tait(d, p.c0, p.rho0, p.gamma_eos, A.p, A.cs)


def oracle_momentum(osys, scheme, gravity=True):
    p = osys._s
    for d, srcs in scheme.mom_src.items():
        A = osys.arrays[d]
        A.au[:] = 0
        A.av[:] = 0
        A.aw[:] = 0
        A.dt_fac[:] = 0
        for s in srcs:
            osys.momentum(d, s, p.alpha, p.beta, p.eta, A.au, A.av, A.aw, A.dt_fac)
        if gravity:
            A.au += p.gx
            A.av += p.gy
            A.aw += p.gz


def rel_err(got, ref, scale=None):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    if scale is None:
        scale = np.max(np.abs(ref))
    if scale == 0:
        return float(np.max(np.abs(got - ref)))
    return float(np.max(np.abs(got - ref)) / scale)


def pairs_from_oracle(osys, d, s):
    off, idx = osys.neighbors(d, s)
    n = len(off) - 1
    di = np.repeat(np.arange(n), np.diff(off))
    order = np.lexsort((idx, di))
    return di[order], idx[order].astype(np.int64)
