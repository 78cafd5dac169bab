"""Edge cases of the pair passes against the oracle, through the C ABI:
an empty source array, a lone particle, two particles at the same
position, and a pair exactly at the kernel's support radius (excluded: the
reference's predicate is the strict r^2 < (2 h_d)^2,
source/pysph/base/nnps.pyx:337,353)."""
import numpy as np
import pytest

from helpers import (oracle_from, oracle_density_eos, oracle_momentum, rel_err,
                     pairs_from_oracle)
from pysph_b200 import workloads as W
from pysph_b200.engine import Engine, fluid_scheme

pytestmark = pytest.mark.gpu

RHO_TOL = {"fp64": 1e-12, "fp32c": 1e-5}
ACC_TOL = {"fp64": 1e-10, "fp32c": 1e-4}


def _props(x, y, h, m=1.0, u=None, v=None, rho=1000.0, cs=10.0):
    n = len(x)
    z = np.zeros(n)
    return dict(x=np.asarray(x, np.float64), y=np.asarray(y, np.float64), z=z,
                u=z.copy() if u is None else np.asarray(u, np.float64),
                v=z.copy() if v is None else np.asarray(v, np.float64),
                w=z.copy(), m=np.full(n, m), h=np.full(n, h), rho=np.full(n, rho),
                p=z.copy(), cs=np.full(n, cs))


PARAMS = dict(dim=2, c0=10.0, rho0=1000.0, gamma=7.0, alpha=0.1, beta=0.0,
              eta=0.1, gravity=(0.0, -9.81, 0.0), dt=1e-5)


def _check(arrays, params, scheme, precision, **kw):
    eng = Engine([(arrays, params)], scheme, dim=2, precision=precision, **kw)
    osys = oracle_from(arrays, params, scheme, 2)
    osys.update()
    oracle_density_eos(osys, scheme)
    oracle_momentum(osys, scheme)
    eng.density()
    eng.momentum()
    eng.check_status()
    for d in scheme.rho_src:
        if len(arrays[d]["x"]) == 0:
            continue
        rho = eng.get(d, "rho").cpu().numpy()
        ref = osys.arrays[d].rho
        assert np.max(np.abs(rho - ref) / np.abs(ref)) <= RHO_TOL[precision], d
    for d in scheme.mom_src:
        if len(arrays[d]["x"]) == 0:
            continue
        O = osys.arrays[d]
        scale = max(np.max(np.abs(O.au)), np.max(np.abs(O.av)))
        for nm, ref in (("au", O.au), ("av", O.av)):
            got = eng.get(d, nm).cpu().numpy()
            assert rel_err(got, ref, scale) <= ACC_TOL[precision], (d, nm)
        dtf = eng.get(d, "dt_fac").cpu().numpy()
        assert rel_err(dtf, O.dt_fac) <= ACC_TOL[precision]
    return eng, osys


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_empty_wall_array(precision):
    # the dam break with a wall array of no particles: the fluid's pairs
    # only, and PC steps run with the empty array in every launch
    arrays, types, params = W.dam_break(dx=0.05)
    wall = {k: np.asarray(v)[:0] for k, v in arrays[1].items()}
    arrs = [arrays[0], wall]
    eng, osys = _check(arrs, params, fluid_scheme(2), precision)
    for _ in range(3):
        eng.pc_step()
    eng.check_status()
    assert len(eng.get(1, "x")) == 0
    assert np.all(np.isfinite(eng.get(0, "x").cpu().numpy()))


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_lone_particle(precision):
    # rho = m W(0, h) from the self pair; no gradient: gravity alone
    arrs = [_props([0.3], [0.7], h=0.013, m=0.1)]
    eng, osys = _check(arrs, PARAMS, fluid_scheme(1), precision)
    assert eng.pair_counts()[0] == 1
    np.testing.assert_array_equal(eng.get(0, "au").cpu().numpy(), [0.0])
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert abs(float(eng.get(0, "av").cpu().numpy()[0]) + 9.81) <= tol * 9.81


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_coincident_particles(precision):
    # particles 0 and 1 at the same position (r_ab = 0 between distinct
    # particles): each is the other's neighbour with W(0) and a zero
    # gradient (the q > 1e-14 guard, source/pysph/base/kernels.pyx:407-412);
    # particle 2 is an ordinary neighbour of both
    arrs = [_props([0.5, 0.5, 0.51], [0.5, 0.5, 0.5], h=0.01, m=0.05,
                   u=[1.0, -1.0, 0.0], v=[0.0, 0.5, 0.0])]
    eng, osys = _check(arrs, PARAMS, fluid_scheme(1), precision)
    di, sa, sj = eng.neighbors(0, 1)
    odi, osj = pairs_from_oracle(osys, 0, 0)
    np.testing.assert_array_equal(di, odi)
    np.testing.assert_array_equal(sj, osj)
    assert set(sj[di == 0]) == {0, 1, 2}


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_pair_at_support_radius_excluded(precision):
    # h = 0.5: particles at distance exactly 1.0 = 2 h (exact in FP32 and
    # FP64) are not neighbours; at 1.0 - 2^-20 they are
    eps = 2.0 ** -20
    arrs = [_props([0.0, 1.0, 3.0, 4.0 - eps], [0.0, 0.0, 0.0, 0.0], h=0.5, m=1.0)]
    eng, osys = _check(arrs, PARAMS, fluid_scheme(1), precision)
    di, sa, sj = eng.neighbors(0, 1)
    pairs = {(int(a), int(b)) for a, b in zip(di, sj)}
    assert (0, 1) not in pairs and (1, 0) not in pairs
    assert (2, 3) in pairs and (3, 2) in pairs
    if precision == "fp64":
        # the FP32C passes test cell-relative FP32 offsets, where a pair at
        # the radius may round in; W and grad W vanish there, so only the
        # pair count can differ
        assert eng.pair_counts()[0] == 4 + 2


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
@pytest.mark.parametrize("lanes", [1, 2])
def test_list_overflow_falls_back_to_the_cell_search(precision, lanes):
    """A 30 x 30 lattice (dx = 0.05, h = 1.3 dx) with a clump of 150 more
    particles within one smoothing length of its centre: their neighbour
    sets (~180) exceed the list capacity (88 slots, 44 a lane with 2 lanes),
    so the density pass marks those lists overflowed (count -1) and every
    pass searches their cells instead.  The first evaluation and two
    predictor-corrector steps still match the oracle.  The EOS exponent is
    1 so that the clump's pressure stays moderate."""
    dx, n = 0.05, 30
    gx, gy = np.meshgrid(np.arange(n) * dx, np.arange(n) * dx)
    h = 1.3 * dx
    rng = np.random.default_rng(3)
    r = h * np.sqrt(rng.random(150))
    t = 2 * np.pi * rng.random(150)
    c = 0.5 * (n - 1) * dx
    x = np.concatenate([gx.ravel(), c + r * np.cos(t)])
    y = np.concatenate([gy.ravel(), c + r * np.sin(t)])
    arr = _props(x, y, h=h, m=1000.0 * dx * dx, rho=1000.0)
    params = dict(PARAMS, gamma=1.0)
    scheme = fluid_scheme(1)
    eng, osys = _check([arr], params, scheme, precision, lanes=lanes, pair_block=128)
    cnt = eng.fields["nbr_cnt"][:lanes * eng.N].view(lanes, eng.N)
    assert bool((cnt == -1).any()), "no list overflowed"
    for _ in range(2):
        eng.pc_step()
        osys.pc_step(1e-5)
    eng.check_status()
    O = osys.arrays[0]
    for nm in ("x", "y"):
        err = float(np.max(np.abs(eng.get(0, nm).cpu().numpy() - getattr(O, nm)))) / dx
        assert err <= (1e-10 if precision == "fp64" else 2e-6), nm
    rho = eng.get(0, "rho").cpu().numpy()
    assert float(np.max(np.abs(rho - O.rho) / O.rho)) <= RHO_TOL[precision]
