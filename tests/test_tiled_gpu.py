"""The tiled pair passes (shared-memory staging of each block's stencil
rows, pair_mode SPHB_PAIRS_TILED) against the oracle and against the
list passes, through the C ABI.

The tiled passes evaluate the same pairs in the same order with the same
FP32 arithmetic as the list passes, so their results agree to the last few
bits; against the oracle they meet the FP32C bars of the other parity tests
(1e-5 relative density error, 1e-4 of the largest acceleration).
"""
import numpy as np
import pytest
import torch

from helpers import oracle_from, oracle_density_eos, oracle_momentum, rel_err
from pysph_b200 import _native as nat
from pysph_b200 import workloads as W
from pysph_b200.engine import Engine, fluid_scheme

pytestmark = pytest.mark.gpu


def small_dam(dx=0.02):
    arrays, types, params = W.dam_break(dx=dx)
    return arrays, params, fluid_scheme(2)


def drop(dx=0.025):
    arrays, types, params = W.elliptical_drop(dx=dx)
    return arrays, dict(params, dt=1e-5), fluid_scheme(1)


CASES = {"dam": small_dam, "drop": drop}


def max_rel(got, ref):
    return float(np.max(np.abs(got - ref) / np.abs(ref)))


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("stencil,block", [(1, 256), (1, 128), (2, 256)])
def test_tiled_first_evaluation_against_oracle(case, stencil, block):
    arrays, params, scheme = CASES[case]()
    eng = Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="tiled",
                 stencil=stencil, pair_block=block)
    assert eng.pairs == "tiled"
    osys = oracle_from(arrays, params, scheme, 2)
    osys.update()
    oracle_density_eos(osys, scheme)
    oracle_momentum(osys, scheme)
    eng.reset_pair_counts()
    eng.eval_stage()
    eng.check_status()
    for a in range(len(arrays)):
        assert max_rel(eng.get(a, "rho").cpu().numpy(), osys.arrays[a].rho) <= 1e-5
    O = osys.arrays[0]
    scale = max(np.max(np.abs(O.au)), np.max(np.abs(O.av)))
    assert rel_err(eng.get(0, "au").cpu().numpy(), O.au, scale) <= 1e-4
    assert rel_err(eng.get(0, "av").cpu().numpy(), O.av, scale) <= 1e-4
    assert rel_err(eng.get(0, "dt_fac").cpu().numpy(), O.dt_fac) <= 1e-4
    pd, pf = eng.pair_counts()
    A = len(arrays)
    tot_rho = sum(len(osys.neighbors(d, s)[1]) for d in range(A) for s in range(A))
    tot_mom = sum(len(osys.neighbors(0, s)[1]) for s in range(A))
    assert abs(pd - tot_rho) <= max(2, tot_rho * 1e-5)
    assert abs(pf - tot_mom) <= max(2, tot_mom * 1e-5)
    # the force pass searching its own cells (no per-stage list) evaluates
    # the same entries in the same order
    got = [eng.get(0, n).clone() for n in ("au", "av", "dt_fac")]
    eng.momentum(mode=0)
    eng.check_status()
    for n, g in zip(("au", "av", "dt_fac"), got):
        assert torch.equal(eng.get(0, n), g), n


def _pair(arrays, params, scheme, **kw):
    a = Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="tiled", **kw)
    b = Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="lists", **kw)
    return a, b


def test_tiled_matches_lists_on_the_full_dam_break():
    """332,018 particles: the tiled and the list passes give the same
    densities, accelerations and dt_fac (the same pairs in the same order),
    the same pair counts, and some blocks (the side walls, whose tiles span
    many cell rows) take the global-memory path."""
    arrays, types, params = W.dam_break()
    a, b = _pair(arrays, params, fluid_scheme(2), pair_block=256)
    for e in (a, b):
        e.reset_pair_counts()
        e.eval_stage()
        e.check_status()
    assert a.pair_counts() == b.pair_counts()
    assert a.fallback_blocks() > 0
    for arr in range(2):
        ra, rb = a.get(arr, "rho").cpu().numpy(), b.get(arr, "rho").cpu().numpy()
        assert max_rel(ra, rb) <= 1e-6
    for n in ("au", "av", "dt_fac"):
        ga, gb = a.get(0, n).cpu().numpy(), b.get(0, n).cpu().numpy()
        assert rel_err(ga, gb) <= 1e-6, n


@pytest.mark.parametrize("case,steps", [("dam", 40), ("drop", 20)])
def test_tiled_steps_match_lists(case, steps):
    """Predictor-corrector steps with the fused stage and the device's
    rebin decisions: the tiled engine tracks the list engine to the FP32C
    trajectory bar and makes the same rebin decisions."""
    arrays, params, scheme = CASES[case]()
    a, b = _pair(arrays, params, scheme)
    da, db = [], []
    for _ in range(steps):
        a.pc_step()
        b.pc_step()
        da.append(a.rebin_count())
        db.append(b.rebin_count())
    a.check_status()
    b.check_status()
    assert da == db
    for n in ("x", "y", "u", "v", "rho"):
        ga, gb = a.get(0, n).cpu().numpy(), b.get(0, n).cpu().numpy()
        assert np.max(np.abs(ga - gb)) <= 1e-5 * max(1.0, np.max(np.abs(gb))), n
    assert a.scene_state()[0].dt == pytest.approx(b.scene_state()[0].dt, rel=1e-6)


def test_tiled_graph_replay_matches_eager():
    arrays, params, scheme = small_dam()
    a = Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="tiled")
    b = Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="tiled")
    for e in (a, b):
        for _ in range(3):
            e.pc_step()
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        a.pc_step()
        b.pc_step()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        a.pc_step()
    for _ in range(15):
        g.replay()
        b.pc_step()
    torch.cuda.synchronize()
    a.check_status()
    b.check_status()
    for n in ("x", "y", "u", "v", "rho", "p"):
        assert torch.equal(a.get(0, n), b.get(0, n)), n
    del g


def test_tiled_batched_scenes():
    """Many scenes of uneven size in one launch per pass."""
    scenes = W.batched_drops(num_scenes=12, seed=3, n_lo=300, n_hi=3000)
    specs = [(arrs, p) for arrs, _, p in scenes]
    eng = Engine(specs, fluid_scheme(1), dim=2, precision="fp32c", pairs="tiled")
    for _ in range(3):
        eng.pc_step()
    eng.check_status()
    for s, (arrs, p) in enumerate(specs):
        osys = oracle_from(arrs, p, fluid_scheme(1), 2)
        for _ in range(3):
            osys.pc_step(p["dt"])
        O = osys.arrays[0]
        rho = eng.get(0, "rho", scene=s).cpu().numpy()
        x = eng.get(0, "x", scene=s).cpu().numpy()
        assert max_rel(rho, O.rho) <= 1e-5
        dx = float(arrs[0]["h"][0]) / 1.3
        assert np.max(np.abs(x - O.x)) / dx <= 2e-6


@pytest.mark.parametrize("kernel", [nat.KERNEL_QUINTIC, nat.KERNEL_WENDLAND])
def test_tiled_other_kernels_match_lists(kernel):
    arrays, params, scheme = drop(dx=0.05)
    a, b = _pair(arrays, params, scheme, kernel=kernel)
    for e in (a, b):
        e.eval_stage()
        e.check_status()
    assert a.pair_counts() == b.pair_counts()
    for n in ("rho", "au", "av"):
        ga, gb = a.get(0, n).cpu().numpy(), b.get(0, n).cpu().numpy()
        assert rel_err(ga, gb) <= 1e-6, n


def test_tiled_rejects_unsupported_configurations():
    from pysph_b200.engine import continuity_scheme
    arrays, params, scheme = drop(dx=0.1)
    with pytest.raises(NotImplementedError):
        Engine([(arrays, params)], scheme, dim=2, precision="fp64", pairs="tiled")
    with pytest.raises(NotImplementedError):
        Engine([(arrays, params)], continuity_scheme(1), dim=2, precision="fp32c",
               pairs="tiled")
    with pytest.raises(ValueError):
        Engine([(arrays, params)], scheme, dim=2, precision="fp32c", pairs="tiled", lanes=2)
