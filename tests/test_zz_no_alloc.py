"""sphb_neighbor_counts_static: neighbour counts for callers that cannot
call cudaMalloc (a host whose memory manager owns the device and hands the
library only its particle arrays, or a latency-critical path that cannot
take cudaMalloc's implicit synchronisation).  Its scratch is an array inside
the library, so the test passes only input and output buffers.

Checked through the C ABI against the engine's own entry point
sphb_neighbors (same FP64 predicate, counts are integers, so they must be
equal) on calls in a row with different particle sets, because every call
reuses the one scratch array.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from pysph_b200 import _native as nat
from pysph_b200 import workloads as W
from pysph_b200.engine import Engine, fluid_scheme

pytestmark = pytest.mark.gpu


def _cols(arr, dim, dev):
    cols = [torch.as_tensor(np.ascontiguousarray(arr[c]), dtype=torch.float64, device=dev)
            for c in ("x", "y", "z", "h")]
    if dim == 2:
        cols[2] = None
    return cols


def engine_counts(arr, dim):
    """Counts from the workspace-based entry point, in the caller's order."""
    eng = Engine([([arr], {})], fluid_scheme(1), dim=dim, precision="fp64")
    counts = torch.zeros(eng.N, dtype=torch.int32, device="cuda")
    eng.call("sphb_neighbors", eng.cur, 1, 1, counts.data_ptr(), None, None, 0)
    eng.check_status()
    idx = eng.bufs[eng.cur]["idx"].long()
    out = torch.empty_like(counts)
    out[idx] = counts
    return out.cpu().numpy()


def static_counts(arr, dim):
    dev = torch.device("cuda")
    x, y, z, h = _cols(arr, dim, dev)
    n = x.numel()
    counts = torch.full((n,), -7, dtype=torch.int32, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = nat.lib().sphb_neighbor_counts_static(
        n, dim, x.data_ptr(), y.data_ptr(), z.data_ptr() if z is not None else None,
        h.data_ptr(), 2.0, counts.data_ptr(), stream)
    assert rc == 0, nat.lib().sphb_last_cuda_error()
    torch.cuda.synchronize()
    return counts.cpu().numpy()


def test_static_counts_match_engine_on_calls_in_a_row():
    drop, _, _ = W.elliptical_drop(dx=0.025)
    lat, _, _ = W.lattice3d(n=16)
    dam, _, _ = W.dam_break(dx=0.02)
    cases = [(drop[0], 2), (lat[0], 3), (dam[0], 2), (drop[0], 2)]
    for arr, dim in cases:
        got = static_counts(arr, dim)
        ref = engine_counts(arr, dim)
        assert got.min() >= 1  # self is always counted
        np.testing.assert_array_equal(got, ref)


def test_static_rejects_oversize_without_device_work():
    n = nat.STATIC_MAX_PARTICLES + 1
    rc = nat.lib().sphb_neighbor_counts_static(n, 2, None, None, None, None, 2.0,
                                                None, None)
    assert rc == -2  # SPHB_ERR_WORKSPACE
    assert nat.lib().sphb_neighbor_counts_static(
        10, 4, None, None, None, None, 2.0, None, None) == -4


def _with_outlier(arr, x_far):
    """arr plus one particle far out on the x axis."""
    out = {k: np.append(np.asarray(v, np.float64), np.asarray(v, np.float64)[0])
           for k, v in arr.items()}
    out["x"][-1] = x_far
    return out


def test_static_counts_far_particles_widen_the_cells():
    """One particle at x = 1e3, then at x = 1e6, beside the drop: the grid
    would need more than 2^19 cells, so the cells grow.  Then the whole drop
    moved to x = 1e9, where cell coordinates at the support's cell size
    would pass 2^30.  The counts stay the engine's on the plain drop (the
    far particle alone counts itself)."""
    drop, _, _ = W.elliptical_drop(dx=0.025)
    ref = engine_counts(drop[0], 2)
    for x_far in (1.0e3, 1.0e6):
        got = static_counts(_with_outlier(drop[0], x_far), 2)
        np.testing.assert_array_equal(got[:-1], ref)
        assert got[-1] == 1
    moved = {k: np.asarray(v, np.float64).copy() for k, v in drop[0].items()}
    moved["x"] = moved["x"] + 1.0e9
    np.testing.assert_array_equal(static_counts(moved, 2), ref)


def test_static_counts_variable_h():
    """Smoothing lengths that vary over the set: the predicate uses each
    particle's own h and the cells cover the largest."""
    drop, _, _ = W.elliptical_drop(dx=0.025)
    arr = {k: np.asarray(v, np.float64).copy() for k, v in drop[0].items()}
    arr["h"] = arr["h"] * (1.0 + 0.3 * np.sin(7.0 * arr["x"]) * np.cos(5.0 * arr["y"]))
    np.testing.assert_array_equal(static_counts(arr, 2), engine_counts(arr, 2))


def test_static_counts_nonfinite_particle_is_minus_one():
    """A NaN position gives -1 for that particle, which is then nobody's
    neighbour: every other count is the engine's on the set without it.  A
    NaN smoothing length gives -1 for that particle alone (the predicate
    takes each particle's own h): the others count it as before."""
    drop, _, _ = W.elliptical_drop(dx=0.025)
    base_arr = {k: np.asarray(v, np.float64).copy() for k, v in drop[0].items()}
    keep = np.ones(len(base_arr["x"]), bool)
    keep[17] = False
    without = engine_counts({k: v[keep] for k, v in base_arr.items()}, 2)
    full = engine_counts(base_arr, 2)
    for prop, ref in (("x", without), ("h", full[keep])):
        arr = {k: v.copy() for k, v in base_arr.items()}
        arr[prop][17] = np.nan
        got = static_counts(arr, 2)
        assert got[17] == -1, prop
        np.testing.assert_array_equal(got[keep], ref, err_msg=prop)
