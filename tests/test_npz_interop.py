"""The solver output format v1 across this build and the reference
(S/solver/utils.py:34-186, 294-340; S/solver/solver.py:605-739), pinned by
files the reference itself wrote and read (tests/golden/make_golden.py,
npz_interop):

* npz_ref_written.npz was written by the reference's own savez from the
  dicts its Solver.dump_output assembles: this build's load must read
  it back to the same arrays and solver data;
* npz_repo_written.npz was written by this build's Solver.dump_output and
  read by the reference's own load, which saw what npz_ref_read.npz
  records: this build must still write the same file, and what the
  reference read must be the arrays that went in.

The workload is the dam break at dx = 0.1 (fluid and wall) with dt = 1e-4,
t = 0.25, count = 7.  CPU only.
"""
import os

import numpy as np
import pytest

import pysph_b200.base.api as base
from pysph_b200 import workloads as W
from pysph_b200.solver import utils
from pysph_b200.solver.solver import Solver

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PROPS = ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "cs")
NAMES = ("fluid", "wall")


def arrays_in():
    """The particle arrays that went into both files, built with this
    build's get_particle_array (the reference's defaults)."""
    arrays, types, _ = W.dam_break(dx=0.1)
    return [base.get_particle_array(name=n, type=t, device="cpu",
                                    **{k: np.asarray(a[k], np.float64) for k in PROPS})
            for a, n, t in zip(arrays, NAMES, types)]


def expected():
    return {pa.name: pa.get_property_arrays(all=False) for pa in arrays_in()}


def _assert_props_equal(got: dict, want: dict, where):
    assert sorted(got) == sorted(want), where
    for k in want:
        np.testing.assert_array_equal(np.asarray(got[k]), np.asarray(want[k]),
                                      err_msg=f"{where}: {k}")


def test_load_reads_the_reference_written_file():
    d = utils.load(os.path.join(GOLD, "npz_ref_written.npz"), device="cpu")
    assert d["solver_data"] == {"dt": 1e-4, "t": 0.25, "count": 7}
    want = expected()
    for name in NAMES:
        pa = d["arrays"][name]
        got = {p: pa.get(p).numpy() for p in pa.get_property_names()}
        got.update(pa.constants)
        _assert_props_equal(got, want[name], name)


def _npz_content(path):
    z = np.load(path, allow_pickle=True)
    out = {k: z[k] for k in z.files}
    out["arrays"] = out["arrays"].reshape(1)[0]
    out["solver_data"] = out["solver_data"].reshape(1)[0]
    return out


def test_dump_output_writes_what_the_reference_read(tmp_path):
    s = Solver(dim=2)
    s.particles = base.Particles(arrays_in())
    s.t, s.count = 0.25, 7
    s.output_directory = str(tmp_path)
    s.fname = "out"
    path = s.dump_output(1e-4)
    now = _npz_content(path)
    then = _npz_content(os.path.join(GOLD, "npz_repo_written.npz"))
    assert sorted(now) == sorted(then) == ["arrays", "solver_data", "version"]
    assert int(now["version"]) == int(then["version"]) == 1
    assert now["solver_data"] == then["solver_data"]
    for name in NAMES:
        _assert_props_equal(now["arrays"][name], then["arrays"][name], name)
    # what the reference's load made of that file
    g = dict(np.load(os.path.join(GOLD, "npz_ref_read.npz")))
    assert (g["solver_dt"], g["solver_t"], g["solver_count"]) == (1e-4, 0.25, 7)
    want = expected()
    for name in NAMES:
        names = [str(n) for n in g[f"{name}__names"]]
        assert sorted(names) == sorted(want[name]), name
        _assert_props_equal({n: g[f"{name}_{n}"] for n in names}, want[name], name)


def test_load_output_resumes_from_the_reference_written_file(tmp_path):
    """Solver.load_output on a file of the reference's name pattern sets
    the arrays' properties, t and count."""
    import shutil
    shutil.copy(os.path.join(GOLD, "npz_ref_written.npz"), tmp_path / "ref_7.npz")
    pas = arrays_in()
    for pa in pas:
        pa.set(x=pa.get("x") * 0.0)
    s = Solver(dim=2)
    s.particles = base.Particles(pas)
    s.output_directory = str(tmp_path)
    s.fname = "ref"
    assert s.load_output("?") == [7]
    s.load_output(7)
    assert (s.t, s.count) == (0.25, 7)
    want = expected()
    for pa in pas:
        np.testing.assert_array_equal(pa.get("x").numpy(), want[pa.name]["x"])
