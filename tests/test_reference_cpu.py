"""The oracle port against the reference's own Cython path run here, through
the driver the bench's CPU reference leg uses (oracle/reference.py; the
reference built by oracle/build_reference.py into oracle/_ref/refbuild --
skipped where that build is absent): the same predictor-corrector steps
give the same states bit for bit, on the dam break at dx = 0.05 with the CFL
rule and on the elliptical drop with a fixed dt.  CPU only."""
import numpy as np
import pytest

from helpers import oracle_from
from oracle import reference as ref
from pysph_b200 import workloads as W
from pysph_b200.engine import fluid_scheme

pytestmark = pytest.mark.skipif(not ref.available(),
                                reason="the reference's Cython build is absent")


def run_both(arrays, types, params, scheme, steps):
    pas, step = ref.stepper(arrays, types, params, 2)
    osys = oracle_from(arrays, params, scheme, 2)
    cfl = params.get("cfl", 0.0) > 0.0
    for _ in range(steps):
        step()
        if cfl:
            osys.pc_step(osys.cfl_time_step(params["cfl"], params["c0"], params["dt_initial"]))
        else:
            osys.pc_step(params["dt"])
    return pas, osys


@pytest.mark.parametrize("case", ["dam", "drop"])
def test_port_reproduces_the_reference_step_by_step(case):
    if case == "dam":
        arrays, types, params = W.dam_break(dx=0.05)
        scheme, steps = fluid_scheme(2), 3
    else:
        arrays, types, params = W.elliptical_drop(dx=0.05)
        params = dict(params, dt=1e-5)
        scheme, steps = fluid_scheme(1), 5
    pas, osys = run_both(arrays, types, params, scheme, steps)
    for pa, oa in zip(pas, osys.arrays):
        for n in ("x", "y", "u", "v", "rho", "p"):
            np.testing.assert_array_equal(np.asarray(pa.get(n)), getattr(oa, n), err_msg=n)


def test_timed_leg_reports_a_rate():
    arrays, types, params = W.elliptical_drop(dx=0.05)
    r = ref.time_steps(arrays, types, dict(params, dt=1e-5), 2, steps=2, warmup=1)
    assert r["steps"] == 2 and r["seconds"] > 0 and r["particles"] == len(arrays[0]["x"])
