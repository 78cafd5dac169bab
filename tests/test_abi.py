"""The C ABI library: it loads, exports every entry point include/sphb.h
declares, and the ctypes mirror matches the header's struct layout (checked
against gcc compiling the header).  No device work is done here."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from pysph_b200 import _native as nat
from pysph_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sphb.h")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(nat.LIB_PATH):
        B.build()
    return nat.lib()


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"SPHB_API\s+[\w\s\*]*?\b(sphb_\w+)\s*\(", src)))


def test_header_declares_the_binding(lib):
    names = declared_symbols()
    assert len(names) >= 16
    assert sorted(nat.EXPORTED) == names


def test_every_symbol_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (sphb_\w+)", out))
    for name in declared_symbols():
        assert name in exported, name
        assert getattr(lib, name) is not None


STRUCTS = {
    "sphb_config": (nat.Config, ["dim", "stencil", "num_particles", "rho_src",
                                 "mom_src", "tait_on", "step_on"]),
    "sphb_scene": (nat.Scene, ["cell_size", "g", "static_lo", "static_hi",
                               "use_cfl"]),
    "sphb_scene_state": (nat.SceneState, ["lo", "n", "cell_base", "box", "dt",
                                          "count", "max_acc2"]),
    "sphb_tile": (nat.Tile, ["seg", "end"]),
    "sphb_buffers": (nat.Buffers, ["x", "w0", "h", "idx", "tag"]),
    "sphb_fields": (nat.Fields, ["rho", "thermo", "cell"]),
    "sphb_work": (nat.Work, ["count", "meta", "status", "pairs"]),
    "sphb_engine": (nat.EngineDesc, ["cfg", "seg_offset", "tiles", "num_tiles",
                                     "num_pair_tiles", "buf", "f", "work"]),
}


def test_struct_layout_matches_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sphb.h"',
             "int main(void){"]
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write("\n".join(lines))
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe])
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(l.split() for l in out.strip().splitlines())
    for cname, (cls, fields) in STRUCTS.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for f in fields:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, (cname, f)


def test_host_helpers(lib):
    import numpy as np
    seg = np.array([0, 300, 300, 1000], np.int32)
    n = ctypes.c_int32()
    assert lib.sphb_make_tiles(seg.ctypes.data, 3, 256, None, ctypes.byref(n)) == 0
    assert n.value == 2 + 0 + 3
    tiles = (nat.Tile * n.value)()
    assert lib.sphb_make_tiles(seg.ctypes.data, 3, 256, ctypes.addressof(tiles),
                               ctypes.byref(n)) == 0
    spans = [(t.seg, t.begin, t.end) for t in tiles]
    assert spans == [(0, 0, 256), (0, 256, 300), (2, 300, 556), (2, 556, 812),
                     (2, 812, 1000)]
    cfg = nat.Config()
    cfg.num_particles = 1000
    cfg.cell_capacity = 5000
    offs = (ctypes.c_size_t * 9)()
    total = ctypes.c_size_t()
    assert lib.sphb_workspace_layout(ctypes.byref(cfg), offs, ctypes.byref(total)) == 0
    assert all(o % 256 == 0 for o in offs)
    assert list(offs) == sorted(offs) and total.value > offs[8]
    assert lib.sphb_workspace_layout(None, offs, ctypes.byref(total)) == -1
    # bad arguments are refused without touching the device
    assert lib.sphb_bin(None, 0, 0, None) == -1
    assert lib.sphb_density(None, 0, 1, 1, None) == -1
    assert lib.sphb_make_tiles(None, 1, 256, None, ctypes.byref(n)) == -1


def test_stage_kinds_checked_on_the_host(lib):
    """sphb_pc_stage and sphb_momentum refuse stage kinds outside 0..7, and
    RK4's kinds 4-7 without the running-sum buffers, before any launch.
    The descriptor's pointers are placeholders: the host checks never
    dereference them, and every call here returns before a launch."""
    d = nat.EngineDesc()
    c = d.cfg
    c.dim, c.precision, c.num_scenes, c.num_arrays = 2, nat.FP64, 1, 1
    c.stencil, c.lanes, c.pair_block = 1, 1, 128
    c.num_particles, c.cell_capacity, c.step_on = 10, 100, 1
    c.mom_src[0] = 1
    p = 0x1000
    d.tiles = d.pair_tiles = d.seg_offset = d.scene = d.sstate = p
    d.num_tiles = d.num_pair_tiles = 1
    for name in ("x", "y", "u", "v", "x0", "y0", "u0", "v0", "m", "h", "idx", "tag"):
        setattr(d.buf[0], name, p)
    d.f.au = d.f.av = d.f.dt_fac = p
    e = ctypes.byref(d)
    for kind in (-1, 8):
        assert lib.sphb_pc_stage(e, 0, kind, None) == -1, kind
    assert lib.sphb_pc_stage(e, 0, 4, None) == -1   # RK4 without its sums
    assert lib.sphb_pc_stage(e, 0, 7, None) == -1
    # the fused stage's kind travels in the mode's bits 8-11
    assert lib.sphb_momentum(e, 0, 1, 1, (8 + 1) << 8, None) == -1
    assert lib.sphb_momentum(e, 0, 1, 1, (4 + 1) << 8, None) == -1
