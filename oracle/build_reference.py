"""Build the reference's own FP64 Cython particle path (PySPH 0.9beta) in a
scratch directory: the checker behind the golden fixtures of tests/golden
and the reference that bench.py times on the host.

    python oracle/build_reference.py --ref <reference checkout> [--out oracle/_ref/refbuild]

The reference location comes from --ref or the PYSPH_REFERENCE environment
variable (there is no default); the build goes to oracle/_ref/refbuild,
which git ignores.

The snapshot is Python 2 / Cython 0.14-era and must be patched mechanically
to build with Python 3.12 and Cython 3: Python-2 syntax and dict methods in
the pure-Python modules (and, in the output format's reader, numpy.load's
allow_pickle for the pickled dicts), numpy aliases, `cpdef inline`, `except -1`
mismatches between .pyx and .pxd, a Cython-3 name-mangling clash, and two
bugs of the snapshot itself (nnps.pyx reads CellManager.coord_x/y/z, which no
longer exist; Particles passes max_radius_scale= / periodic_domain= where
CellManager takes radius_scale= / domain=).  OpenCL-only modules the path
imports (cl_utils, locator, domain_manager) are replaced by stubs: this build
never takes the OpenCL path.  No arithmetic of the particle path is changed.

Nothing here is imported by the product; the build output stays in the
scratch directory (git-ignored) and is used only by the golden-fixture
script and bench.py's CPU legs (through oracle/reference.py).  An existing
build is kept unless --force is given.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

MODULES = [
    "base/carray", "base/fast_utils", "base/point", "base/particle_array",
    "base/polygon_array", "base/kernels", "base/cell", "base/nnps",
    "sph/sph_func", "sph/kernel_correction", "sph/sph_calc",
    "sph/funcs/common", "sph/funcs/basic_funcs", "sph/funcs/density_funcs",
    "sph/funcs/eos_funcs", "sph/funcs/pressure_funcs", "sph/funcs/viscosity_funcs",
    "sph/funcs/position_funcs", "sph/funcs/external_force",
    "sph/funcs/xsph_funcs", "sph/funcs/arithmetic_funcs",
]

STUB_CL_UTILS = '''"""Stub of pysph.solver.cl_utils for a build without OpenCL."""
import numpy
from os import path
HAS_CL = False
def get_real(val, precision):
    return numpy.float64(val)
def get_cl_include():
    return ""
def get_scalar_buffer(val, precision, ctx):
    return None
def get_pysph_root():
    return path.split(path.split(path.abspath(__file__))[0])[0]
def cl_read(filename, precision="double", function_name=None):
    return ""
def get_real_type(precision):
    return "double"
def get_type(precision):
    return numpy.float64
def enqueue_copy(*a, **k):
    raise RuntimeError("no OpenCL in this build")
def create_some_context():
    raise RuntimeError("no OpenCL in this build")
'''

STUB_LOCATOR = '''"""Stub of pysph.base.locator (OpenCL neighbour locators)."""
class OpenCLNeighborLocatorType:
    AllPairNeighborLocator = 0
    LinkedListSPHNeighborLocator = 1
    RadixSortNeighborLocator = 2
class OpenCLNeighborLocator(object):
    pass
class AllPairNeighborLocator(OpenCLNeighborLocator):
    pass
class LinkedListSPHNeighborLocator(OpenCLNeighborLocator):
    pass
class RadixSortNeighborLocator(OpenCLNeighborLocator):
    pass
'''

STUB_DOMAIN_MANAGER = '''"""Stub of pysph.base.domain_manager (OpenCL domain managers)."""
class DomainManagerType:
    DomainManager = 0
    LinkedListManager = 1
    RadixSortManager = 2
class DomainManager(object):
    pass
class LinkedListManager(DomainManager):
    pass
class RadixSortManager(DomainManager):
    pass
'''


def sub(path, pattern, repl, count=0, flags=0, required=True):
    s = open(path).read()
    s2, n = re.subn(pattern, repl, s, count=count, flags=flags)
    if required and n == 0:
        raise RuntimeError(f"patch found nothing in {path}: {pattern}")
    open(path, "w").write(s2)


def patch_common(pkg):
    """Mechanical Python-3 / Cython-3 fixes over every source file."""
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            p = os.path.join(dirpath, f)
            if not f.endswith((".pyx", ".pxd", ".py")):
                continue
            s = open(p).read()
            o = s
            s = re.sub(r"\bcpdef inline\b", "cpdef", s)
            s = re.sub(r"numpy\.float\b(?!\d|_)", "numpy.float64", s)
            s = re.sub(r"numpy\.int\b(?!\d|_|c)", "numpy.int64", s)
            s = re.sub(r"numpy\.long\b", "numpy.int64", s)
            s = re.sub(r"\bnp\.float\b(?!\d|_)", "np.float64", s)
            s = re.sub(r"\bnp\.int\b(?!\d|_|c)", "np.int64", s)
            s = re.sub(r"\.iteritems\(\)", ".items()", s)
            s = re.sub(r"\.itervalues\(\)", ".values()", s)
            s = re.sub(r"\.iterkeys\(\)", ".keys()", s)
            s = re.sub(r"(\w[\w\.\[\]'\"]*)\.has_key\(([^()]*)\)", r"(\2 in \1)", s)
            s = re.sub(r"raise (\w+), (.+)$", r"raise \1(\2)", s, flags=re.M)
            s = re.sub(r"^(\s*)print (?!\()(.*)$", r"\1print(\2)", s, flags=re.M)
            s = re.sub(r"except (\w+), (\w+):", r"except \1 as \2:", s)
            s = re.sub(r"__gradient\b", "py_gradient_scalar", s)
            if f.endswith(".pyx"):
                # buffer dtypes must be C types
                s = re.sub(r"(ndarray\[[^\]]*dtype\s*=\s*(?:numpy|np)\.(?:float64|int64))\]",
                           r"\1_t]", s)
                s = re.sub(r"\b(numpy|np)\.int_t\b", r"\1.int64_t", s)
                s = re.sub(r"\b(numpy|np)\.float_t\b", r"\1.float64_t", s)
                # dict views are not lists in Python 3
                s = re.sub(r"(?<![\w\.])((?:self\.)?[\w]+(?:\.\w+)*)\.(keys|values)\(\)",
                           r"list(\1.\2())", s)
            if s != o:
                open(p, "w").write(s)


def patch_specific(pkg):
    B = os.path.join(pkg, "base")
    S = os.path.join(pkg, "sph")
    # stubs for the OpenCL-only modules
    open(os.path.join(pkg, "solver", "cl_utils.py"), "w").write(STUB_CL_UTILS)
    open(os.path.join(B, "locator.py"), "w").write(STUB_LOCATOR)
    open(os.path.join(B, "domain_manager.py"), "w").write(STUB_DOMAIN_MANAGER)
    # `except -1` declared in the .pxd but not at the definition
    sub(os.path.join(B, "cell.pyx"),
        r"(cdef int get_potential_cells\(self, cPoint pnt, double radius,\s*list cell_list\))",
        r"\1 except -1")
    sub(os.path.join(B, "cell.pyx"), r"(cpdef int update_status\(self, bint variable_h\))",
        r"\1 except -1")
    sub(os.path.join(B, "particle_array.pyx"),
        r"(cpdef int append_parray\(self, ParticleArray parray\))", r"\1 except -1")
    # PyString_AsString(str) comparisons -> str comparisons
    p = os.path.join(B, "particle_array.pyx")
    sub(p, r"strcmp\(PyString_AsString\(data_type\), '(\w+)'\) == 0", r"data_type == '\1'")
    sub(p, r"%PyString_AsString\(data_type\)", "%data_type")
    # snapshot bug: CellManager lost coord_x/y/z
    sub(os.path.join(B, "nnps.pyx"), r"self\.cell_manager\.coord_x", "'x'")
    sub(os.path.join(B, "nnps.pyx"), r"self\.cell_manager\.coord_y", "'y'")
    sub(os.path.join(B, "nnps.pyx"), r"self\.cell_manager\.coord_z", "'z'")
    # snapshot bug: Particles passes kwargs CellManager does not take
    sub(os.path.join(B, "particles.py"), r"max_radius_scale=self\.max_radius_scale",
        "radius_scale=self.max_radius_scale")
    sub(os.path.join(B, "particles.py"), r"periodic_domain=self\.periodic_domain",
        "domain=self.periodic_domain")
    # the output format's reader and writer (S/solver/utils.py): the unused
    # Python-2 `commands` module, `basestring`, and numpy.load of the
    # pickled dicts, which numpy >= 1.16.3 refuses without allow_pickle
    U = os.path.join(pkg, "solver", "utils.py")
    sub(U, r"^import commands$", "", flags=re.M)
    sub(U, r"\bbasestring\b", "str")
    sub(U, r"numpy\.load\(fname\)", "numpy.load(fname, allow_pickle=True)")
    # implicit relative imports of the pure-Python modules
    for f, mods in (("base/particles.py", ["cell", "nnps", "particle_array",
                                            "particle_types", "domain_manager", "locator"]),
                    ("solver/sph_equation.py", []), ("solver/integrator.py", [])):
        p = os.path.join(pkg, f)
        for m in mods:
            sub(p, rf"^from {m} import", f"from pysph.base.{m} import", flags=re.M,
                required=False)
            sub(p, rf"^import {m}$", f"import pysph.base.{m} as {m}", flags=re.M,
                required=False)


SETUP = '''
import numpy
from setuptools import setup, Extension
from Cython.Build import cythonize
mods = {mods!r}
exts = [Extension(m.replace("/", "."), [m + ".pyx"], include_dirs=[numpy.get_include(), "."],
                  language="c++", extra_compile_args=["-O2", "-ffp-contract=off", "-w"])
        for m in ["pysph/" + x for x in mods]]
setup(name="pysph_ref", ext_modules=cythonize(exts, language_level=2, quiet=True,
      compiler_directives={{"legacy_implicit_noexcept": True}}))
'''


def build(ref, out, force=False):
    """Build the reference from the checkout `ref` into `out` (kept when
    already built, unless force)."""
    sys.path.insert(0, ROOT)
    from oracle.reference import available
    if not force and available(out):
        return out
    src = os.path.join(ref, "source", "pysph")
    os.makedirs(out, exist_ok=True)
    pkg = os.path.join(out, "pysph")
    if os.path.exists(pkg):
        shutil.rmtree(pkg)
    shutil.copytree(src, pkg)
    patch_common(pkg)
    patch_specific(pkg)
    open(os.path.join(out, "setup_ref.py"), "w").write(SETUP.format(mods=MODULES))
    r = subprocess.run([sys.executable, "setup_ref.py", "build_ext", "--inplace", "-j", "8"],
                       cwd=out, capture_output=True, text=True)
    open(os.path.join(out, "build.log"), "w").write(r.stdout + r.stderr)
    if r.returncode != 0:
        tail = (r.stdout + r.stderr)[-6000:]
        raise RuntimeError("reference build failed:\n" + tail)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PYSPH_REFERENCE"),
                    help="the reference checkout (default: $PYSPH_REFERENCE)")
    ap.add_argument("--out", default=os.path.join(ROOT, "oracle", "_ref", "refbuild"))
    ap.add_argument("--force", action="store_true", help="rebuild an existing build")
    a = ap.parse_args()
    if not a.ref:
        ap.error("name the reference checkout with --ref or PYSPH_REFERENCE")
    print(build(a.ref, a.out, a.force))
