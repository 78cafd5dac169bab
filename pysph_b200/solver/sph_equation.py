"""SPHOperation / SPHIntegration: build one SPHCalc per destination array
with one function per source array (S/solver/sph_equation.py:10-257)."""
from __future__ import annotations

from ..base.particle_types import ParticleType
from ..sph.sph_calc import SPHCalc
from ..sph.sph_func import SPHFunctionParticle

Fluid = ParticleType.Fluid
Solid = ParticleType.Solid


class SPHOperation:
    def __init__(self, function, on_types, id, updates=(), kernel=None,
                 from_types=(), kernel_correction=-1, integrates=False):
        self.from_types = list(from_types)
        self.on_types = list(on_types)
        self.function = function
        self.updates = list(updates)
        self.id = id
        self.integrates = integrates
        self.kernel = kernel
        self.nbr_info = issubclass(function.get_func_class(), SPHFunctionParticle)
        self.has_kernel_correction = kernel_correction != -1
        self.kernel_correction = kernel_correction
        self.calc_type = SPHCalc

    @staticmethod
    def _matches(arr, types):
        return arr.particle_type in types or arr in types or arr.name in types

    def get_calc_data(self, particles):
        """{dest index: {'sources', 'funcs', 'dnum', 'id', 'snum'}}"""
        if not issubclass(self.function.get_func_class(), SPHFunctionParticle):
            self.nbr_info = False
            if self.from_types:
                raise ValueError(f"Only Subclasses of SPHFunctionParticle need neighbors, "
                                 f"{self.function.get_func_class()} should not provide "
                                 "`from_types` to operation")
        else:
            self.nbr_info = True
        arrays = particles.arrays
        calc_data = {}
        for i, dst in enumerate(arrays):
            if not self._matches(dst, self.on_types):
                continue
            calc_data[i] = {"sources": [], "funcs": [], "dnum": i, "id": "", "snum": str(i)}
            if not self.from_types:
                func = self.function.get_func(dst, dst)
                func.id = self.id
                calc_data[i]["funcs"] = [func]
                calc_data[i]["sources"] = [dst]
                calc_data[i]["id"] = self.id + "_" + dst.name
            else:
                for j, src in enumerate(arrays):
                    if self._matches(src, self.from_types):
                        func = self.function.get_func(source=src, dest=dst)
                        func.id = self.id
                        calc_data[i]["sources"].append(src)
                        calc_data[i]["funcs"].append(func)
                        calc_data[i]["snum"] += str(j)
                        calc_data[i]["id"] = self.id + "_" + dst.name
                if not calc_data[i]["sources"]:
                    raise RuntimeWarning(f"No source found for {self.id} operation")
        return calc_data

    def get_calcs(self, particles, kernel):
        calcs = []
        data = self.get_calc_data(particles)
        for i, dest in enumerate(particles.arrays):
            if i not in data:
                continue
            d = data[i]
            calcs.append(self.calc_type(
                particles=particles, sources=d["sources"], dest=dest, funcs=d["funcs"],
                kernel=kernel, updates=self.updates, integrates=self.integrates,
                dnum=d["dnum"], id=d["id"], dim=kernel.dim, snum=d["snum"],
                kernel_correction=self.kernel_correction, nbr_info=self.nbr_info))
        return calcs


class SPHIntegration(SPHOperation):
    """An integrating SPHOperation: the function computes an acceleration of
    the `updates` properties."""

    def __init__(self, function, on_types, id, updates=(), kernel=None,
                 from_types=(), kernel_correction=-1):
        SPHOperation.__init__(self, function, on_types, id, updates, kernel,
                              from_types=from_types, integrates=True,
                              kernel_correction=kernel_correction)
