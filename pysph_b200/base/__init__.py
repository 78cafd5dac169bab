"""Particle containers, kernels and the neighbour-search view of the API
(the reference's pysph.base)."""
