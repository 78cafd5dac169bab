"""SPH functions and calcs of the particle-update path (the reference's
pysph.sph)."""
