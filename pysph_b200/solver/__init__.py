"""Operations, integrators and the solver loop (the reference's
pysph.solver)."""
