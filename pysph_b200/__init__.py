"""pysph_b200 -- B200-native (sm_100a) particle-update path of PySPH.

The CUDA engine (pysph_b200.engine, C ABI in include/sphb.h) carries
cell-binned neighbour search, summation density + Tait EOS, momentum
(pressure gradient + Monaghan artificial viscosity) + gravity and the
predictor-corrector integrator for batches of scenes.  The reference-shaped
API lives in pysph_b200.base / .sph / .solver.
"""
__version__ = "0.1.0"
