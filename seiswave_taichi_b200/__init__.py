"""seiswave_taichi_b200 -- B200 (sm_100a) elastic staggered-grid finite-difference
time loop, a drop-in for SeisWave_Taichi's ElasticWAVE classes.

Modules named like the reference's (src/...):
  Elastic2D_CPML        2D P-SV, schemes SSG_VS / SSG_SV / RSG, ADE-CPML
  Elastic3D_SSG_CPML    3D SSG, ADE-CPML, point force
  Elastic3D_SSG_Tensor  3D SSG, ADE-CPML, moment tensor, receiver arrays
  Elastic3D_SSG_SPML    3D SSG, split-field PML
  BaseFun               Ricker / Ricker2 / Ricker3 wavelets
  pml                   diff_coff, diff_coff_op, SetADEPML profiles
The kernels live in lib/libseiswave.so (C ABI: include/seiswave.h), built by
build_native.py; there is no CPU fallback.
"""
__version__ = "0.1.0"
