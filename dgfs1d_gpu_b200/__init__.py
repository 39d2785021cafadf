"""B200 (sm_100a) fast-spectral Boltzmann collision operators for DGFS.

Drop-in for the scattering-model and integrator plugins of dgfsStd1D /
dgfsBi1D / dgfsABstd1D: the collision operator Q(f,f) (VHS/HS single species,
VSS binary mixture), the DG advection right-hand side and the explicit /
IMEX stage updates, computed by hand-written CUDA kernels behind the C ABI of
``libdgfs_sm100.so`` (include/dgfs_sm100.h).
"""
__version__ = '0.1.0'
