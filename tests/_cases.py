"""Shared seeded test cases (velocity meshes, distributions) for the tests."""
import numpy as np

from oracle.collision import VHSTables
from oracle.mesh import VelocityMeshStd, vhs_prefactor

SEED = 20261203


def vhs_case(N, M, Nrho, dev, full_sphere, omega=0.81, nslots=1, noise=0.01,
             seed=SEED):
    vm = VelocityMeshStd(Nv=N, M=M, Nrho=Nrho, dev=dev, full_sphere=full_sphere)
    invKn, prefac = vhs_prefactor(vm, omega, 4.17e-10, 273.)
    gamma = 2.0 * (1 - omega)
    rng = np.random.default_rng(seed)
    f = np.empty((nslots, N ** 3))
    cv = vm.cv
    for s in range(nslots):
        uy = rng.uniform(-0.1, 0.1)
        T = rng.uniform(0.95, 1.05)
        m = np.exp(-(cv[0] ** 2 + (cv[1] - uy) ** 2 + cv[2] ** 2) / T) \
            / (np.pi * T) ** 1.5
        f[s] = m * (1 + noise * rng.uniform(-1, 1, m.shape))
    return vm, prefac, gamma, f


def vhs_tables(vm, gamma):
    return VHSTables(vm.Nv, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, gamma,
                     sphere_factor=vm.sphere_factor)


def op_kwargs(vm, prefac, gamma):
    return dict(N=vm.Nv, L=vm.L, qz=vm.qz, qw=vm.qw, sz=vm.sz, sw=vm.sw,
                sphere_factor=vm.sphere_factor, gamma=gamma, prefac=prefac,
                cw=vm.cw, c0=vm.cv[2, :vm.Nv])
