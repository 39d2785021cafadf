"""Shared seeded test cases (velocity meshes, distributions) for the tests."""
from dgfs1d_gpu_b200.workloads import couette_distributions, vhs_mesh_params
from oracle.collision import VHSTables
from oracle.mesh import VelocityMeshStd, vhs_prefactor

SEED = 20261203


def vhs_case(N, M, Nrho, dev, full_sphere, omega=0.81, nslots=1, noise=0.01,
             seed=SEED):
    """Oracle mesh, prefactor, gamma and seeded distributions."""
    vm = VelocityMeshStd(Nv=N, M=M, Nrho=Nrho, dev=dev, full_sphere=full_sphere)
    invKn, prefac = vhs_prefactor(vm, omega, 4.17e-10, 273.)
    gamma = 2.0 * (1 - omega)
    f = couette_distributions(vm.cv[2, :N], nslots, noise=noise, seed=seed)
    return vm, prefac, gamma, f


def vhs_tables(vm, gamma):
    return VHSTables(vm.Nv, vm.L, vm.qz, vm.qw, vm.sz, vm.sw, gamma,
                     sphere_factor=vm.sphere_factor)


def op_kwargs(vm, prefac, gamma):
    return dict(N=vm.Nv, L=vm.L, qz=vm.qz, qw=vm.qw, sz=vm.sz, sw=vm.sw,
                sphere_factor=vm.sphere_factor, gamma=gamma, prefac=prefac,
                cw=vm.cw, c0=vm.cv[2, :vm.Nv])
