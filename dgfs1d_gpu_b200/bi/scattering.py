"""Mixture scattering-model plugins (``[scattering-model] type``).

``vss`` keeps the constructor, parameters and ``fs(idx, d_f1, d_f2, d_Q,
elem, upt, uptout)`` of dgfs1D/bi/scattering.py:47-321 (idx = 'pq'; Q_pq is
accumulated into d_Q).  Precomputation of the pair weights runs on the GPU.
``[scattering-model] precision-mode = fp64|fp32`` selects the operator's
arithmetic (default: fp64 for double, fp32 for float configurations).
"""
import itertools as it
from math import gamma

import numpy as np

from ..collision import VSSOperator
from ..sphericaldesign import get_sphquadrule


class DGFSScatteringModelBi:
    scattering_model = None

    def __init__(self, cfg, velocitymesh, **kwargs):
        self.cfg = cfg
        self.vm = velocitymesh
        self._nspcs = self.vm.nspcs()
        self.load_parameters()
        self.perform_precomputation()


class DGFSBiVSSScatteringModel(DGFSScatteringModelBi):
    scattering_model = 'vss'

    def __init__(self, cfg, velocitymesh, **kwargs):
        self._Ne = kwargs.get('Ne')
        self._max_evals = kwargs.get('max_evals', 64)
        super().__init__(cfg, velocitymesh, **kwargs)

    def load_parameters(self):
        cfg, vm = self.cfg, self.vm
        ssrulepre = cfg.lookup('scattering-model', 'ssrulepre')
        self._Mpre = cfg.lookupint('scattering-model', 'Mpre')
        self._szpre = get_sphquadrule('symmetric', rule=ssrulepre,
                                      npts=self._Mpre).pts
        self._cases = list(it.product(range(self._nspcs), repeat=2))
        ns = self._nspcs
        self._gamma = np.zeros((ns, ns))
        self._eta = np.zeros((ns, ns))
        self._prefactor = np.zeros((ns, ns))
        m = vm.masses()
        for p, q in self._cases:
            pq = f'{p}{q}'
            alpha = cfg.lookupfloat('scattering-model', 'alpha' + pq)
            omega = cfg.lookupfloat('scattering-model', 'omega' + pq)
            dRef = cfg.lookupfloat('scattering-model', 'dRef' + pq)
            Tref = cfg.lookupfloat('scattering-model', 'Tref' + pq)
            self._eta[p, q] = alpha - 1.
            self._gamma[p, q] = 2.0 * (1. - omega)
            invKn = (np.sqrt(1. + m[p] / m[q]) * np.pi * vm.n0() * dRef * dRef
                     * pow(Tref / vm.T0(), omega - 0.5) * vm.H0())
            mu = m[p] * m[q] / (m[p] + m[q])
            self._prefactor[p, q] = invKn * alpha / (
                np.sqrt(1. + m[p] / m[q]) * pow(mu, omega - 0.5)
                * pow(2., 1 + alpha) * gamma(2.5 - omega) * np.pi)

    @property
    def prefac(self):
        return {f'{p}{q}': self._prefactor[p, q] for p, q in self._cases}

    def perform_precomputation(self):
        vm = self.vm
        default = 'fp64' if self.cfg.dtype == np.float64 else 'fp32'
        prec = self.cfg.lookupordefault('scattering-model', 'precision-mode',
                                        default)
        self._op = VSSOperator(vm.Nv(), vm.L(), vm.qz(), vm.qw(), vm.sz(),
                               vm.sw(), self._szpre, vm.masses(), self._gamma,
                               self._eta, self._prefactor,
                               max_evals=self._max_evals, precision=prec)

    @property
    def operator(self):
        return self._op

    def fs(self, idx, d_arr_in1, d_arr_in2, d_arr_out, elem, upt, uptout):
        p, q = int(idx[0]), int(idx[1])
        Ne = self._Ne
        self._op.eval(p, q, d_arr_in1, d_arr_in2, d_arr_out,
                      src_base=upt * Ne + elem, dst_base=uptout * Ne + elem,
                      nevals=1)

    def fs_batch(self, p, q, d_fp, d_fq, d_Qp, src, dst, stream=None):
        self._op.eval(p, q, d_fp, d_fq, d_Qp, src=src, dst=dst, stream=stream)

    def fs_batch_species(self, p, d_fs, d_Qp, src, dst, stream=None):
        """Q_p[dst] += sum_q Q_pq(f_p[src], f_q[src]): the partner loop of
        bi.py:336-342 in one call."""
        self._op.eval_species(p, d_fs, d_Qp, src=src, dst=dst, stream=stream)
