"""Nodal DG bases of the 1-D solvers (host, FP64).

``nodal-sem-gll`` (Lagrange polynomials on Gauss-Lobatto points, lifting by
the boundary quadrature weights) and ``nodal-gll`` (Hesthaven's nodal DG with
mass lumping), as selected by ``[basis] kind`` in the reference
(dgfs1D/basis.py:206-421).  Besides the DG operators, each basis provides the
decomposition of the Galerkin collision tensor
H_mab = int phi_m phi_a phi_b (J. Comput. Phys. 378, 178-208, 2019) that the
drivers use to evaluate Q mode by mode: for nodal bases it is diagonal, so
mode m of Q is Q applied to coefficient m alone (``sigModes[m] == [0]``).
"""
import numpy as np

from .plugins import subclass_where
from .quadrature import (gauss_lobatto_jacobi, lagrange_at, lagrange_deriv_at,
                         legendre_orthonormal)


def _filter(mat, tol=1e-15):
    mat = np.array(mat, dtype=np.float64)
    mat[np.abs(mat) < tol] = 0.0
    return mat


class Basis:
    basis_kind = None

    def __init__(self, cfg):
        self.cfg = cfg
        self.K = cfg.lookupint('basis', 'K')
        self.Nq = self.K
        Nqr = cfg.lookupint('basis', 'Nqr')
        self.z, self.w = gauss_lobatto_jacobi(self.K)
        zr, _ = gauss_lobatto_jacobi(Nqr)
        self.interpMat = lagrange_at(self.z, zr).T          # (K, Nqr)
        self.derivMat = lagrange_deriv_at(self.z, self.z).T
        self._build()
        # SVD of the (inverse-mass weighted) collision tensor, per mode
        self.U, self.V, self.sigModes = [], [], []
        for m in range(self.K):
            u, s, vt = np.linalg.svd(self._invM_H[m])
            Um, Vm = _filter(u), _filter(np.diag(s) @ vt)
            nnzU = np.where(np.sum(Um, axis=0) != 0)[0]
            nnzV = np.where(np.sum(Vm, axis=1) != 0)[0]
            self.U.append(Um)
            self.V.append(Vm)
            self.sigModes.append(np.intersect1d(nnzU, nnzV))
        self.faceOp = _filter(self.Bqf.T)          # (Nqf, K) face traces
        self.derivOp = _filter(self.derivMat)      # ux = derivOp . u
        self.invMassOp = _filter(self.invMassMat)
        # slope-limiter operators (dgfs1D/basis.py:289-301): projections onto
        # the Legendre mode 0 (cell average) and modes 0-1 (linear part, then
        # differentiated), as the nodal values of each element
        Vo = legendre_orthonormal(self.K, self.z).T
        invV = np.linalg.inv(Vo)
        A0, A1 = Vo.copy(), Vo.copy()
        A0[:, 1:] = 0.0
        A1[:, 2:] = 0.0
        self.cellAvgOp = _filter(A0 @ invV)
        self.drLinOp = _filter(self.derivMat @ (A1 @ invV))

    def upwind_ops(self, sigma=-1):
        """Applied volume operators of the upwind summation-by-parts
        discretisation (dgfs1D/basis.py:304-312): (Dm^T, Dp^T) with
        Dp/m = D +- S P^-1 / 2, D = derivMat^T, P = diag(w) and S = sigma q q^T,
        q the last column of the QR factor of the Legendre Vandermonde.  The
        first is used where c_x > 0, the second where c_x < 0."""
        V = legendre_orthonormal(self.K, self.z).T
        Q, _ = np.linalg.qr(V)
        sig = np.zeros(self.K)
        sig[-1] = sigma
        S = Q @ np.diag(sig) @ Q.T
        invP = np.diag(1.0 / self.w)
        D = self.derivMat.T
        Dp, Dm = D + 0.5 * S @ invP, D - 0.5 * S @ invP
        return _filter(Dm.T), _filter(Dp.T)

    def mode_sources(self):
        """For nodal bases: the coefficient slot feeding each (m, r) term.

        Returns [(m, a)] when U[m][:, r] and V[m][r, :] are the same signed
        unit vector e_a (to 1e-12) for the single significant r, so
        Q(U^T u, V u) at mode m equals Q(u_a, u_a) (Q is quadratic /
        bilinear and the signs cancel).  Raises for bases without that
        structure.
        """
        out = []
        for m in range(self.K):
            if len(self.sigModes[m]) != 1:
                raise NotImplementedError('only diagonal collision tensors')
            r = int(self.sigModes[m][0])
            col, row = self.U[m][:, r], self.V[m][r, :]
            a = int(np.argmax(np.abs(col)))
            unit = np.zeros(self.K)
            unit[a] = 1.0
            if not (np.allclose(np.abs(col), unit, rtol=0, atol=1e-12)
                    and np.allclose(np.abs(row), unit, rtol=0, atol=1e-12)
                    and np.sign(col[a]) == np.sign(row[a])):
                raise NotImplementedError('only diagonal collision tensors')
            out.append((m, a))
        return out


class NodalSemGLL(Basis):
    basis_kind = 'nodal-sem-gll'

    def _build(self):
        K = self.K
        B = lagrange_at(self.z, self.z).T
        M = np.einsum('mq,q,lq->ml', B, self.w, B)
        invM = np.linalg.inv(M)
        H = np.einsum('mq,aq,bq,q->mab', B, B, B, self.w)
        self._invM_H = np.einsum('ml,mab->lab', invM, H)
        self.Nqf = 2
        zqf, _ = gauss_lobatto_jacobi(2)
        self.Bqf = lagrange_at(self.z, zqf).T               # (K, 2)
        self.gLD = self.Bqf[:, 0] / self.w[0]
        self.gRD = self.Bqf[:, -1] / self.w[-1]
        self.invMassMat = B.T


class NodalGLL(Basis):
    basis_kind = 'nodal-gll'

    def _build(self):
        K = self.K
        I = np.eye(K)
        B = legendre_orthonormal(K, self.z).T
        invM = B @ B.T
        self._invM_H = np.einsum('mq,aq,bq->mab', I, I, I)
        self.Nqf = K
        self.Bqf = I
        self.gLD, self.gRD = invM[0, :], invM[-1, :]
        self.invMassMat = I


def get_basis(cfg):
    return subclass_where(Basis, basis_kind=cfg.lookup('basis', 'kind'))(cfg)
