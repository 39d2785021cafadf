"""Oracle restatement of the single-species DG solver around Q (float64).

Test infrastructure only (see ``oracle/__init__.py``).  Follows
dgfs1D/std/std.py:37-423 (driver and ``rhs``), dgfs1D/std/kernels/std.mako
(face extraction, upwind flux, lifting), dgfs1D/basis.py:206-421 (nodal
bases), dgfs1D/std/bc.py + kernels/bcs/*.mako (boundary conditions),
dgfs1D/std/integrator.py (explicit schemes), dgfs1D/axnpby.py and
dgfs1D/std/moments.py:11-70 (bulk moments).
"""
import numpy as np

from .mesh import (gauss_lobatto_jacobi, jac_nodal_basis_at, nodal_basis_at,
                   ortho_basis_at)


def filter_tol(mat, tol=1e-15):
    """Zero entries below tol, as the gimmik kernels see them (util.py:16-18)."""
    mat = np.array(mat, dtype=np.float64)
    mat[abs(mat) < tol] = 0.
    return mat


class NodalBasis:
    """``nodal-sem-gll`` (basis.py:206-329) and ``nodal-gll`` (333-421)."""

    def __init__(self, kind, K, Nqr):
        self.kind, self.K = kind, K
        z, w = gauss_lobatto_jacobi(K, 0., 0.)
        self.z, self.w = z, w
        I = np.eye(K)
        zr, _ = gauss_lobatto_jacobi(Nqr, 0., 0.)
        self.interpMat = nodal_basis_at(K, z, zr).T
        D = jac_nodal_basis_at(K, z, z)
        self.derivMat = D.T
        if kind == 'nodal-sem-gll':
            B = nodal_basis_at(K, z, z).T
            M = np.einsum('mq,q,lq->ml', B, w, B)
            invM = np.linalg.inv(M)
            H = np.einsum('mq,aq,bq,q->mab', B, B, B, w)
            invM_H = np.einsum('ml,mab->lab', invM, H)
            self.Nqf = 2
            zqf, _ = gauss_lobatto_jacobi(2, 0., 0.)
            self.Bqf = nodal_basis_at(K, z, zqf).T
            self.gLD = self.Bqf[:, 0] / w[0]
            self.gRD = self.Bqf[:, -1] / w[-1]
            self.invMassMat = B.T
        elif kind == 'nodal-gll':
            B = ortho_basis_at(K, z).T
            invM = B @ B.T
            invM_H = np.einsum('mq,aq,bq->mab', I, I, I)
            self.Nqf = K
            self.Bqf = I
            self.gLD, self.gRD = invM[0, :], invM[-1, :]
            self.invMassMat = I
        else:
            raise ValueError(kind)
        U, V, sig = [], [], []
        for m in range(K):
            u, s, v = np.linalg.svd(invM_H[m, :, :])
            Um, Vm = filter_tol(u), filter_tol(np.dot(np.diag(s), v))
            nnzU = np.where(np.sum(Um, axis=0) != 0)[0]
            nnzV = np.where(np.sum(Vm, axis=1) != 0)[0]
            U.append(Um)
            V.append(Vm)
            sig.append(np.intersect1d(nnzU, nnzV))
        self.U, self.V, self.sigModes = U, V, sig
        # slope-limiter operators (basis.py:289-301): projection onto the
        # Legendre mode 0 (cell average) and modes 0-1 (linear part),
        # differentiated with the nodal derivative
        Vo = ortho_basis_at(K, z).T
        invV = np.linalg.inv(Vo)
        A0 = Vo.copy()
        A0[:, 1:] = 0
        A1 = Vo.copy()
        A1[:, 2:] = 0
        self.cellAvgOp = filter_tol(A0 @ invV)
        self.drLinOp = filter_tol(D.T @ (A1 @ invV))
        # the operators as the kernels apply them (C = A . B, filtered)
        self.bwdFaceOp = filter_tol(self.Bqf.T)      # (Nqf, K)
        self.derivOp = filter_tol(D.T)               # (K, K): ux = D^T u
        self.invMassOp = filter_tol(self.invMassMat)


def classic_mesh(xlo, xhi, Ne, H0):
    """``Mesh.classic`` + non-dimensionalisation (mesh.py:10-18, 88-128)."""
    xmesh = np.linspace(xlo, xhi, Ne + 1) / H0
    h = np.diff(xmesh).reshape(-1, 1)
    return xmesh, h / 2., 2. / h


def face_maps(Ne, Nqf):
    """mapL/mapR of std.py:63-66."""
    mapL, mapR = np.arange(Ne + 1) + (Nqf - 1) * Ne - 1, np.arange(Ne + 1)
    mapL[0], mapR[-1] = 0, Ne * Nqf - 1
    return mapL, mapR


class WallDiffuseBC:
    """Purely diffuse wall (std/bc.py:25-78, dgfs-wall-diffuse.mako)."""

    def __init__(self, cv, cw, T, u, nl):
        self.cx, self.cw, self.nl = cv[0], cw, nl
        self.ux = u[0]
        self.f0 = (1.0 / (np.pi * T) ** 1.5) * np.exp(
            -np.sum((cv - np.reshape(u, (3, 1))) ** 2, axis=0) / T)
        self.nden = None

    def update(self, ul):
        fac = (self.cx - self.ux) * self.nl
        num = (fac >= 0.) * (fac * ul * self.cw)
        den = (fac < 0.) * (fac * self.f0 * self.cw)
        self.nden = -(np.sum(num) / np.sum(den))

    def apply(self, ul):
        fac = (self.cx - self.ux) * self.nl
        return (fac < 0) * (self.f0 * self.nden) + (fac >= 0) * ul


class InletBC:
    """Inlet: incoming from a fixed Maxwellian (dgfs-inlet.mako); with
    ``shift`` = u_x the incoming test is (c_x - u_x) n < 0
    (dgfs-inlet-nondim.mako)."""

    def __init__(self, cv, rho, T, u, nl, shift=0.0):
        self.cx, self.nl, self.shift = cv[0], nl, shift
        self.f0 = (rho / (np.pi * T) ** 1.5) * np.exp(
            -np.sum((cv - np.reshape(u, (3, 1))) ** 2, axis=0) / T)

    def update(self, ul):
        pass

    def apply(self, ul):
        fac = (self.cx - self.shift) * self.nl
        return (fac < 0) * self.f0 + (fac >= 0) * ul


class VanishBC:
    """dgfs-vanish.mako: ghost 0 where c_x n >= 0, the trace elsewhere."""

    def __init__(self, cv, nl):
        self.cx, self.nl = cv[0], nl

    def update(self, ul):
        pass

    def apply(self, ul):
        fac = self.cx * self.nl
        return (fac >= 0) * 0.0 + (fac < 0) * ul


class WallExprBC:
    """dgfs-wall-expr-diffuse.mako (std and bi): diffuse wall with state
    (ux, uy, uz, T) = state(t) (nondimensional) and the unnormalised
    Maxwellian exp(-m |c - u|^2 / T); set ``t`` before each right-hand side."""

    def __init__(self, cv, cw, nl, state, mass=1.0):
        self.cv, self.cw, self.nl, self.state, self.mass = cv, cw, nl, state, mass
        self.t = 0.0

    def _mx(self):
        ux, uy, uz, T = self.state(self.t)
        cv = self.cv
        c2 = (cv[0] - ux) ** 2 + (cv[1] - uy) ** 2 + (cv[2] - uz) ** 2
        return ux, np.exp(-self.mass * c2 / T)

    def update(self, ul):
        ux, mx = self._mx()
        fac = (self.cv[0] - ux) * self.nl
        num = (fac >= 0.) * (fac * ul * self.cw)
        den = (fac < 0.) * (fac * mx * self.cw)
        self.nden = -(np.sum(num) / np.sum(den))

    def apply(self, ul):
        ux, mx = self._mx()
        fac = (self.cv[0] - ux) * self.nl
        return (fac < 0) * (mx * self.nden) + (fac >= 0) * ul


class PeriodicBC:
    """Single-rank ``dgfs-periodic``: ghost = the interior trace
    (dgfs-periodic.mako)."""

    def update(self, ul):
        pass

    def apply(self, ul):
        return ul.copy()


def dg_rhs(basis, invjac, cx, bcl, bcr, u_in, collide=None):
    """Right-hand side of std.py:281-366 for u_in of shape (K, Ne, Nv).

    ``collide(u_in, ux)`` adds the collision term (the fs loop of :349-356).
    """
    K, Ne, Nv = u_in.shape
    usolF = np.einsum('qk,kev->qev', basis.bwdFaceOp, u_in)
    usolF = usolF.reshape(-1, Nv)
    mapL, mapR = face_maps(Ne, basis.Nqf)
    uL = usolF[mapL].copy()
    uR = usolF[mapR].copy()
    bcL = uL[0].copy()
    bcR = uR[Ne].copy()
    bcl.update(bcL)
    uL[0] = bcl.apply(bcL)
    bcr.update(bcR)
    uR[Ne] = bcr.apply(bcR)
    ac = 0.5 * np.abs(cx)
    jL = ac * (uL - uR)
    jR = jL.copy()
    jL = jL + 0.5 * cx * (uR - uL)
    jR = jR + 0.5 * cx * (uL - uR)
    ux = np.einsum('km,mev->kev', basis.derivOp, u_in)
    ux = ux * (-cx)
    for k in range(K):
        for e in range(Ne):
            ux[k, e] += -jL[e + 1] * basis.gRD[k] + jR[e] * basis.gLD[k]
    ux = ux * invjac.reshape(1, Ne, 1)
    if collide is not None:
        collide(u_in, ux)
    return np.einsum('km,mev->kev', basis.invMassOp, ux)


def upwind_ops(basis, sigma=-1):
    """Upwind summation-by-parts operators of basis.py:304-312 as applied
    (Dp^T, Dm^T): S = sigma q q^T with q the last column of the QR of the
    Legendre Vandermonde, P = diag(w), Dp/m = D -/+ ... = D +- S P^-1 / 2,
    D = derivMat^T."""
    K = basis.K
    V = ortho_basis_at(K, basis.z).T
    Vo, _ = np.linalg.qr(V)
    sig = np.zeros(K)
    sig[-1] = sigma
    S = Vo @ np.diag(sig) @ Vo.T
    invP = np.diag(1.0 / basis.w)
    D = basis.derivMat.T
    Dp, Dm = D + 0.5 * S @ invP, D - 0.5 * S @ invP
    return filter_tol(Dp.T), filter_tol(Dm.T)


def dg_rhs_upwind(basis, invjac, cx, bcl, bcr, u_in, sigma=-1, swap=False,
                  collide=None):
    """Explicit right-hand side of dgfsABUstd1D (abstdu.py:295-383): the
    upwind fluxes jL = (uR - uL) min(c, 0), jR = -(uR - uL) max(c, 0) (equal
    to the central-upwind fluxes of dg_rhs), the split volume term
    -(Dm^T max(c,0) u + Dp^T min(c,0) u), lifting, invjac; ``swap`` gives
    each end's boundary the other end's trace (one-rank dgfs-cyclic)."""
    K, Ne, Nv = u_in.shape
    DpT, DmT = upwind_ops(basis, sigma)
    usolF = np.einsum('qk,kev->qev', basis.bwdFaceOp, u_in).reshape(-1, Nv)
    mapL, mapR = face_maps(Ne, basis.Nqf)
    uL = usolF[mapL].copy()
    uR = usolF[mapR].copy()
    bcL, bcR = uL[0].copy(), uR[Ne].copy()
    if swap:
        bcL, bcR = bcR, bcL
    bcl.update(bcL)
    uL[0] = bcl.apply(bcL)
    bcr.update(bcR)
    uR[Ne] = bcr.apply(bcR)
    diff = uR - uL
    jL = diff * np.minimum(cx, 0.0)
    jR = -diff * np.maximum(cx, 0.0)
    f = np.where(cx > 0, cx, 0.0) * u_in
    g = np.where(cx < 0, cx, 0.0) * u_in
    ux = -(np.einsum('km,mev->kev', DmT, f) + np.einsum('km,mev->kev', DpT, g))
    for k in range(K):
        for e in range(Ne):
            ux[k, e] += -jL[e + 1] * basis.gRD[k] + jR[e] * basis.gLD[k]
    ux = ux * invjac.reshape(1, Ne, 1)
    if collide is not None:
        collide(u_in, ux)
    return np.einsum('km,mev->kev', basis.invMassOp, ux)


def log_mean(a, b):
    """aveL of astd/kernels/limiters.mako:163-170 (elementwise)."""
    xi = np.abs(a / (b + 1e-20))
    f = (xi - 1) / (xi + 1)
    u = f * f
    with np.errstate(divide='ignore', invalid='ignore'):
        den = np.where(u < 1e-2, 1 + u / 3 + u * u / 5 + u * u * u / 7,
                       np.log(xi + 1e-20) / 2. / (f + 1e-20))
    return 0.5 * (a + b) / den


def dg_rhs_entropy(basis, invjac, cx, bcl, bcr, u_in, collide=None):
    """Explicit right-hand side of dgfsABE2std1D (abstde2.py:340-380): the
    fluxes, lifting and invjac of dg_rhs with the entropy-stable volume term
    -2 c_x sum_l Dr[k][l] aveL(u_k, u_l) (eDeriv, limiters.mako:173-195)."""
    K, Ne, Nv = u_in.shape
    usolF = np.einsum('qk,kev->qev', basis.bwdFaceOp, u_in).reshape(-1, Nv)
    mapL, mapR = face_maps(Ne, basis.Nqf)
    uL = usolF[mapL].copy()
    uR = usolF[mapR].copy()
    bcL, bcR = uL[0].copy(), uR[Ne].copy()
    bcl.update(bcL)
    uL[0] = bcl.apply(bcL)
    bcr.update(bcR)
    uR[Ne] = bcr.apply(bcR)
    ac = 0.5 * np.abs(cx)
    jL = ac * (uL - uR)
    jR = jL.copy()
    jL = jL + 0.5 * cx * (uR - uL)
    jR = jR + 0.5 * cx * (uL - uR)
    Dr = basis.derivMat
    ux = np.zeros_like(u_in)
    for k in range(K):
        for l in range(K):
            ux[k] += -2 * Dr[k, l] * cx * log_mean(u_in[k], u_in[l])
    for k in range(K):
        for e in range(Ne):
            ux[k, e] += -jL[e + 1] * basis.gRD[k] + jR[e] * basis.gLD[k]
    ux = ux * invjac.reshape(1, Ne, 1)
    if collide is not None:
        collide(u_in, ux)
    return np.einsum('km,mev->kev', basis.invMassOp, ux)


def limit_positivity(basis, u):
    """limitPos of limiters.mako:198-227 (every element): u_k <- a + theta
    (u_k - a), theta = min(1, |(a - 1e-13)/(a - min u)|) rounded to single
    precision (the kernel's fabsf)."""
    K, Ne, Nv = u.shape
    avg = np.einsum('j,jev->ev', basis.cellAvgOp[0], u)
    mn = np.minimum(1e10, u.min(axis=0))
    with np.errstate(divide='ignore', invalid='ignore'):
        ratio = ((avg - 1e-13) / (avg - mn)).astype(np.float32)
    theta = np.minimum(1.0, np.abs(ratio).astype(np.float64))
    return avg[None] + theta[None] * (u - avg[None])


def collide_fs(basis, fs):
    """The collision loop of std.py:349-356 with fs(f, g) -> increment."""
    def collide(u_in, ux):
        K, Ne, Nv = u_in.shape
        for m in range(K):
            d_f = np.einsum('ar,aev->rev', basis.U[m], u_in)
            d_g = np.einsum('rb,bev->rev', basis.V[m], u_in)
            for r in basis.sigModes[m]:
                for e in range(Ne):
                    ux[m, e] += fs(d_f[r, e], d_g[r, e])
    return collide


def axnpby(x0, a0, *terms):
    """x0 <- a0 x0 + sum a_i x_i with the a0 in {0, 1} branches (axnpby.py)."""
    acc = 0.0
    for a, x in zip(terms[::2], terms[1::2]):
        acc = acc + a * x
    if a0 == 0.0:
        x0[...] = acc
    elif a0 == 1.0:
        x0[...] = x0 + acc
    else:
        x0[...] = a0 * x0 + acc


def integrate(kind, rhs, t, dt, u):
    """One step of std/integrator.py:37-157 (in place on u)."""
    if kind == 'euler':
        r0 = rhs(t, u)
        axnpby(u, 1.0, dt, r0)
    elif kind == 'ssp-rk2':
        r0 = rhs(t, u)
        axnpby(r0, dt, 1.0, u)
        r1 = rhs(t + dt, r0)
        axnpby(u, 0.5, 0.5, r0, 0.5 * dt, r1)
    elif kind == 'ssp-rk3':
        r1 = rhs(t, u)
        r0 = np.empty_like(u)
        axnpby(r0, 0.0, 1.0, u, dt, r1)
        r1 = rhs(t + dt, r0)
        axnpby(r0, 0.25, 0.75, u, 0.25 * dt, r1)
        r1 = rhs(t + 0.5 * dt, r0)
        axnpby(u, 1.0 / 3.0, 2.0 / 3.0, r0, 2.0 / 3.0 * dt, r1)
    elif kind == 'lse-rk45':
        a = [0.0, -567301805773.0 / 1357537059087.0,
             -2404267990393.0 / 2016746695238.0,
             -3550918686646.0 / 2091501179385.0,
             -1275806237668.0 / 842570457699.0]
        b = [1432997174477.0 / 9575080441755.0,
             5161836677717.0 / 13612068292357.0,
             1720146321549.0 / 2090206949498.0,
             3134564353537.0 / 4481467310338.0,
             2277821191437.0 / 14882151754819.0]
        c = [0.0, 1432997174477.0 / 9575080441755.0,
             2526269341429.0 / 6820363962896.0,
             2006345519317.0 / 3224310063776.0,
             2802321613138.0 / 2924317926251.0]
        r1 = np.zeros_like(u)
        for s in range(5):
            r0 = rhs(t + c[s] * dt, u)
            axnpby(r1, a[s], dt, r0)
            axnpby(u, 1., b[s], r1)
    else:
        raise ValueError(kind)


def moments(basis, coeff, cv, cw, T0=1.0, rho0=1.0, u0=1.0, R0=8.3144598,
            molarMass0=1.0):
    """Bulk moments of std/moments.py:11-70 at the reconstruction points.

    Returns (Nqr, Ne, 10): rho, Ux, Uy, T, Qx, Qy, Pxx, Pyy, Pxy, p with the
    dimensional scaling of :61-68 (pass T0=rho0=u0=1 for nondimensional).
    """
    K, Ne, Nv = coeff.shape
    soln = np.einsum('mr,mej->rej', basis.interpMat, coeff)
    mcw = cw
    out = np.zeros(soln.shape[:2] + (10,))
    out[:, :, 0] = np.einsum('...j->...', soln) * mcw
    if np.sum(out[:, :, 0]) < 1e-10:      # :35-37 writes zeros
        return np.zeros_like(out)
    out[:, :, 1] = np.einsum('rej,j->re', soln, cv[0]) * mcw / out[:, :, 0]
    out[:, :, 2] = np.einsum('rej,j->re', soln, cv[1]) * mcw / out[:, :, 0]
    Nqr = soln.shape[0]
    cx = cv[0].reshape(1, 1, Nv) - out[:, :, 1].reshape(Nqr, Ne, 1)
    cy = cv[1].reshape(1, 1, Nv) - out[:, :, 2].reshape(Nqr, Ne, 1)
    cz = cv[2].reshape(1, 1, Nv) - np.zeros((Nqr, Ne, 1))
    cSqr = cx * cx + cy * cy + cz * cz
    out[:, :, 3] = np.einsum('...j,...j->...', soln, cSqr) * (2. / 3. * mcw)
    out[:, :, 3] /= out[:, :, 0]
    out[:, :, 4] = np.einsum('...j,...j,...j->...', soln, cSqr, cx) * mcw
    out[:, :, 5] = np.einsum('...j,...j,...j->...', soln, cSqr, cy) * mcw
    out[:, :, 6] = 2 * np.einsum('...j,...j,...j->...', soln, cx, cx) * mcw
    out[:, :, 7] = 2 * np.einsum('...j,...j,...j->...', soln, cy, cy) * mcw
    out[:, :, 8] = 2 * np.einsum('...j,...j,...j->...', soln, cx, cy) * mcw
    out[:, :, 0:9] *= np.array([rho0, u0, u0, T0, 0.5 * rho0 * u0 ** 3,
                                0.5 * rho0 * u0 ** 3, 0.5 * rho0 * u0 ** 2,
                                0.5 * rho0 * u0 ** 2, 0.5 * rho0 * u0 ** 2])
    out[:, :, 9] = (R0 / molarMass0) * out[:, :, 0] * out[:, :, 3]
    return out


def moments_bi(basis, coeffs, cv, cw, masses, T0=1.0, rho0=1.0, u0=1.0,
               R0=8.3144598, NA=6.0221409e+23, molarMass0=1.0):
    """Mixture moments of bi/moments.py:11-113 at the reconstruction points.

    Returns (Nqr, Ne, 7 * nspcs): per species rho, Ux, Uy, T, Qx, p, nden,
    dimensional.  T uses the species velocity, Qx the mixture velocity of
    the species kept (u_z taken as zero in both); a species whose density
    summed over all points is below 1e-10 keeps rho and has zero U and T
    (:43-45).
    """
    ns = len(coeffs)
    im = basis.interpMat
    soln = [np.einsum('mr,mej->rej', im, c) for c in coeffs]
    Nqr, Ne, Nv = soln[0].shape
    out = np.zeros((Nqr, Ne, 7 * ns))
    tot = np.zeros((Nqr, Ne, 3))

    def pec(ux, uy):
        cx = cv[0].reshape(1, 1, Nv) - ux.reshape(Nqr, Ne, 1)
        cy = cv[1].reshape(1, 1, Nv) - uy.reshape(Nqr, Ne, 1)
        cz = cv[2].reshape(1, 1, Nv) - np.zeros((Nqr, Ne, 1))
        return cx, cx * cx + cy * cy + cz * cz

    for p in range(ns):
        m, o, f = masses[p], 7 * p, soln[p]
        mcw = m * cw
        out[:, :, o] = np.sum(f, axis=-1) * mcw
        if np.sum(out[:, :, o]) < 1e-10:
            continue
        out[:, :, o + 1] = np.tensordot(f, cv[0], axes=(-1, 0)) * mcw / out[:, :, o]
        out[:, :, o + 2] = np.tensordot(f, cv[1], axes=(-1, 0)) * mcw / out[:, :, o]
        _, c2 = pec(out[:, :, o + 1], out[:, :, o + 2])
        out[:, :, o + 3] = np.sum(f * c2, axis=-1) * (2. / 3. * mcw * m) / out[:, :, o]
        tot[:, :, 0] += out[:, :, o]
        tot[:, :, 1] += out[:, :, o] * out[:, :, o + 1]
        tot[:, :, 2] += out[:, :, o] * out[:, :, o + 2]
    tot[:, :, 1] /= tot[:, :, 0]
    tot[:, :, 2] /= tot[:, :, 0]
    cx, c2 = pec(tot[:, :, 1], tot[:, :, 2])
    for p in range(ns):
        m, o, f = masses[p], 7 * p, soln[p]
        mcw = m * cw
        out[:, :, o + 4] = m * np.sum(f * c2 * cx, axis=-1) * mcw
        out[:, :, o:o + 5] *= np.array([rho0, u0, u0, T0, 0.5 * rho0 * u0 ** 3])
        out[:, :, o + 5] = (m * R0 / molarMass0) * out[:, :, o] * out[:, :, o + 3]
        out[:, :, o + 6] = (NA / m / molarMass0) * out[:, :, o]
    return out


# -- binary mixture (dgfs1D/bi/bi.py:265-349, bi/integrator.py) -------------

def collide_bi(basis, p, nspcs, fs_pq):
    """Collision loop of bi.py:336-342: sum_q Q_pq(U^T u_p, V u_q)."""
    def collide(us):
        def add(u_in, ux):
            K, Ne, Nv = u_in.shape
            for m in range(K):
                d_f = np.einsum('ar,aev->rev', basis.U[m], us[p])
                for q in range(nspcs):
                    d_g = np.einsum('rb,bev->rev', basis.V[m], us[q])
                    for r in basis.sigModes[m]:
                        for e in range(Ne):
                            ux[m, e] += fs_pq(p, q, d_f[r, e], d_g[r, e])
        return add
    return collide


def bi_integrate(kind, rhs, t, dt, us, compat=False):
    """One step of the mixture integrators; rhs(p, t, us) -> array."""
    ns = len(us)
    if kind == 'euler':
        r0 = [rhs(p, t, us) for p in range(ns)]
        for p in range(ns):
            axnpby(r0[p], dt, 1.0, us[p])
        for p in range(ns):
            us[p][...] = r0[p]
    elif kind == 'ssp-rk2':
        r0 = []
        for p in range(ns):
            r = rhs(p, t, us)
            axnpby(r, dt, 1.0, us[p])
            r0.append(r)
        for p in range(ns):
            r1 = rhs(p, t + dt, r0)
            axnpby(us[p], 0.5, 0.5, r0[p], 0.5 * dt, r1)
    elif kind == 'ssp-rk3':
        r0 = [np.empty_like(u) for u in us]
        for p in range(ns):
            r1 = rhs(p, t, us)
            axnpby(r0[p], 0.0, 1.0, us[p], dt, r1)
        r1s = []
        for p in range(ns):
            r1 = rhs(p, t + dt, r0)
            axnpby(r1, 0.25 * dt, 0.75, us[p], dt if compat else 0.25, r0[p])
            r1s.append(r1)
        for p in range(ns):
            r = rhs(p, t + 0.5 * dt, r1s)
            axnpby(us[p], 1.0 / 3.0, 2.0 / 3.0, r1s[p], 2.0 / 3.0 * dt, r)
    elif kind == 'lse-rk45':
        a = [0.0, -567301805773.0 / 1357537059087.0,
             -2404267990393.0 / 2016746695238.0,
             -3550918686646.0 / 2091501179385.0,
             -1275806237668.0 / 842570457699.0]
        b = [1432997174477.0 / 9575080441755.0,
             5161836677717.0 / 13612068292357.0,
             1720146321549.0 / 2090206949498.0,
             3134564353537.0 / 4481467310338.0,
             2277821191437.0 / 14882151754819.0]
        c = [0.0, 1432997174477.0 / 9575080441755.0,
             2526269341429.0 / 6820363962896.0,
             2006345519317.0 / 3224310063776.0,
             2802321613138.0 / 2924317926251.0]
        r1 = [np.zeros_like(u) for u in us]
        for s in range(5):
            r0 = []
            for p in range(ns):
                r = rhs(p, t + c[s] * dt, us)
                axnpby(r1[p], a[s], dt, r)
                axnpby(r, 0., 1., us[p], b[s], r1[p])
                r0.append(r)
            for p in range(ns):
                us[p][...] = r0[p]
    else:
        raise ValueError(kind)


def _minmod(a, b, c):
    """minmod of limiters.mako:11-15: the smallest magnitude when the three
    signs agree (and none is zero), else 0."""
    sa, sb, sc = np.sign(a), np.sign(b), np.sign(c)
    m = np.trunc((sa + sb + sc) / 3.)
    return np.where(np.abs(m) == 1,
                    m * np.minimum(np.minimum(np.abs(a), np.abs(b)), np.abs(c)),
                    0.)


def limit_linear(basis, invjac, xsol, u, tol=1e-6):
    """The linear slope limiter applied after every step of dgfsABstd1D with
    ``[time-integrator] limiter = 1`` (abstd.py:403-415, limitLin of
    astd/kernels/limiters.mako:17-76): in every interior element whose end
    values differ from the minmod-limited linear reconstruction by more than
    tol, the solution becomes the cell average plus the minmod of its linear
    slope and the two one-sided average differences (divided by h)."""
    K, Ne = u.shape[0], u.shape[1]
    uavg = np.einsum('kj,jev->kev', basis.cellAvgOp, u)
    ulx = np.einsum('kj,jev->kev', basis.drLinOp, u) * np.asarray(invjac).reshape(1, Ne, 1)
    out = u.copy()
    for e in range(1, Ne - 1):
        h = (1. / np.asarray(invjac).ravel()[e]) * 2
        x0 = xsol[0, e] + h / 2
        a, aR, aL = uavg[0, e], uavg[0, min(e + 1, Ne - 1)], uavg[0, max(e - 1, 0)]
        lim = (np.abs(a - _minmod(a - u[0, e], aR - a, a - aL) - u[0, e])
               + np.abs(a + _minmod(u[K - 1, e] - a, aR - a, a - aL) - u[K - 1, e])) > tol
        slope = _minmod(ulx[0, e], (aR - a) / h, (a - aL) / h)
        for k in range(K):
            out[k, e] = np.where(lim, a + (xsol[k, e] - x0) * slope, u[k, e])
    return out
