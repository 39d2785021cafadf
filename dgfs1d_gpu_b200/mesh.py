"""1-D physical mesh (``[mesh]``): the ``classic``, ``glj`` and ``bump``
point distributions of dgfs1D/mesh.py:8-84, non-dimensionalised by H0, with
the element Jacobians h/2 and 2/h (mesh.py:88-128; one rank)."""
import numpy as np

from .quadrature import gauss_lobatto_jacobi


class Mesh:
    def __init__(self, cfg):
        self.cfg = cfg
        kind = cfg.lookupordefault('mesh', 'type', 'classic')
        xlo, xhi = cfg.lookupfloat('mesh', 'xlo'), cfg.lookupfloat('mesh', 'xhi')
        if not xlo < xhi:
            raise ValueError('xlo must be less than xhi')
        Ne = cfg.lookupint('mesh', 'Ne')
        if Ne <= 0:
            raise ValueError('Need atleast one element to define a mesh')
        if kind == 'classic':
            x = np.linspace(xlo, xhi, Ne + 1)
        elif kind == 'glj':
            a = cfg.lookupordefault('mesh', 'alpha', 0.0)
            b = cfg.lookupordefault('mesh', 'beta', 0.0)
            z, _ = gauss_lobatto_jacobi(Ne + 1, a, b)
            x = 0.5 * (xhi + xlo) + 0.5 * (xhi - xlo) * z
        elif kind == 'bump':
            mu = cfg.lookupordefault('mesh', 'mu', 0.0)
            z = np.tanh(2 * mu * np.arange(Ne + 1) / Ne - mu) / np.tanh(mu)
            x = 0.5 * (xhi + xlo) + 0.5 * (xhi - xlo) * z
        else:
            raise ValueError(f'unknown mesh type {kind!r}')
        self.H0 = cfg.lookupfloat('mesh', 'H0')
        x = np.asarray(x, dtype=np.float64) / self.H0
        h = np.diff(x).reshape(-1, 1)
        if np.min(h) <= 1e-8:
            raise ValueError('Too small element size')
        self.xmesh, self.Ne = x, len(x) - 1
        self.jac, self.invjac = h / 2., 2. / h
        self.xlo, self.xhi = x.min(), x.max()
