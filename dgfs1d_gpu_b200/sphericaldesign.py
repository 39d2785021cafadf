"""Symmetric spherical designs (Womersley) used by the collision sums.

Interface of dgfs1D/sphericaldesign/__init__.py:82-105:
``get_sphquadrule('symmetric', rule='womersley', npts=M)`` returns an object
with ``pts`` (M x 3).  The point sets are the published Womersley designs,
bundled in ``data/womersley_symmetric.npz`` (recipe: ``tests/golden/make_sphere_designs.py``);
when several degrees share a point count the highest degree is chosen.
"""
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data',
                     'womersley_symmetric.npz')


class SphericalRule:
    def __init__(self, pts, degree):
        self.pts = np.asarray(pts, dtype=np.float64)
        self.wts = np.full(len(self.pts), 4 * np.pi / len(self.pts))
        self.degree = degree


def available(path=_DATA):
    data = np.load(path)
    return sorted((int(k[7:]), int(k[2:5])) for k in data.files)


def get_sphquadrule(sstype, rule=None, npts=None, qdeg=None, path=_DATA):
    if sstype != 'symmetric':
        raise ValueError(f'unknown spherical design type {sstype!r}')
    if rule not in (None, 'womersley'):
        raise ValueError(f'unknown spherical design rule {rule!r}')
    if not npts and not qdeg:
        raise ValueError('Must specify either npts or qdeg')
    data = np.load(path)
    best = None
    for key in data.files:
        deg, m = int(key[2:5]), int(key[7:])
        if (not npts or npts == m) and (not qdeg or qdeg <= deg):
            if (best is None or (npts and deg > best[1])
                    or (qdeg and m < best[2])):
                best = (key, deg, m)
    if best is None:
        raise ValueError('No suitable spherical quadrature rule found')
    return SphericalRule(data[best[0]], best[1])
