"""Distribution checkpoints (``[dgfsdistwriter]``) and restart.

The reference writes, every ``dt-out``, one HDF5 file per rank holding the
flat coefficient array(s) as dataset ``coeff`` (single species,
std/distribution.py:9-44) or ``coeff0``, ``coeff1``, ... (mixture,
bi/distribution.py:28-44), each with attributes time, K, Ne, Nv, and a
restart reads them back and checks K, Ne and Nv (std.py:234-244,
bi.py:223-236, abstd.py:243-253).  The file name is the configured basename
with ``.h5`` appended when missing, then ``_rank=<rank>``, formatted with
``t``.

The same datasets and attributes are written here.  With h5py importable the
file is that HDF5 file; without it (h5py is not part of every image) the
datasets go into a NumPy ``.npz`` archive under the same name pattern with
extension ``.npz``: array ``<name>`` plus scalars ``<name>.time``,
``<name>.K``, ``<name>.Ne``, ``<name>.Nv``.  ``read_distribution`` accepts
either form (HDF5 only where h5py is importable).
"""
import os

import numpy as np

ATTRS = ('time', 'K', 'Ne', 'Nv')


def _h5py():
    try:
        import h5py
    except ImportError:
        return None
    return h5py


def _rank():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank()
    except Exception:
        pass
    return 0


def write_distribution(path, datasets, time, K, Ne, Nv):
    """Write {name: flat array} with the reference's attributes."""
    h5 = _h5py()
    if h5 is not None and '.h5' in os.path.basename(path):
        with h5.File(path, 'w') as f:
            for name, data in datasets.items():
                d = f.create_dataset(name, data=np.ascontiguousarray(data))
                d.attrs['time'] = time
                d.attrs['K'], d.attrs['Ne'], d.attrs['Nv'] = K, Ne, Nv
        return path
    arrays = {}
    for name, data in datasets.items():
        arrays[name] = np.ascontiguousarray(data)
        for a, v in zip(ATTRS, (time, K, Ne, Nv)):
            arrays['%s.%s' % (name, a)] = np.asarray(v)
    with open(path, 'wb') as fh:          # keep the name exactly as formed
        np.savez(fh, **arrays)
    return path


def read_distribution(path, names, K, Ne, Nv):
    """({name: flat array}, time), checking K, Ne and Nv as the drivers do."""
    out, time = {}, None
    with open(path, 'rb') as fh:
        magic = fh.read(8)
    if magic == b'\x89HDF\r\n\x1a\n':
        h5 = _h5py()
        if h5 is None:
            raise RuntimeError('%s is an HDF5 file and h5py is not available'
                               % path)
        with h5.File(path, 'r') as f:
            for name in names:
                d = f[name]
                out[name] = np.asarray(d[:])
                attrs = {a: d.attrs[a] for a in ATTRS}
                time = _check(attrs, name, K, Ne, Nv)
    else:
        with np.load(path) as z:
            for name in names:
                out[name] = np.asarray(z[name])
                attrs = {a: z['%s.%s' % (name, a)][()] for a in ATTRS}
                time = _check(attrs, name, K, Ne, Nv)
    return out, time


def read_dataset(path, name='coeff'):
    """(flat array, {time, K, Ne, Nv}) of one dataset, without checks."""
    with open(path, 'rb') as fh:
        magic = fh.read(8)
    if magic == b'\x89HDF\r\n\x1a\n':
        h5 = _h5py()
        if h5 is None:
            raise RuntimeError('%s is an HDF5 file and h5py is not available'
                               % path)
        with h5.File(path, 'r') as f:
            d = f[name]
            return np.asarray(d[:]), {a: d.attrs[a] for a in ATTRS}
    with np.load(path) as z:
        return (np.asarray(z[name]),
                {a: z['%s.%s' % (name, a)][()] for a in ATTRS})


def remaining_steps(t, tf, dt):
    """Steps of size dt left from t to tf (the drivers loop while t < tf)."""
    import math
    return max(0, int(math.ceil((tf - t) / dt - 1e-9)))


def _check(attrs, name, K, Ne, Nv):
    for a, want, what in (('K', K, 'K'), ('Ne', Ne, 'Ne'), ('Nv', Nv, 'N')):
        if int(attrs[a]) != want:
            raise ValueError('Inconsistent distribution %s (%s: %d, run: %d)'
                             % (what, name, int(attrs[a]), want))
    return float(attrs['time'])


class DGFSDistributionWriter:
    """Writes the solution every ``dt-out`` after ``tcurr`` (datasets
    ``coeff`` for one species, ``coeff<p>`` for a mixture)."""

    def __init__(self, tcurr, shape, cfg, sect='dgfsdistwriter', nspcs=None):
        self.K, self.Ne, self.Nv = shape
        self.nspcs = nspcs
        self.enabled = cfg.has_section(sect)
        if not self.enabled:
            return
        self.basedir = cfg.lookupordefault(sect, 'basedir', '.')
        extn = '.h5' if _h5py() is not None else '.npz'
        base = cfg.lookup(sect, 'basename')
        if base.endswith('.h5') and extn != '.h5':
            base = base[:-3]
        if not base.endswith(extn):
            base += extn
        self.basename = base + '_rank=' + str(_rank())
        self.dt_out = cfg.lookupfloat(sect, 'dt-out')
        self.tout_next = tcurr + self.dt_out

    def __call__(self, dt, tcurr, coeff):
        if not self.enabled or abs(self.tout_next - tcurr) > 0.5 * dt:
            return None
        if self.nspcs is None:
            data = {'coeff': coeff.detach().cpu().numpy().ravel()}
        else:
            data = {'coeff%d' % p: c.detach().cpu().numpy().ravel()
                    for p, c in enumerate(coeff)}
        path = os.path.join(self.basedir, self.basename.format(t=tcurr))
        write_distribution(path, data, tcurr, self.K, self.Ne, self.Nv)
        self.tout_next = tcurr + self.dt_out
        return path
