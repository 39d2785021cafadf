"""Grid-convergence error between two distribution checkpoints
(``dgfsStdError1D``, dgfs1D/error.py:1-63).

    python -m dgfs1d_gpu_b200.error coarse.npz_rank=0 fine.npz_rank=0

``file2`` must hold twice the elements of ``file1`` with the same number of
nodes per element.  The coarse solution is interpolated to the nodes of the
two fine elements inside each coarse one (GLL nodes of [-1, 0] and [0, 1]
mapped to the coarse element) and the error is the GLL-quadrature L1 norm
of the difference, halved per fine element, summed over elements and
velocities and divided by the fine element count and the velocity count
(compare(), :18-33).  The reference then prints it with ``print(*gerr)``
on a scalar, which raises; here the value is printed.
"""
import argparse
import sys

import numpy as np

from .distribution import read_dataset
from .quadrature import gauss_lobatto_jacobi, lagrange_at


def decode(path):
    """(Ne, Nq, data (Nq, Ne, Nv)) of a single-species checkpoint."""
    data, at = read_dataset(path, 'coeff')
    Nq, Ne, Nv = int(at['K']), int(at['Ne']), int(at['Nv'])
    return Ne, Nq, data.reshape(Nq, Ne, Nv)


def compare(Nq, f, f2):
    _, Ne2, nvars = f2.shape
    r, w = gauss_lobatto_jacobi(Nq)
    r2 = r * 0.5 + 0.5
    r2 = np.concatenate((-np.flip(r2), r2))
    im = lagrange_at(r, r2)                              # (2 Nq, Nq)
    fr = np.einsum('rm,mjk->rjk', im, f)
    fr = fr.swapaxes(0, 2).reshape((-1, Ne2, Nq)).swapaxes(0, 2)
    diff = np.abs(fr - f2)
    L1e = 0.5 * np.einsum('q,qjk->jk', w, diff)
    return np.sum(L1e, axis=(0, 1)) / Ne2 / nvars


def compute_error(file1, file2):
    Ne1, Nq1, u1 = decode(file1)
    Ne2, Nq2, u2 = decode(file2)
    if Ne2 // Ne1 != 2:
        raise ValueError('Elements in file2 != 2 * (elements in file1)')
    if Nq1 != Nq2:
        raise ValueError("Number of quadrature points don't match")
    return compare(Nq1, u1, u2)


def main(argv=None):
    ap = argparse.ArgumentParser(prog='python -m dgfs1d_gpu_b200.error')
    ap.add_argument('file1')
    ap.add_argument('file2')
    a = ap.parse_args(sys.argv[1:] if argv is None else argv)
    err = compute_error(a.file1, a.file2)
    print(err)
    return err


if __name__ == '__main__':
    main()
