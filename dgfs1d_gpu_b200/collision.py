"""Host handles of the native fast-spectral collision operators.

Thin owners of the C-ABI handles in ``libdgfs_sm100.so``; arrays are torch
CUDA tensors (or anything exposing ``data_ptr()``), passed by pointer.
"""
import ctypes

import numpy as np
import torch

from . import _native as nat

_DT = {torch.float32: nat.DGFS_F32, torch.float64: nat.DGFS_F64}
_PREC = {'fp64': nat.DGFS_PREC_FP64, 'fp32': nat.DGFS_PREC_FP32}


def _dptr(a):
    return ctypes.cast(a.ctypes.data, ctypes.POINTER(ctypes.c_double))


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _check_dist(t, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f'{name} must be a CUDA tensor')
    if t.dtype not in _DT:
        raise TypeError(f'{name} must be float32 or float64')
    if not t.is_contiguous():
        raise ValueError(f'{name} must be contiguous')


class VHSOperator:
    """Batched single-species VHS Q(f,f) (``vhs-gll``).

    precision: 'fp64' (all FP64, reference parity) or 'fp32' (FP32 3-D FFTs
    on f - M with the local Maxwellian M in FP64).
    """

    def __init__(self, N, L, qz, qw, sz, sw, sphere_factor, gamma, prefac,
                 cw, c0, precision='fp64', max_evals=64, sinc_eps=1e-15):
        if precision not in _PREC:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.N, self.n = int(N), int(N) ** 3
        self.precision = precision
        self.prefac = float(prefac)
        self.max_evals = int(max_evals)
        self._keep = [np.ascontiguousarray(x, dtype=np.float64)
                      for x in (qz, qw, np.asarray(sz).reshape(-1), c0)]
        qz_, qw_, sz_, c0_ = self._keep
        d = nat.VhsDesc()
        d.N, d.Nrho, d.M = self.N, len(qz_), len(sz_) // 3
        d.L = float(L)
        d.qz, d.qw, d.sz, d.c0 = _dptr(qz_), _dptr(qw_), _dptr(sz_), _dptr(c0_)
        d.sw, d.sphere_factor = float(sw), float(sphere_factor)
        d.gamma, d.prefac, d.sinc_eps = float(gamma), float(prefac), float(sinc_eps)
        d.cw = float(cw)
        d.precision = _PREC[precision]
        d.max_evals = self.max_evals
        h = ctypes.c_void_p()
        nat.check(nat.lib().dgfs_vhs_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.Nrho, self.M = d.Nrho, d.M
        self.variant = 0          # 0: the library's default cluster size

    def _nevals(self, f, Q, src, dst, src_base, dst_base, nevals):
        """Check the arrays and slot ranges; return the evaluation count."""
        nf, nq = f.numel() // self.n, Q.numel() // self.n
        if f.numel() % self.n or Q.numel() % self.n:
            raise ValueError('array sizes must be multiples of N^3')
        if nevals is None:
            nevals = len(src) if src is not None else nf - src_base
        for sl, base, cnt, name in ((src, src_base, nf, 'src'),
                                    (dst, dst_base, nq, 'dst')):
            if sl is None:
                if base < 0 or base + nevals > cnt:
                    raise IndexError(f'{name} slots out of range')
            elif sl.dtype != torch.int32 or not sl.is_cuda or len(sl) < nevals:
                raise TypeError(f'{name} must be a CUDA int32 tensor of '
                                f'length >= nevals')
        return int(nevals)

    def eval(self, f, Q, src=None, dst=None, src_base=0, dst_base=0,
             nevals=None, stream=None):
        """Q[dst(i)] += Q(f[src(i)]) for i < nevals (slot-major arrays)."""
        _check_dist(f, 'f')
        _check_dist(Q, 'Q')
        nevals = self._nevals(f, Q, src, dst, src_base, dst_base, nevals)
        nat.check(nat.lib().dgfs_vhs_eval(
            self._h, ctypes.c_void_p(f.data_ptr()), _DT[f.dtype],
            ctypes.c_void_p(Q.data_ptr()), _DT[Q.dtype],
            ctypes.c_void_p(src.data_ptr() if src is not None else 0), int(src_base),
            ctypes.c_void_p(dst.data_ptr() if dst is not None else 0), int(dst_base),
            nevals, _stream_ptr(stream)))

    def eval_multi(self, f_list, q_list, dtype_f, dtype_q, src, dst,
                   stream=None):
        """Q(f, f) for points of several problems sharing this operator:
        f_list, q_list are CUDA int64 tensors of array addresses (one per
        evaluation), src/dst CUDA int32 slot tensors of the same length."""
        n = len(src)
        for t_, name in ((f_list, 'f_list'), (q_list, 'q_list')):
            if t_.dtype != torch.int64 or not t_.is_cuda or len(t_) != n:
                raise TypeError(f'{name} must be a CUDA int64 tensor of '
                                'length nevals')
        for t_, name in ((src, 'src'), (dst, 'dst')):
            if t_.dtype != torch.int32 or not t_.is_cuda or len(t_) != n:
                raise TypeError(f'{name} must be a CUDA int32 tensor of '
                                'length nevals')
        nat.check(nat.lib().dgfs_vhs_eval_multi(
            self._h, ctypes.c_void_p(f_list.data_ptr()), _DT[dtype_f],
            ctypes.c_void_p(q_list.data_ptr()), _DT[dtype_q],
            ctypes.c_void_p(src.data_ptr()), 0,
            ctypes.c_void_p(dst.data_ptr()), 0, n, _stream_ptr(stream)))

    def eval2(self, f, g, Q, src=None, dst=None, src_base=0, dst_base=0,
              nevals=None, stream=None):
        """Bilinear Q[dst(i)] += Q(f[src(i)], g[src(i)]) (``vhs``): gain of
        the pair (f, g), loss f * Re IFFT(b2 FFT(g)/n); f and g have the same
        dtype and shape.  Two (FP64) or three (FP32) passes of the Q(h, h)
        pipeline."""
        _check_dist(f, 'f')
        _check_dist(g, 'g')
        _check_dist(Q, 'Q')
        if g.dtype != f.dtype or g.shape != f.shape:
            raise TypeError('f and g must have the same dtype and shape')
        nevals = self._nevals(f, Q, src, dst, src_base, dst_base, nevals)
        nat.check(nat.lib().dgfs_vhs_eval2(
            self._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(g.data_ptr()),
            _DT[f.dtype], ctypes.c_void_p(Q.data_ptr()), _DT[Q.dtype],
            ctypes.c_void_p(src.data_ptr() if src is not None else 0), int(src_base),
            ctypes.c_void_p(dst.data_ptr() if dst is not None else 0), int(dst_base),
            nevals, _stream_ptr(stream)))

    def variants(self):
        """Cluster sizes of the FP32 terms kernel compiled for this N."""
        buf = (ctypes.c_int32 * 8)()
        n = nat.lib().dgfs_vhs_variants(self.N, buf, 8)
        if n < 0:
            nat.check(n)
        return list(buf[:n])

    def set_variant(self, cluster):
        nat.check(nat.lib().dgfs_vhs_set_variant(self._h, int(cluster)))
        self.variant = int(cluster)

    def autotune(self, f=None, Q=None, reps=3, stream=None, call=None):
        """Time every terms-kernel variant and keep the fastest: on the
        evaluation of (f, Q), or on ``call()`` (any enqueue of this
        operator's evaluations, e.g. a merged multi-problem call).

        Returns {variant: ms per call}.  Q (or call's outputs) is overwritten.
        """
        if self.precision != 'fp32':
            return {}
        if call is None:
            def call():
                self.eval(f, Q, stream=stream)
        times = {}
        for c in self.variants():
            self.set_variant(c)
            call()                                   # warm-up
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(reps):
                call()
            e.record()
            e.synchronize()
            times[c] = s.elapsed_time(e) / reps
        self.set_variant(min(times, key=times.get))
        return times

    def device_error(self):
        """Waits for the device; nonzero if a bounded wait of the handle's
        kernels gave up since the last call (the flag is then cleared)."""
        out = ctypes.c_int32(0)
        nat.check(nat.lib().dgfs_vhs_device_error(self._h, ctypes.byref(out)))
        return int(out.value)

    def set_projection(self, enable=True):
        """Toggle the FP64 conservation projection of every evaluation."""
        nat.check(nat.lib().dgfs_vhs_set_projection(self._h, int(bool(enable))))

    def close(self):
        if getattr(self, '_h', None):
            nat.release(nat.lib().dgfs_vhs_destroy, self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VSSOperator:
    """Batched binary-mixture VSS Q_pq(f_p, f_q) (``vss``).

    gamma, eta, prefac: (nspcs, nspcs) arrays (pair pq at [p, q]).
    precision: 'fp64' (the reference's) or 'fp32' (FP32 transforms of
    f - M; Maxwellian parts, radial sum, final transform and loss in FP64).
    """

    def __init__(self, N, L, qz, qw, sz, sw, szpre, masses, gamma, eta,
                 prefac, max_evals=64, precision='fp64'):
        if precision not in _PREC:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        self.N, self.n = int(N), int(N) ** 3
        ns = len(masses)
        self.nspcs = ns
        self._keep = [np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
                      for x in (qz, qw, sz, szpre, masses, gamma, eta, prefac)]
        qz_, qw_, sz_, szp_, m_, g_, e_, p_ = self._keep
        d = nat.VssDesc()
        d.N, d.Nrho, d.M, d.Mpre, d.nspcs = self.N, len(qz_), len(sz_) // 3, \
            len(szp_) // 3, ns
        d.L, d.sw = float(L), float(sw)
        d.qz, d.qw, d.sz, d.szpre = _dptr(qz_), _dptr(qw_), _dptr(sz_), _dptr(szp_)
        d.masses, d.gamma, d.eta, d.prefac = _dptr(m_), _dptr(g_), _dptr(e_), \
            _dptr(p_)
        d.max_evals = int(max_evals)
        d.precision = _PREC[precision]
        h = ctypes.c_void_p()
        nat.check(nat.lib().dgfs_vss_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self.prefac = np.asarray(prefac, dtype=np.float64).reshape(ns, ns)

    def eval(self, p, q, fp, fq, Qp, src=None, dst=None, src_base=0,
             dst_base=0, nevals=None, stream=None):
        """Q_p[dst(i)] += Q_pq(f_p[src(i)], f_q[src(i)])."""
        for t, name in ((fp, 'f_p'), (fq, 'f_q'), (Qp, 'Q_p')):
            _check_dist(t, name)
        if fp.dtype != fq.dtype:
            raise TypeError('f_p and f_q must have the same dtype')
        nf = fp.numel() // self.n
        if nevals is None:
            nevals = len(src) if src is not None else nf - src_base
        for sl, base, cnt, name in ((src, src_base, nf, 'src'),
                                    (dst, dst_base, Qp.numel() // self.n, 'dst')):
            if sl is None and (base < 0 or base + nevals > cnt):
                raise IndexError(f'{name} slots out of range')
        nat.check(nat.lib().dgfs_vss_eval(
            self._h, int(p), int(q), ctypes.c_void_p(fp.data_ptr()),
            ctypes.c_void_p(fq.data_ptr()), _DT[fp.dtype],
            ctypes.c_void_p(Qp.data_ptr()), _DT[Qp.dtype],
            ctypes.c_void_p(src.data_ptr() if src is not None else 0), int(src_base),
            ctypes.c_void_p(dst.data_ptr() if dst is not None else 0), int(dst_base),
            int(nevals), _stream_ptr(stream)))

    def eval_species(self, p, fs, Qp, src=None, dst=None, src_base=0,
                     dst_base=0, nevals=None, stream=None):
        """Q_p[dst(i)] += sum_q Q_pq(f_p[src(i)], f_q[src(i)]): every pair
        of species p in one call (fs: one tensor per species)."""
        if len(fs) != self.nspcs:
            raise ValueError('fs must hold one array per species')
        for i, t in enumerate(fs):
            _check_dist(t, f'f[{i}]')
            if t.dtype != fs[0].dtype or t.shape != fs[0].shape:
                raise TypeError('the species arrays must share dtype and shape')
        _check_dist(Qp, 'Q_p')
        nf = fs[0].numel() // self.n
        if nevals is None:
            nevals = len(src) if src is not None else nf - src_base
        for sl, base, cnt, name in ((src, src_base, nf, 'src'),
                                    (dst, dst_base, Qp.numel() // self.n, 'dst')):
            if sl is None and (base < 0 or base + nevals > cnt):
                raise IndexError(f'{name} slots out of range')
        ptrs = (ctypes.c_void_p * self.nspcs)(*[t.data_ptr() for t in fs])
        nat.check(nat.lib().dgfs_vss_eval_species(
            self._h, int(p), ptrs, _DT[fs[0].dtype],
            ctypes.c_void_p(Qp.data_ptr()), _DT[Qp.dtype],
            ctypes.c_void_p(src.data_ptr() if src is not None else 0), int(src_base),
            ctypes.c_void_p(dst.data_ptr() if dst is not None else 0), int(dst_base),
            int(nevals), _stream_ptr(stream)))

    def eval_species_multi(self, p, f_lists, q_list, dtype_f, dtype_q, src,
                           dst, stream=None):
        """eval_species for points of several mixtures sharing this
        operator (FP32 mode): f_lists a CUDA int64 tensor [nspcs * nevals]
        of input array addresses, q_list [nevals] of species-p outputs."""
        n = len(src)
        if f_lists.dtype != torch.int64 or not f_lists.is_cuda or \
                len(f_lists) != self.nspcs * n:
            raise TypeError('f_lists must be a CUDA int64 tensor of length '
                            'nspcs * nevals')
        if q_list.dtype != torch.int64 or not q_list.is_cuda or len(q_list) != n:
            raise TypeError('q_list must be a CUDA int64 tensor of length nevals')
        nat.check(nat.lib().dgfs_vss_eval_species_multi(
            self._h, int(p), ctypes.c_void_p(f_lists.data_ptr()), _DT[dtype_f],
            ctypes.c_void_p(q_list.data_ptr()), _DT[dtype_q],
            ctypes.c_void_p(src.data_ptr()), 0, ctypes.c_void_p(dst.data_ptr()),
            0, n, _stream_ptr(stream)))

    def close(self):
        if getattr(self, '_h', None):
            nat.release(nat.lib().dgfs_vss_destroy, self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
