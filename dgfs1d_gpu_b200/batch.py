"""Many independent problems advanced as one CUDA graph per stage.

Problems that share one operator (the same velocity grid, rules and
parameters) are merged: their points form one list of (array, slot) pairs
and every kernel of the operator runs once for all of them
(``merged_vhs``, ``merged_vss``; dgfs_vhs_eval_multi,
dgfs_vss_eval_species_multi).  Problems of different velocity grids
(N = 16/24/32), rules or species (VHS and VSS) cannot share one kernel
without paying the largest variant's shared memory and registers in every
CTA: the kernels are specialised per N at compile time.  Each group's stage
is enqueued on its own stream, forked from and joined to one capture
stream, and the whole stage is captured once into a CUDA graph; a stage is
then a single graph launch whose branches the GPU schedules concurrently.
"""
import torch


def _lists(parts, n, device):
    """Address and slot tensors of every slot of every part [(f, Q)]."""
    fl, ql, sl = [], [], []
    for f, Q in parts:
        cnt = f.numel() // n
        fl += [f.data_ptr()] * cnt
        ql += [Q.data_ptr()] * cnt
        sl += list(range(cnt))
    as_t = lambda x, dt: torch.tensor(x, dtype=dt, device=device)  # noqa: E731
    return (as_t(fl, torch.int64), as_t(ql, torch.int64),
            as_t(sl, torch.int32))


def merged_vhs(op, parts):
    """One evaluation call of ``op`` for every slot of every (f, Q) in
    ``parts`` (Q[s] += Q(f[s])); returns the enqueue function."""
    f0, q0 = parts[0]
    if any(f.dtype != f0.dtype or Q.dtype != q0.dtype for f, Q in parts):
        raise TypeError('merged problems must share the array dtypes')
    fl, ql, sl = _lists(parts, op.n, f0.device)

    def fn(stream=None):
        op.eval_multi(fl, ql, f0.dtype, q0.dtype, sl, sl, stream=stream)
    fn.keep = (parts, fl, ql, sl)
    return fn


def merged_vss(op, mixtures):
    """One call per species of ``op`` (FP32) for every slot of every mixture
    in ``mixtures`` = [([f_0, f_1, ...], [Q_0, Q_1, ...])]:
    Q_p[s] += sum_q Q_pq(f_p[s], f_q[s])."""
    ns = op.nspcs
    dev = mixtures[0][0][0].device
    fdt, qdt = mixtures[0][0][0].dtype, mixtures[0][1][0].dtype
    per = [_lists([(fs[q], Qs[0]) for fs, Qs in mixtures], op.n, dev)
           for q in range(ns)]
    f_lists = torch.cat([fl for fl, _, _ in per])
    sl = per[0][2]
    q_lists = [_lists([(fs[p], Qs[p]) for fs, Qs in mixtures], op.n, dev)[1]
               for p in range(ns)]

    def fn(stream=None):
        for p in range(ns):
            op.eval_species_multi(p, f_lists, q_lists[p], fdt, qdt, sl, sl,
                                  stream=stream)
    fn.keep = (mixtures, f_lists, q_lists, sl)
    return fn


class StageGraph:
    """Capture ``[fn_0, ..., fn_k]`` (callables enqueuing work on the current
    stream) as concurrent branches of one CUDA graph."""

    def __init__(self, fns, device='cuda'):
        self.fns = list(fns)
        self.device = device
        self.streams = [torch.cuda.Stream(device=device) for _ in self.fns]
        self.graph = None

    def run_eager(self):
        """The same branches without a graph (for comparison)."""
        main = torch.cuda.current_stream()
        for fn, st in zip(self.fns, self.streams):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                fn()
        for st in self.streams:
            main.wait_stream(st)

    def capture(self, warmup=1):
        for _ in range(warmup):
            self.run_eager()
        torch.cuda.synchronize()
        cap = torch.cuda.Stream(device=self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(cap):
            with torch.cuda.graph(g, stream=cap):
                for fn, st in zip(self.fns, self.streams):
                    st.wait_stream(cap)
                    with torch.cuda.stream(st):
                        fn()
                for st in self.streams:
                    cap.wait_stream(st)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()
