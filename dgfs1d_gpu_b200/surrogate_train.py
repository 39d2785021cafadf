"""Training data, training loop and solver coupling of the FNO surrogate.

* ``perturbed_maxwellians`` / ``operator_pairs``: seeded (f, Q) pairs from the
  plain operator -- Maxwellians with density in [0.5, 2], temperature in
  [0.7, 1.5], bulk velocity in [-0.3, 0.3]^3, times (1 + eps U[-1, 1]).
* ``harvest``: (f, Q) pairs along a real run of the plain solver.
* ``train``: Adam with a cosine learning-rate decay on the native kernels.
* ``SurrogateBoltzmann``: the Boltzmann-operator hook of ``DGFSABstd1D``.
  The surrogate replaces Q(f, f) except that every k-th call evaluates the
  plain operator as well; the plain result is used at those calls, and the
  relative L2 residual |Q_pred - Q_plain| / |Q_plain| judges the prediction:
  above ``tol`` the plain operator serves every call until a later check
  passes.  With ``correct=True`` the prediction between checks is the
  surrogate plus the defect d = Q_plain - Q_sur measured at the last check
  (the residual then judges Q_sur + d_previous); a steady state of the
  coupled scheme is then a steady state of the plain one.
* ``run_to_steady``: steps a solver until the relative change of its FP64
  bulk moments per step falls below a tolerance.
"""
import math
import time

import numpy as np
import torch


def grid(c0, device='cuda'):
    c = torch.as_tensor(np.asarray(c0), dtype=torch.float64, device=device)
    cx, cy, cz = torch.meshgrid(c, c, c, indexing='ij')
    return torch.stack([cx.reshape(-1), cy.reshape(-1), cz.reshape(-1)])


def perturbed_maxwellians(c0, count, seed, noise=0.05, rho=(0.5, 2.0),
                          T=(0.7, 1.5), umax=0.3, device='cuda'):
    """[count, N^3] float64 seeded perturbed Maxwellians on the grid c0."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    cv = grid(c0, device)

    def uni(lo, hi, *shape):
        return lo + (hi - lo) * torch.rand(*shape, generator=g, device=device,
                                           dtype=torch.float64)
    r = uni(*rho, count, 1)
    t = uni(*T, count, 1)
    u = uni(-umax, umax, count, 3)
    d2 = ((cv[None] - u[:, :, None]) ** 2).sum(1)
    f = r / (math.pi * t) ** 1.5 * torch.exp(-d2 / t)
    return f * (1 + noise * uni(-1.0, 1.0, *f.shape))


def operator_pairs(op, f, batch=24):
    """Q = op(f) for every row of f (plain operator, accumulate into zeros)."""
    Q = torch.zeros_like(f)
    for i in range(0, f.shape[0], batch):
        op.eval(f[i:i + batch], Q[i:i + batch])
    return Q


def harvest(solver, nsteps, every):
    """Run the plain solver; return its point states every `every` steps as
    [count, N^3] rows (K*Ne points per snapshot)."""
    rows = []
    n = solver.u.shape[-1]
    for s in range(nsteps):
        solver.step()
        if (s + 1) % every == 0:
            rows.append(solver.u.reshape(-1, n).clone())
    return torch.cat(rows) if rows else torch.empty(0, n, dtype=torch.float64,
                                                     device=solver.u.device)


def train(net, f, Q, steps, batch=24, lr=2e-3, lr_final=1e-5, seed=0,
          time_budget=None, log_every=100, tail=0, tail_frac=0.5):
    """Adam on random mini-batches; returns [(step, mean loss)].

    With ``tail`` > 0 a fraction ``tail_frac`` of every batch is drawn from
    the last ``tail`` rows (e.g. states harvested along the target run)."""
    g = torch.Generator(device='cpu')
    g.manual_seed(int(seed))
    n = f.shape[0]
    nt = int(round(batch * tail_frac)) if tail > 0 else 0
    hist, t0 = [], time.time()
    fb = torch.empty((batch, f.shape[1]), dtype=torch.float64, device=f.device)
    qb = torch.empty_like(fb)
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g)
        if nt:
            idx[:nt] = n - tail + torch.randint(0, tail, (nt,), generator=g)
        idx = idx.to(f.device)
        torch.index_select(f, 0, idx, out=fb)
        torch.index_select(Q, 0, idx, out=qb)
        lr_s = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * s / steps))
        net.train_step(fb, qb, lr=lr_s)
        if (s + 1) % log_every == 0 or s == steps - 1:
            hist.append((s + 1, float(net.last_loss(batch).mean())))
        if time_budget is not None and time.time() - t0 > time_budget:
            hist.append((s + 1, float(net.last_loss(batch).mean())))
            break
    return hist


def residuals(net, op, f, batch=24):
    """Per-sample |Q_sur - Q_plain| / |Q_plain| on the rows of f."""
    Qp = operator_pairs(op, f, batch)
    Qs = operator_pairs(net, f, batch)
    return (torch.linalg.norm(Qs - Qp, dim=1)
            / torch.linalg.norm(Qp, dim=1)).cpu().numpy()


class SurrogateBoltzmann:
    """Boltzmann-operator hook for DGFSABstd1D (see the module docstring)."""

    def __init__(self, solver, net, k=10, tol=1e-3, correct=False):
        self.solver, self.net, self.k, self.tol = solver, net, int(k), float(tol)
        self.correct = bool(correct)
        self.calls = 0
        self.fallback = False
        self.checks = []        # (call, residual)
        self.plain_calls = 0
        self._qp = torch.zeros_like(solver.u)
        self._qs = torch.zeros_like(solver.u)
        self._d = torch.zeros_like(solver.u) if correct else None
        self._have_d = False

    def __call__(self, t, u_in, u_out):
        s = self.solver
        check = self.calls % self.k == 0
        self.calls += 1
        if check:
            self._qp.zero_()
            self._qs.zero_()
            s.sm.fs_batch(u_in, self._qp, s.src, s.dst)
            self.net.eval(u_in, self._qs, src=s.src, dst=s.dst)
            pred = self._qs + self._d if (self.correct and self._have_d) else self._qs
            res = float(torch.linalg.norm(pred - self._qp)
                        / torch.linalg.norm(self._qp))
            self.checks.append((self.calls, res))
            if self.correct:
                torch.sub(self._qp, self._qs, out=self._d)
                self._have_d = True
            self.fallback = res > self.tol
            self.plain_calls += 1
            u_out += self._qp
        elif self.fallback:
            self.plain_calls += 1
            s.sm.fs_batch(u_in, u_out, s.src, s.dst)
        else:
            self.net.eval(u_in, u_out, src=s.src, dst=s.dst)
            if self.correct:
                u_out += self._d

    def stats(self):
        res = [r for _, r in self.checks]
        return dict(calls=self.calls, plain_calls=self.plain_calls,
                    checks=len(res),
                    residual_first=res[0] if res else None,
                    residual_median=float(np.median(res)) if res else None,
                    residual_last=res[-1] if res else None,
                    fallback_fraction=self.plain_calls / max(self.calls, 1))


def run_to_steady(solver, tol=1e-8, max_steps=100000, check_every=1):
    """Step until |m^{n+1} - m^n| / |m^n| < tol for the FP64 nondimensional
    bulk moments (per step); returns steps, wall seconds, final moments."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prev = solver.dg.moments(solver.u).clone()
    hist = []
    steps = 0
    res = float('inf')
    while steps < max_steps:
        solver.step()
        steps += 1
        if steps % check_every == 0:
            m = solver.dg.moments(solver.u)
            res = float(torch.linalg.norm(m - prev) / torch.linalg.norm(prev)
                        / check_every)
            hist.append((steps, res))
            prev.copy_(m)
            if res < tol:
                break
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return dict(steps=steps, wall_s=wall, residual=res, history=hist,
                moments=solver.bulk_moments())
