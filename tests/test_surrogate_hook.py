"""Host logic of the surrogate/plain coupling (SurrogateBoltzmann) with fake
operators on the CPU: k-step checks, the residual test, fallback and the
defect-corrected mode."""
import torch

from dgfs1d_gpu_b200.surrogate_train import SurrogateBoltzmann


class _Plain:
    def __init__(self):
        self.calls = 0

    def fs_batch(self, u, out, src, dst):
        self.calls += 1
        out += 2.0 * u


class _Net:
    def __init__(self, err):
        self.err, self.calls = err, 0

    def eval(self, u, out, src=None, dst=None):
        self.calls += 1
        out += (2.0 + self.err) * u


class _Solver:
    def __init__(self):
        self.u = torch.ones(3, 2, 5, dtype=torch.float64)
        self.sm = _Plain()
        self.src = self.dst = None


def _run(err, correct, calls=25, k=10, tol=1e-3):
    s = _Solver()
    net = _Net(err)
    hook = SurrogateBoltzmann(s, net, k=k, tol=tol, correct=correct)
    outs = []
    for _ in range(calls):
        out = torch.zeros_like(s.u)
        hook(0.0, s.u, out)
        outs.append(out)
    return hook, s, net, outs


def test_accurate_surrogate_runs_between_checks():
    hook, s, net, outs = _run(err=1e-5, correct=False)
    st = hook.stats()
    assert st['checks'] == 3 and st['plain_calls'] == 3      # calls 1, 11, 21
    assert s.sm.calls == 3 and net.calls == 25
    assert torch.allclose(outs[1], (2.0 + 1e-5) * s.u)       # surrogate result
    assert torch.equal(outs[0], 2.0 * s.u)                   # plain at checks


def test_inaccurate_surrogate_falls_back_to_the_plain_operator():
    hook, s, net, outs = _run(err=0.1, correct=False)
    st = hook.stats()
    assert st['plain_calls'] == 25 and st['fallback_fraction'] == 1.0
    assert all(torch.equal(o, 2.0 * s.u) for o in outs)
    assert abs(st['residual_median'] - 0.05) < 1e-12


def test_defect_correction_recovers_the_plain_operator_on_a_fixed_state():
    hook, s, net, outs = _run(err=0.1, correct=True)
    st = hook.stats()
    # the first check judges the bare surrogate (no defect yet) and falls
    # back for its k-1 calls; from the second check on the corrected
    # prediction is exact on this fixed state
    assert st['residual_first'] > 1e-3 and st['residual_last'] < 1e-12
    assert st['plain_calls'] == 10 + 2
    assert all(torch.allclose(o, 2.0 * s.u, rtol=0, atol=1e-14) for o in outs)
