"""The uneven multi-problem batch: one CUDA graph per stage.

Six VHS problems (N = 16/24/32, 12-39 points) and two VSS mixtures (N=24)
are captured as concurrent branches of one graph; a replay must give the
same Q as the eager launches, bit for bit, and every slot of every problem
must match the oracle."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module', params=[False, True], ids=['per-problem', 'merged'])
def problems(request):
    """Per problem (one operator and one call per problem), or merged (the
    problems that share an operator evaluated in one call per kernel)."""
    from dgfs1d_gpu_b200 import build
    build.build()
    from dgfs1d_gpu_b200.workloads_c3 import build_c3
    return build_c3(precision='fp32', merged=request.param)


def _members(probs):
    out = []
    for p in probs:
        out += p.get('members', [p])
    return out


def _snapshot(probs):
    out = []
    for p in _members(probs):
        qs = p['Q'] if isinstance(p['Q'], list) else [p['Q']]
        out.append([q.clone() for q in qs])
    return out


def test_graph_replay_equals_eager(problems):
    from dgfs1d_gpu_b200.batch import StageGraph
    sg = StageGraph([p['fn'] for p in problems])
    sg.run_eager()
    torch.cuda.synchronize()
    eager = _snapshot(problems)
    sg.capture()
    for _ in range(2):
        sg.replay()
    torch.cuda.synchronize()
    graph = _snapshot(problems)
    for p, a, b in zip(_members(problems), eager, graph):
        for x, y in zip(a, b):
            if not torch.equal(x, y):
                d = (x - y).abs().reshape(x.shape[0], -1).amax(1)
                raise AssertionError(
                    f"{p['name']}: graph replay differs from the eager launches "
                    f"(max |diff| {float(d.max()):.3e} of max |Q| "
                    f"{float(x.abs().max()):.3e}, slots "
                    f"{torch.nonzero(d).flatten().tolist()})")
    assert all(torch.isfinite(x).all() for a in graph for x in a)


def _projected(ref, prm):
    """The minimal-L2 conservation correction the VHS problems apply."""
    g = np.meshgrid(prm['c0'], prm['c0'], prm['c0'], indexing='ij')
    cv = np.stack([x.ravel() for x in g])
    phi = np.vstack([np.ones(cv.shape[1]), cv, np.sum(cv ** 2, axis=0)])
    G = (phi * prm['cw']) @ phi.T
    return ref - np.linalg.solve(G, (phi * prm['cw']) @ ref.T).T @ phi


def test_every_slot_matches_oracle(problems):
    """Every slot of every problem against the oracle: the six VHS problems
    (FP32 mode with the FP64 conservation projection, applied to the
    oracle's Q as well) and both VSS mixtures (each species' Q is the sum of
    its two pair operators, Q_p = Q_p0(f_p, f_0) + Q_p1(f_p, f_1))."""
    from oracle.collision import VHSTables, VSSTables, vhs_gll_fs, vss_fs
    for p in problems:
        p['fn']()
    torch.cuda.synchronize()
    vss_tabs = {}
    for p in _members(problems):
        prm = p['params']
        if p['name'].startswith('vhs'):
            tab = VHSTables(prm['N'], prm['L'], prm['qz'], prm['qw'], prm['sz'],
                            prm['sw'], prm['gamma'],
                            sphere_factor=prm['sphere_factor'])
            f = p['f'].cpu().numpy()
            Q = p['Q'].cpu().numpy()
            ref = np.stack([vhs_gll_fs(tab, prm['prefac'], x) for x in f])
            ref = _projected(ref, prm)
            for s in range(p['nevals']):
                err = np.linalg.norm(Q[s] - ref[s]) / np.linalg.norm(ref[s])
                assert err < 1e-5, f"{p['name']} slot {s}: rel L2 {err:.3e}"
        else:
            m = prm['masses']
            fs = [x.cpu().numpy() for x in p['f']]
            for sp in range(2):
                Q = p['Q'][sp].cpu().numpy()
                ref = np.zeros_like(Q)
                for q in range(2):
                    key = (prm['gamma'][sp, q], prm['eta'][sp, q],
                           m[q] / (m[sp] + m[q]))
                    if key not in vss_tabs:
                        vss_tabs[key] = VSSTables(
                            prm['N'], prm['L'], prm['qz'], prm['qw'], prm['sz'],
                            prm['sw'], prm['szpre'], *key)
                    ref += np.stack([vss_fs(vss_tabs[key], prm['prefac'][sp, q],
                                            m[sp], m[q], fs[sp][s], fs[q][s])
                                     for s in range(Q.shape[0])])
                for s in range(Q.shape[0]):
                    err = np.linalg.norm(Q[s] - ref[s]) / np.linalg.norm(ref[s])
                    assert err < 1e-5, \
                        f"{p['name']} species {sp} slot {s}: rel L2 {err:.3e}"
