"""Learned scheduler: device forward/backward checked against the CPU
reference, training on engine-logged task costs, counts unchanged by the
schedule, and the schedule's gain over the fixed heuristic on a held-out graph."""
import numpy as np
import pytest

import gpm
import _mlp_ref as ref

pytestmark = pytest.mark.gpu


def test_device_gradient_matches_cpu_reference():
    s = gpm.Sched(seed=3)
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, s.nparams).astype(np.float32)
    s.set_params(p)
    X = rng.normal(0, 1, (777, 8)).astype(np.float32)
    T = rng.normal(0, 1, (777, 6)).astype(np.float32)
    T[rng.random(T.shape) < 0.1] = np.nan
    loss, g = s.grad(X, T)
    assert abs(loss - ref.loss(p, X, T)) <= 1e-4 * max(1.0, abs(loss))
    gr = ref.grad(p, X, T)
    assert np.allclose(g, gr, rtol=2e-3, atol=2e-5), np.abs(g - gr).max()
    idx = rng.choice(s.nparams, 40, replace=False)
    assert np.allclose(gr[idx], ref.fd_grad(p, X, T, idx), rtol=1e-4, atol=1e-7)
    _, _, y = ref.forward(p, X)
    assert np.allclose(s.predict(X), y, rtol=1e-4, atol=1e-4)


HEUR = lambda X: np.where(np.exp2(X[:, 0]) - 1 > 50, 4, 1)  # the fixed schedule: CTA if d > 50, long threshold 64


def totals(X, Y, choice):
    cost = np.exp2(Y) - 1
    return cost[np.arange(len(Y)), choice].sum()


@pytest.fixture(scope="module")
def trained():
    s = gpm.Sched(seed=7)
    rows = 0
    for scale, seed in [(15, 11), (16, 12), (17, 13)]:
        rows += s.collect(gpm.Graph.rmat(scale, 16, seed=seed).orient())
    for n, gam, md, seed in [(60000, 2.2, 24.0, 14), (120000, 2.6, 48.0, 15)]:
        _, a, b = gpm.gen_chung_lu(n, gam, md, seed=seed)
        rows += s.collect(gpm.Graph.from_edges(n, a, b).orient())
    X, Y = s.dataset()
    assert len(X) == rows > 1000 and np.isfinite(Y).all()
    first = s.train(1, 3e-3)
    last = s.train(600, 3e-3)
    return s, first, last


def test_training_reduces_loss(trained):
    s, first, last = trained
    assert last < 0.5 * first, (first, last)


def test_learned_schedule_counts_and_gain(trained):
    s, _, _ = trained
    # held-out graph: different seed and scale
    g = gpm.Graph.rmat(18, 16, seed=99).orient()
    want = g.tc(gpm.V_CENTRIC)
    s.attach(g)
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    g.tc_async(gpm.TC_LEARNED, sp, out.data_ptr())
    torch.cuda.synchronize()
    assert int(out.item()) == want
    # regret on the held-out graph from its own logged costs
    probe = gpm.Sched(seed=1)
    probe.collect(g)
    X, Y = probe.dataset()
    learned = np.argmin(s.predict(X), axis=1)
    best = np.argmin(Y, axis=1)
    t_heur, t_learn, t_best = totals(X, Y, HEUR(X)), totals(X, Y, learned), totals(X, Y, best)
    print(f"held-out R-MAT 18: warp-cycles heuristic {t_heur:.4g} learned {t_learn:.4g} best {t_best:.4g}")
    assert t_best <= t_learn
    assert t_learn <= t_heur, "the trained schedule should not cost more than the fixed heuristic"


def test_scheduler_lifetime():
    """A destroyed scheduler is never used: destroying the process default
    clears it, and a graph whose attached scheduler was destroyed gets an
    error instead of a launch."""
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    g = gpm.Graph.rmat(10, 8, seed=3).orient()
    s = gpm.Sched(seed=5).set_default()
    gpm.Sched._default = None
    s.close()
    with pytest.raises(gpm.GpmError, match="no trained scheduler"):
        g.tc_async(gpm.TC_LEARNED, sp, out.data_ptr())
    s2 = gpm.Sched(seed=6)
    s2.attach(g)
    lib, h = gpm.lib, s2.h
    assert lib.gpm_sched_destroy(h) == 0
    s2.h = None
    with pytest.raises(gpm.GpmError, match="destroyed"):
        g.tc_async(gpm.TC_LEARNED, sp, out.data_ptr())
    assert lib.gpm_sched_set_default(h) != 0
    assert lib.gpm_sched_destroy(h) != 0
    s3 = gpm.Sched.pretrained()
    s3.attach(g)
    g.tc_async(gpm.TC_LEARNED, sp, out.data_ptr())
    torch.cuda.synchronize()
    assert int(out.item()) == g.tc(gpm.V_CENTRIC)
