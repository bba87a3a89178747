"""The learned warm start end to end on a small member of the parametric family (fine level 7,
network grid level 5): device assembly, FP64-multigrid training data, training with the library's
own forward/backward kernels, and what the trained network gains over the zero initial guess on
unseen instances at the same stopping test (||d|| <= 1e-8 ||b||).

What the tests pin: the network learns (validation error well below that of a zero prediction), a
warm start never costs iterations on average (the defect test rejects bad starts), both starts reach
the same solution, and the mechanism itself gains: the exact solution sampled on the network grid,
used as the start the same way, saves at least one PCG iteration on average -- the ceiling any
network can approach."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UNSEEN = range(10_000, 10_032)


@pytest.fixture(scope="module")
def trained(featlib, cuda):
    from featb200.warmstart import ParametricFamily, WarmStart
    fam = ParametricFamily(level=7, net_level=5, precision="f64")
    X, Y, its = fam.generate(range(0, 1024))
    ws = WarmStart(fam, max_batch=32, seed=0)
    hist = ws.fit(X, Y, epochs=30, batch=32, lr=3e-3)
    return fam, ws, hist, its


def test_network_learns(trained, cuda):
    fam, ws, hist, its = trained
    assert np.all(np.isfinite(hist))
    assert hist[-1] < 0.1 * hist[0], hist
    Xv, Yv, _ = fam.generate(UNSEEN)
    err = [float((ws.predict(Xv[j]) - Yv[j]).norm() / Yv[j].norm()) for j in range(len(UNSEEN))]
    print("validation relative error: median", np.median(err))
    assert np.median(err) < 0.25


def test_warm_start_gain(trained):
    from featb200.warmstart import evaluate
    fam, ws, hist, its = trained
    rows = evaluate(ws, UNSEEN)
    assert all(r["ok"] for r in rows)
    zero = np.array([r["it_zero"] for r in rows])
    warm = np.array([r["it_warm"] for r in rows])
    print("iterations zero/warm", zero.mean(), warm.mean(), "network start used",
          np.mean([r["used"] for r in rows]), "median d0/|b|", np.median([r["d0_ratio"] for r in rows]))
    assert warm.mean() <= zero.mean()
    assert np.all(warm <= zero + 1)
    assert max(r["rel_diff"] for r in rows) <= 1e-6


def test_exact_start_ceiling(trained, cuda):
    """The same start built from the exact solution on the network grid saves >= 1 iteration."""
    torch = cuda
    fam, ws, hist, its = trained
    zero, warm = [], []
    for k in UNSEEN:
        fam.setup(k)
        x = torch.zeros(fam.n, dtype=torch.float64, device="cuda")
        _, it0 = fam.solve(x)
        x0 = fam.prolongate(fam.restrict_solution(x).clone())
        _, it1 = fam.solve(x0)
        zero.append(it0)
        warm.append(it1)
    print("exact-start iterations zero/warm", np.mean(zero), np.mean(warm))
    assert np.mean(warm) <= np.mean(zero) - 1.0


def test_fallback_to_zero(trained):
    """A network whose prediction is useless (every parameter 1: a huge output) is rejected by the
    defect test and the solve starts from zero."""
    fam, ws, hist, its = trained
    p = ws.net.get_params()
    try:
        ws.net.set_params(np.ones_like(p))
        fam.setup(10_100)
        x0, used, ratio = ws.initial_guess(10_100)
        assert not used
        assert float(x0.abs().max().item()) == 0.0
    finally:
        ws.net.set_params(p)
