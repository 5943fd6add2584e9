"""Inflow inversion through the adjoint on a small runup problem: the gauge
misfit falls under Adam, and the gradient of the whole chunked simulation
agrees with finite differences of the simulated misfit."""
import pytest
import torch

from diffswe2d_b200.inversion import invert, make_runup_problem

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def small_problem():
    return make_runup_problem(cases=2, seed=3, ny=61, nx=98, dx=0.056, duration=6.0, dt_out=0.3,
                              n_controls=8, n_gauges=3, device=DEV)


def test_inversion_reduces_gauge_misfit(small_problem):
    problem, raw_true = small_problem
    raw0 = torch.zeros_like(raw_true)  # controls at 0.015 m (middle of the bounds)
    res = invert(problem, raw0, lr=0.02, max_iters=40, rmse_tol=1e-6)
    first, last = res.rmse_history[0], res.rmse_history[-1]
    print("rmse first", first, "last", last, "s/iter", res.seconds_per_iteration)
    for b in range(problem.batch):
        assert last[b] < 0.6 * first[b]


def test_chunked_gradient_matches_finite_differences(small_problem):
    problem, raw_true = small_problem
    raw = (raw_true + 0.3).detach().requires_grad_(True)
    sim = problem.simulate(problem.series(raw))
    loss = ((sim - problem.targets) ** 2).mean(dim=(1, 2)).sum()
    loss.backward()
    g = raw.grad.detach().cpu().numpy()

    def f(r):
        with torch.no_grad():
            s = problem.simulate(problem.series(r), differentiable=False)
            return float(((s - problem.targets) ** 2).mean(dim=(1, 2)).sum().double())

    eps = 2e-2
    for b, k in ((0, 2), (1, 5)):
        up, dn = raw.detach().clone(), raw.detach().clone()
        up[b, k] += eps
        dn[b, k] -= eps
        fd = (f(up) - f(dn)) / (2 * eps)
        print("control", b, k, "adjoint", g[b, k], "FD", fd)
        assert abs(g[b, k] - fd) <= 0.05 * abs(fd) + 1e-9
