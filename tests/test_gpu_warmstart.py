"""What the learned warm start gains over the plain inversion, at a small
scale (half the runup resolution in each direction twice over: 61 x 98 at
5.6 cm; 2048 training runs): the network trained by its own kernels on
solver-generated runs predicts held-out controls far better than the cold
start, and the inversion seeded with it starts and ends at a lower gauge
misfit than the same inversion from the cold start."""
import numpy as np
import pytest
import torch

from diffswe2d_b200.inversion import RunupFamily
from diffswe2d_b200.warmstart import WarmStartNet
from diffswe2d_b200.warmstart_study import compare, generate, train

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def trained():
    fam = RunupFamily(ny=61, nx=98, dx=0.056, seed=3, device=DEV)
    data = generate(fam, 2048, seed=11)
    assert data.x.shape == (2048, 6, 1125) and torch.isfinite(data.x).all()
    net = WarmStartNet(DEV, seed=0)
    log = train(net, data, epochs=20, batch=128, lr=2e-3)
    print("data", data.seconds, "s;", data.cell_updates / data.seconds / 1e6, "Mcell/s; train",
          log.seconds, "s; val rmse", log.val_rmse_m, "losses", log.train_loss[::5])
    return fam, net, log


def test_training_fits_controls(trained):
    fam, net, log = trained
    assert log.train_loss[-1] < 0.5 * log.train_loss[0]
    # controls ~ U[-0.012, 0.015]: their spread about the mean is 7.8 mm
    assert log.val_rmse_m < 0.0045


def test_warm_start_beats_cold_start(trained):
    fam, net, _ = trained
    r = compare(fam, net, cases=6, seed=99, max_iters=40, tol=1e-4)
    cold, warm = r["cold"], r["warm"]
    print(r)
    ci, wi = np.array(cold["initial_rmse"]), np.array(warm["initial_rmse"])
    cf, wf = np.array(cold["final_rmse"]), np.array(warm["final_rmse"])
    assert np.median(wi) < 0.5 * np.median(ci)
    assert np.median(wf) < np.median(cf)
