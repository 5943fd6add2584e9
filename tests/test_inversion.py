"""Spline parameterisation of the inflow against the reference's inversion
script (fixtures made from its own functions), on the CPU."""
import numpy as np
import torch

from diffswe2d_b200.inversion import bounded_controls, clamped_bspline_basis, raw_from_controls


def test_basis_matches_reference(golden):
    d = golden("spline")
    for tag, ctl in (("a", 16), ("b", 20), ("c", 16)):
        basis, knots, grev = clamped_bspline_basis(torch.from_numpy(d[f"{tag}_times"]), ctl, 3)
        assert np.allclose(basis.numpy(), d[f"{tag}_basis"], rtol=0, atol=1e-14)
        assert np.allclose(knots.numpy(), d[f"{tag}_knots"], rtol=0, atol=1e-14)
        assert np.allclose(grev.numpy(), d[f"{tag}_greville"], rtol=0, atol=1e-14)
        assert np.allclose(basis.sum(1).numpy(), 1.0)


def test_bounded_controls_match_reference(golden):
    d = golden("spline")
    for tag in ("a", "b", "c"):
        out = bounded_controls(torch.from_numpy(d[f"{tag}_raw"]))
        assert np.allclose(out.numpy(), d[f"{tag}_bounded"], rtol=0, atol=1e-15)


def test_raw_round_trip():
    v = torch.tensor([-0.012, 0.0, 0.015, 0.049], dtype=torch.float64)
    assert torch.allclose(bounded_controls(raw_from_controls(v)), v, atol=1e-12)
