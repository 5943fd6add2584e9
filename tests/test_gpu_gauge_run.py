"""gauge_run (whole run as one autograd node, device clock, checkpointed
adjoint) against the reference's loop of one forward() call per output
interval: gauges and final state bit for bit, gradients to 1e-6."""
import numpy as np
import pytest
import torch

from diffswe2d_b200 import SWE2D, SWEConfig, scenarios
from diffswe2d_b200.adjoint import forward_checkpointed
from diffswe2d_b200.gauge_run import GaugeRunWorkspace, _RecordFull, gauge_run

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
GAUGES = [(20, 30), (31, 12), (40, 55), (20, 30)]


def _model(B, seed=2):
    sc = scenarios.runup(ny=61, nx=98, dx=0.056, seed=seed)
    bed = torch.from_numpy(sc.bed).to(DEV)
    n = torch.from_numpy(sc.roughness).to(DEV)
    if B > 1:
        bump = torch.linspace(0.0, 0.004, B, device=DEV).view(B, 1, 1, 1)
        bed = (bed.view(1, 1, *bed.shape) + bump).contiguous()
        n = n.view(1, 1, *n.shape).expand(B, 1, *n.shape).contiguous()
    m = SWE2D(bed, n, sc.dx, sc.dy, config=SWEConfig(**sc.config), train_dem=False)
    h0 = torch.clamp(-m.bed.detach(), min=0.0).expand(B, 1, 61, 98)
    U0 = torch.cat([h0, torch.zeros_like(h0), torch.zeros_like(h0)], dim=1).contiguous()
    return m, U0


def _levels(B, n_out):
    t = torch.arange(n_out, dtype=torch.float32, device=DEV)
    return torch.stack([0.012 * torch.sin(0.4 * t + b) + 0.004 for b in range(B)])


def _chunked(m, U0, levels, out_dt, grad):
    U, out = U0, []
    for i in range(levels.shape[-1]):
        lv = levels[:, i] if levels.ndim == 2 else levels[i]
        if grad:
            U = forward_checkpointed(m, U, t_end=out_dt, boundary_level=lv)
        else:
            with torch.no_grad():
                U, _ = m(U, t_end=out_dt, start_time=i * out_dt, boundary_level=lv)
        bed = m.bed  # differentiable when the DEM correction requires grad
        out.append(torch.stack([U[:, 0, iy, ix] + bed[:, 0, iy, ix].expand(U.shape[0])
                                for iy, ix in GAUGES], dim=-1))
    return torch.stack(out, dim=1), U


@pytest.mark.parametrize("B,shared", [(1, True), (3, False)])
def test_forward_matches_chunked_forward_calls(B, shared):
    m, U0 = _model(B)
    levels = _levels(B, 12)
    lv = levels[0] if shared else levels
    ref_g, ref_U = _chunked(m, U0, lv, 0.25, grad=False)
    with torch.no_grad():
        g, U = gauge_run(m, U0, lv, 0.25, GAUGES, graph_steps=4, checkpoint_every=8)
    assert torch.equal(g, ref_g)
    assert torch.equal(U, ref_U)


@pytest.mark.parametrize("B,store", [(1, False), (2, False), (1, True), (2, True)])
def test_gradients_match_chunked_checkpointed_autograd(B, store):
    """Both backward modes: states recomputed from checkpoints (store=False)
    and every step's state kept from the forward pass (store=True)."""
    out = []
    for mode in ("run", "chunks"):
        m, U0 = _model(B)
        m.roughness_length.requires_grad_(True)
        U0 = U0.clone().requires_grad_(True)
        levels = _levels(B, 8).requires_grad_(True)
        w = torch.linspace(-1.0, 2.0, B * 8 * len(GAUGES), device=DEV).view(B, 8, len(GAUGES))
        if mode == "run":
            g, U = gauge_run(m, U0, levels, 0.2, GAUGES, graph_steps=2, checkpoint_every=6,
                             store_states=store)
        else:
            g, U = _chunked(m, U0, levels, 0.2, grad=True)
        loss = (w * g).sum() + 1e-2 * (U * U).sum()
        loss.backward()
        out.append((levels.grad.cpu().numpy(), U0.grad.cpu().numpy(),
                    m.roughness_length.grad.cpu().numpy(), g.detach().cpu().numpy()))
    (gl_r, gu_r, gn_r, g_r), (gl_c, gu_c, gn_c, g_c) = out
    assert np.array_equal(g_r, g_c)

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
    print("levels", rel(gl_r, gl_c), "U0", rel(gu_r, gu_c), "n", rel(gn_r, gn_c))
    assert np.abs(gl_c).max() > 0
    assert rel(gl_r, gl_c) <= 1e-6
    assert rel(gu_r, gu_c) <= 1e-6
    assert rel(gn_r, gn_c) <= 1e-6


def test_record_overflow_is_reported_and_retried():
    m, U0 = _model(1)
    levels = _levels(1, 6)[0]
    ws = GaugeRunWorkspace(m, 1, 61, 98, U0.device, 1, 6, GAUGES, graph_steps=2, checkpoint_every=2,
                           record_cap=3)
    with pytest.raises(_RecordFull):
        ws.run(U0, levels.view(-1, 1), 0.25)
    with torch.no_grad():
        g, _ = gauge_run(m, U0, levels, 0.25, GAUGES)
        ref, _ = _chunked(m, U0, levels, 0.25, grad=False)
    assert torch.equal(g, ref)


def test_backward_after_workspace_reuse_raises():
    m, U0 = _model(1)
    levels = _levels(1, 4)[0].clone().requires_grad_(True)
    g1, _ = gauge_run(m, U0, levels, 0.2, GAUGES)
    g2, _ = gauge_run(m, U0, levels, 0.2, GAUGES)
    g2.sum().backward()
    with pytest.raises(RuntimeError, match="ran again"):
        g1.sum().backward()


@pytest.mark.parametrize("store", [False, True])
def test_bed_gradient_matches_chunked_autograd(store):
    """gauge_run's bed (DEM correction) gradient equals the chunk-by-chunk
    forward_checkpointed gradient."""
    out = []
    for mode in ("run", "chunks"):
        m, U0 = _model(1)
        m.dem_correction_parameter.requires_grad_(True)
        levels = _levels(1, 6)
        if mode == "run":
            g, U = gauge_run(m, U0, levels, 0.2, GAUGES, graph_steps=2, checkpoint_every=6,
                             store_states=store)
        else:
            g, U = _chunked(m, U0, levels, 0.2, grad=True)
        (g.sum() + 1e-2 * (U * U).sum()).backward()
        out.append(m.dem_correction_parameter.grad.cpu().numpy())
    a, b = out
    assert np.abs(b).max() > 0
    assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


def test_tuned_checkpoint_interval(tmp_path, monkeypatch):
    """checkpoint_every=None: the autotuner times the run for every k of
    CHECKPOINT_CHOICES, caches the fastest and the run uses it; gradients do
    not depend on k (bit for bit), so the choice is purely a speed one."""
    from diffswe2d_b200 import autotune
    from diffswe2d_b200.gauge_run import _WORKSPACES
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    monkeypatch.setattr(autotune, "_tuned", {})
    m, U0 = _model(2)
    levels = _levels(2, 40)
    U = U0.clone().requires_grad_(True)
    L = levels.clone().requires_grad_(True)
    g, _ = gauge_run(m, U, L, 0.25, GAUGES, checkpoint_every=None)
    g.square().sum().backward()
    ws = list(_WORKSPACES.values())[0]
    assert ws.k in autotune.CHECKPOINT_CHOICES
    tuned = autotune.checkpoint_tuning(DEV)
    assert len(tuned) == 1 and list(tuned.values())[0]["k"] == ws.k
    monkeypatch.setattr(autotune, "_tuned", {})  # the cache is read back from disk
    assert autotune.tuned_checkpoint_every(m, U0, levels, 0.25, GAUGES) == ws.k
    grads = []
    for k in (32, 256):
        U2 = U0.clone().requires_grad_(True)
        L2 = levels.clone().requires_grad_(True)
        g2, _ = gauge_run(m, U2, L2, 0.25, GAUGES, checkpoint_every=k)
        g2.square().sum().backward()
        assert torch.equal(g2, g)
        grads.append((U2.grad, L2.grad))
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])
    assert torch.equal(grads[0][0], U.grad) and torch.equal(grads[0][1], L.grad)
