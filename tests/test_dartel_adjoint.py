"""The hand-written DARTEL data-term adjoint.

CPU: the oracle's restatement of the reference's Gauss-Newton gradient is
pinned bit for bit to the reference's own output (``dartel_adjoint_golden``),
and the oracle's exact adjoint is checked against float64 central finite
differences (h = 1e-4) and against that reference gradient (equal at k = 0;
cosine >= 0.99 for k = 3 and 7, where the reference's pull-back is an
approximation of the derivative).  GPU: ``dartel_data_term``'s forward and
backward against the oracle, finite differences on the device, checkpoint
intervals, batching with per-registration output weights, float32.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import dartel as od

G = np.load(GOLDEN / "dartel_adjoint_golden.npz")
S, T, V = G["source"], G["target"], G["velocity"]
KS = tuple(int(k) for k in G["ks"])


def _fd_pairs(objective, v, count=16, h=1e-4, seed=1):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        c, y, x = rng.integers(2), rng.integers(v.shape[1]), rng.integers(v.shape[2])
        vp, vm = v.copy(), v.copy()
        vp[c, y, x] += h
        vm[c, y, x] -= h
        out.append(((c, y, x), (objective(vp) - objective(vm)) / (2 * h)))
    return out


@pytest.mark.parametrize("k", KS)
def test_oracle_pinned_to_reference_gradient(k):
    np.testing.assert_array_equal(od.gauss_newton_gradient(V, S, T, k), G[f"gradient_{k}"])
    assert od.data_term(V, S, T, k) == G[f"objective_{k}"]


@pytest.mark.parametrize("k", (0, 3, 7))
def test_oracle_adjoint_matches_finite_differences(k):
    g = od.data_term_gradient(V, S, T, k)
    pairs = _fd_pairs(lambda v: od.data_term(v, S, T, k), V)
    fd = np.array([p[1] for p in pairs])
    got = np.array([g[idx] for idx, _ in pairs])
    assert np.abs(got - fd).max() <= 1e-6 * np.abs(fd).max()


@pytest.mark.parametrize("k", KS)
def test_oracle_adjoint_against_reference_gradient(k):
    g = od.data_term_gradient(V, S, T, k)
    ref = G[f"gradient_{k}"]
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    cosine = float((g * ref).sum() / (np.linalg.norm(g) * np.linalg.norm(ref)))
    if k == 0:
        assert rel <= 1e-12
    else:
        assert cosine >= 0.99 and rel <= 0.15


# ------------------------------------------------------------------ GPU


def _cuda(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("k", (0, 3, 7))
def test_gpu_forward_and_backward_match_oracle(native_library, k):
    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term

    v = _cuda(V).requires_grad_(True)
    e = dartel_data_term(v, _cuda(S), _cuda(T), k)
    np.testing.assert_allclose(float(e.detach()), G[f"objective_{k}"], rtol=1e-13)
    e.backward()
    want = od.data_term_gradient(V, S, T, k)
    got = v.grad.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_gpu_gradient_matches_finite_differences(native_library):
    """64 x 32 float64, k = 7, central differences with h = 1e-4 of the device objective."""

    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term

    k = 7
    s_dev, t_dev = _cuda(S), _cuda(T)
    v = _cuda(V).requires_grad_(True)
    dartel_data_term(v, s_dev, t_dev, k).backward()
    g = v.grad.cpu().numpy()
    pairs = _fd_pairs(lambda w: float(dartel_data_term(_cuda(w), s_dev, t_dev, k)), V, count=24, seed=7)
    fd = np.array([p[1] for p in pairs])
    got = np.array([g[idx] for idx, _ in pairs])
    assert np.abs(got - fd).max() <= 1e-6 * np.abs(fd).max()


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_the_gradient(native_library):
    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term

    grads = []
    for every in (1, 2, 3, 7):
        v = _cuda(V).requires_grad_(True)
        dartel_data_term(v, _cuda(S), _cuda(T), 7, checkpoint_every=every).backward()
        grads.append(v.grad.cpu().numpy())
    for g in grads[1:]:
        assert np.abs(g - grads[0]).max() <= 1e-13 * np.abs(grads[0]).max()


@pytest.mark.gpu
def test_batched_registrations_with_output_weights(native_library):
    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term

    batch, k = 4, 5
    src = np.stack([synthetic.smooth_sheet(32, 64, 40 + b) for b in range(batch)])
    tgt = np.stack([synthetic.smooth_sheet(32, 64, 60 + b) for b in range(batch)])
    vel = np.stack([np.stack([synthetic.smooth_sheet(32, 64, 80 + 2 * b + c) - 0.5 for c in range(2)]) * 2.0
                    for b in range(batch)])
    weights = np.array([1.0, -0.5, 2.0, 0.25])
    v = _cuda(vel).requires_grad_(True)
    energies = dartel_data_term(v, _cuda(src), _cuda(tgt), k)
    (energies * _cuda(weights)).sum().backward()
    for b in range(batch):
        np.testing.assert_allclose(float(energies[b].detach()), od.data_term(vel[b], src[b], tgt[b], k), rtol=1e-13)
        want = weights[b] * od.data_term_gradient(vel[b], src[b], tgt[b], k)
        assert np.abs(v.grad[b].cpu().numpy() - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_float32_gradient_tracks_float64(native_library):
    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term

    v32 = _cuda(V, torch.float32).requires_grad_(True)
    dartel_data_term(v32, _cuda(S, torch.float32), _cuda(T, torch.float32), 7).backward()
    want = od.data_term_gradient(V, S, T, 7)
    rel = np.linalg.norm(v32.grad.cpu().numpy() - want) / np.linalg.norm(want)
    assert rel <= 1e-3  # float32 rounding (6e-8) grows through 7 squarings of the map (measured 1.4e-4)
