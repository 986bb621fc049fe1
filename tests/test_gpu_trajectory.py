"""GPU: the checkpointed leapfrog adjoint (sbh_trajectory) against float64
torch autograd of the same kick-drift-kick integration with the direct sum.
beta = 1e6 opens every node, so the tree evaluates the exact direct sum and
the two integrations differ only by float32 rounding."""
import numpy as np
import pytest
import torch

import sbh_trajectory as T
import sbh_workloads as W

pytestmark = pytest.mark.gpu


def _direct_accel64(x, m, eps):
    d = x[:, None, :] - x[None, :, :]
    r2 = (d * d).sum(-1)
    return (-(m[None, :] * (r2 + eps * eps + 1e-12) ** -1.5)[..., None] * d).sum(1)


@pytest.mark.parametrize("ckpt", [1, 3, 10])
def test_trajectory_adjoint_matches_float64_autograd(cuda, ckpt):
    p, m, disp = W.perturbed_lattice(8, seed=3, rms_cells=0.2)
    eps, dt, steps = 2e-2, 2e-3, 7
    rng = np.random.default_rng(4)
    target = p + rng.normal(scale=1e-3, size=p.shape).astype(np.float32)
    lattice = (p - disp).astype(np.float32)
    grav = T.Gravity(beta=1e6, softening=eps, leaf_size=16)
    x0 = torch.tensor(p, device=cuda)
    v0 = torch.zeros_like(x0)
    mt = torch.tensor(m, device=cuda)
    xT, vT, ck = T.forward_with_checkpoints(x0, v0, mt, steps, dt, grav, checkpoint_every=ckpt)
    tgt = torch.tensor(target, device=cuda)
    n = x0.shape[0]
    lx = 2.0 * (xT - tgt) / (n * 3)
    lx0, lv0, gm = T.adjoint(ck, lx, torch.zeros_like(lx), mt, steps, dt, grav, checkpoint_every=ckpt)

    d64 = torch.tensor(disp, dtype=torch.float64, requires_grad=True)
    m64 = torch.tensor(m, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(lattice, dtype=torch.float64) + d64
    v = torch.zeros_like(x)
    h = 0.5 * dt
    a = _direct_accel64(x, m64, eps)
    for _ in range(steps):
        v = v + h * a
        x = x + dt * v
        a = _direct_accel64(x, m64, eps)
        v = v + h * a
    loss = ((x - torch.tensor(target, dtype=torch.float64)) ** 2).mean()
    loss.backward()
    np.testing.assert_allclose(xT.cpu().numpy(), x.detach().numpy(), rtol=1e-5, atol=1e-6)
    g = d64.grad.numpy()
    err = np.linalg.norm(lx0.cpu().numpy() - g) / np.linalg.norm(g)
    assert err < 1e-3, err
    gme = np.linalg.norm(gm.cpu().numpy() - m64.grad.numpy()) / np.linalg.norm(m64.grad.numpy())
    assert gme < 1e-3, gme


def test_trajectory_adjoint_at_config5_settings_against_float64_direct(cuda):
    """Config 5's integration settings (theta 0.6, eps 2e-3, dt 1e-3, 50
    kick-drift-kick steps, checkpoints every 10) on an 8^3 perturbed lattice:
    the tree's trajectory and its checkpointed adjoint against float64
    autograd of the direct-sum integration; the gap is the tree's force
    error carried through the steps."""
    p, m, disp = W.perturbed_lattice(8, seed=5, rms_cells=0.2)
    eps, dt, steps, ckpt = 2e-3, 1e-3, 50, 10
    target = p + np.random.default_rng(6).normal(scale=1e-3, size=p.shape).astype(np.float32)
    lattice = (p - disp).astype(np.float32)
    grav = T.Gravity(beta=1.0 / 0.6, softening=eps, leaf_size=16)
    x0 = torch.tensor(p, device=cuda)
    mt = torch.tensor(m, device=cuda)
    xT, vT, ck = T.forward_with_checkpoints(x0, torch.zeros_like(x0), mt, steps, dt, grav, checkpoint_every=ckpt)
    tgt = torch.tensor(target, device=cuda)
    n = x0.shape[0]
    lx = 2.0 * (xT - tgt) / (n * 3)
    lx0, _, gm = T.adjoint(ck, lx, torch.zeros_like(lx), mt, steps, dt, grav, checkpoint_every=ckpt)

    d64 = torch.tensor(disp, dtype=torch.float64, requires_grad=True)
    m64 = torch.tensor(m, dtype=torch.float64, requires_grad=True)
    x = torch.tensor(lattice, dtype=torch.float64) + d64
    v = torch.zeros_like(x)
    h = 0.5 * dt
    a = _direct_accel64(x, m64, eps)
    for _ in range(steps):
        v = v + h * a
        x = x + dt * v
        a = _direct_accel64(x, m64, eps)
        v = v + h * a
    loss = ((x - torch.tensor(target, dtype=torch.float64)) ** 2).mean()
    loss.backward()
    xe = np.linalg.norm(xT.cpu().numpy() - x.detach().numpy()) / np.linalg.norm(x.detach().numpy())
    g = d64.grad.numpy()
    ge = np.linalg.norm(lx0.cpu().numpy() - g) / np.linalg.norm(g)
    me = np.linalg.norm(gm.cpu().numpy() - m64.grad.numpy()) / np.linalg.norm(m64.grad.numpy())
    print(f"config-5 settings, 512 particles: final positions {xe:.2e}, d/d displacements {ge:.2e}, d/d masses {me:.2e}")
    assert xe < 1e-5  # measured 1.6e-7
    assert ge < 5e-4  # measured 5.5e-5
    assert me < 1e-4  # measured 6.1e-6
