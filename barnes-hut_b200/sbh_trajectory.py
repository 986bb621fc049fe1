"""Differentiable kick-drift-kick leapfrog on the native tree, with a
checkpointed adjoint (the pattern of the reference's
python/dynamics/gaussian_sigma_likelihood_bh.py:50-124, which differentiates
through lax.scan with a custom_vjp BH acceleration and keeps every step's
residuals).

One KDK step with h = dt / 2 and a = softened self-gravity of the native tree:

    v_h = v + h a(x);   x' = x + dt v_h;   v' = v_h + h a(x')

The backward pass walks the steps in reverse with the adjoints (lx, lv):

    lv_h = lv';  lx' += h J_a(x')^T lv'      (adjoint of the second kick)
    lx = lx';    lv_h += dt lx'              (adjoint of the drift)
    lv = lv_h;   lx += h J_a(x)^T lv_h       (adjoint of the first kick)

J_a(x)^T w and the mass gradient come from one sbh_native_force_vjp (the full
adjoint: query side, direct sources and node moments). The kick at the end
of step n and at the start of step n + 1 see the same positions, so their
cotangents are summed into one force+VJP call per distinct position.

Memory: positions and velocities are kept every `checkpoint_every` steps;
each segment is recomputed forward once during the backward pass (one extra
force evaluation per step).
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

import sbh_b200 as B


@dataclass
class Gravity:
    """Softened self-gravity on the native tree. group_size: most targets per
    walk group (None: the library's default of 96, best for clustered
    systems; 64 suits near-uniform ones such as a perturbed lattice)."""
    beta: float = 1.0 / 0.6
    softening: float = 2e-3
    leaf_size: int = 16
    quadrupole: bool = True
    group_size: int | None = None

    def __post_init__(self):
        self.tree = B.NativeTree()

    def accel(self, x: torch.Tensor, m: torch.Tensor) -> torch.Tensor:
        self.tree.build(x, m, leaf_size=self.leaf_size, with_adjoint=False, group_size=self.group_size)
        return self.tree.force(beta=self.beta, softening=self.softening, quadrupole=self.quadrupole)

    def accel_vjp(self, x: torch.Tensor, m: torch.Tensor, w: torch.Tensor):
        """(J_a(x)^T w, d(w . a)/dm)."""
        self.tree.build(x, m, leaf_size=self.leaf_size, with_adjoint=True, group_size=self.group_size)
        _, gx, gm = self.tree.force_vjp(w, beta=self.beta, softening=self.softening, quadrupole=self.quadrupole,
                                        want_force=False)
        return gx, gm


def kdk(x, v, m, steps: int, dt: float, grav: Gravity, a0=None):
    """Integrate `steps` KDK steps; returns (x, v, a(x_final))."""
    h = 0.5 * dt
    a = grav.accel(x, m) if a0 is None else a0
    for _ in range(steps):
        v = v + h * a
        x = x + dt * v
        a = grav.accel(x, m)
        v = v + h * a
    return x, v, a


def forward_with_checkpoints(x0, v0, m, steps: int, dt: float, grav: Gravity, checkpoint_every: int = 10):
    """Forward pass keeping (x, v) every `checkpoint_every` steps."""
    ckpts = [(x0.clone(), v0.clone())]
    x, v, a = x0, v0, None
    done = 0
    while done < steps:
        k = min(checkpoint_every, steps - done)
        x, v, a = kdk(x, v, m, k, dt, grav, a0=a)
        done += k
        if done < steps:
            ckpts.append((x.clone(), v.clone()))
    return x, v, ckpts


def adjoint(ckpts, lx_T, lv_T, m, steps: int, dt: float, grav: Gravity, checkpoint_every: int = 10):
    """Reverse pass from the adjoints of the final state; returns
    (lx_0, lv_0, dL/dm)."""
    h = 0.5 * dt
    lx, lv = lx_T.clone(), lv_T.clone()
    gm = torch.zeros_like(m)
    seg_starts = list(range(0, steps, checkpoint_every))
    pending = None  # cotangent of a(x) waiting to be merged with the next kick at the same x
    for si in reversed(range(len(seg_starts))):
        s0 = seg_starts[si]
        k = min(checkpoint_every, steps - s0)
        x, v = ckpts[si]
        xs = [x]
        a = grav.accel(x, m)
        for _ in range(k):  # recompute the segment's positions
            v = v + h * a
            x = x + dt * v
            a = grav.accel(x, m)
            v = v + h * a
            xs.append(x)
        for j in reversed(range(k)):
            # second kick of step j: v' = v_h + h a(x_{j+1})
            w = h * lv if pending is None else h * lv + pending
            gx, g_m = grav.accel_vjp(xs[j + 1], m, w)
            lx = lx + gx
            gm = gm + g_m
            # drift: x_{j+1} = x_j + dt v_h
            lv = lv + dt * lx
            # first kick: v_h = v_j + h a(x_j); merged with the previous step's second kick
            pending = h * lv
    # the first kick of step 0 at x_0
    gx, g_m = grav.accel_vjp(ckpts[0][0], m, pending)
    lx = lx + gx
    gm = gm + g_m
    return lx, lv, gm
