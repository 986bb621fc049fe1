"""GPU: the library's kernels on the reference's own octree8 buffers (from
the golden fixtures) reproduce the reference's recorded outputs, including
the stochastic estimator at fixed seeds (same curand streams)."""
import os

import numpy as np
import pytest

import sbh_b200 as B
from conftest import rel_l2

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", ["uniform_d5", "plummer_d5"])
def test_kernels_on_reference_buffers(cuda, case):
    path = os.path.join(GOLD, "octree8_reference.npz")
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    g = np.load(path)
    leaf, node, q, cot = g[case + "_leaf"], g[case + "_node"], g[case + "_queries"], g[case + "_cot"]
    got = B.barnes_hut_force_octree8(leaf, node, q, beta=2.0).cpu().numpy()
    assert rel_l2(got, g[case + "_bh_beta2"]) < 1e-5
    for tag, (eps, cut, prune, mult) in {"soft": (5e-2, 1.5, False, 4.0), "softprune": (5e-2, 0.3, True, 2.0),
                                         "plummer": (1e-3, 1e6, True, 4.0)}.items():
        kw = dict(beta=2.0, softening_scale=eps, cutoff_scale=cut, prune_enabled=prune, prune_r_cut_mult=mult)
        got = B.softened_barnes_hut_force_octree8(leaf, node, q, **kw).cpu().numpy()
        assert rel_l2(got, g[case + f"_{tag}"]) < 1e-5
        got = B.softened_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **kw).cpu().numpy()
        assert rel_l2(got, g[case + f"_{tag}_vjp"]) < 1e-5
    for seed in (7, 11):
        for soft in (0, 1):
            kw = dict(samples_per_subdomain=2, seed=seed, beta=1.0)
            if soft:
                kw.update(softening_scale=5e-2, cutoff_scale=1.5, prune_enabled=True, prune_r_cut_mult=4.0)
                f = B.softened_stochastic_barnes_hut_force_octree8(leaf, node, q, **kw)
                v = B.softened_stochastic_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **kw)
            else:
                f = B.stochastic_barnes_hut_force_octree8(leaf, node, q, **kw)
                v = B.stochastic_barnes_hut_force_octree8_vjp(leaf, node, q, cot, **kw)
            for got, want in ((f, g[case + f"_stoch_s{seed}_soft{soft}"]),
                              (v, g[case + f"_stoch_s{seed}_soft{soft}_vjp"])):
                got = got.cpu().numpy()
                row = np.linalg.norm(got - want, axis=1) / np.maximum(np.linalg.norm(want, axis=1), 1e-30)
                assert row.max() < 1e-4  # every row on the reference's sampled paths
