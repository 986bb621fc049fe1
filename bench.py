"""Benchmark: force+VJP evaluations per second of softened self-gravity at
N = 1,048,576 per system (Plummer spheres, a = 1, truncated at 10a, equal
masses, epsilon = 1e-3, theta = 0.5 i.e. beta = 2, float32). One evaluation
= the softened force of every particle of one system + the full adjoint
(d/d positions and masses of sum w . a for a random cotangent w).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--systems S] [--impl reference]

Batched step (the timed region): S systems (default 8) in one forest, one
build + one fused force/adjoint walk + one finalize for all of them; value =
S evaluations / step time. The same step captured in a CUDA graph, the plain
path (build, force, rebuild, force+VJP as separate calls on one system) and
the reference algorithm on this GPU (dense octree8 through the
reference-compatible entry points) are reported beside it.

One process per GPU (torchrun for N > 1); every rank evaluates its own
independent systems (replicas, weak scaling; the path needs no collective).
Timing: CUDA events on the launching stream, L2 flushed (256 MB write)
between steps outside the timed events, the max over ranks. Rank 0 prints one
JSON line.

--impl reference times the reference's own CPU path (its Tree3D build and
evaluateBarnesHut_stackless, compiled from its headers into oracle/_ref)
with all host threads on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "barnes-hut_b200"))

import sbh_workloads as W  # noqa: E402

N_DEFAULT = 1 << 20
BETA = 2.0
EPS = 1e-3
LEAF = 16
METRIC = "force+VJP evals/sec at N=1M, rel-L2<=1e-4 vs FP64 direct; batched vs plain"


def workload(n: int, systems: int) -> str:
    return f"plummer_n{n}_eps1e-3_theta0.5_force_plus_full_vjp_{systems}_systems_per_step"


EXTRAS = ("octree8_plain", "opening_sweep", "forest", "sharded_single_system", "winding_number",
          "winding_number_mesh", "treepm_short_range", "stochastic_octree8", "direct_sum", "trajectory")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="particles per system")
    ap.add_argument("--systems", type=int, default=8, help="systems batched in one step")
    ap.add_argument("--cpu-sample", type=int, default=32768, help="queries timed by the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the octree8, forest, winding-number, stochastic and trajectory measurements")
    ap.add_argument("--extra", action="append", default=None, choices=EXTRAS,
                    help="run only the named extra measurements (repeatable; default: all)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU code (oracle/_ref), bounded sample
# ---------------------------------------------------------------------------
def cpu_reference_eval_time(points, masses, sample: int, threads: int):
    """Seconds for one force+VJP evaluation of the full system by the
    reference's CPU path, extrapolated from a timed sample of queries."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sbh_oracle as O

    n = points.shape[0]
    rng = np.random.default_rng(123)
    idx = np.sort(rng.choice(n, min(sample, n), replace=False))
    q = points[idx]
    cot = rng.normal(size=q.shape).astype(np.float32)
    t0 = time.perf_counter()
    tree = O.RefTree3D(points, masses, variant=0)  # Tree3D<8,1>: leaf size 8
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, counts = tree.eval(q, BETA, O.REF_K_SOFT_FORCE, eps=EPS, threads=threads)
    t_force = time.perf_counter() - t0
    t0 = time.perf_counter()
    tree.eval(q, BETA, O.REF_K_SOFT_FORCE_VJP, eps=EPS, cot=cot, threads=threads)
    t_vjp = time.perf_counter() - t0
    scale = n / q.shape[0]
    # num_contribs of evaluateBarnesHut_stackless (include/barnes_hut.h:29,45,50): the interactions each
    # query takes under the reference's own per-target opening rule
    return t_build + (t_force + t_vjp) * scale, dict(build_s=t_build, force_sample_s=t_force, vjp_sample_s=t_vjp,
                                                     sample_queries=int(q.shape[0]),
                                                     interactions_per_query=float(np.mean(counts)))


def reference_gpu_plugin_time(points, masses, cot):
    """The reference's own GPU plugin (its src/sbh_ffi.cu, unmodified, built
    for sm_100a into oracle/_ref/libsbh_ref_gpu.so) on this GPU, through its
    handlers in the order of the reference's custom_vjp recompute flow
    (python/jax_sbh_ffi.py:1804-1891): octree8 build at depth 7 (corners =
    data min/max -+ 1e-3), softened force, rebuild, softened query-side VJP,
    all N queries, "no cutoff" = 1e6 box lengths, pruning off. One warm-up
    evaluation on 4,096 queries loads the module; one full evaluation is
    timed with CUDA events (it includes the handlers' own cudaMalloc, frees
    and stream synchronisations)."""
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import sbh_oracle as O

    L = O.refgpu()
    dev = torch.device("cuda", 0)
    n = points.shape[0]
    depth = 7
    total = O.octree8_total_nodes(depth)
    P = torch.as_tensor(points, device=dev)
    M = torch.as_tensor(masses, device=dev)
    C = torch.as_tensor(cot, device=dev)
    Z = torch.zeros_like(P)
    MN = torch.as_tensor(points.min(0) - np.float32(1e-3), device=dev)
    MX = torch.as_tensor(points.max(0) + np.float32(1e-3), device=dev)
    leaf = torch.empty(n * 32, dtype=torch.uint8, device=dev)
    node = torch.empty(total * 104, dtype=torch.uint8, device=dev)
    con = torch.empty(total * 32, dtype=torch.uint8, device=dev)
    f = torch.empty((n, 3), device=dev)
    g = torch.empty((n, 3), device=dev)
    cut = 1e6 * float((points.max(0) - points.min(0)).max())
    s = torch.cuda.current_stream().cuda_stream

    def evaluate(nq):
        O.refgpu_check(L.ref_build_octree8(s, P.data_ptr(), Z.data_ptr(), M.data_ptr(), n, MN.data_ptr(),
                                           MX.data_ptr(), leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                           con.data_ptr(), con.numel(), depth))
        O.refgpu_check(L.ref_bh_force_octree8_soft(s, leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                                   P.data_ptr(), nq, f.data_ptr(), BETA, EPS, cut, 0, 4.0, 0, 1.0,
                                                   256))
        O.refgpu_check(L.ref_build_octree8(s, P.data_ptr(), Z.data_ptr(), M.data_ptr(), n, MN.data_ptr(),
                                           MX.data_ptr(), leaf.data_ptr(), leaf.numel(), node.data_ptr(), node.numel(),
                                           con.data_ptr(), con.numel(), depth))
        O.refgpu_check(L.ref_bh_force_octree8_soft_vjp(s, leaf.data_ptr(), leaf.numel(), node.data_ptr(),
                                                       node.numel(), P.data_ptr(), nq, C.data_ptr(), g.data_ptr(),
                                                       BETA, EPS, cut, 0, 4.0, 0, 1.0, 256))

    evaluate(4096)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    evaluate(n)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return dict(ms_per_eval=ms, evals_per_s=1000.0 / ms, n=n, max_depth=depth,
                what="the reference's unmodified GPU plugin: octree8 build, softened force, rebuild, softened "
                     "query-side VJP of all N queries (its custom_vjp recompute flow)")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    p, m = W.plummer(args.n, seed=1000)
    times = []
    info = {}
    for s in range(args.warmup + args.steps):
        t, info = cpu_reference_eval_time(p, m, args.cpu_sample, threads)
        if s >= args.warmup:
            times.append(t)
    t = statistics.mean(times)
    value = 1.0 / t
    sample = (f"Tree3D<8,1> build of all {args.n} points + force and query-side VJP of "
              f"{info['sample_queries']} sampled particles, extrapolated x{args.n / info['sample_queries']:.0f}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": workload(args.n, args.systems), "n": args.n, "beta": BETA, "softening": EPS, "leaf_size": 8,
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "detail": info,
    }
    try:
        import torch

        if torch.cuda.is_available():
            cot = np.random.default_rng(5).normal(size=p.shape).astype(np.float32)
            line["reference_gpu_plugin"] = reference_gpu_plugin_time(p, m, cot)
    except (ImportError, OSError, RuntimeError) as e:  # plugin not built here: the CPU line stands alone
        line["reference_gpu_plugin"] = {"unavailable": str(e).splitlines()[0][:200]}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def fp64_direct_subset(points_d, masses_d, idx, eps):
    """Float64 direct sum at a subset of targets (plain PyTorch, chunked)."""
    import torch

    p = points_d.double()
    m = masses_d.double()
    q = p[idx]
    out = torch.zeros_like(q)
    for a in range(0, q.shape[0], 64):
        d = q[a:a + 64, None, :] - p[None, :, :]
        r2 = (d * d).sum(-1)
        c = -m[None, :] * (r2 + eps * eps + 1e-12) ** -1.5
        out[a:a + 64] = (c[..., None] * d).sum(1)
    return out


def opening_sweep_measurement(B, torch, P0, M0, W0, idx, ref, flush):
    """How much of the walk the accuracy bar needs: one 2^20 system's fused
    force + full adjoint (the step's kernel, same settings) at openings beta
    = 1/theta from the configuration's 2 down to 1.25, with the force's
    rel-L2 against the FP64 direct sum on the accuracy subset. The headline
    stays at theta = 0.5; this only states the headroom."""
    tree = B.NativeTree().build(P0, M0)
    out = dict(what="build once; force + full adjoint per beta (CUDA events, L2 flushed)", points=[])
    for beta in (2.0, 1.75, 1.5, 1.25):
        f, _, _ = tree.force_vjp(W0, beta=beta, softening=EPS)
        torch.cuda.synchronize()
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tree.force_vjp(W0, beta=beta, softening=EPS)
        e1.record()
        torch.cuda.synchronize()
        rel = float(torch.linalg.norm(f[idx].double() - ref) / torch.linalg.norm(ref))
        out["points"].append(dict(beta=beta, theta=1.0 / beta, force_vjp_ms=e0.elapsed_time(e1),
                                  rel_l2_vs_fp64_direct=rel))
    tree.release()
    return out


def forest_measurement(B, torch, dev, rank, world, flush):
    """Config 4: 256 Plummer systems, N log-uniform in [1e3, 2e5]. Batched =
    one forest build + one fused force/adjoint walk for all systems; plain =
    build, force, rebuild, VJP per system (the recompute flow). Systems are
    sharded across ranks with no collective."""
    import sbh_dist

    systems, sizes = W.forest(256, 1000, 200000, seed=0)
    a, b = sbh_dist.shard_systems(sizes, world, rank)
    mine = systems[a:b]
    pts = torch.tensor(np.concatenate([s[0] for s in mine]), device=dev)
    ms = torch.tensor(np.concatenate([s[1] for s in mine]), device=dev)
    offs = torch.tensor(sbh_dist.system_offsets([s[0].shape[0] for s in mine]), device=dev)
    w = torch.randn(pts.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
    n = pts.shape[0]
    F, GX, GM = torch.empty_like(pts), torch.empty_like(pts), torch.empty(n, device=dev)
    prm = B.NativeTree.params(BETA, EPS, 0.0, True)
    tree = B.NativeTree(dev)
    # leaf and group size autotuned on this forest (outside the timed region)
    tune = B.autotune_native(pts, ms, offs, adjoint=True, beta=BETA, softening=EPS)
    leaf, group = tune["leaf_size"], tune["group_size"]

    def batched():
        tree.build(pts, ms, system_offsets=offs, leaf_size=leaf, with_adjoint=True, group_size=group)
        tree.adjoint_walk(w, prm, F)
        tree.adjoint_finalize(GX, GM)

    trees = [B.NativeTree(dev) for _ in range(2)]
    views = [(pts[o0:o1], ms[o0:o1], w[o0:o1]) for o0, o1 in zip(offs[:-1].tolist(), offs[1:].tolist())]

    def plain():
        for p_, m_, w_ in views:
            trees[0].build(p_, m_, leaf_size=leaf, with_adjoint=False, group_size=group)
            trees[0].force(beta=BETA, softening=EPS)
            trees[1].build(p_, m_, leaf_size=leaf, with_adjoint=True, group_size=group)
            trees[1].force_vjp(w_, beta=BETA, softening=EPS, want_force=False)

    # CUDA graph of the batched step (build + walk + finalize, no host sync inside)
    batched()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        batched()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            batched()
    torch.cuda.current_stream(dev).wait_stream(s)
    torch.cuda.synchronize()

    def timed(fn, reps):
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / reps

    plain()
    t_plain = timed(plain, 2)
    t_batched = timed(batched, 3)
    t_graph = timed(g.replay, 3)
    del g
    # accuracy of the graph's forces: 512 targets of the largest and of the smallest system against
    # the FP64 direct sum over their own system
    acc = {}
    sizes_mine = [s_[0].shape[0] for s_ in mine]
    for tag, si in (("largest", int(np.argmax(sizes_mine))), ("smallest", int(np.argmin(sizes_mine)))):
        o0, o1 = int(offs[si]), int(offs[si + 1])
        sub = torch.tensor(np.random.default_rng(7).choice(o1 - o0, min(512, o1 - o0), replace=False), device=dev)
        ref = fp64_direct_subset(pts[o0:o1], ms[o0:o1], sub, EPS)
        acc[tag] = dict(particles=o1 - o0, rel_l2_vs_fp64_direct=float(
            torch.linalg.norm(F[o0:o1][sub].double() - ref) / torch.linalg.norm(ref)))
    return dict(systems=int(b - a), particles=int(n), plain_ms=t_plain, batched_ms=t_batched, graph_ms=t_graph,
                accuracy=acc,
                batched_over_plain=t_plain / t_graph,
                particle_evals_per_s_graph=n / (t_graph * 1e-3), particle_evals_per_s_plain=n / (t_plain * 1e-3),
                autotuned=dict(leaf_size=leaf, group_size=group, trials=tune["trials"]))


def stochastic_measurement(B, torch, P0, M0, idx, ref, flush):
    """Config 2a, stochastic variant: the reference's stochastic octree8
    estimator (MLPCV, src/sbh_ffi.cu:2146-2291) at all 2^20 particles of the
    Plummer system, depth-7 tree; the error against the FP64 direct sum on
    the 1,024-target accuracy subset. The reference has no "nodes per query"
    knob: samples_per_subdomain draws that many particle paths in each of the
    (up to 512) depth-3 subdomains of a query, and each path evaluates the 8
    children of every node it descends through. 32 paths per subdomain is
    the configuration's "32 samples"; 1 path per subdomain is the fewest the
    estimator allows. Classic octree8 BH on the same queries beside it."""
    Q = P0.contiguous()
    Z = torch.zeros_like(P0)
    span = float((P0.max(0).values - P0.min(0).values).max())
    leaf, node = B.build_octree8_buffers(P0, Z, M0, max_depth=7)
    kw = dict(beta=BETA, softening_scale=EPS, cutoff_scale=1e6 * span, prune_enabled=False)

    def timed(fn, warm):
        if warm:
            fn()
            torch.cuda.synchronize()
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    rel = lambda f: float(torch.linalg.norm(f[idx].double() - ref) / torch.linalg.norm(ref))  # noqa: E731
    out = dict(queries=int(Q.shape[0]), max_depth=7,
               mapping=("samples_per_subdomain = particle paths per depth-3 subdomain (the reference has no "
                        "nodes-per-query knob); s32 is the configuration's 32 samples"))
    for sps in (1, 32):
        st, st_ms = timed(lambda: B.softened_stochastic_barnes_hut_force_octree8(  # noqa: B023
            leaf, node, Q, samples_per_subdomain=sps, seed=3, **kw), warm=sps == 1)
        out[f"stochastic_s{sps}"] = dict(ms=st_ms, queries_per_s=Q.shape[0] / (st_ms * 1e-3),
                                         rel_l2_vs_fp64_direct=rel(st))
    cl, cl_ms = timed(lambda: B.softened_barnes_hut_force_octree8(leaf, node, Q, **kw), warm=True)
    out["classic"] = dict(ms=cl_ms, queries_per_s=Q.shape[0] / (cl_ms * 1e-3), rel_l2_vs_fp64_direct=rel(cl))
    # the native stochastic estimator (sbh_native_stochastic_force): the group
    # walk at beta_coarse plus 32 drawn tree nodes per query refined to beta = 2
    tree = B.NativeTree().build(P0, M0)
    nat = dict(samples=32, what=("group walk at beta_coarse + 32 tree nodes per query (shared by a target group) "
                                 "drawn by octupole size and refined to beta 2; unbiased for the beta-2 force walk"))
    for bc in (1.0, 1.25, 1.5):
        st, st_ms = timed(lambda: tree.stochastic_force(beta=BETA, beta_coarse=bc, samples=32, seed=3,  # noqa: B023
                                                        softening=EPS), warm=True)
        nat[f"beta_coarse_{bc}"] = dict(ms=st_ms, queries_per_s=Q.shape[0] / (st_ms * 1e-3),
                                        rel_l2_vs_fp64_direct=rel(st))
    W0s = torch.randn_like(P0)
    for bc in (1.0, 1.5):
        _, vj_ms = timed(lambda: tree.stochastic_force_vjp(W0s, beta=BETA, beta_coarse=bc, samples=32,  # noqa: B023
                                                          seed=3, softening=EPS, want_force=False), warm=True)
        nat[f"beta_coarse_{bc}"]["vjp_ms"] = vj_ms
    nat["vjp_what"] = ("gradients w.r.t. all positions and masses of sum(w . estimate), the draws held fixed "
                       "(one adjoint walk + finalize)")
    _, cv_ms = timed(lambda: tree.force_vjp(W0s, beta=BETA, softening=EPS, want_force=False), warm=True)
    nat["force_walk_vjp_ms"] = cv_ms
    wk, wk_ms = timed(lambda: tree.force(beta=BETA, softening=EPS, quadrupole_radius=0.0, quadrupole_linear=0.0),
                      warm=True)
    nat["force_walk_beta_2"] = dict(ms=wk_ms, rel_l2_vs_fp64_direct=rel(wk),
                                    what="the estimator's expectation: force walk at beta 2, quadrupole everywhere")
    tree.release()
    out["native"] = nat
    return out


def trajectory_measurement(torch, dev, flush):
    """Config 5: 128^3 perturbed lattice (2,097,152 particles, P(k) ~ k^-2,
    rms 0.2 cell), eps 2e-3, theta 0.6, 50 kick-drift-kick steps of dt 1e-3;
    gradient of the mean squared final-position error to a seeded target
    with respect to the initial displacements, checkpointing every 10 steps
    (sbh_trajectory: native force and full adjoint per step)."""
    import sbh_b200 as B
    import sbh_trajectory as T

    p, m, disp = W.perturbed_lattice(128, seed=5, rms_cells=0.2)
    target = p + np.random.default_rng(6).normal(scale=1e-3, size=p.shape).astype(np.float32)
    x0 = torch.tensor(p, device=dev)
    v0 = torch.zeros_like(x0)
    mt = torch.tensor(m, device=dev)
    tgt = torch.tensor(target, device=dev)
    # leaf and group size autotuned on the initial positions (outside the timed region)
    tune = B.autotune_native(x0, mt, adjoint=True, beta=1.0 / 0.6, softening=2e-3)
    grav = T.Gravity(beta=1.0 / 0.6, softening=2e-3, leaf_size=tune["leaf_size"], group_size=tune["group_size"])
    steps, dt, ck = 50, 1e-3, 10
    T.kdk(x0, v0, mt, 1, dt, grav)  # warm-up (workspaces)
    torch.cuda.synchronize()
    flush.zero_()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    xT, vT, ckpts = T.forward_with_checkpoints(x0, v0, mt, steps, dt, grav, checkpoint_every=ck)
    e1.record()
    n = x0.shape[0]
    lx = 2.0 * (xT - tgt) / (n * 3)
    gx0, gv0, gm = T.adjoint(ckpts, lx, torch.zeros_like(lx), mt, steps, dt, grav, checkpoint_every=ck)
    e2.record()
    torch.cuda.synchronize()
    fwd, bwd = e0.elapsed_time(e1), e1.elapsed_time(e2)
    # the per-step force's error: the initial positions' force (theta 0.6, eps 2e-3, the autotuned
    # tree) against the FP64 direct sum on 1,024 particles
    tree = B.NativeTree(dev).build(x0, mt, leaf_size=tune["leaf_size"], with_adjoint=False,
                                   group_size=tune["group_size"])
    f0 = tree.force(beta=1.0 / 0.6, softening=2e-3)
    sub = torch.tensor(np.random.default_rng(8).choice(n, 1024, replace=False), device=dev)
    ref = fp64_direct_subset(x0, mt, sub, 2e-3)
    force_rel = float(torch.linalg.norm(f0[sub].double() - ref) / torch.linalg.norm(ref))
    tree.release()
    return dict(particles=int(n), steps=steps, checkpoint_every=ck, forward_ms=fwd, backward_ms=bwd,
                force_rel_l2_vs_fp64_direct=force_rel,
                total_s=(fwd + bwd) * 1e-3, force_evals=steps + 1, recomputed_forces=steps,
                force_vjp_evals=steps + 1, grad_norm=float(torch.linalg.norm(gx0)),
                loss=float(((xT - tgt) ** 2).mean()),
                autotuned=dict(leaf_size=tune["leaf_size"], group_size=tune["group_size"], trials=tune["trials"]))


def winding_measurement(B, torch, dev, flush):
    """Config 2b: winding number of 262,144 oriented points on the ellipsoid
    (1, 0.7, 0.5) at 1,048,576 queries uniform in [-1.5, 1.5]^3."""
    pts, nrm, wgt = W.ellipsoid_surface(262144, seed=2)
    q = W.uniform_box_queries(1048576, seed=3)
    inside = torch.tensor(W.ellipsoid_inside(q), device=dev)
    P, N, M, Q = (torch.tensor(a, device=dev) for a in (pts, nrm, wgt, q))
    tree = B.NativeTree(dev)

    def step():
        tree.build(P, M, normals=N, leaf_size=LEAF, with_adjoint=False)
        return tree.winding_number(Q, beta=BETA)

    out = step()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(3):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = step()
        e1.record()
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / 3
    err_in = float((out[inside] - 1.0).abs().mean())
    err_out = float(out[~inside].abs().mean())
    # against the FP64 direct sum (signedSolidAngle) at 1,024 of the queries
    sub = np.random.default_rng(9).choice(q.shape[0], 1024, replace=False)
    Qs = Q[sub].double()
    P64, N64, M64 = P.double(), N.double(), M.double()
    ref64 = torch.zeros(1024, dtype=torch.float64, device=dev)
    for a in range(0, 1024, 32):
        d = P64[None, :, :] - Qs[a:a + 32, None, :]
        r = torch.linalg.norm(d, dim=2)
        ref64[a:a + 32] = ((M64[None, :] * (d * N64[None, :, :]).sum(2)) / (4.0 * np.pi * (r ** 3 + 1e-5))).sum(1)
    rel64 = float(torch.linalg.norm(out[sub].double() - ref64) / torch.linalg.norm(ref64))
    del P64, N64, M64
    # the adjoint with respect to queries, source positions, normals and weights (one walk + finalize)
    vtree = B.NativeTree(dev).build(P, M, normals=N, leaf_size=LEAF, with_adjoint=True)
    U = torch.tensor(np.random.default_rng(4).normal(size=q.shape[0]).astype(np.float32), device=dev)

    def vstep():
        vtree.build(P, M, normals=N, leaf_size=LEAF, with_adjoint=True)
        return vtree.winding_number_vjp(Q, U, beta=BETA, want_value=True)

    vstep()
    torch.cuda.synchronize()
    flush.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    vstep()
    e1.record()
    torch.cuda.synchronize()
    vjp_ms = e0.elapsed_time(e1)
    # the reference's algorithm on this GPU: its adaptive Tree3D<1,3> (leaf size 1, built here on the
    # device with the reference CPU builder's bytes) and its warp-vote traversal (src/sbh_gpu.cu)
    def ref_step():
        leaf, node = B.build_octree_buffers(P, N, M, backend="cpu")
        return B.eval_barnes_hut_wn(leaf, node, Q, beta=BETA)[0]

    ref_step()
    torch.cuda.synchronize()
    flush.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rout = ref_step()
    e1.record()
    torch.cuda.synchronize()
    ref_ms = e0.elapsed_time(e1)
    return dict(sources=262144, queries=1048576, ms=ms, queries_per_s=1048576 / (ms * 1e-3),
                mean_abs_err_inside=err_in, mean_abs_err_outside=err_out, rel_l2_vs_fp64_direct=rel64,
                fp64_subset=1024,
                vjp_ms=vjp_ms, vjp_what=("build + winding number and its adjoint with respect to queries, source "
                                         "positions, normals and weights (one walk + finalize)"),
                reference_algorithm_ms=ref_ms, speedup_vs_reference_algorithm=ref_ms / ms,
                reference_algorithm_mean_abs_err_inside=float((rout[inside] - 1.0).abs().mean()),
                reference_algorithm_mean_abs_err_outside=float(rout[~inside].abs().mean()),
                reference_algorithm="Tree3D<1,3> (leaf size 1) + warp-vote Barnes-Hut, beta 2, both on this GPU")


def winding_mesh_measurement(B, torch, dev, flush):
    """Config 2b on mesh-sampled sources: 262,144 points sampled on the
    device from a closed torus mesh (R 1, r 0.4, 16,384 triangles), the tree
    built on them, and the winding number at 1,048,576 queries uniform in
    [-1.5, 1.5]^3. One step = sample + build + walk."""
    V, F = W.torus_mesh(1.0, 0.4, 128, 64)
    Vt = torch.tensor(V, device=dev)
    Ft = torch.tensor(F, device=dev)
    q = W.uniform_box_queries(1048576, seed=3)
    inside = torch.tensor(W.torus_inside(q), device=dev)
    qd = np.abs(np.sqrt((np.sqrt(q[:, 0].astype(np.float64) ** 2 + q[:, 1] ** 2) - 1.0) ** 2 + q[:, 2] ** 2) - 0.4)
    away = torch.tensor(qd > 0.05, device=dev)
    Q = torch.tensor(q, device=dev)
    tree = B.NativeTree(dev)
    ns = 262144

    def step():
        P, N, M = B.sample_points_on_mesh(ns, Vt, Ft, seed=1, device=dev)
        tree.build(P, M, normals=N, leaf_size=LEAF, with_adjoint=False)
        return tree.winding_number(Q, beta=BETA)

    out = step()
    torch.cuda.synchronize()
    # median of 5: the sampler's status read synchronises, so a host-side
    # pause inside that call would otherwise land in a single mean
    tot, tsamp = [], []
    for _ in range(5):
        flush.zero_()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        P, N, M = B.sample_points_on_mesh(ns, Vt, Ft, seed=1, device=dev)
        e1.record()
        tree.build(P, M, normals=N, leaf_size=LEAF, with_adjoint=False)
        out = tree.winding_number(Q, beta=BETA)
        e2.record()
        torch.cuda.synchronize()
        tot.append(e0.elapsed_time(e2))
        tsamp.append(e0.elapsed_time(e1))
    ms = float(np.median(tot))
    err_in = float((out[inside & away] - 1.0).abs().mean())
    err_out = float(out[~inside & away].abs().mean())
    return dict(mesh_faces=int(F.shape[0]), sources=ns, queries=1048576, ms=ms, sample_ms=float(np.median(tsamp)),
                queries_per_s=1048576 / (ms * 1e-3), mean_abs_err_inside=err_in, mean_abs_err_outside=err_out,
                note="errors over queries farther than 0.05 from the surface; the sampler's status check "
                     "synchronises once per call")


def treepm_measurement(B, torch, dev, flush):
    """Short-range half of a TreePM step at scale, in the reference's TreePM
    units (python/cosmology/treepm_jaxpm_demo.py:59-78, defaults :305-331):
    a 128^3 perturbed lattice (2,097,152 particles, rms displacement 0.5
    cells) in a periodic box of 128 mesh cells, r_split 1 cell, softening 0.1,
    beta 1.7, cells beyond 4 r_split pruned. The native periodic walk (build +
    force with target groups of 64, the size for walks bounded by a prune
    radius; also timed with 32 and 96) against the reference's algorithm on this GPU (dense octree8 of
    depth 6, the reference's traversal with the same prune), both checked
    against the FP64 minimum-image erfc direct sum on 1,024 particles."""
    k = 128
    pts, m, _ = W.perturbed_lattice(k, seed=11, rms_cells=0.5)
    L = float(k)
    pts = np.mod(pts.astype(np.float64) * L, L).astype(np.float32)
    m = np.full(pts.shape[0], 1.0, np.float32)
    rs, eps, beta, mult = 1.0, 0.1, 1.7, 4.0
    P, M = torch.tensor(pts, device=dev), torch.tensor(m, device=dev)
    Z = torch.zeros_like(P)
    idx = np.random.default_rng(12).choice(pts.shape[0], 1024, replace=False)
    q = P[idx].double()
    ref = torch.zeros((1024, 3), dtype=torch.float64, device=dev)
    src, ms = P.double(), M.double()
    for a in range(0, 1024, 64):
        d = q[a:a + 64, None, :] - src[None, :, :]
        d -= L * torch.floor(d / L + 0.5)
        r2 = (d * d).sum(-1)
        dist = torch.sqrt(r2 + 1e-12)
        u = dist / (2 * rs)
        att = torch.special.erfc(u) + 2.0 / np.sqrt(np.pi) * u * torch.exp(-u * u)
        ref[a:a + 64] = -(ms[None, :, None] * (att * (r2 + eps * eps + 1e-12) ** -1.5)[..., None] * d).sum(1)
        del d, r2, dist, u, att
    tree = B.NativeTree(dev)
    F = torch.empty_like(P)
    kw = dict(beta=beta, softening=eps, cutoff=rs, quadrupole=False, periodic=True, box_length=L,
              prune_radius=mult * rs)

    def ours(group_size=None):
        tree.build(P, M, leaf_size=LEAF, with_adjoint=False, group_size=group_size)
        tree.force(out=F, **kw)

    lo = torch.zeros(3, device=dev)
    hi = torch.full((3,), L, device=dev)

    def refalg():
        leaf, node = B.build_octree8_buffers(P, Z, M, lo, hi, max_depth=6)
        return B.softened_barnes_hut_force_octree8(leaf, node, P, beta=beta, softening_scale=eps, cutoff_scale=rs,
                                                   prune_enabled=True, prune_r_cut_mult=mult, periodic=True,
                                                   box_length=L)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        tot, out = 0.0, None
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps, out

    ours32_ms, _ = timed(lambda: ours(32), 3)
    ours96_ms, _ = timed(lambda: ours(96), 3)
    ours128_ms, _ = timed(lambda: ours(B.native_group_size()), 3)
    ours_ms, _ = timed(lambda: ours(64), 3)
    st = tree.stats()
    rel = float(torch.linalg.norm(F[idx].double() - ref) / torch.linalg.norm(ref))
    ref_ms, o8 = timed(refalg, 1)
    rel_o8 = float(torch.linalg.norm(o8[idx].double() - ref) / torch.linalg.norm(ref))
    return dict(particles=int(pts.shape[0]), box_cells=k, r_split=rs, prune_radius=mult * rs, softening=eps,
                beta=beta, group_size=64, ms=ours_ms, ms_with_32_target_groups=ours32_ms,
                ms_with_96_target_groups=ours96_ms, ms_with_128_target_groups=ours128_ms,
                rel_l2_vs_fp64_direct=rel,
                interactions_per_particle=(st["far"] + st["near"]) / pts.shape[0],
                octree8_reference_algorithm_ms=ref_ms, octree8_rel_l2_vs_fp64_direct=rel_o8,
                speedup_vs_reference_algorithm=ref_ms / ours_ms)


def sharded_measurement(B, torch, dev, rank, world, n):
    """Strong scaling of one system (runs when world > 1): n Plummer
    particles split by target across the ranks (sbh_dist.sharded_force_vjp).
    Every rank builds the same tree, walks its share of the target groups,
    and one all-reduce of forces and gradients (n x 28 bytes) completes the
    result on every rank. Timed per evaluation (build + walk + finalize +
    all-reduce, max over ranks) beside the same evaluation on one rank."""
    import sbh_dist

    p, m = W.plummer(n, seed=999)
    w = np.random.default_rng(998).normal(size=p.shape).astype(np.float32)
    P, M, Wt = (torch.tensor(a, device=dev) for a in (p, m, w))
    tree = B.NativeTree(dev)

    def sharded():
        tree.build(P, M, leaf_size=LEAF, with_adjoint=True)
        return sbh_dist.sharded_force_vjp(tree, Wt, beta=BETA, softening=EPS)

    def single():
        tree.build(P, M, leaf_size=LEAF, with_adjoint=True)
        return tree.force_vjp(Wt, beta=BETA, softening=EPS)

    def timed(fn, reps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    for _ in range(2):
        sharded()
    single()
    sh_ms = sbh_dist.max_over_ranks(timed(sharded, 5), dev)
    one_ms = timed(single, 3)
    f, gx, _ = sharded()
    f1, gx1, _ = single()
    torch.cuda.synchronize()
    rel_f = sbh_dist.max_over_ranks(float(torch.linalg.norm(f - f1) / torch.linalg.norm(f1)), dev)
    rel_g = sbh_dist.max_over_ranks(float(torch.linalg.norm(gx - gx1) / torch.linalg.norm(gx1)), dev)
    return dict(particles=n, ranks=world, sharded_ms=sh_ms, single_rank_ms=one_ms, speedup=one_ms / sh_ms,
                allreduce_bytes=int(n * 28), rel_force_vs_single=rel_f, rel_grad_vs_single=rel_g)


def direct_measurement(B, torch, P0, M0, W0, flush):
    """The direct sums (the reference's SoftenedDirectForce and its VJP,
    src/sbh_ffi.cu:503-546): all 2^20 x 2^20 pairs of the first Plummer
    system, softening 1e-3, no cutoff (the reference's convention: a cutoff
    of 1e6 box lengths). One launch each."""
    span = float((P0.max(0).values - P0.min(0).values).max())
    kw = dict(softening_scale=1e-3, cutoff_scale=span * 1e6)
    out = {}
    for name, fn in (("force", lambda: B.softened_direct_force(P0, M0, P0, **kw)),
                     ("vjp", lambda: B.softened_direct_force_vjp(P0, M0, P0, W0, **kw))):
        fn()
        torch.cuda.synchronize()
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        pairs = float(P0.shape[0]) ** 2
        out[name] = dict(ms=ms, pair_interactions_per_s=pairs / (ms * 1e-3))
    return dict(sources=int(P0.shape[0]), queries=int(P0.shape[0]), **out)


def measure_fp32_peak(B, torch, dev):
    """FP32 FMA peak in TFLOP/s: the faster of independent scalar FMA chains
    and the same chains two per instruction (packed FFMA2, which the walks
    issue); both run the same flops."""
    buf = torch.zeros(4096, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    blocks, iters = 148 * 16, 2048
    flops = blocks * 256 * 8 * 16 * iters * 2
    best = 0.0
    for probe in (B.lib().sbh_probe_fp32, B.lib().sbh_probe_fp32x2):
        for _ in range(2):
            probe(stream, buf.data_ptr(), blocks, 64)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B._check(probe(stream, buf.data_ptr(), blocks, iters), "probe_fp32")
        e1.record()
        torch.cuda.synchronize()
        best = max(best, flops / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def octree8_plain_measurement(B, torch, P0, M0, W0, idx, ref, flush):
    """The reference's own algorithm on this GPU: the dense octree8 build
    (depth 7, corners = data min/max -+ 1e-3) + softened force + (rebuild) +
    query-side VJP, as separate calls through the reference-compatible
    entry points, the custom_vjp recompute flow of the reference's
    softened_barnes_hut_force_octree8. "No cutoff" in the reference's
    convention is cutoff = 1e6 x the box size; pruning is off."""
    span = float((P0.max(0).values - P0.min(0).values).max())
    cut = 1e6 * span
    kw = dict(beta=BETA, softening_scale=EPS, cutoff_scale=cut, prune_enabled=False)
    Z = torch.zeros_like(P0)

    def call():
        leaf, node = B.build_octree8_buffers(P0, Z, M0, max_depth=7)
        f = B.softened_barnes_hut_force_octree8(leaf, node, P0, **kw)
        leaf, node = B.build_octree8_buffers(P0, Z, M0, max_depth=7)
        B.softened_barnes_hut_force_octree8_vjp(leaf, node, P0, W0, **kw)
        return f

    f = call()
    torch.cuda.synchronize()
    rel = float(torch.linalg.norm(f[idx].double() - ref) / torch.linalg.norm(ref))
    flush.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    call()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # the block size of the warp-cooperative traversal (warps of 32 Morton-ordered queries per block)
    leaf, node = B.build_octree8_buffers(P0, Z, M0, max_depth=7)
    tuned = B.autotune_octree8(leaf, node, P0, **kw)
    return dict(ms_per_eval=ms, evals_per_s=1000.0 / ms, rel_l2_vs_fp64_direct=rel, max_depth=7,
                note="query-side VJP only (the reference's VJP has no source or mass terms)",
                threads=256, force_threads_autotuned=tuned)


def run_ours(args):
    import torch
    import torch.distributed as dist

    import sbh_b200 as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, K = args.n, args.systems
    systems = [W.plummer(n, seed=1000 + rank * K + s) for s in range(K)]
    p = np.concatenate([s_[0] for s_ in systems])
    m = np.concatenate([s_[1] for s_ in systems])
    offs = np.arange(K + 1, dtype=np.int64) * n
    w = np.random.default_rng(77 + rank).normal(size=p.shape).astype(np.float32)
    P = torch.tensor(p, device=dev)
    M = torch.tensor(m, device=dev)
    Wt = torch.tensor(w, device=dev)
    OFFS = torch.tensor(offs, device=dev) if K > 1 else None
    F = torch.empty_like(P)
    GX = torch.empty_like(P)
    GM = torch.empty_like(M)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    prm = B.NativeTree.params(BETA, EPS, 0.0, True)
    tree = B.NativeTree(dev)
    tree.build(P, M, system_offsets=OFFS, leaf_size=LEAF, with_adjoint=True)  # sizes the workspace

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def run_step():
        tree.build(P, M, system_offsets=OFFS, leaf_size=LEAF, with_adjoint=True)
        tree.adjoint_walk(Wt, prm, F)
        tree.adjoint_finalize(GX, GM)

    def step():
        s0, s1, s2 = ev(), ev(), ev()
        s0.record()
        tree.build(P, M, system_offsets=OFFS, leaf_size=LEAF, with_adjoint=True)
        s1.record()
        tree.adjoint_walk(Wt, prm, F)
        s2.record()
        tree.adjoint_finalize(GX, GM)
        return s0, s1, s2

    # accuracy of the timed configuration (outside the timed region): system 0
    step()
    torch.cuda.synchronize()
    idx = torch.tensor(np.random.default_rng(5).choice(n, 1024, replace=False), device=dev)
    ref = fp64_direct_subset(P[:n], M[:n], idx, EPS)
    rel = float(torch.linalg.norm(F[idx].double() - ref) / torch.linalg.norm(ref))
    # rows whose own relative error exceeds 5% (outlier_frac of unified_force_benchmark.py:316-328)
    row_rel = torch.linalg.norm(F[idx].double() - ref, dim=1) / torch.linalg.norm(ref, dim=1).clamp_min(1e-12)
    outlier_frac = float((row_rel > 0.05).double().mean())
    st = tree.stats()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms, walk_ms, build_ms = 0.0, 0.0, 0.0
    marks = []
    for _ in range(args.steps):
        flush.zero_()
        a, b, c = step()
        d = ev()
        d.record()
        marks.append((a, b, c, d))
    torch.cuda.synchronize()
    for a, b, c, d in marks:
        total_ms += a.elapsed_time(d)
        walk_ms += b.elapsed_time(c)
        build_ms += a.elapsed_time(b)
    clocks = sampler.stop()
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * K * 1000.0 / ms_per_step

    # the same step captured in one CUDA graph and replayed
    g = torch.cuda.CUDAGraph()
    gs_ = torch.cuda.Stream(dev)
    gs_.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(gs_):
        run_step()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=gs_):
            run_step()
    torch.cuda.current_stream(dev).wait_stream(gs_)
    torch.cuda.synchronize()
    graph_ms = 0.0
    for _ in range(2):
        flush.zero_()
        a, b = ev(), ev()
        a.record()
        g.replay()
        b.record()
        torch.cuda.synchronize()
        graph_ms += a.elapsed_time(b)
    graph_ms /= 2
    del g

    # plain path on system 0: separate C-ABI calls, the tree rebuilt for the
    # VJP (the reference's custom_vjp recompute flow)
    P0, M0, W0 = P[:n], M[:n], Wt[:n]
    F0 = torch.empty_like(P0)
    t1, t2 = B.NativeTree(dev), B.NativeTree(dev)

    def plain():
        t1.build(P0, M0, leaf_size=LEAF, with_adjoint=False)
        t1.force(beta=BETA, softening=EPS, out=F0)
        t2.build(P0, M0, leaf_size=LEAF, with_adjoint=True)
        t2.force_vjp(W0, beta=BETA, softening=EPS, want_force=False)

    def plain_force():
        t1.build(P0, M0, leaf_size=LEAF, with_adjoint=False)
        t1.force(beta=BETA, softening=EPS, out=F0)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            a, b = ev(), ev()
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps

    plain_ms = timed(plain, 2)
    force_ms = timed(plain_force, 2)
    plain_force_rel = float(torch.linalg.norm(F0[idx].double() - ref) / torch.linalg.norm(ref))

    # e2e: host buffers in, host buffers out, through the public API. Every
    # step uploads its own inputs from pinned host memory and reads its own
    # results back, inside the timed region; as a serving loop would, the
    # copies run on two side streams against two device buffer sets, so the
    # upload of step s + 1 and the download of step s - 1 overlap the walk of
    # step s. The inputs (235 MB) are larger than L2, so no flush is needed.
    Ph, Mh, Wh = (torch.tensor(a_).pin_memory() for a_ in (p, m, w))
    Fh = [torch.empty(P.shape).pin_memory() for _ in range(2)]
    GXh = [torch.empty(P.shape).pin_memory() for _ in range(2)]
    GMh = [torch.empty(M.shape).pin_memory() for _ in range(2)]
    Pd = [torch.empty_like(P) for _ in range(2)]
    Md = [torch.empty_like(M) for _ in range(2)]
    Wd = [torch.empty_like(Wt) for _ in range(2)]
    Fd = [torch.empty_like(F) for _ in range(2)]
    GXd = [torch.empty_like(GX) for _ in range(2)]
    GMd = [torch.empty_like(GM) for _ in range(2)]
    comp = torch.cuda.current_stream(dev)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def e2e_run(steps):
        free = [None, None]  # events: compute done with buffer set b
        done = [None, None]
        t0, t1 = ev(), ev()
        t0.record(comp)
        up.wait_stream(comp)
        down.wait_stream(comp)
        for s_ in range(steps):
            b = s_ % 2
            with torch.cuda.stream(up):
                if free[b] is not None:
                    up.wait_event(free[b])
                Pd[b].copy_(Ph, non_blocking=True)
                Md[b].copy_(Mh, non_blocking=True)
                Wd[b].copy_(Wh, non_blocking=True)
                loaded = torch.cuda.Event()
                loaded.record(up)
            comp.wait_event(loaded)
            if done[b] is not None:
                comp.wait_event(done[b])  # the previous download from these outputs has finished
            tree.build(Pd[b], Md[b], system_offsets=OFFS, leaf_size=LEAF, with_adjoint=True)
            tree.adjoint_walk(Wd[b], prm, Fd[b])
            tree.adjoint_finalize(GXd[b], GMd[b])
            free[b] = torch.cuda.Event()
            free[b].record(comp)
            with torch.cuda.stream(down):
                down.wait_event(free[b])
                Fh[b].copy_(Fd[b], non_blocking=True)
                GXh[b].copy_(GXd[b], non_blocking=True)
                GMh[b].copy_(GMd[b], non_blocking=True)
                done[b] = torch.cuda.Event()
                done[b].record(down)
        comp.wait_stream(down)
        comp.wait_stream(up)
        t1.record(comp)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / steps

    e2e_run(2)
    e_ms = e2e_run(args.steps)
    if world > 1:
        t = torch.tensor([e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())

    # roofline of the dominant kernel (the adjoint walk)
    walk_s = walk_ms / args.steps * 1e-3
    flops_walk = adjoint_walk_flops(st, n * K)
    fp32_peak = measure_fp32_peak(B, torch, dev)
    traffic = WALK_DRAM_BYTES_PER_PARTICLE * n * K
    # the build: HBM-bound, algorithmic bytes per build of K systems
    build_s = build_ms / args.steps * 1e-3
    build_bytes = K * n * BUILD_ALG_BYTES_PER_PARTICLE + st["nodes"] * BUILD_ALG_BYTES_PER_NODE
    hbm_peak, hbm_source = hbm_peak_gbs()

    extras = {}
    if not args.no_extras:
        want = set(args.extra) if args.extra else set(EXTRAS)
        if world == 1 and "octree8_plain" in want:
            extras["octree8_plain"] = octree8_plain_measurement(B, torch, P0, M0, W0, idx, ref, flush)
        if world == 1 and "opening_sweep" in want:
            extras["opening_sweep"] = opening_sweep_measurement(B, torch, P0, M0, W0, idx, ref, flush)
        if "forest" in want:  # every rank takes part (a collective-free shard of the systems)
            extras["forest"] = forest_measurement(B, torch, dev, rank, world, flush)
        if world > 1 and "sharded_single_system" in want:
            extras["sharded_single_system"] = sharded_measurement(B, torch, dev, rank, world, n)
        if world == 1:
            if "winding_number" in want:
                extras["winding_number"] = winding_measurement(B, torch, dev, flush)
            if "winding_number_mesh" in want:
                extras["winding_number_mesh"] = winding_mesh_measurement(B, torch, dev, flush)
            if "treepm_short_range" in want:
                extras["treepm_short_range"] = treepm_measurement(B, torch, dev, flush)
            if "stochastic_octree8" in want:
                extras["stochastic_octree8"] = stochastic_measurement(B, torch, P0, M0, idx, ref, flush)
            if "direct_sum" in want:
                extras["direct_sum"] = direct_measurement(B, torch, P0, M0, W0, flush)
            if "trajectory" in want:
                extras["trajectory"] = trajectory_measurement(torch, dev, flush)

    if rank == 0:
        cpu = None
        ref_rule = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            t_eval, info = cpu_reference_eval_time(systems[0][0], systems[0][1], args.cpu_sample, threads)
            cpu = {"value": 1.0 / t_eval, "unit": "evals/s", "cores": threads, "kind": "reference",
                   "sample": (f"reference Tree3D<8,1> build of all {n} points + force and query-side VJP of "
                              f"{info['sample_queries']} sampled particles (beta 2), extrapolated to all")}
            # the walk's flops by the convention of 20 flop per interaction (GPU Gems 3 ch. 31), the VJP
            # counted as twice the force, with the interactions the reference's per-target rule takes
            inter = info["interactions_per_query"] * n * K
            flops_ref = REF_FLOPS_PER_INTERACTION * (1 + REF_VJP_FACTOR) * inter
            ref_rule = {"flops_per_interaction": REF_FLOPS_PER_INTERACTION, "vjp_factor": REF_VJP_FACTOR,
                        "interactions_per_step": inter,
                        "interactions_per_query": info["interactions_per_query"],
                        "achieved": flops_ref / walk_s / 1e12, "frac": flops_ref / walk_s / 1e12 / fp32_peak,
                        "counted_by": (f"num_contribs of the reference's CPU evaluateBarnesHut_stackless on "
                                       f"Tree3D<8,1> (leaf 8, beta 2) over {info['sample_queries']} sampled "
                                       "queries of system 0")}
        launches = args.steps * (build_launches(K) + WALK_LAUNCHES + FINALIZE_LAUNCHES)
        plain_eps = 1000.0 / plain_ms
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer spheres, a=1, r<10a)",
            "config": {"workload": workload(n, K), "n": n, "systems_per_gpu": K, "beta": BETA, "theta": 1.0 / BETA,
                       "softening": EPS, "leaf_size": LEAF,
                       "far_field": (f"monopole at every target + quadrupole of every accepted node, taken to first "
                                     f"order about the group centre (once per group) where r_g <= "
                                     f"{B.QUADRUPOLE_LINEAR} |c - cell centre|, exact at every target elsewhere"),
                       "vjp": "positions and masses",
                       "batched": f"{K} systems in one forest: one build, one walk, one finalize per step",
                       "l2": "flushed between steps (256 MB write, outside the timed events)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "accuracy": {"rel_l2_vs_fp64_direct": rel, "outlier_frac": outlier_frac,
                         "max_row_rel": float(row_rel.max()), "subset": 1024, "system": 0},
            "batched_vs_plain": {"batched_evals_per_s": value / world, "plain_evals_per_s": plain_eps,
                                 "ratio": value / world / plain_eps, "plain_ms_per_eval": plain_ms,
                                 "graph_ms_per_step": graph_ms, "eager_ms_per_step": ms_per_step,
                                 "plain": "build, force, rebuild, force+VJP as separate calls on one system"},
            "plain_force": {"ms_per_eval": force_ms, "rel_l2_vs_fp64_direct": plain_force_rel,
                            "what": "build + force of one N=1M system (classic BH, theta 0.5)"},
            "roofline": {"kernel": "adjoint_walk_kernel<quad>", "bound": "fp32", "achieved": flops_walk / walk_s / 1e12,
                         "peak": fp32_peak, "unit": "TFLOP/s", "frac": flops_walk / walk_s / 1e12 / fp32_peak,
                         "peak_source": "measured in this run: the faster of sbh_probe_fp32 and sbh_probe_fp32x2 (FMA chains, scalar and packed)",
                         "traffic": traffic, "walk_ms": walk_s * 1e3,
                         "interactions": {"far": st["far"], "far_quadrupole_exact": st["far_quadrupole_exact"],
                                          "far_quadrupole_linear": st["far_quadrupole_linear"],
                                          "linear_pairs": st["linear_pairs"], "near": st["near"]},
                         "flops_counted_as": "per operation of the walk's own formulas (an FMA as 2): per target "
                                             "200 per far node with the exact quadrupole, 45 with the monopole "
                                             "(linearized nodes included), 55 per near pair; 370 per linearized "
                                             "(group, node) pair and 33 per target for the group expansion",
                         "reference_convention": ref_rule,
                         "build": {"bound": "hbm", "achieved": build_bytes / build_s / 1e9, "peak": hbm_peak,
                                   "unit": "GB/s", "frac": build_bytes / build_s / 1e9 / hbm_peak,
                                   "peak_source": hbm_source, "algorithmic_bytes": build_bytes,
                                   "build_ms": build_s * 1e3,
                                   "traffic": (None if BUILD_DRAM_BYTES_PER_PARTICLE is None
                                               else BUILD_DRAM_BYTES_PER_PARTICLE * n * K),
                                   "bytes_counted_as": "per particle 16 read (position, mass) + 20 written "
                                                       "(sorted position and mass, permutation); per node 80 "
                                                       "written"}},
            "cpu_baseline": cpu,
            "e2e": {"value": world * K * 1000.0 / e_ms, "unit": "evals/s",
                    "h2d_bytes_per_step": int(K * n * 28), "d2h_bytes_per_step": int(K * n * 28),
                    "copies": "each step uploads its inputs and reads its results back from pinned host memory "
                              "on two side streams, overlapping the walks of the neighbouring steps"},
            "gpu_launches": launches,
            "clocks": clocks,
            "tree": {"nodes": st["nodes"], "groups": st["groups"]},
            "extras": extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# Kernels per step of the timed path (counted from the host code):
# build of one system: offsets 1 + bbox 3 + keys 1 + 8 radix passes x
#   (count 1 + scan 3 + scatter 1) + levels 1 + slots 1 + scan 3 + emit 1 +
#   node count 1 + gather 1 + moment scan 3 + finalize 1 + roots 1 +
#   groups 3 (count pass, level cursors, emit pass) = 61; a forest of K > 1
#   systems copies its offsets instead of the offsets kernel and adds a
#   stable pass on the system id (gather 1 + ceil(log2 K / 8) radix passes
#   x 5 + gathers 2 + system ids 1)
# walk: zero adjoint 1 + walk 1 = 2; finalize: push 1 + scan 3 + combine 1 = 5
def build_launches(k: int) -> int:
    if k <= 1:
        return 61
    bits = max(1, (k - 1).bit_length())
    return 61 - 1 + 1 + 5 * ((bits + 7) // 8) + 3


WALK_LAUNCHES = 2

# DRAM bytes (read + write) of one adjoint walk per particle, from one ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of the packed walk
# (four targets per lane, node tiles, linearized quadrupoles) over 4 Plummer
# systems of 262,144 particles: 127.01 MB + 39.26 MB for 1,048,576 particles.
# The walk's DRAM traffic is its L2 misses on the tree, the particles and the
# adjoint arrays, which grow with the particle count.
WALK_DRAM_BYTES_PER_PARTICLE = 158.6
FINALIZE_LAUNCHES = 5

# FP32 flops of the adjoint walk (force + adjoint, counted from
# adjoint_walk_kernel and lq_field / lq_node_adjoint, an FMA as 2): per target
# and far node with the exact quadrupole, per target and far node with the
# monopole (the linearized nodes' monopole included), per near pair; per
# (group, node) pair with the linearized quadrupole (field, Jacobian and node
# adjoint, once per group), and per target the group expansion applied at the
# end (force and query-side gradient).
ADJ_FLOPS_FAR_QUAD = 200
ADJ_FLOPS_FAR_MONO = 45
ADJ_FLOPS_NEAR = 55
ADJ_FLOPS_LINEAR_PAIR = 370
ADJ_FLOPS_LINEAR_APPLY = 33


# The roofline convention of the benchmark definition: 20 flop per
# interaction (Nyland, Harris and Prins, GPU Gems 3 ch. 31), the VJP counted
# as twice the force, interactions as the reference's per-target rule counts
# them.
REF_FLOPS_PER_INTERACTION = 20
REF_VJP_FACTOR = 2

# Algorithmic bytes of one native build: per particle the position and mass
# read (16) and the sorted position and mass plus the permutation written
# (16 + 4); per node one 80-byte record written.
BUILD_ALG_BYTES_PER_PARTICLE = 16 + 20
BUILD_ALG_BYTES_PER_NODE = 80

# DRAM bytes (read + write) of one forest build per particle, summed over the
# build's 69 kernels from one ncu capture of the bench's 8 x 2^20 Plummer
# forest (4,911.9 MB read + 1,900.0 MB written).
BUILD_DRAM_BYTES_PER_PARTICLE = 812.0


def hbm_peak_gbs():
    """The measured copy bandwidth of MEASURED_PEAKS.json, else the pool's
    earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, STREAM-style copy)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (6.65 TB/s, an earlier copy measurement on this pool)"


def adjoint_walk_flops(st, n_targets) -> float:
    fq = st["far_quadrupole_exact"]
    lin = ADJ_FLOPS_LINEAR_PAIR * st["linear_pairs"] + (ADJ_FLOPS_LINEAR_APPLY * n_targets if st["linear_pairs"] else 0)
    return ADJ_FLOPS_FAR_QUAD * fq + ADJ_FLOPS_FAR_MONO * (st["far"] - fq) + ADJ_FLOPS_NEAR * st["near"] + lin


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
