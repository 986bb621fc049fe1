// Native adaptive Morton octree ("ntree"): build, group traversal for the
// softened force with monopole + quadrupole far field, the full adjoint
// (w.r.t. positions and masses), the winding number, and the batched forest
// (many independent systems in one build and one launch). The walks also
// take a periodic box with minimum images, the erfc short-range cutoff and a
// prune radius (the short range of TreePM), and a quadrupole radius beyond
// which accepted nodes keep the monopole alone.
//
// Traversal: one warp per target group of at most kGroup targets (kTPL per
// lane), cut from the tree so its box is compact; every opening decision is
// taken on the group's box, so it is warp-uniform; warps take groups from an
// atomic counter (persistent grid).
//
// Tree definition (the CPU oracle restates it; integer fields are pinned
// bit-exactly):
//  1. per system: lo = per-axis min, span = max axis extent (1 if 0);
//     q_a = floor((x_a - lo_a) * (2^21 / span)) in double, clamped to [0, 2^21);
//  2. key = 63-bit Morton code (x in bit 3i, y in 3i+1, z in 3i+2); the sort
//     is stable by (system, key, input index);
//  3. the level-l cell of a key is its top 3l bits; a cell is a node when
//     l == 0 or its parent cell holds more than leaf_size particles; a node
//     is a leaf when it holds at most leaf_size particles or l == 21;
//  4. nodes are numbered in DFS pre-order; skip[k] is the index after k's
//     subtree, so a traversal is "k = accept ? skip[k] : k + 1".
// Node numbering needs only per-position quantities and one scan: with
// d(i) = common levels of key[i-1], key[i] and L(i) = the leaf level of
// position i (1 + the largest common level of key[a], key[a+S] over the
// windows a in [i-S, i]), position i starts internal nodes at levels
// [d(i)+1, L(i)-1] and a leaf at L(i) when d(i) < L(i).
//
// No fast-math in this translation unit: quantisation and the acceptance
// test use IEEE operations (explicit _rn intrinsics, no contraction) so the
// oracle reproduces them bit for bit; the pair kernels use rsqrtf.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>

#include "sbh_common.cuh"
#include "sbh_native.cuh"
#include "sbh_primitives.cuh"

namespace sbh {
namespace nt {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t float_to_ordered(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Segment (system) of element i given seg_off[0..nseg] (nseg >= 1).
__device__ __forceinline__ int seg_of(const int64_t* seg_off, int nseg, int64_t i) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (seg_off[mid] <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1FFFFFull;
  v = (v | (v << 32)) & 0x1F00000000FFFFull;
  v = (v | (v << 16)) & 0x1F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint32_t compact21(uint64_t v) {
  v &= 0x1249249249249249ull;
  v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ull;
  v = (v ^ (v >> 4)) & 0x100F00F00F00F00Full;
  v = (v ^ (v >> 8)) & 0x1F0000FF0000FFull;
  v = (v ^ (v >> 16)) & 0x1F00000000FFFFull;
  v = (v ^ (v >> 32)) & 0x1FFFFFull;
  return static_cast<uint32_t>(v);
}

// Common tree levels (0..21) of two 63-bit keys.
__device__ __forceinline__ int common_levels(uint64_t a, uint64_t b) {
  uint64_t x = a ^ b;
  if (x == 0) return 21;
  return (__clzll(x) - 1) / 3;
}

// ---------------------------------------------------------------------------
// 1. bounding boxes (per system)
// ---------------------------------------------------------------------------
__global__ void bbox_init_kernel(uint32_t* bb, int nseg) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  for (int d = 0; d < 3; d++) {
    bb[6 * s + d] = 0xFFFFFFFFu;  // min (ordered)
    bb[6 * s + 3 + d] = 0u;       // max (ordered)
  }
}

// Per-system bounding boxes (order-preserving uint encoding, min/max by
// atomics). Each block scans a contiguous chunk; a lane keeps running
// min/max for the system its warp is in and the warp reduces and flushes
// them only when that system changes, so the atomics per system are few
// (contiguous systems: about one flush per warp) instead of six per 32
// points. A warp whose 32 points straddle a system boundary adds them with
// per-lane atomics.
__device__ __forceinline__ void bbox_flush(uint32_t* bb, int s, uint32_t* mn, uint32_t* mx, int lane) {
  for (int d = 0; d < 3; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  }
  if (lane == 0 && mn[0] <= mx[0]) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&bb[6 * s + d], mn[d]);
      atomicMax(&bb[6 * s + 3 + d], mx[d]);
    }
  }
}

__global__ void bbox_kernel(const float* __restrict__ pts, int64_t n, const int64_t* __restrict__ seg_off, int nseg,
                            uint32_t* bb) {
  const int lane = threadIdx.x & 31;
  const int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
  const int64_t chunk = (per_block + blockDim.x - 1) / blockDim.x * blockDim.x;
  const int64_t lo = static_cast<int64_t>(blockIdx.x) * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  int run = -1;  // the warp's current system (warp-uniform)
  uint32_t mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
  for (int64_t base = lo; base < hi; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const bool ok = i < hi;
    int s = 0;
    uint32_t o[3] = {0u, 0u, 0u};
    if (ok) {
      s = nseg > 1 ? seg_of(seg_off, nseg, i) : 0;
      for (int d = 0; d < 3; d++) o[d] = float_to_ordered(pts[3 * i + d]);
    }
    const int first = __ffs(__ballot_sync(0xffffffffu, ok)) - 1;
    if (first < 0) continue;  // no point of this warp in range
    const int s0 = __shfl_sync(0xffffffffu, s, first);
    if (__all_sync(0xffffffffu, !ok || s == s0)) {
      if (s0 != run) {
        if (run >= 0) bbox_flush(bb, run, mn, mx, lane);
        run = s0;
        for (int d = 0; d < 3; d++) {
          mn[d] = 0xFFFFFFFFu;
          mx[d] = 0u;
        }
      }
      if (ok) {
        for (int d = 0; d < 3; d++) {
          mn[d] = min(mn[d], o[d]);
          mx[d] = max(mx[d], o[d]);
        }
      }
    } else if (ok) {
      for (int d = 0; d < 3; d++) {
        atomicMin(&bb[6 * s + d], o[d]);
        atomicMax(&bb[6 * s + 3 + d], o[d]);
      }
    }
  }
  if (run >= 0) bbox_flush(bb, run, mn, mx, lane);
}

// SegBox: lo (float3), span (float), scale (double) per system.
__global__ void bbox_finalize_kernel(const uint32_t* bb, int nseg, const int64_t* seg_off, SegBox* boxes) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  SegBox b;
  bool empty = seg_off[s + 1] <= seg_off[s];
  float lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = empty ? 0.0f : ordered_to_float(bb[6 * s + d]);
    hi[d] = empty ? 0.0f : ordered_to_float(bb[6 * s + 3 + d]);
  }
  float span = 0.0f;
  for (int d = 0; d < 3; d++) span = fmaxf(span, __fsub_rn(hi[d], lo[d]));
  if (!(span > 0.0f)) span = 1.0f;
  for (int d = 0; d < 3; d++) b.lo[d] = lo[d];
  b.span = span;
  b.scale = __ddiv_rn(2097152.0, static_cast<double>(span));
  boxes[s] = b;
}

// ---------------------------------------------------------------------------
// 2. keys
// ---------------------------------------------------------------------------
__global__ void keys_kernel(const float* __restrict__ pts, int64_t n, const int64_t* __restrict__ seg_off, int nseg,
                            const SegBox* __restrict__ boxes, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ segkey) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int s = nseg > 1 ? seg_of(seg_off, nseg, i) : 0;
    SegBox b = boxes[s];
    uint64_t key = 0;
    for (int d = 0; d < 3; d++) {
      double t = __dmul_rn(__dsub_rn(static_cast<double>(pts[3 * i + d]), static_cast<double>(b.lo[d])), b.scale);
      double f = floor(t);
      uint64_t q = f < 0.0 ? 0ull : (f > 2097151.0 ? 2097151ull : static_cast<uint64_t>(f));
      key |= spread21(q) << d;
    }
    keys[i] = key;
    if (segkey) segkey[i] = static_cast<uint32_t>(s);
  }
}

// gather sorted (segment id, key) order of the segment pass
__global__ void gather_keys_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ perm, int64_t n,
                                   uint64_t* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = keys[perm[i]];
}

// ---------------------------------------------------------------------------
// 3. topology
// ---------------------------------------------------------------------------
// cl[a] = common levels of key[a], key[a+S] (same system), else -1
// dd[i] = common levels of key[i-1], key[i] (same system), else -1
__global__ void levels_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ sseg, int64_t n, int S,
                              int8_t* __restrict__ cl, int8_t* __restrict__ dd) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t k = keys[i];
    uint32_t s = sseg ? sseg[i] : 0u;
    int c = -1;
    if (i + S < n && (!sseg || sseg[i + S] == s)) c = common_levels(k, keys[i + S]);
    cl[i] = static_cast<int8_t>(c);
    int d = -1;
    if (i > 0 && (!sseg || sseg[i - 1] == s)) d = common_levels(keys[i - 1], k);
    dd[i] = static_cast<int8_t>(d);
  }
}

// leaf level L(i) and node-slot count of position i
__global__ void slots_kernel(const int8_t* __restrict__ cl, const int8_t* __restrict__ dd, int64_t n, int S,
                             int8_t* __restrict__ lv, uint32_t* __restrict__ cnt) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int mx = -1;
    int64_t a0 = i - S < 0 ? 0 : i - S;
    for (int64_t a = a0; a <= i; a++) mx = max(mx, static_cast<int>(cl[a]));
    int L = mx + 1;
    if (L > 21) L = 21;
    int d = dd[i];
    int lo = d + 1;
    int nint = L - lo;
    if (nint < 0) nint = 0;
    int nleaf = d < L ? 1 : 0;
    lv[i] = static_cast<int8_t>(L);
    cnt[i] = static_cast<uint32_t>(nint + nleaf);
  }
}

// end of the level-l cell that starts at i: first j > i outside it
__device__ __forceinline__ int64_t cell_end(const uint64_t* keys, const uint32_t* sseg, int64_t i, int l,
                                            int64_t seg_end) {
  uint64_t pref = l == 0 ? 0ull : keys[i] >> (63 - 3 * l);
  int64_t lo = i + 1, hi = seg_end;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    uint64_t pm = l == 0 ? 0ull : keys[mid] >> (63 - 3 * l);
    if (pm == pref)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void emit_nodes_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ sseg,
                                  const int64_t* __restrict__ sorted_seg_off, int64_t n, const int8_t* __restrict__ dd,
                                  const int8_t* __restrict__ lv, const uint32_t* __restrict__ base,
                                  NodeRec* __restrict__ nodes, int64_t cap, uint32_t* status) {
  uint32_t total = base[n];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int d = dd[i];
    int L = lv[i];
    int lo = d + 1;
    int top = d < L ? L : L - 1;
    uint32_t slot = base[i];
    int64_t seg_end = sseg ? sorted_seg_off[sseg[i] + 1] : n;
    for (int l = lo; l <= top; l++, slot++) {
      if (slot >= cap) {
        raise_status(status, SBH_DEV_ITER_LIMIT);
        return;
      }
      int64_t e = cell_end(keys, sseg, i, l, seg_end);
      uint32_t skip = e < n ? base[e] : total;
      bool leaf = (l == L);
      nodes[slot].topo = make_int4(static_cast<int>(i), static_cast<int>(e), static_cast<int>(skip),
                                   l | (leaf ? kLeafFlag : 0));
    }
  }
}

// ---------------------------------------------------------------------------
// 4. sorted particles and FP64 moments
// ---------------------------------------------------------------------------
__global__ void gather_particles_kernel(const float* __restrict__ pts, const float* __restrict__ masses,
                                        const float* __restrict__ nrm, const uint32_t* __restrict__ perm, int64_t n,
                                        float4* __restrict__ sp, float4* __restrict__ sn) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t s = perm[i];
    sp[i] = make_float4(pts[3 * s], pts[3 * s + 1], pts[3 * s + 2], masses[s]);
    if (sn && nrm) sn[i] = make_float4(nrm[3 * s], nrm[3 * s + 1], nrm[3 * s + 2], 0.0f);
  }
}

// moment vector of sorted particle i relative to its system's box centre
struct MomentLoad {
  const float4* sp;
  const uint32_t* sseg;
  const SegBox* boxes;
  __device__ DVec<10> operator()(int64_t i) const {
    float4 p = sp[i];
    SegBox b = boxes[sseg ? sseg[i] : 0];
    double half = 0.5 * static_cast<double>(b.span);
    double y0 = static_cast<double>(p.x) - (static_cast<double>(b.lo[0]) + half);
    double y1 = static_cast<double>(p.y) - (static_cast<double>(b.lo[1]) + half);
    double y2 = static_cast<double>(p.z) - (static_cast<double>(b.lo[2]) + half);
    double m = p.w;
    DVec<10> r;
    r.v[0] = m;
    r.v[1] = m * y0;
    r.v[2] = m * y1;
    r.v[3] = m * y2;
    r.v[4] = m * y0 * y0;
    r.v[5] = m * y1 * y1;
    r.v[6] = m * y2 * y2;
    r.v[7] = m * y0 * y1;
    r.v[8] = m * y0 * y2;
    r.v[9] = m * y1 * y2;
    return r;
  }
};

struct NormalMomentLoad {
  const float4* sp;
  const float4* sn;
  __device__ DVec<3> operator()(int64_t i) const {
    float4 p = sp[i], q = sn[i];
    double m = p.w;
    DVec<3> r;
    r.v[0] = m * q.x;
    r.v[1] = m * q.y;
    r.v[2] = m * q.z;
    return r;
  }
};

// Node records from topology + moments + cell geometry (NodeRec, 80 B).
// The topology fields were written by emit_nodes_kernel into nodes[k].topo.
__global__ void finalize_nodes_kernel(NodeRec* __restrict__ nodes, const uint32_t* __restrict__ nn_ptr,
                                      const uint64_t* __restrict__ keys, const uint32_t* __restrict__ sseg,
                                      const SegBox* __restrict__ boxes, const DVec<10>* __restrict__ P,
                                      const DVec<3>* __restrict__ PN, float4* __restrict__ nnrm) {
  uint32_t nn = *nn_ptr;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    int4 t = nodes[k].topo;
    int level = t.w & 0xFF;
    int64_t s0 = t.x, e0 = t.y;
    SegBox b = boxes[sseg ? sseg[s0] : 0];
    DVec<10> hi = P[e0], lo = P[s0];
    double v[10];
    for (int c = 0; c < 10; c++) v[c] = hi.v[c] - lo.v[c];
    double M = v[0];
    double half = 0.5 * static_cast<double>(b.span);
    double c0[3] = {static_cast<double>(b.lo[0]) + half, static_cast<double>(b.lo[1]) + half,
                    static_cast<double>(b.lo[2]) + half};
    // cell geometry from the key prefix (exact in double, rounded once)
    uint64_t pref = level == 0 ? 0ull : keys[s0] >> (63 - 3 * level);
    float side = ldexpf(b.span, -level);
    float ctr[3];
    for (int d = 0; d < 3; d++) {
      uint32_t cd = compact21(pref >> d);
      ctr[d] = static_cast<float>(__dadd_rn(static_cast<double>(b.lo[d]),
                                            __dmul_rn(static_cast<double>(cd) + 0.5, static_cast<double>(side))));
    }
    float X[3];
    double S[6] = {0, 0, 0, 0, 0, 0};
    if (M != 0.0) {
      double Y[3] = {v[1] / M, v[2] / M, v[3] / M};
      for (int d = 0; d < 3; d++) X[d] = static_cast<float>(Y[d] + c0[d]);
      S[0] = v[4] - M * Y[0] * Y[0];
      S[1] = v[5] - M * Y[1] * Y[1];
      S[2] = v[6] - M * Y[2] * Y[2];
      S[3] = v[7] - M * Y[0] * Y[1];
      S[4] = v[8] - M * Y[0] * Y[2];
      S[5] = v[9] - M * Y[1] * Y[2];
    } else {
      for (int d = 0; d < 3; d++) X[d] = ctr[d];
    }
    float diag = __fmul_rn(side, 1.7320508f);
    NodeRec r;
    r.com = make_float4(X[0], X[1], X[2], static_cast<float>(M));
    r.cell = make_float4(ctr[0], ctr[1], ctr[2], diag);
    r.quad = make_float4(static_cast<float>(S[0]), static_cast<float>(S[1]), static_cast<float>(S[2]),
                         static_cast<float>(S[3]));
    r.quad2 = make_float4(static_cast<float>(S[4]), static_cast<float>(S[5]), 0.0f, 0.0f);
    r.topo = t;
    nodes[k] = r;
    if (nnrm && PN) {
      DVec<3> nh = PN[e0], nl = PN[s0];
      nnrm[k] = M != 0.0 ? make_float4(static_cast<float>((nh.v[0] - nl.v[0]) / M),
                                       static_cast<float>((nh.v[1] - nl.v[1]) / M),
                                       static_cast<float>((nh.v[2] - nl.v[2]) / M), 1.0f)
                         : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

// Roots: [first node, end of the nodes) of each system.
__global__ void roots_kernel(const int64_t* __restrict__ sorted_seg_off, int nseg, const uint32_t* __restrict__ base,
                             int64_t cap, int2* __restrict__ roots) {
  int s = blockIdx.x;
  if (s >= nseg) return;
  int64_t a = sorted_seg_off[s], b = sorted_seg_off[s + 1];
  uint32_t total = base[sorted_seg_off[nseg]];
  uint32_t r0 = a < b ? base[a] : 0u;
  uint32_t r1 = b < sorted_seg_off[nseg] ? base[b] : total;
  // never walk past the node array, even if the capacity check tripped
  uint32_t ucap = static_cast<uint32_t>(cap);
  r0 = r0 < ucap ? r0 : ucap;
  r1 = r1 < ucap ? r1 : ucap;
  if (threadIdx.x == 0) roots[s] = make_int2(static_cast<int>(r0), static_cast<int>(a < b ? r1 : r0));
}

// Target groups cut from the tree, at most G (<= kGroup) targets each. For
// every node holding more than G particles its children are taken in order;
// each maximal run of consecutive children that hold at most G particles
// each is one range of sorted particles, cut into chunks of G (the last one
// shorter). Children with more particles are handled the same way one level
// down; a leaf with more than G particles (coincident points at level 21)
// and a system root holding at most G are cut into chunks directly. Every
// group lies inside the cell of a node with more than G particles, so its
// bounding box is compact (runs of consecutive Morton positions can straddle
// distant cells), and the chunks fill the lanes better than one group per
// child run. Slots come from an atomic counter: the group order varies
// between runs, each group's result does not. Every group holds at least one
// particle, so n + systems + 1 slots always suffice.
__device__ __forceinline__ void emit_chunks(int4* groups, uint32_t* count, int64_t cap, int s0, int s1, int sys,
                                            int G, uint32_t* status) {
  int ng = (s1 - s0 + G - 1) / G;
  if (ng <= 0) return;
  uint32_t slot = atomicAdd(count, static_cast<uint32_t>(ng));
  for (int g = 0; g < ng; g++) {
    int s = s0 + g * G;
    if (slot + g < cap)
      groups[slot + g] = make_int4(s, min(s + G, s1), sys, 0);
    else
      raise_status(status, SBH_DEV_ITER_LIMIT);
  }
}

__global__ void group_nodes_kernel(const NodeRec* __restrict__ nodes, const uint32_t* __restrict__ nn_ptr,
                                   const uint32_t* __restrict__ sseg, int4* __restrict__ groups, int64_t cap, int G,
                                   uint32_t* __restrict__ count, uint32_t* status) {
  uint32_t nn = *nn_ptr;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    int4 t = nodes[k].topo;
    int cnt = t.y - t.x;
    bool leaf = (t.w & kLeafFlag) != 0;
    bool root = (t.w & 0xFF) == 0;
    int sys = sseg ? static_cast<int>(sseg[t.x]) : 0;
    if (leaf || cnt <= G) {
      if (root || (leaf && cnt > G)) emit_chunks(groups, count, cap, t.x, t.y, sys, G, status);
      continue;
    }
    int run_s = -1, run_e = -1;
    for (uint32_t c = k + 1; c < static_cast<uint32_t>(t.z) && c < nn;) {
      int4 tc = nodes[c].topo;
      if (tc.y - tc.x > G) {
        if (run_s >= 0) emit_chunks(groups, count, cap, run_s, run_e, sys, G, status);
        run_s = -1;
      } else {
        if (run_s < 0) run_s = tc.x;
        run_e = tc.y;
      }
      if (static_cast<uint32_t>(tc.z) <= c) break;  // malformed skip: never loop
      c = static_cast<uint32_t>(tc.z);
    }
    if (run_s >= 0) emit_chunks(groups, count, cap, run_s, run_e, sys, G, status);
  }
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ idx, int64_t n,
                                  uint32_t* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = src[idx[i]];
}

__global__ void sseg_kernel(const int64_t* __restrict__ seg_off, int nseg, int64_t n, uint32_t* __restrict__ sseg) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    sseg[i] = static_cast<uint32_t>(seg_of(seg_off, nseg, i));
}

// meta[0] = number of nodes (base[n]); flags an overflow of the capacity.
__global__ void node_count_kernel(const uint32_t* base, int64_t n, int64_t cap, uint32_t* meta) {
  uint32_t total = base[n];
  meta[0] = total <= cap ? total : static_cast<uint32_t>(cap);
  meta[3] = total > cap ? 1u : 0u;
}


__global__ void single_offsets_kernel(int64_t* seg_off, int64_t n) {
  seg_off[0] = 0;
  seg_off[1] = n;
}

// ---------------------------------------------------------------------------
// 5. traversal
// ---------------------------------------------------------------------------
struct WalkTree {
  const NodeRec* nodes;
  const float4* sp;     // sorted sources (x, y, z, m)
  const float4* sn;     // sorted source normals (winding number)
  const float4* nnrm;   // node mean normals (winding number)
  const int2* roots;    // per system: [root, end of the system's nodes)
};

struct WalkTargets {
  const float4* tp;          // sorted target positions
  const uint32_t* perm;      // sorted slot -> input index
  const int4* groups;        // (start, end, system, 0), <= 32 targets each
  const uint32_t* ngroups;   // device-side group count
  int self;                  // targets are the sources (skip i == j pairs)
  uint32_t* counter;         // work counter, zero at launch
  uint32_t capacity;         // entries of groups (bounds the device-side count)
  int64_t tbeg, tend;        // groups whose first sorted target lies outside [tbeg, tend) are skipped
};

// Persistent walks: the grid holds as many warps as the SMs keep resident,
// and each warp takes its next group from an atomic counter until none is
// left, so a warp that drew cheap groups keeps working while another is
// still on an expensive one (group costs in one tree differ by 10x and
// more between the core and the halo of a clustered distribution).
__device__ __forceinline__ uint32_t next_group(const WalkTargets& G) {
  uint32_t s = 0;
  if ((threadIdx.x & 31) == 0) s = atomicAdd(G.counter, 1u);
  return __shfl_sync(0xffffffffu, s, 0);
}

// Resident blocks of 128 threads per SM the walks are compiled for (this
// caps their registers at 65536 / (128 x blocks)). Measured on a B200 with
// 8 x 2^20 Plummer particles, quadrupole radius 1.6, three targets per
// lane: the adjoint walk takes 412 ms at 5 blocks (96 registers) and 389 ms
// at 6 (80 registers, 56 bytes of spills), where 7 blocks leave 72
// registers and 128 bytes of spills; the force walk 182.5 ms at 5 and 177 ms
// at 6.
#ifndef SBH_ADJOINT_WALK_MIN_BLOCKS
#define SBH_ADJOINT_WALK_MIN_BLOCKS 6
#endif
#ifndef SBH_FORCE_WALK_MIN_BLOCKS
#define SBH_FORCE_WALK_MIN_BLOCKS 6
#endif
constexpr int kAdjointWalkMinBlocks = SBH_ADJOINT_WALK_MIN_BLOCKS;
constexpr int kForceWalkMinBlocks = SBH_FORCE_WALK_MIN_BLOCKS;

struct WalkParams {
  float beta;
  float eps2;      // softening^2 + 1e-12
  float cutoff;    // <= 0: no attenuation
  float box;       // periodic box length (periodic walks)
  float inv_box;   // 1 / box
  float prune_r2;  // > 0: skip nodes whose cell is farther than sqrt(prune_r2) from the group box
  float quad_g;    // > 0: an accepted node takes the quadrupole only when its opening distance^2 is
                   // below quad_g * (beta * diagonal)^2; 0: every accepted node takes it
  float inv_2cut;  // 1 / (2 cutoff) (cutoff walks)
  float cc_coef;   // 1 / (2 sqrt(pi) cutoff^3) (cutoff walks)
};

// Minimum-image displacement of a periodic box (minImageDisplacement,
// include/kernel.h:27-39).
__device__ __forceinline__ float min_image(float d, const WalkParams& P) {
  return d - P.box * floorf(d * P.inv_box + 0.5f);
}

// The periodic image of a cell's centre nearest the group box's centre, per
// axis (IEEE operations, the oracle's order).
__device__ __forceinline__ float4 cell_image(const float4& cell, const float* gmin, const float* gmax,
                                             const WalkParams& P) {
  float c[3] = {cell.x, cell.y, cell.z};
  for (int d = 0; d < 3; d++) {
    float bc = __fmul_rn(__fadd_rn(gmin[d], gmax[d]), 0.5f);
    float k = rintf(__fmul_rn(__fsub_rn(bc, c[d]), P.inv_box));
    c[d] = __fadd_rn(c[d], __fmul_rn(P.box, k));
  }
  return make_float4(c[0], c[1], c[2], cell.w);
}

// AABB prune of the short-range split (the group form of
// octree8_should_prune, src/sbh_ffi.cu:1903-1948): the node is skipped when
// the distance from the group box to its cell exceeds the prune radius. The
// half side is taken a little above diag / (2 sqrt 3), so the test errs on
// the side of keeping a node.
__device__ __forceinline__ bool prune_node(const float4& cell, const float* gmin, const float* gmax, float r2) {
  float half = __fmul_rn(cell.w, 0.2887f);
  float x[3] = {cell.x, cell.y, cell.z};
  float t[3];
  for (int d = 0; d < 3; d++) {
    float a = __fsub_rn(gmin[d], __fadd_rn(x[d], half));
    float b = __fsub_rn(__fsub_rn(x[d], half), gmax[d]);
    float m = a > b ? a : b;
    t[d] = m > 0.0f ? m : 0.0f;
  }
  float d2 = __fadd_rn(__fadd_rn(__fmul_rn(t[0], t[0]), __fmul_rn(t[1], t[1])), __fmul_rn(t[2], t[2]));
  return d2 > r2;
}

// Targets of one group as a lane holds them: slots lane + 32 t, t < kTPL.
// Inactive slots carry the group's first target (inside the group box) and
// a zero cotangent or mass, so they add nothing to the sums over the warp.
struct LaneTargets {
  float x[kTPL], y[kTPL], z[kTPL];
  int idx[kTPL];
  bool act[kTPL];
};

__device__ __forceinline__ void load_targets(const WalkTargets& G, const int4& gr, int lane, LaneTargets& Q) {
#pragma unroll
  for (int t = 0; t < kTPL; t++) {
    int i = gr.x + lane + 32 * t;
    Q.act[t] = i < gr.y;
    Q.idx[t] = i;
    float4 q = G.tp[Q.act[t] ? i : gr.x];
    Q.x[t] = q.x;
    Q.y[t] = q.y;
    Q.z[t] = q.z;
  }
}

// Group bounding box: min/max over every slot of the warp.
__device__ __forceinline__ void group_box(const LaneTargets& Q, float* gmin, float* gmax) {
  float lo[3] = {Q.x[0], Q.y[0], Q.z[0]}, hi[3] = {Q.x[0], Q.y[0], Q.z[0]};
#pragma unroll
  for (int t = 1; t < kTPL; t++) {
    lo[0] = fminf(lo[0], Q.x[t]);
    lo[1] = fminf(lo[1], Q.y[t]);
    lo[2] = fminf(lo[2], Q.z[t]);
    hi[0] = fmaxf(hi[0], Q.x[t]);
    hi[1] = fmaxf(hi[1], Q.y[t]);
    hi[2] = fmaxf(hi[2], Q.z[t]);
  }
#pragma unroll
  for (int d = 0; d < 3; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    gmin[d] = lo[d];
    gmax[d] = hi[d];
  }
}

// Acceptance test: the reference's rule |q - cell centre| / diag >= beta
// (include/tree3d.h:134-153, src/sbh_ffi.cu:1878-1893) made to hold for every
// target of the group: dist(group box, cell centre) > beta * diag. IEEE
// operations in the oracle's order (no contraction).
__device__ __forceinline__ bool accept_node(const float4& cell, const float* gmin, const float* gmax, float beta,
                                            float& d2, float& rc2) {
  float rc = __fmul_rn(cell.w, beta);
  float x[3] = {cell.x, cell.y, cell.z};
  float t[3];
  for (int d = 0; d < 3; d++) {
    float a = __fsub_rn(gmin[d], x[d]);
    float b = __fsub_rn(x[d], gmax[d]);
    float m = a > b ? a : b;
    t[d] = m > 0.0f ? m : 0.0f;
  }
  d2 = __fadd_rn(__fadd_rn(__fmul_rn(t[0], t[0]), __fmul_rn(t[1], t[1])), __fmul_rn(t[2], t[2]));
  rc2 = __fmul_rn(rc, rc);
  return d2 > rc2;
}

// Far-field order of an accepted node (warp-uniform: the inputs are the
// group box and the node). The quadrupole's share of the error falls off
// one power of the distance faster than the monopole's, so beyond
// sqrt(quad_g) opening radii the monopole alone is kept.
__device__ __forceinline__ bool quad_order(float d2, float rc2, const WalkParams& P) {
  return !(P.quad_g > 0.0f) || d2 < __fmul_rn(P.quad_g, rc2);
}

__device__ __forceinline__ bool accept_node(const float4& cell, const float* gmin, const float* gmax, float beta) {
  float rc = __fmul_rn(cell.w, beta);
  float x[3] = {cell.x, cell.y, cell.z};
  float t[3];
  for (int d = 0; d < 3; d++) {
    float a = __fsub_rn(gmin[d], x[d]);
    float b = __fsub_rn(x[d], gmax[d]);
    float m = a > b ? a : b;
    t[d] = m > 0.0f ? m : 0.0f;
  }
  float d2 = __fadd_rn(__fadd_rn(__fmul_rn(t[0], t[0]), __fmul_rn(t[1], t[1])), __fmul_rn(t[2], t[2]));
  return d2 > __fmul_rn(rc, rc);
}

// erfc attenuation of the short-range force and its radial derivative term
// (src/sbh_ffi.cu:142-160, 2062-2090), with u = r / (2 cutoff):
//   att = erfc(u) + (2 / sqrt(pi)) u e^{-u^2},
//   cc  = ir3 r e^{-u^2} / (2 sqrt(pi) cutoff^3);
// att = 1, cc = 0 without cutoff. erfc(u) is the rational approximation of
// Abramowitz & Stegun 7.1.26 (after Hastings): (a1 t + a2 t^2 + a3 t^3 +
// a4 t^4 + a5 t^5) e^{-u^2} with t = 1 / (1 + p u), absolute error at most
// 1.5e-7 for u >= 0. It shares e^{-u^2} with the second term, so one
// exponential serves a pair; the divisions by the cutoff are precomputed.
__device__ __forceinline__ void attenuation(float r2, float ir3, const WalkParams& P, float& att, float& cc) {
  const float r2p = r2 + 1e-12f;
  const float dist = r2p * rsqrtf(r2p);
  const float u = dist * P.inv_2cut;
  const float e = expf(-(u * u));
  const float t = __fdividef(1.0f, fmaf(0.3275911f, u, 1.0f));
  const float poly =
      t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, 1.061405429f, -1.453152027f), 1.421413741f), -0.284496736f), 0.254829592f);
  att = e * fmaf(1.1283791671f, u, poly);  // 2 / sqrt(pi) = 1.1283791671
  cc = ir3 * dist * e * P.cc_coef;
}

// One accepted node's monopole (with the erfc attenuation when CUT, minimum
// image when PER) added to the lane's far-field accumulators.
template <bool CUT, bool PER>
__device__ __forceinline__ void far_mono_force(const float4& A, const LaneTargets& Q, int nslot, const WalkParams& P,
                                               float* fx, float* fy, float* fz) {
#pragma unroll
  for (int t = 0; t < kTPL; t++) {
    if (t >= nslot) break;
    float rx = Q.x[t] - A.x, ry = Q.y[t] - A.y, rz = Q.z[t] - A.z;
    if (PER) {
      rx = min_image(rx, P);
      ry = min_image(ry, P);
      rz = min_image(rz, P);
    }
    float r2 = rx * rx + ry * ry + rz * rz;
    float ir = rsqrtf(r2 + P.eps2);
    float ir3 = ir * ir * ir;
    float c = -A.w * ir3;
    if (CUT) {
      float att, cc;
      attenuation(r2, ir3, P, att, cc);
      c *= att;
    }
    fx[t] += c * rx;
    fy[t] += c * ry;
    fz[t] += c * rz;
  }
}

// One accepted node's monopole + quadrupole (Plummer softening):
// a_q = ir5 (3 S r + 1.5 tr(S) r) - 7.5 (r.S.r) ir7 r.
__device__ __forceinline__ void far_quad_force(const NodeRec* nd, const float4& A, const LaneTargets& Q, int nslot,
                                               const WalkParams& P, float* fx, float* fy, float* fz) {
  const float4 Qd = __ldg(&nd->quad);
  const float4 X = __ldg(&nd->quad2);
  const float tr15 = 1.5f * (Qd.x + Qd.y + Qd.z);
#pragma unroll
  for (int t = 0; t < kTPL; t++) {
    if (t >= nslot) break;
    float rx = Q.x[t] - A.x, ry = Q.y[t] - A.y, rz = Q.z[t] - A.z;
    float r2 = rx * rx + ry * ry + rz * rz;
    float ir = rsqrtf(r2 + P.eps2);
    float ih = ir * ir;
    float ir3 = ir * ih;
    float c = -A.w * ir3;
    float sx = Qd.x * rx + Qd.w * ry + X.x * rz;
    float sy = Qd.w * rx + Qd.y * ry + X.y * rz;
    float sz = X.x * rx + X.y * ry + Qd.z * rz;
    float rsr = rx * sx + ry * sy + rz * sz;
    float ir5 = ir3 * ih;
    float cr = c + ir5 * (tr15 - 7.5f * rsr * ih);
    float c3 = 3.0f * ir5;
    fx[t] += cr * rx + c3 * sx;
    fy[t] += cr * ry + c3 * sy;
    fz[t] += cr * rz + c3 * sz;
  }
}

// Flop accounting used by the roofline (FP32 operations counted from the
// formulas below, an FMA as 2, per target): force walk near pair 20, far
// node 55 (monopole + quadrupole); adjoint walk (force + adjoint) near pair
// 55, far node 200 including the share of the warp reductions.

template <bool QUAD, bool CUT, bool PER>
__global__ void __launch_bounds__(128, kForceWalkMinBlocks)
    force_walk_kernel(WalkTree T, WalkTargets G, WalkParams P, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint32_t ng = min(*G.ngroups, G.capacity);
  for (;;) {
    uint32_t gw = next_group(G);
    if (gw >= ng) break;
    int4 gr = G.groups[gw];
    if (gr.x < G.tbeg || gr.x >= G.tend) continue;  // another rank's targets (warp-uniform)
    LaneTargets Q;
    load_targets(G, gr, lane, Q);
    const int nslot = (gr.y - gr.x + 31) / 32;  // warp-uniform: the target slots in use
    float gmin[3], gmax[3];
    group_box(Q, gmin, gmax);
    int2 rt = T.roots[gr.z];
    float fx[kTPL], fy[kTPL], fz[kTPL];                                     // far field
    float nx[kTPL], ny[kTPL], nz[kTPL], cx[kTPL], cy[kTPL], cz[kTPL];       // near field, compensated
#pragma unroll
    for (int t = 0; t < kTPL; t++) fx[t] = fy[t] = fz[t] = nx[t] = ny[t] = nz[t] = cx[t] = cy[t] = cz[t] = 0.f;
    // Pre-order walk. The next node is known once this node's opening test
    // is done, so its opening data is loaded before this node's terms are
    // evaluated and the load latency hides behind that arithmetic.
    int k = rt.x;
    int4 tp = make_int4(0, 0, rt.y, 0);
    float4 A = make_float4(0.f, 0.f, 0.f, 0.f), C = A;
    if (k < rt.y) {
      tp = __ldg(&T.nodes[k].topo);
      A = __ldg(&T.nodes[k].com);
      C = __ldg(&T.nodes[k].cell);
    }
    while (k < rt.y) {
      const NodeRec* nd = T.nodes + k;
      const float4 Ci = PER ? cell_image(C, gmin, gmax, P) : C;
      const bool live = A.w != 0.0f &&  // mass-zero and pruned nodes are skipped
                        !(CUT && P.prune_r2 > 0.0f && prune_node(Ci, gmin, gmax, P.prune_r2));
      float d2 = 0.0f, rc2 = 0.0f;
      const bool acc = live && accept_node(Ci, gmin, gmax, P.beta, d2, rc2);
      const bool qh = QUAD && quad_order(d2, rc2, P);
      const bool leaf = (tp.w & kLeafFlag) != 0;
      const int next = (!live || acc || leaf) ? tp.z : k + 1;
      int4 tpn = tp;
      float4 An = A, Cn = C;
      if (next < rt.y) {
        tpn = __ldg(&T.nodes[next].topo);
        An = __ldg(&T.nodes[next].com);
        Cn = __ldg(&T.nodes[next].cell);
      }
      if (acc) {
        if (qh) {
          far_quad_force(nd, A, Q, nslot, P, fx, fy, fz);
        } else {
          far_mono_force<CUT, PER>(A, Q, nslot, P, fx, fy, fz);
        }
      } else if (live && leaf) {
        float ax[kTPL], ay[kTPL], az[kTPL];
#pragma unroll
        for (int t = 0; t < kTPL; t++) ax[t] = ay[t] = az[t] = 0.f;
        for (int j = tp.x; j < tp.y; j++) {
          float4 s = __ldg(&T.sp[j]);
#pragma unroll
          for (int t = 0; t < kTPL; t++) {
            if (t >= nslot) break;
            float rx = Q.x[t] - s.x, ry = Q.y[t] - s.y, rz = Q.z[t] - s.z;
            if (PER) {
              rx = min_image(rx, P);
              ry = min_image(ry, P);
              rz = min_image(rz, P);
            }
            float r2 = rx * rx + ry * ry + rz * rz;
            float ir = rsqrtf(r2 + P.eps2);
            float ir3 = ir * ir * ir;
            float c = -s.w * ir3;
            if (CUT) {
              float att, cc;
              attenuation(r2, ir3, P, att, cc);
              c *= att;
            }
            ax[t] += c * rx;
            ay[t] += c * ry;
            az[t] += c * rz;
          }
        }
#pragma unroll
        for (int t = 0; t < kTPL; t++) {
          kahan_add(nx[t], cx[t], ax[t]);
          kahan_add(ny[t], cy[t], ay[t]);
          kahan_add(nz[t], cz[t], az[t]);
        }
      }
      k = next;
      tp = tpn;
      A = An;
      C = Cn;
    }
#pragma unroll
    for (int t = 0; t < kTPL; t++) {
      if (Q.act[t]) {
        uint32_t o = G.perm[Q.idx[t]];
        out[3 * o] = fx[t] + nx[t];
        out[3 * o + 1] = fy[t] + ny[t];
        out[3 * o + 2] = fz[t] + nz[t];
      }
    }
  }
}

// Sum 4 values over the warp with 6 shuffles: afterwards lane 8*v holds the
// warp total of value v (v = 0..3).
__device__ __forceinline__ float reduce4(float v0, float v1, float v2, float v3) {
  int lane = threadIdx.x & 31;
  bool b4 = lane & 16;
  float s0 = b4 ? v0 : v2, s1 = b4 ? v1 : v3;
  float k0 = b4 ? v2 : v0, k1 = b4 ? v3 : v1;
  k0 += __shfl_xor_sync(0xffffffffu, s0, 16);
  k1 += __shfl_xor_sync(0xffffffffu, s1, 16);
  bool b3 = lane & 8;
  float s = b3 ? k0 : k1;
  float v = b3 ? k1 : k0;
  v += __shfl_xor_sync(0xffffffffu, s, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  return v;  // lane with bits (b4, b3): value 2*b4 + b3
}

__device__ __forceinline__ int reduce4_index(int lane) { return ((lane >> 4) & 1) * 2 + ((lane >> 3) & 1); }

// Sum 10 values over the warp with 12 shuffles (a transposed butterfly: at
// each step a lane keeps one half of its values and receives its partner's
// share of that half). Afterwards lane l holds the warp total of value
// reduce10_index(l); lanes where that is -1 hold padding.
__device__ __forceinline__ float reduce10(const float* v) {
  int lane = threadIdx.x & 31;
  bool b = lane & 16;
  float h[6];
#pragma unroll
  for (int j = 0; j < 5; j++) {
    float send = b ? v[j] : v[j + 5];
    float keep = b ? v[j + 5] : v[j];
    h[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  h[5] = 0.f;
  b = lane & 8;
  float g[4];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    float send = b ? h[j] : h[j + 3];
    float keep = b ? h[j + 3] : h[j];
    g[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  g[3] = 0.f;
  b = lane & 4;
  float e[2];
#pragma unroll
  for (int j = 0; j < 2; j++) {
    float send = b ? g[j] : g[j + 2];
    float keep = b ? g[j + 2] : g[j];
    e[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  b = lane & 2;
  float send = b ? e[0] : e[1];
  float d = (b ? e[1] : e[0]) + __shfl_xor_sync(0xffffffffu, send, 2);
  d += __shfl_xor_sync(0xffffffffu, d, 1);
  return d;
}

// Value index held by lane l after reduce10: value (c + 3 b3) + 5 b4 with
// c = b1 + 2 b2, for even lanes with c < 3 and c + 3 b3 < 5; otherwise -1.
__device__ __forceinline__ int reduce10_index(int lane) {
  if (lane & 1) return -1;
  int c = ((lane >> 1) & 1) + 2 * ((lane >> 2) & 1);
  if (c >= 3) return -1;
  int hj = c + 3 * ((lane >> 3) & 1);
  if (hj >= 5) return -1;
  return hj + 5 * ((lane >> 4) & 1);
}

// One accepted node, monopole far field, for the lane's targets: query-side
// gradient and force into the lane's accumulators, the node-side adjoint
// (A_X, A_M) reduced over the warp and added to the node's slots.
template <bool CUT, bool PER>
__device__ __forceinline__ void far_mono_adjoint(const float4& A, const LaneTargets& Q, const float* wx,
                                                 const float* wy, const float* wz, int nslot, const WalkParams& P,
                                                 bool want_force, float* gx, float* gy, float* gz, float* fx,
                                                 float* fy, float* fz, float* __restrict__ na, int lane, int r4) {
  const float M = A.w;
  float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
#pragma unroll
  for (int t = 0; t < kTPL; t++) {
    if (t >= nslot) break;
    float rx = Q.x[t] - A.x, ry = Q.y[t] - A.y, rz = Q.z[t] - A.z;
    if (PER) {
      rx = min_image(rx, P);
      ry = min_image(ry, P);
      rz = min_image(rz, P);
    }
    float r2 = rx * rx + ry * ry + rz * rz;
    float ir = rsqrtf(r2 + P.eps2);
    float ih = ir * ir;
    float ir3 = ir * ih;
    float ir5 = ir3 * ih;
    float rw = rx * wx[t] + ry * wy[t] + rz * wz[t];
    float att = 1.0f, cc = 0.0f;
    if (CUT) attenuation(r2, ir3, P, att, cc);
    float lin = att * ir3;
    float mlin = M * lin, mrad = M * (rw * (3.0f * att * ir5 + cc));
    v3 -= lin * rw;  // A_M
    float qx_ = mrad * rx - mlin * wx[t];
    float qy_ = mrad * ry - mlin * wy[t];
    float qz_ = mrad * rz - mlin * wz[t];
    if (want_force) {
      fx[t] -= mlin * rx;
      fy[t] -= mlin * ry;
      fz[t] -= mlin * rz;
    }
    gx[t] += qx_;
    gy[t] += qy_;
    gz[t] += qz_;
    v0 -= qx_;
    v1 -= qy_;
    v2 -= qz_;
  }
  float tot = reduce4(v0, v1, v2, v3);
  if ((lane & 7) == 0) atomicAdd(&na[r4], tot);
}

// One accepted node with the quadrupole (Plummer softening, no cutoff, not
// periodic): as far_mono_adjoint plus the quadrupole's terms and the node's
// G = sym d(w . a_q)/dS, ten values reduced over the warp.
__device__ __forceinline__ void far_quad_adjoint(const NodeRec* nd, const float4& A, const LaneTargets& Q,
                                                 const float* wx, const float* wy, const float* wz, int nslot,
                                                 const WalkParams& P, bool want_force, float* gx, float* gy,
                                                 float* gz, float* fx, float* fy, float* fz, float* __restrict__ na,
                                                 int r10) {
  const float4 Qd = __ldg(&nd->quad);
  const float4 X = __ldg(&nd->quad2);
  const float M = A.w;
  const float Sxx = Qd.x, Syy = Qd.y, Szz = Qd.z, Sxy = Qd.w, Sxz = X.x, Syz = X.y;
  const float tr15 = 1.5f * (Sxx + Syy + Szz);
  float v[10], vb = 0.f;  // vb: the (r.w) I part of G, added to its diagonal once
#pragma unroll
  for (int j = 0; j < 10; j++) v[j] = 0.f;
#pragma unroll
  for (int t = 0; t < kTPL; t++) {
    if (t >= nslot) break;
    float rx = Q.x[t] - A.x, ry = Q.y[t] - A.y, rz = Q.z[t] - A.z;
    float r2 = rx * rx + ry * ry + rz * rz;
    float ir = rsqrtf(r2 + P.eps2);
    float ih = ir * ir;
    float ir3 = ir * ih;
    float ir5 = ir3 * ih;
    float rw = rx * wx[t] + ry * wy[t] + rz * wz[t];
    float mlin = M * ir3, mrad = M * (rw * (3.0f * ir5));
    v[3] -= ir3 * rw;  // A_M
    float sx = Sxx * rx + Sxy * ry + Sxz * rz;
    float sy = Sxy * rx + Syy * ry + Syz * rz;
    float sz = Sxz * rx + Syz * ry + Szz * rz;
    float swx = Sxx * wx[t] + Sxy * wy[t] + Sxz * wz[t];
    float swy = Sxy * wx[t] + Syy * wy[t] + Syz * wz[t];
    float swz = Sxz * wx[t] + Syz * wy[t] + Szz * wz[t];
    float rsr = rx * sx + ry * sy + rz * sz;
    float rsw = rx * swx + ry * swy + rz * swz;
    float ir7 = ir5 * ih, ir9 = ir7 * ih;
    float c1 = 3.0f * ir5;
    float a1 = 5.0f * ir7 * rw;
    float a3 = 15.0f * ir7 * rsw - 52.5f * ir9 * rsr * rw;
    float cw = tr15 * ir5 - 7.5f * ir7 * rsr - mlin;
    float cr = mrad - tr15 * a1 - a3;
    float c2 = 3.0f * a1;
    float qx_ = c1 * swx - c2 * sx + cw * wx[t] + cr * rx;
    float qy_ = c1 * swy - c2 * sy + cw * wy[t] + cr * ry;
    float qz_ = c1 * swz - c2 * sz + cw * wz[t] + cr * rz;
    // G, off-diagonals doubled (halved once below)
    float al = 1.5f * ir5, ga = 7.5f * ir7 * rw;
    vb += al * rw;
    float ux = 2.0f * al * wx[t] - ga * rx;
    float uy = 2.0f * al * wy[t] - ga * ry;
    float uz = 2.0f * al * wz[t] - ga * rz;
    v[4] += ux * rx;
    v[5] += uy * ry;
    v[6] += uz * rz;
    v[7] += ux * ry + uy * rx;
    v[8] += ux * rz + uz * rx;
    v[9] += uy * rz + uz * ry;
    if (want_force) {
      float cf = ir5 * (tr15 - 7.5f * rsr * ih) - mlin;
      fx[t] += cf * rx + c1 * sx;
      fy[t] += cf * ry + c1 * sy;
      fz[t] += cf * rz + c1 * sz;
    }
    gx[t] += qx_;
    gy[t] += qy_;
    gz[t] += qz_;
    v[0] -= qx_;
    v[1] -= qy_;
    v[2] -= qz_;
  }
  v[4] += vb;
  v[5] += vb;
  v[6] += vb;
  v[7] *= 0.5f;
  v[8] *= 0.5f;
  v[9] *= 0.5f;
  float tot = reduce10(v);
  if (r10 >= 0) atomicAdd(&na[r10], tot);
}

// Fused force + adjoint walk. Per target slot: the query-side gradient
// (written to gq in sorted order); per accepted node: A_X, A_M, G summed over
// the group and added to node_adj; per near source particle: (dx, dm) summed
// over the group and added to part_adj. Forces are written when out != null.
// Every node-side term is linear in the cotangent, so inactive slots (zero
// cotangent) add nothing.
//
// Per (target, node) pair with r = q - X, h = |r|^2 + eps^2, ir = h^-1/2,
// lin = att ir^3, rad = (3 att ir^5 + cc)(r.w), and S the node's second
// moment, the query-side gradient is
//   M (rad r - lin w) + 3 ir^5 S w - 15 ir^7 (r.w) S r
//     + (1.5 tr(S) ir^5 - 7.5 ir^7 rSr) w - (7.5 tr(S) ir^7 (r.w) + a3) r,
// a3 = 15 ir^7 (r.Sw) - 52.5 ir^9 (rSr)(r.w), and the node-side terms are
// A_X = -(that gradient), A_M = -lin (r.w) and
// G = 1.5 ir^5 (w r^T + r w^T) + 1.5 ir^5 (r.w) I - 7.5 ir^7 (r.w) r r^T.
template <bool QUAD, bool CUT, bool PER>
__global__ void __launch_bounds__(128, kAdjointWalkMinBlocks)
    adjoint_walk_kernel(WalkTree T, WalkTargets G, WalkParams P, const float* __restrict__ cot,
                        float* __restrict__ out, float* __restrict__ gq, float* __restrict__ node_adj,
                        float* __restrict__ part_adj) {
  const int lane = threadIdx.x & 31;
  const uint32_t ng = min(*G.ngroups, G.capacity);
  const int r4 = reduce4_index(lane), r10 = reduce10_index(lane);
  for (;;) {
    uint32_t gw = next_group(G);
    if (gw >= ng) break;
    int4 gr = G.groups[gw];
    if (gr.x < G.tbeg || gr.x >= G.tend) continue;  // another rank's targets (warp-uniform)
    LaneTargets Q;
    load_targets(G, gr, lane, Q);
    const int nslot = (gr.y - gr.x + 31) / 32;  // warp-uniform: the target slots in use
    float wx[kTPL], wy[kTPL], wz[kTPL];
#pragma unroll
    for (int t = 0; t < kTPL; t++) {
      const uint32_t o = Q.act[t] ? G.perm[Q.idx[t]] : 0u;
      wx[t] = Q.act[t] ? cot[3 * o] : 0.f;
      wy[t] = Q.act[t] ? cot[3 * o + 1] : 0.f;
      wz[t] = Q.act[t] ? cot[3 * o + 2] : 0.f;
    }
    float gmin[3], gmax[3];
    group_box(Q, gmin, gmax);
    int2 rt = T.roots[gr.z];
    float gx[kTPL], gy[kTPL], gz[kTPL];  // query-side gradient
    float fx[kTPL], fy[kTPL], fz[kTPL];  // force
#pragma unroll
    for (int t = 0; t < kTPL; t++) gx[t] = gy[t] = gz[t] = fx[t] = fy[t] = fz[t] = 0.f;
    int k = rt.x;
    while (k < rt.y) {
      const NodeRec* nd = T.nodes + k;
      int4 tp = __ldg(&nd->topo);
      float4 A = __ldg(&nd->com);
      float4 C = __ldg(&nd->cell);
      if (PER) C = cell_image(C, gmin, gmax, P);
      if (A.w == 0.0f || (CUT && P.prune_r2 > 0.0f && prune_node(C, gmin, gmax, P.prune_r2))) {
        k = tp.z;  // mass-zero and pruned nodes are skipped
        continue;
      }
      float d2, rc2;
      if (accept_node(C, gmin, gmax, P.beta, d2, rc2)) {
        float* na = node_adj + static_cast<int64_t>(k) * kNodeAdj;
        if (QUAD && quad_order(d2, rc2, P)) {
          far_quad_adjoint(nd, A, Q, wx, wy, wz, nslot, P, out != nullptr, gx, gy, gz, fx, fy, fz, na, r10);
        } else {
          far_mono_adjoint<CUT, PER>(A, Q, wx, wy, wz, nslot, P, out != nullptr, gx, gy, gz, fx, fy, fz, na, lane,
                                     r4);
        }
        k = tp.z;
      } else if (tp.w & kLeafFlag) {
        // the self pair (r = 0) only occurs when the leaf overlaps the group
        const bool selfchk = G.self && tp.x < gr.y && gr.x < tp.y;
        for (int j = tp.x; j < tp.y; j++) {
          float4 s = __ldg(&T.sp[j]);
          float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
          for (int t = 0; t < kTPL; t++) {
            if (t >= nslot) break;
            float rx = Q.x[t] - s.x, ry = Q.y[t] - s.y, rz = Q.z[t] - s.z;
            if (PER) {
              rx = min_image(rx, P);
              ry = min_image(ry, P);
              rz = min_image(rz, P);
            }
            float r2 = rx * rx + ry * ry + rz * rz;
            float ir = rsqrtf(r2 + P.eps2);
            float ih = ir * ir;
            float ir3 = ir * ih;
            float ir5 = ir3 * ih;
            float rw = rx * wx[t] + ry * wy[t] + rz * wz[t];
            float att = 1.0f, cc = 0.0f;
            if (CUT) attenuation(r2, ir3, P, att, cc);
            float lin = att * ir3;
            float m = (selfchk && j == Q.idx[t]) ? 0.0f : s.w;
            float mlin = m * lin, mrad = m * (rw * (3.0f * att * ir5 + cc));
            float qx_ = mrad * rx - mlin * wx[t];
            float qy_ = mrad * ry - mlin * wy[t];
            float qz_ = mrad * rz - mlin * wz[t];
            gx[t] += qx_;
            gy[t] += qy_;
            gz[t] += qz_;
            if (out) {
              fx[t] -= mlin * rx;
              fy[t] -= mlin * ry;
              fz[t] -= mlin * rz;
            }
            a0 -= qx_;
            a1 -= qy_;
            a2 -= qz_;
            a3 -= lin * rw;  // zero for the self pair (r = 0) and inactive slots (w = 0)
          }
          float tot = reduce4(a0, a1, a2, a3);
          if ((lane & 7) == 0) atomicAdd(&part_adj[static_cast<int64_t>(j) * kPartAdj + r4], tot);
        }
        k = tp.z;
      } else {
        k++;
      }
    }
#pragma unroll
    for (int t = 0; t < kTPL; t++) {
      if (Q.act[t]) {
        int64_t i = Q.idx[t];
        gq[3 * i] = gx[t];
        gq[3 * i + 1] = gy[t];
        gq[3 * i + 2] = gz[t];
        if (out) {
          const uint32_t o = G.perm[i];  // reloaded: not kept live through the walk
          out[3 * o] = fx[t];
          out[3 * o + 1] = fy[t];
          out[3 * o + 2] = fz[t];
        }
      }
    }
  }
}

// Interaction counts of the force and adjoint walks: the same traversal and
// the same decisions without the sums, so the hot walks carry no counters.
// Per group: accepted nodes (and those that take the quadrupole) and near
// source particles, each times the group's targets.
template <bool QUAD, bool CUT, bool PER>
__global__ void __launch_bounds__(128)
    count_walk_kernel(WalkTree T, WalkTargets G, WalkParams P, unsigned long long* __restrict__ counters) {
  const int lane = threadIdx.x & 31;
  const uint32_t ng = min(*G.ngroups, G.capacity);
  for (;;) {
    uint32_t gw = next_group(G);
    if (gw >= ng) break;
    int4 gr = G.groups[gw];
    if (gr.x < G.tbeg || gr.x >= G.tend) continue;
    LaneTargets Q;
    load_targets(G, gr, lane, Q);
    float gmin[3], gmax[3];
    group_box(Q, gmin, gmax);
    int2 rt = T.roots[gr.z];
    unsigned long long nfar = 0, nnear = 0, nquad = 0;
    int k = rt.x;
    while (k < rt.y) {
      const NodeRec* nd = T.nodes + k;
      const int4 tp = __ldg(&nd->topo);
      const float4 A = __ldg(&nd->com);
      float4 C = __ldg(&nd->cell);
      if (PER) C = cell_image(C, gmin, gmax, P);
      if (A.w == 0.0f || (CUT && P.prune_r2 > 0.0f && prune_node(C, gmin, gmax, P.prune_r2))) {
        k = tp.z;
        continue;
      }
      float d2, rc2;
      if (accept_node(C, gmin, gmax, P.beta, d2, rc2)) {
        nfar++;
        if (QUAD && quad_order(d2, rc2, P)) nquad++;
        k = tp.z;
      } else if (tp.w & kLeafFlag) {
        nnear += static_cast<unsigned long long>(tp.y - tp.x);
        k = tp.z;
      } else {
        k++;
      }
    }
    if (lane == 0) {
      unsigned long long na = static_cast<unsigned long long>(gr.y - gr.x);
      atomicAdd(&counters[0], nfar * na);
      atomicAdd(&counters[1], nnear * na);
      atomicAdd(&counters[2], nquad * na);
    }
  }
}

// Node adjoints -> difference arrays over each node's particle range. Per
// node (coordinates relative to the system's box centre c0, Xc = X - c0):
//   V_X = A_X / M, V_Q = A_M - A_X . Xc / M, G, G Xc, Xc^T G Xc   (14 values)
__global__ void node_push_kernel(const NodeRec* __restrict__ nodes, const uint32_t* __restrict__ nn_ptr,
                                 const float* __restrict__ node_adj, const uint32_t* __restrict__ sseg,
                                 const SegBox* __restrict__ boxes, DVec<14>* __restrict__ D) {
  uint32_t nn = *nn_ptr;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const float* a = node_adj + static_cast<int64_t>(k) * kNodeAdj;
    bool any = false;
    for (int c = 0; c < 10; c++) any |= a[c] != 0.0f;
    if (!any) continue;
    NodeRec r = nodes[k];
    double M = r.com.w;
    if (M == 0.0) continue;
    SegBox b = boxes[sseg ? sseg[r.topo.x] : 0];
    double half = 0.5 * static_cast<double>(b.span);
    double X[3] = {static_cast<double>(r.com.x) - (static_cast<double>(b.lo[0]) + half),
                   static_cast<double>(r.com.y) - (static_cast<double>(b.lo[1]) + half),
                   static_cast<double>(r.com.z) - (static_cast<double>(b.lo[2]) + half)};
    double AX[3] = {a[0], a[1], a[2]};
    double AM = a[3];
    double G[6] = {a[4], a[5], a[6], a[7], a[8], a[9]};
    double GX[3] = {G[0] * X[0] + G[3] * X[1] + G[4] * X[2], G[3] * X[0] + G[1] * X[1] + G[5] * X[2],
                    G[4] * X[0] + G[5] * X[1] + G[2] * X[2]};
    double val[14];
    val[0] = AX[0] / M;
    val[1] = AX[1] / M;
    val[2] = AX[2] / M;
    val[3] = AM - (AX[0] * X[0] + AX[1] * X[1] + AX[2] * X[2]) / M;
    for (int c = 0; c < 6; c++) val[4 + c] = G[c];
    for (int c = 0; c < 3; c++) val[10 + c] = GX[c];
    val[13] = X[0] * GX[0] + X[1] * GX[1] + X[2] * GX[2];
    for (int c = 0; c < 14; c++) {
      atomicAdd(&D[r.topo.x].v[c], val[c]);
      atomicAdd(&D[r.topo.y].v[c], -val[c]);
    }
  }
}

// Per sorted particle: query side + direct-source terms + node terms
// (inclusive prefix of D = exclusive prefix at i + 1).
__global__ void adjoint_combine_kernel(const float4* __restrict__ sp, const uint32_t* __restrict__ perm,
                                       const uint32_t* __restrict__ sseg, const SegBox* __restrict__ boxes, int64_t n,
                                       const float* __restrict__ gq, const float* __restrict__ part_adj,
                                       const DVec<14>* __restrict__ C, float* __restrict__ dx,
                                       float* __restrict__ dm) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float4 p = sp[i];
    SegBox b = boxes[sseg ? sseg[i] : 0];
    double half = 0.5 * static_cast<double>(b.span);
    double x[3] = {static_cast<double>(p.x) - (static_cast<double>(b.lo[0]) + half),
                   static_cast<double>(p.y) - (static_cast<double>(b.lo[1]) + half),
                   static_cast<double>(p.z) - (static_cast<double>(b.lo[2]) + half)};
    const DVec<14>& c = C[i + 1];
    const double* G = &c.v[4];
    double Gx[3] = {G[0] * x[0] + G[3] * x[1] + G[4] * x[2], G[3] * x[0] + G[1] * x[1] + G[5] * x[2],
                    G[4] * x[0] + G[5] * x[1] + G[2] * x[2]};
    double m = p.w;
    uint32_t o = perm[i];
    for (int d = 0; d < 3; d++) {
      double v = static_cast<double>(gq[3 * i + d]) + static_cast<double>(part_adj[kPartAdj * i + d]) +
                 m * (c.v[d] + 2.0 * (Gx[d] - c.v[10 + d]));
      dx[3 * o + d] = static_cast<float>(v);
    }
    double wq = c.v[3] + (c.v[0] * x[0] + c.v[1] * x[1] + c.v[2] * x[2]) +
                (x[0] * Gx[0] + x[1] * Gx[1] + x[2] * Gx[2]) -
                2.0 * (x[0] * c.v[10] + x[1] * c.v[11] + x[2] * c.v[12]) + c.v[13];
    dm[o] = static_cast<float>(static_cast<double>(part_adj[kPartAdj * i + 3]) + wq);
  }
}

// Winding number (include/kernel.h:73-80): w(q) = sum m n.(p - q) / (4 pi (|p-q|^3 + 1e-5));
// far field: node mass and mass-weighted mean normal at the COM, as the
// reference's trees aggregate them (include/tree3d.h:255-264, 310-327).
__global__ void __launch_bounds__(128, 4)
    wn_walk_kernel(WalkTree T, WalkTargets G, float beta, float* __restrict__ out,
                   unsigned long long* __restrict__ counters) {
  const int lane = threadIdx.x & 31;
  const uint32_t ng = min(*G.ngroups, G.capacity);
  const float k4pi = 0.07957747154594767f;  // 1 / (4 pi)
  for (;;) {
    uint32_t gw = next_group(G);
    if (gw >= ng) break;
    int4 gr = G.groups[gw];
    if (gr.x < G.tbeg || gr.x >= G.tend) continue;  // another rank's targets (warp-uniform)
    LaneTargets Q;
    load_targets(G, gr, lane, Q);
    const int nslot = (gr.y - gr.x + 31) / 32;  // warp-uniform: the target slots in use
    float gmin[3], gmax[3];
    group_box(Q, gmin, gmax);
    int2 rt = T.roots[gr.z];
    float far[kTPL], near[kTPL], comp[kTPL];
#pragma unroll
    for (int t = 0; t < kTPL; t++) far[t] = near[t] = comp[t] = 0.f;
    uint32_t nfar = 0, nnear = 0;  // per group (a group's counts stay below n)
    // Pre-order walk. The next node is known once this node's opening test
    // is done, so its opening data is loaded before this node's terms are
    // evaluated and the load latency hides behind that arithmetic.
    int k = rt.x;
    int4 tp = make_int4(0, 0, rt.y, 0);
    float4 A = make_float4(0.f, 0.f, 0.f, 0.f), C = A;
    if (k < rt.y) {
      tp = __ldg(&T.nodes[k].topo);
      A = __ldg(&T.nodes[k].com);
      C = __ldg(&T.nodes[k].cell);
    }
    while (k < rt.y) {
      const bool live = A.w != 0.0f;  // mass-zero nodes are skipped
      const bool acc = live && accept_node(C, gmin, gmax, beta);
      const bool leaf = (tp.w & kLeafFlag) != 0;
      const int next = (!live || acc || leaf) ? tp.z : k + 1;
      int4 tpn = tp;
      float4 An = A, Cn = C;
      if (next < rt.y) {
        tpn = __ldg(&T.nodes[next].topo);
        An = __ldg(&T.nodes[next].com);
        Cn = __ldg(&T.nodes[next].cell);
      }
      if (acc) {
        float4 N = __ldg(&T.nnrm[k]);
#pragma unroll
        for (int t = 0; t < kTPL; t++) {
          if (t >= nslot) break;
          float dx = A.x - Q.x[t], dy = A.y - Q.y[t], dz = A.z - Q.z[t];
          float dist = sqrtf(dx * dx + dy * dy + dz * dz);
          float nd_ = N.x * dx + N.y * dy + N.z * dz;
          far[t] += A.w * nd_ * k4pi / (dist * dist * dist + 1e-5f);
        }
        nfar++;
      } else if (live && leaf) {
        float a[kTPL];
#pragma unroll
        for (int t = 0; t < kTPL; t++) a[t] = 0.f;
        for (int j = tp.x; j < tp.y; j++) {
          float4 s = __ldg(&T.sp[j]);
          float4 nrm = __ldg(&T.sn[j]);
#pragma unroll
          for (int t = 0; t < kTPL; t++) {
            if (t >= nslot) break;
            float dx = s.x - Q.x[t], dy = s.y - Q.y[t], dz = s.z - Q.z[t];
            float dist = sqrtf(dx * dx + dy * dy + dz * dz);
            float nd_ = nrm.x * dx + nrm.y * dy + nrm.z * dz;
            a[t] += s.w * nd_ * k4pi / (dist * dist * dist + 1e-5f);
          }
        }
#pragma unroll
        for (int t = 0; t < kTPL; t++) kahan_add(near[t], comp[t], a[t]);
        nnear += static_cast<uint32_t>(tp.y - tp.x);
      }
      k = next;
      tp = tpn;
      A = An;
      C = Cn;
    }
#pragma unroll
    for (int t = 0; t < kTPL; t++)
      if (Q.act[t]) out[G.perm[Q.idx[t]]] = far[t] + near[t];
    if (counters && lane == 0) {
      unsigned long long na = static_cast<unsigned long long>(gr.y - gr.x);
      atomicAdd(&counters[0], nfar * na);
      atomicAdd(&counters[1], nnear * na);
    }
  }
}

// Query targets: keys in the box of system 0 (clamped), sorted, grouped in
// runs of kQueryGroup (one slot per lane: for queries spread evenly through
// the box, wider groups only add interactions; 2^20 uniform queries over
// 262,144 ellipsoid sources take 9.4 ms with runs of 32, 13.8 ms with 64 or
// 96).
__global__ void query_keys_kernel(const float* __restrict__ q, int64_t nq, const SegBox* __restrict__ boxes,
                                  uint64_t* __restrict__ keys) {
  SegBox b = boxes[0];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nq;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint64_t key = 0;
    for (int d = 0; d < 3; d++) {
      double t = __dmul_rn(__dsub_rn(static_cast<double>(q[3 * i + d]), static_cast<double>(b.lo[d])), b.scale);
      double f = floor(t);
      uint64_t qq = !(f >= 0.0) ? 0ull : (f > 2097151.0 ? 2097151ull : static_cast<uint64_t>(f));
      key |= spread21(qq) << d;
    }
    keys[i] = key;
  }
}

__global__ void query_gather_kernel(const float* __restrict__ q, const uint32_t* __restrict__ perm, int64_t nq,
                                    float4* __restrict__ tp, int4* __restrict__ groups, uint32_t* __restrict__ ngroups) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nq;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t s = perm[i];
    tp[i] = make_float4(q[3 * s], q[3 * s + 1], q[3 * s + 2], 0.0f);
    if (i % kQueryGroup == 0) {
      int64_t e = i + kQueryGroup < nq ? i + kQueryGroup : nq;
      groups[i / kQueryGroup] = make_int4(static_cast<int>(i), static_cast<int>(e), 0, 0);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *ngroups = static_cast<uint32_t>((nq + kQueryGroup - 1) / kQueryGroup);
}

}  // namespace nt
}  // namespace sbh

// ===========================================================================
// host side
// ===========================================================================
namespace sbh {
namespace nt {

struct Layout {
  // tree
  SegBox* boxes;
  uint32_t* bb;
  uint64_t* k0;
  uint64_t* k1;
  uint32_t* v0;
  uint32_t* v1;
  uint32_t* segkey;
  uint32_t* t0;
  uint32_t* t1;
  uint32_t* t2;
  uint32_t* t3;
  uint32_t* hist;
  uint32_t* scan_tmp;
  int8_t* cl;
  int8_t* dd;
  int8_t* lv;
  uint32_t* base;  // n + 1 node-slot offsets
  NodeRec* nodes;
  DVec<10>* P;
  DVec<10>* ptmp;
  DVec<3>* PN;
  DVec<3>* pntmp;
  float4* nnrm;
  float4* sp;
  float4* sn;
  uint32_t* perm;   // sorted slot -> input index (points into v0 or v1)
  uint32_t* sseg;   // sorted slot -> system
  int64_t* seg_off;
  int2* roots;
  int4* groups;
  uint32_t* work;  // persistent-walk work counters
  uint32_t* meta;  // [0] node count, [1] group count, [2] which ping-pong buffer holds perm
  unsigned long long* counters;
  // adjoint scratch
  float* node_adj;
  float* part_adj;
  float* gq;
  DVec<14>* D;
  DVec<14>* dtmp;
  int64_t cap;
};

inline int64_t node_capacity(int64_t n, int nseg, int S) { return 21 * (n / (S + 1)) + n + nseg + 1; }

template <typename C>
void carve(C& c, int64_t n, int nseg, int S, bool normals, bool adjoint, Layout& L) {
  int64_t nn = n > 0 ? n : 1;
  int64_t cap = node_capacity(n, nseg, S);
  L.cap = cap;
  L.meta = c.template take<uint32_t>(8);
  L.counters = c.template take<unsigned long long>(4);
  L.boxes = c.template take<SegBox>(nseg);
  L.bb = c.template take<uint32_t>(6 * nseg);
  L.seg_off = c.template take<int64_t>(nseg + 1);
  L.k0 = c.template take<uint64_t>(nn);
  L.k1 = c.template take<uint64_t>(nn);
  L.v0 = c.template take<uint32_t>(nn);
  L.v1 = c.template take<uint32_t>(nn);
  L.segkey = c.template take<uint32_t>(nn);
  int64_t tn = nseg > 1 ? nn : 1;
  L.t0 = c.template take<uint32_t>(tn);
  L.t1 = c.template take<uint32_t>(tn);
  L.t2 = c.template take<uint32_t>(tn);
  L.t3 = c.template take<uint32_t>(tn);
  int64_t hist_n = radix_hist_elems(nn);
  L.hist = c.template take<uint32_t>(hist_n);
  int64_t st = scan_tiles(hist_n), st2 = scan_tiles(nn + 1);
  L.scan_tmp = c.template take<uint32_t>((st > st2 ? st : st2) + scan_tiles(nseg + 1));
  L.cl = c.template take<int8_t>(nn);
  L.dd = c.template take<int8_t>(nn);
  L.lv = c.template take<int8_t>(nn);
  L.base = c.template take<uint32_t>(nn + 1);
  L.nodes = c.template take<NodeRec>(cap);
  L.P = c.template take<DVec<10>>(nn + 1);
  L.ptmp = c.template take<DVec<10>>(scan_tiles<DVec<10>>(nn));
  L.sp = c.template take<float4>(nn);
  L.sseg = c.template take<uint32_t>(nn);
  L.roots = c.template take<int2>(nseg);
  L.groups = c.template take<int4>(nn + nseg + 1);
  L.work = c.template take<uint32_t>(4);
  if (normals) {
    L.PN = c.template take<DVec<3>>(nn + 1);
    L.pntmp = c.template take<DVec<3>>(scan_tiles<DVec<3>>(nn));
    L.nnrm = c.template take<float4>(cap);
    L.sn = c.template take<float4>(nn);
  } else {
    L.PN = nullptr;
    L.pntmp = nullptr;
    L.nnrm = nullptr;
    L.sn = nullptr;
  }
  if (adjoint) {
    L.node_adj = c.template take<float>(cap * kNodeAdj);
    L.part_adj = c.template take<float>(nn * kPartAdj);
    L.gq = c.template take<float>(nn * 3);
    L.D = c.template take<DVec<14>>(nn + 1);
    L.dtmp = c.template take<DVec<14>>(scan_tiles<DVec<14>>(nn + 1));
  } else {
    L.node_adj = nullptr;
    L.part_adj = nullptr;
    L.gq = nullptr;
    L.D = nullptr;
    L.dtmp = nullptr;
  }
}

// The tree handle stored in the first bytes after the status word: the
// sizes the workspace was carved for, so later calls find the same layout.
struct Header {
  uint64_t magic;
  int64_t n;
  int32_t nseg;
  int32_t leaf_size;
  int32_t normals;
  int32_t adjoint;
  int64_t tbeg = 0, tend = INT64_MAX;  // sorted target range the walks serve
  // the last evaluation: 0 none, 1 a force or adjoint walk (its interaction
  // counts are recounted on demand), 2 the winding number (counted in-walk)
  int32_t last_walk = 0;
  bool counts_fresh = true;
  sbh_native_params last_params{};
  int64_t last_tbeg = 0, last_tend = INT64_MAX;
};
constexpr uint64_t kMagic = 0x5342483230304e54ull;  // "SBH200NT"

inline unsigned gs(int64_t n, int t = 256) {
  int64_t b = (n + t - 1) / t;
  if (b > 148 * 32) b = 148 * 32;
  return static_cast<unsigned>(b < 1 ? 1 : b);
}

struct SegCountLoad {
  const uint32_t* gc;
  __device__ uint32_t operator()(int64_t i) const { return gc[i]; }
};

}  // namespace nt
}  // namespace sbh

using namespace sbh;
using namespace sbh::nt;

namespace {

// Host registry: which tree (sizes) a workspace holds, so evaluation calls
// recover the workspace layout without reading device memory.
std::mutex g_reg_mu;
std::unordered_map<const void*, Header> g_registry;

int register_tree(void* ws, const Header& h) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  g_registry[ws] = h;
  return SBH_OK;
}

int native_layout(void* ws, size_t ws_bytes, const Header& h, Layout& L) {
  Carver c(ws, ws_bytes);
  carve(c, h.n, h.nseg, h.leaf_size, h.normals != 0, h.adjoint != 0, L);
  if (!c.ok) return fail(SBH_ERR_WORKSPACE, "workspace too small for the native tree");
  return SBH_OK;
}

}  // namespace

extern "C" {

int sbh_native_group_size(void) { return kGroup; }

size_t sbh_native_workspace_bytes(int64_t n, int num_systems, int leaf_size, int with_normals, int with_adjoint) {
  if (n < 0 || num_systems < 1 || leaf_size < 1 || leaf_size > 32) return 0;
  Sizer s;
  Layout L;
  carve(s, n, num_systems, leaf_size, with_normals != 0, with_adjoint != 0, L);
  return s.off;
}

int sbh_native_build(cudaStream_t stream, const float* points, const float* masses, const float* normals, int64_t n,
                     const int64_t* system_offsets, int num_systems, int leaf_size, int with_adjoint,
                     void* workspace, size_t workspace_bytes) {
  if (n < 0 || n >= (1ll << 31)) return invalid("number of points must be in [0, 2^31)");
  if (num_systems < 1) return invalid("num_systems must be >= 1");
  if (num_systems > 1 && !system_offsets) return invalid("system_offsets is required when num_systems > 1");
  if (leaf_size < 1 || leaf_size > 32) return invalid("leaf_size must be in [1, 32]");
  if (n > 0 && (!points || !masses)) return invalid("points and masses must be non-null");
  if (!workspace) return fail(SBH_ERR_WORKSPACE, "workspace is null");
  size_t need = sbh_native_workspace_bytes(n, num_systems, leaf_size, normals != nullptr, with_adjoint);
  if (workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Header h{kMagic, n, num_systems, leaf_size, normals != nullptr, with_adjoint != 0};
  Layout L;
  if (int rc = native_layout(workspace, workspace_bytes, h, L)) return rc;
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, 64, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(L.meta, 0, 8 * sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(L.counters, 0, 4 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  // system offsets (device copy, or [0, n] for one system)
  if (num_systems > 1) {
    e = cudaMemcpyAsync(L.seg_off, system_offsets, (num_systems + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice,
                        stream);
  } else {
    single_offsets_kernel<<<1, 1, 0, stream>>>(L.seg_off, n);
  }
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  int nseg = num_systems;
  bbox_init_kernel<<<(nseg + 255) / 256, 256, 0, stream>>>(L.bb, nseg);
  if (n > 0) bbox_kernel<<<gs(n), 256, 0, stream>>>(points, n, L.seg_off, nseg, L.bb);
  bbox_finalize_kernel<<<(nseg + 255) / 256, 256, 0, stream>>>(L.bb, nseg, L.seg_off, L.boxes);
  const uint32_t* perm = L.v0;
  if (n > 0) {
    keys_kernel<<<gs(n), 256, 0, stream>>>(points, n, L.seg_off, nseg, L.boxes, L.k0, nseg > 1 ? L.segkey : nullptr);
    int which = 0;
    e = radix_sort<uint64_t>(stream, L.k0, L.v0, L.k1, L.v1, n, 63, false, L.hist, L.scan_tmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    uint64_t* ksorted = which == 0 ? L.k0 : L.k1;
    uint32_t* vsorted = which == 0 ? L.v0 : L.v1;
    if (nseg > 1) {
      // Stable pass on the system id over the key-sorted order: payload =
      // position in that order, then gather keys and input indices.
      gather_u32_kernel<<<gs(n), 256, 0, stream>>>(L.segkey, vsorted, n, L.t0);
      int bits = 0;
      while ((1 << bits) < nseg) bits++;
      int w2 = 0;
      e = radix_sort<uint32_t>(stream, L.t0, L.t2, L.t1, L.t3, n, bits, false, L.hist, L.scan_tmp, &w2);
      if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
      const uint32_t* p2 = w2 == 0 ? L.t2 : L.t3;
      uint64_t* kout = which == 0 ? L.k1 : L.k0;
      uint32_t* vout = which == 0 ? L.v1 : L.v0;
      gather_keys_kernel<<<gs(n), 256, 0, stream>>>(ksorted, p2, n, kout);
      gather_u32_kernel<<<gs(n), 256, 0, stream>>>(vsorted, p2, n, vout);
      ksorted = kout;
      vsorted = vout;
      sseg_kernel<<<gs(n), 256, 0, stream>>>(L.seg_off, nseg, n, L.sseg);
    }
    if (ksorted != L.k0) {
      e = cudaMemcpyAsync(L.k0, ksorted, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(L.v0, vsorted, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
      if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    }
    perm = L.v0;
    const uint32_t* sseg = nseg > 1 ? L.sseg : nullptr;
    levels_kernel<<<gs(n), 256, 0, stream>>>(L.k0, sseg, n, leaf_size, L.cl, L.dd);
    slots_kernel<<<gs(n), 256, 0, stream>>>(L.cl, L.dd, n, leaf_size, L.lv, L.base);
    e = exclusive_scan<uint32_t>(stream, ArrayLoad<uint32_t>{L.base}, n, L.base, L.scan_tmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    emit_nodes_kernel<<<gs(n), 256, 0, stream>>>(L.k0, sseg, L.seg_off, n, L.dd, L.lv, L.base, L.nodes, L.cap, status);
    node_count_kernel<<<1, 1, 0, stream>>>(L.base, n, L.cap, L.meta);
    gather_particles_kernel<<<gs(n), 256, 0, stream>>>(points, masses, normals, perm, n, L.sp, L.sn);
    e = exclusive_scan<DVec<10>>(stream, MomentLoad{L.sp, sseg, L.boxes}, n, L.P, L.ptmp, true);
    if (e == cudaSuccess && normals)
      e = exclusive_scan<DVec<3>>(stream, NormalMomentLoad{L.sp, L.sn}, n, L.PN, L.pntmp, true);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    finalize_nodes_kernel<<<gs(static_cast<int64_t>(L.cap)), 256, 0, stream>>>(L.nodes, L.meta, L.k0, sseg, L.boxes,
                                                                                L.P, L.PN, L.nnrm);
  } else {
    e = cudaMemsetAsync(L.base, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  }
  // system roots and target groups (meta[1] counts the groups)
  roots_kernel<<<nseg, 32, 0, stream>>>(L.seg_off, nseg, L.base, L.cap, L.roots);
  if (n > 0)
    group_nodes_kernel<<<gs(static_cast<int64_t>(L.cap)), 256, 0, stream>>>(
        L.nodes, L.meta, nseg > 1 ? L.sseg : nullptr, L.groups, n + nseg + 1, kGroup, L.meta + 1, status);
  if (int rc = check_launch("sbh_native_build")) return rc;
  return register_tree(workspace, h);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// evaluation entry points
// ---------------------------------------------------------------------------
namespace {

int lookup(const void* ws, size_t ws_bytes, Header& h, Layout& L) {
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_registry.find(ws);
    if (it == g_registry.end()) return invalid("workspace holds no native tree; call sbh_native_build first");
    h = it->second;
  }
  return native_layout(const_cast<void*>(ws), ws_bytes, h, L);
}

// Records which evaluation last ran on the tree in `ws` (Header::last_walk).
void remember_walk(const void* ws, int kind, const sbh_native_params* p) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  auto it = g_registry.find(ws);
  if (it == g_registry.end()) return;
  Header& h = it->second;
  h.last_walk = kind;
  if (p) h.last_params = *p;
  h.last_tbeg = h.tbeg;
  h.last_tend = h.tend;
  h.counts_fresh = kind != 1;
}

__global__ void zero_node_adj_kernel(float* adj, const uint32_t* meta) {
  int64_t total = static_cast<int64_t>(meta[0]) * kNodeAdj;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    adj[i] = 0.0f;
}

WalkTree tree_view(const Layout& L) { return WalkTree{L.nodes, L.sp, L.sn, L.nnrm, L.roots}; }

WalkTargets self_targets(const Layout& L, const Header& h) {
  return WalkTargets{L.sp,      L.v0, L.groups, L.meta + 1, 1, L.work, static_cast<uint32_t>(h.n + h.nseg + 1),
                     h.tbeg, h.tend};
}

bool partial_range(const Header& h) { return h.tbeg > 0 || h.tend < h.n; }

// Blocks of a persistent walk: resident blocks per SM x SMs, and no more
// than one warp per possible group. Occupancy is queried per kernel and
// device once (a host-side query; nothing is enqueued).
template <typename K>
unsigned walk_blocks(K kernel, int64_t max_groups) {
  struct Key {
    const void* k;
    int dev;
    bool operator<(const Key& o) const { return k < o.k || (k == o.k && dev < o.dev); }
  };
  static std::mutex mu;
  static std::map<Key, unsigned> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  Key key{reinterpret_cast<const void*>(kernel), dev};
  unsigned resident = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) resident = it->second;
  }
  if (resident == 0) {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0) != cudaSuccess || per_sm <= 0)
      per_sm = 4;
    resident = static_cast<unsigned>(sms * per_sm);
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = resident;
  }
  int64_t need = (max_groups + 3) / 4;
  if (need < 1) need = 1;
  return need < resident ? static_cast<unsigned>(need) : resident;
}

// Zeroes the work counter and launches a persistent walk over the groups.
template <typename K, typename... A>
cudaError_t launch_walk(cudaStream_t stream, uint32_t* counter, int64_t max_groups, K kernel, A... args) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  kernel<<<walk_blocks(kernel, max_groups), 128, 0, stream>>>(args...);
  return cudaGetLastError();
}

int check_params(const sbh_native_params* p) {
  if (!p) return invalid("params must be non-null");
  if (!(p->beta > 0.0f)) return invalid("beta must be > 0");
  if (p->softening < 0.0f) return invalid("softening must be >= 0");
  if (p->quadrupole && p->cutoff > 0.0f) return invalid("the quadrupole far field needs cutoff <= 0 (Plummer)");
  if (p->periodic && !(p->box_length > 0.0f)) return invalid("box_length must be > 0 when periodic is set");
  if (p->periodic && p->quadrupole) return invalid("the periodic walk uses the monopole far field (quadrupole = 0)");
  if (p->prune_radius < 0.0f) return invalid("prune_radius must be >= 0");
  if (p->prune_radius > 0.0f && !(p->cutoff > 0.0f)) return invalid("prune_radius needs an erfc cutoff (cutoff > 0)");
  if (!(p->quadrupole_radius >= 0.0f)) return invalid("quadrupole_radius must be >= 0");
  return SBH_OK;
}

WalkParams walk_params(const sbh_native_params* p) {
  float eps = fmaxf(p->softening, 0.0f);
  float box = p->periodic ? p->box_length : 1.0f;
  float qr = p->quadrupole_radius;
  double c = p->cutoff > 0.0f ? static_cast<double>(p->cutoff) : 1.0;
  return WalkParams{p->beta,
                    eps * eps + 1e-12f,
                    p->cutoff,
                    box,
                    1.0f / box,
                    p->prune_radius * p->prune_radius,
                    qr > 0.0f ? qr * qr : 0.0f,
                    static_cast<float>(0.5 / c),
                    static_cast<float>(1.0 / (2.0 * 1.7724538509055160 * c * c * c))};
}

// Recounts the interactions of the last force or adjoint walk (same tree,
// parameters and target range) into the counters, once per walk.
int refresh_counts(cudaStream_t stream, const void* ws, const Header& h, const Layout& L) {
  if (h.last_walk != 1 || h.counts_fresh) return SBH_OK;
  cudaError_t e = cudaMemsetAsync(L.counters, 0, 3 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  const sbh_native_params& p = h.last_params;
  Header hr = h;
  hr.tbeg = h.last_tbeg;
  hr.tend = h.last_tend;
  WalkParams wp = walk_params(&p);
  bool cut = p.cutoff > 0.0f;
  bool per = p.periodic != 0;
  auto k = p.quadrupole ? count_walk_kernel<true, false, false>
           : per ? (cut ? count_walk_kernel<false, true, true> : count_walk_kernel<false, false, true>)
                 : (cut ? count_walk_kernel<false, true, false> : count_walk_kernel<false, false, false>);
  e = launch_walk(stream, L.work, h.n + h.nseg, k, tree_view(L), self_targets(L, hr), wp, L.counters);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_reg_mu);
  auto it = g_registry.find(ws);
  if (it != g_registry.end()) it->second.counts_fresh = true;
  return SBH_OK;
}


}  // namespace

extern "C" {

// Re-cuts the target groups of the tree in `workspace` with at most
// group_size targets each (the build cuts groups of kGroup).
int sbh_native_set_group_size(cudaStream_t stream, void* workspace, size_t workspace_bytes, int group_size) {
  if (group_size < 1 || group_size > kGroup)
    return invalid("group_size must be in [1, " + std::to_string(kGroup) + "]");
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (h.n == 0) return SBH_OK;
  cudaError_t e = cudaMemsetAsync(L.meta + 1, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  group_nodes_kernel<<<gs(static_cast<int64_t>(L.cap)), 256, 0, stream>>>(
      L.nodes, L.meta, h.nseg > 1 ? L.sseg : nullptr, L.groups, h.n + h.nseg + 1, group_size, L.meta + 1,
      static_cast<uint32_t*>(workspace));
  return check_launch("sbh_native_set_group_size");
}

// Restricts the force and adjoint walks on the tree in `workspace` to the
// target groups whose first target lies at sorted positions [begin, end).
// Ranks holding the same tree and a partition of [0, n) into such ranges
// serve every target exactly once; each rank's forces are zero outside its
// targets and its gradients are partial sums, so summing the ranks' outputs
// gives the full force and gradient. A new build resets the range to [0, n).
int sbh_native_set_target_range(cudaStream_t stream, void* workspace, size_t workspace_bytes, int64_t begin,
                                int64_t end) {
  (void)stream;  // host-side state only
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (begin < 0 || end < begin || end > h.n) return invalid("target range must satisfy 0 <= begin <= end <= n");
  std::lock_guard<std::mutex> lk(g_reg_mu);
  auto it = g_registry.find(workspace);
  if (it == g_registry.end()) return invalid("workspace holds no native tree; call sbh_native_build first");
  it->second.tbeg = begin;
  it->second.tend = end;
  return SBH_OK;
}

int sbh_native_force(cudaStream_t stream, const sbh_native_params* params, float* force_out, void* workspace,
                     size_t workspace_bytes) {
  if (int rc = check_params(params)) return rc;
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (h.n == 0) return SBH_OK;
  if (!force_out) return invalid("force_out must be non-null");
  cudaError_t e = cudaSuccess;
  // with a partial target range the other targets' rows are zero (ranks sum their outputs)
  if (partial_range(h)) e = cudaMemsetAsync(force_out, 0, h.n * 3 * sizeof(float), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  WalkParams wp = walk_params(params);
  int64_t mg = h.n + h.nseg;
  bool cut = params->cutoff > 0.0f;
  bool per = params->periodic != 0;
  auto k = params->quadrupole ? force_walk_kernel<true, false, false>
           : per ? (cut ? force_walk_kernel<false, true, true> : force_walk_kernel<false, false, true>)
                 : (cut ? force_walk_kernel<false, true, false> : force_walk_kernel<false, false, false>);
  e = launch_walk(stream, L.work, mg, k, tree_view(L), self_targets(L, h), wp, force_out);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 1, params);
  return check_launch("sbh_native_force");
}

int sbh_native_adjoint_walk(cudaStream_t stream, const sbh_native_params* params, const float* cotangent,
                            float* force_out, void* workspace, size_t workspace_bytes) {
  if (int rc = check_params(params)) return rc;
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.adjoint) return invalid("the tree was built without adjoint scratch (with_adjoint = 0)");
  if (h.n == 0) return SBH_OK;
  if (!cotangent) return invalid("cotangent must be non-null");
  int64_t n = h.n;
  cudaError_t e = cudaMemsetAsync(L.part_adj, 0, n * kPartAdj * sizeof(float), stream);
  // with a partial target range the query-side gradient (added for every particle by the
  // finalize) and the force rows of the other targets are zero
  if (e == cudaSuccess && partial_range(h)) e = cudaMemsetAsync(L.gq, 0, n * 3 * sizeof(float), stream);
  if (e == cudaSuccess && partial_range(h) && force_out)
    e = cudaMemsetAsync(force_out, 0, n * 3 * sizeof(float), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  zero_node_adj_kernel<<<gs(L.cap * kNodeAdj), 256, 0, stream>>>(L.node_adj, L.meta);
  WalkParams wp = walk_params(params);
  bool cut = params->cutoff > 0.0f;
  bool per = params->periodic != 0;
  auto k = params->quadrupole ? adjoint_walk_kernel<true, false, false>
           : per ? (cut ? adjoint_walk_kernel<false, true, true> : adjoint_walk_kernel<false, false, true>)
                 : (cut ? adjoint_walk_kernel<false, true, false> : adjoint_walk_kernel<false, false, false>);
  e = launch_walk(stream, L.work, n + h.nseg, k, tree_view(L), self_targets(L, h), wp, cotangent, force_out, L.gq,
                  L.node_adj, L.part_adj);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 1, params);
  return check_launch("sbh_native_adjoint_walk");
}

int sbh_native_adjoint_finalize(cudaStream_t stream, float* grad_points, float* grad_masses, void* workspace,
                                size_t workspace_bytes) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.adjoint) return invalid("the tree was built without adjoint scratch (with_adjoint = 0)");
  if (h.n == 0) return SBH_OK;
  if (!grad_points || !grad_masses) return invalid("gradient outputs must be non-null");
  int64_t n = h.n;
  cudaError_t e = cudaMemsetAsync(L.D, 0, (n + 1) * sizeof(DVec<14>), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  const uint32_t* sseg = h.nseg > 1 ? L.sseg : nullptr;
  node_push_kernel<<<gs(L.cap), 256, 0, stream>>>(L.nodes, L.meta, L.node_adj, sseg, L.boxes, L.D);
  e = exclusive_scan<DVec<14>>(stream, ArrayLoad<DVec<14>>{L.D}, n + 1, L.D, L.dtmp, false);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  adjoint_combine_kernel<<<gs(n), 256, 0, stream>>>(L.sp, L.v0, sseg, L.boxes, n, L.gq, L.part_adj, L.D, grad_points,
                                                    grad_masses);
  return check_launch("sbh_native_adjoint_finalize");
}

int sbh_native_force_vjp(cudaStream_t stream, const sbh_native_params* params, const float* cotangent,
                         float* force_out, float* grad_points, float* grad_masses, void* workspace,
                         size_t workspace_bytes) {
  if (!grad_points || !grad_masses) return invalid("gradient outputs must be non-null");
  if (int rc = sbh_native_adjoint_walk(stream, params, cotangent, force_out, workspace, workspace_bytes)) return rc;
  return sbh_native_adjoint_finalize(stream, grad_points, grad_masses, workspace, workspace_bytes);
}

size_t sbh_native_query_workspace_bytes(int64_t nq) {
  if (nq < 0) return 0;
  Sizer s;
  int64_t nn = nq > 0 ? nq : 1;
  s.take<uint32_t>(8);
  s.take<uint64_t>(nn);
  s.take<uint64_t>(nn);
  s.take<uint32_t>(nn);
  s.take<uint32_t>(nn);
  s.take<uint32_t>(radix_hist_elems(nn));
  s.take<uint32_t>(scan_tiles(radix_hist_elems(nn)));
  s.take<float4>(nn);
  s.take<int4>(nn / kQueryGroup + 1);
  return s.off;
}

int sbh_native_winding_number(cudaStream_t stream, float beta, const float* queries, int64_t nq, float* out,
                              void* workspace, size_t workspace_bytes, void* query_workspace,
                              size_t query_workspace_bytes) {
  if (!(beta > 0.0f)) return invalid("beta must be > 0");
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.normals) return invalid("the tree was built without normals");
  if (h.nseg != 1) return invalid("query evaluation needs a single-system tree");
  if (nq < 0 || nq >= (1ll << 31)) return invalid("number of queries must be in [0, 2^31)");
  if (nq == 0) return SBH_OK;
  if (!queries || !out) return invalid("queries and out must be non-null");
  size_t need = sbh_native_query_workspace_bytes(nq);
  if (!query_workspace || query_workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "query workspace too small: need " + std::to_string(need) + " bytes");
  if (h.n == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, nq * sizeof(float), stream);
    return e == cudaSuccess ? SBH_OK : fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  }
  Carver c(query_workspace, query_workspace_bytes);
  uint32_t* qmeta = c.take<uint32_t>(8);
  uint64_t* k0 = c.take<uint64_t>(nq);
  uint64_t* k1 = c.take<uint64_t>(nq);
  uint32_t* v0 = c.take<uint32_t>(nq);
  uint32_t* v1 = c.take<uint32_t>(nq);
  uint32_t* hist = c.take<uint32_t>(radix_hist_elems(nq));
  uint32_t* stmp = c.take<uint32_t>(scan_tiles(radix_hist_elems(nq)));
  float4* tp = c.take<float4>(nq);
  int4* groups = c.take<int4>(nq / kQueryGroup + 1);
  query_keys_kernel<<<gs(nq), 256, 0, stream>>>(queries, nq, L.boxes, k0);
  int which = 0;
  cudaError_t e = radix_sort<uint64_t>(stream, k0, v0, k1, v1, nq, 63, false, hist, stmp, &which);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  const uint32_t* qperm = which == 0 ? v0 : v1;
  query_gather_kernel<<<gs(nq), 256, 0, stream>>>(queries, qperm, nq, tp, groups, qmeta);
  e = cudaMemsetAsync(L.counters, 0, 3 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  WalkTargets G{tp, qperm, groups, qmeta, 0, qmeta + 2, static_cast<uint32_t>(nq / kQueryGroup + 1), 0, INT64_MAX};
  e = launch_walk(stream, qmeta + 2, nq / kQueryGroup + 1, wn_walk_kernel, tree_view(L), G, beta, out, L.counters);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 2, nullptr);
  return check_launch("sbh_native_winding_number");
}

// Synchronises the stream and reports [node count, group count, far
// interactions, near interactions] of the last build / evaluation.
int sbh_native_stats(cudaStream_t stream, const void* workspace, size_t workspace_bytes, uint64_t* out4) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  uint32_t meta[8];
  unsigned long long cnt[3];
  if (int rc = refresh_counts(stream, workspace, h, L)) return rc;
  cudaError_t e = cudaMemcpyAsync(meta, L.meta, sizeof(meta), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, L.counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  out4[0] = meta[0];
  out4[1] = meta[1];
  out4[2] = cnt[0];
  out4[3] = cnt[1];
  if (meta[3]) return fail(SBH_ERR_LIMIT, "node capacity exceeded");
  return SBH_OK;
}

int sbh_native_quadrupole_count(cudaStream_t stream, const void* workspace, size_t workspace_bytes,
                                uint64_t* far_quadrupole) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!far_quadrupole) return invalid("far_quadrupole must be non-null");
  if (int rc = refresh_counts(stream, workspace, h, L)) return rc;
  unsigned long long c = 0;
  cudaError_t e = cudaMemcpyAsync(&c, L.counters + 2, sizeof(c), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  *far_quadrupole = c;
  return SBH_OK;
}

// Copies the tree to caller buffers (device pointers; any may be null):
// sorted keys (n), permutation (n, sorted slot -> input index), nodes
// (num_nodes x 80 bytes), and the node count to *num_nodes (synchronises).
int sbh_native_export(cudaStream_t stream, const void* workspace, size_t workspace_bytes, uint64_t* keys_out,
                      uint32_t* perm_out, void* nodes_out, size_t nodes_capacity, uint64_t* num_nodes) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  uint32_t nn = 0;
  cudaError_t e = cudaMemcpyAsync(&nn, L.meta, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (num_nodes) *num_nodes = nn;
  if (keys_out && h.n > 0) e = cudaMemcpyAsync(keys_out, L.k0, h.n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream);
  if (e == cudaSuccess && perm_out && h.n > 0)
    e = cudaMemcpyAsync(perm_out, L.v0, h.n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream);
  if (e == cudaSuccess && nodes_out) {
    if (nodes_capacity < nn) return invalid("nodes_out too small");
    e = cudaMemcpyAsync(nodes_out, L.nodes, static_cast<size_t>(nn) * sizeof(NodeRec), cudaMemcpyDeviceToDevice,
                        stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  return SBH_OK;
}

}  // extern "C"
