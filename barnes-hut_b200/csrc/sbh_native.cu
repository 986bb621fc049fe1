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
#include "sbh_f32x2.cuh"
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
// child run. Every group holds at least one particle, so n + systems + 1
// slots always suffice.
//
// The groups are stored deepest first: a counting pass (COUNT) tallies them
// by the level of the cells they come from, group_bins_kernel turns the
// tallies into cursors, and the emitting pass writes each group at its
// level's cursor. Deeper cells lie in denser regions, where a group has more
// interactions, so the persistent walks hand out the expensive groups first
// and the cheap ones fill the tail. Within a level the order comes from
// atomics and varies between runs; each group's result does not.
constexpr int kGroupBins = 24;  // levels 0..22 (a run of children sits one level below its parent)

template <bool COUNT>
__device__ __forceinline__ void emit_chunks(int4* groups, uint32_t* bins, int64_t cap, int s0, int s1, int sys,
                                            int G, int level, uint32_t* status) {
  int ng = (s1 - s0 + G - 1) / G;
  if (ng <= 0) return;
  const int bin = kGroupBins - 1 - min(level, kGroupBins - 1);
  if (COUNT) {
    atomicAdd(&bins[bin], static_cast<uint32_t>(ng));
    return;
  }
  uint32_t slot = atomicAdd(&bins[bin], static_cast<uint32_t>(ng));
  for (int g = 0; g < ng; g++) {
    int s = s0 + g * G;
    if (slot + g < cap)
      groups[slot + g] = make_int4(s, min(s + G, s1), sys, level);
    else
      raise_status(status, SBH_DEV_ITER_LIMIT);
  }
}

template <bool COUNT>
__global__ void group_nodes_kernel(const NodeRec* __restrict__ nodes, const uint32_t* __restrict__ nn_ptr,
                                   const uint32_t* __restrict__ sseg, int4* __restrict__ groups, int64_t cap, int G,
                                   uint32_t* __restrict__ bins, uint32_t* status) {
  uint32_t nn = *nn_ptr;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    int4 t = nodes[k].topo;
    int cnt = t.y - t.x;
    bool leaf = (t.w & kLeafFlag) != 0;
    int level = t.w & 0xFF;
    bool root = level == 0;
    int sys = sseg ? static_cast<int>(sseg[t.x]) : 0;
    if (leaf || cnt <= G) {
      if (root || (leaf && cnt > G)) emit_chunks<COUNT>(groups, bins, cap, t.x, t.y, sys, G, level, status);
      continue;
    }
    int run_s = -1, run_e = -1;
    for (uint32_t c = k + 1; c < static_cast<uint32_t>(t.z) && c < nn;) {
      int4 tc = nodes[c].topo;
      if (tc.y - tc.x > G) {
        if (run_s >= 0) emit_chunks<COUNT>(groups, bins, cap, run_s, run_e, sys, G, level + 1, status);
        run_s = -1;
      } else {
        if (run_s < 0) run_s = tc.x;
        run_e = tc.y;
      }
      if (static_cast<uint32_t>(tc.z) <= c) break;  // malformed skip: never loop
      c = static_cast<uint32_t>(tc.z);
    }
    if (run_s >= 0) emit_chunks<COUNT>(groups, bins, cap, run_s, run_e, sys, G, level + 1, status);
  }
}

// Tallies per level -> cursors (exclusive offsets, deepest level first) and
// the group count.
__global__ void group_bins_kernel(uint32_t* bins, uint32_t* group_count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t run = 0;
  for (int b = 0; b < kGroupBins; b++) {
    uint32_t c = bins[b];
    bins[b] = run;
    run += c;
  }
  *group_count = run;
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
  float quad_lin;  // kappa^2 > 0: accepted quadrupole nodes with r_g^2 <= kappa^2 |c - cell centre|^2 take
                   // the quadrupole to first order about the group centre c; 0: never
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

// ---------------------------------------------------------------------------
// Linearized quadrupole. An accepted node whose cell lies far from the group
// compared with the group's size (r_g^2 <= kappa^2 |c - cell centre|^2, c the
// group box centre, r_g its half diagonal) takes its quadrupole field to
// first order about c: a_q(x_t - X) ~ a_q(c - X) + J(c - X) (x_t - c), J the
// field's (symmetric) Jacobian. The sum over such nodes of a_q(c - X) and
// J(c - X) is then one 9-value expansion per group, applied to each target
// once at the end of the walk, instead of one quadrupole evaluation per
// (target, node) pair. The monopole stays exact at every target. With
// h = |x|^2 + eps^2 and f_n = h^{-(2n+1)/2}:
//   a_q = (1.5 tr S f2 - 7.5 (x.Sx) f3) x + 3 f2 Sx,
//   J   = (52.5 (x.Sx) f4 - 7.5 tr S f3) x x^T - 15 f3 (Sx x^T + x (Sx)^T)
//         + (1.5 tr S f2 - 7.5 (x.Sx) f3) I + 3 f2 S.
// For the adjoint, a group's linearized terms contribute w_t . (a_q + J dx_t)
// to L; per node that is W . a_q(x) + V : J(x) with W = sum_t w_t and
// V = sym sum_t w_t (x_t - c)^T, whose gradients with respect to x = c - X
// and S (contractions of the third to fifth derivatives of h^{-1/2}) are
//   dL/dx = J W + 0.5 [ -945 f5 (x.Sx)(x.Vx) x
//             + 105 f4 ((tr S (x.Vx) + tr V (x.Sx) + 4 Sx.Vx) x + 2 (x.Vx) Sx + 2 (x.Sx) Vx)
//             - 15 f3 ((tr S tr V + 2 S:V) x + 4 V Sx + 4 S Vx + 2 tr V Sx + 2 tr S Vx) ],
//   dL/dS = c1 x x^T + 1.5 f2 (W x^T + x W^T) - 15 f3 (Vx x^T + x (Vx)^T) + c2 I + 3 f2 V,
//   c1 = -7.5 (W.x) f3 + 52.5 (x.Vx) f4 - 7.5 tr V f3, c2 = 1.5 (W.x) f2 - 7.5 (x.Vx) f3 + 1.5 tr V f2,
// and dL/dX = -dL/dx. Symmetric 3x3 matrices are packed (xx, yy, zz, xy, xz, yz).

__device__ __forceinline__ void lq_symv(const float* A, float x0, float x1, float x2, float* o) {
  o[0] = fmaf(A[0], x0, fmaf(A[3], x1, A[4] * x2));
  o[1] = fmaf(A[3], x0, fmaf(A[1], x1, A[5] * x2));
  o[2] = fmaf(A[4], x0, fmaf(A[5], x1, A[2] * x2));
}

// a_q(x) and J(x) packed, for x = c - X (the second moment S packed).
__device__ __forceinline__ void lq_field(const float* x, const float* S, float eps2, float* a, float* J, float* f) {
  const float h = fmaf(x[0], x[0], fmaf(x[1], x[1], fmaf(x[2], x[2], eps2)));
  const float ir = rsqrtf(h), ih = ir * ir;
  f[0] = ir * ih * ih;  // f2
  f[1] = f[0] * ih;     // f3
  f[2] = f[1] * ih;     // f4
  f[3] = f[2] * ih;     // f5
  float Sx[3];
  lq_symv(S, x[0], x[1], x[2], Sx);
  const float trS = S[0] + S[1] + S[2];
  const float xSx = fmaf(x[0], Sx[0], fmaf(x[1], Sx[1], x[2] * Sx[2]));
  const float be = fmaf(1.5f * trS, f[0], -7.5f * xSx * f[1]);
  const float al = fmaf(52.5f * xSx, f[2], -7.5f * trS * f[1]);
  const float f2x3 = 3.0f * f[0], f3x15 = 15.0f * f[1];
#pragma unroll
  for (int d = 0; d < 3; d++) a[d] = fmaf(be, x[d], f2x3 * Sx[d]);
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int e = 0; e < 6; e++) {
    const int i = ii[e], j = jj[e];
    float v = fmaf(al * x[i], x[j], -f3x15 * fmaf(Sx[i], x[j], x[i] * Sx[j]));
    v = fmaf(f2x3, S[e], v);
    J[e] = i == j ? v + be : v;
  }
}

// dL/dx (g) and dL/dS (G, packed) of L = W . a_q(x) + V : J(x), from
// lq_field's J and radial factors f = (f2, f3, f4, f5).
__device__ __forceinline__ void lq_node_adjoint(const float* x, const float* S, const float* J, const float* f,
                                                const float* W, const float* V, float* g, float* G) {
  float Sx[3], Vx[3], SVx[3], VSx[3];
  lq_symv(S, x[0], x[1], x[2], Sx);
  lq_symv(V, x[0], x[1], x[2], Vx);
  lq_symv(S, Vx[0], Vx[1], Vx[2], SVx);
  lq_symv(V, Sx[0], Sx[1], Sx[2], VSx);
  lq_symv(J, W[0], W[1], W[2], g);  // J W
  const float trS = S[0] + S[1] + S[2], trV = V[0] + V[1] + V[2];
  const float xSx = fmaf(x[0], Sx[0], fmaf(x[1], Sx[1], x[2] * Sx[2]));
  const float xVx = fmaf(x[0], Vx[0], fmaf(x[1], Vx[1], x[2] * Vx[2]));
  const float SxVx = fmaf(Sx[0], Vx[0], fmaf(Sx[1], Vx[1], Sx[2] * Vx[2]));
  const float SdV = fmaf(S[0], V[0], fmaf(S[1], V[1], fmaf(S[2], V[2],
                    2.0f * fmaf(S[3], V[3], fmaf(S[4], V[4], S[5] * V[5])))));
  const float Wx = fmaf(W[0], x[0], fmaf(W[1], x[1], W[2] * x[2]));
  const float f2 = f[0], f3 = f[1], f4 = f[2], f5 = f[3];
  const float kx = fmaf(-945.0f * f5, xSx * xVx,
                        fmaf(105.0f * f4, fmaf(trS, xVx, fmaf(trV, xSx, 4.0f * SxVx)),
                             -15.0f * f3 * fmaf(trS, trV, 2.0f * SdV)));
  const float c4a = 105.0f * f4 * xVx, c4b = 105.0f * f4 * xSx, c3 = -7.5f * f3;  // the 0.5 folded in
#pragma unroll
  for (int d = 0; d < 3; d++) {
    float v = fmaf(0.5f * kx, x[d], fmaf(c4a, Sx[d], c4b * Vx[d]));
    v = fmaf(c3, fmaf(4.0f, VSx[d] + SVx[d], fmaf(2.0f * trV, Sx[d], 2.0f * trS * Vx[d])), v);
    g[d] += v;
  }
  const float c1 = fmaf(-7.5f * Wx, f3, fmaf(52.5f * xVx, f4, -7.5f * trV * f3));
  const float c2 = fmaf(1.5f * Wx, f2, fmaf(-7.5f * xVx, f3, 1.5f * trV * f2));
  const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int e = 0; e < 6; e++) {
    const int i = ii[e], j = jj[e];
    float v = fmaf(c1 * x[i], x[j], 1.5f * f2 * fmaf(W[i], x[j], x[i] * W[j]));
    v = fmaf(-15.0f * f3, fmaf(Vx[i], x[j], x[i] * Vx[j]), v);
    v = fmaf(3.0f * f2, V[e], v);
    G[e] = i == j ? v + c2 : v;
  }
}

// ---------------------------------------------------------------------------
// Node tiles staged in shared memory. The walks visit nodes in pre-order, so
// after an opened node the next one is its neighbour in memory, and an
// accepted node with a small subtree skips only a few records. A warp stages
// the opening data (topology, COM, cell) of 32 consecutive nodes at once, one
// node per lane, with cp.async (16 bytes a copy, cached in L2 only), and
// walks from shared memory until the pre-order index leaves the tile. One L2
// round trip then serves every visit inside the tile, where each visit used
// to wait on its own loads. When a visit's successor lies outside the tile,
// the next tile's copy starts before the visit's terms are evaluated and is
// waited for only after them, so the copy overlaps the arithmetic.
constexpr int kTile = 32;
struct NodeTile {
  int4 topo[kTile];
  float4 com[kTile];
  float4 cell[kTile];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Bulk copies (the TMA unit's non-tensor cp.async.bulk, no multicast) into
// shared memory, completed on an mbarrier. The waits are bounded: a copy
// that never completes makes the wait return false, and the caller flags
// the workspace's status word and stops instead of spinning.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Issued by one lane: orders the warp's earlier reads of the destination
// (generic proxy) before the copy's writes (async proxy), arms the barrier
// for `bytes` and starts the copy. dst, src and bytes are multiples of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Starts staging nodes [base, min(base + kTile, end)) into the warp's tile.
// Every lane calls it (warp-uniform) after it has read what it needs from
// the previous tile; stage_wait() completes the copy for all lanes.
__device__ __forceinline__ void stage_tile_async(const NodeRec* __restrict__ nodes, int base, int end,
                                                 NodeTile* tile, int lane) {
  __syncwarp();  // every lane has finished reading the previous tile
  const int k = base + lane;
  if (k < end) {
    const NodeRec* nd = nodes + k;
    cp_async16(&tile->topo[lane], &nd->topo);
    cp_async16(&tile->com[lane], &nd->com);
    cp_async16(&tile->cell[lane], &nd->cell);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();
}

// Per-warp shared state of the linearized quadrupole during one group's walk:
// the queue of accepted nodes waiting for their one-per-group evaluation (one
// node per lane when 32 have gathered), each lane's running sums of a_q and
// J over the nodes it evaluated, and the group's constants.
struct LinQueue {
  int node[32];
  float acc[9][32];  // [a_q (3), J (6)][lane]
  float grp[16];     // c (3), r_g^2, W (3), V (6)
};

// Group centre and squared half diagonal, IEEE operations in the oracle's
// order (group_centre in oracle/sbh_oracle.c), so both take the same
// linearization decisions.
__device__ __forceinline__ void lq_group_centre(const float* gmin, const float* gmax, float* c4) {
  float hd[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    c4[d] = __fmul_rn(0.5f, __fadd_rn(gmin[d], gmax[d]));
    hd[d] = __fmul_rn(0.5f, __fsub_rn(gmax[d], gmin[d]));
  }
  c4[3] = __fadd_rn(__fadd_rn(__fmul_rn(hd[0], hd[0]), __fmul_rn(hd[1], hd[1])), __fmul_rn(hd[2], hd[2]));
}

// Whether an accepted quadrupole node is linearized (warp-uniform).
__device__ __forceinline__ bool lq_linear(const float* c4, const float4& cell, float k2) {
  const float dx = __fsub_rn(c4[0], cell.x), dy = __fsub_rn(c4[1], cell.y), dz = __fsub_rn(c4[2], cell.z);
  const float R2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  return c4[3] <= __fmul_rn(k2, R2);
}

// Sum over the warp, result in every lane.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Evaluates the queued nodes, one per lane (lanes < cnt): adds a_q and J to
// the lane's sums and, when node_adj is given, the node's dL/dX and dL/dS.
__device__ __forceinline__ void lq_flush(const NodeRec* __restrict__ nodes, LinQueue* lq, int cnt, float eps2,
                                         float* __restrict__ node_adj, int lane) {
  __syncwarp();
  if (lane < cnt) {
    const int k = lq->node[lane];
    const NodeRec* nd = nodes + k;
    const float4 A = __ldg(&nd->com), Qd = __ldg(&nd->quad), X2 = __ldg(&nd->quad2);
    const float x[3] = {lq->grp[0] - A.x, lq->grp[1] - A.y, lq->grp[2] - A.z};
    const float S[6] = {Qd.x, Qd.y, Qd.z, Qd.w, X2.x, X2.y};
    float a[3], J[6], f[4];
    lq_field(x, S, eps2, a, J, f);
#pragma unroll
    for (int c = 0; c < 3; c++) lq->acc[c][lane] += a[c];
#pragma unroll
    for (int c = 0; c < 6; c++) lq->acc[3 + c][lane] += J[c];
    if (node_adj) {
      float g[3], G[6];
      lq_node_adjoint(x, S, J, f, &lq->grp[4], &lq->grp[7], g, G);
      float* na = node_adj + static_cast<int64_t>(k) * kNodeAdj;
#pragma unroll
      for (int c = 0; c < 3; c++) atomicAdd(&na[c], -g[c]);
#pragma unroll
      for (int c = 0; c < 6; c++) atomicAdd(&na[4 + c], G[c]);
    }
  }
  __syncwarp();
}

// The walks are compiled three times: four targets per lane (groups of up
// to 128), three (up to 96) and two (up to 64), each for the occupancy that
// suits it. Measured on a
// B200 over 8 x 2^20 Plummer particles at quadrupole radius 1.6, the adjoint
// walk takes 410 ms with two targets per lane at 7 blocks per SM (72
// registers) and 389 ms with three at 6 blocks (80 registers); 4 per lane at
// 4 blocks takes 411 ms. The adjoint walk's packed form (two slots per FP32
// instruction) then brought three per lane to 367 ms at 5 blocks (96
// registers), against 374 ms for the scalar form at 6 blocks and 397 ms at 5;
// packed at 4 blocks it takes 403 ms. Two per lane packed stays best at 7
// blocks (the 2^21 lattice walk: 33.9 ms, 34.8 at 6, 36.9 at 5; scalar 36.9
// at 7). Four per lane packed (two full pairs, groups of 128) at 4 blocks
// (128 registers) takes 356 ms; its force walk at 5 blocks (102 registers)
// builds + forces one 2^20 Plummer system in 22.7 ms (23.2 at 4 blocks, 24.1
// with groups of 96). Clustered systems gain from the
// larger groups;
// near-uniform ones and walks bounded by a prune radius gain from smaller
// groups (a 2^21 lattice trajectory: 3.76 s with groups of 64, 4.46 s with
// 96), which the two-slot kernels serve. A tree walks with the kernels of its
// current group size (sbh_native_set_group_size).
namespace tpl2 {
constexpr int kTPL = 2;
constexpr int kForceWalkMinBlocks = 7;
constexpr int kAdjointWalkMinBlocks = 7;
#define SBH_NT_WITH_WN_WALK  // the winding-number walk (groups of 32 queries) only here
#include "sbh_native_walks.inc"
#undef SBH_NT_WITH_WN_WALK
}  // namespace tpl2

namespace tpl3 {
constexpr int kTPL = 3;
constexpr int kForceWalkMinBlocks = 6;
constexpr int kAdjointWalkMinBlocks = 5;
#include "sbh_native_walks.inc"
}  // namespace tpl3

namespace tpl4 {
constexpr int kTPL = 4;
constexpr int kForceWalkMinBlocks = 5;
constexpr int kAdjointWalkMinBlocks = 4;
#include "sbh_native_walks.inc"
}  // namespace tpl4

// One of the five variants (quadrupole; periodic and/or cutoff) of a walk
// kernel of namespace NS.
#define SBH_NT_SELECT(NS, KERNEL, QUADV, PERV, CUTV)                                          \
  ((QUADV)  ? NS::KERNEL<true, false, false>                                                  \
   : (PERV) ? ((CUTV) ? NS::KERNEL<false, true, true> : NS::KERNEL<false, false, true>)       \
            : ((CUTV) ? NS::KERNEL<false, true, false> : NS::KERNEL<false, false, false>))

#include "sbh_native_stochastic.inc"

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

// Winding-number node adjoints -> difference arrays over each node's
// particle range: dL/dX / M (3), (dL/dX . Xc) / M (1), dL/dN (3), with Xc the
// COM relative to the system's box centre (single-system trees).
__global__ void wn_node_push_kernel(const NodeRec* __restrict__ nodes, const uint32_t* __restrict__ nn_ptr,
                                    const float* __restrict__ node_adj, const SegBox* __restrict__ boxes,
                                    DVec<14>* __restrict__ D) {
  const uint32_t nn = *nn_ptr;
  const SegBox b = boxes[0];
  const double half = 0.5 * static_cast<double>(b.span);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const float* a = node_adj + static_cast<int64_t>(k) * kNodeAdj;
    bool any = false;
    for (int c = 0; c < 7; c++) any |= a[c] != 0.0f;
    if (!any) continue;
    const NodeRec r = nodes[k];
    const double M = r.com.w;
    if (M == 0.0) continue;
    const double X[3] = {static_cast<double>(r.com.x) - (static_cast<double>(b.lo[0]) + half),
                         static_cast<double>(r.com.y) - (static_cast<double>(b.lo[1]) + half),
                         static_cast<double>(r.com.z) - (static_cast<double>(b.lo[2]) + half)};
    double val[7];
    for (int c = 0; c < 3; c++) val[c] = a[c] / M;
    val[3] = (a[0] * X[0] + a[1] * X[1] + a[2] * X[2]) / M;
    for (int c = 0; c < 3; c++) val[4 + c] = a[4 + c];
    for (int c = 0; c < 7; c++) {
      atomicAdd(&D[r.topo.x].v[c], val[c]);
      atomicAdd(&D[r.topo.y].v[c], -val[c]);
    }
  }
}

// Per sorted source: the direct terms plus the node terms through
// X = sum m p / M and sum m n (inclusive prefix of D = exclusive prefix at i + 1),
// written in input order.
__global__ void wn_combine_kernel(const float4* __restrict__ sp, const float4* __restrict__ sn,
                                  const uint32_t* __restrict__ perm, const SegBox* __restrict__ boxes, int64_t n,
                                  const float* __restrict__ part_adj, const float* __restrict__ part_dn,
                                  const DVec<14>* __restrict__ C, float* __restrict__ dp, float* __restrict__ dn,
                                  float* __restrict__ dm) {
  const SegBox b = boxes[0];
  const double half = 0.5 * static_cast<double>(b.span);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float4 p = sp[i], nr = sn[i];
    const double x[3] = {static_cast<double>(p.x) - (static_cast<double>(b.lo[0]) + half),
                         static_cast<double>(p.y) - (static_cast<double>(b.lo[1]) + half),
                         static_cast<double>(p.z) - (static_cast<double>(b.lo[2]) + half)};
    const DVec<14>& c = C[i + 1];
    const double m = p.w;
    const uint32_t o = perm[i];
    const double nn3[3] = {nr.x, nr.y, nr.z};
    for (int d = 0; d < 3; d++) {
      dp[3 * static_cast<int64_t>(o) + d] =
          static_cast<float>(static_cast<double>(part_adj[kPartAdj * i + d]) + m * c.v[d]);
      dn[3 * static_cast<int64_t>(o) + d] = static_cast<float>(static_cast<double>(part_dn[3 * i + d]) + m * c.v[4 + d]);
    }
    const double q = x[0] * c.v[0] + x[1] * c.v[1] + x[2] * c.v[2] - c.v[3] + nn3[0] * c.v[4] + nn3[1] * c.v[5] +
                     nn3[2] * c.v[6];
    dm[o] = static_cast<float>(static_cast<double>(part_adj[kPartAdj * i + 3]) + q);
  }
}

// The query-side gradient of the last adjoint walk (sorted order) in input order.
__global__ void query_side_kernel(const uint32_t* __restrict__ perm, int64_t n, const float* __restrict__ gq,
                                  float* __restrict__ out) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint32_t o = perm[i];
    for (int d = 0; d < 3; d++) out[3 * static_cast<int64_t>(o) + d] = gq[3 * i + d];
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
  uint32_t* gbins;  // per-level group tallies, then cursors (group_nodes_kernel)
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
  L.gbins = c.template take<uint32_t>(kGroupBins);
  L.counters = c.template take<unsigned long long>(kCounters);
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
  int32_t group_size = kGroup;         // most targets per group (selects the walk kernels)
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

// Host registry: which tree (sizes, group size, target range) a workspace
// holds, keyed by the workspace's address, so evaluation calls recover the
// workspace layout without reading device memory. An entry lives until
// sbh_native_release(workspace) or the next build on the same address.
std::mutex g_reg_mu;
std::unordered_map<const void*, Header> g_registry;

// Target groups of at most G targets, deepest cells first (group_nodes_kernel).
cudaError_t cut_groups(cudaStream_t stream, const Layout& L, int64_t n, int nseg, int G, uint32_t* status) {
  cudaError_t e = cudaMemsetAsync(L.gbins, 0, kGroupBins * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  const unsigned grid = gs(static_cast<int64_t>(L.cap));
  const uint32_t* sseg = nseg > 1 ? L.sseg : nullptr;
  group_nodes_kernel<true><<<grid, 256, 0, stream>>>(L.nodes, L.meta, sseg, L.groups, n + nseg + 1, G, L.gbins,
                                                     status);
  group_bins_kernel<<<1, 32, 0, stream>>>(L.gbins, L.meta + 1);
  group_nodes_kernel<false><<<grid, 256, 0, stream>>>(L.nodes, L.meta, sseg, L.groups, n + nseg + 1, G, L.gbins,
                                                      status);
  return cudaGetLastError();
}

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

int sbh_native_release(const void* workspace) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  g_registry.erase(workspace);
  return SBH_OK;
}

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
  // the node records are read with 16-byte vector loads and bulk copies
  if (reinterpret_cast<uintptr_t>(workspace) % 16 != 0) return invalid("workspace must be 16-byte aligned");
  size_t need = sbh_native_workspace_bytes(n, num_systems, leaf_size, normals != nullptr, with_adjoint);
  if (workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Header h{kMagic, n, num_systems, leaf_size, normals != nullptr, with_adjoint != 0};
  Layout L;
  if (int rc = native_layout(workspace, workspace_bytes, h, L)) return rc;
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, 64, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(L.meta, 0, 8 * sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(L.counters, 0, kCounters * sizeof(unsigned long long), stream);
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
  if (n > 0) {
    cudaError_t ge = cut_groups(stream, L, n, nseg, kGroup, status);
    if (ge != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(ge));
  }
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
  if (!(p->quadrupole_linear >= 0.0f)) return invalid("quadrupole_linear must be >= 0");
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
                    static_cast<float>(1.0 / (2.0 * 1.7724538509055160 * c * c * c)),
                    p->quadrupole && p->quadrupole_linear > 0.0f ? p->quadrupole_linear * p->quadrupole_linear
                                                                  : 0.0f};
}

// Recounts the interactions of the last force or adjoint walk (same tree,
// parameters and target range) into the counters, once per walk.
int refresh_counts(cudaStream_t stream, const void* ws, const Header& h, const Layout& L) {
  if (h.last_walk != 1 || h.counts_fresh) return SBH_OK;
  cudaError_t e = cudaMemsetAsync(L.counters, 0, kCounters * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  const sbh_native_params& p = h.last_params;
  Header hr = h;
  hr.tbeg = h.last_tbeg;
  hr.tend = h.last_tend;
  WalkParams wp = walk_params(&p);
  bool cut = p.cutoff > 0.0f;
  bool per = p.periodic != 0;
  auto k = h.group_size > kGroupThreeSlots ? SBH_NT_SELECT(tpl4, count_walk_kernel, p.quadrupole, per, cut)
           : h.group_size > kGroupTwoSlots ? SBH_NT_SELECT(tpl3, count_walk_kernel, p.quadrupole, per, cut)
                                           : SBH_NT_SELECT(tpl2, count_walk_kernel, p.quadrupole, per, cut);
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
  // the stats keep describing the last walk: count it on its own groups first
  if (int rc = refresh_counts(stream, workspace, h, L)) return rc;
  cudaError_t e = cut_groups(stream, L, h.n, h.nseg, group_size, static_cast<uint32_t*>(workspace));
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    auto it = g_registry.find(workspace);
    if (it != g_registry.end()) it->second.group_size = group_size;
  }
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
  auto k = h.group_size > kGroupThreeSlots ? SBH_NT_SELECT(tpl4, force_walk_kernel, params->quadrupole, per, cut)
           : h.group_size > kGroupTwoSlots ? SBH_NT_SELECT(tpl3, force_walk_kernel, params->quadrupole, per, cut)
                                           : SBH_NT_SELECT(tpl2, force_walk_kernel, params->quadrupole, per, cut);
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
  auto k = h.group_size > kGroupThreeSlots ? SBH_NT_SELECT(tpl4, adjoint_walk_kernel, params->quadrupole, per, cut)
           : h.group_size > kGroupTwoSlots ? SBH_NT_SELECT(tpl3, adjoint_walk_kernel, params->quadrupole, per, cut)
                                           : SBH_NT_SELECT(tpl2, adjoint_walk_kernel, params->quadrupole, per, cut);
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

int sbh_native_adjoint_query_side(cudaStream_t stream, float* grad_points, void* workspace,
                                  size_t workspace_bytes) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.adjoint) return invalid("the tree was built without adjoint scratch (with_adjoint = 0)");
  if (h.n == 0) return SBH_OK;
  if (!grad_points) return invalid("grad_points must be non-null");
  query_side_kernel<<<gs(h.n), 256, 0, stream>>>(L.v0, h.n, L.gq, grad_points);
  return check_launch("sbh_native_adjoint_query_side");
}

int sbh_native_force_vjp(cudaStream_t stream, const sbh_native_params* params, const float* cotangent,
                         float* force_out, float* grad_points, float* grad_masses, void* workspace,
                         size_t workspace_bytes) {
  if (!grad_points || !grad_masses) return invalid("gradient outputs must be non-null");
  if (int rc = sbh_native_adjoint_walk(stream, params, cotangent, force_out, workspace, workspace_bytes)) return rc;
  return sbh_native_adjoint_finalize(stream, grad_points, grad_masses, workspace, workspace_bytes);
}

int sbh_native_stochastic_force(cudaStream_t stream, const sbh_native_params* params, float beta_coarse,
                                int samples, uint64_t seed, float* force_out, void* workspace,
                                size_t workspace_bytes) {
  if (int rc = check_params(params)) return rc;
  if (params->cutoff > 0.0f || params->periodic || params->prune_radius > 0.0f)
    return invalid("the stochastic estimator serves Plummer-softened free-space gravity (no cutoff, periodic box "
                   "or prune radius)");
  if (!(beta_coarse > 0.0f) || beta_coarse > params->beta) return invalid("beta_coarse must be in (0, beta]");
  if (samples < 1 || samples > kStochMaxSamples)
    return invalid("samples must be in [1, " + std::to_string(kStochMaxSamples) + "]");
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (h.n == 0) return SBH_OK;
  if (!force_out) return invalid("force_out must be non-null");
  if (partial_range(h)) return invalid("the stochastic estimator needs the full target range");
  const WalkParams wp = walk_params(params);
  uint32_t* status = static_cast<uint32_t*>(workspace);  // SBH_DEV_ITER_LIMIT if a tile copy never completes
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e == cudaSuccess)
    e = launch_walk(stream, L.work, h.n + h.nseg, stoch_group_kernel, tree_view(L), self_targets(L, h), beta_coarse,
                    params->beta, wp.eps2, samples, seed, force_out, status);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 0, nullptr);
  return check_launch("sbh_native_stochastic_force");
}

int sbh_native_stochastic_force_vjp(cudaStream_t stream, const sbh_native_params* params, float beta_coarse,
                                    int samples, uint64_t seed, const float* cotangent, float* force_out,
                                    float* grad_points, float* grad_masses, void* workspace,
                                    size_t workspace_bytes) {
  if (int rc = check_params(params)) return rc;
  if (params->cutoff > 0.0f || params->periodic || params->prune_radius > 0.0f)
    return invalid("the stochastic estimator serves Plummer-softened free-space gravity (no cutoff, periodic box "
                   "or prune radius)");
  if (!(beta_coarse > 0.0f) || beta_coarse > params->beta) return invalid("beta_coarse must be in (0, beta]");
  if (samples < 1 || samples > kStochMaxSamples)
    return invalid("samples must be in [1, " + std::to_string(kStochMaxSamples) + "]");
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.adjoint) return invalid("the tree was built without adjoint scratch (with_adjoint = 0)");
  if (h.n == 0) return SBH_OK;
  if (!cotangent) return invalid("cotangent must be non-null");
  if (!grad_points || !grad_masses) return invalid("gradient outputs must be non-null");
  if (partial_range(h)) return invalid("the stochastic estimator needs the full target range");
  if (force_out) {  // the estimate itself: the same draws
    if (int rc = sbh_native_stochastic_force(stream, params, beta_coarse, samples, seed, force_out, workspace,
                                             workspace_bytes))
      return rc;
  }
  cudaError_t e = cudaMemsetAsync(L.part_adj, 0, h.n * kPartAdj * sizeof(float), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  zero_node_adj_kernel<<<gs(L.cap * kNodeAdj), 256, 0, stream>>>(L.node_adj, L.meta);
  const WalkParams wp = walk_params(params);
  uint32_t* status = static_cast<uint32_t*>(workspace);
  if (!force_out) e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);  // else the forward cleared it
  if (e == cudaSuccess)
    e = launch_walk(stream, L.work, h.n + h.nseg, stoch_adjoint_kernel, tree_view(L), self_targets(L, h),
                    beta_coarse, params->beta, wp.eps2, samples, seed, cotangent, L.gq, L.node_adj, L.part_adj,
                    status);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 0, nullptr);
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
  e = cudaMemsetAsync(L.counters, 0, kCounters * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  WalkTargets G{tp, qperm, groups, qmeta, 0, qmeta + 2, static_cast<uint32_t>(nq / kQueryGroup + 1), 0, INT64_MAX};
  e = launch_walk(stream, qmeta + 2, nq / kQueryGroup + 1, tpl2::wn_walk_kernel, tree_view(L), G, beta, out,
                  L.counters);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  remember_walk(workspace, 2, nullptr);
  return check_launch("sbh_native_winding_number");
}

int sbh_native_winding_number_vjp(cudaStream_t stream, float beta, const float* queries, int64_t nq,
                                  const float* cotangent, float* out, float* grad_queries, float* grad_points,
                                  float* grad_normals, float* grad_masses, void* workspace, size_t workspace_bytes,
                                  void* query_workspace, size_t query_workspace_bytes) {
  if (!(beta > 0.0f)) return invalid("beta must be > 0");
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!h.normals) return invalid("the tree was built without normals");
  if (!h.adjoint) return invalid("the tree was built without adjoint scratch (with_adjoint = 0)");
  if (h.nseg != 1) return invalid("query evaluation needs a single-system tree");
  if (nq < 0 || nq >= (1ll << 31)) return invalid("number of queries must be in [0, 2^31)");
  if (h.n > 0 && (!grad_points || !grad_normals || !grad_masses))
    return invalid("grad_points, grad_normals and grad_masses must be non-null");
  if (nq > 0 && (!queries || !cotangent || !grad_queries))
    return invalid("queries, cotangent and grad_queries must be non-null");
  size_t need = sbh_native_query_workspace_bytes(nq);
  if (nq > 0 && (!query_workspace || query_workspace_bytes < need))
    return fail(SBH_ERR_WORKSPACE, "query workspace too small: need " + std::to_string(need) + " bytes");
  const int64_t n = h.n;
  cudaError_t e = cudaSuccess;
  if (n > 0) {
    e = cudaMemsetAsync(L.part_adj, 0, n * kPartAdj * sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.gq, 0, n * 3 * sizeof(float), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.D, 0, (n + 1) * sizeof(DVec<14>), stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    zero_node_adj_kernel<<<gs(L.cap * kNodeAdj), 256, 0, stream>>>(L.node_adj, L.meta);
  }
  if (nq > 0 && n == 0) {
    e = cudaMemsetAsync(grad_queries, 0, nq * 3 * sizeof(float), stream);
    if (e == cudaSuccess && out) e = cudaMemsetAsync(out, 0, nq * sizeof(float), stream);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  }
  if (nq > 0 && n > 0) {
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
    e = radix_sort<uint64_t>(stream, k0, v0, k1, v1, nq, 63, false, hist, stmp, &which);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    const uint32_t* qperm = which == 0 ? v0 : v1;
    query_gather_kernel<<<gs(nq), 256, 0, stream>>>(queries, qperm, nq, tp, groups, qmeta);
    WalkTargets G{tp, qperm, groups, qmeta, 0, qmeta + 2, static_cast<uint32_t>(nq / kQueryGroup + 1), 0, INT64_MAX};
    e = launch_walk(stream, qmeta + 2, nq / kQueryGroup + 1, tpl2::wn_adjoint_walk_kernel, tree_view(L), G, beta,
                    cotangent, out, grad_queries, L.node_adj, L.part_adj, L.gq);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  }
  if (n > 0) {
    wn_node_push_kernel<<<gs(L.cap), 256, 0, stream>>>(L.nodes, L.meta, L.node_adj, L.boxes, L.D);
    e = exclusive_scan<DVec<14>>(stream, ArrayLoad<DVec<14>>{L.D}, n + 1, L.D, L.dtmp, false);
    if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
    wn_combine_kernel<<<gs(n), 256, 0, stream>>>(L.sp, L.sn, L.v0, L.boxes, n, L.part_adj, L.gq, L.D, grad_points,
                                                 grad_normals, grad_masses);
  }
  remember_walk(workspace, 2, nullptr);
  return check_launch("sbh_native_winding_number_vjp");
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
  unsigned long long c[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(c, L.counters + 2, sizeof(c), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  *far_quadrupole = c[0] + c[1];
  return SBH_OK;
}

int sbh_native_far_counts(cudaStream_t stream, const void* workspace, size_t workspace_bytes, uint64_t* out3) {
  Header h;
  Layout L;
  if (int rc = lookup(workspace, workspace_bytes, h, L)) return rc;
  if (!out3) return invalid("out3 must be non-null");
  if (int rc = refresh_counts(stream, workspace, h, L)) return rc;
  unsigned long long c[3] = {0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(c, L.counters + 2, sizeof(c), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  for (int i = 0; i < 3; i++) out3[i] = c[i];
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
