// Device-wide primitives written for this library: exclusive scans (u32,
// double and small double vectors) and a stable LSD radix sort of u32/u64
// keys with u32 payloads. All of them are deterministic (no floating-point
// atomics; fixed reduction trees), allocate nothing (temporaries come from
// the caller's workspace) and launch a fixed number of kernels, so they can
// be captured in CUDA graphs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace sbh {

constexpr int kScanThreads = 256;

// Items per thread: 8 for 4-8 byte elements, fewer for the FP64 moment
// vectors so a tile stays in registers without spilling.
template <typename T>
struct ScanCfg {
  static constexpr int kItems = sizeof(T) <= 8 ? 8 : (sizeof(T) <= 32 ? 4 : 2);
  static constexpr int kTile = kScanThreads * kItems;
};

// K doubles summed component-wise.
template <int K>
struct DVec {
  double v[K];
  __host__ __device__ DVec() {
    for (int i = 0; i < K; i++) v[i] = 0.0;
  }
  __host__ __device__ DVec operator+(const DVec& o) const {
    DVec r;
    for (int i = 0; i < K; i++) r.v[i] = v[i] + o.v[i];
    return r;
  }
};

__device__ __forceinline__ uint32_t shfl_up_t(uint32_t x, int d) {
  return __shfl_up_sync(0xffffffffu, x, d);
}
__device__ __forceinline__ uint64_t shfl_up_t(uint64_t x, int d) {
  return __shfl_up_sync(0xffffffffu, x, d);
}
__device__ __forceinline__ double shfl_up_t(double x, int d) {
  return __shfl_up_sync(0xffffffffu, x, d);
}
template <int K>
__device__ __forceinline__ DVec<K> shfl_up_t(const DVec<K>& x, int d) {
  DVec<K> r;
  for (int i = 0; i < K; i++) r.v[i] = __shfl_up_sync(0xffffffffu, x.v[i], d);
  return r;
}

template <typename T>
__device__ __forceinline__ T zero_t() {
  return T();
}
template <>
__device__ __forceinline__ uint32_t zero_t<uint32_t>() {
  return 0u;
}
template <>
__device__ __forceinline__ uint64_t zero_t<uint64_t>() {
  return 0ull;
}
template <>
__device__ __forceinline__ double zero_t<double>() {
  return 0.0;
}

// Inclusive warp scan.
template <typename T>
__device__ __forceinline__ T warp_inclusive(T x) {
  int lane = threadIdx.x & 31;
  for (int d = 1; d < 32; d <<= 1) {
    T y = shfl_up_t(x, d);
    if (lane >= d) x = x + y;
  }
  return x;
}

// Exclusive block scan of one value per thread; returns the exclusive prefix
// and writes the block total to *total. blockDim.x == kScanThreads.
template <typename T>
__device__ T block_exclusive(T x, T* total) {
  __shared__ T warp_tot[kScanThreads / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = warp_inclusive(x);
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < kScanThreads / 32 ? warp_tot[lane] : zero_t<T>();
    T wi = warp_inclusive(w);
    if (lane < kScanThreads / 32) warp_tot[lane] = wi;
  }
  __syncthreads();
  T base = warp == 0 ? zero_t<T>() : warp_tot[warp - 1];
  T t = warp_tot[kScanThreads / 32 - 1];
  __syncthreads();
  if (total) *total = t;
  // exclusive = inclusive - x, computed as base + (inc - x) without subtraction:
  T prev = shfl_up_t(inc, 1);
  if (lane == 0) prev = zero_t<T>();
  return base + prev;
}

// Phase 1: per-tile totals.
template <typename T, typename Load>
__global__ void __launch_bounds__(kScanThreads) scan_tile_totals(Load load, int64_t n, T* tile_tot) {
  constexpr int kItems = ScanCfg<T>::kItems;
  int64_t tile0 = static_cast<int64_t>(blockIdx.x) * ScanCfg<T>::kTile;
  T acc = zero_t<T>();
  for (int k = 0; k < kItems; k++) {
    int64_t i = tile0 + static_cast<int64_t>(threadIdx.x) * kItems + k;
    if (i < n) acc = acc + load(i);
  }
  T tot;
  block_exclusive(acc, &tot);
  if (threadIdx.x == 0) tile_tot[blockIdx.x] = tot;
}

// Phase 2: exclusive scan of the tile totals in one block (any count).
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_tile_offsets(T* tile_tot, int64_t ntiles) {
  __shared__ T carry_s;
  if (threadIdx.x == 0) carry_s = zero_t<T>();
  __syncthreads();
  for (int64_t c0 = 0; c0 < ntiles; c0 += kScanThreads) {
    int64_t i = c0 + threadIdx.x;
    T x = i < ntiles ? tile_tot[i] : zero_t<T>();
    T tot;
    T ex = block_exclusive(x, &tot);
    T carry = carry_s;
    if (i < ntiles) tile_tot[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + tot;
    __syncthreads();
  }
}

// Phase 3: exclusive scan within tiles plus the tile offset; out[n] = total
// when write_total.
template <typename T, typename Load>
__global__ void __launch_bounds__(kScanThreads) scan_tile_apply(Load load, int64_t n,
                                                               const T* tile_off, T* out,
                                                               int write_total, T* total_out) {
  constexpr int kItems = ScanCfg<T>::kItems;
  int64_t tile0 = static_cast<int64_t>(blockIdx.x) * ScanCfg<T>::kTile;
  T items[kItems];
  T acc = zero_t<T>();
  for (int k = 0; k < kItems; k++) {
    int64_t i = tile0 + static_cast<int64_t>(threadIdx.x) * kItems + k;
    items[k] = i < n ? load(i) : zero_t<T>();
    acc = acc + items[k];
  }
  T tot;
  T run = tile_off[blockIdx.x] + block_exclusive(acc, &tot);
  for (int k = 0; k < kItems; k++) {
    int64_t i = tile0 + static_cast<int64_t>(threadIdx.x) * kItems + k;
    if (i < n) out[i] = run;
    run = run + items[k];
  }
  if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) {
    T t = tile_off[blockIdx.x] + tot;
    if (total_out) *total_out = t;
    out[n] = t;
  }
}

// Number of tiles (= temporaries of type T) of a scan over n elements of T.
template <typename T = uint32_t>
inline int64_t scan_tiles(int64_t n) {
  return n <= 0 ? 1 : (n + ScanCfg<T>::kTile - 1) / ScanCfg<T>::kTile;
}

// Exclusive scan of load(0..n-1) into out[0..n-1] (and out[n] = total when
// write_total). tmp: scan_tiles<T>(n) elements of T.
template <typename T, typename Load>
cudaError_t exclusive_scan(cudaStream_t s, Load load, int64_t n, T* out, T* tmp,
                           bool write_total) {
  int64_t nt = scan_tiles<T>(n);
  scan_tile_totals<T, Load><<<static_cast<unsigned>(nt), kScanThreads, 0, s>>>(load, n, tmp);
  scan_tile_offsets<T><<<1, kScanThreads, 0, s>>>(tmp, nt);
  scan_tile_apply<T, Load><<<static_cast<unsigned>(nt), kScanThreads, 0, s>>>(
      load, n, tmp, out, write_total ? 1 : 0, static_cast<T*>(nullptr));
  return cudaGetLastError();
}

template <typename T>
struct ArrayLoad {
  const T* p;
  __device__ T operator()(int64_t i) const { return p[i]; }
};

// --------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits.
// --------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 2048 keys per block

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_count(const K* keys, int64_t n, int shift,
                                                            uint32_t* hist, int64_t nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int64_t t0 = static_cast<int64_t>(blockIdx.x) * kSortTile;
  for (int r = 0; r < kSortRounds; r++) {
    int64_t i = t0 + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[static_cast<uint32_t>(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[static_cast<int64_t>(threadIdx.x) * nblocks + blockIdx.x] = h[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const K* keys_in, const uint32_t* vals_in,
                                                              K* keys_out, uint32_t* vals_out,
                                                              int64_t n, int shift,
                                                              const uint32_t* hist_off,
                                                              int64_t nblocks) {
  __shared__ uint32_t goff[256];
  __shared__ uint32_t wcnt[kSortThreads / 32][256];
  __shared__ uint32_t rtot[256];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  goff[threadIdx.x] = hist_off[static_cast<int64_t>(threadIdx.x) * nblocks + blockIdx.x];
  for (int w = 0; w < kSortThreads / 32; w++) wcnt[w][threadIdx.x] = 0;
  __syncthreads();
  int64_t t0 = static_cast<int64_t>(blockIdx.x) * kSortTile;
  uint32_t lanemask_lt = (1u << lane) - 1u;
  for (int r = 0; r < kSortRounds; r++) {
    int64_t i = t0 + r * kSortThreads + threadIdx.x;
    bool valid = i < n;
    K key = valid ? keys_in[i] : K(0);
    uint32_t d = valid ? (static_cast<uint32_t>(key >> shift) & 255u) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t my = __popc(peers & lanemask_lt);
    if (valid && my == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      uint32_t s = 0;
      for (int w = 0; w < kSortThreads / 32; w++) {
        uint32_t c = wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = s;
        s += c;
      }
      rtot[threadIdx.x] = s;
    }
    __syncthreads();
    if (valid) {
      uint32_t dst = goff[d] + wcnt[warp][d] + my;
      keys_out[dst] = key;
      vals_out[dst] = vals_in ? vals_in[i] : static_cast<uint32_t>(i);
    }
    __syncthreads();
    goff[threadIdx.x] += rtot[threadIdx.x];
    for (int w = 0; w < kSortThreads / 32; w++) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
  }
}

inline int64_t radix_blocks(int64_t n) { return n <= 0 ? 1 : (n + kSortTile - 1) / kSortTile; }

// Workspace elements (u32) for radix_sort's histogram + scan temporaries.
inline int64_t radix_hist_elems(int64_t n) { return 256 * radix_blocks(n); }

// Sorts (keys, vals) stably by the low `bits` bits of the key. vals_in may be
// null (payload = input index). Ping-pongs between (k0, v0) and (k1, v1);
// returns 0 if the sorted data ends in (k0, v0), 1 if in (k1, v1). The input
// must be in k0 (and v0 when given).
template <typename K>
cudaError_t radix_sort(cudaStream_t s, K* k0, uint32_t* v0, K* k1, uint32_t* v1, int64_t n,
                       int bits, bool vals_given, uint32_t* hist, uint32_t* scan_tmp,
                       int* which) {
  int64_t nb = radix_blocks(n);
  int cur = 0;
  bool first = true;
  if (n <= 0) {
    *which = 0;
    return cudaSuccess;
  }
  for (int shift = 0; shift < bits; shift += 8) {
    K* kin = cur == 0 ? k0 : k1;
    uint32_t* vin = cur == 0 ? v0 : v1;
    K* kout = cur == 0 ? k1 : k0;
    uint32_t* vout = cur == 0 ? v1 : v0;
    radix_count<K><<<static_cast<unsigned>(nb), kSortThreads, 0, s>>>(kin, n, shift, hist, nb);
    cudaError_t e = exclusive_scan<uint32_t>(s, ArrayLoad<uint32_t>{hist}, 256 * nb, hist,
                                             scan_tmp, false);
    if (e != cudaSuccess) return e;
    radix_scatter<K><<<static_cast<unsigned>(nb), kSortThreads, 0, s>>>(
        kin, (first && !vals_given) ? nullptr : vin, kout, vout, n, shift, hist, nb);
    first = false;
    cur ^= 1;
  }
  if (first) {
    // zero passes requested: payload = identity
    *which = 0;
    return cudaGetLastError();
  }
  *which = cur;
  return cudaGetLastError();
}

}  // namespace sbh
