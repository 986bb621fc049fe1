// Shared definitions of the sbh_b200 CUDA sources: byte layouts of the
// reference's buffers, the workspace carve-out, error plumbing, and the
// FP32 pair kernels (softened force, its query-side VJP, the un-softened
// gravityGrad, the potential and the signed solid angle).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/sbh_b200.h"

namespace sbh {

// --------------------------------------------------------------------------
// Byte layouts (bhorowitz/barnes-hut include/leaf_data.h, src/sbh_ffi.cu:47-63,
// include/tree3d.h:211-225, include/tree2d.h). They are part of the drop-in
// contract: buffers produced by the reference's builders are read as-is.
// --------------------------------------------------------------------------
struct Leaf3 {
  float pos[3];
  float nrm[3];
  float mass;
  float alpha;
};
static_assert(sizeof(Leaf3) == 32, "Leaf3 must be 32 bytes");

struct Leaf2 {
  float pos[2];
  float nrm[2];
  float mass;
  float alpha;
};
static_assert(sizeof(Leaf2) == 24, "Leaf2 must be 24 bytes");

struct OctreeNode8 {
  uint32_t start, end, parent, first_child;
  uint32_t child[8];
  uint8_t child_mask, depth, is_leaf, pad0;
  float cx, cy, cz, half_size, diameter;
  Leaf3 contrib;
};
static_assert(sizeof(OctreeNode8) == 104, "OctreeNode8 must be 104 bytes");
static_assert(offsetof(OctreeNode8, contrib) == 72, "OctreeNode8 contrib offset");

// Tree3DNode<1,3> / Tree2DNode<1,3>: fields in declaration order with the
// natural alignment the reference's compiler gives them.
template <int N, int BRANCH, int MASK_WORDS, typename LEAF>
struct TreeNodeLayout {
  uint64_t start;
  uint64_t end;
  uint64_t buffer_idx;
  uint64_t parent_idx;
  float bmin[N];
  float bmax[N];
  float diameter;
  LEAF contrib;
  uint64_t mask[MASK_WORDS];
  uint64_t child_idx[BRANCH];
  int32_t num_children;
  int32_t depth;
  int32_t max_depth;
  bool is_leaf;
};
using Node3 = TreeNodeLayout<3, 512, 8, Leaf3>;
using Node2 = TreeNodeLayout<2, 64, 1, Leaf2>;
static_assert(sizeof(Node3) == 4272, "Node3 must match Tree3DNode<1,3> (4272 bytes)");
static_assert(sizeof(Node2) == 616, "Node2 must match Tree2DNode<1,3> (616 bytes)");
static_assert(offsetof(Node3, contrib) == 60, "Node3 contrib offset");
static_assert(offsetof(Node3, mask) == 96, "Node3 mask offset");
static_assert(offsetof(Node3, child_idx) == 160, "Node3 child offset");
static_assert(offsetof(Node3, is_leaf) == 4268, "Node3 is_leaf offset");
static_assert(offsetof(Node2, mask) == 80, "Node2 mask offset");
static_assert(offsetof(Node2, is_leaf) == 612, "Node2 is_leaf offset");

constexpr int kLevel3Split = 8;
constexpr int kLevel3Bins = 512;
constexpr int kLevel3MaxNodes = 513;

// --------------------------------------------------------------------------
// Workspace: [status word | padding to 256 B | carved regions ...]
// --------------------------------------------------------------------------
constexpr size_t kWsAlign = 256;
constexpr size_t kStatusBytes = 256;

inline size_t align_up(size_t x, size_t a = kWsAlign) { return (x + a - 1) / a * a; }

struct Carver {
  char* base;
  size_t off;
  size_t cap;
  bool ok;
  Carver(void* b, size_t c) : base(static_cast<char*>(b)), off(kStatusBytes), cap(c), ok(true) {}
  template <typename T>
  T* take(size_t count) {
    size_t bytes = align_up(count * sizeof(T) + 16);
    if (off + bytes > cap) ok = false;
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return ok ? p : nullptr;
  }
};

// Size-only twin of Carver for *_workspace_bytes().
struct Sizer {
  size_t off = kStatusBytes;
  template <typename T>
  T* take(size_t count) {
    off += align_up(count * sizeof(T) + 16);
    return nullptr;
  }
};

// --------------------------------------------------------------------------
// Host error plumbing
// --------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int check_launch(const char* what);
inline int invalid(const std::string& msg) { return fail(SBH_ERR_INVALID_ARGUMENT, msg); }

// Device status word helpers.
__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bit) {
  if (status) atomicOr(status, bit);
}

// --------------------------------------------------------------------------
// Pair kernels in FP32, written in the reference's operation order
// (src/sbh_ffi.cu:142-160, 431-501, 2044-2090; include/kernel.h:27-94).
// --------------------------------------------------------------------------
struct Periodic {
  int on;
  float box;
};

// minImageDisplacement (include/kernel.h:27-39): floor(x / L + 0.5).
__device__ __forceinline__ float min_image_floor(float d, const Periodic& p) {
  if (p.on && p.box > 0.0f) {
    float inv_l = 1.0f / p.box;
    d = d - p.box * floorf(d * inv_l + 0.5f);
  }
  return d;
}

// Direct-sum minimum image (src/sbh_ffi.cu:437-442): nearbyint(x / L).
__device__ __forceinline__ float min_image_rint(float d, float inv_l, const Periodic& p) {
  if (p.on && p.box > 0.0f) d -= p.box * nearbyintf(d * inv_l);
  return d;
}

// Below this u = r / (2 cutoff) the attenuation erfc(u) + (2/sqrt(pi)) u
// e^{-u^2} = 1 - (4 / (3 sqrt(pi))) u^3 + O(u^5) is within 6e-9 of 1, under
// half an FP32 ulp of 1, so it is taken as 1 without evaluating erfc and exp.
// The reference's "Plummer softening, no cutoff" convention passes a cutoff
// of 1e6 box lengths (python/unified_force_benchmark.py:364-374), which
// puts every pair here.
constexpr float kAttUnityU = 1.0f / 512.0f;

struct Soft {
  float eps;       // max(softening, 0)
  float cutoff;    // <= 0 disables the erfc attenuation
  float unity_r2;  // (2 cutoff kAttUnityU)^2: pairs with r^2 + 1e-12 below it have att = 1
  __host__ __device__ Soft(float e = 0.0f, float c = 0.0f)
      : eps(e), cutoff(c), unity_r2(c > 0.0f ? (2.0f * c * kAttUnityU) * (2.0f * c * kAttUnityU) : 0.0f) {}
};

// coefficient c with f = c * r for the softened force; r = q - p.
__device__ __forceinline__ float soft_coeff(float r2, float mass, const Soft& s) {
  float inv_r = rsqrtf(r2 + s.eps * s.eps + 1e-12f);
  float inv_r3 = inv_r * inv_r * inv_r;
  float att = 1.0f;
  // the square-root and division are only needed outside the att = 1 range
  if (s.cutoff > 0.0f && r2 + 1e-12f >= s.unity_r2) {
    float dist = sqrtf(r2 + 1e-12f);
    float u = dist / (2.0f * s.cutoff);
    if (u >= kAttUnityU) {
      float e = expf(-(u * u));
      att = erfcf(u) + (2.0f / 1.772453850905516f) * u * e;
    }
  }
  return -mass * att * inv_r3;
}

// Query-side VJP of the softened force: acc += -m (lin g - rad r).
__device__ __forceinline__ void soft_vjp_accum(float rx, float ry, float rz, float mass,
                                               float gx, float gy, float gz, const Soft& s,
                                               float& ax, float& ay, float& az) {
  float r2 = rx * rx + ry * ry + rz * rz;
  float inv_r = rsqrtf(r2 + s.eps * s.eps + 1e-12f);
  float inv_r3 = inv_r * inv_r * inv_r;
  float inv_r5 = inv_r3 * inv_r * inv_r;
  float att = 1.0f;
  float cc = 0.0f;
  // below kAttUnityU (r^2 under unity_r2): att = 1, and cc = ir3 r e / (2 sqrt(pi) cutoff^3) is
  // below 1e-4 (r^2 + eps^2) / cutoff^2 of the 3 att ir^5 term it joins, so it is left out
  if (s.cutoff > 0.0f && r2 + 1e-12f >= s.unity_r2) {
    float dist = sqrtf(r2 + 1e-12f);
    float u = dist / (2.0f * s.cutoff);
    float e = 1.0f;
    if (u >= kAttUnityU) {
      e = expf(-(u * u));
      att = erfcf(u) + (2.0f / 1.772453850905516f) * u * e;
    }
    cc = inv_r3 * dist * e / (2.0f * 1.772453850905516f * s.cutoff * s.cutoff * s.cutoff);
  }
  float rg = rx * gx + ry * gy + rz * gz;
  float lin = att * inv_r3;
  float rad = rg * (3.0f * att * inv_r5 + cc);
  ax += -mass * (lin * gx - rad * rx);
  ay += -mass * (lin * gy - rad * ry);
  az += -mass * (lin * gz - rad * rz);
}

// gravityGrad (include/kernel.h:89-94): -m / (|r| + 0.1)^3 * r.
__device__ __forceinline__ float grav_grad_coeff(float r2, float mass) {
  float dist = sqrtf(r2);
  float den = dist + 0.1f;
  return -mass / (den * den * den);
}

// gravityGradVjp (src/sbh_ffi.cu:2044-2060).
__device__ __forceinline__ void grav_grad_vjp_accum(float rx, float ry, float rz, float mass,
                                                    float gx, float gy, float gz, float& ax,
                                                    float& ay, float& az) {
  float r2 = rx * rx + ry * ry + rz * rz;
  float dist = sqrtf(r2 + 1e-12f);
  float den = dist + 0.1f;
  float id3 = 1.0f / (den * den * den);
  float id4 = id3 / den;
  float rg = rx * gx + ry * gy + rz * gz;
  float dinv = 1.0f / (dist + 1e-12f);
  float k = 3.0f * rg * dinv * id4;
  ax += -mass * (id3 * gx - k * rx);
  ay += -mass * (id3 * gy - k * ry);
  az += -mass * (id3 * gz - k * rz);
}

// Kahan-compensated accumulation of a partial sum v into (s, c).
__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  float y = v - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

}  // namespace sbh
