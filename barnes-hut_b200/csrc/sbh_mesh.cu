// Surface sampling of a triangle mesh on the device: the input side of the
// winding-number path when the sources come from a mesh.
//
// The reference samples on the host (python/old_interface/sampler.py:45-78,
// sample_points_on_mesh; python/old_interface/source.py:119-155,
// MeshSurface): a face is chosen with probability area / total area, a
// point uniform in it, and the sample takes the face's unit normal. Here the
// same distribution comes from three launches:
//   1. face_kernel: per face, twice its area and its unit normal (FP64
//      arithmetic from the FP32 vertices, rounded once at the end);
//   2. an FP64 exclusive scan of the doubled areas: the cumulative
//      distribution, its last entry the doubled total area;
//   3. sample_kernel: per sample i, three uniforms from a counter-based
//      generator (outputs 3i+1..3i+3 of splitmix64 seeded with `seed`), the
//      face by binary search of u0 * total in the distribution, and the
//      barycentric pair (u1, u2) reflected into the triangle when
//      u1 + u2 > 1 (the reference rejects and redraws instead; both give the
//      uniform density on the triangle).
// Every sample carries the weight total area / n, the surface measure it
// stands for in the winding-number sum. Results depend only on (seed, i), not
// on the launch shape, so a CPU restatement reproduces them exactly.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "sbh_b200.h"
#include "sbh_common.cuh"
#include "sbh_primitives.cuh"

namespace sbh {
namespace mesh {
namespace {

constexpr int kThreads = 256;

// splitmix64 (S. Vigna, 2015): the output for state x; the generator's k-th
// output from seed s is mix(s + k * 0x9e3779b97f4a7c15).
__device__ __forceinline__ uint64_t splitmix64_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Uniform double in [0, 1) from the top 53 bits.
__device__ __forceinline__ double unit_double(uint64_t z) { return static_cast<double>(z >> 11) * 0x1.0p-53; }

struct Face {
  double e1[3], e2[3], v0[3];
};

__device__ __forceinline__ bool load_face(const float* __restrict__ V, int64_t nv, const int32_t* __restrict__ F,
                                          int64_t f, Face& out) {
  // 64-bit indices: 3 * a overflows int32 for vertex indices past ~7.2e8
  const int64_t a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
  if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) return false;
  for (int d = 0; d < 3; d++) {
    double x0 = V[3 * a + d], x1 = V[3 * b + d], x2 = V[3 * c + d];
    out.v0[d] = x0;
    out.e1[d] = __dsub_rn(x1, x0);
    out.e2[d] = __dsub_rn(x2, x0);
  }
  return true;
}

// Twice the face area (|e1 x e2|, zero for degenerate or NaN faces) and the
// unit normal e1 x e2 / |e1 x e2| (zero when the area is zero).
__global__ void face_kernel(const float* __restrict__ V, int64_t nv, const int32_t* __restrict__ F, int64_t nf,
                            double* __restrict__ area2, float4* __restrict__ normal, uint32_t* status) {
  for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; f < nf;
       f += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    Face t;
    double len = 0.0, c[3] = {0.0, 0.0, 0.0};
    if (load_face(V, nv, F, f, t)) {
      c[0] = __dsub_rn(__dmul_rn(t.e1[1], t.e2[2]), __dmul_rn(t.e1[2], t.e2[1]));
      c[1] = __dsub_rn(__dmul_rn(t.e1[2], t.e2[0]), __dmul_rn(t.e1[0], t.e2[2]));
      c[2] = __dsub_rn(__dmul_rn(t.e1[0], t.e2[1]), __dmul_rn(t.e1[1], t.e2[0]));
      len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(c[0], c[0]), __dmul_rn(c[1], c[1])), __dmul_rn(c[2], c[2])));
      if (!(len > 0.0) || isinf(len)) len = 0.0;
    } else {
      raise_status(status, SBH_DEV_BAD_BOUNDS);
    }
    area2[f] = len;
    float4 nrm = make_float4(0.f, 0.f, 0.f, 0.f);
    if (len > 0.0) {
      nrm.x = __double2float_rn(__ddiv_rn(c[0], len));
      nrm.y = __double2float_rn(__ddiv_rn(c[1], len));
      nrm.z = __double2float_rn(__ddiv_rn(c[2], len));
    }
    normal[f] = nrm;
  }
}

__global__ void sample_kernel(const float* __restrict__ V, int64_t nv, const int32_t* __restrict__ F, int64_t nf,
                              const double* __restrict__ cdf, const float4* __restrict__ normal, int64_t n,
                              uint64_t seed, float* __restrict__ points, float* __restrict__ normals_out,
                              float* __restrict__ weights, uint32_t* status) {
  const double total = cdf[nf];
  const bool ok = total > 0.0 && !isinf(total);
  if (!ok && blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, SBH_DEV_BAD_BOUNDS);
  const float w = ok ? __double2float_rn(__ddiv_rn(__dmul_rn(total, 0.5), static_cast<double>(n))) : 0.0f;
  // largest double below the total: the search target stays inside the last face of positive area
  const double top = ok ? __longlong_as_double(__double_as_longlong(total) - 1) : 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float p[3] = {0.f, 0.f, 0.f};
    float4 nrm = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) {
      const uint64_t base = seed + static_cast<uint64_t>(3 * i + 1) * 0x9e3779b97f4a7c15ull;
      double u0 = unit_double(splitmix64_mix(base));
      double u1 = unit_double(splitmix64_mix(base + 0x9e3779b97f4a7c15ull));
      double u2 = unit_double(splitmix64_mix(base + 2 * 0x9e3779b97f4a7c15ull));
      double target = fmin(__dmul_rn(u0, total), top);
      // first j in [1, nf] with cdf[j] > target; the face is j - 1
      int64_t lo = 1, hi = nf;
      while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > target)
          hi = mid;
        else
          lo = mid + 1;
      }
      const int64_t f = lo - 1;
      if (__dadd_rn(u1, u2) > 1.0) {
        u1 = __dsub_rn(1.0, u1);
        u2 = __dsub_rn(1.0, u2);
      }
      Face t;
      if (load_face(V, nv, F, f, t)) {
        for (int d = 0; d < 3; d++)
          p[d] = __double2float_rn(__dadd_rn(__dadd_rn(t.v0[d], __dmul_rn(u1, t.e1[d])), __dmul_rn(u2, t.e2[d])));
        nrm = normal[f];
      }
    }
    points[3 * i] = p[0];
    points[3 * i + 1] = p[1];
    points[3 * i + 2] = p[2];
    normals_out[3 * i] = nrm.x;
    normals_out[3 * i + 1] = nrm.y;
    normals_out[3 * i + 2] = nrm.z;
    weights[i] = w;
  }
}

unsigned grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return static_cast<unsigned>(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

template <typename C>
void carve(C& c, int64_t nf, double** area2, double** cdf, double** tmp, float4** normal) {
  *area2 = c.template take<double>(static_cast<size_t>(nf));
  *cdf = c.template take<double>(static_cast<size_t>(nf) + 1);
  *tmp = c.template take<double>(static_cast<size_t>(scan_tiles<double>(nf)));
  *normal = c.template take<float4>(static_cast<size_t>(nf));
}

// ---------------------------------------------------------------------------
// Vertex sources (the reference's MeshVertices, python/old_interface/
// source.py:85-115): every vertex is a source, with the area-weighted vertex
// normal of igl.per_vertex_normals(V, F, 1) (the normalised sum of e1 x e2
// over the incident faces) and, as its mass, the diagonal of libigl's
// default (Voronoi) mass matrix: the mixed Voronoi area of Meyer, Desbrun,
// Schroeder and Barr (2003). Per face P0 P1 P2 with cot_i the cotangent of
// the angle at corner i:
//   no obtuse angle: corner i takes (|Pi Pk|^2 cot_j + |Pi Pj|^2 cot_k) / 8;
//   obtuse at corner i: corner i takes area / 2, the other two area / 4.
// The three shares sum to the face's area, so the masses sum to the surface
// area. Faces of zero area add nothing. FP64 throughout; the per-vertex sums
// are FP64 atomics, so the FP32 outputs can differ from a sequential sum in
// the last place.
__global__ void vertex_face_kernel(const float* __restrict__ V, int64_t nv, const int32_t* __restrict__ F,
                                   int64_t nf, double* __restrict__ acc, uint32_t* status) {
  for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; f < nf;
       f += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t id[3] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};  // 64-bit: 3 * id below
    bool ok = true;
    for (int c = 0; c < 3; c++) ok = ok && id[c] >= 0 && id[c] < nv;
    if (!ok) {
      raise_status(status, SBH_DEV_BAD_BOUNDS);
      continue;
    }
    double p[3][3];
    for (int c = 0; c < 3; c++)
      for (int d = 0; d < 3; d++) p[c][d] = V[3 * id[c] + d];
    // e[c]: the edge from corner c to corner c + 1
    double e[3][3];
    for (int c = 0; c < 3; c++)
      for (int d = 0; d < 3; d++) e[c][d] = __dsub_rn(p[(c + 1) % 3][d], p[c][d]);
    double n[3];  // e0 x (P2 - P0) = -(e0 x e2)
    n[0] = __dsub_rn(__dmul_rn(e[2][1], e[0][2]), __dmul_rn(e[2][2], e[0][1]));
    n[1] = __dsub_rn(__dmul_rn(e[2][2], e[0][0]), __dmul_rn(e[2][0], e[0][2]));
    n[2] = __dsub_rn(__dmul_rn(e[2][0], e[0][1]), __dmul_rn(e[2][1], e[0][0]));
    const double dbl = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(n[0], n[0]), __dmul_rn(n[1], n[1])),
                                            __dmul_rn(n[2], n[2])));
    if (!(dbl > 0.0) || isinf(dbl)) continue;  // no area, no share
    const double area = __dmul_rn(dbl, 0.5);
    // squared edge lengths and the corner dot products: corner c sits
    // between e[c] (outgoing) and e[c - 1] (incoming, reversed)
    double l2[3], dot[3];
    for (int c = 0; c < 3; c++) {
      l2[c] = __dadd_rn(__dadd_rn(__dmul_rn(e[c][0], e[c][0]), __dmul_rn(e[c][1], e[c][1])),
                        __dmul_rn(e[c][2], e[c][2]));
      const int b = (c + 2) % 3;
      dot[c] = -__dadd_rn(__dadd_rn(__dmul_rn(e[c][0], e[b][0]), __dmul_rn(e[c][1], e[b][1])),
                          __dmul_rn(e[c][2], e[b][2]));
    }
    double share[3];
    int obtuse = -1;
    for (int c = 0; c < 3; c++)
      if (dot[c] < 0.0) obtuse = c;
    if (obtuse >= 0) {
      for (int c = 0; c < 3; c++) share[c] = c == obtuse ? __dmul_rn(area, 0.5) : __dmul_rn(area, 0.25);
    } else {
      double cot[3];
      for (int c = 0; c < 3; c++) cot[c] = __ddiv_rn(dot[c], dbl);
      // corner c: the edge to c + 1 (l2[c]) faces corner c + 2, the edge to c + 2 (l2[c + 2]) faces c + 1
      for (int c = 0; c < 3; c++)
        share[c] = __dmul_rn(__dadd_rn(__dmul_rn(l2[c], cot[(c + 2) % 3]), __dmul_rn(l2[(c + 2) % 3], cot[(c + 1) % 3])),
                             0.125);
    }
    for (int c = 0; c < 3; c++) {
      double* a = acc + 4 * static_cast<int64_t>(id[c]);
      atomicAdd(a, share[c]);
      atomicAdd(a + 1, n[0]);
      atomicAdd(a + 2, n[1]);
      atomicAdd(a + 3, n[2]);
    }
  }
}

__global__ void vertex_finish_kernel(const double* __restrict__ acc, int64_t nv, float* __restrict__ normals,
                                     float* __restrict__ masses) {
  for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < nv;
       v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double* a = acc + 4 * v;
    const double len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(a[1], a[1]), __dmul_rn(a[2], a[2])),
                                            __dmul_rn(a[3], a[3])));
    const bool unit = len > 0.0 && !isinf(len);
    for (int d = 0; d < 3; d++) normals[3 * v + d] = unit ? __double2float_rn(__ddiv_rn(a[1 + d], len)) : 0.0f;
    masses[v] = __double2float_rn(a[0]);
  }
}

}  // namespace
}  // namespace mesh
}  // namespace sbh

using namespace sbh;

extern "C" {

size_t sbh_mesh_sample_workspace_bytes(int64_t nf) {
  if (nf < 0) return 0;
  Sizer s;
  double *a, *c, *t;
  float4* nrm;
  mesh::carve(s, nf, &a, &c, &t, &nrm);
  return s.off;
}

int sbh_sample_mesh_surface(cudaStream_t stream, const float* vertices, int64_t nv, const int32_t* faces, int64_t nf,
                            int64_t n, uint64_t seed, float* points_out, float* normals_out, float* weights_out,
                            void* workspace, size_t workspace_bytes) {
  if (nv < 0 || nf < 0 || n < 0) return invalid("sizes must be >= 0");
  if (n > 0 && nf == 0) return invalid("the mesh has no faces");
  if (n > 0 && (!vertices || !faces)) return invalid("vertices and faces must be non-null");
  if (n > 0 && (!points_out || !normals_out || !weights_out)) return invalid("outputs must be non-null");
  if (n == 0) return SBH_OK;
  size_t need = sbh_mesh_sample_workspace_bytes(nf);
  if (!workspace || workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes);
  double *area2, *cdf, *tmp;
  float4* normal;
  mesh::carve(c, nf, &area2, &cdf, &tmp, &normal);
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  mesh::face_kernel<<<mesh::grid_for(nf), mesh::kThreads, 0, stream>>>(vertices, nv, faces, nf, area2, normal,
                                                                       status);
  e = exclusive_scan<double>(stream, ArrayLoad<double>{area2}, nf, cdf, tmp, true);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  mesh::sample_kernel<<<mesh::grid_for(n), mesh::kThreads, 0, stream>>>(
      vertices, nv, faces, nf, cdf, normal, n, seed, points_out, normals_out, weights_out, status);
  return check_launch("sample_mesh_surface");
}

size_t sbh_mesh_vertex_workspace_bytes(int64_t nv) {
  if (nv < 0) return 0;
  Sizer s;
  s.take<double>(4 * static_cast<size_t>(nv));
  return s.off;
}

int sbh_mesh_vertex_sources(cudaStream_t stream, const float* vertices, int64_t nv, const int32_t* faces, int64_t nf,
                            float* normals_out, float* masses_out, void* workspace, size_t workspace_bytes) {
  if (nv < 0 || nf < 0) return invalid("sizes must be >= 0");
  if (nv > 0 && (!vertices || !normals_out || !masses_out)) return invalid("vertices and outputs must be non-null");
  if (nf > 0 && !faces) return invalid("faces must be non-null");
  if (nv == 0) return nf == 0 ? SBH_OK : invalid("faces reference vertices of an empty mesh");
  size_t need = sbh_mesh_vertex_workspace_bytes(nv);
  if (!workspace || workspace_bytes < need)
    return fail(SBH_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  Carver c(workspace, workspace_bytes);
  double* acc = c.take<double>(4 * static_cast<size_t>(nv));
  uint32_t* status = static_cast<uint32_t*>(workspace);
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, 4 * sizeof(double) * static_cast<size_t>(nv), stream);
  if (e != cudaSuccess) return fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  if (nf > 0)
    mesh::vertex_face_kernel<<<mesh::grid_for(nf), mesh::kThreads, 0, stream>>>(vertices, nv, faces, nf, acc, status);
  mesh::vertex_finish_kernel<<<mesh::grid_for(nv), mesh::kThreads, 0, stream>>>(acc, nv, normals_out, masses_out);
  return check_launch("mesh_vertex_sources");
}

}  // extern "C"
