// C driver over the REFERENCE's own GPU plugin (bhorowitz/barnes-hut
// src/sbh_ffi.cu), compiled from where it lies by oracle/Makefile with the
// project-written Eigen and XLA-FFI stand-ins in oracle/ref_shim/. With the
// stand-in, XLA_FFI_DEFINE_HANDLER_SYMBOL expands to nothing and every
// reference handler (sbh_ffi::BuildOctree8Buffers, ...) is an ordinary C++
// function; each wrapper below wraps raw device pointers into the stand-in
// buffer types and calls it unchanged on the given stream.
//
// TEST INFRASTRUCTURE ONLY: the GPU parity tests and the golden-fixture
// generator use it as the reference implementation (same inputs -> the
// reference's own outputs, including its curand streams). The product
// library never links it.
#include "sbh_ffi.cu"

#include <cstring>
#include <string>

namespace {

thread_local std::string g_last_error;

using namespace sbh_ffi;

F32R1 f1(const float* p, int64_t n) {
  int64_t d[1] = {n};
  return F32R1(const_cast<float*>(p), d, 1);
}
F32R2 f2(const float* p, int64_t r, int64_t c) {
  int64_t d[2] = {r, c};
  return F32R2(const_cast<float*>(p), d, 2);
}
U8R1 u1(const void* p, int64_t nbytes) {
  int64_t d[1] = {nbytes};
  return U8R1(const_cast<void*>(p), d, 1);
}
F32R1Out f1o(float* p, int64_t n) { return F32R1Out(f1(p, n)); }
F32R2Out f2o(float* p, int64_t r, int64_t c) { return F32R2Out(f2(p, r, c)); }
U8R1Out u1o(void* p, int64_t nbytes) { return U8R1Out(u1(p, nbytes)); }

int ret(const xla::ffi::Error& e) {
  g_last_error = e.message;
  return e.code;
}

cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* ref_gpu_last_error() { return g_last_error.c_str(); }

size_t ref_gpu_leaf3_size() { return sbh_leaf3_size(); }
size_t ref_gpu_node3_size() { return sbh_node3_size(); }
size_t ref_gpu_octree8_node_size() { return sbh_octree8_node_size(); }
size_t ref_gpu_level3_max_nodes() { return sbh_octree_level3_max_nodes(); }

int ref_bruteforce_gravity(void* s, const float* pts, const float* m, int64_t n, int dim,
                           const float* q, int64_t nq, float* out, int periodic,
                           float box, int threads) {
  return ret(BruteForceGravity(S(s), f2(pts, n, dim), f1(m, n), f2(q, nq, dim), f1o(out, nq),
                               periodic, box, threads));
}

int ref_direct_force_soft(void* s, const float* pts, const float* m, int64_t n, const float* q,
                          int64_t nq, float* out, float eps, float cutoff, int periodic,
                          float box, int threads) {
  return ret(SoftenedDirectForce(S(s), f2(pts, n, 3), f1(m, n), f2(q, nq, 3), f2o(out, nq, 3),
                                 eps, cutoff, periodic, box, threads));
}

int ref_direct_force_soft_vjp(void* s, const float* pts, const float* m, int64_t n,
                              const float* q, int64_t nq, const float* cot, float* out,
                              float eps, float cutoff, int periodic, float box, int threads) {
  return ret(SoftenedDirectForceVjp(S(s), f2(pts, n, 3), f1(m, n), f2(q, nq, 3),
                                    f2(cot, nq, 3), f2o(out, nq, 3), eps, cutoff, periodic,
                                    box, threads));
}

int ref_build_octree_level3(void* s, const float* pts, const float* nrm, const float* m,
                            int64_t n, const float* mn, const float* mx, void* leaf,
                            int64_t leaf_bytes, void* node, int64_t node_bytes, void* contrib,
                            int64_t contrib_bytes) {
  return ret(BuildOctreeLevel3Buffers(S(s), f2(pts, n, 3), f2(nrm, n, 3), f1(m, n), f1(mn, 3),
                                      f1(mx, 3), u1o(leaf, leaf_bytes), u1o(node, node_bytes),
                                      u1o(contrib, contrib_bytes)));
}

int ref_build_octree8(void* s, const float* pts, const float* nrm, const float* m, int64_t n,
                      const float* mn, const float* mx, void* leaf, int64_t leaf_bytes,
                      void* node, int64_t node_bytes, void* contrib, int64_t contrib_bytes,
                      int max_depth) {
  return ret(BuildOctree8Buffers(S(s), f2(pts, n, 3), f2(nrm, n, 3), f1(m, n), f1(mn, 3),
                                 f1(mx, 3), u1o(leaf, leaf_bytes), u1o(node, node_bytes),
                                 u1o(contrib, contrib_bytes), max_depth));
}

// dim 2 -> Node2/Leaf2 handlers, dim 3 -> Node3/Leaf3 handlers.
int ref_barnes_hut_gravity(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                           const void* node, int64_t node_bytes, const float* q, int64_t nq,
                           float* out, float beta, int periodic, float box, int threads) {
  if (dim == 2)
    return ret(BarnesHutGravity(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                f2(q, nq, 2), f1o(out, nq), beta, periodic, box, threads));
  return ret(BarnesHutGravity3D(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 3),
                                f1o(out, nq), beta, periodic, box, threads));
}

int ref_barnes_hut_force(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                         const void* node, int64_t node_bytes, const float* q, int64_t nq,
                         float* out, float beta, int periodic, float box, int threads) {
  if (dim == 2)
    return ret(BarnesHutForce(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 2),
                              f2o(out, nq, 2), beta, periodic, box, threads));
  return ret(BarnesHutForce3D(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 3),
                              f2o(out, nq, 3), beta, periodic, box, threads));
}

int ref_barnes_hut_force_soft(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                              const void* node, int64_t node_bytes, const float* q,
                              int64_t nq, float* out, float beta, float eps, float cutoff,
                              int periodic, float box, int threads) {
  if (dim == 2)
    return ret(SoftenedBarnesHutForce(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                      f2(q, nq, 2), f2o(out, nq, 2), beta, eps, cutoff,
                                      periodic, box, threads));
  return ret(SoftenedBarnesHutForce3D(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                      f2(q, nq, 3), f2o(out, nq, 3), beta, eps, cutoff,
                                      periodic, box, threads));
}

int ref_stochastic_bh_gravity(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                              const void* node, int64_t node_bytes, const void* contrib,
                              int64_t contrib_bytes, const float* q, int64_t nq, float* out,
                              int samples, int seed, int periodic, float box, int threads) {
  if (dim == 2)
    return ret(StochasticBarnesHutGravity(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                          u1(contrib, contrib_bytes), f2(q, nq, 2),
                                          f1o(out, nq), samples, seed, periodic, box, threads));
  return ret(StochasticBarnesHutGravity3D(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                          u1(contrib, contrib_bytes), f2(q, nq, 3),
                                          f1o(out, nq), samples, seed, periodic, box, threads));
}

int ref_stochastic_bh_force(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                            const void* node, int64_t node_bytes, const void* contrib,
                            int64_t contrib_bytes, const float* q, int64_t nq, float* out,
                            int samples, int seed, int periodic, float box, int threads) {
  if (dim == 2)
    return ret(StochasticBarnesHutForce(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                        u1(contrib, contrib_bytes), f2(q, nq, 2),
                                        f2o(out, nq, 2), samples, seed, periodic, box, threads));
  return ret(StochasticBarnesHutForce3D(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                        u1(contrib, contrib_bytes), f2(q, nq, 3),
                                        f2o(out, nq, 3), samples, seed, periodic, box, threads));
}

int ref_stochastic_bh_force_soft(void* s, int dim, const void* leaf, int64_t leaf_bytes,
                                 const void* node, int64_t node_bytes, const void* contrib,
                                 int64_t contrib_bytes, const float* q, int64_t nq, float* out,
                                 int samples, int seed, float eps, float cutoff, int periodic,
                                 float box, int threads) {
  if (dim == 2)
    return ret(SoftenedStochasticBarnesHutForce(
        S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), u1(contrib, contrib_bytes),
        f2(q, nq, 2), f2o(out, nq, 2), samples, seed, eps, cutoff, periodic, box, threads));
  return ret(SoftenedStochasticBarnesHutForce3D(
      S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), u1(contrib, contrib_bytes),
      f2(q, nq, 3), f2o(out, nq, 3), samples, seed, eps, cutoff, periodic, box, threads));
}

int ref_bh_force_octree8(void* s, const void* leaf, int64_t leaf_bytes, const void* node,
                         int64_t node_bytes, const float* q, int64_t nq, float* out, float beta,
                         int periodic, float box, int threads) {
  return ret(BarnesHutForceOctree8(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                   f2(q, nq, 3), f2o(out, nq, 3), beta, periodic, box, threads));
}

int ref_bh_force_octree8_soft(void* s, const void* leaf, int64_t leaf_bytes, const void* node,
                              int64_t node_bytes, const float* q, int64_t nq, float* out,
                              float beta, float eps, float cutoff, int prune, float prune_mult,
                              int periodic, float box, int threads) {
  return ret(SoftenedBarnesHutForceOctree8(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                           f2(q, nq, 3), f2o(out, nq, 3), beta, eps, cutoff,
                                           prune, prune_mult, periodic, box, threads));
}

int ref_bh_force_octree8_soft_vjp(void* s, const void* leaf, int64_t leaf_bytes,
                                  const void* node, int64_t node_bytes, const float* q,
                                  int64_t nq, const float* cot, float* out, float beta,
                                  float eps, float cutoff, int prune, float prune_mult,
                                  int periodic, float box, int threads) {
  return ret(SoftenedBarnesHutForceOctree8Vjp(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                              f2(q, nq, 3), f2(cot, nq, 3), f2o(out, nq, 3),
                                              beta, eps, cutoff, prune, prune_mult, periodic,
                                              box, threads));
}

// softened = 0 -> StochasticBarnesHutForceOctree8 (eps/cutoff/prune ignored).
int ref_stochastic_bh_force_octree8(void* s, int softened, const void* leaf,
                                    int64_t leaf_bytes, const void* node, int64_t node_bytes,
                                    const float* q, int64_t nq, float* out, int samples,
                                    int seed, float beta, float eps, float cutoff, int prune,
                                    float prune_mult, int periodic, float box, int threads) {
  if (!softened)
    return ret(StochasticBarnesHutForceOctree8(S(s), u1(leaf, leaf_bytes), u1(node, node_bytes),
                                               f2(q, nq, 3), f2o(out, nq, 3), samples, seed,
                                               beta, periodic, box, threads));
  return ret(SoftenedStochasticBarnesHutForceOctree8(
      S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 3), f2o(out, nq, 3), samples,
      seed, beta, eps, cutoff, prune, prune_mult, periodic, box, threads));
}

int ref_stochastic_bh_force_octree8_vjp(void* s, int softened, const void* leaf,
                                        int64_t leaf_bytes, const void* node,
                                        int64_t node_bytes, const float* q, int64_t nq,
                                        const float* cot, float* out, int samples, int seed,
                                        float beta, float eps, float cutoff, int prune,
                                        float prune_mult, int periodic, float box,
                                        int threads) {
  if (!softened)
    return ret(StochasticBarnesHutForceOctree8Vjp(
        S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 3), f2(cot, nq, 3),
        f2o(out, nq, 3), samples, seed, beta, periodic, box, threads));
  return ret(SoftenedStochasticBarnesHutForceOctree8Vjp(
      S(s), u1(leaf, leaf_bytes), u1(node, node_bytes), f2(q, nq, 3), f2(cot, nq, 3),
      f2o(out, nq, 3), samples, seed, beta, eps, cutoff, prune, prune_mult, periodic, box,
      threads));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The reference's pybind module sbh_gpu (src/sbh_gpu.cu:36-208) evaluates the
// scalar kernels (gravityPotential, signedSolidAngle, smoothDistExp) by brute
// force, warp-vote BH and MLPCV with seed 0, 32 threads per block. These
// test-only kernels call the same reference templates on Node2/Node3
// buffers so that the parity tests can compare against them.
// ---------------------------------------------------------------------------
#include "brute_force_gpu.h"

namespace {

template <typename TREE>
__global__ void ref_vote_scalar(const LeafData<TREE::N>* leaf, const TREE* nodes, const float* q, int nq,
                                float beta, int kind, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  VectorNd<TREE::N> p;
  for (int d = 0; d < TREE::N; d++) p(d) = q[TREE::N * i + d];
  if (kind == 0)
    out[i] = evaluateBarnesHutGPUVote<FLOAT>(leaf, nodes, nodes, p, beta, gravityPotential<TREE::N>);
  else if (kind == 3)
    out[i] = evaluateBarnesHutGPUVote<FLOAT>(leaf, nodes, nodes, p, beta, signedSolidAngle<TREE::N>);
  else
    out[i] = evaluateBarnesHutGPUVote<FLOAT>(leaf, nodes, nodes, p, beta, smoothDistExp<TREE::N>);
}

template <typename TREE>
__global__ void ref_mlpcv_scalar(const LeafData<TREE::N>* leaf, int n, const TREE* nodes,
                                 const LeafData<TREE::N>* contrib, const float* q, int nq, int samples,
                                 int kind, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  VectorNd<TREE::N> p;
  for (int d = 0; d < TREE::N; d++) p(d) = q[TREE::N * i + d];
  if (kind == 0)
    out[i] = multiLevelPrefixControlVariateSampleGPUQuery<FLOAT>(leaf, n, nodes, nodes, contrib, p,
                                                                 gravityPotential<TREE::N>, samples, 0);
  else if (kind == 3)
    out[i] = multiLevelPrefixControlVariateSampleGPUQuery<FLOAT>(leaf, n, nodes, nodes, contrib, p,
                                                                 signedSolidAngle<TREE::N>, samples, 0);
  else
    out[i] = multiLevelPrefixControlVariateSampleGPUQuery<FLOAT>(leaf, n, nodes, nodes, contrib, p,
                                                                 smoothDistExp<TREE::N>, samples, 0);
}

// q_soa: the queries axis by axis (the column-major layout the module reads).
template <int N>
__global__ void ref_brute_scalar(const LeafData<N>* leaf, int n, const float* q_soa, int nq, int kind,
                                 float* out) {
  int i = blockDim.x * blockIdx.x + threadIdx.x;
  float r;
  if (kind == 0)
    r = bruteForceSummationGPU<FLOAT>(leaf, n, q_soa, nq, gravityPotential<N>, i);
  else if (kind == 3)
    r = bruteForceSummationGPU<FLOAT>(leaf, n, q_soa, nq, signedSolidAngle<N>, i);
  else
    r = bruteForceSummationGPU<FLOAT>(leaf, n, q_soa, nq, smoothDistExp<N>, i);
  if (i < nq) out[i] = r;
}

}  // namespace

extern "C" {

int ref_sbhgpu_barnes_hut(void* s, int dim, int kind, const void* leaf, const void* node, const float* q,
                          int64_t nq, float beta, float* out) {
  int g = static_cast<int>((nq + 31) / 32);
  if (dim == 3)
    ref_vote_scalar<Node3><<<g, 32, 0, S(s)>>>(static_cast<const Leaf3*>(leaf), static_cast<const Node3*>(node), q,
                                               static_cast<int>(nq), beta, kind, out);
  else
    ref_vote_scalar<Node2><<<g, 32, 0, S(s)>>>(static_cast<const Leaf2*>(leaf), static_cast<const Node2*>(node), q,
                                               static_cast<int>(nq), beta, kind, out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int ref_sbhgpu_mlpcv(void* s, int dim, int kind, const void* leaf, int64_t n, const void* node,
                     const void* contrib, const float* q, int64_t nq, int samples, float* out) {
  int g = static_cast<int>((nq + 31) / 32);
  if (dim == 3)
    ref_mlpcv_scalar<Node3><<<g, 32, 0, S(s)>>>(static_cast<const Leaf3*>(leaf), static_cast<int>(n),
                                                static_cast<const Node3*>(node),
                                                static_cast<const Leaf3*>(contrib), q, static_cast<int>(nq),
                                                samples, kind, out);
  else
    ref_mlpcv_scalar<Node2><<<g, 32, 0, S(s)>>>(static_cast<const Leaf2*>(leaf), static_cast<int>(n),
                                                static_cast<const Node2*>(node),
                                                static_cast<const Leaf2*>(contrib), q, static_cast<int>(nq),
                                                samples, kind, out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int ref_sbhgpu_brute(void* s, int dim, int kind, const void* leaf, int64_t n, const float* q_soa, int64_t nq,
                     float* out) {
  int g = static_cast<int>((nq + 31) / 32);
  if (dim == 3)
    ref_brute_scalar<3><<<g, 32, 32 * sizeof(Leaf3), S(s)>>>(static_cast<const Leaf3*>(leaf),
                                                             static_cast<int>(n), q_soa, static_cast<int>(nq),
                                                             kind, out);
  else
    ref_brute_scalar<2><<<g, 32, 32 * sizeof(Leaf2), S(s)>>>(static_cast<const Leaf2*>(leaf),
                                                             static_cast<int>(n), q_soa, static_cast<int>(nq),
                                                             kind, out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // extern "C"
