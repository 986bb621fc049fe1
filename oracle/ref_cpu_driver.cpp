// C driver over the REFERENCE's own CPU tree code (bhorowitz/barnes-hut
// include/tree3d.h, tree2d.h, barnes_hut.h, tree_sampler.h, kernel.h),
// compiled from where those headers lie by oracle/Makefile against the
// project-written Eigen shim in oracle/ref_shim/.
//
// TEST INFRASTRUCTURE ONLY (the oracle's "reference" build): tests, the smoke
// check and bench.py's CPU-baseline leg load it through oracle/sbh_oracle.py.
// Nothing in the product library links it.
//
// What it mirrors:
//  * tree construction exactly as PyOctree / PyQuadtree do it
//    (include/py_tree.h:21-75): LeafData from points/normals/masses/alpha,
//    AABB from the given corners, max_depth = 100;
//  * evaluation exactly as evalBarnesHut does it (src/sbh.cpp:49-88): one
//    std::thread per requested thread, query i handled by thread i % T,
//    evaluateBarnesHut_stackless per query, num_contribs per query recorded;
//  * the MLPCV sampler (src/sbh.cpp:108-151 driving
//    include/tree_sampler.h:21-113), except that each query gets its own
//    std::mt19937 seeded with seed + i instead of the reference's single
//    global generator shared by all threads (src/sbh.cpp:40-41), which is a
//    data race and not reproducible.
// The reference CPU module has no force kernel (potential, winding number and
// smooth distance only), so the softened force and its query-side VJP are
// passed in as KernelFuncs restating src/sbh_ffi.cu:142-160 and :2062-2090.
#include <Eigen/Core>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "aabb.h"
#include "barnes_hut.h"
#include "kernel.h"
#include "leaf_data.h"
#include "tree2d.h"
#include "tree3d.h"
#include "tree_sampler.h"
#include "utils.h"

namespace {

FLOAT g_eps = FP(1e-3);
FLOAT g_cutoff = FP(0.0);
thread_local VectorNd<3> g_cot3;

// Softened (Plummer + optional erfc cutoff) force, the reference GPU formula
// (src/sbh_ffi.cu:142-160) evaluated in FLOAT on the host.
VectorNd<3> softForce3(const LeafData<3>& d, VectorNd<3> q) {
  VectorNd<3> r = q - d.position;
  FLOAT r2 = r.squaredNorm();
  FLOAT eps = g_eps > 0 ? g_eps : FP(0.0);
  FLOAT inv_r = FP(1.0) / sqrt(r2 + eps * eps + FP(1e-12));
  FLOAT inv_r3 = inv_r * inv_r * inv_r;
  FLOAT att = FP(1.0);
  if (g_cutoff > 0) {
    FLOAT dist = sqrt(r2 + FP(1e-12));
    FLOAT u = dist / (FP(2.0) * g_cutoff);
    att = std::erfc(u) + (FP(2.0) / FP(1.772453850905516)) * u * exp(-(u * u));
  }
  return (-d.mass * att * inv_r3) * r;
}

// Query-side VJP of softForce3 (src/sbh_ffi.cu:2062-2090).
VectorNd<3> softForceVjp3(const LeafData<3>& d, VectorNd<3> q) {
  VectorNd<3> r = q - d.position;
  VectorNd<3> g = g_cot3;
  FLOAT r2 = r.squaredNorm();
  FLOAT eps = g_eps > 0 ? g_eps : FP(0.0);
  FLOAT inv_r = FP(1.0) / sqrt(r2 + eps * eps + FP(1e-12));
  FLOAT inv_r3 = inv_r * inv_r * inv_r;
  FLOAT inv_r5 = inv_r3 * inv_r * inv_r;
  FLOAT att = FP(1.0);
  FLOAT cc = FP(0.0);
  if (g_cutoff > 0) {
    FLOAT dist = sqrt(r2 + FP(1e-12));
    FLOAT u = dist / (FP(2.0) * g_cutoff);
    FLOAT e = exp(-(u * u));
    att = std::erfc(u) + (FP(2.0) / FP(1.772453850905516)) * u * e;
    cc = inv_r3 * dist * e /
         (FP(2.0) * FP(1.772453850905516) * g_cutoff * g_cutoff * g_cutoff);
  }
  FLOAT rg = r.dot(g);
  VectorNd<3> grad = (att * inv_r3) * g - (rg * (FP(3.0) * att * inv_r5 + cc)) * r;
  return -d.mass * grad;
}

enum KernelId {
  K_POTENTIAL = 0,
  K_WINDING = 1,
  K_SMOOTHDIST = 2,
  K_SOFT_FORCE = 3,
  K_SOFT_FORCE_VJP = 4,
  K_GRAVITY_GRAD = 5,
};

struct Handle3 {
  int variant;
  std::vector<LeafData<3>> leaf;
  std::unique_ptr<Tree3D<8, 1>> t81;
  std::unique_ptr<Tree3D<1, 1>> t11;
  std::unique_ptr<Tree3D<1, 3>> t13;
};

struct Handle2 {
  std::vector<LeafData<2>> leaf;
  std::unique_ptr<Tree2D<1, 3>> t13;
};

int pickThreads(int threads) {
  if (threads > 0) return threads;
  int hc = static_cast<int>(std::thread::hardware_concurrency());
  return hc == 0 ? 8 : hc;
}

template <typename Fn>
void runPool(int64_t m, int threads, Fn fn) {
  int t = pickThreads(threads);
  std::vector<std::thread> pool;
  for (int ti = 0; ti < t; ti++) {
    pool.emplace_back([=]() {
      for (int64_t i = ti; i < m; i += t) fn(i);
    });
  }
  for (auto& th : pool) th.join();
}

template <typename TREE>
int evalTree3(const Handle3* h, const TREE* tree, const float* queries, int64_t m,
              float beta, int kernel, const float* cot, double* out,
              int32_t* counts, int threads) {
  const LeafData<3>* data = h->leaf.data();
  const auto* root = tree->root();
  const auto* buf = tree->node_buffer();
  FLOAT b = static_cast<FLOAT>(beta);
  runPool(m, threads, [&](int64_t i) {
    VectorNd<3> q(static_cast<FLOAT>(queries[3 * i + 0]),
                  static_cast<FLOAT>(queries[3 * i + 1]),
                  static_cast<FLOAT>(queries[3 * i + 2]));
    int nc = 0;
    if (kernel == K_POTENTIAL || kernel == K_WINDING || kernel == K_SMOOTHDIST) {
      KernelFunc<FLOAT, 3> f = kernel == K_POTENTIAL
                                   ? gravityPotential<3>
                                   : (kernel == K_WINDING ? signedSolidAngle<3>
                                                          : smoothDistExp<3>);
      FLOAT r = evaluateBarnesHut_stackless<FLOAT>(data, root, buf, q, b, f, nc);
      out[i] = static_cast<double>(r);
    } else {
      if (kernel == K_SOFT_FORCE_VJP) {
        g_cot3 = VectorNd<3>(static_cast<FLOAT>(cot[3 * i + 0]),
                             static_cast<FLOAT>(cot[3 * i + 1]),
                             static_cast<FLOAT>(cot[3 * i + 2]));
      }
      KernelFunc<VectorNd<3>, 3> f =
          kernel == K_SOFT_FORCE ? softForce3
                                 : (kernel == K_SOFT_FORCE_VJP ? softForceVjp3
                                                               : gravityGrad<3>);
      VectorNd<3> r = evaluateBarnesHut_stackless<VectorNd<3>>(data, root, buf, q, b, f, nc);
      out[3 * i + 0] = static_cast<double>(r(0));
      out[3 * i + 1] = static_cast<double>(r(1));
      out[3 * i + 2] = static_cast<double>(r(2));
    }
    if (counts) counts[i] = nc;
  });
  return 0;
}

template <typename TREE>
int mlpcvTree3(const Handle3* h, const TREE* tree, const float* queries, int64_t m,
               int kernel, int samples, uint32_t seed, double* out, int32_t* counts,
               int threads) {
  const LeafData<3>* data = h->leaf.data();
  const auto* root = tree->root();
  const auto* buf = tree->node_buffer();
  runPool(m, threads, [&](int64_t i) {
    std::mt19937 rng(seed + static_cast<uint32_t>(i));
    VectorNd<3> q(static_cast<FLOAT>(queries[3 * i + 0]),
                  static_cast<FLOAT>(queries[3 * i + 1]),
                  static_cast<FLOAT>(queries[3 * i + 2]));
    if (kernel == K_POTENTIAL || kernel == K_WINDING || kernel == K_SMOOTHDIST) {
      KernelFunc<FLOAT, 3> f = kernel == K_POTENTIAL
                                   ? gravityPotential<3>
                                   : (kernel == K_WINDING ? signedSolidAngle<3>
                                                          : smoothDistExp<3>);
      auto r = multiLevelPrefixControlVariateSample_stackless<FLOAT>(
          data, h->leaf.size(), root, buf, q, f, rng, samples);
      out[i] = static_cast<double>(r.first);
      if (counts) counts[i] = r.second;
    } else {
      KernelFunc<VectorNd<3>, 3> f = kernel == K_SOFT_FORCE ? softForce3 : gravityGrad<3>;
      auto r = multiLevelPrefixControlVariateSample_stackless<VectorNd<3>>(
          data, h->leaf.size(), root, buf, q, f, rng, samples);
      out[3 * i + 0] = static_cast<double>(r.first(0));
      out[3 * i + 1] = static_cast<double>(r.first(1));
      out[3 * i + 2] = static_cast<double>(r.first(2));
      if (counts) counts[i] = r.second;
    }
  });
  return 0;
}

}  // namespace

extern "C" {

// Size in bytes of FLOAT in this build (4, or 8 with -DUSE_DOUBLE).
int ref_float_bytes() { return static_cast<int>(sizeof(FLOAT)); }

void ref_set_softening(double eps, double cutoff) {
  g_eps = static_cast<FLOAT>(eps);
  g_cutoff = static_cast<FLOAT>(cutoff);
}

// variant 0 = Tree3D<8,1> (leaf size 8, binary split per axis),
// variant 1 = Tree3D<1,1> (sbh.Octree1), variant 2 = Tree3D<1,3> (sbh.Octree3).
void* ref_tree3d_build(int variant, const float* points, const float* normals,
                       const float* masses, int64_t n, const float* min_corner,
                       const float* max_corner, float alpha, int max_depth) {
  Handle3* h = new Handle3();
  h->variant = variant;
  h->leaf.resize(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) {
      h->leaf[i].position(d) = static_cast<FLOAT>(points[3 * i + d]);
      h->leaf[i].normal(d) = normals ? static_cast<FLOAT>(normals[3 * i + d]) : FP(0.0);
    }
    h->leaf[i].mass = static_cast<FLOAT>(masses[i]);
    h->leaf[i].alpha = static_cast<FLOAT>(alpha);
  }
  AABB<3> bounds(VectorNd<3>(static_cast<FLOAT>(min_corner[0]), static_cast<FLOAT>(min_corner[1]),
                             static_cast<FLOAT>(min_corner[2])),
                 VectorNd<3>(static_cast<FLOAT>(max_corner[0]), static_cast<FLOAT>(max_corner[1]),
                             static_cast<FLOAT>(max_corner[2])));
  int md = max_depth > 0 ? max_depth : 100;
  if (variant == 0) {
    h->t81 = std::make_unique<Tree3D<8, 1>>(h->leaf, bounds, md);
  } else if (variant == 1) {
    h->t11 = std::make_unique<Tree3D<1, 1>>(h->leaf, bounds, md);
  } else {
    h->t13 = std::make_unique<Tree3D<1, 3>>(h->leaf, bounds, md);
  }
  return h;
}

void ref_tree3d_free(void* p) { delete static_cast<Handle3*>(p); }

int64_t ref_tree3d_num_nodes(void* p) {
  Handle3* h = static_cast<Handle3*>(p);
  if (h->t81) return static_cast<int64_t>(h->t81->node_vector().size());
  if (h->t11) return static_cast<int64_t>(h->t11->node_vector().size());
  return static_cast<int64_t>(h->t13->node_vector().size());
}

int ref_tree3d_max_depth(void* p) {
  Handle3* h = static_cast<Handle3*>(p);
  if (h->t81) return h->t81->global_max_depth();
  if (h->t11) return h->t11->global_max_depth();
  return h->t13->global_max_depth();
}

size_t ref_tree3d_node_size(int variant) {
  if (variant == 0) return sizeof(Tree3DNode<8, 1>);
  if (variant == 1) return sizeof(Tree3DNode<1, 1>);
  return sizeof(Tree3DNode<1, 3>);
}

size_t ref_leaf3_size() { return sizeof(LeafData<3>); }
size_t ref_leaf2_size() { return sizeof(LeafData<2>); }

// Raw byte copies of the reordered leaf array, the node buffer and the
// per-node contrib array (what sbh.Octree*.{leaf_data,node_buffer,
// contrib_data}_bytes() return, src/sbh.cpp:225-249).
void ref_tree3d_copy_leaf(void* p, void* out) {
  Handle3* h = static_cast<Handle3*>(p);
  std::memcpy(out, h->leaf.data(), h->leaf.size() * sizeof(LeafData<3>));
}

void ref_tree3d_copy_nodes(void* p, void* out) {
  Handle3* h = static_cast<Handle3*>(p);
  if (h->t81) {
    std::memcpy(out, h->t81->node_buffer(), h->t81->node_vector().size() * sizeof(Tree3DNode<8, 1>));
  } else if (h->t11) {
    std::memcpy(out, h->t11->node_buffer(), h->t11->node_vector().size() * sizeof(Tree3DNode<1, 1>));
  } else {
    std::memcpy(out, h->t13->node_buffer(), h->t13->node_vector().size() * sizeof(Tree3DNode<1, 3>));
  }
}

void ref_tree3d_copy_contrib(void* p, void* out) {
  Handle3* h = static_cast<Handle3*>(p);
  const std::vector<LeafData<3>>* v = h->t81 ? &h->t81->contrib_data_vector()
                                      : (h->t11 ? &h->t11->contrib_data_vector()
                                                : &h->t13->contrib_data_vector());
  std::memcpy(out, v->data(), v->size() * sizeof(LeafData<3>));
}

// kernel: 0 potential, 1 winding number, 2 smooth distance (scalar, out[m]);
// 3 softened force, 4 softened force query-side VJP (needs cot), 5 gravityGrad
// (vector, out[3m]). counts[i] = interaction count (num_contribs).
int ref_tree3d_eval(void* p, const float* queries, int64_t m, float beta, int kernel,
                    const float* cot, double* out, int32_t* counts, int threads) {
  Handle3* h = static_cast<Handle3*>(p);
  if (h->t81) return evalTree3(h, h->t81.get(), queries, m, beta, kernel, cot, out, counts, threads);
  if (h->t11) return evalTree3(h, h->t11.get(), queries, m, beta, kernel, cot, out, counts, threads);
  return evalTree3(h, h->t13.get(), queries, m, beta, kernel, cot, out, counts, threads);
}

int ref_tree3d_mlpcv(void* p, const float* queries, int64_t m, int kernel, int samples,
                     uint32_t seed, double* out, int32_t* counts, int threads) {
  Handle3* h = static_cast<Handle3*>(p);
  if (h->t81) return mlpcvTree3(h, h->t81.get(), queries, m, kernel, samples, seed, out, counts, threads);
  if (h->t11) return mlpcvTree3(h, h->t11.get(), queries, m, kernel, samples, seed, out, counts, threads);
  return mlpcvTree3(h, h->t13.get(), queries, m, kernel, samples, seed, out, counts, threads);
}

// 2D quadtree Tree2D<1,3> (sbh.Quadtree3): the only builder of the Node2
// layout the 2D FFI targets consume.
void* ref_tree2d_build(const float* points, const float* normals, const float* masses,
                       int64_t n, const float* min_corner, const float* max_corner,
                       float alpha) {
  Handle2* h = new Handle2();
  h->leaf.resize(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; i++) {
    for (int d = 0; d < 2; d++) {
      h->leaf[i].position(d) = static_cast<FLOAT>(points[2 * i + d]);
      h->leaf[i].normal(d) = normals ? static_cast<FLOAT>(normals[2 * i + d]) : FP(0.0);
    }
    h->leaf[i].mass = static_cast<FLOAT>(masses[i]);
    h->leaf[i].alpha = static_cast<FLOAT>(alpha);
  }
  AABB<2> bounds(VectorNd<2>(static_cast<FLOAT>(min_corner[0]), static_cast<FLOAT>(min_corner[1])),
                 VectorNd<2>(static_cast<FLOAT>(max_corner[0]), static_cast<FLOAT>(max_corner[1])));
  h->t13 = std::make_unique<Tree2D<1, 3>>(h->leaf, bounds, 100);
  return h;
}

void ref_tree2d_free(void* p) { delete static_cast<Handle2*>(p); }
int64_t ref_tree2d_num_nodes(void* p) {
  return static_cast<int64_t>(static_cast<Handle2*>(p)->t13->node_vector().size());
}
size_t ref_tree2d_node_size() { return sizeof(Tree2DNode<1, 3>); }
void ref_tree2d_copy_leaf(void* p, void* out) {
  Handle2* h = static_cast<Handle2*>(p);
  std::memcpy(out, h->leaf.data(), h->leaf.size() * sizeof(LeafData<2>));
}
void ref_tree2d_copy_nodes(void* p, void* out) {
  Handle2* h = static_cast<Handle2*>(p);
  std::memcpy(out, h->t13->node_buffer(), h->t13->node_vector().size() * sizeof(Tree2DNode<1, 3>));
}
void ref_tree2d_copy_contrib(void* p, void* out) {
  Handle2* h = static_cast<Handle2*>(p);
  const auto& v = h->t13->contrib_data_vector();
  std::memcpy(out, v.data(), v.size() * sizeof(LeafData<2>));
}

// 2D evaluation: kernel 0 potential, 1 winding number (scalar); 5 gravityGrad (vec2).
int ref_tree2d_eval(void* p, const float* queries, int64_t m, float beta, int kernel,
                    double* out, int32_t* counts, int threads) {
  Handle2* h = static_cast<Handle2*>(p);
  const LeafData<2>* data = h->leaf.data();
  const auto* root = h->t13->root();
  const auto* buf = h->t13->node_buffer();
  FLOAT b = static_cast<FLOAT>(beta);
  runPool(m, threads, [&](int64_t i) {
    VectorNd<2> q(static_cast<FLOAT>(queries[2 * i + 0]), static_cast<FLOAT>(queries[2 * i + 1]));
    int nc = 0;
    if (kernel == K_GRAVITY_GRAD) {
      VectorNd<2> r = evaluateBarnesHut_stackless<VectorNd<2>>(data, root, buf, q, b, gravityGrad<2>, nc);
      out[2 * i + 0] = static_cast<double>(r(0));
      out[2 * i + 1] = static_cast<double>(r(1));
    } else {
      KernelFunc<FLOAT, 2> f = kernel == K_WINDING ? signedSolidAngle<2> : gravityPotential<2>;
      out[i] = static_cast<double>(evaluateBarnesHut_stackless<FLOAT>(data, root, buf, q, b, f, nc));
    }
    if (counts) counts[i] = nc;
  });
  return 0;
}

}  // extern "C"
