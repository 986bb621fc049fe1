/*
 * sbh_b200 -- C ABI of the B200-native Barnes-Hut summation library.
 *
 * Every entry point takes a CUDA stream, raw device pointers and sizes, and
 * parameters by value. The builds, walks and direct sums allocate no device
 * memory and do not synchronise the stream, so they can be called
 * concurrently on different streams and captured in CUDA graphs; the
 * read-backs (status, stats, export) and the adaptive Tree2D/Tree3D builders
 * synchronise, as their comments say. The one piece of process-global state
 * is the native tree's host registry: sbh_native_build records, per
 * workspace address, the tree's sizes, its target-group size and its target
 * range, which the later sbh_native_* calls on that workspace read (guarded
 * by a mutex). sbh_native_release() drops a workspace's entry; call it
 * before the workspace is freed, so that memory reused at the same address
 * is not mistaken for the old tree.
 * Temporary storage comes from a caller-provided workspace whose size the
 * matching *_workspace_bytes() function reports.
 *
 * Return value: SBH_OK (0) or an sbh_status error code; sbh_last_error()
 * returns the message of the calling thread's last failure. Errors detected
 * on the device (a stack-depth or iteration limit, an invalid bounding box)
 * are recorded in a status word at the start of the workspace and read back
 * with sbh_read_device_status().
 *
 * Reference interfaces replaced (bhorowitz/barnes-hut):
 *   src/sbh_ffi.cu       XLA-FFI handlers (:548-3576, symbols :3580-3947)
 *   src/sbh_ffi.cu       layout queries (:3949-3963)
 *   python/jax_sbh_ffi.py target names (:10-34) and attribute defaults
 * The compat entry points keep the reference's byte layouts (Leaf3 32 B,
 * OctreeNode8 104 B, Tree3DNode<1,3> 4272 B, Tree2DNode<1,3> 616 B) and
 * argument meaning; the sbh_native_* entry points are new (the adaptive tree,
 * the full adjoint and the batched forest have no reference counterpart).
 */
#ifndef SBH_B200_H_
#define SBH_B200_H_

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum {
  SBH_OK = 0,
  SBH_ERR_INVALID_ARGUMENT = 1, /* xla::ffi::Error::InvalidArgument in the reference */
  SBH_ERR_CUDA = 2,             /* xla::ffi::Error::Internal(cudaGetErrorString)   */
  SBH_ERR_WORKSPACE = 3,        /* workspace missing or smaller than required     */
  SBH_ERR_LIMIT = 4             /* device-side stack / iteration limit reached    */
} sbh_status;

/* Device status word bits (sbh_read_device_status). */
#define SBH_DEV_STACK_OVERFLOW 0x1u
#define SBH_DEV_BAD_BOUNDS 0x2u
#define SBH_DEV_ITER_LIMIT 0x4u

/* Message of the calling thread's last failed call ("" if none). */
const char* sbh_last_error(void);
/* Library version string. */
const char* sbh_version(void);

/* Copies the device status word stored at the start of `workspace` to
 * *out (synchronises `stream`). Replaces nothing in the reference: the
 * reference reports these conditions by host checks after a stream sync
 * (src/sbh_ffi.cu:1123-1133) or not at all. */
int sbh_read_device_status(cudaStream_t stream, const void* workspace, uint32_t* out);

/* ---------------------------------------------------------------------- */
/* Layout queries -- same symbols as src/sbh_ffi.cu:3949-3963            */
/* ---------------------------------------------------------------------- */
size_t sbh_leaf3_size(void);              /* 32   */
size_t sbh_node3_size(void);              /* 4272 */
size_t sbh_octree_level3_max_nodes(void); /* 513  */
size_t sbh_octree8_node_size(void);       /* 104  */
size_t sbh_leaf2_size(void);              /* 24   */
size_t sbh_node2_size(void);              /* 616  */
/* Dense octree8 node count (8^(d+1) - 1) / 7, python/jax_sbh_ffi.py:90-96. */
uint64_t sbh_octree8_total_nodes(int max_depth);

/* ---------------------------------------------------------------------- */
/* Direct sums                                                            */
/* ---------------------------------------------------------------------- */
/* Replaces BruteForceGravity (src/sbh_ffi.cu:548-598): out[q] = -sum m/(|p-q|+0.1),
 * dim 2 or 3, nearbyint minimum image when periodic. */
int sbh_bruteforce_gravity(cudaStream_t stream, const float* points, const float* masses,
                           int64_t n, int dim, const float* queries, int64_t nq, float* out,
                           int periodic, float box_length, int threads);

/* Replaces SoftenedDirectForce (src/sbh_ffi.cu:600-661). softening >= 0,
 * cutoff > 0 (erfc attenuation), as the reference validates. */
int sbh_direct_force_soft(cudaStream_t stream, const float* points, const float* masses,
                          int64_t n, const float* queries, int64_t nq, float* out,
                          float softening_scale, float cutoff_scale, int periodic,
                          float box_length, int threads);

/* Replaces SoftenedDirectForceVjp (src/sbh_ffi.cu:663-734): query-side VJP. */
int sbh_direct_force_soft_vjp(cudaStream_t stream, const float* points, const float* masses,
                              int64_t n, const float* queries, int64_t nq,
                              const float* cotangent, float* out, float softening_scale,
                              float cutoff_scale, int periodic, float box_length, int threads);

/* ---------------------------------------------------------------------- */
/* octree8 (dense Morton octree, reference layout)                        */
/* ---------------------------------------------------------------------- */
size_t sbh_build_octree8_workspace_bytes(int64_t n, int max_depth);

/* Replaces BuildOctree8Buffers (src/sbh_ffi.cu:1039-1420). min/max corners
 * are DEVICE pointers (3 floats each), as in the reference; the span is
 * computed on the device (no host round trip). Output byte sizes must be
 * exactly n*32, T(d)*104 and T(d)*32. Within one leaf cell particles keep
 * their input order (the reference's order there is nondeterministic). */
int sbh_build_octree8(cudaStream_t stream, const float* points, const float* normals,
                      const float* masses, int64_t n, const float* min_corner,
                      const float* max_corner, int max_depth, void* leaf_out,
                      size_t leaf_bytes, void* node_out, size_t node_bytes, void* contrib_out,
                      size_t contrib_bytes, void* workspace, size_t workspace_bytes);

/* No counterpart in the reference. Same result as sbh_build_octree8, for
 * callers that cannot allocate device memory at call time (an XLA custom
 * call under JAX's preallocating allocator, a fixed memory budget, code that
 * must avoid the implicit synchronisation of cudaMalloc): the temporaries
 * live in a 16 MiB array that is part of the library and stays resident on
 * every GPU that loads it. Nothing is allocated. Sizes whose
 * sbh_build_octree8_workspace_bytes(n, max_depth) exceeds
 * sbh_build_octree8_static_scratch_bytes() are rejected with
 * SBH_ERR_INVALID_ARGUMENT (for example n = 200,000 fits at max_depth 6,
 * n = 100,000 at max_depth 7). The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and caches it; under CUDA's
 * default lazy module loading that lookup is also where the library's device
 * code and this array are loaded onto the device, which can allocate device
 * memory and synchronise. Make that first call before a framework reserves
 * the rest of the GPU and before any stream capture, or set
 * CUDA_MODULE_LOADING=EAGER. The cached address is not valid after
 * cudaDeviceReset on that device. Each call clears what must start at zero
 * (status word, cell counters) itself. All calls share the one array, so
 * calls that may overlap on the GPU (different streams, or several host
 * threads) race and must be serialised by the caller. An invalid bounds span
 * (the largest of max_corner - min_corner over the axes not > 0) is recorded
 * only in the array's own status word, which this entry point does not
 * expose, and leaves a malformed tree: callers check their corners before
 * the call. */
size_t sbh_build_octree8_static_scratch_bytes(void);
int sbh_build_octree8_static(cudaStream_t stream, const float* points, const float* normals,
                             const float* masses, int64_t n, const float* min_corner,
                             const float* max_corner, int max_depth, void* leaf_out,
                             size_t leaf_bytes, void* node_out, size_t node_bytes,
                             void* contrib_out, size_t contrib_bytes);

/* Replaces BarnesHutForceOctree8 (src/sbh_ffi.cu:3133-3181). */
int sbh_barnes_hut_force_octree8(cudaStream_t stream, const void* leaf, size_t leaf_bytes,
                                 const void* nodes, size_t node_bytes, const float* queries,
                                 int64_t nq, float* out, float beta, int periodic,
                                 float box_length, int threads, void* workspace,
                                 size_t workspace_bytes);

/* Query-side VJP of sbh_barnes_hut_force_octree8 (gravityGradVjp,
 * src/sbh_ffi.cu:2044-2060, in the same traversal). No handler counterpart:
 * the reference's barnes_hut_force_octree8_vjp (python/jax_sbh_ffi.py:1372)
 * takes central finite differences of the forward. */
int sbh_barnes_hut_force_octree8_vjp(cudaStream_t stream, const void* leaf, size_t leaf_bytes,
                                     const void* nodes, size_t node_bytes, const float* queries,
                                     int64_t nq, const float* cotangent, float* out, float beta,
                                     int periodic, float box_length, int threads, void* workspace,
                                     size_t workspace_bytes);

/* Replaces SoftenedBarnesHutForceOctree8 (src/sbh_ffi.cu:3183-3248). */
int sbh_barnes_hut_force_octree8_soft(cudaStream_t stream, const void* leaf, size_t leaf_bytes,
                                      const void* nodes, size_t node_bytes,
                                      const float* queries, int64_t nq, float* out, float beta,
                                      float softening_scale, float cutoff_scale,
                                      int prune_enabled, float prune_r_cut_mult, int periodic,
                                      float box_length, int threads, void* workspace,
                                      size_t workspace_bytes);

/* Replaces SoftenedBarnesHutForceOctree8Vjp (src/sbh_ffi.cu:3250-3320). */
int sbh_barnes_hut_force_octree8_soft_vjp(cudaStream_t stream, const void* leaf,
                                          size_t leaf_bytes, const void* nodes,
                                          size_t node_bytes, const float* queries, int64_t nq,
                                          const float* cotangent, float* out, float beta,
                                          float softening_scale, float cutoff_scale,
                                          int prune_enabled, float prune_r_cut_mult,
                                          int periodic, float box_length, int threads,
                                          void* workspace, size_t workspace_bytes);

/* Replaces StochasticBarnesHutForceOctree8 (softened = 0, src/sbh_ffi.cu:3322-3373) and
 * SoftenedStochasticBarnesHutForceOctree8 (softened = 1, :3375-3443). Same curand
 * streams as the reference: curand_init(seed + q) and curand_init((u32)(seed + q +
 * 0x9e3779b9)). */
int sbh_stochastic_bh_force_octree8(cudaStream_t stream, int softened, const void* leaf,
                                    size_t leaf_bytes, const void* nodes, size_t node_bytes,
                                    const float* queries, int64_t nq, float* out,
                                    int samples_per_subdomain, int seed, float beta,
                                    float softening_scale, float cutoff_scale,
                                    int prune_enabled, float prune_r_cut_mult, int periodic,
                                    float box_length, int threads, void* workspace,
                                    size_t workspace_bytes);

/* Replaces StochasticBarnesHutForceOctree8Vjp (:3445-3501) and
 * SoftenedStochasticBarnesHutForceOctree8Vjp (:3503-3576). */
int sbh_stochastic_bh_force_octree8_vjp(cudaStream_t stream, int softened, const void* leaf,
                                        size_t leaf_bytes, const void* nodes,
                                        size_t node_bytes, const float* queries, int64_t nq,
                                        const float* cotangent, float* out,
                                        int samples_per_subdomain, int seed, float beta,
                                        float softening_scale, float cutoff_scale,
                                        int prune_enabled, float prune_r_cut_mult, int periodic,
                                        float box_length, int threads, void* workspace,
                                        size_t workspace_bytes);

/* Measurement helper (no reference counterpart): launches blocks x 256
 * threads of independent FMA chains; flops = blocks*256*8*16*iters*2. Times
 * the FP32 pipe peak that the traversal rooflines are reported against. */
int sbh_probe_fp32(cudaStream_t stream, float* out, int blocks, int iters);

/* As sbh_probe_fp32 with the FMAs issued two per instruction (packed FP32,
 * sm_100); same flops per launch. */
int sbh_probe_fp32x2(cudaStream_t stream, float* out, int blocks, int iters);

/* Bytes of device workspace every octree8 / Node2 / Node3 traversal needs
 * (the device status word). */
size_t sbh_traversal_workspace_bytes(void);

/* Workspace with which the per-query octree8 traversals (classic, softened,
 * their VJPs and the stochastic ones) of nq queries take the queries in
 * Morton order of their positions: a warp's threads then walk nearby paths,
 * and the deterministic ones walk them down one stack per warp, reading each
 * node once for the lanes that reach it. Every query's result is the same in
 * either order (each query takes its own decisions in its own order, its
 * curand streams seeded by its own index); with a smaller workspace, or
 * below 4,096 queries, they run in input order, one thread per query. */
size_t sbh_traversal_ordered_workspace_bytes(int64_t nq);

/* ---------------------------------------------------------------------- */
/* Level-3 tree (Tree3DNode<1,3> layout) and Node2 / Node3 traversals     */
/* ---------------------------------------------------------------------- */
size_t sbh_build_octree_level3_workspace_bytes(int64_t n);

/* Replaces BuildOctreeLevel3Buffers (src/sbh_ffi.cu:736-1037). Outputs must be
 * n*32, 513*4272 and 513*32 bytes. */
int sbh_build_octree_level3(cudaStream_t stream, const float* points, const float* normals,
                            const float* masses, int64_t n, const float* min_corner,
                            const float* max_corner, void* leaf_out, size_t leaf_bytes,
                            void* node_out, size_t node_bytes, void* contrib_out,
                            size_t contrib_bytes, void* workspace, size_t workspace_bytes);

/* kernel: 0 = gravity potential (BarnesHutGravity{,3D}, out[nq]),
 *         1 = gravityGrad force (BarnesHutForce{,3D}, out[nq*dim]),
 *         2 = softened force (SoftenedBarnesHutForce{,3D}, out[nq*dim]),
 *         3 = winding number (new target; the reference only has it in the
 *             pybind module, src/sbh_gpu.cu:100-120), out[nq],
 *         6 = smoothDistExp, exp(-alpha |p - q|) (pybind module only,
 *             src/sbh_gpu.cu:122-141), out[nq].
 * dim 2 -> Node2/Leaf2 bytes, dim 3 -> Node3/Leaf3 bytes. Warp-vote opening
 * exactly as evaluateBarnesHutGPUVote (include/barnes_hut_gpu.h:19-72), with
 * warps formed from `threads`-sized blocks as the reference launches them. */
int sbh_barnes_hut_tree(cudaStream_t stream, int dim, int kernel, const void* leaf,
                        size_t leaf_bytes, const void* nodes, size_t node_bytes,
                        const float* queries, int64_t nq, float* out, float beta,
                        float softening_scale, float cutoff_scale, int periodic,
                        float box_length, int threads, void* workspace,
                        size_t workspace_bytes);

/* Stochastic (MLPCV) on Node2/Node3 trees, multiLevelPrefixControlVariateSampleGPUQuery
 * (include/tree_sampler_gpu.h:25-140); kernel ids as above (0, 1, 2, 3). */
int sbh_stochastic_bh_tree(cudaStream_t stream, int dim, int kernel, const void* leaf,
                           size_t leaf_bytes, const void* nodes, size_t node_bytes,
                           const void* contrib, size_t contrib_bytes, const float* queries,
                           int64_t nq, float* out, int samples_per_subdomain, int seed,
                           float softening_scale, float cutoff_scale, int periodic,
                           float box_length, int threads, void* workspace,
                           size_t workspace_bytes);

/* GPU build of the adaptive quadtree Tree2DNode<1,3> (Node2, 616 bytes) that
 * the reference builds on the CPU (sbh.Quadtree3, include/tree2d.h:237-330,
 * include/py_tree.h:29-45, max_depth 100; used by build_quadtree_buffers,
 * python/jax_sbh_ffi.py:658-724): leaf size 1, an 8 x 8 split per node,
 * nodes in breadth-first order, the same bytes as the reference's builder
 * for distinct points. points / normals (NULL: zeros) are n x 2, masses n,
 * min_corner / max_corner 2 floats on the device. leaf_out is n * 24 bytes;
 * node_out and contrib_out hold up to node_capacity_bytes / 616 nodes and
 * contrib records. Synchronises the stream (once per tree level). On
 * success *num_nodes is the node count; when node_out is too small the call
 * returns SBH_ERR_LIMIT with a larger capacity to retry with in *num_nodes. */
size_t sbh_build_quadtree_workspace_bytes(int64_t n);
int sbh_build_quadtree(cudaStream_t stream, const float* points, const float* normals,
                       const float* masses, int64_t n, const float* min_corner,
                       const float* max_corner, float alpha, void* leaf_out, size_t leaf_bytes,
                       void* node_out, size_t node_capacity_bytes, void* contrib_out,
                       size_t contrib_capacity_bytes, uint64_t* num_nodes, void* workspace,
                       size_t workspace_bytes);

/* The same for the adaptive octree Tree3DNode<1,3> (Node3, 4272 bytes; 8^3
 * split per node) that the reference builds on the CPU (sbh.Octree3,
 * include/tree3d.h:238-327, include/py_tree.h:58-75) for
 * build_octree_buffers(backend="cpu") (python/jax_sbh_ffi.py:805-830).
 * points / normals are n x 3, leaf_out n * 32 bytes, records as above. */
size_t sbh_build_adaptive_octree_workspace_bytes(int64_t n);
int sbh_build_adaptive_octree(cudaStream_t stream, const float* points, const float* normals,
                              const float* masses, int64_t n, const float* min_corner,
                              const float* max_corner, float alpha, void* leaf_out,
                              size_t leaf_bytes, void* node_out, size_t node_capacity_bytes,
                              void* contrib_out, size_t contrib_capacity_bytes,
                              uint64_t* num_nodes, void* workspace, size_t workspace_bytes);

/* The pybind module sbh_gpu's evaluations (src/sbh_gpu.cu:36-661; no FFI
 * handler) on Node2/Node3 buffers, for the scalar kernels kernel = 0
 * (gravityPotential), 3 (signedSolidAngle) or 6 (smoothDistExp,
 * include/kernel.h:82-87). Barnes-Hut is sbh_barnes_hut_tree with these
 * kernel ids. sbh_brute_force_tree sums every leaf record in leaf order with
 * Kahan compensation (bruteForceSummationGPU, include/brute_force_gpu.h);
 * sbh_stochastic_bh_tree_shared_seed is the MLPCV estimate with one seed
 * for every query, as the module passes it (0), instead of the FFI's
 * seed + query index. */
int sbh_brute_force_tree(cudaStream_t stream, int dim, int kernel, const void* leaf,
                         size_t leaf_bytes, const float* queries, int64_t nq, float* out,
                         int threads);
int sbh_stochastic_bh_tree_shared_seed(cudaStream_t stream, int dim, int kernel, const void* leaf,
                                       size_t leaf_bytes, const void* nodes, size_t node_bytes,
                                       const void* contrib, size_t contrib_bytes,
                                       const float* queries, int64_t nq, float* out,
                                       int samples_per_subdomain, int seed, int threads,
                                       void* workspace, size_t workspace_bytes);

/* Query-side VJPs on Node2/Node3 trees: out[nq*dim] = J(q)^T cotangent of the
 * force (softened = 0: gravityGrad, 1: softened force), with the opening
 * decisions of the forward traversal. No handler counterpart: the
 * reference's barnes_hut_force_vjp and softened_barnes_hut_force_vjp
 * (python/jax_sbh_ffi.py:1037-1135) take central finite differences of the
 * forward; these evaluate the derivative kernels gravityGradVjp /
 * gravityGradSoftCutoffVjp (src/sbh_ffi.cu:2044-2090) in the same walk. */
int sbh_barnes_hut_tree_vjp(cudaStream_t stream, int dim, int softened, const void* leaf,
                            size_t leaf_bytes, const void* nodes, size_t node_bytes,
                            const float* queries, int64_t nq, const float* cotangent, float* out,
                            float beta, float softening_scale, float cutoff_scale, int periodic,
                            float box_length, int threads, void* workspace,
                            size_t workspace_bytes);

/* MLPCV query-side VJP with the forward's sampled paths and weights for the
 * same seed (the convention of the reference's stochastic octree8 VJP,
 * src/sbh_ffi.cu:2293-2442); replaces the finite differences of
 * stochastic_barnes_hut_force_vjp and softened_stochastic_barnes_hut_force_vjp
 * (python/jax_sbh_ffi.py:1222-1334). */
int sbh_stochastic_bh_tree_vjp(cudaStream_t stream, int dim, int softened, const void* leaf,
                               size_t leaf_bytes, const void* nodes, size_t node_bytes,
                               const void* contrib, size_t contrib_bytes, const float* queries,
                               int64_t nq, const float* cotangent, float* out,
                               int samples_per_subdomain, int seed, float softening_scale,
                               float cutoff_scale, int periodic, float box_length, int threads,
                               void* workspace, size_t workspace_bytes);

/* ---------------------------------------------------------------------- */
/* Native adaptive octree (no reference counterpart: a new B200 path)     */
/* ---------------------------------------------------------------------- */
/* Opening rule: the reference's |q - cell centre| / cell diagonal >= beta
 * (beta = 1/theta; include/tree3d.h:134-153, src/sbh_ffi.cu:1878-1893) made
 * to hold for every target of a group: accept a node when the distance from
 * the group's bounding box to the cell centre exceeds beta * diagonal.
 * Targets are walked in groups of at most sbh_native_group_size() (packed
 * from the tree's cells). The far field is the node monopole about its
 * centre of mass plus (quadrupole = 1) its second moment about the COM;
 * near-field leaves are summed pairwise. */
typedef struct sbh_native_params {
  float beta;      /* 1 / theta, > 0 */
  float softening; /* Plummer softening epsilon, >= 0 */
  float cutoff;    /* erfc attenuation scale of the short-range split; <= 0 disables */
  int quadrupole;  /* 1: monopole + quadrupole far field (needs cutoff <= 0), 0: monopole */
  int periodic;    /* 1: minimum-image displacements in a cube of side box_length (monopole only);
                      the opening test uses the cell's image nearest the group */
  float box_length;
  float prune_radius; /* > 0 (with cutoff > 0): skip nodes whose cell lies farther than this from
                         every target of the group (the short-range split of TreePM) */
  float quadrupole_radius; /* with quadrupole = 1: > 0 adds the quadrupole only for accepted nodes
                              closer to the group box than quadrupole_radius opening radii
                              (beta * diagonal), the monopole alone beyond; 0: for every
                              accepted node */
  float quadrupole_linear; /* with quadrupole = 1: kappa > 0 takes the quadrupole of an accepted node
                              to first order about the group box centre c, a_q(c - X) + J(c - X)
                              (x - c), instead of at every target, when the group's half diagonal
                              r_g satisfies r_g^2 <= kappa^2 |c - cell centre|^2. The monopole is
                              still evaluated at every target. Such a node costs one evaluation per
                              group instead of one per target; 0: every quadrupole is exact */
} sbh_native_params;

/* Most targets one group holds (one warp walks a group). */
int sbh_native_group_size(void);

/* Forgets the tree recorded for `workspace` in the host registry (sizes,
 * group size, target range). Later sbh_native_* evaluation calls on it fail
 * with SBH_ERR_INVALID_ARGUMENT until the next sbh_native_build. Call it
 * before freeing a workspace. Always returns SBH_OK; device memory is not
 * touched. */
int sbh_native_release(const void* workspace);

/* Re-cuts the target groups of the tree built in `workspace` with at most
 * group_size (1 .. sbh_native_group_size()) targets each; later walks use
 * them. The build cuts groups of sbh_native_group_size(). Smaller groups have
 * tighter boxes: fewer interactions per target where the walk is bounded by
 * a prune radius (the TreePM short range), more per-node overhead per target
 * elsewhere. */
int sbh_native_set_group_size(cudaStream_t stream, void* workspace, size_t workspace_bytes,
                              int group_size);

/* Restricts the force and adjoint walks on the tree in `workspace` to the
 * target groups whose first target lies at sorted positions [begin, end)
 * (0 <= begin <= end <= n). Ranks holding the same tree and a partition of
 * [0, n) serve every target exactly once: each rank's force rows are zero
 * outside its targets and its gradients are partial sums, so the sum over
 * ranks (an all-reduce of N x 16 bytes) is the full result. Host-side state;
 * a new build resets the range to [0, n). */
int sbh_native_set_target_range(cudaStream_t stream, void* workspace, size_t workspace_bytes,
                                int64_t begin, int64_t end);

/* Workspace for a tree of n points in num_systems independent systems. */
size_t sbh_native_workspace_bytes(int64_t n, int num_systems, int leaf_size, int with_normals,
                                  int with_adjoint);

/* Builds the tree(s) inside `workspace`. points (n x 3), masses (n), normals
 * (n x 3, optional: winding number). system_offsets: device int64 array of
 * num_systems + 1 offsets into the concatenated inputs (NULL for one system).
 * leaf_size in [1, 32]. with_adjoint reserves the scratch of
 * sbh_native_force_vjp. Later calls on the same workspace evaluate this tree.
 * The workspace must be 16-byte aligned (cudaMalloc's is). */
int sbh_native_build(cudaStream_t stream, const float* points, const float* masses,
                     const float* normals, int64_t n, const int64_t* system_offsets,
                     int num_systems, int leaf_size, int with_adjoint, void* workspace,
                     size_t workspace_bytes);

/* Softened self-gravity of every point of every system: force_out (n x 3,
 * input order). */
int sbh_native_force(cudaStream_t stream, const sbh_native_params* params, float* force_out,
                     void* workspace, size_t workspace_bytes);

/* Stochastic Barnes-Hut self-gravity on the tree in `workspace`
 * (Plummer softening, free space: params->cutoff <= 0, no periodic box or
 * prune radius; params->beta is the refined opening beta_f, params'
 * quadrupole settings are not used). force_out (n x 3, input order) = the
 * group walk at beta_coarse (monopole + quadrupole everywhere) plus, per
 * target group, `samples` (1..1024) nodes of the group's coarse cut drawn
 * by stratified sampling in proportion to M r_g^3 / r^5 (r from the group
 * box to the node's COM; zero where the box clears beta_f cell diagonals), each adding
 * (group walk of the node's subtree at beta_f - the node's quadrupole) /
 * (samples * probability) at the group's targets. Its expectation is the
 * group walk at beta_f with the quadrupole at every accepted node
 * (sbh_native_force with quadrupole_radius = quadrupole_linear = 0); the
 * draws depend on the seed and the group's first input index only. The
 * stochastic counterpart of the reference's stochastic octree8 traversal
 * (src/sbh_ffi.cu:2146-2291) on this library's tree: `samples` is the
 * number of tree nodes drawn per query. Needs the full target range and
 * allocates nothing. */
int sbh_native_stochastic_force(cudaStream_t stream, const sbh_native_params* params, float beta_coarse,
                                int samples, uint64_t seed, float* force_out, void* workspace,
                                size_t workspace_bytes);

/* The adjoint of sbh_native_stochastic_force's estimate at the same seed,
 * with the draws held fixed (as the reference's stochastic VJPs hold their
 * paths, src/sbh_ffi.cu:2293-2442): grad_points (n x 3) and grad_masses (n)
 * of L = sum_i w_i . a_i, input order, with respect to every particle's
 * position and mass (the tree built with_adjoint). force_out (optional)
 * receives the estimate. */
int sbh_native_stochastic_force_vjp(cudaStream_t stream, const sbh_native_params* params, float beta_coarse,
                                    int samples, uint64_t seed, const float* cotangent, float* force_out,
                                    float* grad_points, float* grad_masses, void* workspace,
                                    size_t workspace_bytes);

/* One traversal computing the force (optional force_out) and the full
 * adjoint of L = sum_i w_i . a_i: grad_points (n x 3) and grad_masses (n),
 * exact for the evaluated approximation (query side, direct sources, and the
 * chain rule through every accepted node's mass, centroid and second moment;
 * opening decisions are recomputed, not stored). */
int sbh_native_force_vjp(cudaStream_t stream, const sbh_native_params* params,
                         const float* cotangent, float* force_out, float* grad_points,
                         float* grad_masses, void* workspace, size_t workspace_bytes);

/* The two phases of sbh_native_force_vjp, for callers that time or overlap
 * them: the traversal (query-side gradient, per-node and per-particle source
 * adjoints, optional force) and the finalize pass (node adjoints pushed down
 * to particles, combined with the traversal's terms, written in input order). */
int sbh_native_adjoint_walk(cudaStream_t stream, const sbh_native_params* params,
                            const float* cotangent, float* force_out, void* workspace,
                            size_t workspace_bytes);
int sbh_native_adjoint_finalize(cudaStream_t stream, float* grad_points, float* grad_masses,
                                void* workspace, size_t workspace_bytes);

/* After sbh_native_adjoint_walk (or sbh_native_force_vjp) on this workspace:
 * the query-side part of the gradient alone, J_i^T w_i of target i's own row
 * (n x 3, input order). This is the quantity the reference's octree8 VJP
 * returns (barnes_hut_force_octree8_soft_vjp_kernel, src/sbh_ffi.cu:2092-2144,
 * which has no source-side terms). It reads the walk's scratch, so it comes
 * before the next walk on the workspace. */
int sbh_native_adjoint_query_side(cudaStream_t stream, float* grad_points, void* workspace,
                                  size_t workspace_bytes);

/* Query workspace of sbh_native_winding_number. */
size_t sbh_native_query_workspace_bytes(int64_t nq);

/* Generalized winding number (include/kernel.h:73-80) of the oriented points
 * of a single-system tree built with normals, at nq query points. Far field:
 * node mass and mass-weighted mean normal at the COM (as the reference's
 * trees aggregate them, include/tree3d.h:255-264). out: nq floats. */
int sbh_native_winding_number(cudaStream_t stream, float beta, const float* queries, int64_t nq,
                              float* out, void* workspace, size_t workspace_bytes,
                              void* query_workspace, size_t query_workspace_bytes);

/* Adjoint of sbh_native_winding_number: with cotangent u (nq floats) and
 * L = sum_i u_i w(q_i), writes dL/dq (grad_queries, nq x 3, input order) and
 * dL/d(points, normals, masses) of the sources (n x 3, n x 3, n, input
 * order), and w itself to out when out is non-null. The tree must be built
 * with normals and with_adjoint. Same plan as the forward (opening decisions
 * recomputed, not stored); the far field of a node is (sum m n) . (X - q) K,
 * so its adjoints reach the sources through X = sum m p / M and sum m n. No
 * reference counterpart: the reference's winding number (signedSolidAngle,
 * include/kernel.h:73-80; src/sbh_gpu.cu:53-187) has no derivative. */
int sbh_native_winding_number_vjp(cudaStream_t stream, float beta, const float* queries, int64_t nq,
                                  const float* cotangent, float* out, float* grad_queries, float* grad_points,
                                  float* grad_normals, float* grad_masses, void* workspace, size_t workspace_bytes,
                                  void* query_workspace, size_t query_workspace_bytes);

/* Synchronises; out4 = {nodes, target groups, far interactions, near
 * interactions} of the last build / evaluation on this workspace. The walks
 * themselves carry no counters: after a force or adjoint walk the counts
 * come from one count-only traversal with that walk's parameters and target
 * range (the same decisions), run here once per walk. */
int sbh_native_stats(cudaStream_t stream, const void* workspace, size_t workspace_bytes,
                     uint64_t* out4);

/* Synchronises; *far_quadrupole = the far interactions (per target) of the
 * last force or adjoint walk on this workspace that took the quadrupole,
 * exact or linearized. */
int sbh_native_quadrupole_count(cudaStream_t stream, const void* workspace, size_t workspace_bytes,
                                uint64_t* far_quadrupole);

/* Synchronises; out3 = {far interactions per target with the exact
 * quadrupole, far interactions per target with the linearized quadrupole,
 * (group, node) pairs of the linearized ones} of the last force or adjoint
 * walk on this workspace. A linearized pair is evaluated once per group. */
int sbh_native_far_counts(cudaStream_t stream, const void* workspace, size_t workspace_bytes, uint64_t* out3);

/* Synchronises; copies sorted keys (n x u64), the permutation (n x u32,
 * sorted slot -> input index) and the 80-byte node records to device buffers
 * (each may be NULL) and the node count to *num_nodes. A node record is
 * {COM x, y, z, mass; cell centre x, y, z, diagonal; S_xx, S_yy, S_zz, S_xy;
 * S_xz, S_yz, 0, 0} as floats, then {start, end, skip, level | 0x100 if
 * leaf} as int32, S being the second moment about the COM. */
int sbh_native_export(cudaStream_t stream, const void* workspace, size_t workspace_bytes,
                      uint64_t* keys_out, uint32_t* perm_out, void* nodes_out,
                      size_t nodes_capacity, uint64_t* num_nodes);

/* ---------------------------------------------------------------------- */
/* Mesh surface sampling (winding-number sources from a triangle mesh)     */
/* ---------------------------------------------------------------------- */
/* Replaces the host-side sampler of the reference's mesh sources
 * (python/old_interface/sampler.py:45-78 sample_points_on_mesh;
 * python/old_interface/source.py:119-155 MeshSurface): n points, each on a
 * face chosen with probability area / total area and uniform inside it, with
 * the face's unit normal (e1 x e2 / |e1 x e2| for the face's vertex order)
 * and the weight total area / n. The random numbers are outputs 3i+1..3i+3 of
 * splitmix64 seeded with `seed` for sample i, so results depend on
 * (seed, i) only. Faces that reference a vertex outside [0, nv) set
 * SBH_DEV_BAD_BOUNDS in the device status word and count as zero area; a mesh
 * without positive area sets it too and yields zeros.
 * vertices: nv x 3 f32, faces: nf x 3 i32 (device). Outputs: points n x 3,
 * normals n x 3, weights n (device, f32). */
size_t sbh_mesh_sample_workspace_bytes(int64_t nf);
int sbh_sample_mesh_surface(cudaStream_t stream, const float* vertices, int64_t nv,
                            const int32_t* faces, int64_t nf, int64_t n, uint64_t seed,
                            float* points_out, float* normals_out, float* weights_out,
                            void* workspace, size_t workspace_bytes);

/* Vertex sources of a triangle mesh, replacing the host-side libigl calls of
 * the reference's MeshVertices (python/old_interface/source.py:85-115:
 * igl.per_vertex_normals(V, F, 1) and the diagonal of igl.massmatrix). Every
 * vertex is a source; its normal is the normalised sum of e1 x e2 over the
 * incident faces (area weighting; zero for a vertex without area), its mass
 * the mixed Voronoi area of Meyer, Desbrun, Schroeder and Barr (2003): per
 * face, corner i takes (|Pi Pk|^2 cot_j + |Pi Pj|^2 cot_k) / 8 when no angle
 * is obtuse, else area / 2 at the obtuse corner and area / 4 at the others.
 * Masses sum to the surface area. Faces that reference a vertex outside
 * [0, nv) set SBH_DEV_BAD_BOUNDS in the device status word and add nothing.
 * vertices: nv x 3 f32, faces: nf x 3 i32 (device). Outputs: normals nv x 3,
 * masses nv (device, f32); the points are the vertices themselves. */
size_t sbh_mesh_vertex_workspace_bytes(int64_t nv);
int sbh_mesh_vertex_sources(cudaStream_t stream, const float* vertices, int64_t nv,
                            const int32_t* faces, int64_t nf, float* normals_out,
                            float* masses_out, void* workspace, size_t workspace_bytes);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* SBH_B200_H_ */
