/*
 * CPU oracle for the Barnes-Hut summation path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithms (bhorowitz/barnes-hut,
 * src/sbh_ffi.cu and include/kernel.h), used by tests/, by the smoke check
 * and by bench.py's CPU-baseline leg as the checker. The product library
 * never calls, links or loads this file.
 *
 * Conventions:
 *  - Opening decisions, quantisation and node geometry are computed in float
 *    in the same operation order as the reference, so that the oracle takes
 *    the same traversal decisions; every kernel contribution and every sum is
 *    then evaluated in double. The result is "the reference's algorithm with
 *    exact arithmetic", the right yardstick for an FP32 GPU implementation.
 *  - The reference compiles with --use_fast_math, so its float divisions are
 *    approximate; decisions and Morton codes that sit exactly on a boundary
 *    can differ from this IEEE oracle. Tests count such cases instead of
 *    requiring them to be zero.
 *  - The reference scatters leaves with an atomic cursor (src/sbh_ffi.cu:1732),
 *    so its order inside one leaf cell is nondeterministic; the oracle keeps
 *    input order inside a cell (a stable counting sort).
 *
 * Native-tree section (orc_native_*): the CPU restatement of this project's
 * own adaptive Morton octree and group traversal, used to pin the GPU build
 * bit-exactly (keys, permutation, topology) and the GPU sums within FP32
 * tolerance.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_SQRT_PI 1.772453850905516
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Byte layouts of the reference (src/sbh_ffi.cu:47-63, include/leaf_data.h) */
/* ------------------------------------------------------------------------ */
typedef struct {
  float pos[3];
  float nrm[3];
  float mass;
  float alpha;
} Leaf3; /* LeafData<3>, 32 bytes */

typedef struct {
  uint32_t start, end, parent, first_child;
  uint32_t child[8];
  uint8_t child_mask, depth, is_leaf, pad0;
  float cx, cy, cz, half_size, diameter;
  Leaf3 contrib;
} OctreeNode8; /* 104 bytes */

_Static_assert(sizeof(Leaf3) == 32, "Leaf3 size");
_Static_assert(sizeof(OctreeNode8) == 104, "OctreeNode8 size");

size_t orc_leaf3_size(void) { return sizeof(Leaf3); }
size_t orc_octree8_node_size(void) { return sizeof(OctreeNode8); }

uint32_t orc_octree8_total_nodes(int max_depth) {
  uint32_t total = 0, level = 1;
  for (int l = 0; l <= max_depth; l++) {
    total += level;
    level <<= 3;
  }
  return total;
}

/* morton3d, src/sbh_ffi.cu:162-171 */
static uint32_t morton3d(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t code = 0;
  for (int i = 0; i < bits; i++) {
    code |= ((x >> i) & 1u) << (3 * i);
    code |= ((y >> i) & 1u) << (3 * i + 1);
    code |= ((z >> i) & 1u) << (3 * i + 2);
  }
  return code;
}

/* quantize_axis, src/sbh_ffi.cu:173-179 (IEEE division here) */
static uint32_t quantize_axis(float v, float min_v, float span, int bits) {
  float t = (v - min_v) / span;
  t = fminf(fmaxf(t, 0.0f), 0.999999f);
  uint32_t max_bin = (1u << bits) - 1u;
  return (uint32_t)(t * (float)(max_bin + 1));
}

/* ------------------------------------------------------------------------ */
/* Softened force and its query-side VJP (src/sbh_ffi.cu:142-160, 431-501,  */
/* 2062-2090), in double. cutoff <= 0 disables the erfc attenuation.        */
/* ------------------------------------------------------------------------ */
typedef struct {
  double eps, cutoff;
  int periodic;
  double box;
} SoftParams;

static void min_image(double* r, const SoftParams* sp, int use_floor) {
  if (sp->periodic && sp->box > 0.0) {
    for (int d = 0; d < 3; d++) {
      double q = r[d] / sp->box;
      r[d] -= sp->box * (use_floor ? floor(q + 0.5) : nearbyint(q));
    }
  }
}

static void soft_force_pair(const double* r, double m, const SoftParams* sp, double* acc) {
  double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  double eps = sp->eps > 0 ? sp->eps : 0.0;
  double inv_r = 1.0 / sqrt(r2 + eps * eps + 1e-12);
  double inv_r3 = inv_r * inv_r * inv_r;
  double att = 1.0;
  if (sp->cutoff > 0.0) {
    double dist = sqrt(r2 + 1e-12);
    double u = dist / (2.0 * sp->cutoff);
    att = erfc(u) + (2.0 / ORC_SQRT_PI) * u * exp(-(u * u));
  }
  double c = -m * att * inv_r3;
  acc[0] += c * r[0];
  acc[1] += c * r[1];
  acc[2] += c * r[2];
}

static void soft_force_pair_vjp(const double* r, double m, const double* g,
                                const SoftParams* sp, double* acc) {
  double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  double eps = sp->eps > 0 ? sp->eps : 0.0;
  double inv_r = 1.0 / sqrt(r2 + eps * eps + 1e-12);
  double inv_r3 = inv_r * inv_r * inv_r;
  double inv_r5 = inv_r3 * inv_r * inv_r;
  double att = 1.0, cc = 0.0;
  if (sp->cutoff > 0.0) {
    double dist = sqrt(r2 + 1e-12);
    double u = dist / (2.0 * sp->cutoff);
    double e = exp(-(u * u));
    att = erfc(u) + (2.0 / ORC_SQRT_PI) * u * e;
    cc = inv_r3 * dist * e / (2.0 * ORC_SQRT_PI * sp->cutoff * sp->cutoff * sp->cutoff);
  }
  double rg = r[0] * g[0] + r[1] * g[1] + r[2] * g[2];
  double lin = att * inv_r3;
  double rad = rg * (3.0 * att * inv_r5 + cc);
  for (int d = 0; d < 3; d++) acc[d] += -m * (lin * g[d] - rad * r[d]);
}

/* gravityGrad (include/kernel.h:89-94): -m (q-p) / (|q-p| + 0.1)^3 */
static void grav_grad_pair(const double* r, double m, double* acc) {
  double dist = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  double den = dist + 0.1;
  double c = -m / (den * den * den);
  acc[0] += c * r[0];
  acc[1] += c * r[1];
  acc[2] += c * r[2];
}

/* gravityGradVjp (src/sbh_ffi.cu:2044-2060) */
static void grav_grad_pair_vjp(const double* r, double m, const double* g, double* acc) {
  double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  double dist = sqrt(r2 + 1e-12);
  double den = dist + 0.1;
  double id3 = 1.0 / (den * den * den);
  double id4 = id3 / den;
  double rg = r[0] * g[0] + r[1] * g[1] + r[2] * g[2];
  double dinv = 1.0 / (dist + 1e-12);
  for (int d = 0; d < 3; d++) acc[d] += -m * (id3 * g[d] - 3.0 * rg * dinv * id4 * r[d]);
}

/* ------------------------------------------------------------------------ */
/* Direct sums (src/sbh_ffi.cu:399-546), double precision                   */
/* ------------------------------------------------------------------------ */

/* softened_direct_force: out[q] = sum_i f(q - p_i), nearbyint min-image */
void orc_direct_force_soft(const float* pts, const float* masses, int64_t n,
                           const float* queries, int64_t nq, double eps, double cutoff,
                           int periodic, double box, double* out) {
  SoftParams sp = {eps, cutoff, periodic, box};
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nq; q++) {
    double acc[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; i++) {
      double r[3] = {(double)queries[3 * q] - pts[3 * i], (double)queries[3 * q + 1] - pts[3 * i + 1],
                     (double)queries[3 * q + 2] - pts[3 * i + 2]};
      min_image(r, &sp, 0);
      soft_force_pair(r, masses[i], &sp, acc);
    }
    out[3 * q] = acc[0];
    out[3 * q + 1] = acc[1];
    out[3 * q + 2] = acc[2];
  }
}

void orc_direct_force_soft_vjp(const float* pts, const float* masses, int64_t n,
                               const float* queries, int64_t nq, const float* cot,
                               double eps, double cutoff, int periodic, double box,
                               double* out) {
  SoftParams sp = {eps, cutoff, periodic, box};
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nq; q++) {
    double acc[3] = {0, 0, 0};
    double g[3] = {cot[3 * q], cot[3 * q + 1], cot[3 * q + 2]};
    for (int64_t i = 0; i < n; i++) {
      double r[3] = {(double)queries[3 * q] - pts[3 * i], (double)queries[3 * q + 1] - pts[3 * i + 1],
                     (double)queries[3 * q + 2] - pts[3 * i + 2]};
      min_image(r, &sp, 0);
      soft_force_pair_vjp(r, masses[i], g, &sp, acc);
    }
    out[3 * q] = acc[0];
    out[3 * q + 1] = acc[1];
    out[3 * q + 2] = acc[2];
  }
}

/*
 * Exact full gradient of L = sum_i w_i . a_i for self-gravity (queries ==
 * sources, a_i = sum_j m_j phi(x_i - x_j), softened, cutoff <= 0 or > 0):
 *   dL/dx_k = sum_j J(x_k - x_j) (m_j w_k - m_k w_j)       (J = d phi/dr, symmetric, even)
 *   dL/dm_k = sum_i w_i . phi(x_i - x_k)
 * A subset of k can be requested (idx); out_dx is (nk, 3), out_dm is (nk,).
 * This is the exact gradient with respect to positions and masses; the
 * reference itself only has the query-side term.
 */
void orc_direct_full_adjoint(const float* pts, const float* masses, int64_t n,
                             const float* w, double eps, double cutoff, const int64_t* idx,
                             int64_t nk, double* out_dx, double* out_dm) {
  SoftParams sp = {eps, cutoff, 0, 1.0};
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t t = 0; t < nk; t++) {
    int64_t k = idx ? idx[t] : t;
    double gx[3] = {0, 0, 0};
    double gm = 0.0;
    double wk[3] = {w[3 * k], w[3 * k + 1], w[3 * k + 2]};
    double mk = masses[k];
    for (int64_t j = 0; j < n; j++) {
      double r[3] = {(double)pts[3 * k] - pts[3 * j], (double)pts[3 * k + 1] - pts[3 * j + 1],
                     (double)pts[3 * k + 2] - pts[3 * j + 2]};
      /* J(r) v via the VJP formula with unit mass: acc = -(J v) ... sign:
       * soft_force_pair_vjp gives acc += -m*(lin g - rad r) = (d/dq of f)^T g
       * where f(q) = m phi(q - p). So J(r)^T g with m=1 is exactly that. */
      double v[3];
      for (int d = 0; d < 3; d++) v[d] = masses[j] * wk[d] - mk * (double)w[3 * j + d];
      soft_force_pair_vjp(r, 1.0, v, &sp, gx);
      /* dL/dm_k: w_j . phi(x_j - x_k) = -w_j . phi(x_k - x_j) */
      double f[3] = {0, 0, 0};
      soft_force_pair(r, 1.0, &sp, f);
      gm -= (double)w[3 * j] * f[0] + (double)w[3 * j + 1] * f[1] + (double)w[3 * j + 2] * f[2];
    }
    out_dx[3 * t] = gx[0];
    out_dx[3 * t + 1] = gx[1];
    out_dx[3 * t + 2] = gx[2];
    out_dm[t] = gm;
  }
}

/* brute_force_gravity (src/sbh_ffi.cu:399-429): -sum m/(|p-q| + 0.1), dim 2 or 3 */
void orc_bruteforce_gravity(const float* pts, const float* masses, int64_t n, int dim,
                            const float* queries, int64_t nq, int periodic, double box,
                            double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nq; q++) {
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) {
      double d2 = 0.0;
      for (int d = 0; d < dim; d++) {
        double diff = (double)pts[dim * i + d] - queries[dim * q + d];
        if (periodic && box > 0.0) diff -= box * nearbyint(diff / box);
        d2 += diff * diff;
      }
      acc += -(double)masses[i] / (sqrt(d2) + 0.1);
    }
    out[q] = acc;
  }
}

/* signedSolidAngle<3> (include/kernel.h:73-80), direct sum in double:
 * w(q) = sum m n.(p-q) / (4 pi (|p-q|^3 + 1e-5)) */
void orc_direct_winding_number(const float* pts, const float* normals, const float* masses,
                               int64_t n, const float* queries, int64_t nq, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nq; q++) {
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) {
      double d[3] = {(double)pts[3 * i] - queries[3 * q], (double)pts[3 * i + 1] - queries[3 * q + 1],
                     (double)pts[3 * i + 2] - queries[3 * q + 2]};
      double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      double nd = normals[3 * i] * d[0] + normals[3 * i + 1] * d[1] + normals[3 * i + 2] * d[2];
      acc += (double)masses[i] * nd / (4.0 * ORC_PI * (dist * dist * dist + 1e-5));
    }
    out[q] = acc;
  }
}

/* ------------------------------------------------------------------------ */
/* octree8 build (src/sbh_ffi.cu:1039-1420, kernels :1682-1876)             */
/* ------------------------------------------------------------------------ */

/*
 * Outputs, exactly sized as the reference's handler requires:
 *   leaf_out    n * 32 bytes, Leaf3 in Morton-cell order (stable inside a cell)
 *   node_out    T(d) * 104 bytes, dense levels 0..d, level l at offset (8^l-1)/7
 *   contrib_out T(d) * 32 bytes, node.contrib copied out
 *   codes_out   (optional) n Morton codes in input order
 *   perm_out    (optional) n input indices in leaf order
 * Returns 0, or 1 for invalid arguments (depth out of [1,10], span <= 0).
 */
int orc_build_octree8(const float* pts, const float* normals, const float* masses, int64_t n,
                      const float* min_corner, const float* max_corner, int max_depth,
                      void* leaf_out, void* node_out, void* contrib_out, uint32_t* codes_out,
                      int64_t* perm_out) {
  if (max_depth < 1 || max_depth > 10) return 1;
  float span = fmaxf(fmaxf(max_corner[0] - min_corner[0], max_corner[1] - min_corner[1]),
                     max_corner[2] - min_corner[2]);
  if (!(span > 0.0f)) return 1;
  uint32_t leaf_count = 1u << (3 * max_depth);
  uint32_t total = orc_octree8_total_nodes(max_depth);

  uint32_t* codes = (uint32_t*)malloc(sizeof(uint32_t) * (n > 0 ? n : 1));
  uint32_t* cnt = (uint32_t*)calloc(leaf_count, sizeof(uint32_t));
  uint32_t* off = (uint32_t*)calloc((size_t)leaf_count + 1, sizeof(uint32_t));
  /* level sums in double: count, mass, m*pos, m*normal */
  uint32_t** lcnt = (uint32_t**)calloc(max_depth + 1, sizeof(uint32_t*));
  double** lsum = (double**)calloc(max_depth + 1, sizeof(double*));
  for (int l = 0; l <= max_depth; l++) {
    lcnt[l] = (uint32_t*)calloc((size_t)1 << (3 * l), sizeof(uint32_t));
    lsum[l] = (double*)calloc(((size_t)1 << (3 * l)) * 7, sizeof(double));
  }
  for (int64_t i = 0; i < n; i++) {
    uint32_t qx = quantize_axis(pts[3 * i], min_corner[0], span, max_depth);
    uint32_t qy = quantize_axis(pts[3 * i + 1], min_corner[1], span, max_depth);
    uint32_t qz = quantize_axis(pts[3 * i + 2], min_corner[2], span, max_depth);
    uint32_t c = morton3d(qx, qy, qz, max_depth);
    codes[i] = c;
    cnt[c]++;
    double m = masses[i];
    double* s = &lsum[max_depth][7 * (size_t)c];
    s[0] += m;
    for (int d = 0; d < 3; d++) {
      s[1 + d] += m * (double)pts[3 * i + d];
      s[4 + d] += m * (double)(normals ? normals[3 * i + d] : 0.0f);
    }
  }
  memcpy(lcnt[max_depth], cnt, sizeof(uint32_t) * leaf_count);
  for (uint32_t c = 0; c < leaf_count; c++) off[c + 1] = off[c] + cnt[c];
  /* stable scatter */
  uint32_t* cur = (uint32_t*)calloc(leaf_count, sizeof(uint32_t));
  Leaf3* leaf = (Leaf3*)leaf_out;
  for (int64_t i = 0; i < n; i++) {
    uint32_t c = codes[i];
    uint32_t dst = off[c] + cur[c]++;
    Leaf3 L;
    for (int d = 0; d < 3; d++) {
      L.pos[d] = pts[3 * i + d];
      L.nrm[d] = normals ? normals[3 * i + d] : 0.0f;
    }
    L.mass = masses[i];
    L.alpha = 1.0f;
    leaf[dst] = L;
    if (perm_out) perm_out[dst] = i;
  }
  /* reduce levels (src/sbh_ffi.cu:1745-1786) */
  for (int l = max_depth - 1; l >= 0; l--) {
    size_t cntl = (size_t)1 << (3 * l);
    for (size_t p = 0; p < cntl; p++) {
      uint32_t cc = 0;
      double s[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int c = 0; c < 8; c++) {
        size_t ch = p * 8 + c;
        if (lcnt[l + 1][ch] == 0) continue;
        cc += lcnt[l + 1][ch];
        for (int k = 0; k < 7; k++) s[k] += lsum[l + 1][7 * ch + k];
      }
      lcnt[l][p] = cc;
      for (int k = 0; k < 7; k++) lsum[l][7 * p + k] = s[k];
    }
  }
  /* nodes (src/sbh_ffi.cu:1788-1876) */
  float cx = min_corner[0] + span * 0.5f;
  float cy = min_corner[1] + span * 0.5f;
  float cz = min_corner[2] + span * 0.5f;
  float half_size = span * 0.5f;
  OctreeNode8* nodes = (OctreeNode8*)node_out;
  Leaf3* contrib = (Leaf3*)contrib_out;
  uint32_t level_off = 0;
  for (int l = 0; l <= max_depth; l++) {
    uint32_t level_nodes = 1u << (3 * l);
    uint32_t parent_off = l == 0 ? 0u : level_off - (1u << (3 * (l - 1)));
    uint32_t child_off = level_off + level_nodes;
    int grid = 1 << l;
    float step = half_size * 2.0f / (float)grid;
    for (uint32_t idx = 0; idx < level_nodes; idx++) {
      OctreeNode8 nd;
      memset(&nd, 0, sizeof(nd));
      uint32_t node_idx = level_off + idx;
      nd.depth = (uint8_t)l;
      nd.parent = l == 0 ? node_idx : parent_off + (idx >> 3);
      nd.is_leaf = l == max_depth ? 1 : 0;
      nd.child_mask = 0;
      nd.first_child = 0xFFFFFFFFu;
      uint32_t first_leaf = idx << (3 * (max_depth - l));
      nd.start = off[first_leaf];
      nd.end = nd.start + lcnt[l][idx];
      int ix = 0, iy = 0, iz = 0;
      for (int b = 0; b < l; b++) {
        ix |= ((idx >> (3 * b + 0)) & 1) << b;
        iy |= ((idx >> (3 * b + 1)) & 1) << b;
        iz |= ((idx >> (3 * b + 2)) & 1) << b;
      }
      /* the GPU contracts (a + b*c) into one fma */
      nd.cx = fmaf((float)ix + 0.5f, step, cx - half_size);
      nd.cy = fmaf((float)iy + 0.5f, step, cy - half_size);
      nd.cz = fmaf((float)iz + 0.5f, step, cz - half_size);
      nd.half_size = step * 0.5f;
      nd.diameter = step * sqrtf(3.0f);
      if (l < max_depth) {
        uint32_t child_base = child_off + (idx << 3);
        uint8_t mask = 0;
        for (uint32_t c = 0; c < 8; c++) {
          nd.child[c] = child_base + c;
          if (lcnt[l + 1][(idx << 3) + c] > 0) {
            mask |= (uint8_t)(1u << c);
            if (nd.first_child == 0xFFFFFFFFu) nd.first_child = child_base + c;
          }
        }
        nd.child_mask = mask;
        if (mask == 0) nd.is_leaf = 1;
      } else {
        for (int c = 0; c < 8; c++) nd.child[c] = 0xFFFFFFFFu;
      }
      double* s = &lsum[l][7 * (size_t)idx];
      nd.contrib.alpha = 1.0f;
      nd.contrib.mass = (float)s[0];
      if ((float)s[0] > 0.0f) {
        for (int d = 0; d < 3; d++) {
          nd.contrib.pos[d] = (float)(s[1 + d] / s[0]);
          nd.contrib.nrm[d] = (float)(s[4 + d] / s[0]);
        }
      }
      nodes[node_idx] = nd;
      contrib[node_idx] = nd.contrib;
    }
    level_off += level_nodes;
  }
  if (codes_out) memcpy(codes_out, codes, sizeof(uint32_t) * (size_t)n);
  free(codes);
  free(cnt);
  free(off);
  free(cur);
  for (int l = 0; l <= max_depth; l++) {
    free(lcnt[l]);
    free(lsum[l]);
  }
  free(lcnt);
  free(lsum);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* octree8 classic BH traversal (src/sbh_ffi.cu:1878-2144)                  */
/* ------------------------------------------------------------------------ */

/* minImageDisplacement (include/kernel.h:27-39), float, floor(x + 0.5) */
static void min_image_f(float* d, int periodic, float box) {
  if (periodic && box > 0.0f) {
    float inv_l = 1.0f / box;
    for (int k = 0; k < 3; k++) d[k] = d[k] - box * floorf(d[k] * inv_l + 0.5f);
  }
}

/* octree8_use_far_field, :1878-1893 */
static int use_far_field(const OctreeNode8* nd, const float* q, float beta, int periodic,
                         float box) {
  if (nd->is_leaf) return 1;
  float dc[3] = {q[0] - nd->cx, q[1] - nd->cy, q[2] - nd->cz};
  min_image_f(dc, periodic, box);
  float dist = sqrtf(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
  return dist / nd->diameter >= beta;
}

static float axis_dist(float q, float lo, float hi) {
  if (q < lo) return lo - q;
  if (q > hi) return q - hi;
  return 0.0f;
}

/* octree8_should_prune, :1903-1948 */
static int should_prune(const OctreeNode8* nd, const float* q, int prune_on, float r_cut_sq,
                        int periodic, float box) {
  if (!prune_on) return 0;
  float qx = q[0], qy = q[1], qz = q[2];
  if (periodic && box > 0.0f) {
    float inv_l = 1.0f / box;
    qx -= box * nearbyintf((qx - nd->cx) * inv_l);
    qy -= box * nearbyintf((qy - nd->cy) * inv_l);
    qz -= box * nearbyintf((qz - nd->cz) * inv_l);
  }
  float dx = axis_dist(qx, nd->cx - nd->half_size, nd->cx + nd->half_size);
  float dy = axis_dist(qy, nd->cy - nd->half_size, nd->cy + nd->half_size);
  float dz = axis_dist(qz, nd->cz - nd->half_size, nd->cz + nd->half_size);
  return dx * dx + dy * dy + dz * dz > r_cut_sq;
}

/* kernel ids for the octree8 evaluators */
enum { ORC_K_GRAV_GRAD = 0, ORC_K_SOFT = 1, ORC_K_SOFT_VJP = 2, ORC_K_GRAV_GRAD_VJP = 3 };

static void eval_source(int kernel, const float* q, const Leaf3* src, const double* g,
                        const SoftParams* sp, double* acc) {
  double r[3] = {(double)q[0] - src->pos[0], (double)q[1] - src->pos[1],
                 (double)q[2] - src->pos[2]};
  min_image(r, sp, 1);
  switch (kernel) {
    case ORC_K_GRAV_GRAD:
      grav_grad_pair(r, src->mass, acc);
      break;
    case ORC_K_SOFT:
      soft_force_pair(r, src->mass, sp, acc);
      break;
    case ORC_K_SOFT_VJP:
      soft_force_pair_vjp(r, src->mass, g, sp, acc);
      break;
    default:
      grav_grad_pair_vjp(r, src->mass, g, acc);
      break;
  }
}

/*
 * barnes_hut_force_octree8{,_soft,_soft_vjp}_kernel (:1950-2144).
 * kernel: 0 gravityGrad, 1 softened force, 2 softened query-side VJP (cot).
 * prune_on / r_cut_sq exactly as the handler derives them (:3235-3237).
 * counts (optional): interactions per query. Returns 0, or 2 if a query's
 * stack would exceed the reference's 128 entries.
 */
int orc_bh_octree8(const void* leaf_bytes, const void* node_bytes, const float* queries,
                   int64_t nq, const float* cot, float beta, int kernel, double eps,
                   double cutoff, int prune_on, float r_cut_sq, int periodic, float box,
                   double* out, int32_t* counts) {
  const Leaf3* leaf = (const Leaf3*)leaf_bytes;
  const OctreeNode8* nodes = (const OctreeNode8*)node_bytes;
  SoftParams sp = {eps, cutoff, periodic, box};
  int status = 0;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t qi = 0; qi < nq; qi++) {
    const float* q = &queries[3 * qi];
    double g[3] = {0, 0, 0};
    if (cot) {
      g[0] = cot[3 * qi];
      g[1] = cot[3 * qi + 1];
      g[2] = cot[3 * qi + 2];
    }
    double acc[3] = {0, 0, 0};
    int32_t nint = 0;
    int stack[128];
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
      int idx = stack[--top];
      const OctreeNode8* nd = &nodes[idx];
      if (nd->contrib.mass == 0.0f) continue;
      if (kernel != ORC_K_GRAV_GRAD && should_prune(nd, q, prune_on, r_cut_sq, periodic, box))
        continue;
      if (use_far_field(nd, q, beta, periodic, box)) {
        if (nd->is_leaf) {
          for (uint32_t i = nd->start; i < nd->end; i++) {
            eval_source(kernel, q, &leaf[i], g, &sp, acc);
            nint++;
          }
        } else {
          eval_source(kernel, q, &nd->contrib, g, &sp, acc);
          nint++;
        }
      } else {
        for (int c = 0; c < 8; c++) {
          if (nd->child_mask & (1u << c)) {
            if (top >= 128) {
              status = 2;
              break;
            }
            stack[top++] = (int)nd->child[c];
          }
        }
      }
    }
    out[3 * qi] = acc[0];
    out[3 * qi + 1] = acc[1];
    out[3 * qi + 2] = acc[2];
    if (counts) counts[qi] = nint;
  }
  return status;
}

/* ======================================================================== */
/* Native adaptive Morton octree (this project's own tree)                  */
/* ======================================================================== */
/*
 * Definition (the GPU build must reproduce every integer field bit-exactly):
 *  1. lo = per-axis min of the points, hi = per-axis max; span = max(hi - lo)
 *     over axes, replaced by 1 when it is 0. All in float, exact.
 *  2. scale = 2097152.0 / (double)span; q_a = floor(((double)x_a - (double)lo_a)
 *     * scale) clamped to [0, 2^21 - 1] (double, no fused operations).
 *  3. key = 63-bit Morton interleave, x in bit 3i, y in 3i+1, z in 3i+2.
 *  4. perm = stable sort of input indices by key.
 *  5. level-l cell of a key = its top 3l bits (l = 0..21). A cell is a node
 *     when l == 0 or its parent cell holds more than leaf_size particles. A
 *     node is a leaf when it holds <= leaf_size particles or l == 21.
 *  6. Nodes are numbered in DFS pre-order (parent before children, children
 *     in Morton order). skip[n] = pre-order index after n's subtree; a node's
 *     particles are the sorted range [start, end).
 */
static int common_levels(uint64_t a, uint64_t b) {
  uint64_t x = a ^ b;
  if (x == 0) return 21;
  int lz = __builtin_clzll(x) - 1; /* 63-bit keys: bit 63 is always 0 */
  return lz / 3;
}

static int cmp_key_idx(const void* a, const void* b) {
  const uint64_t* x = (const uint64_t*)a;
  const uint64_t* y = (const uint64_t*)b;
  if (x[0] < y[0]) return -1;
  if (x[0] > y[0]) return 1;
  if (x[1] < y[1]) return -1;
  if (x[1] > y[1]) return 1;
  return 0;
}

/* Quantisation + keys + stable sort. keys_out[i] is the key of sorted slot i,
 * perm_out[i] the input index stored there. box_out = {lo[3], span}. */
void orc_native_sort(const float* pts, int64_t n, uint64_t* keys_out, int64_t* perm_out,
                     float* box_out) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = 0; i < n; i++)
    for (int d = 0; d < 3; d++) {
      lo[d] = fminf(lo[d], pts[3 * i + d]);
      hi[d] = fmaxf(hi[d], pts[3 * i + d]);
    }
  float span = 0.0f;
  for (int d = 0; d < 3; d++) span = fmaxf(span, hi[d] - lo[d]);
  if (!(span > 0.0f)) span = 1.0f;
  double scale = 2097152.0 / (double)span;
  uint64_t* kv = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (n > 0 ? n : 1));
  for (int64_t i = 0; i < n; i++) {
    uint64_t key = 0;
    for (int d = 0; d < 3; d++) {
      double t = ((double)pts[3 * i + d] - (double)lo[d]) * scale;
      double f = floor(t);
      uint64_t qv = f < 0.0 ? 0 : (f > 2097151.0 ? 2097151u : (uint64_t)f);
      for (int b = 0; b < 21; b++) key |= ((qv >> b) & 1ull) << (3 * b + d);
    }
    kv[2 * i] = key;
    kv[2 * i + 1] = (uint64_t)i;
  }
  qsort(kv, (size_t)n, 2 * sizeof(uint64_t), cmp_key_idx);
  for (int64_t i = 0; i < n; i++) {
    keys_out[i] = kv[2 * i];
    perm_out[i] = (int64_t)kv[2 * i + 1];
  }
  free(kv);
  box_out[0] = lo[0];
  box_out[1] = lo[1];
  box_out[2] = lo[2];
  box_out[3] = span;
}

/*
 * Topology from sorted keys. Returns the node count; when the output arrays
 * are non-NULL they receive (pre-order) start, end, skip and level per node.
 * Every slot count is computed from per-position quantities only:
 *   d(i)  = common levels of key[i-1] and key[i] (cells i starts: levels > d(i))
 *   L(i)  = leaf level of position i = min(21, 1 + max_{a} cl(key[a], key[a+S]))
 *           over windows a in [i-S, i] with a+S < n (S = leaf_size),
 *           or 0 if n <= S.
 *   position i starts internal nodes at levels [lo(i), L(i) - 1] where
 *   lo(i) = 0 for i == 0 else d(i) + 1, and a leaf at level L(i) when
 *   i == 0 or d(i) < L(i).
 */
int64_t orc_native_topology(const uint64_t* keys, int64_t n, int leaf_size, int32_t* start,
                            int32_t* end, int32_t* skip, int8_t* level) {
  if (n <= 0) return 0;
  int S = leaf_size;
  int* cl = (int*)malloc(sizeof(int) * (size_t)n);
  int* Lv = (int*)malloc(sizeof(int) * (size_t)n);
  int64_t* base = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
  for (int64_t a = 0; a < n; a++) cl[a] = (a + S < n) ? common_levels(keys[a], keys[a + S]) : -1;
  for (int64_t i = 0; i < n; i++) {
    if (n <= S) {
      Lv[i] = 0;
      continue;
    }
    int mx = -1;
    int64_t a0 = i - S < 0 ? 0 : i - S;
    for (int64_t a = a0; a <= i; a++)
      if (cl[a] > mx) mx = cl[a];
    int L = mx + 1;
    Lv[i] = L > 21 ? 21 : L;
  }
  base[0] = 0;
  for (int64_t i = 0; i < n; i++) {
    int lo = i == 0 ? 0 : common_levels(keys[i - 1], keys[i]) + 1;
    int d = i == 0 ? -1 : common_levels(keys[i - 1], keys[i]);
    int nint = Lv[i] - lo;
    if (nint < 0) nint = 0;
    int nleaf = (i == 0 || d < Lv[i]) ? 1 : 0;
    base[i + 1] = base[i] + nint + nleaf;
  }
  int64_t total = base[n];
  if (start) {
    for (int64_t i = 0; i < n; i++) {
      int lo = i == 0 ? 0 : common_levels(keys[i - 1], keys[i]) + 1;
      int d = i == 0 ? -1 : common_levels(keys[i - 1], keys[i]);
      int64_t slot = base[i];
      int top = (i == 0 || d < Lv[i]) ? Lv[i] : Lv[i] - 1;
      for (int l = lo; l <= top; l++) {
        /* end: first j > i whose key leaves the level-l cell of key[i] */
        int64_t e = i + 1;
        int64_t lo_s = i + 1, hi_s = n;
        uint64_t pref = l == 0 ? 0 : keys[i] >> (63 - 3 * l);
        while (lo_s < hi_s) {
          int64_t mid = (lo_s + hi_s) >> 1;
          uint64_t pm = l == 0 ? 0 : keys[mid] >> (63 - 3 * l);
          if (pm == pref)
            lo_s = mid + 1;
          else
            hi_s = mid;
        }
        e = lo_s;
        start[slot] = (int32_t)i;
        end[slot] = (int32_t)e;
        level[slot] = (int8_t)l;
        skip[slot] = (int32_t)(e < n ? base[e] : total);
        slot++;
      }
    }
  }
  free(cl);
  free(Lv);
  free(base);
  return total;
}

/* ------------------------------------------------------------------------ */
/* Native tree handle: sorted order, topology, geometry, and a traversal     */
/* plan (per target group: accepted nodes and near-field leaves).            */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t n, nn;
  int leaf_size;
  float lo[3], span;
  uint64_t* keys;
  int64_t* perm;
  int32_t *start, *end, *skip;
  int8_t* level;
  float* center; /* nn x 3, cell centre */
  float* side;   /* nn, cell side */
  /* plan */
  int group_size;
  int64_t ngroups;
  int64_t* far_off; /* ngroups + 1 */
  int32_t* far_idx;
  uint8_t* far_quad; /* per far entry: 1 when the node takes the quadrupole */
  double* far_coef;  /* per far entry: the term's coefficient (NULL: 1), set by orc_native_stochastic_plan */
  double* near_coef; /* per near entry: the leaf's coefficient (NULL: 1) */
  int64_t* near_off;
  int32_t* near_idx; /* near-field leaf node ids */
  int64_t* gstart;
  int64_t* gend;
  float* gcen; /* per group: centre (3) and squared half diagonal of its box (float) */
  /* winding-number plan over external queries (orc_native_wn_plan) */
  int64_t wn_nq, wn_ngroups;
  int64_t* wn_qperm; /* sorted query -> input index */
  int64_t *wn_far_off, *wn_near_off;
  int32_t *wn_far_idx, *wn_near_idx;
} NativeTree;

static void cell_geometry(const NativeTree* t, int64_t nd, uint64_t key) {
  int l = t->level[nd];
  uint64_t p = l == 0 ? 0 : key >> (63 - 3 * l);
  uint32_t c[3] = {0, 0, 0};
  for (int b = 0; b < l; b++)
    for (int d = 0; d < 3; d++) c[d] |= (uint32_t)((p >> (3 * b + d)) & 1u) << b;
  float side = ldexpf(t->span, -l);
  t->side[nd] = side;
  for (int d = 0; d < 3; d++)
    t->center[3 * nd + d] = (float)((double)t->lo[d] + ((double)c[d] + 0.5) * (double)side);
}

void* orc_native_build(const float* pts, int64_t n, int leaf_size) {
  NativeTree* t = (NativeTree*)calloc(1, sizeof(NativeTree));
  t->n = n;
  t->leaf_size = leaf_size;
  t->keys = (uint64_t*)malloc(sizeof(uint64_t) * (n > 0 ? n : 1));
  t->perm = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  float box[4];
  orc_native_sort(pts, n, t->keys, t->perm, box);
  memcpy(t->lo, box, 3 * sizeof(float));
  t->span = box[3];
  int64_t nn = orc_native_topology(t->keys, n, leaf_size, NULL, NULL, NULL, NULL);
  t->nn = nn;
  size_t cap = nn > 0 ? (size_t)nn : 1;
  t->start = (int32_t*)malloc(sizeof(int32_t) * cap);
  t->end = (int32_t*)malloc(sizeof(int32_t) * cap);
  t->skip = (int32_t*)malloc(sizeof(int32_t) * cap);
  t->level = (int8_t*)malloc(cap);
  t->center = (float*)malloc(sizeof(float) * 3 * cap);
  t->side = (float*)malloc(sizeof(float) * cap);
  orc_native_topology(t->keys, n, leaf_size, t->start, t->end, t->skip, t->level);
  for (int64_t k = 0; k < nn; k++) cell_geometry(t, k, t->keys[t->start[k]]);
  return t;
}

void orc_native_free(void* h) {
  NativeTree* t = (NativeTree*)h;
  if (!t) return;
  free(t->keys);
  free(t->perm);
  free(t->start);
  free(t->end);
  free(t->skip);
  free(t->level);
  free(t->center);
  free(t->side);
  free(t->far_off);
  free(t->far_idx);
  free(t->far_quad);
  free(t->far_coef);
  free(t->near_coef);
  free(t->near_off);
  free(t->near_idx);
  free(t->gstart);
  free(t->gend);
  free(t->gcen);
  free(t->wn_qperm);
  free(t->wn_far_off);
  free(t->wn_near_off);
  free(t->wn_far_idx);
  free(t->wn_near_idx);
  free(t);
}

int64_t orc_native_num_nodes(void* h) { return ((NativeTree*)h)->nn; }

void orc_native_get(void* h, uint64_t* keys, int64_t* perm, int32_t* start, int32_t* end,
                    int32_t* skip, int8_t* level, float* center, float* side, float* box) {
  NativeTree* t = (NativeTree*)h;
  if (keys) memcpy(keys, t->keys, sizeof(uint64_t) * t->n);
  if (perm) memcpy(perm, t->perm, sizeof(int64_t) * t->n);
  if (start) memcpy(start, t->start, sizeof(int32_t) * t->nn);
  if (end) memcpy(end, t->end, sizeof(int32_t) * t->nn);
  if (skip) memcpy(skip, t->skip, sizeof(int32_t) * t->nn);
  if (level) memcpy(level, t->level, t->nn);
  if (center) memcpy(center, t->center, sizeof(float) * 3 * t->nn);
  if (side) memcpy(side, t->side, sizeof(float) * t->nn);
  if (box) {
    memcpy(box, t->lo, 3 * sizeof(float));
    box[3] = t->span;
  }
}

/* Node monopoles in double from the sorted particles: mass, mass-weighted
 * centroid, and the float COM the GPU stores. mom: nn x 4 (M, X, Y, Z). */
#define MOM 10
static void native_moments(const NativeTree* t, const float* pts, const float* masses,
                           double* mom) {
  int64_t n = t->n;
  /* prefix sums of m, m y, m y y^T with y = x - box centre (smaller magnitudes) */
  double c0[3];
  for (int d = 0; d < 3; d++) c0[d] = (double)t->lo[d] + 0.5 * (double)t->span;
  double* P = (double*)calloc(((size_t)n + 1) * MOM, sizeof(double));
  for (int64_t i = 0; i < n; i++) {
    int64_t s = t->perm[i];
    double m = masses[s];
    double y[3] = {(double)pts[3 * s] - c0[0], (double)pts[3 * s + 1] - c0[1], (double)pts[3 * s + 2] - c0[2]};
    double v[MOM] = {m, m * y[0], m * y[1], m * y[2], m * y[0] * y[0], m * y[1] * y[1], m * y[2] * y[2],
                     m * y[0] * y[1], m * y[0] * y[2], m * y[1] * y[2]};
    for (int c = 0; c < MOM; c++) P[MOM * (i + 1) + c] = P[MOM * i + c] + v[c];
  }
  for (int64_t k = 0; k < t->nn; k++) {
    double v[MOM];
    for (int c = 0; c < MOM; c++) v[c] = P[MOM * t->end[k] + c] - P[MOM * t->start[k] + c];
    double M = v[0];
    double* o = &mom[MOM * k];
    o[0] = M;
    if (M != 0.0) {
      double Y[3] = {v[1] / M, v[2] / M, v[3] / M};
      for (int d = 0; d < 3; d++) o[1 + d] = Y[d] + c0[d];
      o[4] = v[4] - M * Y[0] * Y[0];
      o[5] = v[5] - M * Y[1] * Y[1];
      o[6] = v[6] - M * Y[2] * Y[2];
      o[7] = v[7] - M * Y[0] * Y[1];
      o[8] = v[8] - M * Y[0] * Y[2];
      o[9] = v[9] - M * Y[1] * Y[2];
    } else {
      for (int d = 0; d < 3; d++) o[1 + d] = (double)t->center[3 * k + d];
      for (int c = 4; c < MOM; c++) o[c] = 0.0;
    }
  }
  free(P);
}

/* S x for the packed symmetric S = (xx, yy, zz, xy, xz, yz) */
static void sym_mul(const double* S, const double* x, double* o) {
  o[0] = S[0] * x[0] + S[3] * x[1] + S[4] * x[2];
  o[1] = S[3] * x[0] + S[1] * x[1] + S[5] * x[2];
  o[2] = S[4] * x[0] + S[5] * x[1] + S[2] * x[2];
}

/*
 * Quadrupole correction of the softened far field about the COM, the exact
 * second-order Taylor term of sum_k m_k phi(x + X - x_k) with
 * phi(r) = -r (r^2 + eps^2)^{-3/2}:
 *   a_q = h^{-5/2} (3 S x + 1.5 tr(S) x) - 7.5 (x^T S x) h^{-7/2} x,  h = |x|^2 + eps^2
 * (x = q - X). Plummer softening only (no cutoff attenuation).
 */
static void quad_force(const double* x, const double* S, double eps, double* acc) {
  double h = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + eps * eps + 1e-12;
  double ih = 1.0 / h;
  double ir = 1.0 / sqrt(h);
  double ir5 = ir * ih * ih;
  double Sx[3];
  sym_mul(S, x, Sx);
  double tr = S[0] + S[1] + S[2];
  double xSx = x[0] * Sx[0] + x[1] * Sx[1] + x[2] * Sx[2];
  for (int d = 0; d < 3; d++) acc[d] += ir5 * (3.0 * Sx[d] + 1.5 * tr * x[d]) - 7.5 * xSx * ir5 * ih * x[d];
}

/* J w for the quadrupole term (J symmetric), and G = sym(d(w . a_q)/dS), the
 * symmetric part of the gradient w.r.t. the full matrix S, packed
 * (G00, G11, G22, G01, G02, G12): for S = sum m y y^T, dL/dy = 2 m G y and
 * dL/dm = y^T G y. */
static void quad_vjp(const double* x, const double* S, const double* w, double eps, double* jw,
                     double* gS) {
  double h = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + eps * eps + 1e-12;
  double ih = 1.0 / h;
  double ir = 1.0 / sqrt(h);
  double ir5 = ir * ih * ih, ir7 = ir5 * ih, ir9 = ir7 * ih;
  double Sx[3], Sw[3];
  sym_mul(S, x, Sx);
  sym_mul(S, w, Sw);
  double tr = S[0] + S[1] + S[2];
  double xSx = x[0] * Sx[0] + x[1] * Sx[1] + x[2] * Sx[2];
  double xw = x[0] * w[0] + x[1] * w[1] + x[2] * w[2];
  double Sxw = Sx[0] * w[0] + Sx[1] * w[1] + Sx[2] * w[2];
  for (int d = 0; d < 3; d++) {
    jw[d] += ir5 * (3.0 * Sw[d] + 1.5 * tr * w[d]) - 5.0 * ir7 * xw * (3.0 * Sx[d] + 1.5 * tr * x[d]) -
             7.5 * ir7 * xSx * w[d] - 7.5 * x[d] * (2.0 * ir7 * Sxw - 7.0 * ir9 * xSx * xw);
  }
  if (gS) {
    /* d(w.a_q)/dS_ij = 1.5 h^-5/2 (w_i x_j + x_i w_j) + 1.5 h^-5/2 (x.w) delta_ij - 7.5 h^-7/2 (x.w) x_i x_j */
    double a = 1.5 * ir5, b = 1.5 * ir5 * xw, c = 7.5 * ir7 * xw;
    gS[0] += a * 2.0 * w[0] * x[0] + b - c * x[0] * x[0];
    gS[1] += a * 2.0 * w[1] * x[1] + b - c * x[1] * x[1];
    gS[2] += a * 2.0 * w[2] * x[2] + b - c * x[2] * x[2];
    gS[3] += a * (w[0] * x[1] + x[0] * w[1]) - c * x[0] * x[1];
    gS[4] += a * (w[0] * x[2] + x[0] * w[2]) - c * x[0] * x[2];
    gS[5] += a * (w[1] * x[2] + x[1] * w[2]) - c * x[1] * x[2];
  }
}

/* The GPU's float COM for node k from double moments. */
static void com_float(const double* mom, int64_t k, float* X, float* M) {
  *M = (float)mom[MOM * k];
  for (int d = 0; d < 3; d++) X[d] = (float)mom[MOM * k + 1 + d];
}

/*
 * Periodic and short-range settings of the native walk (the CUDA walk's
 * sbh_native_params.periodic / box_length / prune_radius):
 *   periodic: displacements take the minimum image in a cube of side box
 *     (minImageDisplacement, include/kernel.h:27-39), and the opening test
 *     and prune use the cell centre's image nearest the group box's centre;
 *   prune_r2 > 0: a node whose cell lies farther than sqrt(prune_r2) from
 *     the group box is skipped (octree8_should_prune, src/sbh_ffi.cu:1903-1948,
 *     for a group), with the half side taken as diag * 0.2887.
 */
static int g_orc_periodic = 0;
static float g_orc_box = 1.0f, g_orc_inv_box = 1.0f, g_orc_prune_r2 = 0.0f;
void orc_native_set_periodic(int on, float box, float prune_radius) {
  g_orc_periodic = on;
  g_orc_box = on ? box : 1.0f;
  g_orc_inv_box = 1.0f / g_orc_box;
  g_orc_prune_r2 = prune_radius * prune_radius;
}

static void native_mi(double* r) {
  if (!g_orc_periodic) return;
  double L = (double)g_orc_box;
  for (int d = 0; d < 3; d++) r[d] -= L * floor(r[d] / L + 0.5);
}

/* The cell centre of node k (its image nearest the group box when periodic). */
static void native_cell(const NativeTree* t, int64_t k, const float* gmin, const float* gmax, float* C) {
  for (int d = 0; d < 3; d++) {
    C[d] = t->center[3 * k + d];
    if (g_orc_periodic) {
      float bc = (gmin[d] + gmax[d]) * 0.5f;
      float kk = rintf((bc - C[d]) * g_orc_inv_box);
      C[d] = C[d] + g_orc_box * kk;
    }
  }
}

static int native_prune(const NativeTree* t, int64_t k, const float* C, const float* gmin, const float* gmax) {
  if (!(g_orc_prune_r2 > 0.0f)) return 0;
  float half = (t->side[k] * 1.7320508f) * 0.2887f;
  float tt[3];
  for (int d = 0; d < 3; d++) {
    float a = gmin[d] - (C[d] + half), b = (C[d] - half) - gmax[d];
    float m = a > b ? a : b;
    tt[d] = m > 0.0f ? m : 0.0f;
  }
  float d2 = tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2];
  return d2 > g_orc_prune_r2;
}

/*
 * Multipole acceptance for target group box [gmin, gmax] (float, no fused
 * operations): the reference's rule |q - cell centre| / diag >= beta
 * (include/tree3d.h:134-153, src/sbh_ffi.cu:1878-1893; beta = 1/theta) made
 * to hold for every target in the box:
 *   accept node k iff dist^2(box, cell centre C) > (side * sqrt(3) * beta)^2.
 * The multipole is expanded about the COM.
 */
static int native_accept(const NativeTree* t, int64_t k, const float* C, const float* gmin,
                         const float* gmax, float beta, float* d2_out, float* rc2_out) {
  float rc = t->side[k] * 1.7320508f * beta;
  float tt[3];
  for (int d = 0; d < 3; d++) {
    float a = gmin[d] - C[d], b = C[d] - gmax[d];
    float m = a > b ? a : b;
    tt[d] = m > 0.0f ? m : 0.0f;
  }
  float d2 = tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2];
  float rc2 = rc * rc;
  *d2_out = d2;
  *rc2_out = rc2;
  return d2 > rc2;
}

/*
 * Far-field order of an accepted node (the CUDA walk's quad_order): with a
 * quadrupole radius q > 0 the quadrupole is added only when the opening
 * distance^2 is below (q*q) * rc^2, in float; q = 0 adds it everywhere.
 */
static float g_orc_quad_g = 0.0f;
void orc_native_set_quadrupole_radius(float q) { g_orc_quad_g = q > 0.0f ? q * q : 0.0f; }

static int native_quad_order(float d2, float rc2) {
  return !(g_orc_quad_g > 0.0f) || d2 < g_orc_quad_g * rc2;
}

static float g_orc_quad_lin2 = 0.0f; /* kappa^2 in float, as the CUDA walk holds it */
void orc_native_set_quad_linear(float kappa) { g_orc_quad_lin2 = kappa > 0.0f ? kappa * kappa : 0.0f; }

/* Far-entry flags of the plan (NativeTree.far_quad). */
#define QUAD_NONE 0
#define QUAD_EXACT 1
#define QUAD_LINEAR 2

/* Group centre c = (gmin + gmax) / 2 and squared half diagonal rg2 of a
 * group box, in float with one rounding per operation (the CUDA walk's
 * order); the quadrupole of an accepted node is linearized about c when
 * rg2 <= kappa^2 |c - cell centre|^2. */
static void group_centre(const float* gmin, const float* gmax, float* c4) {
  float hd[3];
  for (int d = 0; d < 3; d++) {
    c4[d] = 0.5f * (gmin[d] + gmax[d]);
    hd[d] = 0.5f * (gmax[d] - gmin[d]);
  }
  c4[3] = (hd[0] * hd[0] + hd[1] * hd[1]) + hd[2] * hd[2];
}

static int quad_linear(const float* c4, const float* cell) {
  if (!(g_orc_quad_lin2 > 0.0f)) return 0;
  float dx = c4[0] - cell[0], dy = c4[1] - cell[1], dz = c4[2] - cell[2];
  float R2 = (dx * dx + dy * dy) + dz * dz;
  return c4[3] <= g_orc_quad_lin2 * R2;
}


/*
 * Target groups cut from the tree. For every node holding more than G
 * particles its children are taken in order; each maximal run of
 * consecutive children that hold at most G particles each is one range of
 * sorted particles, cut into chunks of G (the last one shorter). Children
 * with more than G particles are handled the same way one level down; a leaf
 * with more than G particles (coincident points) and a root holding at most G
 * are cut into chunks of G directly. Every group lies inside the cell of a
 * node with more than G particles, so its bounding box stays compact, and
 * the chunks fill the walk's lanes better than one group per child run.
 * Writes group starts/ends (sorted positions) and returns the count.
 */
static int64_t emit_chunks(int64_t s0, int64_t s1, int G, int64_t* gs, int64_t* ge, int64_t ng) {
  for (int64_t s = s0; s < s1; s += G) {
    gs[ng] = s;
    ge[ng] = s + G < s1 ? s + G : s1;
    ng++;
  }
  return ng;
}

static int64_t native_node_groups(const NativeTree* t, int G, int64_t* gs, int64_t* ge) {
  int64_t ng = 0;
  for (int64_t k = 0; k < t->nn; k++) {
    int32_t cnt = t->end[k] - t->start[k];
    int is_leaf = (k + 1 >= t->nn) || (t->skip[k] == k + 1);
    int is_root = t->level[k] == 0;
    if (is_leaf || cnt <= G) {
      if (is_root || (is_leaf && cnt > G)) ng = emit_chunks(t->start[k], t->end[k], G, gs, ge, ng);
      continue;
    }
    /* children of k: k+1, skip[k+1], ... until skip[k] */
    int64_t run_s = -1, run_e = -1;
    for (int64_t c = k + 1; c < t->skip[k]; c = t->skip[c]) {
      if (t->end[c] - t->start[c] > G) {
        if (run_s >= 0) ng = emit_chunks(run_s, run_e, G, gs, ge, ng);
        run_s = -1;
        continue;
      }
      if (run_s < 0) run_s = t->start[c];
      run_e = t->end[c];
    }
    if (run_s >= 0) ng = emit_chunks(run_s, run_e, G, gs, ge, ng);
  }
  return ng;
}

int g_orc_group_mode = 1; /* 1: groups cut from the tree (the CUDA walk's definition), 0: runs of G sorted particles */
void orc_native_set_group_mode(int mode) { g_orc_group_mode = mode; }

int64_t orc_native_plan(void* h, const float* pts, const float* masses, double beta,
                        int group_size) {
  NativeTree* t = (NativeTree*)h;
  int64_t n = t->n;
  free(t->far_off);
  free(t->far_idx);
  free(t->far_quad);
  free(t->far_coef);
  free(t->near_coef);
  t->far_coef = t->near_coef = NULL;
  free(t->near_off);
  free(t->near_idx);
  t->group_size = group_size;
  free(t->gstart);
  free(t->gend);
  free(t->gcen);
  t->gstart = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  t->gend = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  int64_t ng;
  if (g_orc_group_mode == 1) {
    ng = native_node_groups(t, group_size, t->gstart, t->gend);
  } else {
    ng = (n + group_size - 1) / group_size;
    for (int64_t g = 0; g < ng; g++) {
      t->gstart[g] = g * group_size;
      t->gend[g] = g * group_size + group_size < n ? g * group_size + group_size : n;
    }
  }
  t->ngroups = ng;
  t->gcen = (float*)malloc(sizeof(float) * 4 * (ng > 0 ? ng : 1));
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  float fbeta = (float)beta;
  int64_t fcap = 1 << 20, ncap = 1 << 18;
  t->far_idx = (int32_t*)malloc(sizeof(int32_t) * fcap);
  t->far_quad = (uint8_t*)malloc(fcap);
  t->near_idx = (int32_t*)malloc(sizeof(int32_t) * ncap);
  t->far_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  t->near_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  int64_t nf = 0, nr = 0, total = 0;
  for (int64_t g = 0; g < ng; g++) {
    t->far_off[g] = nf;
    t->near_off[g] = nr;
    int64_t s0 = t->gstart[g], s1 = t->gend[g];
    float gmin[3] = {INFINITY, INFINITY, INFINITY}, gmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = s0; i < s1; i++)
      for (int d = 0; d < 3; d++) {
        float v = pts[3 * t->perm[i] + d];
        gmin[d] = fminf(gmin[d], v);
        gmax[d] = fmaxf(gmax[d], v);
      }
    group_centre(gmin, gmax, &t->gcen[4 * g]);
    int64_t k = 0, cnt_int = 0;
    while (k < t->nn) {
      float X[3], M, C[3];
      com_float(mom, k, X, &M);
      native_cell(t, k, gmin, gmax, C);
      if (M == 0.0f || native_prune(t, k, C, gmin, gmax)) {
        k = t->skip[k];
        continue;
      }
      int is_leaf = (k + 1 >= t->nn) || (t->skip[k] == k + 1);
      float d2, rc2;
      if (native_accept(t, k, C, gmin, gmax, fbeta, &d2, &rc2)) {
        if (nf == fcap) {
          fcap *= 2;
          t->far_idx = (int32_t*)realloc(t->far_idx, sizeof(int32_t) * fcap);
          t->far_quad = (uint8_t*)realloc(t->far_quad, fcap);
        }
        t->far_quad[nf] = (uint8_t)(!native_quad_order(d2, rc2) ? QUAD_NONE
                                    : quad_linear(&t->gcen[4 * g], C) ? QUAD_LINEAR : QUAD_EXACT);
        t->far_idx[nf++] = (int32_t)k;
        cnt_int += 1;
        k = t->skip[k];
      } else if (is_leaf) {
        if (nr == ncap) {
          ncap *= 2;
          t->near_idx = (int32_t*)realloc(t->near_idx, sizeof(int32_t) * ncap);
        }
        t->near_idx[nr++] = (int32_t)k;
        cnt_int += t->end[k] - t->start[k];
        k = t->skip[k];
      } else {
        k = k + 1;
      }
    }
    total += cnt_int * (s1 - s0);
  }
  t->far_off[ng] = nf;
  t->near_off[ng] = nr;
  free(mom);
  return total;
}

/* The quadrupole field a_q(x) of quad_force and its Jacobian J = da_q/dx
 * (symmetric: a_q is the gradient of 0.5 S : grad grad h^{-1/2}),
 * with h = |x|^2 + eps^2 + 1e-12, tau = 1.5 tr S:
 *   J = h^{-5/2} (3 S + tau I) - 15 h^{-7/2} (S x x^T + x x^T S)
 *       - 5 tau h^{-7/2} x x^T - 7.5 (x^T S x) h^{-7/2} I + 52.5 (x^T S x) h^{-9/2} x x^T.
 * J packed (xx, yy, zz, xy, xz, yz). */
static void quad_field_jacobian(const double* x, const double* S, double eps, double* a, double* J) {
  double h = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + eps * eps + 1e-12;
  double ih = 1.0 / h, ir = 1.0 / sqrt(h);
  double ir5 = ir * ih * ih, ir7 = ir5 * ih, ir9 = ir7 * ih;
  double Sx[3];
  sym_mul(S, x, Sx);
  double tau = 1.5 * (S[0] + S[1] + S[2]);
  double xSx = x[0] * Sx[0] + x[1] * Sx[1] + x[2] * Sx[2];
  for (int d = 0; d < 3; d++) a[d] = ir5 * (3.0 * Sx[d] + tau * x[d]) - 7.5 * xSx * ir7 * x[d];
  static const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int e = 0; e < 6; e++) {
    int i = ii[e], j = jj[e];
    double dij = i == j ? 1.0 : 0.0;
    J[e] = ir5 * (3.0 * S[e] + tau * dij) - 15.0 * ir7 * (Sx[i] * x[j] + x[i] * Sx[j]) - 5.0 * tau * ir7 * x[i] * x[j] -
           7.5 * xSx * ir7 * dij + 52.5 * xSx * ir9 * x[i] * x[j];
  }
}

/* Accepted nodes whose quadrupole is taken to first order about the group
 * box centre c instead of at every target: those with r_g <= kappa |c - X|
 * (r_g the half diagonal of the group box, X the node's COM);
 * a_q(x) ~ a_q(c - X) + J(c - X) (x - c). kappa <= 0: never. */
/* The node side of one linearized quadrupole for a group with cotangent sum
 * W = sum_t w_t and V = sym sum_t w_t (x_t - c)^T (packed xx, yy, zz, xy, xz,
 * yz): L = W . a_q(x) + V : J(x) with x = c - X. Returns g = dL/dx (so
 * dL/dX = -g) and G = dL/dS (the symmetric-gradient convention of quad_vjp).
 * With h = |x|^2 + eps^2 + 1e-12 and f_n = h^{-(2n+1)/2}:
 *   G = c1 x x^T + 1.5 f2 (W x^T + x W^T) - 15 f3 (Vx x^T + x (Vx)^T) + c2 I + 3 f2 V,
 *     c1 = -7.5 (W.x) f3 + 52.5 (x.Vx) f4 - 7.5 tr(V) f3, c2 = 1.5 (W.x) f2 - 7.5 (x.Vx) f3 + 1.5 tr(V) f2;
 *   g = J W + 0.5 [ -945 f5 (x.Sx)(x.Vx) x
 *         + 105 f4 ((tr S (x.Vx) + tr V (x.Sx) + 4 Sx.Vx) x + 2 (x.Vx) Sx + 2 (x.Sx) Vx)
 *         - 15 f3 ((tr S tr V + 2 S:V) x + 4 V Sx + 4 S Vx + 2 tr V Sx + 2 tr S Vx) ]
 * (contractions of the third to fifth derivatives of h^{-1/2}). */
static void quad_linear_node_adjoint(const double* x, const double* S, double eps, const double* W, const double* V,
                                     double* g, double* G) {
  double a[3], J[6];
  quad_field_jacobian(x, S, eps, a, J);
  double h = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + eps * eps + 1e-12;
  double ih = 1.0 / h, ir = 1.0 / sqrt(h);
  double f2 = ir * ih * ih, f3 = f2 * ih, f4 = f3 * ih, f5 = f4 * ih;
  double Sx[3], Vx[3], SVx[3], VSx[3], JW[3];
  sym_mul(S, x, Sx);
  sym_mul(V, x, Vx);
  sym_mul(S, Vx, SVx);
  sym_mul(V, Sx, VSx);
  sym_mul(J, W, JW);
  double trS = S[0] + S[1] + S[2], trV = V[0] + V[1] + V[2];
  double xSx = x[0] * Sx[0] + x[1] * Sx[1] + x[2] * Sx[2];
  double xVx = x[0] * Vx[0] + x[1] * Vx[1] + x[2] * Vx[2];
  double SxVx = Sx[0] * Vx[0] + Sx[1] * Vx[1] + Sx[2] * Vx[2];
  double SdV = S[0] * V[0] + S[1] * V[1] + S[2] * V[2] + 2.0 * (S[3] * V[3] + S[4] * V[4] + S[5] * V[5]);
  double Wx = W[0] * x[0] + W[1] * x[1] + W[2] * x[2];
  double kx = -945.0 * f5 * xSx * xVx + 105.0 * f4 * (trS * xVx + trV * xSx + 4.0 * SxVx) -
              15.0 * f3 * (trS * trV + 2.0 * SdV);
  for (int d = 0; d < 3; d++)
    g[d] = JW[d] + 0.5 * (kx * x[d] + 210.0 * f4 * (xVx * Sx[d] + xSx * Vx[d]) -
                          15.0 * f3 * (4.0 * VSx[d] + 4.0 * SVx[d] + 2.0 * trV * Sx[d] + 2.0 * trS * Vx[d]));
  double c1 = -7.5 * Wx * f3 + 52.5 * xVx * f4 - 7.5 * trV * f3;
  double c2 = 1.5 * Wx * f2 - 7.5 * xVx * f3 + 1.5 * trV * f2;
  static const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
  for (int e = 0; e < 6; e++) {
    int i = ii[e], j = jj[e];
    G[e] = c1 * x[i] * x[j] + 1.5 * f2 * (W[i] * x[j] + x[i] * W[j]) - 15.0 * f3 * (Vx[i] * x[j] + x[i] * Vx[j]) +
           (i == j ? c2 : 0.0) + 3.0 * f2 * V[e];
  }
}

/*
 * Evaluate the planned sums with the given (possibly perturbed) positions
 * and masses: topology, sorted order and decisions stay frozen, node
 * moments are recomputed. out_force: n x 3 in input order. If w is given,
 * *loss = sum_i w_i . a_i. quad != 0 adds the quadrupole term of accepted
 * nodes (Plummer softening, cutoff must be <= 0).
 */
void orc_native_eval(void* h, const float* pts, const float* masses, double eps, double cutoff,
                     int quad, double* out_force, const float* w, double* loss) {
  NativeTree* t = (NativeTree*)h;
  int64_t n = t->n;
  SoftParams sp = {eps, cutoff, 0, 1.0};
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  double L = 0.0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : L)
  for (int64_t g = 0; g < t->ngroups; g++) {
    int64_t s0 = t->gstart[g], s1 = t->gend[g];
    const double gc[3] = {t->gcen[4 * g], t->gcen[4 * g + 1], t->gcen[4 * g + 2]};
    for (int64_t i = s0; i < s1; i++) {
      int64_t qi = t->perm[i];
      double q[3] = {pts[3 * qi], pts[3 * qi + 1], pts[3 * qi + 2]};
      double acc[3] = {0, 0, 0};
      for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++) {
        int32_t k = t->far_idx[e];
        const double* o = &mom[MOM * k];
        double r[3] = {q[0] - o[1], q[1] - o[2], q[2] - o[3]};
        double tm[3] = {0, 0, 0};
        native_mi(r);
        soft_force_pair(r, o[0], &sp, tm);
        if (quad && t->far_quad[e] == QUAD_EXACT) {
          quad_force(r, o + 4, eps, tm);
        } else if (quad && t->far_quad[e] == QUAD_LINEAR) {
          /* first order about the (frozen) group centre */
          double rc[3] = {gc[0] - o[1], gc[1] - o[2], gc[2] - o[3]};
          double a[3], J[6], dl[3] = {q[0] - gc[0], q[1] - gc[1], q[2] - gc[2]}, Jd[3];
          quad_field_jacobian(rc, o + 4, eps, a, J);
          sym_mul(J, dl, Jd);
          for (int d = 0; d < 3; d++) tm[d] += a[d] + Jd[d];
        }
        const double cf = t->far_coef ? t->far_coef[e] : 1.0;
        for (int d = 0; d < 3; d++) acc[d] += cf * tm[d];
      }
      for (int64_t e = t->near_off[g]; e < t->near_off[g + 1]; e++) {
        int32_t k = t->near_idx[e];
        double tm[3] = {0, 0, 0};
        for (int32_t j = t->start[k]; j < t->end[k]; j++) {
          int64_t sj = t->perm[j];
          double r[3] = {q[0] - pts[3 * sj], q[1] - pts[3 * sj + 1], q[2] - pts[3 * sj + 2]};
          native_mi(r);
          soft_force_pair(r, masses[sj], &sp, tm);
        }
        const double cf = t->near_coef ? t->near_coef[e] : 1.0;
        for (int d = 0; d < 3; d++) acc[d] += cf * tm[d];
      }
      if (out_force) {
        out_force[3 * qi] = acc[0];
        out_force[3 * qi + 1] = acc[1];
        out_force[3 * qi + 2] = acc[2];
      }
      if (w) L += w[3 * qi] * acc[0] + w[3 * qi + 1] * acc[1] + w[3 * qi + 2] * acc[2];
    }
  }
  if (loss) *loss = L;
  free(mom);
}

/*
 * Exact adjoint of orc_native_eval's loss w.r.t. positions and masses, with
 * the plan frozen:
 *   query side       dL/dx_i += sum_src J_src(x_i)^T w_i
 *   direct sources   dL/dx_j -= m_j J(x_i - x_j)^T w_i,  dL/dm_j += w_i . phi(x_i - x_j)
 *   node moments     A_X[k] = -sum_i J_k(x_i - X_k)^T w_i   (monopole + quadrupole)
 *                    A_M[k] = sum_i w_i . phi(x_i - X_k)
 *                    G_S[k] = sum_i d(w_i . a_q)/dS
 *                    dL/dx_p += (m_p / M_k) A_X[k] + 2 m_p G_S[k] (x_p - X_k)
 *                    dL/dm_p += A_M[k] + A_X[k] . (x_p - X_k) / M_k + (x_p - X_k)^T G_S[k] (x_p - X_k)
 *   for every particle p of node k (S = sum m y y^T about X has zero derivative
 *   through X because sum m y = 0).
 * dx: n x 3, dm: n, input order.
 */
void orc_native_adjoint(void* h, const float* pts, const float* masses, const float* w,
                        double eps, double cutoff, int quad, double* dx, double* dm) {
  NativeTree* t = (NativeTree*)h;
  int64_t n = t->n;
  SoftParams sp = {eps, cutoff, 0, 1.0};
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  double* AX = (double*)calloc((size_t)(t->nn > 0 ? t->nn : 1) * MOM, sizeof(double));
  memset(dx, 0, sizeof(double) * 3 * n);
  memset(dm, 0, sizeof(double) * n);
  for (int64_t g = 0; g < t->ngroups; g++) {
    int64_t s0 = t->gstart[g], s1 = t->gend[g];
    const double gc[3] = {t->gcen[4 * g], t->gcen[4 * g + 1], t->gcen[4 * g + 2]};
    /* linearized quadrupoles: the group's cotangent sums W = sum w, V = sym sum w (x - c)^T; per node
     * dL/dX = -g, dL/dS = G (quad_linear_node_adjoint); each target's query side takes J w */
    double W[3] = {0, 0, 0}, V[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t i = s0; i < s1; i++) {
      int64_t qi = t->perm[i];
      double wi[3] = {w[3 * qi], w[3 * qi + 1], w[3 * qi + 2]};
      double dl[3] = {pts[3 * qi] - gc[0], pts[3 * qi + 1] - gc[1], pts[3 * qi + 2] - gc[2]};
      for (int d = 0; d < 3; d++) W[d] += wi[d];
      V[0] += wi[0] * dl[0];
      V[1] += wi[1] * dl[1];
      V[2] += wi[2] * dl[2];
      V[3] += 0.5 * (wi[0] * dl[1] + wi[1] * dl[0]);
      V[4] += 0.5 * (wi[0] * dl[2] + wi[2] * dl[0]);
      V[5] += 0.5 * (wi[1] * dl[2] + wi[2] * dl[1]);
    }
    for (int64_t e = t->far_off[g]; quad && e < t->far_off[g + 1]; e++) {
      if (t->far_quad[e] != QUAD_LINEAR) continue;
      int32_t k = t->far_idx[e];
      const double* o = &mom[MOM * k];
      double rc[3] = {gc[0] - o[1], gc[1] - o[2], gc[2] - o[3]};
      double gl[3], Gl[6];
      quad_linear_node_adjoint(rc, o + 4, eps, W, V, gl, Gl);
      for (int d = 0; d < 3; d++) AX[MOM * k + 1 + d] -= gl[d];
      for (int c = 0; c < 6; c++) AX[MOM * k + 4 + c] += Gl[c];
    }
    for (int64_t i = s0; i < s1; i++) {
      int64_t qi = t->perm[i];
      double q[3] = {pts[3 * qi], pts[3 * qi + 1], pts[3 * qi + 2]};
      const double wt[3] = {w[3 * qi], w[3 * qi + 1], w[3 * qi + 2]};
      double gq[3] = {0, 0, 0};
      for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++) {
        int32_t k = t->far_idx[e];
        const double* o = &mom[MOM * k];
        double r[3] = {q[0] - o[1], q[1] - o[2], q[2] - o[3]};
        native_mi(r);
        double jt[3] = {0, 0, 0}, f[3] = {0, 0, 0};
        /* a term with coefficient c: every adjoint is linear in the cotangent, so it takes c w */
        const double cf = t->far_coef ? t->far_coef[e] : 1.0;
        const double wi[3] = {cf * wt[0], cf * wt[1], cf * wt[2]};
        soft_force_pair_vjp(r, o[0], wi, &sp, jt);
        soft_force_pair(r, 1.0, &sp, f);
        if (quad && t->far_quad[e] == QUAD_EXACT) quad_vjp(r, o + 4, wi, eps, jt, &AX[MOM * k + 4]);
        if (quad && t->far_quad[e] == QUAD_LINEAR) {
          double rc[3] = {gc[0] - o[1], gc[1] - o[2], gc[2] - o[3]}, a[3], J[6], Jw[3];
          quad_field_jacobian(rc, o + 4, eps, a, J);
          sym_mul(J, wi, Jw);
          for (int d = 0; d < 3; d++) gq[d] += Jw[d];  /* the node side is added per group above */
        }
        for (int d = 0; d < 3; d++) {
          gq[d] += jt[d];
          AX[MOM * k + 1 + d] -= jt[d];
        }
        AX[MOM * k] += wi[0] * f[0] + wi[1] * f[1] + wi[2] * f[2];
      }
      for (int64_t e = t->near_off[g]; e < t->near_off[g + 1]; e++) {
        int32_t k = t->near_idx[e];
        const double cf = t->near_coef ? t->near_coef[e] : 1.0;
        const double wi[3] = {cf * wt[0], cf * wt[1], cf * wt[2]};
        for (int32_t j = t->start[k]; j < t->end[k]; j++) {
          int64_t sj = t->perm[j];
          double r[3] = {q[0] - pts[3 * sj], q[1] - pts[3 * sj + 1], q[2] - pts[3 * sj + 2]};
          native_mi(r);
          double jt[3] = {0, 0, 0}, f[3] = {0, 0, 0};
          soft_force_pair_vjp(r, 1.0, wi, &sp, jt);
          soft_force_pair(r, 1.0, &sp, f);
          for (int d = 0; d < 3; d++) {
            gq[d] += masses[sj] * jt[d];
            dx[3 * sj + d] -= masses[sj] * jt[d];
          }
          dm[sj] += wi[0] * f[0] + wi[1] * f[1] + wi[2] * f[2];
        }
      }
      for (int d = 0; d < 3; d++) dx[3 * qi + d] += gq[d];
    }
  }
  /* push node adjoints down to the particles of each node */
  for (int64_t k = 0; k < t->nn; k++) {
    const double* o = &mom[MOM * k];
    double M = o[0];
    if (M == 0.0) continue;
    const double* A = &AX[MOM * k];
    int any = 0;
    for (int c = 0; c < MOM; c++) any |= A[c] != 0.0;
    if (!any) continue;
    for (int32_t j = t->start[k]; j < t->end[k]; j++) {
      int64_t sj = t->perm[j];
      double mj = masses[sj];
      double y[3] = {(double)pts[3 * sj] - o[1], (double)pts[3 * sj + 1] - o[2], (double)pts[3 * sj + 2] - o[3]};
      double Gy[3];
      sym_mul(A + 4, y, Gy);
      double proj = A[1] * y[0] + A[2] * y[1] + A[3] * y[2];
      for (int d = 0; d < 3; d++) dx[3 * sj + d] += mj / M * A[1 + d] + 2.0 * mj * Gy[d];
      dm[sj] += A[0] + proj / M + (y[0] * Gy[0] + y[1] * Gy[1] + y[2] * Gy[2]);
    }
  }
  free(AX);
  free(mom);
}

/* Plan statistics: number of groups and list lengths. */
/* Far interactions (per target) of the recorded plan that take the quadrupole. */
int64_t orc_native_quadrupole_interactions(void* h) {
  NativeTree* t = (NativeTree*)h;
  int64_t total = 0;
  for (int64_t g = 0; g < t->ngroups; g++) {
    int64_t c = 0;
    for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++) c += t->far_quad[e] != QUAD_NONE;
    total += c * (t->gend[g] - t->gstart[g]);
  }
  return total;
}

/* Far interactions (per target) of the plan with the linearized quadrupole,
 * and the (group, node) pairs they come from. */
void orc_native_linear_quadrupole_counts(void* h, int64_t* per_target, int64_t* pairs) {
  NativeTree* t = (NativeTree*)h;
  int64_t pt = 0, pr = 0;
  for (int64_t g = 0; g < t->ngroups; g++) {
    int64_t c = 0;
    for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++) c += t->far_quad[e] == QUAD_LINEAR;
    pr += c;
    pt += c * (t->gend[g] - t->gstart[g]);
  }
  *per_target = pt;
  *pairs = pr;
}

void orc_native_plan_stats(void* h, int64_t* ngroups, int64_t* nfar, int64_t* nnear) {
  NativeTree* t = (NativeTree*)h;
  *ngroups = t->ngroups;
  *nfar = t->far_off ? t->far_off[t->ngroups] : 0;
  *nnear = t->near_off ? t->near_off[t->ngroups] : 0;
}

/* Per-group list lengths of the recorded plan: far nodes and near particles. */
void orc_native_group_costs(void* h, int64_t* far, int64_t* near_particles) {
  NativeTree* t = (NativeTree*)h;
  for (int64_t g = 0; g < t->ngroups; g++) {
    far[g] = t->far_off[g + 1] - t->far_off[g];
    int64_t np_ = 0;
    for (int64_t e = t->near_off[g]; e < t->near_off[g + 1]; e++) {
      int32_t k = t->near_idx[e];
      np_ += t->end[k] - t->start[k];
    }
    near_particles[g] = np_;
  }
}

/*
 * Central finite differences, in float64, of the frozen-plan loss
 * L = sum_i w_i . a_i of orc_native_eval (the recorded plan: groups, accepted
 * nodes with their quadrupole flags, near leaves) with respect to the
 * position and the mass of each listed particle: step hx in each coordinate,
 * hm_rel * m_k in the mass. Plummer softening only (cutoff 0, no periodic box
 * or prune radius).
 *
 * Under a frozen plan particle k enters L only through
 *   (1) its own row, target k (its far nodes and near pairs);
 *   (2) the near pairs where it is the source, for every target of the groups
 *       whose near list holds k's leaf;
 *   (3) the mass, centroid and second moment of each node that contains it,
 *       for every target of the groups that accept that node.
 * Only these terms are evaluated, at the perturbed position or mass, and each
 * term's difference f(+) - f(-) is taken before it is summed, so the sum does
 * not lose the small per-particle signal to cancellation. A node's perturbed
 * moments are updated about its unperturbed centroid X:
 *   M' = M - m + m',  D = (m' d1 - m d0) / M',  X' = X + D,
 *   S' = S - m d0 d0^T + m' d1 d1^T - M' D D^T,  d0 = x - X, d1 = x' - X.
 * One particle costs about N far-field evaluations per perturbation instead
 * of the whole loss. dx: nidx x 3 and dm: nidx, in the order of idx.
 */
#define FD_MAX_DEPTH 64
static int native_is_leaf(const NativeTree* t, int64_t k) { return (k + 1 >= t->nn) || (t->skip[k] == k + 1); }

/* nodes containing sorted position s, root first; returns their count */
static int native_ancestors(const NativeTree* t, int64_t s, int32_t* anc) {
  int na = 0;
  int64_t a = 0;
  while (na < FD_MAX_DEPTH) {
    anc[na++] = (int32_t)a;
    if (native_is_leaf(t, a)) break;
    int64_t c = a + 1;
    while (c < t->skip[a] && !(t->start[c] <= s && s < t->end[c])) c = t->skip[c];
    if (c >= t->skip[a]) break;
    a = c;
  }
  return na;
}

/* soft_force_pair (no cutoff) plus, with use_quad, quad_force: the same
 * formulas sharing h = |r|^2 + eps^2 + 1e-12 and its inverse square root */
static inline void far_term(const double* r, double M, const double* S, int use_quad, const SoftParams* sp,
                            double* acc) {
  const double h = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + sp->eps * sp->eps + 1e-12;
  const double ir = 1.0 / sqrt(h), ih = ir * ir, ir3 = ir * ih;
  const double c = -M * ir3;
  if (!use_quad) {
    for (int d = 0; d < 3; d++) acc[d] += c * r[d];
    return;
  }
  const double ir5 = ir3 * ih;
  double Sx[3];
  sym_mul(S, r, Sx);
  const double tr = S[0] + S[1] + S[2];
  const double xSx = r[0] * Sx[0] + r[1] * Sx[1] + r[2] * Sx[2];
  for (int d = 0; d < 3; d++) acc[d] += c * r[d] + ir5 * (3.0 * Sx[d] + 1.5 * tr * r[d]) - 7.5 * xSx * ir5 * ih * r[d];
}

/* The field of one planned far entry at q: the monopole, plus the exact
 * quadrupole (QUAD_EXACT) or its first-order expansion about the frozen group
 * centre gc (QUAD_LINEAR). */
static inline void plan_far_term(const double* q, const double* o, int flag, const double* gc, const SoftParams* sp,
                                 double* acc) {
  double r[3] = {q[0] - o[1], q[1] - o[2], q[2] - o[3]};
  far_term(r, o[0], o + 4, flag == QUAD_EXACT, sp, acc);
  if (flag == QUAD_LINEAR) {
    double rc[3] = {gc[0] - o[1], gc[1] - o[2], gc[2] - o[3]}, a[3], J[6], Jd[3];
    double dl[3] = {q[0] - gc[0], q[1] - gc[1], q[2] - gc[2]};
    quad_field_jacobian(rc, o + 4, sp->eps, a, J);
    sym_mul(J, dl, Jd);
    for (int d = 0; d < 3; d++) acc[d] += a[d] + Jd[d];
  }
}

void orc_native_fd(void* h, const float* pts, const float* masses, const float* w, double eps, int quad,
                   const int64_t* idx, int64_t nidx, double hx, double hm_rel, double* dx, double* dm) {
  NativeTree* t = (NativeTree*)h;
  const int64_t n = t->n, nn = t->nn, ng = t->ngroups;
  SoftParams sp = {eps, 0.0, 0, 1.0};
  double* mom = (double*)malloc(sizeof(double) * MOM * (nn > 0 ? nn : 1));
  native_moments(t, pts, masses, mom);
  double* sx = (double*)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
  double* sw = (double*)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
  double* sm = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  int64_t* inv = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  for (int64_t s = 0; s < n; s++) {
    int64_t j = t->perm[s];
    for (int d = 0; d < 3; d++) {
      sx[3 * s + d] = pts[3 * j + d];
      sw[3 * s + d] = w[3 * j + d];
    }
    sm[s] = masses[j];
    inv[j] = s;
  }
  int64_t* grp = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  for (int64_t g = 0; g < ng; g++)
    for (int64_t s = t->gstart[g]; s < t->gend[g]; s++) grp[s] = g;
  /* nodes that contain a listed particle */
  uint8_t* mark = (uint8_t*)calloc(nn > 0 ? nn : 1, 1);
  for (int64_t j = 0; j < nidx; j++) {
    int32_t anc[FD_MAX_DEPTH];
    int na = native_ancestors(t, inv[idx[j]], anc);
    for (int a = 0; a < na; a++) mark[anc[a]] = 1;
  }
  /* for each marked node: the groups accepting it (with the quadrupole flag),
   * and for each marked leaf: the groups whose near list holds it */
  int64_t* foff = (int64_t*)calloc(nn + 1, sizeof(int64_t));
  int64_t* noff = (int64_t*)calloc(nn + 1, sizeof(int64_t));
  for (int64_t g = 0; g < ng; g++) {
    for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++)
      if (mark[t->far_idx[e]]) foff[t->far_idx[e] + 1]++;
    for (int64_t e = t->near_off[g]; e < t->near_off[g + 1]; e++)
      if (mark[t->near_idx[e]]) noff[t->near_idx[e] + 1]++;
  }
  for (int64_t k = 0; k < nn; k++) {
    foff[k + 1] += foff[k];
    noff[k + 1] += noff[k];
  }
  int32_t* fgrp = (int32_t*)malloc(sizeof(int32_t) * (foff[nn] > 0 ? foff[nn] : 1));
  uint8_t* fq = (uint8_t*)malloc(foff[nn] > 0 ? foff[nn] : 1);
  double* fcf = (double*)malloc(sizeof(double) * (foff[nn] > 0 ? foff[nn] : 1));
  int32_t* ngrp = (int32_t*)malloc(sizeof(int32_t) * (noff[nn] > 0 ? noff[nn] : 1));
  double* ncf = (double*)malloc(sizeof(double) * (noff[nn] > 0 ? noff[nn] : 1));
  int64_t* fcur = (int64_t*)malloc(sizeof(int64_t) * (nn > 0 ? nn : 1));
  int64_t* ncur = (int64_t*)malloc(sizeof(int64_t) * (nn > 0 ? nn : 1));
  memcpy(fcur, foff, sizeof(int64_t) * nn);
  memcpy(ncur, noff, sizeof(int64_t) * nn);
  for (int64_t g = 0; g < ng; g++) {
    for (int64_t e = t->far_off[g]; e < t->far_off[g + 1]; e++) {
      int32_t k = t->far_idx[e];
      if (!mark[k]) continue;
      fgrp[fcur[k]] = (int32_t)g;
      fcf[fcur[k]] = t->far_coef ? t->far_coef[e] : 1.0;
      fq[fcur[k]++] = t->far_quad[e];
    }
    for (int64_t e = t->near_off[g]; e < t->near_off[g + 1]; e++) {
      int32_t k = t->near_idx[e];
      if (!mark[k]) continue;
      ncf[ncur[k]] = t->near_coef ? t->near_coef[e] : 1.0;
      ngrp[ncur[k]++] = (int32_t)g;
    }
  }
  free(fcur);
  free(ncur);

#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t j = 0; j < nidx; j++) {
    const int64_t k = idx[j], sk = inv[k], gk = grp[sk];
    int32_t anc[FD_MAX_DEPTH];
    const int na = native_ancestors(t, sk, anc);
    const double xk[3] = {sx[3 * sk], sx[3 * sk + 1], sx[3 * sk + 2]};
    const double mk = sm[sk];
    /* perturbation c (0..2: coordinate c, 3: mass), side p (0: +, 1: -) */
    double xp[4][2][3], mp[4][2];
    for (int c = 0; c < 4; c++)
      for (int p = 0; p < 2; p++) {
        const double sg = p == 0 ? 1.0 : -1.0;
        for (int d = 0; d < 3; d++) xp[c][p][d] = xk[d];
        mp[c][p] = mk;
        if (c < 3)
          xp[c][p][c] += sg * hx;
        else
          mp[c][p] = mk * (1.0 + sg * hm_rel);
      }
    /* perturbed moments of every ancestor: [ancestor][c][p][M, X(3), S(6)] */
    double(*pm)[4][2][MOM] = malloc(sizeof(double) * (size_t)na * 4 * 2 * MOM);
    for (int a = 0; a < na; a++) {
      const double* o = &mom[MOM * anc[a]];
      for (int c = 0; c < 4; c++)
        for (int p = 0; p < 2; p++) {
          double d0[3], d1[3], D[3];
          const double M1 = o[0] - mk + mp[c][p];
          for (int d = 0; d < 3; d++) {
            d0[d] = xk[d] - o[1 + d];
            d1[d] = xp[c][p][d] - o[1 + d];
            D[d] = (mp[c][p] * d1[d] - mk * d0[d]) / M1;
          }
          double* q = pm[a][c][p];
          q[0] = M1;
          for (int d = 0; d < 3; d++) q[1 + d] = o[1 + d] + D[d];
          static const int ii[6] = {0, 1, 2, 0, 0, 1}, jj[6] = {0, 1, 2, 1, 2, 2};
          for (int e = 0; e < 6; e++)
            q[4 + e] = o[4 + e] - mk * d0[ii[e]] * d0[jj[e]] + mp[c][p] * d1[ii[e]] * d1[jj[e]] -
                       M1 * D[ii[e]] * D[jj[e]];
        }
    }
    double D4[4] = {0, 0, 0, 0};
    const double* wk = &sw[3 * sk];
    /* (1) own row */
    for (int64_t e = t->far_off[gk]; e < t->far_off[gk + 1]; e++) {
      const int32_t K = t->far_idx[e];
      int ai = -1;
      for (int a = 0; a < na; a++)
        if (anc[a] == K) ai = a;
      const int uq = quad ? t->far_quad[e] : QUAD_NONE;
      const double gck[3] = {t->gcen[4 * gk], t->gcen[4 * gk + 1], t->gcen[4 * gk + 2]};
      const double cf = t->far_coef ? t->far_coef[e] : 1.0;
      for (int c = 0; c < 4; c++) {
        double f[2][3] = {{0, 0, 0}, {0, 0, 0}};
        for (int p = 0; p < 2; p++) {
          const double* o = ai >= 0 ? pm[ai][c][p] : &mom[MOM * K];
          plan_far_term(xp[c][p], o, uq, gck, &sp, f[p]);
        }
        D4[c] += cf * (wk[0] * (f[0][0] - f[1][0]) + wk[1] * (f[0][1] - f[1][1]) + wk[2] * (f[0][2] - f[1][2]));
      }
    }
    for (int64_t e = t->near_off[gk]; e < t->near_off[gk + 1]; e++) {
      const int32_t K = t->near_idx[e];
      const double cf = t->near_coef ? t->near_coef[e] : 1.0;
      for (int64_t s = t->start[K]; s < t->end[K]; s++) {
        if (s == sk) continue; /* the self pair is zero on both sides */
        for (int c = 0; c < 3; c++) {
          double f[2][3] = {{0, 0, 0}, {0, 0, 0}};
          for (int p = 0; p < 2; p++) {
            double r[3] = {xp[c][p][0] - sx[3 * s], xp[c][p][1] - sx[3 * s + 1], xp[c][p][2] - sx[3 * s + 2]};
            far_term(r, sm[s], NULL, 0, &sp, f[p]);
          }
          D4[c] += cf * (wk[0] * (f[0][0] - f[1][0]) + wk[1] * (f[0][1] - f[1][1]) + wk[2] * (f[0][2] - f[1][2]));
        }
      }
    }
    /* (2) near pairs with k as the source */
    const int32_t leafk = anc[na - 1];
    for (int64_t e = noff[leafk]; e < noff[leafk + 1]; e++) {
      const int64_t g = ngrp[e];
      const double cf = ncf[e];
      for (int64_t s = t->gstart[g]; s < t->gend[g]; s++) {
        if (s == sk) continue;
        const double* ws = &sw[3 * s];
        for (int c = 0; c < 4; c++) {
          double f[2][3] = {{0, 0, 0}, {0, 0, 0}};
          for (int p = 0; p < 2; p++) {
            double r[3] = {sx[3 * s] - xp[c][p][0], sx[3 * s + 1] - xp[c][p][1], sx[3 * s + 2] - xp[c][p][2]};
            far_term(r, mp[c][p], NULL, 0, &sp, f[p]);
          }
          D4[c] += cf * (ws[0] * (f[0][0] - f[1][0]) + ws[1] * (f[0][1] - f[1][1]) + ws[2] * (f[0][2] - f[1][2]));
        }
      }
    }
    /* (3) the moments of k's ancestors, for the targets that accept them */
    for (int a = 0; a < na; a++) {
      const int32_t A = anc[a];
      for (int64_t e = foff[A]; e < foff[A + 1]; e++) {
        const int64_t g = fgrp[e];
        const double cf = fcf[e];
        const int uq = quad ? fq[e] : QUAD_NONE;
        const double gcg[3] = {t->gcen[4 * g], t->gcen[4 * g + 1], t->gcen[4 * g + 2]};
        for (int64_t s = t->gstart[g]; s < t->gend[g]; s++) {
          if (s == sk) continue; /* target k's row is term (1) */
          const double* ws = &sw[3 * s];
          for (int c = 0; c < 4; c++) {
            double f[2][3] = {{0, 0, 0}, {0, 0, 0}};
            for (int p = 0; p < 2; p++) plan_far_term(&sx[3 * s], pm[a][c][p], uq, gcg, &sp, f[p]);
            D4[c] += cf * (ws[0] * (f[0][0] - f[1][0]) + ws[1] * (f[0][1] - f[1][1]) + ws[2] * (f[0][2] - f[1][2]));
          }
        }
      }
    }
    for (int c = 0; c < 3; c++) dx[3 * j + c] = D4[c] / (2.0 * hx);
    dm[j] = mk != 0.0 ? D4[3] / (2.0 * hm_rel * mk) : 0.0;
    free(pm);
  }
  free(fgrp);
  free(fq);
  free(fcf);
  free(ngrp);
  free(ncf);
  free(foff);
  free(noff);
  free(mark);
  free(grp);
  free(inv);
  free(sm);
  free(sw);
  free(sx);
  free(mom);
}

/*
 * Winding number of external queries on the native tree, as the CUDA
 * sbh_native_winding_number walks it (a single-system tree built with
 * normals): the queries are sorted by the 63-bit Morton key of their position
 * in the tree's box (clamped to it, IEEE double quantisation), stably by
 * index, and cut into groups of 32 consecutive sorted queries; each group's
 * box takes the opening test of the gravity walk (no quadrupole, no prune).
 * Accepted nodes contribute (sum_p m_p n_p) . (X - q) K(|X - q|) with X the
 * node's COM, near sources m n . (p - q) K(|p - q|), K(r) = 1 / (4 pi (r^3 +
 * 1e-5)) (signedSolidAngle, include/kernel.h:73-80). Sums in double.
 */
#define WN_GROUP 32
#define WN_K4PI 0.07957747154594767

static double wn_kernel_d(double r2) {
  double r = sqrt(r2);
  return WN_K4PI / (r2 * r + 1e-5);
}

int64_t orc_native_wn_plan(void* h, const float* pts, const float* masses, const float* queries, int64_t nq,
                           double beta) {
  NativeTree* t = (NativeTree*)h;
  free(t->wn_qperm);
  free(t->wn_far_off);
  free(t->wn_near_off);
  free(t->wn_far_idx);
  free(t->wn_near_idx);
  t->wn_nq = nq;
  double scale = 2097152.0 / (double)t->span;
  uint64_t* kv = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (nq > 0 ? nq : 1));
  for (int64_t i = 0; i < nq; i++) {
    uint64_t key = 0;
    for (int d = 0; d < 3; d++) {
      double tq = ((double)queries[3 * i + d] - (double)t->lo[d]) * scale;
      double f = floor(tq);
      uint64_t qv = !(f >= 0.0) ? 0 : (f > 2097151.0 ? 2097151u : (uint64_t)f);
      for (int b = 0; b < 21; b++) key |= ((qv >> b) & 1ull) << (3 * b + d);
    }
    kv[2 * i] = key;
    kv[2 * i + 1] = (uint64_t)i;
  }
  qsort(kv, (size_t)nq, 2 * sizeof(uint64_t), cmp_key_idx);
  t->wn_qperm = (int64_t*)malloc(sizeof(int64_t) * (nq > 0 ? nq : 1));
  for (int64_t i = 0; i < nq; i++) t->wn_qperm[i] = (int64_t)kv[2 * i + 1];
  free(kv);
  int64_t ng = (nq + WN_GROUP - 1) / WN_GROUP;
  t->wn_ngroups = ng;
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  float fbeta = (float)beta;
  int64_t fcap = 1 << 16, ncap = 1 << 16, nf = 0, nr = 0, total = 0;
  t->wn_far_idx = (int32_t*)malloc(sizeof(int32_t) * fcap);
  t->wn_near_idx = (int32_t*)malloc(sizeof(int32_t) * ncap);
  t->wn_far_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  t->wn_near_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  for (int64_t g = 0; g < ng; g++) {
    t->wn_far_off[g] = nf;
    t->wn_near_off[g] = nr;
    int64_t s0 = g * WN_GROUP, s1 = s0 + WN_GROUP < nq ? s0 + WN_GROUP : nq;
    float gmin[3] = {INFINITY, INFINITY, INFINITY}, gmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = s0; i < s1; i++)
      for (int d = 0; d < 3; d++) {
        float v = queries[3 * t->wn_qperm[i] + d];
        gmin[d] = fminf(gmin[d], v);
        gmax[d] = fmaxf(gmax[d], v);
      }
    int64_t k = 0, cnt = 0;
    while (k < t->nn) {
      float X[3], M, C[3];
      com_float(mom, k, X, &M);
      native_cell(t, k, gmin, gmax, C);
      if (M == 0.0f) {
        k = t->skip[k];
        continue;
      }
      int is_leaf = (k + 1 >= t->nn) || (t->skip[k] == k + 1);
      float d2, rc2;
      if (native_accept(t, k, C, gmin, gmax, fbeta, &d2, &rc2)) {
        if (nf == fcap) t->wn_far_idx = (int32_t*)realloc(t->wn_far_idx, sizeof(int32_t) * (fcap *= 2));
        t->wn_far_idx[nf++] = (int32_t)k;
        cnt += 1;
        k = t->skip[k];
      } else if (is_leaf) {
        if (nr == ncap) t->wn_near_idx = (int32_t*)realloc(t->wn_near_idx, sizeof(int32_t) * (ncap *= 2));
        t->wn_near_idx[nr++] = (int32_t)k;
        cnt += t->end[k] - t->start[k];
        k = t->skip[k];
      } else {
        k = k + 1;
      }
    }
    total += cnt * (s1 - s0);
  }
  t->wn_far_off[ng] = nf;
  t->wn_near_off[ng] = nr;
  free(mom);
  return total;
}

/* node sums of m n (nn x 3) in double, by prefix sums over the sorted order */
static double* wn_node_normals(const NativeTree* t, const float* normals, const float* masses) {
  double* P = (double*)calloc(((size_t)t->n + 1) * 3, sizeof(double));
  for (int64_t i = 0; i < t->n; i++) {
    int64_t s = t->perm[i];
    for (int d = 0; d < 3; d++) P[3 * (i + 1) + d] = P[3 * i + d] + (double)masses[s] * normals[3 * s + d];
  }
  double* Nm = (double*)malloc(sizeof(double) * 3 * (t->nn > 0 ? t->nn : 1));
  for (int64_t k = 0; k < t->nn; k++)
    for (int d = 0; d < 3; d++) Nm[3 * k + d] = P[3 * t->end[k] + d] - P[3 * t->start[k] + d];
  free(P);
  return Nm;
}

/* out[i] = winding number at query i (input order) with the recorded plan */
void orc_native_wn_eval(void* h, const float* pts, const float* normals, const float* masses, const float* queries,
                        double* out) {
  NativeTree* t = (NativeTree*)h;
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  double* Nm = wn_node_normals(t, normals, masses);
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t g = 0; g < t->wn_ngroups; g++) {
    int64_t s0 = g * WN_GROUP, s1 = s0 + WN_GROUP < t->wn_nq ? s0 + WN_GROUP : t->wn_nq;
    for (int64_t i = s0; i < s1; i++) {
      int64_t qi = t->wn_qperm[i];
      double q[3] = {queries[3 * qi], queries[3 * qi + 1], queries[3 * qi + 2]};
      double acc = 0.0;
      for (int64_t e = t->wn_far_off[g]; e < t->wn_far_off[g + 1]; e++) {
        int32_t k = t->wn_far_idx[e];
        const double* o = &mom[MOM * k];
        double d[3] = {o[1] - q[0], o[2] - q[1], o[3] - q[2]};
        acc += (Nm[3 * k] * d[0] + Nm[3 * k + 1] * d[1] + Nm[3 * k + 2] * d[2]) *
               wn_kernel_d(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      }
      for (int64_t e = t->wn_near_off[g]; e < t->wn_near_off[g + 1]; e++) {
        int32_t k = t->wn_near_idx[e];
        for (int32_t j = t->start[k]; j < t->end[k]; j++) {
          int64_t sj = t->perm[j];
          double d[3] = {pts[3 * sj] - q[0], pts[3 * sj + 1] - q[1], pts[3 * sj + 2] - q[2]};
          acc += masses[sj] * (normals[3 * sj] * d[0] + normals[3 * sj + 1] * d[1] + normals[3 * sj + 2] * d[2]) *
                 wn_kernel_d(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        }
      }
      out[qi] = acc;
    }
  }
  free(Nm);
  free(mom);
}

/*
 * Adjoint of orc_native_wn_eval's L = sum_i u_i w(q_i) with the plan frozen.
 * For one term f = a . d K(r), d = p - q, r = |d| (a = m n for a source, the
 * node's sum m n for a far node, p its COM): df/dd = a K - 3 (a . d) r K^2 d / k4pi
 * (K' = -3 r^2 K^2 / k4pi for K = k4pi / (r^3 + 1e-5)), df/dq = -df/dd, df/dp =
 * df/dd, df/da = d K. A source takes dp += u df/dd, dn += u m d K,
 * dm += u (n . d) K; a node's dL/dX = sum u df/dd and dL/d(sum m n) = sum u d K
 * reach its particles through X = sum m p / M and sum m n:
 * dp += (m / M) dL/dX, dn += m dL/dN, dm += dL/dX . (p - X) / M + n . dL/dN.
 * dq: nq x 3 (input order), dp, dn: n x 3, dm: n.
 */
void orc_native_wn_adjoint(void* h, const float* pts, const float* normals, const float* masses,
                           const float* queries, const float* u, double* dq, double* dp, double* dn, double* dm) {
  NativeTree* t = (NativeTree*)h;
  int64_t n = t->n;
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  double* Nm = wn_node_normals(t, normals, masses);
  double* A = (double*)calloc((size_t)(t->nn > 0 ? t->nn : 1) * 6, sizeof(double)); /* dL/dX, dL/dN */
  memset(dq, 0, sizeof(double) * 3 * t->wn_nq);
  memset(dp, 0, sizeof(double) * 3 * n);
  memset(dn, 0, sizeof(double) * 3 * n);
  memset(dm, 0, sizeof(double) * n);
  for (int64_t g = 0; g < t->wn_ngroups; g++) {
    int64_t s0 = g * WN_GROUP, s1 = s0 + WN_GROUP < t->wn_nq ? s0 + WN_GROUP : t->wn_nq;
    for (int64_t i = s0; i < s1; i++) {
      int64_t qi = t->wn_qperm[i];
      double q[3] = {queries[3 * qi], queries[3 * qi + 1], queries[3 * qi + 2]};
      double ui = u[qi];
      for (int64_t e = t->wn_far_off[g]; e < t->wn_far_off[g + 1]; e++) {
        int32_t k = t->wn_far_idx[e];
        const double* o = &mom[MOM * k];
        double d[3] = {o[1] - q[0], o[2] - q[1], o[3] - q[2]};
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2), K = wn_kernel_d(r2);
        double ad = Nm[3 * k] * d[0] + Nm[3 * k + 1] * d[1] + Nm[3 * k + 2] * d[2];
        for (int c = 0; c < 3; c++) {
          double g1 = Nm[3 * k + c] * K - 3.0 * ad * r * K * K * d[c] / WN_K4PI;
          dq[3 * qi + c] -= ui * g1;
          A[6 * k + c] += ui * g1;
          A[6 * k + 3 + c] += ui * d[c] * K;
        }
      }
      for (int64_t e = t->wn_near_off[g]; e < t->wn_near_off[g + 1]; e++) {
        int32_t k = t->wn_near_idx[e];
        for (int32_t j = t->start[k]; j < t->end[k]; j++) {
          int64_t sj = t->perm[j];
          double d[3] = {pts[3 * sj] - q[0], pts[3 * sj + 1] - q[1], pts[3 * sj + 2] - q[2]};
          double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2], r = sqrt(r2), K = wn_kernel_d(r2);
          double mj = masses[sj];
          double nd = normals[3 * sj] * d[0] + normals[3 * sj + 1] * d[1] + normals[3 * sj + 2] * d[2];
          for (int c = 0; c < 3; c++) {
            double g1 = mj * (normals[3 * sj + c] * K - 3.0 * nd * r * K * K * d[c] / WN_K4PI);
            dq[3 * qi + c] -= ui * g1;
            dp[3 * sj + c] += ui * g1;
            dn[3 * sj + c] += ui * mj * d[c] * K;
          }
          dm[sj] += ui * nd * K;
        }
      }
    }
  }
  for (int64_t k = 0; k < t->nn; k++) {
    const double* o = &mom[MOM * k];
    double M = o[0];
    if (M == 0.0) continue;
    const double* a = &A[6 * k];
    int any = 0;
    for (int c = 0; c < 6; c++) any |= a[c] != 0.0;
    if (!any) continue;
    for (int32_t j = t->start[k]; j < t->end[k]; j++) {
      int64_t sj = t->perm[j];
      double mj = masses[sj];
      double y[3] = {(double)pts[3 * sj] - o[1], (double)pts[3 * sj + 1] - o[2], (double)pts[3 * sj + 2] - o[3]};
      for (int c = 0; c < 3; c++) {
        dp[3 * sj + c] += mj / M * a[c];
        dn[3 * sj + c] += mj * a[3 + c];
      }
      dm[sj] += (a[0] * y[0] + a[1] * y[1] + a[2] * y[2]) / M + normals[3 * sj] * a[3] + normals[3 * sj + 1] * a[4] +
                normals[3 * sj + 2] * a[5];
    }
  }
  free(A);
  free(Nm);
  free(mom);
}

/* ------------------------------------------------------------------------ */
/* Native stochastic Barnes-Hut (the CUDA sbh_native_stochastic_force)        */
/* ------------------------------------------------------------------------ */
/*
 * The estimator, per target group (groups cut from the tree as in
 * native_node_groups), on the GPU's own node records:
 *   1. coarse part: the group walk at beta_c (a node is accepted when the
 *      group box clears beta_c diagonals of its cell centre); accepted
 *      nodes add their monopole + quadrupole about the COM at every target,
 *      the leaves reached add their particles directly;
 *   2. weights: an accepted node n gets w_n = M r_g^3 / r^5 (r_g^2 = tr S / M,
 *      r^2 = dist(group box, COM)^2 + eps^2: the size of the octupole the
 *      quadrupole leaves out at the box's nearest point), or 0 when the group box already
 *      clears beta_f diagonals of the cell (there the refined walk below is
 *      the node's own quadrupole);
 *   3. K stratified draws u_k = (k + U_k) W / K, W = sum w_n, each picking
 *      the node whose interval [running sum before n, after n) holds u_k,
 *      U_k uniform from (seed, input index of the group's first target, k);
 *      the group's targets share the draws;
 *   4. a node drawn c times adds c W / (K len_n) (R_n - F_n) at every target,
 *      R_n the group walk of n's subtree at beta_f and F_n the node's
 *      monopole + quadrupole, len_n its interval's length.
 * E[estimate] = coarse part + sum over w_n > 0 of (R_n - F_n) = the group walk
 * at beta_f with the quadrupole at every accepted node. Weights, running sums
 * and draws are computed in float with the CUDA kernel's operation order
 * (IEEE +, *, /, sqrt, no contraction), so the same nodes are drawn; forces
 * are summed in double.
 */
typedef struct {
  float com[4], cell[4], quad[4], quad2[4];
  int32_t topo[4];
} OrcNodeRec;

#define ORC_LEAF_FLAG 0x100

/* SplitMix64's output function (Steele, Lea and Flood, "Fast splittable
 * pseudorandom number generators", OOPSLA 2014) on a Weyl sequence indexed by
 * (index, draw): 24 bits -> a float in [0, 1). */
static float orc_stoch_uniform(uint64_t seed, uint64_t idx, int k) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (idx * 64u + (uint64_t)k + 1u);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (float)(z >> 40) * 0x1p-24f;
}

static int stoch_accept(const float* cell, const float* lo, const float* hi, float beta) {
  float rc = cell[3] * beta;
  float tt[3];
  for (int d = 0; d < 3; d++) {
    float a = lo[d] - cell[d], b = cell[d] - hi[d];
    float m = a > b ? a : b;
    tt[d] = m > 0.0f ? m : 0.0f;
  }
  float d2 = tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2];
  return d2 > rc * rc;
}

/* w_n for the group with box [lo, hi]: r is the distance from the box to the COM */
static float stoch_weight(const OrcNodeRec* nd, const float* lo, const float* hi, float beta_f, float eps2) {
  if (stoch_accept(nd->cell, lo, hi, beta_f)) return 0.0f;
  float trS = (nd->quad[0] + nd->quad[1]) + nd->quad[2];
  trS = trS > 0.0f ? trS : 0.0f;
  float t3[3];
  for (int d = 0; d < 3; d++) {
    float a = lo[d] - nd->com[d], b = nd->com[d] - hi[d];
    float m = a > b ? a : b;
    t3[d] = m > 0.0f ? m : 0.0f;
  }
  float r2 = ((t3[0] * t3[0] + t3[1] * t3[1]) + t3[2] * t3[2]) + eps2;
  float num = trS * sqrtf(trS / nd->com[3]);
  float den = (r2 * r2) * sqrtf(r2);
  return num / den;
}

/* monopole + quadrupole of node c at q, h = |r|^2 + eps2 */
static void stoch_node_far(const OrcNodeRec* c, const float* q, double eps2, double* acc) {
  double r[3] = {(double)q[0] - c->com[0], (double)q[1] - c->com[1], (double)q[2] - c->com[2]};
  double h = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + eps2;
  double ih = 1.0 / h, ir = 1.0 / sqrt(h);
  double ir3 = ir * ih, ir5 = ir3 * ih;
  double S[6] = {c->quad[0], c->quad[1], c->quad[2], c->quad[3], c->quad2[0], c->quad2[1]};
  double Sx[3];
  sym_mul(S, r, Sx);
  double tr = S[0] + S[1] + S[2];
  double xSx = r[0] * Sx[0] + r[1] * Sx[1] + r[2] * Sx[2];
  double M = c->com[3];
  for (int d = 0; d < 3; d++)
    acc[d] += -M * ir3 * r[d] + ir5 * (3.0 * Sx[d] + 1.5 * tr * r[d]) - 7.5 * xSx * ir5 * ih * r[d];
}

static void stoch_direct(const float* sp, int32_t s0, int32_t s1, const float* q, double eps2, double* acc) {
  for (int32_t j = s0; j < s1; j++) {
    double r[3] = {(double)q[0] - sp[4 * j], (double)q[1] - sp[4 * j + 1], (double)q[2] - sp[4 * j + 2]};
    double h = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + eps2;
    double c = -(double)sp[4 * j + 3] / (h * sqrt(h));
    for (int d = 0; d < 3; d++) acc[d] += c * r[d];
  }
}

/* R_n(q) - F_n(q): the group walk of node n0's subtree at beta_f (n0 itself
 * is opened: its weight is positive only when the box does not clear it)
 * minus n0's monopole + quadrupole, at target q. */
static void stoch_correction(const OrcNodeRec* N, const float* sp, int32_t n0, const float* lo, const float* hi,
                             const float* q, float beta_f, double eps2, double* d3) {
  double R[3] = {0, 0, 0}, F[3] = {0, 0, 0};
  const OrcNodeRec* nd = &N[n0];
  if (nd->topo[3] & ORC_LEAF_FLAG) {
    stoch_direct(sp, nd->topo[0], nd->topo[1], q, eps2, R);
  } else {
    for (int32_t k = n0 + 1; k < nd->topo[2];) {
      const OrcNodeRec* c = &N[k];
      if (c->com[3] == 0.0f) {
        k = c->topo[2];
      } else if (stoch_accept(c->cell, lo, hi, beta_f)) {
        stoch_node_far(c, q, eps2, R);
        k = c->topo[2];
      } else if (c->topo[3] & ORC_LEAF_FLAG) {
        stoch_direct(sp, c->topo[0], c->topo[1], q, eps2, R);
        k = c->topo[2];
      } else {
        k = k + 1;
      }
    }
  }
  stoch_node_far(nd, q, eps2, F);
  for (int d = 0; d < 3; d++) d3[d] = R[d] - F[d];
}

/*
 * n targets = the sorted sources sp (n x 4: x, y, z, m), perm: sorted ->
 * input index, nodes: nn records of 80 bytes (the GPU export). out (the
 * estimate) and expect (its expectation, the group walk at beta_f), n x 3 in
 * input order; either may be NULL. Returns the number of subtree walks
 * (distinct drawn nodes) over all groups.
 */
int64_t orc_native_stochastic(const float* sp, const uint32_t* perm, int64_t n, const void* nodes, int64_t nn,
                              int group_size, float beta_c, float beta_f, float eps2, int K, uint64_t seed,
                              double* out, double* expect) {
  const OrcNodeRec* N = (const OrcNodeRec*)nodes;
  NativeTree t;
  memset(&t, 0, sizeof(t));
  t.n = n;
  t.nn = nn;
  size_t cap = nn > 0 ? (size_t)nn : 1;
  t.start = (int32_t*)malloc(sizeof(int32_t) * cap);
  t.end = (int32_t*)malloc(sizeof(int32_t) * cap);
  t.skip = (int32_t*)malloc(sizeof(int32_t) * cap);
  t.level = (int8_t*)malloc(cap);
  for (int64_t k = 0; k < nn; k++) {
    t.start[k] = N[k].topo[0];
    t.end[k] = N[k].topo[1];
    t.skip[k] = N[k].topo[2];
    t.level[k] = (int8_t)(N[k].topo[3] & 0xff);
  }
  int64_t* gs = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  int64_t* ge = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  int64_t ng = native_node_groups(&t, group_size, gs, ge);
  double de2 = (double)eps2;
  int64_t walks = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : walks)
  for (int64_t g = 0; g < ng; g++) {
    int64_t s0 = gs[g], s1 = ge[g], m = s1 - s0;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = s0; i < s1; i++)
      for (int d = 0; d < 3; d++) {
        lo[d] = fminf(lo[d], sp[4 * i + d]);
        hi[d] = fmaxf(hi[d], sp[4 * i + d]);
      }
    int64_t r0 = 0, r1 = nn; /* the root whose particles hold the group */
    for (int64_t k = 0; k < nn; k = N[k].topo[2]) {
      if (N[k].topo[0] <= s0 && s0 < N[k].topo[1]) {
        r0 = k;
        r1 = N[k].topo[2];
        break;
      }
    }
    double* fc = (double*)calloc((size_t)m * 3, sizeof(double));
    double* ex = (double*)calloc((size_t)m * 3, sizeof(double));
    double* co = (double*)calloc((size_t)m * 3, sizeof(double));
    float W = 0.0f;
    /* pass 1: coarse part, W, the expectation of the correction */
    for (int64_t k = r0; k < r1;) {
      const OrcNodeRec* c = &N[k];
      int leaf = (c->topo[3] & ORC_LEAF_FLAG) != 0;
      if (c->com[3] == 0.0f) {
        k = c->topo[2];
      } else if (stoch_accept(c->cell, lo, hi, beta_c)) {
        float w = stoch_weight(c, lo, hi, beta_f, eps2);
        W = W + w;
        for (int64_t i = s0; i < s1; i++) {
          const float q[3] = {sp[4 * i], sp[4 * i + 1], sp[4 * i + 2]};
          stoch_node_far(c, q, de2, &fc[3 * (i - s0)]);
          if (w > 0.0f && expect) {
            double d3[3];
            stoch_correction(N, sp, (int32_t)k, lo, hi, q, beta_f, de2, d3);
            for (int d = 0; d < 3; d++) ex[3 * (i - s0) + d] += d3[d];
          }
        }
        k = c->topo[2];
      } else if (leaf) {
        for (int64_t i = s0; i < s1; i++) {
          const float q[3] = {sp[4 * i], sp[4 * i + 1], sp[4 * i + 2]};
          stoch_direct(sp, c->topo[0], c->topo[1], q, de2, &fc[3 * (i - s0)]);
        }
        k = c->topo[2];
      } else {
        k = k + 1;
      }
    }
    /* pass 2: the K stratified draws, shared by the group's targets */
    if (W > 0.0f) {
      const uint64_t gi = perm[s0];
      float P = 0.0f, step = W / (float)K;
      int kk = 0;
      float u = ((float)kk + orc_stoch_uniform(seed, gi, kk)) * step;
      int32_t last = -1;
      float last_scale = 0.0f;
      for (int64_t k = r0; k < r1 && kk < K;) {
        const OrcNodeRec* c = &N[k];
        int leaf = (c->topo[3] & ORC_LEAF_FLAG) != 0;
        if (c->com[3] == 0.0f) {
          k = c->topo[2];
        } else if (stoch_accept(c->cell, lo, hi, beta_c)) {
          float w = stoch_weight(c, lo, hi, beta_f, eps2);
          float Pn = P + w;
          if (Pn > P) { /* a weight that rounding absorbed has an empty interval */
            float scale = W / ((float)K * (Pn - P));
            int cnt = 0;
            last = (int32_t)k;
            last_scale = scale;
            while (kk < K && u < Pn) {
              cnt++;
              kk++;
              if (kk < K) u = ((float)kk + orc_stoch_uniform(seed, gi, kk)) * step;
            }
            if (cnt > 0) {
              float sc = (float)cnt * scale;
              walks++;
              for (int64_t i = s0; i < s1; i++) {
                const float q[3] = {sp[4 * i], sp[4 * i + 1], sp[4 * i + 2]};
                double d3[3];
                stoch_correction(N, sp, (int32_t)k, lo, hi, q, beta_f, de2, d3);
                for (int d = 0; d < 3; d++) co[3 * (i - s0) + d] += d3[d] * (double)sc;
              }
            }
          }
          P = Pn;
          k = c->topo[2];
        } else if (leaf) {
          k = c->topo[2];
        } else {
          k = k + 1;
        }
      }
      /* draws at the top end that rounding left past the last interval */
      if (kk < K && last >= 0) {
        float sc = (float)(K - kk) * last_scale;
        walks++;
        for (int64_t i = s0; i < s1; i++) {
          const float q[3] = {sp[4 * i], sp[4 * i + 1], sp[4 * i + 2]};
          double d3[3];
          stoch_correction(N, sp, last, lo, hi, q, beta_f, de2, d3);
          for (int d = 0; d < 3; d++) co[3 * (i - s0) + d] += d3[d] * (double)sc;
        }
      }
    }
    for (int64_t i = s0; i < s1; i++) {
      const uint64_t oi = perm[i];
      for (int d = 0; d < 3; d++) {
        if (out) out[3 * oi + d] = fc[3 * (i - s0) + d] + co[3 * (i - s0) + d];
        if (expect) expect[3 * oi + d] = fc[3 * (i - s0) + d] + ex[3 * (i - s0) + d];
      }
    }
    free(fc);
    free(ex);
    free(co);
  }
  free(gs);
  free(ge);
  free(t.start);
  free(t.end);
  free(t.skip);
  free(t.level);
  return walks;
}

/* Node records in the GPU's 80-byte layout from the oracle's tree (float
 * COM and second moments of the double sums; cell centre and diagonal
 * side * sqrt(3); topology with the leaf flag), for CPU-side runs of
 * orc_native_stochastic. */
void orc_native_records(void* h, const float* pts, const float* masses, void* out) {
  NativeTree* t = (NativeTree*)h;
  double* mom = (double*)malloc(sizeof(double) * MOM * (t->nn > 0 ? t->nn : 1));
  native_moments(t, pts, masses, mom);
  OrcNodeRec* R = (OrcNodeRec*)out;
  for (int64_t k = 0; k < t->nn; k++) {
    const double* o = &mom[MOM * k];
    OrcNodeRec r;
    memset(&r, 0, sizeof(r));
    for (int d = 0; d < 3; d++) r.com[d] = (float)o[1 + d];
    r.com[3] = (float)o[0];
    for (int d = 0; d < 3; d++) r.cell[d] = t->center[3 * k + d];
    r.cell[3] = t->side[k] * 1.7320508f;
    for (int c = 0; c < 4; c++) r.quad[c] = (float)o[4 + c];
    r.quad2[0] = (float)o[8];
    r.quad2[1] = (float)o[9];
    r.topo[0] = t->start[k];
    r.topo[1] = t->end[k];
    r.topo[2] = t->skip[k];
    r.topo[3] = (int32_t)t->level[k] | (native_is_leaf(t, k) ? ORC_LEAF_FLAG : 0);
    R[k] = r;
  }
  free(mom);
}

/*
 * The stochastic estimator of orc_native_stochastic as a frozen plan of the
 * tree `h` (built on the same points: its topology is the GPU's), for
 * orc_native_eval, orc_native_adjoint and orc_native_fd with quad = 1:
 * per group, far entries (node, exact quadrupole, coefficient) and near
 * entries (leaf, coefficient). The decisions and draws are taken on the given
 * node records (the GPU export) exactly as orc_native_stochastic takes them:
 *   coarse cut: accepted nodes (+1), leaves reached (+1);
 *   a node n drawn c times with interval scale s: its quadrupole (-c s) and
 *   the group walk of its subtree at beta_f (accepted nodes and leaves, +c s).
 * The adjoint of this plan is the VJP of the estimate with the draws held
 * fixed. Returns the number of far + near entries.
 */
typedef struct {
  int64_t nf, nr, fcap, ncap;
  int32_t *fi, *ni;
  double *fc, *nc;
} StochPlan;

static void sp_far(StochPlan* P, int32_t k, double c) {
  if (P->nf == P->fcap) {
    P->fcap = P->fcap ? 2 * P->fcap : 1024;
    P->fi = (int32_t*)realloc(P->fi, sizeof(int32_t) * P->fcap);
    P->fc = (double*)realloc(P->fc, sizeof(double) * P->fcap);
  }
  P->fi[P->nf] = k;
  P->fc[P->nf++] = c;
}

static void sp_near(StochPlan* P, int32_t k, double c) {
  if (P->nr == P->ncap) {
    P->ncap = P->ncap ? 2 * P->ncap : 1024;
    P->ni = (int32_t*)realloc(P->ni, sizeof(int32_t) * P->ncap);
    P->nc = (double*)realloc(P->nc, sizeof(double) * P->ncap);
  }
  P->ni[P->nr] = k;
  P->nc[P->nr++] = c;
}

/* the entries of sc (R_n - F_n) for a group with box [lo, hi] */
static void sp_refine(StochPlan* P, const OrcNodeRec* N, int32_t n0, double sc, const float* lo, const float* hi,
                      float beta_f) {
  sp_far(P, n0, -sc);
  const OrcNodeRec* nd = &N[n0];
  if (nd->topo[3] & ORC_LEAF_FLAG) {
    sp_near(P, n0, sc);
    return;
  }
  for (int32_t k = n0 + 1; k < nd->topo[2];) {
    const OrcNodeRec* c = &N[k];
    if (c->com[3] == 0.0f) {
      k = c->topo[2];
    } else if (stoch_accept(c->cell, lo, hi, beta_f)) {
      sp_far(P, k, sc);
      k = c->topo[2];
    } else if (c->topo[3] & ORC_LEAF_FLAG) {
      sp_near(P, k, sc);
      k = c->topo[2];
    } else {
      k = k + 1;
    }
  }
}

int64_t orc_native_stochastic_plan(void* h, const float* pts, const void* nodes, int group_size, float beta_c,
                                   float beta_f, float eps2, int K, uint64_t seed) {
  NativeTree* t = (NativeTree*)h;
  const OrcNodeRec* N = (const OrcNodeRec*)nodes;
  const int64_t n = t->n, nn = t->nn;
  free(t->far_off);
  free(t->far_idx);
  free(t->far_quad);
  free(t->far_coef);
  free(t->near_off);
  free(t->near_idx);
  free(t->near_coef);
  free(t->gstart);
  free(t->gend);
  free(t->gcen);
  t->group_size = group_size;
  t->gstart = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  t->gend = (int64_t*)malloc(sizeof(int64_t) * (n + 2));
  const int64_t ng = native_node_groups(t, group_size, t->gstart, t->gend);
  t->ngroups = ng;
  t->gcen = (float*)malloc(sizeof(float) * 4 * (ng > 0 ? ng : 1));
  t->far_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  t->near_off = (int64_t*)malloc(sizeof(int64_t) * (ng + 1));
  StochPlan P;
  memset(&P, 0, sizeof(P));
  for (int64_t g = 0; g < ng; g++) {
    t->far_off[g] = P.nf;
    t->near_off[g] = P.nr;
    const int64_t s0 = t->gstart[g], s1 = t->gend[g];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = s0; i < s1; i++)
      for (int d = 0; d < 3; d++) {
        lo[d] = fminf(lo[d], pts[3 * t->perm[i] + d]);
        hi[d] = fmaxf(hi[d], pts[3 * t->perm[i] + d]);
      }
    float* c4 = &t->gcen[4 * g];
    group_centre(lo, hi, c4);
    int64_t r0 = 0, r1 = nn;
    for (int64_t k = 0; k < nn; k = N[k].topo[2]) {
      if (N[k].topo[0] <= s0 && s0 < N[k].topo[1]) {
        r0 = k;
        r1 = N[k].topo[2];
        break;
      }
    }
    float W = 0.0f;
    for (int64_t k = r0; k < r1;) {
      const OrcNodeRec* c = &N[k];
      if (c->com[3] == 0.0f) {
        k = c->topo[2];
      } else if (stoch_accept(c->cell, lo, hi, beta_c)) {
        sp_far(&P, (int32_t)k, 1.0);
        W = W + stoch_weight(c, lo, hi, beta_f, eps2);
        k = c->topo[2];
      } else if (c->topo[3] & ORC_LEAF_FLAG) {
        sp_near(&P, (int32_t)k, 1.0);
        k = c->topo[2];
      } else {
        k = k + 1;
      }
    }
    if (W > 0.0f) {
      const uint64_t gi = t->perm[s0];
      float Pr = 0.0f, step = W / (float)K;
      int kk = 0;
      float u = ((float)kk + orc_stoch_uniform(seed, gi, kk)) * step;
      int32_t last = -1;
      float last_scale = 0.0f;
      for (int64_t k = r0; k < r1 && kk < K;) {
        const OrcNodeRec* c = &N[k];
        if (c->com[3] == 0.0f) {
          k = c->topo[2];
        } else if (stoch_accept(c->cell, lo, hi, beta_c)) {
          float Pn = Pr + stoch_weight(c, lo, hi, beta_f, eps2);
          if (Pn > Pr) {
            float scale = W / ((float)K * (Pn - Pr));
            int cnt = 0;
            last = (int32_t)k;
            last_scale = scale;
            while (kk < K && u < Pn) {
              cnt++;
              kk++;
              if (kk < K) u = ((float)kk + orc_stoch_uniform(seed, gi, kk)) * step;
            }
            if (cnt > 0) sp_refine(&P, N, (int32_t)k, (double)((float)cnt * scale), lo, hi, beta_f);
          }
          Pr = Pn;
          k = c->topo[2];
        } else if (c->topo[3] & ORC_LEAF_FLAG) {
          k = c->topo[2];
        } else {
          k = k + 1;
        }
      }
      if (kk < K && last >= 0) sp_refine(&P, N, last, (double)((float)(K - kk) * last_scale), lo, hi, beta_f);
    }
  }
  t->far_off[ng] = P.nf;
  t->near_off[ng] = P.nr;
  t->far_idx = P.fi ? P.fi : (int32_t*)malloc(sizeof(int32_t));
  t->far_coef = P.fc ? P.fc : (double*)malloc(sizeof(double));
  t->near_idx = P.ni ? P.ni : (int32_t*)malloc(sizeof(int32_t));
  t->near_coef = P.nc ? P.nc : (double*)malloc(sizeof(double));
  t->far_quad = (uint8_t*)malloc(P.nf > 0 ? (size_t)P.nf : 1);
  memset(t->far_quad, QUAD_EXACT, P.nf > 0 ? (size_t)P.nf : 1);
  return P.nf + P.nr;
}
