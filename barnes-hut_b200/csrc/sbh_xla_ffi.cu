// XLA custom-call handlers with the reference's symbol names, argument
// order and attribute names (src/sbh_ffi.cu:3580-3947), so that the
// reference's python/jax_sbh_ffi.py can load this library and register its
// targets unchanged (jax.ffi.pycapsule(lib.<symbol>), api_version=1).
//
// Each handler decodes XLA's call frame (buffers, scalar attributes looked up
// by name, the stream from the execution context), checks shapes with the
// reference's messages, and forwards to the library's C entry point. Scratch
// for the builds and the traversals' status word comes from XLA's device
// allocator when the runtime provides it (XLA_FFI_DeviceMemory_Allocate; it
// is released when the handler returns, stream-ordered like XLA's own
// scratch), else from cudaMallocAsync / cudaFreeAsync on the handler's
// stream. Nothing here synchronises the stream.
//
// Host-only code: no kernels are defined in this file.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "sbh_b200.h"
#include "sbh_xla_ffi_abi.h"
#include "sbh_xla_ffi.h"

#define SBH_FFI_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr size_t kCallFrameMinSize = offsetof(XLA_FFI_CallFrame, attrs) + sizeof(XLA_FFI_Attrs);

// True when the runtime's API table reaches past `field` and sets it.
#define SBH_API_HAS(api, field)                                                                   \
  ((api) != nullptr && (api)->struct_size >= offsetof(XLA_FFI_Api, field) + sizeof((api)->field) && \
   (api)->field != nullptr)

struct Buf {
  const XLA_FFI_Buffer* b = nullptr;
  int64_t dim(int i) const { return i < b->rank ? b->dims[i] : 1; }
  int64_t count() const {
    int64_t c = 1;
    for (int64_t i = 0; i < b->rank; i++) c *= b->dims[i];
    return c;
  }
  float* f() const { return static_cast<float*>(b->data); }
  void* p() const { return b->data; }
};

const char* dtype_name(XLA_FFI_DataType t) {
  switch (t) {
    case XLA_FFI_DataType_F32:
      return "f32";
    case XLA_FFI_DataType_U8:
      return "u8";
    case XLA_FFI_DataType_S32:
      return "s32";
    default:
      return "other";
  }
}

// One handler invocation: decoding helpers, error construction, scratch.
class Call {
 public:
  explicit Call(XLA_FFI_CallFrame* cf) : cf_(cf), api_(cf->api) {}
  ~Call() {
    for (const Scratch& s : scratch_) {
      if (s.from_xla) {
        XLA_FFI_DeviceMemory_Free_Args a{sizeof(a), nullptr, cf_->ctx, s.bytes, s.ptr};
        XLA_FFI_Error* e = api_->XLA_FFI_DeviceMemory_Free(&a);
        (void)e;  // a failed free leaves the error object to XLA's allocator
      } else {
        cudaFreeAsync(s.ptr, stream_);
      }
    }
  }

  XLA_FFI_Error* error(XLA_FFI_Error_Code code, const std::string& msg) {
    if (!SBH_API_HAS(api_, XLA_FFI_Error_Create)) return nullptr;
    XLA_FFI_Error_Create_Args a{sizeof(a), nullptr, msg.c_str(), code};
    return api_->XLA_FFI_Error_Create(&a);
  }
  XLA_FFI_Error* invalid(const std::string& msg) { return error(XLA_FFI_Error_Code_INVALID_ARGUMENT, msg); }
  // The first decoding failure (kept until the handler returns it).
  XLA_FFI_Error* err() { return err_; }

  // Maps a C entry point's status to XLA's error convention.
  XLA_FFI_Error* rc(int status) {
    if (status == SBH_OK) return nullptr;
    std::string msg = sbh_last_error();
    return error(status == SBH_ERR_INVALID_ARGUMENT ? XLA_FFI_Error_Code_INVALID_ARGUMENT : XLA_FFI_Error_Code_INTERNAL,
                 msg);
  }

  bool counts(int64_t nargs, int64_t nrets, int64_t nattrs) {
    if (cf_->args.size != nargs)
      return fail("Wrong number of arguments: expected " + std::to_string(nargs) + " but got " +
                  std::to_string(cf_->args.size));
    if (cf_->rets.size != nrets)
      return fail("Wrong number of results: expected " + std::to_string(nrets) + " but got " +
                  std::to_string(cf_->rets.size));
    if (cf_->attrs.size != nattrs)
      return fail("Wrong number of attributes: expected " + std::to_string(nattrs) + " but got " +
                  std::to_string(cf_->attrs.size));
    return true;
  }

  bool arg(int i, XLA_FFI_DataType dt, int rank, Buf* out) {
    if (cf_->args.types[i] != XLA_FFI_ArgType_BUFFER) return fail("argument " + std::to_string(i) + " is not a buffer");
    return buffer(static_cast<const XLA_FFI_Buffer*>(cf_->args.args[i]), "argument", i, dt, rank, out);
  }
  bool ret(int i, XLA_FFI_DataType dt, int rank, Buf* out) {
    if (cf_->rets.types[i] != XLA_FFI_RetType_BUFFER) return fail("result " + std::to_string(i) + " is not a buffer");
    return buffer(static_cast<const XLA_FFI_Buffer*>(cf_->rets.rets[i]), "result", i, dt, rank, out);
  }

  bool i32(const char* name, int* v) {
    const XLA_FFI_Scalar* s = scalar(name, XLA_FFI_DataType_S32);
    if (!s) return false;
    std::memcpy(v, s->value, sizeof(int32_t));
    return true;
  }
  bool f32(const char* name, float* v) {
    const XLA_FFI_Scalar* s = scalar(name, XLA_FFI_DataType_F32);
    if (!s) return false;
    std::memcpy(v, s->value, sizeof(float));
    return true;
  }

  bool stream(cudaStream_t* s) {
    if (!SBH_API_HAS(api_, XLA_FFI_Stream_Get)) return fail("the XLA runtime provides no stream");
    XLA_FFI_Stream_Get_Args a{sizeof(a), nullptr, cf_->ctx, nullptr};
    if (XLA_FFI_Error* e = api_->XLA_FFI_Stream_Get(&a)) {
      err_ = e;
      return false;
    }
    *s = stream_ = static_cast<cudaStream_t>(a.stream);
    return true;
  }

  // Device scratch of `bytes` (stream() first). Released when the handler
  // returns, in stream order.
  bool scratch(size_t bytes, void** out) {
    if (bytes == 0) bytes = 256;
    if (SBH_API_HAS(api_, XLA_FFI_DeviceMemory_Allocate) &&
        SBH_API_HAS(api_, XLA_FFI_DeviceMemory_Free)) {
      XLA_FFI_DeviceMemory_Allocate_Args a{sizeof(a), nullptr, cf_->ctx, bytes, 256, nullptr};
      if (XLA_FFI_Error* e = api_->XLA_FFI_DeviceMemory_Allocate(&a)) {
        err_ = e;
        return false;
      }
      if (!a.data) return fail(XLA_FFI_Error_Code_RESOURCE_EXHAUSTED, "XLA's allocator returned no memory");
      scratch_.push_back({a.data, bytes, true});
      *out = a.data;
      return true;
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, stream_);
    if (e != cudaSuccess) return fail(XLA_FFI_Error_Code_RESOURCE_EXHAUSTED, cudaGetErrorString(e));
    scratch_.push_back({p, bytes, false});
    *out = p;
    return true;
  }

 private:
  struct Scratch {
    void* ptr;
    size_t bytes;
    bool from_xla;
  };

  bool fail(const std::string& msg) { return fail(XLA_FFI_Error_Code_INVALID_ARGUMENT, msg); }
  bool fail(XLA_FFI_Error_Code code, const std::string& msg) {
    if (!err_) err_ = error(code, msg);
    return false;
  }

  bool buffer(const XLA_FFI_Buffer* b, const char* what, int i, XLA_FFI_DataType dt, int rank, Buf* out) {
    if (!b) return fail(std::string(what) + " " + std::to_string(i) + " is missing");
    if (b->dtype != dt)
      return fail(std::string("Wrong buffer dtype: expected ") + dtype_name(dt) + " but got " + dtype_name(b->dtype) +
                  " (" + what + " " + std::to_string(i) + ")");
    if (b->rank != rank)
      return fail("Wrong buffer rank: expected " + std::to_string(rank) + " but got " + std::to_string(b->rank) + " (" +
                  what + " " + std::to_string(i) + ")");
    out->b = b;
    return true;
  }

  const XLA_FFI_Scalar* scalar(const char* name, XLA_FFI_DataType dt) {
    const size_t len = std::strlen(name);
    for (int64_t k = 0; k < cf_->attrs.size; k++) {
      const XLA_FFI_ByteSpan* nm = cf_->attrs.names[k];
      if (!nm || nm->len != len || std::memcmp(nm->ptr, name, len) != 0) continue;
      if (cf_->attrs.types[k] != XLA_FFI_AttrType_SCALAR) {
        fail(std::string("attribute '") + name + "' is not a scalar");
        return nullptr;
      }
      const XLA_FFI_Scalar* s = static_cast<const XLA_FFI_Scalar*>(cf_->attrs.attrs[k]);
      if (!s || s->dtype != dt) {
        fail(std::string("Wrong scalar data type for attribute '") + name + "': expected " + dtype_name(dt));
        return nullptr;
      }
      return s;
    }
    fail(std::string("missing attribute '") + name + "'");
    return nullptr;
  }

  XLA_FFI_CallFrame* cf_;
  const XLA_FFI_Api* api_;
  XLA_FFI_Error* err_ = nullptr;
  cudaStream_t stream_ = nullptr;
  std::vector<Scratch> scratch_;
};

// Metadata query at registration, stage filter, then the handler's body.
template <typename Body>
XLA_FFI_Error* handle(XLA_FFI_CallFrame* cf, Body body) {
  if (!cf) return nullptr;
  if (cf->extension_start && cf->extension_start->type == XLA_FFI_Extension_Metadata) {
    auto* ext = reinterpret_cast<XLA_FFI_Metadata_Extension*>(cf->extension_start);
    if (ext->metadata) {
      ext->metadata->api_version = XLA_FFI_Api_Version{sizeof(XLA_FFI_Api_Version), nullptr, kXlaFfiApiMajor,
                                                       kXlaFfiApiMinor};
      ext->metadata->traits = 0;
    }
    return nullptr;
  }
  if (cf->struct_size < kCallFrameMinSize) {
    Call c(cf);
    return c.invalid("XLA_FFI_CallFrame is smaller than this handler expects");
  }
  if (cf->stage != XLA_FFI_ExecutionStage_EXECUTE) return nullptr;  // registered for execution only
  Call c(cf);
  return body(c);
}

// --------------------------------------------------------------------------
// shared bodies
// --------------------------------------------------------------------------
XLA_FFI_Error* direct_soft(Call& c, bool vjp) {
  const int na = vjp ? 4 : 3;
  Buf pts, ms, q, cot, out;
  float eps, cut, box;
  int periodic, threads;
  if (!c.counts(na, 1, 5) || !c.arg(0, XLA_FFI_DataType_F32, 2, &pts) || !c.arg(1, XLA_FFI_DataType_F32, 1, &ms) ||
      !c.arg(2, XLA_FFI_DataType_F32, 2, &q) || (vjp && !c.arg(3, XLA_FFI_DataType_F32, 2, &cot)) ||
      !c.ret(0, XLA_FFI_DataType_F32, 2, &out) || !c.f32("softening_scale", &eps) ||
      !c.f32("cutoff_scale", &cut) || !c.i32("periodic", &periodic) || !c.f32("box_length", &box) ||
      !c.i32("threads", &threads))
    return c.err();
  const int64_t n = pts.dim(0), nq = q.dim(0);
  if (pts.dim(1) != 3 || q.dim(1) != 3)
    return c.invalid(vjp ? "points/queries/cotangent must have dim=3" : "points/queries must have dim=3");
  if (vjp && (cot.dim(0) != nq || cot.dim(1) != 3)) return c.invalid("cotangent shape mismatch");
  if (ms.dim(0) != n) return c.invalid("masses length mismatch");
  if (out.dim(0) != nq || out.dim(1) != 3) return c.invalid("out shape mismatch");
  cudaStream_t s;
  if (!c.stream(&s)) return c.err();
  if (vjp)
    return c.rc(sbh_direct_force_soft_vjp(s, pts.f(), ms.f(), n, q.f(), nq, cot.f(), out.f(), eps, cut, periodic, box,
                                          threads));
  return c.rc(sbh_direct_force_soft(s, pts.f(), ms.f(), n, q.f(), nq, out.f(), eps, cut, periodic, box, threads));
}

// points, normals, masses, min_corner, max_corner -> leaf, node, contrib bytes
bool build_inputs(Call& c, Buf* pts, Buf* nrm, Buf* ms, Buf* mn, Buf* mx, Buf* leaf, Buf* node, Buf* con,
                  XLA_FFI_Error** e) {
  if (!c.arg(0, XLA_FFI_DataType_F32, 2, pts) || !c.arg(1, XLA_FFI_DataType_F32, 2, nrm) ||
      !c.arg(2, XLA_FFI_DataType_F32, 1, ms) || !c.arg(3, XLA_FFI_DataType_F32, 1, mn) ||
      !c.arg(4, XLA_FFI_DataType_F32, 1, mx) || !c.ret(0, XLA_FFI_DataType_U8, 1, leaf) ||
      !c.ret(1, XLA_FFI_DataType_U8, 1, node) || !c.ret(2, XLA_FFI_DataType_U8, 1, con)) {
    *e = c.err();
    return false;
  }
  if (pts->dim(1) != 3) *e = c.invalid("points must have shape (N, 3)");
  else if (nrm->dim(1) != 3) *e = c.invalid("normals must have shape (N, 3)");
  else if (pts->dim(0) != nrm->dim(0)) *e = c.invalid("points/normals row mismatch");
  else if (ms->dim(0) != pts->dim(0)) *e = c.invalid("masses must have shape (N,)");
  else if (mn->dim(0) != 3 || mx->dim(0) != 3) *e = c.invalid("min_corner/max_corner must have shape (3,)");
  else return true;
  return false;
}

XLA_FFI_Error* build_level3(Call& c) {
  Buf pts, nrm, ms, mn, mx, leaf, node, con;
  XLA_FFI_Error* e = nullptr;
  if (!c.counts(5, 3, 0)) return c.err();
  if (!build_inputs(c, &pts, &nrm, &ms, &mn, &mx, &leaf, &node, &con, &e)) return e;
  cudaStream_t s;
  void* ws;
  const int64_t n = pts.dim(0);
  size_t wsb = sbh_build_octree_level3_workspace_bytes(n);
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  return c.rc(sbh_build_octree_level3(s, pts.f(), nrm.f(), ms.f(), n, mn.f(), mx.f(), leaf.p(), leaf.count(), node.p(),
                                      node.count(), con.p(), con.count(), ws, wsb));
}

XLA_FFI_Error* build_octree8(Call& c) {
  Buf pts, nrm, ms, mn, mx, leaf, node, con;
  XLA_FFI_Error* e = nullptr;
  int depth;
  if (!c.counts(5, 3, 1) || !c.i32("max_depth", &depth)) return c.err();
  if (!build_inputs(c, &pts, &nrm, &ms, &mn, &mx, &leaf, &node, &con, &e)) return e;
  if (depth < 1 || depth > 10) return c.invalid("max_depth must be in [1, 10]");
  cudaStream_t s;
  void* ws;
  const int64_t n = pts.dim(0);
  size_t wsb = sbh_build_octree8_workspace_bytes(n, depth);
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  return c.rc(sbh_build_octree8(s, pts.f(), nrm.f(), ms.f(), n, mn.f(), mx.f(), depth, leaf.p(), leaf.count(),
                                node.p(), node.count(), con.p(), con.count(), ws, wsb));
}

// Queries of a tree traversal: (nq, dim), output (nq,) or (nq, dim).
bool query_shapes(Call& c, const Buf& q, const Buf& out, int dim, bool vector_out, XLA_FFI_Error** e) {
  if (q.dim(1) != dim) {
    *e = c.invalid(dim == 2 ? "queries dim must be 2" : "queries dim must be 3");
    return false;
  }
  if (out.dim(0) != q.dim(0) || (vector_out && out.dim(1) != dim)) {
    *e = c.invalid("out shape mismatch");
    return false;
  }
  return true;
}

// Node2/Node3 warp-vote BH: kernel 0 gravity, 1 force, 2 softened force.
XLA_FFI_Error* barnes_hut_tree(Call& c, int dim, int kernel) {
  const bool soft = kernel == 2, vec = kernel != 0;
  Buf leaf, node, q, out;
  float beta, eps = 0.f, cut = 1.f, box;
  int periodic, threads;
  if (!c.counts(3, 1, soft ? 6 : 4) || !c.arg(0, XLA_FFI_DataType_U8, 1, &leaf) ||
      !c.arg(1, XLA_FFI_DataType_U8, 1, &node) || !c.arg(2, XLA_FFI_DataType_F32, 2, &q) ||
      !c.ret(0, XLA_FFI_DataType_F32, vec ? 2 : 1, &out) || !c.f32("beta", &beta) ||
      (soft && (!c.f32("softening_scale", &eps) || !c.f32("cutoff_scale", &cut))) ||
      !c.i32("periodic", &periodic) || !c.f32("box_length", &box) || !c.i32("threads", &threads))
    return c.err();
  XLA_FFI_Error* e = nullptr;
  if (!query_shapes(c, q, out, dim, vec, &e)) return e;
  cudaStream_t s;
  void* ws;
  const size_t wsb = sbh_traversal_workspace_bytes();
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  return c.rc(sbh_barnes_hut_tree(s, dim, kernel, leaf.p(), leaf.count(), node.p(), node.count(), q.f(), q.dim(0),
                                  out.f(), beta, eps, cut, periodic, box, threads, ws, wsb));
}

// Node2/Node3 MLPCV: kernel 0 gravity, 1 force, 2 softened force.
XLA_FFI_Error* stochastic_tree(Call& c, int dim, int kernel) {
  const bool soft = kernel == 2, vec = kernel != 0;
  Buf leaf, node, con, q, out;
  float eps = 0.f, cut = 1.f, box;
  int samples, seed, periodic, threads;
  if (!c.counts(4, 1, soft ? 7 : 5) || !c.arg(0, XLA_FFI_DataType_U8, 1, &leaf) ||
      !c.arg(1, XLA_FFI_DataType_U8, 1, &node) || !c.arg(2, XLA_FFI_DataType_U8, 1, &con) ||
      !c.arg(3, XLA_FFI_DataType_F32, 2, &q) || !c.ret(0, XLA_FFI_DataType_F32, vec ? 2 : 1, &out) ||
      !c.i32("samples_per_subdomain", &samples) || !c.i32("seed", &seed) ||
      (soft && (!c.f32("softening_scale", &eps) || !c.f32("cutoff_scale", &cut))) ||
      !c.i32("periodic", &periodic) || !c.f32("box_length", &box) || !c.i32("threads", &threads))
    return c.err();
  XLA_FFI_Error* e = nullptr;
  if (!query_shapes(c, q, out, dim, vec, &e)) return e;
  cudaStream_t s;
  void* ws;
  const size_t wsb = sbh_traversal_workspace_bytes();
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  return c.rc(sbh_stochastic_bh_tree(s, dim, kernel, leaf.p(), leaf.count(), node.p(), node.count(), con.p(),
                                     con.count(), q.f(), q.dim(0), out.f(), samples, seed, eps, cut, periodic, box,
                                     threads, ws, wsb));
}

// octree8 classic BH: plain (gravityGrad), softened, softened VJP.
enum O8Kind { kO8Plain, kO8Soft, kO8SoftVjp };

XLA_FFI_Error* octree8_bh(Call& c, O8Kind kind) {
  const bool soft = kind != kO8Plain, vjp = kind == kO8SoftVjp;
  Buf leaf, node, q, cot, out;
  float beta, eps = 0.f, cut = 1.f, mult = 4.f, box;
  int prune = 0, periodic, threads;
  if (!c.counts(vjp ? 4 : 3, 1, soft ? 8 : 4) || !c.arg(0, XLA_FFI_DataType_U8, 1, &leaf) ||
      !c.arg(1, XLA_FFI_DataType_U8, 1, &node) || !c.arg(2, XLA_FFI_DataType_F32, 2, &q) ||
      (vjp && !c.arg(3, XLA_FFI_DataType_F32, 2, &cot)) || !c.ret(0, XLA_FFI_DataType_F32, 2, &out) ||
      !c.f32("beta", &beta) ||
      (soft && (!c.f32("softening_scale", &eps) || !c.f32("cutoff_scale", &cut) || !c.i32("prune_enabled", &prune) ||
                !c.f32("prune_r_cut_mult", &mult))) ||
      !c.i32("periodic", &periodic) || !c.f32("box_length", &box) || !c.i32("threads", &threads))
    return c.err();
  XLA_FFI_Error* e = nullptr;
  if (!query_shapes(c, q, out, 3, true, &e)) return e;
  if (vjp && (cot.dim(0) != q.dim(0) || cot.dim(1) != 3)) return c.invalid("cotangent shape mismatch");
  cudaStream_t s;
  void* ws;
  const int64_t nq = q.dim(0);
  const size_t wsb = sbh_traversal_ordered_workspace_bytes(nq);  // room to take the queries in Morton order
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  if (kind == kO8Plain)
    return c.rc(sbh_barnes_hut_force_octree8(s, leaf.p(), leaf.count(), node.p(), node.count(), q.f(), nq, out.f(),
                                             beta, periodic, box, threads, ws, wsb));
  if (kind == kO8Soft)
    return c.rc(sbh_barnes_hut_force_octree8_soft(s, leaf.p(), leaf.count(), node.p(), node.count(), q.f(), nq,
                                                  out.f(), beta, eps, cut, prune, mult, periodic, box, threads, ws,
                                                  wsb));
  return c.rc(sbh_barnes_hut_force_octree8_soft_vjp(s, leaf.p(), leaf.count(), node.p(), node.count(), q.f(), nq,
                                                    cot.f(), out.f(), beta, eps, cut, prune, mult, periodic, box,
                                                    threads, ws, wsb));
}

XLA_FFI_Error* octree8_stochastic(Call& c, bool soft, bool vjp) {
  Buf leaf, node, q, cot, out;
  float beta, eps = 0.f, cut = 1.f, mult = 4.f, box;
  int samples, seed, prune = 0, periodic, threads;
  if (!c.counts(vjp ? 4 : 3, 1, soft ? 10 : 6) || !c.arg(0, XLA_FFI_DataType_U8, 1, &leaf) ||
      !c.arg(1, XLA_FFI_DataType_U8, 1, &node) || !c.arg(2, XLA_FFI_DataType_F32, 2, &q) ||
      (vjp && !c.arg(3, XLA_FFI_DataType_F32, 2, &cot)) || !c.ret(0, XLA_FFI_DataType_F32, 2, &out) ||
      !c.i32("samples_per_subdomain", &samples) || !c.i32("seed", &seed) || !c.f32("beta", &beta) ||
      (soft && (!c.f32("softening_scale", &eps) || !c.f32("cutoff_scale", &cut) || !c.i32("prune_enabled", &prune) ||
                !c.f32("prune_r_cut_mult", &mult))) ||
      !c.i32("periodic", &periodic) || !c.f32("box_length", &box) || !c.i32("threads", &threads))
    return c.err();
  XLA_FFI_Error* e = nullptr;
  if (!query_shapes(c, q, out, 3, true, &e)) return e;
  if (vjp && (cot.dim(0) != q.dim(0) || cot.dim(1) != 3)) return c.invalid("cotangent shape mismatch");
  cudaStream_t s;
  void* ws;
  const int64_t nq = q.dim(0);
  const size_t wsb = sbh_traversal_ordered_workspace_bytes(nq);
  if (!c.stream(&s) || !c.scratch(wsb, &ws)) return c.err();
  if (vjp)
    return c.rc(sbh_stochastic_bh_force_octree8_vjp(s, soft ? 1 : 0, leaf.p(), leaf.count(), node.p(), node.count(),
                                                    q.f(), nq, cot.f(), out.f(), samples, seed, beta, eps, cut, prune,
                                                    mult, periodic, box, threads, ws, wsb));
  return c.rc(sbh_stochastic_bh_force_octree8(s, soft ? 1 : 0, leaf.p(), leaf.count(), node.p(), node.count(), q.f(),
                                              nq, out.f(), samples, seed, beta, eps, cut, prune, mult, periodic, box,
                                              threads, ws, wsb));
}

}  // namespace

// --------------------------------------------------------------------------
// the handler symbols (src/sbh_ffi.cu:3580-3947)
// --------------------------------------------------------------------------
SBH_FFI_EXPORT XLA_FFI_Error* sbh_bruteforce_gravity_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) -> XLA_FFI_Error* {
    Buf pts, ms, q, out;
    int periodic, threads;
    float box;
    if (!c.counts(3, 1, 3) || !c.arg(0, XLA_FFI_DataType_F32, 2, &pts) || !c.arg(1, XLA_FFI_DataType_F32, 1, &ms) ||
        !c.arg(2, XLA_FFI_DataType_F32, 2, &q) || !c.ret(0, XLA_FFI_DataType_F32, 1, &out) ||
        !c.i32("periodic", &periodic) || !c.f32("box_length", &box) || !c.i32("threads", &threads))
      return c.err();
    const int64_t n = pts.dim(0), dim = pts.dim(1), nq = q.dim(0);
    if (q.dim(1) != dim) return c.invalid("queries dim mismatch");
    if (ms.dim(0) != n) return c.invalid("masses length mismatch");
    if (dim != 2 && dim != 3) return c.invalid("only dim=2 or dim=3 supported");
    if (out.dim(0) != nq) return c.invalid("out shape mismatch");
    cudaStream_t s;
    if (!c.stream(&s)) return c.err();
    return c.rc(sbh_bruteforce_gravity(s, pts.f(), ms.f(), n, static_cast<int>(dim), q.f(), nq, out.f(), periodic, box,
                                       threads));
  });
}

SBH_FFI_EXPORT XLA_FFI_Error* sbh_direct_force_soft_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return direct_soft(c, false); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_direct_force_soft_vjp_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return direct_soft(c, true); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_build_octree_level3_buffers_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return build_level3(c); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_build_octree8_buffers_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return build_octree8(c); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_gravity_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 2, 0); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 2, 1); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_gravity_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 3, 0); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 3, 1); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_soft_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 2, 2); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_soft_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return barnes_hut_tree(c, 3, 2); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_octree8_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_bh(c, kO8Plain); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_octree8_soft_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_bh(c, kO8Soft); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_barnes_hut_force_octree8_soft_vjp_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_bh(c, kO8SoftVjp); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_gravity_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 2, 0); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_gravity_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 3, 0); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 2, 1); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 3, 1); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_soft_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 2, 2); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_soft_ffi_3d(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return stochastic_tree(c, 3, 2); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_octree8_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_stochastic(c, false, false); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_octree8_soft_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_stochastic(c, true, false); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_octree8_vjp_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_stochastic(c, false, true); });
}
SBH_FFI_EXPORT XLA_FFI_Error* sbh_stochastic_bh_force_octree8_soft_vjp_ffi(XLA_FFI_CallFrame* cf) {
  return handle(cf, [](Call& c) { return octree8_stochastic(c, true, true); });
}
