// Minimal XLA-FFI stand-in, written for this project, so that the reference's
// src/sbh_ffi.cu compiles without jaxlib's headers (jax is not installed in
// this image). The handler functions of the reference take these buffer and
// error types by value; XLA_FFI_DEFINE_HANDLER_SYMBOL expands to nothing, so
// the reference's handlers are plain C++ functions that oracle/ref_gpu_driver.cu
// calls directly.
//
// TEST INFRASTRUCTURE ONLY: used by the oracle's reference build recipe
// (oracle/Makefile) and never by the product library.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

namespace xla {
namespace ffi {

enum DataType { F32 = 0, U8 = 1 };

template <DataType dt>
struct NativeType;
template <>
struct NativeType<F32> {
  typedef float type;
};
template <>
struct NativeType<U8> {
  typedef uint8_t type;
};

struct Dims {
  const int64_t* d;
  size_t n;
  size_t size() const { return n; }
  int64_t operator[](size_t i) const { return d[i]; }
};

template <DataType dt, int rank>
struct Buffer {
  typedef typename NativeType<dt>::type T;
  void* data;
  int64_t dims[4];
  int nd;

  Buffer() : data(nullptr), nd(rank) {
    for (int i = 0; i < 4; i++) dims[i] = 0;
  }
  Buffer(void* p, const int64_t* shape, int ndims) : data(p), nd(ndims) {
    for (int i = 0; i < 4; i++) dims[i] = (i < ndims) ? shape[i] : 0;
  }
  Dims dimensions() const { return Dims{dims, static_cast<size_t>(nd)}; }
  T* typed_data() const { return static_cast<T*>(data); }
  void* untyped_data() const { return data; }
  size_t element_count() const {
    size_t c = 1;
    for (int i = 0; i < nd; i++) c *= static_cast<size_t>(dims[i]);
    return c;
  }
  size_t size_bytes() const { return element_count() * sizeof(T); }
};

template <DataType dt, int rank>
struct ResultBuffer {
  Buffer<dt, rank> buf;
  ResultBuffer() {}
  explicit ResultBuffer(const Buffer<dt, rank>& b) : buf(b) {}
  Buffer<dt, rank>* operator->() { return &buf; }
  const Buffer<dt, rank>* operator->() const { return &buf; }
};

class Error {
 public:
  int code;
  std::string message;
  Error() : code(0) {}
  Error(int c, const char* m) : code(c), message(m ? m : "") {}
  static Error Success() { return Error(); }
  static Error InvalidArgument(const char* m) { return Error(3, m); }
  static Error Internal(const char* m) { return Error(13, m); }
  static Error InvalidArgument(const std::string& m) { return Error(3, m.c_str()); }
  static Error Internal(const std::string& m) { return Error(13, m.c_str()); }
};

template <typename T>
struct PlatformStream {};

}  // namespace ffi
}  // namespace xla

#define XLA_FFI_DEFINE_HANDLER_SYMBOL(...)
