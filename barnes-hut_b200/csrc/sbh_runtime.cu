// Error plumbing, version, layout queries and the device status read-back of
// the sbh_b200 C ABI.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "sbh_common.cuh"

namespace sbh {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    return fail(SBH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  return SBH_OK;
}

}  // namespace sbh

extern "C" {

const char* sbh_last_error(void) { return sbh::g_last_error.c_str(); }

const char* sbh_version(void) { return "sbh_b200 0.1.0 (sm_100a)"; }

int sbh_read_device_status(cudaStream_t stream, const void* workspace, uint32_t* out) {
  if (!workspace || !out) return sbh::invalid("workspace and out must be non-null");
  cudaError_t e = cudaMemcpyAsync(out, workspace, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return sbh::fail(SBH_ERR_CUDA, cudaGetErrorString(e));
  return SBH_OK;
}

size_t sbh_leaf3_size(void) { return sizeof(sbh::Leaf3); }
size_t sbh_node3_size(void) { return sizeof(sbh::Node3); }
size_t sbh_octree_level3_max_nodes(void) { return static_cast<size_t>(sbh::kLevel3MaxNodes); }
size_t sbh_octree8_node_size(void) { return sizeof(sbh::OctreeNode8); }
size_t sbh_leaf2_size(void) { return sizeof(sbh::Leaf2); }
size_t sbh_node2_size(void) { return sizeof(sbh::Node2); }

uint64_t sbh_octree8_total_nodes(int max_depth) {
  uint64_t total = 0, level = 1;
  for (int l = 0; l <= max_depth; l++) {
    total += level;
    level <<= 3;
  }
  return total;
}

size_t sbh_traversal_workspace_bytes(void) { return sbh::kStatusBytes; }

}  // extern "C"

// ---------------------------------------------------------------------------
// FP32 peak probe: independent FMA chains, 8 per thread, no memory traffic
// inside the loop. Used to report the traversal kernels' FP32-pipe roofline
// against a number measured on the same GPU.
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(256) fp32_probe_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-3f, x2 = x0 + 2e-3f, x3 = x0 + 3e-3f;
  float x4 = x0 + 4e-3f, x5 = x0 + 5e-3f, x6 = x0 + 6e-3f, x7 = x0 + 7e-3f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      x0 = fmaf(x0, a, b);
      x1 = fmaf(x1, a, b);
      x2 = fmaf(x2, a, b);
      x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b);
      x5 = fmaf(x5, a, b);
      x6 = fmaf(x6, a, b);
      x7 = fmaf(x7, a, b);
    }
  }
  float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains alive
}

// The same chains two to an instruction (packed FFMA2 on sm_100): 4 float2
// chains per thread, the same flops per launch.
__global__ void __launch_bounds__(256) fp32x2_probe_kernel(float* out, int iters, float a, float b) {
  const float x0 = threadIdx.x * 1e-7f;
  float2 y0 = make_float2(x0, x0 + 1e-3f), y1 = make_float2(x0 + 2e-3f, x0 + 3e-3f);
  float2 y2 = make_float2(x0 + 4e-3f, x0 + 5e-3f), y3 = make_float2(x0 + 6e-3f, x0 + 7e-3f);
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      y0 = __ffma2_rn(y0, a2, b2);
      y1 = __ffma2_rn(y1, a2, b2);
      y2 = __ffma2_rn(y2, a2, b2);
      y3 = __ffma2_rn(y3, a2, b2);
    }
  }
  float s = y0.x + y0.y + y1.x + y1.y + y2.x + y2.y + y3.x + y3.y;
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the chains alive
}
}  // namespace

extern "C" {
// Launches blocks x 256 threads of 8 independent FMA chains x 16 x iters:
// flops = blocks * 256 * 8 * 16 * iters * 2.
int sbh_probe_fp32(cudaStream_t stream, float* out, int blocks, int iters) {
  if (blocks <= 0 || iters <= 0 || !out) return sbh::invalid("blocks, iters > 0 and out non-null required");
  fp32_probe_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
  return sbh::check_launch("probe_fp32");
}

// As sbh_probe_fp32 with the FMAs issued two per instruction; same flops.
int sbh_probe_fp32x2(cudaStream_t stream, float* out, int blocks, int iters) {
  if (blocks <= 0 || iters <= 0 || !out) return sbh::invalid("blocks, iters > 0 and out non-null required");
  fp32x2_probe_kernel<<<blocks, 256, 0, stream>>>(out, iters, 0.999999f, 1e-7f);
  return sbh::check_launch("probe_fp32x2");
}
}
