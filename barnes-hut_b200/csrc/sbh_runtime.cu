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
