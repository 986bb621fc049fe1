// Device-side records of the native adaptive octree (see sbh_native.cu).
#pragma once

#include <cstdint>

namespace sbh {
namespace nt {

// Bounding cube of one system.
struct SegBox {
  float lo[3];
  float span;
  double scale;  // 2^21 / span
};

// One node, 64 bytes, read by the traversal with four 16-byte loads.
struct NodeRec {
  float4 com;    // COM x, y, z and total mass M
  float4 cell;   // cell centre x, y, z and diag = side * sqrt(3)
  float4 quad;   // S_xx, S_yy, S_zz, S_xy (second moment about the COM)
  float4 quad2;  // S_xz, S_yz, 0, 0
  int4 topo;     // particle range [start, end), skip index, level | 0x100 if leaf
};
static_assert(sizeof(NodeRec) == 80, "NodeRec must be 80 bytes");

constexpr int kLeafFlag = 0x100;
// Targets per lane in the walks (a group of 32 * kTPL targets per warp).
// Measured on a B200, adjoint walk over 8 x 2^20 Plummer particles at
// quadrupole radius 1.6: 410 ms with 2 per lane (7 blocks per SM), 389 ms
// with 3 (6 blocks, 80 registers), 411 ms with 4 (4 blocks); larger groups
// share each node's load, opening test and warp reduction among more
// targets at the price of a larger box and more registers.
#ifndef SBH_TARGETS_PER_LANE
#define SBH_TARGETS_PER_LANE 3
#endif
constexpr int kTPL = SBH_TARGETS_PER_LANE;
constexpr int kGroup = 32 * kTPL;  // targets per group (one warp)
#ifndef SBH_QUERY_GROUP
#define SBH_QUERY_GROUP 32
#endif
constexpr int kQueryGroup = SBH_QUERY_GROUP;  // targets per group of external queries (<= 32 * kTPL)
static_assert(kQueryGroup <= 32 * kTPL, "a query group must fit the lanes' target slots");
constexpr int kNodeAdj = 12;    // per-node adjoint floats: A_X(3) A_M(1) G(6) pad(2)
constexpr int kPartAdj = 4;     // per-particle adjoint floats: dx(3) dm(1)

}  // namespace nt
}  // namespace sbh
