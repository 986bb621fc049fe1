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
// Most targets per group: four per lane of a warp. Groups of at most
// kGroupTwoSlots targets are walked by the two-slot kernels, of at most
// kGroupThreeSlots by the three-slot kernels, larger ones by the four-slot
// kernels.
constexpr int kGroupTwoSlots = 64;
constexpr int kGroupThreeSlots = 96;
constexpr int kGroup = 128;  // targets per group built by default (one warp, four per lane)
#ifndef SBH_QUERY_GROUP
#define SBH_QUERY_GROUP 32
#endif
constexpr int kQueryGroup = SBH_QUERY_GROUP;  // targets per group of external queries
static_assert(kQueryGroup <= kGroupTwoSlots, "query groups are walked by the two-slot kernels");
constexpr int kNodeAdj = 12;    // per-node adjoint floats: A_X(3) A_M(1) G(6) pad(2)
constexpr int kPartAdj = 4;     // per-particle adjoint floats: dx(3) dm(1)
// interaction counters of the count-only walk: far, near (per target), far with the exact
// quadrupole, far with the linearized quadrupole (per target), linearized (group, node) pairs
constexpr int kCounters = 8;

}  // namespace nt
}  // namespace sbh
