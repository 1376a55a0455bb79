// The linear revaluation of a group of netting sets as a matrix product: the device arguments of
// basisRevalueKernel (tables built by buildBasis, basis_plan.h).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "basis_plan.h"
#include "zk_device.cuh"

namespace zk {

// One group: up to 128 netting sets of one scenario with the same margin-call and reporting dates.
struct BasisArgs {
  const float* cube;              // the scenario's factor cube [field][date][path]
  uint32_t nP, nT, nA, nC, nF, fS, fQ, fXf;
  const uint32_t* dates;          // [nT][kBasisDateWords]
  const BasisKg* kgs;
  const float* options;           // [*][8]
  const float4* fixings;          // [*]: A, b, 1 / c, slot
  const uint32_t* chunks;         // [numChunks][2]: byte offset into blob, K-steps
  const unsigned char* blob;      // coefficient images, 16-byte aligned
  const float* scale;             // [nT][kBasisRows]
  const NsArgs<float>* ns;        // the group's netting sets, row order
  uint32_t numNs, numFixSlots, numChunks, pad;
};

// One CTA per (tile of 128 paths, group): grid (tiles, groups), 512 threads, one CTA per SM; descBytes and fixSlots:
// the largest over the groups (BasisImage::descBytes, numFixSlots).
cudaError_t launchBasisRevalue(const BasisArgs* groups, uint32_t numGroups, uint32_t nP, uint32_t descBytes, uint32_t fixSlots,
                               uint32_t* err, cudaStream_t stream);

}  // namespace zk
