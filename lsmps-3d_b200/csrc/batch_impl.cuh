// batch_impl.cuh - the merged form of a batch (batch_merged.cu), used by
// batch.cu.
#pragma once

#include <climits>
#include <string>
#include <vector>

#include "common.cuh"

namespace lsmps {

// All boxes of a batch as one particle set: the merged buffers, the boxes'
// grid table and gather/scatter table on the device, and the context that
// steps the set.
struct MergedBatch {
  lsmps_ctx* ctx = nullptr;
  std::vector<void*> allocations;
  BoxGrid* grids = nullptr;
  PpeBoxOut* box_ppe = nullptr;  // per box: its own PPE matrix (the merged step writes the rows there)
  void* io = nullptr;  // per box: its views, counts and merged bases
  lsmps_step_state state{};
  lsmps_params params{};
  int nbox = 0;
  index_t nf = 0, nw = 0, nc = 0;
  int precision = 0;
};

// True when the boxes differ only in their grid origin and dims.
bool boxes_mergeable(const std::vector<lsmps_params>& params);
// Allocate the merged set, build its neighbour tables and labels from the
// boxes' current positions, reserve and optionally autotune the context
// (outside stream capture).
lsmps_status prepare_merged(MergedBatch& mb, int device, cudaStream_t stream, const std::vector<lsmps_params>& params,
                            const std::vector<lsmps_step_state>& states, int precision, int autotune_repeats,
                            std::string& error);
// Queue one launch's work: gather, the merged step, scatter.
lsmps_status queue_merged(MergedBatch& mb, cudaStream_t stream, std::string& error);
void release_merged(MergedBatch& mb);

}  // namespace lsmps
