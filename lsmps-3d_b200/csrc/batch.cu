// batch.cu - many independent particle boxes stepped by one captured CUDA
// graph (no counterpart in the reference, which steps one box per process).
//
// A batch owns S worker streams, each with its own context (scratch, packs,
// mixed-form arrays), so boxes on different streams never share scratch.  Box
// b is stepped on stream b mod S.  lsmps_batch_capture records, on an origin
// stream: a fork event every worker stream waits on, then each box's
// lsmps_step on its worker stream, then a join (the origin waits on every
// worker's final event), and instantiates the graph.  One lsmps_batch_launch
// then replays all boxes' launch sequences with no host work between them;
// boxes on different streams run concurrently, which fills the 148 SMs even
// when single boxes are small.
//
// Every allocation happens before capture: lsmps_batch_capture reserves each
// worker context for the largest box it will step (lsmps_ctx_reserve), and
// the contexts run asynchronously (device status folded by
// lsmps_batch_synchronize).
#include <algorithm>
#include <vector>

#include "batch_impl.cuh"
#include "impl.cuh"

struct lsmps_batch {
  int device = 0;
  cudaStream_t origin = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<lsmps_ctx*> ctxs;
  std::vector<cudaEvent_t> done;  // one per worker stream (join)
  cudaEvent_t fork = nullptr;
  std::vector<lsmps_params> params;
  std::vector<lsmps_step_state> states;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string last_error;
  // The merged form (batch_merged.cu): used when requested (the default) and
  // the boxes differ only in their grids.
  bool want_merged = true;
  bool merged_active = false;
  lsmps::MergedBatch merged;
};

namespace {

lsmps_status batch_fail(lsmps_batch* b, lsmps_status st, const std::string& what) {
  b->last_error = what;
  return st;
}

void release_graph(lsmps_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  if (b->merged_active) lsmps::release_merged(b->merged);
  b->merged_active = false;
}

// The merged form: one particle set for all boxes, stepped on the origin
// stream (gather, lsmps_step, scatter) and captured as the batch's graph.
lsmps_status capture_merged(lsmps_batch* b, int precision, int autotune_repeats) {
  std::string err;
  lsmps_status st = lsmps::prepare_merged(b->merged, b->device, b->origin, b->params, b->states, precision,
                                          autotune_repeats, err);
  if (st) return batch_fail(b, st, err);
  b->merged_active = true;
  if (cudaStreamSynchronize(b->origin) != cudaSuccess) return batch_fail(b, LSMPS_CUDA_ERROR, "pre-capture sync");
  if (cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return batch_fail(b, LSMPS_CUDA_ERROR, "begin capture failed");
  st = lsmps::queue_merged(b->merged, b->origin, err);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->origin, &graph);
  if (e != cudaSuccess || st) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return st ? batch_fail(b, st, err)
              : batch_fail(b, LSMPS_CUDA_ERROR, std::string("end capture: ") + cudaGetErrorString(e));
  }
  b->graph = graph;
  if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
    cudaGetLastError();
    release_graph(b);
    return batch_fail(b, LSMPS_CUDA_ERROR, "graph instantiation failed");
  }
  return LSMPS_OK;
}

}  // namespace

extern "C" lsmps_status lsmps_batch_create(int device, int streams, lsmps_batch** out) {
  if (!out || streams <= 0 || streams > 64) return LSMPS_INVALID_ARGUMENT;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return LSMPS_CUDA_ERROR;
  lsmps_batch* b = new lsmps_batch();
  b->device = device;
  bool ok = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int s = 0; s < streams && ok; ++s) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    lsmps_ctx* ctx = nullptr;
    ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) b->streams.push_back(st);
    ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (ok) b->done.push_back(ev);
    ok = ok && lsmps_ctx_create(device, &ctx) == LSMPS_OK;
    if (ok) {
      b->ctxs.push_back(ctx);
      lsmps_ctx_set_stream(ctx, st);
      lsmps_ctx_set_synchronous(ctx, 0);
      ctx->csr_cell_blocks = true;
    }
  }
  if (!ok) {
    cudaGetLastError();
    lsmps_batch_destroy(b);
    return LSMPS_CUDA_ERROR;
  }
  *out = b;
  return LSMPS_OK;
}

extern "C" void lsmps_batch_destroy(lsmps_batch* b) {
  if (!b) return;
  if (b->origin) cudaStreamSynchronize(b->origin);
  release_graph(b);
  for (lsmps_ctx* c : b->ctxs) lsmps_ctx_destroy(c);
  for (cudaEvent_t e : b->done) cudaEventDestroy(e);
  for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
}

extern "C" lsmps_status lsmps_batch_add(lsmps_batch* b, const lsmps_params* params, const lsmps_step_state* state) {
  if (!b || !params || !state) return LSMPS_INVALID_ARGUMENT;
  if (b->graph) return batch_fail(b, LSMPS_INVALID_ARGUMENT, "boxes cannot be added after capture");
  b->params.push_back(*params);
  b->states.push_back(*state);
  return LSMPS_OK;
}

extern "C" int lsmps_batch_size(lsmps_batch* b) { return b ? static_cast<int>(b->states.size()) : -1; }

extern "C" lsmps_status lsmps_batch_capture(lsmps_batch* b, int precision, int autotune_repeats) {
  if (!b || b->states.empty()) return LSMPS_INVALID_ARGUMENT;
  if (precision != LSMPS_PRECISION_PLAIN && precision != LSMPS_PRECISION_MIXED) return LSMPS_INVALID_ARGUMENT;
  if (cudaSetDevice(b->device) != cudaSuccess) return LSMPS_CUDA_ERROR;
  release_graph(b);
  if (b->want_merged && lsmps::boxes_mergeable(b->params)) return capture_merged(b, precision, autotune_repeats);
  const int S = static_cast<int>(b->streams.size());
  // Reserve every worker context for its largest box, and tune its knobs on
  // that box, before anything is captured.
  for (int s = 0; s < S; ++s) {
    lsmps_ctx* ctx = b->ctxs[s];
    lsmps_ctx_set_precision(ctx, precision);
    size_t nf = 0, nw = 0, nc = 0;
    int largest = -1;
    for (size_t k = s; k < b->states.size(); k += S) {
      const lsmps_step_state& st = b->states[k];
      if (largest < 0 || st.fluid.count > b->states[largest].fluid.count) largest = static_cast<int>(k);
      nf = std::max(nf, st.fluid.count);
      nw = std::max(nw, st.walls.count);
      nc = std::max(nc, std::max(st.fluid_cells.cell_count, st.wall_cells.cell_count));
    }
    if (largest < 0) continue;
    lsmps_status st = lsmps_ctx_reserve(ctx, nf, nw, nc);
    if (st) return batch_fail(b, st, std::string("reserve: ") + lsmps_ctx_last_error(ctx));
    if (autotune_repeats > 0) {
      st = lsmps_autotune(ctx, &b->params[largest], &b->states[largest], autotune_repeats, nullptr);
      if (st) return batch_fail(b, st, std::string("autotune: ") + lsmps_ctx_last_error(ctx));
    }
  }
  for (int s = 0; s < S; ++s) {
    lsmps_status st = lsmps_ctx_synchronize(b->ctxs[s]);
    if (st) return batch_fail(b, st, std::string("pre-capture: ") + lsmps_ctx_last_error(b->ctxs[s]));
  }
  if (cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return batch_fail(b, LSMPS_CUDA_ERROR, "begin capture failed");
  lsmps_status result = LSMPS_OK;
  cudaEventRecord(b->fork, b->origin);
  for (int s = 0; s < S; ++s) cudaStreamWaitEvent(b->streams[s], b->fork, 0);
  for (size_t k = 0; k < b->states.size() && !result; ++k) {
    lsmps_ctx* ctx = b->ctxs[k % S];
    result = lsmps_step(ctx, &b->params[k], &b->states[k]);
    if (result) b->last_error = std::string("box ") + std::to_string(k) + ": " + lsmps_ctx_last_error(ctx);
  }
  for (int s = 0; s < S; ++s) {
    cudaEventRecord(b->done[s], b->streams[s]);
    cudaStreamWaitEvent(b->origin, b->done[s], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->origin, &graph);
  if (e != cudaSuccess || result) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return result ? result : batch_fail(b, LSMPS_CUDA_ERROR, std::string("end capture: ") + cudaGetErrorString(e));
  }
  b->graph = graph;
  if (cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
    cudaGetLastError();
    release_graph(b);
    return batch_fail(b, LSMPS_CUDA_ERROR, "graph instantiation failed");
  }
  return LSMPS_OK;
}

extern "C" lsmps_status lsmps_batch_launch(lsmps_batch* b, void* stream) {
  if (!b || !b->exec) return LSMPS_NOT_PREPARED;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->origin;
  if (cudaGraphLaunch(b->exec, s) != cudaSuccess) {
    cudaGetLastError();
    return batch_fail(b, LSMPS_CUDA_ERROR, "graph launch failed");
  }
  return LSMPS_OK;
}

extern "C" lsmps_status lsmps_batch_synchronize(lsmps_batch* b) {
  if (!b) return LSMPS_INVALID_ARGUMENT;
  if (cudaStreamSynchronize(b->origin) != cudaSuccess) return batch_fail(b, LSMPS_CUDA_ERROR, "synchronize failed");
  lsmps_status first = LSMPS_OK;
  if (b->merged_active && b->merged.ctx) {
    const lsmps_status st = lsmps_ctx_synchronize(b->merged.ctx);
    if (st) {
      first = st;
      b->last_error = lsmps_ctx_last_error(b->merged.ctx);
    }
  }
  for (lsmps_ctx* c : b->ctxs) {
    const lsmps_status st = lsmps_ctx_synchronize(c);
    if (st && !first) {
      first = st;
      b->last_error = lsmps_ctx_last_error(c);
    }
  }
  return first;
}

extern "C" void* lsmps_batch_stream(lsmps_batch* b) { return b ? static_cast<void*>(b->origin) : nullptr; }

extern "C" const char* lsmps_batch_last_error(lsmps_batch* b) { return b ? b->last_error.c_str() : ""; }

extern "C" lsmps_status lsmps_batch_set_merged(lsmps_batch* b, int on) {
  if (!b || (on != 0 && on != 1)) return LSMPS_INVALID_ARGUMENT;
  if (b->graph) return batch_fail(b, LSMPS_INVALID_ARGUMENT, "the form is chosen before capture");
  b->want_merged = on != 0;
  return LSMPS_OK;
}

extern "C" int lsmps_batch_merged(lsmps_batch* b) { return b && b->merged_active ? 1 : 0; }
