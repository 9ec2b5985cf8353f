// engine.cuh -- the iteration-loop driver shared by the vertex programs.
//
// The reference drives every GAS iteration from the host and reads the frontier
// size back after each one (GASengine/enactor_vertex_centric.cuh:2526-2872,
// cudaMemcpy at :2866-2869). Here the per-iteration kernels are captured once
// into the body of a CUDA-graph WHILE node; the kernel that finishes an
// iteration (last CTA to arrive) decides on the device whether another one runs
// (cudaGraphSetConditional), so a whole run is one graph launch with no host
// round trip. A host-driven loop (one control-block read per iteration) is kept
// for comparison and debugging (mg_opts.use_graph = -1).
#pragma once

#include <cuda_runtime.h>
#include <cstring>
#include <functional>
#include <vector>

#include "mg_internal.h"

// Body enqueuer: launches one iteration's kernels on `s`. When `use_cond` is
// set the kernels must call cudaGraphSetConditional(h, ...) from the CTA that
// ends the iteration.
using LoopBody = std::function<void(cudaStream_t s, cudaGraphConditionalHandle h, int use_cond)>;

// Runs `body` until DevCtl::done is set on the device. `slot` and `sig`
// identify a cached executable graph (reused while the signature matches).
// `max_iters` bounds the host-driven loop.
mg_status run_loop(mg_graph *g, int slot, const void *sig, size_t sig_len, bool use_graph, const LoopBody &body,
                   int64_t max_iters);

// Copies the control block back to the pinned host mirror (synchronises the stream).
mg_status fetch_ctl(mg_graph *g);

// Cache slots.
enum LoopSlot { SLOT_BFS = 0, SLOT_SSSP, SLOT_CC, SLOT_PR, SLOT_PR_REF, SLOT_ADJ, SLOT_MSBFS, SLOT_BSSSP, SLOT_PPR,
                SLOT_MSSSP, SLOT_COUNT };
