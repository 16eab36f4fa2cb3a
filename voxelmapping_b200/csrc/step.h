// Scheduler state of the persistent batch step (step.cu), shared with the
// batch glue (batch.cu), which allocates it and launches the step.
#pragma once

#include "vmap_launch.h"

namespace vmapb {

// The stages of one map's step, in dependency order.
enum { ST_ALLOC, ST_VISIBLE, ST_FUSE, ST_ZRANGE, ST_RAYCAST, ST_NORMALS, ST_COUNT };

struct StepTask {
    int total;  // items, set when the task opens
    int taken;  // items handed out (may run past total)
    int done;   // items finished
    int aux;    // fusion: blocks visible; z-range: the first `aux` task indices are neighbour links
};

// Zeroed before every step. The three counters sit on their own 128-byte
// lines: warps poll them while other warps count items done.
struct StepSched {
    unsigned tail;  // ring entries reserved
    unsigned pad0[31];
    unsigned head;  // ring entries below `head` have no items left
    unsigned pad1[31];
    unsigned mapsDone;
    unsigned pad2[31];
    int ring[kMaxBatch * ST_COUNT];       // task id + 1 of each opened task, 0 = not yet written
    StepTask task[kMaxBatch * ST_COUNT];  // task id = map * ST_COUNT + stage
};

// A warp that waits this long without progress gives up (VMAP_FLAG_STEP_STALLED).
constexpr unsigned long long kStepStallNs = 2000000000ull;

// Clears S and runs one step of every map in `views` as one persistent launch.
// With reserveUnwritten, ring entry 0 is reserved but never written, so the
// step cannot proceed: every warp waits on it until stallNs pass without
// progress (the test of the bounded wait).
cudaError_t launch_step(const ManyViews& views, StepSched* S, int fmt, const Launcher& l, cudaStream_t s,
                        unsigned long long stallNs = kStepStallNs, bool reserveUnwritten = false);

}  // namespace vmapb
