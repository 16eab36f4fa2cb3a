// Persistent batch step: every stage of every map of a batch in ONE launch.
//
// One map's step is a chain of six stage tasks - allocation, visibility,
// fusion, z-range (with the neighbour links), ray marching, normals - and a
// task's item count is known only once the map's previous stage has finished
// (blocks allocated, blocks visible). Open tasks sit in a device-side ring
// in the order they opened; warps take items from the oldest entry that has
// items left and move on once all of its items are handed out. The warp that
// finishes the last item of a map's stage opens that map's next stage, so
// one map's ray marching runs beside another's fusion, and no stage waits
// for the slowest map of the batch. Every item is one warp's work, and the
// item bodies are the stage kernels' own (stages.cuh, march.cuh), so the
// results equal those of the six stage launches.
//
// Memory ordering: each lane fences its writes and the warp syncs before
// lane 0 counts the item done; the warp that completes a stage fences again
// before it publishes the next task; a warp fences after it takes an item
// (acquire). A warp counts its last item done before it looks for the next
// one, and takes the next item of the task it is working on with one atomic. Map data that an earlier stage of the launch wrote is read with
// plain loads (ld_map<false>), never through the read-only path.
//
// Waiting: a warp waits only while the ring holds no task with items left,
// that is while other warps run the items whose completion opens the next
// tasks; no warp waits while it holds an item, so every step completes.
// Each wait is still bounded: after 2 s in which neither the ring nor the
// count of finished maps changed, the warp raises VMAP_FLAG_STEP_STALLED in
// every map of the batch and leaves the kernel.
//
// The reference has no counterpart: VoxelMapping drives one map per call.
#include "march.cuh"
#include "stages.cuh"
#include "step.h"

namespace vmapb {

namespace {

constexpr int kWarpSet = 256;                         // one warp's staged blocks of a 32x8 tile (2 KB)
// Work of one item (one warp) besides the fixed-size ones (a 32x8-pixel tile
// for allocation and normals, a ray tile for the marcher): coarse enough that
// the scheduler's atomics stay far below the items' own memory traffic.
constexpr int kVisGroups = 4;   // visibility: 4 groups of 32 blocks
constexpr int kFuseBlocks = 4;  // fusion: 4 visible blocks
constexpr int kZTasks = 128;    // z-range: 128 link / fold tasks

__device__ __forceinline__ unsigned vload(const unsigned* p) { return *(volatile const unsigned*)p; }
__device__ __forceinline__ int vload(const int* p) { return *(volatile const int*)p; }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Items of stage s of a map, read when the stage opens (its inputs are final).
__device__ __forceinline__ int stage_items(const MapView& v, int s, int tw)
{
    switch (s) {
    case ST_ALLOC: return alloc_tiles<8>(v);
    case ST_VISIBLE: return v.in.active ? (allocated_blocks(v.m) + 32 * kVisGroups - 1) / (32 * kVisGroups) : 0;
    case ST_FUSE: return v.in.active ? ((int)vload(v.m.ctr + C_VISIBLE) + kFuseBlocks - 1) / kFuseBlocks : 0;
    case ST_ZRANGE: return (links_pending(v) + zrange_blocks(v) + kZTasks - 1) / kZTasks;
    case ST_RAYCAST: return ray_tiles(v, tw);
    default: return normal_tiles<8>(v);
    }
}

// Open the first stage >= s of map mi that has items (lane 0 of one warp),
// or count the map finished. The side effects the stage launches take at
// their start happen here: the visible counter is cleared before visibility
// accumulates into it, and the blocks linked by the z-range stage are marked
// before the ray marcher reads their links.
__device__ void open_from(const ManyViews& views, StepSched* S, int mi, int s, int tw)
{
    const MapView& v = views[mi];
    for (; s < ST_COUNT; ++s) {
        if (s == ST_VISIBLE && v.in.active) v.m.ctr[C_VISIBLE] = 0u;
        if (s == ST_RAYCAST && v.out.vmap) v.m.ctr[C_LINKED] = (unsigned)allocated_blocks(v.m);
        const int n = stage_items(v, s, tw);
        if (n > 0) {
            StepTask& t = S->task[mi * ST_COUNT + s];
            t.total = n;
            t.aux = s == ST_ZRANGE ? links_pending(v) : s == ST_FUSE ? (int)vload(v.m.ctr + C_VISIBLE) : 0;
            __threadfence();
            const unsigned pos = atomicAdd(&S->tail, 1u);
            atomicExch(&S->ring[pos], mi * ST_COUNT + s + 1);
            return;
        }
    }
    __threadfence();
    atomicAdd(&S->mapsDone, 1u);
}

struct Grab {
    int task, item, total, aux;
};

// Lane 0: the next item, from the oldest ring entry with items left; task -1
// when every map is finished or the wait stalled.
__device__ Grab grab(const ManyViews& views, StepSched* S, unsigned& h, unsigned long long stallNs)
{
    const unsigned nmaps = (unsigned)views.count();
    unsigned seenTail = ~0u, seenDone = ~0u, sleep = 32;
    unsigned long long since = global_ns();
    for (;;) {
        const unsigned head = vload(&S->head);
        if (head > h) h = head;
        const unsigned tail = vload(&S->tail);
        const unsigned done = vload(&S->mapsDone);
        if (h < tail) {
            const int e = vload(&S->ring[h]);
            if (e != 0) {  // (0: reserved, not yet written)
                __threadfence();
                StepTask* t = &S->task[e - 1];
                const int total = vload(&t->total);
                if (vload(&t->taken) < total) {
                    const int i = atomicAdd(&t->taken, 1);
                    if (i < total) return Grab{e - 1, i, total, vload(&t->aux)};
                }
                atomicMax(&S->head, h + 1);  // every item of entry h is handed out
                ++h;
                continue;
            }
        } else if (done >= nmaps) {
            return Grab{-1, 0, 0, 0};
        }
        if (tail != seenTail || done != seenDone) {
            seenTail = tail;
            seenDone = done;
            since = global_ns();
        } else if (global_ns() - since > stallNs) {
            for (unsigned i = 0; i < nmaps; ++i)
                if (views[i].m.ctr) atomicOr(views[i].m.ctr + C_ERR, VMAP_FLAG_STEP_STALLED);
            return Grab{-1, 0, 0, 0};
        }
        __nanosleep(sleep);
        if (sleep < 1024) sleep <<= 1;
    }
}

template <int FMT>
__global__ void __launch_bounds__(256, 4) step_kernel(const __grid_constant__ ManyViews views, StepSched* S,
                                                       int order, int tw, unsigned long long stallNs)
{
    __shared__ unsigned long long s_wkey[8][kWarpCache];
    __shared__ int s_wslot[8][kWarpCache];
    __shared__ unsigned long long s_set[8][kWarpSet];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long* set = s_set[wid];
    for (int i = lane; i < kWarpSet; i += 32) set[i] = kEmptyKey;
    // warp w of the grid opens the first stage of maps w, w + warps, ...
    if (lane == 0)
        for (int m = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); m < views.count();
             m += (int)((gridDim.x * blockDim.x) >> 5))
            open_from(views, S, m, 0, tw);
    __syncwarp();
    // scheduler state of each warp, kept in shared memory rather than in
    // registers across the item bodies: lane 0's ring cursor, the task the
    // warp takes items from, its item count and aux value, the warp's items
    // of that task not yet counted done, the item in hand, and the map whose
    // blocks the warp's block cache holds
    __shared__ int s_state[8][8];
    int* st = s_state[wid];
    enum { H, CUR, TOTAL, AUX, UNCOUNTED, ITEM, WMAP };
    if (lane == 0) {
        st[H] = st[TOTAL] = st[AUX] = st[UNCOUNTED] = st[ITEM] = 0;
        st[CUR] = st[WMAP] = -1;
    }
    __syncwarp();
    for (;;) {
        // the next item of the current task: one atomic
        const int cur = st[CUR];
        int i = 0;
        if (lane == 0 && cur >= 0) i = atomicAdd(&S->task[cur].taken, 1);
        i = __shfl_sync(full, i, 0);
        if (cur < 0 || i >= st[TOTAL]) {
            // the task has no items left: count this warp's items of it done
            // (before looking for work, so a warp never waits on a stage whose
            // completion it owes), then take an item from the ring
            if (cur >= 0) {
                __threadfence();  // release this lane's writes of those items
                __syncwarp();
                if (lane == 0) {
                    const int n = st[UNCOUNTED];
                    if (atomicAdd(&S->task[cur].done, n) + n == st[TOTAL]) {
                        __threadfence();
                        open_from(views, S, cur / ST_COUNT, cur % ST_COUNT + 1, tw);
                    }
                }
            }
            if (lane == 0) {
                unsigned h = (unsigned)st[H];
                const Grab g = grab(views, S, h, stallNs);
                st[H] = (int)h;
                st[CUR] = g.task;
                st[TOTAL] = g.total;
                st[AUX] = g.aux;
                st[ITEM] = g.item;
                st[UNCOUNTED] = 0;
            }
            __syncwarp();
            if (st[CUR] < 0) break;
            __threadfence();  // acquire: the inputs of the task's stage
            i = st[ITEM];
        }
        const int task = st[CUR], mi = task / ST_COUNT, s = task - mi * ST_COUNT;
        const MapView& v = views[mi];
        switch (s) {
        case ST_ALLOC: {  // a 32x8-pixel tile, a column of 8 pixels per lane (depths loaded first)
            const int tx = (v.cam.W + 31) >> 5;
            const int x = (i % tx) * 32 + lane, y0 = (i / tx) * 8;
            float d[8];
#pragma unroll
            for (int r = 0; r < 8; ++r)
                d[r] = x < v.cam.W && y0 + r < v.cam.H ? read_depth(v.in, x, y0 + r) : __int_as_float(0x7fffffff);
#pragma unroll 1
            for (int r = 0; r < 8; ++r)
                band_blocks_at(v, x, y0 + r, d[r], [&](unsigned long long key, int bx, int by, int bz) {
                    stage_block<kWarpSet>(set, v.m, key, bx, by, bz);
                });
            __syncwarp();
            insert_staged<kWarpSet>(set, v.m, lane, 32);
            __syncwarp();
            break;
        }
        case ST_VISIBLE:  // kVisGroups groups of 32 blocks
            for (int q = 0; q < kVisGroups; ++q) visibility_group(v, i * kVisGroups + q, lane);
            break;
        case ST_FUSE: {  // kFuseBlocks blocks, 16 voxels of each per lane
            const int nvis = st[AUX];
#pragma unroll 1
            for (int k = i * kFuseBlocks; k < min(nvis, (i + 1) * kFuseBlocks); ++k) {
                const int slot = v.m.visList[k];
#pragma unroll 1
                for (int j = 0; j < 4; ++j) fuse_voxels<FMT>(v, slot, 4 * (lane + 32 * j));
            }
            break;
        }
        case ST_ZRANGE: {  // kZTasks tasks: neighbour links first, then z-range folds
            const int nlink = st[AUX], nz = zrange_blocks(v);
            for (int q = 0; q < kZTasks / 32; ++q) {
                const int t = (i * (kZTasks / 32) + q) * 32 + lane;
                if (t < nlink) link_task<false>(v.m, t);
                else if (t - nlink < nz) zrange_block(v, t - nlink);
            }
            break;
        }
        case ST_RAYCAST:
            if (mi != st[WMAP]) {
                warp_cache_clear(s_wkey[wid], lane);  // ends with __syncwarp
                if (lane == 0) st[WMAP] = mi;
            }
            march_tile<FMT, false>(v, mi, i, st[TOTAL], order, tw, s_wkey[wid], s_wslot[wid], lane);
            break;
        default: {  // normals of a 32x8-pixel tile
            const int tx = (v.cam.W + 31) >> 5;
            const int x = (i % tx) * 32 + lane, y0 = (i / tx) * 8;
            for (int r = 0; r < 8; ++r) normal_pixel<false>(v, x, y0 + r);
            break;
        }
        }
        __syncwarp();
        if (lane == 0) ++st[UNCOUNTED];
        __syncwarp();
    }
}

template <int FMT>
cudaError_t launch_step_fmt(const ManyViews& views, StepSched* S, const Launcher& l, cudaStream_t s,
                            unsigned long long stallNs, bool reserveUnwritten)
{
    // resident CTAs per SM (a static initialiser runs once, thread-safely)
    static const int fit = [] {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, step_kernel<FMT>, 256, 0) != cudaSuccess || o < 1) o = 1;
        return o;
    }();
    // CTAs beyond those resident would only start once others finish: cap at occupancy
    const int per_sm = l.raycast > 0 && l.raycast < fit ? l.raycast : fit;
    cudaError_t e = cudaMemsetAsync(S, 0, sizeof(StepSched), s);
    if (e != cudaSuccess) return e;
    if (reserveUnwritten) {  // tail = 1 with ring[0] left 0
        static const unsigned one = 1u;
        if ((e = cudaMemcpyAsync(&S->tail, &one, sizeof one, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    }
    step_kernel<FMT><<<stage_grid(l, per_sm), 256, 0, s>>>(views, S, l.tileOrder, l.tileW, stallNs);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_step(const ManyViews& views, StepSched* S, int fmt, const Launcher& l, cudaStream_t s,
                        unsigned long long stallNs, bool reserveUnwritten)
{
    switch (fmt) {
    case VMAP_VOXEL_REF: return launch_step_fmt<VMAP_VOXEL_REF>(views, S, l, s, stallNs, reserveUnwritten);
    case VMAP_VOXEL_F32: return launch_step_fmt<VMAP_VOXEL_F32>(views, S, l, s, stallNs, reserveUnwritten);
    case VMAP_VOXEL_F16: return launch_step_fmt<VMAP_VOXEL_F16>(views, S, l, s, stallNs, reserveUnwritten);
    case VMAP_VOXEL_I16: return launch_step_fmt<VMAP_VOXEL_I16>(views, S, l, s, stallNs, reserveUnwritten);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace vmapb
