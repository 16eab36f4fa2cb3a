// Map snapshots: save the used blocks and their keys, load them into a map and
// rebuild its hash table.
//
// The reference has no snapshot; its nearest operations are MapStruct::reset
// and release (src/map_struct.cu:29-79). Serving many sessions from one GPU
// needs one to evict an idle map to host memory and bring it back later, and
// the same bytes serve as a checkpoint. Blocks are handed out densely in pool
// order (0, 1, 2, ...), so a snapshot is two contiguous copies (keys, then
// n_blocks * block_bytes of pool) plus a header. Loading copies them back to
// the same pool slots and re-inserts every key with its slot; every kernel
// reads blocks through the hash table or in pool order, so the loaded map
// behaves bit-identically to the saved one whatever its bucket count.
#include <cstring>
#include <string>

#include "vmap_launch.h"

using namespace vmapb;

namespace {

constexpr uint32_t kSnapVersion = 1;
constexpr uint64_t kPoolAlign = 256;

uint64_t pool_offset(uint32_t n)
{
    const uint64_t keys_end = sizeof(vmap_snapshot_header) + 8ull * n;
    return (keys_end + kPoolAlign - 1) / kPoolAlign * kPoolAlign;
}

vmap_status fail(vmap_status st, const std::string& msg)
{
    set_last_error(msg);
    return st;
}

vmap_status cuda_fail(cudaError_t e, const char* what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VMAP_ERR_OUT_OF_MEMORY : VMAP_ERR_CUDA;
}

#define SNAP_CK(expr)                                        \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);  \
    } while (0)

// Inserts `key` with a given pool slot (the probe sequence of hash_insert
// without the bump allocation). A key already present means the snapshot was
// corrupt.
__device__ void hash_insert_slot(const DevMap& m, unsigned long long key, unsigned slot)
{
    const int3 c = unpack_key(key);
    int b = ref_hash_fast(c.x, c.y, c.z, m.nBucket, m.bucketMagic);
#pragma unroll 1
    for (int p = 0; p < kMaxProbe; ++p) {
        ulonglong2* s = m.slots + (size_t)b * kSlots;
#pragma unroll 1
        for (int i = 0; i < kSlots; ++i) {
            unsigned long long cur = __ldcg(&s[i].x);
            if (cur == kEmptyKey) cur = atomicCAS(&s[i].x, kEmptyKey, key);
            if (cur == kEmptyKey) {
                s[i].y = (unsigned long long)slot;
                return;
            }
            if (cur == key) {
                atomicOr(m.ctr + C_ERR, VMAP_FLAG_BAD_SNAPSHOT);
                return;
            }
        }
        b = (b + 1 == m.nBucket) ? 0 : b + 1;
    }
    atomicOr(m.ctr + C_ERR, VMAP_FLAG_HASH_FULL);
}

// Counters were zeroed by the host; thread 0 restores the allocation count and
// the saved sticky flags, every thread re-inserts its blocks' keys.
__global__ void rebuild_hash_kernel(DevMap m, unsigned n, unsigned flags)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        m.ctr[C_ALLOC] = n;
        if (flags) atomicOr(m.ctr + C_ERR, flags);
    }
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long key = m.blockKeys[i];
        if (key >> 63) atomicOr(m.ctr + C_ERR, VMAP_FLAG_BAD_SNAPSHOT);  // the empty key, or bit 63 set
        else hash_insert_slot(m, key, i);
    }
}

__global__ void clear_slots_kernel(DevMap m)
{
    const size_t n = (size_t)m.nBucket * kSlots;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m.slots[i] = make_ulonglong2(kEmptyKey, ~0ull);
}

int sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return 1;
    return sms;
}

// 256-thread CTAs for `items` grid-stride items, at most 8 per SM
int grid_for(size_t items)
{
    const size_t g = (items + 255) / 256;
    const size_t cap = (size_t)sm_count() * 8;
    return (int)(g == 0 ? 1 : (g < cap ? g : cap));
}

}  // namespace

extern "C" {

vmap_status vmap_snapshot_save(vmap_map* map, void* dst, uint64_t capacity, uint64_t* bytes, void* stream)
{
    if (!map || !bytes) return VMAP_ERR_INVALID_ARG;
    vmap_config cfg;
    vmap_stats st;
    vmap_status r = vmap_get_config(map, &cfg);
    if (r != VMAP_OK) return r;
    if ((r = vmap_get_stats(map, stream, &st)) != VMAP_OK) return r;  // synchronises `stream`
    const DevMap& m = map_device_view(map);
    const uint32_t n = st.allocated_blocks;
    vmap_snapshot_header h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "VMAPSNAP", 8);
    h.version = kSnapVersion;
    h.header_bytes = sizeof(vmap_snapshot_header);
    h.voxel_format = cfg.voxel_format;
    h.with_color = cfg.with_color ? 1 : 0;
    h.block_bytes = (uint32_t)m.blockBytes;
    h.n_blocks = n;
    h.voxel_size = cfg.voxel_size;
    h.truncation = cfg.truncation;
    h.max_weight = cfg.max_weight;
    h.error_flags = st.error_flags;
    h.keys_offset = sizeof(vmap_snapshot_header);
    h.pool_offset = pool_offset(n);
    const uint64_t total = h.pool_offset + (uint64_t)n * h.block_bytes;
    *bytes = total;
    if (!dst) return VMAP_OK;
    if (capacity < total)
        return fail(VMAP_ERR_INVALID_ARG, "vmap_snapshot_save: destination holds " + std::to_string(capacity) +
                                              " bytes, the snapshot needs " + std::to_string(total));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* d = static_cast<unsigned char*>(dst);
    SNAP_CK(cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyDefault, s));
    // zero the padding before the aligned pool so equal maps give equal bytes
    static const unsigned char zeros[kPoolAlign] = {};
    const uint64_t keys_end = h.keys_offset + 8ull * n;
    if (h.pool_offset > keys_end)
        SNAP_CK(cudaMemcpyAsync(d + keys_end, zeros, h.pool_offset - keys_end, cudaMemcpyDefault, s));
    if (n) {
        SNAP_CK(cudaMemcpyAsync(d + h.keys_offset, m.blockKeys, 8ull * n, cudaMemcpyDefault, s));
        SNAP_CK(cudaMemcpyAsync(d + h.pool_offset, m.pool, (size_t)n * h.block_bytes, cudaMemcpyDefault, s));
    }
    SNAP_CK(cudaStreamSynchronize(s));  // `h` lives on this stack frame
    return VMAP_OK;
}

vmap_status vmap_snapshot_load(vmap_map* map, const void* src, uint64_t bytes, void* stream)
{
    if (!map || !src) return VMAP_ERR_INVALID_ARG;
    if (bytes < sizeof(vmap_snapshot_header))
        return fail(VMAP_ERR_INVALID_ARG, "vmap_snapshot_load: shorter than a snapshot header");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    vmap_snapshot_header h;
    SNAP_CK(cudaMemcpyAsync(&h, src, sizeof(h), cudaMemcpyDefault, s));
    SNAP_CK(cudaStreamSynchronize(s));
    vmap_config cfg;
    vmap_stats st;
    vmap_status r = vmap_get_config(map, &cfg);
    if (r != VMAP_OK) return r;
    if ((r = vmap_get_stats(map, stream, &st)) != VMAP_OK) return r;
    const DevMap& m = map_device_view(map);
    if (std::memcmp(h.magic, "VMAPSNAP", 8) != 0 || h.version != kSnapVersion ||
        h.header_bytes != sizeof(vmap_snapshot_header) || h.keys_offset != sizeof(vmap_snapshot_header) ||
        h.pool_offset != pool_offset(h.n_blocks) || bytes < h.pool_offset + (uint64_t)h.n_blocks * h.block_bytes)
        return fail(VMAP_ERR_INVALID_ARG, "vmap_snapshot_load: not a version-1 snapshot, or truncated");
    if (h.voxel_format != cfg.voxel_format || h.with_color != (cfg.with_color ? 1 : 0) ||
        h.block_bytes != (uint32_t)m.blockBytes || std::memcmp(&h.voxel_size, &cfg.voxel_size, 4) != 0 ||
        std::memcmp(&h.truncation, &cfg.truncation, 4) != 0 || h.max_weight != cfg.max_weight)
        return fail(VMAP_ERR_INVALID_ARG,
                    "vmap_snapshot_load: voxel format, colour, voxel size, truncation or weight cap differ");
    if (h.n_blocks > (uint32_t)m.capacity)
        return fail(VMAP_ERR_INVALID_ARG, "vmap_snapshot_load: " + std::to_string(h.n_blocks) +
                                              " blocks exceed the pool capacity of " + std::to_string(m.capacity));
    const uint32_t n = h.n_blocks;
    const unsigned char* p = static_cast<const unsigned char*>(src);
    // blocks beyond the snapshot must read as unobserved (zero) once handed out again
    if (st.allocated_blocks > n)
        SNAP_CK(cudaMemsetAsync(m.pool + (size_t)n * m.blockBytes, 0, (size_t)(st.allocated_blocks - n) * m.blockBytes, s));
    SNAP_CK(cudaMemsetAsync(m.ctr, 0, C_COUNT * sizeof(unsigned), s));
    clear_slots_kernel<<<grid_for((size_t)m.nBucket * kSlots), 256, 0, s>>>(m);
    SNAP_CK(cudaGetLastError());
    if (n) {
        SNAP_CK(cudaMemcpyAsync(m.blockKeys, p + h.keys_offset, 8ull * n, cudaMemcpyDefault, s));
        SNAP_CK(cudaMemcpyAsync(m.pool, p + h.pool_offset, (size_t)n * m.blockBytes, cudaMemcpyDefault, s));
    }
    rebuild_hash_kernel<<<grid_for(n), 256, 0, s>>>(m, n, h.error_flags);
    SNAP_CK(cudaGetLastError());
    if ((r = vmap_get_stats(map, stream, &st)) != VMAP_OK) return r;  // also waits for the copies out of src
    const unsigned bad = st.error_flags & ~h.error_flags;
    if (bad & (VMAP_FLAG_HASH_FULL | VMAP_FLAG_BAD_SNAPSHOT)) {
        Launcher l;
        l.numSMs = sm_count();
        SNAP_CK(launch_reset(m, (size_t)m.capacity * m.blockBytes, l, s));
        SNAP_CK(cudaStreamSynchronize(s));
        return bad & VMAP_FLAG_BAD_SNAPSHOT
                   ? fail(VMAP_ERR_INVALID_ARG, "vmap_snapshot_load: invalid or repeated block key; map reset")
                   : fail(VMAP_ERR_HASH_FULL, "vmap_snapshot_load: keys do not fit the hash table; map reset");
    }
    return VMAP_OK;
}

}  // extern "C"
