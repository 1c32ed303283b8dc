// p3m_static.cu — the cell-list build for callers that cannot allocate.
//
// Some hosts may not call cudaMalloc at the point where they need cell
// lists: a renderer or physics callback that runs inside a frame whose
// allocations are forbidden, an allocator that is owned by another runtime
// (a JVM or game engine that hands out all device memory itself), or code
// that must not stall on the driver's allocator. p3m_cell_lists_static serves
// them: it builds the same sorted cell lists as p3m_build_cell_lists, from
// device arrays the caller owns into device arrays the caller owns, and keeps
// its working memory (key/ID ping-pong buffers, radix tile histograms, scan
// partials) in one fixed array compiled into this library.
//
// The array is a file-scope __device__ variable, so every GPU that loads this
// module holds it (about 16.3 MB) until the process exits. Host code cannot
// use its name as a device address; the first call on each device looks the
// address up with cudaGetSymbolAddress (with that device current) and caches
// it. Every call shares the array and it keeps the last call's contents, so
// calls whose work overlaps on the GPU (two streams, or two host threads)
// race: order them on one stream or synchronise between them.

#include "p3m_internal.cuh"

#include <mutex>

namespace {

constexpr int kMaxBodies = P3M_CELL_LISTS_STATIC_MAX_BODIES;
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kTiles = (kMaxBodies + p3m::kSortTile - 1) / p3m::kSortTile;
constexpr size_t kHistEntries = (size_t)p3m::kSortMaxRadix * kTiles;
constexpr size_t kSumEntries = kHistEntries / 4096 + 2;
constexpr size_t kVecBytes = align256((size_t)kMaxBodies * sizeof(uint32_t));
constexpr size_t kOffKeysA = 0;
constexpr size_t kOffValsA = kOffKeysA + kVecBytes;
constexpr size_t kOffKeysB = kOffValsA + kVecBytes;
constexpr size_t kOffValsB = kOffKeysB + kVecBytes;
constexpr size_t kOffHist = kOffValsB + kVecBytes;
constexpr size_t kOffSums = kOffHist + align256(kHistEntries * sizeof(uint32_t));
constexpr size_t kScratchBytes = kOffSums + align256(kSumEntries * sizeof(uint32_t));

// The working memory of every call on a device (see the file comment).
static __device__ __align__(256) unsigned char g_cell_list_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Failures are reported through p3m_last_error(NULL), like p3m_create's.
int fail(int status, const std::string& what) {
    p3m::set_detached_error(what);
    return status;
}

// Device address of the scratch array on the current device, looked up once
// per device.
int scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(P3M_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(P3M_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_cell_list_scratch);
        if (e != cudaSuccess || !p)
            return fail(P3M_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_address[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_address[dev]);
    return P3M_OK;
}

int bits_for(long long count) {
    int b = 1;
    while ((1LL << b) < count) ++b;
    return b;
}

}  // namespace

extern "C" int p3m_cell_lists_static(const float* bodies4, const float* materials4, int32_t n,
                                     int32_t grid_width, int32_t grid_height,
                                     uint32_t* sorted_keys, int32_t* sorted_ids,
                                     int32_t* cell_start, int32_t* cell_count, uint32_t* cell_mass,
                                     float* entries4, void* stream) {
    p3m::set_detached_error("");
    if (n < 0) return fail(P3M_ERR_INVALID_ARGUMENT, "body count must be >= 0");
    if (n > kMaxBodies)
        return fail(P3M_ERR_CAPACITY, "p3m_cell_lists_static handles at most " +
                                          std::to_string(kMaxBodies) + " bodies; got " +
                                          std::to_string(n));
    if (grid_width <= 0 || grid_height <= 0 || (long long)grid_width * grid_height > (1LL << 28))
        return fail(P3M_ERR_INVALID_ARGUMENT, "grid must be positive with at most 2^28 cells");
    if (n > 0 && (!bodies4 || !materials4 || !sorted_keys || !sorted_ids || !entries4))
        return fail(P3M_ERR_INVALID_ARGUMENT, "a body-sized array is NULL");
    if (!cell_start || !cell_count || !cell_mass)
        return fail(P3M_ERR_INVALID_ARGUMENT, "a cell-sized array is NULL");

    unsigned char* base = nullptr;
    int st = scratch_address(&base);
    if (st != P3M_OK) return st;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long P = (long long)grid_width * grid_height;
    p3m::GridShape g{grid_width, grid_height, grid_width, grid_height, 0};
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + kOffKeysA);
    uint32_t* vals = reinterpret_cast<uint32_t*>(base + kOffValsA);
    p3m::SortScratch scratch;
    scratch.keys_alt = reinterpret_cast<uint32_t*>(base + kOffKeysB);
    scratch.vals_alt = reinterpret_cast<uint32_t*>(base + kOffValsB);
    scratch.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    scratch.block_sums = reinterpret_cast<uint32_t*>(base + kOffSums);
    scratch.capacity = kMaxBodies;

    // Counts and masses are summed with atomics: they start at zero every
    // call. The scratch array needs no clearing: keys and IDs are written for
    // every body before they are read, and each radix pass rewrites the
    // histogram entries it scans.
    cudaError_t e = cudaMemsetAsync(cell_count, 0, (size_t)P * sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cell_mass, 0, (size_t)P * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cell_start, 0, (size_t)P * sizeof(int32_t), s);
    if (e == cudaSuccess && n > 0)
        e = p3m::launch_cell_keys(reinterpret_cast<const float4*>(bodies4), n, g, keys, vals, s);
    uint32_t* sk = keys;
    uint32_t* sv = vals;
    if (e == cudaSuccess && n > 0)
        e = p3m::radix_sort_pairs(keys, vals, scratch, n, bits_for(P), s, &sk, &sv);
    if (e == cudaSuccess && n > 0)
        e = p3m::launch_cell_build(sk, sv, n, reinterpret_cast<const float4*>(bodies4),
                                   reinterpret_cast<const float4*>(materials4), cell_start,
                                   cell_count, cell_mass, reinterpret_cast<float4*>(entries4), 0,
                                   s);
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpyAsync(sorted_keys, sk, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpyAsync(sorted_ids, sv, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return fail(P3M_ERR_CUDA, std::string("p3m_cell_lists_static: ") + cudaGetErrorString(e));
    return P3M_OK;
}
