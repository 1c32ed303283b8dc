// p3m_internal.cuh — shared declarations of the sm_100a P3M library.
//
// Layout in HBM (one context):
//   bodies      float4[cap]  (x, y, vx, vy) in unit coordinates, ID order
//   materials   float4[cap]  (mass, friction, solid, block)
//   accel       float2[cap]
//   keys/ids    uint32[cap] x2 ping-pong   cell-key radix sort
//   entries     float4[cap]  bodies gathered into cell order (x, y, mass, id bits)
//   cell_start / cell_count / cell_mass    int32/int32/uint32 [P]
//   density     uint32[M] or int64[M]      fixed-point CIC mesh
//   half        float2[(MW/2+1) * MH]      row-transformed density
//   cols        float4[(MW/2+1) * MH]      column-inverted (Fx, Fy) spectra
//   force       float2[M]                  (fx, fy) long-range mesh force
//   green       float2[(MW/2+1) * MH]      spectral multipliers (gx, gy)
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "../../include/p3m.h"

namespace p3m {

constexpr float kCellMassUnits = 256.0f;        // build_grid.comp:19
constexpr float kMaximumUnit = 0.99999994f;      // collision_build.comp:21
constexpr int kMaxMeshAxis = 4096;
constexpr int kTwiddleLog2 = 12;                 // one table of 4096 roots
constexpr int kTwiddleLength = 1 << kTwiddleLog2;

// ------------------------------------------------------------- index helpers
// floor(x) converted to int the way the GPU's cvt.rzi.s32.f32 converts:
// NaN -> 0, saturation at the int range (the value is already integral).
__host__ __device__ __forceinline__ int float_to_int(float f) {
#ifdef __CUDA_ARCH__
    return __float2int_rz(f);  // cvt.rzi.s32.f32: the same NaN and saturation rules
#else
    if (f != f) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int)0x80000000;
    return (int)f;
#endif
}

// Out-of-line so that the common path below stays two compares.
static __host__ __device__ __noinline__ int wrap_far(int v, int size) {
    v %= size;
    return v < 0 ? v + size : v;
}

// wrapCell / wrapMesh (build_grid.comp:21-37, kick.comp:38-59): one period
// added or subtracted. Every index a position in [0, 1] produces needs no
// more; a position outside that range, handed in by a caller, is reduced
// modulo the size so that no index ever leaves its buffer.
__host__ __device__ __forceinline__ int wrap_index(int v, int size) {
    if (v < 0) v += size;
    else if (v >= size) v -= size;
    if ((unsigned)v >= (unsigned)size) v = wrap_far(v, size);
    return v;
}

// A cell coordinate that stencil offsets (|d| <= size) are added to: kept as
// it is for positions in [0, 1], folded into [0, size) only when it lies so
// far out that adding an offset could overflow.
__host__ __device__ __forceinline__ int guard_coord(int v, int size) {
    return (v < -size || v > 2 * size) ? wrap_index(v, size) : v;
}

// ---------------------------------------------------------------- radix sort
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kSortMaxRadix = 256;

constexpr int kSortMaxPasses = 4;

struct SortScratch {
    uint32_t* keys_alt = nullptr;
    uint32_t* vals_alt = nullptr;
    uint32_t* hist = nullptr;       // kSortMaxRadix * tiles
    uint32_t* block_sums = nullptr; // scan partials
    // One-kernel-per-pass form (all null: three kernels per pass instead).
    // `lookback` holds sort_lookback_words(capacity) words: the digit totals
    // of every pass, the tile counters and the tiles' published counts;
    // `wait_timeouts` counts look-back waits that gave up.
    uint32_t* lookback = nullptr;
    unsigned int* wait_timeouts = nullptr;
    int capacity = 0;
    // Polls of one look-back word before a wait gives up, and the tile whose
    // counts are never published (-1: none). Only the timeout test changes
    // them (p3m_set_lookback_fault): a withheld tile makes its successor's
    // wait run out, as a tile that never arrives would.
    int poll_limit = 200000;
    int withhold_tile = -1;
};

size_t sort_hist_entries(int capacity);
size_t sort_block_sum_entries(int capacity);
size_t sort_lookback_words(int capacity);

// Digit totals of a look-back sort, added by the kernel that writes its keys
// (the drift for the cell sort, the Morton-key kernel for the reorder)
// instead of by a separate pass over the keys. totals == nullptr: the sort
// counts them itself.
struct SortTotals {
    uint32_t* totals = nullptr;  // [pass][kLookbackMaxRadix] digit counts, cleared
    int passes = 0, bits = 0, key_bits = 0;
};
constexpr int kLookbackMaxRadix = 512;  // digits of up to 9 bits

// Clears the look-back words of a sort of n keys over key_bits bits (one
// memset) and says where the keys' producer adds their digit totals. Leaves
// out->totals null (nothing issued; the sort counts its digits itself) from
// 2^21 keys, and when that sort does not take the look-back form.
cudaError_t radix_sort_prepare(const SortScratch& s, int n, int key_bits, cudaStream_t stream,
                               SortTotals* out);

// Adds this thread's key (when `valid`) to the digit totals: counts per pass
// in shared memory (warp-aggregated), then one global atomic per CTA and
// non-zero digit. Every thread of the CTA calls it; `sh` holds
// kSortMaxPasses * kLookbackMaxRadix words.
__device__ __forceinline__ void add_digit_totals(const SortTotals& st, bool valid, uint32_t key,
                                                 uint32_t* sh) {
    const int bins = st.passes * kLookbackMaxRadix;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    for (int p = 0; p < st.passes; ++p) {
        const int pb = min(st.bits, st.key_bits - p * st.bits);
        const uint32_t d = valid ? (key >> (p * st.bits)) & ((1u << pb) - 1u) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int lane = threadIdx.x & 31;
        if (valid && lane == __ffs(peers) - 1)
            atomicAdd(&sh[p * kLookbackMaxRadix + d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < bins; i += blockDim.x)
        if (sh[i]) atomicAdd(&st.totals[i], sh[i]);
}

// Stable LSD radix sort of (keys, vals) on bits [0, key_bits). Passes
// alternate between the inputs and the scratch pair; *out_keys/*out_vals
// name the pair that holds the result. Launches only; no allocation, no
// synchronisation.
// totals_ready: radix_sort_prepare ran for this sort and the keys' producer
// added the digit totals.
// failed (may be null): set to the device word that this sort sets to 1 when
// one of its bounded look-back waits gave up (its output is then not a
// permutation of its input), or to null when the sort has no waits. The
// consumers of the result check it (launch_cell_build, launch_permute).
cudaError_t radix_sort_pairs(uint32_t* keys, uint32_t* vals, const SortScratch& s, int n,
                             int key_bits, cudaStream_t stream, uint32_t** out_keys,
                             uint32_t** out_vals, bool totals_ready = false,
                             const uint32_t** failed = nullptr);

// Exclusive scan of n uint32 in place (n <= 4096 * 4096).
cudaError_t exclusive_scan_u32(uint32_t* data, int n, uint32_t* block_sums,
                               cudaStream_t stream);

// ------------------------------------------------------------- step kernels
struct GridShape {
    int W, H;     // physical grid
    int MW, MH;   // mesh (= physical on the torus, 2x on walls)
    int bounded;
    int fft_lines = 0;  // lines per CTA of the FFT kernels; 0 = automatic
};

// Half kick + drift substeps (collision_build.comp:40-51), then the home-cell
// key of each body, written in descending ID order for the cell sort.
// With totals.totals set (radix_sort_prepare), also adds the keys' digit
// totals for the look-back cell sort.
cudaError_t launch_drift(float4* bodies, const float2* accel, int n, float half_kick,
                         float drift_dt, int substeps, GridShape g, uint32_t* keys,
                         uint32_t* vals, unsigned int* nonfinite, cudaStream_t stream,
                         SortTotals totals = SortTotals());
// Home-cell keys of the current positions (no drift).
cudaError_t launch_cell_keys(const float4* bodies, int n, GridShape g, uint32_t* keys,
                             uint32_t* vals, cudaStream_t stream);
// Morton tile keys (spatial_sort_key.glsl), ascending ID order.
cudaError_t launch_morton_keys(const float4* bodies, int n, int wbits, int hbits,
                               uint32_t* keys, uint32_t* vals, cudaStream_t stream,
                               SortTotals totals = SortTotals());
// Permutation of the Morton reorder (spatial_sort_scatter / _materials.comp).
// When *sort_failed is set (the sort's look-back gave up) the bodies are
// copied in place order instead, so no index taken from the sort is used.
cudaError_t launch_permute(const uint32_t* order, int n, const float4* bodies, const float2* accel,
                           const float4* materials, float4* bodies_out, float2* accel_out,
                           float4* materials_out, uint32_t* destinations, cudaStream_t stream,
                           const uint32_t* sort_failed = nullptr);
// Cell lists from sorted keys: start, count, mass; gathers entries. With
// fill_cells = P > 0, cell_start (P + 1 entries) becomes a full CSR: an empty
// cell starts where the next occupied one does and cell_start[P] = n;
// otherwise only occupied cells are written. When *sort_failed is set (the
// sort's look-back gave up) nothing is written: the cleared counts leave
// every cell empty, and no key or ID from the sort is used as an index.
cudaError_t launch_cell_build(const uint32_t* keys, const uint32_t* ids, int n,
                              const float4* bodies, const float4* materials, int* cell_start,
                              int* cell_count, uint32_t* cell_mass, float4* entries,
                              int fill_cells, cudaStream_t stream,
                              const uint32_t* sort_failed = nullptr);

// CIC deposit (build_grid.comp:53-69) over cell-ordered entries (keys: their
// sorted cells; cell_start: the full CSR). Writes every mesh cell.
// work: deposit_work_entries(capacity, MW, MH) int4 + 1 counter.
size_t deposit_work_entries(int capacity, int MW, int MH);
// Whether launch_deposit reads cell_start for n bodies (it then needs the full
// CSR); otherwise it reads `keys`.
bool deposit_uses_cell_starts(int n);
cudaError_t launch_deposit(const float4* entries, const uint32_t* keys, const int* cell_start,
                           int n, GridShape g, int deposit_mode, float mass_scale, void* density,
                           int4* work, int* work_count, int work_capacity, cudaStream_t stream);

// Real 2D FFT, spectral multiply and inverse (fft_shared.comp, convolve.comp).
cudaError_t launch_fft_forward_rows(const void* density, int deposit_mode, float inv_scale,
                                    GridShape g, const float2* twiddles, float2* half,
                                    cudaStream_t stream);
cudaError_t launch_fft_columns(const float2* half, const float2* green, float inv_total,
                               GridShape g, const float2* twiddles, float4* cols,
                               cudaStream_t stream);
cudaError_t launch_fft_inverse_rows(const float4* cols, GridShape g, const float2* twiddles,
                                    float2* force, cudaStream_t stream);
// FP64 forward 2D FFT (radix-2, exact sincospi twiddles) of the density mesh
// scaled by inv_scale, into z (MW x MH double2): validateFft's reference.
cudaError_t launch_density_spectrum_f64(const void* density, int deposit_mode, double inv_scale,
                                        GridShape g, double2* z, cudaStream_t stream);
// Forward spectrum only (diagnostic): half-spectrum columns transformed.
cudaError_t launch_fft_forward_columns(float2* half, GridShape g, const float2* twiddles,
                                       cudaStream_t stream);

// FP64 Green's function precompute (kernel_init.comp + 2 forward FFTs +
// convolve.comp's deconvolution), unit total mass.
struct GreenParams {
    float aspect, gravity, sigma_cells, window_floor;
};
cudaError_t build_green(GridShape g, GreenParams p, double2* work, float2* green,
                        cudaStream_t stream);

// Interpolation + short range + half kick (kick.comp:66-156).
struct KickParams {
    int n, W, H, MW, MH, bounded, rx, ry, exact, home_limit, initial, mutual;
    int sr_threads;  // block size of the short-range kernel (64..256)
    // The short range's two-slot form (exact limit 2, at least one body per
    // two cells: it reads the per-cell slot table); else the list walk.
    int slot_form;
    float aspect, gravity, sigma_cells, total_mass, min_frac, dt, field_x, field_y;
};
// Short-range correction over the cell stencil (kick.comp:122-151), one
// thread per body; writes a_short[id]. Radii 1..6.
cudaError_t launch_short_range(const float4* bodies, const float4* entries, const int* cell_start,
                               const int* cell_count, const uint32_t* cell_mass,
                               const float4* slots, float2* a_short, KickParams p,
                               cudaStream_t stream);
// The two source slots of every cell for the two-slot short range (exact
// limit 2): the monopole at the cell centre (count > 2), the first one or
// two list entries, or empty slots (mass 0) at the centre. Two planes of W*H
// cells: float4 (x0, x1, y0, y1), then float2 (G m0 / M_tot, G m1 / M_tot).
cudaError_t launch_cell_slots(const int* cell_start, const int* cell_count,
                              const uint32_t* cell_mass, const float4* entries, int W, int H,
                              float gravity, float total_mass, float4* slots,
                              cudaStream_t stream);
// CIC interpolation + field + a_short, then the half kick (kick.comp:82-103,
// :153-154), one thread per body in ID order.
cudaError_t launch_interp_kick(float4* bodies, float2* accel, const float2* force,
                               const float2* a_short, KickParams p, cudaStream_t stream);

// Reverse pass of one gravity-only step (p3m_adjoint.cu). cv: coefficient of
// the velocity cotangent in the acceleration cotangent (dt/2 for a step, 0
// when folding the initial acceleration a0 = F(x0) into x0); fold: update
// only the position cotangent and clear the acceleration cotangent.
struct AdjointParams {
    int n, W, H, MW, MH, bounded, rx, ry, exact, home_limit, mutual, fold;
    float aspect, gravity, sigma_cells, total_mass, min_frac, dt, cv;
};
// wa = la + cv lv per body, and its CIC spread into `cotangent`, a field of
// 2*MH rows of MW floats (row 2y: x component of row y, row 2y+1: y).
cudaError_t launch_adjoint_spread(const float4* bodies, const float4* lam, const float2* lam_a,
                                  float2* wa, float* cotangent, const AdjointParams& p,
                                  cudaStream_t stream);
// Short-range pair and monopole terms, accumulated into g_short (zeroed).
cudaError_t launch_adjoint_short_range(const float4* bodies, const float4* entries,
                                       const int* cell_start, const int* cell_count,
                                       const uint32_t* cell_mass, const float2* wa,
                                       float2* g_short, const AdjointParams& p,
                                       cudaStream_t stream);
// CIC-gradient gather of m mu + wa . E, plus g_short; then the step's
// cotangent update (or the fold).
cudaError_t launch_adjoint_gather(const float4* bodies, const float4* materials, const float2* wa,
                                  const float2* mu2, const float2* force, const float2* g_short,
                                  float4* lam, float2* lam_a, const AdjointParams& p,
                                  cudaStream_t stream);
// Transposed mesh operator: mu = Kx^T X + Ky^T Y for the interleaved
// cotangent field; mu2[(y >> 1) * MW + x] holds rows 2q and 2q+1 as (x, y).
// half2: 2*MH*(MW/2+1) float2; cols: MH*(MW/2+1) float2 (may alias the
// forward's float4 column buffer).
cudaError_t launch_fft_adjoint(const float* cotangent, const float2* green, float inv_total,
                               GridShape g, const float2* twiddles, float2* half2, float4* cols,
                               float2* mu2, cudaStream_t stream);

// Shared-memory opt-ins, once per device (p3m_create), never during capture.
cudaError_t configure_deposit();
cudaError_t configure_fft();

// Host-side twiddle table: e^{-2 pi i m / 4096}, computed in double.
void host_twiddles(float2* out);

// FP64 diagnostics (p3m_diag.cu).
cudaError_t launch_direct_accel(const float4* bodies, const float4* materials, int n,
                                const int* targets, int n_targets, double aspect, double gravity,
                                double total_mass, double min_dist2, int bounded, double2* out,
                                cudaStream_t stream);
int conservation_blocks();
cudaError_t launch_conservation(const float4* bodies, const float4* materials, int n, double w,
                                double h, double* partial, double* out, cudaStream_t stream);

// Process-wide count of kernels launched by this library (p3m_kernel_launches).
void count_launches(int kernels);

// Kernels of the step's chain start with grid_dependency_wait() and are
// launched by launch_chained with programmatic stream serialization: the
// next kernel's CTAs are dispatched while the previous grid drains, and each
// waits at its first statement until that grid has completed and its writes
// are visible, so the order of the chain is unchanged. Launched the ordinary
// way (or after a memset or event), the wait returns at once.
__device__ __forceinline__ void grid_dependency_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... Params, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                                  cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

// Aim previews (trajectory.comp): one warp per preview, `count` previews.
cudaError_t launch_trajectories(const KickParams& k, float2 viewport, float min_dt, float max_dt,
                                float target_segment_px, float max_path_px, float min_dash_px,
                                float restitution, int steps, int count, const float2* origins_px,
                                const float2* velocities_px, const float2* force,
                                const float4* entries, const int* cell_start,
                                const int* cell_count, const uint32_t* cell_mass,
                                float4* vertices, cudaStream_t stream);

// ------------------------------------------------------- batched launches
// One launch runs a stage for many simulations: CTA b runs local block
// b - first[s] of simulation s, where first[] (sims + 1 entries, on the
// device) is the prefix of the simulations' block counts; a simulation with
// no blocks is skipped. Each launcher takes the per-simulation arguments as a
// device array of its Args struct.
__device__ __forceinline__ int2 batch_block(const int* __restrict__ first, int sims) {
    int lo = 0, hi = sims - 1;
    const int b = (int)blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&first[mid]) <= b) lo = mid;
        else hi = mid - 1;
    }
    return make_int2(lo, b - __ldg(&first[lo]));
}

struct BatchGrid {
    const int* first;  // device, sims + 1
    int sims;
    int blocks;        // first[sims]
};

struct DriftArgs {
    float4* bodies; const float2* accel; uint32_t* keys; uint32_t* vals; unsigned int* nonfinite;
    int n; float half_kick, drift_dt; int substeps, bounded, W, H;
};
struct MortonArgs { const float4* bodies; uint32_t* keys; uint32_t* vals; int n, wbits, hbits; };
struct RadixArgs {
    const uint32_t* keys_in; const uint32_t* vals_in; uint32_t* keys_out; uint32_t* vals_out;
    uint32_t* hist; int n, shift, bits, tiles;
};
struct ScanArgs { uint32_t* data; int n; };
struct PermuteArgs {
    const uint32_t* order; const float4* bodies; const float2* accel; const float4* materials;
    float4* bodies_out; float2* accel_out; float4* materials_out; uint32_t* destinations; int n;
};
// The cell build's entries per 256-thread block (two runs of 32 per warp):
// every form (single context, batched, persistent) cuts its blocks so.
constexpr int kCellBuildItems = 2;
constexpr int kCellBuildBlockEntries = 256 * kCellBuildItems;
struct CellBuildArgs {
    const uint32_t* keys; const uint32_t* ids; const float4* bodies; const float4* materials;
    int* cell_start; int* cell_count; uint32_t* cell_mass; float4* entries; int n;
};
struct ZeroArgs { uint32_t* data; long long words; };  // words of 4 bytes
struct DepositArgs {
    const float4* entries; const uint32_t* keys; void* density; int n, W, H, MW, MH; float scale;
};
struct FftRowsArgs {
    const void* density; float2* half; float inv_scale; int MW, MH, per_cta;
};
struct FftColumnsArgs {
    const float2* half; const float2* green; float4* cols; float inv_total; int MW, MH, per_cta;
};
struct FftInverseArgs { const float4* cols; float2* force; int MW, MH, per_cta; };
struct ShortRangeArgs {
    const float4* bodies; const float4* entries; const int* cell_start; const int* cell_count;
    const uint32_t* cell_mass; const float4* slots; float2* a_short; KickParams p;
};
struct SlotsArgs {
    const int* cell_start; const int* cell_count; const uint32_t* cell_mass; const float4* entries;
    float4* slots; int W, H; float gravity, total_mass;
};
struct KickArgs {
    float4* bodies; float2* accel; const float2* force; const float2* a_short; KickParams p;
};

constexpr int kBatchThreads = 256;      // every batched launch but the scan
constexpr int kBatchScanThreads = 1024;
int radix_tiles(int n);                 // tiles (CTAs) of one radix pass over n keys
int radix_scan_limit();                 // largest histogram one scan CTA takes
int chunk_deposit_blocks(int n);        // CTAs of the entry-chunk deposit
int chunk_deposit_smem();               // its shared window, bytes
void fft_batch_shape(const GridShape& g, int* rows_per_cta, int* cols_per_cta, int* inv_per_cta,
                     size_t* rows_smem, size_t* cols_smem, size_t* inv_smem);

cudaError_t batched_drift(const DriftArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_morton_keys(const MortonArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_radix_hist(const RadixArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_scan(const ScanArgs* a, BatchGrid g, cudaStream_t s);  // one CTA each
cudaError_t batched_radix_scatter(const RadixArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_permute(const PermuteArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_cell_build(const CellBuildArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_zero(const ZeroArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_deposit(const DepositArgs* a, BatchGrid g, int deposit_mode, cudaStream_t s);
cudaError_t batched_fft_rows(const FftRowsArgs* a, BatchGrid g, int deposit_mode, size_t smem,
                             const float2* twiddles, cudaStream_t s);
cudaError_t batched_fft_columns(const FftColumnsArgs* a, BatchGrid g, size_t smem,
                                const float2* twiddles, cudaStream_t s);
cudaError_t batched_fft_inverse(const FftInverseArgs* a, BatchGrid g, size_t smem,
                                const float2* twiddles, cudaStream_t s);
cudaError_t batched_short_range(const ShortRangeArgs* a, BatchGrid g, int rx, int ry, int exact2,
                                cudaStream_t s);
cudaError_t batched_interp_kick(const KickArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t batched_cell_slots(const SlotsArgs* a, BatchGrid g, cudaStream_t s);
cudaError_t configure_batched();

// ---- the batched step as one persistent launch (step/p3m_batch_persistent.cu)
// A stage: `blocks` virtual blocks of the batched body `kind` over `sims`
// simulations; `args` and `first` are byte offsets of its argument array and
// block prefix (sims + 1 ints) in the plan's device blob. A phase: stages
// first_stage .. first_stage + stages - 1, independent of one another; a grid
// barrier separates phases.
enum PStageKind {
    kPStageMorton, kPStageRadixHist, kPStageScan, kPStageRadixScatter, kPStagePermute,
    kPStageCopy, kPStageDrift, kPStageZero, kPStageCellBuild, kPStageSlots,
    kPStageShortRangeSlots, kPStageShortRangeLists, kPStageDepositU32, kPStageDepositI64,
    kPStageFftRowsU32, kPStageFftRowsI64, kPStageFftColumns, kPStageFftInverse, kPStageKick
};
struct PStage { int kind, sims, blocks, args, first; };
struct PPhase { int first_stage, stages; };
struct CopyArgs { const uint32_t* src; uint32_t* dst; long long words; };  // 4-byte words
// The persistent kernel's stencil: the short range stages it runs are (3, 3).
constexpr int kPersistentRx = 3, kPersistentRy = 3;
constexpr int kPersistentMaxStamps = 64;  // per-phase timer stamps of one launch
size_t persistent_base_smem();
int persistent_scan_limit();
int persistent_ctas_per_sm(size_t smem);
cudaError_t launch_batch_persistent(const unsigned char* blob, const PStage* stages,
                                    const PPhase* phases, int n_phases, const float2* tw,
                                    unsigned int* sync, int poll_limit, int withhold_cta,
                                    int withhold_phase, int ctas, size_t smem,
                                    unsigned long long* phase_ns, cudaStream_t stream);

// Sets the message p3m_last_error(NULL) returns on this thread (entry points
// without a context).
void set_detached_error(const std::string& what);

}  // namespace p3m

#include <vector>

// Stage timing: CUDA event pairs recorded on the context's stream.
struct p3m_stage_events {
    int stage;
    cudaEvent_t start, stop;
};

// One captured step. Everything a replay bakes in is part of the key: the
// body count, whether the step starts with a Morton reorder, which of the
// ping-pong body buffers is current, and the scalar uniforms.
struct p3m_step_graph {
    int n;
    bool sort;
    const void* bodies;
    int mutual, bounded, mass_scale;
    float field_x, field_y, total_mass;
    cudaGraphExec_t exec;
    long long kernels;
    uint32_t* sorted_keys;
    uint32_t* sorted_ids;
};

// ------------------------------------------------------------------ context
struct p3m_ctx {
    p3m_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    // The short range needs only the cell lists: in a step it runs on `side`
    // beside the deposit and FFT (fork / join events).
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // p3m_step_io: the host copies on their own streams (one per direction,
    // so upload and download overlap), through device staging buffers; the
    // events order each staging buffer's reuse. Created at the first call.
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    float4* stage_in = nullptr;
    float4* stage_out = nullptr;
    cudaEvent_t in_ready = nullptr, in_free = nullptr, out_ready = nullptr, out_free = nullptr;
    p3m::GridShape grid{};
    bool walls_supported = false;
    float aspect = 1.0f;
    int rx = 1, ry = 1;
    int sort_wbits = 0, sort_hbits = 0;
    int bounded = 0;
    int mutual = 1;
    float field_x = 0.0f, field_y = 0.0f;  // unit/s^2
    float mass_excess = 0.0f;
    float normalization_mass = -1.0f;
    int mass_scale = 1;
    long long physics_steps = 0;
    int green_bounded = -1;  // which mesh the Green's table was built for
    int tune_fft_lines = 0;  // launch shapes chosen by the batch autotuner
    int tune_sr_threads = 256;

    // body state
    float4* bodies = nullptr;
    float4* bodies_alt = nullptr;
    float2* accel = nullptr;
    float2* accel_alt = nullptr;
    float4* materials = nullptr;
    float4* materials_alt = nullptr;
    uint32_t* destinations = nullptr;
    unsigned int* status = nullptr;  // [0] non-finite bodies seen by the drift
    // Page-locked copy of status[0..1], read at the synchronising entry
    // points, and the counts already reported to the caller.
    unsigned int* status_host = nullptr;
    unsigned int reported_nonfinite = 0, reported_timeouts = 0;

    // cell lists
    uint32_t* keys = nullptr;
    uint32_t* vals = nullptr;
    p3m::SortScratch sort;
    uint32_t* sorted_keys = nullptr;  // where the last sort left its result
    uint32_t* sorted_ids = nullptr;
    int* cell_start = nullptr;
    int* cell_count = nullptr;
    uint32_t* cell_mass = nullptr;
    float4* entries = nullptr;
    float4* cell_slots = nullptr;  // per cell: the two source slots of the short range (24 B)
    float2* a_short = nullptr;  // short-range accelerations, by body ID
    int4* deposit_work = nullptr;  // pieces of heavy mesh tiles (+1 counter)
    size_t deposit_work_capacity = 0;

    // mesh
    void* density = nullptr;
    float2* half = nullptr;
    float4* cols = nullptr;
    float2* force = nullptr;
    float2* green = nullptr;
    float2* twiddles = nullptr;
    size_t mesh_capacity = 0;  // cells the mesh buffers hold

    // diagnostics scratch
    double* diag = nullptr;  // conservation partials + result

    // differentiated rollout (checkpoints, recompute slots, cotangents)
    struct p3m_adjoint_store* adjoint = nullptr;

    // aim previews: the body count of the last force build (-1: none), and
    // the staging buffers of p3m_trajectories
    int built_n = -1;
    void* traj_scratch = nullptr;
    size_t traj_scratch_bytes = 0;

    // captured steps (CUDA graphs)
    bool use_graphs = true;
    std::vector<p3m_step_graph> graphs;

    // stage profiler
    bool profiling = false;
    std::vector<p3m_stage_events> pending;  // recorded, not yet folded
    std::vector<cudaEvent_t> free_events;
    double stage_ms[P3M_STAGE_COUNT_] = {};
    long long stage_intervals[P3M_STAGE_COUNT_] = {};

    std::string last_error;
};
