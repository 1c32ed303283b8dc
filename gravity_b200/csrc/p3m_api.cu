// p3m_api.cu — the C-ABI of include/p3m.h: context lifecycle, state hand-off
// and the orchestration of GravityPipeline's P3M step
// (src/main/kotlin/dev/gravity/GravityPipeline.kt).

#include "p3m_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <functional>
#include <map>
#include <vector>

namespace p3m {
namespace {
std::atomic<long long> g_launches{0};
}
void count_launches(int kernels) { g_launches.fetch_add(kernels, std::memory_order_relaxed); }
}  // namespace p3m

namespace {

thread_local std::string g_create_error;

int fail(p3m_ctx* ctx, int status, const std::string& what) {
    if (ctx) ctx->last_error = what;
    else g_create_error = what;
    return status;
}

int fail_cuda(p3m_ctx* ctx, const char* where, cudaError_t e) {
    std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(ctx, e == cudaErrorMemoryAllocation ? P3M_ERR_OUT_OF_MEMORY : P3M_ERR_CUDA, m);
}

#define P3M_CUDA(ctx, expr)                                   \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return fail_cuda(ctx, #expr, e_); \
    } while (0)

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

int log2_floor(int v) {
    int b = 0;
    while ((1 << (b + 1)) <= v) ++b;
    return b;
}

int bits_for(long long count) {  // ceil(log2(count)), at least 1
    int b = 1;
    while ((1LL << b) < count) ++b;
    return b;
}

// ------------------------------------------------------------ stage timing
cudaEvent_t take_event(p3m_ctx* ctx) {
    if (!ctx->free_events.empty()) {
        cudaEvent_t e = ctx->free_events.back();
        ctx->free_events.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Folds recorded intervals into the per-stage totals (waits for them).
void fold_stages(p3m_ctx* ctx) {
    if (ctx->pending.empty()) return;
    cudaEventSynchronize(ctx->pending.back().stop);
    for (const auto& p : ctx->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
            ctx->stage_ms[p.stage] += ms;
            ctx->stage_intervals[p.stage] += 1;
        }
        ctx->free_events.push_back(p.start);
        ctx->free_events.push_back(p.stop);
    }
    ctx->pending.clear();
}

// Records one stage interval around a scope when profiling is on.
struct StageScope {
    p3m_ctx* ctx;
    int stage;
    cudaEvent_t start = nullptr;
    StageScope(p3m_ctx* c, int s) : ctx(c), stage(s) {
        if (ctx->profiling) {
            start = take_event(ctx);
            if (start) cudaEventRecord(start, ctx->stream);
        }
    }
    ~StageScope() {
        if (!start) return;
        cudaEvent_t stop = take_event(ctx);
        if (!stop) return;
        cudaEventRecord(stop, ctx->stream);
        ctx->pending.push_back({stage, start, stop});
        if (ctx->pending.size() >= 4096) fold_stages(ctx);
    }
};

// GravityPipeline.kt:1649-1650 sortAxisBits.
int sort_axis_bits(int extent) { return std::min(10, log2_floor(std::max(1, extent / 4))); }

// GravityPipeline.kt:1546-1547 massScaleFor.
int mass_scale_for(float total_mass) {
    const double v = 4000000000.0 / (double)total_mass;
    const long long s = (long long)v;
    return (int)std::min(std::max(s, 1LL), 65536LL);
}

// GravityPipeline.kt:153-169, in Float arithmetic like the Kotlin code.
void neighbor_radii(const p3m_config& c, int* rx, int* ry) {
    const float aspect = (float)c.viewport_width / (float)c.viewport_height;
    const float vx = c.local_search_sigma_multiplier * c.softening_cells * (float)c.grid_width /
                     ((float)c.grid_height * aspect);
    const float vy = c.softening_cells * c.local_search_sigma_multiplier;
    *rx = std::min(std::max((int)std::ceil(vx), c.minimum_neighbor_radius_cells),
                   c.maximum_neighbor_radius_cells);
    *ry = std::min(std::max((int)std::ceil(vy), c.minimum_neighbor_radius_cells),
                   c.maximum_neighbor_radius_cells);
}

// GravityFieldConfig.init (GravityConfig.kt:655-673) with the grid range
// widened to 16..4096 (the reference caps it at 128..2048 because its FFT line
// lives in a 2048-entry shared array, fft_shared.comp:12-14).
int validate(const p3m_config* c, std::string* why) {
    if (!c) { *why = "config is NULL"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->struct_size != (int)sizeof(p3m_config)) {
        *why = "config.struct_size does not match this library's p3m_config";
        return P3M_ERR_INVALID_ARGUMENT;
    }
    if (!pow2(c->grid_width) || c->grid_width < 16 || c->grid_width > p3m::kMaxMeshAxis) {
        *why = "grid width must be a power of two in 16..4096";
        return P3M_ERR_UNSUPPORTED;
    }
    if (!pow2(c->grid_height) || c->grid_height < 16 || c->grid_height > p3m::kMaxMeshAxis) {
        *why = "grid height must be a power of two in 16..4096";
        return P3M_ERR_UNSUPPORTED;
    }
    if (c->viewport_width <= 0 || c->viewport_height <= 0) { *why = "viewport must be positive"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->gravitational_constant >= 0.0f) || !std::isfinite(c->gravitational_constant)) { *why = "gravitational constant must be finite and >= 0"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->softening_cells > 0.0f) || !std::isfinite(c->softening_cells)) { *why = "softening must be finite and > 0"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->local_search_sigma_multiplier > 0.0f) || !std::isfinite(c->local_search_sigma_multiplier)) { *why = "search multiplier must be finite and > 0"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->minimum_neighbor_radius_cells < 1) { *why = "minimum neighbour radius must be >= 1"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->maximum_neighbor_radius_cells < c->minimum_neighbor_radius_cells) { *why = "maximum neighbour radius below minimum"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->exact_neighbor_body_limit < 1) { *why = "exact neighbour body limit must be >= 1"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->maximum_home_body_interactions < 1) { *why = "home interactions must be >= 1"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->minimum_distance_cell_fraction > 0.0f) || !std::isfinite(c->minimum_distance_cell_fraction)) { *why = "minimum distance fraction must be finite and > 0"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->minimum_assignment_window_power > 0.0f) || c->minimum_assignment_window_power > 1.0f) { *why = "window power floor must be in (0, 1]"; return P3M_ERR_INVALID_ARGUMENT; }
    if (!(c->time_step > 0.0f) || !std::isfinite(c->time_step)) { *why = "time step must be finite and > 0"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->drift_substeps < 1) { *why = "drift substeps must be >= 1"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->spatial_sort_interval < 0) { *why = "sort interval must be non-negative"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->capacity <= 0 || c->capacity > (1 << 28)) { *why = "capacity must be in 1..2^28"; return P3M_ERR_INVALID_ARGUMENT; }
    if (c->deposit_mode != P3M_DEPOSIT_U32 && c->deposit_mode != P3M_DEPOSIT_I64) { *why = "unknown deposit mode"; return P3M_ERR_INVALID_ARGUMENT; }
    {
        int rx = 1, ry = 1;
        neighbor_radii(*c, &rx, &ry);
        if (rx > 6 || ry > 6) {
            *why = "neighbour radii above 6 cells are not supported";
            return P3M_ERR_UNSUPPORTED;
        }
    }
    if (c->bounded && 2 * std::max(c->grid_width, c->grid_height) > p3m::kMaxMeshAxis) {
        *why = "walls need an FFT grid of at most 2048 cells per axis";
        return P3M_ERR_UNSUPPORTED;
    }
    return P3M_OK;
}

p3m::GridShape grid_for(const p3m_ctx* ctx) {
    p3m::GridShape g;
    g.W = ctx->cfg.grid_width;
    g.H = ctx->cfg.grid_height;
    g.bounded = ctx->bounded;
    g.MW = ctx->bounded ? 2 * g.W : g.W;
    g.MH = ctx->bounded ? 2 * g.H : g.H;
    g.fft_lines = ctx->tune_fft_lines;
    return g;
}

size_t mesh_cells(const p3m_ctx* ctx) { return (size_t)ctx->grid.MW * ctx->grid.MH; }
size_t half_cells(const p3m_ctx* ctx) { return (size_t)(ctx->grid.MW / 2 + 1) * ctx->grid.MH; }
size_t phys_cells(const p3m_ctx* ctx) { return (size_t)ctx->grid.W * ctx->grid.H; }

template <typename T>
int dalloc(p3m_ctx* ctx, T** p, size_t count, const char* what) {
    void* v = nullptr;
    cudaError_t e = cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail_cuda(ctx, what, e);
    *p = static_cast<T*>(v);
    return P3M_OK;
}

void adjoint_free(p3m_ctx* ctx);

void free_all(p3m_ctx* ctx) {
    adjoint_free(ctx);
    for (cudaStream_t s : {ctx->up_stream, ctx->down_stream})
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    ctx->up_stream = ctx->down_stream = nullptr;
    for (cudaEvent_t* e : {&ctx->in_ready, &ctx->in_free, &ctx->out_ready, &ctx->out_free})
        if (*e) {
            cudaEventDestroy(*e);
            *e = nullptr;
        }
    if (ctx->stage_in) cudaFree(ctx->stage_in);
    if (ctx->stage_out) cudaFree(ctx->stage_out);
    ctx->stage_in = ctx->stage_out = nullptr;
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    ctx->ev_fork = ctx->ev_join = nullptr;
    ctx->side = nullptr;
    fold_stages(ctx);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
    for (cudaEvent_t e : ctx->free_events) cudaEventDestroy(e);
    ctx->free_events.clear();
    if (ctx->traj_scratch) cudaFree(ctx->traj_scratch);
    ctx->traj_scratch = nullptr;
    if (ctx->status_host) cudaFreeHost(ctx->status_host);
    ctx->status_host = nullptr;
    void* ptrs[] = {ctx->diag, ctx->bodies, ctx->bodies_alt, ctx->accel, ctx->accel_alt, ctx->materials,
                    ctx->materials_alt, ctx->destinations, ctx->status, ctx->keys, ctx->vals,
                    ctx->sort.keys_alt, ctx->sort.vals_alt, ctx->sort.hist, ctx->sort.block_sums,
                    ctx->sort.lookback,
                    ctx->cell_start, ctx->cell_count, ctx->entries, ctx->cell_slots,
                    ctx->a_short, ctx->deposit_work, ctx->density,
                    ctx->half, ctx->cols, ctx->force, ctx->green, ctx->twiddles};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

// (Re)builds the Green's table when the mesh changed (initializeKernel on a
// `bounded` change, GravityPipeline.kt:97-103). The table is for unit total
// mass; normalizeTo only changes the 1/M_tot factor the spectral pass applies.
int ensure_green(p3m_ctx* ctx) {
    if (ctx->green_bounded == ctx->bounded) return P3M_OK;
    ctx->grid = grid_for(ctx);
    double2* work = nullptr;
    P3M_CUDA(ctx, cudaMallocAsync((void**)&work, mesh_cells(ctx) * sizeof(double2), ctx->stream));
    p3m::GreenParams gp{ctx->aspect, ctx->cfg.gravitational_constant, ctx->cfg.softening_cells,
                        ctx->cfg.minimum_assignment_window_power};
    cudaError_t e = p3m::build_green(ctx->grid, gp, work, ctx->green, ctx->stream);
    cudaFreeAsync(work, ctx->stream);
    if (e != cudaSuccess) return fail_cuda(ctx, "build_green", e);
    ctx->green_bounded = ctx->bounded;
    return P3M_OK;
}

// GravityPipeline.kt:1326-1331 normalizeTo.
void normalize_to(p3m_ctx* ctx, int n) {
    const float mass = std::max(1.0f, (float)n + ctx->mass_excess);
    if (mass == ctx->normalization_mass) return;
    ctx->normalization_mass = mass;
    ctx->mass_scale = mass_scale_for(mass);
}

int check_n(p3m_ctx* ctx, int n) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (n < 0) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "body count must be >= 0");
    if (n > ctx->cfg.capacity) return fail(ctx, P3M_ERR_CAPACITY, "body count exceeds capacity");
    return P3M_OK;
}

// Queues a copy of the device status words into status_host; read it with
// device_failures() once the stream is synchronised.
cudaError_t queue_status_read(p3m_ctx* ctx) {
    return cudaMemcpyAsync(ctx->status_host, ctx->status, 2 * sizeof(unsigned int),
                           cudaMemcpyDeviceToHost, ctx->stream);
}

// Failures the device detected since the last report, from status_host
// (queue_status_read and a stream synchronisation first): a bounded look-back
// wait that gave up (P3M_ERR_TIMEOUT; every result computed since is
// untrustworthy), then, when `nonfinite` is set, bodies that became non-finite
// (P3M_ERR_NON_FINITE). Each is reported once.
int device_failures(p3m_ctx* ctx, bool nonfinite) {
    const unsigned int waits = ctx->status_host[1];
    const unsigned int bad = ctx->status_host[0];
    if (waits != ctx->reported_timeouts) {
        const unsigned int grown = waits - ctx->reported_timeouts;
        ctx->reported_timeouts = waits;
        return fail(ctx, P3M_ERR_TIMEOUT,
                    std::to_string(grown) + " bounded look-back wait(s) of a sort gave up; "
                    "the cell lists and everything computed from them since are invalid");
    }
    if (nonfinite && bad != ctx->reported_nonfinite) {
        const unsigned int grown = bad - ctx->reported_nonfinite;
        ctx->reported_nonfinite = bad;
        return fail(ctx, P3M_ERR_NON_FINITE,
                    std::to_string(grown) + " non-finite body state(s) seen by the drift");
    }
    return P3M_OK;
}

// Cell lists from keys already written in descending ID order.
// totals_ready: radix_sort_prepare ran and the keys' producer (the drift)
// added their digit totals.
int lists_from_keys(p3m_ctx* ctx, int n, bool totals_ready = false) {
    StageScope scope(ctx, P3M_STAGE_CELL_LISTS);
    const long long P = (long long)phys_cells(ctx);
    uint32_t* sk = ctx->keys;
    uint32_t* sv = ctx->vals;
    const uint32_t* failed = nullptr;
    P3M_CUDA(ctx, p3m::radix_sort_pairs(ctx->keys, ctx->vals, ctx->sort, n, bits_for(P),
                                        ctx->stream, &sk, &sv, totals_ready, &failed));
    ctx->sorted_keys = sk;
    ctx->sorted_ids = sv;
    // Counts and masses are one block (cell_mass follows cell_count): one clear.
    P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_count, 0, 2 * P * sizeof(int), ctx->stream));
    P3M_CUDA(ctx, p3m::launch_cell_build(sk, sv, n, ctx->bodies, ctx->materials, ctx->cell_start,
                                         ctx->cell_count, ctx->cell_mass, ctx->entries,
                                         p3m::deposit_uses_cell_starts(n) ? (int)P : 0,
                                         ctx->stream, failed));
    return P3M_OK;
}

// Deposit + FFT + spectral multiply + inverse (GravityPipeline.kt:907-973
// after the lists).
int mesh_force(p3m_ctx* ctx, int n) {
    int st = ensure_green(ctx);
    if (st != P3M_OK) return st;
    const bool i64 = ctx->cfg.deposit_mode == P3M_DEPOSIT_I64;
    {
        StageScope scope(ctx, P3M_STAGE_DEPOSIT);
        P3M_CUDA(ctx, p3m::launch_deposit(ctx->entries, ctx->sorted_keys, ctx->cell_start, n, ctx->grid,
                                          ctx->cfg.deposit_mode, (float)ctx->mass_scale,
                                          ctx->density, ctx->deposit_work,
                                          reinterpret_cast<int*>(ctx->deposit_work +
                                                                 ctx->deposit_work_capacity),
                                          (int)ctx->deposit_work_capacity, ctx->stream));
    }
    // fft_init.comp's uInverseMassScale = 1f / massScale (GravityPipeline.kt:942).
    const float inv_scale = i64 ? 1.0f / 4294967296.0f : 1.0f / (float)ctx->mass_scale;
    {
        StageScope scope(ctx, P3M_STAGE_FORWARD_FFT);
        P3M_CUDA(ctx, p3m::launch_fft_forward_rows(ctx->density, ctx->cfg.deposit_mode, inv_scale,
                                                   ctx->grid, ctx->twiddles, ctx->half,
                                                   ctx->stream));
    }
    {
        StageScope scope(ctx, P3M_STAGE_SPECTRAL);
        P3M_CUDA(ctx, p3m::launch_fft_columns(ctx->half, ctx->green,
                                              1.0f / ctx->normalization_mass, ctx->grid,
                                              ctx->twiddles, ctx->cols, ctx->stream));
    }
    {
        StageScope scope(ctx, P3M_STAGE_INVERSE_FFT);
        P3M_CUDA(ctx, p3m::launch_fft_inverse_rows(ctx->cols, ctx->grid, ctx->twiddles,
                                                   ctx->force, ctx->stream));
    }
    ctx->built_n = n;
    return P3M_OK;
}

int build_force(p3m_ctx* ctx, int n) {
    P3M_CUDA(ctx, p3m::launch_cell_keys(ctx->bodies, n, ctx->grid, ctx->keys, ctx->vals, ctx->stream));
    int st = lists_from_keys(ctx, n);
    if (st != P3M_OK) return st;
    return mesh_force(ctx, n);
}

p3m::KickParams kick_params(const p3m_ctx* ctx, int n, int initial) {
    p3m::KickParams p;
    p.n = n;
    p.W = ctx->grid.W; p.H = ctx->grid.H; p.MW = ctx->grid.MW; p.MH = ctx->grid.MH;
    p.bounded = ctx->bounded; p.rx = ctx->rx; p.ry = ctx->ry;
    p.exact = ctx->cfg.exact_neighbor_body_limit;
    p.home_limit = ctx->cfg.maximum_home_body_interactions;
    p.initial = initial; p.mutual = ctx->mutual;
    p.aspect = ctx->aspect; p.gravity = ctx->cfg.gravitational_constant;
    p.sigma_cells = ctx->cfg.softening_cells; p.total_mass = ctx->normalization_mass;
    p.min_frac = ctx->cfg.minimum_distance_cell_fraction; p.dt = ctx->cfg.time_step;
    p.field_x = ctx->field_x; p.field_y = ctx->field_y;
    p.sr_threads = ctx->tune_sr_threads;
    // Two-slot form for exact limit 2 unless the simulation is sparse (under
    // one body per two cells): the slot table of mostly empty cells then
    // costs more than the list walk it saves.
    p.slot_form = p.exact == 2 && 2 * (long long)n >= (long long)phys_cells(ctx);
    return p;
}

// The short range over the current cell lists; with exact limit 2 it reads
// the per-cell slot table, built first on the same stream.
int short_range(p3m_ctx* ctx, const p3m::KickParams& p, cudaStream_t stream) {
    if (p.slot_form && p.n > 0)
        P3M_CUDA(ctx, p3m::launch_cell_slots(ctx->cell_start, ctx->cell_count, ctx->cell_mass,
                                             ctx->entries, ctx->grid.W, ctx->grid.H,
                                             p.gravity, p.total_mass, ctx->cell_slots, stream));
    P3M_CUDA(ctx, p3m::launch_short_range(ctx->bodies, ctx->entries, ctx->cell_start,
                                          ctx->cell_count, ctx->cell_mass, ctx->cell_slots,
                                          ctx->a_short, p, stream));
    return P3M_OK;
}

int apply_kick(p3m_ctx* ctx, int n, int initial, bool with_short_range = true) {
    const p3m::KickParams p = kick_params(ctx, n, initial);
    if (ctx->mutual && with_short_range) {
        StageScope scope(ctx, P3M_STAGE_SHORT_RANGE);
        const int st = short_range(ctx, p, ctx->stream);
        if (st != P3M_OK) return st;
    }
    StageScope scope(ctx, P3M_STAGE_KICK);
    P3M_CUDA(ctx, p3m::launch_interp_kick(ctx->bodies, ctx->accel, ctx->force, ctx->a_short, p,
                                          ctx->stream));
    return P3M_OK;
}

// GravityPipeline.kt:1269-1319 sortBodies.
int sort_bodies(p3m_ctx* ctx, int n) {
    if (n <= 0) return P3M_OK;
    StageScope scope(ctx, P3M_STAGE_SPATIAL_SORT);
    const int key_bits = ctx->sort_wbits + ctx->sort_hbits;
    p3m::SortTotals totals;  // the key kernel adds the sort's digit totals
    P3M_CUDA(ctx, p3m::radix_sort_prepare(ctx->sort, n, key_bits, ctx->stream, &totals));
    P3M_CUDA(ctx, p3m::launch_morton_keys(ctx->bodies, n, ctx->sort_wbits, ctx->sort_hbits,
                                          ctx->keys, ctx->vals, ctx->stream, totals));
    uint32_t* sk = ctx->keys;
    uint32_t* sv = ctx->vals;
    const uint32_t* failed = nullptr;
    P3M_CUDA(ctx, p3m::radix_sort_pairs(ctx->keys, ctx->vals, ctx->sort, n, key_bits, ctx->stream,
                                        &sk, &sv, totals.totals != nullptr, &failed));
    P3M_CUDA(ctx, p3m::launch_permute(sv, n, ctx->bodies, ctx->accel, ctx->materials,
                                      ctx->bodies_alt, ctx->accel_alt, ctx->materials_alt,
                                      ctx->destinations, ctx->stream, failed));
    // Slots beyond n (capacity reserved for bodies a caller adds later) keep
    // their contents: carry them into the buffers that become current.
    const size_t tail = (size_t)ctx->cfg.capacity - (size_t)n;
    if (tail > 0) {
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->bodies_alt + n, ctx->bodies + n, tail * sizeof(float4),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->accel_alt + n, ctx->accel + n, tail * sizeof(float2),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->materials_alt + n, ctx->materials + n,
                                      tail * sizeof(float4), cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    }
    std::swap(ctx->bodies, ctx->bodies_alt);
    std::swap(ctx->accel, ctx->accel_alt);
    std::swap(ctx->materials, ctx->materials_alt);
    return P3M_OK;
}

// One gravity-only step (GravityPipeline.kt:445-494 without collisions).
int enqueue_step(p3m_ctx* ctx, int n, bool do_sort) {
    if (do_sort) {
        int st = sort_bodies(ctx, n);
        if (st != P3M_OK) return st;
    }
    // Collision substeps drift the bodies: substep 0 half-kicks with the
    // stored acceleration (GravityPipeline.kt:465-473); the fused kernel also
    // writes the home-cell keys.
    const float dt = ctx->cfg.time_step;
    const float drift_dt = dt / (float)ctx->cfg.drift_substeps;
    p3m::SortTotals totals;  // the drift adds the cell sort's digit totals
    {
        StageScope scope(ctx, P3M_STAGE_DRIFT);
        if (ctx->mutual)
            P3M_CUDA(ctx, p3m::radix_sort_prepare(ctx->sort, n, bits_for(phys_cells(ctx)),
                                                  ctx->stream, &totals));
        P3M_CUDA(ctx, p3m::launch_drift(ctx->bodies, ctx->accel, n, 0.5f * dt, drift_dt,
                                        ctx->cfg.drift_substeps, ctx->grid, ctx->keys, ctx->vals,
                                        ctx->status, ctx->stream, totals));
    }
    if (ctx->mutual) {
        int st = lists_from_keys(ctx, n, totals.totals != nullptr);
        if (st != P3M_OK) return st;
        // The short range reads only the lists: outside the profiler it runs
        // on the side stream beside the deposit and FFT.
        const bool overlap = !ctx->profiling && n > 0;
        if (overlap) {
            P3M_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
            P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
            st = short_range(ctx, kick_params(ctx, n, 0), ctx->side);
            if (st != P3M_OK) return st;
            P3M_CUDA(ctx, cudaEventRecord(ctx->ev_join, ctx->side));
        }
        st = mesh_force(ctx, n);
        if (st != P3M_OK) return st;
        if (overlap) {
            P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
            return apply_kick(ctx, n, 0, false);
        }
    }
    return apply_kick(ctx, n, 0);
}

void swap_body_buffers(p3m_ctx* ctx) {
    std::swap(ctx->bodies, ctx->bodies_alt);
    std::swap(ctx->accel, ctx->accel_alt);
    std::swap(ctx->materials, ctx->materials_alt);
}

void drop_graphs(p3m_ctx* ctx) {
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
    ctx->graphs.clear();
}

bool graph_matches(const p3m_step_graph& g, const p3m_ctx* ctx, int n, bool do_sort) {
    return g.n == n && g.sort == do_sort && g.bodies == ctx->bodies && g.mutual == ctx->mutual &&
           g.bounded == ctx->bounded && g.mass_scale == ctx->mass_scale &&
           g.field_x == ctx->field_x && g.field_y == ctx->field_y &&
           g.total_mass == ctx->normalization_mass;
}

int one_step(p3m_ctx* ctx, int n) {
    normalize_to(ctx, n);
    int st = ensure_green(ctx);
    if (st != P3M_OK) return st;
    const int interval = ctx->cfg.spatial_sort_interval;
    const bool do_sort = interval > 0 && (ctx->physics_steps % interval) == 0;
    if (interval > 0) ctx->physics_steps++;
    if (!ctx->use_graphs || ctx->profiling || n == 0) return enqueue_step(ctx, n, do_sort);

    for (const auto& g : ctx->graphs) {
        if (!graph_matches(g, ctx, n, do_sort)) continue;
        P3M_CUDA(ctx, cudaGraphLaunch(g.exec, ctx->stream));
        p3m::count_launches((int)g.kernels);
        if (ctx->mutual) ctx->built_n = n;
        if (do_sort) swap_body_buffers(ctx);
        ctx->sorted_keys = g.sorted_keys;
        ctx->sorted_ids = g.sorted_ids;
        return P3M_OK;
    }
    // Capture the step once for this key, then launch it.
    p3m_step_graph entry{};
    entry.n = n;
    entry.sort = do_sort;
    entry.bodies = ctx->bodies;
    entry.mutual = ctx->mutual;
    entry.bounded = ctx->bounded;
    entry.mass_scale = ctx->mass_scale;
    entry.field_x = ctx->field_x;
    entry.field_y = ctx->field_y;
    entry.total_mass = ctx->normalization_mass;
    float4* const saved[4] = {ctx->bodies, ctx->bodies_alt, ctx->materials, ctx->materials_alt};
    float2* const saved_accel[2] = {ctx->accel, ctx->accel_alt};
    const long long k0 = p3m_kernel_launches();
    P3M_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    st = enqueue_step(ctx, n, do_sort);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != P3M_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        // Nothing ran: put the buffer roles back as they were.
        ctx->bodies = saved[0];
        ctx->bodies_alt = saved[1];
        ctx->materials = saved[2];
        ctx->materials_alt = saved[3];
        ctx->accel = saved_accel[0];
        ctx->accel_alt = saved_accel[1];
        if (st != P3M_OK) return st;
        return fail_cuda(ctx, "cudaStreamEndCapture", e);
    }
    entry.kernels = p3m_kernel_launches() - k0;
    e = cudaGraphInstantiate(&entry.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail_cuda(ctx, "cudaGraphInstantiate", e);
    entry.sorted_keys = ctx->sorted_keys;
    entry.sorted_ids = ctx->sorted_ids;
    if (ctx->graphs.size() >= 8) {
        cudaGraphExecDestroy(ctx->graphs.front().exec);
        ctx->graphs.erase(ctx->graphs.begin());
    }
    ctx->graphs.push_back(entry);
    P3M_CUDA(ctx, cudaGraphLaunch(entry.exec, ctx->stream));
    return P3M_OK;
}

size_t buffer_bytes(const p3m_ctx* ctx, int which, void** dptr) {
    const size_t cap = (size_t)ctx->cfg.capacity;
    const bool i64 = ctx->cfg.deposit_mode == P3M_DEPOSIT_I64;
    switch (which) {
        case P3M_BUF_BODIES: *dptr = ctx->bodies; return cap * 16;
        case P3M_BUF_ACCELERATION: *dptr = ctx->accel; return cap * 8;
        case P3M_BUF_MATERIALS: *dptr = ctx->materials; return cap * 16;
        case P3M_BUF_CELL_KEYS: *dptr = ctx->sorted_keys ? ctx->sorted_keys : ctx->keys; return cap * 4;
        case P3M_BUF_CELL_BODIES: *dptr = ctx->sorted_ids ? ctx->sorted_ids : ctx->vals; return cap * 4;
        case P3M_BUF_CELL_START: *dptr = ctx->cell_start; return phys_cells(ctx) * 4;
        case P3M_BUF_CELL_COUNT: *dptr = ctx->cell_count; return phys_cells(ctx) * 4;
        case P3M_BUF_CELL_MASS: *dptr = ctx->cell_mass; return phys_cells(ctx) * 4;
        case P3M_BUF_DENSITY: *dptr = ctx->density; return mesh_cells(ctx) * (i64 ? 8 : 4);
        case P3M_BUF_FORCE: *dptr = ctx->force; return mesh_cells(ctx) * 8;
        case P3M_BUF_DESTINATIONS: *dptr = ctx->destinations; return cap * 4;
        case P3M_BUF_GREEN: *dptr = ctx->green; return half_cells(ctx) * 8;
        default: *dptr = nullptr; return 0;
    }
}

int autotune_context(p3m_ctx* c, int n, int trial_steps, int* best_fft_out, int* best_sr_out);

}  // namespace

namespace p3m {
void set_detached_error(const std::string& what) { g_create_error = what; }
}  // namespace p3m

extern "C" {

int p3m_config_default(p3m_config* c) {
    if (!c) return P3M_ERR_INVALID_ARGUMENT;
    std::memset(c, 0, sizeof(*c));
    c->struct_size = (int32_t)sizeof(p3m_config);
    c->viewport_width = 2560;
    c->viewport_height = 1440;
    c->grid_width = 512;
    c->grid_height = 256;
    c->gravitational_constant = 0.035f;
    c->softening_cells = 0.85f;
    c->local_search_sigma_multiplier = 3.0f;
    c->minimum_neighbor_radius_cells = 1;
    c->maximum_neighbor_radius_cells = 6;
    c->exact_neighbor_body_limit = 2;
    c->maximum_home_body_interactions = 8;
    c->minimum_distance_cell_fraction = 0.05f;
    c->minimum_assignment_window_power = 0.08f;
    c->time_step = 1.0f / 120.0f;
    c->drift_substeps = 16;
    c->spatial_sort_interval = 2;
    c->capacity = 400000;
    c->bounded = 0;
    c->deposit_mode = P3M_DEPOSIT_U32;
    c->mutual_gravity = 1;
    return P3M_OK;
}

const char* p3m_status_string(int status) {
    switch (status) {
        case P3M_OK: return "ok";
        case P3M_ERR_INVALID_ARGUMENT: return "invalid argument";
        case P3M_ERR_OUT_OF_MEMORY: return "out of device memory";
        case P3M_ERR_CUDA: return "CUDA error";
        case P3M_ERR_TIMEOUT: return "device wait timed out";
        case P3M_ERR_NON_FINITE: return "non-finite body state";
        case P3M_ERR_CAPACITY: return "body count exceeds capacity";
        case P3M_ERR_UNSUPPORTED: return "unsupported configuration";
        case P3M_ERR_STATE: return "invalid state";
        default: return "unknown status";
    }
}

const char* p3m_last_error(const p3m_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

int p3m_create(const p3m_config* config, p3m_ctx** out) {
    g_create_error.clear();
    if (!out) return fail(nullptr, P3M_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    std::string why;
    int st = validate(config, &why);
    if (st != P3M_OK) return fail(nullptr, st, why);

    p3m_ctx* ctx = new (std::nothrow) p3m_ctx();
    if (!ctx) return fail(nullptr, P3M_ERR_OUT_OF_MEMORY, "host allocation failed");
    ctx->cfg = *config;
    cudaError_t e = cudaGetDevice(&ctx->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        fail_cuda(nullptr, "cudaStreamCreate", e);
        if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return P3M_ERR_CUDA;
    }
    ctx->aspect = (float)config->viewport_width / (float)config->viewport_height;
    neighbor_radii(*config, &ctx->rx, &ctx->ry);
    ctx->sort_wbits = sort_axis_bits(config->viewport_width);
    ctx->sort_hbits = sort_axis_bits(config->viewport_height);
    ctx->bounded = config->bounded;
    ctx->mutual = config->mutual_gravity;
    ctx->walls_supported = 2 * std::max(config->grid_width, config->grid_height) <= p3m::kMaxMeshAxis;
    ctx->grid = grid_for(ctx);

    const size_t cap = (size_t)config->capacity;
    const size_t P = (size_t)config->grid_width * config->grid_height;
    const int mw_max = ctx->walls_supported ? 2 * config->grid_width : config->grid_width;
    const int mh_max = ctx->walls_supported ? 2 * config->grid_height : config->grid_height;
    const size_t M = (size_t)mw_max * mh_max;
    const size_t HALF = (size_t)(mw_max / 2 + 1) * mh_max;
    ctx->mesh_capacity = M;
    ctx->sort.capacity = (int)cap;

#define ALLOC(ptr, count)                                              \
    do {                                                               \
        int s_ = dalloc(ctx, &(ptr), (count), "cudaMalloc(" #ptr ")"); \
        if (s_ != P3M_OK) { g_create_error = ctx->last_error; free_all(ctx); cudaStreamDestroy(ctx->stream); delete ctx; return s_; } \
    } while (0)
    ALLOC(ctx->bodies, cap);
    ALLOC(ctx->bodies_alt, cap);
    ALLOC(ctx->accel, cap);
    ALLOC(ctx->accel_alt, cap);
    ALLOC(ctx->materials, cap);
    ALLOC(ctx->materials_alt, cap);
    ALLOC(ctx->destinations, cap);
    ALLOC(ctx->status, 4);  // [0] non-finite bodies, [1] look-back waits that gave up
    ctx->sort.wait_timeouts = ctx->status + 1;
    {
        cudaError_t he = cudaHostAlloc((void**)&ctx->status_host, 4 * sizeof(unsigned int),
                                       cudaHostAllocDefault);
        if (he != cudaSuccess) {
            ctx->status_host = nullptr;
            fail_cuda(ctx, "cudaHostAlloc(status_host)", he);
            g_create_error = ctx->last_error;
            free_all(ctx);
            cudaStreamDestroy(ctx->stream);
            delete ctx;
            return he == cudaErrorMemoryAllocation ? P3M_ERR_OUT_OF_MEMORY : P3M_ERR_CUDA;
        }
    }
    ALLOC(ctx->keys, cap);
    ALLOC(ctx->vals, cap);
    ALLOC(ctx->sort.keys_alt, cap);
    ALLOC(ctx->sort.vals_alt, cap);
    ALLOC(ctx->sort.hist, p3m::sort_hist_entries((int)cap));
    ALLOC(ctx->sort.block_sums, p3m::sort_block_sum_entries((int)cap));
    ALLOC(ctx->sort.lookback, p3m::sort_lookback_words((int)cap));
    ALLOC(ctx->cell_start, P + 1);
    ALLOC(ctx->cell_count, 2 * P);  // counts, then the masses (cleared together)
    ctx->cell_mass = reinterpret_cast<uint32_t*>(ctx->cell_count + P);
    ALLOC(ctx->cell_slots, (3 * P + 1) / 2);  // float4 plane + float2 plane
    ALLOC(ctx->entries, cap);
    ALLOC(ctx->a_short, cap);
    ctx->deposit_work_capacity = p3m::deposit_work_entries((int)cap, mw_max, mh_max);
    ALLOC(ctx->deposit_work, ctx->deposit_work_capacity + 1);  // + the counter
    {
        unsigned long long* d = nullptr;
        ALLOC(d, M);  // 8 bytes per cell holds either deposit mode
        ctx->density = d;
    }
    ALLOC(ctx->half, HALF);
    ALLOC(ctx->cols, HALF);
    ALLOC(ctx->force, M);
    ALLOC(ctx->green, HALF);
    ALLOC(ctx->twiddles, p3m::kTwiddleLength);
    ALLOC(ctx->diag, (size_t)p3m::conservation_blocks() * 6 + 8);
#undef ALLOC

    auto init = [&]() -> int {
        P3M_CUDA(ctx, p3m::configure_deposit());
        P3M_CUDA(ctx, p3m::configure_fft());
        std::vector<float2> tw(p3m::kTwiddleLength);
        p3m::host_twiddles(tw.data());
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->twiddles, tw.data(), tw.size() * sizeof(float2),
                                      cudaMemcpyHostToDevice, ctx->stream));
        // clearMaterials (GravityPipeline.kt:1493-1503): unit mass, not solid.
        std::vector<float4> mats(cap, make_float4(1.0f, 0.0f, 0.0f, 0.0f));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->materials, mats.data(), cap * sizeof(float4),
                                      cudaMemcpyHostToDevice, ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->bodies, 0, cap * sizeof(float4), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->accel, 0, cap * sizeof(float2), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->destinations, 0, cap * sizeof(uint32_t), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, 4 * sizeof(unsigned), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_count, 0, P * sizeof(int), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_start, 0, (P + 1) * sizeof(int), ctx->stream));
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_mass, 0, P * sizeof(uint32_t), ctx->stream));
        int s = ensure_green(ctx);
        if (s != P3M_OK) return s;
        P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return P3M_OK;
    };
    st = init();
    if (st != P3M_OK) {
        g_create_error = ctx->last_error;
        free_all(ctx);
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return st;
    }
    normalize_to(ctx, 0);
    *out = ctx;
    return P3M_OK;
}

int p3m_destroy(p3m_ctx* ctx) {
    if (!ctx) return P3M_OK;
    cudaStreamSynchronize(ctx->stream);
    free_all(ctx);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return P3M_OK;
}

int p3m_upload_state(p3m_ctx* ctx, const float* bodies4, const float* materials4,
                     const float* acceleration2, int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (bodies4)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->bodies, bodies4, (size_t)n * 16, cudaMemcpyDefault, ctx->stream));
    if (materials4)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->materials, materials4, (size_t)n * 16, cudaMemcpyDefault, ctx->stream));
    if (acceleration2)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->accel, acceleration2, (size_t)n * 8, cudaMemcpyDefault, ctx->stream));
    // Host arrays belong to the caller: finish reading them before returning.
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

int p3m_upload_range(p3m_ctx* ctx, int32_t first, int32_t count, const float* bodies4,
                     const float* materials4, const float* acceleration2) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (first < 0 || count < 0) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "range must be non-negative");
    if ((long long)first + count > ctx->cfg.capacity)
        return fail(ctx, P3M_ERR_CAPACITY, "range exceeds capacity");
    if (bodies4)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->bodies + first, bodies4, (size_t)count * 16, cudaMemcpyDefault, ctx->stream));
    if (materials4)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->materials + first, materials4, (size_t)count * 16, cudaMemcpyDefault, ctx->stream));
    if (acceleration2)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->accel + first, acceleration2, (size_t)count * 8, cudaMemcpyDefault, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

int p3m_download_state(p3m_ctx* ctx, float* bodies4, float* materials4, float* acceleration2,
                       int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (bodies4)
        P3M_CUDA(ctx, cudaMemcpyAsync(bodies4, ctx->bodies, (size_t)n * 16, cudaMemcpyDefault, ctx->stream));
    if (materials4)
        P3M_CUDA(ctx, cudaMemcpyAsync(materials4, ctx->materials, (size_t)n * 16, cudaMemcpyDefault, ctx->stream));
    if (acceleration2)
        P3M_CUDA(ctx, cudaMemcpyAsync(acceleration2, ctx->accel, (size_t)n * 8, cudaMemcpyDefault, ctx->stream));
    P3M_CUDA(ctx, queue_status_read(ctx));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // The arrays are written; a sort whose wait gave up made them invalid.
    return device_failures(ctx, false);
}

int p3m_debug_get(p3m_ctx* ctx, int32_t which, void* host, size_t bytes) {
    if (!ctx || !host) return P3M_ERR_INVALID_ARGUMENT;
    void* d = nullptr;
    const size_t size = buffer_bytes(ctx, which, &d);
    if (!d) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "unknown buffer");
    if (bytes > size) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "more bytes requested than the buffer holds");
    P3M_CUDA(ctx, cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

int p3m_device_pointer(p3m_ctx* ctx, int32_t which, void** device, size_t* bytes) {
    if (!ctx || !device) return P3M_ERR_INVALID_ARGUMENT;
    void* d = nullptr;
    const size_t size = buffer_bytes(ctx, which, &d);
    if (!d) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "unknown buffer");
    *device = d;
    if (bytes) *bytes = size;
    return P3M_OK;
}

int p3m_set_bounded(p3m_ctx* ctx, int32_t bounded) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    const int b = bounded ? 1 : 0;
    if (b == ctx->bounded) return P3M_OK;
    if (b && !ctx->walls_supported)
        return fail(ctx, P3M_ERR_UNSUPPORTED, "walls need an FFT grid of at most 2048 cells per axis");
    ctx->bounded = b;
    ctx->grid = grid_for(ctx);
    return ensure_green(ctx);
}

int p3m_set_field_acceleration(p3m_ctx* ctx, float ax_px, float ay_px) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    ctx->field_x = ax_px / (float)ctx->cfg.viewport_width;
    ctx->field_y = ay_px / (float)ctx->cfg.viewport_height;
    return P3M_OK;
}

int p3m_set_mutual_gravity(p3m_ctx* ctx, int32_t enabled) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    ctx->mutual = enabled ? 1 : 0;
    return P3M_OK;
}

int p3m_set_mass_excess(p3m_ctx* ctx, float mass_excess) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(mass_excess)) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "mass excess must be finite");
    ctx->mass_excess = mass_excess;
    return P3M_OK;
}

int p3m_initialize_acceleration(p3m_ctx* ctx, int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    normalize_to(ctx, n);
    if (ctx->mutual) {
        st = build_force(ctx, n);
        if (st != P3M_OK) return st;
    }
    return apply_kick(ctx, n, 1);
}

int p3m_step(p3m_ctx* ctx, int32_t n, int32_t steps) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (steps < 0) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "steps must be >= 0");
    for (int i = 0; i < steps; ++i) {
        st = one_step(ctx, n);
        if (st != P3M_OK) return st;
    }
    return P3M_OK;
}

int p3m_set_launch_shape(p3m_ctx* ctx, int32_t fft_lines, int32_t short_range_threads) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (fft_lines < 0 || fft_lines > 16)
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "fft_lines must be in [0, 16]");
    if (short_range_threads != 64 && short_range_threads != 128 && short_range_threads != 256)
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "short_range_threads must be 64, 128 or 256");
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->tune_fft_lines = fft_lines;
    ctx->tune_sr_threads = short_range_threads;
    ctx->grid = grid_for(ctx);
    drop_graphs(ctx);
    return P3M_OK;
}

int p3m_autotune(p3m_ctx* ctx, int32_t n, int32_t trial_steps, int32_t* chosen2) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (trial_steps <= 0) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "trial_steps must be > 0");
    if (n == 0) return fail(ctx, P3M_ERR_STATE, "autotune needs active bodies");
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    normalize_to(ctx, n);
    st = ensure_green(ctx);
    if (st != P3M_OK) return st;
    int f = 0, t = 256;
    st = autotune_context(ctx, n, trial_steps, &f, &t);
    if (st != P3M_OK) return st;
    if (chosen2) {
        chosen2[0] = f;
        chosen2[1] = t;
    }
    return P3M_OK;
}

int p3m_sort_bodies(p3m_ctx* ctx, int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    return sort_bodies(ctx, n);
}

int p3m_drift(p3m_ctx* ctx, int32_t n, float kick_dt, float drift_dt) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    // collision_build.comp:43: nothing moves when both are zero.
    if (!(kick_dt != 0.0f || drift_dt != 0.0f)) return P3M_OK;
    P3M_CUDA(ctx, p3m::launch_drift(ctx->bodies, ctx->accel, n, 0.5f * kick_dt, drift_dt, 1,
                                    ctx->grid, nullptr, nullptr, ctx->status, ctx->stream));
    return P3M_OK;
}

int p3m_build_cell_lists(p3m_ctx* ctx, int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    P3M_CUDA(ctx, p3m::launch_cell_keys(ctx->bodies, n, ctx->grid, ctx->keys, ctx->vals, ctx->stream));
    return lists_from_keys(ctx, n);
}

int p3m_build_force(p3m_ctx* ctx, int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    normalize_to(ctx, n);
    return build_force(ctx, n);
}

int p3m_apply_kick(p3m_ctx* ctx, int32_t n, int32_t initial) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    normalize_to(ctx, n);
    return apply_kick(ctx, n, initial ? 1 : 0);
}

int p3m_synchronize(p3m_ctx* ctx) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, queue_status_read(ctx));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // p3m_step_io's copies (the last download follows the last step).
    if (ctx->up_stream) P3M_CUDA(ctx, cudaStreamSynchronize(ctx->up_stream));
    if (ctx->down_stream) P3M_CUDA(ctx, cudaStreamSynchronize(ctx->down_stream));
    return device_failures(ctx, true);
}

int p3m_step_io(p3m_ctx* ctx, int32_t n, const float* host_bodies_in4, float* host_bodies_out4) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (!ctx->up_stream) {  // first call: the copy streams, staging buffers and events
        const size_t cap = (size_t)ctx->cfg.capacity;
        P3M_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->up_stream, cudaStreamNonBlocking));
        P3M_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->down_stream, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&ctx->in_ready, &ctx->in_free, &ctx->out_ready, &ctx->out_free})
            P3M_CUDA(ctx, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        if (cudaMalloc((void**)&ctx->stage_in, cap * sizeof(float4)) != cudaSuccess ||
            cudaMalloc((void**)&ctx->stage_out, cap * sizeof(float4)) != cudaSuccess)
            return fail(ctx, P3M_ERR_OUT_OF_MEMORY, "staging buffers of p3m_step_io");
    }
    const size_t bytes = (size_t)n * sizeof(float4);
    if (host_bodies_in4 && n > 0) {
        // The upload waits only until the previous step has taken the last
        // upload out of the staging buffer, so it overlaps that step.
        P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->up_stream, ctx->in_free, 0));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->stage_in, host_bodies_in4, bytes, cudaMemcpyHostToDevice,
                                      ctx->up_stream));
        P3M_CUDA(ctx, cudaEventRecord(ctx->in_ready, ctx->up_stream));
        P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->in_ready, 0));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->bodies, ctx->stage_in, bytes, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        P3M_CUDA(ctx, cudaEventRecord(ctx->in_free, ctx->stream));
    }
    st = one_step(ctx, n);
    if (st != P3M_OK) return st;
    if (host_bodies_out4 && n > 0) {
        // The stepped bodies go to the staging buffer once the previous
        // download has left it; the download then overlaps the next step.
        P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->out_free, 0));
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->stage_out, ctx->bodies, bytes, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        P3M_CUDA(ctx, cudaEventRecord(ctx->out_ready, ctx->stream));
        P3M_CUDA(ctx, cudaStreamWaitEvent(ctx->down_stream, ctx->out_ready, 0));
        P3M_CUDA(ctx, cudaMemcpyAsync(host_bodies_out4, ctx->stage_out, bytes,
                                      cudaMemcpyDeviceToHost, ctx->down_stream));
        P3M_CUDA(ctx, cudaEventRecord(ctx->out_free, ctx->down_stream));
    }
    return P3M_OK;
}

int p3m_set_lookback_fault(p3m_ctx* ctx, int32_t poll_limit, int32_t withheld_tile) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (poll_limit < 1) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "poll_limit must be >= 1");
    if (withheld_tile < -1) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "withheld_tile must be >= -1");
    // Captured steps bake the sort's launch arguments in: capture anew.
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    drop_graphs(ctx);
    ctx->sort.poll_limit = poll_limit;
    ctx->sort.withhold_tile = withheld_tile;
    return P3M_OK;
}

int p3m_set_graphs(p3m_ctx* ctx, int32_t enabled) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    drop_graphs(ctx);
    ctx->use_graphs = enabled != 0;
    return P3M_OK;
}

int p3m_profile_enable(p3m_ctx* ctx, int32_t enabled) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    fold_stages(ctx);
    if (enabled) {
        for (int i = 0; i < P3M_STAGE_COUNT_; ++i) {
            ctx->stage_ms[i] = 0.0;
            ctx->stage_intervals[i] = 0;
        }
    }
    ctx->profiling = enabled != 0;
    return P3M_OK;
}

int p3m_profile_read(p3m_ctx* ctx, double* total_ms, int64_t* intervals) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    fold_stages(ctx);
    for (int i = 0; i < P3M_STAGE_COUNT_; ++i) {
        if (total_ms) total_ms[i] = ctx->stage_ms[i];
        if (intervals) intervals[i] = ctx->stage_intervals[i];
    }
    return P3M_OK;
}

int64_t p3m_kernel_launches(void) { return p3m::g_launches.load(); }

int p3m_get_stream(p3m_ctx* ctx, void** stream) {
    if (!ctx || !stream) return P3M_ERR_INVALID_ARGUMENT;
    *stream = (void*)ctx->stream;
    return P3M_OK;
}

int p3m_host_alloc(size_t bytes, void** host) {
    if (!host) return P3M_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaHostAlloc(host, std::max<size_t>(bytes, 1), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        *host = nullptr;
        return fail_cuda(nullptr, "cudaHostAlloc", e);
    }
    return P3M_OK;
}

int p3m_host_free(void* host) {
    if (!host) return P3M_OK;
    cudaError_t e = cudaFreeHost(host);
    return e == cudaSuccess ? P3M_OK : fail_cuda(nullptr, "cudaFreeHost", e);
}

int p3m_nonfinite_count(p3m_ctx* ctx, int64_t* count) {
    if (!ctx || !count) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, queue_status_read(ctx));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *count = (int64_t)ctx->status_host[0];
    return P3M_OK;
}

int p3m_wait_timeouts(p3m_ctx* ctx, int64_t* count) {
    if (!ctx || !count) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, queue_status_read(ctx));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *count = (int64_t)ctx->status_host[1];
    return P3M_OK;
}

// The FP32 half spectrum of the last force build, column-transformed into a
// work copy (the force path never stores it: its column pass multiplies by
// the Green's table and inverts in shared memory).
namespace {
int float_spectrum(p3m_ctx* ctx, std::vector<float2>* out) {
    if (ctx->built_n < 0) return fail(ctx, P3M_ERR_STATE, "no force build yet");
    const size_t cells = half_cells(ctx);
    float2* work = nullptr;
    P3M_CUDA(ctx, cudaMallocAsync((void**)&work, cells * sizeof(float2), ctx->stream));
    cudaError_t e = cudaMemcpyAsync(work, ctx->half, cells * sizeof(float2),
                                    cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess) e = p3m::launch_fft_forward_columns(work, ctx->grid, ctx->twiddles, ctx->stream);
    out->resize(cells);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out->data(), work, cells * sizeof(float2), cudaMemcpyDeviceToHost,
                            ctx->stream);
    cudaFreeAsync(work, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail_cuda(ctx, "density spectrum", e);
    return P3M_OK;
}
}  // namespace

int p3m_density_spectrum(p3m_ctx* ctx, float* spectrum2, size_t bytes) {
    if (!ctx || !spectrum2) return P3M_ERR_INVALID_ARGUMENT;
    if (bytes < half_cells(ctx) * sizeof(float2))
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "spectrum needs (MW/2+1)*MH float2 values");
    std::vector<float2> spec;
    const int st = float_spectrum(ctx, &spec);
    if (st != P3M_OK) return st;
    std::memcpy(spectrum2, spec.data(), spec.size() * sizeof(float2));
    return P3M_OK;
}

int p3m_validate_fft(p3m_ctx* ctx, double* out3) {
    if (!ctx || !out3) return P3M_ERR_INVALID_ARGUMENT;
    // GravityPipeline.kt:379: check(!bounded).
    if (ctx->bounded) return fail(ctx, P3M_ERR_STATE, "FFT validation covers the periodic mesh only");
    std::vector<float2> spec;
    int st = float_spectrum(ctx, &spec);
    if (st != P3M_OK) return st;
    const int MW = ctx->grid.MW, MH = ctx->grid.MH, SW = MW / 2 + 1;
    // GravityPipeline.kt:1546-1547 / :390: the density over massScale (the
    // int64 form: over 2^32), in FP64.
    const double inv_scale = ctx->cfg.deposit_mode == P3M_DEPOSIT_I64
                                 ? 1.0 / 4294967296.0
                                 : 1.0 / (double)ctx->mass_scale;
    double2* z = nullptr;
    P3M_CUDA(ctx, cudaMallocAsync((void**)&z, mesh_cells(ctx) * sizeof(double2), ctx->stream));
    std::vector<double2> ref(mesh_cells(ctx));
    cudaError_t e = p3m::launch_density_spectrum_f64(ctx->density, ctx->cfg.deposit_mode,
                                                     inv_scale, ctx->grid, z, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ref.data(), z, ref.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                            ctx->stream);
    cudaFreeAsync(z, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail_cuda(ctx, "p3m_validate_fft", e);
    // GravityPipeline.kt:404-418 over all 2*MW*MH components; columns
    // 1..MW/2-1 of the half spectrum stand for themselves and their mirror.
    double max_abs = 0.0, max_ref = 0.0, sq = 0.0;
    for (int ky = 0; ky < MH; ++ky) {
        for (int kx = 0; kx < SW; ++kx) {
            const double2 r = ref[(size_t)ky * MW + kx];
            const float2 v = spec[(size_t)ky * SW + kx];
            const double ex = std::fabs(r.x - (double)v.x), ey = std::fabs(r.y - (double)v.y);
            const double w = (kx == 0 || 2 * kx == MW) ? 1.0 : 2.0;
            max_abs = std::max(max_abs, std::max(ex, ey));
            max_ref = std::max(max_ref, std::max(std::fabs(r.x), std::fabs(r.y)));
            sq += w * (ex * ex + ey * ey);
        }
    }
    out3[0] = max_abs;
    out3[1] = max_abs / std::max(max_ref, 1e-30);
    out3[2] = std::sqrt(sq / (2.0 * (double)MW * (double)MH));
    return P3M_OK;
}

int p3m_direct_accel_f64(p3m_ctx* ctx, int32_t n, const int32_t* targets, int32_t n_targets,
                         double* out) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (n_targets < 0 || (n_targets > 0 && (!targets || !out)))
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "targets/out missing");
    for (int i = 0; i < n_targets; ++i)
        if (targets[i] < 0 || targets[i] >= n) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "target ID out of range");
    if (n_targets == 0) return P3M_OK;
    normalize_to(ctx, n);
    int* dt = nullptr;
    double2* dout = nullptr;
    P3M_CUDA(ctx, cudaMallocAsync((void**)&dt, (size_t)n_targets * sizeof(int), ctx->stream));
    P3M_CUDA(ctx, cudaMallocAsync((void**)&dout, (size_t)n_targets * sizeof(double2), ctx->stream));
    cudaError_t e = cudaMemcpyAsync(dt, targets, (size_t)n_targets * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    const double aspect = (double)ctx->cfg.viewport_width / (double)ctx->cfg.viewport_height;
    const double cw = aspect / ctx->cfg.grid_width, ch = 1.0 / ctx->cfg.grid_height;
    const double md = (double)ctx->cfg.minimum_distance_cell_fraction * std::min(cw, ch);
    if (e == cudaSuccess)
        e = p3m::launch_direct_accel(ctx->bodies, ctx->materials, n, dt, n_targets, aspect,
                                     (double)ctx->cfg.gravitational_constant,
                                     (double)ctx->normalization_mass, md * md, ctx->bounded, dout,
                                     ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout, (size_t)n_targets * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(dt, ctx->stream);
    cudaFreeAsync(dout, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail_cuda(ctx, "p3m_direct_accel_f64", e);
    return P3M_OK;
}

int p3m_diagnostics_f64(p3m_ctx* ctx, int32_t n, double* out6) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (!out6) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "out is NULL");
    double* partial = ctx->diag;
    double* result = ctx->diag + (size_t)p3m::conservation_blocks() * 6;
    P3M_CUDA(ctx, p3m::launch_conservation(ctx->bodies, ctx->materials, n,
                                           (double)ctx->cfg.viewport_width,
                                           (double)ctx->cfg.viewport_height, partial, result,
                                           ctx->stream));
    P3M_CUDA(ctx, cudaMemcpyAsync(out6, result, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched form: many independent simulations of uneven sizes (the
// application's trajectory previews and ensembles), stepped together.
//
// Every simulation keeps its own context, buffers and stream. A batch step is
// captured once as one CUDA graph: an event on the batch stream forks to every
// simulation's stream, each enqueues its whole step (reorder, drift, lists,
// deposit, FFT, short range, kick), and the batch stream joins them all. The
// graph is replayed with one cudaGraphLaunch per step for the whole batch,
// and the GPU runs the simulations' chains side by side. A replay bakes in
// every simulation's body count, reorder phase, current ping-pong buffer and
// uniforms; the cache keys on all of them and captures a new graph when any
// changes (with the default reorder interval of 2 a steady batch cycles
// through four graphs).

struct p3m_batch {
    std::vector<p3m_ctx*> sims;
    std::vector<int> n;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // fused form: the short range beside the mesh force
    cudaEvent_t side_fork = nullptr, side_join = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    struct Graph {
        std::vector<uint64_t> key;
        cudaGraphExec_t exec;
        long long kernels;
        std::vector<std::pair<uint32_t*, uint32_t*>> sorted;
    };
    std::vector<Graph> graphs;
    // Fused form: the stages of a step over all simulations at once, either
    // as one launch per stage (the default) or as one persistent launch.
    bool fused = true;
    bool persistent = false;
    int persistent_ctas_per_sm = 0;  // 0: as many as stay resident
    // The persistent launch's grid barrier: polls before a wait gives up, and
    // the test hook (a CTA that never arrives at one phase's barrier).
    int barrier_polls = 1 << 20;
    int withhold_cta = -1, withhold_phase = -1;
    unsigned int* sync = nullptr;  // device: arrivals, waits given up
    unsigned int reported_timeouts = 0;
    unsigned long long* phase_ns = nullptr;  // device: the last launch's phase stamps
    int32_t last_info[4] = {0, 0, 0, 0};     // of the last step's plan: see p3m_batch_plan_info
    // p3m_batch_step_io: one copy stream per direction, device staging of all
    // simulations' bodies back to back, the events that order the staging
    // buffers' reuse, and the row-copy arguments between the staging and
    // each simulation's current body buffer (keyed by counts and buffers).
    cudaStream_t up_stream = nullptr, down_stream = nullptr;
    float4* stage_in = nullptr;
    float4* stage_out = nullptr;
    cudaEvent_t in_ready = nullptr, in_free = nullptr, out_ready = nullptr, out_free = nullptr;
    struct IoArgs {
        std::vector<uint64_t> key;
        void* dev = nullptr;  // RowCopy[sims], then the block prefix (sims + 1 ints)
        int blocks = 0;
    };
    std::vector<IoArgs> io_args;
    struct Plan {
        std::vector<uint64_t> key;
        void* blob = nullptr;  // per-simulation arguments and block prefixes
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        bool persistent = false;
        int phases = 0, ctas = 0;
        std::vector<char> swap;  // simulations whose buffers the reorder swapped
        std::vector<std::pair<uint32_t*, uint32_t*>> sorted;
    };
    std::vector<Plan> plans;
    std::string last_error;
};

namespace {

int batch_fail(p3m_batch* b, int status, const std::string& what) {
    if (b) b->last_error = what;
    else g_create_error = what;
    return status;
}

int batch_fail_ctx(p3m_batch* b, size_t sim, int status) {
    return batch_fail(b, status, "simulation " + std::to_string(sim) + ": " + b->sims[sim]->last_error);
}

void batch_drop_graphs(p3m_batch* b) {
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
    for (auto& p : b->plans) {
        if (p.exec) cudaGraphExecDestroy(p.exec);
        if (p.blob) cudaFree(p.blob);
    }
    b->plans.clear();
}

uint64_t bits_of(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Everything one captured batch step bakes in.
std::vector<uint64_t> batch_key(const p3m_batch* b, const std::vector<char>& sort) {
    std::vector<uint64_t> key;
    key.reserve(b->sims.size() * 6);
    for (size_t i = 0; i < b->sims.size(); ++i) {
        const p3m_ctx* c = b->sims[i];
        key.push_back((uint64_t)b->n[i] | ((uint64_t)sort[i] << 32) | ((uint64_t)c->mutual << 33) |
                      ((uint64_t)c->bounded << 34));
        key.push_back((uint64_t)(uintptr_t)c->bodies);
        key.push_back((uint64_t)c->mass_scale | (bits_of(c->normalization_mass) << 32));
        key.push_back(bits_of(c->field_x) | (bits_of(c->field_y) << 32));
        key.push_back((uint64_t)c->tune_fft_lines | ((uint64_t)c->tune_sr_threads << 32));
    }
    return key;
}

int batch_enqueue(p3m_batch* b, const std::vector<char>& sort) {
    cudaError_t e = cudaEventRecord(b->fork, b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    for (size_t i = 0; i < b->sims.size(); ++i) {
        p3m_ctx* c = b->sims[i];
        e = cudaStreamWaitEvent(c->stream, b->fork, 0);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
        int st = enqueue_step(c, b->n[i], sort[i] != 0);
        if (st != P3M_OK) return batch_fail_ctx(b, i, st);
        e = cudaEventRecord(b->join[i], c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[i], 0);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    }
    return P3M_OK;
}

bool fused_supported(const p3m_batch* b);
int batch_fused_step(p3m_batch* b, const std::vector<char>& sort, const std::vector<uint64_t>& key);

// Rows of float4 between the I/O staging buffers and the simulations' body
// buffers, every simulation in one launch (block b: local block b - first[s]
// of simulation s).
struct RowCopy {
    const float4* src;
    float4* dst;
    int n;
};

__global__ void __launch_bounds__(256) batch_rows_copy_kernel(const RowCopy* __restrict__ copies,
                                                              const int* __restrict__ first,
                                                              int sims) {
    const int2 sb = p3m::batch_block(first, sims);
    const RowCopy c = copies[sb.x];
    const int k = sb.y * 256 + (int)threadIdx.x;
    if (k < c.n) c.dst[k] = c.src[k];
}

// The row copies of the batch's current bodies from (in) or to (out) the
// staging buffer, simulation i at row sum(n[j], j < i); built once per set
// of counts and body buffers and kept (the reorder cycles through a few).
const p3m_batch::IoArgs* batch_io_args(p3m_batch* b, bool in) {
    const size_t S = b->sims.size();
    std::vector<uint64_t> key;
    key.reserve(2 * S + 1);
    key.push_back(in ? 1u : 0u);
    for (size_t i = 0; i < S; ++i) {
        key.push_back((uint64_t)(uintptr_t)b->sims[i]->bodies);
        key.push_back((uint64_t)b->n[i]);
    }
    for (const auto& a : b->io_args)
        if (a.key == key) return &a;
    std::vector<RowCopy> copies(S);
    std::vector<int> first(S + 1, 0);
    long long row = 0;
    for (size_t i = 0; i < S; ++i) {
        float4* cur = b->sims[i]->bodies;
        copies[i] = in ? RowCopy{b->stage_in + row, cur, b->n[i]}
                       : RowCopy{cur, b->stage_out + row, b->n[i]};
        first[i + 1] = first[i] + (b->n[i] + 255) / 256;
        row += b->n[i];
    }
    const size_t cbytes = S * sizeof(RowCopy);
    const size_t fbytes = (S + 1) * sizeof(int);
    p3m_batch::IoArgs a;
    a.key = key;
    a.blocks = first[S];
    if (cudaMalloc(&a.dev, cbytes + fbytes) != cudaSuccess) return nullptr;
    // A new buffer: a blocking copy (the default stream does not wait for
    // the batch's non-blocking streams).
    if (cudaMemcpy(a.dev, copies.data(), cbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(static_cast<char*>(a.dev) + cbytes, first.data(), fbytes,
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(a.dev);
        return nullptr;
    }
    if (b->io_args.size() >= 16) {  // dropped only after its last use has run
        cudaStreamSynchronize(b->stream);
        cudaFree(b->io_args.front().dev);
        b->io_args.erase(b->io_args.begin());
    }
    b->io_args.push_back(std::move(a));
    return &b->io_args.back();
}

cudaError_t launch_io_copy(p3m_batch* b, const p3m_batch::IoArgs* a) {
    if (a->blocks <= 0) return cudaSuccess;
    const size_t cbytes = b->sims.size() * sizeof(RowCopy);
    batch_rows_copy_kernel<<<a->blocks, 256, 0, b->stream>>>(
        static_cast<const RowCopy*>(a->dev),
        reinterpret_cast<const int*>(static_cast<const char*>(a->dev) + cbytes),
        (int)b->sims.size());
    p3m::count_launches(1);
    return cudaGetLastError();
}

int batch_one_step(p3m_batch* b) {
    std::vector<char> sort(b->sims.size(), 0);
    for (size_t i = 0; i < b->sims.size(); ++i) {
        p3m_ctx* c = b->sims[i];
        normalize_to(c, b->n[i]);
        int st = ensure_green(c);
        if (st != P3M_OK) return batch_fail_ctx(b, i, st);
        const int interval = c->cfg.spatial_sort_interval;
        sort[i] = (interval > 0 && (c->physics_steps % interval) == 0) ? 1 : 0;
        if (interval > 0) c->physics_steps++;
    }
    const std::vector<uint64_t> key = batch_key(b, sort);
    if (b->fused && fused_supported(b)) return batch_fused_step(b, sort, key);
    for (const auto& g : b->graphs) {
        if (g.key != key) continue;
        cudaError_t e = cudaGraphLaunch(g.exec, b->stream);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
        p3m::count_launches((int)g.kernels);
        for (size_t i = 0; i < b->sims.size(); ++i) {
            if (b->sims[i]->mutual) b->sims[i]->built_n = b->n[i];
            if (sort[i]) swap_body_buffers(b->sims[i]);
            b->sims[i]->sorted_keys = g.sorted[i].first;
            b->sims[i]->sorted_ids = g.sorted[i].second;
        }
        return P3M_OK;
    }
    struct Saved { float4 *b, *ba, *m, *ma; float2 *a, *aa; };
    std::vector<Saved> saved;
    for (p3m_ctx* c : b->sims)
        saved.push_back({c->bodies, c->bodies_alt, c->materials, c->materials_alt, c->accel, c->accel_alt});
    const long long k0 = p3m_kernel_launches();
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    int st = batch_enqueue(b, sort);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(b->stream, &graph);
    if (st != P3M_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        for (size_t i = 0; i < b->sims.size(); ++i) {  // nothing ran: restore buffer roles
            p3m_ctx* c = b->sims[i];
            c->bodies = saved[i].b; c->bodies_alt = saved[i].ba;
            c->materials = saved[i].m; c->materials_alt = saved[i].ma;
            c->accel = saved[i].a; c->accel_alt = saved[i].aa;
        }
        if (st != P3M_OK) return st;
        return batch_fail(b, P3M_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    }
    p3m_batch::Graph entry;
    entry.key = key;
    entry.kernels = p3m_kernel_launches() - k0;
    e = cudaGraphInstantiate(&entry.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    for (p3m_ctx* c : b->sims) entry.sorted.push_back({c->sorted_keys, c->sorted_ids});
    if (b->graphs.size() >= 8) {
        cudaGraphExecDestroy(b->graphs.front().exec);
        b->graphs.erase(b->graphs.begin());
    }
    b->graphs.push_back(std::move(entry));
    e = cudaGraphLaunch(b->graphs.back().exec, b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    return P3M_OK;
}

// ---- fused batch step ------------------------------------------------------
// Every stage of the step runs as one launch over all simulations (CTA b
// takes local block b - first[s] of simulation s; see p3m_internal.cuh), so a
// batch step costs ~25 launches whatever the number of simulations. The
// per-simulation arguments of every launch and the block prefixes live in one
// device blob, written once per plan; the launches are captured in a graph.
// A plan holds for one set of body counts, reorder flags, buffer roles and
// uniforms, like the graphs of the other form.

struct BlobBuilder {
    std::vector<unsigned char> host;
    size_t add(const void* data, size_t bytes) {
        const size_t off = (host.size() + 15) & ~(size_t)15;
        host.resize(off + bytes);
        if (bytes) std::memcpy(host.data() + off, data, bytes);
        return off;
    }
};

// Each stage is recorded twice: as a launch of its batched kernel (the
// per-stage form) and as an entry of the persistent kernel's stage table
// with its phase (stages of one phase are independent of one another). Raw
// launches (copies, stream forks) belong to the per-stage form only; the
// persistent form has its own entries for them.
struct FusedBuilder {
    BlobBuilder blob;
    std::vector<std::function<cudaError_t(unsigned char*, cudaStream_t)>> launches;
    struct PEntry { p3m::PStage st; int phase; };
    std::vector<PEntry> pstages;
    bool persistent_ok = true;  // every stage has a persistent form
    size_t pool = 0;            // the largest dynamic shared memory of a stage

    template <typename Args>
    bool offsets(const std::vector<Args>& args, const std::vector<int>& blocks, size_t* a_off,
                 size_t* f_off, int* total) {
        if (args.empty()) return false;
        std::vector<int> first(args.size() + 1, 0);
        for (size_t i = 0; i < args.size(); ++i) first[i + 1] = first[i] + blocks[i];
        if (first.back() == 0) return false;
        *a_off = blob.add(args.data(), args.size() * sizeof(Args));
        *f_off = blob.add(first.data(), first.size() * sizeof(int));
        *total = first.back();
        return true;
    }
    template <typename Args, typename Fn>
    void stage(const std::vector<Args>& args, const std::vector<int>& blocks, Fn fn, int kind,
               int phase, size_t smem) {
        size_t a_off, f_off;
        int total;
        if (!offsets(args, blocks, &a_off, &f_off, &total)) return;
        const int sims = (int)args.size();
        launches.push_back([=](unsigned char* dev, cudaStream_t st) {
            p3m::BatchGrid g{reinterpret_cast<const int*>(dev + f_off), sims, total};
            return fn(reinterpret_cast<const Args*>(dev + a_off), g, st);
        });
        if (kind < 0) persistent_ok = false;
        pstages.push_back({{kind, sims, total, (int)a_off, (int)f_off}, phase});
        pool = std::max(pool, smem);
    }
    template <typename Args>
    void persistent_stage(const std::vector<Args>& args, const std::vector<int>& blocks, int kind,
                          int phase) {
        size_t a_off, f_off;
        int total;
        if (!offsets(args, blocks, &a_off, &f_off, &total)) return;
        pstages.push_back({{kind, (int)args.size(), total, (int)a_off, (int)f_off}, phase});
    }
    void raw(std::function<cudaError_t(unsigned char*, cudaStream_t)> fn) { launches.push_back(fn); }
};

// Whether the fused form covers this batch: every histogram of a radix pass
// fits one scan CTA.
bool fused_supported(const p3m_batch* b) {
    for (size_t i = 0; i < b->sims.size(); ++i)
        if ((long long)p3m::radix_tiles(b->n[i]) * 256 > p3m::radix_scan_limit()) return false;
    return true;
}

struct SimRoles {
    float4 *bodies, *materials;
    float2* accel;
    uint32_t *sk, *sv;  // the cell sort's result
};

// Radix passes over the simulations listed in `who` (key bits each), with
// keys/vals ping-ponging between (keys, vals) and the sort scratch.
void fused_radix(FusedBuilder& fb, const p3m_batch* b, const std::vector<int>& who,
                 const std::vector<int>& key_bits, std::vector<uint32_t*>& kin,
                 std::vector<uint32_t*>& vin, int& phase) {
    int max_passes = 0;
    std::vector<int> passes(who.size()), bits(who.size());
    for (size_t j = 0; j < who.size(); ++j) {
        passes[j] = (key_bits[j] + 7) / 8;
        bits[j] = (key_bits[j] + passes[j] - 1) / passes[j];
        if (b->n[who[j]] <= 1) passes[j] = 0;
        max_passes = std::max(max_passes, passes[j]);
    }
    std::vector<uint32_t*> kout(who.size()), vout(who.size());
    for (size_t j = 0; j < who.size(); ++j) {
        const p3m_ctx* c = b->sims[who[j]];
        kout[j] = c->sort.keys_alt;
        vout[j] = c->sort.vals_alt;
    }
    for (int pass = 0; pass < max_passes; ++pass) {
        std::vector<p3m::RadixArgs> ra;
        std::vector<p3m::ScanArgs> sa;
        std::vector<int> tiles, ones;
        for (size_t j = 0; j < who.size(); ++j) {
            if (pass >= passes[j]) continue;
            const p3m_ctx* c = b->sims[who[j]];
            const int n = b->n[who[j]];
            const int shift = pass * bits[j];
            const int pbits = std::min(bits[j], key_bits[j] - shift);
            const int t = p3m::radix_tiles(n);
            ra.push_back({kin[j], vin[j], kout[j], vout[j], c->sort.hist, n, shift, pbits, t});
            sa.push_back({c->sort.hist, (1 << pbits) * t});
            tiles.push_back(t);
            ones.push_back(1);
            std::swap(kin[j], kout[j]);
            std::swap(vin[j], vout[j]);
        }
        fb.stage(ra, tiles, p3m::batched_radix_hist, p3m::kPStageRadixHist, ++phase, 0);
        fb.stage(sa, ones, p3m::batched_scan, p3m::kPStageScan, ++phase, 0);
        fb.stage(ra, tiles, p3m::batched_radix_scatter, p3m::kPStageRadixScatter, ++phase,
                 p3m::persistent_base_smem());
    }
}

int build_fused(p3m_batch* b, const std::vector<char>& sort, p3m_batch::Plan& plan) {
    const size_t S = b->sims.size();
    FusedBuilder fb;
    int phase = 0;  // the persistent form's phase of the stages being added
    std::vector<SimRoles> role(S);
    plan.swap.assign(S, 0);
    for (size_t i = 0; i < S; ++i) {
        p3m_ctx* c = b->sims[i];
        role[i] = {c->bodies, c->materials, c->accel, c->keys, c->vals};
    }
    // 1. Morton reorder (simulations whose reorder step this is).
    {
        std::vector<int> who, bits;
        std::vector<p3m::MortonArgs> ma;
        std::vector<int> blocks;
        for (size_t i = 0; i < S; ++i) {
            if (!sort[i] || b->n[i] <= 0) continue;
            p3m_ctx* c = b->sims[i];
            who.push_back((int)i);
            bits.push_back(c->sort_wbits + c->sort_hbits);
            ma.push_back({c->bodies, c->keys, c->vals, b->n[i], c->sort_wbits, c->sort_hbits});
            blocks.push_back((b->n[i] + 255) / 256);
        }
        fb.stage(ma, blocks, p3m::batched_morton_keys, p3m::kPStageMorton, phase, 0);
        std::vector<uint32_t*> kin(who.size()), vin(who.size());
        for (size_t j = 0; j < who.size(); ++j) {
            kin[j] = b->sims[who[j]]->keys;
            vin[j] = b->sims[who[j]]->vals;
        }
        fused_radix(fb, b, who, bits, kin, vin, phase);
        ++phase;
        std::vector<p3m::PermuteArgs> pa;
        std::vector<p3m::CopyArgs> copies;  // the persistent form's tail copies
        std::vector<int> copy_blocks;
        for (size_t j = 0; j < who.size(); ++j) {
            p3m_ctx* c = b->sims[who[j]];
            const int n = b->n[who[j]];
            pa.push_back({vin[j], c->bodies, c->accel, c->materials, c->bodies_alt, c->accel_alt,
                          c->materials_alt, c->destinations, n});
            const size_t tail = (size_t)c->cfg.capacity - (size_t)n;
            if (tail > 0) {
                float4* bs = c->bodies + n; float4* bd = c->bodies_alt + n;
                float2* as = c->accel + n; float2* ad = c->accel_alt + n;
                float4* ms = c->materials + n; float4* md = c->materials_alt + n;
                fb.raw([=](unsigned char*, cudaStream_t st) {
                    cudaError_t e = cudaMemcpyAsync(bd, bs, tail * sizeof(float4), cudaMemcpyDeviceToDevice, st);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(ad, as, tail * sizeof(float2), cudaMemcpyDeviceToDevice, st);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(md, ms, tail * sizeof(float4), cudaMemcpyDeviceToDevice, st);
                    return e;
                });
                auto add_copy = [&](const void* src, void* dst, size_t bytes) {
                    const long long words = (long long)(bytes / 4);
                    copies.push_back({static_cast<const uint32_t*>(src), static_cast<uint32_t*>(dst), words});
                    copy_blocks.push_back((int)((words + p3m::kBatchThreads - 1) / p3m::kBatchThreads));
                };
                add_copy(bs, bd, tail * sizeof(float4));
                add_copy(as, ad, tail * sizeof(float2));
                add_copy(ms, md, tail * sizeof(float4));
            }
            role[who[j]].bodies = c->bodies_alt;
            role[who[j]].accel = c->accel_alt;
            role[who[j]].materials = c->materials_alt;
            plan.swap[who[j]] = 1;
        }
        fb.stage(pa, blocks, p3m::batched_permute, p3m::kPStagePermute, phase, 0);
        fb.persistent_stage(copies, copy_blocks, p3m::kPStageCopy, phase);
        if (!who.empty()) ++phase;
    }
    // 2. Drift, with the home-cell keys.
    {
        std::vector<p3m::DriftArgs> da;
        std::vector<int> blocks;
        for (size_t i = 0; i < S; ++i) {
            if (b->n[i] <= 0) continue;
            p3m_ctx* c = b->sims[i];
            const float dt = c->cfg.time_step;
            da.push_back({role[i].bodies, role[i].accel, c->keys, c->vals, c->status, b->n[i],
                          0.5f * dt, dt / (float)c->cfg.drift_substeps, c->cfg.drift_substeps,
                          c->grid.bounded, c->grid.W, c->grid.H});
            blocks.push_back((b->n[i] + 255) / 256);
        }
        fb.stage(da, blocks, p3m::batched_drift, p3m::kPStageDrift, phase, 0);
    }
    // 3. Cell lists (simulations with mutual gravity). The cell counts and
    // masses and the density mesh are cleared beside the drift: nothing in
    // the step reads them before the cell build and the deposit.
    std::vector<int> mut;
    for (size_t i = 0; i < S; ++i)
        if (b->sims[i]->mutual && b->n[i] > 0) mut.push_back((int)i);
    {
        std::vector<p3m::ZeroArgs> za;
        std::vector<int> zb;
        for (int i : mut) {
            p3m_ctx* c = b->sims[i];
            const long long P = (long long)phys_cells(c);
            const int zblocks = (int)((P + p3m::kBatchThreads * 16 - 1) / (p3m::kBatchThreads * 16));
            za.push_back({reinterpret_cast<uint32_t*>(c->cell_count), P});
            za.push_back({c->cell_mass, P});
            zb.push_back(zblocks);
            zb.push_back(zblocks);
            const bool i64 = c->cfg.deposit_mode == P3M_DEPOSIT_I64;
            const long long words = (long long)mesh_cells(c) * (i64 ? 2 : 1);
            za.push_back({static_cast<uint32_t*>(c->density), words});
            zb.push_back((int)((words + p3m::kBatchThreads * 16 - 1) / (p3m::kBatchThreads * 16)));
        }
        fb.stage(za, zb, p3m::batched_zero, p3m::kPStageZero, phase, 0);
    }
    {
        std::vector<int> bits;
        std::vector<uint32_t*> kin, vin;
        for (int i : mut) {
            bits.push_back(bits_for(phys_cells(b->sims[i])));
            kin.push_back(b->sims[i]->keys);
            vin.push_back(b->sims[i]->vals);
        }
        fused_radix(fb, b, mut, bits, kin, vin, phase);
        std::vector<p3m::CellBuildArgs> ca;
        std::vector<int> cb;
        for (size_t j = 0; j < mut.size(); ++j) {
            p3m_ctx* c = b->sims[mut[j]];
            role[mut[j]].sk = kin[j];
            role[mut[j]].sv = vin[j];
            ca.push_back({kin[j], vin[j], role[mut[j]].bodies, role[mut[j]].materials,
                          c->cell_start, c->cell_count, c->cell_mass, c->entries, b->n[mut[j]]});
            cb.push_back((b->n[mut[j]] + p3m::kCellBuildBlockEntries - 1) / p3m::kCellBuildBlockEntries);
        }
        fb.stage(ca, cb, p3m::batched_cell_build, p3m::kPStageCellBuild, ++phase, 0);
    }
    const int phase_lists = phase;  // the phase of the cell build
    // 4. Short range (by stencil shape) on the side stream: it reads only the
    // cell lists, so it runs beside the deposit and FFT.
    {
        cudaStream_t side = b->side;
        cudaEvent_t fork_ev = b->side_fork;
        fb.raw([=](unsigned char*, cudaStream_t st) {
            cudaError_t e = cudaEventRecord(fork_ev, st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork_ev, 0);
            return e;
        });
        // The two-slot form first builds each cell's slots (kick_params says
        // which simulations take it).
        auto slot_form = [&](int i) { return kick_params(b->sims[i], b->n[i], 0).slot_form != 0; };
        {
            std::vector<p3m::SlotsArgs> sl;
            std::vector<int> slb;
            for (int i : mut) {
                p3m_ctx* c = b->sims[i];
                if (!slot_form(i)) continue;
                const p3m::KickParams kp = kick_params(c, b->n[i], 0);
                sl.push_back({c->cell_start, c->cell_count, c->cell_mass, c->entries,
                              c->cell_slots, c->grid.W, c->grid.H, kp.gravity, kp.total_mass});
                slb.push_back((int)((phys_cells(c) + p3m::kBatchThreads - 1) / p3m::kBatchThreads));
            }
            if (!sl.empty())
                fb.stage(sl, slb, [side](const p3m::SlotsArgs* a, p3m::BatchGrid g, cudaStream_t) {
                    return p3m::batched_cell_slots(a, g, side);
                }, p3m::kPStageSlots, phase_lists + 1, 0);
        }
        std::map<int, std::vector<int>> groups;  // rx * 64 + ry * 2 + two-slot form
        for (int i : mut) {
            const p3m_ctx* c = b->sims[i];
            groups[c->rx * 64 + c->ry * 2 + (slot_form(i) ? 1 : 0)].push_back(i);
        }
        for (const auto& kv : groups) {
            std::vector<p3m::ShortRangeArgs> sa;
            std::vector<int> sb;
            for (int i : kv.second) {
                p3m_ctx* c = b->sims[i];
                sa.push_back({role[i].bodies, c->entries, c->cell_start, c->cell_count, c->cell_mass,
                              c->cell_slots, c->a_short, kick_params(c, b->n[i], 0)});
                sb.push_back((b->n[i] + p3m::kBatchThreads - 1) / p3m::kBatchThreads);
            }
            const int rx = kv.first / 64, ry = (kv.first % 64) / 2, ex = kv.first % 2;
            // The persistent kernel carries the (3, 3) stencil only.
            const int kind = rx == p3m::kPersistentRx && ry == p3m::kPersistentRy
                                 ? (ex ? p3m::kPStageShortRangeSlots : p3m::kPStageShortRangeLists)
                                 : -1;
            fb.stage(sa, sb, [rx, ry, ex, side](const p3m::ShortRangeArgs* a, p3m::BatchGrid g, cudaStream_t) {
                return p3m::batched_short_range(a, g, rx, ry, ex, side);
            }, kind, phase_lists + 2, ex ? p3m::persistent_base_smem() : 0);
        }
        cudaEvent_t join_ev = b->side_join;
        fb.raw([=](unsigned char*, cudaStream_t) { return cudaEventRecord(join_ev, side); });
    }
    // 5. Mesh force (the mesh was cleared beside the drift): deposit, FFT with
    // the Green's multiply, inverse.
    {
        for (int mode : {P3M_DEPOSIT_U32, P3M_DEPOSIT_I64}) {
            std::vector<p3m::DepositArgs> dep;
            std::vector<int> db;
            std::vector<p3m::FftRowsArgs> fr;
            std::vector<int> fblocks;
            size_t smem = 0;
            for (int i : mut) {
                p3m_ctx* c = b->sims[i];
                if (c->cfg.deposit_mode != mode) continue;
                const p3m::GridShape& g = c->grid;
                const bool i64 = mode == P3M_DEPOSIT_I64;
                dep.push_back({c->entries, role[i].sk, c->density, b->n[i], g.W, g.H, g.MW, g.MH,
                               i64 ? 4294967296.0f : (float)c->mass_scale});
                db.push_back(p3m::chunk_deposit_blocks(b->n[i]));
                int rp, cp, ip;
                size_t rs, cs, is;
                p3m::fft_batch_shape(g, &rp, &cp, &ip, &rs, &cs, &is);
                fr.push_back({c->density, c->half, i64 ? 1.0f / 4294967296.0f : 1.0f / (float)c->mass_scale,
                              g.MW, g.MH, rp});
                fblocks.push_back((g.MH / 2 + rp - 1) / rp);
                smem = std::max(smem, rs);
            }
            const bool i64 = mode == P3M_DEPOSIT_I64;
            fb.stage(dep, db, [mode](const p3m::DepositArgs* a, p3m::BatchGrid g, cudaStream_t st) {
                return p3m::batched_deposit(a, g, mode, st);
            }, i64 ? p3m::kPStageDepositI64 : p3m::kPStageDepositU32, phase_lists + 1,
                     p3m::persistent_base_smem());
            const float2* tw0 = mut.empty() ? nullptr : b->sims[mut[0]]->twiddles;
            fb.stage(fr, fblocks, [mode, smem, tw0](const p3m::FftRowsArgs* a, p3m::BatchGrid g, cudaStream_t st) {
                return p3m::batched_fft_rows(a, g, mode, smem, tw0, st);
            }, i64 ? p3m::kPStageFftRowsI64 : p3m::kPStageFftRowsU32, phase_lists + 2, smem);
        }
        std::vector<p3m::FftColumnsArgs> fc;
        std::vector<p3m::FftInverseArgs> fi;
        std::vector<int> cbk, ibk;
        size_t csm = 0, ism = 0;
        for (int i : mut) {
            p3m_ctx* c = b->sims[i];
            const p3m::GridShape& g = c->grid;
            int rp, cp, ip;
            size_t rs, cs, is;
            p3m::fft_batch_shape(g, &rp, &cp, &ip, &rs, &cs, &is);
            fc.push_back({c->half, c->green, c->cols, 1.0f / c->normalization_mass, g.MW, g.MH, cp});
            cbk.push_back((g.MW / 2 + 1 + cp - 1) / cp);
            fi.push_back({c->cols, c->force, g.MW, g.MH, ip});
            ibk.push_back((g.MH + ip - 1) / ip);
            csm = std::max(csm, cs);
            ism = std::max(ism, is);
        }
        const float2* tw0 = mut.empty() ? nullptr : b->sims[mut[0]]->twiddles;
        fb.stage(fc, cbk, [csm, tw0](const p3m::FftColumnsArgs* a, p3m::BatchGrid g, cudaStream_t st) {
            return p3m::batched_fft_columns(a, g, csm, tw0, st);
        }, p3m::kPStageFftColumns, phase_lists + 3, csm);
        fb.stage(fi, ibk, [ism, tw0](const p3m::FftInverseArgs* a, p3m::BatchGrid g, cudaStream_t st) {
            return p3m::batched_fft_inverse(a, g, ism, tw0, st);
        }, p3m::kPStageFftInverse, phase_lists + 4, ism);
    }
    // 6. Interpolation + kick, after the short range has joined.
    {
        cudaEvent_t join_ev = b->side_join;
        fb.raw([=](unsigned char*, cudaStream_t st) { return cudaStreamWaitEvent(st, join_ev, 0); });
        std::vector<p3m::KickArgs> ka;
        std::vector<int> kb;
        for (size_t i = 0; i < S; ++i) {
            if (b->n[i] <= 0) continue;
            p3m_ctx* c = b->sims[i];
            ka.push_back({role[i].bodies, role[i].accel, c->force, c->a_short, kick_params(c, b->n[i], 0)});
            kb.push_back((b->n[i] + p3m::kBatchThreads - 1) / p3m::kBatchThreads);
        }
        fb.stage(ka, kb, p3m::batched_interp_kick, p3m::kPStageKick, phase_lists + 5, 0);
    }
    plan.sorted.resize(S);
    for (size_t i = 0; i < S; ++i) plan.sorted[i] = {role[i].sk, role[i].sv};

    // The persistent form: the stage table ordered by phase (empty phases
    // dropped), in the blob beside the arguments, and the grid that stays
    // resident with the largest stage's shared memory.
    size_t st_off = 0, ph_off = 0, psmem = 0;
    int n_phases = 0, ctas = 0;
    plan.persistent = b->persistent && fb.persistent_ok && !fb.pstages.empty();
    if (plan.persistent) {
        std::stable_sort(fb.pstages.begin(), fb.pstages.end(),
                         [](const FusedBuilder::PEntry& x, const FusedBuilder::PEntry& y) {
                             return x.phase < y.phase;
                         });
        std::vector<p3m::PStage> table;
        std::vector<p3m::PPhase> phases;
        for (size_t k = 0; k < fb.pstages.size(); ++k) {
            if (k == 0 || fb.pstages[k].phase != fb.pstages[k - 1].phase)
                phases.push_back({(int)k, 0});
            phases.back().stages++;
            table.push_back(fb.pstages[k].st);
        }
        n_phases = (int)phases.size();
        st_off = fb.blob.add(table.data(), table.size() * sizeof(p3m::PStage));
        ph_off = fb.blob.add(phases.data(), phases.size() * sizeof(p3m::PPhase));
        psmem = (std::max(fb.pool, p3m::persistent_base_smem()) + 15) & ~(size_t)15;
        const int fit = p3m::persistent_ctas_per_sm(psmem);
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int per_sm = b->persistent_ctas_per_sm > 0 ? std::min(b->persistent_ctas_per_sm, fit) : fit;
        ctas = sms * per_sm;
        if (ctas <= 0) plan.persistent = false;  // cannot stay resident: per-stage launches
    }
    plan.phases = plan.persistent ? n_phases : 0;
    plan.ctas = plan.persistent ? ctas : 0;

    // Upload the arguments, capture the launches.
    cudaError_t e = cudaMalloc(&plan.blob, std::max<size_t>(fb.blob.host.size(), 16));
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_OUT_OF_MEMORY, "fused plan arguments");
    e = cudaMemcpyAsync(plan.blob, fb.blob.host.data(), fb.blob.host.size(), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    unsigned char* dev = static_cast<unsigned char*>(plan.blob);
    const long long k0 = p3m_kernel_launches();
    e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    cudaError_t le = cudaSuccess;
    if (plan.persistent) {
        const float2* tw0 = mut.empty() ? nullptr : b->sims[mut[0]]->twiddles;
        le = p3m::launch_batch_persistent(
            dev, reinterpret_cast<const p3m::PStage*>(dev + st_off),
            reinterpret_cast<const p3m::PPhase*>(dev + ph_off), n_phases, tw0, b->sync,
            b->barrier_polls, b->withhold_cta, b->withhold_phase, ctas, psmem, b->phase_ns,
            b->stream);
    } else {
        for (auto& fn : fb.launches) {
            le = fn(dev, b->stream);
            if (le != cudaSuccess) break;
        }
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(b->stream, &graph);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return batch_fail(b, P3M_ERR_CUDA, std::string("fused capture: ") +
                                               cudaGetErrorString(le != cudaSuccess ? le : e));
    }
    plan.kernels = p3m_kernel_launches() - k0;
    e = cudaGraphInstantiate(&plan.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, std::string("fused instantiate: ") + cudaGetErrorString(e));
    return P3M_OK;
}

int batch_fused_step(p3m_batch* b, const std::vector<char>& sort, const std::vector<uint64_t>& key) {
    p3m_batch::Plan* plan = nullptr;
    for (auto& p : b->plans)
        if (p.key == key) { plan = &p; break; }
    if (!plan) {
        p3m_batch::Plan fresh;
        fresh.key = key;
        int st = build_fused(b, sort, fresh);
        if (st != P3M_OK) {
            if (fresh.exec) cudaGraphExecDestroy(fresh.exec);
            if (fresh.blob) cudaFree(fresh.blob);
            return st;
        }
        if (b->plans.size() >= 8) {
            cudaGraphExecDestroy(b->plans.front().exec);
            cudaFree(b->plans.front().blob);
            b->plans.erase(b->plans.begin());
        }
        b->plans.push_back(std::move(fresh));
        plan = &b->plans.back();
    }
    cudaError_t e = cudaGraphLaunch(plan->exec, b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    p3m::count_launches((int)plan->kernels);
    b->last_info[0] = plan->persistent ? 1 : 0;
    b->last_info[1] = (int32_t)plan->kernels;
    b->last_info[2] = plan->phases;
    b->last_info[3] = plan->ctas;
    for (size_t i = 0; i < b->sims.size(); ++i) {
        p3m_ctx* c = b->sims[i];
        if (plan->swap[i]) swap_body_buffers(c);
        if (c->mutual) c->built_n = b->n[i];
        if (c->mutual && b->n[i] > 0) {
            c->sorted_keys = plan->sorted[i].first;
            c->sorted_ids = plan->sorted[i].second;
        }
    }
    return P3M_OK;
}

// Device time of `steps` direct (not captured) steps of one simulation.
int time_direct_steps(p3m_ctx* c, int n, int steps, float* ms) {
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    P3M_CUDA(c, cudaEventCreate(&t0));
    P3M_CUDA(c, cudaEventCreate(&t1));
    P3M_CUDA(c, cudaEventRecord(t0, c->stream));
    for (int s = 0; s < steps; ++s) {
        normalize_to(c, n);
        const int interval = c->cfg.spatial_sort_interval;
        const bool sort = interval > 0 && (c->physics_steps % interval) == 0;
        if (interval > 0) c->physics_steps++;
        int st = enqueue_step(c, n, sort);
        if (st != P3M_OK) return st;
    }
    P3M_CUDA(c, cudaEventRecord(t1, c->stream));
    P3M_CUDA(c, cudaEventSynchronize(t1));
    P3M_CUDA(c, cudaEventElapsedTime(ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return P3M_OK;
}

// Launch shapes of one context by timing: `trial_steps` direct steps (after
// one untimed step) under each FFT line count per CTA (automatic, 1, 2, 4,
// 8), then each short-range block (64, 128, 256 threads) with the best line
// count. The trials step the context; its bodies, materials, accelerations
// and step counter are put back afterwards (the buffer roles may have
// swapped: the contents are what matter). Leaves the best shapes set.
int autotune_context(p3m_ctx* c, int n, int trial_steps, int* best_fft_out, int* best_sr_out) {
    const size_t cap = (size_t)c->cfg.capacity;
    float4 *sb = nullptr, *sm = nullptr;
    float2* sa = nullptr;
    const long long steps_before = c->physics_steps;
    P3M_CUDA(c, cudaMallocAsync((void**)&sb, cap * sizeof(float4), c->stream));
    P3M_CUDA(c, cudaMallocAsync((void**)&sm, cap * sizeof(float4), c->stream));
    P3M_CUDA(c, cudaMallocAsync((void**)&sa, cap * sizeof(float2), c->stream));
    P3M_CUDA(c, cudaMemcpyAsync(sb, c->bodies, cap * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    P3M_CUDA(c, cudaMemcpyAsync(sm, c->materials, cap * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    P3M_CUDA(c, cudaMemcpyAsync(sa, c->accel, cap * sizeof(float2), cudaMemcpyDeviceToDevice, c->stream));
    auto trial = [&](float* ms) -> int {
        c->grid = grid_for(c);
        int st = time_direct_steps(c, n, 1, ms);  // warm-up
        if (st == P3M_OK) st = time_direct_steps(c, n, trial_steps, ms);
        return st;
    };
    const int fft_choices[] = {0, 1, 2, 4, 8};
    const int sr_choices[] = {64, 128, 256};
    int best_fft = 0, best_sr = 256;
    float best = 3.4e38f, ms = 0.0f;
    c->tune_sr_threads = 256;
    for (int f : fft_choices) {
        c->tune_fft_lines = f;
        int st = trial(&ms);
        if (st != P3M_OK) return st;
        if (ms < best) { best = ms; best_fft = f; }
    }
    c->tune_fft_lines = best_fft;
    best = 3.4e38f;
    for (int t : sr_choices) {
        c->tune_sr_threads = t;
        int st = trial(&ms);
        if (st != P3M_OK) return st;
        if (ms < best) { best = ms; best_sr = t; }
    }
    c->tune_sr_threads = best_sr;
    c->grid = grid_for(c);
    P3M_CUDA(c, cudaMemcpyAsync(c->bodies, sb, cap * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    P3M_CUDA(c, cudaMemcpyAsync(c->materials, sm, cap * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    P3M_CUDA(c, cudaMemcpyAsync(c->accel, sa, cap * sizeof(float2), cudaMemcpyDeviceToDevice, c->stream));
    cudaFreeAsync(sb, c->stream);
    cudaFreeAsync(sm, c->stream);
    cudaFreeAsync(sa, c->stream);
    P3M_CUDA(c, cudaStreamSynchronize(c->stream));
    c->physics_steps = steps_before;
    drop_graphs(c);
    *best_fft_out = best_fft;
    *best_sr_out = best_sr;
    return P3M_OK;
}

// The fused form's autotuner. It times whole batch steps, the launches the
// batch really runs: first the form (one launch per stage, or the persistent
// launch with as many CTAs per SM as stay resident), then coordinate descent
// over the FFT lines per CTA of each distinct grid in turn (the other grids
// held), then, for the persistent form, over its CTAs per SM. Every
// simulation's bodies, materials, accelerations and step counter are saved
// first and put back after.
int autotune_fused(p3m_batch* b, int trial_steps, int32_t* chosen) {
    const size_t S = b->sims.size();
    struct Saved { float4* bodies = nullptr; float4* materials = nullptr; float2* accel = nullptr; long long steps = 0; };
    std::vector<Saved> saved(S);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    auto finish = [&](int st) {
        for (auto& v : saved) {
            if (v.bodies) cudaFree(v.bodies);
            if (v.materials) cudaFree(v.materials);
            if (v.accel) cudaFree(v.accel);
        }
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        return st;
    };
    auto cuda_fail = [&](cudaError_t e) { return finish(batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e))); };
    cudaError_t e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    if (e != cudaSuccess) return cuda_fail(e);
    for (size_t i = 0; i < S; ++i) {
        p3m_ctx* c = b->sims[i];
        const size_t cap = (size_t)c->cfg.capacity;
        e = cudaMalloc((void**)&saved[i].bodies, cap * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc((void**)&saved[i].materials, cap * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc((void**)&saved[i].accel, cap * sizeof(float2));
        if (e != cudaSuccess) return finish(batch_fail(b, P3M_ERR_OUT_OF_MEMORY, "autotune state copies"));
        e = cudaMemcpyAsync(saved[i].bodies, c->bodies, cap * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(saved[i].materials, c->materials, cap * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(saved[i].accel, c->accel, cap * sizeof(float2), cudaMemcpyDeviceToDevice, b->stream);
        if (e != cudaSuccess) return cuda_fail(e);
        saved[i].steps = c->physics_steps;
    }
    // One trial: fresh plans, four untimed steps (every plan of the reorder
    // and buffer cycle built), then `trial_steps` timed steps.
    auto trial = [&](float* ms) -> int {
        batch_drop_graphs(b);
        for (int w = 0; w < 4; ++w) {
            int st = batch_one_step(b);
            if (st != P3M_OK) return st;
        }
        cudaError_t te = cudaEventRecord(t0, b->stream);
        for (int k = 0; k < trial_steps && te == cudaSuccess; ++k) {
            int st = batch_one_step(b);
            if (st != P3M_OK) return st;
        }
        if (te == cudaSuccess) te = cudaEventRecord(t1, b->stream);
        if (te == cudaSuccess) te = cudaEventSynchronize(t1);
        if (te == cudaSuccess) te = cudaEventElapsedTime(ms, t0, t1);
        if (te != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(te));
        return P3M_OK;
    };
    // The distinct grids, each with its simulations.
    std::vector<std::vector<size_t>> groups;
    for (size_t i = 0; i < S; ++i) {
        const p3m_ctx* c = b->sims[i];
        bool placed = false;
        for (auto& g : groups) {
            const p3m_ctx* q = b->sims[g[0]];
            if (q->grid.W == c->grid.W && q->grid.H == c->grid.H && q->bounded == c->bounded) {
                g.push_back(i);
                placed = true;
                break;
            }
        }
        if (!placed) groups.push_back({i});
    }
    auto set_lines = [&](const std::vector<size_t>& g, int lines) {
        for (size_t i : g) {
            b->sims[i]->tune_fft_lines = lines;
            b->sims[i]->grid = grid_for(b->sims[i]);
        }
    };
    const int fft_choices[] = {0, 1, 2, 4, 8};
    std::vector<int> best_lines(groups.size(), 0);
    float ms = 0.0f;
    {
        float best = 3.4e38f;
        bool best_form = false;
        for (bool form : {false, true}) {
            b->persistent = form;
            b->persistent_ctas_per_sm = 0;
            int st = trial(&ms);
            if (st != P3M_OK) return finish(st);
            if (ms < best) { best = ms; best_form = form; }
        }
        b->persistent = best_form;
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
        float best = 3.4e38f;
        for (int f : fft_choices) {
            set_lines(groups[gi], f);
            int st = trial(&ms);
            if (st != P3M_OK) return finish(st);
            if (ms < best) { best = ms; best_lines[gi] = f; }
        }
        set_lines(groups[gi], best_lines[gi]);
    }
    if (b->persistent) {
        float best = 3.4e38f;
        int best_ctas = 0;
        for (int per_sm : {0, 1, 2, 3}) {
            b->persistent_ctas_per_sm = per_sm;
            int st = trial(&ms);
            if (st != P3M_OK) return finish(st);
            if (ms < best) { best = ms; best_ctas = per_sm; }
        }
        b->persistent_ctas_per_sm = best_ctas;
    }
    // Put every simulation's state back (the buffer roles may have swapped;
    // the contents are what matter).
    e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    batch_drop_graphs(b);
    for (size_t i = 0; i < S; ++i) {
        p3m_ctx* c = b->sims[i];
        const size_t cap = (size_t)c->cfg.capacity;
        e = cudaMemcpyAsync(c->bodies, saved[i].bodies, cap * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->materials, saved[i].materials, cap * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->accel, saved[i].accel, cap * sizeof(float2), cudaMemcpyDeviceToDevice, b->stream);
        if (e != cudaSuccess) return cuda_fail(e);
        c->physics_steps = saved[i].steps;
    }
    e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    for (size_t gi = 0; gi < groups.size() && chosen && gi < 64; ++gi) {
        const p3m_ctx* c = b->sims[groups[gi][0]];
        chosen[4 * gi + 0] = c->grid.W;
        chosen[4 * gi + 1] = c->grid.H;
        chosen[4 * gi + 2] = best_lines[gi];
        chosen[4 * gi + 3] = p3m::kBatchThreads;
    }
    return finish(P3M_OK);
}

}  // namespace

extern "C" {

int p3m_batch_create(const p3m_config* configs, int32_t count, p3m_batch** out) {
    g_create_error.clear();
    if (!out || !configs || count <= 0) return batch_fail(nullptr, P3M_ERR_INVALID_ARGUMENT, "configs, count and out are required");
    *out = nullptr;
    p3m_batch* b = new (std::nothrow) p3m_batch();
    if (!b) return batch_fail(nullptr, P3M_ERR_OUT_OF_MEMORY, "host allocation failed");
    auto undo = [&](int st) {
        for (p3m_ctx* c : b->sims) p3m_destroy(c);
        if (b->sync) cudaFree(b->sync);
        if (b->phase_ns) cudaFree(b->phase_ns);
        for (cudaEvent_t e : b->join) cudaEventDestroy(e);
        if (b->fork) cudaEventDestroy(b->fork);
        if (b->side_fork) cudaEventDestroy(b->side_fork);
        if (b->side_join) cudaEventDestroy(b->side_join);
        if (b->side) cudaStreamDestroy(b->side);
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return st;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->side_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->side_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return undo(fail_cuda(nullptr, "batch stream/event", e));
    e = cudaMalloc((void**)&b->sync, 2 * sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMalloc((void**)&b->phase_ns, p3m::kPersistentMaxStamps * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(b->sync, 0, 2 * sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMemset(b->phase_ns, 0, p3m::kPersistentMaxStamps * sizeof(unsigned long long));
    if (e != cudaSuccess) return undo(fail_cuda(nullptr, "batch barrier words", e));
    for (int32_t i = 0; i < count; ++i) {
        p3m_ctx* c = nullptr;
        int st = p3m_create(&configs[i], &c);
        if (st != P3M_OK) {
            g_create_error = "simulation " + std::to_string(i) + ": " + g_create_error;
            return undo(st);
        }
        b->sims.push_back(c);
        b->n.push_back(0);
        cudaEvent_t j = nullptr;
        e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        if (e != cudaSuccess) return undo(fail_cuda(nullptr, "batch event", e));
        b->join.push_back(j);
    }
    *out = b;
    return P3M_OK;
}

int p3m_batch_destroy(p3m_batch* b) {
    if (!b) return P3M_OK;
    cudaStreamSynchronize(b->stream);
    for (cudaStream_t s : {b->up_stream, b->down_stream})
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    for (cudaEvent_t e : {b->in_ready, b->in_free, b->out_ready, b->out_free})
        if (e) cudaEventDestroy(e);
    for (auto& a : b->io_args) cudaFree(a.dev);
    if (b->stage_in) cudaFree(b->stage_in);
    if (b->stage_out) cudaFree(b->stage_out);
    batch_drop_graphs(b);
    for (p3m_ctx* c : b->sims) p3m_destroy(c);
    cudaFree(b->sync);
    cudaFree(b->phase_ns);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    cudaEventDestroy(b->fork);
    cudaEventDestroy(b->side_fork);
    cudaEventDestroy(b->side_join);
    cudaStreamSynchronize(b->side);
    cudaStreamDestroy(b->side);
    cudaStreamDestroy(b->stream);
    delete b;
    return P3M_OK;
}

const char* p3m_batch_last_error(const p3m_batch* b) {
    return b ? b->last_error.c_str() : g_create_error.c_str();
}

int p3m_batch_size(const p3m_batch* b, int32_t* count) {
    if (!b || !count) return P3M_ERR_INVALID_ARGUMENT;
    *count = (int32_t)b->sims.size();
    return P3M_OK;
}

int p3m_batch_context(p3m_batch* b, int32_t sim, p3m_ctx** ctx) {
    if (!b || !ctx) return P3M_ERR_INVALID_ARGUMENT;
    if (sim < 0 || sim >= (int32_t)b->sims.size()) return batch_fail(b, P3M_ERR_INVALID_ARGUMENT, "simulation index out of range");
    *ctx = b->sims[sim];
    return P3M_OK;
}

int p3m_batch_upload(p3m_batch* b, int32_t sim, const float* bodies4, const float* materials4,
                     int32_t n) {
    p3m_ctx* c = nullptr;
    int st = p3m_batch_context(b, sim, &c);
    if (st != P3M_OK) return st;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    st = p3m_upload_state(c, bodies4, materials4, nullptr, n);
    if (st != P3M_OK) return batch_fail_ctx(b, (size_t)sim, st);
    b->n[sim] = n;
    return P3M_OK;
}

int p3m_batch_initialize_acceleration(p3m_batch* b) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    for (size_t i = 0; i < b->sims.size(); ++i) {
        int st = p3m_initialize_acceleration(b->sims[i], b->n[i]);
        if (st != P3M_OK) return batch_fail_ctx(b, i, st);
    }
    for (size_t i = 0; i < b->sims.size(); ++i) {
        int st = p3m_synchronize(b->sims[i]);
        if (st != P3M_OK) return batch_fail_ctx(b, i, st);
    }
    return P3M_OK;
}

int p3m_batch_step(p3m_batch* b, int32_t steps) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    if (steps < 0) return batch_fail(b, P3M_ERR_INVALID_ARGUMENT, "steps must be >= 0");
    for (int32_t s = 0; s < steps; ++s) {
        int st = batch_one_step(b);
        if (st != P3M_OK) return st;
    }
    return P3M_OK;
}

int p3m_batch_autotune(p3m_batch* b, int32_t trial_steps, int32_t* chosen) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    if (trial_steps <= 0) return batch_fail(b, P3M_ERR_INVALID_ARGUMENT, "trial_steps must be > 0");
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    batch_drop_graphs(b);
    if (b->fused && fused_supported(b)) return autotune_fused(b, trial_steps, chosen);
    // One probe per distinct grid: the simulation with the most bodies.
    std::vector<size_t> probes;
    for (size_t i = 0; i < b->sims.size(); ++i) {
        const p3m_ctx* c = b->sims[i];
        bool placed = false;
        for (size_t& p : probes) {
            const p3m_ctx* q = b->sims[p];
            if (q->grid.W == c->grid.W && q->grid.H == c->grid.H && q->bounded == c->bounded) {
                if (b->n[i] > b->n[p]) p = i;
                placed = true;
                break;
            }
        }
        if (!placed) probes.push_back(i);
    }
    int tuned = 0;
    for (size_t p : probes) {
        p3m_ctx* c = b->sims[p];
        int best_fft = 0, best_sr = 256;
        int st = autotune_context(c, b->n[p], trial_steps, &best_fft, &best_sr);
        if (st != P3M_OK) return batch_fail_ctx(b, p, st);
        for (size_t i = 0; i < b->sims.size(); ++i) {
            p3m_ctx* o = b->sims[i];
            if (o->grid.W == c->grid.W && o->grid.H == c->grid.H && o->bounded == c->bounded) {
                o->tune_fft_lines = best_fft;
                o->tune_sr_threads = best_sr;
                o->grid = grid_for(o);
                drop_graphs(o);
            }
        }
        if (chosen && tuned < 64) {
            chosen[4 * tuned + 0] = c->grid.W;
            chosen[4 * tuned + 1] = c->grid.H;
            chosen[4 * tuned + 2] = best_fft;
            chosen[4 * tuned + 3] = best_sr;
        }
        ++tuned;
    }
    return P3M_OK;
}

int p3m_batch_set_fused(p3m_batch* b, int32_t enabled) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    batch_drop_graphs(b);
    b->fused = enabled != 0;
    return P3M_OK;
}

int p3m_batch_synchronize(p3m_batch* b) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    // p3m_batch_step_io's copies (the last download follows the last step).
    if (e == cudaSuccess && b->up_stream) e = cudaStreamSynchronize(b->up_stream);
    if (e == cudaSuccess && b->down_stream) e = cudaStreamSynchronize(b->down_stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    unsigned int gave_up = 0;  // grid-barrier waits that ran out, over all launches
    e = cudaMemcpy(&gave_up, b->sync + 1, sizeof(gave_up), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    if (gave_up != b->reported_timeouts) {
        b->reported_timeouts = gave_up;
        return batch_fail(b, P3M_ERR_TIMEOUT,
                          "a grid barrier of the persistent batch step gave up waiting (" +
                              std::to_string(gave_up) + " waits so far); the simulations' "
                              "state is incomplete and must be uploaded again");
    }
    return P3M_OK;
}

int p3m_batch_step_io(p3m_batch* b, const float* host_bodies_in4, float* host_bodies_out4) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaSuccess;
    if (!b->up_stream) {  // first call: copy streams, staging, events
        size_t cap = 0;
        for (p3m_ctx* c : b->sims) cap += (size_t)c->cfg.capacity;
        e = cudaStreamCreateWithFlags(&b->up_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->down_stream, cudaStreamNonBlocking);
        for (cudaEvent_t* ev : {&b->in_ready, &b->in_free, &b->out_ready, &b->out_free})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
        if (cudaMalloc((void**)&b->stage_in, std::max<size_t>(cap, 1) * sizeof(float4)) != cudaSuccess ||
            cudaMalloc((void**)&b->stage_out, std::max<size_t>(cap, 1) * sizeof(float4)) != cudaSuccess)
            return batch_fail(b, P3M_ERR_OUT_OF_MEMORY, "staging buffers of p3m_batch_step_io");
    }
    long long rows = 0;
    for (int v : b->n) rows += v;
    const size_t bytes = (size_t)rows * sizeof(float4);
    if (host_bodies_in4 && rows > 0) {
        const p3m_batch::IoArgs* a = batch_io_args(b, true);
        if (!a) return batch_fail(b, P3M_ERR_OUT_OF_MEMORY, "row-copy arguments");
        // The upload waits only until the previous step has taken the last
        // upload out of the staging buffer, so it overlaps that step.
        e = cudaStreamWaitEvent(b->up_stream, b->in_free, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->stage_in, host_bodies_in4, bytes, cudaMemcpyHostToDevice, b->up_stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->in_ready, b->up_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->in_ready, 0);
        if (e == cudaSuccess) e = launch_io_copy(b, a);
        if (e == cudaSuccess) e = cudaEventRecord(b->in_free, b->stream);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    }
    int st = batch_one_step(b);
    if (st != P3M_OK) return st;
    if (host_bodies_out4 && rows > 0) {
        const p3m_batch::IoArgs* a = batch_io_args(b, false);  // the buffers after the step
        if (!a) return batch_fail(b, P3M_ERR_OUT_OF_MEMORY, "row-copy arguments");
        // The stepped bodies go to the staging buffer once the previous
        // download has left it; the download then overlaps the next step.
        e = cudaStreamWaitEvent(b->stream, b->out_free, 0);
        if (e == cudaSuccess) e = launch_io_copy(b, a);
        if (e == cudaSuccess) e = cudaEventRecord(b->out_ready, b->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->down_stream, b->out_ready, 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host_bodies_out4, b->stage_out, bytes, cudaMemcpyDeviceToHost,
                                b->down_stream);
        if (e == cudaSuccess) e = cudaEventRecord(b->out_free, b->down_stream);
        if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    }
    return P3M_OK;
}

int p3m_batch_set_persistent(p3m_batch* b, int32_t enabled, int32_t ctas_per_sm) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    if (ctas_per_sm < 0) return batch_fail(b, P3M_ERR_INVALID_ARGUMENT, "ctas_per_sm must be >= 0");
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    batch_drop_graphs(b);
    b->persistent = enabled != 0;
    b->persistent_ctas_per_sm = ctas_per_sm;
    return P3M_OK;
}

int p3m_batch_set_barrier_fault(p3m_batch* b, int32_t poll_limit, int32_t withheld_cta,
                                int32_t phase) {
    if (!b) return P3M_ERR_INVALID_ARGUMENT;
    if (poll_limit <= 0 || withheld_cta < -1 || phase < -1)
        return batch_fail(b, P3M_ERR_INVALID_ARGUMENT,
                          "poll_limit must be > 0, withheld_cta and phase >= -1");
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    batch_drop_graphs(b);  // the plans bake the barrier's arguments in
    b->barrier_polls = poll_limit;
    b->withhold_cta = withheld_cta;
    b->withhold_phase = phase;
    return P3M_OK;
}

int p3m_batch_plan_info(p3m_batch* b, int32_t* info4) {
    if (!b || !info4) return P3M_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < 4; ++i) info4[i] = b->last_info[i];
    return P3M_OK;
}

int p3m_batch_phase_times(p3m_batch* b, double* ms, int32_t capacity, int32_t* phases) {
    if (!b || !phases || capacity < 0 || (capacity > 0 && !ms)) return P3M_ERR_INVALID_ARGUMENT;
    *phases = 0;
    if (!b->last_info[0]) return P3M_OK;
    const int np = std::min(b->last_info[2], p3m::kPersistentMaxStamps - 1);
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    std::vector<unsigned long long> ns(np + 1, 0);
    e = cudaMemcpy(ns.data(), b->phase_ns, ns.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return batch_fail(b, P3M_ERR_CUDA, cudaGetErrorString(e));
    for (int i = 0; i < np && i < capacity; ++i)
        ms[i] = ns[i + 1] >= ns[i] ? (double)(ns[i + 1] - ns[i]) * 1e-6 : 0.0;
    *phases = np;
    return P3M_OK;
}

int p3m_batch_get_stream(p3m_batch* b, void** stream) {
    if (!b || !stream) return P3M_ERR_INVALID_ARGUMENT;
    *stream = (void*)b->stream;
    return P3M_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Differentiated rollout: the gravity-only step (GravityPipeline.kt:445-494
// without collisions) run forward with checkpoints, then reversed with the
// hand-written adjoint of p3m_adjoint.cu. The reference has no adjoint.
//
// Forward: `steps` plain steps (graph-replayed like p3m_step), with the
// bodies and accelerations saved every `interval` steps. Backward: for each
// segment from the last, the segment's checkpoint is restored and its steps
// recomputed, keeping for every step the positions, cell lists and mesh
// force the reverse step needs (the memory of one segment), then the steps
// are reversed. The context's state is put back to the forward's end.
// Memory: (steps/interval + 2) x 24 B per body of checkpoints, plus
// (interval + 1) x (32 B per body + 12 B per cell + 8 B per mesh cell) of
// recompute slots, plus the cotangents.

struct p3m_adjoint_store {
    int n = 0, steps = 0, interval = 0, initial = 0, slots = 0;
    size_t P = 0, M = 0;
    bool recorded = false;
    std::vector<void*> blocks;
    float4* ck_bodies = nullptr;  // [checkpoints + 1][n], the last: the final state
    float2* ck_accel = nullptr;
    float4* slot_bodies = nullptr;  // [slots][n]
    float4* slot_entries = nullptr;
    int* slot_start = nullptr;      // [slots][P]
    int* slot_count = nullptr;
    uint32_t* slot_mass = nullptr;
    float2* slot_force = nullptr;   // [slots][M]
    float4* lam = nullptr;          // cotangents of (x, y, vx, vy)
    float2* lam_a = nullptr;        // cotangents of a
    float2* wa = nullptr;
    float2* g_short = nullptr;
    float* cot = nullptr;           // 2*MH x MW
    float2* half2 = nullptr;        // 2*MH x (MW/2+1)
    float2* mu2 = nullptr;          // MH/2 x MW
    // One captured reverse step per slot (its pointers are the slot's), with
    // the parameters it was captured with; re-captured when they change.
    struct ReverseGraph {
        cudaGraphExec_t exec = nullptr;
        p3m::AdjointParams p{};
        const void* buffers[4] = {};  // the context buffers it reads
        long long kernels = 0;
    };
    std::vector<ReverseGraph> reverse_graphs;
};

namespace {

void adjoint_free(p3m_ctx* ctx) {
    if (!ctx->adjoint) return;
    for (auto& g : ctx->adjoint->reverse_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (void* b : ctx->adjoint->blocks) cudaFree(b);
    delete ctx->adjoint;
    ctx->adjoint = nullptr;
}

int checkpoints_for(int steps, int interval) { return (steps + interval - 1) / interval; }

template <typename T>
int adjoint_alloc(p3m_ctx* ctx, p3m_adjoint_store* a, T** out, size_t count) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return fail_cuda(ctx, "adjoint storage", e);
    a->blocks.push_back(p);
    *out = static_cast<T*>(p);
    return P3M_OK;
}

int adjoint_prepare(p3m_ctx* ctx, int n, int steps, int interval) {
    p3m_adjoint_store* a = ctx->adjoint;
    const size_t P = phys_cells(ctx), M = mesh_cells(ctx);
    if (a && a->n == n && a->steps == steps && a->interval == interval && a->P == P && a->M == M)
        return P3M_OK;
    adjoint_free(ctx);
    a = new (std::nothrow) p3m_adjoint_store();
    if (!a) return fail(ctx, P3M_ERR_OUT_OF_MEMORY, "host allocation failed");
    ctx->adjoint = a;
    a->n = n;
    a->steps = steps;
    a->interval = interval;
    a->P = P;
    a->M = M;
    a->slots = interval + 1;
    const size_t nn = (size_t)n, ck = (size_t)checkpoints_for(steps, interval) + 1;
    const size_t S = (size_t)a->slots;
    const size_t SW = (size_t)ctx->grid.MW / 2 + 1, MH = (size_t)ctx->grid.MH, MW = (size_t)ctx->grid.MW;
    int st = P3M_OK;
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->ck_bodies, ck * nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->ck_accel, ck * nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_bodies, S * nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_entries, S * nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_start, S * P);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_count, S * P);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_mass, S * P);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->slot_force, S * M);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->lam, nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->lam_a, nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->wa, nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->g_short, nn);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->cot, 2 * MH * MW);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->half2, 2 * MH * SW);
    if (st == P3M_OK) st = adjoint_alloc(ctx, a, &a->mu2, MH / 2 * MW);
    if (st != P3M_OK) adjoint_free(ctx);
    return st;
}

#define P3M_COPY(ctx, dst, src, bytes) \
    P3M_CUDA(ctx, cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyDeviceToDevice, (ctx)->stream))

// Keeps what the reverse step at the current state needs.
// Up to six device-to-device copies in one launch (16-byte words; every
// segment here starts on a 16-byte boundary and is a multiple of 16 bytes).
struct CopySegments {
    uint4* dst[6];
    const uint4* src[6];
    long long words[6];
    int count;
};

__global__ void __launch_bounds__(256) copy_segments_kernel(CopySegments c) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int k = 0; k < c.count; ++k)
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < c.words[k];
             i += stride)
            c.dst[k][i] = c.src[k][i];
}

// The state a reverse step needs, saved into recompute slot `slot` with one
// kernel (a backward pass saves a slot per step: six copies each would be
// six launches).
int adjoint_save_slot(p3m_ctx* ctx, int slot) {
    p3m_adjoint_store* a = ctx->adjoint;
    const size_t n = (size_t)a->n, P = a->P, M = a->M, s = (size_t)slot;
    CopySegments c{};
    auto add = [&](void* dst, const void* src, size_t bytes) {
        c.dst[c.count] = static_cast<uint4*>(dst);
        c.src[c.count] = static_cast<const uint4*>(src);
        c.words[c.count] = (long long)(bytes / sizeof(uint4));
        ++c.count;
    };
    add(a->slot_bodies + s * n, ctx->bodies, n * sizeof(float4));
    add(a->slot_entries + s * n, ctx->entries, n * sizeof(float4));
    add(a->slot_start + s * P, ctx->cell_start, P * sizeof(int));  // P is a multiple of 16
    add(a->slot_count + s * P, ctx->cell_count, P * sizeof(int));
    add(a->slot_mass + s * P, ctx->cell_mass, P * sizeof(uint32_t));
    add(a->slot_force + s * M, ctx->force, M * sizeof(float2));
    copy_segments_kernel<<<4 * 148, 256, 0, ctx->stream>>>(c);
    p3m::count_launches(1);
    P3M_CUDA(ctx, cudaGetLastError());
    return P3M_OK;
}

int adjoint_checkpoint(p3m_ctx* ctx, int index, bool restore) {
    p3m_adjoint_store* a = ctx->adjoint;
    const size_t n = (size_t)a->n, k = (size_t)index;
    if (restore) {
        P3M_COPY(ctx, ctx->bodies, a->ck_bodies + k * n, n * sizeof(float4));
        P3M_COPY(ctx, ctx->accel, a->ck_accel + k * n, n * sizeof(float2));
    } else {
        P3M_COPY(ctx, a->ck_bodies + k * n, ctx->bodies, n * sizeof(float4));
        P3M_COPY(ctx, a->ck_accel + k * n, ctx->accel, n * sizeof(float2));
    }
    return P3M_OK;
}

p3m::AdjointParams adjoint_params(const p3m_ctx* ctx, int n) {
    p3m::AdjointParams p;
    p.n = n;
    p.W = ctx->grid.W; p.H = ctx->grid.H; p.MW = ctx->grid.MW; p.MH = ctx->grid.MH;
    p.bounded = ctx->bounded; p.rx = ctx->rx; p.ry = ctx->ry;
    p.exact = ctx->cfg.exact_neighbor_body_limit;
    p.home_limit = ctx->cfg.maximum_home_body_interactions;
    p.mutual = ctx->mutual;
    p.fold = 0;
    p.aspect = ctx->aspect; p.gravity = ctx->cfg.gravitational_constant;
    p.sigma_cells = ctx->cfg.softening_cells; p.total_mass = ctx->normalization_mass;
    p.min_frac = ctx->cfg.minimum_distance_cell_fraction; p.dt = ctx->cfg.time_step;
    p.cv = 0.5f * ctx->cfg.time_step;
    return p;
}

// One reverse step against recompute slot `slot`.
int adjoint_reverse_enqueue(p3m_ctx* ctx, int slot, const p3m::AdjointParams& p) {
    p3m_adjoint_store* a = ctx->adjoint;
    const size_t n = (size_t)a->n, P = a->P, M = a->M, s = (size_t)slot;
    const float4* bodies = a->slot_bodies + s * n;
    P3M_CUDA(ctx, cudaMemsetAsync(a->cot, 0, 2 * M * sizeof(float), ctx->stream));
    P3M_CUDA(ctx, cudaMemsetAsync(a->g_short, 0, n * sizeof(float2), ctx->stream));
    P3M_CUDA(ctx, p3m::launch_adjoint_spread(bodies, a->lam, a->lam_a, a->wa, a->cot, p, ctx->stream));
    P3M_CUDA(ctx, p3m::launch_adjoint_short_range(bodies, a->slot_entries + s * n,
                                                  a->slot_start + s * P, a->slot_count + s * P,
                                                  a->slot_mass + s * P, a->wa, a->g_short, p,
                                                  ctx->stream));
    if (p.mutual)
        P3M_CUDA(ctx, p3m::launch_fft_adjoint(a->cot, ctx->green, 1.0f / ctx->normalization_mass,
                                              ctx->grid, ctx->twiddles, a->half2, ctx->cols,
                                              a->mu2, ctx->stream));
    P3M_CUDA(ctx, p3m::launch_adjoint_gather(bodies, ctx->materials, a->wa, a->mu2,
                                             a->slot_force + s * M, a->g_short, a->lam, a->lam_a,
                                             p, ctx->stream));
    return P3M_OK;
}

// One reverse step (two clears and six kernels), replayed from a CUDA graph
// captured once per slot: a backward pass runs hundreds of them, each too
// short to hide eight launches.
int adjoint_reverse(p3m_ctx* ctx, int slot, const p3m::AdjointParams& p) {
    p3m_adjoint_store* a = ctx->adjoint;
    if (!ctx->use_graphs || ctx->profiling) return adjoint_reverse_enqueue(ctx, slot, p);
    if ((int)a->reverse_graphs.size() < a->slots) a->reverse_graphs.resize(a->slots);
    auto& g = a->reverse_graphs[slot];
    const void* buffers[4] = {ctx->materials, ctx->green, ctx->cols, ctx->twiddles};
    if (g.exec && std::memcmp(&g.p, &p, sizeof(p)) == 0 &&
        std::memcmp(g.buffers, buffers, sizeof(buffers)) == 0) {
        P3M_CUDA(ctx, cudaGraphLaunch(g.exec, ctx->stream));
        p3m::count_launches((int)g.kernels);
        return P3M_OK;
    }
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    const long long k0 = p3m_kernel_launches();
    P3M_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int st = adjoint_reverse_enqueue(ctx, slot, p);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != P3M_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (st != P3M_OK) return st;
        return fail_cuda(ctx, "cudaStreamEndCapture", e);
    }
    g.kernels = p3m_kernel_launches() - k0;
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g.exec = nullptr;
        return fail_cuda(ctx, "cudaGraphInstantiate", e);
    }
    g.p = p;
    std::memcpy(g.buffers, buffers, sizeof(buffers));
    P3M_CUDA(ctx, cudaGraphLaunch(g.exec, ctx->stream));
    return P3M_OK;
}

}  // namespace

extern "C" {

int p3m_adjoint_forward(p3m_ctx* ctx, int32_t n, int32_t steps, int32_t interval, int32_t flags) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (steps < 1 || interval < 1) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "steps and interval must be >= 1");
    if (n < 1) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "the rollout needs at least one body");
    if (flags & ~P3M_ADJOINT_INITIAL_ACCELERATION) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "unknown flags");
    if (ctx->bounded) return fail(ctx, P3M_ERR_UNSUPPORTED, "the differentiated rollout covers the torus only");
    if (ctx->cfg.spatial_sort_interval != 0)
        return fail(ctx, P3M_ERR_UNSUPPORTED, "the differentiated rollout keeps body order: spatial_sort_interval must be 0");
    normalize_to(ctx, n);
    st = ensure_green(ctx);
    if (st != P3M_OK) return st;
    st = adjoint_prepare(ctx, n, steps, interval);
    if (st != P3M_OK) return st;
    p3m_adjoint_store* a = ctx->adjoint;
    a->recorded = false;
    a->initial = (flags & P3M_ADJOINT_INITIAL_ACCELERATION) ? 1 : 0;
    if (a->initial) {
        st = p3m_initialize_acceleration(ctx, n);
        if (st != P3M_OK) return st;
    }
    for (int k = 0; k < steps; ++k) {
        if (k % interval == 0) {
            st = adjoint_checkpoint(ctx, k / interval, false);
            if (st != P3M_OK) return st;
        }
        st = one_step(ctx, n);
        if (st != P3M_OK) return st;
    }
    st = adjoint_checkpoint(ctx, checkpoints_for(steps, interval), false);
    if (st != P3M_OK) return st;
    a->recorded = true;
    return P3M_OK;
}

int p3m_adjoint_backward(p3m_ctx* ctx, const float* seed_bodies4, const float* seed_accel2,
                         float* grad_bodies4, float* grad_accel2) {
    if (!ctx || !seed_bodies4 || !grad_bodies4) return P3M_ERR_INVALID_ARGUMENT;
    p3m_adjoint_store* a = ctx->adjoint;
    if (!a || !a->recorded) return fail(ctx, P3M_ERR_STATE, "no recorded rollout: call p3m_adjoint_forward first");
    const int n = a->n;
    normalize_to(ctx, n);
    P3M_CUDA(ctx, cudaMemcpyAsync(a->lam, seed_bodies4, (size_t)n * sizeof(float4), cudaMemcpyDefault, ctx->stream));
    if (seed_accel2)
        P3M_CUDA(ctx, cudaMemcpyAsync(a->lam_a, seed_accel2, (size_t)n * sizeof(float2), cudaMemcpyDefault, ctx->stream));
    else
        P3M_CUDA(ctx, cudaMemsetAsync(a->lam_a, 0, (size_t)n * sizeof(float2), ctx->stream));
    const p3m::AdjointParams p = adjoint_params(ctx, n);
    const int init_slot = a->slots - 1;
    int st = P3M_OK;
    for (int seg = checkpoints_for(a->steps, a->interval) - 1; seg >= 0; --seg) {
        const int first = seg * a->interval;
        const int count = std::min(a->interval, a->steps - first);
        st = adjoint_checkpoint(ctx, seg, true);
        if (st != P3M_OK) return st;
        if (seg == 0 && a->initial && ctx->mutual) {
            st = build_force(ctx, n);
            if (st == P3M_OK) st = adjoint_save_slot(ctx, init_slot);
            if (st != P3M_OK) return st;
        }
        for (int s = 0; s < count; ++s) {
            st = one_step(ctx, n);
            if (st == P3M_OK) st = adjoint_save_slot(ctx, s);
            if (st != P3M_OK) return st;
        }
        for (int s = count - 1; s >= 0; --s) {
            st = adjoint_reverse(ctx, s, p);
            if (st != P3M_OK) return st;
        }
    }
    if (a->initial && ctx->mutual) {
        p3m::AdjointParams q = p;
        q.cv = 0.0f;
        q.fold = 1;
        st = adjoint_reverse(ctx, init_slot, q);
        if (st != P3M_OK) return st;
    } else if (a->initial) {
        P3M_CUDA(ctx, cudaMemsetAsync(a->lam_a, 0, (size_t)n * sizeof(float2), ctx->stream));
    }
    st = adjoint_checkpoint(ctx, checkpoints_for(a->steps, a->interval), true);
    if (st != P3M_OK) return st;
    P3M_CUDA(ctx, cudaMemcpyAsync(grad_bodies4, a->lam, (size_t)n * sizeof(float4), cudaMemcpyDefault, ctx->stream));
    if (grad_accel2)
        P3M_CUDA(ctx, cudaMemcpyAsync(grad_accel2, a->lam_a, (size_t)n * sizeof(float2), cudaMemcpyDefault, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

int p3m_adjoint_release(p3m_ctx* ctx) {
    if (!ctx) return P3M_ERR_INVALID_ARGUMENT;
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    adjoint_free(ctx);
    return P3M_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Aim previews (updateTrajectory, GravityPipeline.kt:514-600; trajectory.comp).

extern "C" {

int p3m_trajectory_config_default(p3m_trajectory_config* c) {
    if (!c) return P3M_ERR_INVALID_ARGUMENT;
    // TrajectoryConfig (GravityConfig.kt:739-745), CollisionConfig
    // restitutionCoefficient (GravityConfig.kt:682).
    c->struct_size = (int32_t)sizeof(p3m_trajectory_config);
    c->steps = 1024;
    c->maximum_time_step = 1.0f;
    c->target_segment_pixels = 6.0f;
    c->maximum_path_viewport_diagonals = 1.0f;
    c->minimum_dash_pixels = 3.0f;
    c->restitution_coefficient = 0.0f;
    return P3M_OK;
}

int p3m_trajectories(p3m_ctx* ctx, int32_t n, const p3m_trajectory_config* tc, int32_t count,
                     const float* origins_px2, const float* velocities_px2, float* vertices4) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (!tc || tc->struct_size != (int32_t)sizeof(p3m_trajectory_config))
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "trajectory config missing or of another version");
    // TrajectoryConfig's checks (GravityConfig.kt:747-756).
    if (tc->steps < 1 || tc->steps > 65536)
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "steps must be in 1..65536");
    auto positive = [](float v) { return v > 0.0f && std::isfinite(v); };
    if (!positive(tc->maximum_time_step) || !positive(tc->target_segment_pixels) ||
        !positive(tc->maximum_path_viewport_diagonals) || !positive(tc->minimum_dash_pixels))
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "trajectory lengths and times must be positive and finite");
    if (!(tc->restitution_coefficient >= 0.0f && tc->restitution_coefficient <= 1.0f))
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "restitution must be in [0, 1]");
    if (count < 0) return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "count must be >= 0");
    if (count == 0) return P3M_OK;
    if (!origins_px2 || !velocities_px2 || !vertices4)
        return fail(ctx, P3M_ERR_INVALID_ARGUMENT, "origins, velocities and vertices are required");
    if (ctx->mutual && ctx->built_n != n)
        return fail(ctx, P3M_ERR_STATE, "no force built for this body count: step or initialize first");
    const size_t in_bytes = (size_t)count * sizeof(float2);
    const size_t out_bytes = (size_t)count * (size_t)tc->steps * 6 * sizeof(float4);
    const size_t need = 2 * in_bytes + out_bytes + 64;
    if (ctx->traj_scratch_bytes < need) {
        if (ctx->traj_scratch) cudaFree(ctx->traj_scratch);
        ctx->traj_scratch = nullptr;
        ctx->traj_scratch_bytes = 0;
        cudaError_t e = cudaMalloc(&ctx->traj_scratch, need);
        if (e != cudaSuccess) return fail_cuda(ctx, "trajectory buffers", e);
        ctx->traj_scratch_bytes = need;
    }
    unsigned char* base = static_cast<unsigned char*>(ctx->traj_scratch);
    float2* d_origins = reinterpret_cast<float2*>(base);
    float2* d_vel = reinterpret_cast<float2*>(base + in_bytes);
    float4* d_out = reinterpret_cast<float4*>(base + ((2 * in_bytes + 15) & ~(size_t)15));
    P3M_CUDA(ctx, cudaMemcpyAsync(d_origins, origins_px2, in_bytes, cudaMemcpyDefault, ctx->stream));
    P3M_CUDA(ctx, cudaMemcpyAsync(d_vel, velocities_px2, in_bytes, cudaMemcpyDefault, ctx->stream));
    const p3m::KickParams k = kick_params(ctx, n, 0);
    const float vw = (float)ctx->cfg.viewport_width, vh = (float)ctx->cfg.viewport_height;
    const float max_path = tc->maximum_path_viewport_diagonals * std::sqrt(vw * vw + vh * vh);
    P3M_CUDA(ctx, p3m::launch_trajectories(k, make_float2(vw, vh), ctx->cfg.time_step,
                                           tc->maximum_time_step, tc->target_segment_pixels,
                                           max_path, tc->minimum_dash_pixels,
                                           tc->restitution_coefficient, tc->steps, count, d_origins,
                                           d_vel, ctx->force, ctx->entries, ctx->cell_start,
                                           ctx->cell_count, ctx->cell_mass, d_out, ctx->stream));
    P3M_CUDA(ctx, cudaMemcpyAsync(vertices4, d_out, out_bytes, cudaMemcpyDefault, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

}  // extern "C"
