// p3m_api.cu — the C-ABI of include/p3m.h: context lifecycle, state hand-off
// and the orchestration of GravityPipeline's P3M step
// (src/main/kotlin/dev/gravity/GravityPipeline.kt).

#include "p3m_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

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

void free_all(p3m_ctx* ctx) {
    void* ptrs[] = {ctx->bodies, ctx->bodies_alt, ctx->accel, ctx->accel_alt, ctx->materials,
                    ctx->materials_alt, ctx->destinations, ctx->status, ctx->keys, ctx->vals,
                    ctx->sort.keys_alt, ctx->sort.vals_alt, ctx->sort.hist, ctx->sort.block_sums,
                    ctx->cell_start, ctx->cell_count, ctx->cell_mass, ctx->entries, ctx->density,
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

// Cell lists from keys already written in descending ID order.
int lists_from_keys(p3m_ctx* ctx, int n) {
    const long long P = (long long)phys_cells(ctx);
    uint32_t* sk = ctx->keys;
    uint32_t* sv = ctx->vals;
    P3M_CUDA(ctx, p3m::radix_sort_pairs(ctx->keys, ctx->vals, ctx->sort, n, bits_for(P),
                                        ctx->stream, &sk, &sv));
    ctx->sorted_keys = sk;
    ctx->sorted_ids = sv;
    P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_count, 0, P * sizeof(int), ctx->stream));
    P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_mass, 0, P * sizeof(uint32_t), ctx->stream));
    P3M_CUDA(ctx, p3m::launch_cell_build(sk, sv, n, ctx->bodies, ctx->materials, ctx->cell_start,
                                         ctx->cell_count, ctx->cell_mass, ctx->entries,
                                         ctx->stream));
    return P3M_OK;
}

// Deposit + FFT + spectral multiply + inverse (GravityPipeline.kt:907-973
// after the lists).
int mesh_force(p3m_ctx* ctx, int n) {
    int st = ensure_green(ctx);
    if (st != P3M_OK) return st;
    const bool i64 = ctx->cfg.deposit_mode == P3M_DEPOSIT_I64;
    const size_t M = mesh_cells(ctx);
    P3M_CUDA(ctx, cudaMemsetAsync(ctx->density, 0, M * (i64 ? 8 : 4), ctx->stream));
    P3M_CUDA(ctx, p3m::launch_deposit(ctx->entries, ctx->sorted_keys, n, ctx->grid,
                                      ctx->cfg.deposit_mode, (float)ctx->mass_scale, ctx->density,
                                      ctx->stream));
    // fft_init.comp's uInverseMassScale = 1f / massScale (GravityPipeline.kt:942).
    const float inv_scale = i64 ? 1.0f / 4294967296.0f : 1.0f / (float)ctx->mass_scale;
    P3M_CUDA(ctx, p3m::launch_fft_forward_rows(ctx->density, ctx->cfg.deposit_mode, inv_scale,
                                               ctx->grid, ctx->twiddles, ctx->half, ctx->stream));
    P3M_CUDA(ctx, p3m::launch_fft_columns(ctx->half, ctx->green, 1.0f / ctx->normalization_mass,
                                          ctx->grid, ctx->twiddles, ctx->cols, ctx->stream));
    P3M_CUDA(ctx, p3m::launch_fft_inverse_rows(ctx->cols, ctx->grid, ctx->twiddles, ctx->force,
                                               ctx->stream));
    return P3M_OK;
}

int build_force(p3m_ctx* ctx, int n) {
    P3M_CUDA(ctx, p3m::launch_cell_keys(ctx->bodies, n, ctx->grid, ctx->keys, ctx->vals, ctx->stream));
    int st = lists_from_keys(ctx, n);
    if (st != P3M_OK) return st;
    return mesh_force(ctx, n);
}

int apply_kick(p3m_ctx* ctx, int n, int initial) {
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
    P3M_CUDA(ctx, p3m::launch_kick(ctx->bodies, ctx->accel, ctx->force, ctx->cell_start,
                                   ctx->cell_count, ctx->cell_mass, ctx->entries, p, ctx->stream));
    return P3M_OK;
}

// GravityPipeline.kt:1269-1319 sortBodies.
int sort_bodies(p3m_ctx* ctx, int n) {
    if (n <= 0) return P3M_OK;
    P3M_CUDA(ctx, p3m::launch_morton_keys(ctx->bodies, n, ctx->sort_wbits, ctx->sort_hbits,
                                          ctx->keys, ctx->vals, ctx->stream));
    uint32_t* sk = ctx->keys;
    uint32_t* sv = ctx->vals;
    P3M_CUDA(ctx, p3m::radix_sort_pairs(ctx->keys, ctx->vals, ctx->sort, n,
                                        ctx->sort_wbits + ctx->sort_hbits, ctx->stream, &sk, &sv));
    P3M_CUDA(ctx, p3m::launch_permute(sv, n, ctx->bodies, ctx->accel, ctx->materials,
                                      ctx->bodies_alt, ctx->accel_alt, ctx->materials_alt,
                                      ctx->destinations, ctx->stream));
    std::swap(ctx->bodies, ctx->bodies_alt);
    std::swap(ctx->accel, ctx->accel_alt);
    std::swap(ctx->materials, ctx->materials_alt);
    return P3M_OK;
}

int one_step(p3m_ctx* ctx, int n) {
    normalize_to(ctx, n);
    const int interval = ctx->cfg.spatial_sort_interval;
    if (interval > 0 && (ctx->physics_steps++ % interval) == 0) {
        int st = sort_bodies(ctx, n);
        if (st != P3M_OK) return st;
    }
    // Collision substeps drift the bodies: substep 0 half-kicks with the
    // stored acceleration (GravityPipeline.kt:465-473); the fused kernel also
    // writes the home-cell keys.
    const float dt = ctx->cfg.time_step;
    const float drift_dt = dt / (float)ctx->cfg.drift_substeps;
    P3M_CUDA(ctx, p3m::launch_drift(ctx->bodies, ctx->accel, n, 0.5f * dt, drift_dt,
                                    ctx->cfg.drift_substeps, ctx->grid, ctx->keys, ctx->vals,
                                    ctx->status, ctx->stream));
    if (ctx->mutual) {
        int st = lists_from_keys(ctx, n);
        if (st != P3M_OK) return st;
        st = mesh_force(ctx, n);
        if (st != P3M_OK) return st;
    }
    return apply_kick(ctx, n, 0);
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

}  // namespace

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
    if (e != cudaSuccess) {
        fail_cuda(nullptr, "cudaStreamCreate", e);
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
    ALLOC(ctx->status, 4);
    ALLOC(ctx->keys, cap);
    ALLOC(ctx->vals, cap);
    ALLOC(ctx->sort.keys_alt, cap);
    ALLOC(ctx->sort.vals_alt, cap);
    ALLOC(ctx->sort.hist, p3m::sort_hist_entries((int)cap));
    ALLOC(ctx->sort.block_sums, p3m::sort_block_sum_entries((int)cap));
    ALLOC(ctx->cell_start, P);
    ALLOC(ctx->cell_count, P);
    ALLOC(ctx->cell_mass, P);
    ALLOC(ctx->entries, cap);
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
#undef ALLOC

    auto init = [&]() -> int {
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
        P3M_CUDA(ctx, cudaMemsetAsync(ctx->cell_start, 0, P * sizeof(int), ctx->stream));
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
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->bodies, bodies4, (size_t)n * 16, cudaMemcpyHostToDevice, ctx->stream));
    if (materials4)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->materials, materials4, (size_t)n * 16, cudaMemcpyHostToDevice, ctx->stream));
    if (acceleration2)
        P3M_CUDA(ctx, cudaMemcpyAsync(ctx->accel, acceleration2, (size_t)n * 8, cudaMemcpyHostToDevice, ctx->stream));
    // Host arrays belong to the caller: finish reading them before returning.
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

int p3m_download_state(p3m_ctx* ctx, float* bodies4, float* materials4, float* acceleration2,
                       int32_t n) {
    int st = check_n(ctx, n);
    if (st != P3M_OK) return st;
    if (bodies4)
        P3M_CUDA(ctx, cudaMemcpyAsync(bodies4, ctx->bodies, (size_t)n * 16, cudaMemcpyDeviceToHost, ctx->stream));
    if (materials4)
        P3M_CUDA(ctx, cudaMemcpyAsync(materials4, ctx->materials, (size_t)n * 16, cudaMemcpyDeviceToHost, ctx->stream));
    if (acceleration2)
        P3M_CUDA(ctx, cudaMemcpyAsync(acceleration2, ctx->accel, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
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
    P3M_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return P3M_OK;
}

}  // extern "C"
