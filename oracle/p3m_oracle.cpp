// p3m_oracle.cpp — CPU restatement of Gravity's P3M gravity step.
//
// TEST INFRASTRUCTURE ONLY. This file is the oracle the CUDA library is
// checked against, and the CPU baseline that the benchmark times beside it.
// Nothing in the product (gravity_b200/) may link, load or call it.
//
// The reference runs this path as GLSL 4.30 compute shaders; it has no CPU
// implementation. Each function below restates one shader (or one piece of
// GravityPipeline.kt host logic) line by line and cites it. Paths are within
// the reference project:
//   S/ = src/main/resources/shaders/
//   K/ = src/main/kotlin/dev/gravity/
//
// Canonical choices where GLSL leaves the result to the implementation:
//   * Linked-list order: build_grid.comp pushes with atomicExchange, so the
//     list order depends on thread timing. Here bodies are pushed in
//     ascending ID order by one thread, so every list runs in DESCENDING ID
//     order (last pushed first).
//   * round(): ties to even (rintf).
//   * No floating-point contraction: built with -ffp-contract=off, so every
//     a*b+c rounds twice, exactly like separate GLSL multiply and add.
//   * Spatial reorder: a stable sort by Morton tile key (ties keep ascending
//     ID); the reference's scatter rank within a tile comes from an atomic
//     and is nondeterministic (S/spatial_sort_scatter.comp:21).
//   * GLSL exp/sin/cos are the C library's expf/sinf/cosf.
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/p3m.h"

namespace {

constexpr float kCellMassUnits = 256.0f;        // S/build_grid.comp:19
constexpr float kMaximumUnit = 0.99999994f;      // S/collision_build.comp:21
constexpr float kTau = 6.28318530717958647692f;  // S/twiddle_init.comp:9
constexpr float kPi = 3.14159265358979323846f;   // S/convolve.comp:14

struct f2 { float x, y; };
struct d2 { double x, y; };

inline f2 cmul(f2 a, f2 b) {  // S/fft_shared.comp:16-18, S/convolve.comp:16-18
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
inline float fractf(float v) { return v - std::floor(v); }  // GLSL fract
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }  // GLSL mix

int log2i(int v) { int b = 0; while ((1 << (b + 1)) <= v) ++b; return b; }
uint32_t reverse_bits(uint32_t v) {
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0f0f0f0fu) | ((v & 0x0f0f0f0fu) << 4);
    v = ((v >> 8) & 0x00ff00ffu) | ((v & 0x00ff00ffu) << 8);
    return (v >> 16) | (v << 16);
}

}  // namespace

extern "C" {

struct oracle_sim {
    p3m_config cfg;
    int capacity;
    int W, H;              // physical grid
    float aspect;          // viewport w / h
    int rx, ry;            // neighbour radii, K/GravityPipeline.kt:153-169
    int bounded;
    int mutual;
    float field_x, field_y;  // unit/s^2
    float mass_excess;
    float normalization_mass;
    long long physics_steps;
    std::vector<float> bodies, accel, materials;
    std::vector<uint32_t> destinations;
    std::vector<float> twiddles;            // vec4 per entry, S/twiddle_init.comp
    std::vector<f2> kernel_x, kernel_y;     // spectra
    std::vector<uint32_t> density;
    std::vector<int64_t> density64;
    std::vector<int> heads, next, counts;
    std::vector<uint32_t> cell_masses;
    std::vector<f2> fft, force_x, force_y;
    int mesh_w() const { return bounded ? 2 * W : W; }
    int mesh_h() const { return bounded ? 2 * H : H; }
};

void oracle_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ---------------------------------------------------------------------------
// S/spatial_sort_key.glsl:7-25 — Morton key of a sort tile.
static uint32_t spread_bits(uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

uint32_t oracle_morton_key(float x, float y, int wbits, int hbits) {
    int sw = 1 << wbits, sh = 1 << hbits;
    // ivec2(floor(position * vec2(size))) then clamp; a non-finite value
    // converts to some int and is clamped (GLSL leaves the value undefined;
    // here NaN maps to 0 and +-inf to the clamp limits).
    auto tile_of = [](float p, int size) {
        float f = std::floor(p * (float)size);
        int t;
        if (std::isnan(f)) t = 0;
        else if (f >= 2147483647.0f) t = 2147483647;
        else if (f <= -2147483648.0f) t = (int)0x80000000;
        else t = (int)f;
        return (uint32_t)std::min(std::max(t, 0), size - 1);
    };
    uint32_t tx = tile_of(x, sw), ty = tile_of(y, sh);
    int common = std::min(wbits, hbits);
    uint32_t low = (1u << common) - 1u;
    uint32_t morton = spread_bits(tx & low) | (spread_bits(ty & low) << 1);
    return morton | (((tx | ty) >> common) << (2 * common));
}

// K/GravityPipeline.kt:1649-1650 sortAxisBits: power-of-two tiles of ~4 px.
int oracle_sort_axis_bits(int extent) {
    int tiles = std::max(1, extent / 4);
    return std::min(10, log2i(tiles));
}

// ---------------------------------------------------------------------------
// Host scalars.

// K/GravityPipeline.kt:1546-1547
int oracle_mass_scale(float total_mass) {
    double v = 4000000000.0 / (double)total_mass;
    long long s = (long long)v;  // toLong truncates
    return (int)std::min(std::max(s, 1LL), 65536LL);
}

// K/GravityPipeline.kt:153-169 (Float arithmetic, as in Kotlin)
void oracle_neighbor_radii(const p3m_config* c, int* rx, int* ry) {
    float aspect = (float)c->viewport_width / (float)c->viewport_height;
    float vx = c->local_search_sigma_multiplier * c->softening_cells * (float)c->grid_width /
               ((float)c->grid_height * aspect);
    float vy = c->softening_cells * c->local_search_sigma_multiplier;
    int ix = (int)std::ceil(vx), iy = (int)std::ceil(vy);
    *rx = std::min(std::max(ix, c->minimum_neighbor_radius_cells), c->maximum_neighbor_radius_cells);
    *ry = std::min(std::max(iy, c->minimum_neighbor_radius_cells), c->maximum_neighbor_radius_cells);
}

// ---------------------------------------------------------------------------
// S/twiddle_init.comp:11-25 + K/GravityPipeline.kt:1359-1371: one table for
// every axis length; entries of half width h start at h - 1.
static void init_twiddles(std::vector<float>& tw, int max_axis) {
    tw.assign((size_t)std::max(1, max_axis - 1) * 4, 0.0f);
    for (int h = 1; h < max_axis; h *= 2) {
        for (int id = 0; id < h; ++id) {
            float fwd = -kTau * (float)id / (float)(h * 2);
            float inv = kTau * (float)id / (float)(h * 2);
            float* e = &tw[(size_t)(h - 1 + id) * 4];
            e[0] = std::cos(fwd); e[1] = std::sin(fwd);
            e[2] = std::cos(inv); e[3] = std::sin(inv);
        }
    }
}

// S/fft_shared.comp:26-81 — in-place radix-2 DIT complex FFT of every line of
// one axis; bit reversal folded into the load; inverse unscaled.
static void fft_axis_f32(f2* values, int width, int height, int axis, int inverse,
                         const float* tw) {
    const int axis_size = axis == 0 ? width : height;
    const int lines = axis == 0 ? height : width;
    const int bits = log2i(axis_size);
#pragma omp parallel
    {
        std::vector<f2> line(axis_size);
#pragma omp for schedule(static)
        for (int l = 0; l < lines; ++l) {
            auto gidx = [&](int coord) -> size_t {
                return axis == 0 ? (size_t)coord + (size_t)l * width
                                 : (size_t)l + (size_t)coord * width;
            };
            for (int c = 0; c < axis_size; ++c) {
                uint32_t src = bits ? reverse_bits((uint32_t)c) >> (32 - bits) : 0u;
                line[c] = values[gidx((int)src)];
            }
            for (int stage = 2; stage <= axis_size; stage <<= 1) {
                int half = stage >> 1;
                for (int b = 0; b < axis_size / 2; ++b) {
                    int within = b & (half - 1);
                    int lower = (b / half) * stage + within;
                    const float* t = &tw[(size_t)(half - 1 + within) * 4];
                    f2 w = inverse ? f2{t[2], t[3]} : f2{t[0], t[1]};
                    f2 lo = line[lower];
                    f2 up = cmul(w, line[lower + half]);
                    line[lower] = {lo.x + up.x, lo.y + up.y};
                    line[lower + half] = {lo.x - up.x, lo.y - up.y};
                }
            }
            for (int c = 0; c < axis_size; ++c) values[gidx(c)] = line[c];
        }
    }
}

// K/GravityPipeline.kt:1373-1386 transform(): rows, then columns.
static void transform_f32(f2* values, int w, int h, int inverse, const float* tw) {
    fft_axis_f32(values, w, h, 0, inverse, tw);
    fft_axis_f32(values, w, h, 1, inverse, tw);
}

// Stand-alone FP32 mirror transform (interleaved complex), with its own table.
void oracle_fft2d_f32(float* values, int width, int height, int inverse) {
    std::vector<float> tw;
    init_twiddles(tw, std::max(width, height));
    transform_f32(reinterpret_cast<f2*>(values), width, height, inverse, tw.data());
}

// FP64 radix-2 2D transform in the same layout (K/GravityPipeline.kt:1388-1436
// cpuFft2d): exact-angle twiddles in double.
void oracle_fft2d_f64(double* values, int width, int height, int inverse) {
    d2* v = reinterpret_cast<d2*>(values);
    for (int axis = 0; axis < 2; ++axis) {
        const int axis_size = axis == 0 ? width : height;
        const int lines = axis == 0 ? height : width;
        const int bits = log2i(axis_size);
#pragma omp parallel
        {
            std::vector<d2> line(axis_size);
#pragma omp for schedule(static)
            for (int l = 0; l < lines; ++l) {
                auto gidx = [&](int coord) -> size_t {
                    return axis == 0 ? (size_t)coord + (size_t)l * width
                                     : (size_t)l + (size_t)coord * width;
                };
                for (int c = 0; c < axis_size; ++c) {
                    uint32_t src = bits ? reverse_bits((uint32_t)c) >> (32 - bits) : 0u;
                    line[c] = v[gidx((int)src)];
                }
                for (int stage = 2; stage <= axis_size; stage <<= 1) {
                    int half = stage / 2;
                    double scale = (inverse ? 2.0 : -2.0) * M_PI / stage;
                    for (int base = 0; base < axis_size; base += stage) {
                        for (int k = 0; k < half; ++k) {
                            double wr = std::cos(scale * k), wi = std::sin(scale * k);
                            d2 up = line[base + k + half], lo = line[base + k];
                            double ur = up.x * wr - up.y * wi, ui = up.x * wi + up.y * wr;
                            line[base + k] = {lo.x + ur, lo.y + ui};
                            line[base + k + half] = {lo.x - ur, lo.y - ui};
                        }
                    }
                }
                for (int c = 0; c < axis_size; ++c) v[gidx(c)] = line[c];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// S/kernel_init.comp:16-46 — real-space long-range force kernel on the mesh.
static void kernel_init(oracle_sim* s) {
    const int gw = s->mesh_w(), gh = s->mesh_h();
    const float g = s->cfg.gravitational_constant;
    const float total = s->normalization_mass;
    const float sigma_cells = s->cfg.softening_cells;
    s->kernel_x.assign((size_t)gw * gh, f2{0, 0});
    s->kernel_y.assign((size_t)gw * gh, f2{0, 0});
#pragma omp parallel for schedule(static)
    for (long long id = 0; id < (long long)gw * gh; ++id) {
        int raw_x = (int)(id % gw), raw_y = (int)(id / gw);
        int off_x = raw_x <= gw / 2 ? raw_x : raw_x - gw;
        int off_y = raw_y <= gh / 2 ? raw_y : raw_y - gh;
        float dx = (float)off_x * s->aspect / (float)s->W;
        float dy = (float)off_y / (float)s->H;
        float r2 = dx * dx + dy * dy;
        if (r2 == 0.0f) continue;
        float sigma = sigma_cells / (float)s->H;
        float long_w = 1.0f - std::exp(-r2 / (2.0f * sigma * sigma));
        float dir_x = raw_x * 2 == gw ? 0.0f : dx;
        float dir_y = raw_y * 2 == gh ? 0.0f : dy;
        float scale = -g * long_w / (total * r2);
        s->kernel_x[id] = {scale * dir_x / s->aspect, 0.0f};
        s->kernel_y[id] = {scale * dir_y, 0.0f};
    }
}

// K/GravityPipeline.kt:1341-1357 initializeKernel: kernel_init + 2 forward FFTs.
static void initialize_kernel(oracle_sim* s) {
    kernel_init(s);
    transform_f32(s->kernel_x.data(), s->mesh_w(), s->mesh_h(), 0, s->twiddles.data());
    transform_f32(s->kernel_y.data(), s->mesh_w(), s->mesh_h(), 0, s->twiddles.data());
}

// K/GravityPipeline.kt:1326-1331 normalizeTo.
static void normalize_to(oracle_sim* s, int n) {
    float mass = std::max(1.0f, (float)n + s->mass_excess);
    if (mass == s->normalization_mass) return;
    s->normalization_mass = mass;
    initialize_kernel(s);
}

int oracle_validate(const p3m_config* c) {
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    if (!c) return P3M_ERR_INVALID_ARGUMENT;
    if (!pow2(c->grid_width) || !pow2(c->grid_height) || c->grid_width < 16 ||
        c->grid_height < 16 || c->grid_width > 4096 || c->grid_height > 4096)
        return P3M_ERR_UNSUPPORTED;
    if (c->bounded && 2 * std::max(c->grid_width, c->grid_height) > 4096) return P3M_ERR_UNSUPPORTED;
    if (c->viewport_width <= 0 || c->viewport_height <= 0 || c->capacity <= 0 ||
        c->drift_substeps <= 0 || c->spatial_sort_interval < 0)
        return P3M_ERR_INVALID_ARGUMENT;
    return P3M_OK;
}

oracle_sim* oracle_create(const p3m_config* c) {
    if (oracle_validate(c) != P3M_OK) return nullptr;
    oracle_sim* s = new oracle_sim();
    s->cfg = *c;
    s->capacity = c->capacity;
    s->W = c->grid_width;
    s->H = c->grid_height;
    s->aspect = (float)c->viewport_width / (float)c->viewport_height;
    oracle_neighbor_radii(c, &s->rx, &s->ry);
    s->bounded = c->bounded;
    s->mutual = c->mutual_gravity;
    s->field_x = s->field_y = 0.0f;
    s->mass_excess = 0.0f;
    s->normalization_mass = -1.0f;  // forces the first normalize_to to build
    s->physics_steps = 0;
    size_t cap = (size_t)c->capacity;
    s->bodies.assign(cap * 4, 0.0f);
    s->accel.assign(cap * 2, 0.0f);
    s->materials.assign(cap * 4, 0.0f);
    for (size_t i = 0; i < cap; ++i) s->materials[i * 4] = 1.0f;  // clearMaterials, :1493-1503
    s->destinations.assign(cap, 0u);
    // maximumFftAxis (K/GravityPipeline.kt:236-237): the largest mesh axis.
    int max_axis = std::max(s->W, s->H) * 2;
    init_twiddles(s->twiddles, max_axis);
    normalize_to(s, 0);
    return s;
}

void oracle_destroy(oracle_sim* s) { delete s; }

void oracle_set_bounded(oracle_sim* s, int b) {
    if (s->bounded == b) return;
    s->bounded = b;
    initialize_kernel(s);
}
void oracle_set_field(oracle_sim* s, float ax_px, float ay_px) {
    s->field_x = ax_px / (float)s->cfg.viewport_width;   // :1230-1234
    s->field_y = ay_px / (float)s->cfg.viewport_height;
}
void oracle_set_mutual_gravity(oracle_sim* s, int m) { s->mutual = m; }
void oracle_set_mass_excess(oracle_sim* s, float e) { s->mass_excess = e; }

void oracle_upload(oracle_sim* s, const float* b, const float* m, const float* a, int n) {
    if (b) std::memcpy(s->bodies.data(), b, (size_t)n * 16);
    if (m) std::memcpy(s->materials.data(), m, (size_t)n * 16);
    if (a) std::memcpy(s->accel.data(), a, (size_t)n * 8);
}
void oracle_download(oracle_sim* s, float* b, float* m, float* a, int n) {
    if (b) std::memcpy(b, s->bodies.data(), (size_t)n * 16);
    if (m) std::memcpy(m, s->materials.data(), (size_t)n * 16);
    if (a) std::memcpy(a, s->accel.data(), (size_t)n * 8);
}

// ---------------------------------------------------------------------------
// S/clear_grid.comp:12-20 + S/build_grid.comp:49-76 — CIC deposit and the
// home-cell linked lists.
// wrapCell / wrapMesh (S/build_grid.comp:21-37): one period added or
// subtracted, which covers every position in [0, 1]. Positions outside that
// range (caller input) are reduced modulo the size instead of indexing past
// the buffer, and a cell coordinate that offsets are added to is folded first
// when it lies so far out that the addition could overflow.
static inline int wrap1(int v, int size) {
    if (v < 0) v += size; else if (v >= size) v -= size;
    if ((unsigned)v >= (unsigned)size) { v %= size; if (v < 0) v += size; }
    return v;
}
static inline int guard(int v, int size) { return (v < -size || v > 2 * size) ? wrap1(v, size) : v; }
// floor()ed float to int as a GPU converts it: NaN -> 0, saturating.
static inline int f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int)0x80000000;
    return (int)f;
}
// uint(round(x)) / int64(round(x)) with round-half-even, saturating, NaN -> 0.
static inline uint32_t u32_rn(float x) {
    if (!(x > 0.0f)) return 0u;
    float r = std::nearbyint(x);
    return r >= 4294967295.0f ? 0xffffffffu : (uint32_t)r;
}
static inline int64_t i64_rn(float x) {
    if (x != x) return 0;
    float r = std::nearbyint(x);
    if (r >= 9.2233720368547758e18f) return INT64_MAX;
    if (r <= -9.2233720368547758e18f) return INT64_MIN;
    return (int64_t)r;
}

static void build_grid(oracle_sim* s, int n) {
    const int W = s->W, H = s->H, MW = s->mesh_w(), MH = s->mesh_h();
    const size_t M = (size_t)MW * MH, P = (size_t)W * H;
    const bool i64 = s->cfg.deposit_mode == P3M_DEPOSIT_I64;
    // clear_grid.comp
    if (i64) s->density64.assign(M, 0); else s->density.assign(M, 0u);
    s->heads.assign(P, -1);
    s->counts.assign(P, 0);
    s->cell_masses.assign(P, 0u);
    s->next.assign((size_t)std::max(n, 1), -1);
    const int mass_scale = oracle_mass_scale(s->normalization_mass);
    const float scale = (float)mass_scale;
    const float* bodies = s->bodies.data();
    const float* mats = s->materials.data();
    uint32_t* dens = s->density.data();
    int64_t* dens64 = s->density64.data();
    // Deposit: integer atomics commute, so a parallel loop gives the same grid.
#pragma omp parallel for schedule(static)
    for (int id = 0; id < n; ++id) {
        float px = bodies[(size_t)id * 4], py = bodies[(size_t)id * 4 + 1];
        float mass = mats[(size_t)id * 4];
        float gx = px * (float)W - 0.5f, gy = py * (float)H - 0.5f;
        float flx = std::floor(gx), fly = std::floor(gy);
        int bx = guard(f2i(flx), MW), by = guard(f2i(fly), MH);
        float fx = gx - flx, fy = gy - fly;  // fract
        float w[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
        for (int k = 0; k < 4; ++k) w[k] *= mass;
        const int ox[4] = {0, 1, 0, 1}, oy[4] = {0, 0, 1, 1};
        for (int k = 0; k < 4; ++k) {
            int mx = wrap1(bx + ox[k], MW), my = wrap1(by + oy[k], MH);
            size_t idx = (size_t)mx + (size_t)my * MW;
            if (i64) {
                // Precision form: 2^-32 mass quanta in int64.
                int64_t q = i64_rn(w[k] * 4294967296.0f);
#pragma omp atomic
                dens64[idx] += q;
            } else {
                uint32_t q = u32_rn(w[k] * scale);
#pragma omp atomic
                dens[idx] += q;
            }
        }
    }
    // Lists: one thread, ascending ID, so each list runs in descending ID.
    for (int id = 0; id < n; ++id) {
        float px = bodies[(size_t)id * 4], py = bodies[(size_t)id * 4 + 1];
        int hx = wrap1(f2i(std::floor(px * (float)W)), W), hy = wrap1(f2i(std::floor(py * (float)H)), H);
        size_t home = (size_t)hx + (size_t)hy * W;
        s->next[id] = s->heads[home];
        s->heads[home] = id;
        s->counts[home] += 1;
        s->cell_masses[home] += u32_rn(mats[(size_t)id * 4] * kCellMassUnits);
    }
}

// S/fft_init.comp:11-17 — fixed point to complex.
static void fft_init(oracle_sim* s) {
    const size_t M = (size_t)s->mesh_w() * s->mesh_h();
    s->fft.assign(M, f2{0, 0});
    if (s->cfg.deposit_mode == P3M_DEPOSIT_I64) {
        const float inv = 1.0f / 4294967296.0f;
        for (size_t i = 0; i < M; ++i) s->fft[i] = {(float)s->density64[i] * inv, 0.0f};
    } else {
        const float inv = 1.0f / (float)oracle_mass_scale(s->normalization_mass);
        for (size_t i = 0; i < M; ++i) s->fft[i] = {(float)s->density[i] * inv, 0.0f};
    }
}

// S/convolve.comp:24-47 — spectral multiply with CIC deconvolution.
static float sincf(float v) { return std::fabs(v) < 1e-6f ? 1.0f : std::sin(v) / v; }

static void convolve(oracle_sim* s) {
    const int gw = s->mesh_w(), gh = s->mesh_h();
    const float floor_power = s->cfg.minimum_assignment_window_power;
    s->force_x.assign((size_t)gw * gh, f2{0, 0});
    s->force_y.assign((size_t)gw * gh, f2{0, 0});
#pragma omp parallel for schedule(static)
    for (long long id = 0; id < (long long)gw * gh; ++id) {
        int raw_x = (int)(id % gw), raw_y = (int)(id / gw);
        int kx = raw_x <= gw / 2 ? raw_x : raw_x - gw;
        int ky = raw_y <= gh / 2 ? raw_y : raw_y - gh;
        float sx = sincf(kPi * (float)kx / (float)gw);
        float sy = sincf(kPi * (float)ky / (float)gh);
        float window = sx * sx * sy * sy;
        float deconv = 1.0f / std::max(window * window, floor_power);
        float inv_size = 1.0f / (float)(gw * gh);
        float scale = deconv * inv_size;
        f2 rho = s->fft[id];
        f2 a = cmul(rho, s->kernel_x[id]), b = cmul(rho, s->kernel_y[id]);
        s->force_x[id] = {a.x * scale, a.y * scale};
        s->force_y[id] = {b.x * scale, b.y * scale};
    }
}

// K/GravityPipeline.kt:907-973 buildForce.
static void build_force(oracle_sim* s, int n) {
    build_grid(s, n);
    fft_init(s);
    transform_f32(s->fft.data(), s->mesh_w(), s->mesh_h(), 0, s->twiddles.data());
    convolve(s);
    transform_f32(s->force_x.data(), s->mesh_w(), s->mesh_h(), 1, s->twiddles.data());
    transform_f32(s->force_y.data(), s->mesh_w(), s->mesh_h(), 1, s->twiddles.data());
}

// ---------------------------------------------------------------------------
// S/kick.comp:66-80 localAcceleration.
struct KickParams {
    int W, H, MW, MH, bounded, rx, ry, exact, home_limit, initial, mutual;
    float aspect, g, sigma_cells, total, min_frac, dt, field_x, field_y;
};

static inline f2 local_acceleration(const KickParams& k, f2 src, f2 tgt, float m) {
    float dx = src.x - tgt.x, dy = src.y - tgt.y;
    if (k.bounded == 0) {
        dx -= std::floor(dx + 0.5f);
        dy -= std::floor(dy + 0.5f);
    }
    float px = dx * k.aspect, py = dy * 1.0f;
    float r2 = px * px + py * py;
    float sigma = k.sigma_cells / (float)k.H;
    float local_w = std::exp(-r2 / (2.0f * sigma * sigma));
    float cw = k.aspect / (float)k.W, ch = 1.0f / (float)k.H;
    float md = k.min_frac * std::min(cw, ch);
    float phys = k.g * m * local_w / (k.total * std::max(r2, md * md));
    return {phys * px / k.aspect, phys * py / 1.0f};
}

// S/kick.comp:82-103 interpolateForce (force meshes hold complex values; the
// real part is the force).
static inline f2 interpolate_force(const KickParams& k, const f2* fx, const f2* fy, f2 p) {
    float gx = p.x * (float)k.W - 0.5f, gy = p.y * (float)k.H - 0.5f;
    float flx = std::floor(gx), fly = std::floor(gy);
    int bx = guard(f2i(flx), k.MW), by = guard(f2i(fly), k.MH);
    float tx = gx - flx, ty = gy - fly;
    auto at = [&](int ox, int oy) {
        int mx = wrap1(bx + ox, k.MW), my = wrap1(by + oy, k.MH);
        size_t i = (size_t)mx + (size_t)my * k.MW;
        return f2{fx[i].x, fy[i].x};
    };
    f2 v00 = at(0, 0), v10 = at(1, 0), v01 = at(0, 1), v11 = at(1, 1);
    f2 a = {mixf(v00.x, v10.x, tx), mixf(v00.y, v10.y, tx)};
    f2 b = {mixf(v01.x, v11.x, tx), mixf(v01.y, v11.y, tx)};
    return {mixf(a.x, b.x, ty), mixf(a.y, b.y, ty)};
}

// S/kick.comp:105-156 main (every body awake: sleep is not on this path).
static void apply_kick(oracle_sim* s, int n, int initial) {
    KickParams k;
    k.W = s->W; k.H = s->H; k.MW = s->mesh_w(); k.MH = s->mesh_h();
    k.bounded = s->bounded; k.rx = s->rx; k.ry = s->ry;
    k.exact = s->cfg.exact_neighbor_body_limit;
    k.home_limit = s->cfg.maximum_home_body_interactions;
    k.initial = initial; k.mutual = s->mutual;
    k.aspect = s->aspect; k.g = s->cfg.gravitational_constant;
    k.sigma_cells = s->cfg.softening_cells; k.total = s->normalization_mass;
    k.min_frac = s->cfg.minimum_distance_cell_fraction; k.dt = s->cfg.time_step;
    k.field_x = s->field_x; k.field_y = s->field_y;
    float* bodies = s->bodies.data();
    float* acc = s->accel.data();
    const float* mats = s->materials.data();
    const f2* fxm = s->force_x.data();
    const f2* fym = s->force_y.data();
    const int* heads = s->heads.data();
    const int* next = s->next.data();
    const int* counts = s->counts.data();
    const uint32_t* cmass = s->cell_masses.data();
#pragma omp parallel for schedule(dynamic, 256)
    for (int id = 0; id < n; ++id) {
        float* body = &bodies[(size_t)id * 4];
        if (k.mutual == 0) {
            if (initial == 0) {
                body[2] += k.field_x * (0.5f * k.dt);
                body[3] += k.field_y * (0.5f * k.dt);
            }
            acc[(size_t)id * 2] = k.field_x;
            acc[(size_t)id * 2 + 1] = k.field_y;
            continue;
        }
        f2 p = {body[0], body[1]};
        f2 interp = interpolate_force(k, fxm, fym, p);
        f2 r = {interp.x + k.field_x, interp.y + k.field_y};
        int hx = guard(f2i(std::floor(p.x * (float)k.W)), k.W), hy = guard(f2i(std::floor(p.y * (float)k.H)), k.H);
        for (int dy = -k.ry; dy <= k.ry; ++dy) {
            for (int dx = -k.rx; dx <= k.rx; ++dx) {
                int cx = hx + dx, cy = hy + dy;
                if (k.bounded != 0 && (cx < 0 || cy < 0 || cx >= k.W || cy >= k.H)) continue;
                int wx = wrap1(cx, k.W), wy = wrap1(cy, k.H);
                int index = wx + wy * k.W;
                int count = counts[index];
                bool home = dx == 0 && dy == 0;
                f2 a;
                if (!home && count > k.exact) {
                    f2 center = {((float)wx + 0.5f) / (float)k.W, ((float)wy + 0.5f) / (float)k.H};
                    float agg = (float)cmass[index] / kCellMassUnits;
                    a = local_acceleration(k, center, p, agg);
                    r.x += a.x; r.y += a.y;
                } else {
                    int other = heads[index];
                    int visited = 0;
                    int limit = home ? k.home_limit : k.exact;
                    while (other >= 0 && visited < limit) {
                        if (other != id) {
                            f2 sp = {bodies[(size_t)other * 4], bodies[(size_t)other * 4 + 1]};
                            a = local_acceleration(k, sp, p, mats[(size_t)other * 4]);
                            r.x += a.x; r.y += a.y;
                        }
                        other = next[other];
                        visited++;
                    }
                }
            }
        }
        if (initial == 0) {
            body[2] += r.x * (0.5f * k.dt);
            body[3] += r.y * (0.5f * k.dt);
        }
        acc[(size_t)id * 2] = r.x;
        acc[(size_t)id * 2 + 1] = r.y;
    }
}

// The kick reads the velocity it updates but positions of other bodies only,
// and the loop above writes only body[2..3] and acc: positions stay fixed, so
// the parallel loop equals the shader's one-pass semantics.

// ---------------------------------------------------------------------------
// S/collision_build.comp:40-51 — the drift part of a collision substep.
void oracle_drift_raw(float* bodies, const float* acc, int n, float kick_dt, float drift_dt,
                      int bounded) {
    if (!(kick_dt != 0.0f || drift_dt != 0.0f)) return;
#pragma omp parallel for schedule(static)
    for (int id = 0; id < n; ++id) {
        float* b = &bodies[(size_t)id * 4];
        b[2] += acc[(size_t)id * 2] * (0.5f * kick_dt);
        b[3] += acc[(size_t)id * 2 + 1] * (0.5f * kick_dt);
        b[0] += b[2] * drift_dt;
        b[1] += b[3] * drift_dt;
        if (bounded) {
            b[0] = std::min(std::max(b[0], 0.0f), kMaximumUnit);
            b[1] = std::min(std::max(b[1], 0.0f), kMaximumUnit);
        } else {
            b[0] = fractf(b[0]);
            b[1] = fractf(b[1]);
        }
    }
}

void oracle_drift(oracle_sim* s, int n, float kick_dt, float drift_dt) {
    oracle_drift_raw(s->bodies.data(), s->accel.data(), n, kick_dt, drift_dt, s->bounded);
}

// ---------------------------------------------------------------------------
// K/GravityPipeline.kt:1269-1319 sortBodies + S/spatial_sort_*.comp: a pure
// permutation of bodies, accelerations and materials along the Morton key.
void oracle_sort_bodies(oracle_sim* s, int n) {
    int wb = oracle_sort_axis_bits(s->cfg.viewport_width);
    int hb = oracle_sort_axis_bits(s->cfg.viewport_height);
    std::vector<uint32_t> key(n);
    for (int i = 0; i < n; ++i)
        key[i] = oracle_morton_key(s->bodies[(size_t)i * 4], s->bodies[(size_t)i * 4 + 1], wb, hb);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<float> nb((size_t)n * 4), na((size_t)n * 2), nm((size_t)n * 4);
    for (int t = 0; t < n; ++t) {
        int src = order[t];
        std::memcpy(&nb[(size_t)t * 4], &s->bodies[(size_t)src * 4], 16);
        std::memcpy(&na[(size_t)t * 2], &s->accel[(size_t)src * 2], 8);
        std::memcpy(&nm[(size_t)t * 4], &s->materials[(size_t)src * 4], 16);
        s->destinations[src] = (uint32_t)t;
    }
    std::memcpy(s->bodies.data(), nb.data(), nb.size() * 4);
    std::memcpy(s->accel.data(), na.data(), na.size() * 4);
    std::memcpy(s->materials.data(), nm.data(), nm.size() * 4);
}

// ---------------------------------------------------------------------------
// Orchestration: K/GravityPipeline.kt:366-370 and :445-494 without the
// collision contacts, liquid, sleep and block bookkeeping.
void oracle_build_force(oracle_sim* s, int n) { build_force(s, n); }
void oracle_apply_kick(oracle_sim* s, int n, int initial) { apply_kick(s, n, initial); }
void oracle_build_grid(oracle_sim* s, int n) { build_grid(s, n); }

void oracle_initialize_acceleration(oracle_sim* s, int n) {
    normalize_to(s, n);
    if (s->mutual) build_force(s, n);
    apply_kick(s, n, 1);
}

void oracle_step(oracle_sim* s, int n, int steps) {
    for (int it = 0; it < steps; ++it) {
        normalize_to(s, n);
        int interval = s->cfg.spatial_sort_interval;
        if (interval > 0 && (s->physics_steps++ % interval) == 0) oracle_sort_bodies(s, n);
        const int sub = s->cfg.drift_substeps;
        const float drift_dt = s->cfg.time_step / (float)sub;
        for (int k = 0; k < sub; ++k)
            oracle_drift(s, n, k == 0 ? s->cfg.time_step : 0.0f, drift_dt);
        if (s->mutual) build_force(s, n);
        apply_kick(s, n, 0);
        // The final zero-drift collision pass (kickDt = driftDt = 0) leaves
        // gravity-only bodies unchanged (S/collision_build.comp:43).
    }
}

// ---------------------------------------------------------------------------
// S/trajectory.comp (one preview, the shader's one thread) and the host
// placement of K/GravityPipeline.kt:514-600, 773-779.

static inline f2 traj_local(const KickParams& k, f2 src, f2 tgt, float m) {
    return local_acceleration(k, src, tgt, m);  // S/trajectory.comp:78-95 == S/kick.comp:66-80
}

static f2 traj_acceleration(const oracle_sim* s, const KickParams& k, f2 p) {
    if (k.mutual == 0) return {k.field_x, k.field_y};
    f2 interp = interpolate_force(k, s->force_x.data(), s->force_y.data(), p);
    f2 r = {interp.x + k.field_x, interp.y + k.field_y};
    int hx = f2i(std::floor(p.x * (float)k.W)), hy = f2i(std::floor(p.y * (float)k.H));
    for (int dy = -k.ry; dy <= k.ry; ++dy) {
        for (int dx = -k.rx; dx <= k.rx; ++dx) {
            int cx = hx + dx, cy = hy + dy;
            if (k.bounded != 0 && (cx < 0 || cy < 0 || cx >= k.W || cy >= k.H)) continue;
            int wx = wrap1(cx, k.W), wy = wrap1(cy, k.H);
            int index = wx + wy * k.W;
            int count = s->counts[index];
            bool home = dx == 0 && dy == 0;
            if (!home && count > k.exact) {
                f2 center = {((float)wx + 0.5f) / (float)k.W, ((float)wy + 0.5f) / (float)k.H};
                f2 a = traj_local(k, center, p, (float)s->cell_masses[index] / kCellMassUnits);
                r.x += a.x; r.y += a.y;
            } else {
                int other = s->heads[index];
                int visited = 0;
                int limit = home ? k.home_limit : k.exact;
                while (other >= 0 && visited < limit) {
                    f2 sp = {s->bodies[(size_t)other * 4], s->bodies[(size_t)other * 4 + 1]};
                    f2 a = traj_local(k, sp, p, s->materials[(size_t)other * 4]);
                    r.x += a.x; r.y += a.y;
                    other = s->next[other];
                    visited++;
                }
            }
        }
    }
    return r;
}

static void traj_emit(float* out, int step, f2 start, f2 delta, float sd, float dist, float sdc,
                      float dc) {
    float* v = out + (size_t)step * 6 * 4;
    for (int i = 0; i < 6; ++i) { v[4 * i] = 0; v[4 * i + 1] = 0; v[4 * i + 2] = 0; v[4 * i + 3] = -1; }
    f2 end = {start.x + delta.x, start.y + delta.y};
    float cuts[4];
    int cut_count = 2;
    cuts[0] = 0.0f; cuts[1] = 1.0f;
    if (end.x < 0.0f) cuts[cut_count++] = -start.x / delta.x;
    else if (end.x >= 1.0f) cuts[cut_count++] = (1.0f - start.x) / delta.x;
    if (end.y < 0.0f) cuts[cut_count++] = -start.y / delta.y;
    else if (end.y >= 1.0f) cuts[cut_count++] = (1.0f - start.y) / delta.y;
    for (int index = 1; index < cut_count; ++index) {
        float value = std::min(std::max(cuts[index], 0.0f), 1.0f);
        int ins = index;
        while (ins > 0 && cuts[ins - 1] > value) { cuts[ins] = cuts[ins - 1]; ins--; }
        cuts[ins] = value;
    }
    float uniq[4];
    int uc = 0;
    for (int index = 0; index < cut_count; ++index)
        if (uc == 0 || std::fabs(cuts[index] - uniq[uc - 1]) > 1e-6f) uniq[uc++] = cuts[index];
    for (int piece = 0; piece < uc - 1; ++piece) {
        float f0 = uniq[piece], f1 = uniq[piece + 1];
        float mid = 0.5f * (f0 + f1);
        float tx = std::floor(start.x + delta.x * mid), ty = std::floor(start.y + delta.y * mid);
        float* q = v + piece * 2 * 4;
        q[0] = std::min(std::max(start.x + delta.x * f0 - tx, 0.0f), 1.0f);
        q[1] = std::min(std::max(start.y + delta.y * f0 - ty, 0.0f), 1.0f);
        q[2] = sdc + dc * f0;
        q[3] = sd + dist * f0;
        q[4] = std::min(std::max(start.x + delta.x * f1 - tx, 0.0f), 1.0f);
        q[5] = std::min(std::max(start.y + delta.y * f1 - ty, 0.0f), 1.0f);
        q[6] = sdc + dc * f1;
        q[7] = sd + dist * f1;
    }
}

// params: steps, max_dt, target_segment_px, path_diagonals, min_dash_px,
// restitution. out: steps * 6 vec4.
void oracle_trajectory(oracle_sim* s, int n, const float* params, float origin_x_px,
                       float origin_y_px, float vx_px, float vy_px, float* out) {
    normalize_to(s, n);
    KickParams k;
    k.W = s->W; k.H = s->H; k.MW = s->mesh_w(); k.MH = s->mesh_h();
    k.bounded = s->bounded; k.rx = s->rx; k.ry = s->ry;
    k.exact = s->cfg.exact_neighbor_body_limit;
    k.home_limit = s->cfg.maximum_home_body_interactions;
    k.initial = 0; k.mutual = s->mutual;
    k.aspect = s->aspect; k.g = s->cfg.gravitational_constant;
    k.sigma_cells = s->cfg.softening_cells; k.total = s->normalization_mass;
    k.min_frac = s->cfg.minimum_distance_cell_fraction; k.dt = s->cfg.time_step;
    k.field_x = s->field_x; k.field_y = s->field_y;
    const int steps = (int)params[0];
    const float max_dt = params[1], target = params[2], diagonals = params[3];
    const float min_dash = params[4], restitution = params[5];
    const float vw = (float)s->cfg.viewport_width, vh = (float)s->cfg.viewport_height;
    const float max_path = diagonals * std::sqrt(vw * vw + vh * vh);
    const float min_dt = s->cfg.time_step;
    // placeX / placeY, then S/trajectory.comp:262-329.
    float ox, oy;
    if (s->bounded) {
        ox = std::min(std::max(origin_x_px, 0.0f), vw * kMaximumUnit);
        oy = std::min(std::max(origin_y_px, 0.0f), vh * kMaximumUnit);
    } else {
        ox = origin_x_px - std::floor(origin_x_px / vw) * vw;
        oy = origin_y_px - std::floor(origin_y_px / vh) * vh;
    }
    f2 pos = {ox / vw, oy / vh}, vel = {vx_px / vw, vy_px / vh};
    f2 acc = traj_acceleration(s, k, pos);
    float path = 0.0f, dash = 0.0f;
    bool finished = false;
    for (int step = 0; step < steps; ++step) {
        if (finished) {
            float* v = out + (size_t)step * 24;
            for (int i = 0; i < 6; ++i) { v[4 * i] = 0; v[4 * i + 1] = 0; v[4 * i + 2] = 0; v[4 * i + 3] = -1; }
            continue;
        }
        float sp = std::sqrt((vel.x * vw) * (vel.x * vw) + (vel.y * vh) * (vel.y * vh));
        float ap = std::sqrt((acc.x * vw) * (acc.x * vw) + (acc.y * vh) * (acc.y * vh));
        float dt;
        if (ap > 1e-5f) dt = (std::sqrt(sp * sp + 2.0f * ap * target) - sp) / ap;
        else dt = target / std::max(sp, 1e-5f);
        dt = std::min(std::max(dt, min_dt), max_dt);
        f2 half = {vel.x + acc.x * (0.5f * dt), vel.y + acc.y * (0.5f * dt)};
        f2 delta = {half.x * dt, half.y * dt};
        if (s->bounded) {
            float nx = pos.x + delta.x, ny = pos.y + delta.y;
            float cx = std::min(std::max(nx, 0.0f), kMaximumUnit), cy = std::min(std::max(ny, 0.0f), kMaximumUnit);
            if (nx != cx) half.x = -restitution * half.x;
            if (ny != cy) half.y = -restitution * half.y;
            delta = {cx - pos.x, cy - pos.y};
        }
        float step_px = std::sqrt((delta.x * vw) * (delta.x * vw) + (delta.y * vh) * (delta.y * vh));
        float remaining = max_path - path;
        if (step_px > remaining) {
            delta.x *= remaining / step_px;
            delta.y *= remaining / step_px;
            step_px = remaining;
            finished = true;
        }
        float mult = 1.0f + std::sqrt(half.x * half.x + half.y * half.y);
        float dash_len = min_dash * mult;
        float step_dash = step_px * min_dash / dash_len;
        traj_emit(out, step, pos, delta, path, step_px, dash, step_dash);
        path += step_px;
        dash += step_dash;
        if (s->bounded) pos = {pos.x + delta.x, pos.y + delta.y};
        else pos = {fractf(pos.x + delta.x), fractf(pos.y + delta.y)};
        if (path >= max_path - 1e-4f) { finished = true; continue; }
        acc = traj_acceleration(s, k, pos);
        vel = {half.x + acc.x * (0.5f * dt), half.y + acc.y * (0.5f * dt)};
    }
    float inv = 1.0f / std::max(path, 1e-6f);
    for (int v = 0; v < steps * 6; ++v) {
        float& w = out[(size_t)v * 4 + 3];
        if (w >= 0.0f) w = std::min(std::max(w * inv, 0.0f), 1.0f);
    }
}

// ---------------------------------------------------------------------------
// Readback of intermediate buffers, in the library's layouts.

int oracle_normalization(oracle_sim* s, float* total_mass, int* mass_scale) {
    *total_mass = s->normalization_mass;
    *mass_scale = oracle_mass_scale(s->normalization_mass);
    return 0;
}

void oracle_radii(oracle_sim* s, int* rx, int* ry) { *rx = s->rx; *ry = s->ry; }

// Cell lists as CSR: each cell's list in walk order, cells ascending.
void oracle_cell_lists(oracle_sim* s, int n, uint32_t* keys, int* bodies_sorted, int* start,
                       int* count, uint32_t* mass) {
    const int P = s->W * s->H;
    int pos = 0;
    for (int c = 0; c < P; ++c) {
        start[c] = s->counts[c] > 0 ? pos : 0;
        count[c] = s->counts[c];
        mass[c] = s->cell_masses[c];
        for (int o = s->heads[c]; o >= 0; o = s->next[o]) {
            keys[pos] = (uint32_t)c;
            bodies_sorted[pos++] = o;
        }
    }
    (void)n;
}

void oracle_density_u32(oracle_sim* s, uint32_t* out) {
    std::memcpy(out, s->density.data(), s->density.size() * 4);
}
void oracle_density_i64(oracle_sim* s, int64_t* out) {
    std::memcpy(out, s->density64.data(), s->density64.size() * 8);
}
// Real parts of the inverse-transformed force meshes, interleaved (fx, fy).
void oracle_force(oracle_sim* s, float* out) {
    size_t M = s->force_x.size();
    for (size_t i = 0; i < M; ++i) {
        out[i * 2] = s->force_x[i].x;
        out[i * 2 + 1] = s->force_y[i].x;
    }
}
// Density spectrum after the forward transform (interleaved complex, M bins).
void oracle_density_spectrum(oracle_sim* s, float* out) {
    std::memcpy(out, s->fft.data(), s->fft.size() * 8);
}
void oracle_kernel_spectra(oracle_sim* s, float* kx, float* ky) {
    std::memcpy(kx, s->kernel_x.data(), s->kernel_x.size() * 8);
    std::memcpy(ky, s->kernel_y.data(), s->kernel_y.size() * 8);
}
void oracle_destinations(oracle_sim* s, uint32_t* out, int n) {
    std::memcpy(out, s->destinations.data(), (size_t)n * 4);
}

// ---------------------------------------------------------------------------
// FP64 direct sum: the law the P3M split approximates, summed over every
// source for a subsample of targets (S/kick.comp:66-80 with the Gaussian
// split removed, i.e. long + short = G m d / (M max(r^2, r_min^2))).
// Torus: minimum image, the displacement the periodic mesh kernel uses
// (S/kernel_init.comp:22-28); walls: the open sum.
void oracle_direct_sum_f64(const float* bodies4, const float* materials4, int n,
                           const int* targets, int n_targets, const p3m_config* c,
                           float total_mass, int bounded, double* out2) {
    const double aspect = (double)c->viewport_width / (double)c->viewport_height;
    const double cw = aspect / c->grid_width, ch = 1.0 / c->grid_height;
    const double md = (double)c->minimum_distance_cell_fraction * std::min(cw, ch);
    const double md2 = md * md;
    const double g = c->gravitational_constant;
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < n_targets; ++t) {
        const int id = targets[t];
        const double tx = bodies4[(size_t)id * 4], ty = bodies4[(size_t)id * 4 + 1];
        double ax = 0.0, ay = 0.0;
        for (int j = 0; j < n; ++j) {
            if (j == id) continue;
            double dx = bodies4[(size_t)j * 4] - tx, dy = bodies4[(size_t)j * 4 + 1] - ty;
            if (!bounded) {
                dx -= std::floor(dx + 0.5);
                dy -= std::floor(dy + 0.5);
            }
            double px = dx * aspect, py = dy;
            double r2 = px * px + py * py;
            double s = g * materials4[(size_t)j * 4] / ((double)total_mass * std::max(r2, md2));
            ax += s * px;
            ay += s * py;
        }
        out2[(size_t)t * 2] = ax / aspect;
        out2[(size_t)t * 2 + 1] = ay;
    }
}

}  // extern "C"
