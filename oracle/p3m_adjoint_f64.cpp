// p3m_adjoint_f64.cpp — FP64 reference model of the differentiated P3M
// rollout: forward and hand-written adjoint.
//
// TEST INFRASTRUCTURE ONLY. The CUDA adjoint is checked against this file (and
// this file against central finite differences of its own forward). Nothing
// in the product may link, load or call it.
//
// The reference has no adjoint; what is differentiated is its gravity-only
// step (K/GravityPipeline.kt:445-494 without collisions, no spatial reorder)
// on the torus, as the continuous model behind the FP32 shaders:
//   S/collision_build.comp:40-51   v_h = v + a dt/2, x' = fract(x + v_h dt)
//                                  (the substeps after the first kick 0)
//   S/build_grid.comp              CIC deposit rho(c) = sum_j m_j w_j(c)
//                                  (here in FP64, not fixed point), cell lists
//   S/kernel_init.comp:16-46,      E = real(IFFT(FFT(rho) K^ deconv / size))
//   S/convolve.comp:24-47
//   S/kick.comp:66-156             a = interp(E, x) + field + short range
//                                  (exact pairs / monopoles as listed)
//                                  v' = v_h + a' dt/2
// Paths: S/ = src/main/resources/shaders/, K/ = src/main/kotlin/dev/gravity/.
//
// The cell topology (which cells are monopoles, which list entries are
// summed) is piecewise constant in the positions and is held fixed when
// differentiating; the mesh transpose uses the conjugate spectrum (the exact
// transpose of a real circulant), independently of the antisymmetry of the
// gradient kernels that the CUDA adjoint uses.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/p3m.h"

extern "C" {
void oracle_fft2d_f64(double* values, int width, int height, int inverse);
void oracle_neighbor_radii(const p3m_config* c, int* rx, int* ry);
}

namespace {

struct c64 { double re, im; };

struct Lists {
    std::vector<int> head, next, count;
    std::vector<double> cell_mass;
};

struct adj64 {
    p3m_config cfg{};
    int n = 0, W = 0, H = 0, rx = 1, ry = 1, exact = 2, home_limit = 8, initial_accel = 1;
    double aspect = 1, g = 1, sigma = 1, min_d2 = 0, total = 1, dt = 0, field_x = 0, field_y = 0;
    std::vector<c64> kx_hat, ky_hat;       // spectra x deconvolution / size
    std::vector<double> mass;              // per body
    std::vector<std::vector<double>> xs;   // positions (n x 2) at every step
    std::vector<double> v, a;              // final velocity and acceleration
    int steps = 0;
};

inline int wrapi(long long v, int size) {
    long long r = v % size;
    return (int)(r < 0 ? r + size : r);
}

double sincd(double v) { return std::fabs(v) < 1e-12 ? 1.0 : std::sin(v) / v; }

// S/kernel_init.comp:16-46 in FP64, FFT'd, times the CIC deconvolution and
// 1/size of S/convolve.comp:24-47.
void build_spectra(adj64* s) {
    const int W = s->W, H = s->H;
    const size_t P = (size_t)W * H;
    std::vector<double> zx(2 * P, 0.0), zy(2 * P, 0.0);
    for (size_t id = 0; id < P; ++id) {
        const int raw_x = (int)(id % W), raw_y = (int)(id / W);
        const int off_x = raw_x <= W / 2 ? raw_x : raw_x - W;
        const int off_y = raw_y <= H / 2 ? raw_y : raw_y - H;
        const double dx = (double)off_x * s->aspect / W, dy = (double)off_y / H;
        const double r2 = dx * dx + dy * dy;
        if (r2 == 0.0) continue;
        const double long_w = 1.0 - std::exp(-r2 / (2.0 * s->sigma * s->sigma));
        const double dir_x = raw_x * 2 == W ? 0.0 : dx;
        const double dir_y = raw_y * 2 == H ? 0.0 : dy;
        const double scale = -s->g * long_w / (s->total * r2);
        zx[2 * id] = scale * dir_x / s->aspect;
        zy[2 * id] = scale * dir_y;
    }
    oracle_fft2d_f64(zx.data(), W, H, 0);
    oracle_fft2d_f64(zy.data(), W, H, 0);
    s->kx_hat.resize(P);
    s->ky_hat.resize(P);
    const double floor_power = s->cfg.minimum_assignment_window_power;
    for (size_t id = 0; id < P; ++id) {
        const int raw_x = (int)(id % W), raw_y = (int)(id / W);
        const int kx = raw_x <= W / 2 ? raw_x : raw_x - W;
        const int ky = raw_y <= H / 2 ? raw_y : raw_y - H;
        const double sx = sincd(M_PI * kx / W), sy = sincd(M_PI * ky / H);
        const double window = sx * sx * sy * sy;
        const double f = 1.0 / std::max(window * window, floor_power) / (double)P;
        s->kx_hat[id] = {zx[2 * id] * f, zx[2 * id + 1] * f};
        s->ky_hat[id] = {zy[2 * id] * f, zy[2 * id + 1] * f};
    }
}

// Cell lists: bodies pushed in ascending ID, so each list runs in
// descending ID (the canonical order of the CUDA lists).
void build_lists(const adj64* s, const double* x, Lists& L) {
    const size_t P = (size_t)s->W * s->H;
    L.head.assign(P, -1);
    L.next.assign(s->n, -1);
    L.count.assign(P, 0);
    L.cell_mass.assign(P, 0.0);
    for (int i = 0; i < s->n; ++i) {
        const int hx = wrapi((long long)std::floor(x[2 * i] * s->W), s->W);
        const int hy = wrapi((long long)std::floor(x[2 * i + 1] * s->H), s->H);
        const size_t c = (size_t)hy * s->W + hx;
        L.next[i] = L.head[c];
        L.head[c] = i;
        L.count[c] += 1;
        // Fixed-point cell mass units of S/build_grid.comp:19.
        L.cell_mass[c] += std::nearbyint(s->mass[i] * 256.0) / 256.0;
    }
}

struct Cic {
    int x0, x1, y0, y1;
    double tx, ty;
};

inline Cic cic(const adj64* s, double px, double py) {
    const double gx = px * s->W - 0.5, gy = py * s->H - 0.5;
    const double fx = std::floor(gx), fy = std::floor(gy);
    Cic c;
    c.tx = gx - fx;
    c.ty = gy - fy;
    c.x0 = wrapi((long long)fx, s->W);
    c.x1 = wrapi((long long)fx + 1, s->W);
    c.y0 = wrapi((long long)fy, s->H);
    c.y1 = wrapi((long long)fy + 1, s->H);
    return c;
}

// y = real(IFFT(FFT(x) * spec)) (conj: the transpose operator).
void convolve(const adj64* s, const double* in, const std::vector<c64>& spec, bool conj,
              double* out) {
    const size_t P = (size_t)s->W * s->H;
    std::vector<double> z(2 * P);
    for (size_t i = 0; i < P; ++i) { z[2 * i] = in[i]; z[2 * i + 1] = 0.0; }
    oracle_fft2d_f64(z.data(), s->W, s->H, 0);
    for (size_t i = 0; i < P; ++i) {
        const double ar = z[2 * i], ai = z[2 * i + 1];
        const double br = spec[i].re, bi = conj ? -spec[i].im : spec[i].im;
        z[2 * i] = ar * br - ai * bi;
        z[2 * i + 1] = ar * bi + ai * br;
    }
    oracle_fft2d_f64(z.data(), s->W, s->H, 1);
    for (size_t i = 0; i < P; ++i) out[i] = z[2 * i];
}

// Pair term of S/kick.comp:66-80 (d = source - target on the minimum image)
// and the transposed Jacobian of it with respect to d applied to w.
struct PairOut { double ax, ay, jx, jy; };

inline PairOut pair(const adj64* s, double dx, double dy, double m, double wx, double wy) {
    dx -= std::floor(dx + 0.5);
    dy -= std::floor(dy + 0.5);
    const double px = dx * s->aspect;
    const double r2 = px * px + dy * dy;
    const double w = std::exp(-r2 / (2.0 * s->sigma * s->sigma));
    const double den = std::max(r2, s->min_d2);
    const double phys = s->g * m * w / (s->total * den);
    double dphys = -phys / (2.0 * s->sigma * s->sigma);
    if (r2 > s->min_d2) dphys -= phys / r2;
    const double wd = wx * dx + wy * dy;
    PairOut o;
    o.ax = phys * dx;
    o.ay = phys * dy;
    o.jx = phys * wx + dphys * wd * 2.0 * s->aspect * s->aspect * dx;
    o.jy = phys * wy + dphys * wd * 2.0 * dy;
    return o;
}

// Visits the sources of target i: fn(source body or -1 for a monopole,
// source x, source y, mass).
template <typename Fn>
void for_sources(const adj64* s, const Lists& L, const double* x, int i, Fn&& fn) {
    const double px = x[2 * i], py = x[2 * i + 1];
    const int hx = wrapi((long long)std::floor(px * s->W), s->W);
    const int hy = wrapi((long long)std::floor(py * s->H), s->H);
    for (int dy = -s->ry; dy <= s->ry; ++dy) {
        for (int dx = -s->rx; dx <= s->rx; ++dx) {
            const int wx = wrapi(hx + dx, s->W), wy = wrapi(hy + dy, s->H);
            const size_t c = (size_t)wy * s->W + wx;
            const int count = L.count[c];
            const bool home = dx == 0 && dy == 0;
            if (!home && count > s->exact) {
                fn(-1, (wx + 0.5) / s->W, (wy + 0.5) / s->H, L.cell_mass[c]);
            } else {
                const int limit = home ? s->home_limit : s->exact;
                int visited = 0;
                for (int o = L.head[c]; o >= 0 && visited < limit; o = L.next[o], ++visited)
                    if (o != i) fn(o, x[2 * o], x[2 * o + 1], s->mass[o]);
            }
        }
    }
}

// a(x) and the mesh force E it interpolated.
void force(const adj64* s, const double* x, double* acc, std::vector<double>& ex,
           std::vector<double>& ey, Lists& L) {
    const size_t P = (size_t)s->W * s->H;
    build_lists(s, x, L);
    std::vector<double> rho(P, 0.0);
    for (int j = 0; j < s->n; ++j) {
        const Cic c = cic(s, x[2 * j], x[2 * j + 1]);
        const double m = s->mass[j];
        rho[(size_t)c.y0 * s->W + c.x0] += m * (1 - c.tx) * (1 - c.ty);
        rho[(size_t)c.y0 * s->W + c.x1] += m * c.tx * (1 - c.ty);
        rho[(size_t)c.y1 * s->W + c.x0] += m * (1 - c.tx) * c.ty;
        rho[(size_t)c.y1 * s->W + c.x1] += m * c.tx * c.ty;
    }
    ex.resize(P);
    ey.resize(P);
    convolve(s, rho.data(), s->kx_hat, false, ex.data());
    convolve(s, rho.data(), s->ky_hat, false, ey.data());
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < s->n; ++i) {
        const Cic c = cic(s, x[2 * i], x[2 * i + 1]);
        auto interp = [&](const std::vector<double>& f) {
            const double a = f[(size_t)c.y0 * s->W + c.x0] * (1 - c.tx) + f[(size_t)c.y0 * s->W + c.x1] * c.tx;
            const double b = f[(size_t)c.y1 * s->W + c.x0] * (1 - c.tx) + f[(size_t)c.y1 * s->W + c.x1] * c.tx;
            return a * (1 - c.ty) + b * c.ty;
        };
        double ax = interp(ex) + s->field_x, ay = interp(ey) + s->field_y;
        for_sources(s, L, x, i, [&](int, double sx, double sy, double m) {
            const PairOut o = pair(s, sx - x[2 * i], sy - x[2 * i + 1], m, 0.0, 0.0);
            ax += o.ax;
            ay += o.ay;
        });
        acc[2 * i] = ax;
        acc[2 * i + 1] = ay;
    }
}

// Adds (d a / d x)^T wa to gx, for a = force(x) with the topology held fixed.
void force_adjoint(const adj64* s, const double* x, const double* wa, double* gx) {
    const size_t P = (size_t)s->W * s->H;
    std::vector<double> ex, ey, acc((size_t)2 * s->n);
    Lists L;
    force(s, x, acc.data(), ex, ey, L);
    // Spread the cotangent with the interpolation weights, then apply the
    // transposed mesh operator: mu = Kx^T lx + Ky^T ly.
    std::vector<double> lx(P, 0.0), ly(P, 0.0), mu(P), tmp(P);
    for (int i = 0; i < s->n; ++i) {
        const Cic c = cic(s, x[2 * i], x[2 * i + 1]);
        const double w[4] = {(1 - c.tx) * (1 - c.ty), c.tx * (1 - c.ty), (1 - c.tx) * c.ty, c.tx * c.ty};
        const size_t idx[4] = {(size_t)c.y0 * s->W + c.x0, (size_t)c.y0 * s->W + c.x1,
                               (size_t)c.y1 * s->W + c.x0, (size_t)c.y1 * s->W + c.x1};
        for (int k = 0; k < 4; ++k) {
            lx[idx[k]] += w[k] * wa[2 * i];
            ly[idx[k]] += w[k] * wa[2 * i + 1];
        }
    }
    convolve(s, lx.data(), s->kx_hat, true, mu.data());
    convolve(s, ly.data(), s->ky_hat, true, tmp.data());
    for (size_t c = 0; c < P; ++c) mu[c] += tmp[c];
    // Gradient of the CIC weights of body j against phi = m_j mu + wa_j . E
    // (its deposit and its interpolation).
    std::vector<double> g((size_t)2 * s->n, 0.0);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < s->n; ++j) {
        const Cic c = cic(s, x[2 * j], x[2 * j + 1]);
        const size_t i00 = (size_t)c.y0 * s->W + c.x0, i10 = (size_t)c.y0 * s->W + c.x1;
        const size_t i01 = (size_t)c.y1 * s->W + c.x0, i11 = (size_t)c.y1 * s->W + c.x1;
        auto phi = [&](size_t k) { return s->mass[j] * mu[k] + wa[2 * j] * ex[k] + wa[2 * j + 1] * ey[k]; };
        const double f00 = phi(i00), f10 = phi(i10), f01 = phi(i01), f11 = phi(i11);
        g[2 * j] = s->W * ((f10 - f00) * (1 - c.ty) + (f11 - f01) * c.ty);
        g[2 * j + 1] = s->H * ((f01 - f00) * (1 - c.tx) + (f11 - f10) * c.tx);
    }
    // Short range: the target moves against d, an exact source with it
    // (per-thread sums, added in thread order).
#pragma omp parallel
    {
        std::vector<double> part(g.size(), 0.0);
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < s->n; ++i) {
            const double wx = wa[2 * i], wy = wa[2 * i + 1];
            for_sources(s, L, x, i, [&](int src, double sx, double sy, double m) {
                const PairOut o = pair(s, sx - x[2 * i], sy - x[2 * i + 1], m, wx, wy);
                part[2 * i] -= o.jx;
                part[2 * i + 1] -= o.jy;
                if (src >= 0) {
                    part[2 * src] += o.jx;
                    part[2 * src + 1] += o.jy;
                }
            });
        }
#pragma omp for ordered schedule(static, 1)
        for (int t = 0; t < omp_get_num_threads(); ++t) {
#pragma omp ordered
            for (size_t k = 0; k < g.size(); ++k) g[k] += part[k];
        }
    }
    for (size_t k = 0; k < g.size(); ++k) gx[k] += g[k];
}

}  // namespace

extern "C" {

adj64* oracle_adj_create(const p3m_config* c, const double* materials4, int n, double field_x,
                         double field_y) {
    if (!c || n <= 0 || c->bounded) return nullptr;
    adj64* s = new adj64();
    s->cfg = *c;
    s->n = n;
    s->W = c->grid_width;
    s->H = c->grid_height;
    s->aspect = (double)c->viewport_width / (double)c->viewport_height;
    oracle_neighbor_radii(c, &s->rx, &s->ry);
    s->exact = c->exact_neighbor_body_limit;
    s->home_limit = c->maximum_home_body_interactions;
    s->g = c->gravitational_constant;
    s->sigma = (double)c->softening_cells / s->H;
    const double cw = s->aspect / s->W, ch = 1.0 / s->H;
    const double md = c->minimum_distance_cell_fraction * std::min(cw, ch);
    s->min_d2 = md * md;
    s->total = std::max(1.0, (double)n);
    s->dt = c->time_step;
    s->field_x = field_x;
    s->field_y = field_y;
    s->mass.resize(n);
    for (int i = 0; i < n; ++i) s->mass[i] = materials4[4 * i];
    build_spectra(s);
    return s;
}

void oracle_adj_destroy(adj64* s) { delete s; }

// Accelerations (n x 2) at positions (n x 2).
void oracle_adj_force(adj64* s, const double* pos2, double* acc2) {
    std::vector<double> ex, ey;
    Lists L;
    force(s, pos2, acc2, ex, ey, L);
}

// The mesh force (two W x H fields) at positions (n x 2).
void oracle_adj_mesh_force(adj64* s, const double* pos2, double* ex_out, double* ey_out) {
    std::vector<double> ex, ey, acc((size_t)2 * s->n);
    Lists L;
    force(s, pos2, acc.data(), ex, ey, L);
    std::memcpy(ex_out, ex.data(), ex.size() * sizeof(double));
    std::memcpy(ey_out, ey.data(), ey.size() * sizeof(double));
}

// Forward rollout from bodies4 (x, y, vx, vy). initial_accel: a0 = force(x0),
// otherwise accel2 holds a0. Writes the final state and acceleration.
void oracle_adj_forward(adj64* s, const double* bodies4, const double* accel2, int initial_accel,
                        int steps, double* final4, double* final_accel2) {
    const int n = s->n;
    const double dt = s->dt;
    s->steps = steps;
    s->initial_accel = initial_accel;
    s->xs.assign((size_t)steps + 1, std::vector<double>((size_t)2 * n));
    std::vector<double> v((size_t)2 * n), a((size_t)2 * n);
    for (int i = 0; i < n; ++i) {
        s->xs[0][2 * i] = bodies4[4 * i];
        s->xs[0][2 * i + 1] = bodies4[4 * i + 1];
        v[2 * i] = bodies4[4 * i + 2];
        v[2 * i + 1] = bodies4[4 * i + 3];
    }
    if (initial_accel) oracle_adj_force(s, s->xs[0].data(), a.data());
    else std::memcpy(a.data(), accel2, sizeof(double) * 2 * n);
    for (int k = 0; k < steps; ++k) {
        const std::vector<double>& x = s->xs[k];
        std::vector<double>& xn = s->xs[k + 1];
        for (int q = 0; q < 2 * n; ++q) {
            v[q] += 0.5 * dt * a[q];
            const double p = x[q] + dt * v[q];
            xn[q] = p - std::floor(p);
        }
        oracle_adj_force(s, xn.data(), a.data());
        for (int q = 0; q < 2 * n; ++q) v[q] += 0.5 * dt * a[q];
    }
    s->v = v;
    s->a = a;
    for (int i = 0; i < n; ++i) {
        final4[4 * i] = s->xs[steps][2 * i];
        final4[4 * i + 1] = s->xs[steps][2 * i + 1];
        final4[4 * i + 2] = v[2 * i];
        final4[4 * i + 3] = v[2 * i + 1];
    }
    if (final_accel2) std::memcpy(final_accel2, a.data(), sizeof(double) * 2 * n);
}

// Replaces the positions (n x 2) recorded for step k of the last forward,
// so the reverse pass can be evaluated along another trajectory (the CUDA
// one, to compare the adjoints' arithmetic alone).
void oracle_adj_set_positions(adj64* s, int k, const double* pos2) {
    if (k < 0 || k > s->steps) return;
    std::memcpy(s->xs[k].data(), pos2, sizeof(double) * 2 * s->n);
}

// Reverse pass: seed4 = dL/d(final x, y, vx, vy), seed_accel2 = dL/d(final a)
// (may be NULL). Writes dL/d(initial x, y, vx, vy) and, when the forward did
// not compute a0 itself, dL/d(a0) (else zeros).
void oracle_adj_backward(adj64* s, const double* seed4, const double* seed_accel2, double* grad4,
                         double* grad_accel2) {
    const int n = s->n;
    const double dt = s->dt;
    std::vector<double> lx((size_t)2 * n), lv((size_t)2 * n), la((size_t)2 * n, 0.0), wa((size_t)2 * n);
    for (int i = 0; i < n; ++i) {
        lx[2 * i] = seed4[4 * i];
        lx[2 * i + 1] = seed4[4 * i + 1];
        lv[2 * i] = seed4[4 * i + 2];
        lv[2 * i + 1] = seed4[4 * i + 3];
    }
    if (seed_accel2) std::memcpy(la.data(), seed_accel2, sizeof(double) * 2 * n);
    for (int k = s->steps - 1; k >= 0; --k) {
        for (int q = 0; q < 2 * n; ++q) wa[q] = la[q] + 0.5 * dt * lv[q];
        force_adjoint(s, s->xs[k + 1].data(), wa.data(), lx.data());
        for (int q = 0; q < 2 * n; ++q) {
            lv[q] += dt * lx[q];
            la[q] = 0.5 * dt * lv[q];
        }
    }
    if (s->initial_accel) {
        force_adjoint(s, s->xs[0].data(), la.data(), lx.data());
        std::fill(la.begin(), la.end(), 0.0);
    }
    for (int i = 0; i < n; ++i) {
        grad4[4 * i] = lx[2 * i];
        grad4[4 * i + 1] = lx[2 * i + 1];
        grad4[4 * i + 2] = lv[2 * i];
        grad4[4 * i + 3] = lv[2 * i + 1];
    }
    if (grad_accel2) std::memcpy(grad_accel2, la.data(), sizeof(double) * 2 * n);
}

}  // extern "C"
