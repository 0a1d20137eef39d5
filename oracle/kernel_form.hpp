// Oracle, kernel form -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of HydroPol2D's surface-flow step in the algebraically identical form
// the CUDA kernels compute, in float or double.  The tests require the CUDA kernels to
// reproduce this restatement bit for bit, and require this restatement (in double) to
// agree with the literal FP64 restatement (oracle/literal.py) to round-off.
//
// Differences from the literal reference order, each algebraically exact:
//   * SI state inside: h [m], face discharge per unit width q [m^2/s], I [m], T [s].
//     The reference carries mm and mm/h (Local_Inertial_Model_D4.m:198, :309).
//   * Split slope: S = (dz + (h_R - h_L)) / dx with dz = z_R - z_L precomputed from the
//     FP64 DEM, and Hf = max(max(h_L - max(dz,0), h_R + min(dz,0)), 0), which equals
//     max(max(y_L, y_R) - max(z_L, z_R), 0) (Local_Inertial_Model_D4.m:91-134).
//   * Bates update as (num * Hf^(7/3)) / (Hf^(7/3) + g dt n^2 |q_p|), equal to
//     num / (1 + g dt n^2 |q_p| / Hf^(7/3)) (Inertial_Solver.m:24-25), one division.
//   * Hf^(7/3), h^(5/3): x^2 * cbrt(x) and x * cbrt(x)^2 with cbrt(x) = x * r^2 and
//     r = x^(-1/3) from a fixed Newton iteration (no libm), so that CPU and GPU round
//     identically.  The seed is the exponent-field division of the IEEE representation
//     (the classic bit-level log2 approximation), refined by r <- r + r(1 - x r^3)/3 with
//     the residual and the update as explicit fused multiply-adds (std::fma here, fma on
//     the GPU: both correctly rounded).
//   * Draining limiter compares rates per unit width (both sides divided by dx).
//   * CFL velocities q/Hf (refreshing_timestep.m:71-77 after unit cancellation); the
//     minimum of alfa*dx/c over cells is taken as alfa*dx/max(c), which is exact because
//     division by a positive number is monotone.
// Compile with -ffp-contract=off: no fused multiply-add may appear.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <algorithm>

#include "hp2d.h"

namespace hp2d_oracle {

constexpr double kG = 9.81;

template <typename R> struct FloatBits;
template <> struct FloatBits<float> {
    using U = uint32_t;
    static constexpr U seed = 0x54AAAAABu;                  // (4/3) * 127 * 2^23
    static constexpr int iters = 3;
    static float tiny() { return 1.17549435e-38f; }         // smallest normal
    static constexpr float up = 16777216.0f;                // 2^24
    static constexpr float down_r = 256.0f;                 // 2^8
};
template <> struct FloatBits<double> {
    using U = uint64_t;
    static constexpr U seed = 0x5540000000000000ull;        // (4/3) * 1023 * 2^52
    static constexpr int iters = 5;
    static double tiny() { return 2.2250738585072014e-308; }
    static constexpr double up = 18014398509481984.0;       // 2^54
    static constexpr double down_r = 262144.0;              // 2^18
};

// x^(-1/3) for finite x > 0.
template <typename R> inline R rcbrt(R x) {
    using FB = FloatBits<R>;
    R scale = R(1);
    if (x < FB::tiny()) { x = x * FB::up; scale = FB::down_r; }
    typename FB::U u;
    std::memcpy(&u, &x, sizeof(R));
    u = FB::seed - u / 3;
    R r;
    std::memcpy(&r, &u, sizeof(R));
    const R third = R(1.0 / 3.0);
    for (int it = 0; it < FB::iters; ++it) {
        R t = x * r;
        t = t * r;
        const R e = std::fma(-t, r, R(1));
        r = std::fma(r * e, third, r);
    }
    return r * scale;
}
template <typename R> inline R pow73(R x) {       // x^(7/3), x >= 0
    if (!(x > R(0))) return R(0);
    R r = rcbrt(x);
    R c = x * (r * r);
    return (x * x) * c;
}
template <typename R> inline R pow53(R x) {       // x^(5/3), x >= 0
    if (!(x > R(0))) return R(0);
    R r = rcbrt(x);
    R c = x * (r * r);
    return x * (c * c);
}

// a / b for b > 0 as the kernels compute it: FP32 reciprocal from the bit seed
// 0x7EF311C3 - bits(b), three Newton steps, quotient with one residual correction
// (b raised to the smallest normal first); FP64 the IEEE division.
inline float qdiv(float a, float b) {
    b = std::fmax(b, 1.17549435e-38f);
    uint32_t u;
    std::memcpy(&u, &b, 4);
    u = 0x7EF311C3u - u;
    float r;
    std::memcpy(&r, &u, 4);
    float e = std::fma(-b, r, 1.0f);
    r = std::fma(r, e, r);
    e = std::fma(-b, r, 1.0f);
    r = std::fma(r, e, r);
    e = std::fma(-b, r, 1.0f);
    r = std::fma(r, e, r);
    const float q = a * r;
    return std::fma(std::fma(-b, q, a), r, q);
}
inline double qdiv(double a, double b) { return a / b; }

template <typename R> inline bool finite(R v) { return std::isfinite(v); }

template <typename R> struct Consts {
    R dt, gdt, dt_over_dx, dx_over_dt, inv_dt, inv_dx, g, tol, thr,
      clamp_eps, neg_eps, ten, half, stagnant, celer_floor, big_depth;
    Consts(double dt_s, double res, double tol_mm, double thr_mm) {
        dt = R(dt_s);
        gdt = R(kG * dt_s);
        dt_over_dx = R(dt_s / res);
        dx_over_dt = R(res / dt_s);
        inv_dt = R(1.0 / dt_s);
        inv_dx = R(1.0 / res);
        g = R(kG);
        tol = R(tol_mm / 1000.0);
        thr = R(thr_mm / 1000.0);
        clamp_eps = R(1e-9);
        neg_eps = R(-1e-11);
        ten = R(10);
        half = R(0.5);
        stagnant = R(0.01);
        celer_floor = R(1e-10);
        big_depth = R(1e9);
    }
};

template <typename R> class Model {
public:
    int ny, nx;
    double res;
    hp2d_params p;
    // static
    std::vector<R> dzx, dzy, n2;
    std::vector<int32_t> outlet_idx;
    std::vector<R> outlet_coef;
    std::vector<uint8_t> soil;          // empty or ny*nx, 255 = none
    std::vector<R> ks, psi, dth, lu, kout, tr, minsm;   // per class
    // rain
    std::vector<double> rain_t, rain_r;
    int n_maps = 0, my = 0, mx = 0;
    double map_dt = 5.0;
    std::vector<double> map_t;   // empty: map m over [m, m+1) x map_dt; else [map_t[m], map_t[m+1])
    std::vector<float> maps;
    // state
    std::vector<R> h, qx, qy, I, T, dmax, arrival;
    // outputs of the last li step
    std::vector<R> hfx, hfy, hf3, qo;    // hf3/qo per outlet entry
    std::vector<R> qx_unl, qy_unl, scale, hn;
    // clock
    double t_min = 0, time_step = 0, tsp = 0;   // clock [min], step [min], time_save_previous
    int64_t k = 1;
    // rain interval of the current step and the loop's t_previous [min]; the first step's
    // comes from the update_spatial_BC call before the loop (HydroPol2D_Main_While.m:115)
    // with t_previous = 0 (:120)
    double rain_a = 0, rain_b = 0, t_prev = 0;
    // diagnostics
    double vmax_last = 0, rain_vol = 0, inf_vol = 0, out_vol = 0;
    int64_t neg_warn = 0, unstable = 0;
    int omp_threads = 1;

    Model(const hp2d_grid& g, const hp2d_params& prm) : ny(g.ny), nx(g.nx), res(g.resolution), p(prm) {
        size_t n = size_t(ny) * nx;
        dzx.assign(n, R(0)); dzy.assign(n, R(0)); n2.assign(n, R(0));
        h.assign(n, R(0)); qx.assign(n, R(0)); qy.assign(n, R(0));
        I.assign(n, R(0)); T.assign(n, R(0));
        dmax.assign(n, -std::numeric_limits<R>::infinity());
        arrival.assign(n, std::numeric_limits<R>::infinity());
        hfx.assign(n, R(0)); hfy.assign(n, R(0));
        qx_unl.assign(n, R(0)); qy_unl.assign(n, R(0)); scale.assign(n, R(1));
        time_step = p.min_time_step / 60.0;   // HydroPol2D_preprocessing.m:2469
        t_min = p.min_time_step / 60.0;
        rain_b = t_min;
    }

    // the clock setter of the unfused drivers: k = 1 starts a run, k + 1 is the loop's
    // advance (HydroPol2D_Main_While.m:721, :734-738), any other k re-seeds the rain
    // interval as if the last two steps had taken time_step
    void set_clock(double t, double ts, int64_t kk) {
        if (kk == 1) {
            rain_a = 0.0; rain_b = t; t_prev = 0.0;
        } else if (kk == k + 1) {
            rain_a = t_prev; rain_b = t_min; t_prev = k == 1 ? ts : t_min;
        } else {
            rain_a = t - 2.0 * ts; rain_b = t - ts; t_prev = t - ts;
        }
        t_min = t; time_step = ts; k = kk;
    }

    size_t at(int i, int j) const { return size_t(i) * nx + j; }

    std::vector<uint8_t> wall;   // NaN elevation (idx_nan): may hold a NaN depth
    void upload_static(const double* z, const double* n, const int32_t* rows, const int32_t* cols,
                       int nout, const double* slopes) {
        wall.assign(size_t(ny) * nx, 0);
        for (size_t c = 0; c < wall.size(); ++c) wall[c] = std::isnan(z[c]) ? 1 : 0;
        // domain-edge faces +inf, faces next to a NaN elevation NaN (see face())
        const double edge = std::numeric_limits<double>::infinity();
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                double dx_ = (j + 1 < nx) ? z[at(i, j + 1)] - z[c] : edge;
                double dy_ = (i >= 1) ? z[at(i - 1, j)] - z[c] : edge;
                dzx[c] = R(dx_);
                dzy[c] = R(dy_);
                n2[c] = R(n[c] * n[c]);
            }
        // outlet cells in increasing linear-index order, duplicates dropped (a repeated
        // index in MATLAB's d_t(outlet_sub) assignment writes the same value twice)
        std::vector<std::pair<int32_t, R>> outs;
        for (int o = 0; o < nout; ++o) {
            size_t c = at(rows[o], cols[o]);
            double coef;
            if (p.outlet_type == 1) {
                double s = slopes ? slopes[o] : p.slope_outlet;
                coef = std::sqrt(std::fabs(s)) / (n[c] * res);
            } else {
                coef = std::sqrt(kG) / res;
            }
            outs.emplace_back(int32_t(c), R(coef));
        }
        std::sort(outs.begin(), outs.end(), [](auto& a, auto& b) { return a.first < b.first; });
        outs.erase(std::unique(outs.begin(), outs.end(), [](auto& a, auto& b) { return a.first == b.first; }),
                   outs.end());
        outlet_idx.resize(outs.size());
        outlet_coef.resize(outs.size());
        for (size_t o = 0; o < outs.size(); ++o) {
            outlet_idx[o] = outs[o].first;
            outlet_coef[o] = outs[o].second;
        }
        hf3.assign(outs.size(), R(0));
        qo.assign(outs.size(), R(0));
    }

    void set_soil(const uint8_t* cls, int ncls, const double* ksat, const double* psi_mm,
                  const double* dtheta, const double* Lu, const double* kout_mmh,
                  const double* Tr_h, const double* minsm_mm) {
        soil.assign(cls, cls + size_t(ny) * nx);
        ks.resize(ncls); psi.resize(ncls); dth.resize(ncls); lu.resize(ncls);
        kout.resize(ncls); tr.resize(ncls); minsm.resize(ncls);
        for (int c = 0; c < ncls; ++c) {
            ks[c] = R(ksat[c] / 3.6e6);
            psi[c] = R(psi_mm[c] / 1000.0);
            dth[c] = R(dtheta[c]);
            lu[c] = R(Lu[c]);
            kout[c] = R(kout_mmh[c] / 3.6e6);
            tr[c] = R(Tr_h[c] * 3600.0);
            minsm[c] = R(minsm_mm[c] / 1000.0);
        }
        reset_timer();
    }

    void set_state(const double* d_mm, const double* outflow, const double* I_mm) {
        size_t n = size_t(ny) * nx;
        for (size_t c = 0; c < n; ++c) {
            h[c] = R(d_mm[c] / 1000.0);
            // outflow_bates [mm/h] -> q [m^2/s]: mm/h / 1000 / 3600 * dx
            qx[c] = outflow ? R(outflow[c] / 3.6e6 * res) : R(0);
            qy[c] = outflow ? R(outflow[n + c] / 3.6e6 * res) : R(0);
            if (I_mm) I[c] = R(I_mm[c] / 1000.0);
            dmax[c] = -std::numeric_limits<R>::infinity();
            arrival[c] = std::numeric_limits<R>::infinity();
        }
        reset_timer();
    }

    // recovery timer starts at Tr (HydroPol2D_Main_While_Ensemble.m:266)
    void reset_timer() {
        for (size_t c = 0; c < T.size(); ++c)
            T[c] = (!soil.empty() && soil[c] != 255) ? tr[soil[c]] : R(0);
    }

    // test hook: overwrite the depth only [mm]
    void set_depth(const double* d_mm) {
        for (size_t c = 0; c < h.size(); ++c) h[c] = R(d_mm[c] / 1000.0);
    }

    // ---------------- rain of a step (update_spatial_BC.m:435-470, :536-558) ----------------
    // A step applies the rain of the clock interval [rain_a, rain_b]: the exact integral of
    // the piecewise-constant rate over it (localAverageRateOverStep x interval,
    // update_spatial_BC.m:1131-1184; maps :1287-1359) / 60 -> mm, here in metres.  Uniform
    // rates hold from rain_t[q] up to rain_t[q+1] (the last for ever); map m holds over
    // [m, m+1) x map_dt (or over [map_t[m], map_t[m+1]) for end-stamped input maps,
    // update_spatial_BC.m:497-517) and nothing after the last map; an interval overlaps at most
    // two maps (every map interval >= max_time_step, checked by the library).
    struct StepRain {
        R depth = R(0);        // uniform [m]
        int nm = 0;
        int m[2] = {0, 0};
        R w[2] = {R(0), R(0)}; // overlap [min] / 60000
    };
    StepRain step_rain(double a, double b) const {
        StepRain s;
        if (!rain_r.empty()) {
            double acc = 0.0;
            if (b > a) {
                const size_t nq = rain_r.size();
                for (size_t q = 0; q < nq; ++q) {
                    const double lo = rain_t[q];
                    const double hi = q + 1 < nq ? rain_t[q + 1] : b;
                    const double ov = std::fmax(0.0, std::fmin(b, hi) - std::fmax(a, lo));
                    if (ov > 0.0 && std::isfinite(rain_r[q])) acc += rain_r[q] * ov;
                }
            }
            s.depth = R(acc / 60000.0);
        }
        if (n_maps > 0 && b > a) {
            int m0 = 0;
            if (!map_t.empty()) {   // the first map that ends after a
                while (m0 < n_maps && !(map_t[size_t(m0) + 1] > a)) ++m0;
            } else {
                m0 = std::max(0, int(std::floor(a / map_dt)) - 1);
            }
            for (int q = m0; q < n_maps && s.nm < 2; ++q) {
                const double lo = map_t.empty() ? q * map_dt : map_t[size_t(q)];
                const double hi = map_t.empty() ? (q + 1) * map_dt : map_t[size_t(q) + 1];
                if (lo >= b) break;
                const double ov = std::fmin(b, hi) - std::fmax(a, lo);
                if (ov > 0.0) {
                    s.m[s.nm] = q;
                    s.w[s.nm] = R(ov / 60000.0);
                    ++s.nm;
                }
            }
        }
        return s;
    }
    // cell-centred bilinear sample of map m at cell (i, j) [mm/h]
    R map_sample(int m, int i, int j) const {
        const float* f = maps.data() + size_t(m) * my * mx;
        const R half = R(0.5);
        R fy = (R(i) + half) * R(double(my) / ny) - half;
        R fx = (R(j) + half) * R(double(mx) / nx) - half;
        fy = std::fmin(std::fmax(fy, R(0)), R(my - 1));
        fx = std::fmin(std::fmax(fx, R(0)), R(mx - 1));
        int iy0 = int(std::floor(fy)), ix0 = int(std::floor(fx));
        int iy1 = std::min(iy0 + 1, my - 1), ix1 = std::min(ix0 + 1, mx - 1);
        R wy = fy - R(iy0), wx = fx - R(ix0);
        R f00 = R(f[iy0 * mx + ix0]), f01 = R(f[iy0 * mx + ix1]);
        R f10 = R(f[iy1 * mx + ix0]), f11 = R(f[iy1 * mx + ix1]);
        R top = (R(1) - wx) * f00 + wx * f01;
        R bot = (R(1) - wx) * f10 + wx * f11;
        return (R(1) - wy) * top + wy * bot;
    }
    // rain depth [m] the step adds at cell (i, j)
    R rain_depth(const StepRain& s, int i, int j) const {
        if (n_maps <= 0) return s.depth;
        if (s.nm == 0) return R(0);
        R r = s.w[0] * map_sample(s.m[0], i, j);
        if (s.nm > 1) r = r + s.w[1] * map_sample(s.m[1], i, j);
        return r;
    }

    // ---------------- inflow hydrographs (update_spatial_BC.m:359-395) ----------------
    // gauge g's rate holds from inf_t[q] up to inf_t[q+1] (the last for ever); a cell of the
    // gauge receives the integral over the step's rain interval / 60 mm after the
    // infiltration (Hydrological_Model.m:27-28); cells of several gauges sum them in
    // increasing gauge order
    int inf_ng = 0, inf_nt = 0;
    std::vector<double> inf_t, inf_r, inf_gcells;
    std::vector<int32_t> inf_entry, inf_off, inf_gauge;
    std::vector<R> inf_depth;
    double inflow_vol = 0;

    void set_inflow(int ng, int nt, const double* t0, const double* rate, int nc, const int32_t* rows,
                    const int32_t* cols, const int32_t* gauge, const double* z) {
        const size_t n = size_t(ny) * nx;
        inf_ng = ng; inf_nt = nt;
        inf_t.assign(t0, t0 + (ng ? nt : 0));
        inf_r.assign(rate, rate + (ng ? size_t(nt) * ng : 0));
        inf_entry.assign(n, -1);
        inf_off.assign(1, 0);
        inf_gauge.clear();
        inf_gcells.assign(size_t(ng), 0.0);
        inf_depth.assign(size_t(ng), R(0));
        std::vector<std::vector<int32_t>> per(n);
        for (int q = 0; q < (ng ? nc : 0); ++q) per[at(rows[q], cols[q])].push_back(gauge[q]);
        for (size_t c = 0; c < n; ++c) {
            if (per[c].empty()) continue;
            std::sort(per[c].begin(), per[c].end());
            inf_entry[c] = int32_t(inf_off.size() - 1);
            for (int32_t g : per[c]) {
                inf_gauge.push_back(g);
                if (std::isfinite(z[c])) inf_gcells[size_t(g)] += 1.0;
            }
            inf_off.push_back(int32_t(inf_gauge.size()));
        }
    }
    void inflow_depths(double a, double b) {
        for (int g = 0; g < inf_ng; ++g) {
            double acc = 0.0;
            if (b > a) {
                for (int q = 0; q < inf_nt; ++q) {
                    const double lo = inf_t[q];
                    const double hi = q + 1 < inf_nt ? inf_t[q + 1] : b;
                    const double ov = std::fmax(0.0, std::fmin(b, hi) - std::fmax(a, lo));
                    const double r = inf_r[size_t(q) * inf_ng + g];
                    if (ov > 0.0 && std::isfinite(r)) acc += r * ov;
                }
            }
            inf_depth[g] = R(acc / 60000.0);
        }
    }

    // ---------------- stage hydrographs (update_spatial_BC.m:316-357) ----------------
    // after the step's timestep refresh, a stage cell's depth becomes its gauge's water depth
    // at the step's clock (the last record starting at or before it, else the first); a cell
    // of several masks takes the highest gauge (the reference overwrites in gauge order)
    int stg_ng = 0, stg_nt = 0;
    std::vector<double> stg_t, stg_d;
    std::vector<int32_t> stg_cell;   // per cell: gauge or -1
    double stage_vol = 0;
    void set_stage(int ng, int nt, const double* t0, const double* d, int nc, const int32_t* rows,
                   const int32_t* cols, const int32_t* gauge) {
        stg_ng = ng; stg_nt = nt;
        stg_t.assign(t0, t0 + (ng ? nt : 0));
        stg_d.assign(d, d + (ng ? size_t(nt) * ng : 0));
        stg_cell.assign(size_t(ny) * nx, -1);
        for (int q = 0; q < (ng ? nc : 0); ++q) {
            int32_t& c = stg_cell[at(rows[q], cols[q])];
            c = std::max(c, gauge[q]);
        }
    }
    void apply_stage() {
        if (!stg_ng) return;
        std::vector<R> now(static_cast<size_t>(stg_ng), R(0));
        for (int g = 0; g < stg_ng; ++g) {
            int z = 0;
            for (int q = 0; q < stg_nt; ++q)
                if (stg_t[q] <= t_min) z = q;
            now[g] = R(stg_d[size_t(z) * stg_ng + g]);
        }
        double v = 0;
        for (size_t c = 0; c < h.size(); ++c) {
            if (stg_cell[c] < 0) continue;
            const R sv = now[size_t(stg_cell[c])];
            v += double(sv) - double(h[c]);
            h[c] = sv;
        }
        stage_vol += v * res * res;
    }

    // ---------------- reservoir / control structures (Local_Inertial_Model_D4.m:318-344) ------
    // From the depth the fluxes use, in structure order: dtsup = d_tot(res)/1000 (with the
    // earlier structures' additions to d_tot), dh = min(k1 max(dtsup-h1,0)^k2 / A 1000 3600,
    // 1000 max(dtsup-h1,0)/dt_h) dt_h mm; the reservoir's Vol_Flux gains dh (the reference's
    // sign), ds1 gains dh, and with a second structure ds1 gains dh again, then dh2 goes the
    // same way to ds2.  Each cell's additions (in mm, FP64) join its depth before the
    // continuity as one extra: hn = (h + extra) + flux term.
    int st_n = 0;
    std::vector<double> st_coef;          // [n][6] k1 h1 k2 k3 h2 k4
    std::vector<int32_t> st_slot;         // [n][3] slot of res, ds1, ds2 (-1: none)
    std::vector<size_t> st_cell;          // slot -> cell
    double struct_vol = 0;
    void set_reservoirs(int n, const int32_t* rr, const int32_t* rc, const double* k1, const double* h1,
                        const double* k2, const int32_t* d1r, const int32_t* d1c, const double* k3,
                        const double* h2, const double* k4, const int32_t* d2r, const int32_t* d2c) {
        st_n = n;
        st_coef.assign(size_t(n) * 6, 0.0);
        st_slot.assign(size_t(n) * 3, -1);
        st_cell.clear();
        auto slot_of = [&](int r, int c) {
            const size_t k = at(r, c);
            for (size_t q = 0; q < st_cell.size(); ++q)
                if (st_cell[q] == k) return int32_t(q);
            st_cell.push_back(k);
            return int32_t(st_cell.size() - 1);
        };
        for (int i = 0; i < n; ++i) {
            const double cf[6] = {k1[i], h1[i], k2[i], k3[i], h2[i], k4[i]};
            for (int q = 0; q < 6; ++q) st_coef[size_t(i) * 6 + q] = cf[q];
            st_slot[3 * i] = slot_of(rr[i], rc[i]);
            if (d1r[i] >= 0) st_slot[3 * i + 1] = slot_of(d1r[i], d1c[i]);
            if (d2r[i] >= 0) st_slot[3 * i + 2] = slot_of(d2r[i], d2c[i]);
        }
    }
    // extras [m] per slot from the depth h the fluxes use; time_step [min]
    std::vector<R> structure_extras(double ts_min) const {
        const size_t m = st_cell.size();
        std::vector<double> ds(m, 0.0), rv(m, 0.0);
        const double dt_h = ts_min / 60.0, area = res * res;
        for (int i = 0; i < st_n; ++i) {
            const double* c = &st_coef[size_t(i) * 6];
            const int sr = st_slot[3 * i], s1 = st_slot[3 * i + 1], s2 = st_slot[3 * i + 2];
            double dh = 0.0, dtsup = 0.0;
            if (s1 >= 0) {
                dtsup = (double(h[st_cell[size_t(sr)]]) * 1000.0 + ds[size_t(sr)]) / 1000.0;
                const double q = std::fmax(dtsup - c[1], 0.0);
                const double avail = 1000.0 * q / dt_h;
                dh = std::fmin(c[0] * std::pow(q, c[2]) / area * 1000.0 * 3600.0, avail) * dt_h;
                rv[size_t(sr)] += dh;
                dtsup = dtsup - dh / 1000.0;
                ds[size_t(s1)] += dh;
            }
            if (s2 >= 0) {
                ds[size_t(s1)] += dh;
                const double q = std::fmax(dtsup - c[4], 0.0);
                const double avail = 1000.0 * q / dt_h;
                const double dh2 = std::fmin(c[3] * std::pow(q, c[5]) / area * 1000.0 * 3600.0, avail) * dt_h;
                rv[size_t(sr)] += dh2;
                ds[size_t(s2)] += dh2;
            }
        }
        std::vector<R> ex(m);
        for (size_t q = 0; q < m; ++q) ex[q] = R((ds[q] + rv[q]) / 1000.0);
        return ex;
    }

    // ---------------- hydrology: rain + Green-Ampt + clamp ----------------
    void hydrology(double dts) {
        Consts<R> K(dts, res, p.depth_tolerance, p.arrival_threshold);
        const StepRain SR = step_rain(rain_a, rain_b);
        if (inf_ng) {
            inflow_depths(rain_a, rain_b);
            double v = 0.0;
            for (int g = 0; g < inf_ng; ++g) v += double(inf_depth[g]) * inf_gcells[g];
            inflow_vol += v * res * res;
        }
        size_t n = size_t(ny) * nx;
        double rv = 0, iv = 0;
        const bool ga = p.flag_infiltration == 1 && !soil.empty();
#pragma omp parallel for schedule(static) reduction(+ : rv, iv)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R r = rain_depth(SR, i, j);
                R hh = h[c] + r;
                if (std::isfinite(double(hh))) rv += double(r);
                if (ga && soil[c] != 255) {
                    int s = soil[c];
                    R Ip = I[c];
                    R C = ks[s] * (R(1) + ((hh + psi[s]) * dth[s]) / Ip);
                    if (Ip > lu[s]) C = ks[s];
                    R ia = hh * K.inv_dt;
                    bool idxC = ia <= C;
                    R Tn = T[c] - K.dt;
                    if (ia > C) Tn = tr[s];
                    bool idxT = Tn < R(0);
                    R f = std::fmin(C, ia);
                    R In = Ip + f * K.dt;
                    if (idxC) In = In - kout[s] * K.dt;
                    In = std::fmax(In, minsm[s]);
                    if (idxT) In = minsm[s];
                    I[c] = In;
                    T[c] = Tn;
                    R fd = f * K.dt;
                    hh = hh - fd;
                    if (hh < R(0)) hh = R(0);
                    if (std::isfinite(double(fd))) iv += double(fd);
                }
                if (inf_ng && inf_entry[c] >= 0) {   // BC_States.inflow is summed over gauges first
                    const int e = inf_entry[c];
                    R v = R(0);
                    for (int q = inf_off[e]; q < inf_off[e + 1]; ++q) v = v + inf_depth[inf_gauge[q]];
                    hh = hh + v;
                }
                h[c] = hh;
            }
        rain_vol += rv * res * res;
        inf_vol += iv * res * res;
        bool any_neg = false;
#pragma omp parallel for schedule(static) reduction(|| : any_neg)
        for (size_t c = 0; c < n; ++c)
            if (h[c] < K.neg_eps) any_neg = true;
        if (any_neg) ++neg_warn;
#pragma omp parallel for schedule(static)
        for (size_t c = 0; c < n; ++c) {
            if (!any_neg && h[c] < K.clamp_eps) h[c] = R(0);
            if (h[c] < R(0)) h[c] = R(0);
        }
    }

    // ---------------- Local_Inertial_Model_D4 ----------------
    // one face: returns (Hf, q) from neighbour depths; for x faces (a, b) = (L, R);
    // for y faces (a, b) = (U, D) and dz = z_U - z_D, so the roles of max/min swap.
    // q_lo / q_hi: previous fluxes of the same direction one face before / after, used by
    // flag_numerical_scheme 2 (s-upwind) and 3 (s-centred), Inertial_Solver.m:29-121 (zero
    // outside the interior columns / rows)
    inline void face(R ha, R hb, R dz, R qp, R n2c, bool is_x, const Consts<R>& K, R& Hf, R& q, R q_lo = R(0),
                     R q_hi = R(0)) const {
        // non-finite dz: +inf on the domain edge (Hf = 0, Local_Inertial_Model_D4.m:139-140),
        // NaN next to an idx_nan cell: MATLAB's max skips the NaN, so Hf is the inside
        // cell's depth (:133-134) and the NaN slope sends q to 0 (:264)
        if (!(std::fabs(dz) <= R(3.0e38))) {
            Hf = std::isnan(dz) ? std::fmax(std::fmax(ha, hb), R(0)) : R(0);
            q = R(0);
            return;
        }
        ha = std::fmax(ha, R(0));
        hb = std::fmax(hb, R(0));
        R S;
        if (is_x) {
            Hf = std::fmax(std::fmax(ha - std::fmax(dz, R(0)), hb + std::fmin(dz, R(0))), R(0));
            S = (dz + (hb - ha)) * K.inv_dx;
        } else {
            Hf = std::fmax(std::fmax(ha + std::fmin(dz, R(0)), hb - std::fmax(dz, R(0))), R(0));
            S = (dz + (ha - hb)) * K.inv_dx;
        }
        if (!(Hf > R(0))) { q = R(0); return; }
        R qn = qp;
        if (p.flag_numerical_scheme != 1) {
            // theta = 1 - dt/dx min(|q_p|/Hf, sqrt(g Hf)); the momentum term mixes q_p with the
            // upwind (scheme 2) or centred (scheme 3) neighbour flux
            const R th = R(1) - K.dt_over_dx * std::fmin(qdiv(std::fabs(qp), Hf), std::sqrt(K.g * Hf));
            const R qnb = p.flag_numerical_scheme == 2 ? (qp < R(0) ? q_hi : q_lo) : R(0.5) * (q_lo + q_hi);
            qn = th * qp + (R(1) - th) * qnb;
        }
        R num = std::fma(-(K.gdt * Hf), S, qn);
        R h73 = pow73(Hf);
        R den = std::fma(K.gdt * n2c, std::fabs(qp), h73);
        q = qdiv(num * h73, den);
        if (!std::isfinite(q)) q = R(0);
        if (p.flag_critical == 1) {
            R crit = Hf * std::sqrt(K.g * Hf);
            q = std::fmin(std::fmax(q, -crit), crit);
        }
        R thr = Hf * K.ten;
        q = std::fmin(std::fmax(q, -thr), thr);
    }

    void li(double dts, double ts_min) {
        Consts<R> K(dts, res, p.depth_tolerance, p.arrival_threshold);
        // faces (unlimited)
#pragma omp parallel for schedule(static)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R Hf, q;
                R hR = (j + 1 < nx) ? h[at(i, j + 1)] : R(0);
                const bool inx = j >= 1 && j + 1 < nx, iny = i >= 1 && i + 1 < ny;
                face(h[c], hR, dzx[c], qx[c], n2[c], true, K, Hf, q, inx ? qx[c - 1] : R(0), inx ? qx[c + 1] : R(0));
                hfx[c] = Hf; qx_unl[c] = q;
                R hU = (i >= 1) ? h[at(i - 1, j)] : R(0);
                face(hU, h[c], dzy[c], qy[c], n2[c], false, K, Hf, q, iny ? qy[at(i - 1, j)] : R(0),
                     iny ? qy[at(i + 1, j)] : R(0));
                hfy[c] = Hf; qy_unl[c] = q;
            }
        // donor scale
#pragma omp parallel for schedule(static)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R out = std::fmax(qx_unl[c], R(0));
                if (j >= 1) out = out + std::fmax(-qx_unl[at(i, j - 1)], R(0));
                out = out + std::fmax(qy_unl[c], R(0));
                if (i + 1 < ny) out = out + std::fmax(-qy_unl[at(i + 1, j)], R(0));
                R avail = std::fmax(h[c], R(0)) * K.dx_over_dt;
                R s = R(1);
                if (out > avail && out > R(0)) s = avail / out;
                if (!std::isfinite(s)) s = R(0);
                scale[c] = std::fmax(std::fmin(s, R(1)), R(0));
            }
        // limited faces
#pragma omp parallel for schedule(static)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R q = qx_unl[c];
                if (j + 1 < nx) {
                    if (q > R(0)) q = q * scale[c];
                    else if (q < R(0)) q = q * scale[at(i, j + 1)];
                } else q = R(0);
                if (!std::isfinite(q)) q = R(0);
                qx[c] = q;
                q = qy_unl[c];
                if (i >= 1) {
                    if (q > R(0)) q = q * scale[c];
                    else if (q < R(0)) q = q * scale[at(i - 1, j)];
                } else q = R(0);
                if (!std::isfinite(q)) q = R(0);
                qy[c] = q;
            }
        // control structures: extras from the depth the fluxes used, joining h first
        if (st_n) {
            const std::vector<R> ex = structure_extras(ts_min);
            double v = 0.0;
            for (size_t q = 0; q < ex.size(); ++q) {
                h[st_cell[q]] = h[st_cell[q]] + ex[q];
                v += double(ex[q]) * res * res;
            }
            struct_vol += v;
        }
        // continuity
        hn.resize(h.size());
#pragma omp parallel for schedule(static)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R qL = (j >= 1) ? qx[at(i, j - 1)] : R(0);
                R qD = (i + 1 < ny) ? qy[at(i + 1, j)] : R(0);
                R hnew = h[c] + K.dt_over_dx * (((qL - qx[c]) - qy[c]) + qD);
                if (hnew < R(0)) hnew = R(0);
                hn[c] = hnew;
            }
        h.swap(hn);
        // outlet sink
        double ov = 0;
        for (size_t o = 0; o < outlet_idx.size(); ++o) {
            size_t c = size_t(outlet_idx[o]);
            R hc = h[c];
            R hout = std::fmax(hc, R(0));
            R qq;
            if (p.outlet_type == 1) qq = outlet_coef[o] * pow53(hout);
            else qq = outlet_coef[o] * (hout * std::sqrt(hout));
            R qmax = hout * K.inv_dt;
            qq = std::fmin(qq, qmax);
            if (!std::isfinite(qq)) qq = R(0);
            h[c] = hc - qq * K.dt;
            hf3[o] = hout;
            qo[o] = qq;
            ov += double(qq * K.dt);
        }
        out_vol += ov * res * res;
    }

    // ---------------- refreshing_timestep (refresh branch) ----------------
    // returns time_calculation_routing [s]; fills vmax
    // ---------------- velocity / hazard maxima (save_output_maps.m:588-604) ----------------
    // the velocity raster max(|vr|, |vu|, |vb|) of the last refresh, and running maxima of it
    // and of depth x velocity (0 below 0.01 m or non-finite, NaN where the depth is NaN)
    bool hz_on = false;
    std::vector<R> vras, vmaxm, hzmaxm;
    void set_hazard_tracking(bool on) {
        hz_on = on;
        if (on) {
            vras.assign(h.size(), R(0));
            vmaxm.assign(h.size(), R(0));
            hzmaxm.assign(h.size(), R(0));
        }
    }
    void track_hazard() {
        for (size_t c = 0; c < h.size(); ++c) {
            const R vr = vras[c];
            vmaxm[c] = vr > vmaxm[c] ? vr : vmaxm[c];
            const R hd = std::fmax(h[c], R(0));
            R hz = hd * vr;
            if (hd < R(0.01) || !std::isfinite(hz)) hz = R(0);
            hzmaxm[c] = std::isnan(h[c]) ? h[c] : (hz > hzmaxm[c] ? hz : hzmaxm[c]);
        }
    }

    double cfl(double dts, double* vmax_out) {
        Consts<R> K(dts, res, p.depth_tolerance, p.arrival_threshold);
        std::vector<R> hf3c(h.size(), R(0));
        for (size_t o = 0; o < outlet_idx.size(); ++o) hf3c[outlet_idx[o]] = hf3[o];
        R vmax = R(0), cmax = R(0);
#pragma omp parallel
        {
        R tv = R(0), tc = R(0);
#pragma omp for schedule(static)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t c = at(i, j);
                R sx = hfx[c] < K.tol ? K.big_depth : hfx[c];
                R sy = hfy[c] < K.tol ? K.big_depth : hfy[c];
                R vr = qdiv(qx[c], sx);
                R vu = qdiv(qy[c], sy);
                R vb = R(0);
                if (i + 1 < ny) {
                    size_t cb = at(i + 1, j);
                    R sb = hfy[cb] < K.tol ? K.big_depth : hfy[cb];
                    vb = qdiv(qy[cb], sb);
                }
                if (hz_on) vras[c] = std::fmax(std::fmax(std::fabs(vr), std::fabs(vu)), std::fabs(vb));
                R rc = (j == 0) ? K.half * vr : vr;
                R uc = K.half * (vu + vb);
                R tot = std::sqrt(rc * rc + uc * uc);
                tv = std::fmax(tv, tot);
                if (tot >= K.stagnant) {
                    R dts_ = std::fmax(std::fmax(hfx[c], hfy[c]), hf3c[c]);
                    R wc = std::fmax(std::sqrt(K.g * std::fmax(dts_, R(0))), K.celer_floor);
                    if (p.flag_adaptive_timestepping != 1) {
                        R ras = std::fmax(std::fmax(std::fabs(vr), std::fabs(vu)), std::fabs(vb));
                        wc = ras + wc;
                    }
                    tc = std::fmax(tc, wc);
                }
            }
#pragma omp critical
        {
            vmax = std::fmax(vmax, tv);
            cmax = std::fmax(cmax, tc);
        }
        }
        *vmax_out = double(vmax);
        return finalize_dt(double(vmax), double(cmax));
    }

    double finalize_dt(double vmax, double cmax) const {
        double dt_adv;
        if (vmax > 0) {
            dt_adv = 1.0 * res / std::max(vmax, 1e-10);
            double tsf = std::max(p.alfa_max - 2.0 * std::max(vmax - 5.0, 0.0), p.alfa_min);
            dt_adv = std::min(dt_adv * tsf, max_dt());
        } else {
            dt_adv = max_dt();
        }
        double dt_wave = cmax > 0 ? (p.alfa_min * res) / cmax : max_dt();
        double nw = p.flag_timestep == 1 ? std::min(dt_adv, dt_wave) : dt_wave;
        if (std::isnan(nw) || std::isinf(nw)) nw = max_dt();
        double tcr = std::max(p.time_step_increments * std::floor(nw / p.time_step_increments),
                              p.min_time_step);
        return std::min(tcr, max_dt());
    }

    void track(double t_end_s) {
        R thr = R(p.arrival_threshold / 1000.0);
        R te = R(t_end_s);
#pragma omp parallel for schedule(static)
        for (size_t c = 0; c < h.size(); ++c) {
            if (dmax[c] < thr && h[c] >= thr) arrival[c] = te;
            dmax[c] = std::fmax(h[c], dmax[c]);
        }
    }

    // ---------------- map records (save_output_maps.m:25-27, :160-166) ----------------
    // after a step whose t_save = t + new dt passes a record time (index above rec_last),
    // the depth after the step is kept with the step's clock
    std::vector<double> rec_times;
    int rec_last = 0;
    std::vector<std::vector<R>> rec_maps;
    std::vector<double> rec_t;
    void set_map_records(int nt, const double* times) {
        rec_times.assign(times, times + nt);
        rec_maps.clear();
        rec_t.clear();
        rec_last = nt > 0 ? last_below(t_min) : 0;
    }
    int last_below(double t) const {   // last index with rec_times[i] < t, -1 if none
        int idx = -1;
        for (size_t i = 0; i < rec_times.size(); ++i)
            if (rec_times[i] < t) idx = int(i);
        return idx;
    }

    // ---------------- failure handling (HydroPol2D_Main_While.m:926-993) ----------------
    // A step is rejected when more cells end it with a depth that is non-finite or below
    // -depth_tolerance than had a non-finite depth when the call began (idx_nan walls), or when
    // the test hook asks for it.  The rejected attempt is undone (d_t = d_p, I_t = I_p, and the
    // clock, counters and volumes it touched) and retried as the catch block does: clock back
    // by the step, catch_index + 1, new step factor * alfa_min * dx / celerity with
    // factor = 1/catch_index/factor_reduction and celerity sqrt(g max(max(d_tot), max(d_p)))
    // (+ the last refresh's maximum velocity when flag_adaptive_timestepping = 0), max_time_step
    // lowered to 1.5 x the new step, the new step capped by it (infinite -> min_time_step), the
    // rain interval [rewound clock, new clock].  The velocity and hazard maxima keep the
    // attempt's contribution (as the library's in-place maps do).
    int refresh_every = 1;          // temporal blocking K: refresh on step 1 and when (k-1) % K == 0
    int64_t fault_k = -1;
    int fault_n = 0;
    int catch_index = 1;
    double max_dt_eff = -1.0;       // running_control.max_time_step as lowered by retries [s]
    int max_retries = 8;
    double factor_reduction = 2.0;
    int dt_floor_stop = 0;
    int64_t retries = 0, rej_k = -1;
    int rej_n = 0;
    uint64_t n_bad0 = 0;
    double max_dt() const { return max_dt_eff > 0 ? max_dt_eff : p.max_time_step; }
    enum StepResult { kAccepted = 0, kRetried = 1, kDtFloor = 2, kFailed = 3 };

    // cells whose depth is non-finite (counted at the start of a call) / bad after a step
    uint64_t count_bad(bool after_step) const {
        uint64_t nb = 0;
        const R negtol = -R(p.depth_tolerance / 1000.0);
        for (size_t c = 0; c < h.size(); ++c)
            nb += after_step ? !(h[c] >= negtol) : !std::isfinite(double(h[c]));
        return nb;
    }
    // a non-finite depth in a cell of finite elevation: the state is unusable
    bool bad_domain() const {
        for (size_t c = 0; c < h.size(); ++c)
            if (!std::isfinite(double(h[c])) && !(c < wall.size() && wall[c])) return true;
        return false;
    }

    // ---------------- one accepted step (HydroPol2D_Main_While.m:403-782) ----------------
    // The step is carried in minutes, as the reference does (time_step, min), and the
    // seconds of the step are time_step*60 (Local_Inertial_Model_D4.m:201).
    int step() {
        // what a rejected attempt restores
        const std::vector<R> h0 = h, qx0 = qx, qy0 = qy, I0 = I, T0 = T, dmax0 = dmax, arr0 = arrival;
        const double sv[] = {rain_vol, inf_vol, out_vol, inflow_vol, stage_vol, struct_vol, tsp, vmax_last};
        const int64_t neg0 = neg_warn, uns0 = unstable;
        const size_t nrec0 = rec_maps.size();
        const int rec_last0 = rec_last;
        double dts = time_step * 60.0;
        hydrology(dts);
        R dmx = R(0);   // max(d_p, d_tot), NaN skipped
        for (size_t c = 0; c < h.size(); ++c) dmx = std::fmax(std::fmax(dmx, h0[c]), h[c]);
        li(dts, time_step);
        double pos_save = std::ceil((t_min * 60.0) / p.time_step_change);
        double time_save = (pos_save - 1.0) * p.time_step_change / 60.0;
        double delta = time_save - tsp;
        tsp = time_save;
        double tcr = time_step * 60.0;
        bool floor_hit = false;
        if ((delta > 0 || k == 1) && (refresh_every <= 1 || k == 1 || (k - 1) % refresh_every == 0)) {
            double vm;
            tcr = cfl(dts, &vm);
            vmax_last = vm;
            if (tcr == p.min_time_step) { ++unstable; floor_hit = true; }
        }
        apply_stage();
        track(t_min * 60.0 + dts);
        if (hz_on) track_hazard();
        bool reject = count_bad(true) > n_bad0;
        if (fault_n > 0 && k == fault_k) { --fault_n; reject = true; }
        if (reject) {
            h = h0; qx = qx0; qy = qy0; I = I0; T = T0; dmax = dmax0; arrival = arr0;
            rain_vol = sv[0]; inf_vol = sv[1]; out_vol = sv[2]; inflow_vol = sv[3]; stage_vol = sv[4];
            struct_vol = sv[5]; tsp = sv[6]; vmax_last = sv[7];
            neg_warn = neg0; unstable = uns0;
            rec_maps.resize(nrec0); rec_t.resize(nrec0); rec_last = rec_last0;
            if (k == rej_k) ++rej_n;
            else { rej_k = k; rej_n = 1; }
            if (rej_n > max_retries) { rej_n = 0; return kFailed; }
            const double wc = std::sqrt(kG * double(dmx));
            ++catch_index;
            const double factor = 1.0 / catch_index / factor_reduction;
            double nt = p.flag_adaptive_timestepping == 1 ? factor * (p.alfa_min * res / wc)
                                                          : factor * (p.alfa_min * res / (vmax_last + wc));
            if (catch_index > 1) max_dt_eff = std::fmin(nt * 1.5, max_dt());
            nt = std::fmin(nt, max_dt());
            if (std::isinf(nt)) nt = p.min_time_step;
            const double t0 = t_min - time_step;
            t_prev = t0;
            time_step = nt / 60.0;
            t_min = t0 + time_step;
            rain_a = t_prev;
            rain_b = t_min;
            ++retries;
            return kRetried;
        }
        if (!rec_times.empty()) {
            const int idx = last_below(t_min + tcr / 60.0);
            if (idx > rec_last) {
                rec_maps.push_back(h);
                rec_t.push_back(t_min);
                rec_last = idx;
            }
        }
        // the next step's rain interval: [t_previous, t] (HydroPol2D_Main_While.m:721), then
        // t_previous <- the increment on the first step, t after it (:734-738)
        rain_a = t_prev;
        rain_b = t_min;
        t_prev = k == 1 ? tcr / 60.0 : t_min;
        time_step = tcr / 60.0;
        t_min = tcr / 60.0 + t_min;
        ++k;
        return floor_hit && dt_floor_stop ? kDtFloor : kAccepted;
    }

    bool finished() const { return !(t_min <= p.routing_time + p.min_time_step / 60.0); }
};

}  // namespace hp2d_oracle
