// Device-side arithmetic of the surface-flow step, shared by the fused and the unfused
// kernels.  Every function here is the per-cell or per-face form of a reference line:
//   face_flux      Local_Inertial_Model_D4.m:31-44, :89-142 (split slope), :198,
//                  Inertial_Solver.m:24-25, LIM_D4.m:264, :272-275, :292-294
//   donor_scale    apply_coarse_draining_limiter, LIM_D4.m:814-829
//   limit_face     LIM_D4.m:831-857
//   continuity     LIM_D4.m:313-315, :389-393, :415
//   outlet_sink    LIM_D4.m:417-498
//   green_ampt     HydroPol2D_Main_While_Ensemble.m:274-298 with Infiltration_Module.m
//                  :179 and :444-445 (supply and depth update)
//   cfl_cell       refreshing_timestep.m:61-89, :139-150, :181-238
// The whole library is compiled with -fmad=false: every a*b+c below rounds twice unless it
// is written as fma() (one rounding, as std::fma on the CPU), so the results are
// reproducible on any IEEE machine that evaluates the same expressions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hp2d {

constexpr double kG = 9.81;

// ---------------- x^(-1/3) by a fixed Newton iteration -------------------------------
// Seed: dividing the IEEE exponent field by three (bits(x)/3 subtracted from the bits of
// 2^(4/3 * bias)), then r <- r + r (1 - x r^3) / 3, quadratically convergent.  The residual
// and the update are single fused multiply-adds (correctly rounded on every IEEE machine,
// so the CPU restatement reproduces them exactly).
template <typename R> struct RcbrtTraits;
template <> struct RcbrtTraits<float> {
    static constexpr int iters = 3;
};
template <> struct RcbrtTraits<double> {
    static constexpr int iters = 5;
};

__device__ __forceinline__ float bits_seed(float x) {
    uint32_t u = __float_as_uint(x);
    return __uint_as_float(0x54AAAAABu - u / 3u);
}
__device__ __forceinline__ double bits_seed(double x) {
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return __longlong_as_double((long long)(0x5540000000000000ull - u / 3ull));
}
__device__ __forceinline__ bool below_normal(float x) { return x < 1.17549435e-38f; }
__device__ __forceinline__ bool below_normal(double x) { return x < 2.2250738585072014e-308; }
template <typename R> __device__ __forceinline__ R sub_up();
template <> __device__ __forceinline__ float sub_up<float>() { return 16777216.0f; }
template <> __device__ __forceinline__ double sub_up<double>() { return 18014398509481984.0; }
template <typename R> __device__ __forceinline__ R sub_down();
template <> __device__ __forceinline__ float sub_down<float>() { return 256.0f; }
template <> __device__ __forceinline__ double sub_down<double>() { return 262144.0; }

template <typename R> __device__ __forceinline__ R rcbrt(R x) {
    R scale = R(1);
    if (below_normal(x)) { x = x * sub_up<R>(); scale = sub_down<R>(); }
    R r = bits_seed(x);
    const R third = R(1.0 / 3.0);
#pragma unroll
    for (int it = 0; it < RcbrtTraits<R>::iters; ++it) {
        R t = x * r;
        t = t * r;
        const R e = fma(-t, r, R(1));
        r = fma(r * e, third, r);
    }
    return r * scale;
}
template <typename R> __device__ __forceinline__ R pow73(R x) {
    if (!(x > R(0))) return R(0);
    R r = rcbrt(x);
    R c = x * (r * r);
    return (x * x) * c;
}
// ---------------- quotient a / b for b > 0 ---------------------------------------------
// FP32: the reciprocal from a bit-level seed (0x7EF311C3 minus the bits of b, relative
// error below 1/8), three Newton steps r <- r + r (1 - b r) (the error squares each step),
// then a r with one residual correction q + (a - b q) r.  Branch-free and built only from
// IEEE multiplies and fused multiply-adds, so the CPU restatement reproduces it bit for
// bit; within about one ulp of the IEEE quotient.  b is raised to the smallest normal
// float first (the seed needs a normal b; a quotient by anything smaller is either zero
// or discarded by the callers' clips).  FP64 uses the IEEE division.
__device__ __forceinline__ float qdiv(float a, float b) {
    b = fmaxf(b, 1.17549435e-38f);
    float r = __uint_as_float(0x7EF311C3u - __float_as_uint(b));
    float e = fmaf(-b, r, 1.0f);
    r = fmaf(r, e, r);
    e = fmaf(-b, r, 1.0f);
    r = fmaf(r, e, r);
    e = fmaf(-b, r, 1.0f);
    r = fmaf(r, e, r);
    const float q = a * r;
    return fmaf(fmaf(-b, q, a), r, q);
}
__device__ __forceinline__ double qdiv(double a, double b) { return a / b; }

// x^(7/3) for x > 0 (callers that have established it)
template <typename R> __device__ __forceinline__ R pow73_pos(R x) {
    R r = rcbrt(x);
    R c = x * (r * r);
    return (x * x) * c;
}
template <typename R> __device__ __forceinline__ R pow53(R x) {
    if (!(x > R(0))) return R(0);
    R r = rcbrt(x);
    R c = x * (r * r);
    return x * (c * c);
}

// ---------------- per-step constants (computed in FP64, rounded once) ------------------
template <typename R> struct StepConsts {
    R dt, gdt, dt_over_dx, dx_over_dt, inv_dt, inv_dx, g, tol, thr;
    __device__ __host__ void make(double dt_s, double res, double tol_mm, double thr_mm) {
        dt = R(dt_s);
        gdt = R(kG * dt_s);
        dt_over_dx = R(dt_s / res);
        dx_over_dt = R(res / dt_s);
        inv_dt = R(1.0 / dt_s);
        inv_dx = R(1.0 / res);
        g = R(kG);
        tol = R(tol_mm / 1000.0);
        thr = R(thr_mm / 1000.0);
    }
};

// ---------------- device state of the clock and of the step reductions ----------------
struct StepScalars {
    double t_min;          // clock at the start of the next step [min]
    double time_step;      // step the next step applies [min]; dt = time_step*60 s
                           // (Local_Inertial_Model_D4.m:201)
    double tsp;            // running_control.time_save_previous [min]
    long long k;           // step counter (1-based)
    int cur;               // which of the double buffers holds the state
    int skip_clamp;        // next step skips the 1e-6 mm clamp (Hydrological_Model.m:45-50)
    double vmax_last;      // velocities.max_velocity of the last refresh
    double rain_vol, inf_vol, out_vol;   // cumulative [m^3]
    long long neg_warn, unstable;
    unsigned int status;   // kStatus* bits
    unsigned int counter;  // CTAs done with the current step
    unsigned long long acc_vmax;   // max speed of the step (ordered bits)
    unsigned long long acc_cmax;   // max wave celerity of non-stagnant cells (ordered bits)
    double acc_rain, acc_inf, acc_out; // step sums [m] (times cell area later)
    int acc_neg;           // unfused path: some depth < -1e-8 mm after hydrology
    int pad;
    unsigned long long n_finite;   // cells with a finite depth (walls excluded)
    // rain of the current step: the depth update_spatial_BC computed over the clock interval
    // [rain_a, rain_b] at the end of the previous step, and the loop's t_previous [min]
    double rain_a, rain_b, t_prev;
    int skip_next;         // fused step: some outlet cell ends below -1e-11 m after the next rain
    int pad2;
    double inflow_vol;     // cumulative inflow-hydrograph volume [m^3]
    double stage_vol;      // cumulative volume the stage overwrites added [m^3]
    double acc_stage;      // step sum [m] (times cell area later)
    // map records (save_output_maps.m:25-27, :160-166): index of the last record time below
    // t_save, records taken, and whether the next step's input depth is to be recorded
    long long rec_count;
    int rec_last, rec_pending;
    double struct_vol;     // cumulative volume the control structures added [m^3]
    unsigned long long skipped_cells;   // cumulative cell records a fused step found unchanged
                                        // in its output buffer and did not rewrite
    unsigned long long skipped_read_cells;   // of those, cells of whole skipped row blocks
                                             // (their records were not read either)
    // Failure handling (HydroPol2D_Main_While.m:926-993).  A step is rejected when more cells
    // end it with a depth that is non-finite or below -depth_tolerance than had a non-finite
    // depth when the run started (idx_nan walls keep theirs), when a row copy timed out, or
    // when the host's test hook asks for it; a rejected step commits nothing (the state stays
    // in the buffer it was read from, the clock and counters stay) and halts the launches
    // until the host has prepared its retry.
    unsigned long long acc_bad;     // step sum: cells ending non-finite or too negative
    unsigned long long n_bad0;      // cells with a non-finite depth at the start of the run
    int halted;                     // 1: launches are no-ops until the host clears it
    int catch_index;                // the reference's catch_index (1 before any failure)
    long long fault_k;              // test hook: attempts of step fault_k are rejected ...
    int fault_n;                    // ... this many times
    int dt_floor_stop;              // 1: a step whose refreshed dt equals min_time_step halts after it
    double max_dt;                  // running_control.max_time_step [s], lowered by retries
    long long retries;              // rejected attempts so far
    unsigned long long retry_dmax;  // retry scan: max depth of d_p and d_tot [m] (ordered bits)
    int bad_domain;                 // start-of-run scan: a cell of finite elevation holds a
                                    // non-finite depth
    int refresh_every;              // temporal blocking K: the time step is refreshed only on step
                                    // 1 and on the steps k with (k - 1) % K == 0 (<= 1: every step)
    // the last step's reduced CFL maxima (ordered bits as acc_vmax / acc_cmax), whether it
    // refreshed the time step and whether that refresh hit min_time_step: a grid split into row
    // slabs redoes the refresh with the maxima of all slabs (hp2d_apply_refresh)
    unsigned long long last_vbits, last_cbits;
    int last_refreshed, last_unstable;
};
// StepScalars::status bits
constexpr unsigned kStatusNumerical = 1u;   // a step was rejected (non-finite / negative depth)
constexpr unsigned kStatusTimeout = 2u;     // a row copy did not land within the wait limit
constexpr unsigned kStatusDtFloor = 4u;     // the refreshed dt hit min_time_step (dt_floor_stop)

// ---------------- map records (save_output_maps.m) -----------------------------------
// After a step whose t_save = t + new dt passes a record time (time_records, 0-based index
// above rec_last), the depth d_t after that step is kept in slot rec_count % n_slots (the next
// step copies its input depth there, or the host when no step follows).
template <typename R> struct RecordDesc {
    int n_times, n_slots;
    const double* times;   // [n_times] [min], increasing
    R* snap;               // [n_slots][ny*nx] depth [m]
    double* snap_t;        // [n_slots] clock t of the step whose result the slot holds [min]
};
// last index i with times[i] < t (-1 when none)
__device__ __host__ inline int last_record_below(const double* times, int n, double t) {
    int lo = 0, hi = n;   // first index with times[i] >= t, by bisection
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (times[mid] < t) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}

// non-negative floats/doubles order like their bit patterns
__device__ __forceinline__ unsigned long long ord_bits(float v) { return (unsigned long long)__float_as_uint(v); }
__device__ __forceinline__ unsigned long long ord_bits(double v) { return (unsigned long long)__double_as_longlong(v); }
__host__ __device__ inline double from_ord(unsigned long long b, bool is_double) {
    if (is_double) {
        double d;
        memcpy(&d, &b, 8);
        return d;
    }
    unsigned int u = (unsigned int)b;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

// ---------------- vectorised cell records ---------------------------------------------
// static record  {dz_x, dz_y, n^2, meta}: meta holds, in the bits of the last element,
//                the soil class (bits 0-7, 255 = no soil) and outlet ordinal + 1 (bits
//                8-31, 0 = not an outlet cell)
// state record   {h, q_x, q_y, dmax}, double-buffered
// soil record    {I, T}, double-buffered (Green-Ampt runs only)
template <typename R> struct Vec;
template <> struct Vec<float> {
    using V4 = float4;
    using V2 = float2;
};
template <> struct Vec<double> {
    using V4 = double4;
    using V2 = double2;
};
__host__ __device__ inline unsigned meta_bits(float v) {
    unsigned u;
    memcpy(&u, &v, 4);
    return u;
}
__host__ __device__ inline unsigned meta_bits(double v) {
    unsigned long long u;
    memcpy(&u, &v, 8);
    return unsigned(u);
}
template <typename R> __host__ __device__ inline R make_meta(unsigned m);
template <> __host__ __device__ inline float make_meta<float>(unsigned m) {
    float f;
    memcpy(&f, &m, 4);
    return f;
}
template <> __host__ __device__ inline double make_meta<double>(unsigned m) {
    unsigned long long u = m;
    double d;
    memcpy(&d, &u, 8);
    return d;
}

// ---------------- bulk async copies (TMA, 1-D) into shared memory ----------------------
// Local-memory sources only (this GPU's global memory); no cluster multicast anywhere.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// retire a barrier whose every phase has completed, before its word is initialised again
__device__ __forceinline__ void mbar_inval(uint32_t bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false when the phase did not complete within `limit` polls
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// generic-proxy reads of a shared buffer complete before the async proxy rewrites it
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// bulk copy global -> shared, completion counted in bytes on `bar`; 16-byte aligned
// addresses, size a multiple of 16
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// ---------------- Green-Ampt soil class table -----------------------------------------
template <typename R> struct SoilClass {
    R ks, psi, dth, lu, kout, tr, minsm, pad;
};

struct OutletList {
    const int32_t* cell;     // sorted linear indices
    int32_t n;
};

// ---------------- rain ---------------------------------------------------------------
struct RainDesc {
    int n_uniform;           // entries in the uniform table (0 = none)
    const double* t_start;   // [min]
    const double* rate;      // [mm/h]
    int n_maps, my, mx;
    double map_dt;           // [min]
    const float* maps;       // n_maps * my * mx
    const double* map_t;     // null: map m over [m, m+1) x map_dt; else over [map_t[m], map_t[m+1]) [min]
};

// Integral [mm/h x min] over [a, b] of the uniform series: rate q holds from t_start[q] up to
// t_start[q+1] (the last one for ever); non-finite rates add nothing
// (update_spatial_BC.m:1131-1184 on the equivalent end-stamped series)
__device__ __host__ inline double uniform_integral(const RainDesc& rd, double a, double b) {
    double acc = 0.0;
    if (!(b > a)) return acc;
    for (int q = 0; q < rd.n_uniform; ++q) {
        const double lo = rd.t_start[q];
        const double hi = q + 1 < rd.n_uniform ? rd.t_start[q + 1] : b;
        const double ov = fmax(0.0, fmin(b, hi) - fmax(a, lo));
        if (ov > 0.0 && isfinite(rd.rate[q])) acc += rd.rate[q] * ov;
    }
    return acc;
}

template <typename R>
__device__ __forceinline__ R map_rate(const RainDesc& rd, const float* f, int i, int j, int ny, int nx);

// ---------------- inflow hydrographs (flag_inflow, update_spatial_BC.m:359-395) ----------
// Gauge g's rate [mm/h] holds from t_start[q] up to t_start[q+1] (the last for ever); a
// step adds to every cell of the gauge the integral over the step's rain interval / 60
// [mm] (delta_inflow_agg x inflow_cells), after the infiltration (Hydrological_Model.m:27-28).
// Inflow cells carry kInflowBit in their meta word and, in bits 8..30, their entry e: the
// cell's gauges are cell_gauge[cell_off[e] .. cell_off[e+1]) in increasing order.
constexpr unsigned kInflowBit = 0x80000000u;
// The same entries carry the stage-hydrograph cells (flag_stage_hydrograph,
// update_spatial_BC.m:316-357): cell_stage[e] is the stage gauge whose depth overwrites the
// cell's depth after the step (-1: none).
template <typename R> struct InflowDesc {
    int n_gauges, n_times;
    const double* t_start;      // [n_times] [min]
    const double* rate;         // [n_times][n_gauges] [mm/h]
    R* depth;                   // [n_gauges] this step's depth [m]
    const int32_t* cell_off;    // [entries + 1]
    const int32_t* cell_gauge;
    const double* gauge_cells;  // [n_gauges] cells of the gauge with a finite elevation
    int n_stage, n_stage_times;
    const double* stage_t;      // [n_stage_times] [min], start-stamped
    const double* stage_d;      // [n_stage_times][n_stage] water depth [m]
    R* stage_now;               // [n_stage] this step's stage depth [m]
    const int32_t* cell_stage;  // [entries]
    const int32_t* cell_struct; // [entries] control-structure slot of the cell (-1: none)
};
// stage depth of gauge g at clock t: the last record starting at or before t, else the
// first (update_spatial_BC.m:322-330)
template <typename R>
__device__ __host__ inline double stage_at(const InflowDesc<R>& d, int g, double t) {
    int z = 0;
    for (int q = 0; q < d.n_stage_times; ++q)
        if (d.stage_t[q] <= t) z = q;
    return d.stage_d[size_t(z) * d.n_stage + g];
}
template <typename R>
__device__ __host__ inline double inflow_integral(const InflowDesc<R>& d, int g, double a, double b) {
    double acc = 0.0;
    if (!(b > a)) return acc;
    for (int q = 0; q < d.n_times; ++q) {
        const double lo = d.t_start[q];
        const double hi = q + 1 < d.n_times ? d.t_start[q + 1] : b;
        const double ov = fmax(0.0, fmin(b, hi) - fmax(a, lo));
        const double r = d.rate[size_t(q) * d.n_gauges + g];
        if (ov > 0.0 && isfinite(r)) acc += r * ov;
    }
    return acc;
}
// adds the inflow depth [m] of the cell with meta word `meta` to hh (BC_States.inflow is the
// sum over the cell's gauges, added once); cells without inflow gauges are left alone
template <typename R> __device__ __forceinline__ void add_inflow(const InflowDesc<R>& d, unsigned meta, R& hh) {
    if (!(meta & kInflowBit)) return;
    const unsigned e = (meta >> 8) & 0x7FFFFFu;
    const int q0 = d.cell_off[e], q1 = d.cell_off[e + 1];
    if (q0 == q1) return;
    R v = R(0);
    for (int q = q0; q < q1; ++q) v = v + d.depth[d.cell_gauge[q]];
    hh = hh + v;
}
// ---------------- reservoir / control structures (flag_reservoir) ----------------------
// Local_Inertial_Model_D4.m:318-344: structure i drains its reservoir cell through up to two
// rating curves Q = k (h - h_crest)^p into downstream cells ds1 and ds2, once per step, from
// the depth d_tot entering the step's fluxes.  As the reference, in structure order:
//   dtsup = d_tot(res)/1000 (with the earlier structures' additions to d_tot);
//   dh = min(k1 max(dtsup-h1,0)^k2 / A 1000 3600, 1000 max(dtsup-h1,0)/dt_h) dt_h [mm];
//   Vol_Flux(res) += dh/1000 A (the reservoir cell GAINS dh: the reference's sign);
//   dtsup -= dh/1000; d_tot(ds1) += dh; with a second structure d_tot(ds1) += dh again (the
//   reference adds the first transfer twice), then dh2 from (h2, k3, k4) as above,
//   Vol_Flux(res) += dh2/1000 A, d_tot(ds2) += dh2.
// Every addition lands in d_t = d_tot + 1000 Vol_Flux / A after the fluxes, so each taking
// cell ("slot") gets one extra depth that enters its continuity: hn = (h + extra) + flux term.
template <typename R> struct StructDesc {
    int n, n_slots;
    const double* coef;       // [n][6]: k1, h1, k2, k3, h2, k4
    const int32_t* slot;      // [n][3]: slot of the reservoir, ds1 and ds2 cells (-1: none)
    const int32_t* slot_cell; // [n_slots] linear cell index
    R* hres;                  // [n] depth of the reservoir cell entering the step [m] (scratch)
    double* acc;              // [2][n_slots] ds additions, Vol_Flux additions [mm] (scratch)
    R* extra;                 // [n_slots] the step's extra depth of the cell [m]
};
// time_step [min] of the step; area = cell area [m^2]; fills s.extra from s.hres; returns
// the volume [m^3] the extras add
template <typename R>
__device__ __host__ inline double structure_transfers(const StructDesc<R>& s, double time_step, double area) {
    double* ds = s.acc;
    double* rv = s.acc + s.n_slots;
    for (int q = 0; q < s.n_slots; ++q) ds[q] = rv[q] = 0.0;
    const double dt_h = time_step / 60.0;
    for (int i = 0; i < s.n; ++i) {
        const double* c = s.coef + 6 * size_t(i);
        const int sr = s.slot[3 * i], s1 = s.slot[3 * i + 1], s2 = s.slot[3 * i + 2];
        double dh = 0.0, dtsup = 0.0;
        if (s1 >= 0) {
            dtsup = (double(s.hres[i]) * 1000.0 + ds[sr]) / 1000.0;
            const double q = fmax(dtsup - c[1], 0.0);
            const double avail = 1000.0 * q / dt_h;
            dh = fmin(c[0] * pow(q, c[2]) / area * 1000.0 * 3600.0, avail) * dt_h;
            rv[sr] += dh;
            dtsup = dtsup - dh / 1000.0;
            ds[s1] += dh;
        }
        if (s2 >= 0) {
            ds[s1] += dh;
            const double q = fmax(dtsup - c[4], 0.0);
            const double avail = 1000.0 * q / dt_h;
            const double dh2 = fmin(c[3] * pow(q, c[5]) / area * 1000.0 * 3600.0, avail) * dt_h;
            rv[sr] += dh2;
            ds[s2] += dh2;
        }
    }
    double vol = 0.0;
    for (int q = 0; q < s.n_slots; ++q) {
        const R e = R((ds[q] + rv[q]) / 1000.0);
        s.extra[q] = e;
        vol += double(e) * area;
    }
    return vol;
}
// outlet entry + 1 of a meta word (0: not an outlet)
__device__ __host__ inline unsigned outlet_ord(unsigned meta) { return (meta & kInflowBit) ? 0u : meta >> 8; }

// Rain of one step over the clock interval [a, b] [min]: a uniform depth, or the (at most
// two) rate maps overlapping the interval with their overlaps (map m holds over
// [m, m+1) x map_dt, or over [map_t[m], map_t[m+1]) for end-stamped input maps, nothing
// after the last map; update_spatial_BC.m:1287-1359).  Depths are rate [mm/h] x
// overlap [min] / 60 [mm], in metres.
template <typename R> struct RainStep {
    R depth;       // uniform series [m]
    int nm;        // maps overlapping the interval (0..2)
    int m[2];
    R w[2];        // overlap / 60000: mm/h -> m
    __device__ __host__ void make(const RainDesc& rd, double a, double b) {
        depth = rd.n_uniform ? R(uniform_integral(rd, a, b) / 60000.0) : R(0);
        nm = 0;
        m[0] = m[1] = 0;
        w[0] = w[1] = R(0);
        if (!rd.n_maps || !(b > a)) return;
        int m0;
        if (rd.map_t) {   // the first map that ends after a
            int lo = 0, hi = rd.n_maps;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (rd.map_t[mid + 1] > a) hi = mid;
                else lo = mid + 1;
            }
            m0 = lo;
        } else {
            m0 = max(0, int(floor(a / rd.map_dt)) - 1);
        }
        for (int q = m0; q < rd.n_maps && nm < 2; ++q) {
            const double lo = rd.map_t ? rd.map_t[q] : q * rd.map_dt;
            const double hi = rd.map_t ? rd.map_t[q + 1] : (q + 1) * rd.map_dt;
            if (lo >= b) break;
            const double ov = fmin(b, hi) - fmax(a, lo);
            if (ov > 0.0) {
                m[nm] = q;
                w[nm] = R(ov / 60000.0);
                ++nm;
            }
        }
    }
    // depth [m] the step adds at cell (i, j)
    __device__ R at(const RainDesc& rd, int i, int j, int ny, int nx) const {
        if (!rd.n_maps) return depth;
        if (nm == 0) return R(0);
        R r = w[0] * map_rate<R>(rd, rd.maps + size_t(m[0]) * rd.my * rd.mx, i, j, ny, nx);
#pragma unroll 1
        for (int q = 1; q < nm; ++q)   // a step across a map boundary (one sampler in the code)
            r = r + w[q] * map_rate<R>(rd, rd.maps + size_t(m[q]) * rd.my * rd.mx, i, j, ny, nx);
        return r;
    }
};


template <typename R>
__device__ __forceinline__ R map_rate(const RainDesc& rd, const float* f, int i, int j, int ny, int nx) {
    const R half = R(0.5);
    R fy = (R(i) + half) * R(double(rd.my) / ny) - half;
    R fx = (R(j) + half) * R(double(rd.mx) / nx) - half;
    fy = fmin(fmax(fy, R(0)), R(rd.my - 1));
    fx = fmin(fmax(fx, R(0)), R(rd.mx - 1));
    int iy0 = (int)floor(fy), ix0 = (int)floor(fx);
    int iy1 = min(iy0 + 1, rd.my - 1), ix1 = min(ix0 + 1, rd.mx - 1);
    R wy = fy - R(iy0), wx = fx - R(ix0);
    R f00 = R(f[iy0 * rd.mx + ix0]), f01 = R(f[iy0 * rd.mx + ix1]);
    R f10 = R(f[iy1 * rd.mx + ix0]), f11 = R(f[iy1 * rd.mx + ix1]);
    R top = (R(1) - wx) * f00 + wx * f01;
    R bot = (R(1) - wx) * f10 + wx * f11;
    return (R(1) - wy) * top + wy * bot;
}

// ---------------- Green-Ampt (one cell) -----------------------------------------------
// h [m] after rain; I [m]; T [s]; returns infiltrated depth [m]; updates h, I, T.
template <typename R>
__device__ __forceinline__ R green_ampt(R& hh, R& Ic, R& Tc, const SoilClass<R>& s, const StepConsts<R>& K) {
    R Ip = Ic;
    R C = s.ks * (R(1) + ((hh + s.psi) * s.dth) / Ip);
    if (Ip > s.lu) C = s.ks;
    R ia = hh * K.inv_dt;
    bool idxC = ia <= C;
    R Tn = Tc - K.dt;
    if (ia > C) Tn = s.tr;
    bool idxT = Tn < R(0);
    R f = fmin(C, ia);
    R In = Ip + f * K.dt;
    if (idxC) In = In - s.kout * K.dt;
    In = fmax(In, s.minsm);
    if (idxT) In = s.minsm;
    Ic = In;
    Tc = Tn;
    R fd = f * K.dt;
    hh = hh - fd;
    if (hh < R(0)) hh = R(0);
    return fd;
}

// ---------------- van Genuchten-Mualem Darcy closure (one cell) ------------------------
// The single-layer branch of the current Infiltration_Module.m (:143-473), in SI units:
// h [m] after rain, I = soil storage I_t [m], zwt = depth to the water table [m]
// (:192-199, from the soil depth, groundwater head and elevation; static here).  Returns
// the infiltrated depth [m]; updates h and I.  Powers with non-integer exponents use the
// CUDA math library (not reproduced bit for bit by the CPU restatement).
template <typename R> struct SoilClassVG {
    R ks;         // saturated conductivity [m/s]
    R theta_r, theta_s, alpha;   // residual / saturated water content [-], alpha [1/m]
    R inv_n, m, inv_m, pad;      // 1/n, m = 1 - 1/n, 1/m
};
template <typename R> struct VGGlobals {
    R ell, ltop, dh_max, wk;     // Mualem l, Ltop [m] (>= 1e-6), dh_max [m], Ksurf_weight in [0, 1]
};
__device__ __forceinline__ float rpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double rpow(double a, double b) { return pow(a, b); }

template <typename R>
__device__ __forceinline__ R vg_infiltration(R& hh, R& Ic, R zwt, const SoilClassVG<R>& s, const VGGlobals<R>& g,
                                             const StepConsts<R>& K) {
    const R ia = hh * K.inv_dt;                              // supply rate (:179) [m/s]
    const R h0 = fmax(hh, R(0));                             // ponding head (:182)
    const R dth = s.theta_s - s.theta_r;
    const R uzmax = zwt * dth;                               // :205-206
    const R S = fmax(Ic, R(0));                              // :209
    const R srem = fmax(uzmax - S, R(0));                    // :214
    const bool no_uz = !(zwt > R(0)) || !(uzmax > R(0));    // :217
    const R zs = fmax(zwt, R(1e-6));
    R tb = s.theta_r + S / zs;                               // :262-265
    tb = fmin(fmax(tb, s.theta_r), s.theta_s);
    const R dsafe = fmax(dth, R(1e-12));
    R seb = fmin(fmax((tb - s.theta_r) / dsafe, R(1e-6)), R(1));
    R hb = -(R(1) / s.alpha) * rpow(rpow(seb, -s.inv_m) - R(1), s.inv_n);   // :272-276
    if (seb >= R(0.999999)) hb = R(0);
    const R w_avail = h0;                                    // :281
    const R w_def = g.ltop * fmax(s.theta_s - tb, R(0));     // :292 (Lmix = Ltop)
    R w_wet = fmin(w_avail, srem);
    w_wet = fmax(fmin(w_wet, w_def), R(0));
    R tt = tb + w_wet / g.ltop;                              // :300-302
    tt = fmin(fmax(tt, s.theta_r), s.theta_s);
    const R set = fmin(fmax((tt - s.theta_r) / dsafe, R(1e-6)), R(1));
    R term = R(1) - rpow(set, s.inv_m);                      // :307-309
    term = fmin(fmax(term, R(0)), R(1));
    const R om = R(1) - rpow(term, s.m);
    R kr = rpow(set, g.ell) * (om * om);
    kr = fmin(fmax(kr, R(0)), R(1));
    const R ktop = s.ks * kr;
    R ksoil = ktop;                                          // :326-333
    if (ia > R(0) || h0 > R(0)) ksoil = g.wk * s.ks + (R(1) - g.wk) * ktop;
    ksoil = fmin(fmax(ksoil, R(0)), s.ks);
    const R dh = fmin(fmax(h0 - hb, R(0)), g.dh_max);        // :336-338
    const R cap = ksoil * (dh / g.ltop + R(1));              // :340-342
    const R flim = srem * K.inv_dt;                          // :345
    R f = fmin(fmin(ia, cap), flim);                         // :347-352
    if (no_uz || isnan(f)) f = R(0);
    f = fmax(f, R(0));
    const R fd = f * K.dt;                                   // :356-365
    Ic = fmax(fmin(Ic + fd, uzmax), R(0));
    hh = hh - fd;                                            // :371-372
    if (hh < R(0)) hh = R(0);
    return fd;
}

// momentum term of schemes 2 and 3 for a face with Hf > 0 (see face_flux)
template <typename R>
__device__ __forceinline__ R diffused_momentum(R qp, R q_lo, R q_hi, R Hf, const StepConsts<R>& K, int scheme) {
    const R th = R(1) - K.dt_over_dx * fmin(qdiv(fabs(qp), Hf), sqrt(K.g * Hf));
    const R qnb = scheme == 2 ? (qp < R(0) ? q_hi : q_lo) : R(0.5) * (q_lo + q_hi);
    return th * qp + (R(1) - th) * qnb;
}

// ---------------- one face of the local-inertial momentum update ----------------------
// x face: (ha, hb) = (left, right) cells, dz = z_right - z_left.
// y face: (ha, hb) = (upper, lower) cells (row i-1, row i), dz = z_upper - z_lower.
// Closed faces carry a non-finite dz: +inf on the domain edge (Hf(:,end) = 0 and
// Hf(1,:) = 0, Local_Inertial_Model_D4.m:139-140) and NaN next to a cell outside the
// domain (idx_nan, NaN elevation).  There MATLAB's max ignores the NaN, so the face depth
// is the inside cell's depth (:133-134) while the NaN slope sends q to 0 (:264); that
// depth still enters the wave celerity of refreshing_timestep.
// Faces that carry no water leave early: whole warps of them skip the power and the
// division, which matters on wet/dry fronts.
//
// SCH = 0: Bates (flag_numerical_scheme 1, Inertial_Solver.m:23-26).  SCH = 1: the schemes
// with numerical diffusion chosen at run time by `scheme` (Inertial_Solver.m:29-121): the
// momentum term q_p of the numerator becomes theta q_p + (1 - theta) q_nb with
//   theta = 1 - dt/dx min(|q_p|/Hf, sqrt(g Hf))           (:61, :84; NaN -> 1 at :86 is
//                                                          never reached for Hf > 0)
//   q_nb  = q_lo if q_p >= 0, else q_hi                    (scheme 2, s-upwind, :35-58)
//   q_nb  = (q_lo + q_hi) / 2                              (scheme 3, s-centred, :91-98)
// where q_lo / q_hi are the previous fluxes of the same direction one face before / after
// (x: columns j-1, j+1; y: rows i-1, i+1), zero on the first and last column (x) or row
// (y), as the reference's interior ranges 2:(end-1) leave them.  The friction term keeps
// |q_p| (total_flux = q_p, :31, :101).
template <typename R, bool IS_X, int SCH = 0>
__device__ __forceinline__ void face_flux(R ha, R hb, R dz, R qp, R n2c, const StepConsts<R>& K,
                                          int flag_critical, R& Hf, R& q, int scheme = 1, R q_lo = R(0),
                                          R q_hi = R(0)) {
    if (!(fabs(dz) <= R(3.0e38))) {
        // NaN dz: MATLAB's max over the two sides skips the NaN one
        Hf = isnan(dz) ? fmax(fmax(ha, hb), R(0)) : R(0);
        q = R(0);
        return;
    }
    ha = fmax(ha, R(0));
    hb = fmax(hb, R(0));
    R S;
    if (IS_X) {
        Hf = fmax(fmax(ha - fmax(dz, R(0)), hb + fmin(dz, R(0))), R(0));
        S = (dz + (hb - ha)) * K.inv_dx;
    } else {
        Hf = fmax(fmax(ha + fmin(dz, R(0)), hb - fmax(dz, R(0))), R(0));
        S = (dz + (ha - hb)) * K.inv_dx;
    }
    if (!(Hf > R(0))) { q = R(0); return; }
    R qn = qp;
    if (SCH) qn = diffused_momentum(qp, q_lo, q_hi, Hf, K, scheme);
    R num = fma(-(K.gdt * Hf), S, qn);   // one rounding for qn - (g dt Hf) S
    R h73 = pow73_pos(Hf);
    R den = fma(K.gdt * n2c, fabs(qp), h73);
    R qq = qdiv(num * h73, den);
    if (!isfinite(qq)) qq = R(0);
    if (flag_critical == 1) {
        R crit = Hf * sqrt(K.g * Hf);
        qq = fmin(fmax(qq, -crit), crit);
    }
    R thr = Hf * R(10);
    q = fmin(fmax(qq, -thr), thr);
}

// face_flux split in two for the fused kernel's interleaved faces: face_geom gives the face
// depth Hf, the slope S and whether the face carries water (open and Hf > 0); face_momentum is
// the update of a wet face, written without branches so that the independent faces of a row
// (two directions, CPL cells per lane) can be interleaved.  For a wet face the two together
// perform the same operations on the same values as face_flux; a face that is not wet is given
// q = 0 (its momentum is evaluated on harmless operands and discarded).
template <typename R, bool IS_X>
__device__ __forceinline__ bool face_geom(R ha, R hb, R dz, R& Hf, R& S, const StepConsts<R>& K) {
    const bool open = fabs(dz) <= R(3.0e38);
    const R a = fmax(ha, R(0)), b = fmax(hb, R(0));
    R Ho;
    if (IS_X) {
        Ho = fmax(fmax(a - fmax(dz, R(0)), b + fmin(dz, R(0))), R(0));
        S = (dz + (b - a)) * K.inv_dx;
    } else {
        Ho = fmax(fmax(a + fmin(dz, R(0)), b - fmax(dz, R(0))), R(0));
        S = (dz + (a - b)) * K.inv_dx;
    }
    // closed faces: NaN dz (next to an idx_nan cell) keeps the inside cell's depth, +inf none
    Hf = open ? Ho : (isnan(dz) ? fmax(fmax(ha, hb), R(0)) : R(0));
    return open && Ho > R(0);
}
template <typename R, int SCH = 0>
__device__ __forceinline__ R face_momentum(bool wet, R Hf, R S, R qp, R n2c, const StepConsts<R>& K, int flag_critical,
                                           int scheme = 1, R q_lo = R(0), R q_hi = R(0)) {
    const R H = wet ? Hf : R(1);
    const R Sl = wet ? S : R(0);
    R qn = qp;
    if (SCH) qn = diffused_momentum(qp, q_lo, q_hi, H, K, scheme);
    const R num = fma(-(K.gdt * H), Sl, qn);
    const R h73 = pow73_pos(H);
    const R den = fma(K.gdt * n2c, fabs(qp), h73);
    R qq = qdiv(num * h73, den);
    qq = isfinite(qq) ? qq : R(0);
    if (flag_critical == 1) {
        const R crit = H * sqrt(K.g * H);
        qq = fmin(fmax(qq, -crit), crit);
    }
    const R thr = H * R(10);
    qq = fmin(fmax(qq, -thr), thr);
    return wet ? qq : R(0);
}

// outgoing rate of a cell over its four faces and its donor scale factor
template <typename R>
__device__ __forceinline__ R donor_scale(R qR, R qL, R qU, R qD, R hc, const StepConsts<R>& K) {
    R out = fmax(qR, R(0));
    out = out + fmax(-qL, R(0));
    out = out + fmax(qU, R(0));
    out = out + fmax(-qD, R(0));
    R avail = fmax(hc, R(0)) * K.dx_over_dt;
    R s = R(1);
    if (out > avail && out > R(0)) s = avail / out;
    if (!isfinite(s)) s = R(0);
    return fmax(fmin(s, R(1)), R(0));
}

// donor_scale without the checks that cannot fire when the four faces are finite:
// avail >= 0, so out > avail implies out > 0 and 0 <= avail/out <= 1 (a finite value
// that the clamps and the NaN test of donor_scale leave unchanged)
template <typename R>
__device__ __forceinline__ R donor_scale_finite(R qR, R qL, R qU, R qD, R hc, const StepConsts<R>& K) {
    R out = fmax(qR, R(0));
    out = out + fmax(-qL, R(0));
    out = out + fmax(qU, R(0));
    out = out + fmax(-qD, R(0));
    const R avail = fmax(hc, R(0)) * K.dx_over_dt;
    return out > avail ? avail / out : R(1);
}
// limit_face for a finite q and scales in [0, 1] (the product is finite)
template <typename R>
__device__ __forceinline__ R limit_face_finite(R q, R s_pos, R s_neg) {
    return q > R(0) ? q * s_pos : (q < R(0) ? q * s_neg : q);
}

// face limited by the scale of its donor cell; s_pos = donor when q > 0
template <typename R>
__device__ __forceinline__ R limit_face(R q, R s_pos, R s_neg) {
    if (q > R(0)) q = q * s_pos;
    else if (q < R(0)) q = q * s_neg;
    if (!isfinite(q)) q = R(0);
    return q;
}

template <typename R>
__device__ __forceinline__ R continuity(R htot, R qL, R qR, R qU, R qD, const StepConsts<R>& K) {
    // separately rounded product and sum, as the reference evaluates it: a cell drained by
    // the limiter then ends at (or clamps to) zero alike in FP32 and FP64
    R hn = htot + K.dt_over_dx * (((qL - qR) - qU) + qD);
    if (hn < R(0)) hn = R(0);
    return hn;
}

// outlet sink; coef = sqrt|S|/(n dx) (type 1) or sqrt(g)/dx (type 2)
template <typename R>
__device__ __forceinline__ R outlet_sink(R& hn, R coef, int outlet_type, const StepConsts<R>& K, R& hout) {
    hout = fmax(hn, R(0));
    R qq = outlet_type == 1 ? coef * pow53(hout) : coef * (hout * sqrt(hout));
    R qmax = hout * K.inv_dt;
    qq = fmin(qq, qmax);
    if (!isfinite(qq)) qq = R(0);
    hn = hn - qq * K.dt;
    return qq;
}

// CFL contribution of one cell: speed and (if not stagnant) wave celerity
template <typename R>
__device__ __forceinline__ void cfl_cell(R qx, R qy, R qyb, R hfx, R hfy, R hfyb, R hf3, bool first_col,
                                         int adaptive, const StepConsts<R>& K, R& speed, R& celer) {
    const R big = R(1e9);
    R sx = hfx < K.tol ? big : hfx;
    R sy = hfy < K.tol ? big : hfy;
    R sb = hfyb < K.tol ? big : hfyb;
    R vr = qdiv(qx, sx);
    R vu = qdiv(qy, sy);
    R vb = qdiv(qyb, sb);
    R rc = first_col ? R(0.5) * vr : vr;
    R uc = R(0.5) * (vu + vb);
    speed = sqrt(rc * rc + uc * uc);
    celer = R(0);
    if (speed >= R(0.01)) {
        R dts = fmax(fmax(hfx, hfy), hf3);
        R wc = fmax(sqrt(K.g * fmax(dts, R(0))), R(1e-10));
        if (adaptive != 1) wc = fmax(fmax(fabs(vr), fabs(vu)), fabs(vb)) + wc;
        celer = wc;
    }
}

// binary search of a sorted outlet list; returns ordinal or -1
__device__ __forceinline__ int find_outlet(const int32_t* cells, int n, int c) {
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = __ldg(cells + mid);
        if (v == c) return mid;
        if (v < c) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

}  // namespace hp2d
