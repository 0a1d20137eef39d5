// Fused surface-flow step: one launch = one accepted step of HydroPol2D_Main_While.m
// :403-782 (rain + Green-Ampt + clamp, local-inertial fluxes, draining limiter,
// continuity, outlet sink, running maximum / arrival time, CFL reductions, and the
// timestep refresh + clock advance done by the last CTA to finish).
//
// Warp-streaming layout.  Each warp owns a strip of 32*CPL columns (CPL = 1 or 2 cells per
// lane; cell h of lane L sits at column 32h + L), of which all but two columns on each side
// are its output, and walks down a block of rows.  The draining limiter makes a cell's new
// depth depend on cells two away (face <- donor scale <- donor's four faces <- their far
// cells); in x those neighbours come from other lanes by warp shuffles (hence the
// two-column apron on each side), in y from a rolling window of registers that holds the
// previous two rows.  Per row a lane does, for each of its cells: hydrology of (r, j), the
// x face (r, j) and y face (r-1|r, j), the donor scale of (r-1, j), the limited faces of
// row r-1 and the continuity / outlet / maxima / CFL of row r-2.  No CTA barrier inside the
// row loop.
//
// Memory: a cell is two 16-byte records -- the static {dz_x, dz_y, n^2, meta} and the
// state {h, q_x, q_y, dmax} -- read and one state record written.  A strip's records of one
// row are contiguous, so one 1-D bulk copy (TMA) brings each record row into a per-warp
// ring of shared-memory stages, counted in bytes by the stage's mbarrier; the rows after
// row k are in flight while row k is computed.
//
// Dry rows: a vote per row tells whether the strip's depths are all zero after the
// hydrology.  Faces and limiter are skipped when rows r-2..r are dry, continuity and CFL
// when rows r-3..r-1 are, and a row r with rows r-3..r dry (deep-dry) only writes row r-2's
// zero depth and fluxes and its running maximum; each shortcut stores exactly what the
// full computation would.
//
// CFL reductions: the step needs max(speed) and, over non-stagnant cells, max of the wave
// celerity sqrt(g*depth).  Because IEEE sqrt is correctly rounded and monotone, max of
// sqrt(x_i) equals sqrt(max x_i) exactly, so the kernel reduces speed^2 and g*depth and
// takes one square root at the end; the stagnant test speed < 0.01 becomes
// speed^2 < stag_s2 with stag_s2 the smallest value whose rounded root reaches 0.01.
//
// The state is double-buffered (StepScalars::cur selects the read side), so a CUDA graph
// of many launches needs no host involvement, and a launch after the end of the
// simulation is a no-op that leaves the buffers and the clock alone.
#pragma once

#include "hp2d_device.cuh"

namespace hp2d {

constexpr int kStripOut = 28;   // output columns of a 32-lane strip (lanes 2..29)
#ifndef HP2D_STAGES
#define HP2D_STAGES 4
#endif
constexpr int kStages = HP2D_STAGES;   // shared-memory ring depth of the row pipeline
#ifndef HP2D_ROW_UNROLL
#define HP2D_ROW_UNROLL 1
#endif
constexpr int kRowUnroll = HP2D_ROW_UNROLL;   // row-loop unroll (register renaming of the window)
#ifndef HP2D_FACE_ILP
#define HP2D_FACE_ILP 1   // 1: interleaved faces in every instantiation, 0: infiltration / rain maps only, -1: none
#endif
// The faces of a row as interleaved, branch-free momentum updates (face_geom + face_momentum)
// rather than one face_flux after the other: measured faster on every workload (wet 2048^2 40.2
// vs 39.1 GCUPS, 60-minute dam-break 98.3 vs 96.3, Green-Ampt + rain maps 21.4 vs 21.0).
template <int INF, bool MAP> constexpr bool kFaceIlp = HP2D_FACE_ILP > 0 || (HP2D_FACE_ILP == 0 && (INF != 0 || MAP));
// Phase (F) without a per-lane branch around each cell's body (stores and reductions masked
// instead), so that the CPL cells interleave: wet 2048^2 41.6 vs 40.8 GCUPS, 60-minute dam-break
// 115.5 vs 111.8, 128-member ensemble 44.6 vs 43.0; the Green-Ampt + rain-map instantiation ran
// 20.3 vs 21.2 with it and keeps the branch.
template <int INF, bool MAP> constexpr bool kFlatF = INF == 0 && !MAP;

// dynamic shared memory of k_fused_step: per warp kStages x (2 records x 32*CPL cells)
template <typename R, int CPL = 1> constexpr size_t fused_smem_bytes(int nt) {
    return size_t(nt / 32) * kStages * 64 * CPL * sizeof(typename Vec<R>::V4);
}

template <typename R> struct FusedArgs {
    using V4 = typename Vec<R>::V4;
    using V2 = typename Vec<R>::V2;
    int ny, nx;
    int n_strips, rows_per_warp, n_warps_total;
    double res;
    double tol_mm, thr_mm;
    double t_end;                // routing_time + min_time_step/60 [min]
    double min_dt, max_dt, inc, tsc, alfa_min, alfa_max;
    int flag_timestep, adaptive, flag_critical, outlet_type, ga;   // ga: infiltration on (either model)
    int scheme;                  // flag_numerical_scheme: 1 Bates, 2 s-upwind, 3 s-centred
    unsigned int wait_polls;     // polls of a row-copy wait before it gives up (HP2D_TIMEOUT)
    int own_r0, own_r1;          // rows whose cells enter the CFL maxima, ledgers and checks (a
                                 // row slab's own rows; the others are halo rows of other slabs)
    unsigned int n_ctas;
    R stag_s2;
    const V4* stat;
    V4* st0; V4* st1;            // state records, double buffer
    V2* gs0; V2* gs1;            // soil records, double buffer
    const SoilClass<R>* classes;       // Green-Ampt classes
    const SoilClassVG<R>* classes_vg;  // van Genuchten classes
    VGGlobals<R> vg;
    const int32_t* outlet_cells; const R* outlet_coef; int n_outlets;
    R* hf3; R* qo;
    R* arrival;
    RainDesc rain;
    InflowDesc<R> inflow;
    RecordDesc<R> rec;
    StructDesc<R> strct;         // reservoir / control structures (n = 0: none)
    R* vmax; R* hzmax;           // velocity / hazard maxima [m/s], [m^2/s] (null: not tracked)
    // [2][n_strips][dry_rows]: 1 when a deep-dry row of the strip wrote its records into state
    // buffer b; the same row deep-dry again two steps later would write identical values
    // (null: off; dry_rows is ny rounded up to a multiple of 4, rows_per_warp <= 128 and a
    // multiple of 4, so that a warp reads its rows' flags as one word per lane)
    unsigned char* dryflag;
    int dry_rows;
    StepScalars* sc;
};

__device__ __host__ inline double finalize_dt(double vmax, double cmax, double res, double alfa_min,
                                              double alfa_max, double min_dt, double max_dt, double inc,
                                              int flag_timestep) {
    double dt_adv;
    if (vmax > 0) {
        dt_adv = 1.0 * res / fmax(vmax, 1e-10);
        double tsf = fmax(alfa_max - 2.0 * fmax(vmax - 5.0, 0.0), alfa_min);
        dt_adv = fmin(dt_adv * tsf, max_dt);
    } else {
        dt_adv = max_dt;
    }
    double dt_wave = cmax > 0 ? (alfa_min * res) / cmax : max_dt;
    double nw = flag_timestep == 1 ? fmin(dt_adv, dt_wave) : dt_wave;
    if (isnan(nw) || isinf(nw)) nw = max_dt;
    double tcr = fmax(inc * floor(nw / inc), min_dt);
    return fmin(tcr, max_dt);
}

// compensated (Kahan) running sum: s + c tracks the exact sum of the added terms to about one
// rounding of the state precision, however many terms (the library builds without contraction,
// so the compensation is not folded away)
template <typename R> struct Kahan {
    R s = R(0), c = R(0);
    __device__ __forceinline__ void add(R x) {
        const R y = x - c;
        const R t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return double(s) - double(c); }
};

template <typename R> __device__ __forceinline__ R warp_max(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R> __device__ __forceinline__ R bits_to(unsigned long long b);
template <> __device__ __forceinline__ float bits_to<float>(unsigned long long b) { return __uint_as_float((unsigned)b); }
template <> __device__ __forceinline__ double bits_to<double>(unsigned long long b) { return __longlong_as_double((long long)b); }

// Neighbour exchange across a warp's strip of 32*CPL columns (cell h of lane L sits at
// column 32h + L): value of the cell to the right / to the left.  With two cells per lane
// one indexed shuffle carries the value across the boundary between the two halves.
template <typename R, int CPL>
__device__ __forceinline__ void right_of(const R (&v)[CPL], R (&out)[CPL], int lane) {
    if (CPL == 1) {
        out[0] = __shfl_down_sync(0xffffffffu, v[0], 1);
    } else {
        out[0] = __shfl_sync(0xffffffffu, lane == 0 ? v[CPL - 1] : v[0], (lane + 1) & 31);
        out[CPL - 1] = __shfl_down_sync(0xffffffffu, v[CPL - 1], 1);
    }
}
template <typename R, int CPL>
__device__ __forceinline__ void left_of(const R (&v)[CPL], R (&out)[CPL], int lane) {
    if (CPL == 1) {
        out[0] = __shfl_up_sync(0xffffffffu, v[0], 1);
    } else {
        out[CPL - 1] = __shfl_sync(0xffffffffu, lane == 31 ? v[0] : v[CPL - 1], (lane + 31) & 31);
        out[0] = __shfl_up_sync(0xffffffffu, v[0], 1);
    }
}

// resident CTAs per SM the register budget is sized for (float: 8 x 128 threads)
#ifndef HP2D_MINB_F32
#define HP2D_MINB_F32 8
#endif
#ifndef HP2D_MINB_F32_PAIR
#define HP2D_MINB_F32_PAIR 4
#endif
template <typename R, int CPL = 1> struct FusedOcc { static constexpr int minb = CPL == 1 ? HP2D_MINB_F32 : HP2D_MINB_F32_PAIR; };
template <int CPL> struct FusedOcc<double, CPL> { static constexpr int minb = CPL == 1 ? 3 : 2; };

// One CTA-sized work item of the fused step: warps blk*NT/32 .. of the grid described by
// `a`.  k_fused_step runs item blockIdx.x of one grid; k_ens_step runs items of many grids
// pulled from a queue.  Every thread of the CTA calls it; it may return early for all of
// them together.  Returns false when a row copy timed out (the CTA must stop using its
// shared-memory ring).
// INF: infiltration model (0 none, 1 Green-Ampt, 2 van Genuchten); MAP: rain from coarse
// maps (else a uniform rate); INFL: inflow hydrographs present (the grids without them do not
// carry the lookup); SCH: 0 Bates faces, 1 the schemes with numerical diffusion
// (flag_numerical_scheme 2 or 3, a.scheme), whose faces also read the previous fluxes of the
// neighbouring faces of the same direction
// The depth d_tot a step hands to its fluxes at each control structure's reservoir cell --
// phase (A) of that cell restated: rain, infiltration, inflow, clamps, from the state and
// soil records `st`/`gs` the step starts from -- then the structures' transfers (one thread,
// in structure order).  The last CTA of a step runs it for the next step; k_struct_prime for
// the first step of a call.
template <typename R, int INF, bool MAP, bool INFL>
__device__ __noinline__ void structure_prepare(const FusedArgs<R>& a, const RainStep<R>& rs, bool skip,
                                               const StepConsts<R>& K, const typename Vec<R>::V4* st,
                                               const typename Vec<R>::V2* gs, int tid, int nt, double time_step) {
    for (int i = tid; i < a.strct.n; i += nt) {
        const int c = a.strct.slot_cell[a.strct.slot[3 * i]];
        const int r = c / a.nx, j = c % a.nx;
        R hh = st[c].x;
        const R rr = MAP ? rs.at(a.rain, r, j, a.ny, a.nx) : rs.depth;
        hh = hh + rr;
        const unsigned meta = meta_bits(a.stat[c].w);
        if (INF) {
            const unsigned scl = meta & 255u;
            if (scl != 255u) {
                R Ic = gs[c].x, Tc = gs[c].y;
                if (INF == 1) green_ampt(hh, Ic, Tc, a.classes[scl], K);
                else vg_infiltration(hh, Ic, Tc, a.classes_vg[scl], a.vg, K);
            }
        }
        if (INFL) add_inflow(a.inflow, meta, hh);
        if (!skip && hh < R(1e-9)) hh = R(0);
        if (hh < R(0)) hh = R(0);
        a.strct.hres[i] = hh;
    }
    __syncthreads();
    if (tid == 0) structure_transfers(a.strct, time_step, a.res * a.res);
}

template <typename R, int NT, int INF, bool MAP, int CPL = 1, bool INFL = false, int SCH = 0>
__device__ __forceinline__ bool fused_item(const FusedArgs<R>& a, const unsigned blk) {
    using V4 = typename Vec<R>::V4;
    using V2 = typename Vec<R>::V2;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ StepConsts<R> s_K;
    __shared__ double s_tmin, s_dts;
    __shared__ int s_cur, s_skip, s_done, s_last;
    __shared__ int s_negn;   // an outlet cell would go below -1e-11 m after the next rain
    __shared__ int s_rec;    // slot that receives this step's input depth (-1: none)
    __shared__ double s_stage;   // depth the stage overwrites of this CTA added [m]
    __shared__ unsigned s_skipw;  // cells whose unchanged record this CTA did not rewrite
    __shared__ unsigned s_skipr;  // of those, cells of skipped blocks (not read either)
    __shared__ RainStep<R> s_rs, s_rsn;   // this step's rain and the next one's
    __shared__ R red_s2[NT / 32];
    __shared__ unsigned long long red_c[NT / 32];
    __shared__ double red_d[3][NT / 32];
    __shared__ int red_to[NT / 32];
    __shared__ unsigned red_bad[NT / 32];
    __shared__ __align__(8) unsigned long long s_bar[NT / 32][kStages];
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    bool timed_out = false;

    const int tid = threadIdx.x;
    if (tid == 0) {
        StepScalars* sc = a.sc;
        s_tmin = sc->t_min;
        s_dts = sc->time_step * 60.0;
        s_cur = sc->cur;
        s_skip = sc->skip_clamp;
        s_negn = 0;
        s_stage = 0.0;
        s_skipw = 0u;
        s_skipr = 0u;
        s_rec = (sc->rec_pending && a.rec.n_slots > 0) ? int(sc->rec_count % a.rec.n_slots) : -1;
        s_done = !(s_tmin <= a.t_end) || sc->halted;
        s_K.make(s_dts, a.res, a.tol_mm, a.thr_mm);
        s_rs.make(a.rain, sc->rain_a, sc->rain_b);
        // the next step applies the rain of [t_previous, t] (HydroPol2D_Main_While.m:721)
        s_rsn.make(a.rain, sc->t_prev, s_tmin);
        if (!s_done && s_skip && blk == 0) sc->neg_warn += 1;
    }
    __syncthreads();
    if (s_done) return true;

    const StepConsts<R> K = s_K;
    const int ny = a.ny, nx = a.nx;
    const int cur = s_cur;
    const bool skip = s_skip != 0;
    const RainStep<R> RS = s_rs;
    const V4* __restrict__ sin = cur ? a.st1 : a.st0;
    V4* __restrict__ sout = cur ? a.st0 : a.st1;
    const V2* __restrict__ gin = cur ? a.gs1 : a.gs0;
    V2* __restrict__ gout = cur ? a.gs0 : a.gs1;
    const V4* __restrict__ stat = a.stat;
    const R t_arr = R(s_tmin * 60.0 + s_dts);
    const R NaNR = R(__int_as_float(0x7fc00000));

    const int lane = tid & 31, warp = tid >> 5;
    const int wg = int(blk) * (NT / 32) + warp;

    double rain_acc = 0.0, inf_acc = 0.0, out_acc = 0.0;
    // per-lane partial sums of the volume ledger in the state precision, Kahan-compensated
    // (the warps' sums and everything after them are FP64)
    Kahan<R> rain_acc_r, inf_acc_r, out_acc_r;
    unsigned nbad = 0u;                       // own cells ending non-finite or below -tol
    unsigned dry = 0u;                        // bit i: row r-i dry across the strip
    R s2max = R(0);
    R cmaxv = R(-1);   // largest celerity term of a non-stagnant cell (-1: none yet)

    if (wg < a.n_warps_total) {
        constexpr int SW = 32 * CPL;       // strip width: CPL cells per lane
        const int strip = wg % a.n_strips;
        const int rb = wg / a.n_strips;
        const int j_first = strip * (SW - 4) - 2;   // 2-column apron on each side
        int j[CPL];
        bool col_ok[CPL], own_lane[CPL];
#pragma unroll
        for (int h = 0; h < CPL; ++h) {
            j[h] = j_first + 32 * h + lane;
            col_ok[h] = j[h] >= 0 && j[h] < nx;
            own_lane[h] = (h > 0 || lane >= 2) && (h < CPL - 1 || lane < 30) && j[h] < nx;
        }
        const int r0 = rb * a.rows_per_warp;
        const int r_end = min(r0 + a.rows_per_warp, ny);
        unsigned char* const dfl =
            a.dryflag ? a.dryflag + (size_t(cur ^ 1) * a.n_strips + strip) * size_t(a.dry_rows) : nullptr;
        unsigned own_n = 0;   // cells of the strip this warp stores
#pragma unroll
        for (int h = 0; h < CPL; ++h) own_n += __popc(__ballot_sync(FULL, own_lane[h]));
        // the flags of this warp's rows in the output buffer and in the input buffer, four per
        // lane (read once: each row's output flag changes only at that row, the input flags not
        // at all during the step)
        unsigned dfw = 0u, dfw_in = 0u;
        if (dfl && r0 + 4 * lane < r_end) {
            dfw = *reinterpret_cast<const unsigned*>(dfl + r0 + 4 * lane);
            dfw_in = *reinterpret_cast<const unsigned*>(a.dryflag + (size_t(cur) * a.n_strips + strip) * size_t(a.dry_rows) +
                                                        r0 + 4 * lane);
        }
        // The whole block of rows: when this step adds no rain and no infiltration and records
        // no map, and the flags show every input row r0-1..r_end+1 of this strip and of its
        // neighbours (the 2-column aprons) deep-dry and every output row already holding the
        // record the deep-dry path would write, the loop below would store nothing and
        // contribute nothing: skip it, copies included.  (A flag is only ever set on a row
        // whose 64 columns hold no outlet or boundary cell, so no inflow, stage or structure
        // water can reach the rows the flags cover, and the deep-dry path updates no velocity
        // or hazard maximum.)
        bool blk_skip = false;
        if constexpr (INF == 0 && !MAP) {
            if (dfl && s_rec < 0 && RS.depth == R(0) && K.thr > R(0)) {
                const int nrow = r_end - r0;
                const int nb = min(max(nrow - 4 * lane, 0), 4);
                const unsigned mask = nb == 4 ? 0xffffffffu : (1u << (8 * nb)) - 1u;
                const unsigned want = 0x01010101u & mask;
                bool ok = (dfw & mask) == want;
                const unsigned char* fin = a.dryflag + size_t(cur) * a.n_strips * size_t(a.dry_rows);
                for (int q = max(strip - 1, 0); q <= min(strip + 1, a.n_strips - 1); ++q) {
                    const unsigned char* fq = fin + size_t(q) * a.dry_rows;
                    if (nb > 0) ok = ok && (*reinterpret_cast<const unsigned*>(fq + r0 + 4 * lane) & mask) == want;
                    if (lane < 3) {
                        const int rr = lane == 0 ? r0 - 1 : r_end + lane - 1;
                        if (rr >= 0 && rr < ny) ok = ok && fq[rr] == 1;
                    }
                }
                blk_skip = __all_sync(FULL, ok);
            }
        }
        if (blk_skip) {
            if (lane == 0) {
                atomicAdd(&s_skipw, own_n * unsigned(r_end - r0));
                atomicAdd(&s_skipr, own_n * unsigned(r_end - r0));
            }
        } else {

        // rolling window (suffix = rows back), one entry per cell of the lane
        R hT1[CPL], hT2[CPL], qxu1[CPL], qyu1[CPL], hfx1[CPL], hfx2[CPL], hfy1[CPL], hfy2[CPL];
        R sc2[CPL], qxl2[CPL], qyl2[CPL], dm1[CPL], dm2[CPL];
        R qyp1[CPL];   // schemes 2/3: previous q_y of the row before
        // velocity of the face below row r-3, computed by the (F) of row r-3: after the shift it
        // is the face above row r-2 (qyl2 / hfy2 then hold the values it was computed from), so
        // the next (F) takes it instead of dividing again; vcar_ok (warp-uniform) says whether
        // the last row's (F) computed it
        R vcar[CPL];
        bool vcar_ok = false;
        unsigned mt1[CPL], mt2[CPL];
#pragma unroll
        for (int h = 0; h < CPL; ++h) {
            qyp1[h] = R(0);
            vcar[h] = R(0);
            hT1[h] = hT2[h] = qxu1[h] = qyu1[h] = R(0);
            hfx1[h] = hfx2[h] = hfy1[h] = hfy2[h] = R(0);
            sc2[h] = R(1);
            qxl2[h] = qyl2[h] = dm1[h] = dm2[h] = R(0);
            mt1[h] = mt2[h] = 0u;
        }

        // TMA pipeline: the warp's two row records (static, state) of rows k+1..k+kStages-1
        // are in flight in a ring of kStages shared-memory stages while row k is
        // computed.  One 1-D bulk copy per record row (the strip's cells are contiguous),
        // the stage's mbarrier counts the bytes.
        const int seg_j0 = max(j_first, 0);
        const int seg_n = min(j_first + SW, nx) - seg_j0;
        const int seg_off = seg_j0 - j_first;
        const int last_k = (r_end + 1) - (r0 - 2);
        V4* ring = reinterpret_cast<V4*>(smem_dyn) + size_t(warp) * kStages * 2 * SW;
        const uint32_t bar0 = smem_addr(&s_bar[warp][0]);
        // lane 0 arms the stage's barrier (arrive + expected bytes) and copies the static
        // row, lane 1 copies the state row; a copy that lands before the arming only makes
        // the transaction count negative for a moment, and the phase cannot complete
        // before lane 0's arrival
        const uint32_t ring_base = smem_addr(ring + seg_off);
        const uint32_t bytes = uint32_t(seg_n) * uint32_t(sizeof(V4));
        const V4* src_base = lane == 0 ? stat : sin;
        const uint32_t dst_half = lane == 0 ? 0u : uint32_t(SW * sizeof(V4));
        auto issue = [&](int k) {
            const int s = k % kStages;
            const uint32_t bar = bar0 + 8u * s;
            const int rr = r0 - 2 + k;
            if (rr >= 0 && rr < ny && seg_n > 0) {
                if (lane == 0) mbar_expect_tx(bar, 2u * bytes);
                bulk_g2s(ring_base + uint32_t(s) * uint32_t(2 * SW * sizeof(V4)) + dst_half,
                         src_base + (size_t(rr) * nx + seg_j0), bytes, bar);
            } else if (lane == 0) {
                mbar_arrive(bar);
            }
        };
        if (lane == 0) {
            for (int s = 0; s < kStages; ++s) mbar_init(bar0 + 8u * s, 1u);
            mbar_fence_init();
        }
        __syncwarp();
        if (lane < 2) {
            fence_proxy_async_smem();   // reads of the ring by an earlier item come first
            for (int k = 0; k < kStages && k <= last_k; ++k) issue(k);
        }
        V2 nG[CPL];
#pragma unroll
        for (int h = 0; h < CPL; ++h) {
            nG[h] = V2{R(0), R(0)};
            if (INF && col_ok[h] && r0 - 2 >= 0) nG[h] = gin[size_t(r0 - 2) * nx + j[h]];
        }
#pragma unroll kRowUnroll
        for (int k = 0; k <= last_k; ++k) {
            const int r = r0 - 2 + k;
            const int s = k % kStages;
            // the dry flag of the output row r-2 in the buffer this step writes
            const bool frow_f = r - 2 >= r0 && r - 2 < r_end;
            const int fri = frow_f ? r - 2 - r0 : 0;
            const unsigned flg = frow_f ? (__shfl_sync(FULL, dfw, fri >> 2) >> (8 * (fri & 3))) & 255u : 0u;
            const unsigned flg_in = frow_f ? (__shfl_sync(FULL, dfw_in, fri >> 2) >> (8 * (fri & 3))) & 255u : 0u;
            const bool landed = mbar_wait_bounded(bar0 + 8u * s, uint32_t((k / kStages) & 1), a.wait_polls);
            if (__any_sync(FULL, !landed)) {   // the whole warp leaves the loop together
                timed_out = true;
                // let every copy still in flight (rows k .. k+kStages-1, this one included) land
                // before the CTA leaves, with the long limit whatever a.wait_polls is
                for (int kk = k; kk < k + kStages && kk <= last_k; ++kk)
                    mbar_wait_bounded(bar0 + 8u * (kk % kStages), uint32_t((kk / kStages) & 1), 1u << 22);
                break;
            }
            V4 S[CPL], X[CPL];
#pragma unroll
            for (int h = 0; h < CPL; ++h) {
                S[h] = ring[s * 2 * SW + 32 * h + lane];
                X[h] = ring[s * 2 * SW + SW + 32 * h + lane];
            }
            __syncwarp();
            if (lane < 2 && k + kStages <= last_k) {
                fence_proxy_async_smem();
                issue(k + kStages);
            }
            const bool rok = r >= 0 && r < ny;
            const bool own_row = r >= r0 && r < r_end;
            R hT0[CPL];
            unsigned meta[CPL];
            bool all_dry = true;
#pragma unroll
            for (int h = 0; h < CPL; ++h) {
                const V2 Gs = nG[h];
                if (INF && col_ok[h] && r + 1 >= 0 && r + 1 < ny) nG[h] = gin[size_t(r + 1) * nx + j[h]];
                meta[h] = meta_bits(S[h].w);
                // (A) hydrology of (r, j)
                hT0[h] = R(0);
                if (col_ok[h] && rok) {
                    const size_t c = size_t(r) * nx + j[h];
                    R hh = X[h].x;
                    // a pending map record keeps the depth this step starts from
                    if (s_rec >= 0 && own_lane[h] && own_row) a.rec.snap[size_t(s_rec) * (size_t(ny) * nx) + c] = hh;
                    // map weights are read from shared memory where they are used
                    const R rr = MAP ? s_rs.at(a.rain, r, j[h], ny, nx) : RS.depth;
                    hh = hh + rr;
                    const bool own = own_lane[h] && own_row && r >= a.own_r0 && r < a.own_r1;
                    // uniform rain volume comes from the count of finite cells at the end
                    if (MAP && own && isfinite(hh)) rain_acc_r.add(rr);
                    if (INF) {
                        const unsigned sc = meta[h] & 255u;
                        V2 go = Gs;
                        if (sc != 255u) {
                            R Ic = Gs.x, Tc = Gs.y;
                            // Green-Ampt: {I, recovery timer}; van Genuchten: {I, water-table depth}
                            const R fd = INF == 1 ? green_ampt(hh, Ic, Tc, a.classes[sc], K)
                                                  : vg_infiltration(hh, Ic, Tc, a.classes_vg[sc], a.vg, K);
                            go.x = Ic;
                            go.y = Tc;
                            if (own && isfinite(fd)) inf_acc_r.add(fd);
                        }
                        if (own) gout[c] = go;
                    }
                    // inflow hydrographs after the infiltration (Hydrological_Model.m:27-28)
                    if (INFL) add_inflow(a.inflow, meta[h], hh);
                    if (!skip && hh < R(1e-9)) hh = R(0);
                    if (hh < R(0)) hh = R(0);
                    hT0[h] = hh;
                }
                all_dry = all_dry && hT0[h] == R(0);
            }
            // rows r-2..r dry across the whole strip: every face flux of row r and r-1 is
            // zero (Hf = 0), the donor scale of row r-1 is one and its limited faces are
            // zero, so (B)-(E) are skipped; the values below are what they would compute
            dry = (dry << 1) | (__all_sync(FULL, all_dry) ? 1u : 0u);
            // Deep-dry row: rows r-3..r dry across the strip and no outlet cell in row r-2.
            // Then (B)-(E) of this row and of the one before were skipped, so the window's
            // flux, face-depth and limited-flux registers hold +0 and the donor scale 1,
            // which is what this row's (B)-(E) and shift would store again; (F) for row r-2
            // gives depth hT2 + 0 = +0 (hT2 is a dry zero), fluxes +0 and the unchanged
            // maximum, with no arrival, outlet or CFL contribution.  Only the depth, maximum
            // and meta registers move.  (hfx2/hfy2 are left one row stale: they are read
            // only by a non-quiet (F), and the (F) after a deep-dry row is quiet.)  A depth
            // of +0 reaches the arrival threshold only when that is not positive.
            if ((dry & 15u) == 15u && K.thr > R(0)) {
                bool plain = true;
#pragma unroll
                for (int h = 0; h < CPL; ++h) plain = plain && (mt2[h] >> 8) == 0u;
                if (__all_sync(FULL, plain)) {
                    const int rm2 = r - 2;
                    if (frow_f && flg && flg_in) {
                        // this buffer already holds the row as this step would write it: the
                        // deep-dry record of two steps ago, and the step between wrote the
                        // deep-dry record into the other buffer (so the running maximum did not
                        // move; a row that got water in between and lost it again by the next
                        // step -- rain soaked up by the soil -- is written)
                        if (lane == 0) atomicAdd(&s_skipw, own_n);
                    } else if (frow_f) {
#pragma unroll
                        for (int h = 0; h < CPL; ++h)
                            if (own_lane[h]) {
                                V4 o4;
                                o4.x = R(0);
                                o4.y = R(0);
                                o4.z = R(0);
                                o4.w = R(0) > dm2[h] ? R(0) : dm2[h];
                                sout[size_t(rm2) * nx + j[h]] = o4;
                            }
                        if (dfl && lane == 0) dfl[rm2] = 1;
                    }
#pragma unroll
                    for (int h = 0; h < CPL; ++h) {
                        hT2[h] = hT1[h]; hT1[h] = hT0[h];
                        dm2[h] = dm1[h]; dm1[h] = X[h].w;
                        mt2[h] = mt1[h]; mt1[h] = meta[h];
                        if (SCH) qyp1[h] = X[h].z;
                    }
                    vcar_ok = false;
                    continue;
                }
            }
            R qxu0[CPL], hfx0[CPL], qyu0[CPL], hfy0[CPL], sc1[CPL], qxl1[CPL], qyl1[CPL];
#pragma unroll
            for (int h = 0; h < CPL; ++h) {
                qxu0[h] = hfx0[h] = qyu0[h] = hfy0[h] = qxl1[h] = qyl1[h] = R(0);
                sc1[h] = R(1);
            }
            if ((dry & 7u) != 7u) {
                // (B) x face (r, j) between (r, j) and (r, j+1)
                R hR[CPL];
                right_of<R, CPL>(hT0, hR, lane);
                // schemes 2/3: previous q_x of the faces j-1 and j+1 (interior columns only);
                // lane 0's left neighbour lies outside the strip and is read from memory
                R qxa[CPL], qxb[CPL];
                if (SCH) {
                    R xq[CPL];
#pragma unroll
                    for (int h = 0; h < CPL; ++h) xq[h] = X[h].y;
                    left_of<R, CPL>(xq, qxa, lane);
                    right_of<R, CPL>(xq, qxb, lane);
                    if (lane == 0 && rok && j[0] >= 1) qxa[0] = sin[size_t(r) * nx + (j[0] - 1)].y;
#pragma unroll
                    for (int h = 0; h < CPL; ++h)
                        if (!(j[h] >= 1 && j[h] + 1 < nx)) qxa[h] = qxb[h] = R(0);
                }
                if constexpr (kFaceIlp<INF, MAP>) {
                // (B) and (C) interleaved: the geometry of the 2 x CPL faces, then -- unless no
                // lane of the warp has a wet one -- their momentum updates without branches
                R Sx[CPL], Sy[CPL], ya[CPL], yb[CPL];
                bool wx[CPL], wy[CPL];
                bool any_wet = false;
#pragma unroll
                for (int h = 0; h < CPL; ++h) {
                    const bool inx = col_ok[h] && rok;
                    const bool iny = inx && r >= r0 - 1;
                    R H;
                    wx[h] = face_geom<R, true>(hT0[h], hR[h], S[h].x, H, Sx[h], K) && inx;
                    hfx0[h] = inx ? H : R(0);
                    wy[h] = face_geom<R, false>(hT1[h], hT0[h], S[h].y, H, Sy[h], K) && iny;
                    hfy0[h] = iny ? H : R(0);
                    any_wet = any_wet || wx[h] || wy[h];
                    ya[h] = yb[h] = R(0);
                    // schemes 2/3: the previous q_y of rows r-1 (kept from the row before) and r+1
                    if (SCH && wy[h] && r >= 1 && r + 1 < ny) {
                        ya[h] = qyp1[h];
                        yb[h] = sin[size_t(r + 1) * nx + j[h]].z;
                    }
                }
                if (__any_sync(FULL, any_wet)) {
#pragma unroll
                    for (int h = 0; h < CPL; ++h) {
                        qxu0[h] = face_momentum<R, SCH>(wx[h], hfx0[h], Sx[h], X[h].y, S[h].z, K, a.flag_critical,
                                                         a.scheme, SCH ? qxa[h] : R(0), SCH ? qxb[h] : R(0));
                        qyu0[h] = face_momentum<R, SCH>(wy[h], hfy0[h], Sy[h], X[h].z, S[h].z, K, a.flag_critical,
                                                         a.scheme, ya[h], yb[h]);
                    }
                }
                } else {
#pragma unroll
                for (int h = 0; h < CPL; ++h)
                    if (col_ok[h] && rok)
                        face_flux<R, true, SCH>(hT0[h], hR[h], S[h].x, X[h].y, S[h].z, K, a.flag_critical, hfx0[h],
                                                qxu0[h], a.scheme, SCH ? qxa[h] : R(0), SCH ? qxb[h] : R(0));
                // (C) y face (r, j) between (r-1, j) and (r, j); schemes 2/3 read the previous
                // q_y of rows r-1 (kept from the row before) and r+1 (from memory)
#pragma unroll
                for (int h = 0; h < CPL; ++h)
                    if (col_ok[h] && rok && r >= r0 - 1) {
                        R ya = R(0), yb = R(0);
                        if (SCH && r >= 1 && r + 1 < ny) {
                            ya = qyp1[h];
                            yb = sin[size_t(r + 1) * nx + j[h]].z;
                        }
                        face_flux<R, false, SCH>(hT1[h], hT0[h], S[h].y, X[h].z, S[h].z, K, a.flag_critical, hfy0[h],
                                                 qyu0[h], a.scheme, ya, yb);
                    }
                }
                // (D) donor scale of (r-1, j)
                R qxu1_left[CPL];
                left_of<R, CPL>(qxu1, qxu1_left, lane);
                const bool drow = r >= r0 && r - 1 >= 0 && r - 1 < ny;
#pragma unroll
                for (int h = 0; h < CPL; ++h)
                    if (col_ok[h] && drow) sc1[h] = donor_scale_finite(qxu1[h], qxu1_left[h], qyu1[h], qyu0[h], hT1[h], K);
                // (E) limited faces of row r-1
                R sc1_right[CPL];
                right_of<R, CPL>(sc1, sc1_right, lane);
#pragma unroll
                for (int h = 0; h < CPL; ++h) {
                    qxl1[h] = limit_face_finite(qxu1[h], sc1[h], sc1_right[h]);
                    qyl1[h] = limit_face_finite(qyu1[h], sc1[h], sc2[h]);
                }
            }
            // (F) continuity, outlet, maxima and CFL of row r-2.  When rows r-3..r-1 are dry
            // across the strip every flux into row r-2 is +0 (and so are its face depths):
            // continuity gives hT2 + 0 and the cell adds nothing to the CFL reductions.
            const bool quiet = (dry & 14u) == 14u;
            R qxl2_left[CPL];
            if (quiet) {
#pragma unroll
                for (int h = 0; h < CPL; ++h) qxl2_left[h] = R(0);
            } else {
                left_of<R, CPL>(qxl2, qxl2_left, lane);
            }
            const int rm2 = r - 2;
            const bool frow = rm2 >= r0 && rm2 < r_end;
            const bool mine = rm2 >= a.own_r0 && rm2 < a.own_r1;   // enters the reductions
            if constexpr (kFlatF<INF, MAP>) {
                // The cells of the lane are computed without a per-lane branch (an apron lane's values
                // are computed and dropped: `act` masks every store and every reduction), so that the
                // compiler can interleave the CPL cells' arithmetic; frow is the same for the warp.
                if (frow) {
                    R hn_[CPL], hf3_[CPL];
    #pragma unroll
                    for (int h = 0; h < CPL; ++h) {
                        const bool act = own_lane[h];
                        const size_t c2 = size_t(rm2) * nx + j[h];
                        // a control structure's transfers join the depth after the fluxes
                        // (Local_Inertial_Model_D4.m:318-344, :390)
                        R h_in = hT2[h];
                        if (INFL && act && (mt2[h] & kInflowBit)) {
                            const int ss = a.inflow.cell_struct[(mt2[h] >> 8) & 0x7FFFFFu];
                            if (ss >= 0) h_in = h_in + a.strct.extra[ss];
                        }
                        R hn = quiet ? h_in + R(0) : continuity(h_in, qxl2_left[h], qxl2[h], qyl2[h], qyl1[h], K);
                        const R negtol = -K.tol;
                        R hf3 = R(0);
                        const unsigned ord = outlet_ord(mt2[h]);
                        if (act && ord) {
                            const int o = int(ord) - 1;
                            R ho;
                            const R qq = outlet_sink(hn, a.outlet_coef[o], a.outlet_type, K, ho);
                            hf3 = ho;
                            a.hf3[o] = ho;
                            a.qo[o] = qq;
                            if (mine) out_acc_r.add(qq * K.dt);
                            // the next step's clamp is skipped when an outlet cell (outside the
                            // infiltrating soils) stays negative after the next rain
                            // (Hydrological_Model.m:45-50); only outlet cells can end negative
                            if (mine && !(a.ga && (mt2[h] & 255u) != 255u) &&
                                hn + (MAP ? s_rsn.at(a.rain, rm2, j[h], ny, nx) : s_rsn.depth) < R(-1e-11))
                                s_negn = 1;   // rare: kept in shared memory, not a register
                        }
                        // stage hydrograph: the cell's depth becomes the gauge's stage
                        // (update_spatial_BC.m:332-341, after the step's refreshing_timestep)
                        if (INFL && act && (mt2[h] & kInflowBit)) {
                            const int sg = a.inflow.cell_stage[(mt2[h] >> 8) & 0x7FFFFFu];
                            if (sg >= 0) {
                                const R sv = a.inflow.stage_now[sg];
                                atomicAdd(&s_stage, double(sv) - double(hn));
                                hn = sv;
                            }
                        }
                        // a non-finite depth (NaN walls included, counted against the run's start)
                        // or one below -depth_tolerance
                        nbad += (hn >= negtol || !mine || !act) ? 0u : 1u;
                        if (act && dm2[h] < K.thr && hn >= K.thr) a.arrival[c2] = t_arr;
                        hn_[h] = hn;
                        hf3_[h] = hf3;
                    }
                    // refreshing_timestep.m:61-89, :139-150, :181-238 for these cells
                    R vras[CPL];   // velocity raster: largest |face velocity| (refreshing_timestep.m:109-111)
    #pragma unroll
                    for (int h = 0; h < CPL; ++h) vras[h] = R(0);
                    if (!quiet && mine) {
                        const R big = R(1e9);
    #pragma unroll
                        for (int h = 0; h < CPL; ++h) {
                            const bool act = own_lane[h];
                            const R vr = qxl2[h] == R(0) ? qxl2[h] : qdiv(qxl2[h], hfx2[h] < K.tol ? big : hfx2[h]);
                            R vu;
                            if (vcar_ok) vu = vcar[h];
                            else vu = qyl2[h] == R(0) ? qyl2[h] : qdiv(qyl2[h], hfy2[h] < K.tol ? big : hfy2[h]);
                            const R vb = qyl1[h] == R(0) ? qyl1[h] : qdiv(qyl1[h], hfy1[h] < K.tol ? big : hfy1[h]);
                            vcar[h] = vb;
                            if (INFL) vras[h] = fmax(fmax(fabs(vr), fabs(vu)), fabs(vb));
                            const R rc = j[h] == 0 ? R(0.5) * vr : vr;
                            const R uc = R(0.5) * (vu + vb);
                            const R s2 = rc * rc + uc * uc;
                            if (act) s2max = fmax(s2max, s2);
                            const R dts = fmax(fmax(hfx2[h], hfy2[h]), hf3_[h]);
                            R cval;
                            if (a.adaptive == 1) {
                                cval = K.g * fmax(dts, R(0));
                            } else {
                                const R wc = fmax(sqrt(K.g * fmax(dts, R(0))), R(1e-10));
                                cval = fmax(fmax(fabs(vr), fabs(vu)), fabs(vb)) + wc;
                            }
                            if (act && s2 >= a.stag_s2) cmaxv = fmax(cmaxv, cval);
                        }
                    }
    #pragma unroll
                    for (int h = 0; h < CPL; ++h) {
                        if (!own_lane[h]) continue;
                        const size_t c2 = size_t(rm2) * nx + j[h];
                        const R hn = hn_[h];
                        const R dm = dm2[h];
                        V4 o4;
                        o4.x = hn;
                        o4.y = qxl2[h];
                        o4.z = qyl2[h];
                        o4.w = hn > dm ? hn : dm;   // save_output_maps.m:598, max(d_t, dmax)
                        sout[c2] = o4;
                        // running maxima of the velocity raster and of depth x velocity
                        // (save_output_maps.m:588-604, snisb_velocity_hazard_snapshot :832-848)
                        if (INFL && a.vmax) {
                            const R vo = a.vmax[c2];
                            a.vmax[c2] = vras[h] > vo ? vras[h] : vo;
                            const R hd = fmax(hn, R(0));
                            R hz = hd * vras[h];
                            if (hd < R(0.01) || !isfinite(hz)) hz = R(0);
                            const R ho = a.hzmax[c2];
                            a.hzmax[c2] = isnan(hn) ? hn : (hz > ho ? hz : ho);
                        }
                    }
                }
            } else {
            // the infiltration and rain-map instantiations keep the per-lane branch around the cell
            // body (fewer live registers: measured faster there)
    #pragma unroll
                for (int h = 0; h < CPL; ++h) {
                    if (own_lane[h] && frow) {
                        const size_t c2 = size_t(rm2) * nx + j[h];
                        // a control structure's transfers join the depth after the fluxes
                        // (Local_Inertial_Model_D4.m:318-344, :390)
                        R h_in = hT2[h];
                        if (INFL && (mt2[h] & kInflowBit)) {
                            const int ss = a.inflow.cell_struct[(mt2[h] >> 8) & 0x7FFFFFu];
                            if (ss >= 0) h_in = h_in + a.strct.extra[ss];
                        }
                        R hn = quiet ? h_in + R(0) : continuity(h_in, qxl2_left[h], qxl2[h], qyl2[h], qyl1[h], K);
                        const R negtol = -K.tol;
                        R hf3 = R(0);
                        const unsigned ord = outlet_ord(mt2[h]);
                        if (ord) {
                            const int o = int(ord) - 1;
                            R ho;
                            const R qq = outlet_sink(hn, a.outlet_coef[o], a.outlet_type, K, ho);
                            hf3 = ho;
                            a.hf3[o] = ho;
                            a.qo[o] = qq;
                            if (mine) out_acc_r.add(qq * K.dt);
                            // the next step's clamp is skipped when an outlet cell (outside the
                            // infiltrating soils) stays negative after the next rain
                            // (Hydrological_Model.m:45-50); only outlet cells can end negative
                            if (mine && !(a.ga && (mt2[h] & 255u) != 255u) &&
                                hn + (MAP ? s_rsn.at(a.rain, rm2, j[h], ny, nx) : s_rsn.depth) < R(-1e-11))
                                s_negn = 1;   // rare: kept in shared memory, not a register
                        }
                        // stage hydrograph: the cell's depth becomes the gauge's stage
                        // (update_spatial_BC.m:332-341, after the step's refreshing_timestep)
                        if (INFL && (mt2[h] & kInflowBit)) {
                            const int sg = a.inflow.cell_stage[(mt2[h] >> 8) & 0x7FFFFFu];
                            if (sg >= 0) {
                                const R sv = a.inflow.stage_now[sg];
                                atomicAdd(&s_stage, double(sv) - double(hn));
                                hn = sv;
                            }
                        }
                        // a non-finite depth (NaN walls included, counted against the run's start)
                        // or one below -depth_tolerance
                        nbad += (hn >= negtol || !mine) ? 0u : 1u;
                        const R dm = dm2[h];
                        if (dm < K.thr && hn >= K.thr) a.arrival[c2] = t_arr;
                        // refreshing_timestep.m:61-89, :139-150, :181-238 for this cell
                        R vras = R(0);   // velocity raster: largest |face velocity| (refreshing_timestep.m:109-111)
                        if (!quiet && mine) {
                            const R big = R(1e9);
                            const R vr = qxl2[h] == R(0) ? qxl2[h] : qdiv(qxl2[h], hfx2[h] < K.tol ? big : hfx2[h]);
                            R vu;
                            if (vcar_ok) vu = vcar[h];
                            else vu = qyl2[h] == R(0) ? qyl2[h] : qdiv(qyl2[h], hfy2[h] < K.tol ? big : hfy2[h]);
                            const R vb = qyl1[h] == R(0) ? qyl1[h] : qdiv(qyl1[h], hfy1[h] < K.tol ? big : hfy1[h]);
                            vcar[h] = vb;
                            if (INFL) vras = fmax(fmax(fabs(vr), fabs(vu)), fabs(vb));
                            const R rc = j[h] == 0 ? R(0.5) * vr : vr;
                            const R uc = R(0.5) * (vu + vb);
                            const R s2 = rc * rc + uc * uc;
                            s2max = fmax(s2max, s2);
                            if (s2 >= a.stag_s2) {
                                const R dts = fmax(fmax(hfx2[h], hfy2[h]), hf3);
                                R cval;
                                if (a.adaptive == 1) {
                                    cval = K.g * fmax(dts, R(0));
                                } else {
                                    const R wc = fmax(sqrt(K.g * fmax(dts, R(0))), R(1e-10));
                                    cval = fmax(fmax(fabs(vr), fabs(vu)), fabs(vb)) + wc;
                                }
                                cmaxv = fmax(cmaxv, cval);
                            }
                        }
                        V4 o4;
                        o4.x = hn;
                        o4.y = qxl2[h];
                        o4.z = qyl2[h];
                        o4.w = hn > dm ? hn : dm;   // save_output_maps.m:598, max(d_t, dmax)
                        sout[c2] = o4;
                        // running maxima of the velocity raster and of depth x velocity
                        // (save_output_maps.m:588-604, snisb_velocity_hazard_snapshot :832-848)
                        if (INFL && a.vmax) {
                            const R vo = a.vmax[c2];
                            a.vmax[c2] = vras > vo ? vras : vo;
                            const R hd = fmax(hn, R(0));
                            R hz = hd * vras;
                            if (hd < R(0.01) || !isfinite(hz)) hz = R(0);
                            const R ho = a.hzmax[c2];
                            a.hzmax[c2] = isnan(hn) ? hn : (hz > ho ? hz : ho);
                        }
                    }
                }
            }
            vcar_ok = !quiet && mine && frow;
            if (flg && lane == 0) dfl[r - 2] = 0;   // rewritten: no longer known dry
            // (G) shift the window down one row
#pragma unroll
            for (int h = 0; h < CPL; ++h) {
                hT2[h] = hT1[h]; hT1[h] = hT0[h];
                qxu1[h] = qxu0[h]; qyu1[h] = qyu0[h];
                hfx2[h] = hfx1[h]; hfx1[h] = hfx0[h];
                hfy2[h] = hfy1[h]; hfy1[h] = hfy0[h];
                sc2[h] = sc1[h];
                qxl2[h] = qxl1[h]; qyl2[h] = qyl1[h];
                dm2[h] = dm1[h]; dm1[h] = X[h].w;
                mt2[h] = mt1[h]; mt1[h] = meta[h];
                if (SCH) qyp1[h] = X[h].z;
            }
        }
        // every phase of the ring's barriers has completed: retire them so that the next
        // item of a persistent CTA can initialise them again
        __syncwarp();
        if (lane == 0 && !timed_out)
            for (int s = 0; s < kStages; ++s) mbar_inval(bar0 + 8u * s);
        }  // !blk_skip
    }

    // ---- CTA reductions ---------------------------------------------------------------
    // (the last CTA reads only the step accumulators, which thread 0 publishes before its
    // ticket; the state records reach the next launch through the kernel boundary)
    rain_acc += rain_acc_r.value();
    inf_acc += inf_acc_r.value();
    out_acc += out_acc_r.value();
    const int lane_ = tid & 31, warp_ = tid >> 5;
    s2max = warp_max(s2max);
    // 0: no non-stagnant cell; else the bits of the (non-negative, +0 for -0) maximum + 1
    unsigned long long cenc = cmaxv >= R(0) ? ord_bits(cmaxv + R(0)) + 1ull : 0ull;
    cenc = warp_max_u(cenc);
    rain_acc = warp_sum(rain_acc);
    inf_acc = warp_sum(inf_acc);
    out_acc = warp_sum(out_acc);
    const int to_any = __any_sync(0xffffffffu, timed_out);
    nbad = __reduce_add_sync(0xffffffffu, nbad);
    if (lane_ == 0) {
        red_bad[warp_] = nbad;
        red_s2[warp_] = s2max;
        red_c[warp_] = cenc;
        red_d[0][warp_] = rain_acc;
        red_d[1][warp_] = inf_acc;
        red_d[2][warp_] = out_acc;
        red_to[warp_] = to_any;
    }
    __syncthreads();
    const int negn = s_negn;
    if (tid == 0) {
        int to = 0;
        for (int w = 0; w < NT / 32; ++w) to |= red_to[w];
        if (to) atomicOr(&a.sc->status, kStatusTimeout);   // a row copy did not arrive in time
        unsigned bad = 0u;
        for (int w = 0; w < NT / 32; ++w) bad += red_bad[w];
        if (bad) atomicAdd(&a.sc->acc_bad, (unsigned long long)bad);
        for (int w = 1; w < NT / 32; ++w) {
            s2max = fmax(s2max, red_s2[w]);
            cenc = red_c[w] > cenc ? red_c[w] : cenc;
            rain_acc += red_d[0][w];
            inf_acc += red_d[1][w];
            out_acc += red_d[2][w];
        }
        StepScalars* sc = a.sc;
        if (s2max > R(0)) atomicMax(&sc->acc_vmax, ord_bits(s2max));
        if (cenc) atomicMax(&sc->acc_cmax, cenc);
        if (rain_acc != 0.0) atomicAdd(&sc->acc_rain, rain_acc);
        if (inf_acc != 0.0) atomicAdd(&sc->acc_inf, inf_acc);
        if (out_acc != 0.0) atomicAdd(&sc->acc_out, out_acc);
        if (negn) atomicOr(&sc->skip_next, 1);
        if (INFL && s_stage != 0.0) atomicAdd(&sc->acc_stage, s_stage);
        if (s_skipw) atomicAdd(&sc->skipped_cells, (unsigned long long)s_skipw);
        if (s_skipr) atomicAdd(&sc->skipped_read_cells, (unsigned long long)s_skipr);
        __threadfence();
        const unsigned int ticket = atomicAdd(&sc->counter, 1u);
        s_last = (ticket == a.n_ctas - 1);
    }
    __syncthreads();
    bool cta_ok = true;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) cta_ok = cta_ok && red_to[w] == 0;
    if (!s_last) return cta_ok;

    // ---- last CTA: refreshing_timestep + clock (HydroPol2D_Main_While.m:691-705, :779)
    __threadfence();
    // a rejected step commits nothing: the state stays in buffer cur, the clock, counters and
    // volumes stay, and the launches halt until the host has prepared the retry
    // (HydroPol2D_Main_While.m:926-993); s_last doubles as the verdict for the CTA below
    if (tid == 0) {
        StepScalars* sc = a.sc;
        bool reject = (atomicAdd(&sc->status, 0u) & kStatusTimeout) != 0u;
        if (atomicAdd(&sc->acc_bad, 0ull) > sc->n_bad0) {
            reject = true;
            sc->status |= kStatusNumerical;
        }
        if (sc->fault_n > 0 && sc->k == sc->fault_k) {   // the host's test hook
            sc->fault_n -= 1;
            reject = true;
            sc->status |= kStatusNumerical;
        }
        if (reject) {
            sc->halted = 1;
            if (s_skip) sc->neg_warn -= 1;   // the attempt's clamp warning is withdrawn
            sc->acc_vmax = 0ull;
            sc->acc_cmax = 0ull;
            sc->acc_rain = 0.0;
            sc->acc_inf = 0.0;
            sc->acc_out = 0.0;
            sc->acc_stage = 0.0;
            sc->acc_bad = 0ull;
            sc->counter = 0u;
            atomicExch(&sc->skip_next, 0);
            s_last = 0;
        }
    }
    __syncthreads();
    if (!s_last) return cta_ok;
    if (tid == 0) {
        StepScalars* sc = a.sc;
        const unsigned long long vbits = atomicAdd(&sc->acc_vmax, 0ull);
        const unsigned long long cbits = atomicAdd(&sc->acc_cmax, 0ull);
        const R vR = sqrt(bits_to<R>(vbits));
        double vm = double(vR);
        double cm = 0.0;
        if (cbits) {
            const R v = bits_to<R>(cbits - 1ull);
            cm = a.adaptive == 1 ? double(fmax(sqrt(v), R(1e-10))) : double(v);
        }
        double rain_s = atomicAdd(&sc->acc_rain, 0.0);
        // uniform rain: the same depth on every cell with a finite depth
        if (a.rain.n_uniform) rain_s += double(s_rs.depth) * double(sc->n_finite);
        const double inf_s = atomicAdd(&sc->acc_inf, 0.0);
        const double out_s = atomicAdd(&sc->acc_out, 0.0);
        const double t = s_tmin;
        const double pos_save = ceil((t * 60.0) / a.tsc);
        const double time_save = (pos_save - 1.0) * a.tsc / 60.0;
        const double delta = time_save - sc->tsp;
        sc->tsp = time_save;
        double tcr = sc->time_step * 60.0;   // refreshing_timestep.m:361-365
        sc->last_vbits = vbits;
        sc->last_cbits = cbits;
        sc->last_refreshed = 0;
        sc->last_unstable = 0;
        if ((delta > 0 || sc->k == 1) &&
            (sc->refresh_every <= 1 || sc->k == 1 || (sc->k - 1) % sc->refresh_every == 0)) {
            tcr = finalize_dt(vm, cm, a.res, a.alfa_min, a.alfa_max, a.min_dt, sc->max_dt, a.inc,
                              a.flag_timestep);
            sc->vmax_last = vm;
            sc->last_refreshed = 1;
            sc->last_unstable = tcr == a.min_dt;
            if (tcr == a.min_dt) {   // refreshing_timestep.m:357-359 (unstable)
                sc->unstable += 1;
                if (sc->dt_floor_stop) {
                    sc->status |= kStatusDtFloor;
                    sc->halted = 1;   // this step is kept; the next launches wait for the host
                }
            }
        }
        const double area = a.res * a.res;
        sc->rain_vol += rain_s * area;
        sc->inf_vol += inf_s * area;
        sc->out_vol += out_s * area;
        if (a.inflow.n_gauges) {   // every cell of a gauge with a finite elevation got its depth
            double v = 0.0;
            for (int g = 0; g < a.inflow.n_gauges; ++g) v += double(a.inflow.depth[g]) * a.inflow.gauge_cells[g];
            sc->inflow_vol += v * area;
        }
        if (a.inflow.n_stage) {
            sc->stage_vol += __ldcg(&sc->acc_stage) * area;
            sc->acc_stage = 0.0;
        }
        if (INFL && a.strct.n) {   // the structures' extras this step applied
            double v = 0.0;
            for (int q = 0; q < a.strct.n_slots; ++q) v += double(a.strct.extra[q]) * area;
            sc->struct_vol += v;
        }
        // the next step's rain: update_spatial_BC over [t_previous, t]
        // (HydroPol2D_Main_While.m:721), then t_previous <- the clock increment on the first
        // step and t after it (:734-738), and the clock advances by the new step (:779)
        sc->rain_a = sc->t_prev;
        sc->rain_b = t;
        sc->t_prev = sc->k == 1 ? tcr / 60.0 : t;
        if (a.rec.n_times > 0) {   // save_output_maps.m:25-27 with t_save = t + new dt (:740)
            if (sc->rec_pending) { sc->rec_count += 1; sc->rec_pending = 0; }   // recorded by this step
            const int idx = last_record_below(a.rec.times, a.rec.n_times, t + tcr / 60.0);
            if (idx > sc->rec_last && a.rec.n_slots > 0) {
                sc->rec_pending = 1;
                a.rec.snap_t[sc->rec_count % a.rec.n_slots] = t;
            }
            if (idx > sc->rec_last) sc->rec_last = idx;
        }
        sc->time_step = tcr / 60.0;
        sc->t_min = tcr / 60.0 + t;
        sc->k += 1;
        sc->cur = cur ^ 1;
        sc->acc_vmax = 0ull;
        sc->acc_cmax = 0ull;
        sc->acc_rain = 0.0;
        sc->acc_inf = 0.0;
        sc->acc_out = 0.0;
        sc->acc_bad = 0ull;
        sc->counter = 0u;
        sc->skip_clamp = atomicExch(&sc->skip_next, 0);   // gathered by every CTA's outlets
    }
    if (a.inflow.n_gauges || a.inflow.n_stage) {   // the next step's gauge depths and stages
        __syncthreads();
        const double ra = a.sc->rain_a, rb = a.sc->rain_b, tn = a.sc->t_min;
        for (int g = tid; g < a.inflow.n_gauges; g += NT)
            a.inflow.depth[g] = R(inflow_integral(a.inflow, g, ra, rb) / 60000.0);
        for (int g = tid; g < a.inflow.n_stage; g += NT) a.inflow.stage_now[g] = R(stage_at(a.inflow, g, tn));
    }
    if constexpr (INFL) {
        if (a.strct.n) {   // the next step's structure transfers, from its d_tot
            __syncthreads();
            __shared__ StepConsts<R> s_Kn;
            __shared__ int s_skn;
            __shared__ double s_tsn;
            if (tid == 0) {
                s_tsn = a.sc->time_step;
                s_Kn.make(s_tsn * 60.0, a.res, a.tol_mm, a.thr_mm);
                s_skn = a.sc->skip_clamp;
            }
            __syncthreads();
            structure_prepare<R, INF, MAP, INFL>(a, s_rsn, s_skn != 0, s_Kn, sout, gout, tid, NT, s_tsn);
        }
    }
    return cta_ok;
}

// Rain maps from gauges by inverse-distance weighting, one full-resolution map per record
// interval (Rainfall_Interpolator.m / idw_function.m with p = 2, the Euclidean norm and no
// radius): cell (i, j) sits at (x_ul + res (j+1), y_ul - res (i+1))
// (HydroPol2D_preprocessing.m:2420-2421); distance d = sqrt(dx^2 + dy^2), 0 -> eps, weight
// 1/d^2; gauges whose record is NaN are left out of that interval's map, and an interval
// without any gauge is dry.  Sums run over the gauges in order, in FP64.
static __global__ void k_idw_maps(int ny, int nx, double res, double x_ul, double y_ul, int ng, const double* xg,
                           const double* yg, int nt, const double* rate, float* maps) {
    const size_t n = size_t(ny) * nx;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / nx), j = int(c % nx);
        const double X = x_ul + res * double(j + 1), Y = y_ul - res * double(i + 1);
        for (int m = 0; m < nt; ++m) {
            double num = 0.0, den = 0.0;
            for (int g = 0; g < ng; ++g) {
                const double r = rate[size_t(m) * ng + g];
                if (isnan(r)) continue;
                const double dx = fabs(X - xg[g]), dy = fabs(Y - yg[g]);
                double d = sqrt(dx * dx + dy * dy);
                if (d == 0.0) d = 2.220446049250313e-16;
                const double w = 1.0 / (d * d);
                num = num + w * r;
                den = den + w;
            }
            maps[size_t(m) * n + c] = den > 0.0 ? float(num / den) : 0.0f;
        }
    }
}

// ---------------- host boundary on the device: records built from the caller's arrays ----
// static record {dz_x, dz_y, n^2, meta} and the unfused path's copies, from the elevation and
// roughness in FP64 (dz formed in FP64 and rounded once; the closed domain edges +inf).  A cell
// of NaN elevation (idx_nan) gets n^2 = NaN: its own faces are closed by their NaN dz before
// n^2 is read, so the NaN only marks the cell as outside the domain (k_skip_flag reads it).
template <typename R>
__global__ void k_build_static(int ny, int nx, const double* z, const double* rough, const uint32_t* meta,
                               typename Vec<R>::V4* stat, R* dzx, R* dzy, R* n2) {
    const size_t n = size_t(ny) * nx;
    const double edge = __longlong_as_double(0x7ff0000000000000ll);   // +inf
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const int i = int(k / nx), j = int(k % nx);
        const R a = R((j + 1 < nx) ? z[k + 1] - z[k] : edge);
        const R b = R((i >= 1) ? z[k - nx] - z[k] : edge);
        const R c = isnan(z[k]) ? R(__longlong_as_double(0x7ff8000000000000ll)) : R(rough[k] * rough[k]);
        stat[k] = typename Vec<R>::V4{a, b, c, make_meta<R>(meta[k])};
        if (dzx) {
            dzx[k] = a;
            dzy[k] = b;
            n2[k] = c;
        }
    }
}
// the unfused entry points' structure-of-arrays copies of the static record
template <typename R>
__global__ void k_static_soa(size_t n, const typename Vec<R>::V4* stat, R* dzx, R* dzy, R* n2) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const auto v = stat[k];
        dzx[k] = v.x;
        dzy[k] = v.y;
        n2[k] = v.z;
    }
}
// state record {h, q_x, q_y, dmax = -inf} from depths.d_t [mm] and outflow_bates pages 1-2
// [mm/h] (NULL: zero fluxes)
template <typename R>
__global__ void k_build_state(size_t n, const double* d, const double* outflow, double res,
                              typename Vec<R>::V4* st) {
    const R ninf = R(__longlong_as_double(0xfff0000000000000ll));
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        typename Vec<R>::V4 x;
        x.x = R(d[k] / 1000.0);
        // outflow_bates [mm/h] -> q [m^2/s]: mm/h / 1000 / 3600 * dx (LIM_D4.m:198)
        x.y = outflow ? R(outflow[k] / 3.6e6 * res) : R(0);
        x.z = outflow ? R(outflow[n + k] / 3.6e6 * res) : R(0);
        x.w = ninf;
        st[k] = x;
    }
}
template <typename R> __global__ void k_fill(size_t n, R* p, R v) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        p[k] = v;
}
// one component of the state records (0..3 = h, q_x, q_y, dmax), for read-back
template <typename R>
__global__ void k_state_component(size_t n, const typename Vec<R>::V4* st, int comp, R* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const auto v = st[k];
        out[k] = comp == 0 ? v.x : comp == 1 ? v.y : comp == 2 ? v.z : v.w;
    }
}

// read-back into FP64: one component of the state records (0..3 = h, q_x, q_y, dmax) or a plain
// array, times `scale` (the conversion to the caller's units happens on the device)
template <typename R>
__global__ void k_state_component_f64(size_t n, const typename Vec<R>::V4* st, int comp, double scale, double* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const auto v = st[k];
        const R x = comp == 0 ? v.x : comp == 1 ? v.y : comp == 2 ? v.z : v.w;
        out[k] = double(x) * scale;
    }
}
template <typename R> __global__ void k_scaled_f64(size_t n, const R* src, double scale, double* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        out[k] = double(src[k]) * scale;
}
template <typename R> __global__ void k_divided_f64(size_t n, const R* src, double div, double* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        out[k] = double(src[k]) / div;
}
// the soil storage I of the soil records, times `scale`
template <typename R>
__global__ void k_soil_component_f64(size_t n, const typename Vec<R>::V2* gs, double scale, double* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x)
        out[k] = double(gs[k].x) * scale;
}
// qout_left (-q_x of the cell to the left, -0 on the first column) or qout_down (-q_y of the
// cell below, -0 on the last row) [mm/h] (Local_Inertial_Model_D4.m:347-350)
template <typename R>
__global__ void k_shifted_flux_f64(int ny, int nx, const typename Vec<R>::V4* st, int down, double scale, double* out) {
    const size_t n = size_t(ny) * nx;
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const int i = int(k / nx), j = int(k % nx);
        if (down) out[k] = i + 1 == ny ? -0.0 : -double(st[k + nx].z) * scale;
        else out[k] = j == 0 ? -0.0 : -double(st[k - 1].y) * scale;
    }
}
// CA_States.I_tot_end_cell [m^3] (Local_Inertial_Model_D4.m:512-514): |right + up + outlet flux|
// [mm/h] x dt over the cell area, from the state records and each outlet cell's sink rate
template <typename R>
__global__ void k_itot_f64(size_t n, const typename Vec<R>::V4* st, const typename Vec<R>::V4* stat, const R* qo,
                           double to_mmh, double dts, double res, double* out) {
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const auto v = st[k];
        const unsigned ord = outlet_ord(meta_bits(stat[k].w));
        const double of = ord ? double(qo[ord - 1]) * 3.6e6 : 0.0;
        out[k] = fabs(double(v.y) * to_mmh + double(v.z) * to_mmh + of) * dts / 1000.0 / 3600.0 * res * res;
    }
}

// a map record taken by the host when no step follows the one that triggered it
template <typename R> __global__ void k_record_depth(size_t n, const typename Vec<R>::V4* st, R* dst) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        dst[c] = st[c].x;
}

// gauge depths of the current rain interval (after a host change of the inflow or clock)
template <typename R> __global__ void k_inflow_depth(InflowDesc<R> d, const StepScalars* sc) {
    const double ra = sc->rain_a, rb = sc->rain_b, t = sc->t_min;
    for (int g = threadIdx.x; g < d.n_gauges; g += blockDim.x)
        d.depth[g] = R(inflow_integral(d, g, ra, rb) / 60000.0);
    for (int g = threadIdx.x; g < d.n_stage; g += blockDim.x) d.stage_now[g] = R(stage_at(d, g, t));
}

// Retry of a rejected step (HydroPol2D_Main_While.m:928-951): the reference's new step needs
// the wave celerity sqrt(g max(max(d_tot), max(d_p))) of the attempt.  Over the state the
// attempt started from (buffer cur, untouched by it) this restates phase (A) per cell -- rain,
// infiltration, inflow and clamps give d_tot -- and reduces max(d_p, d_tot) (NaN skipped, as
// MATLAB's max) into sc->retry_dmax.  It also takes back the arrival times the attempt wrote:
// a cell whose arrival equals the attempt's t_arr and whose start-of-step maximum is below the
// threshold was marked by it (a block of temporal blocking marks with the times of its
// sub-steps, the range [t_arr_lo, t_arr_hi]).  inf: 0 none, 1 Green-Ampt, 2 van Genuchten.
template <typename R>
__global__ void k_retry_scan(const FusedArgs<R> a, int inf, R t_arr_lo, R t_arr_hi) {
    StepScalars* sc = a.sc;
    RainStep<R> RS;
    RS.make(a.rain, sc->rain_a, sc->rain_b);
    StepConsts<R> K;
    K.make(sc->time_step * 60.0, a.res, a.tol_mm, a.thr_mm);
    const bool skip = sc->skip_clamp != 0;
    const typename Vec<R>::V4* st = sc->cur ? a.st1 : a.st0;
    const typename Vec<R>::V2* gs = sc->cur ? a.gs1 : a.gs0;
    const size_t n = size_t(a.ny) * a.nx;
    R m = R(0);
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int r = int(c / a.nx), j = int(c % a.nx);
        const auto rec = st[c];
        R hh = rec.x;
        m = fmax(m, hh);
        hh = hh + RS.at(a.rain, r, j, a.ny, a.nx);
        const unsigned meta = meta_bits(a.stat[c].w);
        if (inf && (meta & 255u) != 255u) {
            R Ic = gs[c].x, Tc = gs[c].y;
            if (inf == 1) green_ampt(hh, Ic, Tc, a.classes[meta & 255u], K);
            else vg_infiltration(hh, Ic, Tc, a.classes_vg[meta & 255u], a.vg, K);
        }
        if (a.inflow.n_gauges) add_inflow(a.inflow, meta, hh);
        if (!skip && hh < R(1e-9)) hh = R(0);
        if (hh < R(0)) hh = R(0);
        m = fmax(m, hh);
        const R ar = a.arrival[c];
        if (ar >= t_arr_lo && ar <= t_arr_hi && rec.w < K.thr) a.arrival[c] = R(__int_as_float(0x7f800000));
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m > R(0)) atomicMax(&sc->retry_dmax, ord_bits(m));
}

// the structure transfers of the first fused step of a call (one block)
template <typename R, int INF, bool MAP>
__global__ void k_struct_prime(const FusedArgs<R> a) {
    __shared__ RainStep<R> s_r;
    __shared__ StepConsts<R> s_k;
    __shared__ int s_skip, s_cur;
    __shared__ double s_ts;
    if (threadIdx.x == 0) {
        const StepScalars* sc = a.sc;
        s_r.make(a.rain, sc->rain_a, sc->rain_b);
        s_ts = sc->time_step;
        s_k.make(s_ts * 60.0, a.res, a.tol_mm, a.thr_mm);
        s_skip = sc->skip_clamp;
        s_cur = sc->cur;
    }
    __syncthreads();
    structure_prepare<R, INF, MAP, true>(a, s_r, s_skip != 0, s_k, s_cur ? a.st1 : a.st0, s_cur ? a.gs1 : a.gs0,
                                         threadIdx.x, blockDim.x, s_ts);
}

template <typename R, int NT, int INF, bool MAP, int CPL = 1, bool INFL = false, int SCH = 0>
__global__ void __launch_bounds__(NT, FusedOcc<R, CPL>::minb) k_fused_step(const FusedArgs<R> a) {
    fused_item<R, NT, INF, MAP, CPL, INFL, SCH>(a, blockIdx.x);
}

// ---- batched ensemble ----------------------------------------------------------------
// Members are independent grids, each with its own FusedArgs (clock, dt, buffers).  Each
// step, k_ens_plan lists the CTA-sized items of the members still running (exclusive
// prefix over members) and k_ens_step -- a persistent grid sized to the resident CTA
// slots -- pulls items from a queue head.  Items of one launch never wait on each other;
// the CTA that completes a member's last item refreshes that member's dt and clock.
struct EnsQueue {
    unsigned head;       // next item to hand out
    unsigned total;      // items of this step
    unsigned n_active;   // members running this step
    unsigned stalled;    // members stopped by a failed row copy
};

template <typename R>
__global__ void k_ens_plan(const FusedArgs<R>* __restrict__ members, int n_members, unsigned* prefix, EnsQueue* q) {
    // one CTA of 1024 threads; members are scanned in chunks of 1024
    __shared__ unsigned s_run[1024];
    __shared__ unsigned s_base, s_act, s_stall;
    const int tid = threadIdx.x;
    if (tid == 0) { s_base = 0; s_act = 0; s_stall = 0; }
    __syncthreads();
    for (int m0 = 0; m0 < n_members; m0 += 1024) {
        const int m = m0 + tid;
        unsigned items = 0;
        if (m < n_members) {
            const FusedArgs<R>& a = members[m];
            const StepScalars* sc = a.sc;
            const bool stalled = (sc->status & kStatusTimeout) != 0u;
            const bool running = sc->t_min <= a.t_end && !stalled && !sc->halted;
            items = running ? a.n_ctas : 0u;
            if (running) atomicAdd(&s_act, 1u);
            if (stalled) atomicAdd(&s_stall, 1u);
        }
        s_run[tid] = items;
        __syncthreads();
        // Hillis-Steele inclusive scan over the chunk
        for (int o = 1; o < 1024; o <<= 1) {
            const unsigned v = tid >= o ? s_run[tid - o] : 0u;
            __syncthreads();
            s_run[tid] += v;
            __syncthreads();
        }
        if (m < n_members) prefix[m] = s_base + s_run[tid] - items;
        __syncthreads();
        if (tid == 0) s_base += s_run[1023];
        __syncthreads();
    }
    if (tid == 0) {
        prefix[n_members] = s_base;
        q->head = 0;
        q->total = s_base;
        q->n_active = s_act;
        q->stalled = s_stall;
    }
}

template <typename R, int NT, int INF, bool MAP, int CPL = 1, bool INFL = false, int SCH = 0>
__global__ void __launch_bounds__(NT, FusedOcc<R, CPL>::minb)
k_ens_step(const FusedArgs<R>* __restrict__ members, int n_members, const unsigned* __restrict__ prefix,
           EnsQueue* q) {
    __shared__ FusedArgs<R> s_a;
    __shared__ unsigned s_item, s_local;
    __shared__ int s_m;
    const int tid = threadIdx.x;
    const unsigned total = q->total;   // written by k_ens_plan before this launch
    for (;;) {
        __syncthreads();   // the previous item is finished with s_a and the ring
        if (tid == 0) {
            const unsigned it = atomicAdd(&q->head, 1u);
            s_item = it;
            if (it < total) {
                // member m with prefix[m] <= it < prefix[m+1] (members without items have
                // prefix[m] == prefix[m+1] and are passed over)
                int lo = 0, hi = n_members - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (prefix[mid] <= it) lo = mid; else hi = mid - 1;
                }
                s_m = lo;
                s_local = it - prefix[lo];
            }
        }
        __syncthreads();
        if (s_item >= total) return;
        {
            const unsigned* src = reinterpret_cast<const unsigned*>(members + s_m);
            unsigned* dst = reinterpret_cast<unsigned*>(&s_a);
            for (int w = tid; w < int(sizeof(FusedArgs<R>) / 4); w += NT) dst[w] = src[w];
        }
        __syncthreads();
        if (!fused_item<R, NT, INF, MAP, CPL, INFL, SCH>(s_a, s_local)) return;   // ring unusable after a timeout
    }
}

// Clamp-skip flag for the first fused step of a call, over every cell (the state may
// have been set from the host).  sc->skip_clamp must be zero on entry.  Also counts the cells
// with a finite depth (n_finite) and with a non-finite one (n_bad0, the count a healthy step
// keeps), and flags a non-finite depth in a cell of finite elevation (bad_domain).
template <typename R>
__global__ void k_skip_flag(const typename Vec<R>::V4* st, const typename Vec<R>::V4* stat, int ny, int nx,
                            RainDesc rain, int ga, double res, double tol_mm, double thr_mm, StepScalars* sc,
                            int own_r0, int own_r1) {
    const size_t n = size_t(ny) * nx;
    RainStep<R> RS;
    RS.make(rain, sc->rain_a, sc->rain_b);
    int neg = 0;
    unsigned long long fin = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const R hc = st[c].x;
        const auto sr = stat[c];
        const int ci = int(c / nx);
        if (ci < own_r0 || ci >= own_r1) continue;   // a row slab counts its own rows only
        if (isfinite(hc)) ++fin;
        else {
            atomicAdd(&sc->n_bad0, 1ull);
            if (!isnan(sr.z)) atomicOr(&sc->bad_domain, 1);
        }
        if (ga && (meta_bits(sr.w) & 255u) != 255u) continue;
        const int i = int(c / nx), j = int(c % nx);
        if (hc + RS.at(rain, i, j, ny, nx) < R(-1e-11)) neg = 1;
    }
    for (int o = 16; o > 0; o >>= 1) fin += __shfl_xor_sync(0xffffffffu, fin, o);
    if ((threadIdx.x & 31) == 0 && fin) atomicAdd(&sc->n_finite, fin);
    if (__syncthreads_or(neg) && threadIdx.x == 0) atomicOr(&sc->skip_clamp, 1);
}

// SoA <-> record conversion for the unfused entry points
template <typename R>
__global__ void k_unpack(size_t n, const typename Vec<R>::V4* st, const typename Vec<R>::V2* gs, R* h, R* qx, R* qy,
                         R* dmax, R* I, R* T) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const auto v = st[c];
        h[c] = v.x;
        qx[c] = v.y;
        qy[c] = v.z;
        dmax[c] = v.w;
        if (gs) {
            const auto g = gs[c];
            I[c] = g.x;
            T[c] = g.y;
        }
    }
}
template <typename R>
__global__ void k_pack(size_t n, typename Vec<R>::V4* st, typename Vec<R>::V2* gs, const R* h, const R* qx,
                       const R* qy, const R* dmax, const R* I, const R* T) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        typename Vec<R>::V4 v;
        v.x = h[c];
        v.y = qx[c];
        v.z = qy[c];
        v.w = dmax[c];
        st[c] = v;
        if (gs) {
            typename Vec<R>::V2 g;
            g.x = I[c];
            g.y = T[c];
            gs[c] = g;
        }
    }
}

}  // namespace hp2d
