// Temporal blocking of the fused step (opt-in, hp2d_set_temporal_blocking): one launch advances
// K accepted steps at the fixed time step of the last refresh; the refresh (refreshing_timestep)
// runs at the end of the block, from the block's last state.  The reference refreshes every step
// (time_step_change is a fraction of the smallest step), so results differ from the per-step
// path by the frozen time step; the kernel-form oracle restates the same schedule (a refresh only
// on step 1 and on the steps k with (k - 1) % K == 0).
//
// A CTA owns a tile of 64 x 32 output cells.  One TMA copy brings the tile's static and state
// records with a halo of 2K cells on every side into shared memory (3-D boxes over the record
// arrays viewed as [ny][nx][4] floats; the halo reaches outside the grid as zeros, and the
// static records there are set to closed faces).  Sub-step s then updates, in four passes
// separated by CTA barriers, the cells 2s away from the halo's outer edge: the draining
// limiter's dependency radius is 2 (face <- donor scale <- donor's faces <- their cells), so
// after K sub-steps the 64 x 32 output cells are exact.  The output cells' records go back to
// HBM once per block: per step the tile moves (48 B x (1 + halo) + 16 B) / K per cell.
//
// Within a block the clamp of the next step's depth (Hydrological_Model.m:45-50) is applied
// unless an outlet cell ended a sub-step below -1e-11 m -- a decision over the whole grid that a
// tile cannot make -- so a block in which that happens is not committed and the host replays its
// steps one per launch (the same rollback as a rejected step).  Rain, infiltration, inflow,
// stage, control structures, map records and hazard maps are not supported in this mode.
#pragma once

#include <cuda.h>

#include "hp2d_device.cuh"
#include "hp2d_fused.cuh"

namespace hp2d {

constexpr int kTbTX = 64;        // output columns of a tile
constexpr int kTbTY = 32;        // output rows of a tile
constexpr int kTbThreads = 512;
constexpr unsigned kStatusTbReplay = 8u;   // StepScalars::status: replay the block step by step

template <int K> struct TbGeom {
    static constexpr int H = 2 * K;                 // halo
    static constexpr int EX = kTbTX + 2 * H, EY = kTbTY + 2 * H, NE = EX * EY;
    // static records (16 B) and the state records' landing zone (16 B, later qxu, qyu, hfx,
    // hfy) per halo cell, h, qx, qy and the donor scale per halo cell, dmax per output cell
    static constexpr size_t smem = size_t(NE) * 16 * 2 + size_t(NE) * 4 * 4 + size_t(kTbTX) * kTbTY * 4;
};

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}


template <int K>
__global__ void __launch_bounds__(kTbThreads, 1)
k_tb_block(const FusedArgs<float> a, const __grid_constant__ CUtensorMap tm_st0,
           const __grid_constant__ CUtensorMap tm_st1, const __grid_constant__ CUtensorMap tm_stat, int ntx) {
    using G = TbGeom<K>;
    constexpr int EX = G::EX, EY = G::EY, NE = G::NE, H = G::H;
    constexpr int NT = kTbThreads;
    extern __shared__ __align__(128) unsigned char smem_tb[];
    float4* s_stat = reinterpret_cast<float4*>(smem_tb);
    float4* s_land = s_stat + NE;
    float* s_qxu = reinterpret_cast<float*>(s_land);
    float* s_qyu = s_qxu + NE;
    float* s_hfx = s_qyu + NE;
    float* s_hfy = s_hfx + NE;
    float* s_h = reinterpret_cast<float*>(s_land + NE);
    float* s_qx = s_h + NE;
    float* s_qy = s_qx + NE;
    float* s_sc = s_qy + NE;
    float* s_dm = s_sc + NE;
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ double s_tmin, s_ts;
    __shared__ int s_cur, s_skip, s_done, s_keff, s_last, s_to, s_replay, s_negn;
    __shared__ float red_s2[NT / 32];
    __shared__ unsigned long long red_c[NT / 32];
    __shared__ double red_o[NT / 32];
    __shared__ unsigned red_b[NT / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    StepScalars* sc = a.sc;
    if (tid == 0) {
        s_tmin = sc->t_min;
        s_ts = sc->time_step;
        s_cur = sc->cur;
        s_skip = sc->skip_clamp;
        s_to = 0;
        s_replay = 0;
        s_negn = 0;
        // sub-steps that run: those starting at or before the end of the simulation
        int keff = 0;
        double t = s_tmin;
        for (int s = 0; s < K && t <= a.t_end; ++s) {
            ++keff;
            t = (s_ts * 60.0) / 60.0 + t;
        }
        s_keff = keff;
        s_done = keff == 0 || sc->halted;
    }
    __syncthreads();
    if (s_done) return;
    const int keff = s_keff;
    const int ny = a.ny, nx = a.nx;
    const int ty = int(blockIdx.x) / ntx, tx = int(blockIdx.x) % ntx;
    const int gx0 = tx * kTbTX - H, gy0 = ty * kTbTY - H;   // global cell of halo cell (0, 0)
    StepConsts<float> Kc;
    Kc.make(s_ts * 60.0, a.res, a.tol_mm, a.thr_mm);

    // ---- the tile's records by TMA (halo included; outside the grid reads zeros) ------------
    const uint32_t bar = smem_addr(&s_bar);
    if (tid == 0) {
        mbar_init(bar, 1u);
        mbar_fence_init();
        mbar_expect_tx(bar, uint32_t(2 * NE * 16));
        tma_load_3d(smem_addr(s_stat), &tm_stat, 0, gx0, gy0, bar);
        tma_load_3d(smem_addr(s_land), s_cur ? &tm_st1 : &tm_st0, 0, gx0, gy0, bar);
    }
    __syncthreads();
    if (!mbar_wait_bounded(bar, 0u, a.wait_polls)) {
        s_to = 1;   // benign race: every writer stores 1
        mbar_wait_bounded(bar, 0u, 1u << 22);   // let the copies land before anything else
    }
    __syncthreads();
    const bool timed_out = s_to != 0;

    float s2max = 0.f, cmaxv = -1.f;
    Kahan<float> out_k;
    unsigned nbad = 0u;
    if (!timed_out) {
        // records outside the grid: closed faces, no outlet; the first step's clamp
        for (int e = tid; e < NE; e += NT) {
            const int gi = gy0 + e / EX, gj = gx0 + e % EX;
            const float4 rec = s_land[e];
            if (gi < 0 || gi >= ny || gj < 0 || gj >= nx)
                s_stat[e] = make_float4(__int_as_float(0x7f800000), __int_as_float(0x7f800000), 0.f,
                                        make_meta<float>(255u));
            float hh = rec.x;
            if (!s_skip && hh < 1e-9f) hh = 0.f;
            if (hh < 0.f) hh = 0.f;
            s_h[e] = hh;
            s_qx[e] = rec.y;
            s_qy[e] = rec.z;
            const int oi = e / EX - H, oj = e % EX - H;
            if (oi >= 0 && oi < kTbTY && oj >= 0 && oj < kTbTX) s_dm[oi * kTbTX + oj] = rec.w;
        }
        __syncthreads();

        double t_s = s_tmin;   // clock at the start of sub-step s, as the per-step finalize advances it
        for (int s = 1; s <= keff; ++s) {
            const int lo = 2 * (s - 1), hx = EX - 2 * (s - 1), hy = EY - 2 * (s - 1);
            // (B)+(C) unlimited faces of the cells whose depth is valid
            {
                const int w = hx - lo, n = w * (hy - lo);
                for (int q = tid; q < n; q += NT) {
                    const int i = lo + q / w, j = lo + q % w, e = i * EX + j;
                    const float4 st = s_stat[e];
                    const float hc = s_h[e];
                    const float hr = j + 1 < EX ? s_h[e + 1] : 0.f;
                    const float hu = i >= 1 ? s_h[e - EX] : 0.f;
                    float Hx, Sx, Hy, Sy;
                    const bool wx = face_geom<float, true>(hc, hr, st.x, Hx, Sx, Kc) && j + 1 < EX;
                    const bool wy = face_geom<float, false>(hu, hc, st.y, Hy, Sy, Kc) && i >= 1;
                    s_hfx[e] = j + 1 < EX ? Hx : 0.f;
                    s_hfy[e] = i >= 1 ? Hy : 0.f;
                    s_qxu[e] = face_momentum<float>(wx, Hx, Sx, s_qx[e], st.z, Kc, a.flag_critical);
                    s_qyu[e] = face_momentum<float>(wy, Hy, Sy, s_qy[e], st.z, Kc, a.flag_critical);
                }
            }
            __syncthreads();
            // (D) donor scales
            {
                const int l = lo + 1, w = hx - 1 - l, n = w * (hy - 1 - l);
                for (int q = tid; q < n; q += NT) {
                    const int i = l + q / w, j = l + q % w, e = i * EX + j;
                    s_sc[e] = donor_scale_finite(s_qxu[e], s_qxu[e - 1], s_qyu[e], s_qyu[e + EX], s_h[e], Kc);
                }
            }
            __syncthreads();
            // (E) limited faces: the new fluxes (the previous ones were read in (B)/(C))
            {
                const int l = lo + 1, w = hx - 2 - l, n = w * (hy - 1 - (l + 1));
                for (int q = tid; q < n; q += NT) {
                    const int i = l + 1 + q / w, j = l + q % w, e = i * EX + j;
                    s_qx[e] = limit_face_finite(s_qxu[e], s_sc[e], s_sc[e + 1]);
                    s_qy[e] = limit_face_finite(s_qyu[e], s_sc[e], s_sc[e - EX]);
                }
            }
            __syncthreads();
            // (F) continuity, outlets, maxima / arrival of the output cells, CFL at the end
            {
                const int l = lo + 2, w = hx - 2 - l, n = w * (hy - 2 - l);
                const float t_arr = float(t_s * 60.0 + s_ts * 60.0);
                for (int q = tid; q < n; q += NT) {
                    const int i = l + q / w, j = l + q % w, e = i * EX + j;
                    float hn = continuity(s_h[e], s_qx[e - 1], s_qx[e], s_qy[e], s_qy[e + EX], Kc);
                    const int oi = i - H, oj = j - H;
                    const bool out = oi >= 0 && oi < kTbTY && oj >= 0 && oj < kTbTX && gy0 + i < ny && gx0 + j < nx;
                    const unsigned ord = outlet_ord(meta_bits(s_stat[e].w));
                    float hf3 = 0.f;
                    if (ord) {
                        float ho;
                        const float qq = outlet_sink(hn, a.outlet_coef[ord - 1], a.outlet_type, Kc, ho);
                        hf3 = ho;
                        if (out) {
                            if (s == keff) {
                                a.hf3[ord - 1] = ho;
                                a.qo[ord - 1] = qq;
                            }
                            out_k.add(qq * Kc.dt);
                            if (hn < -1e-11f) {
                                if (s < keff) s_replay = 1;
                                else s_negn = 1;
                            }
                        }
                    }
                    if (out) {
                        nbad += (hn >= -Kc.tol) ? 0u : 1u;
                        const size_t c = size_t(gy0 + i) * nx + (gx0 + j);
                        const float dm = s_dm[oi * kTbTX + oj];
                        if (dm < Kc.thr && hn >= Kc.thr) a.arrival[c] = t_arr;
                        s_dm[oi * kTbTX + oj] = hn > dm ? hn : dm;
                        if (s == keff) {   // refreshing_timestep's per-cell terms of the last state
                            const float big = 1e9f;
                            const float vr = qdiv(s_qx[e], s_hfx[e] < Kc.tol ? big : s_hfx[e]);
                            const float vu = qdiv(s_qy[e], s_hfy[e] < Kc.tol ? big : s_hfy[e]);
                            const float vb = qdiv(s_qy[e + EX], s_hfy[e + EX] < Kc.tol ? big : s_hfy[e + EX]);
                            const float rc = gx0 + j == 0 ? 0.5f * vr : vr;
                            const float uc = 0.5f * (vu + vb);
                            const float s2 = rc * rc + uc * uc;
                            s2max = fmaxf(s2max, s2);
                            if (s2 >= a.stag_s2) {
                                const float dts = fmaxf(fmaxf(s_hfx[e], s_hfy[e]), hf3);
                                float cval;
                                if (a.adaptive == 1) {
                                    cval = Kc.g * fmaxf(dts, 0.f);
                                } else {
                                    const float wc = fmaxf(sqrtf(Kc.g * fmaxf(dts, 0.f)), 1e-10f);
                                    cval = fmaxf(fmaxf(fabsf(vr), fabsf(vu)), fabsf(vb)) + wc;
                                }
                                cmaxv = fmaxf(cmaxv, cval);
                            }
                        }
                    }
                    // the next sub-step's depth entering its fluxes: the clamp without the skip
                    // (a block whose outlets asked for the skip is replayed)
                    if (s < keff) {
                        if (hn < 1e-9f) hn = 0.f;
                    }
                    s_h[e] = hn;
                }
            }
            t_s = (s_ts * 60.0) / 60.0 + t_s;
            __syncthreads();
        }
        // ---- the output cells' records back to HBM ----------------------------------------
        float4* sout = s_cur ? a.st0 : a.st1;
        for (int q = tid; q < kTbTX * kTbTY; q += NT) {
            const int oi = q / kTbTX, oj = q % kTbTX;
            const int gi = ty * kTbTY + oi, gj = tx * kTbTX + oj;
            if (gi < ny && gj < nx) {
                const int e = (oi + H) * EX + (oj + H);
                sout[size_t(gi) * nx + gj] = make_float4(s_h[e], s_qx[e], s_qy[e], s_dm[q]);
            }
        }
    }

    // ---- CTA reductions, then the block's bookkeeping in the last CTA ----------------------
    s2max = warp_max(s2max);
    unsigned long long cenc = cmaxv >= 0.f ? ord_bits(cmaxv + 0.f) + 1ull : 0ull;
    cenc = warp_max_u(cenc);
    double out_acc = warp_sum(out_k.value());
    nbad = __reduce_add_sync(0xffffffffu, nbad);
    if (lane == 0) {
        red_s2[warp] = s2max;
        red_c[warp] = cenc;
        red_o[warp] = out_acc;
        red_b[warp] = nbad;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned bad = 0u;
        for (int w = 0; w < NT / 32; ++w) {
            s2max = fmaxf(s2max, red_s2[w]);
            cenc = red_c[w] > cenc ? red_c[w] : cenc;
            bad += red_b[w];
            if (w) out_acc += red_o[w];
        }
        if (s2max > 0.f) atomicMax(&sc->acc_vmax, ord_bits(s2max));
        if (cenc) atomicMax(&sc->acc_cmax, cenc);
        if (out_acc != 0.0) atomicAdd(&sc->acc_out, out_acc);
        if (bad) atomicAdd(&sc->acc_bad, (unsigned long long)bad);
        if (timed_out) atomicOr(&sc->status, kStatusTimeout);
        if (s_replay) atomicOr(&sc->status, kStatusTbReplay);
        if (s_negn) atomicOr(&sc->skip_next, 1);
        __threadfence();
        const unsigned ticket = atomicAdd(&sc->counter, 1u);
        s_last = ticket == a.n_ctas - 1;
    }
    __syncthreads();
    if (!s_last || tid != 0) return;
    __threadfence();
    // A block is not committed when a row copy timed out (the call reports HP2D_TIMEOUT), or when
    // it cannot stand for the per-step path: an outlet cell asked for the clamp skip inside it,
    // a depth went non-finite or too negative, or the test hook names one of its steps.  Those
    // blocks are replayed one step per launch by the host, where the per-step rules (and the
    // retry of a rejected step) apply; the test hook's attempts are left for the replay.
    const unsigned status = atomicAdd(&sc->status, 0u);
    bool reject = (status & (kStatusTimeout | kStatusTbReplay)) != 0u;
    if (atomicAdd(&sc->acc_bad, 0ull) > sc->n_bad0 * (unsigned long long)keff ||
        (sc->fault_n > 0 && sc->fault_k >= sc->k && sc->fault_k < sc->k + keff)) {
        reject = true;
        if (!(status & kStatusTimeout)) sc->status |= kStatusTbReplay;
    }
    if (reject) {
        sc->halted = 1;
    } else {
        const double area = a.res * a.res;
        sc->out_vol += atomicAdd(&sc->acc_out, 0.0) * area;
        if (s_skip) sc->neg_warn += 1;   // the block's first step ran without the clamp
        for (int s = 0; s < keff; ++s) {   // the per-step bookkeeping of each sub-step
            const double t = sc->t_min;
            const double pos_save = ceil((t * 60.0) / a.tsc);
            const double time_save = (pos_save - 1.0) * a.tsc / 60.0;
            const double delta = time_save - sc->tsp;
            sc->tsp = time_save;
            double tcr = sc->time_step * 60.0;
            if (s == K - 1 && (delta > 0 || sc->k == 1)) {   // the block's last step refreshes
                const unsigned long long vbits = atomicAdd(&sc->acc_vmax, 0ull);
                const unsigned long long cbits = atomicAdd(&sc->acc_cmax, 0ull);
                const double vm = double(sqrtf(__uint_as_float(unsigned(vbits))));
                double cm = 0.0;
                if (cbits) {
                    const float v = __uint_as_float(unsigned(cbits - 1ull));
                    cm = a.adaptive == 1 ? double(fmaxf(sqrtf(v), 1e-10f)) : double(v);
                }
                tcr = finalize_dt(vm, cm, a.res, a.alfa_min, a.alfa_max, a.min_dt, sc->max_dt, a.inc, a.flag_timestep);
                sc->vmax_last = vm;
                if (tcr == a.min_dt) {
                    sc->unstable += 1;
                    if (sc->dt_floor_stop) {
                        sc->status |= kStatusDtFloor;
                        sc->halted = 1;
                    }
                }
            }
            sc->rain_a = sc->t_prev;
            sc->rain_b = t;
            sc->t_prev = sc->k == 1 ? tcr / 60.0 : t;
            sc->time_step = tcr / 60.0;
            sc->t_min = tcr / 60.0 + t;
            sc->k += 1;
        }
        sc->cur = s_cur ^ 1;
        sc->skip_clamp = atomicExch(&sc->skip_next, 0);
    }
    sc->acc_vmax = 0ull;
    sc->acc_cmax = 0ull;
    sc->acc_out = 0.0;
    sc->acc_bad = 0ull;
    sc->counter = 0u;
    if (reject) atomicExch(&sc->skip_next, 0);
}

}  // namespace hp2d
