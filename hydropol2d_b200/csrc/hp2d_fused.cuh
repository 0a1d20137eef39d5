// Fused surface-flow step: one launch = one accepted step of HydroPol2D_Main_While.m
// :403-782 (rain + Green-Ampt + clamp, local-inertial fluxes, draining limiter,
// continuity, outlet sink, running maximum / arrival time, CFL reductions, and the
// timestep refresh + clock advance done by the last CTA to finish).
//
// Tiling: each CTA owns a BY x BX block of cells.  The draining limiter makes a cell's
// new depth depend on cells two away (face <- donor scale <- donor's four faces <- their
// far cells), so the CTA stages a (BY+4) x (BX+4) depth tile (hydrology applied in
// place), computes the faces touching cells within one cell of the block, the donor
// scales within one cell, the limited faces of the block, and the block's continuity.
// All of that lives in shared memory; the only global traffic is one read of each input
// field and one write of each output field (halo reads mostly hit L2).
//
// The state is double-buffered (StepScalars::cur selects the read side), so a CUDA graph
// of many launches needs no host involvement, and a launch after the end of the
// simulation is a no-op that leaves the buffers and the clock alone.
#pragma once

#include "hp2d_device.cuh"

namespace hp2d {

template <typename R> struct FusedArgs {
    int ny, nx;
    double res;
    double tol_mm, thr_mm;
    double t_end;                // routing_time + min_time_step/60 [min]
    double min_dt, max_dt, inc, tsc, alfa_min, alfa_max;
    int flag_timestep, adaptive, flag_critical, outlet_type, ga;
    unsigned int n_ctas;
    const R* dzx; const R* dzy; const R* n2;
    const uint8_t* soil; const SoilClass<R>* classes;
    const uint32_t* outlet_bits; int bit_words;   // words per row
    const int32_t* outlet_cells; const R* outlet_coef; int n_outlets;
    R* hf3; R* qo;
    R* h0; R* h1; R* qx0; R* qx1; R* qy0; R* qy1; R* I0; R* I1; R* T0; R* T1;
    R* dmax; R* arrival;
    RainDesc rain;
    StepScalars* sc;
};

__device__ inline double finalize_dt(double vmax, double cmax, double res, double alfa_min,
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

template <typename R> __device__ __forceinline__ R warp_max(R v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R, int BY, int BX>
struct FusedSmem {
    static constexpr int HH = BY + 4, HW = BX + 4;   // depth tile, origin (r0-2, c0-2)
    static constexpr int XH = BY + 2, XW = BX + 3;   // x faces, origin (r0-1, c0-2)
    static constexpr int YH = BY + 3, YW = BX + 2;   // y faces, origin (r0-1, c0-1)
    static constexpr int SH = BY + 2, SW = BX + 2;   // donor scale, origin (r0-1, c0-1)
    static constexpr size_t n_elems = size_t(HH) * HW + 2 * size_t(XH) * XW + 2 * size_t(YH) * YW + size_t(SH) * SW;
    static constexpr size_t bytes = n_elems * sizeof(R);
};

template <typename R, int BY, int BX, int NT>
__global__ void __launch_bounds__(NT) k_fused_step(const FusedArgs<R> a) {
    using SM = FusedSmem<R, BY, BX>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sH = reinterpret_cast<R*>(smem_raw);
    R* sQx = sH + SM::HH * SM::HW;
    R* sHx = sQx + SM::XH * SM::XW;
    R* sQy = sHx + SM::XH * SM::XW;
    R* sHy = sQy + SM::YH * SM::YW;
    R* sS = sHy + SM::YH * SM::YW;

    __shared__ StepConsts<R> K;
    __shared__ double s_tmin, s_dts;
    __shared__ int s_cur, s_skip, s_done, s_map, s_last;
    __shared__ R s_rain;
    __shared__ R red_r[2][NT / 32];
    __shared__ double red_d[3][NT / 32];

    const int tid = threadIdx.x;
    if (tid == 0) {
        StepScalars* sc = a.sc;
        s_tmin = sc->t_min;
        s_dts = sc->time_step * 60.0;
        s_cur = sc->cur;
        s_skip = sc->skip_clamp;
        s_done = !(s_tmin <= a.t_end);
        K.make(s_dts, a.res, a.tol_mm, a.thr_mm);
        s_rain = a.rain.n_uniform ? R(uniform_rate(a.rain, s_tmin)) : R(0);
        s_map = a.rain.n_maps ? map_index(a.rain, s_tmin) : -1;
        if (!s_done && s_skip && blockIdx.x == 0 && blockIdx.y == 0) sc->neg_warn += 1;
    }
    __syncthreads();
    if (s_done) return;

    const int ny = a.ny, nx = a.nx;
    const int r0 = blockIdx.y * BY, c0 = blockIdx.x * BX;
    const int cur = s_cur;
    const R* hin = cur ? a.h1 : a.h0;
    const R* qxin = cur ? a.qx1 : a.qx0;
    const R* qyin = cur ? a.qy1 : a.qy0;
    const R* Iin = cur ? a.I1 : a.I0;
    const R* Tin = cur ? a.T1 : a.T0;
    R* hout = cur ? a.h0 : a.h1;
    R* qxout = cur ? a.qx0 : a.qx1;
    R* qyout = cur ? a.qy0 : a.qy1;
    R* Iout = cur ? a.I0 : a.I1;
    R* Tout = cur ? a.T0 : a.T1;
    const float* map = s_map >= 0 ? a.rain.maps + size_t(s_map) * a.rain.my * a.rain.mx : nullptr;

    double rain_acc = 0.0, inf_acc = 0.0, out_acc = 0.0;

    // ---- phase 0: depth tile with rain, Green-Ampt and the clamp ----------------------
    for (int e = tid; e < SM::HH * SM::HW; e += NT) {
        const int li = e / SM::HW, lj = e - li * SM::HW;
        const int i = r0 - 2 + li, j = c0 - 2 + lj;
        R hh = R(0);
        if (i >= 0 && i < ny && j >= 0 && j < nx) {
            const size_t c = size_t(i) * nx + j;
            const bool own = li >= 2 && li < BY + 2 && lj >= 2 && lj < BX + 2;
            hh = hin[c];
            const R rate = map ? map_rate<R>(a.rain, map, i, j, ny, nx) : s_rain;
            const R r = rate * K.rain_scale;
            hh = hh + r;
            if (own && isfinite(hh)) rain_acc += double(r);
            if (a.ga) {
                const uint8_t s = a.soil[c];
                if (s != 255) {
                    R Ic = Iin[c], Tc = Tin[c];
                    const R fd = green_ampt(hh, Ic, Tc, a.classes[s], K);
                    if (own) {
                        Iout[c] = Ic;
                        Tout[c] = Tc;
                        if (isfinite(fd)) inf_acc += double(fd);
                    }
                } else if (own) {
                    Iout[c] = Iin[c];
                    Tout[c] = Tin[c];
                }
            }
            if (!s_skip && hh < R(1e-9)) hh = R(0);
            if (hh < R(0)) hh = R(0);
        }
        sH[li * SM::HW + lj] = hh;
    }
    __syncthreads();

    // ---- phase 1: unlimited face fluxes ----------------------------------------------
    for (int e = tid; e < SM::XH * SM::XW; e += NT) {
        const int li = e / SM::XW, lj = e - li * SM::XW;
        const int i = r0 - 1 + li, j = c0 - 2 + lj;
        R Hf = R(0), q = R(0);
        if (i >= 0 && i < ny && j >= 0 && j < nx) {
            const size_t c = size_t(i) * nx + j;
            const R dz = a.dzx[c];
            if (!isnan(dz)) {
                const R ha = sH[(li + 1) * SM::HW + lj], hb = sH[(li + 1) * SM::HW + lj + 1];
                face_flux<R, true>(ha, hb, dz, qxin[c], a.n2[c], K, a.flag_critical, Hf, q);
            }
        }
        sQx[e] = q;
        sHx[e] = Hf;
    }
    for (int e = tid; e < SM::YH * SM::YW; e += NT) {
        const int li = e / SM::YW, lj = e - li * SM::YW;
        const int i = r0 - 1 + li, j = c0 - 1 + lj;
        R Hf = R(0), q = R(0);
        if (i >= 0 && i < ny && j >= 0 && j < nx) {
            const size_t c = size_t(i) * nx + j;
            const R dz = a.dzy[c];
            if (!isnan(dz)) {
                const R ha = sH[li * SM::HW + lj + 1], hb = sH[(li + 1) * SM::HW + lj + 1];
                face_flux<R, false>(ha, hb, dz, qyin[c], a.n2[c], K, a.flag_critical, Hf, q);
            }
        }
        sQy[e] = q;
        sHy[e] = Hf;
    }
    __syncthreads();

    // ---- phase 2: donor scale factors ------------------------------------------------
    for (int e = tid; e < SM::SH * SM::SW; e += NT) {
        const int li = e / SM::SW, lj = e - li * SM::SW;
        const int i = r0 - 1 + li, j = c0 - 1 + lj;
        R s = R(1);
        if (i >= 0 && i < ny && j >= 0 && j < nx) {
            const R qR = sQx[li * SM::XW + lj + 1];
            const R qL = sQx[li * SM::XW + lj];
            const R qU = sQy[li * SM::YW + lj];
            const R qD = sQy[(li + 1) * SM::YW + lj];
            s = donor_scale(qR, qL, qU, qD, sH[(li + 1) * SM::HW + lj + 1], K);
        }
        sS[e] = s;
    }
    __syncthreads();

    // ---- phase 3: limited faces of the block (in place) ------------------------------
    for (int e = tid; e < BY * (BX + 1); e += NT) {
        const int ra = e / (BX + 1), cb = e - ra * (BX + 1);
        R* q = &sQx[(ra + 1) * SM::XW + cb + 1];
        *q = limit_face(*q, sS[(ra + 1) * SM::SW + cb], sS[(ra + 1) * SM::SW + cb + 1]);
    }
    for (int e = tid; e < (BY + 1) * BX; e += NT) {
        const int ra = e / BX, cb = e - ra * BX;
        R* q = &sQy[(ra + 1) * SM::YW + cb + 1];
        *q = limit_face(*q, sS[(ra + 1) * SM::SW + cb + 1], sS[ra * SM::SW + cb + 1]);
    }
    __syncthreads();

    // ---- phase 4: continuity, outlet, maxima, CFL -------------------------------------
    R vmax = R(0), cmax = R(0);
    const R t_arr = R(s_tmin * 60.0 + s_dts);
    for (int e = tid; e < BY * BX; e += NT) {
        const int ra = e / BX, cb = e - ra * BX;
        const int i = r0 + ra, j = c0 + cb;
        if (i >= ny || j >= nx) continue;
        const size_t c = size_t(i) * nx + j;
        const R htot = sH[(ra + 2) * SM::HW + cb + 2];
        const R qR = sQx[(ra + 1) * SM::XW + cb + 2];
        const R qL = sQx[(ra + 1) * SM::XW + cb + 1];
        const R qU = sQy[(ra + 1) * SM::YW + cb + 1];
        const R qD = sQy[(ra + 2) * SM::YW + cb + 1];
        R hn = continuity(htot, qL, qR, qU, qD, K);
        R hf3 = R(0);
        if (a.n_outlets && ((__ldg(a.outlet_bits + size_t(i) * a.bit_words + (j >> 5)) >> (j & 31)) & 1u)) {
            const int o = find_outlet(a.outlet_cells, a.n_outlets, int(c));
            if (o >= 0) {
                R ho;
                const R qq = outlet_sink(hn, a.outlet_coef[o], a.outlet_type, K, ho);
                hf3 = ho;
                a.hf3[o] = ho;
                a.qo[o] = qq;
                out_acc += double(qq * K.dt);
            }
        }
        const R dm = a.dmax[c];
        if (dm < K.thr && hn >= K.thr) a.arrival[c] = t_arr;
        if (hn > dm) a.dmax[c] = hn;
        R speed, celer;
        cfl_cell(qR, qU, qD, sHx[(ra + 1) * SM::XW + cb + 2], sHy[(ra + 1) * SM::YW + cb + 1],
                 sHy[(ra + 2) * SM::YW + cb + 1], hf3, j == 0, a.adaptive, K, speed, celer);
        vmax = fmax(vmax, speed);
        cmax = fmax(cmax, celer);
        hout[c] = hn;
        qxout[c] = qR;
        qyout[c] = qU;
    }

    // ---- CTA reductions ---------------------------------------------------------------
    // every thread publishes its stores before the CTA takes its ticket, so the last
    // CTA can read the new outlet depths
    __threadfence();
    const int lane = tid & 31, warp = tid >> 5;
    vmax = warp_max(vmax);
    cmax = warp_max(cmax);
    rain_acc = warp_sum(rain_acc);
    inf_acc = warp_sum(inf_acc);
    out_acc = warp_sum(out_acc);
    if (lane == 0) {
        red_r[0][warp] = vmax;
        red_r[1][warp] = cmax;
        red_d[0][warp] = rain_acc;
        red_d[1][warp] = inf_acc;
        red_d[2][warp] = out_acc;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < NT / 32; ++w) {
            vmax = fmax(vmax, red_r[0][w]);
            cmax = fmax(cmax, red_r[1][w]);
            rain_acc += red_d[0][w];
            inf_acc += red_d[1][w];
            out_acc += red_d[2][w];
        }
        StepScalars* sc = a.sc;
        if (vmax > R(0)) atomicMax(&sc->acc_vmax, ord_bits(vmax));
        if (cmax > R(0)) atomicMax(&sc->acc_cmax, ord_bits(cmax));
        if (rain_acc != 0.0) atomicAdd(&sc->acc_rain, rain_acc);
        if (inf_acc != 0.0) atomicAdd(&sc->acc_inf, inf_acc);
        if (out_acc != 0.0) atomicAdd(&sc->acc_out, out_acc);
        __threadfence();
        const unsigned int ticket = atomicAdd(&sc->counter, 1u);
        s_last = (ticket == a.n_ctas - 1);
    }
    __syncthreads();
    if (!s_last) return;

    // ---- last CTA: refreshing_timestep + clock (HydroPol2D_Main_While.m:691-705, :779)
    __threadfence();
    __shared__ double s_tnew, s_dtnew;
    if (tid == 0) {
        StepScalars* sc = a.sc;
        const bool is_d = sizeof(R) == 8;
        const double vm = from_ord(atomicAdd(&sc->acc_vmax, 0ull), is_d);
        const double cm = from_ord(atomicAdd(&sc->acc_cmax, 0ull), is_d);
        const double rain_s = atomicAdd(&sc->acc_rain, 0.0);
        const double inf_s = atomicAdd(&sc->acc_inf, 0.0);
        const double out_s = atomicAdd(&sc->acc_out, 0.0);
        const double t = s_tmin;
        const double pos_save = ceil((t * 60.0) / a.tsc);
        const double time_save = (pos_save - 1.0) * a.tsc / 60.0;
        const double delta = time_save - sc->tsp;
        sc->tsp = time_save;
        double tcr = sc->time_step * 60.0;   // refreshing_timestep.m:361-365
        if (delta > 0 || sc->k == 1) {
            tcr = finalize_dt(vm, cm, a.res, a.alfa_min, a.alfa_max, a.min_dt, a.max_dt, a.inc,
                              a.flag_timestep);
            sc->vmax_last = vm;
            if (tcr == a.min_dt) sc->unstable += 1;
        }
        const double area = a.res * a.res;
        sc->rain_vol += rain_s * area;
        sc->inf_vol += inf_s * area;
        sc->out_vol += out_s * area;
        sc->time_step = tcr / 60.0;
        sc->t_min = tcr / 60.0 + t;
        sc->k += 1;
        sc->cur = cur ^ 1;
        sc->acc_vmax = 0ull;
        sc->acc_cmax = 0ull;
        sc->acc_rain = 0.0;
        sc->acc_inf = 0.0;
        sc->acc_out = 0.0;
        sc->counter = 0u;
        s_tnew = sc->t_min;
        s_dtnew = sc->time_step * 60.0;
    }
    __syncthreads();
    // skip flag of the next step's clamp: only outlet cells can hold a negative depth
    // after a step (continuity clamps every other cell at zero).
    int neg = 0;
    if (a.n_outlets) {
        StepConsts<R> K2;
        K2.make(s_dtnew, a.res, a.tol_mm, a.thr_mm);
        const int m2 = a.rain.n_maps ? map_index(a.rain, s_tnew) : -1;
        const float* map2 = m2 >= 0 ? a.rain.maps + size_t(m2) * a.rain.my * a.rain.mx : nullptr;
        const R ru = a.rain.n_uniform ? R(uniform_rate(a.rain, s_tnew)) : R(0);
        for (int o = tid; o < a.n_outlets; o += NT) {
            const int c = a.outlet_cells[o];
            if (a.ga && a.soil[c] != 255) continue;
            const int i = c / nx, j = c - (c / nx) * nx;
            const R rate = map2 ? map_rate<R>(a.rain, map2, i, j, ny, nx) : ru;
            const R hv = __ldcg(hout + c) + rate * K2.rain_scale;
            if (hv < R(-1e-11)) neg = 1;
        }
    }
    neg = __syncthreads_or(neg);
    if (tid == 0) a.sc->skip_clamp = neg;
}

// Clamp-skip flag for the first fused step of a call, over every cell (the state may
// have been set from the host).  sc->skip_clamp must be zero on entry.
template <typename R>
__global__ void k_skip_flag(const R* h, int ny, int nx, RainDesc rain, const uint8_t* soil, int ga,
                            double res, double tol_mm, double thr_mm, StepScalars* sc) {
    const size_t n = size_t(ny) * nx;
    const double t = sc->t_min, dts = sc->time_step * 60.0;
    StepConsts<R> K;
    K.make(dts, res, tol_mm, thr_mm);
    const int m = rain.n_maps ? map_index(rain, t) : -1;
    const float* map = m >= 0 ? rain.maps + size_t(m) * rain.my * rain.mx : nullptr;
    const R ru = rain.n_uniform ? R(uniform_rate(rain, t)) : R(0);
    int neg = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        if (ga && soil[c] != 255) continue;
        const int i = int(c / nx), j = int(c % nx);
        const R rate = map ? map_rate<R>(rain, map, i, j, ny, nx) : ru;
        if (h[c] + rate * K.rain_scale < R(-1e-11)) neg = 1;
    }
    if (__syncthreads_or(neg) && threadIdx.x == 0) atomicOr(&sc->skip_clamp, 1);
}

}  // namespace hp2d
