// Unfused kernels: one reference function per C-ABI call (hp2d_hydrology_step,
// hp2d_li_step, hp2d_cfl_dt, hp2d_track_maxima).  They exist so that a MATLAB caller that
// keeps calling Local_Inertial_Model_D4 / Infiltration_Module / refreshing_timestep
// separately gets the same numbers as the fused step; they share every formula with it
// (hp2d_device.cuh) and run one grid-wide pass per stage, in place on the current
// buffers.
#pragma once

#include "hp2d_device.cuh"

namespace hp2d {

template <typename R> struct GridView {
    int ny, nx;
    double res, tol_mm, thr_mm;
};

// rain + Green-Ampt (Hydrological_Model.m:14-42); records whether any depth < -1e-8 mm
template <typename R>
__global__ void k_hydro_rain_ga(GridView<R> g, double rain_a, double rain_b, double dt_s, RainDesc rain, R* h, R* I, R* T,
                                const uint8_t* soil, const SoilClass<R>* classes, const SoilClassVG<R>* classes_vg,
                                VGGlobals<R> vg, int inf, InflowDesc<R> inflow, const typename Vec<R>::V4* stat,
                                StepScalars* sc) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    RainStep<R> RS;
    RS.make(rain, rain_a, rain_b);
    const size_t n = size_t(g.ny) * g.nx;
    double racc = 0, iacc = 0;
    int neg = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        const R r = RS.at(rain, i, j, g.ny, g.nx);
        R hh = h[c] + r;
        if (isfinite(hh)) racc += double(r);
        if (inf && soil[c] != 255) {
            R Ic = I[c], Tc = T[c];   // T: recovery timer (Green-Ampt) or water-table depth (van Genuchten)
            const R fd = inf == 1 ? green_ampt(hh, Ic, Tc, classes[soil[c]], K)
                                  : vg_infiltration(hh, Ic, Tc, classes_vg[soil[c]], vg, K);
            I[c] = Ic;
            T[c] = Tc;
            if (isfinite(fd)) iacc += double(fd);
        }
        if (inflow.n_gauges) add_inflow(inflow, meta_bits(stat[c].w), hh);   // Hydrological_Model.m:27-28
        if (hh < R(-1e-11)) neg = 1;
        h[c] = hh;
    }
    for (int o = 16; o > 0; o >>= 1) {
        racc += __shfl_xor_sync(0xffffffffu, racc, o);
        iacc += __shfl_xor_sync(0xffffffffu, iacc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (racc != 0.0) atomicAdd(&sc->acc_rain, racc);
        if (iacc != 0.0) atomicAdd(&sc->acc_inf, iacc);
    }
    if (__syncthreads_or(neg) && threadIdx.x == 0) atomicOr(&sc->acc_neg, 1);
}

// depth clamp (Hydrological_Model.m:45-52)
template <typename R>
__global__ void k_hydro_clamp(size_t n, R* h, const StepScalars* sc) {
    const bool skip = sc->acc_neg != 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        R hh = h[c];
        if (!skip && hh < R(1e-9)) hh = R(0);
        if (hh < R(0)) hh = R(0);
        h[c] = hh;
    }
}

// unlimited faces (LIM_D4.m:31-294); face (i,j): x = right face of cell (i,j), y = upper face.
// scheme = flag_numerical_scheme (Inertial_Solver.m): 1 Bates, 2 s-upwind, 3 s-centred; the
// neighbouring previous fluxes of schemes 2/3 exist on interior columns (x) / rows (y) only.
template <typename R>
__global__ void k_faces(GridView<R> g, double dt_s, const R* h, const R* dzx, const R* dzy, const R* n2,
                        const R* qx, const R* qy, R* hfx, R* hfy, R* qxu, R* qyu, int flag_critical, int scheme) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    const size_t n = size_t(g.ny) * g.nx;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        R Hf, q;
        const R hR = (j + 1 < g.nx) ? h[c + 1] : R(0);
        if (scheme == 1) {
            face_flux<R, true>(h[c], hR, dzx[c], qx[c], n2[c], K, flag_critical, Hf, q);
        } else {
            const bool in = j >= 1 && j + 1 < g.nx;
            face_flux<R, true, 1>(h[c], hR, dzx[c], qx[c], n2[c], K, flag_critical, Hf, q, scheme,
                                  in ? qx[c - 1] : R(0), in ? qx[c + 1] : R(0));
        }
        hfx[c] = Hf;
        qxu[c] = q;
        const R hU = (i >= 1) ? h[c - g.nx] : R(0);
        if (scheme == 1) {
            face_flux<R, false>(hU, h[c], dzy[c], qy[c], n2[c], K, flag_critical, Hf, q);
        } else {
            const bool in = i >= 1 && i + 1 < g.ny;
            face_flux<R, false, 1>(hU, h[c], dzy[c], qy[c], n2[c], K, flag_critical, Hf, q, scheme,
                                   in ? qy[c - g.nx] : R(0), in ? qy[c + g.nx] : R(0));
        }
        hfy[c] = Hf;
        qyu[c] = q;
    }
}

// donor scales (LIM_D4.m:814-829)
template <typename R>
__global__ void k_scale(GridView<R> g, double dt_s, const R* h, const R* qxu, const R* qyu, R* scale) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    const size_t n = size_t(g.ny) * g.nx;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        const R qL = j >= 1 ? qxu[c - 1] : R(0);
        const R qD = i + 1 < g.ny ? qyu[c + g.nx] : R(0);
        scale[c] = donor_scale(qxu[c], qL, qyu[c], qD, h[c], K);
    }
}

// limited faces into the state flux buffers (LIM_D4.m:831-857)
template <typename R>
__global__ void k_limit(GridView<R> g, const R* qxu, const R* qyu, const R* scale, R* qx, R* qy) {
    const size_t n = size_t(g.ny) * g.nx;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        const R sR = j + 1 < g.nx ? scale[c + 1] : R(1);
        const R sU = i >= 1 ? scale[c - g.nx] : R(1);
        qx[c] = limit_face(qxu[c], scale[c], sR);
        qy[c] = limit_face(qyu[c], scale[c], sU);
    }
}

// continuity (LIM_D4.m:313-315, :389-393, :415), in place on h
template <typename R>
__global__ void k_continuity(GridView<R> g, double dt_s, R* h, const R* qx, const R* qy) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    const size_t n = size_t(g.ny) * g.nx;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        const R qL = j >= 1 ? qx[c - 1] : R(0);
        const R qD = i + 1 < g.ny ? qy[c + g.nx] : R(0);
        h[c] = continuity(h[c], qL, qx[c], qy[c], qD, K);
    }
}

// control-structure transfers of an unfused step (Local_Inertial_Model_D4.m:318-344), one
// thread: from the d_tot the fluxes used, the extras join h before the continuity kernel
template <typename R>
__global__ void k_struct_unfused(StructDesc<R> s, R* h, double time_step, double area, StepScalars* sc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < s.n; ++i) s.hres[i] = h[s.slot_cell[s.slot[3 * i]]];
    sc->struct_vol += structure_transfers(s, time_step, area);
    for (int q = 0; q < s.n_slots; ++q) h[s.slot_cell[q]] = h[s.slot_cell[q]] + s.extra[q];
}

// outlet sink (LIM_D4.m:417-498), one thread per outlet cell
template <typename R>
__global__ void k_outlet(GridView<R> g, double dt_s, R* h, const int32_t* cells, const R* coef, int n_out,
                         int outlet_type, R* hf3, R* qo, StepScalars* sc) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    double acc = 0;
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n_out; o += gridDim.x * blockDim.x) {
        const int c = cells[o];
        R hn = h[c], ho;
        const R qq = outlet_sink(hn, coef[o], outlet_type, K, ho);
        h[c] = hn;
        hf3[o] = ho;
        qo[o] = qq;
        acc += double(qq * K.dt);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(&sc->acc_out, acc);
}

// CFL reductions (refreshing_timestep.m:61-238); accumulates into sc->acc_vmax/acc_cmax
template <typename R>
__global__ void k_cfl(GridView<R> g, double dt_s, const R* qx, const R* qy, const R* hfx, const R* hfy,
                      const uint32_t* outlet_bits, int bit_words, const int32_t* cells, const R* hf3,
                      int n_out, int adaptive, StepScalars* sc) {
    StepConsts<R> K;
    K.make(dt_s, g.res, g.tol_mm, g.thr_mm);
    const size_t n = size_t(g.ny) * g.nx;
    R vmax = R(0), cmax = R(0);
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const int i = int(c / g.nx), j = int(c % g.nx);
        R h3 = R(0);
        if (n_out && ((outlet_bits[size_t(i) * bit_words + (j >> 5)] >> (j & 31)) & 1u)) {
            const int o = find_outlet(cells, n_out, int(c));
            if (o >= 0) h3 = hf3[o];
        }
        const bool last = i + 1 >= g.ny;
        const R qyb = last ? R(0) : qy[c + g.nx];
        const R hfb = last ? R(0) : hfy[c + g.nx];
        R sp, ce;
        cfl_cell(qx[c], qy[c], qyb, hfx[c], hfy[c], hfb, h3, j == 0, adaptive, K, sp, ce);
        vmax = fmax(vmax, sp);
        cmax = fmax(cmax, ce);
    }
    for (int o = 16; o > 0; o >>= 1) {
        vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (vmax > R(0)) atomicMax(&sc->acc_vmax, ord_bits(vmax));
        if (cmax > R(0)) atomicMax(&sc->acc_cmax, ord_bits(cmax));
    }
}

// running maximum depth and arrival time (save_output_maps.m:588-600)
template <typename R>
__global__ void k_track(size_t n, const R* h, R* dmax, R* arrival, R thr, R t_end) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const R hn = h[c], dm = dmax[c];
        if (dm < thr && hn >= thr) arrival[c] = t_end;
        if (hn > dm) dmax[c] = hn;
    }
}

// stored volume sum(h) in FP64 (NaN walls skipped)
template <typename R>
__global__ void k_volume(size_t n, const R* h, double* out) {
    double acc = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const R v = h[c];
        if (isfinite(v)) acc += double(v);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(out, acc);
}

}  // namespace hp2d
