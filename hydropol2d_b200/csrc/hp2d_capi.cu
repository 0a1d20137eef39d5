// C ABI of the B200 surface-flow step (include/hp2d.h).  One translation unit: the
// kernels are templates instantiated here for float and double.  Build with
//   nvcc -gencode arch=compute_100a,code=sm_100a -fmad=false -O3 -shared ...
// (-fmad=false keeps every product and sum separately rounded, which the parity tests
// against the CPU restatement rely on).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "hp2d.h"
#include "hp2d_device.cuh"
#include "hp2d_fused.cuh"
#include "hp2d_unfused.cuh"

using namespace hp2d;

namespace {

thread_local std::string g_create_error;

constexpr int kThreads = 256;

struct CudaFail {
    cudaError_t e;
    const char* what;
};

#define HP_CK(call)                                              \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) throw CudaFail{_e, #call};        \
    } while (0)

struct Base {
    virtual ~Base() = default;
};

template <typename R> struct Dev {
    R* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free();
        if (count == 0) return;
        HP_CK(cudaMalloc(&p, count * sizeof(R)));
        n = count;
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~Dev() { free(); }
};

template <typename R> constexpr int fused_by() { return 16; }
template <typename R> constexpr int fused_bx() { return sizeof(R) == 4 ? 64 : 32; }

}  // namespace

struct hp2d_ctx {
    hp2d_grid g{};
    hp2d_params p{};
    int device = 0;
    std::string err;
    cudaStream_t stream = nullptr;
    std::unique_ptr<Base> impl;
};

namespace {

template <typename R> struct Impl : Base {
    hp2d_ctx* ctx;
    int ny, nx;
    size_t n;
    double res;
    Dev<R> dzx, dzy, n2;
    Dev<uint8_t> soil;
    Dev<SoilClass<R>> classes;
    int n_classes = 0;
    Dev<uint32_t> outlet_bits;
    int bit_words = 0;
    Dev<int32_t> outlet_cells;
    Dev<R> outlet_coef, hf3, qo;
    int n_out = 0;
    Dev<R> h[2], qx[2], qy[2], I[2], T[2], dmax, arrival;
    Dev<R> hfx, hfy, qxu, qyu, scale;
    Dev<double> rain_t, rain_r;
    Dev<float> maps;
    RainDesc rain{};
    Dev<StepScalars> sc;
    StepScalars hs{};
    Dev<double> vol;
    bool static_ready = false, state_ready = false, dirty = true;
    double last_dt_s = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;

    explicit Impl(hp2d_ctx* c) : ctx(c) {
        ny = c->g.ny;
        nx = c->g.nx;
        n = size_t(ny) * nx;
        res = c->g.resolution;
        dzx.alloc(n); dzy.alloc(n); n2.alloc(n);
        for (int b = 0; b < 2; ++b) {
            h[b].alloc(n); qx[b].alloc(n); qy[b].alloc(n);
            HP_CK(cudaMemset(h[b].p, 0, n * sizeof(R)));
            HP_CK(cudaMemset(qx[b].p, 0, n * sizeof(R)));
            HP_CK(cudaMemset(qy[b].p, 0, n * sizeof(R)));
        }
        dmax.alloc(n); arrival.alloc(n);
        sc.alloc(1);
        vol.alloc(1);
        bit_words = (nx + 31) / 32;
        outlet_bits.alloc(size_t(ny) * bit_words);
        HP_CK(cudaMemset(outlet_bits.p, 0, size_t(ny) * bit_words * sizeof(uint32_t)));
        std::memset(&hs, 0, sizeof(hs));
        hs.t_min = c->p.min_time_step / 60.0;
        hs.time_step = c->p.min_time_step / 60.0;   // HydroPol2D_preprocessing.m:2469
        hs.k = 1;
        push_sc();
        reset_maxima();
    }
    ~Impl() override {
        if (graph) cudaGraphExecDestroy(graph);
    }

    cudaStream_t st() const { return ctx->stream; }
    void push_sc() { HP_CK(cudaMemcpyAsync(sc.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st())); HP_CK(cudaStreamSynchronize(st())); }
    void pull_sc() { HP_CK(cudaMemcpyAsync(&hs, sc.p, sizeof(hs), cudaMemcpyDeviceToHost, st())); HP_CK(cudaStreamSynchronize(st())); }

    void fill(R* p, size_t count, R v) {
        std::vector<R> tmp(count, v);
        HP_CK(cudaMemcpyAsync(p, tmp.data(), count * sizeof(R), cudaMemcpyHostToDevice, st()));
        HP_CK(cudaStreamSynchronize(st()));
    }
    void reset_maxima() {
        fill(dmax.p, n, -std::numeric_limits<R>::infinity());
        fill(arrival.p, n, std::numeric_limits<R>::infinity());
    }
    void upload(R* dst, const std::vector<R>& v) {
        HP_CK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(R), cudaMemcpyHostToDevice, st()));
        HP_CK(cudaStreamSynchronize(st()));
    }
    std::vector<R> fetch(const R* src, size_t count) {
        std::vector<R> v(count);
        if (count) {
            HP_CK(cudaMemcpyAsync(v.data(), src, count * sizeof(R), cudaMemcpyDeviceToHost, st()));
            HP_CK(cudaStreamSynchronize(st()));
        }
        return v;
    }
    GridView<R> view() const {
        GridView<R> gv;
        gv.ny = ny; gv.nx = nx; gv.res = res;
        gv.tol_mm = ctx->p.depth_tolerance;
        gv.thr_mm = ctx->p.arrival_threshold;
        return gv;
    }
    int blocks_for(size_t count) const {
        size_t b = (count + kThreads - 1) / kThreads;
        return int(std::max<size_t>(1, std::min<size_t>(b, 148 * 16)));
    }

    hp2d_status upload_static(const double* z, const double* rough, const int32_t* rows, const int32_t* cols,
                              int32_t nout, const double* slopes) {
        const double qnan = std::numeric_limits<double>::quiet_NaN();
        std::vector<R> a(n), b(n), c(n);
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                size_t k = size_t(i) * nx + j;
                a[k] = R((j + 1 < nx) ? z[k + 1] - z[k] : qnan);
                b[k] = R((i >= 1) ? z[k - nx] - z[k] : qnan);
                c[k] = R(rough[k] * rough[k]);
            }
        upload(dzx.p, a); upload(dzy.p, b); upload(n2.p, c);
        std::vector<std::pair<int32_t, R>> outs;
        for (int o = 0; o < nout; ++o) {
            if (rows[o] < 0 || rows[o] >= ny || cols[o] < 0 || cols[o] >= nx) {
                ctx->err = "outlet cell outside the grid";
                return HP2D_INVALID_ARG;
            }
            size_t k = size_t(rows[o]) * nx + cols[o];
            double coef = ctx->p.outlet_type == 1
                              ? std::sqrt(std::fabs(slopes ? slopes[o] : ctx->p.slope_outlet)) / (rough[k] * res)
                              : std::sqrt(kG) / res;
            outs.emplace_back(int32_t(k), R(coef));
        }
        std::sort(outs.begin(), outs.end(), [](auto& x, auto& y) { return x.first < y.first; });
        outs.erase(std::unique(outs.begin(), outs.end(), [](auto& x, auto& y) { return x.first == y.first; }), outs.end());
        n_out = int(outs.size());
        std::vector<int32_t> cells(n_out);
        std::vector<R> coefs(n_out);
        std::vector<uint32_t> bits(size_t(ny) * bit_words, 0u);
        for (int o = 0; o < n_out; ++o) {
            cells[o] = outs[o].first;
            coefs[o] = outs[o].second;
            int i = cells[o] / nx, j = cells[o] % nx;
            bits[size_t(i) * bit_words + (j >> 5)] |= 1u << (j & 31);
        }
        outlet_cells.alloc(std::max(n_out, 1));
        outlet_coef.alloc(std::max(n_out, 1));
        hf3.alloc(std::max(n_out, 1));
        qo.alloc(std::max(n_out, 1));
        if (n_out) {
            HP_CK(cudaMemcpy(outlet_cells.p, cells.data(), n_out * sizeof(int32_t), cudaMemcpyHostToDevice));
            upload(outlet_coef.p, coefs);
        }
        fill(hf3.p, std::max(n_out, 1), R(0));
        fill(qo.p, std::max(n_out, 1), R(0));
        HP_CK(cudaMemcpy(outlet_bits.p, bits.data(), bits.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        static_ready = true;
        invalidate_graph();
        return HP2D_OK;
    }

    hp2d_status set_soil(const uint8_t* cls, int32_t ncls, const double* ksat, const double* psi,
                         const double* dtheta, const double* Lu, const double* kout, const double* Tr,
                         const double* minsm) {
        if (ncls <= 0 || ncls > 255) { ctx->err = "n_classes must be in 1..255"; return HP2D_INVALID_ARG; }
        for (size_t k = 0; k < n; ++k)
            if (cls[k] != 255 && cls[k] >= ncls) { ctx->err = "soil class index out of range"; return HP2D_INVALID_ARG; }
        std::vector<SoilClass<R>> t(ncls);
        for (int c = 0; c < ncls; ++c) {
            t[c].ks = R(ksat[c] / 3.6e6);
            t[c].psi = R(psi[c] / 1000.0);
            t[c].dth = R(dtheta[c]);
            t[c].lu = R(Lu[c]);
            t[c].kout = R(kout[c] / 3.6e6);
            t[c].tr = R(Tr[c] * 3600.0);
            t[c].minsm = R(minsm[c] / 1000.0);
            t[c].pad = R(0);
        }
        soil.alloc(n);
        classes.alloc(ncls);
        HP_CK(cudaMemcpy(soil.p, cls, n, cudaMemcpyHostToDevice));
        HP_CK(cudaMemcpy(classes.p, t.data(), ncls * sizeof(SoilClass<R>), cudaMemcpyHostToDevice));
        n_classes = ncls;
        host_soil.assign(cls, cls + n);
        host_tr.resize(ncls);
        for (int c = 0; c < ncls; ++c) host_tr[c] = t[c].tr;
        for (int b = 0; b < 2; ++b) {
            if (!I[b].p) { I[b].alloc(n); fill(I[b].p, n, R(0)); }
            if (!T[b].p) { T[b].alloc(n); fill(T[b].p, n, R(0)); }
        }
        reset_timer();
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    // recovery timer starts at Tr (HydroPol2D_Main_While_Ensemble.m:266)
    void reset_timer() {
        if (!T[0].p || host_soil.empty()) return;
        std::vector<R> v(n);
        for (size_t k = 0; k < n; ++k) v[k] = host_soil[k] != 255 ? host_tr[host_soil[k]] : R(0);
        upload(T[hs.cur].p, v);
    }
    std::vector<uint8_t> host_soil;
    std::vector<R> host_tr;

    hp2d_status set_state(const double* d, const double* outflow, const double* Imm) {
        std::vector<R> a(n), b(n), c(n);
        for (size_t k = 0; k < n; ++k) {
            a[k] = R(d[k] / 1000.0);
            b[k] = outflow ? R(outflow[k] / 3.6e6 * res) : R(0);
            c[k] = outflow ? R(outflow[n + k] / 3.6e6 * res) : R(0);
        }
        int cur = hs.cur;
        upload(h[cur].p, a); upload(qx[cur].p, b); upload(qy[cur].p, c);
        if (Imm) {
            if (!I[0].p) for (int q = 0; q < 2; ++q) { I[q].alloc(n); T[q].alloc(n); fill(T[q].p, n, R(0)); }
            std::vector<R> v(n);
            for (size_t k = 0; k < n; ++k) v[k] = R(Imm[k] / 1000.0);
            upload(I[cur].p, v);
        }
        reset_timer();
        reset_maxima();
        state_ready = true;
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_clock(double t, double time_step, int64_t k) {
        pull_sc();
        hs.t_min = t;
        hs.time_step = time_step;
        hs.k = k;
        push_sc();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_rain_uniform(int32_t cnt, const double* t0, const double* rate) {
        rain_t.alloc(std::max(cnt, 1)); rain_r.alloc(std::max(cnt, 1));
        if (cnt) {
            HP_CK(cudaMemcpy(rain_t.p, t0, cnt * sizeof(double), cudaMemcpyHostToDevice));
            HP_CK(cudaMemcpy(rain_r.p, rate, cnt * sizeof(double), cudaMemcpyHostToDevice));
        }
        rain.n_uniform = cnt;
        rain.t_start = rain_t.p;
        rain.rate = rain_r.p;
        rain.n_maps = 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_rain_maps(int32_t nm, int32_t my, int32_t mx, const float* rate, double map_dt) {
        if (nm <= 0 || my <= 0 || mx <= 0 || !(map_dt > 0)) { ctx->err = "bad rain map shape"; return HP2D_INVALID_ARG; }
        size_t cnt = size_t(nm) * my * mx;
        maps.alloc(cnt);
        HP_CK(cudaMemcpy(maps.p, rate, cnt * sizeof(float), cudaMemcpyHostToDevice));
        rain.n_maps = nm; rain.my = my; rain.mx = mx; rain.map_dt = map_dt; rain.maps = maps.p;
        rain.n_uniform = 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    bool ga() const { return ctx->p.flag_infiltration == 1 && n_classes > 0; }

    void fold_accumulators() {
        pull_sc();
        double area = res * res;
        hs.rain_vol += hs.acc_rain * area;
        hs.inf_vol += hs.acc_inf * area;
        hs.out_vol += hs.acc_out * area;
        hs.acc_rain = hs.acc_inf = hs.acc_out = 0;
        hs.acc_vmax = hs.acc_cmax = 0;
        hs.acc_neg = 0;
        push_sc();
    }

    // ---------------- unfused entry points ----------------
    hp2d_status hydrology_step(double time_step) {
        pull_sc();
        hs.acc_neg = 0;
        push_sc();
        int cur = hs.cur;
        double dts = time_step * 60.0;
        k_hydro_rain_ga<R><<<blocks_for(n), kThreads, 0, st()>>>(view(), hs.t_min, dts, rain, h[cur].p,
                                                               I[cur].p, T[cur].p, soil.p, classes.p, ga() ? 1 : 0, sc.p);
        HP_CK(cudaGetLastError());
        k_hydro_clamp<R><<<blocks_for(n), kThreads, 0, st()>>>(n, h[cur].p, sc.p);
        HP_CK(cudaGetLastError());
        pull_sc();
        if (hs.acc_neg) hs.neg_warn += 1;
        push_sc();
        fold_accumulators();
        dirty = true;
        return HP2D_OK;
    }

    void ensure_scratch() {
        if (!hfx.p) { hfx.alloc(n); hfy.alloc(n); qxu.alloc(n); qyu.alloc(n); scale.alloc(n); }
    }

    hp2d_status li_step(double time_step) {
        ensure_scratch();
        pull_sc();
        int cur = hs.cur;
        double dts = time_step * 60.0;
        auto gv = view();
        int nb = blocks_for(n);
        k_faces<R><<<nb, kThreads, 0, st()>>>(gv, dts, h[cur].p, dzx.p, dzy.p, n2.p, qx[cur].p, qy[cur].p,
                                            hfx.p, hfy.p, qxu.p, qyu.p, ctx->p.flag_critical);
        HP_CK(cudaGetLastError());
        k_scale<R><<<nb, kThreads, 0, st()>>>(gv, dts, h[cur].p, qxu.p, qyu.p, scale.p);
        HP_CK(cudaGetLastError());
        k_limit<R><<<nb, kThreads, 0, st()>>>(gv, qxu.p, qyu.p, scale.p, qx[cur].p, qy[cur].p);
        HP_CK(cudaGetLastError());
        k_continuity<R><<<nb, kThreads, 0, st()>>>(gv, dts, h[cur].p, qx[cur].p, qy[cur].p);
        HP_CK(cudaGetLastError());
        if (n_out) {
            k_outlet<R><<<(n_out + kThreads - 1) / kThreads, kThreads, 0, st()>>>(
                gv, dts, h[cur].p, outlet_cells.p, outlet_coef.p, n_out, ctx->p.outlet_type, hf3.p, qo.p, sc.p);
            HP_CK(cudaGetLastError());
        }
        last_dt_s = dts;
        fold_accumulators();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status cfl_dt(double* ts_out, double* vmax_out) {
        if (!hfx.p) { ctx->err = "hp2d_cfl_dt needs a preceding hp2d_li_step"; return HP2D_NOT_READY; }
        pull_sc();
        hs.acc_vmax = hs.acc_cmax = 0;
        push_sc();
        int cur = hs.cur;
        k_cfl<R><<<blocks_for(n), kThreads, 0, st()>>>(view(), last_dt_s, qx[cur].p, qy[cur].p, hfx.p, hfy.p,
                                                     outlet_bits.p, bit_words, outlet_cells.p, hf3.p, n_out,
                                                     ctx->p.flag_adaptive_timestepping, sc.p);
        HP_CK(cudaGetLastError());
        pull_sc();
        const bool is_d = sizeof(R) == 8;
        double vm = from_ord(hs.acc_vmax, is_d), cm = from_ord(hs.acc_cmax, is_d);
        const hp2d_params& p = ctx->p;
        double dt_adv;
        if (vm > 0) {
            dt_adv = 1.0 * res / std::fmax(vm, 1e-10);
            double tsf = std::fmax(p.alfa_max - 2.0 * std::fmax(vm - 5.0, 0.0), p.alfa_min);
            dt_adv = std::fmin(dt_adv * tsf, p.max_time_step);
        } else {
            dt_adv = p.max_time_step;
        }
        double dt_wave = cm > 0 ? (p.alfa_min * res) / cm : p.max_time_step;
        double nw = p.flag_timestep == 1 ? std::fmin(dt_adv, dt_wave) : dt_wave;
        if (std::isnan(nw) || std::isinf(nw)) nw = p.max_time_step;
        double tcr = std::fmax(p.time_step_increments * std::floor(nw / p.time_step_increments), p.min_time_step);
        tcr = std::fmin(tcr, p.max_time_step);
        hs.acc_vmax = hs.acc_cmax = 0;
        hs.vmax_last = vm;
        if (tcr == p.min_time_step) hs.unstable += 1;
        push_sc();
        *ts_out = tcr / 60.0;
        if (vmax_out) *vmax_out = vm;
        return HP2D_OK;
    }

    hp2d_status track_maxima(double t_end) {
        int cur = hs.cur;
        R thr = R(ctx->p.arrival_threshold / 1000.0);
        k_track<R><<<blocks_for(n), kThreads, 0, st()>>>(n, h[cur].p, dmax.p, arrival.p, thr, R(t_end * 60.0));
        HP_CK(cudaGetLastError());
        HP_CK(cudaStreamSynchronize(st()));
        return HP2D_OK;
    }

    // ---------------- fused path ----------------
    FusedArgs<R> fused_args() {
        FusedArgs<R> a{};
        const hp2d_params& p = ctx->p;
        a.ny = ny; a.nx = nx; a.res = res;
        a.tol_mm = p.depth_tolerance; a.thr_mm = p.arrival_threshold;
        a.t_end = p.routing_time + p.min_time_step / 60.0;
        a.min_dt = p.min_time_step; a.max_dt = p.max_time_step; a.inc = p.time_step_increments;
        a.tsc = p.time_step_change; a.alfa_min = p.alfa_min; a.alfa_max = p.alfa_max;
        a.flag_timestep = p.flag_timestep; a.adaptive = p.flag_adaptive_timestepping;
        a.flag_critical = p.flag_critical; a.outlet_type = p.outlet_type; a.ga = ga() ? 1 : 0;
        constexpr int BY = fused_by<R>(), BX = fused_bx<R>();
        a.n_ctas = unsigned((nx + BX - 1) / BX) * unsigned((ny + BY - 1) / BY);
        a.dzx = dzx.p; a.dzy = dzy.p; a.n2 = n2.p;
        a.soil = soil.p; a.classes = classes.p;
        a.outlet_bits = outlet_bits.p; a.bit_words = bit_words;
        a.outlet_cells = outlet_cells.p; a.outlet_coef = outlet_coef.p; a.n_outlets = n_out;
        a.hf3 = hf3.p; a.qo = qo.p;
        a.h0 = h[0].p; a.h1 = h[1].p; a.qx0 = qx[0].p; a.qx1 = qx[1].p; a.qy0 = qy[0].p; a.qy1 = qy[1].p;
        a.I0 = I[0].p; a.I1 = I[1].p; a.T0 = T[0].p; a.T1 = T[1].p;
        a.dmax = dmax.p; a.arrival = arrival.p;
        a.rain = rain;
        a.sc = sc.p;
        return a;
    }

    void launch_fused(const FusedArgs<R>& a) {
        constexpr int BY = fused_by<R>(), BX = fused_bx<R>();
        using SM = FusedSmem<R, BY, BX>;
        dim3 grid((nx + BX - 1) / BX, (ny + BY - 1) / BY);
        k_fused_step<R, BY, BX, kThreads><<<grid, kThreads, SM::bytes, st()>>>(a);
    }

    void invalidate_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_steps = 0;
    }

    void prologue() {
        if (!dirty) return;
        pull_sc();
        hs.skip_clamp = 0;
        hs.counter = 0;
        hs.acc_vmax = hs.acc_cmax = 0;
        hs.acc_rain = hs.acc_inf = hs.acc_out = 0;
        push_sc();
        k_skip_flag<R><<<blocks_for(n), kThreads, 0, st()>>>(h[hs.cur].p, ny, nx, rain, soil.p, ga() ? 1 : 0, res,
                                                           ctx->p.depth_tolerance, ctx->p.arrival_threshold, sc.p);
        HP_CK(cudaGetLastError());
        dirty = false;
    }

    static constexpr int kGraphChunk = 32;

    hp2d_status fused_steps(int32_t nsteps, cudaEvent_t after = nullptr) {
        if (!static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        if (ctx->p.flag_infiltration == 1 && n_classes == 0) { ctx->err = "flag_infiltration=1 needs hp2d_set_soil"; return HP2D_NOT_READY; }
        prologue();
        FusedArgs<R> a = fused_args();
        int remaining = nsteps;
        if (remaining >= kGraphChunk) {
            if (!graph) {
                cudaGraph_t gr;
                HP_CK(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                for (int s = 0; s < kGraphChunk; ++s) launch_fused(a);
                HP_CK(cudaStreamEndCapture(st(), &gr));
                HP_CK(cudaGraphInstantiate(&graph, gr, 0));
                HP_CK(cudaGraphDestroy(gr));
                graph_steps = kGraphChunk;
            }
            while (remaining >= graph_steps) {
                HP_CK(cudaGraphLaunch(graph, st()));
                remaining -= graph_steps;
            }
        }
        for (int s = 0; s < remaining; ++s) launch_fused(a);
        HP_CK(cudaGetLastError());
        if (after) HP_CK(cudaEventRecord(after, st()));
        pull_sc();
        return HP2D_OK;
    }

    hp2d_status fused_steps_timed(int32_t nsteps, float* ms) {
        if (!static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        prologue();
        HP_CK(cudaStreamSynchronize(st()));
        cudaEvent_t e0, e1;
        HP_CK(cudaEventCreate(&e0));
        HP_CK(cudaEventCreate(&e1));
        HP_CK(cudaEventRecord(e0, st()));
        hp2d_status s = fused_steps(nsteps, e1);   // e1 recorded before the clock readback
        HP_CK(cudaEventSynchronize(e1));
        HP_CK(cudaEventElapsedTime(ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return s;
    }

    hp2d_status run(int64_t max_steps, int64_t* done) {
        const double t_end = ctx->p.routing_time + ctx->p.min_time_step / 60.0;
        int64_t k0 = hs.k;
        while (hs.t_min <= t_end) {
            int64_t left = max_steps > 0 ? max_steps - (hs.k - k0) : int64_t(1) << 40;
            if (left <= 0) break;
            int32_t chunk = int32_t(std::min<int64_t>(left, 1024));
            hp2d_status s = fused_steps(chunk);
            if (s != HP2D_OK) return s;
        }
        if (done) *done = hs.k - k0;
        return HP2D_OK;
    }

    // ---------------- outputs ----------------
    hp2d_status download(int32_t field, double* out, size_t count) {
        if (count != n) { ctx->err = "count must be ny*nx"; return HP2D_INVALID_ARG; }
        pull_sc();
        int cur = hs.cur;
        const double to_mmh = 3.6e6 / res;
        auto per_outlet_map = [&](const Dev<R>& src, double scale) {
            std::fill(out, out + n, 0.0);
            if (!n_out) return;
            std::vector<int32_t> cells(n_out);
            HP_CK(cudaMemcpy(cells.data(), outlet_cells.p, n_out * sizeof(int32_t), cudaMemcpyDeviceToHost));
            auto v = fetch(src.p, n_out);
            for (int o = 0; o < n_out; ++o) out[cells[o]] = double(v[o]) * scale;
        };
        switch (field) {
            case HP2D_FIELD_DEPTH: { auto v = fetch(h[cur].p, n); for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) * 1000.0; break; }
            case HP2D_FIELD_QOUT_RIGHT: { auto v = fetch(qx[cur].p, n); for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) * to_mmh; break; }
            case HP2D_FIELD_QOUT_UP: { auto v = fetch(qy[cur].p, n); for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) * to_mmh; break; }
            case HP2D_FIELD_QOUT_LEFT: {
                auto v = fetch(qx[cur].p, n);
                for (int i = 0; i < ny; ++i)
                    for (int j = 0; j < nx; ++j) out[size_t(i) * nx + j] = j == 0 ? -0.0 : -double(v[size_t(i) * nx + j - 1]) * to_mmh;
                break;
            }
            case HP2D_FIELD_QOUT_DOWN: {
                auto v = fetch(qy[cur].p, n);
                for (int i = 0; i < ny; ++i)
                    for (int j = 0; j < nx; ++j) out[size_t(i) * nx + j] = i + 1 == ny ? -0.0 : -double(v[size_t(i + 1) * nx + j]) * to_mmh;
                break;
            }
            case HP2D_FIELD_OUTLET_FLOW: per_outlet_map(qo, 3.6e6); break;
            case HP2D_FIELD_HF_X: case HP2D_FIELD_HF_Y: {
                if (!hfx.p) { ctx->err = "Hf is materialised by hp2d_li_step only"; return HP2D_NOT_READY; }
                auto v = fetch(field == HP2D_FIELD_HF_X ? hfx.p : hfy.p, n);
                for (size_t k = 0; k < n; ++k) out[k] = double(v[k]);
                break;
            }
            case HP2D_FIELD_HF_OUTLET: per_outlet_map(hf3, 1.0); break;
            case HP2D_FIELD_DMAX: { auto v = fetch(dmax.p, n); for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) * 1000.0; break; }
            case HP2D_FIELD_ARRIVAL: { auto v = fetch(arrival.p, n); for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) / 60.0; break; }
            case HP2D_FIELD_SOIL_STORAGE: {
                if (!I[cur].p) { ctx->err = "no soil storage (hp2d_set_soil not called)"; return HP2D_NOT_READY; }
                auto v = fetch(I[cur].p, n);
                for (size_t k = 0; k < n; ++k) out[k] = double(v[k]) * 1000.0;
                break;
            }
            case HP2D_FIELD_I_TOT_END_CELL: {
                auto a = fetch(qx[cur].p, n), b = fetch(qy[cur].p, n);
                std::vector<double> of(n, 0.0);
                if (n_out) {
                    std::vector<int32_t> cells(n_out);
                    HP_CK(cudaMemcpy(cells.data(), outlet_cells.p, n_out * sizeof(int32_t), cudaMemcpyDeviceToHost));
                    auto v = fetch(qo.p, n_out);
                    for (int o = 0; o < n_out; ++o) of[cells[o]] = double(v[o]) * 3.6e6;
                }
                double dts = last_dt_s > 0 ? last_dt_s : hs.time_step * 60.0;
                for (size_t k = 0; k < n; ++k)
                    out[k] = std::fabs(double(a[k]) * to_mmh + double(b[k]) * to_mmh + of[k]) * dts / 1000.0 / 3600.0 * res * res;
                break;
            }
            default: ctx->err = "unknown field"; return HP2D_INVALID_ARG;
        }
        return HP2D_OK;
    }

    hp2d_status download_native(int32_t field, void* out, size_t bytes) {
        pull_sc();
        int cur = hs.cur;
        const R* src = nullptr;
        size_t cnt = n;
        switch (field) {
            case 0: src = h[cur].p; break;
            case 1: src = qx[cur].p; break;
            case 2: src = qy[cur].p; break;
            case 3: src = I[cur].p; break;
            case 4: src = T[cur].p; break;
            case 5: src = dmax.p; break;
            case 6: src = arrival.p; break;
            case 7: src = hfx.p; break;
            case 8: src = hfy.p; break;
            case 9: src = hf3.p; cnt = size_t(n_out); break;
            case 10: src = qo.p; cnt = size_t(n_out); break;
            default: ctx->err = "unknown native field"; return HP2D_INVALID_ARG;
        }
        if (!src) { ctx->err = "field not materialised"; return HP2D_NOT_READY; }
        if (bytes != cnt * sizeof(R)) { ctx->err = "byte count mismatch"; return HP2D_INVALID_ARG; }
        if (cnt) {
            HP_CK(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, st()));
            HP_CK(cudaStreamSynchronize(st()));
        }
        return HP2D_OK;
    }

    hp2d_status diag(hp2d_diag* o) {
        pull_sc();
        o->t = hs.t_min;
        o->time_step = hs.time_step;
        o->k = hs.k;
        o->max_velocity = hs.vmax_last;
        o->rain_volume = hs.rain_vol;
        o->infiltration_volume = hs.inf_vol;
        o->outlet_volume = hs.out_vol;
        o->neg_depth_warnings = hs.neg_warn;
        o->unstable_steps = hs.unstable;
        o->status_bits = hs.status;
        return HP2D_OK;
    }

    hp2d_status stored_volume(double* v) {
        pull_sc();
        HP_CK(cudaMemsetAsync(vol.p, 0, sizeof(double), st()));
        k_volume<R><<<blocks_for(n), kThreads, 0, st()>>>(n, h[hs.cur].p, vol.p);
        HP_CK(cudaGetLastError());
        double s = 0;
        HP_CK(cudaMemcpyAsync(&s, vol.p, sizeof(double), cudaMemcpyDeviceToHost, st()));
        HP_CK(cudaStreamSynchronize(st()));
        *v = s * res * res;
        return HP2D_OK;
    }
};

template <typename F> hp2d_status guarded(hp2d_ctx* ctx, F&& fn) {
    if (!ctx || !ctx->impl) return HP2D_INVALID_ARG;
    try {
        HP_CK(cudaSetDevice(ctx->device));
        return fn();
    } catch (const CudaFail& f) {
        ctx->err = std::string(f.what) + ": " + cudaGetErrorString(f.e);
        return HP2D_CUDA_ERROR;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return HP2D_INVALID_ARG;
    }
}

template <typename F> hp2d_status with_impl(hp2d_ctx* ctx, F&& fn) {
    return guarded(ctx, [&]() -> hp2d_status {
        if (ctx->g.precision == HP2D_FP32) return fn(*static_cast<Impl<float>*>(ctx->impl.get()));
        return fn(*static_cast<Impl<double>*>(ctx->impl.get()));
    });
}

template <typename R> void set_smem_attr() {
    constexpr int BY = fused_by<R>(), BX = fused_bx<R>();
    using SM = FusedSmem<R, BY, BX>;
    HP_CK(cudaFuncSetAttribute(k_fused_step<R, BY, BX, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(SM::bytes)));
}

}  // namespace

extern "C" {

const char* hp2d_create_error(void) { return g_create_error.c_str(); }

hp2d_status hp2d_create(const hp2d_grid* grid, const hp2d_params* params, int32_t device, hp2d_ctx** out) {
    g_create_error.clear();
    if (!grid || !params || !out) { g_create_error = "null argument"; return HP2D_INVALID_ARG; }
    *out = nullptr;
    const hp2d_params& p = *params;
    if (grid->ny <= 0 || grid->nx <= 0 || !(grid->resolution > 0)) { g_create_error = "grid must have ny, nx > 0 and resolution > 0"; return HP2D_INVALID_ARG; }
    if (grid->precision != HP2D_FP32 && grid->precision != HP2D_FP64) { g_create_error = "precision must be HP2D_FP32 or HP2D_FP64"; return HP2D_INVALID_ARG; }
    if (p.flag_subgrid != 0) { g_create_error = "flag_subgrid=1 is not supported"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_D8 != 0) { g_create_error = "flag_D8=1 is not supported"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_reservoir != 0) { g_create_error = "flag_reservoir=1 is not supported"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_numerical_scheme != 1) { g_create_error = "only flag_numerical_scheme=1 (Bates) is supported"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_infiltration != 0 && p.flag_infiltration != 1) { g_create_error = "flag_infiltration must be 0 or 1"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_critical != 0 && p.flag_critical != 1) { g_create_error = "flag_critical must be 0 or 1"; return HP2D_INVALID_ARG; }
    if (p.outlet_type != 1 && p.outlet_type != 2) { g_create_error = "outlet_type must be 1 or 2"; return HP2D_INVALID_ARG; }
    if (!(p.min_time_step > 0) || !(p.max_time_step >= p.min_time_step) || !(p.time_step_increments > 0) ||
        !(p.time_step_change > 0)) {
        g_create_error = "time-step controls must be positive with max >= min";
        return HP2D_INVALID_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_create_error = "no CUDA device";
        return HP2D_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) { g_create_error = "device index out of range"; return HP2D_INVALID_ARG; }
    auto* ctx = new hp2d_ctx();
    ctx->g = *grid;
    ctx->p = p;
    ctx->device = device;
    try {
        HP_CK(cudaSetDevice(device));
        HP_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        if (grid->precision == HP2D_FP32) {
            set_smem_attr<float>();
            ctx->impl.reset(new Impl<float>(ctx));
        } else {
            set_smem_attr<double>();
            ctx->impl.reset(new Impl<double>(ctx));
        }
    } catch (const CudaFail& f) {
        g_create_error = std::string(f.what) + ": " + cudaGetErrorString(f.e);
        ctx->impl.reset();
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return HP2D_CUDA_ERROR;
    }
    *out = ctx;
    return HP2D_OK;
}

hp2d_status hp2d_destroy(hp2d_ctx* ctx) {
    if (!ctx) return HP2D_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->impl.reset();
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return HP2D_OK;
}

const char* hp2d_last_error(const hp2d_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

hp2d_status hp2d_upload_static(hp2d_ctx* ctx, const double* z, const double* roughness, const int32_t* rows,
                               const int32_t* cols, int32_t n_outlets, const double* slopes) {
    if (!z || !roughness || n_outlets < 0 || (n_outlets > 0 && (!rows || !cols))) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.upload_static(z, roughness, rows, cols, n_outlets, slopes); });
}

hp2d_status hp2d_set_soil(hp2d_ctx* ctx, const uint8_t* soil_class, int32_t n_classes, const double* ksat,
                          const double* psi, const double* dtheta, const double* Lu, const double* k_out,
                          const double* Tr, const double* min_soil_moisture) {
    if (!soil_class || !ksat || !psi || !dtheta || !Lu || !k_out || !Tr || !min_soil_moisture) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        return m.set_soil(soil_class, n_classes, ksat, psi, dtheta, Lu, k_out, Tr, min_soil_moisture);
    });
}

hp2d_status hp2d_set_state(hp2d_ctx* ctx, const double* d, const double* outflow, const double* soil_storage) {
    if (!d) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_state(d, outflow, soil_storage); });
}

hp2d_status hp2d_set_clock(hp2d_ctx* ctx, double t, double time_step, int64_t k) {
    if (!(time_step > 0) || k < 1) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_clock(t, time_step, k); });
}

hp2d_status hp2d_set_rain_uniform(hp2d_ctx* ctx, int32_t n, const double* t_start, const double* rate) {
    if (n < 0 || (n > 0 && (!t_start || !rate))) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_rain_uniform(n, t_start, rate); });
}

hp2d_status hp2d_set_rain_maps(hp2d_ctx* ctx, int32_t n_maps, int32_t my, int32_t mx, const float* rate, double map_dt) {
    if (!rate) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_rain_maps(n_maps, my, mx, rate, map_dt); });
}

hp2d_status hp2d_hydrology_step(hp2d_ctx* ctx, double time_step) {
    if (!(time_step > 0)) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.hydrology_step(time_step); });
}

hp2d_status hp2d_li_step(hp2d_ctx* ctx, double time_step) {
    if (!(time_step > 0)) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        if (!m.static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        return m.li_step(time_step);
    });
}

hp2d_status hp2d_cfl_dt(hp2d_ctx* ctx, double* time_step, double* max_velocity) {
    if (!time_step) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.cfl_dt(time_step, max_velocity); });
}

hp2d_status hp2d_track_maxima(hp2d_ctx* ctx, double t_end) {
    return with_impl(ctx, [&](auto& m) { return m.track_maxima(t_end); });
}

hp2d_status hp2d_fused_steps(hp2d_ctx* ctx, int32_t nsteps) {
    if (nsteps < 0) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.fused_steps(nsteps); });
}

hp2d_status hp2d_fused_steps_timed(hp2d_ctx* ctx, int32_t nsteps, float* elapsed_ms) {
    if (nsteps < 0 || !elapsed_ms) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.fused_steps_timed(nsteps, elapsed_ms); });
}

hp2d_status hp2d_run(hp2d_ctx* ctx, int64_t max_steps, int64_t* steps_done) {
    return with_impl(ctx, [&](auto& m) { return m.run(max_steps, steps_done); });
}

hp2d_status hp2d_download(hp2d_ctx* ctx, int32_t field, double* host, size_t count) {
    if (!host) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.download(field, host, count); });
}

hp2d_status hp2d_download_native(hp2d_ctx* ctx, int32_t field, void* host, size_t bytes) {
    if (!host && bytes) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.download_native(field, host, bytes); });
}

hp2d_status hp2d_get_diag(hp2d_ctx* ctx, hp2d_diag* out) {
    if (!out) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.diag(out); });
}

hp2d_status hp2d_stored_volume(hp2d_ctx* ctx, double* volume) {
    if (!volume) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.stored_volume(volume); });
}

}  // extern "C"
