// C ABI of the B200 surface-flow step (include/hp2d.h).  One translation unit: the
// kernels are templates instantiated here for float and double.  Build with
//   nvcc -gencode arch=compute_100a,code=sm_100a -fmad=false -O3 -shared ...
// (-fmad=false keeps every product and sum separately rounded, which the parity tests
// against the CPU restatement rely on).
//
// Device layout of one context (n = ny*nx cells, R = float or double):
//   stat      n x {dz_x, dz_y, n^2, meta}            static record (16 or 32 B)
//   st4[2]    n x {h, q_x, q_y, dmax}                state record, double-buffered
//   gs2[2]    n x {I, T}                             Green-Ampt record, double-buffered
//   arrival   n x R
//   per outlet: coefficient, Hf(:,:,3) and sink rate
// plus, for the unfused entry points only, structure-of-arrays copies (dz_x, dz_y, n^2,
// soil class, outlet bitmask) and scratch (h, q, dmax, I, T, Hf, unlimited q, scale).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "hp2d.h"
#include "hp2d_device.cuh"
#include "hp2d_fused.cuh"
#include "hp2d_unfused.cuh"
#include "hp2d_tb.cuh"

using namespace hp2d;

namespace {

thread_local std::string g_create_error;

constexpr int kThreads = 128;

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

template <typename T> struct Dev {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free();
        if (count == 0) return;
        HP_CK(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~Dev() { free(); }
};



// Copies between a caller's host array and device memory.  Page-locked (or registered) caller
// memory moves in one cudaMemcpyAsync at the link rate.  Pageable arrays of at least kMin bytes
// are staged through this context's page-locked chunks by kLanes host threads, each with its
// own stream and two chunks, so that one chunk's host memcpy overlaps the other's DMA; smaller
// pageable arrays go in one copy, which the driver stages itself.  The chunks are allocated on
// the first staged copy and kept with the context.
struct HostStage {
    static constexpr size_t kChunk = size_t(8) << 20;
    static constexpr size_t kMin = size_t(32) << 20;
    static constexpr int kLanes = 4;
    struct Lane {
        void* pin[2] = {nullptr, nullptr};
        cudaStream_t s = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        cudaError_t err = cudaSuccess;
    };
    Lane lanes[kLanes];
    bool ready = false;

    ~HostStage() {
        for (Lane& l : lanes) {
            if (l.s) cudaStreamSynchronize(l.s);
            for (int b = 0; b < 2; ++b) {
                if (l.pin[b]) cudaFreeHost(l.pin[b]);
                if (l.ev[b]) cudaEventDestroy(l.ev[b]);
            }
            if (l.s) cudaStreamDestroy(l.s);
        }
    }
    static bool page_locked(const void* p) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    }
    void setup() {
        if (ready) return;
        for (Lane& l : lanes) {
            HP_CK(cudaStreamCreateWithFlags(&l.s, cudaStreamNonBlocking));
            for (int b = 0; b < 2; ++b) {
                HP_CK(cudaMallocHost(&l.pin[b], kChunk));
                HP_CK(cudaEventCreateWithFlags(&l.ev[b], cudaEventDisableTiming));
            }
        }
        ready = true;
    }
    // host -> device (to_device) or device -> host; returns after the data has landed.  Work
    // queued on `main` before the call completes first.
    void copy(void* dev, void* host, size_t bytes, bool to_device, cudaStream_t main, int device) {
        if (bytes == 0) return;
        const cudaMemcpyKind kind = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
        if (bytes < kMin || page_locked(host)) {
            HP_CK(to_device ? cudaMemcpyAsync(dev, host, bytes, kind, main) : cudaMemcpyAsync(host, dev, bytes, kind, main));
            HP_CK(cudaStreamSynchronize(main));
            return;
        }
        setup();
        HP_CK(cudaStreamSynchronize(main));
        const size_t nchunks = (bytes + kChunk - 1) / kChunk;
        auto lane_work = [&](int t) {
            Lane& l = lanes[t];
            l.err = cudaSetDevice(device);
            int use = 0, pb = -1;
            size_t poff = 0, plen = 0;
            for (size_t c = size_t(t); c < nchunks && l.err == cudaSuccess; c += kLanes) {
                const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
                const int b = use++ & 1;
                char* d = static_cast<char*>(dev) + off;
                char* h = static_cast<char*>(host) + off;
                if (to_device) {   // the chunk's last DMA must be done before it is refilled
                    if ((l.err = cudaEventSynchronize(l.ev[b])) != cudaSuccess) break;
                    std::memcpy(l.pin[b], h, len);
                    if ((l.err = cudaMemcpyAsync(d, l.pin[b], len, kind, l.s)) != cudaSuccess) break;
                    if ((l.err = cudaEventRecord(l.ev[b], l.s)) != cudaSuccess) break;
                } else {           // this chunk's DMA runs while the previous one is copied out
                    if ((l.err = cudaMemcpyAsync(l.pin[b], d, len, kind, l.s)) != cudaSuccess) break;
                    if ((l.err = cudaEventRecord(l.ev[b], l.s)) != cudaSuccess) break;
                    if (pb >= 0) {
                        if ((l.err = cudaEventSynchronize(l.ev[pb])) != cudaSuccess) break;
                        std::memcpy(static_cast<char*>(host) + poff, l.pin[pb], plen);
                    }
                    pb = b;
                    poff = off;
                    plen = len;
                }
            }
            if (!to_device && pb >= 0 && l.err == cudaSuccess) {
                l.err = cudaEventSynchronize(l.ev[pb]);
                if (l.err == cudaSuccess) std::memcpy(static_cast<char*>(host) + poff, l.pin[pb], plen);
            }
            const cudaError_t e = cudaStreamSynchronize(l.s);
            if (l.err == cudaSuccess) l.err = e;
        };
        std::vector<std::thread> pool;
        const int used = int(std::min<size_t>(kLanes, nchunks));
        for (int t = 1; t < used; ++t) pool.emplace_back(lane_work, t);
        lane_work(0);
        for (auto& th : pool) th.join();
        for (int t = 0; t < used; ++t) HP_CK(lanes[t].err);
    }
};

// f(begin, end) over [0, n) on up to 16 host threads (one for small n): the per-cell host loops of
// the set-up calls, whose first touch of fresh pages dominates on large grids
template <typename F> void host_parallel(size_t n, F f) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < (size_t(1) << 20) || hw == 1) {
        f(size_t(0), n);
        return;
    }
    const size_t chunk = (n + hw - 1) / hw;
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < hw; ++t) {
        const size_t a = t * chunk, b = std::min(n, a + chunk);
        if (a < b) pool.emplace_back(f, a, b);
    }
    f(size_t(0), std::min(n, chunk));
    for (auto& th : pool) th.join();
}
// allocator whose value-initialisation is a no-op, so that a large vector is filled once, in parallel
template <typename T> struct NoInitAlloc : std::allocator<T> {
    template <typename U> struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <typename U> NoInitAlloc(const NoInitAlloc<U>&) {}
    template <typename U> void construct(U* p) { ::new (static_cast<void*>(p)) U; }
    template <typename U, typename... A> void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};

// meta words of a grid without soil classes (255 everywhere, filled first): the outlet ordinal + 1
// in bits 8..30 of the outlet cells (cells sorted, one entry per cell)
__global__ void k_outlet_meta_scatter(const int32_t* __restrict__ cells, int n_out, uint32_t* __restrict__ meta) {
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n_out; o += gridDim.x * blockDim.x)
        meta[cells[o]] = 255u | (uint32_t(o + 1) << 8);
}

// smallest x >= 0 whose correctly rounded square root reaches R(0.01): the stagnant
// test sqrt(s2) < 0.01 of refreshing_timestep.m:184 is then s2 < x exactly
template <typename R> R stagnant_threshold() {
    const R target = R(0.01);
    R x = target * target;
    while (x > R(0) && std::sqrt(std::nextafter(x, R(0))) >= target) x = std::nextafter(x, R(0));
    while (std::sqrt(x) < target) x = std::nextafter(x, R(1));
    return x;
}

template <typename R>
__global__ void k_write_meta(size_t n, typename Vec<R>::V4* stat, const uint32_t* meta) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x)
        stat[c].w = make_meta<R>(meta[c]);
}

template <typename R>
__global__ void k_volume4(size_t n, const typename Vec<R>::V4* st, double* out) {
    double acc = 0;
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < n; c += size_t(gridDim.x) * blockDim.x) {
        const R v = st[c].x;
        if (isfinite(v)) acc += double(v);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(out, acc);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
typedef CUresult (*TensorMapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                      const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TensorMapEncodeFn tensor_map_encoder() {
    static TensorMapEncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TensorMapEncodeFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}
// an array of ny x nx float4 records as a [ny][nx][4] float tensor, boxes of ex x ey records
// (coordinates outside the array read as zeros)
bool record_map(CUtensorMap* m, const void* base, int ny, int nx, int ex, int ey) {
    TensorMapEncodeFn fn = tensor_map_encoder();
    if (!fn) return false;
    cuuint64_t dims[3] = {4, cuuint64_t(nx), cuuint64_t(ny)};
    cuuint64_t strides[2] = {16, cuuint64_t(nx) * 16};
    cuuint32_t box[3] = {4, cuuint32_t(ex), cuuint32_t(ey)};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

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
    using V4 = typename Vec<R>::V4;
    using V2 = typename Vec<R>::V2;
    hp2d_ctx* ctx;
    int ny, nx;
    size_t n;
    double res;
    // fused-path records
    Dev<V4> stat, st4[2];
    Dev<V2> gs2[2];
    void alloc_soil_records() {
        for (int b = 0; b < 2; ++b) if (!gs2[b].p) gs2[b].alloc(n);
    }
    Dev<R> arrival;
    Dev<SoilClass<R>> classes;
    int n_classes = 0;
    Dev<int32_t> outlet_cells;
    Dev<R> outlet_coef, hf3, qo;
    int n_out = 0;
    // unfused path: structure-of-arrays copies and scratch
    Dev<R> dzx, dzy, n2;
    Dev<uint8_t> soil;
    Dev<uint32_t> outlet_bits;
    int bit_words = 0;
    Dev<R> h, qx, qy, dmax, I, T;
    Dev<R> hfx, hfy, qxu, qyu, scale;
    // forcing, clock
    Dev<double> rain_t, rain_r;
    // inflow hydrographs
    Dev<double> inf_t, inf_r, inf_cells;
    Dev<R> inf_depth;
    Dev<int32_t> inf_off, inf_gauge;
    InflowDesc<R> inflow{};
    std::vector<double> host_gcells;
    // map records
    Dev<double> rec_times, rec_t;
    Dev<R> rec_snap;
    // records kept in page-locked host memory mapped into the device's address space
    // (hp2d_set_record_target(ctx, 1)): the step that takes a record writes it across the host
    // link itself, overlapped with its other work, and reading it back is a host-side read
    R* rec_host = nullptr;
    size_t rec_host_n = 0;
    int rec_target = 0;
    void free_rec_host() {
        if (rec_host) cudaFreeHost(rec_host);
        rec_host = nullptr;
        rec_host_n = 0;
    }
    RecordDesc<R> rec{};
    Dev<float> maps;
    RainDesc rain{};
    Dev<StepScalars> sc;
    StepScalars hs{};
    Dev<double> vol;
    // host copies needed to rebuild records
    std::vector<uint32_t, NoInitAlloc<uint32_t>> host_meta;   // meta word per cell (host mirror)
    std::vector<uint8_t> host_soil;
    std::vector<R> host_tr;
    // van Genuchten infiltration: classes, globals, water-table depth per cell, DEM copy
    Dev<SoilClassVG<R>> classes_vg;
    int n_classes_vg = 0;
    VGGlobals<R> vgg{};
    std::vector<R> host_zwt;
    std::vector<double> host_z;   // host copy of the DEM, fetched from z_keep when a setter needs it
    Dev<double> z_keep;           // the caller's DEM (FP64) as uploaded
    const std::vector<double>& hz() {
        if (host_z.size() != n) host_z = fetch(z_keep.p, n);
        return host_z;
    }
    bool static_ready = false, dirty = true;
    double last_dt_s = 0;
    int rows_per_warp = 64;
    bool rpw_chosen = false;   // set by hp2d_set_tuning / hp2d_autotune / an ensemble
    int n_sms = 0;
    // Rows per warp when none was chosen.  FP32 two-cell strips: of 40, 32, 24 and 16 rows the
    // one that best fills whole waves of resident CTAs (4 per SM) after the 4 halo rows per
    // block -- on a 4096 x 8192 grid 40 (3528 CTAs, 5.96 waves), on 2048 x 2048 32 (560 CTAs,
    // one wave; 40 rows leave 455 CTAs for 592 slots).  Other layouts keep rows_per_warp.
    int default_rows(int cpl) {
        if (sizeof(R) != 4 || cpl != 2) return rows_per_warp;
        if (!n_sms) HP_CK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, ctx->device));
        const double slots = double(FusedOcc<float, 2>::minb) * n_sms;
        const int strips = (nx + 59) / 60;
        int best = rows_per_warp;
        double best_score = -1.0;
        for (int r : {40, 32, 24, 16}) {
            const double ctas = std::ceil(double(strips) * ((ny + r - 1) / r) / 4.0);
            const double waves = std::ceil(ctas / slots);
            const double score = ctas / (waves * slots) * double(r) / double(r + 4);
            if (score > best_score + 1e-12) { best_score = score; best = r; }
        }
        return best;
    }
    int cells_per_lane = 1;   // fused-step layout: 1 (32-column strips) or 2 (64-column strips)
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;

    explicit Impl(hp2d_ctx* c) : ctx(c) {
        if (sizeof(R) == 4) {   // measured defaults for FP32 (hp2d_autotune refines them per grid)
            cells_per_lane = 2;
            rows_per_warp = 40;   // 4096 x 8192 dam-break: 94.7 GCUPS vs 93.5 at 32
        }
        ny = c->g.ny;
        nx = c->g.nx;
        n = size_t(ny) * nx;
        res = c->g.resolution;
        stat.alloc(n);
        for (int b = 0; b < 2; ++b) st4[b].alloc(n);
        arrival.alloc(n);
        sc.alloc(1);
        vol.alloc(1);
        bit_words = (nx + 31) / 32;
        host_meta.resize(n);
        host_parallel(n, [&](size_t a, size_t b) { std::fill(host_meta.begin() + a, host_meta.begin() + b, 255u); });
        std::memset(&hs, 0, sizeof(hs));
        hs.t_min = c->p.min_time_step / 60.0;
        hs.time_step = c->p.min_time_step / 60.0;   // HydroPol2D_preprocessing.m:2469
        hs.k = 1;
        // the first step's rain: update_spatial_BC before the loop (HydroPol2D_Main_While.m:115)
        // over [t_previous, t] with t_previous = 0 (:120)
        hs.rain_a = 0.0;
        hs.rain_b = hs.t_min;
        hs.t_prev = 0.0;
        hs.catch_index = 1;                      // HydroPol2D_Main_While.m:266
        hs.max_dt = c->p.max_time_step;
        hs.fault_k = -1;
        push_sc();
        // closed faces everywhere until hp2d_upload_static, dry state
        const R qn = std::numeric_limits<R>::quiet_NaN();
        fill(stat.p, n, V4{qn, qn, R(0), make_meta<R>(255u)});
        const V4 dry{R(0), R(0), R(0), -std::numeric_limits<R>::infinity()};
        fill(st4[0].p, n, dry);
        fill(st4[1].p, n, dry);
        fill(arrival.p, n, std::numeric_limits<R>::infinity());
    }
    ~Impl() override {
        if (graph) cudaGraphExecDestroy(graph);
        free_rec_host();
    }

    cudaStream_t st() const { return ctx->stream; }
    HostStage stage;   // staging of pageable caller arrays
    void h2d(void* dev, const void* host, size_t bytes) {
        stage.copy(dev, const_cast<void*>(host), bytes, true, st(), ctx->device);
    }
    void push_sc() { HP_CK(cudaMemcpyAsync(sc.p, &hs, sizeof(hs), cudaMemcpyHostToDevice, st())); HP_CK(cudaStreamSynchronize(st())); }
    void pull_sc() { HP_CK(cudaMemcpyAsync(&hs, sc.p, sizeof(hs), cudaMemcpyDeviceToHost, st())); HP_CK(cudaStreamSynchronize(st())); }

    // the library's own host vectors: one copy (the driver stages pageable memory itself; the
    // context's staging chunks are for the caller's large arrays, whose page-locked allocation
    // would cost more than it saves here)
    template <typename T, typename A> void upload(T* dst, const std::vector<T, A>& v) {
        if (v.empty()) return;
        HP_CK(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st()));
        HP_CK(cudaStreamSynchronize(st()));
    }
    template <typename T> std::vector<T> fetch(const T* src, size_t count) {
        std::vector<T> v(count);
        if (count) {
            HP_CK(cudaMemcpyAsync(v.data(), src, count * sizeof(T), cudaMemcpyDeviceToHost, st()));
            HP_CK(cudaStreamSynchronize(st()));
        }
        return v;
    }
    template <typename T> void fill(T* p, size_t count, T v) {   // on the device, no host staging
        if (!count) return;
        k_fill<T><<<blocks_for(count), kThreads, 0, st()>>>(count, p, v);
        HP_CK(cudaGetLastError());
        HP_CK(cudaStreamSynchronize(st()));
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
        return int(std::max<size_t>(1, std::min<size_t>(b, 148 * 32)));
    }
    // infiltration model in use: 0 none, 1 Green-Ampt, 2 van Genuchten
    int inf_mode() const {
        if (ctx->p.flag_infiltration == 1 && n_classes > 0) return 1;
        if (ctx->p.flag_infiltration == 2 && n_classes_vg > 0) return 2;
        return 0;
    }
    bool ga() const { return inf_mode() != 0; }
    bool soil_missing() const {
        return (ctx->p.flag_infiltration == 1 && n_classes == 0) || (ctx->p.flag_infiltration == 2 && n_classes_vg == 0);
    }
    // initial second component of a soil record: recovery timer (Green-Ampt) or water-table depth
    R soil_y(size_t k) const {
        if (host_soil.empty() || host_soil[k] == 255) return R(0);
        return inf_mode() == 2 ? host_zwt[k] : host_tr[host_soil[k]];
    }


    void write_meta() {
        Dev<uint32_t> m;
        m.alloc(n);
        upload(m.p, host_meta);
        k_write_meta<R><<<blocks_for(n), kThreads, 0, st()>>>(n, stat.p, m.p);
        HP_CK(cudaGetLastError());
        HP_CK(cudaStreamSynchronize(st()));
    }

    hp2d_status upload_static(const double* z, const double* rough, const int32_t* rows, const int32_t* cols,
                              int32_t nout, const double* slopes) {
        host_z.clear();
        const double edge = std::numeric_limits<double>::infinity();   // closed domain-edge face
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
        if (size_t(outs.size()) >= (1u << 23)) { ctx->err = "too many outlet cells"; return HP2D_INVALID_ARG; }
        std::sort(outs.begin(), outs.end(), [](auto& x, auto& y) { return x.first < y.first; });
        outs.erase(std::unique(outs.begin(), outs.end(), [](auto& x, auto& y) { return x.first == y.first; }), outs.end());
        n_out = int(outs.size());
        host_parallel(n, [&](size_t a, size_t b) {   // outlets and inflow cells are set anew
            for (size_t k = a; k < b; ++k) host_meta[k] &= 255u;
        });
        inflow.n_gauges = 0;
        inflow.n_stage = 0;
        inflow_cells_h = BcCells{};
        stage_cells_h = BcCells{};
        strct = StructDesc<R>{};   // the structures' cells are set anew too
        struct_cells_h.clear();
        std::vector<int32_t> cells(n_out);
        std::vector<R> coefs(n_out);
        std::vector<uint32_t> bits(size_t(ny) * bit_words, 0u);
        for (int o = 0; o < n_out; ++o) {
            cells[o] = outs[o].first;
            coefs[o] = outs[o].second;
            host_meta[cells[o]] |= uint32_t(o + 1) << 8;
            int i = cells[o] / nx, j = cells[o] % nx;
            bits[size_t(i) * bit_words + (j >> 5)] |= 1u << (j & 31);
        }
        // the records (and the unfused entry points' structure-of-arrays copies) are built
        // on the device from the caller's FP64 arrays
        {
            Dev<double> dr_;
            Dev<uint32_t> dm_;
            if (z_keep.n != n) z_keep.alloc(n);   // kept: setters that need the DEM fetch it
            dr_.alloc(n); dm_.alloc(n);
            h2d(z_keep.p, z, n * sizeof(double));
            h2d(dr_.p, rough, n * sizeof(double));
            if (host_soil.empty()) {   // the same words as the host mirror, built on the device
                Dev<int32_t> dc;
                dc.alloc(size_t(std::max(n_out, 1)));
                if (n_out) upload(dc.p, cells);
                fill(dm_.p, n, 255u);
                if (n_out) k_outlet_meta_scatter<<<(n_out + kThreads - 1) / kThreads, kThreads, 0, st()>>>(dc.p, n_out, dm_.p);
                HP_CK(cudaGetLastError());
                HP_CK(cudaStreamSynchronize(st()));
            } else {
                upload(dm_.p, host_meta);
            }
            // the unfused entry points' copies are extracted from the records on first use
            dzx.free(); dzy.free(); n2.free();
            k_build_static<R><<<blocks_for(n), kThreads, 0, st()>>>(ny, nx, z_keep.p, dr_.p, dm_.p, stat.p, nullptr,
                                                                     nullptr, nullptr);
            HP_CK(cudaGetLastError());
            HP_CK(cudaStreamSynchronize(st()));
        }
        (void)edge;
        outlet_bits.alloc(bits.size());
        upload(outlet_bits.p, bits);
        outlet_cells.alloc(std::max(n_out, 1));
        outlet_coef.alloc(std::max(n_out, 1));
        hf3.alloc(std::max(n_out, 1));
        qo.alloc(std::max(n_out, 1));
        upload(outlet_cells.p, cells);
        upload(outlet_coef.p, coefs);
        fill(hf3.p, std::max(n_out, 1), R(0));
        fill(qo.p, std::max(n_out, 1), R(0));
        static_ready = true;
        invalidate_graph();
        dirty = true;
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
        classes.alloc(ncls);
        upload(classes.p, t);
        n_classes = ncls;
        host_soil.assign(cls, cls + n);
        host_tr.resize(ncls);
        for (int c = 0; c < ncls; ++c) host_tr[c] = t[c].tr;
        host_parallel(n, [&](size_t a, size_t b) {
            for (size_t k = a; k < b; ++k) host_meta[k] = (host_meta[k] & ~255u) | cls[k];
        });
        write_meta();
        soil.alloc(n);
        upload(soil.p, host_soil);
        // soil records: keep I if present, recovery timer restarts at Tr
        std::vector<V2> g(n);
        if (gs2[0].p) g = fetch(gs2[hs.cur].p, n);
        else for (size_t k = 0; k < n; ++k) g[k] = V2{R(0), R(0)};
        for (size_t k = 0; k < n; ++k) g[k].y = soil_y(k);
        alloc_soil_records();
        upload(gs2[hs.cur].p, g);
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_soil_vg(const uint8_t* cls, int32_t ncls, const double* theta_r, const double* theta_s,
                            const double* n_vg, const double* alpha, const double* ksat, const double* soil_depth,
                            const double* gw_head, double l_vg, double ltop, double dh_max, double wk) {
        if (!static_ready) { ctx->err = "hp2d_upload_static first (the water-table depth needs the DEM)"; return HP2D_NOT_READY; }
        if (ncls <= 0 || ncls > 255) { ctx->err = "n_classes must be in 1..255"; return HP2D_INVALID_ARG; }
        for (size_t k = 0; k < n; ++k)
            if (cls[k] != 255 && cls[k] >= ncls) { ctx->err = "soil class index out of range"; return HP2D_INVALID_ARG; }
        std::vector<SoilClassVG<R>> t(ncls);
        for (int c = 0; c < ncls; ++c) {
            if (!(n_vg[c] > 1.0) || !(alpha[c] > 0.0) || !(theta_s[c] >= theta_r[c])) {
                ctx->err = "van Genuchten classes need n > 1, alpha > 0 and theta_sat >= theta_r";
                return HP2D_INVALID_ARG;
            }
            const double m = 1.0 - 1.0 / n_vg[c];
            t[c].ks = R(ksat[c] / 1000.0 / 3600.0);
            t[c].theta_r = R(theta_r[c]);
            t[c].theta_s = R(theta_s[c]);
            t[c].alpha = R(alpha[c]);
            t[c].inv_n = R(1.0 / n_vg[c]);
            t[c].m = R(m);
            t[c].inv_m = R(1.0 / m);
            t[c].pad = R(0);
        }
        classes_vg.alloc(ncls);
        upload(classes_vg.p, t);
        n_classes_vg = ncls;
        vgg.ell = R(l_vg);
        vgg.ltop = R(std::max(ltop, 1e-6));                    // Infiltration_Module.m:232
        vgg.dh_max = R(dh_max);
        vgg.wk = R(std::min(std::max(wk, 0.0), 1.0));          // :321
        // water-table depth (Infiltration_Module.m:192-199): GW_Depth = h_t - (z - Soil_Depth),
        // zwt = max(Soil_Depth - GW_Depth, 0); no head given = water table at the soil bottom
        host_zwt.assign(n, R(0));
        const std::vector<double>& zz = hz();
        for (size_t k = 0; k < n; ++k) {
            const double sd = soil_depth[k];
            const double ht = gw_head ? gw_head[k] : zz[k] - sd;
            const double gwd = ht - (zz[k] - sd);
            host_zwt[k] = R(std::max(sd - gwd, 0.0));
        }
        host_soil.assign(cls, cls + n);
        host_parallel(n, [&](size_t a, size_t b) {
            for (size_t k = a; k < b; ++k) host_meta[k] = (host_meta[k] & ~255u) | cls[k];
        });
        write_meta();
        soil.alloc(n);
        upload(soil.p, host_soil);
        std::vector<V2> g(n);
        if (gs2[0].p) g = fetch(gs2[hs.cur].p, n);
        else for (size_t k = 0; k < n; ++k) g[k] = V2{R(0), R(0)};
        for (size_t k = 0; k < n; ++k) g[k].y = soil_y(k);
        alloc_soil_records();
        upload(gs2[hs.cur].p, g);
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_state(const double* d, const double* outflow, const double* Imm) {
        pull_sc();
        {   // records built on the device from the caller's arrays
            Dev<double> dq;
            double* dd = readback_buffer();   // the read-back buffer doubles as upload staging
            h2d(dd, d, n * sizeof(double));
            if (outflow) {
                dq.alloc(2 * n);
                h2d(dq.p, outflow, 2 * n * sizeof(double));
            }
            k_build_state<R><<<blocks_for(n), kThreads, 0, st()>>>(n, dd, outflow ? dq.p : nullptr, res,
                                                                    st4[hs.cur].p);
            HP_CK(cudaGetLastError());
            HP_CK(cudaStreamSynchronize(st()));
        }
        if (Imm || gs2[0].p) {
            alloc_soil_records();
            std::vector<V2> g(n);
            std::vector<V2> old;
            if (!Imm) old = fetch(gs2[hs.cur].p, n);
            for (size_t k = 0; k < n; ++k) {
                g[k].x = Imm ? R(Imm[k] / 1000.0) : old[k].x;
                g[k].y = soil_y(k);
            }
            upload(gs2[hs.cur].p, g);
        }
        fill(arrival.p, n, std::numeric_limits<R>::infinity());
        hs.halted = 0;   // a new state starts over after a failed call
        push_sc();
        dirty = true;
        return HP2D_OK;
    }

    // The rain interval follows the clock: k = 1 starts as a fresh run; k one above the
    // current counter is the loop's advance (the interval becomes [t_previous, old clock]
    // and t_previous the increment time_step on the first step, the old clock after it);
    // any other k re-seeds it as if the last two steps had taken time_step
    // (hp2d_set_rain_clock sets it exactly).
    hp2d_status set_clock(double t, double time_step, int64_t k) {
        pull_sc();
        if (k == 1) {
            hs.rain_a = 0.0;
            hs.rain_b = t;
            hs.t_prev = 0.0;
        } else if (k == hs.k + 1) {
            hs.rain_a = hs.t_prev;
            hs.rain_b = hs.t_min;
            hs.t_prev = hs.k == 1 ? time_step : hs.t_min;
        } else {
            hs.rain_a = t - 2.0 * time_step;
            hs.rain_b = t - time_step;
            hs.t_prev = t - time_step;
        }
        hs.t_min = t;
        hs.time_step = time_step;
        hs.k = k;
        hs.halted = 0;
        push_sc();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_rain_clock(double rain_a, double rain_b, double t_previous) {
        pull_sc();
        hs.rain_a = rain_a;
        hs.rain_b = rain_b;
        hs.t_prev = t_previous;
        push_sc();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_rain_uniform(int32_t cnt, const double* t0, const double* rate) {
        rain_t.alloc(std::max(cnt, 1));
        rain_r.alloc(std::max(cnt, 1));
        if (cnt) {
            upload(rain_t.p, std::vector<double>(t0, t0 + cnt));
            upload(rain_r.p, std::vector<double>(rate, rate + cnt));
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
        if (map_dt * 60.0 < ctx->p.max_time_step) {   // a step's rain interval spans at most two maps
            ctx->err = "rain map interval shorter than max_time_step";
            return HP2D_INVALID_ARG;
        }
        size_t cnt = size_t(nm) * my * mx;
        maps.alloc(cnt);
        upload(maps.p, std::vector<float>(rate, rate + cnt));
        rain.n_maps = nm; rain.my = my; rain.mx = mx; rain.map_dt = map_dt; rain.maps = maps.p;
        rain.map_t = nullptr;
        rain.n_uniform = 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    // End-stamped input rain maps (flag_input_rainfall_map = 1): map m holds over
    // [t_end[m-1], t_end[m]), the first one from t_end[0] - dt_force
    Dev<double> map_edges;
    hp2d_status set_rain_maps_end_stamped(int32_t nm, int32_t my, int32_t mx, const float* rate, const double* t_end,
                                          double dt_force) {
        if (nm <= 0 || my <= 0 || mx <= 0 || !rate || !t_end || !(dt_force >= 0)) {
            ctx->err = "bad input rain maps";
            return HP2D_INVALID_ARG;
        }
        std::vector<double> e(size_t(nm) + 1);
        e[0] = t_end[0] - dt_force;
        for (int q = 0; q < nm; ++q) e[size_t(q) + 1] = t_end[q];
        for (int q = 0; q < nm; ++q) {
            if (!(e[size_t(q) + 1] >= e[q]) || !std::isfinite(e[q]) || !std::isfinite(e[size_t(q) + 1])) {
                ctx->err = "map end times must be finite and non-decreasing";
                return HP2D_INVALID_ARG;
            }
            // an interval shorter than a step could make a step's rain span three maps
            if (e[size_t(q) + 1] > e[q] && (e[size_t(q) + 1] - e[q]) * 60.0 < ctx->p.max_time_step) {
                ctx->err = "rain map interval shorter than max_time_step";
                return HP2D_INVALID_ARG;
            }
        }
        size_t cnt = size_t(nm) * my * mx;
        maps.alloc(cnt);
        upload(maps.p, std::vector<float>(rate, rate + cnt));
        map_edges.alloc(e.size());
        upload(map_edges.p, e);
        rain.n_maps = nm; rain.my = my; rain.mx = mx; rain.map_dt = 0.0; rain.maps = maps.p;
        rain.map_t = map_edges.p;
        rain.n_uniform = 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    // Rain gauges: one IDW map per record interval of dt minutes, computed on the device and
    // used as full-resolution rain maps
    hp2d_status set_rain_gauges(int32_t ng, const double* xg, const double* yg, int32_t nt, double dt,
                                const double* rate, double x_ul, double y_ul) {
        if (ng <= 0 || nt <= 0 || !(dt > 0)) { ctx->err = "bad rain gauge table"; return HP2D_INVALID_ARG; }
        if (dt * 60.0 < ctx->p.max_time_step) {
            ctx->err = "rain record interval shorter than max_time_step";
            return HP2D_INVALID_ARG;
        }
        Dev<double> dx, dy, dr;
        dx.alloc(size_t(ng)); dy.alloc(size_t(ng)); dr.alloc(size_t(nt) * ng);
        upload(dx.p, std::vector<double>(xg, xg + ng));
        upload(dy.p, std::vector<double>(yg, yg + ng));
        upload(dr.p, std::vector<double>(rate, rate + size_t(nt) * ng));
        maps.alloc(size_t(nt) * n);
        k_idw_maps<<<blocks_for(n), kThreads, 0, st()>>>(ny, nx, res, x_ul, y_ul, ng, dx.p, dy.p, nt, dr.p, maps.p);
        HP_CK(cudaGetLastError());
        HP_CK(cudaStreamSynchronize(st()));
        rain.n_maps = nt; rain.my = ny; rain.mx = nx; rain.map_dt = dt; rain.maps = maps.p;
        rain.map_t = nullptr;
        rain.n_uniform = 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    // Boundary-condition cells: inflow hydrographs and stage hydrographs share one entry table
    // (meta bit 31 + entry); each setter keeps its cell list and rebuilds the table.
    struct BcCells { std::vector<size_t> cell; std::vector<int32_t> gauge; };
    BcCells inflow_cells_h, stage_cells_h;
    Dev<double> stage_t, stage_d;
    Dev<R> stage_now;
    Dev<int32_t> bc_stage;

    hp2d_status check_bc_cells(int32_t ng, int32_t nc, const int32_t* rows, const int32_t* cols,
                               const int32_t* gauge, BcCells& out, const char* what) {
        out.cell.clear();
        out.gauge.clear();
        for (int q = 0; q < (ng ? nc : 0); ++q) {
            if (rows[q] < 0 || rows[q] >= ny || cols[q] < 0 || cols[q] >= nx || gauge[q] < 0 || gauge[q] >= ng) {
                ctx->err = std::string(what) + " cell or gauge out of range";
                return HP2D_INVALID_ARG;
            }
            const size_t k = size_t(rows[q]) * nx + cols[q];
            if (!(host_meta[k] & kInflowBit) && (host_meta[k] >> 8) != 0u) {
                ctx->err = std::string("an outlet cell cannot also be an ") + what + " cell";
                return HP2D_INVALID_ARG;
            }
            out.cell.push_back(k);
            out.gauge.push_back(gauge[q]);
        }
        return HP2D_OK;
    }

    void rebuild_bc_cells() {
        const int ng = inflow.n_gauges;
        std::vector<std::vector<int32_t>> per(n);
        std::vector<int32_t> stg(n, -1);
        std::vector<size_t> used;
        auto mark = [&](size_t k) {
            if (per[k].empty() && stg[k] < 0) used.push_back(k);
        };
        for (size_t q = 0; q < inflow_cells_h.cell.size(); ++q) {
            mark(inflow_cells_h.cell[q]);
            per[inflow_cells_h.cell[q]].push_back(inflow_cells_h.gauge[q]);
        }
        for (size_t q = 0; q < stage_cells_h.cell.size(); ++q) {   // the reference overwrites in
            const size_t k = stage_cells_h.cell[q];                  // gauge order: the last wins
            if (per[k].empty() && stg[k] < 0) used.push_back(k);
            stg[k] = std::max(stg[k], stage_cells_h.gauge[q]);
        }
        for (size_t q = 0; q < struct_cells_h.size(); ++q) used.push_back(struct_cells_h[q]);
        for (size_t k = 0; k < n; ++k)
            if (host_meta[k] & kInflowBit) host_meta[k] &= 255u;
        std::sort(used.begin(), used.end());
        used.erase(std::unique(used.begin(), used.end()), used.end());
        std::vector<int32_t> off(1, 0), gl, st, ss;
        host_gcells.assign(size_t(ng), 0.0);
        for (size_t e = 0; e < used.size(); ++e) {
            const size_t k = used[e];
            auto& v = per[k];
            std::sort(v.begin(), v.end());   // a cell listed twice for a gauge gets it twice
            for (int32_t g : v) {
                gl.push_back(g);
                if (std::isfinite(hz()[k])) host_gcells[size_t(g)] += 1.0;
            }
            off.push_back(int32_t(gl.size()));
            st.push_back(stg[k]);
            const auto it = std::find(struct_cells_h.begin(), struct_cells_h.end(), k);
            ss.push_back(it == struct_cells_h.end() ? -1 : int32_t(it - struct_cells_h.begin()));
            host_meta[k] = (host_meta[k] & 255u) | kInflowBit | (uint32_t(e) << 8);
        }
        write_meta();
        inf_off.alloc(off.size());
        inf_gauge.alloc(std::max<size_t>(gl.size(), 1));
        bc_stage.alloc(std::max<size_t>(st.size(), 1));
        bc_struct.alloc(std::max<size_t>(ss.size(), 1));
        upload(inf_off.p, off);
        if (!gl.empty()) upload(inf_gauge.p, gl);
        if (!st.empty()) upload(bc_stage.p, st);
        if (!ss.empty()) upload(bc_struct.p, ss);
        if (ng) {
            inf_cells.alloc(size_t(ng));
            upload(inf_cells.p, host_gcells);
        }
        inflow.cell_off = inf_off.p;
        inflow.cell_gauge = inf_gauge.p;
        inflow.cell_stage = bc_stage.p;
        inflow.cell_struct = bc_struct.p;
        inflow.gauge_cells = inf_cells.p;
        invalidate_graph();
        dirty = true;
    }

    // Inflow hydrographs: gauge rates [n_times][n_gauges] on the start-stamped table t_start,
    // (row, col, gauge) cells; replaces any earlier inflow (n_gauges = 0 removes it).
    hp2d_status set_inflow(int32_t ng, int32_t nt, const double* t0, const double* rate, int32_t nc,
                           const int32_t* rows, const int32_t* cols, const int32_t* gauge) {
        if (!static_ready) { ctx->err = "hp2d_upload_static must come before hp2d_set_inflow"; return HP2D_NOT_READY; }
        if (ng < 0 || (ng > 0 && (nt < 1 || nc < 1))) { ctx->err = "bad inflow table shape"; return HP2D_INVALID_ARG; }
        BcCells cells;
        hp2d_status s = check_bc_cells(ng, nc, rows, cols, gauge, cells, "inflow");
        if (s != HP2D_OK) return s;
        if (inflow_cells_h.cell.size() + stage_cells_h.cell.size() + cells.cell.size() >= (1u << 23)) {
            ctx->err = "too many inflow cells";
            return HP2D_INVALID_ARG;
        }
        if (ng) {
            inf_t.alloc(size_t(nt));
            inf_r.alloc(size_t(nt) * ng);
            inf_depth.alloc(size_t(ng));
            upload(inf_t.p, std::vector<double>(t0, t0 + nt));
            upload(inf_r.p, std::vector<double>(rate, rate + size_t(nt) * ng));
        }
        inflow.n_gauges = ng;
        inflow.n_times = nt;
        inflow.t_start = inf_t.p;
        inflow.rate = inf_r.p;
        inflow.depth = inf_depth.p;
        inflow_cells_h = std::move(cells);
        rebuild_bc_cells();
        return HP2D_OK;
    }

    // Stage hydrographs: gauge water depths [m] [n_times][n_gauges] on the start-stamped table
    // t_start, (row, col, gauge) cells; n_gauges = 0 removes them.
    hp2d_status set_stage(int32_t ng, int32_t nt, const double* t0, const double* depth, int32_t nc,
                          const int32_t* rows, const int32_t* cols, const int32_t* gauge) {
        if (!static_ready) { ctx->err = "hp2d_upload_static must come before hp2d_set_stage"; return HP2D_NOT_READY; }
        if (ng < 0 || (ng > 0 && (nt < 1 || nc < 1))) { ctx->err = "bad stage table shape"; return HP2D_INVALID_ARG; }
        BcCells cells;
        hp2d_status s = check_bc_cells(ng, nc, rows, cols, gauge, cells, "stage");
        if (s != HP2D_OK) return s;
        for (size_t k : cells.cell)
            if (!std::isfinite(hz()[k])) { ctx->err = "a stage cell needs a finite elevation"; return HP2D_INVALID_ARG; }
        if (inflow_cells_h.cell.size() + stage_cells_h.cell.size() + cells.cell.size() >= (1u << 23)) {
            ctx->err = "too many stage cells";
            return HP2D_INVALID_ARG;
        }
        if (ng) {
            stage_t.alloc(size_t(nt));
            stage_d.alloc(size_t(nt) * ng);
            stage_now.alloc(size_t(ng));
            upload(stage_t.p, std::vector<double>(t0, t0 + nt));
            upload(stage_d.p, std::vector<double>(depth, depth + size_t(nt) * ng));
        }
        inflow.n_stage = ng;
        inflow.n_stage_times = nt;
        inflow.stage_t = stage_t.p;
        inflow.stage_d = stage_d.p;
        inflow.stage_now = stage_now.p;
        stage_cells_h = std::move(cells);
        rebuild_bc_cells();
        return HP2D_OK;
    }

    // Reservoir / control structures (flag_reservoir, Local_Inertial_Model_D4.m:318-344):
    // structure i drains cell (res_row, res_col) through rating curve (k1, h1, k2) into
    // (ds1_row, ds1_col) and, when ds2_row >= 0, through (k3, h2, k4) into (ds2_row, ds2_col);
    // 0-based cells, ds1_row < 0 for none.  n = 0 removes them.
    StructDesc<R> strct{};
    std::vector<size_t> struct_cells_h;   // slot -> cell
    Dev<double> st_coef, st_acc;
    Dev<int32_t> st_slot, st_slot_cell, bc_struct;
    Dev<R> st_hres, st_extra;

    hp2d_status set_reservoirs(int32_t ns, const int32_t* rr, const int32_t* rc, const double* k1, const double* h1,
                               const double* k2, const int32_t* d1r, const int32_t* d1c, const double* k3,
                               const double* h2, const double* k4, const int32_t* d2r, const int32_t* d2c) {
        if (!static_ready) { ctx->err = "hp2d_upload_static must come before hp2d_set_reservoirs"; return HP2D_NOT_READY; }
        if (ns < 0) { ctx->err = "negative structure count"; return HP2D_INVALID_ARG; }
        if (ns > 0 && ctx->p.flag_reservoir != 1) { ctx->err = "structures need flag_reservoir = 1"; return HP2D_INVALID_ARG; }
        std::vector<size_t> cells;
        std::vector<int32_t> slot(size_t(ns) * 3, -1);
        std::vector<double> coef(size_t(ns) * 6);
        auto slot_of = [&](int32_t r, int32_t c, int32_t& out) -> hp2d_status {
            if (r < 0 || r >= ny || c < 0 || c >= nx) { ctx->err = "structure cell out of range"; return HP2D_INVALID_ARG; }
            const size_t k = size_t(r) * nx + c;
            if (!(host_meta[k] & kInflowBit) && (host_meta[k] >> 8) != 0u) {
                ctx->err = "an outlet cell cannot also be a structure cell";
                return HP2D_INVALID_ARG;
            }
            if (!std::isfinite(hz()[k])) { ctx->err = "a structure cell needs a finite elevation"; return HP2D_INVALID_ARG; }
            auto it = std::find(cells.begin(), cells.end(), k);
            out = int32_t(it - cells.begin());
            if (it == cells.end()) cells.push_back(k);
            return HP2D_OK;
        };
        for (int i = 0; i < ns; ++i) {
            const double cf[6] = {k1[i], h1[i], k2[i], k3[i], h2[i], k4[i]};
            for (int q = 0; q < 6; ++q) coef[size_t(i) * 6 + q] = cf[q];
            hp2d_status s = slot_of(rr[i], rc[i], slot[3 * i]);
            if (s != HP2D_OK) return s;
            if (d1r[i] >= 0) {
                if (!(std::isfinite(k1[i]) && std::isfinite(h1[i]) && std::isfinite(k2[i]))) {
                    ctx->err = "non-finite rating curve";
                    return HP2D_INVALID_ARG;
                }
                if ((s = slot_of(d1r[i], d1c[i], slot[3 * i + 1])) != HP2D_OK) return s;
            }
            if (d2r[i] >= 0) {
                // the reference indexes ds1 in the second structure's branch
                if (d1r[i] < 0) { ctx->err = "a second structure needs a first downstream cell"; return HP2D_INVALID_ARG; }
                if (!(std::isfinite(k3[i]) && std::isfinite(h2[i]) && std::isfinite(k4[i]))) {
                    ctx->err = "non-finite rating curve";
                    return HP2D_INVALID_ARG;
                }
                if ((s = slot_of(d2r[i], d2c[i], slot[3 * i + 2])) != HP2D_OK) return s;
            }
        }
        if (inflow_cells_h.cell.size() + stage_cells_h.cell.size() + cells.size() >= (1u << 23)) {
            ctx->err = "too many boundary cells";
            return HP2D_INVALID_ARG;
        }
        strct = StructDesc<R>{};
        if (ns > 0) {
            const size_t m = cells.size();
            st_coef.alloc(coef.size());
            st_slot.alloc(slot.size());
            st_slot_cell.alloc(m);
            st_hres.alloc(size_t(ns));
            st_acc.alloc(2 * m);
            st_extra.alloc(m);
            upload(st_coef.p, coef);
            upload(st_slot.p, slot);
            std::vector<int32_t> sc32(cells.begin(), cells.end());
            upload(st_slot_cell.p, sc32);
            fill(st_extra.p, m, R(0));
            strct = StructDesc<R>{ns, int(m), st_coef.p, st_slot.p, st_slot_cell.p, st_hres.p, st_acc.p, st_extra.p};
        }
        struct_cells_h = std::move(cells);
        rebuild_bc_cells();
        return HP2D_OK;
    }

    // Map records at the reference's record times (save_output_maps.m): n_slots depth maps
    // kept on the device, the oldest overwritten first; n_times = 0 switches them off.
    hp2d_status set_map_records(int32_t nt, const double* times, int32_t nslots) {
        if (nt < 0 || (nt > 0 && (!times || nslots < 1))) { ctx->err = "bad map record table"; return HP2D_INVALID_ARG; }
        for (int q = 1; q < nt; ++q)
            if (!(times[q] > times[q - 1])) { ctx->err = "record times must increase"; return HP2D_INVALID_ARG; }
        rec = RecordDesc<R>{};
        rec_snap.free();
        free_rec_host();
        if (nt > 0) {
            rec_times.alloc(size_t(nt));
            upload(rec_times.p, std::vector<double>(times, times + nt));
            R* snap = nullptr;
            if (rec_target == 1) {
                HP_CK(cudaHostAlloc(reinterpret_cast<void**>(&rec_host), size_t(nslots) * n * sizeof(R),
                                    cudaHostAllocMapped | cudaHostAllocPortable));
                rec_host_n = size_t(nslots) * n;
                HP_CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&snap), rec_host, 0));
            } else {
                rec_snap.alloc(size_t(nslots) * n);
                snap = rec_snap.p;
            }
            rec_t.alloc(size_t(nslots));
            rec = RecordDesc<R>{nt, nslots, rec_times.p, snap, rec_t.p};
        }
        pull_sc();
        hs.rec_count = 0;
        hs.rec_pending = 0;
        hs.rec_last = nt > 0 ? last_record_below(times, nt, hs.t_min) : 0;
        push_sc();
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }
    // a record whose step had no successor copies the current depth now (hs pulled)
    void flush_records() {
        if (!rec.n_slots || !hs.rec_pending) return;
        const int64_t slot = hs.rec_count % rec.n_slots;
        k_record_depth<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[hs.cur].p, rec.snap + size_t(slot) * n);
        HP_CK(cudaGetLastError());
        hs.rec_count += 1;
        hs.rec_pending = 0;
        push_sc();
    }
    hp2d_status set_record_target(int32_t target, int32_t n_times, const double* times, int32_t n_slots) {
        if (target != 0 && target != 1) { ctx->err = "record target must be 0 (device) or 1 (mapped host memory)"; return HP2D_INVALID_ARG; }
        rec_target = target;
        return set_map_records(n_times, times, n_slots);
    }
    hp2d_status map_records(int64_t* count) {
        pull_sc();
        flush_records();
        *count = hs.rec_count;
        return HP2D_OK;
    }
    hp2d_status download_map_record(int64_t index, double* depth_mm, double* t_min) {
        pull_sc();
        flush_records();
        if (!rec.n_slots || index < 0 || index >= hs.rec_count || index < hs.rec_count - rec.n_slots) {
            ctx->err = "map record not held (never taken or overwritten)";
            return HP2D_INVALID_ARG;
        }
        const size_t slot = size_t(index % rec.n_slots);
        if (rec_host) {   // already in host memory: the steps wrote it there
            HP_CK(cudaStreamSynchronize(st()));
            const R* v = rec_host + slot * n;
            for (size_t k = 0; k < n; ++k) depth_mm[k] = double(v[k]) * 1000.0;
        } else {
            double* d = readback_buffer();
            k_scaled_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, rec.snap + slot * n, 1000.0, d);
            copy_out(d, depth_mm);
        }
        if (t_min) {
            double t = 0;
            HP_CK(cudaMemcpyAsync(&t, rec.snap_t + slot, sizeof(double), cudaMemcpyDeviceToHost, st()));
            HP_CK(cudaStreamSynchronize(st()));
            *t_min = t;
        }
        return HP2D_OK;
    }

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
    // each call unpacks the records of the current buffer into the SoA scratch, runs
    // the stage kernels and packs the result back
    void ensure_scratch() {
        if (!h.p) {
            h.alloc(n); qx.alloc(n); qy.alloc(n); dmax.alloc(n); I.alloc(n); T.alloc(n);
            hfx.alloc(n); hfy.alloc(n); qxu.alloc(n); qyu.alloc(n); scale.alloc(n);
            fill(hfx.p, n, R(0));
            fill(hfy.p, n, R(0));
        }
    }
    void unpack() {
        ensure_scratch();
        const int cur = hs.cur;
        k_unpack<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[cur].p, gs2[cur].p, h.p, qx.p, qy.p, dmax.p, I.p, T.p);
        HP_CK(cudaGetLastError());
    }
    void pack() {
        const int cur = hs.cur;
        k_pack<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[cur].p, gs2[cur].p, h.p, qx.p, qy.p, dmax.p, I.p, T.p);
        HP_CK(cudaGetLastError());
    }

    hp2d_status hydrology_step(double time_step) {
        pull_sc();
        hs.acc_neg = 0;
        push_sc();
        unpack();
        double dts = time_step * 60.0;
        if (inflow.n_gauges) {   // gauge depths of the current rain interval
            k_inflow_depth<R><<<1, kThreads, 0, st()>>>(inflow, sc.p);
            HP_CK(cudaGetLastError());
        }
        k_hydro_rain_ga<R><<<blocks_for(n), kThreads, 0, st()>>>(view(), hs.rain_a, hs.rain_b, dts, rain, h.p, I.p, T.p, soil.p,
                                                               classes.p, classes_vg.p, vgg, inf_mode(), inflow,
                                                               stat.p, sc.p);
        HP_CK(cudaGetLastError());
        k_hydro_clamp<R><<<blocks_for(n), kThreads, 0, st()>>>(n, h.p, sc.p);
        HP_CK(cudaGetLastError());
        pack();
        std::vector<R> gd;
        if (inflow.n_gauges) gd = fetch(inf_depth.p, size_t(inflow.n_gauges));
        pull_sc();
        if (hs.acc_neg) hs.neg_warn += 1;
        for (size_t g = 0; g < gd.size(); ++g) hs.inflow_vol += double(gd[g]) * host_gcells[g] * res * res;
        push_sc();
        fold_accumulators();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status li_step(double time_step) {
        pull_sc();
        unpack();
        double dts = time_step * 60.0;
        auto gv = view();
        int nb = blocks_for(n);
        if (!dzx.p) {   // structure-of-arrays copies of the static record, made once
            dzx.alloc(n); dzy.alloc(n); n2.alloc(n);
            k_static_soa<R><<<nb, kThreads, 0, st()>>>(n, stat.p, dzx.p, dzy.p, n2.p);
            HP_CK(cudaGetLastError());
        }
        k_faces<R><<<nb, kThreads, 0, st()>>>(gv, dts, h.p, dzx.p, dzy.p, n2.p, qx.p, qy.p, hfx.p, hfy.p, qxu.p,
                                            qyu.p, ctx->p.flag_critical, ctx->p.flag_numerical_scheme);
        HP_CK(cudaGetLastError());
        k_scale<R><<<nb, kThreads, 0, st()>>>(gv, dts, h.p, qxu.p, qyu.p, scale.p);
        HP_CK(cudaGetLastError());
        k_limit<R><<<nb, kThreads, 0, st()>>>(gv, qxu.p, qyu.p, scale.p, qx.p, qy.p);
        HP_CK(cudaGetLastError());
        if (strct.n) {
            k_struct_unfused<R><<<1, 32, 0, st()>>>(strct, h.p, time_step, res * res, sc.p);
            HP_CK(cudaGetLastError());
        }
        k_continuity<R><<<nb, kThreads, 0, st()>>>(gv, dts, h.p, qx.p, qy.p);
        HP_CK(cudaGetLastError());
        if (n_out) {
            k_outlet<R><<<(n_out + kThreads - 1) / kThreads, kThreads, 0, st()>>>(
                gv, dts, h.p, outlet_cells.p, outlet_coef.p, n_out, ctx->p.outlet_type, hf3.p, qo.p, sc.p);
            HP_CK(cudaGetLastError());
        }
        pack();
        last_dt_s = dts;
        fold_accumulators();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status cfl_dt(double* ts_out, double* vmax_out) {
        if (!(last_dt_s > 0)) { ctx->err = "hp2d_cfl_dt needs a preceding hp2d_li_step"; return HP2D_NOT_READY; }
        pull_sc();
        hs.acc_vmax = hs.acc_cmax = 0;
        push_sc();
        unpack();
        k_cfl<R><<<blocks_for(n), kThreads, 0, st()>>>(view(), last_dt_s, qx.p, qy.p, hfx.p, hfy.p, outlet_bits.p,
                                                     bit_words, outlet_cells.p, hf3.p, n_out,
                                                     ctx->p.flag_adaptive_timestepping, sc.p);
        HP_CK(cudaGetLastError());
        pull_sc();
        const bool is_d = sizeof(R) == 8;
        double vm = from_ord(hs.acc_vmax, is_d), cm = from_ord(hs.acc_cmax, is_d);
        const hp2d_params& p = ctx->p;
        double tcr = finalize_dt(vm, cm, res, p.alfa_min, p.alfa_max, p.min_time_step, hs.max_dt,
                                 p.time_step_increments, p.flag_timestep);
        hs.acc_vmax = hs.acc_cmax = 0;
        hs.vmax_last = vm;
        if (tcr == p.min_time_step) hs.unstable += 1;
        push_sc();
        *ts_out = tcr / 60.0;
        if (vmax_out) *vmax_out = vm;
        return HP2D_OK;
    }

    hp2d_status track_maxima(double t_end) {
        pull_sc();
        unpack();
        R thr = R(ctx->p.arrival_threshold / 1000.0);
        k_track<R><<<blocks_for(n), kThreads, 0, st()>>>(n, h.p, dmax.p, arrival.p, thr, R(t_end * 60.0));
        HP_CK(cudaGetLastError());
        pack();
        HP_CK(cudaStreamSynchronize(st()));
        dirty = true;   // the records were rewritten from outside a fused step
        return HP2D_OK;
    }

    // ---------------- fused path ----------------
    FusedArgs<R> fused_args(int cpl = 0) {
        if (cpl <= 0) cpl = cells_per_lane;
        FusedArgs<R> a{};
        const hp2d_params& p = ctx->p;
        a.ny = ny; a.nx = nx; a.res = res;
        a.tol_mm = p.depth_tolerance; a.thr_mm = p.arrival_threshold;
        a.t_end = p.routing_time + p.min_time_step / 60.0;
        a.min_dt = p.min_time_step; a.max_dt = p.max_time_step; a.inc = p.time_step_increments;
        a.tsc = p.time_step_change; a.alfa_min = p.alfa_min; a.alfa_max = p.alfa_max;
        a.flag_timestep = p.flag_timestep; a.adaptive = p.flag_adaptive_timestepping;
        a.flag_critical = p.flag_critical; a.outlet_type = p.outlet_type; a.ga = ga() ? 1 : 0;
        a.scheme = p.flag_numerical_scheme;
        a.wait_polls = wait_polls;
        a.own_r0 = own_r0;
        a.own_r1 = own_r1 < 0 ? ny : own_r1;
        const int out_cols = 32 * cpl - 4;   // a strip's output columns (2-column apron each side)
        a.n_strips = (nx + out_cols - 1) / out_cols;
        const int rpw = rpw_chosen ? rows_per_warp : default_rows(cpl);
        a.rows_per_warp = rpw;
        a.n_warps_total = a.n_strips * ((ny + rpw - 1) / rpw);
        a.n_ctas = unsigned((a.n_warps_total + kThreads / 32 - 1) / (kThreads / 32));
        a.stag_s2 = stagnant_threshold<R>();
        a.stat = stat.p;
        a.st0 = st4[0].p; a.st1 = st4[1].p;
        a.gs0 = gs2[0].p; a.gs1 = gs2[1].p;
        a.classes = classes.p;
        a.classes_vg = classes_vg.p;
        a.vg = vgg;
        a.outlet_cells = outlet_cells.p; a.outlet_coef = outlet_coef.p; a.n_outlets = n_out;
        a.hf3 = hf3.p; a.qo = qo.p;
        a.arrival = arrival.p;
        a.rain = rain;
        a.inflow = inflow;
        a.rec = rec;
        a.strct = strct;
        a.dry_rows = dry_rows();
        a.dryflag = dry_usable(rpw) && tb_chosen <= 1 && !slab() ? dryf.p : nullptr;
        a.vmax = hz_on ? vmaxm.p : nullptr;
        a.hzmax = hz_on ? hzmaxm.p : nullptr;
        a.sc = sc.p;
        return a;
    }

    // kernels whose ring needs more than the default 48 KB of dynamic shared memory opt in
    // once per instantiation and device (before any graph capture: fused_steps and autotune
    // call this); the per-device flags of an instantiation are guarded by its own mutex, so
    // host threads sharing a device opt in once
    template <int INF, bool MAP, int CPL, bool INFL, int SCH = 0> static void opt_in_smem() {
        static std::mutex mu;
        static std::vector<char> done;
        const size_t sm = fused_smem_bytes<R, CPL>(kThreads);
        if (sm <= 40 * 1024) return;   // the static shared memory counts too
        int dev = 0;
        HP_CK(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lock(mu);
        if (done.size() <= size_t(dev)) done.resize(size_t(dev) + 1, 0);
        if (!done[size_t(dev)]) {
            HP_CK(cudaFuncSetAttribute(k_fused_step<R, kThreads, INF, MAP, CPL, INFL, SCH>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
            done[size_t(dev)] = 1;
        }
    }
    template <int INF, int CPL> void opt_in_i() {
        opt_in_smem<INF, false, CPL, false>(); opt_in_smem<INF, true, CPL, false>();
        opt_in_smem<INF, false, CPL, true>(); opt_in_smem<INF, true, CPL, true>();
        opt_in_smem<INF, false, CPL, true, 1>(); opt_in_smem<INF, true, CPL, true, 1>();
    }
    template <int CPL> void opt_in_t() { opt_in_i<0, CPL>(); opt_in_i<1, CPL>(); opt_in_i<2, CPL>(); }
    void opt_in() { opt_in_t<1>(); opt_in_t<2>(); }

    template <int INF, bool MAP, int CPL, bool INFL, int SCH = 0> void launch_one(const FusedArgs<R>& a) {
        const size_t sm = fused_smem_bytes<R, CPL>(kThreads);
        k_fused_step<R, kThreads, INF, MAP, CPL, INFL, SCH><<<a.n_ctas, kThreads, sm, st()>>>(a);
    }
    template <int INF, int CPL> void launch_i(const FusedArgs<R>& a) {
        const bool map = rain.n_maps > 0, infl = bc_kernel();
        if (ctx->p.flag_numerical_scheme != 1) {   // schemes 2/3: the general (boundary-cell) variant
            if (map) launch_one<INF, true, CPL, true, 1>(a); else launch_one<INF, false, CPL, true, 1>(a);
            return;
        }
        if (map) {
            if (infl) launch_one<INF, true, CPL, true>(a); else launch_one<INF, true, CPL, false>(a);
        } else {
            if (infl) launch_one<INF, false, CPL, true>(a); else launch_one<INF, false, CPL, false>(a);
        }
    }
    template <int CPL> void launch_fused_t(const FusedArgs<R>& a) {
        switch (inf_mode()) {
            case 1: launch_i<1, CPL>(a); break;
            case 2: launch_i<2, CPL>(a); break;
            default: launch_i<0, CPL>(a);
        }
    }
    void launch_fused(const FusedArgs<R>& a) {
        if (cells_per_lane == 2) launch_fused_t<2>(a);
        else launch_fused_t<1>(a);
    }

    // the fused kernel variant with boundary-condition cells (inflow, stage, structures)
    bool bc_kernel() const { return inflow.n_gauges > 0 || inflow.n_stage > 0 || strct.n > 0 || hz_on; }

    // Velocity and hazard maxima (velocities.vmax_final, velocities.hazardmax_final of
    // save_output_maps.m:588-604) tracked by the fused step; on = 1 (re)starts them at zero.
    // Every step must refresh the velocities (time_step_change at most half min_time_step).
    bool hz_on = false;
    Dev<R> vmaxm, hzmaxm;
    hp2d_status set_hazard_tracking(int32_t on) {
        if (on != 0 && on != 1) { ctx->err = "on must be 0 or 1"; return HP2D_INVALID_ARG; }
        if (on && !(2.0 * ctx->p.time_step_change <= ctx->p.min_time_step)) {
            ctx->err = "hazard maps need a velocity refresh every step (time_step_change <= min_time_step / 2)";
            return HP2D_INVALID_ARG;
        }
        if (on) {
            vmaxm.alloc(n);
            hzmaxm.alloc(n);
            fill(vmaxm.p, n, R(0));
            fill(hzmaxm.p, n, R(0));
        }
        hz_on = on != 0;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }

    template <int INF> void struct_prime_t(const FusedArgs<R>& a) {
        if (rain.n_maps > 0) k_struct_prime<R, INF, true><<<1, kThreads, 0, st()>>>(a);
        else k_struct_prime<R, INF, false><<<1, kThreads, 0, st()>>>(a);
    }

    void invalidate_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_steps = 0;
    }

    // Dry-row flags of the fused step ([2][ny][strips of the narrowest layout]): zero is always
    // valid ("not known to hold the dry record"); they are cleared whenever something other
    // than a fused step of the current layout wrote the state buffers.
    Dev<unsigned char> dryf;
    int dry_layout = -1;
    int dry_rows() const { return (ny + 3) & ~3; }
    void reset_dry() {
        if (!dryf.p) dryf.alloc(2 * size_t(dry_rows()) * size_t((nx + 27) / 28));
        HP_CK(cudaMemsetAsync(dryf.p, 0, dryf.n, st()));
    }
    // the launches use the flags only with rows per warp a multiple of 4 up to 128; launches
    // without them do not maintain them, so any change of layout or of flag use clears them
    bool dry_enabled = true;   // hp2d_set_dry_skip
    bool dry_usable(int rpw) const { return dry_enabled && rpw % 4 == 0 && rpw <= 128; }
    int dry_key(int cpl) {
        const int rpw = rpw_chosen ? rows_per_warp : default_rows(cpl);
        return dry_usable(rpw) ? cpl : -cpl;
    }
    void dry_for_layout(int cpl) {
        const int key = dry_key(cpl);
        if (dry_layout != key || !dryf.p) {
            reset_dry();
            dry_layout = key;
        }
    }

    // set by the prologue's scan: a cell of finite elevation holds a non-finite depth
    bool bad_state = false;
    void prologue() {
        dry_for_layout(cells_per_lane);
        if (!dirty) return;
        reset_dry();
        pull_sc();
        hs.skip_clamp = 0;
        hs.counter = 0;
        hs.acc_vmax = hs.acc_cmax = 0;
        hs.acc_rain = hs.acc_inf = hs.acc_out = 0;
        hs.n_finite = 0;
        hs.n_bad0 = 0;
        hs.acc_bad = 0;
        hs.bad_domain = 0;
        push_sc();
        k_skip_flag<R><<<blocks_for(n), kThreads, 0, st()>>>(st4[hs.cur].p, stat.p, ny, nx, rain, ga() ? 1 : 0, res,
                                                           ctx->p.depth_tolerance, ctx->p.arrival_threshold, sc.p,
                                                           own_r0, own_r1 < 0 ? ny : own_r1);
        HP_CK(cudaGetLastError());
        if (inflow.n_gauges || inflow.n_stage) {
            k_inflow_depth<R><<<1, kThreads, 0, st()>>>(inflow, sc.p);
            HP_CK(cudaGetLastError());
        }
        if (strct.n) {   // after the gauge depths and the skip flag it reads
            const FusedArgs<R> a = fused_args();
            switch (inf_mode()) {
                case 1: struct_prime_t<1>(a); break;
                case 2: struct_prime_t<2>(a); break;
                default: struct_prime_t<0>(a);
            }
            HP_CK(cudaGetLastError());
        }
        dirty = false;
        pull_sc();
        bad_state = hs.bad_domain != 0;
    }

    static constexpr int kGraphChunk = 32;

    // the CUDA graph of kGraphChunk fused launches (captured once per context and launch
    // shape; invalidate_graph drops it when an argument it holds changes)
    void ensure_graph(const FusedArgs<R>& a) {
        if (graph) return;
        cudaGraph_t gr;
        HP_CK(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < kGraphChunk; ++s) launch_fused(a);
        HP_CK(cudaStreamEndCapture(st(), &gr));
        HP_CK(cudaGraphInstantiate(&graph, gr, 0));
        HP_CK(cudaGraphDestroy(gr));
        graph_steps = kGraphChunk;
    }

    void launch_steps(int64_t count) {
        FusedArgs<R> a = fused_args();
        int64_t remaining = count;
        if (remaining >= kGraphChunk) {
            ensure_graph(a);
            while (remaining >= graph_steps) {
                HP_CK(cudaGraphLaunch(graph, st()));
                remaining -= graph_steps;
            }
        }
        for (int64_t s = 0; s < remaining; ++s) launch_fused(a);
        HP_CK(cudaGetLastError());
    }

    // `nsteps` accepted steps.  A rejected step halts the remaining launches of the batch; the
    // host then prepares its retry (handle_halt) and launches the steps still missing, until the
    // retries of one step run out.
    hp2d_status fused_steps(int32_t nsteps, cudaEvent_t after = nullptr) {
        if (!static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        if (soil_missing()) { ctx->err = "flag_infiltration=1 needs hp2d_set_soil, =2 hp2d_set_soil_vg"; return HP2D_NOT_READY; }
        if (tb_chosen > 1) return blocked_steps(nsteps, after);
        opt_in();
        prologue();
        if (bad_state) return bad_state_error();
        const int64_t k_target = hs.k + nsteps;
        int64_t todo = nsteps;
        hp2d_status status = HP2D_OK;
        for (;;) {
            launch_steps(todo);
            if (after) HP_CK(cudaEventRecord(after, st()));
            pull_sc();
            if (!hs.halted) break;
            status = handle_halt();
            if (status != HP2D_OK) break;
            todo = k_target - hs.k;
            if (todo <= 0) break;
            prologue();
            if (bad_state) { status = bad_state_error(); break; }
        }
        flush_records();
        return status;
    }

    // ---------------- row slabs of one grid (hp2d_set_owned_rows) ----------------
    // A context that holds one slab of rows of a larger grid plus halo rows that other slabs own:
    // its steps reduce the CFL maxima, ledgers and checks over its own rows only; the caller
    // combines the slabs' maxima (hp2d_step_maxima, hp2d_apply_refresh) and refreshes the halo
    // rows from their owners (hp2d_copy_rows) after every step.
    int own_r0 = 0, own_r1 = -1;   // -1: every row
    bool slab() const { return own_r0 != 0 || (own_r1 >= 0 && own_r1 != ny); }
    hp2d_status set_owned_rows(int32_t r0, int32_t r1) {
        if (r0 < 0 || r1 > ny || r0 >= r1) { ctx->err = "owned rows must satisfy 0 <= row0 < row1 <= ny"; return HP2D_INVALID_ARG; }
        own_r0 = r0;
        own_r1 = r1;
        invalidate_graph();
        dirty = true;
        return HP2D_OK;
    }
    hp2d_status step_maxima(uint64_t* vbits, uint64_t* cbits, int32_t* skip) {
        pull_sc();
        *vbits = hs.last_vbits;
        *cbits = hs.last_cbits;
        if (skip) *skip = hs.skip_clamp;
        return HP2D_OK;
    }
    // the last step's refresh redone with the maxima of every slab (the same arithmetic as the
    // step's own finalize), and the clamp skip of the next step set to every slab's verdict
    hp2d_status apply_refresh(uint64_t vbits, uint64_t cbits, int32_t skip) {
        pull_sc();
        if (hs.last_refreshed) {
            const hp2d_params& p = ctx->p;
            const bool is_d = sizeof(R) == 8;
            const R vR = std::sqrt(R(from_ord(vbits, is_d)));
            const double vm = double(vR);
            double cm = 0.0;
            if (cbits) {
                const R v = R(from_ord(cbits - 1ull, is_d));
                cm = p.flag_adaptive_timestepping == 1 ? double(std::fmax(std::sqrt(v), R(1e-10))) : double(v);
            }
            const double tcr = finalize_dt(vm, cm, res, p.alfa_min, p.alfa_max, p.min_time_step, hs.max_dt,
                                           p.time_step_increments, p.flag_timestep);
            const double t_old = hs.rain_b;   // the clock the step started from
            const int uns = tcr == p.min_time_step;
            hs.unstable += uns - hs.last_unstable;
            hs.last_unstable = uns;
            hs.vmax_last = vm;
            hs.time_step = tcr / 60.0;
            hs.t_min = tcr / 60.0 + t_old;
            hs.t_prev = hs.k - 1 == 1 ? tcr / 60.0 : t_old;
            hs.last_vbits = vbits;
            hs.last_cbits = cbits;
        }
        hs.skip_clamp = skip;
        push_sc();
        return HP2D_OK;
    }
    hp2d_status copy_rows(int32_t row0, int32_t nrows, void* buf, int32_t into_state) {
        if (row0 < 0 || nrows < 0 || row0 + nrows > ny || (nrows > 0 && !buf)) {
            ctx->err = "rows outside the grid";
            return HP2D_INVALID_ARG;
        }
        if (gs2[0].p && inf_mode()) { ctx->err = "row copies carry the state records only (no infiltration)"; return HP2D_UNSUPPORTED_FLAG; }
        pull_sc();
        V4* rows = st4[hs.cur].p + size_t(row0) * nx;
        const size_t bytes = size_t(nrows) * nx * sizeof(V4);
        if (into_state) HP_CK(cudaMemcpyAsync(rows, buf, bytes, cudaMemcpyDefault, st()));
        else HP_CK(cudaMemcpyAsync(buf, rows, bytes, cudaMemcpyDefault, st()));
        HP_CK(cudaStreamSynchronize(st()));
        return HP2D_OK;
    }

    // ---------------- temporal blocking (hp2d_set_temporal_blocking) ----------------
    int tb_k = 1;                 // requested: 1 off, 2..4 steps per block, 0 chosen by hp2d_autotune
    int tb_chosen = 1;            // steps per block in use
    int64_t tb_replay_until = 0;  // steps before this one run one per launch (a replayed block)
    CUtensorMap tb_map[3];        // state buffers 0 and 1, static records
    int tb_map_k = 0;             // K the maps' boxes were made for
    int tb_ntx = 0, tb_nty = 0;

    const char* tb_unsupported() const {
        if (sizeof(R) != 4) return "temporal blocking is built for FP32 contexts";
        if (inf_mode() != 0) return "temporal blocking does not support infiltration";
        if (rain.n_uniform || rain.n_maps) return "temporal blocking does not support rain";
        if (bc_kernel()) return "temporal blocking does not support inflow, stage, control structures or hazard maps";
        if (rec.n_times > 0) return "temporal blocking does not support map records";
        if (ctx->p.flag_numerical_scheme != 1) return "temporal blocking supports flag_numerical_scheme 1";
        return nullptr;
    }
    hp2d_status set_temporal_blocking(int32_t k) {
        if (k < 0 || k > 4) { ctx->err = "steps per block must be 0 (chosen by hp2d_autotune) or 1..4"; return HP2D_INVALID_ARG; }
        if (k != 1 && sizeof(R) != 4) { ctx->err = "temporal blocking is built for FP32 contexts"; return HP2D_UNSUPPORTED_FLAG; }
        tb_k = k;
        use_block_depth(k == 0 ? 1 : k);
        return HP2D_OK;
    }
    void use_block_depth(int k) {
        tb_chosen = k;
        pull_sc();
        hs.refresh_every = k;
        push_sc();
        invalidate_graph();
        dirty = true;   // the dry flags are not kept while blocks run
    }
    template <int K> void tb_launch_k(const FusedArgs<R>& a0) {
        if constexpr (sizeof(R) == 4) {
            using G = TbGeom<K>;
            static std::mutex mu;
            static std::vector<char> done;
            {
                int dev = 0;
                HP_CK(cudaGetDevice(&dev));
                std::lock_guard<std::mutex> lock(mu);
                if (done.size() <= size_t(dev)) done.resize(size_t(dev) + 1, 0);
                if (!done[size_t(dev)]) {
                    HP_CK(cudaFuncSetAttribute(k_tb_block<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(G::smem)));
                    done[size_t(dev)] = 1;
                }
            }
            if (tb_map_k != K) {
                if (!record_map(&tb_map[0], st4[0].p, ny, nx, G::EX, G::EY) ||
                    !record_map(&tb_map[1], st4[1].p, ny, nx, G::EX, G::EY) ||
                    !record_map(&tb_map[2], stat.p, ny, nx, G::EX, G::EY))
                    throw std::runtime_error("cuTensorMapEncodeTiled rejected the record arrays");
                tb_map_k = K;
            }
            FusedArgs<float> a = a0;
            tb_ntx = (nx + kTbTX - 1) / kTbTX;
            tb_nty = (ny + kTbTY - 1) / kTbTY;
            a.n_ctas = unsigned(tb_ntx * tb_nty);
            k_tb_block<K><<<a.n_ctas, kTbThreads, G::smem, st()>>>(a, tb_map[0], tb_map[1], tb_map[2], tb_ntx);
        }
    }
    void tb_launch(const FusedArgs<R>& a, int k) {
        if (k == 2) tb_launch_k<2>(a);
        else if (k == 3) tb_launch_k<3>(a);
        else tb_launch_k<4>(a);
    }
    // nsteps accepted steps with blocks of tb_chosen steps where the step counter is aligned
    // (a block starts at a step k with (k - 2) % K == 0, so that its last step is a refresh step)
    // and single launches elsewhere; a block that cannot be committed is replayed step by step
    hp2d_status blocked_steps(int32_t nsteps, cudaEvent_t after) {
        if (const char* why = tb_unsupported()) { ctx->err = why; return HP2D_UNSUPPORTED_FLAG; }
        opt_in();
        prologue();
        if (bad_state) return bad_state_error();
        const int K = tb_chosen;
        const int64_t k_target = hs.k + nsteps;
        hp2d_status status = HP2D_OK;
        for (;;) {
            const FusedArgs<R> a = fused_args();
            int64_t k = hs.k;
            while (k < k_target) {
                if (k >= tb_replay_until && k >= 2 && (k - 2) % K == 0 && k_target - k >= K) {
                    tb_launch(a, K);
                    k += K;
                } else {
                    launch_fused(a);
                    k += 1;
                }
            }
            HP_CK(cudaGetLastError());
            if (after) HP_CK(cudaEventRecord(after, st()));
            pull_sc();
            if (!hs.halted) break;
            status = handle_halt();
            if (status != HP2D_OK) break;
            if (k_target - hs.k <= 0) break;
            prologue();
            if (bad_state) { status = bad_state_error(); break; }
        }
        flush_records();
        return status;
    }

    // ---------------- failure handling (HydroPol2D_Main_While.m:926-993) ----------------
    int max_retries = 8;              // attempts of one step rejected before the call fails
    double factor_reduction = 2.0;    // running_control.factor_reduction (input_data_script.m:486)
    unsigned int wait_polls = 1u << 22;
    int64_t rej_k = -1;               // step whose attempts were rejected last, and how often
    int rej_n = 0;

    hp2d_status bad_state_error() {
        ctx->err = "the state holds a non-finite depth in a cell of finite elevation (only idx_nan cells, of NaN "
                   "elevation, may hold NaN); nothing was stepped";
        return HP2D_NUMERICAL;
    }

    // The launches halted: a row copy timed out (the step was rejected), the refreshed dt hit
    // the floor with dt_floor_stop on (the step was kept), or a step was rejected for its
    // depths.  The last is retried as the reference's catch block does: the attempt's state is
    // already the rolled-back one (d_t = d_p, I_t = I_p: the buffer the attempt read), the clock
    // goes back by the attempt's step, catch_index grows, the new step is
    //   factor * alfa_min * dx / c,  factor = 1 / catch_index / factor_reduction,
    //   c = sqrt(g max(max(d_tot), max(d_p)))  (+ the last refresh's maximum velocity when
    //   flag_adaptive_timestepping = 0, for the reference's velocity-raster maximum),
    // max_time_step drops to min(1.5 x new step, max_time_step), the new step is capped by it
    // (an infinite one becomes min_time_step), the clock advances by it and the rain interval
    // becomes [rewound clock, new clock] (update_spatial_BC after the catch).
    hp2d_status handle_halt() {
        if (hs.status & kStatusDtFloor) {   // a kept step
            hs.status &= ~kStatusDtFloor;
            hs.halted = 0;
            push_sc();
            ctx->err = "the refreshed time step reached min_time_step (refreshing_timestep.m:357-359) at step " +
                       std::to_string(hs.k - 1) + "; that step was kept";
            return HP2D_DT_FLOOR;
        }
        // a rejected step: take back its arrival marks and find max(d_p, d_tot) for the retry
        hs.retry_dmax = 0ull;
        push_sc();
        {
            // the launch marked arrivals with the times of at most tb_chosen steps from the clock
            const FusedArgs<R> a = fused_args();
            const double dts = hs.time_step * 60.0;
            double t = hs.t_min;
            const R lo = R(t * 60.0 + dts);
            for (int q = 1; q < std::max(tb_chosen, 1); ++q) t = dts / 60.0 + t;
            const R hi = R(t * 60.0 + dts);
            k_retry_scan<R><<<blocks_for(n), kThreads, 0, st()>>>(a, inf_mode(), lo, hi);
            HP_CK(cudaGetLastError());
        }
        pull_sc();
        if (hs.status & kStatusTbReplay) {   // a block of temporal blocking: its steps one by one
            hs.status &= ~kStatusTbReplay;
            hs.halted = 0;
            tb_replay_until = hs.k + tb_chosen;
            push_sc();
            dirty = true;
            return HP2D_OK;
        }
        if (hs.status & kStatusTimeout) {
            hs.status &= ~kStatusTimeout;
            hs.halted = 0;
            push_sc();
            dirty = true;
            ctx->err = "a row copy into shared memory did not complete within its wait limit; that step was "
                       "rejected and the state is the last accepted one";
            return HP2D_TIMEOUT;
        }
        if (hs.k == rej_k) ++rej_n;
        else { rej_k = hs.k; rej_n = 1; }
        if (rej_n > max_retries) {
            hs.halted = 0;
            push_sc();
            dirty = true;
            ctx->err = "step " + std::to_string(hs.k) + " was rejected " + std::to_string(rej_n) +
                       " times (a depth went non-finite or below -depth_tolerance); the state is the last accepted one";
            rej_n = 0;
            return HP2D_NUMERICAL;
        }
        const double dmx = from_ord(hs.retry_dmax, sizeof(R) == 8);
        const double wc = std::sqrt(kG * dmx);
        const hp2d_params& p = ctx->p;
        hs.catch_index += 1;
        const double factor = 1.0 / hs.catch_index / factor_reduction;
        double nt = p.flag_adaptive_timestepping == 1 ? factor * (p.alfa_min * res / wc)
                                                      : factor * (p.alfa_min * res / (hs.vmax_last + wc));
        if (hs.catch_index > 1) hs.max_dt = std::fmin(nt * 1.5, hs.max_dt);
        nt = std::fmin(nt, hs.max_dt);
        if (std::isinf(nt)) nt = p.min_time_step;
        const double t0 = hs.t_min - hs.time_step;
        hs.t_prev = t0;
        hs.time_step = nt / 60.0;
        hs.t_min = t0 + hs.time_step;
        hs.rain_a = hs.t_prev;
        hs.rain_b = hs.t_min;
        hs.halted = 0;
        hs.retries += 1;
        push_sc();
        dirty = true;
        return HP2D_OK;
    }

    hp2d_status set_retry_policy(int32_t retries, double factor, int32_t dt_floor_is_error) {
        if (retries < 0 || !(factor > 0) || (dt_floor_is_error != 0 && dt_floor_is_error != 1)) {
            ctx->err = "max_retries >= 0, factor_reduction > 0 and dt_floor_is_error 0 or 1";
            return HP2D_INVALID_ARG;
        }
        max_retries = retries;
        factor_reduction = factor;
        pull_sc();
        hs.dt_floor_stop = dt_floor_is_error;
        push_sc();
        return HP2D_OK;
    }
    hp2d_status inject_fault(int64_t k, int32_t attempts) {
        if (attempts < 0) { ctx->err = "attempts must be >= 0"; return HP2D_INVALID_ARG; }
        pull_sc();
        hs.fault_k = k;
        hs.fault_n = attempts;
        push_sc();
        return HP2D_OK;
    }

    hp2d_status fused_steps_timed(int32_t nsteps, float* ms) {
        if (!static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        prologue();
        if (nsteps >= kGraphChunk && !soil_missing()) {   // set-up, not a step: outside the timed region
            opt_in();
            ensure_graph(fused_args());
        }
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

    // ---------------- autotuning ----------------
    // Copies of everything a fused step writes, so that trial steps can be undone.
    struct Snapshot {
        Dev<V4> st[2];
        Dev<V2> gs[2];
        Dev<R> arr, hf3s, qos;
        Dev<StepScalars> scs;
    };
    template <typename T> void copy_dev(T* dst, const T* src, size_t count) {
        if (count) HP_CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice, st()));
    }
    void take(Snapshot& s) {
        for (int b = 0; b < 2; ++b) {
            s.st[b].alloc(n);
            copy_dev(s.st[b].p, st4[b].p, n);
            if (gs2[b].p) { s.gs[b].alloc(n); copy_dev(s.gs[b].p, gs2[b].p, n); }
        }
        s.arr.alloc(n);
        copy_dev(s.arr.p, arrival.p, n);
        if (n_out) {
            s.hf3s.alloc(n_out); copy_dev(s.hf3s.p, hf3.p, n_out);
            s.qos.alloc(n_out); copy_dev(s.qos.p, qo.p, n_out);
        }
        s.scs.alloc(1);
        copy_dev(s.scs.p, sc.p, 1);
        reset_dry();   // trial layouts may differ from the current one
        HP_CK(cudaStreamSynchronize(st()));
    }
    void put_back(const Snapshot& s) {
        for (int b = 0; b < 2; ++b) {
            copy_dev(st4[b].p, s.st[b].p, n);
            if (gs2[b].p) copy_dev(gs2[b].p, s.gs[b].p, n);
        }
        copy_dev(arrival.p, s.arr.p, n);
        if (n_out) { copy_dev(hf3.p, s.hf3s.p, n_out); copy_dev(qo.p, s.qos.p, n_out); }
        copy_dev(sc.p, s.scs.p, 1);
        reset_dry();
        HP_CK(cudaStreamSynchronize(st()));
        pull_sc();
    }

    // Times `trial` fused steps per launch shape (rows each warp streams) from the current
    // state, undoes them, and keeps the fastest shape.  Results never depend on the shape.
    hp2d_status autotune(int32_t trial, int32_t* chosen) {
        if (!static_ready) { ctx->err = "hp2d_upload_static not called"; return HP2D_NOT_READY; }
        if (soil_missing()) { ctx->err = "flag_infiltration=1 needs hp2d_set_soil, =2 hp2d_set_soil_vg"; return HP2D_NOT_READY; }
        opt_in();
        prologue();
        Snapshot snap;
        take(snap);
        const int cands[] = {16, 24, 32, 40, 44, 48, 56, 64, 96, 128};
        if (!rpw_chosen) rows_per_warp = default_rows(cells_per_lane);
        rpw_chosen = true;
        const int keep = rows_per_warp, keep_cpl = cells_per_lane;
        int best = keep, best_cpl = keep_cpl;
        float best_ms = std::numeric_limits<float>::infinity();
        bool timed_out = false;
        cudaEvent_t e0, e1;
        HP_CK(cudaEventCreate(&e0));
        HP_CK(cudaEventCreate(&e1));
        for (int cpl = 1; cpl <= 2; ++cpl)
        for (int c : cands) {
            if (c > std::max(ny, 4) && c != 16) continue;
            rows_per_warp = c;
            cells_per_lane = cpl;
            const FusedArgs<R> a = fused_args();
            launch_fused(a);   // warm-up
            HP_CK(cudaEventRecord(e0, st()));
            for (int s = 0; s < trial; ++s) launch_fused(a);
            HP_CK(cudaEventRecord(e1, st()));
            HP_CK(cudaGetLastError());
            HP_CK(cudaEventSynchronize(e1));
            float ms = 0;
            HP_CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best_ms) { best_ms = ms; best = c; best_cpl = cpl; }
            pull_sc();
            timed_out = timed_out || (hs.status & kStatusTimeout) != 0;
            put_back(snap);
        }
        rows_per_warp = best;
        cells_per_lane = best_cpl;
        // temporal blocking left to the tuner: blocks of 2, 3 and 4 steps against single steps,
        // per step (the state is put back after each trial; the blocks' results differ from the
        // single steps' by the frozen time step, which the caller accepted with steps_per_block 0)
        if (tb_k == 0 && !tb_unsupported() && !timed_out) {
            int best_k = 1;
            float best_step = best_ms / float(std::max(trial, 1));
            const FusedArgs<R> a = fused_args(best_cpl);
            for (int kb = 2; kb <= 4; ++kb) {
                tb_chosen = kb;
                tb_launch(a, kb);   // warm-up
                HP_CK(cudaEventRecord(e0, st()));
                for (int s = 0; s < trial; ++s) tb_launch(a, kb);
                HP_CK(cudaEventRecord(e1, st()));
                HP_CK(cudaGetLastError());
                HP_CK(cudaEventSynchronize(e1));
                float ms = 0;
                HP_CK(cudaEventElapsedTime(&ms, e0, e1));
                pull_sc();
                timed_out = timed_out || (hs.status & kStatusTimeout) != 0;
                put_back(snap);
                const float per = ms / float(std::max(trial, 1) * kb);
                if (per < best_step) { best_step = per; best_k = kb; }
            }
            use_block_depth(best_k);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        invalidate_graph();
        if (timed_out) { ctx->err = "a row copy did not complete within its wait limit"; return HP2D_TIMEOUT; }
        if (chosen) *chosen = best;
        return HP2D_OK;
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
    // A field goes to the caller's FP64 array in one copy: a kernel converts it (one component of
    // the state records, or a plain array, times `scale`) into this context's FP64 read-back
    // buffer, allocated on the first read-back and kept, and one cudaMemcpyAsync moves it to the
    // caller's memory (page-locked memory is read at the full link rate).  Nothing is shared
    // between contexts.
    Dev<double> rb;
    double* readback_buffer() {
        if (rb.n != n) rb.alloc(n);
        return rb.p;
    }
    void copy_out(const double* dev, double* out) {
        HP_CK(cudaGetLastError());
        stage.copy(const_cast<double*>(dev), out, n * sizeof(double), false, st(), ctx->device);
    }
    void fetch_scaled(const R* src, double scale, double* out) {
        double* d = readback_buffer();
        k_scaled_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, src, scale, d);
        copy_out(d, out);
    }
    void fetch_component_scaled(int comp, double scale, double* out) {
        pull_sc();
        double* d = readback_buffer();
        k_state_component_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[hs.cur].p, comp, scale, d);
        copy_out(d, out);
    }


    hp2d_status download(int32_t field, double* out, size_t count) {
        if (count != n) { ctx->err = "count must be ny*nx"; return HP2D_INVALID_ARG; }
        const double to_mmh = 3.6e6 / res;
        auto per_outlet_map = [&](const Dev<R>& src, double scale_) {
            std::fill(out, out + n, 0.0);
            if (!n_out) return;
            auto cells = fetch(outlet_cells.p, size_t(n_out));
            auto v = fetch(src.p, size_t(n_out));
            for (int o = 0; o < n_out; ++o) out[cells[o]] = double(v[o]) * scale_;
        };
        switch (field) {
            case HP2D_FIELD_DEPTH: fetch_component_scaled(0, 1000.0, out); break;
            case HP2D_FIELD_QOUT_RIGHT: fetch_component_scaled(1, to_mmh, out); break;
            case HP2D_FIELD_QOUT_UP: fetch_component_scaled(2, to_mmh, out); break;
            case HP2D_FIELD_QOUT_LEFT: case HP2D_FIELD_QOUT_DOWN: {
                pull_sc();
                double* d = readback_buffer();
                k_shifted_flux_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(ny, nx, st4[hs.cur].p,
                                                                            field == HP2D_FIELD_QOUT_DOWN, to_mmh, d);
                copy_out(d, out);
                break;
            }
            case HP2D_FIELD_OUTLET_FLOW: per_outlet_map(qo, 3.6e6); break;
            case HP2D_FIELD_HF_X: case HP2D_FIELD_HF_Y: {
                if (!(last_dt_s > 0)) { ctx->err = "Hf is materialised by hp2d_li_step only"; return HP2D_NOT_READY; }
                fetch_scaled(field == HP2D_FIELD_HF_X ? hfx.p : hfy.p, 1.0, out);
                break;
            }
            case HP2D_FIELD_HF_OUTLET: per_outlet_map(hf3, 1.0); break;
            case HP2D_FIELD_DMAX: fetch_component_scaled(3, 1000.0, out); break;
            case HP2D_FIELD_ARRIVAL: {
                double* d = readback_buffer();
                k_divided_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, arrival.p, 60.0, d);
                copy_out(d, out);
                break;
            }
            case HP2D_FIELD_VMAX: case HP2D_FIELD_HAZARD_MAX: {
                if (!hz_on) { ctx->err = "velocity / hazard maxima are off (hp2d_set_hazard_tracking)"; return HP2D_NOT_READY; }
                fetch_scaled(field == HP2D_FIELD_VMAX ? vmaxm.p : hzmaxm.p, 1.0, out);
                break;
            }
            case HP2D_FIELD_SOIL_STORAGE: {
                if (!gs2[0].p) { ctx->err = "no soil storage (hp2d_set_soil not called)"; return HP2D_NOT_READY; }
                pull_sc();
                double* d = readback_buffer();
                k_soil_component_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, gs2[hs.cur].p, 1000.0, d);
                copy_out(d, out);
                break;
            }
            case HP2D_FIELD_I_TOT_END_CELL: {
                pull_sc();
                const double dts = last_dt_s > 0 ? last_dt_s : hs.time_step * 60.0;
                double* d = readback_buffer();
                k_itot_f64<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[hs.cur].p, stat.p, qo.p, to_mmh, dts, res, d);
                copy_out(d, out);
                break;
            }
            default: ctx->err = "unknown field"; return HP2D_INVALID_ARG;
        }
        return HP2D_OK;
    }

    hp2d_status download_native(int32_t field, void* out, size_t bytes) {
        size_t cnt = (field == 9 || field == 10) ? size_t(n_out) : n;
        if (bytes != cnt * sizeof(R)) { ctx->err = "byte count mismatch"; return HP2D_INVALID_ARG; }
        R* o = static_cast<R*>(out);
        switch (field) {
            case 0: case 1: case 2: case 5: {   // one component, gathered on the device
                pull_sc();
                R* d = reinterpret_cast<R*>(readback_buffer());
                k_state_component<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[hs.cur].p, field == 5 ? 3 : field, d);
                HP_CK(cudaGetLastError());
                HP_CK(cudaMemcpyAsync(o, d, n * sizeof(R), cudaMemcpyDeviceToHost, st()));
                HP_CK(cudaStreamSynchronize(st()));
                break;
            }
            case 3: case 4: {
                if (!gs2[0].p) { ctx->err = "no soil records"; return HP2D_NOT_READY; }
                pull_sc();
                auto v = fetch(gs2[hs.cur].p, n);
                for (size_t k = 0; k < n; ++k) o[k] = field == 3 ? v[k].x : v[k].y;
                break;
            }
            case 6: { auto v = fetch(arrival.p, n); std::copy(v.begin(), v.end(), o); break; }
            case 7: case 8: {
                if (!hfx.p) { ctx->err = "Hf is materialised by hp2d_li_step only"; return HP2D_NOT_READY; }
                auto v = fetch(field == 7 ? hfx.p : hfy.p, n);
                std::copy(v.begin(), v.end(), o);
                break;
            }
            case 9: case 10: {
                auto v = fetch(field == 9 ? hf3.p : qo.p, cnt);
                std::copy(v.begin(), v.end(), o);
                break;
            }
            default: ctx->err = "unknown native field"; return HP2D_INVALID_ARG;
        }
        return HP2D_OK;
    }

    hp2d_status diag(hp2d_diag* o) {
        pull_sc();
        o->t = hs.t_min;
        o->time_step = hs.time_step;
        o->k = hs.k;
        o->rain_t0 = hs.rain_a;
        o->rain_t1 = hs.rain_b;
        o->t_previous = hs.t_prev;
        o->inflow_volume = hs.inflow_vol;
        o->stage_volume = hs.stage_vol;
        o->structure_volume = hs.struct_vol;
        o->skipped_cells = int64_t(hs.skipped_cells);
        o->skipped_read_cells = int64_t(hs.skipped_read_cells);
        o->max_velocity = hs.vmax_last;
        o->rain_volume = hs.rain_vol;
        o->infiltration_volume = hs.inf_vol;
        o->outlet_volume = hs.out_vol;
        o->neg_depth_warnings = hs.neg_warn;
        o->unstable_steps = hs.unstable;
        o->status_bits = hs.status;
        o->retries = hs.retries;
        o->catch_index = hs.catch_index;
        o->steps_per_block = tb_chosen;
        o->max_time_step = hs.max_dt;
        return HP2D_OK;
    }

    hp2d_status stored_volume(double* v) {
        pull_sc();
        HP_CK(cudaMemsetAsync(vol.p, 0, sizeof(double), st()));
        k_volume4<R><<<blocks_for(n), kThreads, 0, st()>>>(n, st4[hs.cur].p, vol.p);
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


}  // namespace

// Batched ensemble: FP32 member contexts on one device advanced together, one persistent
// launch per step (k_ens_plan + k_ens_step), chunks of steps captured in a CUDA graph.
struct hp2d_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<hp2d_ctx*> members;
    Dev<FusedArgs<float>> args;
    Dev<unsigned> prefix;
    Dev<EnsQueue> queue;
    int rows_per_warp = 32;
    int cells_per_lane = 2;   // layout of the streamed strips (as hp2d_set_layout)
    int ga = -1, map = -1;
    bool infl = false;   // some member has inflow hydrographs
    int sch = 0;         // members' faces: 0 Bates, 1 schemes 2/3 (members agree on the kind)
    int grid_for[3][3] = {};
    cudaGraphExec_t graph = nullptr;
    int graph_members = -1, graph_rpw = -1, graph_cpl = -1, graph_kind = -1;
    // the kernel variant a captured graph launches
    int kind() const { return sch * 16 + ga * 4 + map * 2 + (infl ? 1 : 0); }

    Impl<float>& impl(int m) { return *static_cast<Impl<float>*>(members[m]->impl.get()); }

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }

    template <int INF, bool MAP, int CPL, bool INFL, int SCH = 0> void launch_t(int nm) {
        const size_t smem = fused_smem_bytes<float, CPL>(kThreads);
        int& grid = grid_for[CPL][INFL ? 1 + SCH : 0];
        if (grid == 0) {
            int per_sm = 0, sms = 0;
            HP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_ens_step<float, kThreads, INF, MAP, CPL, INFL, SCH>, kThreads, smem));
            HP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
            grid = std::max(1, per_sm) * sms;
        }
        k_ens_plan<float><<<1, 1024, 0, stream>>>(args.p, nm, prefix.p, queue.p);
        k_ens_step<float, kThreads, INF, MAP, CPL, INFL, SCH><<<grid, kThreads, smem, stream>>>(args.p, nm, prefix.p,
                                                                                             queue.p);
    }
    template <int INF, int CPL> void launch_m(int nm) {
        if (sch) {
            if (map) launch_t<INF, true, CPL, true, 1>(nm); else launch_t<INF, false, CPL, true, 1>(nm);
            return;
        }
        if (map) {
            if (infl) launch_t<INF, true, CPL, true>(nm); else launch_t<INF, true, CPL, false>(nm);
        } else {
            if (infl) launch_t<INF, false, CPL, true>(nm); else launch_t<INF, false, CPL, false>(nm);
        }
    }
    template <int CPL> void launch_c(int nm) {
        if (ga == 1) launch_m<1, CPL>(nm);
        else if (ga == 2) launch_m<2, CPL>(nm);
        else launch_m<0, CPL>(nm);
    }
    void launch(int nm) {
        if (cells_per_lane == 2) launch_c<2>(nm);
        else launch_c<1>(nm);
    }

    // members' pending work done, their first-step prologues run, argument table current
    hp2d_status prepare() {
        const int nm = int(members.size());
        if (nm == 0) { err = "the ensemble has no members"; return HP2D_NOT_READY; }
        std::vector<FusedArgs<float>> host(nm);
        for (int m = 0; m < nm; ++m) {
            Impl<float>& im = impl(m);
            if (!im.static_ready) { err = "member " + std::to_string(m) + ": hp2d_upload_static not called"; return HP2D_NOT_READY; }
            if (im.soil_missing()) {
                err = "member " + std::to_string(m) + ": its infiltration model needs its soil tables";
                return HP2D_NOT_READY;
            }
            const int mga = im.inf_mode(), mmap = im.rain.n_maps > 0 ? 1 : 0;
            const int msch = members[m]->p.flag_numerical_scheme != 1 ? 1 : 0;
            if (m == 0) { ga = mga; map = mmap; infl = false; sch = msch; }
            if (im.bc_kernel()) infl = true;
            if (mga != ga || mmap != map) {
                err = "members must agree on the infiltration model and on the kind of rain forcing";
                return HP2D_INVALID_ARG;
            }
            if (msch != sch) {
                err = "members must agree on Bates (flag_numerical_scheme 1) against the schemes 2/3";
                return HP2D_INVALID_ARG;
            }
            HP_CK(cudaSetDevice(device));
            if (im.rows_per_warp != rows_per_warp || !im.rpw_chosen) {
                im.rows_per_warp = rows_per_warp;
                im.rpw_chosen = true;
                im.invalidate_graph();
            }
            im.prologue();
            if (im.bad_state) {
                err = "member " + std::to_string(m) + ": " + (im.bad_state_error(), members[m]->err);
                return HP2D_NUMERICAL;
            }
            im.dry_for_layout(cells_per_lane);   // the ensemble's layout may differ from the member's
            HP_CK(cudaStreamSynchronize(im.st()));
            host[m] = im.fused_args(cells_per_lane);
        }
        // a captured graph holds these pointers: reallocate (and recapture) only on a size change
        if (args.n != size_t(nm)) {
            drop_graph();
            args.alloc(size_t(nm));
            prefix.alloc(size_t(nm) + 1);
        }
        HP_CK(cudaMemcpyAsync(args.p, host.data(), host.size() * sizeof(FusedArgs<float>), cudaMemcpyHostToDevice, stream));
        if (!queue.p) queue.alloc(1);
        HP_CK(cudaStreamSynchronize(stream));
        return HP2D_OK;
    }

    static constexpr int kChunk = 32;

    // the CUDA graph of kChunk launches for the current members and launch shape
    void ensure_graph(int nm) {
        if (graph && (graph_members != nm || graph_rpw != rows_per_warp || graph_cpl != cells_per_lane ||
                      graph_kind != kind())) drop_graph();
        if (graph) return;
        cudaGraph_t gr;
        HP_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < kChunk; ++k) launch(nm);
        HP_CK(cudaStreamEndCapture(stream, &gr));
        HP_CK(cudaGraphInstantiate(&graph, gr, 0));
        HP_CK(cudaGraphDestroy(gr));
        graph_members = nm;
        graph_rpw = rows_per_warp;
        graph_cpl = cells_per_lane;
        graph_kind = kind();
    }

    // `after` (optional) is recorded once the launches and the plan pass are queued, before
    // the host reads the members' clocks back
    hp2d_status steps(int32_t nsteps, int32_t* n_active, cudaEvent_t after = nullptr) {
        hp2d_status s = prepare();
        if (s != HP2D_OK) return s;
        const int nm = int(members.size());
        int remaining = nsteps;
        if (remaining >= kChunk) {
            ensure_graph(nm);
            while (remaining >= kChunk) {
                HP_CK(cudaGraphLaunch(graph, stream));
                remaining -= kChunk;
            }
        }
        for (int k = 0; k < remaining; ++k) launch(nm);
        HP_CK(cudaGetLastError());
        // one more plan pass counts the members still running after these steps
        k_ens_plan<float><<<1, 1024, 0, stream>>>(args.p, nm, prefix.p, queue.p);
        if (after) HP_CK(cudaEventRecord(after, stream));
        EnsQueue q{};
        HP_CK(cudaMemcpyAsync(&q, queue.p, sizeof(q), cudaMemcpyDeviceToHost, stream));
        HP_CK(cudaStreamSynchronize(stream));
        for (int m = 0; m < nm; ++m) {
            impl(m).pull_sc();
            impl(m).flush_records();
        }
        unsigned retried = 0;
        for (int m = 0; m < nm; ++m) {   // a rejected member step: its retry, as on its own
            Impl<float>& im = impl(m);
            if (!im.hs.halted || (im.hs.status & kStatusTimeout)) continue;
            const hp2d_status s = im.handle_halt();
            if (s != HP2D_OK) {
                err = "member " + std::to_string(m) + ": " + members[m]->err;
                return s;
            }
            ++retried;   // halted members were not counted as running
        }
        if (n_active) *n_active = int32_t(q.n_active + retried);
        if (q.stalled) {
            err = std::to_string(q.stalled) + " member(s) stopped: a row copy did not complete within its wait limit";
            return HP2D_TIMEOUT;
        }
        return HP2D_OK;
    }

    hp2d_status run(int64_t max_steps, int64_t* launches) {
        int64_t done = 0;
        int32_t active = 1;
        while (active > 0 && (max_steps <= 0 || done < max_steps)) {
            const int64_t left = max_steps > 0 ? max_steps - done : int64_t(1) << 40;
            const int32_t chunk = int32_t(std::min<int64_t>(left, 256));
            hp2d_status s = steps(chunk, &active);
            if (s != HP2D_OK) return s;
            done += chunk;
        }
        if (launches) *launches = done;
        return HP2D_OK;
    }

    // every member's state copied aside, trial steps per launch shape, state put back
    hp2d_status autotune(int32_t trial, int32_t* chosen) {
        const int cands[] = {8, 16, 24, 32, 48, 64};
        const int nm = int(members.size());
        std::vector<std::unique_ptr<Impl<float>::Snapshot>> snaps;
        hp2d_status s = prepare();
        if (s != HP2D_OK) return s;
        for (int m = 0; m < nm; ++m) {
            snaps.emplace_back(new Impl<float>::Snapshot());
            impl(m).take(*snaps.back());
        }
        const int keep = rows_per_warp, keep_cpl = cells_per_lane;
        int best = keep, best_cpl = keep_cpl;
        float best_ms = std::numeric_limits<float>::infinity();
        cudaEvent_t e0, e1;
        HP_CK(cudaEventCreate(&e0));
        HP_CK(cudaEventCreate(&e1));
        bool stalled = false;
        for (int cpl = 1; cpl <= 2; ++cpl)
        for (int c : cands) {
            rows_per_warp = c;
            cells_per_lane = cpl;
            s = prepare();
            if (s != HP2D_OK) break;
            launch(nm);   // warm-up
            HP_CK(cudaEventRecord(e0, stream));
            for (int k = 0; k < trial; ++k) launch(nm);
            HP_CK(cudaEventRecord(e1, stream));
            HP_CK(cudaGetLastError());
            HP_CK(cudaEventSynchronize(e1));
            float ms = 0;
            HP_CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best_ms) { best_ms = ms; best = c; best_cpl = cpl; }
            for (int m = 0; m < nm; ++m) {
                impl(m).pull_sc();
                stalled = stalled || (impl(m).hs.status & kStatusTimeout) != 0;
                impl(m).put_back(*snaps[m]);
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        rows_per_warp = best;
        cells_per_lane = best_cpl;
        drop_graph();
        if (s != HP2D_OK) return s;
        if (stalled) { err = "a row copy did not complete within its wait limit"; return HP2D_TIMEOUT; }
        if (chosen) *chosen = best;
        return prepare();
    }
};

namespace {
template <typename F> hp2d_status ens_guarded(hp2d_ensemble* e, F&& fn) {
    if (!e) return HP2D_INVALID_ARG;
    try {
        HP_CK(cudaSetDevice(e->device));
        return fn();
    } catch (const CudaFail& f) {
        e->err = std::string(f.what) + ": " + cudaGetErrorString(f.e);
        return HP2D_CUDA_ERROR;
    } catch (const std::exception& ex) {
        e->err = ex.what();
        return HP2D_INVALID_ARG;
    }
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
    if (p.flag_reservoir != 0 && p.flag_reservoir != 1) { g_create_error = "flag_reservoir must be 0 or 1"; return HP2D_INVALID_ARG; }
    if (p.flag_numerical_scheme < 1 || p.flag_numerical_scheme > 3) { g_create_error = "flag_numerical_scheme must be 1 (Bates), 2 (s-upwind) or 3 (s-centred)"; return HP2D_UNSUPPORTED_FLAG; }
    if (p.flag_infiltration < 0 || p.flag_infiltration > 2) { g_create_error = "flag_infiltration must be 0, 1 (Green-Ampt) or 2 (van Genuchten)"; return HP2D_UNSUPPORTED_FLAG; }
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
            ctx->impl.reset(new Impl<float>(ctx));
        } else {
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

hp2d_status hp2d_set_soil_vg(hp2d_ctx* ctx, const uint8_t* soil_class, int32_t n_classes, const double* theta_r,
                             const double* theta_sat, const double* n_vg, const double* alpha_vg, const double* ksat,
                             const double* soil_depth, const double* gw_head, double l_vg, double Ltop, double dh_max,
                             double ksurf_weight) {
    if (!soil_class || !theta_r || !theta_sat || !n_vg || !alpha_vg || !ksat || !soil_depth) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        return m.set_soil_vg(soil_class, n_classes, theta_r, theta_sat, n_vg, alpha_vg, ksat, soil_depth, gw_head, l_vg,
                             Ltop, dh_max, ksurf_weight);
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

hp2d_status hp2d_set_inflow(hp2d_ctx* ctx, int32_t n_gauges, int32_t n_times, const double* t_start,
                            const double* rates, int32_t n_cells, const int32_t* rows, const int32_t* cols,
                            const int32_t* gauge) {
    if (n_gauges > 0 && (!t_start || !rates || !rows || !cols || !gauge)) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_inflow(n_gauges, n_times, t_start, rates, n_cells, rows, cols, gauge); });
}

hp2d_status hp2d_set_map_records(hp2d_ctx* ctx, int32_t n_times, const double* time_records, int32_t n_slots) {
    return with_impl(ctx, [&](auto& m) { return m.set_record_target(0, n_times, time_records, n_slots); });
}

hp2d_status hp2d_set_map_records_host(hp2d_ctx* ctx, int32_t n_times, const double* time_records, int32_t n_slots) {
    return with_impl(ctx, [&](auto& m) { return m.set_record_target(1, n_times, time_records, n_slots); });
}

hp2d_status hp2d_map_records(hp2d_ctx* ctx, int64_t* count) {
    if (!count) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.map_records(count); });
}

hp2d_status hp2d_download_map_record(hp2d_ctx* ctx, int64_t index, double* depth_mm, double* t_min) {
    if (!depth_mm) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.download_map_record(index, depth_mm, t_min); });
}

hp2d_status hp2d_set_reservoirs(hp2d_ctx* ctx, int32_t n, const int32_t* res_row, const int32_t* res_col,
                                const double* k1, const double* h1, const double* k2, const int32_t* ds1_row,
                                const int32_t* ds1_col, const double* k3, const double* h2, const double* k4,
                                const int32_t* ds2_row, const int32_t* ds2_col) {
    if (n > 0 && (!res_row || !res_col || !k1 || !h1 || !k2 || !ds1_row || !ds1_col || !k3 || !h2 || !k4 || !ds2_row ||
                  !ds2_col))
        return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        return m.set_reservoirs(n, res_row, res_col, k1, h1, k2, ds1_row, ds1_col, k3, h2, k4, ds2_row, ds2_col);
    });
}

hp2d_status hp2d_set_dry_skip(hp2d_ctx* ctx, int32_t on) {
    if (on != 0 && on != 1) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        m.dry_enabled = on != 0;
        m.invalidate_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_set_hazard_tracking(hp2d_ctx* ctx, int32_t on) {
    return with_impl(ctx, [&](auto& m) { return m.set_hazard_tracking(on); });
}

hp2d_status hp2d_set_stage(hp2d_ctx* ctx, int32_t n_gauges, int32_t n_times, const double* t_start,
                           const double* depth_m, int32_t n_cells, const int32_t* rows, const int32_t* cols,
                           const int32_t* gauge) {
    if (n_gauges > 0 && (!t_start || !depth_m || !rows || !cols || !gauge)) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.set_stage(n_gauges, n_times, t_start, depth_m, n_cells, rows, cols, gauge); });
}

hp2d_status hp2d_set_rain_gauges(hp2d_ctx* ctx, int32_t n_gauges, const double* x_gauge, const double* y_gauge,
                                 int32_t n_times, double record_dt, const double* rates, double x_ul, double y_ul) {
    if (!x_gauge || !y_gauge || !rates) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        return m.set_rain_gauges(n_gauges, x_gauge, y_gauge, n_times, record_dt, rates, x_ul, y_ul);
    });
}

hp2d_status hp2d_set_rain_clock(hp2d_ctx* ctx, double rain_t0, double rain_t1, double t_previous) {
    return with_impl(ctx, [&](auto& m) { return m.set_rain_clock(rain_t0, rain_t1, t_previous); });
}

hp2d_status hp2d_set_rain_maps_end_stamped(hp2d_ctx* ctx, int32_t n_maps, int32_t my, int32_t mx, const float* rate,
                                           const double* t_end, double dt_force) {
    return with_impl(ctx, [&](auto& m) { return m.set_rain_maps_end_stamped(n_maps, my, mx, rate, t_end, dt_force); });
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

hp2d_status hp2d_set_layout(hp2d_ctx* ctx, int32_t cells_per_lane) {
    if (cells_per_lane != 1 && cells_per_lane != 2) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        m.cells_per_lane = cells_per_lane;
        m.invalidate_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_set_tuning(hp2d_ctx* ctx, int32_t rows_per_warp) {
    if (rows_per_warp < 4) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        m.rows_per_warp = rows_per_warp;
        m.rpw_chosen = true;
        m.invalidate_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_run(hp2d_ctx* ctx, int64_t max_steps, int64_t* steps_done) {
    return with_impl(ctx, [&](auto& m) { return m.run(max_steps, steps_done); });
}

hp2d_status hp2d_set_retry_policy(hp2d_ctx* ctx, int32_t max_retries, double factor_reduction,
                                  int32_t dt_floor_is_error) {
    return with_impl(ctx, [&](auto& m) { return m.set_retry_policy(max_retries, factor_reduction, dt_floor_is_error); });
}

hp2d_status hp2d_set_wait_limit(hp2d_ctx* ctx, int64_t polls) {
    if (polls < 0 || polls > int64_t(0xffffffffu)) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) {
        m.wait_polls = unsigned(polls);
        m.invalidate_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_inject_step_fault(hp2d_ctx* ctx, int64_t k, int32_t attempts) {
    return with_impl(ctx, [&](auto& m) { return m.inject_fault(k, attempts); });
}

hp2d_status hp2d_set_owned_rows(hp2d_ctx* ctx, int32_t row0, int32_t row1) {
    return with_impl(ctx, [&](auto& m) { return m.set_owned_rows(row0, row1); });
}

hp2d_status hp2d_step_maxima(hp2d_ctx* ctx, uint64_t* speed2_bits, uint64_t* celerity_bits, int32_t* clamp_skip) {
    if (!speed2_bits || !celerity_bits) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.step_maxima(speed2_bits, celerity_bits, clamp_skip); });
}

hp2d_status hp2d_apply_refresh(hp2d_ctx* ctx, uint64_t speed2_bits, uint64_t celerity_bits, int32_t clamp_skip) {
    return with_impl(ctx, [&](auto& m) { return m.apply_refresh(speed2_bits, celerity_bits, clamp_skip); });
}

hp2d_status hp2d_copy_rows(hp2d_ctx* ctx, int32_t row0, int32_t nrows, void* buffer, int32_t into_state) {
    return with_impl(ctx, [&](auto& m) { return m.copy_rows(row0, nrows, buffer, into_state); });
}

hp2d_status hp2d_set_temporal_blocking(hp2d_ctx* ctx, int32_t steps_per_block) {
    return with_impl(ctx, [&](auto& m) { return m.set_temporal_blocking(steps_per_block); });
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

extern "C" {

hp2d_status hp2d_autotune(hp2d_ctx* ctx, int32_t trial_steps, int32_t* rows_per_warp) {
    if (trial_steps < 1) return HP2D_INVALID_ARG;
    return with_impl(ctx, [&](auto& m) { return m.autotune(trial_steps, rows_per_warp); });
}

hp2d_status hp2d_ensemble_create(int32_t device, hp2d_ensemble** out) {
    if (!out) return HP2D_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_create_error = "no CUDA device";
        return HP2D_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) { g_create_error = "device index out of range"; return HP2D_INVALID_ARG; }
    auto* e = new hp2d_ensemble();
    e->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        g_create_error = "cannot create the ensemble's stream";
        delete e;
        return HP2D_CUDA_ERROR;
    }
    *out = e;
    return HP2D_OK;
}

hp2d_status hp2d_ensemble_destroy(hp2d_ensemble* e) {
    if (!e) return HP2D_INVALID_ARG;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    e->drop_graph();
    e->args.free();
    e->prefix.free();
    e->queue.free();
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return HP2D_OK;
}

const char* hp2d_ensemble_last_error(const hp2d_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

hp2d_status hp2d_ensemble_add(hp2d_ensemble* e, hp2d_ctx* member) {
    return ens_guarded(e, [&]() -> hp2d_status {
        if (!member || !member->impl) { e->err = "null member"; return HP2D_INVALID_ARG; }
        if (member->g.precision != HP2D_FP32) { e->err = "ensemble members must be FP32 contexts"; return HP2D_INVALID_ARG; }
        if (member->device != e->device) { e->err = "member lives on another device"; return HP2D_INVALID_ARG; }
        for (auto* m : e->members)
            if (m == member) { e->err = "member added twice"; return HP2D_INVALID_ARG; }
        e->members.push_back(member);
        e->drop_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_ensemble_set_tuning(hp2d_ensemble* e, int32_t rows_per_warp) {
    if (rows_per_warp < 4) return HP2D_INVALID_ARG;
    return ens_guarded(e, [&]() -> hp2d_status {
        e->rows_per_warp = rows_per_warp;
        e->drop_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_ensemble_set_layout(hp2d_ensemble* e, int32_t cells_per_lane) {
    if (cells_per_lane != 1 && cells_per_lane != 2) return HP2D_INVALID_ARG;
    return ens_guarded(e, [&]() -> hp2d_status {
        e->cells_per_lane = cells_per_lane;
        e->drop_graph();
        return HP2D_OK;
    });
}

hp2d_status hp2d_ensemble_autotune(hp2d_ensemble* e, int32_t trial_steps, int32_t* rows_per_warp) {
    if (trial_steps < 1) return HP2D_INVALID_ARG;
    return ens_guarded(e, [&]() { return e->autotune(trial_steps, rows_per_warp); });
}

hp2d_status hp2d_ensemble_steps(hp2d_ensemble* e, int32_t nsteps, int32_t* n_active) {
    if (nsteps < 0) return HP2D_INVALID_ARG;
    return ens_guarded(e, [&]() { return e->steps(nsteps, n_active); });
}

hp2d_status hp2d_ensemble_steps_timed(hp2d_ensemble* e, int32_t nsteps, int32_t* n_active, float* elapsed_ms) {
    if (nsteps < 0 || !elapsed_ms) return HP2D_INVALID_ARG;
    return ens_guarded(e, [&]() -> hp2d_status {
        hp2d_status s = e->prepare();
        if (s != HP2D_OK) return s;
        if (nsteps >= hp2d_ensemble::kChunk) e->ensure_graph(int(e->members.size()));   // set-up, untimed
        HP_CK(cudaStreamSynchronize(e->stream));
        cudaEvent_t e0, e1;
        HP_CK(cudaEventCreate(&e0));
        HP_CK(cudaEventCreate(&e1));
        HP_CK(cudaEventRecord(e0, e->stream));
        s = e->steps(nsteps, n_active, e1);
        HP_CK(cudaEventSynchronize(e1));
        HP_CK(cudaEventElapsedTime(elapsed_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return s;
    });
}

hp2d_status hp2d_ensemble_run(hp2d_ensemble* e, int64_t max_steps, int64_t* steps_done) {
    return ens_guarded(e, [&]() { return e->run(max_steps, steps_done); });
}

}  // extern "C"
