// hp2d_cfl_dt_noalloc: refreshing_timestep's refresh branch on caller-owned device arrays
// that allocates no memory at all.
//
// Who needs it: callers that may not allocate GPU memory while they run -- a MEX gateway
// living inside MATLAB, whose GPU memory pool owns the device and is the only allocator
// allowed to grow; real-time drivers that forbid allocation after start-up.  They already
// hold the face fluxes and face depths on the device and only want the next time step.
// The call ends by copying the two maxima into host memory and synchronising the caller's
// stream.
//
// The reduction scratch (one partial maximum per block of 16 rows, plus the two final
// maxima) is the file-scope array g_noalloc_scratch below: 64 KB that every GPU which
// loads this library keeps until the process exits.  It bounds the grid to 65,536 rows.
// Host code cannot use the array's name as a device address (in host code it names a
// host-side shadow), so the first call on each device, with that device current, looks
// the address up with cudaGetSymbolAddress and keeps it; that first call should happen
// before any stream capture begins.  Every call shares the array, so calls that overlap
// on the GPU (other streams, other host threads) race; each call overwrites every slot
// it reads before reading it, so nothing needs clearing between calls.
#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "hp2d.h"
#include "hp2d_device.cuh"
#include "hp2d_fused.cuh"

namespace {

constexpr int kNoAllocRowsPerBlock = 16;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocMaxRows = kNoAllocRowsPerBlock * kNoAllocMaxBlocks;   // 65,536
constexpr int kNoAllocThreads = 256;

struct NoAllocScratch {
    unsigned long long s2max[kNoAllocMaxBlocks];   // speed^2 (ordered bits), per block
    unsigned long long cenc[kNoAllocMaxBlocks];    // celerity value bits + 1, 0 = none
    unsigned long long result[2];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
NoAllocScratch* g_noalloc_ptr[kMaxDevices] = {};

// per block: max speed^2 and encoded max celerity over its rows (refreshing_timestep.m
// :61-89, :139-150, :181-238, the same per-cell arithmetic as hp2d_cfl_dt)
__global__ void __launch_bounds__(kNoAllocThreads) k_cfl_partials_noalloc(
    int ny, int nx, double res, double tol_mm, const float* __restrict__ qx, const float* __restrict__ qy,
    const float* __restrict__ hf, int adaptive, float stag_s2, NoAllocScratch* s) {
    hp2d::StepConsts<float> K;
    K.make(1.0, res, tol_mm, 0.0);
    const size_t n = size_t(ny) * nx;
    const int r0 = blockIdx.x * kNoAllocRowsPerBlock;
    const int r1 = min(r0 + kNoAllocRowsPerBlock, ny);
    float s2max = 0.f;
    unsigned long long cenc = 0ull;
    const size_t c0 = size_t(r0) * nx, c1 = size_t(r1) * nx;
    for (size_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const int i = int(c / nx), j = int(c - size_t(i) * nx);
        const bool last = i + 1 >= ny;
        const float qyb = last ? 0.f : qy[c + nx];
        const float hfb = last ? 0.f : hf[n + c + nx];
        const float hfx = hf[c], hfy = hf[n + c], hf3 = hf[2 * n + c];
        const float big = 1e9f;
        const float vr = hp2d::qdiv(qx[c], hfx < K.tol ? big : hfx);
        const float vu = hp2d::qdiv(qy[c], hfy < K.tol ? big : hfy);
        const float vb = hp2d::qdiv(qyb, hfb < K.tol ? big : hfb);
        const float rc = j == 0 ? 0.5f * vr : vr;
        const float uc = 0.5f * (vu + vb);
        const float s2 = rc * rc + uc * uc;
        s2max = fmaxf(s2max, s2);
        if (s2 >= stag_s2) {
            const float dts = fmaxf(fmaxf(hfx, hfy), hf3);
            float cval;
            if (adaptive == 1) {
                cval = K.g * fmaxf(dts, 0.f);
            } else {
                const float wc = fmaxf(sqrtf(K.g * fmaxf(dts, 0.f)), 1e-10f);
                cval = fmaxf(fmaxf(fabsf(vr), fabsf(vu)), fabsf(vb)) + wc;
            }
            const unsigned long long e = hp2d::ord_bits(cval) + 1ull;
            cenc = e > cenc ? e : cenc;
        }
    }
    __shared__ float ss[kNoAllocThreads / 32];
    __shared__ unsigned long long sc[kNoAllocThreads / 32];
    s2max = hp2d::warp_max(s2max);
    cenc = hp2d::warp_max_u(cenc);
    if ((threadIdx.x & 31) == 0) {
        ss[threadIdx.x >> 5] = s2max;
        sc[threadIdx.x >> 5] = cenc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kNoAllocThreads / 32; ++w) {
            s2max = fmaxf(s2max, ss[w]);
            cenc = sc[w] > cenc ? sc[w] : cenc;
        }
        s->s2max[blockIdx.x] = hp2d::ord_bits(s2max);
        s->cenc[blockIdx.x] = cenc;
    }
}

// one block: maxima over the block partials
__global__ void __launch_bounds__(kNoAllocThreads) k_cfl_final_noalloc(int nblocks, NoAllocScratch* s) {
    unsigned long long a = 0ull, b = 0ull;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a = s->s2max[i] > a ? s->s2max[i] : a;
        b = s->cenc[i] > b ? s->cenc[i] : b;
    }
    a = hp2d::warp_max_u(a);
    b = hp2d::warp_max_u(b);
    __shared__ unsigned long long sa[kNoAllocThreads / 32], sb[kNoAllocThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kNoAllocThreads / 32; ++w) {
            a = sa[w] > a ? sa[w] : a;
            b = sb[w] > b ? sb[w] : b;
        }
        s->result[0] = a;
        s->result[1] = b;
    }
}

float stagnant_threshold_f32() {
    const float target = 0.01f;
    float x = target * target;
    while (x > 0.f && std::sqrt(std::nextafter(x, 0.f)) >= target) x = std::nextafter(x, 0.f);
    while (std::sqrt(x) < target) x = std::nextafter(x, 1.f);
    return x;
}

thread_local std::string g_noalloc_error;

hp2d_status fail(hp2d_status st, const char* what, cudaError_t e = cudaSuccess) {
    g_noalloc_error = what;
    if (e != cudaSuccess) {
        g_noalloc_error += ": ";
        g_noalloc_error += cudaGetErrorString(e);
    }
    return st;
}

}  // namespace

extern "C" {

const char* hp2d_noalloc_error(void) { return g_noalloc_error.c_str(); }

hp2d_status hp2d_cfl_dt_noalloc(int32_t ny, int32_t nx, double resolution, const hp2d_params* params,
                                const float* q_x, const float* q_y, const float* hf, void* stream,
                                double* time_step, double* max_velocity) {
    g_noalloc_error.clear();
    if (!params || !q_x || !q_y || !hf || !time_step) return fail(HP2D_INVALID_ARG, "null argument");
    if (ny <= 0 || nx <= 0 || !(resolution > 0)) return fail(HP2D_INVALID_ARG, "grid must have ny, nx > 0 and resolution > 0");
    if (ny > kNoAllocMaxRows)
        return fail(HP2D_INVALID_ARG,
                    "grid has more than 65536 rows: the fixed scratch of hp2d_cfl_dt_noalloc holds partial maxima "
                    "for at most 4096 blocks of 16 rows; use hp2d_cfl_dt on a context instead");
    if (int64_t(ny) * nx > int64_t(INT32_MAX)) return fail(HP2D_INVALID_ARG, "grid has more than 2^31-1 cells");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(HP2D_NO_DEVICE, "cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return fail(HP2D_INVALID_ARG, "device index beyond 63");
    NoAllocScratch* s = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail(HP2D_CUDA_ERROR, "cudaGetSymbolAddress(g_noalloc_scratch)", e);
            g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(p);
        }
        s = g_noalloc_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call ends with a read-back and a stream synchronisation, neither of which a stream
    // under capture allows: refuse before anything enters the caller's capture
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return fail(HP2D_CUDA_ERROR, "cudaStreamIsCapturing", e);
    if (cap != cudaStreamCaptureStatusNone)
        return fail(HP2D_INVALID_ARG, "the stream is being captured: hp2d_cfl_dt_noalloc reads its result back "
                                      "and synchronises the stream");
    const int nblocks = (ny + kNoAllocRowsPerBlock - 1) / kNoAllocRowsPerBlock;
    k_cfl_partials_noalloc<<<nblocks, kNoAllocThreads, 0, st>>>(ny, nx, resolution, params->depth_tolerance, q_x, q_y,
                                                               hf, params->flag_adaptive_timestepping,
                                                               stagnant_threshold_f32(), s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HP2D_CUDA_ERROR, "k_cfl_partials_noalloc launch", e);
    k_cfl_final_noalloc<<<1, kNoAllocThreads, 0, st>>>(nblocks, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HP2D_CUDA_ERROR, "k_cfl_final_noalloc launch", e);
    unsigned long long res2[2] = {0ull, 0ull};
    e = cudaMemcpyAsync(res2, s->result, sizeof(res2), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(HP2D_CUDA_ERROR, "reading the maxima back", e);
    const float vR = std::sqrt(hp2d::from_ord(res2[0], false) > 0 ? float(hp2d::from_ord(res2[0], false)) : 0.f);
    const double vm = double(vR);
    double cm = 0.0;
    if (res2[1]) {
        const float v = float(hp2d::from_ord(res2[1] - 1ull, false));
        cm = params->flag_adaptive_timestepping == 1 ? double(std::fmax(std::sqrt(v), 1e-10f)) : double(v);
    }
    const hp2d_params& p = *params;
    const double tcr = hp2d::finalize_dt(vm, cm, resolution, p.alfa_min, p.alfa_max, p.min_time_step, p.max_time_step,
                                         p.time_step_increments, p.flag_timestep);
    *time_step = tcr / 60.0;
    if (max_velocity) *max_velocity = vm;
    return HP2D_OK;
}

}  // extern "C"
