// BF16 tensor-core GEMM for the learned screening network (sm_100a, tcgen05 + TMA).
//
//   C[M x N] = A[M x K] * B[N x K]^T   (+ bias, ReLU, split-K accumulation)
//
// A and B are K-major BF16 (K contiguous), accumulation is FP32 in tensor memory.  One CTA
// of 128 threads computes a 128 x BN tile:
//   * thread 0 streams 128 x 64 and BN x 64 tiles of A and B into a ring of kStages
//     shared-memory stages with 2-D TMA copies (128-byte swizzle), completion counted in
//     bytes on the stage's `full` barrier;
//   * thread 32 issues four tcgen05.mma (M = 128, N = BN, K = 16) per stage into a TMEM
//     accumulator of BN columns and frees the stage with tcgen05.commit on `empty`;
//   * after the last stage a commit on `done` releases the epilogue: warp w reads TMEM
//     lanes 32w..32w+31 (tile rows) with tcgen05.ld and writes its rows to global memory.
// Every wait has an iteration limit; on expiry the kernel records an error code, lets its
// own copies land (again with a limit), frees its TMEM and returns.  No cluster multicast.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "hp2d_device.cuh"

namespace hp2d {
namespace nn {

constexpr int kBM = 128;         // tile rows (tcgen05 M)
constexpr int kBK = 64;          // tile depth: 64 BF16 = one 128-byte swizzle row
constexpr int kGemmStages = 4;
constexpr uint32_t kWaitLimit = 1u << 24;

enum Epilogue : int {
    EPI_F32 = 0,          // C fp32 = acc
    EPI_F32_ATOMIC = 1,   // C fp32 += acc (split-K partial sums, gradient accumulation)
    EPI_BF16_BIAS_RELU = 2,
    EPI_BF16_BIAS = 3,
    EPI_F32_BIAS = 4,
};

template <int BN, int KB = kBK> constexpr size_t gemm_smem_bytes() {
    return size_t(kGemmStages) * (kBM * KB * 2 + BN * KB * 2) + 1024;   // + alignment slack
}

// Geometry of an implicit-GEMM 3x3 convolution (A is read straight from the NHWC input):
// the 128 output pixels of a tile are 128 consecutive pixels of one image (W >= 128) or
// 128/W whole rows (W < 128); k tile kt is tap kt / cblocks, channel block kt % cblocks.
struct ConvGeom {
    int H, W, cblocks;
};

// ---- PTX wrappers ----------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the 128-byte
// swizzle: rows of 128 bytes, groups of 8 rows 1024 bytes apart (stride byte offset),
// descriptor version 1, layout type 2 (128-byte swizzle).  Addresses in 16-byte units.
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= uint64_t((smem_addr >> 4) & 0x3FFFu);
    d |= uint64_t(1u) << 16;                 // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(1024u >> 4) << 32;         // stride byte offset: 8 rows x 128 B
    d |= uint64_t(1u) << 46;                 // descriptor version
    d |= uint64_t(2u) << 61;                 // 128-byte swizzle
    return d;
}
// 32-element (64-byte) rows with the 64-byte swizzle: groups of 8 rows 512 bytes apart
__device__ __forceinline__ uint64_t sw64_kmajor_desc(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= uint64_t((smem_addr >> 4) & 0x3FFFu);
    d |= uint64_t(1u) << 16;
    d |= uint64_t(512u >> 4) << 32;          // stride byte offset: 8 rows x 64 B
    d |= uint64_t(1u) << 46;
    d |= uint64_t(4u) << 61;                 // 64-byte swizzle
    return d;
}
template <int KB> __device__ __forceinline__ uint64_t kmajor_desc(uint32_t a) {
    return KB == 64 ? sw128_kmajor_desc(a) : sw64_kmajor_desc(a);
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = BN
template <int BN> __device__ __forceinline__ constexpr uint32_t bf16_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(kBM >> 4) << 24);
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    return mbar_wait_bounded(bar, parity, kWaitLimit);
}

// round-to-nearest-even FP32 -> BF16
__device__ __forceinline__ uint16_t f2bf(float f) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

// One thread's 32 accumulator columns (tile row `row`, output columns col0..col0+31) through the
// epilogue `epi` into C.
__device__ __forceinline__ void store_row32(float (&v)[32], int row, int col0, int M, int N, void* C, int ldc,
                                            const float* __restrict__ bias, int epi) {
    if (row >= M || col0 >= N) return;
    const int ncol = min(32, N - col0);
    if (epi == EPI_F32 || epi == EPI_F32_BIAS) {
        float* out = static_cast<float*>(C) + size_t(row) * ldc + col0;
        if (epi == EPI_F32_BIAS)
            for (int i = 0; i < ncol; ++i) v[i] += bias[col0 + i];
        if (ncol == 32 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) {
#pragma unroll
            for (int i = 0; i < 32; i += 4)
                *reinterpret_cast<float4*>(out + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        } else {
            for (int i = 0; i < ncol; ++i) out[i] = v[i];
        }
    } else if (epi == EPI_F32_ATOMIC) {
        float* out = static_cast<float*>(C) + size_t(row) * ldc + col0;
        for (int i = 0; i < ncol; ++i) atomicAdd(out + i, v[i]);
    } else {
        uint16_t* out = static_cast<uint16_t*>(C) + size_t(row) * ldc + col0;
        const bool relu = epi == EPI_BF16_BIAS_RELU;
        uint32_t pk[16];
#pragma unroll
        for (int i = 0; i < 32; i += 2) {
            float a = v[i] + (col0 + i < N ? bias[col0 + i] : 0.0f);
            float b = v[i + 1] + (col0 + i + 1 < N ? bias[col0 + i + 1] : 0.0f);
            if (relu) { a = fmaxf(a, 0.0f); b = fmaxf(b, 0.0f); }
            pk[i / 2] = uint32_t(f2bf(a)) | (uint32_t(f2bf(b)) << 16);
        }
        if (ncol == 32 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) {
#pragma unroll
            for (int i = 0; i < 16; i += 4)
                *reinterpret_cast<uint4*>(out + 2 * i) = make_uint4(pk[i], pk[i + 1], pk[i + 2], pk[i + 3]);
        } else {
            for (int i = 0; i < ncol; ++i) out[i] = uint16_t(pk[i / 2] >> (16 * (i & 1)));
        }
    }
}

// KB: k-tile depth (64 with the 128-byte swizzle, 32 with the 64-byte swizzle); IM2COL: A is
// the NHWC input of a 3x3 convolution read through a 4-D tensor map (see ConvGeom).
template <int BN, int KB = kBK, bool IM2COL = false>
__global__ void __launch_bounds__(128, 1)
k_gemm_bf16(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
            int kt_total, int kt_per_split, void* C, int ldc, const float* __restrict__ bias, int epi,
            int* err, const ConvGeom g) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN");
    static_assert(KB == 64 || KB == 32, "KB");
    static_assert(KB == 64 || IM2COL, "32-deep tiles are for 32-channel convolutions");
    constexpr uint32_t kABytes = kBM * KB * 2;
    constexpr uint32_t kBBytes = BN * KB * 2;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) unsigned long long bar_full[kGemmStages], bar_empty[kGemmStages], bar_done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_addr(smem_raw) + 1023u) & ~1023u;
    const uint32_t sA0 = base, sB0 = base + kGemmStages * kABytes;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kt0 = blockIdx.z * kt_per_split;
    const int nk = min(kt0 + kt_per_split, kt_total) - kt0;

    if (warp == 0) tmem_alloc(smem_addr(&s_tmem), uint32_t(BN));
    if (tid == 0) {
        for (int s = 0; s < kGemmStages; ++s) {
            mbar_init(smem_addr(&bar_full[s]), 1u);
            mbar_init(smem_addr(&bar_empty[s]), 1u);
        }
        mbar_init(smem_addr(&bar_done), 1u);
        mbar_fence_init();
        s_fail = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    int issued = 0;
    if (tid == 0 && nk > 0) {
        // producer: TMA tiles of A (rows m0..) and B (rows n0..), k tile kt0 + i
        int img = 0, y0 = 0, x0 = 0;
        if (IM2COL) {
            const int hw = g.H * g.W;
            img = m0 / hw;
            const int rem = m0 - img * hw;
            y0 = rem / g.W;
            x0 = rem - y0 * g.W;
        }
        for (int i = 0; i < nk; ++i) {
            const int s = i % kGemmStages;
            const uint32_t fb = smem_addr(&bar_full[s]);
            if (i >= kGemmStages && !bar_wait(smem_addr(&bar_empty[s]), uint32_t(((i / kGemmStages) - 1) & 1))) {
                atomicExch(&s_fail, 1);
                break;
            }
            mbar_expect_tx(fb, kABytes + kBBytes);
            const int kt = kt0 + i;
            const int kx = kt * KB;
            if (IM2COL) {
                // tap (dy, dx) shifts the pixel box; TMA fills outside the image with zeros
                const int tap = kt / g.cblocks, cb = kt - tap * g.cblocks;
                tma_load_4d(sA0 + uint32_t(s) * kABytes, &tmA, cb * KB, x0 + tap % 3 - 1, y0 + tap / 3 - 1, img, fb);
            } else {
                tma_load_2d(sA0 + uint32_t(s) * kABytes, &tmA, kx, m0, fb);
            }
            tma_load_2d(sB0 + uint32_t(s) * kBBytes, &tmB, kx, n0, fb);
            issued = i + 1;
        }
    } else if (tid == 32) {
        // MMA issuer
        constexpr uint32_t idesc = bf16_idesc<BN>();
        for (int i = 0; i < nk; ++i) {
            const int s = i % kGemmStages;
            if (!bar_wait(smem_addr(&bar_full[s]), uint32_t((i / kGemmStages) & 1))) {
                atomicExch(&s_fail, 1);
                break;
            }
            tc_fence_after();
            const uint64_t da = kmajor_desc<KB>(sA0 + uint32_t(s) * kABytes);
            const uint64_t db = kmajor_desc<KB>(sB0 + uint32_t(s) * kBBytes);
#pragma unroll
            for (int kk = 0; kk < KB / 16; ++kk)   // +32 bytes per K=16 step inside the swizzled row
                tc_mma_bf16(tmem, da + uint64_t(2 * kk), db + uint64_t(2 * kk), idesc, (i | kk) != 0 ? 1u : 0u);
            tc_commit(smem_addr(&bar_empty[s]));
        }
        tc_commit(smem_addr(&bar_done));   // arrives once every MMA issued above has completed
    }
    __syncwarp();
    // epilogue: all 128 threads
    const bool landed = nk > 0 ? bar_wait(smem_addr(&bar_done), 0u) : true;
    if (!landed) atomicExch(&s_fail, 1);
    tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    if (landed && nk > 0) {
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
            store_row32(v, row, n0 + c0, M, N, C, ldc, bias, epi);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (s_fail) {
        if (tid == 0) {
            atomicExch(err, 1);
            // let the copies already issued land before the shared memory is released
            for (int i = max(0, issued - kGemmStages); i < issued; ++i)
                bar_wait(smem_addr(&bar_full[i % kGemmStages]), uint32_t((i / kGemmStages) & 1));
        }
        __syncthreads();
    }
    if (warp == 0) tmem_dealloc(tmem, uint32_t(BN));
}


// Persistent form (grids of more tiles than SMs).  One CTA of 192 threads per SM walks the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... of the (m, n, split) tile grid, m fastest:
//   * warp 0 lane 0 streams the k tiles of every tile through the same stage ring;
//   * warp 1 lane 0 issues the MMAs of the CTA's i-th tile into TMEM accumulator i % 2 (2 x BN
//     columns allocated) and commits `acc_full[i % 2]` after its last k tile;
//   * warps 2-5 drain accumulator i % 2 (warp w reads TMEM lanes 32 (w % 4) ..) through the
//     epilogue and release it on `acc_empty[i % 2]` (128 arrivals),
// so the epilogue of one tile overlaps the loads and MMAs of the next.  Every wait is bounded; a
// role whose wait expires sets the CTA's failure flag, the others stop at their next check, the
// MMA thread waits for its own MMAs, the producer for its own copies, and the TMEM is freed.
constexpr int kPtThreads = 192;

__device__ __forceinline__ bool pt_failed(const volatile int* f) { return *f != 0; }

template <int BN, int KB = kBK, bool IM2COL = false>
__global__ void __launch_bounds__(kPtThreads, 1)
k_gemm_bf16_pt(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
               int kt_total, int kt_per_split, void* C, int ldc, const float* __restrict__ bias, int epi,
               int* err, const ConvGeom g, int mtiles, int ntiles, int splits) {
    static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "BN");
    static_assert(KB == 64 || KB == 32, "KB");
    static_assert(KB == 64 || IM2COL, "32-deep tiles are for 32-channel convolutions");
    constexpr uint32_t kABytes = kBM * KB * 2;
    constexpr uint32_t kBBytes = BN * KB * 2;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) unsigned long long bar_full[kGemmStages], bar_empty[kGemmStages];
    __shared__ __align__(8) unsigned long long acc_full[2], acc_empty[2], bar_done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    volatile int* fail = &s_fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_addr(smem_raw) + 1023u) & ~1023u;
    const uint32_t sA0 = base, sB0 = base + kGemmStages * kABytes;
    const int total = mtiles * ntiles * splits;

    if (warp == 0) tmem_alloc(smem_addr(&s_tmem), uint32_t(2 * BN));
    if (tid == 0) {
        for (int s = 0; s < kGemmStages; ++s) {
            mbar_init(smem_addr(&bar_full[s]), 1u);
            mbar_init(smem_addr(&bar_empty[s]), 1u);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_addr(&acc_full[b]), 1u);
            mbar_init(smem_addr(&acc_empty[b]), 128u);
        }
        mbar_init(smem_addr(&bar_done), 1u);
        mbar_fence_init();
        s_fail = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    // tile t: rows m0.., columns n0.., k tiles kt0 .. kt0 + nk - 1
    auto tile = [&](int t, int& m0, int& n0, int& kt0, int& nk) {
        const int mt = t % mtiles, rest = t / mtiles;
        m0 = mt * kBM;
        n0 = (rest % ntiles) * BN;
        kt0 = (rest / ntiles) * kt_per_split;
        nk = min(kt0 + kt_per_split, kt_total) - kt0;
    };

    uint32_t issued = 0;   // producer: k tiles whose copies were issued
    if (warp == 0) {
        if (lane == 0) {
            for (int t = blockIdx.x; t < total && !pt_failed(fail); t += gridDim.x) {
                int m0, n0, kt0, nk;
                tile(t, m0, n0, kt0, nk);
                int img = 0, y0 = 0, x0 = 0;
                if (IM2COL) {
                    const int hw = g.H * g.W;
                    img = m0 / hw;
                    const int rem = m0 - img * hw;
                    y0 = rem / g.W;
                    x0 = rem - y0 * g.W;
                }
                for (int i = 0; i < nk; ++i) {
                    const uint32_t it = issued;
                    const int s = int(it % kGemmStages);
                    const uint32_t fb = smem_addr(&bar_full[s]);
                    if (it >= uint32_t(kGemmStages) &&
                        !bar_wait(smem_addr(&bar_empty[s]), ((it / kGemmStages) - 1u) & 1u)) {
                        *fail = 1;
                        break;
                    }
                    mbar_expect_tx(fb, kABytes + kBBytes);
                    const int kt = kt0 + i;
                    if (IM2COL) {
                        const int tap = kt / g.cblocks, cb = kt - tap * g.cblocks;
                        tma_load_4d(sA0 + uint32_t(s) * kABytes, &tmA, cb * KB, x0 + tap % 3 - 1, y0 + tap / 3 - 1,
                                    img, fb);
                    } else {
                        tma_load_2d(sA0 + uint32_t(s) * kABytes, &tmA, kt * KB, m0, fb);
                    }
                    tma_load_2d(sB0 + uint32_t(s) * kBBytes, &tmB, kt * KB, n0, fb);
                    issued = it + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = bf16_idesc<BN>();
            uint32_t it = 0;
            int lt = 0;
            for (int t = blockIdx.x; t < total && !pt_failed(fail); t += gridDim.x) {
                int m0, n0, kt0, nk;
                tile(t, m0, n0, kt0, nk);
                if (nk <= 0) continue;
                const int b = lt & 1;
                if (lt >= 2 && !bar_wait(smem_addr(&acc_empty[b]), uint32_t((lt >> 1) - 1) & 1u)) {
                    *fail = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + uint32_t(b * BN);
                bool ok = true;
                for (int i = 0; i < nk; ++i, ++it) {
                    const int s = int(it % kGemmStages);
                    if (!bar_wait(smem_addr(&bar_full[s]), (it / kGemmStages) & 1u)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t da = kmajor_desc<KB>(sA0 + uint32_t(s) * kABytes);
                    const uint64_t db = kmajor_desc<KB>(sB0 + uint32_t(s) * kBBytes);
#pragma unroll
                    for (int kk = 0; kk < KB / 16; ++kk)
                        tc_mma_bf16(acc, da + uint64_t(2 * kk), db + uint64_t(2 * kk), idesc, (i | kk) != 0 ? 1u : 0u);
                    tc_commit(smem_addr(&bar_empty[s]));
                }
                if (!ok) {
                    *fail = 1;
                    break;
                }
                tc_commit(smem_addr(&acc_full[b]));
                ++lt;
            }
            // every MMA this thread issued has completed before the TMEM can be released
            tc_commit(smem_addr(&bar_done));
            if (!bar_wait(smem_addr(&bar_done), 0u)) *fail = 1;
        }
    } else {
        const int q = warp & 3;   // TMEM lanes 32q .. 32q + 31 = tile rows
        int lt = 0;
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            int m0, n0, kt0, nk;
            tile(t, m0, n0, kt0, nk);
            if (nk <= 0) continue;
            const int b = lt & 1;
            bool ready = !pt_failed(fail) && bar_wait(smem_addr(&acc_full[b]), uint32_t(lt >> 1) & 1u);
            if (!__all_sync(0xffffffffu, ready)) {
                if (lane == 0) *fail = 1;
                break;
            }
            tc_fence_after();
            const int row = m0 + q * 32 + lane;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(b * BN + c0), v);
                store_row32(v, row, n0 + c0, M, N, C, ldc, bias, epi);
            }
            tc_fence_before();
            mbar_arrive(smem_addr(&acc_empty[b]));
            ++lt;
        }
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (s_fail) {
        if (tid == 0) {
            atomicExch(err, 1);
            // let the copies already issued land before the shared memory is released
            for (uint32_t i = issued > uint32_t(kGemmStages) ? issued - kGemmStages : 0u; i < issued; ++i)
                bar_wait(smem_addr(&bar_full[i % kGemmStages]), (i / kGemmStages) & 1u);
        }
        __syncthreads();
    }
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, uint32_t(2 * BN));
}

}  // namespace nn
}  // namespace hp2d
