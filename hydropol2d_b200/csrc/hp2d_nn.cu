// Kernels of the learned screening network (include/hp2d_nn.h): the tcgen05 GEMM host
// side (tensor maps, tile choice) and the memory-bound layers around it.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "hp2d.h"
#include "hp2d_nn.h"
#include "hp2d_nn_gemm.cuh"

using namespace hp2d;
using namespace hp2d::nn;

namespace {

thread_local std::string g_nn_error;
__device__ int g_nn_err_flag = 0;

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// K-major BF16 matrix [rows, K] with pitch ld (elements), box kb x box_rows; 128-byte swizzle
// for 64-element (128-byte) rows, 64-byte swizzle for 32-element rows
bool make_map(CUtensorMap* m, const void* base, int rows, int K, int ld, int box_rows, int kb = kBK) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {cuuint64_t(K), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(ld) * 2};
    cuuint32_t box[2] = {cuuint32_t(kb), cuuint32_t(box_rows)};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, kb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// NHWC BF16 activations [B, H, W, C] as a 4-D map (C innermost); box kb channels x
// min(W, 128) pixels x 128/min(W,128) rows x 1 image = the 128 pixels of one GEMM tile.
// Coordinates outside the image read as zeros (the convolution's padding).
bool make_map_nhwc(CUtensorMap* m, const void* base, int B, int H, int W, int C, int kb) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int bw = W < kBM ? W : kBM;
    cuuint64_t dims[4] = {cuuint64_t(C), cuuint64_t(W), cuuint64_t(H), cuuint64_t(B)};
    cuuint64_t strides[3] = {cuuint64_t(C) * 2, cuuint64_t(W) * C * 2, cuuint64_t(H) * W * C * 2};
    cuuint32_t box[4] = {cuuint32_t(kb), cuuint32_t(bw), cuuint32_t(kBM / bw), 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, kb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

hp2d_status fail(const std::string& msg, hp2d_status st = HP2D_INVALID_ARG) {
    g_nn_error = msg;
    return st;
}

hp2d_status launched(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string(what) + ": " + cudaGetErrorString(e), HP2D_CUDA_ERROR);
    return HP2D_OK;
}

// the current device's copy of the kernels' error flag (resolved once per device)
int* err_ptr() {
    static std::mutex mu;
    static int* ptr[64] = {};
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[d]) {
        void* q = nullptr;
        if (cudaGetSymbolAddress(&q, g_nn_err_flag) != cudaSuccess) return nullptr;
        ptr[d] = static_cast<int*>(q);
    }
    return ptr[d];
}

std::mutex g_launch_init_mutex;   // first-use set-up of the GEMM launches, per device

int sm_count(int dev) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
}

// a grid of more tiles than the persistent kernel's resident CTAs runs persistently
// (k_gemm_bf16_pt), a smaller one one tile per CTA
template <int BN, int KB, bool IM2COL>
hp2d_status launch_tiles(const CUtensorMap& ma, const CUtensorMap& mb, int M, int N, int kt, int per, int mtiles,
                         int ntiles, int splits, void* C, int ldc, const float* bias, int epi, int* err, ConvGeom g,
                         cudaStream_t st) {
    // per device: attributes set and the persistent kernel's resident CTAs per SM (by registers and
    // shared memory, and by TMEM: 2 x BN of its 512 columns per CTA)
    constexpr int kDevs = 64;
    static int per_sm[kDevs] = {};
    static int sms[kDevs] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kDevs) return fail("device index beyond 63");
    const size_t smem = gemm_smem_bytes<BN, KB>();
    std::unique_lock<std::mutex> lock(g_launch_init_mutex);
    if (!per_sm[dev]) {
        if (cudaFuncSetAttribute(k_gemm_bf16<BN, KB, IM2COL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess ||
            cudaFuncSetAttribute(k_gemm_bf16_pt<BN, KB, IM2COL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)) != cudaSuccess)
            return launched("cudaFuncSetAttribute");
        // the largest shared-memory carveout, so that CTAs of several tiles can share an SM
        cudaFuncSetAttribute(k_gemm_bf16_pt<BN, KB, IM2COL>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncAttributes fa{};
        int smem_sm = 0;
        if (cudaFuncGetAttributes(&fa, k_gemm_bf16_pt<BN, KB, IM2COL>) != cudaSuccess ||
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
            return launched("cudaFuncGetAttributes");
        const int regs = ((fa.numRegs + 7) / 8) * 8;
        const int by_regs = 65536 / std::max(1, regs * kPtThreads);
        const int by_smem = smem_sm / int(smem + fa.sharedSizeBytes + 1024);
        per_sm[dev] = std::max(1, std::min({by_regs, by_smem, 512 / (2 * BN), 4}));
        sms[dev] = sm_count(dev);
    }
    const int ctas = per_sm[dev], n_sms = sms[dev];
    lock.unlock();
    const long total = long(mtiles) * ntiles * splits;
    // split-K partial sums (atomic epilogue) run one CTA per SM: measured faster in the training
    // step's weight-gradient GEMMs than several CTAs adding into the same outputs
    const int grid_pt = n_sms * (epi == EPI_F32_ATOMIC ? 1 : ctas);
    if (total > grid_pt) {
        k_gemm_bf16_pt<BN, KB, IM2COL><<<grid_pt, kPtThreads, smem, st>>>(ma, mb, M, N, kt, per, C, ldc, bias, epi,
                                                                          err, g, mtiles, ntiles, splits);
        return launched("k_gemm_bf16_pt");
    }
    k_gemm_bf16<BN, KB, IM2COL><<<dim3(mtiles, ntiles, splits), 128, smem, st>>>(ma, mb, M, N, kt, per, C, ldc, bias,
                                                                               epi, err, g);
    return launched("k_gemm_bf16");
}

template <int BN>
hp2d_status gemm_bn(int M, int N, int K, const void* A, int lda, const void* B, int ldb, void* C, int ldc,
                    const float* bias, int epi, int split_k, cudaStream_t st) {
    CUtensorMap ma, mb;
    if (!make_map(&ma, A, M, K, lda, kBM) || !make_map(&mb, B, N, K, ldb, BN))
        return fail("cuTensorMapEncodeTiled rejected an operand (alignment or pitch)");
    const int kt = K / kBK;
    const int per = (kt + split_k - 1) / split_k;
    const int splits = (kt + per - 1) / per;   // every split gets at least one k tile
    int* err = err_ptr();
    if (!err) return fail("cannot resolve the error flag", HP2D_CUDA_ERROR);
    return launch_tiles<BN, kBK, false>(ma, mb, M, N, kt, per, (M + kBM - 1) / kBM, (N + BN - 1) / BN, splits, C,
                                        ldc, bias, epi, err, ConvGeom{0, 0, 0}, st);
}

template <int BN, int KB>
hp2d_status conv_bn(const void* x, int B, int H, int W, int Cin, const void* w, int ldw, int Co, const float* bias,
                    void* y, int ldy, int epi, cudaStream_t st) {
    CUtensorMap ma, mb;
    if (!make_map_nhwc(&ma, x, B, H, W, Cin, KB) || !make_map(&mb, w, Co, 9 * Cin, ldw, BN, KB))
        return fail("cuTensorMapEncodeTiled rejected an operand (alignment or pitch)");
    int* err = err_ptr();
    if (!err) return fail("cannot resolve the error flag", HP2D_CUDA_ERROR);
    const int M = B * H * W;
    const int kt = 9 * Cin / KB;
    return launch_tiles<BN, KB, true>(ma, mb, M, Co, kt, kt, M / kBM, (Co + BN - 1) / BN, 1, y, ldy, bias, epi, err,
                                      ConvGeom{H, W, Cin / KB}, st);
}

template <int KB>
hp2d_status conv_kb(const void* x, int B, int H, int W, int Cin, const void* w, int ldw, int Co, const float* bias,
                    void* y, int ldy, int epi, cudaStream_t st) {
    if (Co <= 32) return conv_bn<32, KB>(x, B, H, W, Cin, w, ldw, Co, bias, y, ldy, epi, st);
    if (Co <= 64) return conv_bn<64, KB>(x, B, H, W, Cin, w, ldw, Co, bias, y, ldy, epi, st);
    if (Co <= 128) return conv_bn<128, KB>(x, B, H, W, Cin, w, ldw, Co, bias, y, ldy, epi, st);
    return conv_bn<256, KB>(x, B, H, W, Cin, w, ldw, Co, bias, y, ldy, epi, st);
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
inline int blocks(int64_t n, int t = 256) { return int(std::min<int64_t>((n + t - 1) / t, 148 * 32)); }

__device__ __forceinline__ float bf(uint16_t u) { return __uint_as_float(uint32_t(u) << 16); }

// ---- layers ------------------------------------------------------------------------------
__global__ void k_im2col(const uint16_t* __restrict__ x, int B, int H, int W, int C, uint16_t* __restrict__ cols,
                         int Kp) {
    const int64_t P = int64_t(B) * H * W;
    const int64_t n = P * Kp;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = e / Kp;
        const int k = int(e - p * Kp);
        uint16_t v = 0;
        if (k < 9 * C) {
            const int tap = k / C, c = k - tap * C;
            const int b = int(p / (int64_t(H) * W));
            const int rem = int(p - int64_t(b) * H * W);
            const int y = rem / W + tap / 3 - 1, xx = rem % W + tap % 3 - 1;
            if (y >= 0 && y < H && xx >= 0 && xx < W) v = x[((int64_t(b) * H + y) * W + xx) * C + c];
        }
        cols[e] = v;
    }
}
// 8 channels (16 bytes) per thread when C % 8 == 0
__global__ void k_im2col_v8(const uint4* __restrict__ x, int B, int H, int W, int C8, uint4* __restrict__ cols,
                            int Kp8) {
    const int64_t P = int64_t(B) * H * W;
    const int64_t n = P * Kp8;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = e / Kp8;
        const int k = int(e - p * Kp8);
        uint4 v = make_uint4(0, 0, 0, 0);
        if (k < 9 * C8) {
            const int tap = k / C8, c = k - tap * C8;
            const int b = int(p / (int64_t(H) * W));
            const int rem = int(p - int64_t(b) * H * W);
            const int y = rem / W + tap / 3 - 1, xx = rem % W + tap % 3 - 1;
            if (y >= 0 && y < H && xx >= 0 && xx < W) v = x[((int64_t(b) * H + y) * W + xx) * C8 + c];
        }
        cols[e] = v;
    }
}
// transposed im2col: cols[k, p], consecutive threads along p
__global__ void k_im2col_t(const uint16_t* __restrict__ x, int B, int H, int W, int C, uint16_t* __restrict__ cols,
                           int Kp) {
    const int64_t P = int64_t(B) * H * W;
    const int64_t n = P * Kp;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(e / P);
        const int64_t p = e - int64_t(k) * P;
        uint16_t v = 0;
        if (k < 9 * C) {
            const int tap = k / C, c = k - tap * C;
            const int b = int(p / (int64_t(H) * W));
            const int rem = int(p - int64_t(b) * H * W);
            const int y = rem / W + tap / 3 - 1, xx = rem % W + tap % 3 - 1;
            if (y >= 0 && y < H && xx >= 0 && xx < W) v = x[((int64_t(b) * H + y) * W + xx) * C + c];
        }
        cols[e] = v;
    }
}

__global__ void k_transpose(const uint16_t* __restrict__ in, int rows, int cols, int ldi, uint16_t* __restrict__ out,
                            int ldo) {
    __shared__ uint16_t tile[32][33];
    // row tiles on x (up to 2^31 - 1 of them: batches of large images), column tiles on y
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        tile[i][threadIdx.x] = (r < rows && c < cols) ? in[int64_t(r) * ldi + c] : 0;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[int64_t(c) * ldo + r] = tile[threadIdx.x][i];
    }
}

__global__ void k_maxpool2(const uint16_t* __restrict__ x, int B, int H, int W, int C, uint16_t* __restrict__ y) {
    const int Ho = H / 2, Wo = W / 2;
    const int64_t n = int64_t(B) * Ho * Wo * C;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % C);
        int64_t q = e / C;
        const int xo = int(q % Wo);
        q /= Wo;
        const int yo = int(q % Ho);
        const int b = int(q / Ho);
        const int64_t i00 = ((int64_t(b) * H + 2 * yo) * W + 2 * xo) * C + c;
        float m = bf(x[i00]);
        uint16_t best = x[i00];
        const int64_t offs[3] = {int64_t(C), int64_t(W) * C, int64_t(W) * C + C};
        for (int t = 0; t < 3; ++t) {
            const uint16_t u = x[i00 + offs[t]];
            if (bf(u) > m) { m = bf(u); best = u; }
        }
        y[e] = best;
    }
}
__global__ void k_maxpool2_bwd(const uint16_t* __restrict__ x, const uint16_t* __restrict__ y,
                               const uint16_t* __restrict__ dy, int B, int H, int W, int C, uint16_t* __restrict__ dx,
                               int acc) {
    const int Ho = H / 2, Wo = W / 2;
    const int64_t n = int64_t(B) * Ho * Wo * C;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % C);
        int64_t q = e / C;
        const int xo = int(q % Wo);
        q /= Wo;
        const int yo = int(q % Ho);
        const int b = int(q / Ho);
        const int64_t i00 = ((int64_t(b) * H + 2 * yo) * W + 2 * xo) * C + c;
        const int64_t offs[4] = {0, int64_t(C), int64_t(W) * C, int64_t(W) * C + C};
        const float m = bf(y[e]);
        bool routed = false;
        for (int t = 0; t < 4; ++t) {
            const bool hit = !routed && bf(x[i00 + offs[t]]) == m;
            if (acc) {
                if (hit) dx[i00 + offs[t]] = f2bf(bf(dx[i00 + offs[t]]) + bf(dy[e]));
            } else {
                dx[i00 + offs[t]] = hit ? dy[e] : uint16_t(0);
            }
            routed = routed || hit;
        }
    }
}

__global__ void k_upsample2(const uint16_t* __restrict__ x, int B, int H, int W, int C, uint16_t* __restrict__ y) {
    const int64_t n = int64_t(B) * (2 * H) * (2 * W) * C;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % C);
        int64_t q = e / C;
        const int xo = int(q % (2 * W));
        q /= 2 * W;
        const int yo = int(q % (2 * H));
        const int b = int(q / (2 * H));
        y[e] = x[((int64_t(b) * H + yo / 2) * W + xo / 2) * C + c];
    }
}
__global__ void k_upsample2_bwd(const uint16_t* __restrict__ dy, int B, int H, int W, int C, uint16_t* __restrict__ dx) {
    const int64_t n = int64_t(B) * H * W * C;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(e % C);
        int64_t q = e / C;
        const int xi = int(q % W);
        q /= W;
        const int yi = int(q % H);
        const int b = int(q / H);
        const int64_t W2 = 2 * W;
        const int64_t i00 = ((int64_t(b) * 2 * H + 2 * yi) * W2 + 2 * xi) * C + c;
        const float s = (bf(dy[i00]) + bf(dy[i00 + C])) + (bf(dy[i00 + W2 * C]) + bf(dy[i00 + W2 * C + C]));
        dx[e] = f2bf(s);
    }
}

__global__ void k_copy_channels(const uint16_t* __restrict__ in, int cin, int c0, int nch, int64_t P,
                                uint16_t* __restrict__ out, int cout, int o0) {
    const int64_t n = P * nch;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = e / nch;
        const int c = int(e - p * nch);
        out[p * cout + o0 + c] = in[p * cin + c0 + c];
    }
}

__global__ void k_relu_bwd(const uint16_t* __restrict__ y, uint16_t* __restrict__ dy, int64_t n) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x)
        if (!(bf(y[e]) > 0.0f)) dy[e] = 0;
}

// one block per 32 columns x a slab of rows; warp-level partial sums, one atomic per column
__global__ void k_colsum(const uint16_t* __restrict__ dz, int64_t P, int C, int ld, float* __restrict__ out) {
    const int c = blockIdx.x * 32 + threadIdx.x;
    float acc = 0.0f;
    if (c < C)
        for (int64_t p = blockIdx.y * int64_t(blockDim.y) + threadIdx.y; p < P; p += int64_t(gridDim.y) * blockDim.y)
            acc += bf(dz[p * ld + c]);
    __shared__ float part[8][33];
    part[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && c < C) {
        float s = 0.0f;
        for (int i = 0; i < int(blockDim.y); ++i) s += part[i][threadIdx.x];
        atomicAdd(out + c, s);
    }
}

__global__ void k_mse(const float* __restrict__ pred, int ldp, const float* __restrict__ t, const float* __restrict__ w,
                      int64_t P, int nch, float scale, float* loss, uint16_t* __restrict__ dpred, int ldd) {
    float acc = 0.0f;
    for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < P; p += int64_t(gridDim.x) * blockDim.x) {
        for (int c = 0; c < ldd; ++c) {
            uint16_t g = 0;
            if (c < nch) {
                const float d = pred[p * ldp + c] - t[p * nch + c];
                const float wc = w ? w[p * nch + c] : 1.0f;
                acc += wc * d * d;
                g = f2bf(2.0f * wc * d * scale);
            }
            dpred[p * ldd + c] = g;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0f) atomicAdd(loss, acc * scale);
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint16_t* __restrict__ wb, int64_t n, float lr, float b1, float b2, float eps, float wd,
                       float c1, float c2) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const float gi = g[e];
        const float mi = b1 * m[e] + (1.0f - b1) * gi;
        const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        const float mh = mi / c1, vh = vi / c2;
        float wi = w[e] * (1.0f - lr * wd);
        wi = wi - lr * mh / (sqrtf(vh) + eps);
        w[e] = wi;
        if (wb) wb[e] = f2bf(wi);
    }
}

__global__ void k_flip3x3(const float* __restrict__ w, int Co, int Ci, int Kp, uint16_t* __restrict__ wt, int Kp2) {
    const int64_t n = int64_t(Ci) * Kp2;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x) {
        const int ci = int(e / Kp2);
        const int k2 = int(e - int64_t(ci) * Kp2);
        float v = 0.0f;
        if (k2 < 9 * Co) {
            const int tap = k2 / Co, co = k2 - tap * Co;
            v = w[int64_t(co) * Kp + (8 - tap) * Ci + ci];
        }
        wt[e] = f2bf(v);
    }
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, uint16_t* __restrict__ out, int64_t n) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n; e += int64_t(gridDim.x) * blockDim.x)
        out[e] = f2bf(in[e]);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" {

const char* hp2d_nn_error(void) { return g_nn_error.c_str(); }

hp2d_status hp2d_nn_check(void) {
    int* p = err_ptr();
    if (!p) return fail("no device", HP2D_NO_DEVICE);
    int v = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) return launched("cudaDeviceSynchronize");
    if (cudaMemcpyFromSymbol(&v, g_nn_err_flag, sizeof(int)) != cudaSuccess) return launched("read error flag");
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_nn_err_flag, &zero, sizeof(int));
        return fail("a GEMM wait ran out of its iteration limit", HP2D_TIMEOUT);
    }
    return HP2D_OK;
}

hp2d_status hp2d_nn_gemm(int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B, int32_t ldb,
                         void* C, int32_t ldc, const float* bias, int32_t epi, int32_t split_k, void* stream) {
    if (M <= 0 || N <= 0 || K <= 0 || K % kBK) return fail("M, N > 0 and K a positive multiple of 64");
    if (!A || !B || !C) return fail("null operand");
    if (lda < K || ldb < K || lda % 8 || ldb % 8 || !aligned16(A) || !aligned16(B))
        return fail("A and B need pitches >= K, multiples of 8, and 16-byte aligned bases");
    if (ldc < N) return fail("ldc < N");
    if (epi < 0 || epi > 4) return fail("unknown epilogue");
    if ((epi == HP2D_NN_EPI_BF16_BIAS_RELU || epi == HP2D_NN_EPI_BF16_BIAS || epi == HP2D_NN_EPI_F32_BIAS) && !bias)
        return fail("bias epilogue without bias");
    if (split_k < 1 || (split_k > 1 && epi != HP2D_NN_EPI_F32_ATOMIC)) return fail("split_k > 1 needs the atomic epilogue");
    cudaStream_t st = S(stream);
    if (N <= 32) return gemm_bn<32>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, split_k, st);
    if (N <= 64) return gemm_bn<64>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, split_k, st);
    if (N <= 128) return gemm_bn<128>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, split_k, st);
    return gemm_bn<256>(M, N, K, A, lda, B, ldb, C, ldc, bias, epi, split_k, st);
}

hp2d_status hp2d_nn_conv3x3(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, const uint16_t* w,
                            int32_t ldw, int32_t Co, const float* bias, void* y, int32_t ldy, int32_t epi,
                            void* stream) {
    if (!x || !w || !y || B <= 0 || H <= 0 || W <= 0 || Co <= 0) return fail("conv3x3: bad shape");
    if (C < 32 || C % 32) return fail("conv3x3: the input needs a multiple of 32 channels");
    const bool rows_ok = (W % kBM == 0) || (kBM % W == 0 && H % (kBM / W) == 0);
    if (!rows_ok || (int64_t(H) * W) % kBM) return fail("conv3x3: H*W must tile into 128-pixel rows or row groups");
    if (ldw < 9 * C || ldw % 8 || !aligned16(x) || !aligned16(w)) return fail("conv3x3: weight pitch or alignment");
    if (ldy < Co) return fail("conv3x3: ldy < Co");
    if (epi != HP2D_NN_EPI_F32 && epi != HP2D_NN_EPI_BF16_BIAS_RELU && epi != HP2D_NN_EPI_BF16_BIAS &&
        epi != HP2D_NN_EPI_F32_BIAS)
        return fail("conv3x3: unsupported epilogue");
    if (epi != HP2D_NN_EPI_F32 && !bias) return fail("conv3x3: bias epilogue without bias");
    cudaStream_t st = S(stream);
    if (C % 64 == 0) return conv_kb<64>(x, B, H, W, C, w, ldw, Co, bias, y, ldy, epi, st);
    return conv_kb<32>(x, B, H, W, C, w, ldw, Co, bias, y, ldy, epi, st);
}

hp2d_status hp2d_nn_im2col3x3(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* cols,
                              int32_t Kp, int32_t transpose, void* stream) {
    if (!x || !cols || B <= 0 || H <= 0 || W <= 0 || C <= 0 || Kp < 9 * C) return fail("im2col: bad shape");
    const int64_t n = int64_t(B) * H * W * Kp;
    if (transpose) {
        k_im2col_t<<<blocks(n), 256, 0, S(stream)>>>(x, B, H, W, C, cols, Kp);
    } else if (C % 8 == 0 && Kp % 8 == 0 && aligned16(x) && aligned16(cols)) {
        k_im2col_v8<<<blocks(n / 8), 256, 0, S(stream)>>>(reinterpret_cast<const uint4*>(x), B, H, W, C / 8,
                                                          reinterpret_cast<uint4*>(cols), Kp / 8);
    } else {
        k_im2col<<<blocks(n), 256, 0, S(stream)>>>(x, B, H, W, C, cols, Kp);
    }
    return launched("im2col");
}

hp2d_status hp2d_nn_transpose(const uint16_t* in, int32_t rows, int32_t cols, int32_t ldi, uint16_t* out, int32_t ldo,
                              void* stream) {
    if (!in || !out || rows <= 0 || cols <= 0 || ldi < cols || ldo < rows) return fail("transpose: bad shape");
    if ((cols + 31) / 32 > 65535) return fail("transpose: more than 65535 column tiles");
    dim3 grid((rows + 31) / 32, (cols + 31) / 32);
    k_transpose<<<grid, dim3(32, 8), 0, S(stream)>>>(in, rows, cols, ldi, out, ldo);
    return launched("transpose");
}

hp2d_status hp2d_nn_maxpool2(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* y, void* stream) {
    if (!x || !y || H % 2 || W % 2 || B <= 0 || C <= 0) return fail("maxpool2: bad shape");
    k_maxpool2<<<blocks(int64_t(B) * H * W * C / 4), 256, 0, S(stream)>>>(x, B, H, W, C, y);
    return launched("maxpool2");
}

hp2d_status hp2d_nn_maxpool2_bwd(const uint16_t* x, const uint16_t* y, const uint16_t* dy, int32_t B, int32_t H,
                                 int32_t W, int32_t C, uint16_t* dx, int32_t accumulate, void* stream) {
    if (!x || !y || !dy || !dx || H % 2 || W % 2) return fail("maxpool2_bwd: bad shape");
    k_maxpool2_bwd<<<blocks(int64_t(B) * H * W * C / 4), 256, 0, S(stream)>>>(x, y, dy, B, H, W, C, dx, accumulate);
    return launched("maxpool2_bwd");
}

hp2d_status hp2d_nn_upsample2(const uint16_t* x, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* y, void* stream) {
    if (!x || !y) return fail("upsample2: null");
    k_upsample2<<<blocks(int64_t(B) * H * W * C * 4), 256, 0, S(stream)>>>(x, B, H, W, C, y);
    return launched("upsample2");
}

hp2d_status hp2d_nn_upsample2_bwd(const uint16_t* dy, int32_t B, int32_t H, int32_t W, int32_t C, uint16_t* dx,
                                  void* stream) {
    if (!dy || !dx) return fail("upsample2_bwd: null");
    k_upsample2_bwd<<<blocks(int64_t(B) * H * W * C), 256, 0, S(stream)>>>(dy, B, H, W, C, dx);
    return launched("upsample2_bwd");
}

hp2d_status hp2d_nn_copy_channels(const uint16_t* in, int32_t cin, int32_t c0, int32_t n, int64_t P, uint16_t* out,
                                  int32_t cout, int32_t o0, void* stream) {
    if (!in || !out || c0 + n > cin || o0 + n > cout || n <= 0) return fail("copy_channels: bad range");
    k_copy_channels<<<blocks(P * n), 256, 0, S(stream)>>>(in, cin, c0, n, P, out, cout, o0);
    return launched("copy_channels");
}

hp2d_status hp2d_nn_relu_bwd(const uint16_t* y, uint16_t* dy, int64_t n, void* stream) {
    if (!y || !dy) return fail("relu_bwd: null");
    k_relu_bwd<<<blocks(n), 256, 0, S(stream)>>>(y, dy, n);
    return launched("relu_bwd");
}

hp2d_status hp2d_nn_colsum(const uint16_t* dz, int64_t P, int32_t C, int32_t ld, float* out, void* stream) {
    if (!dz || !out || ld < C) return fail("colsum: bad shape");
    dim3 grid((C + 31) / 32, int(std::min<int64_t>((P + 255) / 256, 1024)));
    k_colsum<<<grid, dim3(32, 8), 0, S(stream)>>>(dz, P, C, ld, out);
    return launched("colsum");
}

hp2d_status hp2d_nn_mse(const float* pred, int32_t ldp, const float* target, const float* w, int64_t P, int32_t nch,
                        float scale, float* loss, uint16_t* dpred, int32_t ldd, void* stream) {
    if (!pred || !target || !loss || !dpred || ldp < nch || ldd < nch) return fail("mse: bad shape");
    k_mse<<<blocks(P), 256, 0, S(stream)>>>(pred, ldp, target, w, P, nch, scale, loss, dpred, ldd);
    return launched("mse");
}

hp2d_status hp2d_nn_adam(float* w, const float* g, float* m, float* v, uint16_t* w_bf16, int64_t n, float lr,
                         float beta1, float beta2, float eps, float weight_decay, int32_t step, void* stream) {
    if (!w || !g || !m || !v || step < 1) return fail("adam: bad arguments");
    const float c1 = 1.0f - powf(beta1, float(step)), c2 = 1.0f - powf(beta2, float(step));
    k_adam<<<blocks(n), 256, 0, S(stream)>>>(w, g, m, v, w_bf16, n, lr, beta1, beta2, eps, weight_decay, c1, c2);
    return launched("adam");
}

hp2d_status hp2d_nn_flip3x3(const float* w, int32_t Co, int32_t Ci, int32_t Kp, uint16_t* wt, int32_t Kp2, void* stream) {
    if (!w || !wt || Kp < 9 * Ci || Kp2 < 9 * Co) return fail("flip3x3: bad shape");
    k_flip3x3<<<blocks(int64_t(Ci) * Kp2), 256, 0, S(stream)>>>(w, Co, Ci, Kp, wt, Kp2);
    return launched("flip3x3");
}

hp2d_status hp2d_nn_f32_to_bf16(const float* in, uint16_t* out, int64_t n, void* stream) {
    if (!in || !out) return fail("f32_to_bf16: null");
    k_f32_to_bf16<<<blocks(n), 256, 0, S(stream)>>>(in, out, n);
    return launched("f32_to_bf16");
}

}  // extern "C"
