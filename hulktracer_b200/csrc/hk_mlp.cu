// hk_mlp.cu -- the learned split proposer's network (no reference
// counterpart): 200 -> 256 -> 256 -> 256 -> 96, ReLU between layers.
//
// * Inference: BF16 weights and activations on the tensor cores, FP32
//   accumulate, 64-row tiles (hk_mlp_tile.cuh, shared with the builder);
//   weights are packed once into the per-lane B-fragment order.
// * Training: FP32 master weights; hand-written tiled SGEMM (with transposed
//   operands), bias / ReLU epilogues, softmax cross-entropy, ReLU backward,
//   column sums and Adam. Gradients are checked against a CPU FP32 reference.
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>
#include <algorithm>

#include <cstdlib>
#include <cstring>

#include "hk_mlp.h"
#include "hk_mlp_tc.cuh"
#include "hk_mlp_tile.cuh"

namespace hk {

// ---------------------------------------------------------------------------
// tiled FP32 GEMM: C[M x N] = op(A) op(B) (+ bias, ReLU); row-major storage
//   op(A)(m, k) = TA ? A[k * lda + m] : A[m * lda + k]
//   op(B)(k, n) = TB ? B[n * ldb + k] : B[k * ldb + n]
// ---------------------------------------------------------------------------
constexpr int GT = 64, GK = 16;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(const float *__restrict__ A, const float *__restrict__ B,
                                               float *__restrict__ C, const float *__restrict__ bias, int M, int N,
                                               int K, int lda, int ldb, int ldc, int relu, int accumulate) {
    __shared__ float As[GK][GT + 1];
    __shared__ float Bs[GK][GT + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * GT, n0 = blockIdx.x * GT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int i = threadIdx.x; i < GK * GT; i += 256) {
            int kk = i / GT, mm = i % GT;
            int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? (TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : 0.0f;
            int n = n0 + mm;
            Bs[kk][mm] = (n < N && k < K) ? (TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                a[i] = As[kk][ty * 4 + i];
                b[i] = Bs[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (accumulate) v += C[(size_t)m * ldc + n];
            if (bias) v += bias[n];
            if (relu) v = v > 0.0f ? v : 0.0f;
            C[(size_t)m * ldc + n] = v;
        }
    }
}

cudaError_t sgemm(bool ta, bool tb, const float *A, const float *B, float *C, const float *bias, int M, int N, int K,
                  int lda, int ldb, int ldc, bool relu, bool accumulate, cudaStream_t s) {
    dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
    if (!ta && !tb) k_sgemm<false, false><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, ldc, relu, accumulate);
    else if (ta && !tb) k_sgemm<true, false><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, ldc, relu, accumulate);
    else if (!ta && tb) k_sgemm<false, true><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, ldc, relu, accumulate);
    else k_sgemm<true, true><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, ldc, relu, accumulate);
    return cudaGetLastError();
}

// softmax cross-entropy over 96 logits per row; dZ = (p - onehot) / rows,
// loss accumulated (sum over rows of -log p_y) into *loss
__global__ void k_softmax_xent(const float *__restrict__ Z, const int32_t *__restrict__ y, int rows,
                               float *__restrict__ dZ, float *loss) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const float *z = Z + (size_t)warp * kMlpOut;
    float v[3];
    float mx = -INFINITY;
    for (int k = 0; k < 3; k++) {
        v[k] = z[lane + 32 * k];
        mx = fmaxf(mx, v[k]);
    }
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float sum = 0.0f;
    for (int k = 0; k < 3; k++) {
        v[k] = expf(v[k] - mx);
        sum += v[k];
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    int label = y[warp];
    float inv_rows = 1.0f / (float)rows;
    for (int k = 0; k < 3; k++) {
        int c = lane + 32 * k;
        float p = v[k] / sum;
        dZ[(size_t)warp * kMlpOut + c] = (p - (c == label ? 1.0f : 0.0f)) * inv_rows;
        if (c == label) atomicAdd(loss, -logf(fmaxf(p, 1e-30f)));
    }
}

__global__ void k_relu_back(float *__restrict__ dH, const float *__restrict__ H, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!(H[i] > 0.0f)) dH[i] = 0.0f;
}

__global__ void k_colsum(const float *__restrict__ dZ, int rows, int cols, float *__restrict__ db) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += dZ[(size_t)r * cols + c];
    db[c] = s;
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.0f - b1) * gi;
        float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

cudaError_t softmax_xent(const float *Z, const int32_t *y, int rows, float *dZ, float *loss, cudaStream_t s) {
    if (rows) k_softmax_xent<<<(rows * 32 + 255) / 256, 256, 0, s>>>(Z, y, rows, dZ, loss);
    return cudaGetLastError();
}
cudaError_t relu_back(float *dH, const float *H, size_t n, cudaStream_t s) {
    if (n) k_relu_back<<<(int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(dH, H, n);
    return cudaGetLastError();
}
cudaError_t colsum(const float *dZ, int rows, int cols, float *db, cudaStream_t s) {
    k_colsum<<<(cols + 127) / 128, 128, 0, s>>>(dZ, rows, cols, db);
    return cudaGetLastError();
}
cudaError_t adam(float *p, const float *g, float *m, float *v, size_t n, float lr, int step, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// BF16 inference on the tensor cores
// ---------------------------------------------------------------------------
// pack W (K x N fp32, row-major) into m16n8k16 B fragments: for k-tile kt,
// n-tile nt and lane l (g = l >> 2, t = l & 3): reg0 = {W[kt*16+2t][n],
// W[kt*16+2t+1][n]}, reg1 = the same 8 rows down, n = nt*8 + g. Rows past K
// are zero.
__global__ void k_pack_b(const float *__restrict__ W, int K, int N, int KT, uint32_t *__restrict__ out) {
    const int NT = N / 8;
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= KT * NT * 32) return;
    int lane = idx & 31, tile = idx >> 5;
    int kt = tile / NT, nt = tile % NT;
    int g = lane >> 2, t = lane & 3;
    int n = nt * 8 + g;
    auto w = [&](int k) { return k < K ? W[(size_t)k * N + n] : 0.0f; };
    int k0 = kt * 16 + 2 * t;
    __nv_bfloat162 r0 = __floats2bfloat162_rn(w(k0), w(k0 + 1));
    __nv_bfloat162 r1 = __floats2bfloat162_rn(w(k0 + 8), w(k0 + 9));
    out[2 * (size_t)idx] = *reinterpret_cast<uint32_t *>(&r0);
    out[2 * (size_t)idx + 1] = *reinterpret_cast<uint32_t *>(&r1);
}

cudaError_t pack_b(const float *W, int K, int N, uint32_t *out, cudaStream_t s) {
    int KT = (K + 15) / 16;
    int total = KT * (N / 8) * 32;
    k_pack_b<<<(total + 255) / 256, 256, 0, s>>>(W, K, N, KT, out);
    return cudaGetLastError();
}

// the tcgen05 chunk layout (hk_mlp_tc.cuh): element (k, n) of layer l's W
// (K x N, row-major FP32; K padded with zeros to 256) at chunk kc = k / 64,
// byte (n / 8) * 1024 + ((k % 64) / 8) * 128 + (n % 8) * 16 + (k % 8) * 2
__global__ void k_pack_umma(const float *__restrict__ W, int K, int N, unsigned char *__restrict__ out, int layer) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   // over 256 x N
    if (i >= kTcAK * N) return;
    const int k = i / N, n = i % N;
    const float v = k < K ? W[(size_t)k * N + n] : 0.0f;
    const int kc = k / kTcChunkK, kk = k % kTcChunkK;
    const size_t off = tc_chunk_off(layer, kc) + (size_t)(n / 8) * kTcBSbo + (size_t)(kk / 8) * 128 + (n % 8) * 16 +
                       (kk % 8) * 2;
    *reinterpret_cast<__nv_bfloat16 *>(out + off) = __float2bfloat16_rn(v);
}

size_t tc_packed_bytes() { return kTcPackedBytes; }

cudaError_t pack_umma(const float *P, unsigned char *out, cudaStream_t s) {
    const size_t offs[4] = {kOffW1, kOffW2, kOffW3, kOffW4};
    const int Ks[4] = {kMlpIn, kMlpHid, kMlpHid, kMlpHid};
    for (int l = 0; l < 4; l++) {
        const int N = (int)tc_layer_n(l);
        k_pack_umma<<<(kTcAK * N + 255) / 256, 256, 0, s>>>(P + offs[l], Ks[l], N, out, l);
    }
    return cudaGetLastError();
}

bool mlp_use_tcgen05() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("HK_MLP_PATH");
        v = (e && strcmp(e, "mma") == 0) ? 0 : 1;
    }
    return v == 1;
}

__device__ __forceinline__ void mma_bf16(float *c, const uint32_t *a, const uint32_t *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---------------------------------------------------------------------------
// Inference over host-visible batches (hk_mlp_forward): 64-row tiles, one CTA
// each, the same tile_forward the builder's k_learn runs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 1)
    k_mlp_fwd(MlpDevice M, const float *__restrict__ X, const uint32_t *rows_dev, uint32_t rows_host,
              float *__restrict__ logits) {
    extern __shared__ __align__(16) unsigned char fwd_smem[];
    const TileSmem S = tile_smem(fwd_smem);
    const uint32_t rows = rows_dev ? min(*rows_dev, rows_host) : rows_host;
    for (uint32_t row0 = blockIdx.x * kTileRows; row0 < rows; row0 += gridDim.x * kTileRows) {
        tile_forward(M, X, row0, rows, S);
        for (uint32_t i = threadIdx.x; i < (uint32_t)kTileRows * kMlpOut; i += blockDim.x) {
            const uint32_t r = row0 + i / kMlpOut;
            if (r < rows) logits[(size_t)r * kMlpOut + i % kMlpOut] = S.logits[i];
        }
        __syncthreads();
    }
}

// The same on the 5th-generation tensor cores: 128-row tiles (hk_mlp_tc.cuh);
// a pipeline wait that runs out sets *err and the CTA stops.
__global__ void __launch_bounds__(256, 1)
    k_mlp_fwd_tc(MlpDevice M, const float *__restrict__ X, const uint32_t *rows_dev, uint32_t rows_host,
                 float *__restrict__ logits, uint32_t *err) {
    extern __shared__ __align__(1024) unsigned char fwd_tc_smem[];
    const TcSmem S = tc_smem(fwd_tc_smem);
    const uint32_t rows = rows_dev ? min(*rows_dev, rows_host) : rows_host;
    if (blockIdx.x * kTcRows >= rows) return;   // no tile for this CTA: no TMEM taken
    const uint32_t tmem = tc_setup(S);
    uint32_t g = 0;
    for (uint32_t row0 = blockIdx.x * kTcRows; row0 < rows; row0 += gridDim.x * kTcRows) {
        if (!tc_tile_forward(M, X, row0, rows, S, tmem, g, err)) break;
        for (uint32_t i = threadIdx.x; i < (uint32_t)kTcRows * kMlpOut; i += blockDim.x) {
            const uint32_t m = i / kMlpOut, j = i % kMlpOut, r = row0 + m;
            if (r < rows) logits[(size_t)r * kMlpOut + j] = S.logits[m * kTcLogitStride + j];
        }
        __syncthreads();
    }
    tc_teardown(tmem);
}

cudaError_t mlp_setup() {
    // the shared-memory opt-in is per device; set it once for each
    static uint64_t attr_set = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !((attr_set >> dev) & 1u)) {
        e = cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_mlp_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_set |= 1ull << dev;
    }
    return cudaSuccess;
}

cudaError_t mlp_infer(const MlpDevice &M, const float *X, const uint32_t *rows_dev, uint32_t rows_host, float *logits,
                      int grid, cudaStream_t s, uint32_t *err) {
    cudaError_t e = mlp_setup();
    if (e != cudaSuccess) return e;
    if (mlp_use_tcgen05() && M.tcw && err) {
        const uint32_t tiles = (rows_host + kTcRows - 1) / kTcRows;
        const int g = (int)std::max<uint32_t>(1u, std::min<uint32_t>(tiles, (uint32_t)grid));
        k_mlp_fwd_tc<<<g, 256, kTcSmem, s>>>(M, X, rows_dev, rows_host, logits, err);
    } else {
        const uint32_t tiles = (rows_host + kTileRows - 1) / kTileRows;
        const int g = (int)std::max<uint32_t>(1u, std::min<uint32_t>(tiles, (uint32_t)grid));
        k_mlp_fwd<<<g, 256, kTileSmem, s>>>(M, X, rows_dev, rows_host, logits);
    }
    return cudaGetLastError();
}

__global__ void k_gather_rows(const float *__restrict__ X, const int32_t *__restrict__ y,
                              const uint32_t *__restrict__ idx, int n, float *__restrict__ Xb, int32_t *__restrict__ yb) {
    int i = blockIdx.x, r = idx[i];
    for (int c = threadIdx.x; c < kMlpIn; c += blockDim.x) Xb[(size_t)i * kMlpIn + c] = X[(size_t)r * kMlpIn + c];
    if (threadIdx.x == 0) yb[i] = y[r];
    (void)n;
}

cudaError_t gather_rows(const float *X, const int32_t *y, const uint32_t *idx, int n, float *Xb, int32_t *yb,
                        cudaStream_t s) {
    if (n) k_gather_rows<<<n, 128, 0, s>>>(X, y, idx, n, Xb, yb);
    return cudaGetLastError();
}

}  // namespace hk
