// hk_mlp.cu -- the learned split proposer's network (no reference
// counterpart): 200 -> 256 -> 256 -> 256 -> 96, ReLU between layers.
//
// * Inference: BF16 weights and activations on the tensor cores
//   (mma.sync m16n8k16, FP32 accumulate). One CTA owns 128 rows (8 warps x
//   16 rows); activations stay in shared memory between layers; weights are
//   packed once into the per-lane B-fragment order so that a warp reads each
//   fragment with one coalesced 8-byte load per lane.
// * Training: FP32 master weights; hand-written tiled SGEMM (with transposed
//   operands), bias / ReLU epilogues, softmax cross-entropy, ReLU backward,
//   column sums and Adam. Gradients are checked against a CPU FP32 reference.
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>
#include <cooperative_groups.h>
#include <algorithm>

#include "hk_mlp.h"

namespace hk {

namespace cg = cooperative_groups;

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

__device__ __forceinline__ void mma_bf16(float *c, const uint32_t *a, const uint32_t *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---------------------------------------------------------------------------
// Inference kernel: a cluster of kClusterN CTAs shares every 64-row tile. CTA
// r of the cluster owns the r-th quarter of each layer's output columns and
// keeps the matching slices of all four layers' packed weights resident in
// shared memory for the whole launch (staged once with 16-byte cp.async). A
// layer's outputs are written, as BF16, into the activation buffer of every
// CTA of the cluster (distributed shared memory), and a cluster barrier
// separates the layers. The logits go straight to global memory.
// Per tile a warp (row group rg of 16 rows, column half ch) runs m16n8k16
// MMAs over its CTA's n-tiles; the arithmetic per output element is the same
// MMA sequence as one CTA computing all columns.
// ---------------------------------------------------------------------------
constexpr int kClusterN = 4;
constexpr int kRowsCta = 64;      // 4 row groups of 16 x 2 column halves = 8 warps
constexpr int kActStride = 264;   // bf16 elements per activation row (256 + 8: conflict-free fragment loads)
constexpr int kKT1 = kMlpInPad / 16, kKT = kMlpHid / 16;
constexpr int kNTcH = kMlpHid / 8 / kClusterN;   // hidden n-tiles per CTA (8)
constexpr int kNTcO = kMlpOut / 8 / kClusterN;   // output n-tiles per CTA (3)
constexpr size_t kW1Words = (size_t)kKT1 * kNTcH * 32 * 2, kWHWords = (size_t)kKT * kNTcH * 32 * 2,
                 kW4Words = (size_t)kKT * kNTcO * 32 * 2;
constexpr size_t kActBytes = 2 * (size_t)kRowsCta * kActStride * 2;
constexpr size_t kInferSmem = kActBytes + 4 * (kW1Words + 2 * kWHWords + kW4Words);
static_assert(kMlpHid % (8 * kClusterN) == 0 && kMlpOut % (8 * kClusterN) == 0, "column split");

// this CTA's n-tile slice [r*NTc, (r+1)*NTc) of a packed layer (KT x NT tiles)
__device__ __forceinline__ void stage_slice(uint32_t *dst, const uint32_t *__restrict__ Wp, int KT, int NT, int NTc,
                                            int r) {
    const int chunks = KT * NTc * 16;   // 16 x 16 bytes per (k-tile, n-tile)
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(dst);
    for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
        const int tile = i >> 4, part = i & 15;
        const int kt = tile / NTc, nt = tile % NTc;
        const uint32_t *src = Wp + ((size_t)(kt * NT + r * NTc + nt) * 32) * 2 + 4 * part;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sbase + 16u * i), "l"(src) : "memory");
    }
}

// one layer, this CTA's columns: warp (rg, ch) computes 16 rows x its n-tiles
// of act(in[16 x K] W + b); hidden layers write BF16 into the act buffer of
// every CTA of the cluster, the last layer writes FP32 logits
template <bool LAST>
__device__ __forceinline__ void cluster_layer(const __nv_bfloat16 *in, int KT, const uint32_t *Ws, int NTc, int r,
                                              const float *__restrict__ bias, __nv_bfloat16 *const *out,
                                              float *__restrict__ logits, int row0, int rows) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warp = threadIdx.x >> 5;
    const int wrow = (warp & 3) * 16;
    const int half = (NTc + 1) / 2;
    const int nt0 = (warp >> 2) * half, nt1 = min(NTc, nt0 + half);
    if (nt0 >= nt1) return;
    const uint2 *Wf = reinterpret_cast<const uint2 *>(Ws);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    const int nj = nt1 - nt0;
    for (int kt = 0; kt < KT; kt++) {
        const int c = kt * 16 + 2 * t;
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t *>(in + (wrow + g) * kActStride + c);
        a[1] = *reinterpret_cast<const uint32_t *>(in + (wrow + g + 8) * kActStride + c);
        a[2] = *reinterpret_cast<const uint32_t *>(in + (wrow + g) * kActStride + c + 8);
        a[3] = *reinterpret_cast<const uint32_t *>(in + (wrow + g + 8) * kActStride + c + 8);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (j >= nj) break;
            const uint2 bf = Wf[(size_t)(kt * NTc + nt0 + j) * 32 + lane];
            uint32_t b[2] = {bf.x, bf.y};
            mma_bf16(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j >= nj) break;
        const int col = (r * NTc + nt0 + j) * 8 + 2 * t;
        float v0 = acc[j][0] + bias[col], v1 = acc[j][1] + bias[col + 1];
        float v2 = acc[j][2] + bias[col], v3 = acc[j][3] + bias[col + 1];
        if (LAST) {
            const int rr = row0 + wrow + g;
            if (rr < rows) {
                logits[(size_t)rr * kMlpOut + col] = v0;
                logits[(size_t)rr * kMlpOut + col + 1] = v1;
            }
            if (rr + 8 < rows) {
                logits[(size_t)(rr + 8) * kMlpOut + col] = v2;
                logits[(size_t)(rr + 8) * kMlpOut + col + 1] = v3;
            }
        } else {
            const __nv_bfloat162 lo = __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
            const __nv_bfloat162 hi = __floats2bfloat162_rn(fmaxf(v2, 0.0f), fmaxf(v3, 0.0f));
#pragma unroll
            for (int q = 0; q < kClusterN; q++) {
                *reinterpret_cast<__nv_bfloat162 *>(out[q] + (wrow + g) * kActStride + col) = lo;
                *reinterpret_cast<__nv_bfloat162 *>(out[q] + (wrow + g + 8) * kActStride + col) = hi;
            }
        }
    }
}

__global__ void __cluster_dims__(kClusterN, 1, 1) __launch_bounds__(256)
    k_mlp_infer(MlpDevice M, const float *__restrict__ X, const uint32_t *rows_dev, uint32_t rows_host,
                float *__restrict__ logits) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    __nv_bfloat16 *act0 = reinterpret_cast<__nv_bfloat16 *>(sm_raw);
    __nv_bfloat16 *act1 = act0 + kRowsCta * kActStride;
    uint32_t *w1 = reinterpret_cast<uint32_t *>(sm_raw + kActBytes);
    uint32_t *w2 = w1 + kW1Words, *w3 = w2 + kWHWords, *w4 = w3 + kWHWords;
    // rows_dev (device count, e.g. written by the builder) is clamped to
    // rows_host, the capacity of X and logits; the same for every CTA
    const int rows = (int)(rows_dev ? min(*rows_dev, rows_host) : rows_host);
    const int nclusters = (int)(gridDim.x / kClusterN);
    const int cid = (int)(blockIdx.x / kClusterN);
    if (cid * kRowsCta >= rows) return;   // no tile for this cluster (uniform across it)
    // the activation buffers of every CTA of the cluster
    __nv_bfloat16 *out0[kClusterN], *out1[kClusterN];
#pragma unroll
    for (int q = 0; q < kClusterN; q++) {
        out0[q] = cluster.map_shared_rank(act0, q);
        out1[q] = cluster.map_shared_rank(act1, q);
    }
    stage_slice(w1, M.w1p, kKT1, kMlpHid / 8, kNTcH, r);
    stage_slice(w2, M.w2p, kKT, kMlpHid / 8, kNTcH, r);
    stage_slice(w3, M.w3p, kKT, kMlpHid / 8, kNTcH, r);
    stage_slice(w4, M.w4p, kKT, kMlpOut / 8, kNTcO, r);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    bool waited = false;
    for (int row0 = cid * kRowsCta; row0 < rows; row0 += nclusters * kRowsCta) {
        // the tile's rows as BF16 (features 200 -> padded 208 with zeros), in
        // every CTA (each needs all input columns)
        for (int i = threadIdx.x; i < kRowsCta * kMlpInPad; i += blockDim.x) {
            const int rr = i / kMlpInPad, c = i % kMlpInPad;
            const float v = (row0 + rr < rows && c < kMlpIn) ? X[(size_t)(row0 + rr) * kMlpIn + c] : 0.0f;
            act0[rr * kActStride + c] = __float2bfloat16_rn(v);
        }
        if (!waited) {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            waited = true;
        }
        __syncthreads();
        cluster_layer<false>(act0, kKT1, w1, kNTcH, r, M.b1, out1, nullptr, row0, rows);
        cluster.sync();
        cluster_layer<false>(act1, kKT, w2, kNTcH, r, M.b2, out0, nullptr, row0, rows);
        cluster.sync();
        cluster_layer<false>(act0, kKT, w3, kNTcH, r, M.b3, out1, nullptr, row0, rows);
        cluster.sync();
        cluster_layer<true>(act1, kKT, w4, kNTcO, r, M.b4, nullptr, logits, row0, rows);
        cluster.sync();   // act0 / act1 are rewritten by the next tile
    }
    if (!waited) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

cudaError_t mlp_setup() {
    // the attribute is per device; set it once for each
    static uint64_t attr_set = 0;
    const size_t smem = kInferSmem;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !((attr_set >> dev) & 1u)) {
        e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_set |= 1ull << dev;
    }
    return cudaSuccess;
}

cudaError_t mlp_infer(const MlpDevice &M, const float *X, const uint32_t *rows_dev, uint32_t rows_host, float *logits,
                      int grid, cudaStream_t s) {
    cudaError_t e = mlp_setup();
    if (e != cudaSuccess) return e;
    // whole clusters; pass the SM count: one CTA per SM fits (the shared
    // memory holds a quarter of the weights)
    const int g = std::max(kClusterN, (grid / kClusterN) * kClusterN);
    k_mlp_infer<<<g, 256, kInferSmem, s>>>(M, X, rows_dev, rows_host, logits);
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
