// hk_mlp_tile.cuh -- the split proposer's network on one tile of 64 rows, for
// one CTA of 256 threads (8 warps). Used by the builder's learned level kernel
// (k_learn) and by hk_mlp_forward, so both run the same arithmetic.
//
// 200 -> 256 -> 256 -> 256 -> 96, ReLU between layers, BF16 weights and
// activations on the tensor cores (mma.sync m16n8k16, FP32 accumulate), FP32
// bias. The tile's activations stay in shared memory between layers. The
// packed weights (B fragments, see pack_b) are not resident: each layer is
// staged from global memory (L2-resident, 414 KB in all) through two 32 KB
// shared-memory buffers in chunks of 8 output n-tiles x all k-tiles, the next
// chunk's 16-byte cp.async copies in flight while the current chunk is
// multiplied, so every weight crosses from L2 once per 64-row tile.
// Warp w computes rows 16 (w & 3) .. + 16 and n-tiles 4 (w >> 2) .. + 4 of each
// chunk.
#pragma once
#include <cuda_bf16.h>

#include "hk_mlp.h"

namespace hk {

constexpr int kTileRows = 64;
constexpr int kTileStride = 264;   // bf16 per activation row (256 + 8: conflict-free fragment loads)
constexpr int kStageNT = 8;        // n-tiles per staged chunk
constexpr int kStageKT = 16;       // k-tiles of the widest layer
constexpr size_t kStageWords = (size_t)kStageKT * kStageNT * 32 * 2;            // 32 KB
constexpr size_t kTileActBytes = (size_t)kTileRows * kTileStride * 2;          // 33,792
constexpr size_t kTileSmem = 2 * kTileActBytes + 2 * kStageWords * 4;          // 133,120
constexpr int kTileChunks = 4 + 4 + 4 + 2;                                      // n-chunks of the 4 layers
static_assert((size_t)kTileRows * kMlpOut * 4 <= kTileActBytes, "logits overlay the first activation buffer");

struct TileSmem {
    __nv_bfloat16 *act0, *act1;
    uint32_t *stage[2];
    float *logits;   // kTileRows x 96, over act0 once the last layer runs
};

__device__ __forceinline__ TileSmem tile_smem(unsigned char *base) {
    TileSmem S;
    S.act0 = reinterpret_cast<__nv_bfloat16 *>(base);
    S.act1 = reinterpret_cast<__nv_bfloat16 *>(base + kTileActBytes);
    S.stage[0] = reinterpret_cast<uint32_t *>(base + 2 * kTileActBytes);
    S.stage[1] = S.stage[0] + kStageWords;
    S.logits = reinterpret_cast<float *>(base);
    return S;
}

struct TileChunk {
    const uint32_t *W;     // packed weights of the layer
    const float *bias;
    int layer, KT, NT, nt0, nc;
};

__device__ __forceinline__ TileChunk tile_chunk(const MlpDevice &M, int q) {
    TileChunk c;
    if (q < 12) {
        c.layer = q / 4;
        c.KT = c.layer == 0 ? kMlpInPad / 16 : kMlpHid / 16;
        c.NT = kMlpHid / 8;
        c.nt0 = (q % 4) * kStageNT;
        c.nc = kStageNT;
        c.W = c.layer == 0 ? M.w1p : (c.layer == 1 ? M.w2p : M.w3p);
        c.bias = c.layer == 0 ? M.b1 : (c.layer == 1 ? M.b2 : M.b3);
    } else {
        c.layer = 3;
        c.KT = kMlpHid / 16;
        c.NT = kMlpOut / 8;
        c.nt0 = (q - 12) * kStageNT;
        c.nc = min(kStageNT, c.NT - c.nt0);
        c.W = M.w4p;
        c.bias = M.b4;
    }
    return c;
}

// the chunk's fragments (k-tiles 0..KT, n-tiles nt0..nt0+nc) into dst[kt][j][lane]
// (uint2 each): per k-tile nc x 256 contiguous bytes, copied in 16-byte pieces
__device__ __forceinline__ void tile_stage(uint32_t *dst, const TileChunk &c) {
    const int per_kt = c.nc * 16;
    const int total = c.KT * per_kt;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(dst);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        const int kt = i / per_kt, rem = i % per_kt;
        const uint32_t *src = c.W + ((size_t)(kt * c.NT + c.nt0) * 32) * 2 + 4 * rem;
        const uint32_t d = sbase + 4u * (uint32_t)(kt * kStageNT * 32 * 2 + 4 * rem);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void tile_mma(float *c, const uint32_t *a, const uint32_t *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// one chunk: act(in W + b) for the chunk's columns; hidden layers write BF16
// activations, the last layer FP32 logits
__device__ __forceinline__ void tile_chunk_compute(const TileChunk &c, const uint32_t *stage, const TileSmem &S) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, warp = threadIdx.x >> 5;
    const int wrow = (warp & 3) * 16;
    const int j0 = (warp >> 2) * 4, nj = min(4, c.nc - j0);
    if (nj <= 0) return;
    const __nv_bfloat16 *in = (c.layer & 1) ? S.act1 : S.act0;
    __nv_bfloat16 *out = (c.layer & 1) ? S.act0 : S.act1;
    const uint2 *Wf = reinterpret_cast<const uint2 *>(stage);
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    for (int kt = 0; kt < c.KT; kt++) {
        const int col = kt * 16 + 2 * t;
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t *>(in + (wrow + g) * kTileStride + col);
        a[1] = *reinterpret_cast<const uint32_t *>(in + (wrow + g + 8) * kTileStride + col);
        a[2] = *reinterpret_cast<const uint32_t *>(in + (wrow + g) * kTileStride + col + 8);
        a[3] = *reinterpret_cast<const uint32_t *>(in + (wrow + g + 8) * kTileStride + col + 8);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (j >= nj) break;
            const uint2 bf = Wf[(size_t)(kt * kStageNT + j0 + j) * 32 + lane];
            const uint32_t b[2] = {bf.x, bf.y};
            tile_mma(acc[j], a, b);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j >= nj) break;
        const int col = (c.nt0 + j0 + j) * 8 + 2 * t;
        const float b0 = c.bias[col], b1 = c.bias[col + 1];
        const float v0 = acc[j][0] + b0, v1 = acc[j][1] + b1, v2 = acc[j][2] + b0, v3 = acc[j][3] + b1;
        if (c.layer == 3) {
            float *L = S.logits;
            L[(wrow + g) * kMlpOut + col] = v0;
            L[(wrow + g) * kMlpOut + col + 1] = v1;
            L[(wrow + g + 8) * kMlpOut + col] = v2;
            L[(wrow + g + 8) * kMlpOut + col + 1] = v3;
        } else {
            *reinterpret_cast<__nv_bfloat162 *>(out + (wrow + g) * kTileStride + col) =
                __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
            *reinterpret_cast<__nv_bfloat162 *>(out + (wrow + g + 8) * kTileStride + col) =
                __floats2bfloat162_rn(fmaxf(v2, 0.0f), fmaxf(v3, 0.0f));
        }
    }
}

// The network on rows row0 .. row0 + 63 of X (200 FP32 features per row; rows
// at or past `rows` are zero): logits in S.logits[r][96] on return. All 256
// threads call it; it ends with a barrier.
__device__ __forceinline__ void tile_forward(const MlpDevice &M, const float *__restrict__ X, uint32_t row0,
                                             uint32_t rows, const TileSmem &S) {
    tile_stage(S.stage[0], tile_chunk(M, 0));
    for (int i = threadIdx.x; i < kTileRows * kMlpInPad; i += blockDim.x) {
        const int rr = i / kMlpInPad, c = i % kMlpInPad;
        const uint32_t r = row0 + (uint32_t)rr;
        const float v = (r < rows && c < kMlpIn) ? X[(size_t)r * kMlpIn + c] : 0.0f;
        S.act0[rr * kTileStride + c] = __float2bfloat16_rn(v);
    }
    for (int q = 0; q < kTileChunks; q++) {
        if (q + 1 < kTileChunks) {
            tile_stage(S.stage[(q + 1) & 1], tile_chunk(M, q + 1));
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();   // the chunk's weights and the previous layer's outputs are visible
        tile_chunk_compute(tile_chunk(M, q), S.stage[q & 1], S);
        __syncthreads();   // stage buffer q & 1 is refilled at iteration q + 1
    }
}

}  // namespace hk
