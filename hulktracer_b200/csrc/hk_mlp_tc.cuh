// hk_mlp_tc.cuh -- the split proposer's network on the 5th-generation tensor
// cores (tcgen05), one tile of 128 rows per CTA of 256 threads.
//
// 200 -> 256 -> 256 -> 256 -> 96, ReLU between layers, BF16 operands, FP32
// accumulation in tensor memory (TMEM, 128 lanes = rows x 256 columns).
//   * Weights: packed once (pack_umma) into the canonical K-major layout of
//     the UMMA shared-memory descriptor without swizzle, in chunks of 64 K
//     values: chunk (layer, kc) holds the layer's N output rows x K values
//     kc*64 .. kc*64+63, 8 x 8 core matrices of 128 bytes,
//       byte(n, k) = (n / 8) * 1024 + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2.
//     Each chunk (32 KB, 12 KB for the last layer) is one bulk copy
//     (cp.async.bulk, completion counted on an mbarrier) from global memory
//     (L2-resident) into a ring of four shared-memory buffers: three chunks
//     are in flight ahead of the one being multiplied, so a tile pays the
//     copy latency about once instead of once per chunk, and the next
//     layer's first chunks arrive during the epilogue.
//   * Activations: the tile's 128 rows x 256 K values in the same canonical
//     layout (byte(m, k) = (m / 8) * 4096 + (k / 8) * 128 + (m % 8) * 16 +
//     (k % 8) * 2), rewritten in place by each layer's epilogue.
//   * One thread issues tcgen05.mma (kind::f16, M = 128, N = 256 or 96, K =
//     16 per instruction) and tcgen05.commit to an mbarrier; all 8 warps then
//     read the accumulators with tcgen05.ld (warp w: lanes 32 (w % 4) ..,
//     columns of half w / 4), add the bias, apply ReLU and store BF16 back as
//     the next layer's A operand (fence.proxy.async before the next MMA).
// Every mbarrier wait is bounded; one that runs out sets *err and the tile is
// abandoned (the caller reports the error) after the copies in flight land.
#pragma once
#include <cuda_bf16.h>

#include "hk_mlp.h"

namespace hk {

constexpr int kTcRows = 128;
constexpr int kTcAK = 256;                                   // K extent of the activation operand
constexpr uint32_t kTcASbo = kTcAK / 8 * 128;                // 4096: next 8-row group
constexpr uint32_t kTcABytes = (uint32_t)kTcRows * kTcAK * 2;   // 65536
constexpr int kTcChunkK = 64;
constexpr uint32_t kTcBSbo = kTcChunkK / 8 * 128;            // 1024: next 8 output rows
constexpr uint32_t kTcBBytes = 256u * kTcChunkK * 2;         // 32768, the largest chunk
constexpr int kTcChunks = 16;                                // 4 layers x 4 chunks of 64 K values
constexpr uint32_t kTcTmemCols = 256;
constexpr int kTcNBuf = 4;                                   // weight-chunk ring
constexpr uint32_t kTcAhead = kTcNBuf - 1;                   // chunks in flight ahead of the multiplied one
constexpr uint32_t kTcBarOff = kTcABytes + kTcNBuf * kTcBBytes;   // 196608: 8 mbarriers + the TMEM address
constexpr uint32_t kTcBiasOff = kTcBarOff + 128;                 // the four bias vectors (864 floats)
constexpr uint32_t kTcBiasN = 3 * kMlpHid + kMlpOut;
constexpr size_t kTcSmem = kTcBiasOff + kTcBiasN * 4;
constexpr uint32_t kTcSpin = 1u << 20;                       // try_wait attempts before giving up
constexpr uint32_t kErrTensorWait = 32u;                     // *err bit: a tensor-core pipeline wait ran out
// row stride of the tile's logits in shared memory: one float more than a row,
// so that lanes holding consecutive rows touch different banks
constexpr uint32_t kTcLogitStride = (uint32_t)kMlpOut + 1u;
static_assert((size_t)kTcRows * kTcLogitStride * 4 <= kTcNBuf * kTcBBytes, "logits overlay the weight buffers");
static_assert(kTcSmem <= 227 * 1024, "shared memory of one CTA");

__host__ __device__ constexpr uint32_t tc_layer_n(int l) { return l == 3 ? (uint32_t)kMlpOut : (uint32_t)kMlpHid; }
__host__ __device__ constexpr uint32_t tc_chunk_bytes(int l) { return tc_layer_n(l) * kTcChunkK * 2; }
// byte offset of chunk (l, kc) in the packed weights
__host__ __device__ constexpr size_t tc_chunk_off(int l, int kc) {
    return (size_t)(l < 3 ? l : 3) * 4 * ((size_t)kMlpHid * kTcChunkK * 2) + (size_t)kc * tc_chunk_bytes(l);
}
constexpr size_t kTcPackedBytes = tc_chunk_off(3, 4);       // 3 x 128 KB + 48 KB

// UMMA shared-memory descriptor: canonical K-major, no swizzle (layout type
// 0), start address / leading byte offset (next core matrix along K) /
// stride byte offset (next 8 rows) in 16-byte units, version 1 (bit 46)
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor, kind::f16: D F32 (bit 4), A and B BF16 (bits 7, 10),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t tc_idesc(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool tc_mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t i = 0; i < kTcSpin; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// one bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global memory into shared memory, counted on the mbarrier
__device__ __forceinline__ void tc_bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 or 32 consecutive accumulator columns of the warp's 32 lanes; the load
// and its wait are one asm statement, so no use of the registers can be
// scheduled before the wait
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

struct TcSmem {
    unsigned char *A;      // activations (canonical layout)
    unsigned char *B0;     // weight chunk ring: buffer b at B0 + b * kTcBBytes
    float *logits;         // kTcRows rows of kTcLogitStride, over the weight buffers after the last layer
    uint32_t bars;         // copy mbarriers (8 bytes each), then the MMA mbarriers
    uint32_t *tmem_addr;
    float *bias;           // b1 | b2 | b3 | b4, copied at the start of every tile
    __device__ __forceinline__ uint32_t buf(uint32_t b) const { return smem_u32(B0) + b * kTcBBytes; }
    __device__ __forceinline__ uint32_t bar_load(uint32_t b) const { return bars + 8u * b; }
    __device__ __forceinline__ uint32_t bar_mma(uint32_t b) const { return bars + 8u * (kTcNBuf + b); }
};

__device__ __forceinline__ TcSmem tc_smem(unsigned char *base) {
    TcSmem S;
    S.A = base;
    S.B0 = base + kTcABytes;
    S.bars = smem_u32(base + kTcBarOff);
    S.logits = reinterpret_cast<float *>(base + kTcABytes);
    S.tmem_addr = reinterpret_cast<uint32_t *>(base + kTcBarOff + 16 * kTcNBuf);
    S.bias = reinterpret_cast<float *>(base + kTcBiasOff);
    return S;
}

// Kernel prologue (all threads): barriers initialised by thread 0, 256 TMEM
// columns allocated by warp 0. Pair with tc_teardown.
__device__ __forceinline__ uint32_t tc_setup(const TcSmem &S) {
    if (threadIdx.x == 0) {
        for (uint32_t b = 0; b < (uint32_t)kTcNBuf; b++) {
            tc_mbar_init(S.bar_load(b), 1);
            tc_mbar_init(S.bar_mma(b), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(S.tmem_addr)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *S.tmem_addr;
}

__device__ __forceinline__ void tc_teardown(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
}

// byte offset of (row m, column k) in the activation operand
__device__ __forceinline__ uint32_t tc_a_off(uint32_t m, uint32_t k) {
    return (m >> 3) * kTcASbo + (k >> 3) * 128u + (m & 7u) * 16u + (k & 7u) * 2u;
}

// The network on rows row0 .. row0 + 127 of X (rows at or past `rows` are
// zero); logits in S.logits[r * kTcLogitStride + j] on return. `g` counts
// the chunks every earlier call of this CTA consumed: chunk g + q of the CTA
// goes to buffer (g + q) % 4 and is that buffer's use (g + q) / 4 (the
// mbarrier phase parity); it advances by kTcChunks. All 256 threads call it. Returns false
// (on every thread) when a wait ran out; *err then holds kErrTensorWait.
__device__ __forceinline__ bool tc_tile_forward(const MlpDevice &M, const float *__restrict__ X, uint32_t row0,
                                                uint32_t rows, const TcSmem &S, uint32_t tmem, uint32_t &g,
                                                uint32_t *err) {
    __shared__ uint32_t s_ok, s_issued;
    const unsigned char *__restrict__ Wp = M.tcw;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    // thread 0: copy chunk q of this tile into its buffer once the MMAs of the
    // buffer's previous chunk (kTcNBuf chunks earlier) are done
    auto issue = [&](uint32_t q) -> bool {
        const uint32_t gq = g + q, b = gq % kTcNBuf, u = gq / kTcNBuf;
        if (u >= 1 && !tc_mbar_wait(S.bar_mma(b), (u - 1) & 1u)) return false;
        const int l = (int)q / 4, kc = (int)q % 4;
        tc_bulk_load(S.buf(b), Wp + tc_chunk_off(l, kc), tc_chunk_bytes(l), S.bar_load(b));
        s_issued = q + 1;
        return true;
    };
    if (tid == 0) {
        s_ok = 1;
        s_issued = 0;
        // the buffers were last read by generic loads (the previous tile's logits)
        tc_fence_async_smem();
        for (uint32_t q = 0; q < kTcAhead && s_ok; q++)
            if (!issue(q)) s_ok = 0;
    }
    // the biases, read by every epilogue: loaded now, stored to shared memory
    // after the features (all of a thread's loads in flight at once)
    constexpr uint32_t kBiasPer = (kTcBiasN + 255u) / 256u;
    float bias_v[kBiasPer];
#pragma unroll
    for (uint32_t u = 0; u < kBiasPer; u++) {
        const uint32_t i = tid + u * blockDim.x, l = i / kMlpHid, j = i % kMlpHid;
        const float *bp = l == 0 ? M.b1 : (l == 1 ? M.b2 : (l == 2 ? M.b3 : M.b4));
        bias_v[u] = i < kTcBiasN ? bp[j] : 0.0f;
    }
    // the tile's features as BF16 in the canonical layout, K 200 .. 255 zero
    // (a row of 200 floats starts 800-byte aligned: 8 values are two float4;
    // eight loads in flight per thread before any is converted). Item i is
    // row m = (i / 256) * 8 + i % 8, values k0 = ((i / 8) % 32) * 8 .. + 7,
    // whose 16 bytes sit at tc_a_off(m, k0) = 16 i: a warp stores 512
    // consecutive bytes, and reads 8 rows x 128 bytes.
    constexpr uint32_t kStage = 8;
    for (uint32_t i0 = tid; i0 < (uint32_t)kTcRows * (kTcAK / 8); i0 += kStage * blockDim.x) {
        float4 x0[kStage], x1[kStage];
#pragma unroll
        for (uint32_t u = 0; u < kStage; u++) {
            const uint32_t i = i0 + u * blockDim.x;
            const uint32_t m = (i >> 8) * 8u + (i & 7u), k0 = ((i >> 3) & 31u) * 8u;
            const uint32_t r = row0 + m;
            x0[u] = x1[u] = make_float4(0, 0, 0, 0);
            if (i < (uint32_t)kTcRows * (kTcAK / 8) && r < rows && k0 < (uint32_t)kMlpIn) {
                const float4 *src = reinterpret_cast<const float4 *>(X + (size_t)r * kMlpIn + k0);
                x0[u] = src[0];
                x1[u] = src[1];
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < kStage; u++) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i >= (uint32_t)kTcRows * (kTcAK / 8)) break;
            const float v[8] = {x0[u].x, x0[u].y, x0[u].z, x0[u].w, x1[u].x, x1[u].y, x1[u].z, x1[u].w};
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                w[j] = *reinterpret_cast<const uint32_t *>(&h);
            }
            *reinterpret_cast<uint4 *>(S.A + 16u * i) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
#pragma unroll
    for (uint32_t u = 0; u < kBiasPer; u++)
        if (tid + u * blockDim.x < kTcBiasN) S.bias[tid + u * blockDim.x] = bias_v[u];
    tc_fence_async_smem();
    tc_fence_before();
    __syncthreads();
    const uint32_t abase = smem_u32(S.A);
    uint32_t consumed = 0;   // chunks whose copy thread 0 has waited for
    for (int l = 0; l < 4; l++) {
        const uint32_t N = tc_layer_n(l);
        const uint32_t idesc = tc_idesc(kTcRows, N);
        if (tid == 0 && s_ok) {
            tc_fence_after();
            for (int kc = 0; kc < 4 && s_ok; kc++) {
                const uint32_t q = (uint32_t)(l * 4 + kc), gq = g + q, b = gq % kTcNBuf;
                if (!tc_mbar_wait(S.bar_load(b), (gq / kTcNBuf) & 1u)) {
                    s_ok = 0;
                    break;
                }
                consumed = q + 1;
                tc_fence_after();
                const uint32_t bbase = S.buf(b);
                // layer 0 has K = 200: its last chunk has one step of real data (192 .. 207)
                const int steps = (l == 0 && kc == 3) ? 1 : 4;
                for (int s = 0; s < steps; s++) {
                    const uint64_t da = tc_sdesc(abase + (uint32_t)(kc * 8 + s * 2) * 128u, 128u, kTcASbo);
                    const uint64_t db = tc_sdesc(bbase + (uint32_t)s * 256u, 128u, kTcBSbo);
                    tc_mma(tmem, da, db, idesc, (kc > 0 || s > 0) ? 1u : 0u);
                }
                tc_commit(S.bar_mma(b));
                // refill the ring: the buffer of chunk q - 1, whose MMAs precede
                // these (a layer's last chunk was issued before the epilogue)
                if (q + kTcAhead < (uint32_t)kTcChunks && (kc != 0 || l == 0) && !issue(q + kTcAhead)) s_ok = 0;
            }
        }
        __syncthreads();
        // every thread waits for the layer's last chunk (its commit covers all
        // MMAs issued before it)
        const uint32_t glast = g + (uint32_t)(l * 4 + 3);
        bool ok = s_ok != 0;
        if (ok && !tc_mbar_wait(S.bar_mma(glast % kTcNBuf), (glast / kTcNBuf) & 1u)) ok = false;
        if (!ok) s_ok = 0;
        __syncthreads();
        if (!s_ok) break;
        // the next layer's last chunk into the buffer this layer's last chunk
        // has just freed, so that its copy runs during the epilogue
        if (tid == 0 && l < 3 && !issue((uint32_t)(l * 4 + 4 + kTcAhead))) s_ok = 0;
        tc_fence_after();
        // epilogue: warp w reads lanes 32 (w % 4) .. + 31 (rows), columns of half w / 4
        const uint32_t m = 32u * (warp & 3u) + lane;
        const uint32_t half = N / 2, c0 = (warp >> 2) * half;
        const float *bl = S.bias + (uint32_t)l * kMlpHid;
        const uint32_t trow = tmem + ((32u * (warp & 3u)) << 16);
        // columns c .. c + 15 from r: bias, ReLU and BF16 into the next
        // layer's operand, or bias into the logits after the last layer
        auto epi16 = [&](const uint32_t *r, uint32_t c) {
            if (l < 3) {
                uint32_t w[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float a = fmaxf(__uint_as_float(r[2 * j]) + bl[c + 2 * j], 0.0f);
                    const float b = fmaxf(__uint_as_float(r[2 * j + 1]) + bl[c + 2 * j + 1], 0.0f);
                    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
                    w[j] = *reinterpret_cast<const uint32_t *>(&h);
                }
                *reinterpret_cast<uint4 *>(S.A + tc_a_off(m, c)) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4 *>(S.A + tc_a_off(m, c + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
            } else {
#pragma unroll
                for (int j = 0; j < 16; j++) S.logits[m * kTcLogitStride + c + j] = __uint_as_float(r[j]) + bl[c + j];
            }
        };
        // 32 columns per TMEM load while they last (half is 128 or 48)
        uint32_t c = c0;
        for (; c + 32 <= c0 + half; c += 32) {
            uint32_t r[32];
            tc_ld32(trow + c, r);
            epi16(r, c);
            epi16(r + 16, c + 16);
        }
        if (c < c0 + half) {
            uint32_t r[16];
            tc_ld16(trow + c, r);
            epi16(r, c);
        }
        tc_fence_async_smem();
        tc_fence_before();
        __syncthreads();
    }
    if (!s_ok) {
        // let every copy this tile started land before the CTA moves on
        if (tid == 0) {
            atomicOr(err, kErrTensorWait);
            for (uint32_t q = consumed; q < s_issued; q++) {
                const uint32_t gq = g + q;
                tc_mbar_wait(S.bar_load(gq % kTcNBuf), (gq / kTcNBuf) & 1u);
            }
        }
        __syncthreads();
        g += kTcChunks;
        return false;
    }
    g += kTcChunks;
    return true;
}

}  // namespace hk
