// hk_mlp.h -- the split proposer's network: sizes, device view, kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace hk {

constexpr int kMlpIn = 200;     // features per node
constexpr int kMlpInPad = 208;  // K of the first layer rounded up to 16
constexpr int kMlpHid = 256;
constexpr int kMlpOut = 96;     // 3 axes x 32 bins (bin 0 unused)

// parameter offsets in the flat FP32 vector: W1 b1 W2 b2 W3 b3 W4 b4 (W as in x out, row-major)
constexpr size_t kOffW1 = 0;
constexpr size_t kOffB1 = kOffW1 + (size_t)kMlpIn * kMlpHid;
constexpr size_t kOffW2 = kOffB1 + kMlpHid;
constexpr size_t kOffB2 = kOffW2 + (size_t)kMlpHid * kMlpHid;
constexpr size_t kOffW3 = kOffB2 + kMlpHid;
constexpr size_t kOffB3 = kOffW3 + (size_t)kMlpHid * kMlpHid;
constexpr size_t kOffW4 = kOffB3 + kMlpHid;
constexpr size_t kOffB4 = kOffW4 + (size_t)kMlpHid * kMlpOut;
constexpr size_t kMlpParams = kOffB4 + kMlpOut;

// packed BF16 weights for inference + FP32 biases (pointers into device memory)
struct MlpDevice {
    const uint32_t *w1p, *w2p, *w3p, *w4p;   // mma.sync B fragments
    const float *b1, *b2, *b3, *b4;
    const unsigned char *tcw;                // tcgen05 weight chunks (pack_umma)
};

cudaError_t sgemm(bool ta, bool tb, const float *A, const float *B, float *C, const float *bias, int M, int N, int K,
                  int lda, int ldb, int ldc, bool relu, bool accumulate, cudaStream_t s);
cudaError_t softmax_xent(const float *Z, const int32_t *y, int rows, float *dZ, float *loss, cudaStream_t s);
cudaError_t relu_back(float *dH, const float *H, size_t n, cudaStream_t s);
cudaError_t colsum(const float *dZ, int rows, int cols, float *db, cudaStream_t s);
cudaError_t adam(float *p, const float *g, float *m, float *v, size_t n, float lr, int step, cudaStream_t s);
cudaError_t pack_b(const float *W, int K, int N, uint32_t *out, cudaStream_t s);
// all four layers (flat FP32 parameters P) into the tcgen05 chunk layout
// (hk_mlp_tc.cuh); out holds tc_packed_bytes() bytes, 16-byte aligned
size_t tc_packed_bytes();
cudaError_t pack_umma(const float *P, unsigned char *out, cudaStream_t s);
// which network kernels run: tcgen05 (true, the default) or mma.sync; read
// from HK_MLP_PATH ("mma" selects mma.sync) once
bool mlp_use_tcgen05();
// allows the inference kernel its shared memory on the current device (once
// per device; call before capturing a graph that holds the kernel)
cudaError_t mlp_setup();
// logits[r][96] for rows r < min(*rows_dev, rows_host) (rows_host alone when rows_dev is null) of X[r][200]
// (the tcgen05 kernel, when selected and M.tcw is set, reports a pipeline
// wait that ran out in *err; without err the mma.sync kernel runs)
cudaError_t mlp_infer(const MlpDevice &M, const float *X, const uint32_t *rows_dev, uint32_t rows_host, float *logits,
                      int grid, cudaStream_t s, uint32_t *err = nullptr);

cudaError_t gather_rows(const float *X, const int32_t *y, const uint32_t *idx, int n, float *Xb, int32_t *yb,
                        cudaStream_t s);

inline size_t packed_words(int K, int N) { return (size_t)((K + 15) / 16) * (N / 8) * 32 * 2; }

}  // namespace hk
