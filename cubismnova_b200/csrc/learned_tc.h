// learned_tc.h -- tensor-core (tcgen05) convolution layers of the learned
// smoother, used by learned.cu for grid inference (see learned_tc.cu).
#pragma once

#include "cn_internal.h"

#include <cstdint>

namespace cn {
namespace nntc {

// bytes of one layer's packed BF16 weights ([27][2][16][8])
constexpr size_t kPackedWeightBytes = 27 * 512;

// kernel form: 1 (default) persistent warp-specialised pipeline, 0 one brick per CTA
void set_form(int form);
// block cells must be multiples of the 16 x 16 x 4 brick
bool supported(const int n[3]);
// FP32 [27][cin][cout] -> packed BF16 B tiles (cin, cout <= 16, zero padded)
cn_status pack_weights(const float *W, int cin, int cout, uint16_t *out, cudaStream_t st);
// hidden layer (also the first, on the packed features): BF16 activations -> (ReLU) -> BF16 activations
cn_status conv_hidden(const uint16_t *act, const int nb[3], const int n[3], const uint16_t *w, int relu,
                      uint16_t *out, int *err, cudaStream_t st);
// last layer (output channel 0) fused with p = (zero_guess ? 0 : p) + (omega x0 + y)
cn_status conv_update(const uint16_t *act, const int nb[3], const int n[3], const uint16_t *w, const float *x0,
                      int64_t xbs, float *p, int64_t pbs, float omega, int zero_guess, int *err, cudaStream_t st);
// CUDA-core forms of the first and last layers (learned_cc.cu): the first
// layer from the FP32 features (x0, x1; block stride xbs) to 16 BF16
// channels with ReLU; the last from 16 BF16 channels to the update of p.
// Weights FP32 [27][cin][cout].
cn_status conv_first_cc(const float *x0, const float *x1, int64_t xbs, const int nb[3], const int n[3],
                        const float *W1, uint16_t *out, cudaStream_t st);
cn_status conv_update_cc(const uint16_t *act, const int nb[3], const int n[3], const float *W3, const float *x0,
                         int64_t xbs, float *p, int64_t pbs, float omega, int zero_guess, cudaStream_t st);


// Training with the hidden layer on the tensor cores (learned_train_tc.cu):
// batches of B patches, x [B][2][(P+8)^3] FP32, weights W and gradients gW
// FP32 [W1 | W2 | W3].  The forward writes y [B][(P+2)^3]; the backward
// reads gc = d loss / d y and writes gW.
struct TrainBufs {
    uint16_t *h1, *h2;     // BF16 channels-last activations [B][(P+6)^3][16], [B][(P+4)^3][16]
    uint16_t *gh1, *gh2;   // their gradients (ReLU-masked)
    uint16_t *wfwd, *wbwd; // packed hidden-layer B tiles: forward, backward-data (kPackedWeightBytes each)
    float *y, *gc;         // the last layer's output and its gradient [B][(P+2)^3]
    int *err;              // device error word (bounded waits that ran out)
};
cn_status train_forward_tc(const TrainBufs &T, const float *x, const float *W, int B, int P, cudaStream_t st);
cn_status train_backward_tc(const TrainBufs &T, const float *x, const float *W, float *gW, int B, int P,
                            cudaStream_t st);

} // namespace nntc
} // namespace cn
