// The MLP of the learned coarse initial guess (mlp.cu): n_in -> h -> h ->
// n_out with ReLU, BF16 weights/activations, FP32 master weights and Adam.
#pragma once

#include "device.h"

namespace xg {

struct Mlp {
    struct Layer {
        uint32_t in = 0, out = 0;
        DevBuf w, b;          // FP32 master W^T [out][in], bias [out]
        DevBuf gw, gb;        // gradients (FP32)
        DevBuf mw, vw, mb, vb;  // Adam moments
        DevBuf wt_bf, w_bf;   // BF16 W^T [out][in] and W [in][out]
    };
    uint32_t n_in = 0, h = 0, n_out = 0;
    Layer layer[3];
    uint64_t step = 0;
    uint32_t cap = 0;  // batch the activation buffers are sized for
    DevBuf X, Xt, H1, H2, H1t, H2t, Y, dY, dYt, dH2, dH1, dH2t, dH1t, sse;

    void init(uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed);
    // Y = MLP(X) for `batch` rows of FP32 X [batch][n_in] into FP32 Y (or the
    // internal buffer when Y is null)
    void forward(uint32_t batch, const float *X, float *Y);
    // gradients of the mean squared error against T at the current weights;
    // returns the loss
    double gradients(uint32_t batch, const float *X, const float *T);
    // one Adam step; returns the loss before the step
    double train_step(uint32_t batch, const float *X, const float *T, float lr);
    uint64_t param_count() const;
    void copy_params(float *host, bool set, bool grads);

  private:
    void ensure(uint32_t batch);
    void refresh_bf16();
    void transpose(const void *in, void *out, uint32_t rows, uint32_t cols);
    static cudaStream_t S() { return ctx().stream; }
};

}  // namespace xg
