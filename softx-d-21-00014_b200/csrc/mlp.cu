// The small MLP of the learned coarse initial guess: three dense layers
// (n_in -> h -> h -> n_out, ReLU after the first two), BF16 weights and
// activations with FP32 accumulation on the tcgen05 GEMM (gemm.cu), FP32
// master weights trained with Adam on a mean-squared-error loss. Forward and
// backward passes are GEMMs with fused epilogues plus a few element-wise
// kernels here (transpose, loss gradient, bias gradient, Adam).
#include <cuda_bf16.h>

#include <cmath>
#include <random>

#include "device.h"
#include "mlp.h"
#include "ops.h"

namespace xg {

namespace {

__global__ void k_f32_to_bf16(const float *__restrict__ in, __nv_bfloat16 *__restrict__ out,
                              uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix (32 x 32 tiles)
__global__ void k_transpose_bf16(const __nv_bfloat16 *__restrict__ in,
                                 __nv_bfloat16 *__restrict__ out, uint32_t rows, uint32_t cols) {
    __shared__ __nv_bfloat16 t[32][33];
    const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (uint32_t j = threadIdx.y; j < 32; j += blockDim.y) {
        const uint32_t r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[j][threadIdx.x] = in[(uint64_t)r * cols + c];
    }
    __syncthreads();
    for (uint32_t j = threadIdx.y; j < 32; j += blockDim.y) {
        const uint32_t c = c0 + j, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(uint64_t)c * rows + r] = t[threadIdx.x][j];
    }
}

// dY = scale * (Y - T) in BF16; sum of squared errors into *sse
__global__ void k_mse_grad(const float *__restrict__ Y, const float *__restrict__ T,
                           __nv_bfloat16 *__restrict__ dY, uint64_t n, float scale, double *sse) {
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float d = Y[i] - T[i];
        acc += (double)d * d;
        dY[i] = __float2bfloat16_rn(scale * d);
    }
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(sse, acc);
}

// db[c] = sum over rows of G[r][c] (BF16 in, FP32 out); one thread per column
__global__ void k_colsum_bf16(const __nv_bfloat16 *__restrict__ G, float *__restrict__ db,
                              uint32_t rows, uint32_t cols) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (uint32_t r = 0; r < rows; ++r) s += __bfloat162float(G[(uint64_t)r * cols + c]);
    db[c] = s;
}

// Adam (Kingma & Ba 2015) on FP32 master parameters; bf16 receives the
// rounded weights when given.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, __nv_bfloat16 *__restrict__ bf16, uint64_t n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        if (bf16) bf16[i] = __float2bfloat16_rn(pi);
    }
}

unsigned grid_for(uint64_t n) { return (unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

void Mlp::init(uint32_t n_in_, uint32_t n_hidden, uint32_t n_out_, uint64_t seed) {
    XG_REQUIRE(n_in_ % 128 == 0 && n_hidden % 128 == 0 && n_out_ % 128 == 0 && n_in_ && n_hidden &&
                   n_out_,
               XAMG_ERR_INVALID_ARG, "mlp: layer widths must be positive multiples of 128");
    n_in = n_in_;
    h = n_hidden;
    n_out = n_out_;
    const uint32_t fan_in[3] = {n_in, h, h}, fan_out[3] = {h, h, n_out};
    std::mt19937_64 rng(seed);
    for (int l = 0; l < 3; ++l) {
        Layer &L = layer[l];
        L.in = fan_in[l];
        L.out = fan_out[l];
        // uniform(-1/sqrt(in), 1/sqrt(in)) weights, zero biases
        const float a = 1.0f / std::sqrt((float)L.in);
        std::uniform_real_distribution<float> U(-a, a);
        std::vector<float> w((size_t)L.out * L.in);
        for (auto &x : w) x = U(rng);
        upload(L.w, w, S());
        upload(L.b, std::vector<float>(L.out, 0.f), S());
        const size_t nw = w.size();
        L.gw.alloc(nw * 4);
        L.gb.alloc(L.out * 4);
        L.mw.alloc(nw * 4);
        L.vw.alloc(nw * 4);
        L.mb.alloc(L.out * 4);
        L.vb.alloc(L.out * 4);
        for (DevBuf *z : {&L.mw, &L.vw, &L.mb, &L.vb})
            XG_CUDA(cudaMemsetAsync(z->p, 0, z->bytes, S()));
        L.wt_bf.alloc(nw * 2);
        L.w_bf.alloc(nw * 2);
    }
    refresh_bf16();
    step = 0;
}

// BF16 copies of the weights: W^T as [out][in] for the forward pass, W as
// [in][out] for the input gradients.
void Mlp::refresh_bf16() {
    for (Layer &L : layer) {
        const uint64_t nw = (uint64_t)L.out * L.in;
        k_f32_to_bf16<<<grid_for(nw), 256, 0, S()>>>(L.w.as<float>(),
                                                     L.wt_bf.as<__nv_bfloat16>(), nw);
        transpose(L.wt_bf.p, L.w_bf.p, L.out, L.in);
        g_kernel_launches += 1;
    }
    XG_CUDA(cudaGetLastError());
}

void Mlp::transpose(const void *in, void *out, uint32_t rows, uint32_t cols) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    k_transpose_bf16<<<grid, block, 0, S()>>>((const __nv_bfloat16 *)in, (__nv_bfloat16 *)out,
                                             rows, cols);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

void Mlp::ensure(uint32_t batch) {
    XG_REQUIRE(batch > 0 && batch % 128 == 0, XAMG_ERR_INVALID_ARG,
               "mlp: the batch must be a positive multiple of 128");
    if (batch <= cap) return;
    cap = batch;
    const uint64_t B = batch;
    X.alloc(B * n_in * 2);
    Xt.alloc(B * n_in * 2);
    H1.alloc(B * h * 2);
    H2.alloc(B * h * 2);
    H1t.alloc(B * h * 2);
    H2t.alloc(B * h * 2);
    Y.alloc(B * n_out * 4);
    dY.alloc(B * n_out * 2);
    dYt.alloc(B * n_out * 2);
    dH2.alloc(B * h * 2);
    dH1.alloc(B * h * 2);
    dH2t.alloc(B * h * 2);
    dH1t.alloc(B * h * 2);
    sse.alloc(8);
}

void Mlp::forward(uint32_t batch, const float *Xf, float *Yout) {
    ensure(batch);
    const uint64_t B = batch;
    k_f32_to_bf16<<<grid_for(B * n_in), 256, 0, S()>>>(Xf, X.as<__nv_bfloat16>(), B * n_in);
    ++g_kernel_launches;
    using ops::mm::gemm_bf16;
    gemm_bf16(B, h, n_in, X.p, layer[0].wt_bf.p, H1.p, h, 2, layer[0].b.as<float>(), nullptr, 0,
              S());
    gemm_bf16(B, h, h, H1.p, layer[1].wt_bf.p, H2.p, h, 2, layer[1].b.as<float>(), nullptr, 0,
              S());
    gemm_bf16(B, n_out, h, H2.p, layer[2].wt_bf.p, Yout ? (void *)Yout : Y.p, n_out, 0,
              layer[2].b.as<float>(), nullptr, 0, S());
}

double Mlp::gradients(uint32_t batch, const float *Xf, const float *T) {
    forward(batch, Xf, nullptr);
    const uint64_t B = batch;
    using ops::mm::gemm_bf16;
    XG_CUDA(cudaMemsetAsync(sse.p, 0, 8, S()));
    const float scale = 2.0f / (float)(B * n_out);
    k_mse_grad<<<grid_for(B * n_out), 256, 0, S()>>>(Y.as<float>(), T, dY.as<__nv_bfloat16>(),
                                                     B * n_out, scale, sse.as<double>());
    ++g_kernel_launches;
    // layer 3: dW3^T = dY^T H2, db3 = colsum dY, dH2 = (dY W3^T^T) masked by H2 > 0
    transpose(dY.p, dYt.p, batch, n_out);
    transpose(H2.p, H2t.p, batch, h);
    gemm_bf16(n_out, h, B, dYt.p, H2t.p, layer[2].gw.p, h, 0, nullptr, nullptr, 0, S());
    k_colsum_bf16<<<(n_out + 127) / 128, 128, 0, S()>>>(dY.as<__nv_bfloat16>(),
                                                        layer[2].gb.as<float>(), batch, n_out);
    gemm_bf16(B, h, n_out, dY.p, layer[2].w_bf.p, dH2.p, h, 3, nullptr, H2.p, h, S());
    // layer 2
    transpose(dH2.p, dH2t.p, batch, h);
    transpose(H1.p, H1t.p, batch, h);
    gemm_bf16(h, h, B, dH2t.p, H1t.p, layer[1].gw.p, h, 0, nullptr, nullptr, 0, S());
    k_colsum_bf16<<<(h + 127) / 128, 128, 0, S()>>>(dH2.as<__nv_bfloat16>(),
                                                    layer[1].gb.as<float>(), batch, h);
    gemm_bf16(B, h, h, dH2.p, layer[1].w_bf.p, dH1.p, h, 3, nullptr, H1.p, h, S());
    // layer 1
    transpose(dH1.p, dH1t.p, batch, h);
    transpose(X.p, Xt.p, batch, n_in);
    gemm_bf16(h, n_in, B, dH1t.p, Xt.p, layer[0].gw.p, n_in, 0, nullptr, nullptr, 0, S());
    k_colsum_bf16<<<(h + 127) / 128, 128, 0, S()>>>(dH1.as<__nv_bfloat16>(),
                                                    layer[0].gb.as<float>(), batch, h);
    g_kernel_launches += 3;
    XG_CUDA(cudaGetLastError());
    double s = 0;
    XG_CUDA(cudaMemcpyAsync(&s, sse.p, 8, cudaMemcpyDeviceToHost, S()));
    XG_CUDA(cudaStreamSynchronize(S()));
    return s / (double)(B * n_out);
}

double Mlp::train_step(uint32_t batch, const float *Xf, const float *T, float lr) {
    const double loss = gradients(batch, Xf, T);
    ++step;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    for (Layer &L : layer) {
        const uint64_t nw = (uint64_t)L.out * L.in;
        k_adam<<<grid_for(nw), 256, 0, S()>>>(L.w.as<float>(), L.gw.as<float>(),
                                              L.mw.as<float>(), L.vw.as<float>(), nullptr, nw, lr,
                                              b1, b2, eps, c1, c2);
        k_adam<<<grid_for(L.out), 256, 0, S()>>>(L.b.as<float>(), L.gb.as<float>(),
                                                 L.mb.as<float>(), L.vb.as<float>(), nullptr,
                                                 L.out, lr, b1, b2, eps, c1, c2);
        g_kernel_launches += 2;
    }
    XG_CUDA(cudaGetLastError());
    refresh_bf16();
    return loss;
}

// Parameters in the order W1^T [h][in], b1, W2^T [h][h], b2, W3^T [out][h], b3.
uint64_t Mlp::param_count() const {
    uint64_t n = 0;
    for (const Layer &L : layer) n += (uint64_t)L.out * L.in + L.out;
    return n;
}

void Mlp::copy_params(float *host, bool set, bool grads) {
    XG_CUDA(cudaStreamSynchronize(S()));
    uint64_t off = 0;
    for (Layer &L : layer) {
        const uint64_t nw = (uint64_t)L.out * L.in;
        DevBuf &w = grads ? L.gw : L.w, &b = grads ? L.gb : L.b;
        if (set) {
            XG_CUDA(cudaMemcpy(w.p, host + off, nw * 4, cudaMemcpyHostToDevice));
            XG_CUDA(cudaMemcpy(b.p, host + off + nw, L.out * 4, cudaMemcpyHostToDevice));
        } else {
            XG_CUDA(cudaMemcpy(host + off, w.p, nw * 4, cudaMemcpyDeviceToHost));
            XG_CUDA(cudaMemcpy(host + off + nw, b.p, L.out * 4, cudaMemcpyDeviceToHost));
        }
        off += nw + L.out;
    }
    if (set && !grads) refresh_bf16();
}

}  // namespace xg
