// Flat element-wise launchers, the process context, and CSR upload/download
// with XAMG's index narrowing.
#include <algorithm>
#include <cstring>

#include "ops.h"

namespace xg {

static Ctx g_ctx;
uint64_t g_kernel_launches = 0;

Ctx &ctx() {
    if (!g_ctx.ready) g_ctx.init();
    return g_ctx;
}

Ctx &ctx_uninit() { return g_ctx; }

void DVec::alloc(uint64_t n_, int nv_, bool f32_) {
    n = n_;
    nv = nv_;
    f32 = f32_;
    buf = std::make_shared<DevBuf>(n * nv * (f32 ? 4 : 8));
    if (buf->bytes) {
        XG_CUDA(cudaMemsetAsync(buf->p, 0, buf->bytes, ctx().stream));
        XG_CUDA(cudaStreamSynchronize(ctx().stream));
    }
    zero = true;
    init = false;
}

// Creates a lane's stream, scratch and pinned slots (the fields of Ctx or of
// a parked Lane).
static void lane_create(cudaStream_t &stream, DevBuf &part, DevBuf &ticket, DevBuf &out,
                        double *&pinned) {
    XG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    part.alloc((size_t)k::BMAX * 32 * 4 * sizeof(double));
    ticket.alloc(sizeof(unsigned) * 4);
    out.alloc(128 * sizeof(double));
    XG_CUDA(cudaMemsetAsync(ticket.p, 0, ticket.bytes, stream));
    XG_CUDA(cudaMallocHost((void **)&pinned, 256 * sizeof(double)));
    XG_CUDA(cudaStreamSynchronize(stream));
}

static void lane_swap(Ctx &c, Lane &l) {
    std::swap(c.stream, l.stream);
    std::swap(c.red_part, l.red_part);
    std::swap(c.red_ticket, l.red_ticket);
    std::swap(c.red_out, l.red_out);
    std::swap(c.pinned, l.pinned);
}

void Ctx::use_lane(int i) {
    XG_REQUIRE(i >= 0 && i <= 4096, XAMG_ERR_INVALID_ARG, "lane out of range");
    if (i == lane) return;
    if ((int)lanes.size() <= std::max(i, lane)) lanes.resize(std::max(i, lane) + 1);
    Lane &l = lanes[i];
    if (!l.stream) lane_create(l.stream, l.red_part, l.red_ticket, l.red_out, l.pinned);
    lane_swap(*this, lanes[lane]);  // park the current lane
    lane_swap(*this, lanes[i]);     // take lane i
    lane = i;
}

void Ctx::init() {
    if (ready) return;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        throw Error(XAMG_ERR_CUDA, std::string("no CUDA device available: ") +
                                       (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
    if (device_request >= 0) XG_CUDA(cudaSetDevice(device_request));
    XG_CUDA(cudaGetDevice(&device));
    XG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    lane_create(stream, red_part, red_ticket, red_out, pinned);
    const int rc = ops::noalloc_prepare_current_device();
    if (rc != XAMG_OK)
        throw Error(rc, "cannot resolve the scratch array of XAMG_b200_dot_noalloc");
    lane = 0;
    ready = true;
}

void Ctx::check_flags() {
    unsigned *pf = (unsigned *)(pinned + 255);
    XG_CUDA(cudaMemcpyAsync(pf, red_ticket.as<unsigned>() + 2, sizeof(unsigned),
                            cudaMemcpyDeviceToHost, stream));
    XG_CUDA(cudaStreamSynchronize(stream));
    if (*pf) {
        XG_CUDA(cudaMemsetAsync(red_ticket.as<unsigned>() + 2, 0, sizeof(unsigned), stream));
        XG_CUDA(cudaStreamSynchronize(stream));
        throw Error(XAMG_ERR_TIMEOUT, "a kernel gave up waiting for its staged matrix entries");
    }
}

void Ctx::shutdown() {
    if (!ready) return;
    use_lane(0);
    for (Lane &l : lanes) {
        if (!l.stream) continue;
        cudaStreamSynchronize(l.stream);
        l.red_part.release();
        l.red_ticket.release();
        l.red_out.release();
        if (l.pinned) cudaFreeHost(l.pinned);
        l.pinned = nullptr;
        cudaStreamDestroy(l.stream);
        l.stream = nullptr;
    }
    lanes.clear();
    cudaStreamSynchronize(stream);
    red_part.release();
    red_ticket.release();
    red_out.release();
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    cudaStreamDestroy(stream);
    stream = nullptr;
    ready = false;
}

namespace ops {

template <class Op>
static void flat(uint64_t m, const Op &op, cudaStream_t s) {
    if (m == 0) return;
    uint64_t blocks = (m + k::CT - 1) / k::CT;
    if (blocks > (uint64_t)k::BMAX * 4) blocks = (uint64_t)k::BMAX * 4;
    k::k_flat<Op><<<(unsigned)blocks, k::CT, 0, s>>>(m, op);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

void s_update(uint64_t n, double *s_, const double *r, const double *v, const double *sc, int nv,
              cudaStream_t s) {
    flat(n * nv, k::OpSUpdate{s_, r, v, sc, nv}, s);
}
void x_update(uint64_t n, double *x, const double *pa, const double *sa, const double *sc,
              int nv, cudaStream_t s) {
    flat(n * nv, k::OpXUpdate{x, pa, sa, sc, nv}, s);
}
void x_update(uint64_t n, double *x, const float *pa, const float *sa, const double *sc, int nv,
              cudaStream_t s) {
    flat(n * nv, k::OpXUpdateT<float>{x, pa, sa, sc, nv}, s);
}
void p_update(uint64_t n, double *p, const double *r, const double *v, const double *sc, int nv,
              cudaStream_t s) {
    flat(n * nv, k::OpPUpdate{p, r, v, sc, nv}, s);
}
void pcg_xr(uint64_t n, double *x, double *r, const double *p, const double *Ap,
            const double *sc, bool x_zero, int nv, cudaStream_t s) {
    flat(n * nv, k::OpPcgXR{x, r, p, Ap, sc, nv, x_zero}, s);
}
void pcg_p(uint64_t n, double *p, const double *z, const double *sc, int nv, cudaStream_t s) {
    flat(n * nv, k::OpPcgP{p, z, sc, nv}, s);
}
void rb_t(uint64_t n, double *t_, const double *z, const double *s_, const double *sc, bool z_zero,
          bool s_zero, int nv, cudaStream_t s) {
    flat(n * nv, k::OpRbT{t_, z, s_, sc, nv, z_zero, s_zero}, s);
}
void rb_r(uint64_t n, double *r, double *x, const double *t, const double *v_, const double *t_,
          const double *sc, bool x_zero, int nv, cudaStream_t s) {
    flat(n * nv, k::OpRbR{r, x, t, v_, t_, sc, nv, x_zero}, s);
}
void rb_x(uint64_t n, double *x, const double *v_, const double *t_, const double *sc,
          bool x_zero, int nv, cudaStream_t s) {
    flat(n * nv, k::OpRbX{x, v_, t_, sc, nv, x_zero}, s);
}
void rb_group2(uint64_t n, double *x, double *v_, double *z, const double *t_, const double *s_,
               const double *sc, bool merged, bool x_zero, int nv, cudaStream_t s) {
    flat(n * nv, k::OpRbG2{x, v_, z, t_, s_, sc, nv, merged, x_zero}, s);
}
void group5(uint64_t n, double *x, double *p, const double *s_, const double *r, const double *v,
            const double *sc, int nv, cudaStream_t s) {
    flat(n * nv, k::OpGroup5{x, p, s_, r, v, sc, nv}, s);
}

template <typename F>
void jacobi_zero(uint64_t n, F *x, const F *b, const F *d, F relax, int nv, cudaStream_t s) {
    flat(n * nv, k::OpJacobiZero<F>{x, b, d, relax, nv}, s);
}
template void jacobi_zero<double>(uint64_t, double *, const double *, const double *, double, int,
                                  cudaStream_t);
template void jacobi_zero<float>(uint64_t, float *, const float *, const float *, float, int,
                                 cudaStream_t);

template <typename T>
void fill(T *x, uint64_t m, T v, cudaStream_t s) {
    flat(m, k::OpFill<T>{x, v}, s);
}
template void fill<double>(double *, uint64_t, double, cudaStream_t);
template void fill<float>(float *, uint64_t, float, cudaStream_t);

template <typename TD, typename TS>
void convert(TD *d, const TS *src, uint64_t m, cudaStream_t s) {
    flat(m, k::OpConvert<TD, TS>{d, src}, s);
}
template void convert<float, double>(float *, const double *, uint64_t, cudaStream_t);
template void convert<double, float>(double *, const float *, uint64_t, cudaStream_t);
template void convert<double, double>(double *, const double *, uint64_t, cudaStream_t);
template void convert<float, float>(float *, const float *, uint64_t, cudaStream_t);

template <typename T>
void add_into(T *y, const T *x, uint64_t m, bool y_zero, cudaStream_t s) {
    flat(m, k::OpAddInto<T>{y, x, (int)y_zero}, s);
}
template void add_into<double>(double *, const double *, uint64_t, bool, cudaStream_t);
template void add_into<float>(float *, const float *, uint64_t, bool, cudaStream_t);

template <typename F>
void scale_rows(F *y, const F *d, uint64_t n, int nv, cudaStream_t s) {
    flat(n * nv, k::OpScaleRows<F>{y, d, nv}, s);
}
template void scale_rows<double>(double *, const double *, uint64_t, int, cudaStream_t);
template void scale_rows<float>(float *, const float *, uint64_t, int, cudaStream_t);

template <typename F>
void axpy_k(F *y, const F *x, const double *coef, uint64_t n, int nv, bool y_zero,
            cudaStream_t s) {
    flat(n * nv, k::OpAxpyK<F>{y, x, coef, nv, (int)y_zero}, s);
}
template void axpy_k<double>(double *, const double *, const double *, uint64_t, int, bool,
                             cudaStream_t);
template void axpy_k<float>(float *, const float *, const double *, uint64_t, int, bool,
                            cudaStream_t);

}  // namespace ops

// ---------------------------------------------------------------------------
// CSR upload with XAMG's narrowing (matrix_block::assemble, matrix.h:78-93:
// hash from encode_hash, values converted to float when reduced).
// ---------------------------------------------------------------------------
void upload_csr(const HCsr &h, DCsr &d, bool f32, int narrow, cudaStream_t s, int tune,
                bool bf16) {
    d.tune_on = tune != 0;
    d.bf16 = f32 && bf16;
    d.nrows = h.nrows;
    d.ncols = h.ncols;
    d.nnz = h.nnz();
    d.f32 = f32;
    d.hash = encode_hash(d.nnz, d.ncols, d.nrows, d.ncols, false, f32);
    const uint16_t i2 = define_int_type(d.ncols);
    d.col_bytes = narrow ? int_type_bytes(i2 > I32_TYPE ? I32_TYPE : i2) : 4;
    XG_REQUIRE(d.ncols <= UINT32_MAX && d.nnz <= UINT32_MAX, XAMG_ERR_UNSUPPORTED,
               "matrix exceeds 32-bit indexing");
    if (narrow >= 2 && d.col_bytes == 4 && h.nrows == h.ncols) {
        bool fits = true;
        for (uint64_t i = 0; i < h.nrows && fits; ++i)
            for (uint64_t j = h.row[i]; j < h.row[i + 1]; ++j) {
                const int64_t off = (int64_t)h.col[j] - (int64_t)i;
                if (off < -32767 || off > 32767) {
                    fits = false;
                    break;
                }
            }
        if (fits) d.col_bytes = -2;
    }
    for (int l = 0; l < 6; ++l) {
        const uint64_t R = (uint64_t)k::CT >> l;
        uint32_t mx = 0;
        for (uint64_t r0 = 0; r0 < h.nrows; r0 += R) {
            const uint64_t r1 = std::min<uint64_t>(r0 + R, h.nrows);
            mx = std::max<uint32_t>(mx, h.row[r1] - h.row[r0]);
        }
        d.tile_max[l] = mx;
    }
    upload(d.row, h.row, s);
    if (d.col_bytes == -2) {
        std::vector<int16_t> c(h.col.size());
        for (uint64_t i = 0; i < h.nrows; ++i)
            for (uint64_t j = h.row[i]; j < h.row[i + 1]; ++j)
                c[j] = (int16_t)((int64_t)h.col[j] - (int64_t)i);
        upload(d.col, c, s);
        XG_CUDA(cudaStreamSynchronize(s));
    } else if (d.col_bytes == 4) {
        upload(d.col, h.col, s);
    } else if (d.col_bytes == 2) {
        std::vector<uint16_t> c(h.col.begin(), h.col.end());
        upload(d.col, c, s);
        XG_CUDA(cudaStreamSynchronize(s));
    } else {
        std::vector<uint8_t> c(h.col.begin(), h.col.end());
        upload(d.col, c, s);
        XG_CUDA(cudaStreamSynchronize(s));
    }
    if (d.bf16) {
        std::vector<__nv_bfloat16> v(h.val.size());
        for (size_t i = 0; i < v.size(); ++i) v[i] = __float2bfloat16_rn((float)h.val[i]);
        upload(d.val, v, s);
        XG_CUDA(cudaStreamSynchronize(s));
    } else if (f32) {
        std::vector<float> v(h.val.size());
        for (size_t i = 0; i < v.size(); ++i) v[i] = (float)h.val[i];
        upload(d.val, v, s);
        XG_CUDA(cudaStreamSynchronize(s));
    } else {
        upload(d.val, h.val, s);
    }
    XG_CUDA(cudaStreamSynchronize(s));
}

void download_csr(const DCsr &d, uint32_t *row, void *col, void *val) {
    if (row && d.row.bytes) XG_CUDA(cudaMemcpy(row, d.row.p, d.row.bytes, cudaMemcpyDeviceToHost));
    if (col && d.col.bytes) XG_CUDA(cudaMemcpy(col, d.col.p, d.col.bytes, cudaMemcpyDeviceToHost));
    if (val && d.val.bytes) XG_CUDA(cudaMemcpy(val, d.val.p, d.val.bytes, cudaMemcpyDeviceToHost));
}

}  // namespace xg
