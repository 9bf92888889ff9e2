// Host-side launchers of the device kernels. Each takes plain device pointers,
// the right-hand-side count nv (1, 2, 4, 8, 16 or 32) and the stream, picks the
// kernel instantiation for (value type, nv, column width) and launches it on
// the canonical schedule. None of them synchronises.
#pragma once

#include "device.h"

namespace xg {
namespace ops {

// --- SpMV family (blas2) ----------------------------------------------------
// y = A x  /  y += A x   (csr_matvec.inl:148-260 / 32-144)
// Launches a wait that must run out after limit_ns (raises the timeout flag).
void wait_selftest(uint64_t limit_ns, cudaStream_t s);

// The persistent preconditioned BiCGStab (csrc/persist.cu): whether the
// matrix's canonical blocks can all be resident at once, and the launch.
// share: canonical blocks each physical block plays (gpu_persistent).
bool pbicgstab_persist_fits(const DCsr &A, int nv, int share);
void pbicgstab_persist(const DCsr &A, const k::PersistArgs &P, int nv, int share,
                       cudaStream_t s);
// A grid barrier that one block never reaches: its waits run out after
// limit_ns and raise *flag.
void grid_selftest(unsigned *count_gen, unsigned *flag, uint64_t limit_ns, cudaStream_t s);

// The convergence tests of a BiCGStab solve recorded as one graph
// (csrc/loop.cu): after r0 = b - A x (loop_start) and after each iteration's
// residual (loop_check); they set the graph's conditional handles in c and
// keep the statistics in out (k::LOOP_* layout).
void loop_start(double *sc, double *out, const k::LoopCtl &c, cudaStream_t s);
void loop_check(double *sc, double *out, const k::LoopCtl &c, cudaStream_t s);

// Resolves the fixed scratch array of XAMG_b200_dot_noalloc and loads its
// kernels on the current device (csrc/noalloc.cu); returns an XAMG status.
int noalloc_prepare_current_device();

template <typename F>
void spmv(const DCsr &A, const F *x, F *y, int nv, bool axpy, cudaStream_t s);

// b_H = R x_double with R in float (restriction after vector::convert, mg.inl:209-214)
void spmv_f32_from_f64(const DCsr &A, const double *x, float *y, int nv, cudaStream_t s);

// r = b - A x, optionally norm[k] = (r,r)_k written to device `norm_out`
template <typename F>
void residual(const DCsr &A, const F *x, const F *b, F *r, int nv, double *norm_out,
              cudaStream_t s);

// r0 = b - A x; p = r = r0; rho0 = rho = (r0,r0)  (merged_bicgstab.inl:103-119)
void group1(const DCsr &A, const double *x, const double *b, double *r0, double *p, double *r,
            double *sc, int nv, cudaStream_t s);
// group1 when x is zero-flagged: r0 = b - 0 without the SpMV
void group1_zero(uint64_t n, const double *b, double *r0, double *p, double *r, double *sc,
                 int nv, cudaStream_t s);

// v = A pa; scal1 = (v, r0); alpha = rho/scal1
void spmv_dot_alpha(const DCsr &A, const double *pa, double *v, const double *r0, double *sc,
                    int nv, cudaStream_t s);
// ... with pa stored in float (an FP32 preconditioner's result, widened
// exactly as it is read: the same sums)
void spmv_dot_alpha(const DCsr &A, const float *pa, double *v, const double *r0, double *sc,
                    int nv, cudaStream_t s);

// t = A sa; phi, psi, theta; omega; res; alpha_c; omega_c
// PCG: Ap = A p with (p, Ap) and alpha; (r, z) and (r, r) with beta;
// x, r updates; p = z + beta p (pcg.inl:103-150)
void pcg_ap(const DCsr &A, const double *p, double *Ap, double *sc, int nv, cudaStream_t s);
void pcg_dots(uint64_t n, const double *r, const double *z, double *sc, bool first, int nv,
              cudaStream_t s);
void pcg_xr(uint64_t n, double *x, double *r, const double *p, const double *Ap,
            const double *sc, bool x_zero, int nv, cudaStream_t s);
void pcg_p(uint64_t n, double *p, const double *z, const double *sc, int nv, cudaStream_t s);
// Reordered BiCGStab (rbicgstab.inl, merged_rbicgstab.inl)
void rb_group1(uint64_t n, double *r, const double *v, const double *t, const double *r0,
               double *sc, int nv, cudaStream_t s);
void rb_t(uint64_t n, double *t_, const double *z, const double *s_, const double *sc, bool z_zero,
          bool s_zero, int nv, cudaStream_t s);
void rb_r(uint64_t n, double *r, double *x, const double *t, const double *v_, const double *t_,
          const double *sc, bool x_zero, int nv, cudaStream_t s);
void rb_x(uint64_t n, double *x, const double *v_, const double *t_, const double *sc,
          bool x_zero, int nv, cudaStream_t s);
void rb_group2(uint64_t n, double *x, double *v_, double *z, const double *t_, const double *s_,
               const double *sc, bool merged, bool x_zero, int nv, cudaStream_t s);
namespace mm {
// C[M][N] = A[M][K] * B[N][K]^T in BF16 with FP32 accumulation on the
// tcgen05 tensor cores (gemm.cu); mode 0 FP32 out (+ bias), 1 BF16 out
// (+ bias), 2 BF16 ReLU(acc + bias), 3 BF16 acc masked by aux > 0.
void gemm_bf16(uint64_t M, uint64_t N, uint64_t K, const void *A, const void *B, void *C,
               uint64_t ldc, int mode, const float *bias, const void *aux, uint64_t ld_aux,
               cudaStream_t s);
}  // namespace mm

void spmv_dot3(const DCsr &A, const double *sa, double *t, const double *s_, double *sc, int nv,
               cudaStream_t s);
void spmv_dot3(const DCsr &A, const float *sa, double *t, const double *s_, double *sc, int nv,
               cudaStream_t s);

// One Jacobi sweep xout = xin + relax*d*(b - A xin)
template <typename F>
void jacobi_sweep(const DCsr &A, const F *xin, F *xout, const F *b, const F *d, F relax, int nv,
                  cudaStream_t s);
template <typename F>
void jacobi_zero(uint64_t n, F *x, const F *b, const F *d, F relax, int nv, cudaStream_t s);

// Chebyshev steps (see ECheby0 / ECheby1 in kernels.cuh)
template <typename F>
void cheby_first(const DCsr &A, const F *x, bool x_zero, const F *b, const F *isd, F c, F *rs,
                 F *t1s, int nv, cudaStream_t s);
template <typename F>
void cheby_step(const DCsr &A, const F *t1s, const F *rs, const F *isd, F c, F *out, bool last,
                bool x_zero, int nv, cudaStream_t s);

// x = 1*(double)(P x_H) + 1*x with P in float (mg.inl:241-249)
void prolong_mixed(const DCsr &P, const float *xH, double *x, bool x_zero, int nv,
                   cudaStream_t s);

// HSGS: forward+backward sweeps over GS blocks (t = b - A_off x_old given)
template <typename F>
void hsgs_sweep(const DCsr &Adiag, const uint64_t *boff, int nblocks, const F *t, F *x,
                const F *d, const double *relax_sc, int nv, cudaStream_t s);

// Dense y = A_inv x (Direct coarse solve)
template <typename F>
void dense_apply(const F *a, uint64_t n, const F *x, F *y, int nv, cudaStream_t s);

// --- vector kernels (blas / blas_merged) -----------------------------------
template <typename F>
void dot(uint64_t n, const F *x, const F *y, double *out, int nv, cudaStream_t s);
void group2(uint64_t n, const double *t, const double *s_, double *out96, int nv,
            cudaStream_t s);
// r = s - omega*t; rho = (r, r0) -> beta, nscal, alpha_c, omega_c; with_x also
// does x = alpha_c*pa + omega_c*sa + x first.
void group4(uint64_t n, const double *s_, const double *t, const double *r0, double *r,
            double *x, const double *pa, const double *sa, bool with_x, double *sc, int nv,
            cudaStream_t s);
void group4(uint64_t n, const double *s_, const double *t, const double *r0, double *r,
            double *x, const float *pa, const float *sa, double *sc, int nv, cudaStream_t s);
void s_update(uint64_t n, double *s_, const double *r, const double *v, const double *sc, int nv,
              cudaStream_t s);
void x_update(uint64_t n, double *x, const double *pa, const double *sa, const double *sc,
              int nv, cudaStream_t s);
void x_update(uint64_t n, double *x, const float *pa, const float *sa, const double *sc, int nv,
              cudaStream_t s);
void p_update(uint64_t n, double *p, const double *r, const double *v, const double *sc, int nv,
              cudaStream_t s);
void group5(uint64_t n, double *x, double *p, const double *s_, const double *r, const double *v,
            const double *sc, int nv, cudaStream_t s);

template <typename T>
void fill(T *x, uint64_t m, T v, cudaStream_t s);
template <typename TD, typename TS>
void convert(TD *d, const TS *src, uint64_t m, cudaStream_t s);
template <typename T>
void add_into(T *y, const T *x, uint64_t m, bool y_zero, cudaStream_t s);
template <typename F>
void scale_rows(F *y, const F *d, uint64_t n, int nv, cudaStream_t s);
template <typename F>
void axpy_k(F *y, const F *x, const double *coef, uint64_t n, int nv, bool y_zero,
            cudaStream_t s);

}  // namespace ops
}  // namespace xg
