// The device side of a BiCGStab solve recorded as one graph (gpu_solve_graph):
// the convergence tests of base_solver::convergence_check / converged
// (solver.h:173-241) run in one-thread kernels between the iteration's
// kernels, and their verdicts drive the graph's conditional nodes (the
// iteration loop, and which of "rest of the iteration" / "final x update"
// follows), so the host launches the whole solve once and reads the
// statistics at the end.
#include "ops.h"

namespace xg {
namespace k {

// base_solver::converged (solver.h:186-241) on the device, as the host's
// host_converged computes it: float tolerances compared against double
// norms; right-hand sides that converge keep the residuals of that
// iteration; when not every one has, the converged ones are masked out of
// the alpha/omega updates (iconv).
__device__ static bool loop_converged(double *sc, double *out, const LoopCtl &c, int res_row) {
    if (!c.check) return false;
    double *iconv = sc + SC_ICONV * SC_STRIDE;
    const double *res = sc + res_row * SC_STRIDE;
    const double *res0 = sc + SC_RHO0 * SC_STRIDE;
    bool flag = true;
    for (int k = 0; k < c.nv; ++k) {
        if (iconv[k] != 0.0) {
            const double a = sqrt(res[k]);
            const double r = a / sqrt(res0[k]);
            if ((a > (double)c.abs_tol) && (r > (double)c.rel_tol)) {
                flag = false;
            } else if (out[LOOP_CONV + k] == 0.0) {
                out[LOOP_ABS + k] = a;
                out[LOOP_REL + k] = r;
                out[LOOP_CONV + k] = 1.0;
            }
        }
    }
    if (flag) return true;
    for (int k = 0; k < c.nv; ++k) iconv[k] = mul(iconv[k], (double)(out[LOOP_CONV + k] == 0.0));
    return false;
}

// begin() + started(): every right-hand side active, statistics cleared,
// the test against rho0 itself; the loop runs unless that already passes
// (its first iteration runs whatever max_iters is, as the host loop's does).
__global__ void k_loop_start(double *sc, double *out, LoopCtl c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int k = 0; k < c.nv; ++k) {
        sc[SC_ICONV * SC_STRIDE + k] = 1.0;
        out[LOOP_ABS + k] = 0.0;
        out[LOOP_REL + k] = 0.0;
        out[LOOP_CONV + k] = 0.0;
    }
    const bool done = loop_converged(sc, out, c, SC_RHO0);
    out[LOOP_ITERS] = 0.0;
    out[LOOP_DONE] = done ? 1.0 : 0.0;
    cudaGraphSetConditional(c.loop, done ? 0u : 1u);
}

// stepped(): after the iteration's residual, either the rest of the iteration
// (not converged: it runs at max_iters too, as finish() does) or the final x
// update (converged); the loop goes on while neither converged nor at
// max_iters.
__global__ void k_loop_check(double *sc, double *out, LoopCtl c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int it = (int)out[LOOP_ITERS] + 1;
    out[LOOP_ITERS] = (double)it;
    const bool done = loop_converged(sc, out, c, SC_RES);
    out[LOOP_DONE] = done ? 1.0 : 0.0;
    cudaGraphSetConditional(c.rest, done ? 0u : 1u);
    cudaGraphSetConditional(c.last, done ? 1u : 0u);
    cudaGraphSetConditional(c.loop, (!done && it < c.max_iters) ? 1u : 0u);
}

}  // namespace k

namespace ops {

void loop_start(double *sc, double *out, const k::LoopCtl &c, cudaStream_t s) {
    k::k_loop_start<<<1, 32, 0, s>>>(sc, out, c);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

void loop_check(double *sc, double *out, const k::LoopCtl &c, cudaStream_t s) {
    k::k_loop_check<<<1, 32, 0, s>>>(sc, out, c);
    XG_CUDA(cudaGetLastError());
    ++g_kernel_launches;
}

}  // namespace ops
}  // namespace xg
