/*
 * Extension entry points of the B200 solve-phase library (libxamg_c_api.so).
 *
 * These stand beside the reference C API of xamg_c_api.h. They expose the
 * device kernels one by one (device pointers in, for kernel-level parity
 * tests and benchmarks), the setup results a caller may want to inspect
 * (narrowed index arrays, hierarchy, statistics), and the matrix generators
 * of the benchmark configurations. Each entry names the reference function
 * whose behaviour it carries, or says that it has no counterpart.
 */
#ifndef XAMG_B200_H_
#define XAMG_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference returns 0 from every call and asserts on
 * errors (api/c/xamg_c_api.cpp:170-597); here errors come back as these. */
#define XAMG_OK 0
#define XAMG_ERR_INVALID_HANDLE (-1)
#define XAMG_ERR_INVALID_ARG (-2)
#define XAMG_ERR_NV_MISMATCH (-3)
#define XAMG_ERR_CUDA (-4)
#define XAMG_ERR_BREAKDOWN (-5)
#define XAMG_ERR_TIMEOUT (-6)
#define XAMG_ERR_NOT_INITIALIZED (-7)
#define XAMG_ERR_UNSUPPORTED (-8)
#define XAMG_ERR_ALLOC (-9)
#define XAMG_ERR_INTERNAL (-10)

/* Message of the last failed call (no counterpart in the reference). */
int XAMG_b200_last_error(char *buf, size_t len);

/* Build information: returns the number of kernels compiled in and writes
 * the target architecture string (no counterpart in the reference). */
int XAMG_b200_build_info(char *buf, size_t len);

/* A CSR block resident in device memory, with XAMG's narrowed column type
 * (col_bytes = 1, 2 or 4; csr_matrix.h:47-86 with I2 in {u8,u16,u32}), or
 * col_bytes = -2: signed 16-bit offsets col - row, a form with no
 * counterpart in the reference, used for square matrices whose entries all
 * lie within 32767 of the diagonal (parameter gpu_index_compress = 2).
 * Row pointers are 32-bit. Values are double (val_f32 = 0), float (1), or
 * BF16 with float arithmetic (2: the FP32 cycle levels that parameter
 * gpu_level_bf16 selects; no counterpart in the reference). Level matrices
 * may also report 3: FP16 values with float arithmetic, each stored divided
 * by the level's power-of-two scale (parameter gpu_level_fp16 = 1 with
 * gpu_level_bf16 = L; no counterpart in the reference). A descriptor of
 * form 3 carries no scale and is not accepted as input;
 * XAMG_b200_solver_level_download returns its values widened to float with
 * the scale applied. */
typedef struct {
    uint64_t nrows, ncols, nnz;
    const uint32_t *row;
    const void *col;
    const void *val;
    int col_bytes;
    int val_f32;
} XAMG_b200_csr;

/* y = A x (mode 0, blas2::Ax_y, src/blas2/detail/csr_matvec.inl:148-260) or
 * y += A x (mode 1, blas2::Axpy, csr_matvec.inl:32-144). x and y are device
 * arrays [rows][nv] (element (i,k) at i*nv+k) of the matrix value type.
 * Each (row, k) is accumulated sequentially over the row's entries with
 * separately rounded multiply and add, as the reference does. */
int XAMG_b200_spmv(const XAMG_b200_csr *A, const void *x, void *y, int nv, int mode,
                   void *stream);

/* v = A x and dot[k] = (v, z)_k in one pass (the blas2::Ax_y + blas::dot pair
 * of merged_pbicgstab.inl:140-153). Double only; dot_out is a host array of
 * nv values; the call synchronises the stream. */
int XAMG_b200_spmv_dot(const XAMG_b200_csr *A, const double *x, double *v, const double *z,
                       double *dot_out, int nv, void *stream);

/* dot[k] = (x, y)_k over n rows (blas::dot, src/blas/detail/blas.inl:463-532)
 * in the library's fixed reduction order. Host output; synchronises. */
int XAMG_b200_dot(uint64_t n, int nv, const double *x, const double *y, double *dot_out,
                  void *stream);

/* The dot product of XAMG_b200_dot for callers that cannot allocate device
 * memory (for example an application whose device memory is owned by its own
 * pool allocator, or a latency-bound loop where a cudaMalloc, which may
 * synchronise the device, is not allowed). No counterpart in the reference.
 * It allocates nothing: its scratch is a fixed __device__ array of this
 * library (1184 x 32 partial sums, 303,104 bytes, plus a counter) whose device
 * address is looked up on the first call on each device, so that first call
 * should precede any stream capture. x, y and dot_out (nv doubles) are device
 * arrays; nv must be 1, 2, 4, 8, 16 or 32 (XAMG_ERR_INVALID_ARG otherwise).
 * The result equals XAMG_b200_dot's bit for bit. All calls share the scratch:
 * calls whose kernels overlap on the GPU race. */
int XAMG_b200_dot_noalloc(uint64_t n, int nv, const double *x, const double *y, double *dot_out,
                          void *stream);

/* merged_bicgstab_group1/2/4 (blas_merged_bicgstab.inl:32-194) on device
 * arrays; the reductions come back in host arrays of nv values. */
int XAMG_b200_group1(uint64_t n, int nv, double *r0, const double *b, double *p, double *r,
                     double *rho0_out, void *stream);
int XAMG_b200_group2(uint64_t n, int nv, const double *t, const double *s, double *phi_out,
                     double *psi_out, double *theta_out, void *stream);
int XAMG_b200_group4(uint64_t n, int nv, const double *s, const double *t, const double *r0,
                     double *r, const double *omega_host, double *rho_out, void *stream);

/* XAMG's index narrowing (bit_operations.h:119-129, csr_matrix.h:455-461). */
uint16_t XAMG_b200_define_int_type(uint64_t range);
uint16_t XAMG_b200_encode_hash(uint64_t nnz, uint64_t ncols, uint64_t block_nrows,
                               uint64_t block_ncols, int f32, int reduced_prec);

/* Matrix generators of the benchmark configurations (host arrays; return
 * the number of nonzeros, or a negative status). The arrays must hold
 * nx*ny*nz+1 row pointers and 7 (or 27) entries per row.
 *  - cube: the reference's 7-point Laplacian, examples/common/generator/cube.inl:28-174.
 *  - diffusion: variable-coefficient diffusion with per-cell coefficient
 *    kappa = exp(sigma * N(0,1)) from `seed`, 7-point finite volumes with
 *    harmonic face averages (stencil 7) or trilinear Q1 finite elements
 *    (stencil 27); aniso_z scales the z-direction conductivity. No
 *    counterpart in the reference. */
int64_t XAMG_b200_generate_cube(uint64_t nx, uint64_t ny, uint64_t nz, uint32_t *row,
                                uint32_t *col, double *val);
int64_t XAMG_b200_generate_diffusion(int stencil, uint64_t nx, uint64_t ny, uint64_t nz,
                                     double sigma, double aniso_z, uint64_t seed, uint32_t *row,
                                     uint32_t *col, double *val);

/* Solver introspection (no counterpart in the reference; it keeps the same
 * data in solver_stats, solver.h:48-66). nv entries per array. */
int XAMG_b200_solver_stats(size_t sid, int *iters, int *conv, double *abs_res, double *rel_res,
                           int nv);

/* The multigrid hierarchy a solver built and uploaded: number of levels
 * (1 when the solver has no multigrid). */
int XAMG_b200_solver_nlevels(size_t sid);

/* Shape of level matrix `which` (0 = A, 1 = R, 2 = P, 3 = the operator the
 * multigrid cycle applies on the level: A, or on level 0 the FP32 copy when
 * gpu_precond_f32 is set) as uploaded: sizes, narrowed column width, value
 * type (val_f32 as in XAMG_b200_csr), XAMG hash, eigenvalue estimates. */
int XAMG_b200_solver_level_info(size_t sid, int level, int which, uint64_t *nrows,
                                uint64_t *ncols, uint64_t *nnz, int *col_bytes, int *val_f32,
                                uint16_t *hash, double *min_eig, double *max_eig);

/* The SpMV launch shapes the autotuner (parameter gpu_spmv_tune, default 1)
 * picked for level matrix `which` (no counterpart): 24 codes, index
 * [value type is float][x type is float][log2 nv]; 0 = not tuned (yet), else
 * 1 + 9 * (right-hand sides a thread: 0 the default of 2 for double and 4 for
 * float x, 1 the other one, 2 eight for float x at nv >= 8) + 3 * (staging: 0 one
 * buffer, 1 two, 2 none) +
 * (consecutive tiles a block takes: 0 one, 1 four, 2 sixteen), or 28: one warp per row (its
 * gathers in flight together, products summed in entry order; a candidate for matrices of at
 * most 2^20 rows times nv), or 29 + 3 * (right-hand sides a thread, as above) + (staging, as
 * above): the plane walk, where a block takes tiles one grid plane apart in turn so that the x
 * rows of the planes it gathered last are still in its SM's L1 (a candidate for square
 * matrices whose rows reach a next plane; gpu_spmv_tune = 5 forces it there without
 * measuring). Only SpMVs without dot products are tuned; every shape gives the same results
 * bit for bit. */
int XAMG_b200_solver_level_tuned(size_t sid, int level, int which, uint8_t *codes);

/* Grid-stencil storage (parameter gpu_index_compress = 3; no counterpart in
 * the reference, whose CSR blocks always carry column indices). A square
 * matrix whose entries all lie on the offsets dz*S2 + dy*S + dx (|dz|, |dy|,
 * |dx| <= 1) of a 27-point box (pattern 0) or a 7-point star (pattern 1) is
 * also stored without column indices: one value array per stencil slot and
 * a bit mask of the entries each row has. The SpMVs without dot products then
 * read that copy and sum each row in the CSR order, so results are unchanged
 * bit for bit. Rows must all be sorted by column, or all store their
 * diagonal first and the rest sorted (*diag_first = 1).
 * XAMG_b200_stencil_layout runs the detection on host CSR arrays (no GPU):
 * *pattern = -1 where the matrix does not qualify.
 * XAMG_b200_solver_level_stencil reports a level matrix's copy (pattern -1:
 * none). */
/* The nv a level matrix's x-staged copy was built for (0: none; no
 * counterpart). With gpu_spmv_tune = 4 (and gpu_index_compress >= 2),
 * multigrid levels whose rows average at least 16 entries, with at least 4,096
 * rows and a tile's x rows within shared memory, get one, and their SpMVs
 * without dot products run the x-staged kernel (each tile's x rows copied once
 * into shared memory by unique column; the same results bit for bit). */
int XAMG_b200_solver_level_xstaged(size_t sid, int level, int which, int *nv);
int XAMG_b200_stencil_layout(uint64_t nrows, const uint32_t *row, const uint32_t *col,
                             int *pattern, uint32_t *S, uint32_t *S2, int *diag_first);
int XAMG_b200_solver_level_stencil(size_t sid, int level, int which, int *pattern, uint32_t *S,
                                   uint32_t *S2, int *diag_first);

/* Copy level matrix `which` back from the device exactly as stored: row
 * pointers (u32), narrowed columns (col_bytes each), values (float/double;
 * BF16 bits for val_f32 = 2; for val_f32 = 3 the FP16 values widened to
 * float with the level's scale applied, 4 bytes each). */
int XAMG_b200_solver_level_download(size_t sid, int level, int which, uint32_t *row, void *col,
                                    void *val);

/* The double-precision hierarchy the host setup built, before narrowing and
 * precision conversion (the equivalent of what hypre hands to XAMG in
 * hypre_base.inl:337-403): which = 0 A_l, 2 P_l. */
int XAMG_b200_solver_hierarchy_export(size_t sid, int level, int which, uint32_t *row,
                                      uint32_t *col, double *val);

/* Device pointers of an uploaded level matrix (which as above), for
 * running the kernel entry points on the solver's own data (no counterpart). */
int XAMG_b200_solver_level_csr(size_t sid, int level, int which, XAMG_b200_csr *out);

/* XAMG's binary system file (src/io/detail/reader.inl:47-177, read by
 * XAMG::io::read_system): u32 nrows, u32 nnz, u32 row[nrows+1], u32
 * col[nnz], f64 val[nnz], then optionally f64 b[nrows*nv] and f64
 * x[nrows*nv] ([row][rhs] interleaved). read_system_size gives the sizes to
 * allocate; read_system fills row/col/val and, when not NULL, b and x, with
 * b = 1 and x = 0 where the file holds none (as read_system does); *found
 * gets bit 0 for b read, bit 1 for x read. write_system writes the same
 * format (x only after b). The reference reads x from the start of the file
 * (reader.inl:160, SEEK_SET with a relative offset); here x is read where it
 * is stored, after b. */
int XAMG_b200_read_system_size(const char *path, uint32_t *nrows, uint32_t *nnz);
int XAMG_b200_read_system(const char *path, uint16_t nv, uint32_t *row, uint32_t *col,
                          double *val, double *b, double *x, int *found);
int XAMG_b200_write_system(const char *path, uint32_t nrows, uint32_t nnz, const uint32_t *row,
                           const uint32_t *col, const double *val, uint16_t nv, const double *b,
                           const double *x);

/* Multigrid hierarchy files (no counterpart: the reference rebuilds the
 * hierarchy through hypre on every run). save writes the host hierarchy a
 * solver's multigrid was built from (every level but the finest, which is the
 * matrix itself, the interpolations, the eigenvalue estimates) with its setup
 * parameters and a fingerprint of the matrix; load attaches such a file to a
 * constructed matrix with the same arrays, so that a solver created on it with
 * the same multigrid setup parameters skips the setup. */
int XAMG_b200_solver_hierarchy_save(size_t sid, const char *path);
int XAMG_b200_matrix_hierarchy_load(size_t mid, const char *path);

/* Dense BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation (no
 * counterpart: the dense layers of the learned coarse initial guess).
 * C[M][N] = A[M][K] * B[N][K]^T; A, B row-major BF16 on the device, C with
 * row stride ldc. mode 0: C FP32 = acc (+ bias[N] if not NULL); 1: C BF16 =
 * acc (+ bias); 2: C BF16 = max(acc + bias, 0); 3: C BF16 = acc where
 * aux[M][ld_aux] (BF16) > 0, else 0. M and N multiples of 128, K a multiple
 * of 64, pointers 16-byte aligned. */
int XAMG_b200_gemm_bf16(uint64_t M, uint64_t N, uint64_t K, const void *A, const void *B,
                        void *C, uint64_t ldc, int mode, const float *bias, const void *aux,
                        uint64_t ld_aux, void *stream);

/* The MLP of the learned coarse initial guess (no counterpart): n_in -> h ->
 * h -> n_out dense layers with ReLU, BF16 weights and activations on the
 * tcgen05 GEMM with FP32 accumulation, FP32 master weights trained by Adam on
 * the mean squared error. Widths and batches are multiples of 128. X, T, Y
 * are FP32 device arrays [batch][n_in] / [batch][n_out]. Parameters (and
 * gradients) are laid out W1^T [h][n_in], b1 [h], W2^T [h][h], b2 [h],
 * W3^T [n_out][h], b3 [n_out] in host FP32 arrays of *count values. */
int XAMG_b200_mlp_create(uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed,
                         size_t *id);
int XAMG_b200_mlp_destroy(size_t id);
int XAMG_b200_mlp_predict(size_t id, uint32_t batch, const float *X, float *Y);
int XAMG_b200_mlp_train_step(size_t id, uint32_t batch, const float *X, const float *T, float lr,
                             double *loss);
int XAMG_b200_mlp_gradients(size_t id, uint32_t batch, const float *X, const float *T,
                            float *grads, double *loss);
int XAMG_b200_mlp_params(size_t id, float *params, int set, uint64_t *count);

/* y = A x (mode 0) or y += A x (mode 1) with level matrix `which` of a
 * solver, as its solves run it: on the library's own copy, with the x-staging
 * plan it has for nv (no counterpart; the kernel-level view of the solver's
 * SpMV for tests and timing). x and y are device arrays of the level's value
 * type, nrows x nv and ncols x nv. */
int XAMG_b200_solver_level_spmv(size_t sid, int level, int which, const void *x, void *y, int nv,
                                int mode, void *stream);

/* Number of kernels this library has launched since it was loaded (no
 * counterpart; used to account for the device work of a timed region). */
uint64_t XAMG_b200_kernel_launches(void);

/* The CUDA stream every library call is ordered on (a cudaStream_t), for
 * callers that time or order their own work against it (no counterpart). */
void *XAMG_b200_stream(void);

/* Select the CUDA device the library will use; must precede XAMG_init and
 * the first call that touches the GPU (no counterpart: the reference binds
 * ranks to cores through XAMG_NUMACONF instead). */
int XAMG_b200_set_device(int device);

/* Architecture of the library's device code as the CUDA runtime reports it
 * for a kernel of the library (cudaFuncGetAttributes): binary_version 100
 * means sm_100 machine code (no counterpart in the reference). */
int XAMG_b200_kernel_arch(int *binary_version, int *ptx_version);

/* Device address of a vector's [size][nv] storage (no counterpart). */
int XAMG_b200_vector_device_ptr(size_t vid, void **ptr);

/* Exercises the bounded waits of the library's kernels (no counterpart): a
 * kernel waits on a barrier that nothing completes, gives up after `seconds`
 * (at most 1) and raises the timeout flag that every solve checks; on return
 * *timed_out is 1 and the GPU context is still usable. Kernels that stage
 * matrix entries wait at most 2 s per copy and report XAMG_ERR_TIMEOUT from
 * the solve call. */
int XAMG_b200_wait_selftest(double seconds, int *timed_out);

/* Exercises the bounded grid barrier of the persistent BiCGStab launch (no
 * counterpart): four blocks wait at a barrier that expects a fifth, each wait
 * gives up after `seconds` (at most 1) and raises the timeout flag; on return
 * *timed_out is 1 and the GPU context is still usable. The persistent solve
 * waits at most 1 s at each barrier and reports XAMG_ERR_TIMEOUT. */
int XAMG_b200_grid_selftest(double seconds, int *timed_out);

/* Solves `count` independent systems together: entry i is
 * XAMG_solver_solve2(nv[i], xids[i], bids[i], sids[i]) (xamg_c_api.h:112),
 * with the same results bit for bit, but every system runs on a stream and
 * reduction scratch of its own so that their kernels run concurrently, and
 * the merged BiCGStab forms advance in lockstep with one host
 * synchronisation per iteration for the whole batch (no counterpart in the
 * reference, which solves one system per call). Solvers and solution vectors
 * must be distinct; the call returns when every system is finished. */
int XAMG_b200_solver_solve_batch(int count, const uint16_t *nv, const size_t *xids,
                                 const size_t *bids, const size_t *sids);

#ifdef __cplusplus
}
#endif

#endif /* XAMG_B200_H_ */
