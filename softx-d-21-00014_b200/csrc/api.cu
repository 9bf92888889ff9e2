// The C ABI: XAMG_* functions of the reference C API
// (api/c/xamg_c_api.cpp:149-597) and the XAMG_b200_* extension entry points.
// Handles are indices into process-wide tables, as in the reference
// (xamg_c_api.cpp:66-85). Every entry point catches errors and returns a
// negative XAMG_ERR_* code; the message is kept for XAMG_b200_last_error().
#include <sys/time.h>

#include <cstring>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/xamg_c_api.h"
#include "ops.h"
#include "io.h"
#include "mlp.h"
#include "solver.h"

#ifndef XAMG_NV
#define XAMG_NV 1
#endif

namespace xg {
namespace {

std::string g_last_error;

struct PartObj {
    uint64_t size = 0;
};
struct VecObj {
    int mode = 0;
    uint64_t ext_offset = 0;
    DVec v;
    bool allocated = false;
};
struct CsrObj {
    HCsr h;
    uint64_t row_offset = 0, col_offset = 0;
};
struct MatObj {
    HCsr h;
    bool constructed = false;
    HierCache hcache;  // host multigrid hierarchies built for this matrix
    // device copies keyed by the narrowing switch and the tuning switch
    std::map<int, std::unique_ptr<DCsr>> dev;
    const DCsr *device(int narrow, int tune) {
        auto &p = dev[narrow * 2 + (tune ? 1 : 0)];
        if (!p) {
            p.reset(new DCsr());
            upload_csr(h, *p, false, narrow, ctx().stream, tune);
        }
        return p.get();
    }
};
struct SolverObj {
    std::unique_ptr<SolverHierarchy> sh;
    size_t mid = 0;
    size_t xid = (size_t)-1, bid = (size_t)-1;
    int nv = 0;
};

std::vector<std::unique_ptr<Params>> g_params;
std::vector<std::unique_ptr<std::map<std::string, std::string>>> g_ovs;
std::vector<std::unique_ptr<PartObj>> g_parts;
std::vector<std::unique_ptr<VecObj>> g_vecs;
std::vector<std::unique_ptr<CsrObj>> g_csrs;
std::vector<std::unique_ptr<MatObj>> g_mats;
std::vector<std::unique_ptr<SolverObj>> g_solvers;

template <typename T>
T &get(std::vector<std::unique_ptr<T>> &tab, size_t id, const char *what) {
    if (id >= tab.size() || !tab[id])
        throw Error(XAMG_ERR_INVALID_HANDLE, std::string("invalid ") + what + " handle " +
                                                 std::to_string(id));
    return *tab[id];
}

template <typename T>
size_t push(std::vector<std::unique_ptr<T>> &tab, T *obj) {
    tab.emplace_back(obj);
    return tab.size() - 1;
}

template <class Fn>
int guarded(Fn &&fn) {
    try {
        fn();
        return XAMG_OK;
    } catch (const Error &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return XAMG_ERR_INTERNAL;
    }
}

void check_nv(int nv) {
    XG_REQUIRE(nv_supported(nv), XAMG_ERR_NV_MISMATCH,
               "nv must be one of 1, 2, 4, 8, 16, 32 (got " + std::to_string(nv) + ")");
}

PValue pv_s(const char *s) {
    PValue v;
    v.type = 'S';
    v.s = s ? s : "";
    return v;
}
PValue pv_i(uint16_t i) {
    PValue v;
    v.type = 'I';
    v.i = i;
    return v;
}
PValue pv_f(float f) {
    PValue v;
    v.type = 'F';
    v.f = f;
    return v;
}

// A non-owning DCsr over caller device memory
struct BorrowedCsr {
    DCsr d;
    explicit BorrowedCsr(const XAMG_b200_csr *A) {
        XG_REQUIRE(A && A->row && ((A->col && A->val) || A->nnz == 0), XAMG_ERR_INVALID_ARG,
                   "null CSR descriptor");
        XG_REQUIRE(A->col_bytes == 1 || A->col_bytes == 2 || A->col_bytes == 4 ||
                       A->col_bytes == -2,
                   XAMG_ERR_INVALID_ARG, "col_bytes must be 1, 2, 4 or -2");
        d.nrows = A->nrows;
        d.ncols = A->ncols;
        d.nnz = A->nnz;
        d.col_bytes = A->col_bytes;
        XG_REQUIRE(A->val_f32 >= 0 && A->val_f32 <= 2, XAMG_ERR_INVALID_ARG,
                   "val_f32 must be 0, 1 or 2");
        d.f32 = A->val_f32 != 0;
        d.bf16 = A->val_f32 == 2;
        d.row.p = (void *)A->row;
        d.col.p = (void *)A->col;
        d.val.p = (void *)A->val;
    }
    ~BorrowedCsr() {
        d.row.p = d.col.p = d.val.p = nullptr;
    }
};

cudaStream_t pick(void *stream) { return stream ? (cudaStream_t)stream : ctx().stream; }

void read_host(const double *dev, double *host, int n, cudaStream_t s) {
    XG_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    XG_CUDA(cudaStreamSynchronize(s));
}

MultiGrid *solver_mg(size_t sid) {
    SolverObj &so = get(g_solvers, sid, "solver");
    return so.sh ? so.sh->mg : nullptr;
}

}  // namespace
}  // namespace xg

using namespace xg;

extern "C" {

// ------------------------------------------------------------------ id / init
int XAMG_id_get_proc() { return 0; }
int XAMG_id_get_nprocs() { return 1; }
void *XAMG_id_get_comm_ptr() { return nullptr; }

int XAMG_init(int argc, char **argv, char *conf) {
    (void)argc;
    (void)argv;
    (void)conf;
    return guarded([&] { ctx(); });
}

int XAMG_finalize() {
    return guarded([&] {
        g_solvers.clear();
        g_mats.clear();
        g_csrs.clear();
        g_vecs.clear();
        g_parts.clear();
        g_ovs.clear();
        g_params.clear();
        ctx().shutdown();
    });
}

int XAMG_get_nv() { return XAMG_NV; }

double XAMG_timer() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int XAMG_barrier() {
    return guarded([&] { XG_CUDA(cudaStreamSynchronize(ctx().stream)); });
}

// ------------------------------------------------------------------ params
int XAMG_param_create(XAMG_param_id *pid) {
    return guarded([&] {
        XG_REQUIRE(pid, XAMG_ERR_INVALID_ARG, "null id pointer");
        *pid = push(g_params, new Params());
    });
}
int XAMG_param_add_value_s(char *role, char *key, char *value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").add_value(role, key, pv_s(value)); });
}
int XAMG_param_add_value_i(char *role, char *key, uint16_t value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").add_value(role, key, pv_i(value)); });
}
int XAMG_param_add_value_d(char *role, char *key, float value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").add_value(role, key, pv_f(value)); });
}
int XAMG_param_change_value_s(char *role, char *key, char *value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").change_value(role, key, pv_s(value)); });
}
int XAMG_param_change_value_i(char *role, char *key, uint16_t value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").change_value(role, key, pv_i(value)); });
}
int XAMG_param_change_value_d(char *role, char *key, float value, XAMG_param_id pid) {
    return guarded([&] { get(g_params, pid, "param").change_value(role, key, pv_f(value)); });
}
int XAMG_param_forced_change_value_s(char *role, char *key, char *value, XAMG_param_id pid) {
    return guarded(
        [&] { get(g_params, pid, "param").forced_change_value(role, key, pv_s(value)); });
}
int XAMG_param_forced_change_value_i(char *role, char *key, uint16_t value, XAMG_param_id pid) {
    return guarded(
        [&] { get(g_params, pid, "param").forced_change_value(role, key, pv_i(value)); });
}
int XAMG_param_forced_change_value_d(char *role, char *key, float value, XAMG_param_id pid) {
    return guarded(
        [&] { get(g_params, pid, "param").forced_change_value(role, key, pv_f(value)); });
}
int XAMG_param_override_create(XAMG_param_override_id *ovid) {
    return guarded([&] {
        XG_REQUIRE(ovid, XAMG_ERR_INVALID_ARG, "null id pointer");
        *ovid = push(g_ovs, new std::map<std::string, std::string>());
    });
}
int XAMG_param_override_add_value(char *key, char *val, XAMG_param_override_id ovid) {
    return guarded([&] { get(g_ovs, ovid, "override").insert({key, val}); });
}
int XAMG_param_override_apply(char *role, XAMG_param_id pid, XAMG_param_override_id ovid) {
    return guarded(
        [&] { get(g_params, pid, "param").add_override(role, get(g_ovs, ovid, "override")); });
}
int XAMG_param_override_destroy(XAMG_param_override_id ovid) {
    return guarded([&] {
        if (ovid < g_ovs.size()) g_ovs[ovid].reset();
    });
}
void XAMG_param_set_default(XAMG_param_id pid) {
    guarded([&] { get(g_params, pid, "param").set_defaults(); });
}
int XAMG_param_print(XAMG_param_id pid) {
    return guarded([&] {
        std::string s = get(g_params, pid, "param").to_string();
        fputs(s.c_str(), stdout);
        fflush(stdout);
    });
}
int XAMG_param_destroy(XAMG_param_id pid) {
    return guarded([&] {
        if (pid < g_params.size()) g_params[pid].reset();
    });
}

// ------------------------------------------------------------------ part
int XAMG_part_create(XAMG_part_id *pid) {
    return guarded([&] {
        XG_REQUIRE(pid, XAMG_ERR_INVALID_ARG, "null id pointer");
        *pid = push(g_parts, new PartObj());
    });
}
int XAMG_part_construct(int size, XAMG_part_id pid) {
    return guarded([&] {
        XG_REQUIRE(size >= 0, XAMG_ERR_INVALID_ARG, "negative size");
        get(g_parts, pid, "part").size = (uint64_t)size;
    });
}
int XAMG_part_get_numa_size(XAMG_part_id pid) {
    try {
        return (int)get(g_parts, pid, "part").size;
    } catch (const Error &e) {
        g_last_error = e.what();
        return e.code;
    }
}
int XAMG_part_destroy(XAMG_part_id pid) {
    return guarded([&] {
        if (pid < g_parts.size()) g_parts[pid].reset();
    });
}

// ------------------------------------------------------------------ vectors
int XAMG_vector_create(XAMG_vector_id *vid, vector_alloc_mode mode) {
    return guarded([&] {
        XG_REQUIRE(vid, XAMG_ERR_INVALID_ARG, "null id pointer");
        VecObj *v = new VecObj();
        v->mode = (int)mode;
        *vid = push(g_vecs, v);
    });
}
int XAMG_vector_offset(uint64_t offset, XAMG_vector_id vid) {
    return guarded([&] { get(g_vecs, vid, "vector").ext_offset = offset; });
}
int XAMG_vector_alloc_d(int size, uint16_t nv, XAMG_vector_id vid) {
    return guarded([&] {
        check_nv(nv);
        XG_REQUIRE(size >= 0, XAMG_ERR_INVALID_ARG, "negative size");
        VecObj &v = get(g_vecs, vid, "vector");
        ctx();
        v.v.alloc((uint64_t)size, nv, false);
        v.allocated = true;
    });
}
int XAMG_vector_set_part(XAMG_part_id pid, XAMG_vector_id vid) {
    return guarded([&] {
        get(g_parts, pid, "part");
        get(g_vecs, vid, "vector");
    });
}
// set_const forced (xamg_c_api.cpp:342-348): the vector is written and not
// zero-flagged even for 0
int XAMG_vector_set_val_d(double val, XAMG_vector_id vid) {
    return guarded([&] {
        VecObj &v = get(g_vecs, vid, "vector");
        XG_REQUIRE(v.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
        ops::fill<double>(v.v.p<double>(), v.v.elems(), val, ctx().stream);
        v.v.zero = false;
        v.v.init = true;
    });
}
// blas::upload (blas_ext.inl:243-285): block_size rows at block_offset
int XAMG_vector_upload_d(double *ptr, uint64_t block_size, uint64_t block_offset, uint16_t nv,
                         XAMG_vector_id vid) {
    return guarded([&] {
        VecObj &v = get(g_vecs, vid, "vector");
        XG_REQUIRE(v.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
        XG_REQUIRE(nv == v.v.nv, XAMG_ERR_NV_MISMATCH, "nv differs from the vector's nv");
        XG_REQUIRE(block_offset + block_size <= v.v.n, XAMG_ERR_INVALID_ARG,
                   "block exceeds the vector");
        XG_REQUIRE(ptr || block_size == 0, XAMG_ERR_INVALID_ARG, "null host pointer");
        if (block_size)
            XG_CUDA(cudaMemcpyAsync(v.v.p<double>() + block_offset * nv, ptr,
                                    block_size * nv * sizeof(double), cudaMemcpyDefault,
                                    ctx().stream));
        XG_CUDA(cudaStreamSynchronize(ctx().stream));
        v.v.zero = false;
        v.v.init = true;
    });
}
int XAMG_vector_download_d(double *ptr, uint64_t block_size, uint64_t block_offset, uint16_t nv,
                           XAMG_vector_id vid) {
    return guarded([&] {
        VecObj &v = get(g_vecs, vid, "vector");
        XG_REQUIRE(v.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
        XG_REQUIRE(nv == v.v.nv, XAMG_ERR_NV_MISMATCH, "nv differs from the vector's nv");
        XG_REQUIRE(block_offset + block_size <= v.v.n, XAMG_ERR_INVALID_ARG,
                   "block exceeds the vector");
        if (block_size) {
            cudaPointerAttributes pa;
            const bool on_device = cudaPointerGetAttributes(&pa, ptr) == cudaSuccess &&
                                   pa.type == cudaMemoryTypeDevice;
            cudaGetLastError();
            if (v.v.zero && on_device) {
                XG_CUDA(cudaMemsetAsync(ptr, 0, block_size * nv * sizeof(double), ctx().stream));
            } else if (v.v.zero) {
                std::memset(ptr, 0, block_size * nv * sizeof(double));
            } else {
                XG_CUDA(cudaMemcpyAsync(ptr, v.v.p<double>() + block_offset * nv,
                                        block_size * nv * sizeof(double), cudaMemcpyDefault,
                                        ctx().stream));
            }
        }
        XG_CUDA(cudaStreamSynchronize(ctx().stream));
    });
}
// blas::copy of a local vector into a distributed one at its external offset
// (blas.inl:259-295)
int XAMG_vector_upload_v(XAMG_vector_id vin, XAMG_vector_id vout) {
    return guarded([&] {
        VecObj &a = get(g_vecs, vin, "vector");
        VecObj &b = get(g_vecs, vout, "vector");
        XG_REQUIRE(a.allocated && b.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
        XG_REQUIRE(a.v.nv == b.v.nv, XAMG_ERR_NV_MISMATCH, "nv differs");
        const uint64_t off = a.ext_offset >= b.ext_offset ? a.ext_offset - b.ext_offset : 0;
        XG_REQUIRE(off + a.v.n <= b.v.n, XAMG_ERR_INVALID_ARG, "source exceeds the target");
        if (a.v.zero) {
            ops::fill<double>(b.v.p<double>() + off * a.v.nv, a.v.elems(), 0.0, ctx().stream);
        } else if (a.v.n) {
            XG_CUDA(cudaMemcpyAsync(b.v.p<double>() + off * a.v.nv, a.v.p<double>(),
                                    a.v.elems() * sizeof(double), cudaMemcpyDeviceToDevice,
                                    ctx().stream));
        }
        b.v.zero = false;
        b.v.init = true;
    });
}
int XAMG_vector_destroy(XAMG_vector_id vid) {
    return guarded([&] {
        if (vid < g_vecs.size()) g_vecs[vid].reset();
    });
}

// ------------------------------------------------------------------ csr matrix
int XAMG_csr_matrix_create(XAMG_csr_matrix_id *id) {
    return guarded([&] {
        XG_REQUIRE(id, XAMG_ERR_INVALID_ARG, "null id pointer");
        *id = push(g_csrs, new CsrObj());
    });
}
int XAMG_csr_matrix_alloc(uint64_t nrows, uint64_t nnz, XAMG_csr_matrix_id id) {
    return guarded([&] {
        CsrObj &c = get(g_csrs, id, "csr_matrix");
        XG_REQUIRE(nrows < UINT32_MAX && nnz < UINT32_MAX, XAMG_ERR_UNSUPPORTED,
                   "sizes exceed 32-bit indexing");
        c.h.nrows = nrows;
        c.h.ncols = nrows;
        c.h.row.assign(nrows + 1, 0);
        c.h.col.assign(nnz, 0);
        c.h.val.assign(nnz, 0.0);
    });
}
// int -> uint32 and double copies (xamg_c_api.cpp:414-423)
int XAMG_csr_matrix_fill(int *row, int *col, double *val, XAMG_matrix_id id) {
    return guarded([&] {
        CsrObj &c = get(g_csrs, id, "csr_matrix");
        XG_REQUIRE(row && (col || c.h.col.empty()) && (val || c.h.val.empty()),
                   XAMG_ERR_INVALID_ARG, "null array");
        const uint64_t nnz = c.h.col.size();
        for (uint64_t i = 0; i <= c.h.nrows; ++i) {
            XG_REQUIRE(row[i] >= 0 && (uint64_t)row[i] <= nnz, XAMG_ERR_INVALID_ARG,
                       "row pointer out of range");
            c.h.row[i] = (uint32_t)row[i];
        }
        XG_REQUIRE(c.h.row[0] == 0 && c.h.row[c.h.nrows] == nnz, XAMG_ERR_INVALID_ARG,
                   "row pointers must start at 0 and end at nnz");
        uint64_t maxc = 0;
        for (uint64_t j = 0; j < nnz; ++j) {
            XG_REQUIRE(col[j] >= 0, XAMG_ERR_INVALID_ARG, "negative column index");
            c.h.col[j] = (uint32_t)col[j];
            maxc = std::max<uint64_t>(maxc, (uint64_t)col[j] + 1);
            c.h.val[j] = val[j];
        }
        for (uint64_t i = 0; i < c.h.nrows; ++i)
            XG_REQUIRE(c.h.row[i] <= c.h.row[i + 1], XAMG_ERR_INVALID_ARG,
                       "row pointers must not decrease");
        c.h.ncols = std::max<uint64_t>(c.h.nrows, maxc);
    });
}
int XAMG_csr_matrix_offset(int row_offset, int col_offset, XAMG_matrix_id id) {
    return guarded([&] {
        CsrObj &c = get(g_csrs, id, "csr_matrix");
        c.row_offset = (uint64_t)row_offset;
        c.col_offset = (uint64_t)col_offset;
    });
}
uint32_t XAMG_csr_matrix_get_nrows(XAMG_csr_matrix_id id) {
    if (id >= g_csrs.size() || !g_csrs[id]) return 0;
    return (uint32_t)g_csrs[id]->h.nrows;
}
int XAMG_csr_matrix_destroy(XAMG_csr_matrix_id id) {
    return guarded([&] {
        if (id < g_csrs.size()) g_csrs[id].reset();
    });
}

// ------------------------------------------------------------------ matrix
int XAMG_matrix_create(XAMG_matrix_id *mid) {
    return guarded([&] {
        XG_REQUIRE(mid, XAMG_ERR_INVALID_ARG, "null id pointer");
        *mid = push(g_mats, new MatObj());
    });
}
int XAMG_matrix_set_part(XAMG_part_id pid, XAMG_matrix_id mid) {
    return guarded([&] {
        get(g_parts, pid, "part");
        get(g_mats, mid, "matrix");
    });
}
// matrix::construct (matrix.inl:368-380): one rank holds the whole matrix as
// its diagonal block; the device copy is made when a solver first needs it
int XAMG_matrix_construct(XAMG_csr_matrix_id cid, XAMG_matrix_id mid) {
    return guarded([&] {
        CsrObj &c = get(g_csrs, cid, "csr_matrix");
        MatObj &m = get(g_mats, mid, "matrix");
        XG_REQUIRE(c.h.ncols == c.h.nrows, XAMG_ERR_UNSUPPORTED,
                   "the single-GPU solve phase needs a square matrix on one rank");
        m.h = c.h;
        m.dev.clear();
        m.hcache.clear();
        m.constructed = true;
    });
}
int XAMG_matrix_destroy(XAMG_matrix_id mid) {
    return guarded([&] {
        if (mid < g_mats.size()) g_mats[mid].reset();
    });
}

// ------------------------------------------------------------------ solvers
static void build_solver(SolverObj &so, const Params &P, int nv) {
    MatObj &m = get(g_mats, so.mid, "matrix");
    XG_REQUIRE(m.constructed, XAMG_ERR_INVALID_ARG, "matrix not constructed");
    SolverCfg c = resolve_cfg(P.get("solver"), "solver");
    const int narrow = c.gpu_index_compress;
    const DCsr *A = m.device(narrow, c.gpu_spmv_tune);
    so.sh.reset(new SolverHierarchy());
    so.sh->build(P, m.h, A, nv, &m.hcache);
    so.nv = nv;
}

int XAMG_solver_create1(XAMG_matrix_id mid, XAMG_param_id pid, XAMG_solver_id *sid) {
    return guarded([&] {
        XG_REQUIRE(sid, XAMG_ERR_INVALID_ARG, "null id pointer");
        Params &P = get(g_params, pid, "param");
        SolverObj *so = new SolverObj();
        so->mid = mid;
        std::unique_ptr<SolverObj> guard(so);
        build_solver(*so, P, XAMG_NV);
        guard.release();
        *sid = push(g_solvers, so);
    });
}

int XAMG_solver_create2(XAMG_matrix_id mid, XAMG_param_id pid, XAMG_vector_id xid,
                        XAMG_vector_id bid, XAMG_solver_id *sid) {
    return guarded([&] {
        XG_REQUIRE(sid, XAMG_ERR_INVALID_ARG, "null id pointer");
        Params &P = get(g_params, pid, "param");
        VecObj &x = get(g_vecs, xid, "vector");
        VecObj &b = get(g_vecs, bid, "vector");
        XG_REQUIRE(x.allocated && b.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
        XG_REQUIRE(x.v.nv == b.v.nv, XAMG_ERR_NV_MISMATCH, "x and b differ in nv");
        SolverObj *so = new SolverObj();
        std::unique_ptr<SolverObj> guard(so);
        so->mid = mid;
        so->xid = xid;
        so->bid = bid;
        build_solver(*so, P, x.v.nv);
        guard.release();
        *sid = push(g_solvers, so);
    });
}

// base_solver::renew_params (solver.h:277-288): override the listed values of
// the solver and preconditioner lists without rebuilding the hierarchy
int XAMG_solver_renew_params(XAMG_param_id pid, XAMG_solver_id sid) {
    return guarded([&] {
        Params &P = get(g_params, pid, "param");
        SolverObj &so = get(g_solvers, sid, "solver");
        SolverHierarchy &sh = *so.sh;
        for (auto &l : P.lists)
            for (auto &kv : l.second.kv) sh.params.lists[l.first].set(kv.first, kv.second);
        for (auto &o : P.overrides) sh.params.overrides[o.first] = o.second;
        const Params &Q = sh.params;
        SolverCfg c = resolve_cfg(Q.get("solver"), "solver");
        auto keep_gpu = [](SolverCfg &dst, const SolverCfg &src) {
            dst.gpu_index_compress = src.gpu_index_compress;
            dst.gpu_hsgs_rows = src.gpu_hsgs_rows;
            dst.gpu_spmv_tune = src.gpu_spmv_tune;
        };
        keep_gpu(c, sh.root->cfg);
        sh.root->cfg = c;
        Krylov *kr = dynamic_cast<Krylov *>(sh.root.get());
        // recorded graphs hold the old parameters in their kernels
        if (kr) {
            XG_CUDA(cudaStreamSynchronize(ctx().stream));
            kr->drop_graphs();
        }
        SolverBase *M = kr ? kr->M.get() : nullptr;
        if (M && Q.has("preconditioner")) {
            SolverCfg pc = resolve_cfg(Q.get("preconditioner"), "preconditioner");
            keep_gpu(pc, M->cfg);
            M->cfg = pc;
        }
        if (sh.mg) {
            for (size_t l = 0; l < sh.mg->pre.size(); ++l) {
                SolverCfg a = resolve_cfg(Q.get("pre_smoother", (int)l), "pre_smoother");
                SolverCfg b = resolve_cfg(Q.get("post_smoother", (int)l), "post_smoother");
                XG_REQUIRE(a.method == sh.mg->pre[l]->cfg.method &&
                               b.method == sh.mg->post[l]->cfg.method,
                           XAMG_ERR_UNSUPPORTED, "renew_params cannot change a smoother method");
                keep_gpu(a, sh.mg->pre[l]->cfg);
                keep_gpu(b, sh.mg->post[l]->cfg);
                sh.mg->pre[l]->cfg = a;
                sh.mg->post[l]->cfg = b;
            }
        }
    });
}

static void do_solve(SolverObj &so, VecObj &x, VecObj &b, int nv) {
    check_nv(nv);
    XG_REQUIRE(x.allocated && b.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
    XG_REQUIRE(x.v.nv == nv && b.v.nv == nv, XAMG_ERR_NV_MISMATCH,
               "nv differs from the vectors' nv");
    MatObj &m = get(g_mats, so.mid, "matrix");
    XG_REQUIRE(x.v.n == m.h.nrows && b.v.n == m.h.nrows, XAMG_ERR_INVALID_ARG,
               "vector size differs from the matrix size");
    if (nv != so.nv) build_solver(so, so.sh->params, nv);
    so.sh->solve(x.v, b.v);
    ctx().check_flags();
}

int XAMG_solver_solve1(uint16_t nv, XAMG_solver_id sid) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        XG_REQUIRE(so.xid != (size_t)-1, XAMG_ERR_INVALID_ARG,
                   "solve1 needs a solver created with XAMG_solver_create2");
        do_solve(so, get(g_vecs, so.xid, "vector"), get(g_vecs, so.bid, "vector"), nv);
    });
}

int XAMG_solver_solve2(uint16_t nv, XAMG_vector_id xid, XAMG_vector_id bid, XAMG_solver_id sid) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        do_solve(so, get(g_vecs, xid, "vector"), get(g_vecs, bid, "vector"), nv);
    });
}

int XAMG_b200_solver_solve_batch(int count, const uint16_t *nv, const XAMG_vector_id *xids,
                                 const XAMG_vector_id *bids, const XAMG_solver_id *sids) {
    return guarded([&] {
        XG_REQUIRE(count >= 0 && count <= 4095, XAMG_ERR_INVALID_ARG,
                   "batch size must be in [0, 4095]");
        if (count == 0) return;
        XG_REQUIRE(nv && xids && bids && sids, XAMG_ERR_INVALID_ARG, "null array");
        std::vector<SolverHierarchy *> hs;
        std::vector<DVec *> xs, bs;
        std::set<size_t> seen_s, seen_x;
        for (int i = 0; i < count; ++i) {
            SolverObj &so = get(g_solvers, sids[i], "solver");
            VecObj &x = get(g_vecs, xids[i], "vector");
            VecObj &b = get(g_vecs, bids[i], "vector");
            XG_REQUIRE(seen_s.insert(sids[i]).second && seen_x.insert(xids[i]).second,
                       XAMG_ERR_INVALID_ARG, "a solver or solution vector appears twice");
            check_nv(nv[i]);
            XG_REQUIRE(x.allocated && b.allocated, XAMG_ERR_INVALID_ARG, "vector not allocated");
            XG_REQUIRE(x.v.nv == nv[i] && b.v.nv == nv[i], XAMG_ERR_NV_MISMATCH,
                       "nv differs from the vectors' nv");
            MatObj &m = get(g_mats, so.mid, "matrix");
            XG_REQUIRE(x.v.n == m.h.nrows && b.v.n == m.h.nrows, XAMG_ERR_INVALID_ARG,
                       "vector size differs from the matrix size");
            if (nv[i] != so.nv) build_solver(so, so.sh->params, nv[i]);
            hs.push_back(so.sh.get());
            xs.push_back(&x.v);
            bs.push_back(&b.v);
        }
        solve_batch(hs, xs, bs);
    });
}

int XAMG_solver_get_convergence_info(int *conv, uint16_t nv, XAMG_solver_id sid) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        XG_REQUIRE(conv, XAMG_ERR_INVALID_ARG, "null array");
        XG_REQUIRE(nv == so.nv, XAMG_ERR_NV_MISMATCH, "nv differs from the solver's nv");
        for (int k = 0; k < nv; ++k) conv[k] = so.sh->root->st.conv[k];
    });
}

int XAMG_solver_destroy(XAMG_solver_id sid) {
    return guarded([&] {
        if (sid < g_solvers.size()) g_solvers[sid].reset();
    });
}

// ================================================================== extension
int XAMG_b200_last_error(char *buf, size_t len) {
    if (buf && len) {
        std::strncpy(buf, g_last_error.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return (int)g_last_error.size();
}

// Never launched: its attributes tell which architecture the library's
// device code was compiled for.
static __global__ void k_arch_query() {}

int XAMG_b200_kernel_arch(int *binary_version, int *ptx_version) {
    return guarded([&] {
        XG_REQUIRE(binary_version && ptx_version, XAMG_ERR_INVALID_ARG, "null pointer");
        ctx();
        cudaFuncAttributes a;
        XG_CUDA(cudaFuncGetAttributes(&a, k_arch_query));
        *binary_version = a.binaryVersion;
        *ptx_version = a.ptxVersion;
    });
}

int XAMG_b200_build_info(char *buf, size_t len) {
    const char *s = "sm_100a";
    if (buf && len) {
        std::strncpy(buf, s, len - 1);
        buf[len - 1] = 0;
    }
    return 1;
}

int XAMG_b200_spmv(const XAMG_b200_csr *A, const void *x, void *y, int nv, int mode,
                   void *stream) {
    return guarded([&] {
        check_nv(nv);
        BorrowedCsr B(A);
        cudaStream_t s = pick(stream);
        if (B.d.f32)
            ops::spmv<float>(B.d, (const float *)x, (float *)y, nv, mode == 1, s);
        else
            ops::spmv<double>(B.d, (const double *)x, (double *)y, nv, mode == 1, s);
    });
}

int XAMG_b200_spmv_dot(const XAMG_b200_csr *A, const double *x, double *v, const double *z,
                       double *dot_out, int nv, void *stream) {
    return guarded([&] {
        check_nv(nv);
        BorrowedCsr B(A);
        XG_REQUIRE(!B.d.f32, XAMG_ERR_INVALID_ARG, "spmv_dot is double only");
        cudaStream_t s = pick(stream);
        DevBuf sc(k::SC_COUNT * k::SC_STRIDE * sizeof(double));
        XG_CUDA(cudaMemsetAsync(sc.p, 0, sc.bytes, s));
        ops::spmv_dot_alpha(B.d, x, v, z, sc.as<double>(), nv, s);
        read_host(sc.as<double>() + k::SC_SCAL1 * k::SC_STRIDE, dot_out, nv, s);
    });
}

int XAMG_b200_dot(uint64_t n, int nv, const double *x, const double *y, double *dot_out,
                  void *stream) {
    return guarded([&] {
        check_nv(nv);
        cudaStream_t s = pick(stream);
        double *o = ctx().red_out.as<double>();
        if (n == 0) {
            for (int k = 0; k < nv; ++k) dot_out[k] = 0.0;
            return;
        }
        ops::dot<double>(n, x, y, o, nv, s);
        read_host(o, dot_out, nv, s);
    });
}

int XAMG_b200_group1(uint64_t n, int nv, double *r0, const double *b, double *p, double *r,
                     double *rho0_out, void *stream) {
    return guarded([&] {
        check_nv(nv);
        cudaStream_t s = pick(stream);
        // group1 on a given r0 (= A x): r0 = b - r0 via an identity "matrix"
        // is not needed; run the element-wise form with r0 as the SpMV result
        DevBuf sc(k::SC_COUNT * k::SC_STRIDE * sizeof(double));
        XG_CUDA(cudaMemsetAsync(sc.p, 0, sc.bytes, s));
        // build a diagonal identity CSR so that A*r0 = r0 exactly (1*x = x)
        std::vector<uint32_t> row(n + 1), col(n);
        std::vector<double> one(n, 1.0);
        for (uint64_t i = 0; i <= n; ++i) row[i] = (uint32_t)i;
        for (uint64_t i = 0; i < n; ++i) col[i] = (uint32_t)i;
        HCsr I;
        I.nrows = I.ncols = n;
        I.row = row;
        I.col = col;
        I.val = one;
        DCsr D;
        upload_csr(I, D, false, false, s);
        DevBuf tmp(n * nv * sizeof(double));
        XG_CUDA(cudaMemcpyAsync(tmp.p, r0, n * nv * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ops::group1(D, tmp.as<double>(), b, r0, p, r, sc.as<double>(), nv, s);
        read_host(sc.as<double>() + k::SC_RHO0 * k::SC_STRIDE, rho0_out, nv, s);
    });
}

int XAMG_b200_group2(uint64_t n, int nv, const double *t, const double *s_, double *phi_out,
                     double *psi_out, double *theta_out, void *stream) {
    return guarded([&] {
        check_nv(nv);
        cudaStream_t s = pick(stream);
        double *o = ctx().red_out.as<double>();
        ops::group2(n, t, s_, o, nv, s);
        double h[96];
        read_host(o, h, 96, s);
        for (int k = 0; k < nv; ++k) {
            phi_out[k] = h[k];
            psi_out[k] = h[32 + k];
            theta_out[k] = h[64 + k];
        }
    });
}

int XAMG_b200_group4(uint64_t n, int nv, const double *s_, const double *t, const double *r0,
                     double *r, const double *omega_host, double *rho_out, void *stream) {
    return guarded([&] {
        check_nv(nv);
        cudaStream_t s = pick(stream);
        std::vector<double> h(k::SC_COUNT * k::SC_STRIDE, 0.0);
        for (int k2 = 0; k2 < nv; ++k2) {
            h[k::SC_OMEGA * k::SC_STRIDE + k2] = omega_host[k2];
            h[k::SC_RHO * k::SC_STRIDE + k2] = 1.0;
            h[k::SC_ALPHA * k::SC_STRIDE + k2] = 1.0;
        }
        DevBuf sc(h.size() * sizeof(double));
        XG_CUDA(cudaMemcpyAsync(sc.p, h.data(), sc.bytes, cudaMemcpyHostToDevice, s));
        ops::group4(n, s_, t, r0, r, nullptr, nullptr, nullptr, false, sc.as<double>(), nv, s);
        read_host(sc.as<double>() + k::SC_SCAL1 * k::SC_STRIDE, rho_out, nv, s);
    });
}

uint16_t XAMG_b200_define_int_type(uint64_t range) { return define_int_type(range); }

uint16_t XAMG_b200_encode_hash(uint64_t nnz, uint64_t ncols, uint64_t bnrows, uint64_t bncols,
                               int f32, int reduced) {
    return encode_hash(nnz, ncols, bnrows, bncols, f32 != 0, reduced != 0);
}

int XAMG_b200_solver_stats(size_t sid, int *iters, int *conv, double *abs_res, double *rel_res,
                           int nv) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        const Stats &st = so.sh->root->st;
        XG_REQUIRE(nv == so.nv, XAMG_ERR_NV_MISMATCH, "nv differs from the solver's nv");
        if (iters) *iters = st.iters;
        for (int k = 0; k < nv; ++k) {
            if (conv) conv[k] = k < (int)st.conv.size() ? st.conv[k] : 0;
            if (abs_res) abs_res[k] = k < (int)st.abs_res.size() ? st.abs_res[k] : 0.0;
            if (rel_res) rel_res[k] = k < (int)st.rel_res.size() ? st.rel_res[k] : 0.0;
        }
    });
}

int XAMG_b200_solver_nlevels(size_t sid) {
    try {
        MultiGrid *mg = solver_mg(sid);
        return mg ? (int)mg->L.size() : 1;
    } catch (const Error &e) {
        g_last_error = e.what();
        return e.code;
    }
}

static const DCsr &level_matrix(size_t sid, int level, int which) {
    SolverObj &so = get(g_solvers, sid, "solver");
    MultiGrid *mg = so.sh->mg;
    if (!mg) {
        XG_REQUIRE(level == 0 && which == 0, XAMG_ERR_INVALID_ARG, "no multigrid hierarchy");
        return *so.sh->A;
    }
    XG_REQUIRE(level >= 0 && level < (int)mg->L.size(), XAMG_ERR_INVALID_ARG, "bad level");
    XG_REQUIRE(which >= 0 && which <= 3, XAMG_ERR_INVALID_ARG, "which must be 0, 1, 2 or 3");
    if (which == 0) return level == 0 ? *so.sh->A : mg->L[level].A;
    if (which == 3) return level == 0 && !mg->full32 ? *so.sh->A : mg->L[level].A;
    XG_REQUIRE(level + 1 < (int)mg->L.size(), XAMG_ERR_INVALID_ARG, "coarsest level has no R/P");
    return which == 1 ? mg->L[level].R : mg->L[level].P;
}

int XAMG_b200_solver_level_info(size_t sid, int level, int which, uint64_t *nrows,
                                uint64_t *ncols, uint64_t *nnz, int *col_bytes, int *val_f32,
                                uint16_t *hash, double *min_eig, double *max_eig) {
    return guarded([&] {
        const DCsr &d = level_matrix(sid, level, which);
        if (nrows) *nrows = d.nrows;
        if (ncols) *ncols = d.ncols;
        if (nnz) *nnz = d.nnz;
        if (col_bytes) *col_bytes = d.col_bytes;
        if (val_f32) *val_f32 = d.fp16 ? 3 : d.bf16 ? 2 : d.f32 ? 1 : 0;
        if (hash) *hash = d.hash;
        MultiGrid *mg = solver_mg(sid);
        if (min_eig) *min_eig = mg ? mg->L[level].min_eig : 0.0;
        if (max_eig) *max_eig = mg ? mg->L[level].max_eig : 0.0;
    });
}

int XAMG_b200_stencil_layout(uint64_t nrows, const uint32_t *row, const uint32_t *col,
                             int *pattern, uint32_t *S, uint32_t *S2, int *diag_first) {
    return guarded([&] {
        XG_REQUIRE(row && col && pattern && S && S2 && diag_first, XAMG_ERR_INVALID_ARG,
                   "null array");
        HCsr h;
        h.nrows = h.ncols = nrows;
        h.row.assign(row, row + nrows + 1);
        h.col.assign(col, col + h.row[nrows]);
        h.val.assign(h.col.size(), 0.0);
        int pat = -1;
        uint32_t s1 = 0, s2 = 0;
        bool df = false;
        if (!stencil_layout(h, pat, s1, s2, df)) pat = -1;
        *pattern = pat;
        *S = s1;
        *S2 = s2;
        *diag_first = df ? 1 : 0;
    });
}

int XAMG_b200_solver_level_stencil(size_t sid, int level, int which, int *pattern, uint32_t *S,
                                   uint32_t *S2, int *diag_first) {
    return guarded([&] {
        const DCsr &d = level_matrix(sid, level, which);
        if (pattern) *pattern = d.st_pat;
        if (S) *S = d.st_S;
        if (S2) *S2 = d.st_S2;
        if (diag_first) *diag_first = d.st_diag_first ? 1 : 0;
    });
}

int XAMG_b200_solver_level_xstaged(size_t sid, int level, int which, int *nv) {
    return guarded([&] {
        XG_REQUIRE(nv, XAMG_ERR_INVALID_ARG, "null pointer");
        *nv = level_matrix(sid, level, which).xs_nv;
    });
}

int XAMG_b200_solver_level_tuned(size_t sid, int level, int which, uint8_t *codes) {
    return guarded([&] {
        XG_REQUIRE(codes, XAMG_ERR_INVALID_ARG, "null array");
        const DCsr &d = level_matrix(sid, level, which);
        std::memcpy(codes, &d.tuned[0][0][0], 24);
    });
}

int XAMG_b200_solver_level_download(size_t sid, int level, int which, uint32_t *row, void *col,
                                    void *val) {
    return guarded([&] {
        const DCsr &d = level_matrix(sid, level, which);
        XG_CUDA(cudaStreamSynchronize(ctx().stream));
        download_csr(d, row, col, val);
    });
}

int XAMG_b200_solver_hierarchy_export(size_t sid, int level, int which, uint32_t *row,
                                      uint32_t *col, double *val) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        MultiGrid *mg = so.sh->mg;
        const HCsr *h = nullptr;
        if (!mg) {
            XG_REQUIRE(level == 0 && which == 0, XAMG_ERR_INVALID_ARG, "no multigrid hierarchy");
            h = &so.sh->hA;
        } else {
            XG_REQUIRE(level >= 0 && level < (int)mg->H->lv.size(), XAMG_ERR_INVALID_ARG,
                       "bad level");
            XG_REQUIRE(which == 0 || which == 2, XAMG_ERR_INVALID_ARG, "which must be 0 or 2");
            h = which == 0 ? &mg->H->lv[level].A : &mg->H->lv[level].P;
        }
        if (row) std::memcpy(row, h->row.data(), h->row.size() * sizeof(uint32_t));
        if (col) std::memcpy(col, h->col.data(), h->col.size() * sizeof(uint32_t));
        if (val) std::memcpy(val, h->val.data(), h->val.size() * sizeof(double));
    });
}

int XAMG_b200_solver_level_csr(size_t sid, int level, int which, XAMG_b200_csr *out) {
    return guarded([&] {
        XG_REQUIRE(out, XAMG_ERR_INVALID_ARG, "null descriptor");
        const DCsr &d = level_matrix(sid, level, which);
        out->nrows = d.nrows;
        out->ncols = d.ncols;
        out->nnz = d.nnz;
        out->row = d.row.as<uint32_t>();
        out->col = d.col.p;
        out->val = d.val.p;
        out->col_bytes = d.col_bytes;
        out->val_f32 = d.fp16 ? 3 : d.bf16 ? 2 : d.f32 ? 1 : 0;
    });
}

int XAMG_b200_read_system_size(const char *path, uint32_t *nrows, uint32_t *nnz) {
    return guarded([&] {
        XG_REQUIRE(nrows && nnz, XAMG_ERR_INVALID_ARG, "null argument");
        const SystemSize z = read_system_size(path);
        *nrows = z.nrows;
        *nnz = z.nnz;
    });
}

int XAMG_b200_read_system(const char *path, uint16_t nv, uint32_t *row, uint32_t *col,
                          double *val, double *b, double *x, int *found) {
    return guarded([&] {
        check_nv(nv);
        const int f = read_system(path, nv, row, col, val, b, x);
        if (found) *found = f;
    });
}

int XAMG_b200_write_system(const char *path, uint32_t nrows, uint32_t nnz, const uint32_t *row,
                           const uint32_t *col, const double *val, uint16_t nv, const double *b,
                           const double *x) {
    return guarded([&] {
        check_nv(nv);
        write_system(path, nrows, nnz, row, col, val, nv, b, x);
    });
}

int XAMG_b200_solver_hierarchy_save(size_t sid, const char *path) {
    return guarded([&] {
        SolverObj &so = get(g_solvers, sid, "solver");
        MultiGrid *mg = so.sh->mg;
        XG_REQUIRE(mg && mg->H, XAMG_ERR_INVALID_ARG, "the solver has no multigrid hierarchy");
        save_hierarchy(path, hierarchy_key(mg->cfg), so.sh->hA, *mg->H);
    });
}

int XAMG_b200_matrix_hierarchy_load(XAMG_matrix_id mid, const char *path) {
    return guarded([&] {
        MatObj &m = get(g_mats, mid, "matrix");
        XG_REQUIRE(m.constructed, XAMG_ERR_INVALID_ARG, "matrix not constructed");
        std::string key;
        auto H = load_hierarchy(path, m.h, key);
        m.hcache[key] = H;
    });
}

int XAMG_b200_gemm_bf16(uint64_t M, uint64_t N, uint64_t K, const void *A, const void *B,
                        void *C, uint64_t ldc, int mode, const float *bias, const void *aux,
                        uint64_t ld_aux, void *stream) {
    return guarded([&] {
        ops::mm::gemm_bf16(M, N, K, A, B, C, ldc, mode, bias, aux, ld_aux, pick(stream));
    });
}

static std::vector<std::unique_ptr<Mlp>> g_mlps;

int XAMG_b200_mlp_create(uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed,
                         size_t *id) {
    return guarded([&] {
        XG_REQUIRE(id, XAMG_ERR_INVALID_ARG, "null id");
        std::unique_ptr<Mlp> m(new Mlp());
        m->init(n_in, n_hidden, n_out, seed);
        g_mlps.push_back(std::move(m));
        *id = g_mlps.size() - 1;
    });
}

int XAMG_b200_mlp_destroy(size_t id) {
    return guarded([&] {
        get(g_mlps, id, "mlp");
        XG_CUDA(cudaStreamSynchronize(ctx().stream));
        g_mlps[id].reset();
    });
}

int XAMG_b200_mlp_predict(size_t id, uint32_t batch, const float *X, float *Y) {
    return guarded([&] {
        XG_REQUIRE(X && Y, XAMG_ERR_INVALID_ARG, "null argument");
        get(g_mlps, id, "mlp").forward(batch, X, Y);
    });
}

int XAMG_b200_mlp_train_step(size_t id, uint32_t batch, const float *X, const float *T, float lr,
                             double *loss) {
    return guarded([&] {
        XG_REQUIRE(X && T, XAMG_ERR_INVALID_ARG, "null argument");
        const double l = get(g_mlps, id, "mlp").train_step(batch, X, T, lr);
        if (loss) *loss = l;
        ctx().check_flags();
    });
}

int XAMG_b200_mlp_gradients(size_t id, uint32_t batch, const float *X, const float *T,
                            float *grads, double *loss) {
    return guarded([&] {
        XG_REQUIRE(X && T && grads, XAMG_ERR_INVALID_ARG, "null argument");
        Mlp &m = get(g_mlps, id, "mlp");
        const double l = m.gradients(batch, X, T);
        m.copy_params(grads, false, true);
        if (loss) *loss = l;
        ctx().check_flags();
    });
}

int XAMG_b200_mlp_params(size_t id, float *params, int set, uint64_t *count) {
    return guarded([&] {
        Mlp &m = get(g_mlps, id, "mlp");
        if (count) *count = m.param_count();
        if (params) m.copy_params(params, set != 0, false);
    });
}

int XAMG_b200_solver_level_spmv(size_t sid, int level, int which, const void *x, void *y, int nv,
                                int mode, void *stream) {
    return guarded([&] {
        check_nv(nv);
        const DCsr &d = level_matrix(sid, level, which);
        cudaStream_t s = pick(stream);
        if (d.f32)
            ops::spmv<float>(d, (const float *)x, (float *)y, nv, mode == 1, s);
        else
            ops::spmv<double>(d, (const double *)x, (double *)y, nv, mode == 1, s);
    });
}

uint64_t XAMG_b200_kernel_launches(void) { return g_kernel_launches; }

void *XAMG_b200_stream(void) {
    try {
        return (void *)ctx().stream;
    } catch (const Error &e) {
        g_last_error = e.what();
        return nullptr;
    }
}

int XAMG_b200_set_device(int device) {
    return guarded([&] {
        Ctx &c = ctx_uninit();
        XG_REQUIRE(!c.ready || c.device == device, XAMG_ERR_INVALID_ARG,
                   "the library is already running on another device");
        c.device_request = device;
    });
}

int XAMG_b200_vector_device_ptr(size_t vid, void **ptr) {
    return guarded([&] {
        VecObj &v = get(g_vecs, vid, "vector");
        XG_REQUIRE(ptr, XAMG_ERR_INVALID_ARG, "null pointer");
        *ptr = v.v.p<double>();
    });
}

int XAMG_b200_wait_selftest(double seconds, int *timed_out) {
    return guarded([&] {
        XG_REQUIRE(timed_out && seconds > 0 && seconds <= 1.0, XAMG_ERR_INVALID_ARG,
                   "seconds must be in (0, 1]");
        Ctx &c = ctx();
        *timed_out = 0;
        ops::wait_selftest((uint64_t)(seconds * 1e9), c.stream);
        try {
            c.check_flags();
        } catch (const Error &e) {
            if (e.code != XAMG_ERR_TIMEOUT) throw;
            *timed_out = 1;
        }
    });
}

int XAMG_b200_grid_selftest(double seconds, int *timed_out) {
    return guarded([&] {
        XG_REQUIRE(timed_out && seconds > 0 && seconds <= 1.0, XAMG_ERR_INVALID_ARG,
                   "seconds must be in (0, 1]");
        Ctx &c = ctx();
        *timed_out = 0;
        DevBuf cg(2 * sizeof(unsigned));
        ops::grid_selftest(cg.as<unsigned>(), c.red().flag, (uint64_t)(seconds * 1e9), c.stream);
        try {
            c.check_flags();
        } catch (const Error &e) {
            if (e.code != XAMG_ERR_TIMEOUT) throw;
            *timed_out = 1;
        }
    });
}

}  // extern "C"
