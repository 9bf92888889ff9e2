/* A stand-in, written for this repository, for the part of hypre's interface
 * that the reference calls (src/hypre/*). hypre 2.20.0 is not available here,
 * so its BoomerAMG setup does not run: HYPRE_BoomerAMGSetup hands back a
 * hierarchy registered beforehand with xamg_ref_hypre_set_hierarchy() (the one
 * the library's host setup builds, so that the reference, the oracle and the
 * GPU solve the same hierarchy), in hypre's own ParCSR / ParAMGData structures
 * that the reference parses (hypre_base.inl:243-403). The other hypre solvers
 * (the reference's --mode hypre) are not available and abort if called.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref). */
#ifndef XAMG_REF_SHIM_HYPRE_H_
#define XAMG_REF_SHIM_HYPRE_H_

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef int HYPRE_Int;
typedef int HYPRE_BigInt;
typedef double HYPRE_Real;
typedef double HYPRE_Complex;

#define HYPRE_PARCSR 5555

struct hypre_CSRMatrix {
    HYPRE_Int num_rows, num_cols, num_nonzeros;
    HYPRE_Int *i, *j;
    HYPRE_Complex *data;
};
struct hypre_ParCSRMatrix {
    HYPRE_BigInt global_num_rows, global_num_cols;
    HYPRE_BigInt first_row_index, first_col_diag;
    hypre_CSRMatrix *diag, *offd;
    HYPRE_BigInt *col_map_offd;
};
struct hypre_ParVector {
    HYPRE_BigInt size;
    std::vector<HYPRE_Complex> data;
};
struct hypre_ParAMGData {
    HYPRE_Int num_levels;
    hypre_ParCSRMatrix **A_array, **P_array;
    HYPRE_Real *min_eig_est, *max_eig_est;
    HYPRE_Int max_levels;
};

#define hypre_ParCSRMatrixDiag(m) ((m)->diag)
#define hypre_ParCSRMatrixOffd(m) ((m)->offd)
#define hypre_ParCSRMatrixColMapOffd(m) ((m)->col_map_offd)
#define hypre_ParCSRMatrixFirstColDiag(m) ((m)->first_col_diag)
#define hypre_ParCSRMatrixFirstRowIndex(m) ((m)->first_row_index)

typedef hypre_ParCSRMatrix *HYPRE_ParCSRMatrix;
typedef hypre_ParVector *HYPRE_ParVector;
struct hypre_Solver_struct;
typedef hypre_Solver_struct *HYPRE_Solver;
typedef HYPRE_Int (*HYPRE_PtrToSolverFcn)(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector,
                                           HYPRE_ParVector);

/* IJ matrix: rows collected by SetValues, turned into a ParCSR on Assemble */
struct hypre_IJMatrix_shim {
    HYPRE_Int ilower, iupper;
    std::vector<std::vector<HYPRE_Int>> cols;
    std::vector<std::vector<HYPRE_Complex>> vals;
    hypre_ParCSRMatrix *par;
};
typedef hypre_IJMatrix_shim *HYPRE_IJMatrix;
struct hypre_IJVector_shim {
    hypre_ParVector *par;
};
typedef hypre_IJVector_shim *HYPRE_IJVector;

namespace xamg_ref_hypre {
/* one level of the registered hierarchy: A_l (square) and P_l (absent on the
 * last level), CSR with 0-based columns, plus the eigenvalue estimates */
struct Level {
    std::vector<HYPRE_Int> arow, acol, prow, pcol;
    std::vector<HYPRE_Complex> aval, pval;
    HYPRE_Int n = 0, pncols = 0;
    double min_eig = 0, max_eig = 0;
};
inline std::vector<Level> &registry() {
    static std::vector<Level> r;
    return r;
}
inline void fail(const char *what) {
    std::fprintf(stderr, "hypre stand-in: %s is not available\n", what);
    std::abort();
}
inline hypre_CSRMatrix *csr(HYPRE_Int nr, HYPRE_Int nc, const std::vector<HYPRE_Int> &r,
                            const std::vector<HYPRE_Int> &c, const std::vector<HYPRE_Complex> &v) {
    hypre_CSRMatrix *m = new hypre_CSRMatrix;
    m->num_rows = nr;
    m->num_cols = nc;
    m->num_nonzeros = (HYPRE_Int)c.size();
    m->i = new HYPRE_Int[nr + 1];
    m->j = new HYPRE_Int[c.size() + 1];
    m->data = new HYPRE_Complex[v.size() + 1];
    for (HYPRE_Int k = 0; k <= nr; ++k) m->i[k] = r.empty() ? 0 : r[k];
    for (size_t k = 0; k < c.size(); ++k) m->j[k] = c[k];
    for (size_t k = 0; k < v.size(); ++k) m->data[k] = v[k];
    return m;
}
inline hypre_ParCSRMatrix *par(hypre_CSRMatrix *diag, HYPRE_Int ncols) {
    hypre_ParCSRMatrix *p = new hypre_ParCSRMatrix;
    p->global_num_rows = diag->num_rows;
    p->global_num_cols = ncols;
    p->first_row_index = 0;
    p->first_col_diag = 0;
    p->diag = diag;
    static std::vector<HYPRE_Int> none(1, 0);
    p->offd = csr(diag->num_rows, 0, std::vector<HYPRE_Int>(diag->num_rows + 1, 0), {}, {});
    p->col_map_offd = nullptr;
    return p;
}
inline void free_par(hypre_ParCSRMatrix *p) {
    if (!p) return;
    for (hypre_CSRMatrix *m : {p->diag, p->offd}) {
        delete[] m->i;
        delete[] m->j;
        delete[] m->data;
        delete m;
    }
    delete p;
}
}  // namespace xamg_ref_hypre

/* registers the hierarchy the next BoomerAMG setups return: for level l,
 * A_l (n[l] rows) and, for l < nlev-1, P_l (n[l] x n[l+1]) */
inline void xamg_ref_hypre_set_hierarchy(int nlev, const int *n, const uint32_t *const *arow,
                                         const uint32_t *const *acol, const double *const *aval,
                                         const uint32_t *const *prow, const uint32_t *const *pcol,
                                         const double *const *pval, const double *min_eig,
                                         const double *max_eig) {
    auto &R = xamg_ref_hypre::registry();
    R.assign(nlev, xamg_ref_hypre::Level());
    for (int l = 0; l < nlev; ++l) {
        auto &L = R[l];
        L.n = n[l];
        L.arow.assign(arow[l], arow[l] + n[l] + 1);
        L.acol.assign(acol[l], acol[l] + arow[l][n[l]]);
        L.aval.assign(aval[l], aval[l] + arow[l][n[l]]);
        L.min_eig = min_eig[l];
        L.max_eig = max_eig[l];
        if (l + 1 < nlev) {
            L.pncols = n[l + 1];
            L.prow.assign(prow[l], prow[l] + n[l] + 1);
            L.pcol.assign(pcol[l], pcol[l] + prow[l][n[l]]);
            L.pval.assign(pval[l], pval[l] + prow[l][n[l]]);
        }
    }
}

inline HYPRE_Int HYPRE_IJMatrixCreate(int, HYPRE_BigInt il, HYPRE_BigInt iu, HYPRE_BigInt,
                                      HYPRE_BigInt, HYPRE_IJMatrix *m) {
    *m = new hypre_IJMatrix_shim;
    (*m)->ilower = il;
    (*m)->iupper = iu;
    (*m)->cols.assign(iu - il + 1, {});
    (*m)->vals.assign(iu - il + 1, {});
    (*m)->par = nullptr;
    return 0;
}
inline HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int) { return 0; }
inline HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix) { return 0; }
inline HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix m, HYPRE_Int nrows, HYPRE_Int *ncols,
                                         const HYPRE_BigInt *rows, const HYPRE_BigInt *cols,
                                         const HYPRE_Complex *vals) {
    HYPRE_Int k = 0;
    for (HYPRE_Int r = 0; r < nrows; ++r) {
        auto &c = m->cols[rows[r] - m->ilower];
        auto &v = m->vals[rows[r] - m->ilower];
        for (HYPRE_Int q = 0; q < ncols[r]; ++q, ++k) {
            c.push_back(cols[k]);
            v.push_back(vals[k]);
        }
    }
    return 0;
}
inline HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix m) {
    const HYPRE_Int n = m->iupper - m->ilower + 1;
    std::vector<HYPRE_Int> r(n + 1, 0), c;
    std::vector<HYPRE_Complex> v;
    for (HYPRE_Int i = 0; i < n; ++i) {
        c.insert(c.end(), m->cols[i].begin(), m->cols[i].end());
        v.insert(v.end(), m->vals[i].begin(), m->vals[i].end());
        r[i + 1] = (HYPRE_Int)c.size();
    }
    m->par = xamg_ref_hypre::par(xamg_ref_hypre::csr(n, n, r, c, v), n);
    return 0;
}
inline HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix m, void **obj) {
    *obj = m->par;
    return 0;
}
inline HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix m) {
    if (m) {
        xamg_ref_hypre::free_par(m->par);
        delete m;
    }
    return 0;
}
inline HYPRE_Int HYPRE_IJMatrixPrint(HYPRE_IJMatrix, const char *) { return 0; }

inline HYPRE_Int HYPRE_IJVectorCreate(int, HYPRE_BigInt il, HYPRE_BigInt iu, HYPRE_IJVector *v) {
    *v = new hypre_IJVector_shim;
    (*v)->par = new hypre_ParVector;
    (*v)->par->size = iu - il + 1;
    (*v)->par->data.assign(iu - il + 1, 0.0);
    return 0;
}
inline HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int) { return 0; }
inline HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
inline HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx,
                                         const HYPRE_Complex *vals) {
    for (HYPRE_Int i = 0; i < n; ++i) v->par->data[idx[i]] = vals[i];
    return 0;
}
inline HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt *idx,
                                         HYPRE_Complex *vals) {
    for (HYPRE_Int i = 0; i < n; ++i) vals[i] = v->par->data[idx[i]];
    return 0;
}
inline HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector) { return 0; }
inline HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **obj) {
    *obj = v->par;
    return 0;
}
inline HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector v) {
    if (v) {
        delete v->par;
        delete v;
    }
    return 0;
}

/* BoomerAMG: the setup returns the registered hierarchy from the level whose
 * matrix has the assembled matrix's size, at most max_levels levels */
inline HYPRE_Int HYPRE_BoomerAMGCreate(HYPRE_Solver *s) {
    hypre_ParAMGData *d = new hypre_ParAMGData;
    d->num_levels = 0;
    d->A_array = d->P_array = nullptr;
    d->min_eig_est = d->max_eig_est = nullptr;
    d->max_levels = 25;
    *s = (HYPRE_Solver)d;
    return 0;
}
inline HYPRE_Int HYPRE_BoomerAMGSetMaxLevels(HYPRE_Solver s, HYPRE_Int n) {
    ((hypre_ParAMGData *)s)->max_levels = n;
    return 0;
}
inline HYPRE_Int HYPRE_BoomerAMGSetup(HYPRE_Solver s, HYPRE_ParCSRMatrix A, HYPRE_ParVector,
                                      HYPRE_ParVector) {
    hypre_ParAMGData *d = (hypre_ParAMGData *)s;
    auto &R = xamg_ref_hypre::registry();
    int k = -1;
    for (size_t l = 0; l < R.size(); ++l)
        if (R[l].n == A->diag->num_rows && (HYPRE_Int)R[l].acol.size() == A->diag->num_nonzeros) {
            k = (int)l;
            break;
        }
    if (k < 0) xamg_ref_hypre::fail("a BoomerAMG setup of an unregistered matrix");
    const int nl = std::min<int>(d->max_levels, (int)R.size() - k);
    d->num_levels = nl;
    d->A_array = new hypre_ParCSRMatrix *[nl];
    d->P_array = new hypre_ParCSRMatrix *[nl];
    d->min_eig_est = new HYPRE_Real[nl];
    d->max_eig_est = new HYPRE_Real[nl];
    for (int i = 0; i < nl; ++i) {
        const auto &L = R[k + i];
        d->A_array[i] = i == 0 ? A
                               : xamg_ref_hypre::par(xamg_ref_hypre::csr(L.n, L.n, L.arow, L.acol,
                                                                         L.aval),
                                                     L.n);
        d->P_array[i] = i + 1 < nl ? xamg_ref_hypre::par(xamg_ref_hypre::csr(L.n, L.pncols, L.prow,
                                                                             L.pcol, L.pval),
                                                         L.pncols)
                                   : nullptr;
        d->min_eig_est[i] = L.min_eig;
        d->max_eig_est[i] = L.max_eig;
    }
    return 0;
}
inline HYPRE_Int HYPRE_BoomerAMGDestroy(HYPRE_Solver s) {
    hypre_ParAMGData *d = (hypre_ParAMGData *)s;
    if (!d) return 0;
    for (int i = 0; i < d->num_levels; ++i) {
        if (i > 0) xamg_ref_hypre::free_par(d->A_array[i]);
        xamg_ref_hypre::free_par(d->P_array[i]);
    }
    delete[] d->A_array;
    delete[] d->P_array;
    delete[] d->min_eig_est;
    delete[] d->max_eig_est;
    delete d;
    return 0;
}
/* configuration calls: the registered hierarchy was built with the matching
 * parameters by the caller, so they are accepted and ignored */
#define XAMG_REF_HYPRE_SET(name, T)                                                         \
    inline HYPRE_Int name(HYPRE_Solver, T) { return 0; }
#define XAMG_REF_HYPRE_SET2(name, T, U)                                                     \
    inline HYPRE_Int name(HYPRE_Solver, T, U) { return 0; }
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetMaxIter, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetTol, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetPrintLevel, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetLogging, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetConvergeType, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetRestriction, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetRAP2, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetMaxCoarseSize, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetStrongThreshold, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetTruncFactor, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetNumPaths, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetCoarsenType, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetInterpType, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetMaxRowSum, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetPMaxElmts, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetNonGalerkinTol, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggNumLevels, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggInterpType, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggTruncFactor, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggP12TruncFactor, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggPMaxElmts, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetAggP12MaxElmts, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetRelaxOrder, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetNumSweeps, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetOldDefault, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetRelaxWt, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BoomerAMGSetChebyOrder, HYPRE_Int)
XAMG_REF_HYPRE_SET2(HYPRE_BoomerAMGSetLevelNonGalerkinTol, HYPRE_Real, HYPRE_Int)
XAMG_REF_HYPRE_SET2(HYPRE_BoomerAMGSetCycleRelaxType, HYPRE_Int, HYPRE_Int)
XAMG_REF_HYPRE_SET2(HYPRE_BoomerAMGSetCycleNumSweeps, HYPRE_Int, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BiCGSTABSetMaxIter, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BiCGSTABSetTol, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BiCGSTABSetAbsoluteTol, HYPRE_Real)
XAMG_REF_HYPRE_SET(HYPRE_BiCGSTABSetPrintLevel, HYPRE_Int)
XAMG_REF_HYPRE_SET(HYPRE_BiCGSTABSetLogging, HYPRE_Int)

inline HYPRE_Int HYPRE_BoomerAMGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector,
                                      HYPRE_ParVector) {
    xamg_ref_hypre::fail("HYPRE_BoomerAMGSolve");
    return 1;
}
inline HYPRE_Int HYPRE_BoomerAMGGetNumIterations(HYPRE_Solver, HYPRE_Int *) { return 0; }
inline HYPRE_Int HYPRE_BoomerAMGGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real *) {
    return 0;
}
inline HYPRE_Int HYPRE_ParCSRBiCGSTABCreate(int, HYPRE_Solver *) {
    xamg_ref_hypre::fail("HYPRE_ParCSRBiCGSTABCreate");
    return 1;
}
inline HYPRE_Int HYPRE_ParCSRBiCGSTABSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector,
                                           HYPRE_ParVector) {
    return 1;
}
inline HYPRE_Int HYPRE_ParCSRBiCGSTABSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector,
                                           HYPRE_ParVector) {
    return 1;
}
inline HYPRE_Int HYPRE_ParCSRBiCGSTABDestroy(HYPRE_Solver) { return 0; }
inline HYPRE_Int HYPRE_BiCGSTABSetPrecond(HYPRE_Solver, HYPRE_PtrToSolverFcn, HYPRE_PtrToSolverFcn,
                                          HYPRE_Solver) {
    return 0;
}
inline HYPRE_Int HYPRE_BiCGSTABGetNumIterations(HYPRE_Solver, HYPRE_Int *) { return 0; }
inline HYPRE_Int HYPRE_BiCGSTABGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real *) {
    return 0;
}

#endif
