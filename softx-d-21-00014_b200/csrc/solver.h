// Solver objects of the B200 solve phase: the XAMG method set (solver.h:417-441)
// on device data. Each class restates the control flow of the reference's
// solvers/detail/*.inl, keeps XAMG's zero-flag short-circuits (they decide
// which kernels run) and replaces each blas/blas2 call sequence with fused
// kernels that write the same values.
#pragma once

#include <functional>
#include <map>
#include <tuple>
#include <memory>
#include <string>
#include <vector>

#include "amg.h"
#include "device.h"
#include "params.h"

namespace xg {

struct Stats {
    std::vector<int> conv;
    std::vector<double> abs_res, rel_res;
    int iters = 0;
};

struct SolverBase {
    SolverCfg cfg;
    std::string role;
    int NV = 1;
    bool f32 = false;
    const DCsr *A = nullptr;
    uint64_t n = 0;
    Stats st;
    std::vector<DVec> buf;
    virtual ~SolverBase() {}
    virtual void setup() {}
    // conv: NV entries, 1 = still active, 0 = converged (the "iconv" vector)
    virtual void solve(DVec &x, DVec &b, const std::vector<double> &conv) = 0;
    void reset_stats();
    void alloc_buffers(int count);
};

struct MgLevel {
    bool f32 = false;       // working precision of A and the smoothers
    bool tf32 = false;      // precision of R and P
    DCsr A, R, P;
    DVec temp, bH, xH;
    double min_eig = 0, max_eig = 0;
    HCsr hA;                // host copy (for the smoothers' setup)
};

std::unique_ptr<SolverBase> make_smoother(const SolverCfg &cfg, const std::string &role,
                                          const DCsr &A, const HCsr &hA, bool f32, int nv,
                                          double min_eig, double max_eig);

// Host hierarchies already built for a matrix, keyed by the setup parameters
// they depend on (the reference rebuilds the hierarchy for every solver; here
// solvers that differ only in precision or smoothers share one build).
using HierCache = std::map<std::string, std::shared_ptr<const Hierarchy>>;
// The cache key of a hierarchy: the setup parameters it was built with.
std::string hierarchy_key(const SolverCfg &c);

class MultiGrid : public SolverBase {
  public:
    std::vector<MgLevel> L;
    std::vector<std::unique_ptr<SolverBase>> pre, post;
    std::unique_ptr<SolverBase> coarse;
    std::shared_ptr<const Hierarchy> H;  // kept for export
    // gpu_precond_f32 = 1 (preconditioner only): the finest level too is
    // stored and smoothed in float; input and output are converted here
    bool full32 = false;
    DVec b32, x32;
    void build(const HCsr &A0, const DCsr *A0dev, const Params &P, const std::string &role,
               int nv, HierCache *cache);
    void solve(DVec &x, DVec &b, const std::vector<double> &conv) override;
    // full32 only: the result stays in float in x32 (zero-flagged on entry
    // when the application starts from zero)
    void solve_to32(DVec &x32, DVec &b, const std::vector<double> &conv);

  private:
    void cycle(int level, DVec &x, DVec &b, int cyc, const std::vector<double> &iconv);
};

// A preconditioner application captured as a CUDA graph: the kernels that
// M->solve(out, in) launches for one (out, in, in.zero) combination, and the
// zero flag it leaves on out.
struct MGraph {
    cudaGraphExec_t exec = nullptr;
    int calls = 0;          // direct runs before the capture
    bool failed = false;    // capture not possible: always run directly
    bool out_zero = false;
    uint64_t launches = 0;  // kernels in the graph
    std::vector<uint8_t> flags;  // step graphs: zero/init of every work vector after the step
};

class Krylov : public SolverBase {
  public:
    bool precond_form = true;  // (P)BiCGStab structure; false: MergedBiCGStab
    bool pcg = false;          // preconditioned conjugate gradients (pcg.inl)
    bool rbicgstab = false;    // reordered BiCGStab (rbicgstab.inl)
    bool rb_merged = false;    // ... in its merged form (merged_rbicgstab.inl)
    std::unique_ptr<SolverBase> M;
    DevBuf sc;                 // scalar block (kernels.cuh Sc)
    // an FP32 multigrid preconditioner (gpu_precond_f32 = 1, V- or W-cycles)
    // hands its results over in float: pa32 = M^-1 p, sa32 = M^-1 s
    bool f32io = false;        // decided at the start of every solve
    bool f32io_ready = false;  // pa32/sa32 allocated
    DVec pa32, sa32;
    void enable_f32io();
    void setup() override;
    void solve(DVec &x, DVec &b, const std::vector<double> &conv) override;
    ~Krylov() override;

    // The merged BiCGStab forms (MergedPBiCGStab, PBiCGStab, MergedBiCGStab,
    // BiCGStab) in steps, one host synchronisation apart, so that a batch of
    // independent solves can run in lockstep on separate lanes (solve() is
    // these steps on one system): begin() launches r0 = b - A x and posts
    // rho0; started() (after the lane's stream is synchronised) tests it;
    // step() launches the rest of the previous iteration, if one is pending,
    // and one iteration up to its residual, and posts it; stepped() tests it
    // and launches the final x update, or leaves the rest of the iteration
    // pending. started()/stepped() return true when the solve is finished;
    // finish() launches a pending rest when the solve stops at max_iters.
    bool steppable() const { return !pcg && !rbicgstab; }
    // gpu_solve_graph (default 1): a merged BiCGStab solve from the root
    // (every right-hand side active) as one graph launch: r0 = b - A x, the
    // convergence test of rho0, then a device-side loop (a conditional WHILE
    // node) over the iteration up to its residual, its convergence test (a
    // one-thread kernel that sets the loop's conditions, csrc/loop.cu) and,
    // as conditional IF nodes, the rest of the iteration or the final x
    // update. The same kernels in the same order as begin/step/stepped/finish,
    // so the same results bit for bit, without a host round trip an
    // iteration. launch_loop() returns false where the solve cannot be
    // recorded (it then runs the steps); loop_done() reads the statistics
    // once the stream has passed the graph.
    bool loop_ok() const;
    bool launch_loop(DVec &x, DVec &b);
    void loop_done(DVec &x);
    // Releases every recorded graph (preconditioner applications, iterations,
    // whole solves): their kernels carry the parameters they were recorded
    // with, so XAMG_solver_renew_params drops them and they are recorded
    // again with the new ones.
    void drop_graphs();
    void begin(DVec &x, DVec &b, const std::vector<double> &conv);
    bool started();
    void step();
    bool stepped();
    void finish();

  private:
    bool check(const double *res, const double *res0, std::vector<double> &iconv);
    void apply_M(DVec &out, DVec &in);
    void run_M(DVec &out, DVec &in);
    void solve_pcg(DVec &x, DVec &b, const std::vector<double> &conv);
    void solve_rbicgstab(DVec &x, DVec &b, const std::vector<double> &conv);
    void upload_iconv(const std::vector<double> &iconv);
    void step_body();
    void step_tail();
    // the whole iteration in one cooperative launch (k_pbicgstab_persist)
    bool persistent_ok() const;
    void run_persistent(DVec &x);
    DevBuf psync, pout;  // grid barrier counters; the launch's statistics
    MGraph &step_graph(const std::tuple<int, bool, const void *> &key);
    void run_graphed(MGraph &g, DVec *x, const std::function<void()> &body);
    // per (out, in, in.zero, lane): a graph's kernels carry its lane's scratch
    std::map<std::tuple<const void *, const void *, bool, int>, MGraph> graphs_;
    // iteration graphs: BiCGStab per (lane, tail, x), PCG and RBiCGStab per
    // (lane, x.zero, x); the work vectors are fixed from setup on, x is the
    // caller's
    std::map<std::tuple<int, bool, const void *>, MGraph> step_graphs_;
    bool capturing_ = false;  // recording step(): preconditioner runs inline
    // whole-solve graphs per (lane, x, b, x.zero at the start)
    struct LoopGraph {
        cudaGraphExec_t exec = nullptr;
        int calls = 0;        // solves run by steps before the recording
        bool failed = false;  // not recordable: always run by steps
        // kernels of the start, of one pass of the loop body (iteration and
        // test), of the rest of an iteration and of the final x update
        uint64_t n_start = 0, n_body = 0, n_rest = 0, n_last = 0;
        std::vector<uint8_t> flags;  // work vectors' zero/init after a solve
    };
    std::map<std::tuple<int, const void *, const void *, bool>, LoopGraph> loop_graphs_;
    DevBuf lout;               // the loop's statistics (k::LOOP_COUNT doubles)
    bool loop_x_zero_ = false; // x.zero when the running loop graph started
    const LoopGraph *loop_run_ = nullptr;  // the loop graph launched last
    bool in_loop_ = false;     // recording the loop body (no host read-back)
    bool record_loop(LoopGraph &g, DVec &x, DVec &b);
    // state of the merged BiCGStab solve between its steps
    struct Run {
        DVec *x = nullptr, *b = nullptr, *pa = nullptr, *sa = nullptr;
        std::vector<double> iconv, rho0, res;
        bool tail = false;  // the rest of the last iteration is not launched yet
    } run_;
};

// The solver hierarchy of XAMG_solver_create* (construct_solver_hierarchy,
// solver.h:481-500): outer method, optional preconditioner.
struct SolverHierarchy {
    Params params;
    HCsr hA;            // host copy of the fine matrix
    const DCsr *A = nullptr;
    int NV = 1;
    std::unique_ptr<SolverBase> root;
    MultiGrid *mg = nullptr;  // the multigrid object, if any
    void build(const Params &P, const HCsr &hA_, const DCsr *A_, int nv, HierCache *cache);
    void solve(DVec &x, DVec &b);
};

// Solves independent systems together (XAMG_b200_solver_solve_batch): system i
// runs on lane i + 1 (its own stream and reduction scratch), so the systems'
// kernels run concurrently. A system whose solve runs as one graph
// (gpu_solve_graph) is launched once and read back at the end; the other
// merged BiCGStab forms advance in lockstep: every round launches one
// iteration of each unfinished system, then the host synchronises the lanes
// once and tests each residual. Other methods run to the end on their lane. The lanes start after the work already queued on
// lane 0, and lane 0 waits for all of them before the call returns.
void solve_batch(const std::vector<SolverHierarchy *> &hs, const std::vector<DVec *> &xs,
                 const std::vector<DVec *> &bs);

}  // namespace xg
