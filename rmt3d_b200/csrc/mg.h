// Device-resident geometric multigrid for the two pressure Poisson problems of
// the step: the cell-centred 7-point MAC problem (simp_mac,
// Utilities/mg_probs.hh:497-530) and the nodal 27-point Q1 FEM problem
// (simp_fem, :458-495).  The V-cycle control reproduces mg_prob::run and
// mg_pred (Utilities/mg_probs.cc:3-83, mg_probs.hh:37-78): the predicted
// number of cycles, extra rounds until the max-norm residual is below the
// problem's tolerance (at most 20 rounds), then two insurance cycles.
#pragma once
#include <cuda_runtime.h>
#include <vector>

namespace rmt3d {

enum mg_kind { MG_MAC = 0, MG_FEM = 1 };

// Opt-in launch timing of one kernel class: CUDA events recorded on the
// launching stream around each launch, summed on read.
struct kernel_profiler {
    int target = -1;  // 0 fem_gs (fine level), 1 mac_rb (fine level)
    std::vector<cudaEvent_t> ev;
    size_t used = 0;
    double points = 0;  // points updated by the timed launches
    double bytes = 0;   // algorithmic bytes of the timed launches
    void begin(cudaStream_t st) {
        if (used + 2 > ev.size()) return;
        cudaEventRecord(ev[used], st);
    }
    void end(cudaStream_t st, double pts, double byt) {
        if (used + 2 > ev.size()) return;
        cudaEventRecord(ev[used + 1], st);
        used += 2;
        points += pts;
        bytes += byt;
    }
};

struct mg_level {
    int n[3];
    int prd[3];
    double *x = nullptr;    // solution
    double *r = nullptr;    // source
    double *res = nullptr;  // residual scratch
    float *xs = nullptr, *rs = nullptr, *ress = nullptr;  // FP32 copies (mixed form)
    size_t npts() const { return (size_t)n[0] * n[1] * n[2]; }
};

// mg_pred (mg_probs.hh:37-78); alpha is the integer quotient 1/(3*iP) = 0
// exactly as the reference computes it, so the averages never move.
struct mg_pred_state {
    int iP = 16;
    int iV = 32;
    double V_avg = 32;
    double V_var = 1e6;
    double alpha = 1 / (3 * 16);
    int iters() const { return iV / iP; }
    void update(int extras);
};

class mg_solver {
  public:
    mg_kind kind;
    std::vector<mg_level> lv;
    double max_norm_tol;
    int v_up = 2, v_down = 2;
    mg_pred_state pred;
    long long cycles_total = 0;
    int last_cycles = 0;
    bool mixed = false;  // FP32 cycles inside FP64 iterative refinement
    bool exact = false;  // iterate each solve until the residual stagnates
    long long *launches = nullptr;
    kernel_profiler *prof = nullptr;

    mg_solver() = default;
    mg_solver(const mg_solver &) = delete;
    mg_solver &operator=(const mg_solver &) = delete;
    ~mg_solver();
    // n: fine points per axis; prd: periodic flags
    int setup(mg_kind k, const int n[3], const int prd[3], bool mixed_form, cudaStream_t st);
    // the level hierarchy setup() builds; 0 or an error code
    static int plan(mg_kind k, const int n[3], const int prd[3], std::vector<mg_level> &out);
    // device bytes setup() allocates for this hierarchy (0 if it cannot coarsen)
    static size_t footprint(mg_kind k, const int n[3], const int prd[3], bool mixed_form);
    size_t bytes_alloc = 0;  // device bytes held
    double *rhs() { return lv[0].r; }
    double *sol() { return lv[0].x; }
    // one solve with the reference's control logic; returns the final max-norm
    // residual (NaN propagates)
    double run(cudaStream_t st);
    // one cooperative launch per solve with the control loop on the device
    bool persistent = false;
    double *dense = nullptr;  // inverse of the coarsest operator (row-major), or null
    int cf = 0;  // first level whose whole sub-cycle runs in one CTA
    bool hard_error = false;  // the persistent launch failed or its barrier timed out
    int setup_persistent(cudaStream_t st);
    double run_persistent(cudaStream_t st);
    double residual_max(cudaStream_t st);
    void vcycle(cudaStream_t st);

  private:
    double *d_max = nullptr;   // device scalar for reductions
    void *pstate = nullptr;    // persistent solver: predictor state, barrier, partial maxima
    int pgrid = 0;
    int build_dense(cudaStream_t st);
    double *h_max = nullptr;   // pinned host mirror
    void cycle(int l, cudaStream_t st);
    void cycle_f32(int l, cudaStream_t st);
    void smooth(int l, int sweeps, cudaStream_t st);
    void smooth_f32(int l, int sweeps, cudaStream_t st);
    void refine_step(cudaStream_t st);
};

}  // namespace rmt3d
