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
    // variable density: 1/rho per cell of the level (shared with the other
    // solver of the scene), FP64 and FP32; null for constant density
    const double *ri = nullptr;
    const float *ris = nullptr;
    size_t npts() const { return (size_t)n[0] * n[1] * n[2]; }
};

// Device-resident control state of one solver: the mg_pred predictor
// (mg_probs.hh:37-78; alpha is the integer quotient 1/(3*iP) = 0 exactly as
// the reference computes it, so the averages never move) and the position in
// the mg_prob::run loop (Utilities/mg_probs.cc:3-83).  The host reads it back
// after a solve or a step.
struct mg_ctl {
    int iV;            // predicted V-cycles x iP
    int phase;         // 0 predicted cycles, 1 extra rounds, 2 insurance, 3 stagnation loop
    int todo;          // cycles left in the current phase
    int extra;         // extra rounds so far
    int it;            // stagnation-loop iterations
    int count;         // cycles of the current solve
    int last_cycles;   // cycles of the last finished solve
    int active;        // the current solve continues
    int nan;           // the last solve ended with a NaN residual
    int need_res;      // the next iteration ends at a point where the control reads the residual
    long long cycles_total;
    double V_avg, V_var;
    double prev, res_out;  // previous / reported max-norm residual
};

constexpr int kMgIP = 16;
constexpr int kMgMaxCycles = 4096;  // bound on the cycles of one solve

struct graph_builder;
struct pmg_args;

// sizes of the arrays carved out of one allocation: 256-byte multiples
inline size_t slab_pad(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

class mg_solver {
  public:
    mg_kind kind;
    std::vector<mg_level> lv;
    double max_norm_tol;
    int v_up = 2, v_down = 2;
    long long cycles_total = 0;  // host mirrors of the device control state
    int last_cycles = 0;
    bool mixed = false;  // FP32 cycles inside FP64 iterative refinement
    bool exact = false;  // iterate each solve until the residual stagnates
    double rtol = 0;     // mixed form: relative tolerance (x max |rhs|), no insurance cycles
    long long *launches = nullptr;
    kernel_profiler *prof = nullptr;
    mg_ctl *ctl = nullptr;       // device control block (owned by the scene)
    mg_ctl *h_ctl = nullptr;     // pinned mirror (owned by the scene)
    bool use_graph = true;       // false: run() issues every kernel from the host
    bool vd = false;             // variable density: levels carry 1/rho (no one-block coarse sub-cycle)
    // one launch per solve in a thread-block cluster (k_mgc.cu), or (default)
    // one launch per phase inside a graph WHILE loop; measured on a B200 the
    // per-phase launches over the whole GPU win for a single scene (64^3:
    // 4.1 vs 14 ms per step), and the batch autotuner picks per grid size
    int cluster_size = 0;        // CTAs per cluster supported here (0: none)
    bool use_cluster = false;
    bool cluster_mode() const { return use_cluster && cluster_size > 0; }
    int setup_cluster();
    cudaError_t launch_cluster(cudaStream_t st);

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
    unsigned char *slab = nullptr;  // every level's arrays, one allocation
    double *rhs() { return lv[0].r; }
    double *sol() { return lv[0].x; }
    double *dense = nullptr;  // inverse of the coarsest operator (row-major), or null
    // smoothing: 0 one launch per colour pass (in place); 1 one launch per
    // whole sweep on shared-memory tiles (mg_tile.cuh), alternating between
    // a level's x and its residual array
    int smoother = 0;
    // first level (>= 1) of the coarse part of a V-cycle run as one
    // thread-block-cluster launch (k_mg_coarse_cluster), -1 none
    int ccl = -1;
    int cluster_coarse_pts = 0;  // largest level handed to that launch (0: none)
    int set_cluster_coarse(int pts);
    int cf = 0;  // first level whose whole sub-cycle runs in one CTA
    int coarse_pts = 0;  // largest level handed to the one-CTA sub-cycle (0: none)
    int set_coarse(int pts);

    // One solve with the reference's control logic, issued eagerly and
    // waited for; returns the reported max-norm residual (NaN propagates).
    // Uses the solver's own graph unless a kernel profiler is active.
    double run(cudaStream_t st);
    // Append one solve to the graph `cur` is capturing: an arming kernel and a
    // WHILE node whose body is one iteration, the residual norm and the
    // control kernel.  Returns the kernels per loop iteration.
    int capture_solve(cudaStream_t cur, graph_builder &gb);
    int outside_kernels = 1;   // kernels of a solve outside its loop body (set by capture_solve)
    int body_kernels = 0;      // kernels per loop iteration (set by capture_solve)
    void invalidate();         // drop the solver's own graph (schedule changed)
    void release();            // free the device memory (stream-ordered, on the set-up stream)
    void sync_host_mirror();   // cycles from the pinned control mirror
    unsigned long long *max_slots() const { return d_max; }

  private:
    cudaStream_t alloc_stream = nullptr;
    unsigned long long *d_max = nullptr;  // residual max-norm (ordered bit pattern)
    cudaGraphExec_t solve_exec = nullptr;
    cudaStream_t cap_main = nullptr;
    graph_builder *own_gb = nullptr;
    int build_dense(cudaStream_t st);
    int build_solve_graph();
    void launch_body(cudaStream_t st, bool armed, unsigned long long h);
    void iterate(cudaStream_t st);
    // a V-cycle from level l down; returns the array holding the level's
    // solution afterwards (0 its x, 1 its residual array)
    int cycle(int l, cudaStream_t st);
    int cycle_f32(int l, cudaStream_t st);
    int smooth(int l, int sweeps, int cur, cudaStream_t st);
    int smooth_f32(int l, int sweeps, int cur, cudaStream_t st);
    void refine_step(cudaStream_t st);
};

// the coarse part of a V-cycle from level l0 in one cluster launch: one
// scene, or every running scene of a group (one cluster each; A: device
// array of the scenes' level tables)
class mg_solver;
cudaError_t coarse_cluster(const mg_solver &m, int l0, bool f32, cudaStream_t st);
cudaError_t coarse_cluster_b(const pmg_args *A, const int *run, int B, int l0, int csize, bool f32, cudaStream_t st);
pmg_args level_args(const mg_solver &m);
// the tiled sweep kernels' shared-memory limits (once per process)
int tile_setup();

// One multigrid solve for every scene of a group of equally sized scenes
// with the same form and schedule, each phase one launch over all of them
// (k_mgb.cu).  The scenes' own solvers keep the level arrays and control
// state; the group holds device tables of their pointers.
struct mgb_level_tab {
    double **x, **r, **res;
    float **xs, **rs, **ress;
    const double **ri;
    const float **ris;
};

class mg_group {
  public:
    int B = 0;
    mg_kind kind = MG_MAC;
    std::vector<mg_level> lv;
    bool mixed = false, exact = false, vd = false;
    double tol = 0, rtol = 0;
    int v_down = 2, v_up = 2;
    int smoother = 0;
    int ccl = -1, csize = 0;     // the cluster coarse sub-cycle (see mg_solver)
    pmg_args *dargs = nullptr;   // device copies of the scenes' level tables for it
    const double *dense = nullptr;
    std::vector<mgb_level_tab> tab;  // device tables per level
    mg_ctl **ctls = nullptr;         // device table of the scenes' control blocks
    unsigned long long **mx = nullptr;  // device table of the scenes' residual slots
    int *part = nullptr;             // device flags: scene b takes part in the next solve
    int *run = nullptr;              // device flags: scene b's solve is still running
    int body_kernels = 0, outside_kernels = 1;

    mg_group() = default;
    mg_group(const mg_group &) = delete;
    mg_group &operator=(const mg_group &) = delete;
    ~mg_group();
    // tables allocated stream-ordered on st (no device-wide synchronisation
    // when groups come and go next to running ones)
    int setup(const std::vector<mg_solver *> &solvers, cudaStream_t st);
    void release();  // frees the tables on the set-up stream (still alive)
    // append the group's solve (arming kernel + WHILE loop) to the capture
    int capture(cudaStream_t cur, graph_builder &gb);

  private:
    void *dev_tables = nullptr;
    cudaStream_t tstream = nullptr;
    void iterate(cudaStream_t st);
};

}  // namespace rmt3d
