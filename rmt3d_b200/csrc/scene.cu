// Scene object and C ABI: construction (fluid_3d ctor + sim_manager set-up),
// initialisation (fluid_3d::initialize / init_iter), the time step
// (fluid_3d::step_forward, F3D_Source/fluid_3d.cc:429-577) as a sequence of
// device kernels on the scene's stream, and state import/export in the
// reference's AoS layout.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>

#include "graph_build.h"
#include "host_common.h"
#include "kernels.h"
#include "mg.h"
#include "rmt3d_gpu.h"
#include "solid.h"

namespace rmt3d {

static thread_local std::string g_err;
int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

}  // namespace rmt3d

using namespace rmt3d;

extern "C" const char *rmt3d_last_error(void) { return g_err.c_str(); }

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(RMT3D_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------
// host-side mirrors of the reference's object and manager arithmetic
// ---------------------------------------------------------------------------
namespace {

struct host_obj {
    int type;
    double c[3], R, eig[3], omega[3];
    double rho, G, cs, ex_visc_mult, ev_trans_mult, dt_pad, dt_ex_pad, ex_mu, volume;
    // basic_sphere::phi (object.cc:76-82)
    double phi(const double xi[3]) const {
        double sq = 0;
        for (int i = 0; i < 3; i++) sq += (xi[i] - c[i]) * (xi[i] - c[i]);
        return sqrt(sq) - R;
    }
    // object::rm0 / sphere::rm0 (object.hh:40-42, :110-114)
    void rm0(const double x[3], double xi[3]) const {
        if (type == RMT3D_OBJ_SPHERE)
            for (int i = 0; i < 3; i++) xi[i] = (x[i] - c[i]) * eig[i] + c[i];
        else
            for (int i = 0; i < 3; i++) xi[i] = x[i];
    }
    // object::velocity (object.hh:48-54)
    void velocity(const double rv[3], double &u, double &v, double &w) const {
        double L[3];
        for (int i = 0; i < 3; i++) L[i] = rv[i] - c[i];
        u += omega[1] * L[2] - omega[2] * L[1];
        v -= omega[0] * L[2] - omega[2] * L[0];
        w += omega[0] * L[1] - omega[1] * L[0];
    }
    // sl_mat::cfl (sim_manager.hh:59-64)
    double cfl(double dx) const {
        double xxsp3 = 3 / (dx * dx);
        double dt1 = 0.5 * rho / (ex_mu * (ev_trans_mult + 1) * xxsp3) * dt_ex_pad;
        double dt0 = dx / cs * dt_pad;
        return (dt0 < dt1) ? dt0 : dt1;
    }
};

inline dim3 blk() { return dim3(32, 4, 2); }
inline dim3 grd(int a, int b, int c) { return dim3((a + 31) / 32, (b + 3) / 4, (c + 1) / 2); }
// Block shapes (x, y, z) of the bulk stencil kernels of the step, 256 threads
// each: the tile of cells a block covers, chosen per kind of scene by the
// batch autotuner (rmt3d_scene_set_block_shape).  Shape 0 is the default.
constexpr int kBlockShapes[][3] = {{32, 4, 2}, {32, 8, 1}, {64, 4, 1}, {32, 2, 4}, {128, 2, 1}};
constexpr int kNumBlockShapes = (int)(sizeof(kBlockShapes) / sizeof(kBlockShapes[0]));
static_assert(kNumBlockShapes == RMT3D_BLOCK_SHAPES, "block shape table and header disagree");
inline dim3 blk_of(int shape) {
    return dim3(kBlockShapes[shape][0], kBlockShapes[shape][1], kBlockShapes[shape][2]);
}
inline dim3 grd_of(int shape, int a, int b, int c) {
    const dim3 t = blk_of(shape);
    return dim3((a + t.x - 1) / t.x, (b + t.y - 1) / t.y, (c + t.z - 1) / t.z);
}
inline unsigned lin_blocks(int n) { return (unsigned)((n + 255) / 256); }

}  // namespace

// Device-resident control block of a scene, copied to a pinned mirror after
// every solve or step: simulation time, the step graph's halt flag and status,
// the per-step error counters and both solvers' multigrid control state.
struct scene_ctl {
    double time;
    int halted;  // a step of the step graph failed: its later launches do nothing
    int steps;   // steps the step graph has executed
    int status;  // status of the failing step
    int run_flag;  // the current step of a group graph runs for this scene
    int counters[8];  // [0..1] frontier sizes, [2] extrapolation errors, [3] corrector problems,
                      // [4] redraw fatal, [5] refmap-derivative errors, [7] TMA waits that gave up
    mg_ctl mac, fem;
};

struct rmt3d_scene {
    rmt3d_scene_desc d;
    grid_dev g;
    fields_dev hF;
    fields_dev *dF = nullptr;
    cudaStream_t st = 0;
    bool own_stream = false;
    std::vector<void *> allocs;
    double *lx = nullptr, *ly = nullptr, *lz = nullptr;
    std::vector<double> hlx, hly, hlz;
    host_obj obj[RMT3D_MAX_OBJ];
    mg_solver mac, fem;
    gradphi_t gradphi;
    bc_face faces[6];
    bool wall[6];
    double dt = 0, time = 0, dt_reg = 0, eps = 0, vmax = 1, K_stiff = 0;
    double min_wall_acc = 0, wall_acc_mult = 0;
    // dt_reg, K_stiff and vmax as sim_manager leaves them at construction,
    // before init_fluid's CFL recheck (a checkpoint restart skips it)
    double dt_reg0 = 0, K_stiff0 = 0, vmax0 = 1;
    int init_err = 1;  // fluid_3d::initialize's result: 0 restarted, 1 from scratch
    int nt = 0;
    long long launches = 0;
    kernel_profiler prof;
    // extrapolation scratch
    uint8_t *lay = nullptr;  // per object: layer tags
    int *inl = nullptr;      // per object: layer that claimed the cell (0: none)
    int *front[2] = {nullptr, nullptr};  // per object: ncell entries each
    int *fcnt = nullptr;                  // frontier lengths, [2][kMaxObj]
    // lanes per frontier cell of the least-squares extrapolation: a warp when
    // the scene steps on its own, 4 when it steps inside a group with others
    int extrap_lanes = 32;
    // rmt3d_snapshot_fields: device staging copies and their own copy stream
    double *snap = nullptr;
    size_t snap_cap = 0;  // doubles
    cudaStream_t cst = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_d2h = nullptr;
    bool d2h_pending = false;
    // velocity edge states through TMA-staged tiles (k_edge_vel_tma): the
    // tensor maps of vel[0..2], made when the rows are 16-byte aligned
    bool edge_tma = false;
    int bshape = 0;  // block shape of the bulk stencil kernels (kBlockShapes)
    CUtensorMap tm_vel[3];
    int *mlist = nullptr, *mcnt = nullptr;  // cells holding a map, for the stress kernel
    // passive tracers (dump_code bit 1 and ntracers > 0, fluid_3d.cc:217-219)
    int ntr = 0;
    int *tr_pc = nullptr;
    double *tr_rp = nullptr;
    uint8_t *tr_alive = nullptr;
    scene_ctl *ctl = nullptr;    // device control block
    scene_ctl *h_ctl = nullptr;  // pinned mirror
    int *counters = nullptr;     // = ctl->counters
    int *h_counters = nullptr;   // = h_ctl->counters
    // the step as one CUDA graph (built on first use, rebuilt when dt, the
    // FEM basis or the multigrid schedule change)
    graph_builder gb;
    cudaGraphExec_t step_exec = nullptr;
    bool graph_dirty = true;
    bool capturing = false;
    bool use_graph = true;
    long long graph_fixed = 0;  // kernels per step outside the multigrid loops
    long long param_version = 0;  // bumped whenever captured step parameters change
    double *d_diag = nullptr;  // solid diagnostics: [0..7] totals, then per-block partials
    unsigned *diag_ticket = nullptr;
    double *d_mean = nullptr;  // [0] mean, [1..] per-block partial sums
    unsigned *mean_ticket = nullptr;
    double *h_scalar = nullptr;
    double *d_red = nullptr;
    size_t dev_bytes = 0;  // bytes held through alloc()
    // variable density: 1/rho per cell on every multigrid level (MAC level
    // dimensions; the FEM levels' cells are the same), FP64 and FP32
    std::vector<double *> rinv;
    std::vector<float *> rinvs;

    // The per-cell arrays in one allocation: plan() records each array in
    // order, commit_slab() allocates their total and carves them at 256-byte
    // boundaries.  One pool request instead of about a hundred, and the
    // arrays' relative placement is the same for every scene whatever the
    // state of the memory pool.
    std::vector<std::pair<void **, size_t>> slab_req;
    template <typename T>
    int plan(T **p, size_t n) {
        slab_req.push_back({(void **)p, slab_pad(n * sizeof(T))});
        return 0;
    }
    int commit_slab() {
        size_t total = 0;
        for (auto &r : slab_req) total += r.second;
        unsigned char *b = nullptr;
        if (cudaMallocAsync((void **)&b, total, st) != cudaSuccess) return fail(RMT3D_ERR_OOM, "device allocation failed");
        allocs.push_back(b);
        dev_bytes += total;
        cudaMemsetAsync(b, 0, total, st);
        size_t off = 0;
        for (auto &r : slab_req) {
            *r.first = b + off;
            off += r.second;
        }
        slab_req.clear();
        return 0;
    }

    // stream-ordered allocation from the device's memory pool (no device-wide
    // synchronisation when scenes are created or destroyed)
    template <typename T>
    int alloc(T **p, size_t n) {
        if (cudaMallocAsync((void **)p, n * sizeof(T), st) != cudaSuccess)
            return fail(RMT3D_ERR_OOM, "device allocation failed");
        allocs.push_back(*p);
        dev_bytes += n * sizeof(T);
        cudaMemsetAsync(*p, 0, n * sizeof(T), st);
        return 0;
    }
    void count(int n = 1) { launches += n; }
};

// the step's captured parameters (dt, FEM basis, multigrid schedule) changed:
// graphs that hold this scene's step must be captured again
static void mark_dirty(rmt3d_scene *s);

// the extrapolation's lanes per frontier cell; a change re-captures the
// scene's own step graph
static void set_extrap_lanes(rmt3d_scene *s, int lanes) {
    if (s->extrap_lanes == lanes) return;
    s->extrap_lanes = lanes;
    mark_dirty(s);
}

static void mark_dirty(rmt3d_scene *s) {
    s->graph_dirty = true;
    s->param_version++;
}

// A blocking copy ordered on the scene's (non-blocking) stream: plain
// cudaMemcpy runs on the legacy stream, which does not wait for it.
static cudaError_t copy_sync(rmt3d_scene *s, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s->st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s->st);
}

// The velocity face states are FP32 in the FP32-advection form (g.f32face): zeroed,
// read and written from the host through these, widened to and narrowed from
// FP64 on the host side.
// FP32 face states and advection arithmetic: the RMT3D_MIXED_BULK32 form
static bool face32(const rmt3d_scene_desc &d) { return d.precision == RMT3D_MIXED_BULK32; }
// FP32 V-cycles inside FP64 refinement: both mixed forms
static bool mixed_form(int precision) { return precision == RMT3D_MIXED || precision == RMT3D_MIXED_BULK32; }

static cudaError_t zero_faces(rmt3d_scene *s) {
    const size_t n = s->g.ncell;
    for (int c = 0; c < 18; c++) {
        cudaError_t e = s->g.f32face ? cudaMemsetAsync(s->hF.fvel32[c], 0, n * sizeof(float), s->st)
                                     : cudaMemsetAsync(s->hF.fvel[c], 0, n * sizeof(double), s->st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static int faces_to_host(rmt3d_scene *s, int c, double *dst) {
    const size_t n = s->g.ncell;
    if (!s->g.f32face) {
        CK(copy_sync(s, dst, s->hF.fvel[c], n * sizeof(double), cudaMemcpyDeviceToHost));
        return RMT3D_OK;
    }
    std::vector<float> t(n);
    CK(copy_sync(s, t.data(), s->hF.fvel32[c], n * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; i++) dst[i] = t[i];
    return RMT3D_OK;
}

static int faces_from_host(rmt3d_scene *s, int c, const double *src) {
    const size_t n = s->g.ncell;
    if (!s->g.f32face) {
        CK(copy_sync(s, s->hF.fvel[c], src, n * sizeof(double), cudaMemcpyHostToDevice));
        return RMT3D_OK;
    }
    std::vector<float> t(n);
    for (size_t i = 0; i < n; i++) t[i] = (float)src[i];
    CK(copy_sync(s, s->hF.fvel32[c], t.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    return RMT3D_OK;
}

// ---------------------------------------------------------------------------
// ghost-frame helpers
// ---------------------------------------------------------------------------
static void periodic(rmt3d_scene *s, std::initializer_list<double *> arrs, std::initializer_list<int *> iarrs,
                     int corner) {
    if (!(s->g.prd[0] || s->g.prd[1] || s->g.prd[2])) return;
    ptr_list pl;
    pl.n = 0;
    pl.ni = 0;
    pl.nf = 0;
    for (double *a : arrs) pl.p[pl.n++] = a;
    for (int *a : iarrs) pl.ip[pl.ni++] = a;
    k_periodic_copy<<<grd(s->g.sm4, s->g.sn4, s->g.so4), blk(), 0, s->st>>>(s->g, pl, corner);
    s->count();
}

// fill_boundary_cc: set_bc_cc then communicate<1> (fluid_3d.cc:145-152)
static void fill_boundary_cc(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    const int ext[3] = {g.sm4, g.sn4, g.so4};
    for (int n = 0; n < 3; n++) {  // walls come in pairs: both faces of an axis at once
        if (!s->wall[2 * n]) continue;
        int t0 = (n == 0) ? 1 : 0, t1 = (n == 2) ? 1 : 2;
        dim3 gr((ext[t0] + 31) / 32, (ext[t1] + 7) / 8, 4);
        k_bc_cc<<<gr, dim3(32, 8, 1), 0, s->st>>>(g, n, s->faces[2 * n], s->faces[2 * n + 1], s->hF.vel[0],
                                                  s->hF.vel[1], s->hF.vel[2]);
        s->count();
    }
    periodic(s, {s->hF.vel[0], s->hF.vel[1], s->hF.vel[2]}, {}, 0);
}

// fill_boundary_cf: set_bc_cf then communicate<4> (fluid_3d.cc:155-165)
static void fill_boundary_cf(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    int walls = 0;
    bc_faces bcs;
    for (int f = 0; f < 6; f++) {
        bcs.f[f] = s->faces[f];
        if (s->wall[f]) walls |= 1 << f;
    }
    if (walls) {
        const int mx = std::max(g.sm4, std::max(g.sn4, g.so4));
        dim3 gr((mx + 31) / 32, (mx + 7) / 8, 6);
        k_bc_cf<<<gr, dim3(32, 8, 1), 0, s->st>>>(g, walls, bcs, s->dF);
        s->count();
    }
    if (g.prd[0] || g.prd[1] || g.prd[2]) {
        ptr_list pl;
        pl.n = g.f32face ? 0 : 18;
        pl.ni = 0;
        pl.nf = g.f32face ? 18 : 0;
        for (int a = 0; a < 18; a++) {
            pl.p[a] = s->hF.fvel[a];
            pl.fp[a] = s->hF.fvel32[a];
        }
        k_periodic_copy<<<grd(g.sm4, g.sn4, g.so4), blk(), 0, s->st>>>(g, pl, 0);
        s->count();
    }
}

// communicate<2>: p, dp, q on the nodal table
static void comm_pressure(rmt3d_scene *s) { periodic(s, {s->hF.p, s->hF.dp, s->hF.q}, {}, 1); }
// communicate<2048>: dvel
static void comm_dvel(rmt3d_scene *s) { periodic(s, {s->hF.dvel[0], s->hF.dvel[1], s->hF.dvel[2]}, {}, 0); }

// communicate<4|64> + communicate_extrap_fx: face states of the maps
static void comm_face_maps(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (!(g.prd[0] || g.prd[1] || g.prd[2])) return;
    for (int o = 0; o < g.n_obj; o++) {
        ptr_list pl;
        pl.n = 18;
        pl.ni = 0;
        pl.nf = 0;
        for (int a = 0; a < 18; a++) pl.p[a] = s->hF.om[o].fx[a];
        k_periodic_copy<<<grd(g.sm4, g.sn4, g.so4), blk(), 0, s->st>>>(g, pl, 0);
        s->count();
    }
}

// communicate<8> + <16|32>: the primary maps' id, x and xpred
static void comm_primary(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (!(g.prd[0] || g.prd[1] || g.prd[2])) return;
    for (int o = 0; o < g.n_obj; o++) {
        objmap_dev &m = s->hF.om[o];
        ptr_list pl;
        pl.n = 0;
        pl.nf = 0;
        for (int a = 0; a < 3; a++) pl.p[pl.n++] = m.x[a];
        for (int a = 0; a < 3; a++) pl.p[pl.n++] = m.xp[a];
        pl.ni = 1;
        pl.ip[0] = m.code;
        k_periodic_copy<<<grd(g.sm4, g.sn4, g.so4), blk(), 0, s->st>>>(g, pl, 0);
        s->count();
    }
}

// ---------------------------------------------------------------------------
// extrapolation, fluid_3d::extrapolate (fluid_3d_ex.cc:31-47)
// ---------------------------------------------------------------------------
// lay_ready: the layer tags and claims are already initialised (by the
// snapshot pass of the reference-map update)
static void extrapolate(rmt3d_scene *s, bool lay_ready = false) {
    const grid_dev &g = s->g;
    if (g.n_obj == 0) return;
    const int nb = lin_blocks(g.ncell);
    const int per_warp_blocks = 148 * 8;
    // without a periodic axis no ghost cell is the image of an interior
    // cell, and the two ghost-copy kernels would find nothing to do
    const bool prd = g.prd[0] || g.prd[1] || g.prd[2];
    int *cnt[2] = {s->fcnt, s->fcnt + kMaxObj};
    if (!lay_ready) {
        k_lay_init<<<nb, 256, 0, s->st>>>(g, s->dF, s->lay, s->inl);
        s->count();
    }
    cudaMemsetAsync(s->fcnt, 0, 2 * kMaxObj * sizeof(int), s->st);
    k_lay_push<<<nb, 256, 0, s->st>>>(g, nullptr, nullptr, 1, s->lay, s->inl, 1, s->front[0], cnt[0]);
    s->count();
    if (prd) {
        k_lay_ghost<<<nb, 256, 0, s->st>>>(g, s->lay, s->inl, 1, s->front[0], cnt[0]);
        s->count();
    }
    int cur = 0;
    for (int L = 1; L <= s->d.nlayers; L++) {
        auto kern = s->extrap_lanes == 4 ? k_extrap_layer<4> : k_extrap_layer<32>;
        kern<<<per_warp_blocks, 128, 0, s->st>>>(g, s->dF, s->front[cur], cnt[cur], L, s->d.max_extrap_rs,
                                                 s->d.weight_fac, s->lx, s->ly, s->lz, s->counters + 2);
        s->count();
        if (prd) {
            k_layer_ghost_copy<<<nb, 256, 0, s->st>>>(g, s->dF, L);
            s->count();
        }
        if (L < s->d.nlayers) {
            int nxt = cur ^ 1;
            cudaMemsetAsync(cnt[nxt], 0, kMaxObj * sizeof(int), s->st);
            k_lay_push<<<per_warp_blocks, 256, 0, s->st>>>(g, s->front[cur], cnt[cur], 0, s->lay, s->inl, L + 1,
                                                           s->front[nxt], cnt[nxt]);
            s->count();
            if (prd) {
                k_lay_ghost<<<nb, 256, 0, s->st>>>(g, s->lay, s->inl, L + 1, s->front[nxt], cnt[nxt]);
                s->count();
            }
            cur = nxt;
        }
    }
}

// ---------------------------------------------------------------------------
// host initial conditions (fluid_3d.cc:292-400) -- evaluated on the host
// exactly as the reference does, then uploaded
// ---------------------------------------------------------------------------
static void host_velocity(rmt3d_scene *s, double x, double y, double z, double &u, double &v, double &w) {
    const rmt3d_scene_desc &d = s->d;
    if (d.sim_type == RMT3D_SIM_FTEST) {  // sim_ftest::velocity (sim_manager.cc:139-146)
        u = -sin(2 * M_PI * x) * cos(2 * M_PI * y) * cos(2 * M_PI * z);
        v = 0.5 * cos(2 * M_PI * x) * sin(2 * M_PI * y) * cos(2 * M_PI * z);
        w = 0.5 * cos(2 * M_PI * x) * cos(2 * M_PI * y) * sin(2 * M_PI * z);
    } else if (d.sim_type == RMT3D_SIM_STEST) {  // sim_stest::velocity (:203-210)
        const double a = 0.01, k = 2 * M_PI;
        u = 2 * M_PI * a * sin(k * z);
        v = 2 * M_PI * a * sin(k * z);
        w = 0;
    } else {  // sim_manager::velocity (:102-131)
        u = 0;
        v = 0;
        w = 0;
        const double coords[3] = {x, y, z};
        double rx[3] = {0, 0, 0};
        for (int i = 0; i < d.vel_prof_num; i++) {
            int vt = static_cast<int>(d.vel_profile[2 * i]);
            double amp = d.vel_profile[2 * i + 1];
            if (vt == 0) continue;
            else if (vt == 1) u += amp;
            else if (vt == 2) v += amp;
            else if (vt == 3) w += amp;
        }
        for (int i = 0; i < d.n_obj; i++) {
            s->obj[i].rm0(coords, rx);
            if (s->obj[i].phi(rx) < 0.) s->obj[i].velocity(rx, u, v, w);
        }
    }
    double tmp = sqrt(u * u + v * v + w * w);
    if (tmp > s->vmax) s->vmax = tmp;
}

static void host_exact(rmt3d_scene *s, double x, double y, double z, double t, double h, double &u, double &v,
                       double &w, double &p) {
    const rmt3d_scene_desc &d = s->d;
    if (d.sim_type == RMT3D_SIM_FTEST) {  // sim_ftest::exact (sim_manager.cc:152-167)
        host_velocity(s, x, y, z, u, v, w);
        u *= cos(2 * M_PI * t);
        v *= cos(2 * M_PI * t);
        w *= cos(2 * M_PI * t);
        x -= 0.5 * h;
        y -= 0.5 * h;
        z -= 0.5 * h;
        p = 3 * M_PI * d.fmu * cos(2 * M_PI * x) * cos(2 * M_PI * y) * cos(2 * M_PI * z);
        p *= (cos(2 * M_PI * t) - sin(2 * M_PI * t) / (6 * M_PI * d.fmu));
    } else if (d.sim_type == RMT3D_SIM_STEST) {  // sim_stest::exact (:187-197)
        const double a = 0.01, k = 2 * M_PI, om = 2 * M_PI;
        u = om * a * sin(k * z - om * t);
        v = om * a * sin(k * z - om * t);
        w = 0;
        z -= 0.5 * h;
        p = -s->obj[0].G * a * a * k * (-k * cos(2 * (k * z - om * t)) + cos(2 * om * t - k) * sin(k)) / 3;
    } else {
        u = v = w = p = 0;
    }
}

static double host_pressure(rmt3d_scene *s, double x, double y, double z) {
    const rmt3d_scene_desc &d = s->d;
    if (d.sim_type == RMT3D_SIM_FTEST) return 3 * M_PI * d.fmu * cos(2 * M_PI * x) * cos(2 * M_PI * y) * cos(2 * M_PI * z);
    if (d.sim_type == RMT3D_SIM_STEST) {
        const double a = 0.01, k = 2 * M_PI;
        return -s->obj[0].G * a * a * k * (-k * cos(2 * k * z) + cos(-k) * sin(k)) / 3;
    }
    return 0;
}

// obligatory_cfl_recheck (sim_manager.cc:56-66)
static void cfl_recheck(rmt3d_scene *s) {
    double dh = std::min(s->g.dx, std::min(s->g.dy, s->g.dz));
    double dt_min = s->d.fdt_pad * dh / s->vmax;
    if (s->dt_reg > dt_min) {
        s->dt_reg = dt_min;
        if (s->d.dt < s->dt_reg) s->dt_reg = s->d.dt;
    }
    s->K_stiff = 0.0025 / (s->dt_reg * s->dt_reg);
    s->g.K_stiff = s->K_stiff;
}

static int read_ctl(rmt3d_scene *s);
static bool graph_mode(rmt3d_scene *s);
static int build_step_graph(rmt3d_scene *s);

// ---- initial conditions on the device (the objects simulation) ------------
struct vel_profile_dev {
    int n;
    double e[2 * RMT3D_MAX_VEL_PROF];
};

// sim_manager::velocity (sim_manager.cc:102-131) at every cell of the ghosted
// box, with the running maximum of |u| for the CFL recheck (as ordered bits)
__global__ void k_init_velocity(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                                const double *lz, vel_profile_dev prof, unsigned long long *vmax_bits) {
    const int ind = blockIdx.x * blockDim.x + threadIdx.x;
    double tmp = 0;
    if (ind < g.ncell) {
        const int i = ind % g.sm4, j = (ind / g.sm4) % g.sn4, k = ind / g.smn4;
        const double coords[3] = {lx[i], ly[j], lz[k]};
        double u = 0, v = 0, w = 0;
        for (int q = 0; q < prof.n; q++) {
            const int vt = static_cast<int>(prof.e[2 * q]);
            const double amp = prof.e[2 * q + 1];
            if (vt == 1) u += amp;
            else if (vt == 2) v += amp;
            else if (vt == 3) w += amp;
        }
        for (int o = 0; o < g.n_obj; o++) {
            const obj_dev &ob = g.obj[o];
            double rx[3];
            for (int a = 0; a < 3; a++)
                rx[a] = (ob.type == RMT3D_OBJ_SPHERE) ? (coords[a] - ob.c[a]) * ob.eig[a] + ob.c[a] : coords[a];
            if (obj_phi(g, o, rx[0], rx[1], rx[2]) < 0.) {
                double L[3];
                for (int a = 0; a < 3; a++) L[a] = rx[a] - ob.c[a];
                u += ob.omega[1] * L[2] - ob.omega[2] * L[1];
                v -= ob.omega[0] * L[2] - ob.omega[2] * L[0];
                w += ob.omega[0] * L[1] - ob.omega[1] * L[0];
            }
        }
        F->vel[0][ind] = u;
        F->vel[1][ind] = v;
        F->vel[2][ind] = w;
        tmp = sqrt(u * u + v * v + w * w);
        if (F->rho) F->rho[ind] = g.frho;
    }
    unsigned long long b = (unsigned long long)__double_as_longlong(tmp);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
        b = t > b ? t : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(vmax_bits, b);
}

// fluid_3d::init_refmap (fluid_3d.cc:348-400) on the device: every map reset;
// each interior cell takes the initial map of each object in turn (the last
// one stays in x, as the reference's loop leaves it) and belongs to the first
// object whose level set is negative there
__global__ void k_init_refmap(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                              const double *lz, int *err) {
    const int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    const int i = ind % g.sm4, j = (ind / g.sm4) % g.sn4, k = ind / g.smn4;
    const bool interior = i >= 2 && i < g.sm4 - 2 && j >= 2 && j < g.sn4 - 2 && k >= 2 && k < g.so4 - 2;
    double X[3] = {0, 0, 0};
    int owner = -1;
    if (interior) {
        const double tx[3] = {lx[i], ly[j], lz[k]};
        for (int o = 0; o < g.n_obj; o++) {
            const obj_dev &ob = g.obj[o];
            for (int a = 0; a < 3; a++)
                X[a] = (ob.type == RMT3D_OBJ_SPHERE) ? (tx[a] - ob.c[a]) * ob.eig[a] + ob.c[a] : tx[a];
            if (obj_phi(g, o, X[0], X[1], X[2]) < 0) {
                if (owner < 0) owner = o;
                else atomicAdd(err, 1);
            }
        }
    }
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        m.code[ind] = (owner == o) ? 0 : -1;
        for (int a = 0; a < 3; a++) {
            m.x[a][ind] = X[a];
            m.xp[a][ind] = X[a];
        }
        for (int a = 0; a < 9; a++) m.gp[a][ind] = -kBig;
        for (int a = 0; a < 18; a++) m.fx[a][ind] = 0;
    }
}

// the objects simulation's initial state is computed on the device; the
// manufactured-solution and shear-test cases keep the host path (trigonometric
// initial fields evaluated with the host's libm, as the reference does)
static bool device_init(const rmt3d_scene *s) {
    return s->d.sim_type == RMT3D_SIM_OBJECTS && !s->d.has_exact;
}

// init_fluid (fluid_3d.cc:292-320): every cell reset (p kept), velocities from
// the initial condition, periodic exchange, CFL recheck, dt = dt_reg
static int init_fluid(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    const size_t n = g.ncell;
    if (device_init(s)) {
        CK(cudaMemsetAsync(s->d_red, 0, sizeof(double), s->st));
        vel_profile_dev prof;
        memset(&prof, 0, sizeof(prof));
        prof.n = s->d.vel_prof_num;
        for (int q = 0; q < 2 * RMT3D_MAX_VEL_PROF; q++) prof.e[q] = s->d.vel_profile[q];
        k_init_velocity<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, prof,
                                                                 (unsigned long long *)s->d_red);
        s->count();
        CK(cudaMemsetAsync(s->hF.q, 0, n * 8, s->st));
        CK(cudaMemsetAsync(s->hF.dp, 0, n * 8, s->st));
        for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(s->hF.dvel[c], 0, n * 8, s->st));
        CK(zero_faces(s));
        for (int c = 0; c < 9; c++) CK(cudaMemsetAsync(s->hF.sigma[c], 0, n * 8, s->st));
        CK(cudaMemcpyAsync(s->h_scalar, s->d_red, sizeof(double), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        if (*s->h_scalar > s->vmax) s->vmax = *s->h_scalar;
        periodic(s, {s->hF.vel[0], s->hF.vel[1], s->hF.vel[2]}, {}, 0);
        cfl_recheck(s);
        rmt3d_set_dt(s, s->dt_reg);
        return 0;
    }
    std::vector<double> u(n), v(n), w(n);
    for (int k = 0; k < g.so4; k++)
        for (int j = 0; j < g.sn4; j++)
            for (int i = 0; i < g.sm4; i++) {
                double p, t[3];
                if (s->d.has_exact) host_exact(s, s->hlx[i], s->hly[j], s->hlz[k], s->time, g.dx, t[0], t[1], t[2], p);
                else host_velocity(s, s->hlx[i], s->hly[j], s->hlz[k], t[0], t[1], t[2]);
                size_t id = gidx(g, i, j, k);
                u[id] = t[0];
                v[id] = t[1];
                w[id] = t[2];
            }
    CK(cudaMemcpyAsync(s->hF.vel[0], u.data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->hF.vel[1], v.data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->hF.vel[2], w.data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->hF.q, 0, n * 8, s->st));
    CK(cudaMemsetAsync(s->hF.dp, 0, n * 8, s->st));
    for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(s->hF.dvel[c], 0, n * 8, s->st));
    CK(zero_faces(s));
    for (int c = 0; c < 9; c++) CK(cudaMemsetAsync(s->hF.sigma[c], 0, n * 8, s->st));
    if (s->d.var_den) {
        std::vector<double> r(n, s->d.frho);
        CK(cudaMemcpyAsync(s->hF.rho, r.data(), n * 8, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    periodic(s, {s->hF.vel[0], s->hF.vel[1], s->hF.vel[2]}, {}, 0);
    cfl_recheck(s);
    rmt3d_set_dt(s, s->dt_reg);
    return 0;
}

__global__ void k_zero_pres(grid_dev g, double *p) {
    const int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    const int i = ind % g.sm4, j = (ind / g.sm4) % g.sn4, k = ind / g.smn4;
    if (i >= 2 && i < g.sm4 - 1 && j >= 2 && j < g.sn4 - 1 && k >= 2 && k < g.so4 - 1) p[ind] = 0;
}

// init_pres (fluid_3d.cc:326-343)
static int init_pres(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    const size_t n = g.ncell;
    if (device_init(s)) {
        // sim_manager::pressure is 0 for the objects simulation; the reference
        // writes it to the nodes 2..s+2 and keeps the rest of p
        k_zero_pres<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->hF.p);
        s->count();
        CK(cudaMemsetAsync(s->hF.q, 0, n * 8, s->st));
        comm_pressure(s);
        return 0;
    }
    std::vector<double> p(n);
    CK(cudaMemcpyAsync(p.data(), s->hF.p, n * 8, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    double hdx = g.dx * 0.5, hdy = g.dy * 0.5, hdz = g.dz * 0.5;
    for (int k = 2; k < g.so4 - 1; k++)
        for (int j = 2; j < g.sn4 - 1; j++)
            for (int i = 2; i < g.sm4 - 1; i++)
                p[gidx(g, i, j, k)] = host_pressure(s, s->hlx[i] - hdx, s->hly[j] - hdy, s->hlz[k] - hdz);
    CK(cudaMemcpyAsync(s->hF.p, p.data(), n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->hF.q, 0, n * 8, s->st));
    CK(cudaStreamSynchronize(s->st));
    comm_pressure(s);
    return 0;
}

// init_refmap (fluid_3d.cc:348-400): every map reset; interior cells take the
// initial map of each object in turn and belong to the first object whose
// level set is negative there
static int init_refmap(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (g.n_obj == 0) return 0;
    CK(cudaMemsetAsync(s->counters + 6, 0, sizeof(int), s->st));
    k_init_refmap<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, s->counters + 6);
    s->count();
    int e = read_ctl(s);
    if (e) return e;
    if (s->h_counters[6] > 0) return fail(RMT3D_ERR_INVALID, "init_refmap: overlapping primary points");
    comm_primary(s);
    return 0;
}

// update_rho (fluid_3d.cc:1104-1143), VAR_DEN only
__global__ void k_update_rho(grid_dev g, const fields_dev *__restrict__ F) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    F->rho[ind] = cell_rho(g, F, ind);
}

static void update_rho(rmt3d_scene *s) {
    if (!s->d.var_den) return;
    k_update_rho<<<lin_blocks(s->g.ncell), 256, 0, s->st>>>(s->g, s->dF);
    s->count();
}

// set_rhoinv (Utilities/mg_probs.cc:90-94) on the interior cells, then the
// coarse levels as means of their 8 children
__global__ void k_rinv_fine(grid_dev g, const fields_dev *__restrict__ F, double *ri, float *ris) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.sm || j >= g.sn || k >= g.so) return;
    const double v = 1. / F->rho[gidx(g, i + 2, j + 2, k + 2)];
    const int id = i + g.sm * (j + g.sn * k);
    ri[id] = v;
    if (ris) ris[id] = (float)v;
}

__global__ void k_rinv_coarse(int f0, int f1, int c0, int c1, int c2, const double *rf, double *rc, float *rcs) {
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    int J = blockIdx.y * blockDim.y + threadIdx.y;
    int K = blockIdx.z * blockDim.z + threadIdx.z;
    if (I >= c0 || J >= c1 || K >= c2) return;
    double s = 0;
    for (int c = 0; c < 2; c++)
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) s += rf[(2 * I + a) + f0 * ((2 * J + b) + f1 * (2 * K + c))];
    const int id = I + c0 * (J + c1 * K);
    rc[id] = 0.125 * s;
    if (rcs) rcs[id] = (float)(0.125 * s);
}

static void update_rinv(rmt3d_scene *s) {
    if (!s->d.var_den) return;
    const grid_dev &g = s->g;
    const bool f32 = mixed_form(s->d.precision);
    k_rinv_fine<<<grd(g.sm, g.sn, g.so), blk(), 0, s->st>>>(g, s->dF, s->rinv[0], f32 ? s->rinvs[0] : nullptr);
    s->count();
    for (size_t l = 1; l < s->rinv.size(); l++) {
        const mg_level &F = s->mac.lv[l - 1], &C = s->mac.lv[l];
        k_rinv_coarse<<<grd(C.n[0], C.n[1], C.n[2]), blk(), 0, s->st>>>(F.n[0], F.n[1], C.n[0], C.n[1], C.n[2],
                                                                        s->rinv[l - 1], s->rinv[l],
                                                                        f32 ? s->rinvs[l] : nullptr);
        s->count();
    }
}

// init_extrapolate (fluid_3d_ex.cc:16-27)
static void init_extrapolate(rmt3d_scene *s) {
    if (s->g.n_obj == 0) return;
    extrapolate(s);
    k_extraps_full<<<lin_blocks(s->g.ncell), 256, 0, s->st>>>(s->g, s->dF);
    s->count();
}

// compute_grad_basis (fluid_3d.cc:2506-2517), evaluated with the current dt
static void compute_grad_basis(rmt3d_scene *s) {
    double fac = 3 * s->g.dx / s->dt;
    for (int i = 0; i < 8; i++) {
        s->gradphi.v[i][0] = (2 * (i % 2) - 1) * fac;
        s->gradphi.v[i][1] = (2 * ((i / 2) % 2) - 1) * fac;
        s->gradphi.v[i][2] = (2 * (i / 4) - 1) * fac;
    }
}

// ---------------------------------------------------------------------------
// step phases
// ---------------------------------------------------------------------------
static void compute_stress(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    const bool maps = g.n_obj > 0;
    if (maps) cudaMemsetAsync(s->mcnt, 0, sizeof(int), s->st);
    k_stress_fluid<<<grd_of(s->bshape, g.sm + 4, g.sn + 4, g.so + 4), blk_of(s->bshape), 0, s->st>>>(g, s->dF, maps ? s->mlist : nullptr,
                                                                          s->mcnt);
    s->count();
    if (maps) {
        k_stress<<<148 * 8, 128, 0, s->st>>>(g, s->dF, s->mlist, s->mcnt);
        s->count();
    }
}

// ---- simulation time, kept on the device (read by the kernels) -----------
__global__ void k_time_set(scene_ctl *c, double t) { c->time = t; }
__global__ void k_time_add(scene_ctl *c, double dt_half) { c->time += dt_half; }

static void set_time(rmt3d_scene *s, double t) {
    s->time = t;
    k_time_set<<<1, 1, 0, s->st>>>(s->ctl, t);
    s->count();
}

// time += dt/2 (the two halves of fluid_3d::step_forward, fluid_3d.cc:456,
// :541); the host mirror follows in eager mode and is read back after a
// graph step
static void advance_half(rmt3d_scene *s) {
    if (!s->capturing) s->time += 0.5 * s->dt;
    k_time_add<<<1, 1, 0, s->st>>>(s->ctl, 0.5 * s->dt);
    s->count();
}

// ---- phases of fluid_3d::step_forward (fluid_3d.cc:429-577) ----------------
// compute_half_time_edge_velocities/refmap with their limited derivatives
static void ph_edges(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (s->edge_tma)
        launch_edge_vel_tma(g, s->dF, s->tm_vel, s->lx, s->ly, s->lz, s->dt, &s->ctl->time, s->d.var_den,
                            s->counters + 7, s->st);
    else if (g.f32face)
        k_edge_vel<float><<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, s->dt,
                                                                       &s->ctl->time, s->d.var_den);
    else
        k_edge_vel<double><<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, s->dt,
                                                                        &s->ctl->time, s->d.var_den);
    s->count();
    if (g.n_obj > 0) {
        k_edge_refmap<<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->dt, s->counters + 5);
        s->count();
    }
    advance_half(s);
}

// godunov_upwinding_set between the boundary fills
static void ph_upwind(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    fill_boundary_cf(s);
    comm_face_maps(s);
    if (g.f32face) k_upwind<float><<<grd_of(s->bshape, g.sm + 1, g.sn + 1, g.so + 1), blk_of(s->bshape), 0, s->st>>>(g, s->dF);
    else k_upwind<double><<<grd_of(s->bshape, g.sm + 1, g.sn + 1, g.so + 1), blk_of(s->bshape), 0, s->st>>>(g, s->dF);
    s->count();
    fill_boundary_cf(s);
}

// mac_solve (fluid_3d.cc:2209-2241) before and after the multigrid solve.
// The solve uses the density of the end of the previous step (or of the
// set-up), as mac.set_rhoinv(lrho) does: update_rho last ran with the full
// map update (:1304), before redraw_boundary.
static void ph_mac_pre(rmt3d_scene *s, double cdt) {
    const grid_dev &g = s->g;
    update_rinv(s);
    k_mac_rhs<<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->mac.rhs(), cdt);
    s->count();
}

static void ph_mac_post(rmt3d_scene *s, double cdt) {
    const grid_dev &g = s->g;
    k_mac_extract<<<grd(g.sm, g.sn, g.so), blk(), 0, s->st>>>(g, s->dF, s->mac.sol());
    s->count();
    comm_pressure(s);
    k_sub_qgrad<<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, cdt, s->d.var_den);
    s->count();
    fill_boundary_cf(s);
}

// update_reference_map (fluid_3d.cc:1149-1255) up to the corrector, whose
// problem count lands in counters[3]
static void ph_refmap(rmt3d_scene *s, double cdt) {
    const grid_dev &g = s->g;
    // without a periodic axis nothing changes the codes between the snapshot
    // and the extrapolation, so the snapshot pass sets the layer tags too
    const bool prd = g.prd[0] || g.prd[1] || g.prd[2];
    k_refmap_predict<<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, cdt);
    k_snapshot_reset<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, prd ? nullptr : s->lay, s->inl);
    s->count(2);
    comm_primary(s);
    extrapolate(s, !prd);
    // update_rho follows in the same pass (var_den)
    k_refmap_correct<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, s->counters + 3, s->d.var_den);
    s->count();
}

static void ph_revert(rmt3d_scene *s) {
    k_refmap_revert<<<lin_blocks(s->g.ncell), 256, 0, s->st>>>(s->g, s->dF);
    s->count();
}

// compute_ustar (fluid_3d.cc:1309-1352) and its boundary fills
static void ph_ustar(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (g.f32face)
        k_ustar<float><<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, s->dt,
                                                                    &s->ctl->time, s->d.var_den);
    else
        k_ustar<double><<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, s->dt,
                                                                     &s->ctl->time, s->d.var_den);
    s->count();
    fill_boundary_cc(s);
    comm_dvel(s);
    advance_half(s);
}

// Mean of x in a fixed summation order: each block writes its partial sum,
// and the last block to finish adds the partials in block order, so the
// result does not depend on scheduling (scenes give the same answer alone
// and when they share the device with others).
constexpr int kMeanBlocks = 148;
constexpr int kDiagVals = 8;

__global__ void k_mean(const double *x, size_t n, double scale, double *out, unsigned *ticket) {
    double sum = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        sum += x[i] * scale;
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    __shared__ double sh[32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) {
            out[1 + blockIdx.x] = v;
            __threadfence();
            last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const volatile double *part = out + 1;
        double t = 0;
        for (unsigned b = 0; b < gridDim.x; b++) t += part[b];
        out[0] = t;
        *ticket = 0;
    }
}

// pp_solve (fluid_3d.cc:2653-2681) before and after the multigrid solve
static void ph_pp_pre(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    // the density is already that of the current maps: update_rho ran after
    // the reference-map update, and nothing since has moved a map
    update_rinv(s);
    k_fem_rhs<<<grd_of(s->bshape, g.fm, g.fn, g.fo), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->fem.rhs(), s->gradphi);
    s->count();
}

static void ph_pp_post(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    size_t nn = (size_t)g.fm * g.fn * g.fo;
    k_mean<<<kMeanBlocks, 256, 0, s->st>>>(s->fem.sol(), nn, 1 / (double)nn, s->d_mean, s->mean_ticket);
    k_fem_extract<<<grd(g.fm, g.fn, g.fo), blk(), 0, s->st>>>(g, s->dF, s->fem.sol(), s->d_mean);
    s->count(2);
    comm_pressure(s);
    k_sub_pgrad<<<grd_of(s->bshape, g.sm, g.sn, g.so), blk_of(s->bshape), 0, s->st>>>(g, s->dF, s->dt, s->d.var_den);
    s->count();
}

// update_reference_map_full, update_rho, redraw_boundary, boundary fills
// (fluid_3d.cc:559-574)
static void ph_final(rmt3d_scene *s) {
    const grid_dev &g = s->g;
    if (g.n_obj > 0) {
        // update_rho follows in the same pass (var_den)
        k_refmap_full<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, s->d.var_den);
        s->count();
        k_redraw<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, s->d.nlayers, s->counters + 4);
        s->count();
    }
    fill_boundary_cc(s);
    comm_dvel(s);
}

// ---------------------------------------------------------------------------
// passive tracers (Utilities/tracers.{hh,cc}); kernels in k_tracer.cu
// ---------------------------------------------------------------------------
static tracer_args tr_args(const rmt3d_scene *s) {
    tracer_args A;
    memset(&A, 0, sizeof(A));
    A.pc = s->tr_pc;
    A.rp = s->tr_rp;
    A.alive = s->tr_alive;
    const double h[3] = {s->g.dx, s->g.dy, s->g.dz};
    const double ax[3] = {s->g.ax, s->g.ay, s->g.az};
    const int cells[3] = {s->g.sm, s->g.sn, s->g.so};
    for (int f = 0; f < 3; f++) {
        A.h[f] = h[f];
        A.low[f] = ax[f] + (0 + 0 - 2 + 0.5) * h[f];  // lx[0] (fluid_3d.cc:136-138)
        const double g0 = ax[f] + (0 + 0.5) * h[f];  // gx[0] (fluid_3d.cc:132-134)
        A.lo[f] = g0 - 0.5 * h[f];
        A.hi[f] = A.lo[f] + cells[f] * h[f];
        for (int lr = 0; lr < 2; lr++)
            A.homog[f][lr] = s->d.bct[f][2 * f + lr] == 1 && s->d.bcv[f][2 * f + lr] == 0;
    }
    A.dt = s->dt;
    return A;
}

// tracers::predict at the start of a step, tracers::advect at its end
// (fluid_3d.cc:459-461, 570-572)
static void tracer_predict(rmt3d_scene *s) {
    if (!s->ntr) return;
    k_tracer_predict<<<(s->ntr + 127) / 128, 128, 0, s->st>>>(s->g, s->dF, tr_args(s), s->ntr);
    s->count();
}
static void tracer_advect(rmt3d_scene *s) {
    if (!s->ntr) return;
    k_tracer_advect<<<(s->ntr + 127) / 128, 128, 0, s->st>>>(s->g, s->dF, tr_args(s), s->ntr);
    s->count();
}

// tracers::set for every tracer, from host coordinates xyz[3 * ntr]
static int tracers_place(rmt3d_scene *s, const double *xyz) {
    double *d = nullptr;
    const size_t bytes = 3 * (size_t)s->ntr * sizeof(double);
    CK(cudaMallocAsync((void **)&d, bytes, s->st));
    cudaError_t ce = cudaMemcpyAsync(d, xyz, bytes, cudaMemcpyHostToDevice, s->st);
    if (ce == cudaSuccess) {
        k_tracer_place<<<(s->ntr + 127) / 128, 128, 0, s->st>>>(s->g, tr_args(s), s->ntr, d);
        s->count();
        ce = cudaStreamSynchronize(s->st);
    }
    cudaFreeAsync(d, s->st);
    CK(ce);
    return 0;
}

// The tracers constructor (tracers.cc:7-70): a fresh start scatters them
// uniformly over the domain; a restart reads the checkpoint's tr.<chk_num>
// file.  The uniform draws are SplitMix64 (Steele, Lea and Flood 2014,
// seed 1), not GSL's taus generator, so a fresh start places the tracers
// elsewhere than the reference does; a restart places them identically.
static int alloc_tracers(rmt3d_scene *s, const char *chk_dir) {
    if (!s->ntr) return 0;
    std::vector<double> xyz(3 * (size_t)s->ntr);
    if (chk_dir) {
        char fn[700];
        snprintf(fn, sizeof(fn), "%s/tr.%05d", chk_dir, s->d.run.chk_num);
        std::vector<float> pos;
        int e = tracer_read_file(fn, s->ntr, pos);
        if (e) return e;
        for (size_t i = 0; i < xyz.size(); i++) xyz[i] = pos[i];
    } else {
        uint64_t state = 1;
        auto uniform = [&]() {
            uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            z ^= z >> 31;
            return (double)(z >> 11) * (1.0 / 9007199254740992.0);
        };
        const double h[3] = {s->g.dx, s->g.dy, s->g.dz};
        const double ax[3] = {s->g.ax, s->g.ay, s->g.az};
        const int cells[3] = {s->g.sm, s->g.sn, s->g.so};
        for (int t = 0; t < s->ntr; t++)
            for (int f = 0; f < 3; f++) {
                const double lo = (ax[f] + 0.5 * h[f]) - 0.5 * h[f];
                xyz[3 * t + f] = lo + cells[f] * h[f] * uniform();
            }
    }
    return tracers_place(s, xyz.data());
}

static int read_ctl(rmt3d_scene *s) {
    CK(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(scene_ctl), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

static int extrap_errors(rmt3d_scene *s) {
    if (s->h_counters[2] > 0) return fail(RMT3D_ERR_EXTRAP, "Extrapolation failed: no eligible points or degenerate matrix");
    if (s->h_counters[5] > 0)
        return fail(RMT3D_ERR_EXTRAP, "normal_derivatives_refmap: missing necessary cells to carry out finite differences");
    return 0;
}

// The step issued kernel by kernel with the host checking each solve and
// each error counter where the reference does (used for the set-up
// iterations, phase-by-phase inspection and kernel profiling).  `stop`
// ends the step after that phase group.
static int step_forward(rmt3d_scene *s, int debug, int stop = 99) {
    const grid_dev &g = s->g;
    (void)debug;
    s->nt++;
    CK(cudaMemsetAsync(s->counters + 2, 0, 6 * sizeof(int), s->st));
    tracer_predict(s);
    compute_stress(s);
    if (stop <= 1) return RMT3D_OK;
    ph_edges(s);
    if (s->edge_tma) {
        int e = read_ctl(s);
        if (e) return e;
        if (s->h_counters[7] > 0) return fail(RMT3D_ERR_CUDA, "k_edge_vel_tma: a staged velocity plane never arrived");
    }
    if (stop <= 2) return RMT3D_OK;
    ph_upwind(s);
    if (stop <= 3) return RMT3D_OK;
    ph_mac_pre(s, s->dt);
    double res = s->mac.run(s->st);
    if (std::isnan(res)) {
        CK(cudaGetLastError());
        return fail(RMT3D_ERR_NAN, "fluid_3d::mac_solve(): NaN detected in multigrid solve");
    }
    ph_mac_post(s, s->dt);
    if (stop <= 4) return RMT3D_OK;
    if (g.n_obj > 0) {
        ph_refmap(s, s->dt);
        int e = read_ctl(s);
        if (!e) e = extrap_errors(s);
        if (e) return e;
        if (s->h_counters[3]) {
            ph_revert(s);
            return RMT3D_REFMAP_UPDATE_ERR;
        }
    }
    if (stop <= 5) return RMT3D_OK;
    compute_stress(s);
    if (stop <= 6) return RMT3D_OK;
    ph_ustar(s);
    if (stop <= 7) return RMT3D_OK;
    ph_pp_pre(s);
    res = s->fem.run(s->st);
    if (std::isnan(res)) return RMT3D_PROJECTION_ERR;
    ph_pp_post(s);
    if (stop <= 8) return RMT3D_OK;
    ph_final(s);
    tracer_advect(s);
    if (g.n_obj > 0) {
        int e = read_ctl(s);
        if (e) return e;
        if (s->h_counters[4] > 0)
            return fail(RMT3D_ERR_INVALID, "redraw_boundary(): Two deep maps try to be inside a cell at the same time!");
    }
    CK(cudaGetLastError());
    return RMT3D_OK;
}

// ---- the step as one CUDA graph --------------------------------------------
// Gate: a step runs only while no earlier step of the graph failed; the
// per-step error counters start at zero.
__global__ void k_step_gate(scene_ctl *c, cudaGraphConditionalHandle h) {
    const bool run = c->halted == 0;
    if (run)
        for (int i = 2; i < 8; i++) c->counters[i] = 0;
    cudaGraphSetConditional(h, run ? 1u : 0u);
}

// After update_reference_map: continue, or revert the maps (corrector
// problem), or neither (an error already ends the step).
__global__ void k_step_branch(scene_ctl *c, cudaGraphConditionalHandle h_rest, cudaGraphConditionalHandle h_rev) {
    const bool err = c->mac.nan || c->counters[2] > 0 || c->counters[5] > 0;
    cudaGraphSetConditional(h_rest, (!err && c->counters[3] == 0) ? 1u : 0u);
    cudaGraphSetConditional(h_rev, (!err && c->counters[3] != 0) ? 1u : 0u);
}

// The step's status, in the order the eager step reports them.
__global__ void k_step_end(scene_ctl *c, int with_objects) {
    int st = 0;
    if (c->counters[7] > 0) st = RMT3D_ERR_CUDA;  // a TMA-staged tile never arrived
    else if (c->mac.nan) st = RMT3D_ERR_NAN;
    else if (with_objects && (c->counters[2] > 0 || c->counters[5] > 0)) st = RMT3D_ERR_EXTRAP;
    else if (with_objects && c->counters[3] != 0) st = RMT3D_REFMAP_UPDATE_ERR;
    else if (c->fem.nan) st = RMT3D_PROJECTION_ERR;
    else if (with_objects && c->counters[4] > 0) st = RMT3D_ERR_INVALID;
    c->status = st;
    c->halted = st != 0;
    c->steps++;
}

// phases 6-9 (after a successful reference-map update)
static int capture_rest(rmt3d_scene *s) {
    compute_stress(s);
    ph_ustar(s);
    ph_pp_pre(s);
    if (s->fem.capture_solve(s->st, s->gb) < 0) return 1;
    s->launches += s->fem.outside_kernels;
    ph_pp_post(s);
    ph_final(s);
    tracer_advect(s);
    return 0;
}

static int build_step_graph(rmt3d_scene *s) {
    if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
    s->step_exec = nullptr;
    if (s->gb.init()) return fail(RMT3D_ERR_CUDA, "stream creation failed");
    s->gb.err = cudaSuccess;
    s->gb.depth = 0;
    const cudaStream_t main = s->st;
    const long long saved = s->launches;
    s->launches = 0;
    s->capturing = true;
    int bad = 0;
    CK(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
    cudaGraphConditionalHandle h_step = s->gb.handle(main);
    k_step_gate<<<1, 1, 0, main>>>(s->ctl, h_step);
    s->count();
    cudaStream_t b1 = s->gb.open(main, h_step, cudaGraphCondTypeIf);
    if (b1) {
        s->st = b1;
        tracer_predict(s);
        compute_stress(s);
        ph_edges(s);
        ph_upwind(s);
        ph_mac_pre(s, s->dt);
        if (s->mac.capture_solve(s->st, s->gb) < 0) bad = 1;
        s->launches += s->mac.outside_kernels;
        ph_mac_post(s, s->dt);
        if (s->g.n_obj > 0) {
            ph_refmap(s, s->dt);
            cudaGraphConditionalHandle h_rev = s->gb.handle(b1), h_rest = s->gb.handle(b1);
            k_step_branch<<<1, 1, 0, b1>>>(s->ctl, h_rest, h_rev);
            s->count();
            cudaStream_t b2 = s->gb.open(b1, h_rev, cudaGraphCondTypeIf);
            if (b2) {
                const long long l0 = s->launches;
                s->st = b2;
                ph_revert(s);
                s->launches = l0;  // the revert branch is not part of a normal step
                s->gb.close(b2);
            }
            b2 = s->gb.open(b1, h_rest, cudaGraphCondTypeIf);
            if (b2) {
                s->st = b2;
                bad |= capture_rest(s);
                s->gb.close(b2);
            }
            s->st = b1;
        } else {
            bad |= capture_rest(s);
        }
        k_step_end<<<1, 1, 0, b1>>>(s->ctl, s->g.n_obj > 0);
        s->count();
        s->gb.close(b1);
    }
    s->st = main;
    cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(scene_ctl), cudaMemcpyDeviceToHost, main);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(main, &graph);
    s->capturing = false;
    s->graph_fixed = s->launches;
    s->launches = saved;
    if (bad || e != cudaSuccess || s->gb.err != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return fail(RMT3D_ERR_CUDA, std::string("step graph capture failed: ") +
                                        cudaGetErrorString(e != cudaSuccess ? e : s->gb.err));
    }
    e = cudaGraphInstantiate(&s->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(RMT3D_ERR_CUDA, std::string("step graph instantiation: ") + cudaGetErrorString(e));
    s->graph_dirty = false;
    return 0;
}

struct pending_steps_g {
    long long c0 = 0, f0 = 0;
    int steps0 = 0;
};

// ---- groups: equally sized scenes stepped by one graph ---------------------
// The per-scene phases run as parallel branches of one graph (one branch per
// scene, forked and joined around the solves); each of the two multigrid
// solves is one batched solve over the group (k_mgb.cu), each phase one
// launch over all scenes.  A scene's gates are device flags: a halted scene
// skips its branches and sits out the solves; a scene whose MAC solve gave
// NaN or whose reference-map update must be reverted sits out the FEM solve.

// step start: run only while not halted; per-step counters to zero; the
// scene takes part in the MAC solve when it runs
__global__ void k_gstep_gate(scene_ctl *c, int *mac_part, cudaGraphConditionalHandle h) {
    const int run = c->halted == 0;
    if (run)
        for (int i = 2; i < 8; i++) c->counters[i] = 0;
    c->run_flag = run;
    *mac_part = run;
    cudaGraphSetConditional(h, run ? 1u : 0u);
}

// after the MAC solve: continue when the step runs and the solve is finite;
// the FEM solve flag starts cleared and is set by the branch that reaches it
__global__ void k_gstep_seg2(scene_ctl *c, int *fem_part, cudaGraphConditionalHandle h) {
    *fem_part = 0;
    cudaGraphSetConditional(h, (c->run_flag && !c->mac.nan) ? 1u : 0u);
}

// after update_reference_map (objects): continue or revert, and take part in
// the FEM solve only when continuing
__global__ void k_gstep_branch(scene_ctl *c, int *fem_part, cudaGraphConditionalHandle h_rest,
                               cudaGraphConditionalHandle h_rev) {
    const bool err = c->mac.nan || c->counters[2] > 0 || c->counters[5] > 0;
    const bool rest = !err && c->counters[3] == 0;
    *fem_part = rest;
    cudaGraphSetConditional(h_rest, rest ? 1u : 0u);
    cudaGraphSetConditional(h_rev, (!err && c->counters[3] != 0) ? 1u : 0u);
}

__global__ void k_set_flag(int *f, int v) { *f = v; }

// after the FEM solve: the rest of the step for the scenes that took part
__global__ void k_gstep_seg3(const int *fem_part, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, *fem_part ? 1u : 0u);
}

__global__ void k_gstep_end(scene_ctl *c, int with_objects) {
    if (!c->run_flag) return;
    int st = 0;
    if (c->counters[7] > 0) st = RMT3D_ERR_CUDA;  // a TMA-staged tile never arrived
    else if (c->mac.nan) st = RMT3D_ERR_NAN;
    else if (with_objects && (c->counters[2] > 0 || c->counters[5] > 0)) st = RMT3D_ERR_EXTRAP;
    else if (with_objects && c->counters[3] != 0) st = RMT3D_REFMAP_UPDATE_ERR;
    else if (c->fem.nan) st = RMT3D_PROJECTION_ERR;
    else if (with_objects && c->counters[4] > 0) st = RMT3D_ERR_INVALID;
    c->status = st;
    c->halted = st != 0;
    c->steps++;
}

// Small pinned host blocks (the control mirrors) are recycled within the
// process instead of being freed: cudaFreeHost would synchronise the whole
// device, which scenes that come and go next to running ones (serving) must
// not do.
namespace {
std::mutex g_pin_mu;
std::map<size_t, std::vector<void *>> g_pin_free;
}  // namespace

static void *pinned_get(size_t n) {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto &v = g_pin_free[n];
        if (!v.empty()) {
            void *p = v.back();
            v.pop_back();
            return p;
        }
    }
    void *p = nullptr;
    return cudaMallocHost(&p, n) == cudaSuccess ? p : nullptr;
}

static void pinned_put(void *p, size_t n) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free[n].push_back(p);
}

namespace rmt3d {
struct scene_group {
    std::vector<rmt3d_scene *> sc;
    mg_group mac, fem;
    graph_builder gb;
    cudaStream_t st = nullptr;
    std::vector<cudaStream_t> br;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> fixed;     // per scene: its own kernels per step
    std::vector<long long> version;   // the scenes' parameter versions at capture
    long long mg_launches = 0;        // batched multigrid kernels issued so far
    std::vector<pending_steps_g> pend;
    ~scene_group() {
        if (st) cudaStreamSynchronize(st);
        mac.release();  // stream-ordered frees on st, before st goes
        fem.release();
        if (exec) cudaGraphExecDestroy(exec);
        gb.release();
        for (cudaStream_t b : br) cudaStreamDestroy(b);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (cudaEvent_t e : ev_join) cudaEventDestroy(e);
        if (st) cudaStreamDestroy(st);
    }
};
}  // namespace rmt3d

// fork the capture of `main` into the scenes' branch streams
static int g_fork(scene_group &G, cudaStream_t main) {
    CK(cudaEventRecord(G.ev_fork, main));
    for (cudaStream_t b : G.br) CK(cudaStreamWaitEvent(b, G.ev_fork, 0));
    return 0;
}
static int g_join(scene_group &G, cudaStream_t main) {
    for (size_t b = 0; b < G.br.size(); b++) {
        CK(cudaEventRecord(G.ev_join[b], G.br[b]));
        CK(cudaStreamWaitEvent(main, G.ev_join[b], 0));
    }
    return 0;
}

// capture work of scene b on its branch stream, counting its kernels
template <typename F>
static void g_on(scene_group &G, size_t b, F fn) {
    rmt3d_scene *s = G.sc[b];
    const cudaStream_t saved = s->st;
    const long long l0 = s->launches;
    s->st = G.br[b];
    s->capturing = true;
    fn(s);
    s->capturing = false;
    G.fixed[b] += s->launches - l0;
    s->launches = l0;
    s->st = saved;
}

// an IF node on scene b's current stream whose handle a kernel has just set
template <typename F>
static void g_if(scene_group &G, rmt3d_scene *s, cudaGraphConditionalHandle h, F body) {
    const cudaStream_t cur = s->st;
    cudaStream_t bs = G.gb.open(cur, h, cudaGraphCondTypeIf);
    if (!bs) return;
    s->st = bs;
    body();
    s->st = cur;
    G.gb.close(bs);
}

static int build_group_graph(scene_group &G) {
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
    if (G.gb.init()) return fail(RMT3D_ERR_CUDA, "stream creation failed");
    G.gb.err = cudaSuccess;
    G.gb.depth = 0;
    const size_t B = G.sc.size();
    G.fixed.assign(B, 0);
    G.version.clear();
    for (rmt3d_scene *s : G.sc) G.version.push_back(s->param_version);
    const cudaStream_t main = G.st;
    CK(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
    // phases 1-4 up to the MAC solve
    g_fork(G, main);
    for (size_t b = 0; b < B; b++)
        g_on(G, b, [&](rmt3d_scene *s) {
            cudaGraphConditionalHandle h = G.gb.handle(s->st);
            k_gstep_gate<<<1, 1, 0, s->st>>>(s->ctl, G.mac.part + b, h);
            s->count();
            g_if(G, s, h, [&]() {
                tracer_predict(s);
                compute_stress(s);
                ph_edges(s);
                ph_upwind(s);
                ph_mac_pre(s, s->dt);
            });
        });
    g_join(G, main);
    if (G.mac.capture(main, G.gb)) G.gb.note(cudaErrorUnknown);
    // phases 4-7 up to the FEM solve
    g_fork(G, main);
    for (size_t b = 0; b < B; b++)
        g_on(G, b, [&](rmt3d_scene *s) {
            int *fp = G.fem.part + b;
            cudaGraphConditionalHandle h2 = G.gb.handle(s->st);
            k_gstep_seg2<<<1, 1, 0, s->st>>>(s->ctl, fp, h2);
            s->count();
            g_if(G, s, h2, [&]() {
                ph_mac_post(s, s->dt);
                auto rest = [&]() {
                    compute_stress(s);
                    ph_ustar(s);
                    ph_pp_pre(s);
                };
                if (s->g.n_obj > 0) {
                    ph_refmap(s, s->dt);
                    cudaGraphConditionalHandle h_rev = G.gb.handle(s->st), h_rest = G.gb.handle(s->st);
                    k_gstep_branch<<<1, 1, 0, s->st>>>(s->ctl, fp, h_rest, h_rev);
                    s->count();
                    g_if(G, s, h_rev, [&]() {
                        const long long l0 = s->launches;
                        ph_revert(s);
                        s->launches = l0;  // not part of a normal step
                    });
                    g_if(G, s, h_rest, rest);
                } else {
                    rest();
                    k_set_flag<<<1, 1, 0, s->st>>>(fp, 1);
                    s->count();
                }
            });
        });
    g_join(G, main);
    if (G.fem.capture(main, G.gb)) G.gb.note(cudaErrorUnknown);
    // phases 8-9 and the step's status
    g_fork(G, main);
    for (size_t b = 0; b < B; b++)
        g_on(G, b, [&](rmt3d_scene *s) {
            cudaGraphConditionalHandle h3 = G.gb.handle(s->st);
            k_gstep_seg3<<<1, 1, 0, s->st>>>(G.fem.part + b, h3);
            s->count();
            g_if(G, s, h3, [&]() {
                ph_pp_post(s);
                ph_final(s);
                tracer_advect(s);
            });
            k_gstep_end<<<1, 1, 0, s->st>>>(s->ctl, s->g.n_obj > 0);
            s->count();
            cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(scene_ctl), cudaMemcpyDeviceToHost, s->st);
        });
    g_join(G, main);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(main, &graph);
    if (e != cudaSuccess || G.gb.err != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return fail(RMT3D_ERR_CUDA, std::string("group graph capture failed: ") +
                                        cudaGetErrorString(e != cudaSuccess ? e : G.gb.err));
    }
    e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(RMT3D_ERR_CUDA, std::string("group graph instantiation: ") + cudaGetErrorString(e));
    return 0;
}

namespace rmt3d {
int group_create(rmt3d_scene *const *scenes, int n, scene_group **out) {
    *out = nullptr;
    scene_group *G = new scene_group();
    G->sc.assign(scenes, scenes + n);
    std::vector<mg_solver *> ms, fs;
    for (rmt3d_scene *s : G->sc) {
        ms.push_back(&s->mac);
        fs.push_back(&s->fem);
        const rmt3d_scene *s0 = G->sc[0];
        if (s->g.sm != s0->g.sm || s->g.sn != s0->g.sn || s->g.so != s0->g.so || s->g.prd[0] != s0->g.prd[0] ||
            s->g.prd[1] != s0->g.prd[1] || s->g.prd[2] != s0->g.prd[2]) {
            delete G;
            return fail(RMT3D_ERR_INVALID, "scenes of a group must have the same grid");
        }
    }
    int e = cudaStreamCreateWithFlags(&G->st, cudaStreamNonBlocking) != cudaSuccess ? RMT3D_ERR_CUDA : 0;
    if (!e) e = G->mac.setup(ms, G->st);
    if (!e) e = G->fem.setup(fs, G->st);
    if (!e && cudaEventCreateWithFlags(&G->ev_fork, cudaEventDisableTiming) != cudaSuccess) e = RMT3D_ERR_CUDA;
    for (int b = 0; b < n && !e; b++) {
        cudaStream_t bs;
        cudaEvent_t ev;
        if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            e = RMT3D_ERR_CUDA;
            break;
        }
        G->br.push_back(bs);
        G->ev_join.push_back(ev);
    }
    // the group's launches must follow each scene's outstanding work
    for (rmt3d_scene *s : G->sc)
        if (!e && cudaStreamSynchronize(s->st) != cudaSuccess) e = RMT3D_ERR_CUDA;
    // scenes that share the GPU with the rest of their group extrapolate with
    // 4 lanes per frontier cell (more cells in flight)
    if (!e)
        for (rmt3d_scene *s : G->sc) set_extrap_lanes(s, n > 1 ? 4 : 32);
    if (!e) e = build_group_graph(*G);
    if (e) {
        delete G;
        return e < 0 ? e : fail(RMT3D_ERR_CUDA, "group set-up failed");
    }
    *out = G;
    return 0;
}

void group_destroy(scene_group *G) {
    if (!G) return;
    cudaStreamSynchronize(G->st);
    for (rmt3d_scene *s : G->sc) set_extrap_lanes(s, 32);
    delete G;
}

int group_launch(scene_group *G, int nsteps) {
    G->pend.assign(G->sc.size(), pending_steps_g{});
    for (size_t b = 0; b < G->sc.size(); b++) {
        rmt3d_scene *s = G->sc[b];
        if (s->param_version != G->version[b]) {
            // dt, basis or schedule of a scene changed since the capture
            int e = build_group_graph(*G);
            if (e) return e;
        }
        G->pend[b].c0 = s->mac.cycles_total;
        G->pend[b].f0 = s->fem.cycles_total;
        G->pend[b].steps0 = s->h_ctl->steps;
        CK(cudaMemsetAsync(&s->ctl->halted, 0, sizeof(int), G->st));
        CK(cudaMemsetAsync(&s->ctl->status, 0, sizeof(int), G->st));
    }
    for (int i = 0; i < nsteps; i++) CK(cudaGraphLaunch(G->exec, G->st));
    G->mg_launches += (long long)nsteps * (G->mac.outside_kernels + G->fem.outside_kernels);
    return 0;
}

bool group_done(scene_group *G) { return cudaStreamQuery(G->st) != cudaErrorNotReady; }

int group_finish(scene_group *G, int *status) {
    CK(cudaStreamSynchronize(G->st));
    CK(cudaGetLastError());
    int first_err = 0;
    std::string msg;
    long long cmax = 0, fmax = 0;
    for (size_t b = 0; b < G->sc.size(); b++) {
        rmt3d_scene *s = G->sc[b];
        const scene_ctl &h = *s->h_ctl;
        const int done = h.steps - G->pend[b].steps0;
        s->nt += done;
        s->time = h.time;
        s->mac.sync_host_mirror();
        s->fem.sync_host_mirror();
        cmax = std::max(cmax, s->mac.cycles_total - G->pend[b].c0);
        fmax = std::max(fmax, s->fem.cycles_total - G->pend[b].f0);
        s->launches += (long long)done * G->fixed[b];
        status[b] = h.status;
        if (h.status < 0 && !first_err) {
            first_err = h.status;
            msg = "scene " + std::to_string(b) + ": step status " + std::to_string(h.status);
        }
    }
    // the batched loops ran as many iterations as the slowest scene needed
    G->mg_launches += cmax * G->mac.body_kernels + fmax * G->fem.body_kernels;
    if (first_err) return fail(first_err, msg);
    return 0;
}

long long group_mg_launches(const scene_group *G) { return G->mg_launches; }
}  // namespace rmt3d

struct pending_steps {
    long long c0, f0;
    int steps0;
    int eager_status;
    int eager_err;
};
static thread_local std::vector<std::pair<rmt3d_scene *, pending_steps>> t_pending;

static pending_steps *pending_of(rmt3d_scene *s) {
    for (auto &p : t_pending)
        if (p.first == s) return &p.second;
    t_pending.push_back({s, pending_steps{}});
    return &t_pending.back().second;
}

static int graph_launch(rmt3d_scene *s, int nsteps, pending_steps &p) {
    if (s->graph_dirty || !s->step_exec) {
        int e = build_step_graph(s);
        if (e) return e;
    }
    p.c0 = s->mac.cycles_total;
    p.f0 = s->fem.cycles_total;
    p.steps0 = s->h_ctl->steps;
    CK(cudaMemsetAsync(&s->ctl->halted, 0, sizeof(int), s->st));
    CK(cudaMemsetAsync(&s->ctl->status, 0, sizeof(int), s->st));
    for (int i = 0; i < nsteps; i++) CK(cudaGraphLaunch(s->step_exec, s->st));
    return 0;
}

static int graph_finish(rmt3d_scene *s, const pending_steps &p, int *status) {
    CK(cudaStreamSynchronize(s->st));
    CK(cudaGetLastError());
    const scene_ctl &h = *s->h_ctl;
    const int done = h.steps - p.steps0;
    s->nt += done;
    s->time = h.time;
    s->mac.sync_host_mirror();
    s->fem.sync_host_mirror();
    s->launches += (long long)done * s->graph_fixed + (s->mac.cycles_total - p.c0) * s->mac.body_kernels +
                   (s->fem.cycles_total - p.f0) * s->fem.body_kernels;
    *status = h.status;
    switch (h.status) {
        case RMT3D_ERR_NAN: return fail(RMT3D_ERR_NAN, "fluid_3d::mac_solve(): NaN detected in multigrid solve");
        case RMT3D_ERR_EXTRAP: return extrap_errors(s);
        case RMT3D_ERR_INVALID:
            return fail(RMT3D_ERR_INVALID, "redraw_boundary(): Two deep maps try to be inside a cell at the same time!");
        default: return 0;
    }
}

static int run_graph(rmt3d_scene *s, int nsteps, int *status) {
    pending_steps p;
    int e = graph_launch(s, nsteps, p);
    if (e) return e;
    return graph_finish(s, p, status);
}

// div_u (fluid_3d_utils.cc:507-560): weighted L2 norm of the FEM rhs, reduced
// in a fixed order
static int div_u(rmt3d_scene *s, double *out) {
    const grid_dev &g = s->g;
    k_fem_rhs<<<grd(g.fm, g.fn, g.fo), blk(), 0, s->st>>>(g, s->dF, s->fem.rhs(), s->gradphi);
    k_divu_l2<<<kMeanBlocks, 256, 0, s->st>>>(g, s->fem.rhs(), s->d_diag, s->diag_ticket);
    s->count(2);
    CK(cudaMemcpyAsync(s->h_scalar, s->d_diag, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    *out = sqrt(*s->h_scalar / ((double)g.fm * g.fn * g.fo));
    return 0;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int rmt3d_scene_create(const rmt3d_scene_desc *desc, void *stream, rmt3d_scene **out) {
    if (!desc || !out) return fail(RMT3D_ERR_INVALID, "null argument");
    *out = nullptr;
    const rmt3d_scene_desc &d = *desc;
    for (int a = 0; a < 3; a++)
        if (d.sys_size[a] < 4 || d.sys_size[a] > 1024) return fail(RMT3D_ERR_INVALID, "sys_size outside 4..1024");
    if (d.n_obj < 0 || d.n_obj > RMT3D_MAX_OBJ) return fail(RMT3D_ERR_TOO_LARGE, "n_obj outside 0..16");
    if (d.implicit_visc) return fail(RMT3D_ERR_UNSUPPORTED, "implicit viscosity is outside this path");
    if (!d.godunov) return fail(RMT3D_ERR_UNSUPPORTED, "only the Godunov scheme is on this path");
    if (d.sim_type == RMT3D_SIM_STEST) return fail(RMT3D_ERR_UNSUPPORTED, "stest (shear cube object) is outside this path");
    for (int o = 0; o < d.n_obj; o++)
        if (d.obj[o].type != RMT3D_OBJ_BASIC_SPHERE && d.obj[o].type != RMT3D_OBJ_SPHERE)
            return fail(RMT3D_ERR_UNSUPPORTED, "object type " + std::to_string(d.obj[o].type) + " is outside this path");
    if (d.nlayers < 1 || d.nlayers > 60) return fail(RMT3D_ERR_INVALID, "nlayers outside 1..60");
    if (d.precision < RMT3D_FP64 || d.precision > RMT3D_MIXED_BULK32)
        return fail(RMT3D_ERR_INVALID, "precision must be RMT3D_FP64, RMT3D_MIXED or RMT3D_MIXED_BULK32");

    rmt3d_scene *s = new rmt3d_scene();
    s->d = d;
    if (stream) {
        s->st = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
            delete s;
            return fail(RMT3D_ERR_CUDA, "stream creation failed");
        }
        s->own_stream = true;
    }
    {
        // keep up to 16 GB of freed scene memory in the device's pool, so that
        // scenes created after others were destroyed reuse it without a trip
        // to the driver's allocator
        static std::mutex mu;
        static bool done[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64 && !done[dev]) {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t thr = 16ull << 30;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            }
            done[dev] = true;
        }
    }
    grid_dev &g = s->g;
    memset(&g, 0, sizeof(g));
    g.sm = d.sys_size[0];
    g.sn = d.sys_size[1];
    g.so = d.sys_size[2];
    g.sm4 = g.sm + 4;
    g.sn4 = g.sn + 4;
    g.so4 = g.so + 4;
    g.smn4 = g.sm4 * g.sn4;
    g.ncell = g.smn4 * g.so4;
    for (int a = 0; a < 3; a++) g.prd[a] = d.periodic[a];
    g.fm = g.sm + (g.prd[0] ? 0 : 1);
    g.fn = g.sn + (g.prd[1] ? 0 : 1);
    g.fo = g.so + (g.prd[2] ? 0 : 1);
    // sim_params.cc:368-370
    double lxx = d.bounds[1] - d.bounds[0], lyy = d.bounds[3] - d.bounds[2], lzz = d.bounds[5] - d.bounds[4];
    g.dx = lxx / d.sys_size[0];
    g.dy = lyy / d.sys_size[1];
    g.dz = lzz / d.sys_size[2];
    g.dxsp = 1.0 / g.dx;
    g.dysp = 1.0 / g.dy;
    g.dzsp = 1.0 / g.dz;
    g.ax = d.bounds[0];
    g.ay = d.bounds[2];
    g.az = d.bounds[4];
    g.mu = d.fmu;
    g.frho = d.frho;
    g.n_obj = d.n_obj;
    g.sim_type = d.sim_type;
    g.has_exact = d.has_exact;
    g.f32face = face32(d);
    g.gravity = d.gravity;
    for (int f = 0; f < 6; f++) {
        g.walls[f] = d.walls[f];
        g.wall_pos[f] = d.wall_pos[f];
    }
    g.wall_dist = d.wall_dist;
    g.winv = 1 / d.wall_dist;
    const double dh = std::min(g.dx, std::min(g.dy, g.dz));

    // sim_manager::create_objs (sim_manager.cc:68-81)
    for (int o = 0; o < d.n_obj; o++) {
        host_obj &ob = s->obj[o];
        const rmt3d_object_desc &od = d.obj[o];
        ob.type = od.type;
        for (int c = 0; c < 3; c++) ob.c[c] = od.basic[c];
        ob.R = od.basic[3];
        ob.rho = od.rho;
        ob.G = od.G;
        ob.cs = sqrt(ob.G / ob.rho);
        ob.ex_visc_mult = d.ex_visc_mult;
        ob.ev_trans_mult = d.ev_trans_mult;
        ob.dt_pad = d.sdt_pad;
        ob.dt_ex_pad = d.dt_ex_pad;
        ob.ex_mu = ob.ex_visc_mult * d.fmu;  // the override at sim_manager.cc:72
        ob.volume = M_PI * 4 / 3 * pow(ob.R, 3);
        for (int c = 0; c < 3; c++) {
            ob.eig[c] = 1;
            ob.omega[c] = 0;
        }
        if (ob.type == RMT3D_OBJ_SPHERE) {
            int sd = int(od.extra[0]);
            double sl = od.extra[1];
            for (int c = 0; c < 3; c++) {
                ob.eig[c] = sl;
                ob.omega[c] = od.extra[2 + c];
            }
            ob.eig[sd] = 1. / (sl * sl);
        }
        obj_dev &gd = g.obj[o];
        gd.type = ob.type;
        for (int c = 0; c < 3; c++) {
            gd.c[c] = ob.c[c];
            gd.eig[c] = ob.eig[c];
            gd.omega[c] = ob.omega[c];
        }
        gd.R = ob.R;
        gd.G = ob.G;
        gd.rho = ob.rho;
        gd.ex_mu = ob.ex_mu;
        gd.ev_trans_mult = ob.ev_trans_mult;
    }
    // sim_manager::setup_const (sim_manager.cc:37-53)
    {
        double xxsp3 = 3.0 / (dh * dh);
        double dt_s = 100000;
        for (int o = 0; o < d.n_obj; o++) {
            double odt = s->obj[o].cfl(dh);
            if (odt < dt_s) dt_s = odt;
        }
        double dt_f = 0.5 * d.frho / (d.fmu * xxsp3) * d.fdt_pad;
        s->dt_reg = (dt_s < dt_f) ? dt_s : dt_f;
        s->eps = d.wt_n * dh;
        g.eps = s->eps;
        g.tf1 = 0.5 / s->eps;
        g.tf2 = 0.5 / M_PI;
        g.tf3 = M_PI / s->eps;
        if (d.dt < s->dt_reg) s->dt_reg = d.dt;
        s->K_stiff = 0.0025 / (s->dt_reg * s->dt_reg);
        g.K_stiff = s->K_stiff;
    }
    // vmax: sim_manager ctor value 1; sim_objects::set_wall_acc (sim_manager.hh:411-444)
    s->vmax = 1;
    if (d.sim_type == RMT3D_SIM_OBJECTS) {
        double winv = g.winv;
        s->min_wall_acc = 20 * winv;
        double mvsq = -1, mvol = -1;
        for (int o = 0; o < d.n_obj; o++) {
            double rho_s = s->obj[o].rho;
            double vsq = 0.5 * fabs((rho_s - d.frho) * d.gravity) / d.frho;
            double mvol_fact = s->obj[o].volume / s->obj[o].R / s->obj[o].R;
            vsq *= mvol_fact;
            if (vsq > mvsq) mvsq = vsq;
            if (mvol_fact > mvol) mvol = mvol_fact;
            double support_acc = fabs((rho_s - d.frho) * d.gravity * winv * mvol_fact / rho_s);
            if (support_acc > s->min_wall_acc) s->min_wall_acc = support_acc;
        }
        s->wall_acc_mult = 0.5 * mvol * pow(winv, 2);
        mvsq = sqrt(mvsq);
        s->vmax = mvsq;  // NaN without objects, exactly as in the reference
    }
    g.min_wall_acc = s->min_wall_acc;
    g.wall_acc_mult = s->wall_acc_mult;
    // fluid_3d::setup_faces (fluid_3d.cc:2952-2974)
    for (int f = 0; f < 6; f++) {
        for (int c = 0; c < 3; c++) {
            s->faces[f].bct[c] = d.bct[c][f];
            s->faces[f].bcv[c] = d.bcv[c][f];
            if (d.bct[c][f] == 1 && d.bcv[c][f] > s->vmax) s->vmax = d.bcv[c][f];
        }
        s->faces[f].h = (f / 2 == 0) ? g.dx : ((f / 2 == 1) ? g.dy : g.dz);
        s->wall[f] = !g.prd[f / 2];
        if (s->wall[f])
            for (int c = 0; c < 3; c++)
                if (d.bct[c][f] != 1 && d.bct[c][f] != 2) {
                    rmt3d_scene_destroy(s);
                    return fail(RMT3D_ERR_INVALID, "bad boundary condition type");
                }
    }
    s->dt = d.dt;

    // coordinates (fluid_3d.cc:137-139)
    s->hlx.resize(g.sm4);
    s->hly.resize(g.sn4);
    s->hlz.resize(g.so4);
    for (int i = 0; i < g.sm4; i++) s->hlx[i] = g.ax + (0 + i - 2 + 0.5) * g.dx;
    for (int j = 0; j < g.sn4; j++) s->hly[j] = g.ay + (0 + j - 2 + 0.5) * g.dy;
    for (int k = 0; k < g.so4; k++) s->hlz[k] = g.az + (0 + k - 2 + 0.5) * g.dz;

    // device state
    const size_t n = g.ncell;
    int e = 0;
    fields_dev &F = s->hF;
    memset(&F, 0, sizeof(F));
    for (int c = 0; c < 3; c++) s->plan(&F.vel[c], n), s->plan(&F.dvel[c], n);
    s->plan(&F.p, n), s->plan(&F.dp, n), s->plan(&F.q, n);
    for (int c = 0; c < 18; c++) g.f32face ? s->plan(&F.fvel32[c], n) : s->plan(&F.fvel[c], n);
    for (int c = 0; c < 9; c++) s->plan(&F.sigma[c], n);
    if (d.var_den) s->plan(&F.rho, n);
    for (int o = 0; o < d.n_obj; o++) {
        objmap_dev &m = F.om[o];
        s->plan(&m.code, n), s->plan(&m.code_prev, n);
        for (int c = 0; c < 3; c++)
            s->plan(&m.x[c], n), s->plan(&m.xp[c], n), s->plan(&m.x_prev[c], n), s->plan(&m.det[c], n), s->plan(&m.el[c], n);
        for (int c = 0; c < 18; c++) s->plan(&m.fx[c], n);
        for (int c = 0; c < 9; c++) s->plan(&m.gp[c], n), s->plan(&m.gp_prev[c], n);
    }
    if (d.n_obj > 0) {
        const size_t no = (size_t)d.n_obj * n;
        s->plan(&s->lay, no), s->plan(&s->inl, no), s->plan(&s->front[0], no), s->plan(&s->front[1], no);
        s->plan(&s->fcnt, 2 * kMaxObj), s->plan(&s->mlist, n), s->plan(&s->mcnt, 1);
    }
    e |= s->commit_slab();
    for (int o = 0; o < d.n_obj && !e; o++) {
        cudaMemsetAsync(F.om[o].code, 0xff, n * sizeof(int), s->st);
        cudaMemsetAsync(F.om[o].code_prev, 0xff, n * sizeof(int), s->st);
    }
    e |= s->alloc(&s->lx, g.sm4) | s->alloc(&s->ly, g.sn4) | s->alloc(&s->lz, g.so4);
    e |= s->alloc(&s->dF, 1);
    if ((d.run.dump_code & 1) && d.run.ntracers > 0) {
        s->ntr = d.run.ntracers;
        e |= s->alloc(&s->tr_pc, 3 * (size_t)s->ntr) | s->alloc(&s->tr_rp, 6 * (size_t)s->ntr) |
             s->alloc(&s->tr_alive, (size_t)s->ntr);
    }
    e |= s->alloc(&s->ctl, 1) | s->alloc(&s->d_mean, 1 + kMeanBlocks) | s->alloc(&s->d_red, 4) |
         s->alloc(&s->mean_ticket, 1) | s->alloc(&s->d_diag, kDiagVals * (1 + kMeanBlocks)) |
         s->alloc(&s->diag_ticket, 1);
    s->h_ctl = (scene_ctl *)pinned_get(sizeof(scene_ctl));
    s->h_scalar = (double *)pinned_get(sizeof(double));
    if (e || !s->h_ctl || !s->h_scalar) {
        rmt3d_scene_destroy(s);
        return fail(RMT3D_ERR_OOM, "allocation failed");
    }
    {
        // control block: time 0, no halt, predictor state iV = 32,
        // V_avg = 32, V_var = 1e6 (mg_pred, mg_probs.hh:44-50)
        scene_ctl c;
        memset(&c, 0, sizeof(c));
        for (mg_ctl *m : {&c.mac, &c.fem}) {
            m->iV = 2 * kMgIP;
            m->V_avg = 2 * kMgIP;
            m->V_var = 1e6;
        }
        *s->h_ctl = c;
        cudaMemcpyAsync(s->ctl, s->h_ctl, sizeof(scene_ctl), cudaMemcpyHostToDevice, s->st);
    }
    s->counters = s->ctl->counters;
    s->h_counters = s->h_ctl->counters;
    s->mac.ctl = &s->ctl->mac;
    s->mac.h_ctl = &s->h_ctl->mac;
    s->fem.ctl = &s->ctl->fem;
    s->fem.h_ctl = &s->h_ctl->fem;
    {
        // The TMA-staged edge kernel where it was measured faster (x extent
        // of 128 cells and more: 4.5% per FP64 step at 128^3; equal at 96^3,
        // 7% slower at 64^3, where its 32 x 8 tiles leave too few blocks);
        // RMT3D_EDGE_TMA=0 or 1 forces either form (the same bits)
        const char *et = getenv("RMT3D_EDGE_TMA");
        const bool want = et ? et[0] == '1' : s->g.sm >= 128;
        if (want) {
            bool ok = true;
            for (int c = 0; c < 3 && ok; c++) ok = edge_vel_tensor_map(s->g, s->hF.vel[c], &s->tm_vel[c]);
            s->edge_tma = ok;
        }
    }
    {
        const char *ge = getenv("RMT3D_GRAPH");
        s->use_graph = !(ge && ge[0] == '0');
        s->mac.use_graph = s->fem.use_graph = s->use_graph;
    }
    cudaMemcpyAsync(s->lx, s->hlx.data(), g.sm4 * 8, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(s->ly, s->hly.data(), g.sn4 * 8, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(s->lz, s->hlz.data(), g.so4 * 8, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(s->dF, &F, sizeof(F), cudaMemcpyHostToDevice, s->st);
    s->mac.launches = &s->launches;
    s->fem.launches = &s->launches;
    s->mac.prof = &s->prof;
    s->fem.prof = &s->prof;
    int nm[3] = {g.sm, g.sn, g.so}, nf[3] = {g.fm, g.fn, g.fo};
    bool mixed = mixed_form(d.precision);
    s->mac.exact = s->fem.exact = d.mg_exact != 0;
    s->mac.rtol = s->fem.rtol = (mixed && d.mixed_rtol > 0) ? d.mixed_rtol : 0;
    s->mac.vd = s->fem.vd = d.var_den != 0;
    if ((e = s->mac.setup(MG_MAC, nm, g.prd, mixed, s->st)) != 0 || (e = s->fem.setup(MG_FEM, nf, g.prd, mixed, s->st)) != 0) {
        rmt3d_scene_destroy(s);
        return e;
    }
    if (d.var_den) {
        // one 1/rho array per level, shared: FEM level l has the MAC level's cells
        const size_t nl = s->mac.lv.size();
        for (size_t l = 0; l < s->fem.lv.size(); l++)
            for (int a = 0; a < 3; a++) {
                const mg_level &F = s->fem.lv[l];
                const int cells = F.prd[a] ? F.n[a] : F.n[a] - 1;
                if (l >= nl || cells != s->mac.lv[l].n[a]) {
                    rmt3d_scene_destroy(s);
                    return fail(RMT3D_ERR_UNSUPPORTED, "variable density needs matching MAC and FEM hierarchies");
                }
            }
        s->rinv.assign(nl, nullptr);
        s->rinvs.assign(nl, nullptr);
        for (size_t l = 0; l < nl && !e; l++) {
            e |= s->alloc(&s->rinv[l], s->mac.lv[l].npts());
            if (mixed) e |= s->alloc(&s->rinvs[l], s->mac.lv[l].npts());
        }
        if (e) {
            rmt3d_scene_destroy(s);
            return fail(RMT3D_ERR_OOM, "allocation failed");
        }
        for (size_t l = 0; l < nl; l++) {
            s->mac.lv[l].ri = s->rinv[l];
            s->mac.lv[l].ris = s->rinvs[l];
            if (l < s->fem.lv.size()) {
                s->fem.lv[l].ri = s->rinv[l];
                s->fem.lv[l].ris = s->rinvs[l];
            }
        }
    }
    if (cudaStreamSynchronize(s->st) != cudaSuccess) {
        rmt3d_scene_destroy(s);
        return fail(RMT3D_ERR_CUDA, "scene set-up failed");
    }
    s->dt_reg0 = s->dt_reg;
    s->K_stiff0 = s->K_stiff;
    s->vmax0 = s->vmax;
    *out = s;
    return RMT3D_OK;
}

// ---------------------------------------------------------------------------
// checkpoints (F3D_Source/fluid_3d_chk_pt.cc)
// ---------------------------------------------------------------------------
// doubles per slice of a checkpoint field file: (m+1)(n+1), the reference's
// u_global (fluid_3d_chk_pt.cc:16, :91)
static size_t chk_slice_len(const rmt3d_scene *s) { return (size_t)(s->g.sm + 1) * (s->g.sn + 1); }

// fluid_3d::initialize_from_chk_point (fluid_3d_chk_pt.cc:74-163).  All eight
// files are read before the device state is touched, so a missing or empty
// file (*status 1 or 2) leaves the scene as it was.
static int read_chk_pt(rmt3d_scene *s, const char *dir, int *status) {
    const grid_dev &g = s->g;
    const size_t n = g.ncell;
    const size_t L = chk_slice_len(s), total = L * g.so * kChkFields;
    std::vector<double> h(total);
    int e = chk_read_files(dir, h.data(), L, g.so, status);
    if (e || *status) return e;
    double *dbuf = nullptr;
    CK(cudaMallocAsync((void **)&dbuf, total * sizeof(double) + sizeof(double), s->st));
    int *bad = (int *)(dbuf + total);
    cudaError_t ce = cudaMemcpyAsync(dbuf, h.data(), total * sizeof(double), cudaMemcpyHostToDevice, s->st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(bad, 0, sizeof(int), s->st);
    // the values of a freshly constructed fluid_3d that the files do not set
    const fields_dev &F = s->hF;
    if (ce == cudaSuccess) ce = cudaMemsetAsync(F.dp, 0, n * 8, s->st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(F.q, 0, n * 8, s->st);
    for (int c = 0; c < 3 && ce == cudaSuccess; c++) ce = cudaMemsetAsync(F.dvel[c], 0, n * 8, s->st);
    if (ce == cudaSuccess) ce = zero_faces(s);
    for (int c = 0; c < 9 && ce == cudaSuccess; c++) ce = cudaMemsetAsync(F.sigma[c], 0, n * 8, s->st);
    int hbad = 0;
    if (ce == cudaSuccess) {
        k_chk_unpack<<<lin_blocks(g.ncell), 256, 0, s->st>>>(g, s->dF, dbuf, bad);
        s->count();
        ce = cudaMemcpyAsync(s->h_scalar, bad, sizeof(int), cudaMemcpyDeviceToHost, s->st);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->st);
    if (ce == cudaSuccess) memcpy(&hbad, s->h_scalar, sizeof(int));
    cudaFreeAsync(dbuf, s->st);
    CK(ce);
    if (hbad) return fail(RMT3D_ERR_INVALID, std::string("checkpoint ") + dir + ": OID names no object");
    // communicate<1>, <2>, <8>, <16|32>; init_extrapolate; update_rho
    periodic(s, {F.vel[0], F.vel[1], F.vel[2]}, {}, 0);
    comm_pressure(s);
    comm_primary(s);
    init_extrapolate(s);
    update_rho(s);
    set_time(s, s->d.run.current_time);
    s->nt = s->d.run.chk_step;
    s->dt_reg = s->dt_reg0;
    s->K_stiff = s->K_stiff0;
    s->g.K_stiff = s->K_stiff0;
    s->vmax = s->vmax0;
    return 0;
}

// the end of fluid_3d::initialize shared by both starts (fluid_3d.cc:212-232)
static int init_finish(rmt3d_scene *s) {
    fill_boundary_cc(s);
    compute_grad_basis(s);
    int re = read_ctl(s);
    if (re) return re;
    if (s->h_counters[2] > 0) return fail(RMT3D_ERR_EXTRAP, "Extrapolation failed: no eligible points or degenerate matrix");
    CK(cudaGetLastError());
    return RMT3D_OK;
}

extern "C" int rmt3d_initialize(rmt3d_scene *s) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    mark_dirty(s);
    int e;
    rmt3d_run_desc &r = s->d.run;
    s->init_err = 1;
    if (r.chk_num > 0) {
        char dir[600];
        snprintf(dir, sizeof(dir), "%s/chk.%05d", r.recover_dirname, r.chk_num);
        if ((e = read_chk_pt(s, dir, &s->init_err))) return e;
    }
    if (s->init_err > 0) {
        r.chk_num = 0;
        set_time(s, 0);
        if ((e = init_fluid(s))) return e;
        if ((e = init_pres(s))) return e;
        if ((e = init_refmap(s))) return e;
        init_extrapolate(s);
        update_rho(s);
    }
    // alloc_tracers (fluid_3d.cc:217-219): from the checkpoint's tracer file
    // on a restart, scattered afresh otherwise
    if (s->ntr) {
        char dir[600];
        snprintf(dir, sizeof(dir), "%s/chk.%05d", r.recover_dirname, r.chk_num);
        if ((e = alloc_tracers(s, r.chk_num > 0 ? dir : nullptr))) return e;
    }
    return init_finish(s);
}

extern "C" int rmt3d_read_chk_pt(rmt3d_scene *s, const char *chk_dirname, int *status) {
    if (!s || !chk_dirname || !status) return fail(RMT3D_ERR_INVALID, "null argument");
    int e = read_chk_pt(s, chk_dirname, status);
    if (e || *status) return e;
    mark_dirty(s);
    s->init_err = 0;
    return init_finish(s);
}

extern "C" int rmt3d_write_chk_pt(rmt3d_scene *s, int snum, int fnum, const char *chk_dirname, int compress) {
    if (!s || !chk_dirname) return fail(RMT3D_ERR_INVALID, "null argument");
    CK(cudaStreamSynchronize(s->st));
    const grid_dev &g = s->g;
    const size_t L = chk_slice_len(s), per = L * g.so, total = per * kChkFields;
    std::vector<double> h(total);
    double *dbuf = nullptr;
    CK(cudaMallocAsync((void **)&dbuf, total * sizeof(double), s->st));
    const int blocks = (int)std::min<size_t>((per + 255) / 256, 148 * 16);
    k_chk_pack<<<blocks, 256, 0, s->st>>>(g, s->dF, dbuf);
    s->count();
    cudaError_t ce = cudaMemcpyAsync(h.data(), dbuf, total * sizeof(double), cudaMemcpyDeviceToHost, s->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->st);
    cudaFreeAsync(dbuf, s->st);
    CK(ce);
    int e = chk_make_dir(chk_dirname);
    if (!e) e = chk_write_files(chk_dirname, h.data(), L, g.so, compress);
    if (e) return e;
    // the tracer file of this frame (the reference copies the stepper's
    // tr.<fnum>, fluid_3d_chk_pt.cc:22-33)
    if (s->ntr) {
        char fn[700];
        snprintf(fn, sizeof(fn), "%s/tr.%05d", chk_dirname, fnum);
        if ((e = rmt3d_write_tracers(s, fn, 1))) return e;
    }
    // set_current_chk_num / _chk_step / _time, then write_params
    s->d.run.chk_num = fnum;
    s->d.run.chk_step = snum;
    s->d.run.current_time = s->time;
    return chk_write_recover_cfg(chk_dirname, s->d, s->dt);
}

extern "C" int rmt3d_set_dt(rmt3d_scene *s, double dt) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (dt != s->dt) mark_dirty(s);
    s->dt = dt;
    return RMT3D_OK;
}

extern "C" int rmt3d_init_iter(rmt3d_scene *s) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    const double tol = 1e-4;
    for (int i = 0; s->init_err > 0 && i < s->d.num_iters; i++) {
        set_time(s, 0);
        fill_boundary_cc(s);
        int e = step_forward(s, 0);
        if (e < 0) return e;
        double divu;
        if ((e = div_u(s, &divu))) return e;
        if ((e = init_fluid(s))) return e;
        if ((e = init_refmap(s))) return e;
        if (s->g.n_obj > 0) {
            k_reset_extraps<<<lin_blocks(s->g.ncell), 256, 0, s->st>>>(s->g, s->dF);
            s->count();
        }
        init_extrapolate(s);
        update_rho(s);
        if (divu < tol) break;
    }
    if (s->init_err > 0) {
        s->nt = 0;
        set_time(s, 0.0);
    }
    compute_stress(s);
    CK(cudaStreamSynchronize(s->st));
    CK(cudaGetLastError());
    return RMT3D_OK;
}

extern "C" int rmt3d_prepare(rmt3d_scene *s) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    int e = rmt3d_initialize(s);
    if (e) return e;
    double dt;
    if ((e = rmt3d_stepper_dt(&s->d, s->dt_reg, &dt, nullptr))) return e;
    rmt3d_set_dt(s, dt);
    if ((e = rmt3d_init_iter(s))) return e;
    rmt3d_set_dt(s, dt);  // stepper::run re-links dt (stepper.hh:336)
    // build the step graph now, so that the first step's latency is a step's
    if (graph_mode(s) && (s->graph_dirty || !s->step_exec) && (e = build_step_graph(s))) return e;
    return RMT3D_OK;
}

// Steps run as graph launches unless a kernel profiler is active or graphs
// are switched off (RMT3D_GRAPH=0); both forms issue the same kernels.
static bool graph_mode(rmt3d_scene *s) { return s->use_graph && s->prof.target < 0; }

extern "C" int rmt3d_step(rmt3d_scene *s, int debug, int *status) {
    if (!s || !status) return fail(RMT3D_ERR_INVALID, "null argument");
    if (graph_mode(s)) {
        int e = run_graph(s, 1, status);
        if (e < 0) *status = e;
        return e < 0 ? e : RMT3D_OK;
    }
    int e = step_forward(s, debug);
    *status = e;
    return e < 0 ? e : RMT3D_OK;
}

extern "C" int rmt3d_step_phases(rmt3d_scene *s, int last_phase, int *status) {
    if (!s || !status) return fail(RMT3D_ERR_INVALID, "null argument");
    if (last_phase < 1 || last_phase > 9) return fail(RMT3D_ERR_INVALID, "phase outside 1..9");
    int e = step_forward(s, 0, last_phase);
    *status = e;
    if (e < 0) return e;
    CK(cudaStreamSynchronize(s->st));
    return RMT3D_OK;
}

extern "C" int rmt3d_run(rmt3d_scene *s, int nsteps, int *status) {
    if (!s || !status) return fail(RMT3D_ERR_INVALID, "null argument");
    *status = 0;
    if (nsteps <= 0) return RMT3D_OK;
    if (graph_mode(s)) {
        int e = run_graph(s, nsteps, status);
        if (e < 0) *status = e;
        return e < 0 ? e : RMT3D_OK;
    }
    for (int i = 0; i < nsteps; i++) {
        int e = rmt3d_step(s, 0, status);
        if (e) return e;
        if (*status) return RMT3D_OK;
    }
    return RMT3D_OK;
}

namespace rmt3d {
int steps_launch(rmt3d_scene *s, int nsteps) {
    pending_steps *p = pending_of(s);
    *p = pending_steps{};
    if (graph_mode(s)) return graph_launch(s, nsteps, *p);
    p->eager_err = rmt3d_run(s, nsteps, &p->eager_status);
    return 0;
}

int steps_finish(rmt3d_scene *s, int *status) {
    pending_steps q = *pending_of(s);
    for (size_t i = 0; i < t_pending.size(); i++)
        if (t_pending[i].first == s) {
            t_pending.erase(t_pending.begin() + i);
            break;
        }
    if (!graph_mode(s)) {
        *status = q.eager_status;
        return q.eager_err;
    }
    int e = graph_finish(s, q, status);
    if (e < 0) *status = e;
    return e < 0 ? e : RMT3D_OK;
}
}  // namespace rmt3d

extern "C" int rmt3d_get_scalar(rmt3d_scene *s, int which, double *v) {
    if (!s || !v) return fail(RMT3D_ERR_INVALID, "null argument");
    switch (which) {
        case 0: *v = s->dt; break;
        case 1: *v = s->time; break;
        case 2: *v = s->dt_reg; break;
        case 3: *v = s->eps; break;
        case 4: *v = s->nt; break;
        case 5: *v = s->mac.last_cycles; break;
        case 6: *v = s->fem.last_cycles; break;
        case 7: *v = (double)s->mac.cycles_total; break;
        case 8: *v = (double)s->fem.cycles_total; break;
        case 9: {
            long long cnt = 0;
            std::vector<int> code(s->g.ncell);
            for (int o = 0; o < s->g.n_obj; o++) {
                CK(copy_sync(s, code.data(), s->hF.om[o].code, s->g.ncell * sizeof(int), cudaMemcpyDeviceToHost));
                for (int c : code) cnt += (c > 0);
            }
            *v = (double)cnt;
            break;
        }
        case 10: *v = s->K_stiff; break;
        case 11: *v = s->vmax; break;
        case 12: *v = (double)(s->dev_bytes + s->mac.bytes_alloc + s->fem.bytes_alloc); break;
        case 13: *v = s->init_err; break;
        default: return fail(RMT3D_ERR_INVALID, "unknown scalar");
    }
    return RMT3D_OK;
}

extern "C" int rmt3d_get_dims(rmt3d_scene *s, int dims[6]) {
    if (!s || !dims) return fail(RMT3D_ERR_INVALID, "null argument");
    dims[0] = s->g.sm4;
    dims[1] = s->g.sn4;
    dims[2] = s->g.so4;
    dims[3] = s->g.fm;
    dims[4] = s->g.fn;
    dims[5] = s->g.fo;
    return RMT3D_OK;
}

static double *field_ptr(rmt3d_scene *s, int which) {
    fields_dev &F = s->hF;
    if (which >= 0 && which < 3) return F.vel[which];
    if (which == 3) return F.p;
    if (which == 4) return F.dp;
    if (which == 5) return F.q;
    if (which >= 6 && which < 9) return F.dvel[which - 6];
    if (which >= 9 && which < 27) return F.fvel[which - 9];  // null when the faces are FP32
    if (which >= 27 && which < 36) return F.sigma[which - 27];
    return nullptr;
}

extern "C" int rmt3d_get_field(rmt3d_scene *s, int which, double *dst) {
    if (!s || !dst) return fail(RMT3D_ERR_INVALID, "null argument");
    if (which >= 9 && which < 27 && s->g.f32face) {
        CK(cudaStreamSynchronize(s->st));
        return faces_to_host(s, which - 9, dst);
    }
    double *p = field_ptr(s, which);
    if (!p) return fail(RMT3D_ERR_INVALID, "unknown field");
    CK(cudaStreamSynchronize(s->st));
    CK(copy_sync(s, dst, p, s->g.ncell * sizeof(double), cudaMemcpyDeviceToHost));
    return RMT3D_OK;
}

extern "C" int rmt3d_snapshot_fields(rmt3d_scene *s, const int *which, int n, double *const *host_dst) {
    if (!s || !which || !host_dst || n < 1 || n > 36) return fail(RMT3D_ERR_INVALID, "bad snapshot arguments");
    const size_t nc = s->g.ncell;
    for (int i = 0; i < n; i++)
        if (!field_ptr(s, which[i]) || !host_dst[i])
            return fail(RMT3D_ERR_INVALID, "unknown field, FP32 face state (read it with rmt3d_get_field), or null buffer");
    if (!s->cst) {
        CK(cudaStreamCreateWithFlags(&s->cst, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&s->ev_snap, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s->ev_d2h, cudaEventDisableTiming));
    }
    // the staging copies of the previous snapshot must have reached the host
    if (s->d2h_pending) CK(cudaStreamWaitEvent(s->st, s->ev_d2h, 0));
    if (s->snap_cap < n * nc) {
        if (s->snap) CK(cudaFreeAsync(s->snap, s->st));
        s->snap = nullptr;
        CK(cudaMallocAsync((void **)&s->snap, n * nc * sizeof(double), s->st));
        s->snap_cap = n * nc;
    }
    for (int i = 0; i < n; i++)
        CK(cudaMemcpyAsync(s->snap + i * nc, field_ptr(s, which[i]), nc * sizeof(double), cudaMemcpyDeviceToDevice,
                           s->st));
    CK(cudaEventRecord(s->ev_snap, s->st));
    CK(cudaStreamWaitEvent(s->cst, s->ev_snap, 0));
    for (int i = 0; i < n; i++)
        CK(cudaMemcpyAsync(host_dst[i], s->snap + i * nc, nc * sizeof(double), cudaMemcpyDeviceToHost, s->cst));
    CK(cudaEventRecord(s->ev_d2h, s->cst));
    s->d2h_pending = true;
    return RMT3D_OK;
}

extern "C" int rmt3d_snapshot_wait(rmt3d_scene *s) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (s->cst) CK(cudaStreamSynchronize(s->cst));
    return RMT3D_OK;
}

extern "C" int rmt3d_get_refmap(rmt3d_scene *s, int obj, int *code, double *x, double *xpred) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (obj < 0 || obj >= s->g.n_obj) return fail(RMT3D_ERR_INVALID, "object index out of range");
    const size_t n = s->g.ncell;
    objmap_dev &m = s->hF.om[obj];
    CK(cudaStreamSynchronize(s->st));
    if (code) CK(copy_sync(s, code, m.code, n * sizeof(int), cudaMemcpyDeviceToHost));
    for (int c = 0; c < 3; c++) {
        if (x) CK(copy_sync(s, x + c * n, m.x[c], n * 8, cudaMemcpyDeviceToHost));
        if (xpred) CK(copy_sync(s, xpred + c * n, m.xp[c], n * 8, cudaMemcpyDeviceToHost));
    }
    return RMT3D_OK;
}

// AoS offsets of struct field (360 B) and struct ref_map (488 B), fields.hh
namespace {
// field: vel[3], p, dp, q, dvel[3], nv_der[3][3], fvel[6][3], sigma[3][3]
constexpr int F_VEL = 0, F_P = 3, F_DP = 4, F_Q = 5, F_DVEL = 6, F_FVEL = 18, F_SIGMA = 36, F_N = 45;
// ref_map (in doubles after the 8-byte id word): x[3], xpred[3], nv_der[3][3],
// fx[6][3], sigma[3][3], elastic_energy[3], detF[3], grad_phi[3][3], act_power[3]
constexpr int R_X = 1, R_XP = 4, R_FX = 16, R_EL = 43, R_DET = 46, R_GP = 49;
}  // namespace

extern "C" int rmt3d_import_reference(rmt3d_scene *s, const void *field_aos, const void *refmap_aos,
                                      const int *ext_index, const void *ext_refmaps, int n_ext, double dt,
                                      double time) {
    if (!s || !field_aos) return fail(RMT3D_ERR_INVALID, "null argument");
    const size_t n = s->g.ncell;
    const double *fa = (const double *)field_aos;
    std::vector<double> buf(n);
    auto put = [&](double *dst, const double *src, int stride, int off) -> int {
        for (size_t i = 0; i < n; i++) buf[i] = src[i * stride + off];
        CK(copy_sync(s, dst, buf.data(), n * 8, cudaMemcpyHostToDevice));
        return 0;
    };
    int e = 0;
    for (int c = 0; c < 3; c++) e |= put(s->hF.vel[c], fa, F_N, F_VEL + c) | put(s->hF.dvel[c], fa, F_N, F_DVEL + c);
    e |= put(s->hF.p, fa, F_N, F_P) | put(s->hF.dp, fa, F_N, F_DP) | put(s->hF.q, fa, F_N, F_Q);
    for (int c = 0; c < 18; c++) {
        if (!s->g.f32face) {
            e |= put(s->hF.fvel[c], fa, F_N, F_FVEL + c);
            continue;
        }
        for (size_t i = 0; i < n; i++) buf[i] = fa[i * F_N + F_FVEL + c];
        e |= faces_from_host(s, c, buf.data());
    }
    for (int c = 0; c < 9; c++) e |= put(s->hF.sigma[c], fa, F_N, F_SIGMA + c);
    if (e) return e;
    const int no = s->g.n_obj;
    if (no > 0 && refmap_aos) {
        std::vector<int> code(n);
        std::vector<double> X(n * 3), XP(n * 3), FX(n * 18), GP(n * 9), DT(n * 3), EL(n * 3);
        auto rd = [&](const unsigned char *rec, int off) { return ((const double *)rec)[off]; };
        for (int o = 0; o < no; o++) {
            std::fill(code.begin(), code.end(), -1);
            std::fill(GP.begin(), GP.end(), -kBig);
            const unsigned char *ra = (const unsigned char *)refmap_aos;
            auto take = [&](size_t cell, const unsigned char *rec, int cd) {
                code[cell] = cd;
                for (int c = 0; c < 3; c++) {
                    X[c * n + cell] = rd(rec, R_X + c);
                    XP[c * n + cell] = rd(rec, R_XP + c);
                    DT[c * n + cell] = rd(rec, R_DET + c);
                    EL[c * n + cell] = rd(rec, R_EL + c);
                }
                for (int c = 0; c < 18; c++) FX[c * n + cell] = rd(rec, R_FX + c);
                for (int c = 0; c < 9; c++) GP[c * n + cell] = rd(rec, R_GP + c);
            };
            for (size_t i = 0; i < n; i++) {
                const unsigned char *rec = ra + i * 488;
                unsigned int cc = *(const unsigned int *)rec;
                if ((int)(cc & 1023) == o + 1) take(i, rec, (cc >> 10) & 63);
            }
            const unsigned char *ea = (const unsigned char *)ext_refmaps;
            for (int q = 0; q < n_ext; q++) {
                const unsigned char *rec = ea + (size_t)q * 488;
                unsigned int cc = *(const unsigned int *)rec;
                if ((int)(cc & 1023) == o + 1) take(ext_index[q], rec, (cc >> 10) & 63);
            }
            objmap_dev &m = s->hF.om[o];
            CK(copy_sync(s, m.code, code.data(), n * sizeof(int), cudaMemcpyHostToDevice));
            for (int c = 0; c < 3; c++) {
                CK(copy_sync(s, m.x[c], X.data() + c * n, n * 8, cudaMemcpyHostToDevice));
                CK(copy_sync(s, m.xp[c], XP.data() + c * n, n * 8, cudaMemcpyHostToDevice));
                CK(copy_sync(s, m.det[c], DT.data() + c * n, n * 8, cudaMemcpyHostToDevice));
                CK(copy_sync(s, m.el[c], EL.data() + c * n, n * 8, cudaMemcpyHostToDevice));
            }
            for (int c = 0; c < 18; c++) CK(copy_sync(s, m.fx[c], FX.data() + c * n, n * 8, cudaMemcpyHostToDevice));
            for (int c = 0; c < 9; c++) CK(copy_sync(s, m.gp[c], GP.data() + c * n, n * 8, cudaMemcpyHostToDevice));
        }
    }
    rmt3d_set_dt(s, dt);
    set_time(s, time);
    update_rho(s);  // the density the reference derives from the imported maps
    mark_dirty(s);
    CK(cudaStreamSynchronize(s->st));
    return RMT3D_OK;
}

extern "C" int rmt3d_export_reference(rmt3d_scene *s, void *field_aos, void *refmap_aos, int *ext_index,
                                      void *ext_refmaps, int max_ext, int *n_ext) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    const size_t n = s->g.ncell;
    CK(cudaStreamSynchronize(s->st));
    std::vector<double> buf(n);
    if (field_aos) {
        double *fa = (double *)field_aos;
        memset(fa, 0, n * 360);
        auto get = [&](const double *src, int off) -> int {
            CK(copy_sync(s, buf.data(), src, n * 8, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; i++) fa[i * F_N + off] = buf[i];
            return 0;
        };
        int e = 0;
        for (int c = 0; c < 3; c++) e |= get(s->hF.vel[c], F_VEL + c) | get(s->hF.dvel[c], F_DVEL + c);
        e |= get(s->hF.p, F_P) | get(s->hF.dp, F_DP) | get(s->hF.q, F_Q);
        for (int c = 0; c < 18; c++) {
            if (!s->g.f32face) {
                e |= get(s->hF.fvel[c], F_FVEL + c);
                continue;
            }
            e |= faces_to_host(s, c, buf.data());
            for (size_t i = 0; i < n; i++) fa[i * F_N + F_FVEL + c] = buf[i];
        }
        for (int c = 0; c < 9; c++) e |= get(s->hF.sigma[c], F_SIGMA + c);
        if (e) return e;
    }
    int ne = 0;
    if (refmap_aos) memset(refmap_aos, 0, n * 488);
    std::vector<int> code(n);
    std::vector<double> X(3 * n), XP(3 * n), FX(18 * n), GP(9 * n), DT(3 * n), EL(3 * n);
    for (int o = 0; o < s->g.n_obj; o++) {
        objmap_dev &m = s->hF.om[o];
        CK(copy_sync(s, code.data(), m.code, n * sizeof(int), cudaMemcpyDeviceToHost));
        for (int c = 0; c < 3; c++) {
            CK(copy_sync(s, X.data() + c * n, m.x[c], n * 8, cudaMemcpyDeviceToHost));
            CK(copy_sync(s, XP.data() + c * n, m.xp[c], n * 8, cudaMemcpyDeviceToHost));
            CK(copy_sync(s, DT.data() + c * n, m.det[c], n * 8, cudaMemcpyDeviceToHost));
            CK(copy_sync(s, EL.data() + c * n, m.el[c], n * 8, cudaMemcpyDeviceToHost));
        }
        for (int c = 0; c < 18; c++) CK(copy_sync(s, FX.data() + c * n, m.fx[c], n * 8, cudaMemcpyDeviceToHost));
        for (int c = 0; c < 9; c++) CK(copy_sync(s, GP.data() + c * n, m.gp[c], n * 8, cudaMemcpyDeviceToHost));
        auto fill = [&](unsigned char *rec, size_t cell, int cd) {
            *(unsigned int *)rec = (unsigned)(o + 1) | ((unsigned)cd << 10);
            double *r = (double *)rec;
            for (int c = 0; c < 3; c++) {
                r[R_X + c] = X[c * n + cell];
                r[R_XP + c] = XP[c * n + cell];
                r[R_DET + c] = DT[c * n + cell];
                r[R_EL + c] = EL[c * n + cell];
            }
            for (int c = 0; c < 18; c++) r[R_FX + c] = FX[c * n + cell];
            for (int c = 0; c < 9; c++) r[R_GP + c] = GP[c * n + cell];
        };
        for (size_t i = 0; i < n; i++) {
            if (code[i] == 0 && refmap_aos) fill((unsigned char *)refmap_aos + i * 488, i, 0);
            if (code[i] > 0) {
                if (ne < max_ext && ext_refmaps && ext_index) {
                    ext_index[ne] = (int)i;
                    fill((unsigned char *)ext_refmaps + (size_t)ne * 488, i, code[i]);
                }
                ne++;
            }
        }
    }
    if (n_ext) *n_ext = ne;
    return RMT3D_OK;
}

// Solid diagnostics over the interior cells, reduced in a fixed order (block
// partials, summed by the last block in block order):
//  [0] sum H(phi) and [1..3] sum x H(phi), y H(phi), z H(phi) over the primary
//      maps (compute_centroid, fluid_3d_utils.cc:1348-1379);
//  [4] sum of squared mean |det F - 1| over the six faces of each primary
//      map's cell, [5] its maximum (total_dev_in_detF, :1032-1084).
__global__ void k_solid_diag(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                             const double *lz, double *out, unsigned *ticket) {
    double v[kDiagVals] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int ncell = g.sm * g.sn * g.so;
    const int strides[3] = {1, g.sm4, g.smn4};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
        const int i = t % g.sm + 2, j = (t / g.sm) % g.sn + 2, k = t / (g.sm * g.sn) + 2;
        const int ind = gidx(g, i, j, k);
        for (int o = 0; o < g.n_obj; o++) {
            const objmap_dev &m = F->om[o];
            if (m.code[ind] != 0) continue;
            const double sf = heaviside(g, obj_phi(g, o, m.x[0][ind], m.x[1][ind], m.x[2][ind]));
            v[0] += sf;
            v[1] += lx[i] * sf;
            v[2] += ly[j] * sf;
            v[3] += lz[k] * sf;
            double dev = 0;
            for (int a = 0; a < 3; a++) {
                dev += fabs(m.det[a][ind] - 1);
                const int nb = ind + strides[a];
                if (m.code[nb] >= 0) dev += fabs(m.det[a][nb] - 1);
            }
            dev /= 6.;
            v[4] += dev * dev;
            v[5] = fmax(v[5], dev * dev);
        }
    }
    __shared__ double sh[kDiagVals][32];
    __shared__ bool last;
    for (int c = 0; c < kDiagVals; c++) {
        double a = v[c];
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = (c == 5) ? fmax(a, b) : a + b;
        }
        if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < kDiagVals; c++) {
            double a = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) a = (c == 5) ? fmax(a, sh[c][w]) : a + sh[c][w];
            out[kDiagVals * (1 + blockIdx.x) + c] = a;
        }
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x < kDiagVals) {
        __threadfence();
        const int c = threadIdx.x;
        const volatile double *part = out + kDiagVals;
        double a = 0;
        for (unsigned b = 0; b < gridDim.x; b++) a = (c == 5) ? fmax(a, part[kDiagVals * b + c]) : a + part[kDiagVals * b + c];
        out[c] = a;
        if (c == 0) *ticket = 0;
    }
}

static int solid_diag(rmt3d_scene *s, double out[kDiagVals]) {
    k_solid_diag<<<kMeanBlocks, 256, 0, s->st>>>(s->g, s->dF, s->lx, s->ly, s->lz, s->d_diag, s->diag_ticket);
    s->count();
    CK(cudaMemcpyAsync(out, s->d_diag, kDiagVals * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

extern "C" int rmt3d_diag(rmt3d_scene *s, int kind, double *value) {
    if (!s || !value) return fail(RMT3D_ERR_INVALID, "null argument");
    if (kind == 0) return div_u(s, value);
    if (kind < 1 || kind > 6) return fail(RMT3D_ERR_INVALID, "unknown diagnostic");
    double v[kDiagVals];
    int e = solid_diag(s, v);
    if (e) return e;
    const double dv = s->g.dx * s->g.dy * s->g.dz;
    switch (kind) {
        case 1: *value = v[0] * dv; break;                 // compute_centroid's vol
        case 2: case 3: case 4: *value = v[kind - 1] / v[0]; break;  // centroid x, y, z
        case 5: *value = sqrt(v[4] * dv); break;           // total_dev_in_detF
        case 6: *value = sqrt(v[5]); break;                // its max_dev
    }
    return RMT3D_OK;
}

// ---------------------------------------------------------------------------
// frame diagnostics and slices (Sim/stepper.hh:378-474, fluid_3d_io.cc:3-434)
// ---------------------------------------------------------------------------
extern "C" int rmt3d_macro(rmt3d_scene *s, rmt3d_macro_data *out) {
    if (!s || !out) return fail(RMT3D_ERR_INVALID, "null argument");
    memset(out, 0, sizeof(*out));
    const grid_dev &g = s->g;
    out->time = s->time;
    out->n_obj = g.n_obj;
    int e = div_u(s, &out->div_u_l2);
    if (e) return e;
    double v[8];
    k_macro_cells<<<kMeanBlocks, 256, 0, s->st>>>(g, s->dF, s->lz, s->d.var_den, s->d_diag, s->diag_ticket);
    s->count();
    CK(copy_sync(s, v, s->d_diag, 8 * sizeof(double), cudaMemcpyDeviceToHost));
    // total_momentum: sum * dx * dy * dz; total_energy: each sum * (dx dy dz)
    for (int c = 0; c < 3; c++) out->momentum[c] = v[c] * g.dx * g.dy * g.dz;
    const double dv = g.dx * g.dy * g.dz;
    out->elastic = v[5] * dv;
    out->kinetic = v[3] * dv;
    out->potential = v[4] * dv;
    out->power = 0;
    out->energy = out->elastic + out->kinetic + out->potential;
    out->div_u_max = v[6];
    out->div_u_min = -v[7];
    for (int o = 0; o < g.n_obj; o++) {
        double w[7];
        k_macro_obj<<<kMeanBlocks, 256, 0, s->st>>>(g, s->dF, s->lx, s->ly, s->lz, o, s->d_diag, s->diag_ticket);
        s->count();
        CK(copy_sync(s, w, s->d_diag, 7 * sizeof(double), cudaMemcpyDeviceToHost));
        // sim_manager::compute_avgs: means, 0 for an object without weight
        for (int c = 0; c < 3; c++) {
            out->velocity[o][c] = w[0] != 0. ? w[4 + c] / w[0] : 0.;
            out->centroid[o][c] = w[0] != 0. ? w[1 + c] / w[0] : 0.;
        }
    }
    if (g.n_obj > 0) {
        double d[kDiagVals];
        if ((e = solid_diag(s, d))) return e;
        out->dev_detF = sqrt(d[4] * dv);
        out->max_dev_detF = sqrt(d[5]);
    }
    return RMT3D_OK;
}

// extents of a slice: the two axes other than dim, in increasing order, over
// the cells or (types 3, 4, 5, 7, 18) the nodes
static void slice_dims(const rmt3d_scene *s, int type, int dim, int *d1, int *d2) {
    const bool corner = (type >= 3 && type < 6) || type == 7 || type == 18;
    int ext[3] = {s->g.sm, s->g.sn, s->g.so};
    if (corner) {
        ext[0] = s->g.fm;
        ext[1] = s->g.fn;
        ext[2] = s->g.fo;
    }
    *d1 = ext[dim == 0 ? 1 : 0];
    *d2 = ext[dim == 2 ? 1 : 2];
}

extern "C" int rmt3d_slice(rmt3d_scene *s, int type, int dim, int point, int obj_id, double *out, int *d1,
                           int *d2) {
    if (!s || !d1 || !d2) return fail(RMT3D_ERR_INVALID, "null argument");
    if (type < 0 || type > 21) return fail(RMT3D_ERR_INVALID, "output type outside 0..21");
    if (dim < 0 || dim > 2) return fail(RMT3D_ERR_INVALID, "slice axis outside 0..2");
    if (obj_id != -1 && (obj_id < 1 || obj_id > s->g.n_obj)) return fail(RMT3D_ERR_INVALID, "object id outside -1, 1..n_obj");
    slice_dims(s, type, dim, d1, d2);
    if (!out) return RMT3D_OK;
    const size_t n = (size_t)*d1 * *d2;
    const int cells[3] = {s->g.sm, s->g.sn, s->g.so};
    if (point < 0 || point >= cells[dim]) {
        memset(out, 0, n * sizeof(double));
        return RMT3D_OK;
    }
    const grid_dev &g = s->g;
    if (type == 18) {  // fill_pp_rhs first (fluid_3d_io.cc:162-164)
        k_fem_rhs<<<grd(g.fm, g.fn, g.fo), blk(), 0, s->st>>>(g, s->dF, s->fem.rhs(), s->gradphi);
        s->count();
    }
    double *d = nullptr;
    CK(cudaMallocAsync((void **)&d, n * sizeof(double), s->st));
    k_slice<<<lin_blocks((int)n), 256, 0, s->st>>>(g, s->dF, s->fem.rhs(), type, dim, point, obj_id, s->d.var_den,
                                                  *d1, *d2, d);
    s->count();
    cudaError_t ce = cudaMemcpyAsync(out, d, n * sizeof(double), cudaMemcpyDeviceToHost, s->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->st);
    cudaFreeAsync(d, s->st);
    CK(ce);
    return RMT3D_OK;
}

extern "C" int rmt3d_write_slice(rmt3d_scene *s, int type, int dim, int point, int obj_id, int format,
                                 const char *filename) {
    if (!s || !filename) return fail(RMT3D_ERR_INVALID, "null argument");
    if (format < 0 || format > 2) return fail(RMT3D_ERR_INVALID, "slice format outside 0..2");
    int d1, d2;
    int e = rmt3d_slice(s, type, dim, point, obj_id, nullptr, &d1, &d2);
    if (e) return e;
    std::vector<double> u((size_t)d1 * d2);
    if ((e = rmt3d_slice(s, type, dim, point, obj_id, u.data(), &d1, &d2))) return e;
    // the coordinates of the two axes: cell centres (gx, gy, gz of
    // fluid_3d.cc:132-134), continued by the ghost centre for the last node
    // of a nodal axis
    const std::vector<double> *ax[3] = {&s->hlx, &s->hly, &s->hlz};
    const int a1 = dim == 0 ? 1 : 0, a2 = dim == 2 ? 1 : 2;
    std::vector<double> c1(d1), c2(d2);
    for (int i = 0; i < d1; i++) c1[i] = (*ax[a1])[i + 2];
    for (int j = 0; j < d2; j++) c2[j] = (*ax[a2])[j + 2];
    return slice_write_file(filename, u.data(), d1, d2, format, c1.data(), c2.data(), s->g.sm);
}

extern "C" int rmt3d_tracer_positions(rmt3d_scene *s, float *xyz, int max_tracers, int *n) {
    if (!s || !n) return fail(RMT3D_ERR_INVALID, "null argument");
    *n = s->ntr;
    if (!s->ntr || !xyz) return RMT3D_OK;
    float *d = nullptr;
    const size_t bytes = 3 * (size_t)s->ntr * sizeof(float);
    CK(cudaMallocAsync((void **)&d, bytes, s->st));
    k_tracer_positions<<<(s->ntr + 127) / 128, 128, 0, s->st>>>(tr_args(s), s->ntr, d);
    s->count();
    std::vector<float> h(3 * (size_t)s->ntr);
    cudaError_t ce = cudaMemcpyAsync(h.data(), d, bytes, cudaMemcpyDeviceToHost, s->st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->st);
    cudaFreeAsync(d, s->st);
    CK(ce);
    const int m = max_tracers < s->ntr ? max_tracers : s->ntr;
    memcpy(xyz, h.data(), 3 * (size_t)(m > 0 ? m : 0) * sizeof(float));
    return RMT3D_OK;
}

extern "C" int rmt3d_tracer_place(rmt3d_scene *s, const double *xyz, int n) {
    if (!s || !xyz) return fail(RMT3D_ERR_INVALID, "null argument");
    if (n != s->ntr) return fail(RMT3D_ERR_INVALID, "tracer count differs from the scene's ntracers");
    if (!s->ntr) return RMT3D_OK;
    return tracers_place(s, xyz);
}

extern "C" int rmt3d_write_tracers(rmt3d_scene *s, const char *filename, int binary) {
    if (!s || !filename) return fail(RMT3D_ERR_INVALID, "null argument");
    if (!s->ntr) return fail(RMT3D_ERR_INVALID, "the scene has no tracers (dump_code bit 1, ntracers)");
    std::vector<float> pos(3 * (size_t)s->ntr);
    int n = 0;
    int e = rmt3d_tracer_positions(s, pos.data(), s->ntr, &n);
    if (e) return e;
    return tracer_write_file(filename, pos.data(), n, binary);
}

extern "C" int rmt3d_sync(rmt3d_scene *s) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    CK(cudaStreamSynchronize(s->st));
    return RMT3D_OK;
}

extern "C" int rmt3d_launch_count(rmt3d_scene *s, long long *count) {
    if (!s || !count) return fail(RMT3D_ERR_INVALID, "null argument");
    *count = s->launches;
    return RMT3D_OK;
}

extern "C" int rmt3d_scene_set_mg_launch(rmt3d_scene *s, int cluster) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (cluster && (!s->mac.cluster_size || !s->fem.cluster_size))
        return fail(RMT3D_ERR_UNSUPPORTED, "thread-block clusters of 8 or more CTAs are not available");
    s->mac.use_cluster = s->fem.use_cluster = cluster != 0;
    s->mac.invalidate();
    s->fem.invalidate();
    mark_dirty(s);
    return RMT3D_OK;
}

extern "C" int rmt3d_scene_set_schedule(rmt3d_scene *s, int v_down, int v_up, int coarse_pts) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (v_down < 0 || v_up < 0 || v_down + v_up < 1 || v_down > 8 || v_up > 8)
        return fail(RMT3D_ERR_INVALID, "smoothing counts outside 0..8 (sum >= 1)");
    s->mac.v_down = s->fem.v_down = v_down;
    s->mac.v_up = s->fem.v_up = v_up;
    s->mac.invalidate();
    s->fem.invalidate();
    mark_dirty(s);
    if (coarse_pts >= 0 && (s->mac.set_coarse(coarse_pts) || s->fem.set_coarse(coarse_pts)))
        return fail(RMT3D_ERR_CUDA, "coarse multigrid kernel configuration failed");
    return RMT3D_OK;
}

namespace rmt3d {
void scene_schedule(rmt3d_scene *s, int out[5]) {
    out[0] = s->mac.v_down;
    out[1] = s->mac.v_up;
    out[2] = s->mac.smoother;
    out[3] = s->mac.use_cluster ? 1 : 0;
    out[4] = s->mac.cluster_coarse_pts;
}
}  // namespace rmt3d

extern "C" int rmt3d_scene_set_coarse_cluster(rmt3d_scene *s, int pts) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (pts < 0) return fail(RMT3D_ERR_INVALID, "negative level size");
    if (pts > 0 && (!s->mac.cluster_size || !s->fem.cluster_size))
        return fail(RMT3D_ERR_UNSUPPORTED, "thread-block clusters of 8 or more CTAs are not available");
    s->mac.set_cluster_coarse(pts);
    s->fem.set_cluster_coarse(pts);
    mark_dirty(s);
    return RMT3D_OK;
}

extern "C" int rmt3d_scene_set_block_shape(rmt3d_scene *s, int shape) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (shape < 0 || shape >= kNumBlockShapes) return fail(RMT3D_ERR_INVALID, "block shape index out of range");
    s->bshape = shape;
    mark_dirty(s);
    return RMT3D_OK;
}

extern "C" int rmt3d_scene_set_smoother(rmt3d_scene *s, int mode) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (mode < 0 || mode > 1) return fail(RMT3D_ERR_INVALID, "smoother mode must be 0 (colour passes) or 1 (tiled sweeps)");
    s->mac.smoother = s->fem.smoother = mode;
    s->mac.invalidate();
    s->fem.invalidate();
    mark_dirty(s);
    return RMT3D_OK;
}

extern "C" size_t rmt3d_scene_footprint(const rmt3d_scene_desc *d) {
    // mirrors the allocations of rmt3d_scene_create and mg_solver::setup
    if (!d || d->sys_size[0] < 1 || d->sys_size[1] < 1 || d->sys_size[2] < 1) return 0;
    const size_t n = (size_t)(d->sys_size[0] + 4) * (d->sys_size[1] + 4) * (d->sys_size[2] + 4);
    // the per-cell slab (commit_slab): arrays at 256-byte boundaries
    size_t b = slab_pad(n * sizeof(double)) * (18 + (d->var_den ? 1 : 0)) +
               18 * slab_pad(n * (face32(*d) ? sizeof(float) : sizeof(double)));
    b += (size_t)d->n_obj * (2 * slab_pad(n * sizeof(int)) + 51 * slab_pad(n * sizeof(double)));
    if (d->n_obj > 0) {
        const size_t no = (size_t)d->n_obj * n;
        b += slab_pad(no * sizeof(uint8_t)) + 3 * slab_pad(no * sizeof(int)) + slab_pad(2 * kMaxObj * sizeof(int)) +
             slab_pad(n * sizeof(int)) + slab_pad(sizeof(int));
    }
    if ((d->run.dump_code & 1) && d->run.ntracers > 0)
        b += (size_t)d->run.ntracers * (3 * sizeof(int) + 6 * sizeof(double) + sizeof(uint8_t));
    b += (size_t)(d->sys_size[0] + 4 + d->sys_size[1] + 4 + d->sys_size[2] + 4) * sizeof(double);
    b += sizeof(fields_dev) + sizeof(scene_ctl) + (1 + kMeanBlocks + 4) * sizeof(double) + sizeof(unsigned);
    b += kDiagVals * (1 + kMeanBlocks) * sizeof(double) + sizeof(unsigned);
    int prd[3], nm[3], nf[3];
    for (int a = 0; a < 3; a++) {
        prd[a] = d->periodic[a] != 0;
        nm[a] = d->sys_size[a];
        nf[a] = d->sys_size[a] + (prd[a] ? 0 : 1);
    }
    const bool mixed = mixed_form(d->precision);
    const size_t mac = mg_solver::footprint(MG_MAC, nm, prd, mixed), fem = mg_solver::footprint(MG_FEM, nf, prd, mixed);
    if (!mac || !fem) return 0;
    if (d->var_den) {
        std::vector<mg_level> lv;
        mg_solver::plan(MG_MAC, nm, prd, lv);
        for (auto &l : lv) b += l.npts() * (sizeof(double) + (mixed ? sizeof(float) : 0));
    }
    return b + mac + fem;
}

extern "C" int rmt3d_scene_checksum(rmt3d_scene *s, double out[4]) {
    if (!s || !out) return fail(RMT3D_ERR_INVALID, "null argument");
    const grid_dev &g = s->g;
    static_assert(4 <= kDiagVals, "checksum partials exceed the diagnostics area");
    k_checksum<<<kMeanBlocks, 256, 0, s->st>>>(g, s->dF, s->d_diag, s->diag_ticket);
    s->count();
    CK(cudaMemcpyAsync(out, s->d_diag, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return RMT3D_OK;
}

extern "C" int rmt3d_profile_kernel(rmt3d_scene *s, int kernel, int max_launches) {
    if (!s) return fail(RMT3D_ERR_INVALID, "null scene");
    if (kernel < -1 || kernel > 1) return fail(RMT3D_ERR_INVALID, "unknown kernel class");
    CK(cudaStreamSynchronize(s->st));
    for (cudaEvent_t e : s->prof.ev) cudaEventDestroy(e);
    s->prof.ev.clear();
    s->prof.used = 0;
    s->prof.points = s->prof.bytes = 0;
    s->prof.target = kernel;
    if (kernel >= 0) {
        s->prof.ev.resize(2 * (size_t)max_launches);
        for (auto &e : s->prof.ev) CK(cudaEventCreate(&e));
    }
    return RMT3D_OK;
}

extern "C" int rmt3d_profile_read(rmt3d_scene *s, double *ms_total, long long *launches, double *bytes_total) {
    if (!s || !ms_total || !launches || !bytes_total) return fail(RMT3D_ERR_INVALID, "null argument");
    CK(cudaStreamSynchronize(s->st));
    double tot = 0;
    for (size_t i = 0; i + 1 < s->prof.used; i += 2) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, s->prof.ev[i], s->prof.ev[i + 1]));
        tot += ms;
    }
    *ms_total = tot;
    *launches = (long long)(s->prof.used / 2);
    *bytes_total = s->prof.bytes;
    return RMT3D_OK;
}

extern "C" int rmt3d_scene_destroy(rmt3d_scene *s) {
    if (!s) return RMT3D_OK;
    cudaStreamSynchronize(s->st);
    if (s->cst) {
        cudaStreamSynchronize(s->cst);
        cudaStreamDestroy(s->cst);
        cudaEventDestroy(s->ev_snap);
        cudaEventDestroy(s->ev_d2h);
    }
    if (s->snap) cudaFreeAsync(s->snap, s->st);
    for (cudaEvent_t e : s->prof.ev) cudaEventDestroy(e);
    if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
    s->gb.release();
    for (void *p : s->allocs) cudaFreeAsync(p, s->st);
    s->mac.release();
    s->fem.release();
    cudaStreamSynchronize(s->st);
    if (s->h_ctl) pinned_put(s->h_ctl, sizeof(scene_ctl));
    if (s->h_scalar) pinned_put(s->h_scalar, sizeof(double));
    if (s->own_stream) cudaStreamDestroy(s->st);
    delete s;
    return RMT3D_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the divergence diagnostic.
//
// Some hosts cannot allocate device memory at the point where they want this
// diagnostic: a host that runs inside a memory pool it must not grow, a plugin
// that is only handed device pointers by its host application, or code that
// must not synchronise the device through cudaMalloc/cudaFree.  For them the
// scratch of div_u -- the FEM right-hand side over the node grid, the
// reduction accumulator and the small argument block the kernels read --
// lives in the fixed array below instead of in per-scene allocations.
//
// The array is sized for at most kNoallocMaxNodes FEM nodes (65^3, the node
// grid of a 64^3 box with walls) and is held by every GPU that loads this
// library until the process exits.  All calls share it and it keeps the last
// call's contents: the accumulator is cleared on every call, and calls that
// overlap on the GPU (different streams or threads) race on it.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoallocMaxNodes = 65 * 65 * 65;
constexpr size_t kNoallocHeader = 16384;  // accumulator + argument block, 256-aligned
constexpr size_t kNoallocBytes = kNoallocHeader + kNoallocMaxNodes * sizeof(double);
// [0, 256): reduction ticket; [256, kNoallocRed): argument block;
// [kNoallocRed, ...): fixed-order reduction partials of k_divu_l2
constexpr size_t kNoallocRed = 256 + (sizeof(fields_dev) + 255) / 256 * 256;
static_assert(kNoallocRed + (1 + kMeanBlocks) * sizeof(double) <= kNoallocHeader, "argument block does not fit");
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

namespace {
// Device address of the scratch array for the current device.  The symbol's
// name in host code is only a host-side stand-in, so the address is looked up
// with the device current, on every call: the lookup is cheap next to the
// call's own synchronisation, and a cached address would go stale if the
// host reset the device and the module were loaded again.
int noalloc_scratch(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(RMT3D_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = (unsigned char *)p;
    return RMT3D_OK;
}
}  // namespace

extern "C" int rmt3d_div_u_noalloc(const int sys_size[3], const int periodic[3], const double bounds[6],
                                   double dt_basis, const double *const dvel[3],
                                   const double *const face_normal_vel[6], void *stream, double *norm_out) {
    if (!sys_size || !periodic || !bounds || !dvel || !norm_out) return fail(RMT3D_ERR_INVALID, "null argument");
    for (int c = 0; c < 3; c++)
        if (!dvel[c]) return fail(RMT3D_ERR_INVALID, "null dvel pointer");
    grid_dev g;
    memset(&g, 0, sizeof(g));
    g.sm = sys_size[0];
    g.sn = sys_size[1];
    g.so = sys_size[2];
    if (g.sm < 1 || g.sn < 1 || g.so < 1) return fail(RMT3D_ERR_INVALID, "sys_size must be positive");
    for (int a = 0; a < 3; a++) g.prd[a] = periodic[a] ? 1 : 0;
    g.fm = g.sm + (g.prd[0] ? 0 : 1);
    g.fn = g.sn + (g.prd[1] ? 0 : 1);
    g.fo = g.so + (g.prd[2] ? 0 : 1);
    const size_t nodes = (size_t)g.fm * g.fn * g.fo;
    if (nodes > kNoallocMaxNodes)
        return fail(RMT3D_ERR_TOO_LARGE, "rmt3d_div_u_noalloc: at most 274625 FEM nodes (65^3); got " +
                                             std::to_string(nodes));
    for (int f = 0; f < 6; f++)
        if (!g.prd[f / 2] && (!face_normal_vel || !face_normal_vel[f]))
            return fail(RMT3D_ERR_INVALID, "a wall face needs its normal face-velocity array");
    g.sm4 = g.sm + 4;
    g.sn4 = g.sn + 4;
    g.so4 = g.so + 4;
    g.smn4 = g.sm4 * g.sn4;
    g.ncell = g.smn4 * g.so4;
    g.dx = (bounds[1] - bounds[0]) / g.sm;
    g.dy = (bounds[3] - bounds[2]) / g.sn;
    g.dz = (bounds[5] - bounds[4]) / g.so;
    // compute_grad_basis (fluid_3d.cc:2506-2517)
    gradphi_t gp;
    const double fac = 3 * g.dx / dt_basis;
    for (int i = 0; i < 8; i++) {
        gp.v[i][0] = (2 * (i % 2) - 1) * fac;
        gp.v[i][1] = (2 * ((i / 2) % 2) - 1) * fac;
        gp.v[i][2] = (2 * (i / 4) - 1) * fac;
    }
    // argument block: only the arrays div_u reads
    static thread_local fields_dev hf;
    memset(&hf, 0, sizeof(hf));
    for (int c = 0; c < 3; c++) hf.dvel[c] = const_cast<double *>(dvel[c]);
    for (int f = 0; f < 6; f++)
        if (face_normal_vel && face_normal_vel[f]) hf.fvel[3 * f + f / 2] = const_cast<double *>(face_normal_vel[f]);
    unsigned char *base = nullptr;
    int e = noalloc_scratch(&base);
    if (e) return e;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *ticket = (unsigned *)base;
    fields_dev *dF = (fields_dev *)(base + 256);
    double *red = (double *)(base + kNoallocRed);
    double *rhs = (double *)(base + kNoallocHeader);
    CK(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
    CK(cudaMemcpyAsync(dF, &hf, sizeof(hf), cudaMemcpyHostToDevice, st));
    k_fem_rhs<<<grd(g.fm, g.fn, g.fo), blk(), 0, st>>>(g, dF, rhs, gp);
    k_divu_l2<<<kMeanBlocks, 256, 0, st>>>(g, rhs, red, ticket);
    double sum = 0;
    CK(cudaMemcpyAsync(&sum, red, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    *norm_out = sqrt(sum / ((double)g.fm * g.fn * g.fo));
    return RMT3D_OK;
}
