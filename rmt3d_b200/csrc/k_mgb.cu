// Batched multigrid: one solve for every scene of a group of equally sized
// scenes, each phase one launch over all of them.
//
// The scenes keep their own level arrays, right-hand sides and control state
// (mg_ctl); the group holds device tables of their pointers.  Every batched
// kernel maps blockIdx.z (or blockIdx.y) to (scene, block within the scene)
// and runs the same body as the single-scene kernel (mg_body.cuh), so each
// scene's solve is bit-identical to its solo solve.  Scenes take part in
// a solve when their flag part[b] is set (a halted or reverted scene sits
// out); a scene whose own control has finished stops being touched while the
// others continue (run[b]).  The graph WHILE loop repeats while any scene of
// the group is still running; each scene's number of cycles is exactly its
// solo number.
#include <cstring>

#include "graph_build.h"
#include "host_common.h"
#include "mg.h"
#include "mg_body.cuh"
#include "mg_ops.cuh"
#include "mg_tile.cuh"
#include "rmt3d_gpu.h"

namespace rmt3d {

// scene of this block and the block's z index within the scene
#define MGB_SCENE(zb)                             \
    const int b_ = blockIdx.z / (zb);             \
    if (!run[b_]) return;                         \
    const int bz_ = blockIdx.z - b_ * (zb);

template <typename T>
__global__ void k_mac_rb_b(lvl_dev L, T *const *x, T *const *r, const T *const *ri, int colour, const int *run,
                           int zb) {
    MGB_SCENE(zb)
    body_mac_rb<T>(L, x[b_], r[b_], colour, ri ? ri[b_] : nullptr, blockIdx.x, blockIdx.y, bz_);
}
// FP32: at most 51 registers, five 256-thread blocks per SM; FP64 keeps
// four (64 registers; its stencil state spills at 51)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 5 : 4) k_fem_gs_b(lvl_dev L, T *const *x, T *const *r, const T *const *ri, int colour, const int *run,
                           int zb) {
    MGB_SCENE(zb)
    body_fem_gs<T>(L, x[b_], r[b_], colour, ri ? ri[b_] : nullptr, blockIdx.x, blockIdx.y, bz_);
}
template <typename T, int KIND>
__global__ void k_resid_b(lvl_dev L, T *const *x, T *const *r, T *const *res, const T *const *ri,
                          unsigned long long *const *mx, const int *run, int zb) {
    MGB_SCENE(zb)
    const double a = body_resid<T, KIND>(L, x[b_], r[b_], res ? res[b_] : nullptr, ri ? ri[b_] : nullptr,
                                         blockIdx.x, blockIdx.y, bz_);
    if (mx) warp_max_into(a, mx[b_]);
}
// the control's residual: only for scenes whose control will read it
template <int KIND>
__global__ void k_resid_ctl_b(lvl_dev L, double *const *x, double *const *r, const double *const *ri,
                              unsigned long long *const *mx, mg_ctl *const *ctl, const int *run, int zb) {
    MGB_SCENE(zb)
    if (!ctl[b_]->need_res) return;
    const double a = body_resid<double, KIND>(L, x[b_], r[b_], nullptr, ri ? ri[b_] : nullptr, blockIdx.x,
                                              blockIdx.y, bz_);
    warp_max_into(a, mx[b_]);
}
template <typename T>
__global__ void k_mac_restrict_b(lvl_dev F, lvl_dev C, T *const *res, T *const *rc, T *const *xc, const int *run,
                                 int zb) {
    MGB_SCENE(zb)
    body_mac_restrict<T>(F, C, res[b_], rc[b_], xc[b_], blockIdx.x, blockIdx.y, bz_);
}
template <typename T>
__global__ void k_fem_restrict_b(lvl_dev F, lvl_dev C, T *const *res, T *const *rc, T *const *xc, const int *run,
                                 int zb) {
    MGB_SCENE(zb)
    body_fem_restrict<T>(F, C, res[b_], rc[b_], xc[b_], blockIdx.x, blockIdx.y, bz_);
}
template <int KIND>
__global__ void k_resid_to_f32_b(lvl_dev L, double *const *x, double *const *r, const double *const *ri,
                                 float *const *rs, float *const *xs, const int *run, int zb) {
    MGB_SCENE(zb)
    body_resid_to_f32<KIND>(L, x[b_], r[b_], ri ? ri[b_] : nullptr, rs[b_], xs[b_], blockIdx.x, blockIdx.y, bz_);
}
template <typename T>
__global__ void k_mac_prolong_b(lvl_dev F, lvl_dev C, T *const *x, T *const *xc, const int *run, int zb) {
    MGB_SCENE(zb)
    body_mac_prolong<T>(F, C, x[b_], xc[b_], blockIdx.x, blockIdx.y, bz_);
}
template <typename T>
__global__ void k_fem_prolong_b(lvl_dev F, lvl_dev C, T *const *x, T *const *xc, const int *run, int zb) {
    MGB_SCENE(zb)
    body_fem_prolong<T>(F, C, x[b_], xc[b_], blockIdx.x, blockIdx.y, bz_);
}
// one tiled sweep (mg_tile.cuh) of every running scene: blockIdx.z = scene x
// z box
template <typename T, int KIND, bool VD>
__global__ void __launch_bounds__(512) k_tile_sweep_b(lvl_dev L, T *const *xin, T *const *xout, T *const *r,
                                                      const T *const *ri, const int *run, int zb) {
    extern __shared__ __align__(16) unsigned char tile_smem[];
    MGB_SCENE(zb)
    using S = tile_shape<T, KIND, VD>;
    body_tile_sweep<T, KIND, VD>(L, xin[b_], xout[b_], r[b_], VD ? ri[b_] : nullptr, blockIdx.x * S::TX,
                                 blockIdx.y * S::TY, bz_ * S::TZ, tile_smem);
}

template <typename T, int KIND, bool VD>
static int tile_attr_b() {
    return cudaFuncSetAttribute((const void *)k_tile_sweep_b<T, KIND, VD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tile_smem_bytes<T, KIND, VD>()) != cudaSuccess;
}

int tile_setup_batched() {
    return tile_attr_b<double, 0, false>() | tile_attr_b<double, 0, true>() | tile_attr_b<double, 1, false>() |
           tile_attr_b<double, 1, true>() | tile_attr_b<float, 0, false>() | tile_attr_b<float, 0, true>() |
           tile_attr_b<float, 1, false>() | tile_attr_b<float, 1, true>();
}

template <typename T>
__global__ void k_copy_b(T *const *a, T *const *b, size_t n, const int *run) {
    if (!run[blockIdx.y]) return;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[blockIdx.y][i] = a[blockIdx.y][i];
}

// one-dimensional phases: blockIdx.y is the scene
template <typename T>
__global__ void k_coarse_dense_b(int np, const double *__restrict__ B, T *const *x, T *const *r, const int *run) {
    if (!run[blockIdx.y]) return;
    body_coarse_dense<T>(np, B, x[blockIdx.y], r[blockIdx.y], blockIdx.x, gridDim.x);
}
template <typename T, int KIND>
__global__ void k_coarse_solve_b(lvl_dev L, T *const *x, T *const *r, int sweeps, const int *run) {
    if (!run[blockIdx.x]) return;
    body_coarse_solve<T, KIND>(L, x[blockIdx.x], r[blockIdx.x], sweeps);
}
__global__ void k_to_f32_b(double *const *a, float *const *b, size_t n, const int *run) {
    if (!run[blockIdx.y]) return;
    body_to_f32(a[blockIdx.y], b[blockIdx.y], n, blockIdx.x);
}
__global__ void k_add_f32_b(double *const *a, float *const *b, size_t n, const int *run) {
    if (!run[blockIdx.y]) return;
    body_add_f32(a[blockIdx.y], b[blockIdx.y], n, blockIdx.x);
}
template <typename T>
__global__ void k_zero_b(T *const *a, size_t n, const int *run) {
    if (!run[blockIdx.y]) return;
    body_zero<T>(a[blockIdx.y], n, blockIdx.x);
}
__global__ void k_absmax_b(double *const *r, size_t n, unsigned long long *const *mx, const int *run) {
    if (!run[blockIdx.y]) return;
    const double *rr = r[blockIdx.y];
    double a = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = fabs(rr[i]);
        if (v != v || v > a) a = (v != v) ? __longlong_as_double(0x7ff8000000000000LL) : v;
    }
    unsigned long long bb = (unsigned long long)__double_as_longlong(a);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, bb, o);
        bb = t > bb ? t : bb;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(mx[blockIdx.y] + 1, bb);
}

// arm the group's solve: the taking-part scenes start their control state;
// the loop runs if any scene takes part (one block, one thread per scene)
__global__ void k_mgb_begin(mg_ctl *const *ctl, unsigned long long *const *mx, const int *part, int *run, int B,
                            cudaGraphConditionalHandle h) {
    const int b = threadIdx.x;
    int on = 0;
    if (b < B) {
        on = part[b] != 0;
        run[b] = on;
        if (on) mg_begin_state(ctl[b], mx[b]);
    }
    const int any = __syncthreads_or(on);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// after an iteration: every running scene steps its own control; the loop
// continues while any scene is still running
__global__ void k_mgb_ctl(mg_ctl *const *ctl, unsigned long long *const *mx, int *run, int B, double tol,
                          double rtol, int exact, cudaGraphConditionalHandle h) {
    const int b = threadIdx.x;
    int on = 0;
    if (b < B && run[b]) {
        on = mg_ctl_step(ctl[b], mx[b], tol, rtol, exact) ? 0 : 1;
        run[b] = on;
    }
    const int any = __syncthreads_or(on);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// ---- host side -------------------------------------------------------------
static lvl_dev ldv(const mg_level &l) { return lvl_dev{l.n[0], l.n[1], l.n[2], l.prd[0], l.prd[1], l.prd[2]}; }
static dim3 gblk() { return dim3(32, 4, 2); }
// per-scene grid of a level phase over (a, b, c) points; z spans the scenes
static dim3 ggrid(int a, int b, int c, int B, int &zb) {
    zb = (c + 1) / 2;
    return dim3((a + 31) / 32, (b + 3) / 4, zb * B);
}

void mg_group::release() {
    if (dev_tables) cudaFreeAsync(dev_tables, tstream);
    if (dargs) cudaFreeAsync(dargs, tstream);
    dev_tables = nullptr;
    dargs = nullptr;
}

mg_group::~mg_group() { release(); }

int mg_group::setup(const std::vector<mg_solver *> &solvers, cudaStream_t st) {
    tstream = st;
    if (solvers.empty() || solvers.size() > 1024) return fail(RMT3D_ERR_INVALID, "group of 1..1024 scenes");
    const mg_solver &s0 = *solvers[0];
    B = (int)solvers.size();
    kind = s0.kind;
    lv = s0.lv;
    mixed = s0.mixed;
    exact = s0.exact;
    vd = s0.vd;
    tol = s0.max_norm_tol;
    rtol = s0.rtol;
    v_down = s0.v_down;
    v_up = s0.v_up;
    smoother = s0.smoother;
    ccl = s0.ccl;
    csize = s0.cluster_size;
    dense = s0.dense;
    for (const mg_solver *m : solvers) {
        bool same = m->kind == kind && m->lv.size() == lv.size() && m->mixed == mixed && m->exact == exact &&
                    m->vd == vd && m->rtol == rtol && m->dense == dense && m->v_down == v_down && m->v_up == v_up &&
                    m->smoother == smoother && m->ccl == ccl && m->cluster_size == csize;
        for (size_t l = 0; same && l < lv.size(); l++)
            for (int d = 0; d < 3; d++) same = same && m->lv[l].n[d] == lv[l].n[d] && m->lv[l].prd[d] == lv[l].prd[d];
        if (!same) return fail(RMT3D_ERR_INVALID, "scenes of a multigrid group must match in size, form and schedule");
    }
    // one device block: per level 8 pointer tables of B entries, then the
    // control pointers, the residual slots' pointers and part/run flags
    const size_t L = lv.size();
    const size_t nptr = L * 8 * B + 2 * B;
    const size_t bytes = nptr * sizeof(void *) + 2 * B * sizeof(int);
    if (cudaMallocAsync(&dev_tables, bytes, st) != cudaSuccess)
        return fail(RMT3D_ERR_OOM, "group table allocation failed");
    std::vector<void *> h(nptr, nullptr);
    for (size_t l = 0; l < L; l++)
        for (int b = 0; b < B; b++) {
            const mg_level &q = solvers[b]->lv[l];
            void **row = &h[(l * 8) * B];
            row[0 * B + b] = q.x;
            row[1 * B + b] = q.r;
            row[2 * B + b] = q.res;
            row[3 * B + b] = q.xs;
            row[4 * B + b] = q.rs;
            row[5 * B + b] = q.ress;
            row[6 * B + b] = (void *)q.ri;
            row[7 * B + b] = (void *)q.ris;
        }
    for (int b = 0; b < B; b++) {
        h[L * 8 * B + b] = solvers[b]->ctl;
        h[L * 8 * B + B + b] = solvers[b]->max_slots();
    }
    cudaMemcpyAsync(dev_tables, h.data(), nptr * sizeof(void *), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync((char *)dev_tables + nptr * sizeof(void *), 0, 2 * B * sizeof(int), st);
    void **d = (void **)dev_tables;
    tab.resize(L);
    for (size_t l = 0; l < L; l++) {
        void **row = d + (l * 8) * B;
        tab[l].x = (double **)(row + 0 * B);
        tab[l].r = (double **)(row + 1 * B);
        tab[l].res = (double **)(row + 2 * B);
        tab[l].xs = (float **)(row + 3 * B);
        tab[l].rs = (float **)(row + 4 * B);
        tab[l].ress = (float **)(row + 5 * B);
        tab[l].ri = vd ? (const double **)(row + 6 * B) : nullptr;
        tab[l].ris = vd ? (const float **)(row + 7 * B) : nullptr;
    }
    ctls = (mg_ctl **)(d + L * 8 * B);
    mx = (unsigned long long **)(d + L * 8 * B + B);
    part = (int *)(d + nptr);
    run = part + B;
    if (ccl >= 0) {
        std::vector<pmg_args> ha;
        for (const mg_solver *m : solvers) ha.push_back(level_args(*m));
        if (cudaMallocAsync(&dargs, B * sizeof(pmg_args), st) != cudaSuccess)
            return fail(RMT3D_ERR_OOM, "group table allocation failed");
        cudaMemcpyAsync(dargs, ha.data(), B * sizeof(pmg_args), cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);  // the host copy of the tables goes out of scope
    }
    cudaStreamSynchronize(st);
    return cudaGetLastError() == cudaSuccess ? 0 : fail(RMT3D_ERR_CUDA, "group table upload failed");
}

template <typename T, int KIND, bool VD>
static void tile_sweep_bk(mg_group &g, const mg_level &L, T *const *xin, T *const *xout, T *const *r,
                          const T *const *ri, cudaStream_t st) {
    using S = tile_shape<T, KIND, VD>;
    const int zb = (L.n[2] + S::TZ - 1) / S::TZ;
    const dim3 gr((L.n[0] + S::TX - 1) / S::TX, (L.n[1] + S::TY - 1) / S::TY, zb * g.B);
    k_tile_sweep_b<T, KIND, VD><<<gr, S::NT, tile_smem_bytes<T, KIND, VD>(), st>>>(ldv(L), xin, xout, r, ri, g.run,
                                                                                     zb);
}

template <typename T>
static void tile_sweep_b(mg_group &g, int l, T *const *xin, T *const *xout, T *const *r, const T *const *ri,
                         cudaStream_t st) {
    const mg_level &L = g.lv[l];
    if (g.kind == MG_MAC) {
        if (ri) tile_sweep_bk<T, 0, true>(g, L, xin, xout, r, ri, st);
        else tile_sweep_bk<T, 0, false>(g, L, xin, xout, r, ri, st);
    } else {
        if (ri) tile_sweep_bk<T, 1, true>(g, L, xin, xout, r, ri, st);
        else tile_sweep_bk<T, 1, false>(g, L, xin, xout, r, ri, st);
    }
    g.body_kernels++;
}

// ν sweeps of level l starting in array `cur` (0 x, 1 residual array);
// returns the array holding the result
template <typename T>
static int smooth_b(mg_group &g, int l, int sweeps, int cur, cudaStream_t st, T *const *const xb[2], T *const *r,
                    const T *const *ri) {
    const mg_level &L = g.lv[l];
    const lvl_dev d = ldv(L);
    for (int s = 0; s < sweeps; s++) {
        if (g.smoother == 1) {
            tile_sweep_b<T>(g, l, xb[cur], xb[cur ^ 1], r, ri, st);
            cur ^= 1;
        } else if (g.kind == MG_MAC) {
            int zb = (L.n[2] + 1) / 2;
            dim3 gr((L.n[0] / 2 + 1 + 31) / 32, (L.n[1] + 3) / 4, zb * g.B);
            for (int c = 0; c < 2; c++) {
                k_mac_rb_b<T><<<gr, gblk(), 0, st>>>(d, xb[cur], r, ri, c, g.run, zb);
                g.body_kernels++;
            }
        } else {
            int zb = (L.n[2] + 1) / 2;
            dim3 gr(((L.n[0] + 1) / 2 + 31) / 32, ((L.n[1] + 1) / 2 + 3) / 4, zb * g.B);
            for (int c = 0; c < 4; c++) {
                k_fem_gs_b<T><<<gr, gblk(), 0, st>>>(d, xb[cur], r, ri, c, g.run, zb);
                g.body_kernels++;
            }
        }
    }
    return cur;
}

template <typename T>
static int cycle_b(mg_group &g, int l, cudaStream_t st) {
    const bool f32 = sizeof(T) == 4;
    auto X = [&](int q) { return f32 ? (T *const *)g.tab[q].xs : (T *const *)g.tab[q].x; };
    auto Rr = [&](int q) { return f32 ? (T *const *)g.tab[q].rs : (T *const *)g.tab[q].r; };
    auto S = [&](int q) { return f32 ? (T *const *)g.tab[q].ress : (T *const *)g.tab[q].res; };
    auto RI = [&](int q) { return f32 ? (const T *const *)g.tab[q].ris : (const T *const *)g.tab[q].ri; };
    const mg_level &F = g.lv[l];
    const int nl = (int)g.lv.size();
    if (l == g.ccl) {
        coarse_cluster_b(g.dargs, g.run, g.B, l, g.csize, sizeof(T) == 4, st);
        g.body_kernels++;
        return 0;
    }
    if (l == nl - 1) {
        if (g.dense) {
            const int np = (int)F.npts();
            k_coarse_dense_b<T><<<dim3((np + 7) / 8, g.B), 256, 0, st>>>(np, g.dense, X(l), Rr(l), g.run);
            g.body_kernels++;
        } else {
            // no dense inverse for this level shape: the solo fallback, one block per scene
            if (g.kind == MG_MAC)
                k_coarse_solve_b<T, 0><<<g.B, 512, 0, st>>>(ldv(F), X(l), Rr(l), 80, g.run);
            else
                k_coarse_solve_b<T, 1><<<g.B, 512, 0, st>>>(ldv(F), X(l), Rr(l), 80, g.run);
            g.body_kernels++;
        }
        return 0;
    }
    T *const *const xb[2] = {X(l), S(l)};
    int cur = smooth_b<T>(g, l, g.v_down, 0, st, xb, Rr(l), RI(l));
    const mg_level &C = g.lv[l + 1];
    int zbf, zbc;
    const dim3 gf = ggrid(F.n[0], F.n[1], F.n[2], g.B, zbf), gc = ggrid(C.n[0], C.n[1], C.n[2], g.B, zbc);
    if (g.kind == MG_MAC) {
        k_resid_b<T, 0><<<gf, gblk(), 0, st>>>(ldv(F), xb[cur], Rr(l), xb[cur ^ 1], RI(l), nullptr, g.run, zbf);
        k_mac_restrict_b<T><<<gc, gblk(), 0, st>>>(ldv(F), ldv(C), xb[cur ^ 1], Rr(l + 1), X(l + 1), g.run, zbc);
    } else {
        k_resid_b<T, 1><<<gf, gblk(), 0, st>>>(ldv(F), xb[cur], Rr(l), xb[cur ^ 1], RI(l), nullptr, g.run, zbf);
        k_fem_restrict_b<T><<<gc, gblk(), 0, st>>>(ldv(F), ldv(C), xb[cur ^ 1], Rr(l + 1), X(l + 1), g.run, zbc);
    }
    g.body_kernels += 2;
    const int cc = cycle_b<T>(g, l + 1, st);
    T *const *xc = cc ? S(l + 1) : X(l + 1);
    if (g.kind == MG_MAC) k_mac_prolong_b<T><<<gf, gblk(), 0, st>>>(ldv(F), ldv(C), xb[cur], xc, g.run, zbf);
    else k_fem_prolong_b<T><<<gf, gblk(), 0, st>>>(ldv(F), ldv(C), xb[cur], xc, g.run, zbf);
    g.body_kernels++;
    return smooth_b<T>(g, l, g.v_up, cur, st, xb, Rr(l), RI(l));
}

// one iteration for every running scene: a V-cycle, or the mixed form's
// refinement step (FP64 residual, FP32 V-cycle on the correction, update)
void mg_group::iterate(cudaStream_t st) {
    if (!mixed) {
        if (cycle_b<double>(*this, 0, st)) {
            // the fine level's solution ended in its residual array
            const size_t n = lv[0].npts();
            k_copy_b<double><<<dim3((unsigned)((n + 255) / 256), B), 256, 0, st>>>(tab[0].res, tab[0].x, n, run);
            body_kernels++;
        }
        return;
    }
    const mg_level &F = lv[0];
    int zbf;
    const dim3 gf = ggrid(F.n[0], F.n[1], F.n[2], B, zbf);
    const size_t n = F.npts();
    const dim3 g1((unsigned)((n + 255) / 256), B);
    // FP64 residual -> FP32 right-hand side, FP32 start value zero (one pass)
    if (kind == MG_MAC)
        k_resid_to_f32_b<0><<<gf, gblk(), 0, st>>>(ldv(F), tab[0].x, tab[0].r, tab[0].ri, tab[0].rs, tab[0].xs, run, zbf);
    else
        k_resid_to_f32_b<1><<<gf, gblk(), 0, st>>>(ldv(F), tab[0].x, tab[0].r, tab[0].ri, tab[0].rs, tab[0].xs, run, zbf);
    body_kernels++;
    const int cur = cycle_b<float>(*this, 0, st);
    k_add_f32_b<<<g1, 256, 0, st>>>(tab[0].x, cur ? tab[0].ress : tab[0].xs, n, run);
    body_kernels++;
}

int mg_group::capture(cudaStream_t cur, graph_builder &gb) {
    cudaGraphConditionalHandle h = gb.handle(cur);
    if (gb.err != cudaSuccess) return -1;
    k_mgb_begin<<<1, 1024, 0, cur>>>(ctls, mx, part, run, B, h);
    outside_kernels = 1;
    if (rtol > 0) {
        k_absmax_b<<<dim3(148, B), 256, 0, cur>>>(tab[0].r, lv[0].npts(), mx, run);
        outside_kernels = 2;
    }
    cudaStream_t body = gb.open(cur, h, cudaGraphCondTypeWhile);
    if (!body) return -1;
    body_kernels = 0;
    iterate(body);
    const mg_level &F = lv[0];
    int zbf;
    const dim3 gf = ggrid(F.n[0], F.n[1], F.n[2], B, zbf);
    if (kind == MG_MAC)
        k_resid_ctl_b<0><<<gf, gblk(), 0, body>>>(ldv(F), tab[0].x, tab[0].r, tab[0].ri, mx, ctls, run, zbf);
    else
        k_resid_ctl_b<1><<<gf, gblk(), 0, body>>>(ldv(F), tab[0].x, tab[0].r, tab[0].ri, mx, ctls, run, zbf);
    k_mgb_ctl<<<1, 1024, 0, body>>>(ctls, mx, run, B, tol, rtol, exact ? 1 : 0, h);
    body_kernels += 2;
    gb.close(body);
    return gb.err == cudaSuccess ? 0 : -1;
}

}  // namespace rmt3d
