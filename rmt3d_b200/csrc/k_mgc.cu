// Multigrid solve in one thread-block cluster: one launch per Poisson solve.
//
// The whole solve -- every V-cycle (or FP64 refinement iteration of the mixed
// form), the max-norm residual after each, and the reference's control logic
// (mg_prob::run, Utilities/mg_probs.cc:3-83, with mg_pred, mg_probs.hh:37-78) --
// runs inside one cluster of up to 16 CTAs.  Phases are separated by the
// hardware cluster barrier (release/acquire at cluster scope), which makes
// the global-memory writes of one phase visible to every CTA of the next.
// The residual maximum is reduced through distributed shared memory; every
// CTA reads the same partials in the same order, so the loop decisions -- and
// with them the sequence of barriers -- are identical in all CTAs.  There is
// no spin-wait: every loop is bounded (levels, sweeps, colours, kMgMaxCycles).
//
// Small, latency-bound levels run far more efficiently this way than as one
// full-GPU launch per phase: a 64^3 solve occupies 16 SMs, and the other SMs
// are free for other scenes' solves.
#include <cooperative_groups.h>

#include <cmath>
#include <cstring>

#include "host_common.h"
#include "mg.h"
#include "mg_ops.cuh"
#include "rmt3d_gpu.h"

namespace cg = cooperative_groups;

namespace rmt3d {

constexpr int kClThreads = 512;

struct cmg_args {
    pmg_args A;
    double tol, rtol;
    int exact, mixed;
    mg_ctl *ctl;
};

// NaN-sticky maximum over the cluster (every thread gets the same value)
__device__ double cl_max(cg::cluster_group &cl, double m) {
    __shared__ double wred[kClThreads / 32];
    __shared__ double cta, all;
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, m, o);
        if (v != v || v > m) m = v;
    }
    if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            if (wred[w] != wred[w] || wred[w] > b) b = wred[w];
        cta = b;
    }
    cl.sync();
    if (threadIdx.x == 0) {
        double g = 0;
        for (unsigned rk = 0; rk < cl.num_blocks(); rk++) {
            const double v = *cl.map_shared_rank(&cta, rk);
            if (v != v || v > g) g = v;
        }
        all = g;
    }
    cl.sync();  // every CTA has read every partial before any is rewritten
    return all;
}

// a V-cycle from level l0 down (l0 > 0: the coarse part of a cycle whose
// finer levels run elsewhere; level l0's x starts at zero)
template <typename T>
__device__ void cl_vcycle(const pmg_args &A, cg::cluster_group &cl, int t0, int ts, int l0 = 0) {
    const int nc = A.kind == 0 ? 2 : 4;
    for (int l = l0; l < A.nlev - 1; l++) {
        const pmg_level &F = A.lv[l];
        for (int s = 0; s < A.v_down; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LRI<T>(F), c, t0, ts);
                cl.sync();
            }
        ph_resid<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LS<T>(F), LRI<T>(F), t0, ts);
        cl.sync();
        const pmg_level &C = A.lv[l + 1];
        ph_restrict<T>(A.kind, ldev(F), ldev(C), LS<T>(F), LR<T>(C), LX<T>(C), t0, ts);
        cl.sync();
    }
    {  // coarsest level
        const pmg_level &L = A.lv[A.nlev - 1];
        const int np = L.n[0] * L.n[1] * L.n[2];
        T *x = LX<T>(L);
        const T *r = LR<T>(L);
        if (A.dense) {
            // one warp per row of the (row-major) inverse
            const int warp = t0 >> 5, lane = t0 & 31, nw = ts >> 5;
            for (int row = warp; row < np; row += nw) {
                const double *b = A.dense + (size_t)row * np;
                double acc = 0;
                for (int c = lane; c < np; c += 32) acc += b[c] * (double)r[c];
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) x[row] = (T)acc;
            }
            cl.sync();
        } else {
            for (int p = t0; p < np; p += ts) x[p] = 0;
            cl.sync();
            for (int s = 0; s < 80; s++)
                for (int c = 0; c < nc; c++) {
                    ph_smooth_colour<T>(A.kind, ldev(L), x, r, LRI<T>(L), c, t0, ts);
                    cl.sync();
                }
        }
    }
    for (int l = A.nlev - 2; l >= l0; l--) {
        const pmg_level &F = A.lv[l];
        const pmg_level &C = A.lv[l + 1];
        ph_prolong<T>(A.kind, ldev(F), ldev(C), LX<T>(F), LX<T>(C), t0, ts);
        cl.sync();
        for (int s = 0; s < A.v_up; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LRI<T>(F), c, t0, ts);
                cl.sync();
            }
    }
}

// one iteration of the solver: a V-cycle, or in the mixed form one FP64
// refinement step around an FP32 V-cycle on the correction
__device__ void cl_iterate(const cmg_args &P, cg::cluster_group &cl, int t0, int ts) {
    if (!P.mixed) {
        cl_vcycle<double>(P.A, cl, t0, ts);
        return;
    }
    const pmg_level &L = P.A.lv[0];
    const int tot = L.n[0] * L.n[1] * L.n[2];
    ph_resid<double>(P.A.kind, ldev(L), L.x, L.r, L.res, L.ri, t0, ts);
    cl.sync();
    for (int t = t0; t < tot; t += ts) {
        L.rs[t] = (float)L.res[t];
        L.xs[t] = 0;
    }
    cl.sync();
    cl_vcycle<float>(P.A, cl, t0, ts);
    for (int t = t0; t < tot; t += ts) L.x[t] += (double)L.xs[t];
    cl.sync();
}

__global__ void __launch_bounds__(kClThreads, 1) k_mg_cluster(cmg_args P) {
    cg::cluster_group cl = cg::this_cluster();
    const int t0 = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    const int ts = (int)cl.num_blocks() * blockDim.x;
    const pmg_level &L0 = P.A.lv[0];
    // control state, identical in every thread of the cluster
    const int iV = P.ctl->iV;
    const double V_avg = P.ctl->V_avg, V_var = P.ctl->V_var;
    const long long total0 = P.ctl->cycles_total;
    int phase = 0, todo = iV / kMgIP, extra = 0, it = 0, count = 0;
    if (todo < 1) todo = 1;
    double prev = 0, res_out = 0;
    bool done = false;
    double tol = P.tol;
    if (P.rtol > 0) {
        // the mixed form's relative tolerance: mixed_rtol x max |rhs|
        double a = 0;
        const int n0 = L0.n[0] * L0.n[1] * L0.n[2];
        for (int t = t0; t < n0; t += ts) {
            const double v = fabs(L0.r[t]);
            if (v != v || v > a) a = v;
        }
        const double rhs = cl_max(cl, a);
        if (P.rtol * rhs > tol) tol = P.rtol * rhs;
    }
    while (!done) {
        cl_iterate(P, cl, t0, ts);
        const double r = cl_max(cl, ph_resid<double>(P.A.kind, ldev(L0), L0.x, L0.r, nullptr, L0.ri, t0, ts));
        count++;
        if (phase <= 1) {
            if (--todo <= 0) {
                res_out = r;
                if (r > tol && extra < 20) {
                    extra++;
                    todo = extra;
                    phase = 1;
                } else if (P.rtol > 0 && !P.exact) {
                    done = true;  // the relaxed form skips the insurance cycles
                } else {
                    phase = 2;
                    todo = 2;
                }
            }
        } else if (phase == 2) {
            if (--todo <= 0) {
                if (P.exact) {
                    prev = 1e300;
                    res_out = r;
                    it = 0;
                    if (r > 0 && r < 0.7 * prev) phase = 3;
                    else done = true;
                } else {
                    done = true;
                }
            }
        } else {
            prev = res_out;
            res_out = r;
            it++;
            if (!(it < 60 && r > 0 && r < 0.7 * prev)) done = true;
        }
        if (count >= kMgMaxCycles) done = true;
    }
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
        // mg_pred::update (alpha = 0)
        mg_ctl *c = P.ctl;
        const double alpha = 1 / (3 * kMgIP);
        const double dV = iV - V_avg;
        int exreduce = static_cast<int>(dV / sqrt(V_var));
        exreduce = exreduce > 0 ? exreduce : 0;
        int nv = iV + kMgIP * extra * (extra + 1) / 2 - 1 - exreduce;
        if (nv < kMgIP) nv = 2 * kMgIP - 1;
        c->iV = nv;
        c->V_avg = (1 - alpha) * V_avg + alpha * nv;
        c->V_var = (1 - alpha) * (V_var + alpha * dV * dV);
        c->phase = phase;
        c->todo = todo;
        c->extra = extra;
        c->it = it;
        c->count = count;
        c->last_cycles = count;
        c->cycles_total = total0 + count;
        c->active = 0;
        c->prev = prev;
        c->res_out = res_out;
        c->nan = (res_out != res_out);
    }
}

// The coarse part of a V-cycle -- levels l0 .. coarsest, smoothing,
// residuals, transfers and the dense coarsest solve -- in one cluster launch
// instead of one full-GPU launch per phase: these levels are small, and each
// of their phases is a launch latency long when issued on its own.
template <typename T>
__global__ void __launch_bounds__(kClThreads, 1) k_mg_coarse_cluster(pmg_args A, int l0) {
    cg::cluster_group cl = cg::this_cluster();
    const int t0 = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    const int ts = (int)cl.num_blocks() * blockDim.x;
    cl_vcycle<T>(A, cl, t0, ts, l0);
}

// the same for every running scene of a group: cluster b works on scene b
template <typename T>
__global__ void __launch_bounds__(kClThreads, 1) k_mg_coarse_cluster_b(const pmg_args *A, const int *run, int l0) {
    cg::cluster_group cl = cg::this_cluster();
    const int b = blockIdx.x / (int)cl.num_blocks();
    if (!run[b]) return;  // the whole cluster leaves together
    const int t0 = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    const int ts = (int)cl.num_blocks() * blockDim.x;
    cl_vcycle<T>(A[b], cl, t0, ts, l0);
}

static cudaError_t coarse_cluster_launch(const void *fn, void **args, int clusters, int csize, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(clusters * csize);
    cfg.blockDim = dim3(kClThreads);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = csize;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

// ---- host side -------------------------------------------------------------
int mg_solver::setup_cluster() {
    cluster_size = 0;
    if (cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    for (int c : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(kClThreads);
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_mg_cluster, &cfg) == cudaSuccess && n >= 1) {
            cluster_size = c;
            for (const void *fn : {(const void *)k_mg_coarse_cluster<double>, (const void *)k_mg_coarse_cluster<float>,
                                   (const void *)k_mg_coarse_cluster_b<double>,
                                   (const void *)k_mg_coarse_cluster_b<float>})
                if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
                    cudaGetLastError();
                    cluster_size = 0;
                }
            return 0;
        }
        cudaGetLastError();
    }
    return 0;
}

pmg_args level_args(const mg_solver &m) {
    pmg_args A;
    memset(&A, 0, sizeof(A));
    A.kind = (m.kind == MG_MAC) ? 0 : 1;
    A.nlev = (int)m.lv.size();
    for (int l = 0; l < A.nlev && l < kMaxLev; l++) {
        pmg_level &P = A.lv[l];
        for (int d = 0; d < 3; d++) {
            P.n[d] = m.lv[l].n[d];
            P.prd[d] = m.lv[l].prd[d];
        }
        P.x = m.lv[l].x;
        P.r = m.lv[l].r;
        P.res = m.lv[l].res;
        P.xs = m.lv[l].xs;
        P.rs = m.lv[l].rs;
        P.ress = m.lv[l].ress;
        P.ri = m.lv[l].ri;
        P.ris = m.lv[l].ris;
    }
    A.dense = m.dense;
    A.v_up = m.v_up;
    A.v_down = m.v_down;
    return A;
}

cudaError_t mg_solver::launch_cluster(cudaStream_t st) {
    cmg_args P;
    memset(&P, 0, sizeof(P));
    P.A = level_args(*this);
    P.tol = max_norm_tol;
    P.rtol = rtol;
    P.exact = exact ? 1 : 0;
    P.mixed = mixed ? 1 : 0;
    P.ctl = ctl;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster_size);
    cfg.blockDim = dim3(kClThreads);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cluster_size;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_mg_cluster, P);
}

}  // namespace rmt3d

namespace rmt3d {
cudaError_t coarse_cluster(const mg_solver &m, int l0, bool f32, cudaStream_t st) {
    pmg_args A = level_args(m);
    void *args[2] = {&A, &l0};
    return coarse_cluster_launch(f32 ? (const void *)k_mg_coarse_cluster<float> : (const void *)k_mg_coarse_cluster<double>,
                                 args, 1, m.cluster_size, st);
}

cudaError_t coarse_cluster_b(const pmg_args *A, const int *run, int B, int l0, int csize, bool f32, cudaStream_t st) {
    void *args[3] = {(void *)&A, (void *)&run, &l0};
    return coarse_cluster_launch(f32 ? (const void *)k_mg_coarse_cluster_b<float>
                                     : (const void *)k_mg_coarse_cluster_b<double>,
                                 args, B, csize, st);
}
}  // namespace rmt3d
