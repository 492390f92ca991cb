// Persistent multigrid solve (opt-in, RMT3D_MG_PERSISTENT=1): one cooperative
// launch runs a whole Poisson
// solve with the reference's control logic on the device (mg_prob::run,
// Utilities/mg_probs.cc:3-83, with mg_pred, mg_probs.hh:37-78): the predicted
// number of V-cycles, extra rounds of 1, 2, 3, ... cycles while the max-norm
// residual is above the tolerance (at most 20 rounds), two insurance cycles
// and the predictor update.
//
// Levels with more than kCoarsePts points are processed by every CTA with
// grid-stride loops, one phase at a time, separated by a grid barrier; the
// remaining coarse levels -- a few thousand points -- run inside CTA 0 with
// block-level synchronisation only.  The grid barrier spins with a bounded
// iteration count: on timeout it raises an error flag and every CTA returns.
// The launch is cooperative, so all CTAs are co-resident.
#include <cooperative_groups.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "host_common.h"
#include "mg.h"
#include "mg_ops.cuh"
#include "rmt3d_gpu.h"

namespace rmt3d {

// bounded grid barrier (all CTAs co-resident: cooperative launch)
__device__ bool grid_bar(const pmg_args &A) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = A.bar + 1;
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(A.bar, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(A.bar, 0u);
            __threadfence();
            atomicAdd((unsigned *)(A.bar + 1), 1u);
        } else {
            long long it = 0;
            while (*gen == g) {
                if (++it > (1LL << 24)) {
                    atomicExch(A.err, 1);
                    break;
                }
                __nanosleep(40);
            }
        }
        __threadfence();
        ok = (*(volatile int *)A.err == 0);
    }
    __syncthreads();
    return ok != 0;
}

// one V-cycle over all levels; false if a barrier timed out
template <typename T>
__device__ bool vcycle(const pmg_args &A) {
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;
    const int nc = A.kind == 0 ? 2 : 4;
    const int cf = A.cf;
    for (int l = 0; l < cf; l++) {
        const pmg_level &F = A.lv[l];
        for (int s = 0; s < A.v_down; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), c, t0, ts);
                if (!grid_bar(A)) return false;
            }
        ph_resid<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LS<T>(F), t0, ts);
        if (!grid_bar(A)) return false;
        const pmg_level &C = A.lv[l + 1];
        ph_restrict<T>(A.kind, ldev(F), ldev(C), LS<T>(F), LR<T>(C), LX<T>(C), t0, ts);
        if (!grid_bar(A)) return false;
    }
    if (blockIdx.x == 0) coarse_cycle<T>(A, cf);
    if (!grid_bar(A)) return false;
    for (int l = cf - 1; l >= 0; l--) {
        const pmg_level &F = A.lv[l];
        const pmg_level &C = A.lv[l + 1];
        ph_prolong<T>(A.kind, ldev(F), ldev(C), LX<T>(F), LX<T>(C), t0, ts);
        if (!grid_bar(A)) return false;
        for (int s = 0; s < A.v_up; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), c, t0, ts);
                if (!grid_bar(A)) return false;
            }
    }
    return true;
}

// one iteration: a plain FP64 V-cycle, or in the mixed form one refinement
// step (FP64 residual, FP32 V-cycle on the correction, FP64 update)
__device__ bool iterate(const pmg_args &A) {
    if (!A.mixed) return vcycle<double>(A);
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;
    const pmg_level &L = A.lv[0];
    const int tot = L.n[0] * L.n[1] * L.n[2];
    ph_resid<double>(A.kind, ldev(L), L.x, L.r, L.res, t0, ts);
    if (!grid_bar(A)) return false;
    for (int t = t0; t < tot; t += ts) {
        L.rs[t] = (float)L.res[t];
        L.xs[t] = 0;
    }
    if (!grid_bar(A)) return false;
    if (!vcycle<float>(A)) return false;
    for (int t = t0; t < tot; t += ts) L.x[t] += (double)L.xs[t];
    return grid_bar(A);
}

// max-norm residual of the finest level, identical in every CTA
__device__ bool resmax(const pmg_args &A, double &out) {
    __shared__ double red[kThreads / 32];
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, ts = gridDim.x * blockDim.x;
    const pmg_level &L = A.lv[0];
    double m = ph_resid<double>(A.kind, ldev(L), L.x, L.r, nullptr, t0, ts);
    for (int o = 16; o > 0; o >>= 1) {
        double v = __shfl_xor_sync(0xffffffffu, m, o);
        if (v != v || v > m) m = v;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++)
            if (red[w] != red[w] || red[w] > b) b = red[w];
        A.partial[blockIdx.x] = b;
    }
    if (!grid_bar(A)) return false;
    double g = 0;
    for (unsigned b = 0; b < gridDim.x; b++) {
        double v = ((volatile double *)A.partial)[b];
        if (v != v || v > g) g = v;
    }
    out = g;
    return true;
}

__global__ void __launch_bounds__(kThreads) k_mg_solve(pmg_args A) {
    const int hard_cap = 20;
    int cycles = 0;
    const int iV = *(volatile int *)A.pred_iV;
    const int iters = iV / 16;
    for (int i = 0; i < iters; i++) {
        if (!iterate(A)) return;
        cycles++;
    }
    double res;
    if (!resmax(A, res)) return;
    int extra = 0;
    while (res > A.tol && extra < hard_cap) {
        extra++;
        for (int n = 0; n < extra; n++) {
            if (!iterate(A)) return;
            cycles++;
        }
        if (!resmax(A, res)) return;
    }
    for (int i = 0; i < 2; i++) {
        if (!iterate(A)) return;
        cycles++;
    }
    if (A.exact) {
        double prev = 1e300;
        if (!resmax(A, res)) return;
        for (int it = 0; it < 60 && res > 0 && res < 0.7 * prev; it++) {
            if (!iterate(A)) return;
            cycles++;
            prev = res;
            if (!resmax(A, res)) return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // mg_pred::update(extras), alpha = 0 (mg_probs.hh:51-66)
        double avg = *A.pred_avg, var = *A.pred_var;
        double dV = iV - avg;
        int exreduce = static_cast<int>(dV / sqrt(var));
        exreduce = exreduce > 0 ? exreduce : 0;
        int nv = iV + 16 * extra * (extra + 1) / 2 - 1 - exreduce;
        if (nv < 16) nv = 2 * 16 - 1;
        *A.pred_iV = nv;
        A.out[0] = res;
        A.out[1] = cycles;
        A.out[2] = extra;
    }
}

// ---- host side -------------------------------------------------------------
int mg_solver::setup_persistent(cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_mg_solve, kThreads, 0);
    if (occ < 1) return fail(RMT3D_ERR_CUDA, "persistent multigrid kernel cannot be resident");
    size_t fine = lv[0].npts();
    int want = (int)((fine / 4 + kThreads - 1) / kThreads);
    int cap = prop.multiProcessorCount;  // one CTA per SM keeps the grid barrier cheap
    pgrid = want < cap ? want : cap;
    if (pgrid < 1) pgrid = 1;
    if (cudaMalloc(&pstate, 64 * sizeof(double) + (size_t)pgrid * sizeof(double)) != cudaSuccess)
        return fail(RMT3D_ERR_OOM, "multigrid state allocation failed");
    cudaMemsetAsync(pstate, 0, 64 * sizeof(double) + (size_t)pgrid * sizeof(double), st);
    // predictor initial state: iV = 32, V_avg = 32, V_var = 1e6
    int iv = 32;
    double av = 32, vv = 1e6;
    char *b = (char *)pstate;
    cudaMemcpyAsync(b + 0, &iv, sizeof(int), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b + 8, &av, sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b + 16, &vv, sizeof(double), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    return 0;
}

double mg_solver::run_persistent(cudaStream_t st) {
    pmg_args A;
    memset(&A, 0, sizeof(A));
    A.kind = (kind == MG_MAC) ? 0 : 1;
    A.nlev = (int)lv.size();
    if (A.nlev > kMaxLev) return NAN;
    A.cf = A.nlev - 1;
    for (int l = 0; l < A.nlev; l++)
        if (lv[l].npts() <= (size_t)kCoarsePts) {
            A.cf = l;
            break;
        }
    for (int l = 0; l < A.nlev; l++) {
        pmg_level &P = A.lv[l];
        for (int d = 0; d < 3; d++) {
            P.n[d] = lv[l].n[d];
            P.prd[d] = lv[l].prd[d];
        }
        P.x = lv[l].x;
        P.r = lv[l].r;
        P.res = lv[l].res;
        P.xs = lv[l].xs;
        P.rs = lv[l].rs;
        P.ress = lv[l].ress;
    }
    A.dense = dense;
    A.tol = max_norm_tol;
    A.v_up = v_up;
    A.v_down = v_down;
    A.exact = exact ? 1 : 0;
    A.mixed = mixed ? 1 : 0;
    char *b = (char *)pstate;
    A.pred_iV = (int *)(b + 0);
    A.pred_avg = (double *)(b + 8);
    A.pred_var = (double *)(b + 16);
    A.bar = (unsigned *)(b + 24);
    A.err = (int *)(b + 32);
    A.out = (double *)(b + 40);
    A.partial = (double *)(b + 64 * sizeof(double));
    void *args[] = {&A};
    cudaError_t e = cudaLaunchCooperativeKernel((void *)k_mg_solve, dim3(pgrid), dim3(kThreads), args, 0, st);
    if (launches) (*launches)++;
    if (e != cudaSuccess) {
        hard_error = true;
        fail(RMT3D_ERR_CUDA, std::string("cooperative multigrid launch: ") + cudaGetErrorString(e));
        return NAN;
    }
    double out[3];
    int err = 0;
    cudaMemcpyAsync(out, A.out, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&err, A.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if (err) {
        hard_error = true;
        fail(RMT3D_ERR_CUDA, "multigrid grid barrier timed out");
        return NAN;
    }
    last_cycles = (int)out[1];
    cycles_total += last_cycles;
    return out[0];
}

}  // namespace rmt3d
