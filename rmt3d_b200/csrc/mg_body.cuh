// Bodies of the multigrid phase kernels, with the block coordinates passed
// in: the single-scene kernels (k_mg.cu) and the batched kernels that run a
// phase for every scene of a group in one launch (k_mgb.cu) call the same
// code, so a scene's solve gives the same bits alone and in a group.
#pragma once
#include <cuda_runtime.h>

#include "mg.h"
#include "mg_ops.cuh"

namespace rmt3d {

// ---- smoothing -------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void body_mac_rb(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int colour, const T *__restrict__ ri, int bx_, int by_, int bz_) {
    int hi = bx_ * blockDim.x + threadIdx.x;
    int j = by_ * blockDim.y + threadIdx.y;
    int k = bz_ * blockDim.z + threadIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    int i = 2 * hi + ((j + k + colour) & 1);
    if (i >= L.n0) return;
    T diag;
    T s = ri ? mac_offdiag_vd(L, x, ri, i, j, k, diag) : mac_offdiag(L, x, i, j, k, diag);
    int id = i + L.n0 * (j + L.n1 * k);
    x[id] = (r[id] - s) / diag;
}

// The Q1 stencil couples a node only to its edge and corner neighbours (the
// face entries are zero), so colouring by the parities of i and j alone never
// puts two coupled nodes in one colour: four colour passes are an exact
// Gauss-Seidel sweep.
template <typename T>
__device__ __forceinline__ void body_fem_gs(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int colour, const T *__restrict__ ri, int bx_, int by_, int bz_) {
    int i = 2 * (bx_ * blockDim.x + threadIdx.x) + (colour & 1);
    int j = 2 * (by_ * blockDim.y + threadIdx.y) + ((colour >> 1) & 1);
    int k = bz_ * blockDim.z + threadIdx.z;
    if (i >= L.n0 || j >= L.n1 || k >= L.n2) return;
    T diag;
    const int id = i + L.n0 * (j + L.n1 * k);
    if (ri) {
        const T s = fem_offdiag_vd(L, x, ri, i, j, k, diag);
        x[id] = (r[id] - s) / diag;
    } else {
        const T s = fem_offdiag(L, x, i, j, k, diag);
        x[id] = (r[id] - s) * fem_inv_diag<T>(L, i, j, k);
    }
}

// residual res = r - A x, and max |res| into *mx (as ordered bit pattern)
template <typename T, int KIND>
__device__ __forceinline__ double body_resid(lvl_dev L, const T *__restrict__ x, const T *__restrict__ r,
                                             T *__restrict__ res, const T *__restrict__ ri, int bx_, int by_,
                                             int bz_) {
    int i = bx_ * blockDim.x + threadIdx.x;
    int j = by_ * blockDim.y + threadIdx.y;
    int k = bz_ * blockDim.z + threadIdx.z;
    double a = 0;
    if (i < L.n0 && j < L.n1 && k < L.n2) {
        T diag;
        T s = op_offdiag<T>(KIND, L, x, ri, i, j, k, diag);
        int id = i + L.n0 * (j + L.n1 * k);
        T v = r[id] - s - diag * x[id];
        if (res) res[id] = v;
        a = fabs((double)v);
        if (a != a) a = __longlong_as_double(0x7ff8000000000000LL);
    }
    return a;
}

// The mixed form's FP64 residual handed to the FP32 cycle in one pass: the
// residual r - A x in FP64 (body_resid's expression), rounded to FP32 as the
// cycle's right-hand side, and the cycle's FP32 start value zeroed.
template <int KIND>
__device__ __forceinline__ void body_resid_to_f32(lvl_dev L, const double *__restrict__ x,
                                                  const double *__restrict__ r, const double *__restrict__ ri,
                                                  float *__restrict__ rs, float *__restrict__ xs, int bx_, int by_,
                                                  int bz_) {
    int i = bx_ * blockDim.x + threadIdx.x;
    int j = by_ * blockDim.y + threadIdx.y;
    int k = bz_ * blockDim.z + threadIdx.z;
    if (i >= L.n0 || j >= L.n1 || k >= L.n2) return;
    double diag;
    const double s = op_offdiag<double>(KIND, L, x, ri, i, j, k, diag);
    const int id = i + L.n0 * (j + L.n1 * k);
    const double v = r[id] - s - diag * x[id];
    rs[id] = (float)v;
    xs[id] = 0;
}

// max of a (non-negative, NaN sticky as the largest bit pattern) over the
// block's warps into *mx
__device__ __forceinline__ void warp_max_into(double a, unsigned long long *mx) {
    unsigned long long b = (unsigned long long)__double_as_longlong(a);
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
        b = t > b ? t : b;
    }
    if ((threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) % 32 == 0) atomicMax(mx, b);
}

// ---- grid transfer ---------------------------------------------------------
template <typename T>
__device__ __forceinline__ void body_mac_restrict(lvl_dev F, lvl_dev C, const T *__restrict__ res, T *__restrict__ rc,
                               T *__restrict__ xc0, int bx_, int by_, int bz_) {
    int I = bx_ * blockDim.x + threadIdx.x;
    int J = by_ * blockDim.y + threadIdx.y;
    int K = bz_ * blockDim.z + threadIdx.z;
    if (I >= C.n0 || J >= C.n1 || K >= C.n2) return;
    T s = 0;
    for (int c = 0; c < 2; c++)
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) s += res[(2 * I + a) + F.n0 * ((2 * J + b) + F.n1 * (2 * K + c))];
    rc[I + C.n0 * (J + C.n1 * K)] = (T)0.5 * s;
    xc0[I + C.n0 * (J + C.n1 * K)] = 0;
}

template <typename T>
__device__ __forceinline__ void body_mac_prolong(lvl_dev F, lvl_dev C, T *__restrict__ x, const T *__restrict__ xc, int bx_, int by_, int bz_) {
    int i = bx_ * blockDim.x + threadIdx.x;
    int j = by_ * blockDim.y + threadIdx.y;
    int k = bz_ * blockDim.z + threadIdx.z;
    if (i >= F.n0 || j >= F.n1 || k >= F.n2) return;
    const int f[3] = {i, j, k};
    const int nc[3] = {C.n0, C.n1, C.n2}, p[3] = {C.p0, C.p1, C.p2};
    int ci[3][2];
    T w[3][2];
    for (int d = 0; d < 3; d++) {
        int I = f[d] >> 1;
        int J = wrapi(I + ((f[d] & 1) ? 1 : -1), nc[d], p[d]);
        ci[d][0] = I;
        if (J < 0) {
            w[d][0] = 1;
            ci[d][1] = I;
            w[d][1] = 0;
        } else {
            w[d][0] = (T)0.75;
            ci[d][1] = J;
            w[d][1] = (T)0.25;
        }
    }
    T e = 0;
    for (int c = 0; c < 2; c++)
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                T wt = w[0][a] * w[1][b] * w[2][c];
                if (wt != 0) e += wt * xc[ci[0][a] + C.n0 * (ci[1][b] + C.n1 * ci[2][c])];
            }
    x[i + F.n0 * (j + F.n1 * k)] += e;
}

template <typename T>
__device__ __forceinline__ void body_fem_restrict(lvl_dev F, lvl_dev C, const T *__restrict__ res, T *__restrict__ rc,
                               T *__restrict__ xc0, int bx_, int by_, int bz_) {
    int I = bx_ * blockDim.x + threadIdx.x;
    int J = by_ * blockDim.y + threadIdx.y;
    int K = bz_ * blockDim.z + threadIdx.z;
    if (I >= C.n0 || J >= C.n1 || K >= C.n2) return;
    const int nf[3] = {F.n0, F.n1, F.n2}, p[3] = {F.p0, F.p1, F.p2};
    const int c[3] = {I, J, K};
    int idx[3][3];
    T w[3][3];
    for (int d = 0; d < 3; d++)
        for (int o = -1; o <= 1; o++) {
            int v = wrapi(2 * c[d] + o, nf[d], p[d]);
            idx[d][o + 1] = v;
            w[d][o + 1] = (v < 0) ? (T)0 : (o == 0 ? (T)1 : (T)0.5);
        }
    T s = 0;
    for (int oc = 0; oc < 3; oc++) {
        if (idx[2][oc] < 0) continue;
        for (int ob = 0; ob < 3; ob++) {
            if (idx[1][ob] < 0) continue;
            for (int oa = 0; oa < 3; oa++) {
                if (idx[0][oa] < 0) continue;
                s += w[0][oa] * w[1][ob] * w[2][oc] * res[idx[0][oa] + F.n0 * (idx[1][ob] + F.n1 * idx[2][oc])];
            }
        }
    }
    rc[I + C.n0 * (J + C.n1 * K)] = (T)0.5 * s;
    xc0[I + C.n0 * (J + C.n1 * K)] = 0;
}

template <typename T>
__device__ __forceinline__ void body_fem_prolong(lvl_dev F, lvl_dev C, T *__restrict__ x, const T *__restrict__ xc, int bx_, int by_, int bz_) {
    int i = bx_ * blockDim.x + threadIdx.x;
    int j = by_ * blockDim.y + threadIdx.y;
    int k = bz_ * blockDim.z + threadIdx.z;
    if (i >= F.n0 || j >= F.n1 || k >= F.n2) return;
    const int f[3] = {i, j, k};
    const int nc[3] = {C.n0, C.n1, C.n2}, p[3] = {C.p0, C.p1, C.p2};
    int ci[3][2];
    T w[3][2];
    int cnt[3];
    for (int d = 0; d < 3; d++) {
        if ((f[d] & 1) == 0) {
            ci[d][0] = f[d] >> 1;
            w[d][0] = 1;
            cnt[d] = 1;
        } else {
            ci[d][0] = f[d] >> 1;
            ci[d][1] = wrapi((f[d] >> 1) + 1, nc[d], p[d]);
            w[d][0] = w[d][1] = (T)0.5;
            cnt[d] = 2;
        }
    }
    T e = 0;
    for (int c = 0; c < cnt[2]; c++)
        for (int b = 0; b < cnt[1]; b++)
            for (int a = 0; a < cnt[0]; a++)
                e += w[0][a] * w[1][b] * w[2][c] * xc[ci[0][a] + C.n0 * (ci[1][b] + C.n1 * ci[2][c])];
    x[i + F.n0 * (j + F.n1 * k)] += e;
}

// coarsest grid: x = B r with the precomputed dense inverse B (row-major)
template <typename T>
__device__ __forceinline__ void body_coarse_dense(int np, const double *__restrict__ B, T *__restrict__ x,
                                                  const T *__restrict__ r, int bx_, int gx_) {
    __shared__ double rs[1024];
    for (int p = threadIdx.x; p < np; p += blockDim.x) rs[p] = (double)r[p];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int row = bx_ * (blockDim.x >> 5) + warp; row < np; row += gx_ * (blockDim.x >> 5)) {
        const double *b = B + (size_t)row * np;
        double acc = 0;
        for (int c = lane; c < np; c += 32) acc += b[c] * rs[c];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[row] = (T)acc;
    }
}

// coarsest grid fallback: many Gauss-Seidel sweeps inside one thread block
template <typename T, int KIND>
__device__ __forceinline__ void body_coarse_solve(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int sweeps) {
    const int np = L.n0 * L.n1 * L.n2;
    for (int p = threadIdx.x; p < np; p += blockDim.x) x[p] = 0;
    __syncthreads();
    const int ncol = (KIND == 0) ? 2 : 8;
    for (int s = 0; s < sweeps; s++)
        for (int col = 0; col < ncol; col++) {
            for (int p = threadIdx.x; p < np; p += blockDim.x) {
                int i = p % L.n0, j = (p / L.n0) % L.n1, k = p / (L.n0 * L.n1);
                int my = (KIND == 0) ? ((i + j + k) & 1) : ((i & 1) | ((j & 1) << 1) | ((k & 1) << 2));
                if (my != col) continue;
                T diag;
                T sum = (KIND == 0) ? mac_offdiag(L, x, i, j, k, diag) : fem_offdiag(L, x, i, j, k, diag);
                x[p] = (r[p] - sum) / diag;
            }
            __syncthreads();
        }
}

// FP64 <-> FP32 helpers of the mixed form
__device__ __forceinline__ void body_to_f32(const double *__restrict__ a, float *__restrict__ b, size_t n, int bx_) {
    size_t i = bx_ * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}
__device__ __forceinline__ void body_add_f32(double *__restrict__ a, const float *__restrict__ b, size_t n, int bx_) {
    size_t i = bx_ * (size_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] += (double)b[i];
}
template <typename T>
__device__ __forceinline__ void body_zero(T *a, size_t n, int bx_) {
    size_t i = bx_ * (size_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0;
}


// ---- the control of one solve (mg_prob::run, Utilities/mg_probs.cc:3-83) ---
__device__ __forceinline__ void mg_begin_state(mg_ctl *c, unsigned long long *mx) {
    c->phase = 0;
    c->todo = c->iV / kMgIP;
    if (c->todo < 1) c->todo = 1;
    c->extra = 0;
    c->it = 0;
    c->count = 0;
    c->active = 1;
    c->need_res = c->todo == 1;
    mx[0] = 0;
    mx[1] = 0;
}

// One step of the control after an iteration, with the fine-level max-norm
// residual in mx[0] (and max |rhs| in mx[1] for the relative tolerance);
// returns true when the solve is finished (the predictor is then updated).
__device__ __forceinline__ bool mg_ctl_step(mg_ctl *c, unsigned long long *mx, double tol, double rtol, int exact) {
    const double r = __longlong_as_double((long long)mx[0]);
    mx[0] = 0;
    // the mixed form's relative tolerance (mixed_rtol x max |rhs|)
    const double rhs = __longlong_as_double((long long)mx[1]);
    const double tol_eff = (rtol > 0 && rtol * rhs > tol) ? rtol * rhs : tol;
    c->count++;
    c->cycles_total++;
    bool done = false;
    if (c->phase <= 1) {
        if (--c->todo <= 0) {
            c->res_out = r;
            if (r > tol_eff && c->extra < 20) {
                c->extra++;
                c->todo = c->extra;
                c->phase = 1;
            } else if (rtol > 0 && !exact) {
                done = true;  // the relaxed form skips the insurance cycles
            } else {
                c->phase = 2;
                c->todo = 2;
            }
        }
    } else if (c->phase == 2) {
        if (--c->todo <= 0) {
            if (exact) {
                c->prev = 1e300;
                c->res_out = r;
                c->it = 0;
                if (r > 0 && r < 0.7 * c->prev) c->phase = 3;
                else done = true;
            } else {
                done = true;
            }
        }
    } else {
        c->prev = c->res_out;
        c->res_out = r;
        c->it++;
        if (!(c->it < 60 && r > 0 && r < 0.7 * c->prev)) done = true;
    }
    if (c->count >= kMgMaxCycles) done = true;
    if (done) {
        // mg_pred::update (alpha = 0)
        const double alpha = 1 / (3 * kMgIP);
        double dV = c->iV - c->V_avg;
        int exreduce = static_cast<int>(dV / sqrt(c->V_var));
        exreduce = exreduce > 0 ? exreduce : 0;
        c->iV += kMgIP * c->extra * (c->extra + 1) / 2 - 1 - exreduce;
        if (c->iV < kMgIP) c->iV = 2 * kMgIP - 1;
        c->V_avg = (1 - alpha) * c->V_avg + alpha * c->iV;
        c->V_var = (1 - alpha) * (c->V_var + alpha * dV * dV);
        c->last_cycles = c->count;
        c->active = 0;
        c->nan = (c->res_out != c->res_out);
    }
    // the residual is read only where a phase ends (and every cycle of the
    // stagnation loop): the next iteration computes it only then
    c->need_res = (c->phase <= 1 && c->todo == 1) || (c->phase == 2 && c->todo == 1 && exact) || c->phase == 3;
    return done;
}

}  // namespace rmt3d
