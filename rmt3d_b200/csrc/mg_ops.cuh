// Multigrid operator helpers of the V-cycle kernels (k_mg.cu): rediscretised
// MAC 7-point and FEM Q1 27-point stencils with the boundary rules of
// stencil_set::set_partials (Utilities/mg_probs.hh:281-343), and the phases of
// the one-block coarse sub-cycle.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace rmt3d {

struct lvl_dev {
    int n0, n1, n2;
    int p0, p1, p2;
};

__host__ __device__ __forceinline__ int wrapi(int v, int n, int prd) {
    if (v < 0) return prd ? v + n : -1;
    if (v >= n) return prd ? v - n : -1;
    return v;
}

// v / num for num in {1, 2, 4, 8} as an exact power-of-two scaling (the same
// bits as the division, without its instruction sequence)
template <typename T>
__device__ __forceinline__ T div_pow2(T v, int num) {
    return num == 1 ? v : num == 2 ? v * (T)0.5 : num == 4 ? v * (T)0.25 : num == 8 ? v * (T)0.125 : v / (T)num;
}

// ---- operator application -------------------------------------------------
template <typename T>
__device__ __forceinline__ T mac_offdiag(const lvl_dev L, const T *__restrict__ x, int i, int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        const int sy = L.n0, sz = L.n0 * L.n1;
        const T *c = x + i + sy * j + sz * k;
        diag = (T)-6;
        return ((c[-1] + c[1]) + (c[-sy] + c[sy])) + (c[-sz] + c[sz]);
    }
    T s = 0;
    int missing = 0;
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
    const int st[3] = {1, L.n0, L.n0 * L.n1};
    const int base = i + L.n0 * (j + L.n1 * k);
    for (int d = 0; d < 3; d++) {
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            int v = wrapi(c[d] + sgn, n[d], p[d]);
            if (v < 0) {
                missing++;
                continue;
            }
            s += x[base + (v - c[d]) * st[d]];
        }
    }
    diag = (T)(-6 + missing);
    return s;
}

template <typename T>
__device__ __forceinline__ T fem_offdiag(const lvl_dev L, const T *__restrict__ x, int i, int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        // interior node: edges -2, corners -1, faces 0
        const int sy = L.n0, sz = L.n0 * L.n1;
        const T *c = x + i + sy * j + sz * k;
        const T *zm = c - sz, *zp = c + sz;
        T e = (c[-1 - sy] + c[1 - sy]) + (c[-1 + sy] + c[1 + sy]);
        e += (zm[-1] + zm[1]) + (zm[-sy] + zm[sy]);
        e += (zp[-1] + zp[1]) + (zp[-sy] + zp[sy]);
        T q = (zm[-1 - sy] + zm[1 - sy]) + (zm[-1 + sy] + zm[1 + sy]);
        q += (zp[-1 - sy] + zp[1 - sy]) + (zp[-1 + sy] + zp[1 + sy]);
        diag = (T)32;
        return (T)-2 * e - q;
    }
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
    bool bd[3];
    for (int d = 0; d < 3; d++) bd[d] = !p[d] && (c[d] == 0 || c[d] == n[d] - 1);
    int nb[3][3];
    for (int d = 0; d < 3; d++)
        for (int o = -1; o <= 1; o++) nb[d][o + 1] = wrapi(c[d] + o, n[d], p[d]);
    T s = 0;
    for (int oc = 0; oc < 3; oc++) {
        int kk = nb[2][oc];
        if (kk < 0) continue;
        for (int ob = 0; ob < 3; ob++) {
            int jj = nb[1][ob];
            if (jj < 0) continue;
            const T *row = x + (size_t)L.n0 * (jj + (size_t)L.n1 * kk);
            for (int oa = 0; oa < 3; oa++) {
                int ii = nb[0][oa];
                if (ii < 0) continue;
                int nz = (oa != 1) + (ob != 1) + (oc != 1);
                if (nz == 0 || nz == 1) continue;  // centre handled below, faces are 0
                T co = (nz == 2) ? (T)-2 : (T)-1;
                int halve = (bd[0] && oa == 1) + (bd[1] && ob == 1) + (bd[2] && oc == 1);
                if (halve == 1) co *= (T)0.5;
                else if (halve == 2) co *= (T)0.25;
                s += co * row[ii];
            }
        }
    }
    int hc = bd[0] + bd[1] + bd[2];
    diag = (T)32 / (T)(1 << hc);
    return s;
}


// 1 / diag of the constant-density FEM stencil at node (i, j, k).  diag is
// 32 / 2^h, h the number of walled axes on whose end planes the node lies,
// so the reciprocal 2^h / 32 is exact and (r - s) times it has the same bits
// as (r - s) / diag, without a division's instruction sequence.
template <typename T>
__device__ __forceinline__ T fem_inv_diag(const lvl_dev L, int i, int j, int k) {
    const int h = (!L.p0 && (i == 0 || i == L.n0 - 1)) + (!L.p1 && (j == 0 || j == L.n1 - 1)) +
                  (!L.p2 && (k == 0 || k == L.n2 - 1));
    return (T)(1 << h) * (T)0.03125;
}

// ---- variable density (VAR_DEN) ---------------------------------------------
// ri: 1/rho per cell of the level (cell-centred, MAC level dimensions; for a
// FEM level with n nodes per axis there are n-1 cells on a walled axis and n
// on a periodic one).  Coarse levels carry the mean of their 8 children.

// var_den_mac::set_stencils (Utilities/mg_probs.cc:196-308): each face
// coefficient is the mean of 1/rho of the two cells it joins; the centre is
// the (Neumann-fixed) centre entry times the mean of the face coefficients,
// accumulated direction by direction as the reference does.
template <typename T>
__device__ __forceinline__ T mac_offdiag_vd(const lvl_dev L, const T *__restrict__ x, const T *__restrict__ ri, int i,
                                            int j, int k, T &diag) {
    const int base = i + L.n0 * (j + L.n1 * k);
    const T rc = ri[base];
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        // interior cell: all six faces, the same operations in the same order
        const int sy = L.n0, sz = L.n0 * L.n1;
        const T ax1 = (T)0.5 * (ri[base - 1] + rc), ax2 = (T)0.5 * (rc + ri[base + 1]);
        const T ay1 = (T)0.5 * (ri[base - sy] + rc), ay2 = (T)0.5 * (rc + ri[base + sy]);
        const T az1 = (T)0.5 * (ri[base - sz] + rc), az2 = (T)0.5 * (rc + ri[base + sz]);
        T s = 0, csum = 0;
        s += ax1 * x[base - 1] + ax2 * x[base + 1];
        csum += ax1 + ax2;
        s += ay1 * x[base - sy] + ay2 * x[base + sy];
        csum += ay1 + ay2;
        s += az1 * x[base - sz] + az2 * x[base + sz];
        csum += az1 + az2;
        diag = (T)(-6) * (csum / (T)6);
        return s;
    }
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
    const int st[3] = {1, L.n0, L.n0 * L.n1};
    T s = 0, csum = 0;
    int cnt = 0;
    for (int d = 0; d < 3; d++) {
        const int lo = wrapi(c[d] - 1, n[d], p[d]), hi = wrapi(c[d] + 1, n[d], p[d]);
        const int il = base + (lo - c[d]) * st[d], ih = base + (hi - c[d]) * st[d];
        if (lo >= 0 && hi >= 0) {
            const T a1 = (T)0.5 * (ri[il] + rc), a2 = (T)0.5 * (rc + ri[ih]);
            s += a1 * x[il] + a2 * x[ih];
            csum += a1 + a2;
            cnt += 2;
        } else if (lo >= 0) {
            const T a1 = (T)0.5 * (ri[il] + rc);
            s += a1 * x[il];
            csum += a1;
            cnt += 1;
        } else if (hi >= 0) {
            const T a2 = (T)0.5 * (rc + ri[ih]);
            s += a2 * x[ih];
            csum += a2;
            cnt += 1;
        }
    }
    diag = (T)(-cnt) * (csum / (T)cnt);
    return s;
}

// var_den_fem::set_stencils (Utilities/mg_probs.cc:97-150): every entry of the
// (boundary-halved) Q1 stencil is scaled by the mean of 1/rho over the cells
// adjacent to both the node and that neighbour -- 1 cell for a corner
// neighbour, 2 for an edge neighbour, all (up to 8) for the centre -- summed
// in the reference's cell order.
template <typename T>
__device__ __forceinline__ T fem_offdiag_vd(const lvl_dev L, const T *__restrict__ x, const T *__restrict__ ri, int i,
                                            int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        // interior node (all 8 cells exist, no halving): corners take one
        // cell, edges the mean of two (lower index first), the centre the
        // mean of all eight in (z, y, x) order; the means multiply by 1/2 and
        // 1/8, the same bits as the divisions without their instruction
        // sequences
        const int sy = L.n0, sz = L.n0 * L.n1;
        const int ncx = L.p0 ? L.n0 : L.n0 - 1, ncy = L.p1 ? L.n1 : L.n1 - 1;
        const int c0 = (i - 1) + ncx * ((j - 1) + ncy * (k - 1));  // cell below-left-front
        const int cy = ncx, cz = ncx * ncy;
        T v[2][2][2];
        v[0][0][0] = ri[c0];
        v[0][0][1] = ri[c0 + 1];
        v[0][1][0] = ri[c0 + cy];
        v[0][1][1] = ri[c0 + cy + 1];
        v[1][0][0] = ri[c0 + cz];
        v[1][0][1] = ri[c0 + cz + 1];
        v[1][1][0] = ri[c0 + cz + cy];
        v[1][1][1] = ri[c0 + cz + cy + 1];
        const T *xc = x + i + sy * j + sz * k;
        T s = 0;
#pragma unroll
        for (int oc = 0; oc < 3; oc++)
#pragma unroll
            for (int ob = 0; ob < 3; ob++)
#pragma unroll
                for (int oa = 0; oa < 3; oa++) {
                    const int nz = (oa != 1) + (ob != 1) + (oc != 1);
                    if (nz <= 1) continue;
                    const T xv = xc[(oa - 1) + sy * (ob - 1) + sz * (oc - 1)];
                    T cf;
                    if (nz == 3) {
                        cf = -v[oc >> 1][ob >> 1][oa >> 1];
                    } else if (oc == 1) {
                        cf = (T)-2 * ((v[0][ob >> 1][oa >> 1] + v[1][ob >> 1][oa >> 1]) * (T)0.5);
                    } else if (ob == 1) {
                        cf = (T)-2 * ((v[oc >> 1][0][oa >> 1] + v[oc >> 1][1][oa >> 1]) * (T)0.5);
                    } else {
                        cf = (T)-2 * ((v[oc >> 1][ob >> 1][0] + v[oc >> 1][ob >> 1][1]) * (T)0.5);
                    }
                    s += cf * xv;
                }
        T c8 = 0;
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int e = 0; e < 2; e++) c8 += v[a][b][e];
        diag = (T)32 * (c8 * (T)0.125);
        return s;
    }
    // boundary or wrapped node; every loop below unrolls to constant indices
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int nc[3] = {p[0] ? n[0] : n[0] - 1, p[1] ? n[1] : n[1] - 1, p[2] ? n[2] : n[2] - 1};
    const int c[3] = {i, j, k};
    int cell[3][2];  // cells below / above the node on each axis (-1: none)
    bool bd[3];
    int nb[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bd[d] = !p[d] && (c[d] == 0 || c[d] == n[d] - 1);
        cell[d][0] = (c[d] - 1 >= 0) ? c[d] - 1 : (p[d] ? c[d] - 1 + nc[d] : -1);
        cell[d][1] = (c[d] < nc[d]) ? c[d] : (p[d] ? c[d] - nc[d] : -1);
#pragma unroll
        for (int o = -1; o <= 1; o++) nb[d][o + 1] = wrapi(c[d] + o, n[d], p[d]);
    }
    // the up to 8 adjacent cells' 1/rho, [cz][cy][cx]
    T v[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const bool ok = cell[0][e] >= 0 && cell[1][b] >= 0 && cell[2][a] >= 0;
                v[a][b][e] = ok ? ri[cell[0][e] + nc[0] * (cell[1][b] + nc[1] * cell[2][a])] : (T)0;
            }
    T s = 0;
#pragma unroll
    for (int oc = 0; oc < 3; oc++) {
#pragma unroll
        for (int ob = 0; ob < 3; ob++) {
#pragma unroll
            for (int oa = 0; oa < 3; oa++) {
                const int nz = (oa != 1) + (ob != 1) + (oc != 1);
                if (nz <= 1) continue;  // centre handled below, faces are 0
                const int kk = nb[2][oc], jj = nb[1][ob], ii = nb[0][oa];
                if (kk < 0 || jj < 0 || ii < 0) continue;
                T co = (nz == 2) ? (T)-2 : (T)-1;
                const int halve = (bd[0] && oa == 1) + (bd[1] && ob == 1) + (bd[2] && oc == 1);
                if (halve == 1) co *= (T)0.5;
                else if (halve == 2) co *= (T)0.25;
                // cells shared by the node and this neighbour, in (z, y, x) order
                T sum = 0;
                int num = 0;
#pragma unroll
                for (int a = (oc == 2 ? 1 : 0); a <= (oc == 0 ? 0 : 1); a++)
#pragma unroll
                    for (int b = (ob == 2 ? 1 : 0); b <= (ob == 0 ? 0 : 1); b++)
#pragma unroll
                        for (int e = (oa == 2 ? 1 : 0); e <= (oa == 0 ? 0 : 1); e++)
                            if (cell[2][a] >= 0 && cell[1][b] >= 0 && cell[0][e] >= 0) {
                                sum += v[a][b][e];
                                num++;
                            }
                s += co * div_pow2(sum, num) * x[ii + L.n0 * (jj + L.n1 * kk)];
            }
        }
    }
    T sum = 0;
    int num = 0;
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 0; e < 2; e++)
                if (cell[2][a] >= 0 && cell[1][b] >= 0 && cell[0][e] >= 0) {
                    sum += v[a][b][e];
                    num++;
                }
    const int hc = bd[0] + bd[1] + bd[2];
    diag = ((T)32 / (T)(1 << hc)) * div_pow2(sum, num);
    return s;
}

template <typename T>
__device__ __forceinline__ T op_offdiag(int kind, const lvl_dev L, const T *__restrict__ x, const T *__restrict__ ri,
                                        int i, int j, int k, T &diag) {
    if (ri) return kind == 0 ? mac_offdiag_vd(L, x, ri, i, j, k, diag) : fem_offdiag_vd(L, x, ri, i, j, k, diag);
    return kind == 0 ? mac_offdiag(L, x, i, j, k, diag) : fem_offdiag(L, x, i, j, k, diag);
}

constexpr int kMaxLev = 12;
constexpr int kDensePts = 1000;  // coarsening stops at the first level with at most this many points
constexpr int kDenseMax = 1024;  // largest level solved by a dense inverse
constexpr int kThreads = 256;

struct pmg_level {
    int n[3];
    int prd[3];
    double *x, *r, *res;
    float *xs, *rs, *ress;
    const double *ri;  // variable density: 1/rho per cell (null: constant)
    const float *ris;
};

struct pmg_args {
    int kind;  // 0 MAC, 1 FEM
    int nlev;
    pmg_level lv[kMaxLev];
    const double *dense;  // inverse of the coarsest operator, or null
    int v_up, v_down;
};

__device__ __forceinline__ lvl_dev ldev(const pmg_level &L) {
    return lvl_dev{L.n[0], L.n[1], L.n[2], L.prd[0], L.prd[1], L.prd[2]};
}

// ---- one phase over a level, for the points [t0, total) with stride ts ----
template <typename T>
__device__ void ph_smooth_colour(int kind, const lvl_dev L, T *x, const T *r, const T *ri, int colour, int t0, int ts) {
    if (kind == 0) {
        const int h = (L.n0 + 1) / 2;
        const int tot = h * L.n1 * L.n2;
        for (int t = t0; t < tot; t += ts) {
            int hi = t % h, j = (t / h) % L.n1, k = t / (h * L.n1);
            int i = 2 * hi + ((j + k + colour) & 1);
            if (i >= L.n0) continue;
            T diag;
            T s = op_offdiag<T>(0, L, x, ri, i, j, k, diag);
            int id = i + L.n0 * (j + L.n1 * k);
            x[id] = (r[id] - s) / diag;
        }
    } else {
        const int ha = (L.n0 + 1) / 2, hb = (L.n1 + 1) / 2;
        const int tot = ha * hb * L.n2;
        for (int t = t0; t < tot; t += ts) {
            int a = t % ha, b = (t / ha) % hb, k = t / (ha * hb);
            int i = 2 * a + (colour & 1), j = 2 * b + ((colour >> 1) & 1);
            if (i >= L.n0 || j >= L.n1) continue;
            T diag;
            T s = op_offdiag<T>(1, L, x, ri, i, j, k, diag);
            int id = i + L.n0 * (j + L.n1 * k);
            x[id] = (r[id] - s) / diag;
        }
    }
}

template <typename T>
__device__ double ph_resid(int kind, const lvl_dev L, const T *x, const T *r, T *res, const T *ri, int t0, int ts) {
    const int tot = L.n0 * L.n1 * L.n2;
    double mx = 0;
    for (int t = t0; t < tot; t += ts) {
        int i = t % L.n0, j = (t / L.n0) % L.n1, k = t / (L.n0 * L.n1);
        T diag;
        T s = op_offdiag<T>(kind, L, x, ri, i, j, k, diag);
        T v = r[t] - s - diag * x[t];
        if (res) res[t] = v;
        double a = fabs((double)v);
        if (a != a || a > mx) mx = a;  // NaN sticks
    }
    return mx;
}

template <typename T>
__device__ void ph_restrict(int kind, const lvl_dev F, const lvl_dev C, const T *res, T *rc, T *xc, int t0, int ts) {
    const int tot = C.n0 * C.n1 * C.n2;
    for (int t = t0; t < tot; t += ts) {
        int I = t % C.n0, J = (t / C.n0) % C.n1, K = t / (C.n0 * C.n1);
        T s = 0;
        if (kind == 0) {
            for (int c = 0; c < 2; c++)
                for (int b = 0; b < 2; b++)
                    for (int a = 0; a < 2; a++) s += res[(2 * I + a) + F.n0 * ((2 * J + b) + F.n1 * (2 * K + c))];
        } else {
            const int nf[3] = {F.n0, F.n1, F.n2}, p[3] = {F.p0, F.p1, F.p2};
            const int cc[3] = {I, J, K};
            int idx[3][3];
            T w[3][3];
            for (int d = 0; d < 3; d++)
                for (int o = -1; o <= 1; o++) {
                    int v = wrapi(2 * cc[d] + o, nf[d], p[d]);
                    idx[d][o + 1] = v;
                    w[d][o + 1] = (v < 0) ? (T)0 : (o == 0 ? (T)1 : (T)0.5);
                }
            for (int oc = 0; oc < 3; oc++) {
                if (idx[2][oc] < 0) continue;
                for (int ob = 0; ob < 3; ob++) {
                    if (idx[1][ob] < 0) continue;
                    for (int oa = 0; oa < 3; oa++) {
                        if (idx[0][oa] < 0) continue;
                        s += w[0][oa] * w[1][ob] * w[2][oc] *
                             res[idx[0][oa] + F.n0 * (idx[1][ob] + F.n1 * idx[2][oc])];
                    }
                }
            }
        }
        rc[t] = (T)0.5 * s;
        xc[t] = 0;
    }
}

template <typename T>
__device__ void ph_prolong(int kind, const lvl_dev F, const lvl_dev C, T *x, const T *xc, int t0, int ts) {
    const int tot = F.n0 * F.n1 * F.n2;
    const int nc[3] = {C.n0, C.n1, C.n2}, p[3] = {C.p0, C.p1, C.p2};
    for (int t = t0; t < tot; t += ts) {
        int i = t % F.n0, j = (t / F.n0) % F.n1, k = t / (F.n0 * F.n1);
        const int f[3] = {i, j, k};
        int ci[3][2];
        T w[3][2];
        int cnt[3];
        for (int d = 0; d < 3; d++) {
            if (kind == 0) {
                int I = f[d] >> 1;
                int J = wrapi(I + ((f[d] & 1) ? 1 : -1), nc[d], p[d]);
                ci[d][0] = I;
                if (J < 0) {
                    w[d][0] = 1;
                    cnt[d] = 1;
                } else {
                    w[d][0] = (T)0.75;
                    ci[d][1] = J;
                    w[d][1] = (T)0.25;
                    cnt[d] = 2;
                }
            } else if ((f[d] & 1) == 0) {
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
        x[t] += e;
    }
}

template <typename T>
__device__ __forceinline__ void set_level_ptrs(pmg_level &L, T *x, T *r, T *res) {
    if constexpr (sizeof(T) == 8) {
        L.x = (double *)x;
        L.r = (double *)r;
        L.res = (double *)res;
    } else {
        L.xs = (float *)x;
        L.rs = (float *)r;
        L.ress = (float *)res;
    }
}

template <typename T>
__device__ __forceinline__ const T *LRI(const pmg_level &L) {
    if constexpr (sizeof(T) == 8) return (const T *)L.ri;
    else return (const T *)L.ris;
}

template <typename T>
__device__ __forceinline__ T *LX(const pmg_level &L) {
    if constexpr (sizeof(T) == 8) return (T *)L.x;
    else return (T *)L.xs;
}
template <typename T>
__device__ __forceinline__ T *LR(const pmg_level &L) {
    if constexpr (sizeof(T) == 8) return (T *)L.r;
    else return (T *)L.rs;
}
template <typename T>
__device__ __forceinline__ T *LS(const pmg_level &L) {
    if constexpr (sizeof(T) == 8) return (T *)L.res;
    else return (T *)L.ress;
}

// coarse levels cf..nlev-1 of one V-cycle inside the calling CTA
template <typename T>
__device__ void coarse_cycle(const pmg_args &A, int cf) {
    const int t0 = threadIdx.x, ts = blockDim.x;
    const int nc = A.kind == 0 ? 2 : 4;
    for (int l = cf; l < A.nlev - 1; l++) {
        const pmg_level &F = A.lv[l];
        for (int s = 0; s < A.v_down; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LRI<T>(F), c, t0, ts);
                __syncthreads();
            }
        ph_resid<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LS<T>(F), LRI<T>(F), t0, ts);
        __syncthreads();
        const pmg_level &C = A.lv[l + 1];
        ph_restrict<T>(A.kind, ldev(F), ldev(C), LS<T>(F), LR<T>(C), LX<T>(C), t0, ts);
        __syncthreads();
    }
    {  // coarsest level
        const pmg_level &L = A.lv[A.nlev - 1];
        const int np = L.n[0] * L.n[1] * L.n[2];
        T *x = LX<T>(L);
        const T *r = LR<T>(L);
        if (A.dense) {
            // one warp per row of the (row-major) inverse: coalesced reads
            const int warp = t0 >> 5, lane = t0 & 31, nw = ts >> 5;
            for (int row = warp; row < np; row += nw) {
                const double *b = A.dense + (size_t)row * np;
                double acc = 0;
                for (int c = lane; c < np; c += 32) acc += b[c] * (double)r[c];
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) x[row] = (T)acc;
            }
            __syncthreads();
        } else {
            for (int p = t0; p < np; p += ts) x[p] = 0;
            __syncthreads();
            for (int s = 0; s < 80; s++)
                for (int c = 0; c < nc; c++) {
                    ph_smooth_colour<T>(A.kind, ldev(L), x, r, LRI<T>(L), c, t0, ts);
                    __syncthreads();
                }
        }
    }
    for (int l = A.nlev - 2; l >= cf; l--) {
        const pmg_level &F = A.lv[l];
        const pmg_level &C = A.lv[l + 1];
        ph_prolong<T>(A.kind, ldev(F), ldev(C), LX<T>(F), LX<T>(C), t0, ts);
        __syncthreads();
        for (int s = 0; s < A.v_up; s++)
            for (int c = 0; c < nc; c++) {
                ph_smooth_colour<T>(A.kind, ldev(F), LX<T>(F), LR<T>(F), LRI<T>(F), c, t0, ts);
                __syncthreads();
            }
    }
}

}  // namespace rmt3d
