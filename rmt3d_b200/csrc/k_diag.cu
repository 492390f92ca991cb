// Frame diagnostics and slice output on the device: the quantities the
// reference's stepper writes to macro.dat and centroid.dat
// (Sim/stepper.hh:378-474) and the slices of fluid_3d::write_slice
// (F3D_Source/fluid_3d_io.cc:3-434).
#include "kernels.h"

namespace rmt3d {

// Reduce NV per-thread values over the grid in a fixed order: warp
// shuffles, then the warps of a block in index order, then (in the block
// that finishes last) the blocks in index order.  Bit c of max_mask makes
// value c a maximum instead of a sum.  out holds NV totals followed by NV
// partials per block; *ticket returns to 0.  blockDim.x is a multiple of 32.
template <int NV>
__device__ void fixed_order_reduce(double (&v)[NV], unsigned max_mask, double *out, unsigned *ticket) {
    __shared__ double sh[NV][32];
    __shared__ bool last;
    for (int c = 0; c < NV; c++) {
        const bool mx = (max_mask >> c) & 1u;
        double a = v[c];
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < NV; c++) {
            const bool mx = (max_mask >> c) & 1u;
            double a = sh[c][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) a = mx ? fmax(a, sh[c][w]) : a + sh[c][w];
            out[NV * (1 + blockIdx.x) + c] = a;
        }
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && threadIdx.x < NV) {
        __threadfence();
        const int c = threadIdx.x;
        const bool mx = (max_mask >> c) & 1u;
        const volatile double *part = out + NV;
        double a = part[c];
        for (unsigned b = 1; b < gridDim.x; b++) a = mx ? fmax(a, part[NV * b + c]) : a + part[NV * b + c];
        out[c] = a;
        if (c == 0) *ticket = 0;
    }
}

// Sums of u^2, v^2, w^2 and p^2 over the interior cells, in a fixed order
// (the same bits on every run)
__global__ void k_checksum(grid_dev g, const fields_dev *__restrict__ F, double *out, unsigned *ticket) {
    double v[4] = {0, 0, 0, 0};
    const int ncell = g.sm * g.sn * g.so;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
        const int ind = gidx(g, t % g.sm + 2, (t / g.sm) % g.sn + 2, t / (g.sm * g.sn) + 2);
        for (int c = 0; c < 3; c++) v[c] += F->vel[c][ind] * F->vel[c][ind];
        v[3] += F->p[ind] * F->p[ind];
    }
    fixed_order_reduce<4>(v, 0u, out, ticket);
}

// Interior-cell sums and extremes of one frame:
//  [0..2] sum of velocity (times density in the variable-density form)
//         (total_momentum, fluid_3d_utils.cc:783-800);
//  [3] sum of |u|^2 / 2; [4] sum of gravity (z - az) over primary cells;
//  [5] sum over primary cells of the mean elastic energy of the cell's six
//      faces, its own three lower faces and the lower faces of its upper
//      neighbours (total_energy, :806-872);
//  [6] max and [7] -min of the divergence of the face velocities
//      (div_u, :579-600).
__global__ void k_macro_cells(grid_dev g, const fields_dev *__restrict__ F, const double *lz, int var_den,
                              double *out, unsigned *ticket) {
    double v[8] = {0, 0, 0, 0, 0, 0, -1e200, -1e200};
    const int ncell = g.sm * g.sn * g.so;
    const int strides[3] = {1, g.sm4, g.smn4};
    const double dhsp[3] = {g.dxsp, g.dysp, g.dzsp};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
        const int i = t % g.sm + 2, j = (t / g.sm) % g.sn + 2, k = t / (g.sm * g.sn) + 2;
        const int ind = gidx(g, i, j, k);
        for (int s = 0; s < 3; s++) {
            const double u = F->vel[s][ind];
            v[s] += var_den ? u * F->rho[ind] : u;
            v[3] += 0.5 * u * u;
        }
        double div = 0;
        for (int f = 0; f < 3; f++)
            div += dhsp[f] * (face_ld(g, F, 3 * (2 * f + 1) + f, ind) - face_ld(g, F, 3 * (2 * f) + f, ind));
        v[6] = fmax(v[6], div);
        v[7] = fmax(v[7], -div);
        for (int o = 0; o < g.n_obj; o++) {
            const objmap_dev &m = F->om[o];
            if (m.code[ind] != 0) continue;
            if (g.gravity != 0) v[4] += g.gravity * (lz[k] - g.az);
            double el = 0;
            for (int s = 0; s < 3; s++) {
                el += m.el[s][ind];
                const int nb = ind + strides[s];
                if (m.code[nb] >= 0) el += m.el[s][nb];
            }
            v[5] += el / 6.;
        }
    }
    fixed_order_reduce<8>(v, (1u << 6) | (1u << 7), out, ticket);
}

// Heaviside-weighted sums over the primary cells of object o
// (compute_v_centroid, fluid_3d_utils.cc:1290-1346): [0] weight, [1..3]
// weighted x, y, z, [4..6] weighted velocity.
__global__ void k_macro_obj(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                            const double *lz, int o, double *out, unsigned *ticket) {
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    const int ncell = g.sm * g.sn * g.so;
    const objmap_dev &m = F->om[o];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
        const int i = t % g.sm + 2, j = (t / g.sm) % g.sn + 2, k = t / (g.sm * g.sn) + 2;
        const int ind = gidx(g, i, j, k);
        if (m.code[ind] != 0) continue;
        const double sf = heaviside(g, obj_phi(g, o, m.x[0][ind], m.x[1][ind], m.x[2][ind]));
        v[0] += sf;
        v[1] += lx[i] * sf;
        v[2] += ly[j] * sf;
        v[3] += lz[k] * sf;
        for (int s = 0; s < 3; s++) v[4 + s] += F->vel[s][ind] * sf;
    }
    fixed_order_reduce<7>(v, 0u, out, ticket);
}

// Weighted sum of squares of the FEM right-hand side (div_u's L2 norm,
// fluid_3d_utils.cc:517-547): half weight on each non-periodic boundary
// plane of the nodal grid.
__global__ void k_divu_l2(grid_dev g, const double *r, double *out, unsigned *ticket) {
    double v[1] = {0};
    const int nn = g.fm * g.fn * g.fo;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += gridDim.x * blockDim.x) {
        const int a = t % g.fm, b = (t / g.fm) % g.fn, c = t / (g.fm * g.fn);
        double nk = (c == 0 || c == g.fo - 1) ? 0.5 : 1.0;
        if (g.prd[2]) nk = 1.0;
        double nj = (b == 0 || b == g.fn - 1) ? 0.5 : 1.0;
        if (g.prd[1]) nj = 1.0;
        double ni = (a == 0 || a == g.fm - 1) ? 0.5 : 1.0;
        if (g.prd[0]) ni = 1.0;
        const double rr = r[t];
        v[0] += ni * nj * nk * rr * rr;
    }
    fixed_order_reduce<1>(v, 0u, out, ticket);
}

// One value of output type `type` at interior-relative cell or node
// (i, j, k), as fluid_3d::copy_slice_to_buf computes it
// (fluid_3d_io.cc:257-418).  obj_id -1 takes the map of least level set at
// the cell, obj_id >= 1 that object's map; map quantities are 100 (OID 0)
// where there is none.
__device__ double slice_value(const grid_dev &g, const fields_dev *__restrict__ F, const double *r, int type,
                              int obj_id, int var_den, int i, int j, int k) {
    const int eid = gidx(g, i + 2, j + 2, k + 2);
    const int lo = eid - g.smn4;
    const int s4 = g.sm4;
    const double *u = F->vel[0], *v = F->vel[1], *w = F->vel[2];
    switch (type) {
        case 0: case 1: case 2: return F->vel[type][eid];
        case 3:
            return 0.25 * g.dysp * (w[eid] - w[eid - s4] + w[eid - 1] - w[eid - 1 - s4] + w[lo] - w[lo - s4] + w[lo - 1] - w[lo - 1 - s4]) -
                   0.25 * g.dzsp * (v[eid] - v[lo] + v[eid - 1] - v[lo - 1] + v[eid - s4] - v[lo - s4] + v[eid - 1 - s4] - v[lo - 1 - s4]);
        case 4:
            return 0.25 * g.dzsp * (u[eid] - u[lo] + u[eid - 1] - u[lo - 1] + u[eid - s4] - u[lo - s4] + u[eid - 1 - s4] - u[lo - 1 - s4]) -
                   0.25 * g.dxsp * (w[eid] - w[eid - 1] + w[eid - s4] - w[eid - s4 - 1] + w[lo] - w[lo - 1] + w[lo - s4] - w[lo - s4 - 1]);
        case 5:
            return 0.25 * g.dxsp * (v[eid] - v[eid - 1] + v[eid - s4] - v[eid - s4 - 1] + v[lo] - v[lo - 1] + v[lo - s4] - v[lo - s4 - 1]) -
                   0.25 * g.dysp * (u[eid] - u[eid - s4] + u[eid - 1] - u[eid - 1 - s4] + u[lo] - u[lo - s4] + u[lo - 1] - u[lo - 1 - s4]);
        case 6: {
            double t = 0;
            for (int c = 0; c < 3; c++) t += F->vel[c][eid] * F->vel[c][eid];
            return sqrt(t);
        }
        case 7: return F->p[eid];
        case 18: return r[i + g.fm * (j + g.fn * k)];
        case 19:
            return g.dxsp * (face_ld(g, F, 3, eid) - face_ld(g, F, 0, eid)) +
                   g.dysp * (face_ld(g, F, 10, eid) - face_ld(g, F, 7, eid)) +
                   g.dzsp * (face_ld(g, F, 17, eid) - face_ld(g, F, 14, eid));
        case 20: return var_den ? F->rho[eid] : 0.;
        case 21: return 100.;
        default: break;
    }
    // reference-map quantities, types 8..17
    int prim = -1;
    for (int o = 0; o < g.n_obj; o++)
        if (F->om[o].code[eid] == 0) prim = o;
    int sel = obj_id - 1;
    if (obj_id == -1) {
        sel = prim;
        double mphi = 1e30;
        if (prim >= 0) {
            const objmap_dev &mp = F->om[prim];
            mphi = obj_phi(g, prim, mp.x[0][eid], mp.x[1][eid], mp.x[2][eid]);
        }
        for (int o = 0; o < g.n_obj; o++) {
            const objmap_dev &me = F->om[o];
            if (me.code[eid] <= 0) continue;
            const double t = obj_phi(g, o, me.x[0][eid], me.x[1][eid], me.x[2][eid]);
            if (t < mphi) {
                mphi = t;
                sel = o;
            }
        }
    }
    if (sel < 0 || sel >= g.n_obj || F->om[sel].code[eid] < 0) return type == 12 ? 0. : 100.;
    const objmap_dev &m = F->om[sel];
    const int code = m.code[eid];
    switch (type) {
        case 8: return obj_phi(g, sel, m.x[0][eid], m.x[1][eid], m.x[2][eid]);
        case 9: case 10: case 11: return m.x[type - 9][eid];
        case 12: return code == 0 ? (double)(sel + 1) : 0.;
        case 13: return (double)code;
        case 14: return obj_phi(g, sel, m.xp[0][eid], m.xp[1][eid], m.xp[2][eid]);
        default: return m.xp[type - 15][eid];
    }
}

// The slice at index `point` of axis `dim` as the reference's global slice
// array: out[a + d1 b] with (a, b) running over the two other axes in
// increasing axis order, over the cell extents or, for the nodal types
// 3, 4, 5, 7, 18, the nodal extents (fluid_3d_io.cc:98-255, 479-505).
__global__ void k_slice(grid_dev g, const fields_dev *__restrict__ F, const double *r, int type, int dim, int point,
                        int obj_id, int var_den, int d1, int d2, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d1 * d2) return;
    const int a = t % d1, b = t / d1;
    const int i = dim == 0 ? point : a;
    const int j = dim == 0 ? a : (dim == 1 ? point : b);
    const int k = dim == 2 ? point : b;
    out[t] = slice_value(g, F, r, type, obj_id, var_den, i, j, k);
}

}  // namespace rmt3d
