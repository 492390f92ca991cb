// Passive tracers on the device (Utilities/tracers.{hh,cc}): one thread per
// tracer.  A tracer keeps the reference's local coordinates: the corner
// p_crd of the 4x4x4 cube of cell centres it is interpolated from, and its
// position rp within the central cell of that cube, in units of the spacing
// and in [-0.5, 0.5] about the cube's centre.  Tracers live on a single
// domain, so a tracer that leaves it through a periodic face comes back on
// the other side (the reference's send to itself) and one that leaves
// through a wall is lost, as when the reference sends it to no process.
#include "kernels.h"

namespace rmt3d {

// tricubic interpolation of the cell-centred velocity at (rx, ry, rz) of the
// cube whose corner cell is (ti, tj, tk) (tracers::interp_vels,
// tracers.cc:395-457).  The reference fits the 64 values with the inverse of
// the 64x64 Vandermonde matrix of the monomials x^i y^j z^k (i, j, k <= 3)
// at the nodes -1.5, -0.5, 0.5, 1.5 of each axis; that interpolant is the
// tensor product of the cubic Lagrange polynomials through those nodes,
// evaluated here axis by axis.
__device__ inline void lagrange4(double r, double (&w)[4]) {
    const double a = r + 1.5, b = r + 0.5, c = r - 0.5, d = r - 1.5;
    w[0] = b * c * d / -6.0;
    w[1] = a * c * d / 2.0;
    w[2] = a * b * d / -2.0;
    w[3] = a * b * c / 6.0;
}

__device__ void tracer_interp(const grid_dev &g, const fields_dev *__restrict__ F, int ti, int tj, int tk,
                              const double (&r)[3], double (&v)[3]) {
    // the reference clamps a cube that leaves the box (tracers.cc:401-426)
    ti = min(max(ti, 0), g.sm4 - 4);
    tj = min(max(tj, 0), g.sn4 - 4);
    tk = min(max(tk, 0), g.so4 - 4);
    double wx[4], wy[4], wz[4];
    lagrange4(r[0], wx);
    lagrange4(r[1], wy);
    lagrange4(r[2], wz);
    for (int c = 0; c < 3; c++) {
        const double *u = F->vel[c];
        double acc = 0;
        for (int k = 0; k < 4; k++) {
            double sy = 0;
            for (int j = 0; j < 4; j++) {
                const double *row = u + gidx(g, ti, tj + j, tk + k);
                const double sx = ((wx[0] * row[0] + wx[1] * row[1]) + wx[2] * row[2]) + wx[3] * row[3];
                sy += wy[j] * sx;
            }
            acc += wz[k] * sy;
        }
        v[c] = acc;
    }
}

// tracers::dx (tracers.hh:346-439): the displacement dt v along axis f,
// slowed near a homogeneous Dirichlet wall the tracer moves towards and kept
// 1% of the domain length away from it.  xx is the tracer's coordinate.
__device__ double tracer_dx(const tracer_args &A, int f, double v, double xx) {
    double update = A.dt * v;
    const int lr = (v < 0) ? 0 : 1;
    if (!A.homog[f][lr]) return update;
    const double lo = A.lo[f], hi = A.hi[f];
    const double min_sep = 0.01 * (hi - lo);
    double sep;
    if (v == 0) {
        const double v1 = fabs(xx - lo), v2 = fabs(hi - xx);
        sep = v2 < v1 ? (hi - xx) : (xx - lo);
    } else {
        sep = (v < 0) ? (xx - lo) : (hi - xx);
    }
    const double vn = fabs(v);
    if (sep <= min_sep) {
        if (v == 0) {
            const double v1 = fabs(xx - lo), v2 = fabs(hi - xx);
            return (v2 < v1) ? (hi - min_sep - xx) : (lo + min_sep - xx);
        }
        return (v < 0) ? (lo + min_sep - xx) : (hi - min_sep - xx);
    }
    if (fabs(update) > 0.1 * sep) update = (exp(-A.dt * vn / sep) - 1) * ((v < 0) ? sep : -sep);
    if ((v < 0 && (xx + update) < (lo + min_sep)) || (v > 0 && (xx + update) > (hi - min_sep)))
        return (v < 0) ? (lo + min_sep - xx) : (hi - min_sep - xx);
    return update;
}

// tracers::proc_adjust (tracers.cc:261-301) followed, for a tracer that left
// the box, by the single-domain exchange (fill_buffer / communicate /
// empty_buffer, :303-371): it returns when every axis it left through is
// periodic, with its cube moved to the image, and is lost otherwise.  `st`
// 0 tests rpf (after the predictor), 1 tests rp0 (after the corrector).
// Returns false for a lost tracer.
__device__ bool tracer_adjust(const grid_dev &g, const tracer_args &A, int (&pc)[3], double (&rp0)[3],
                              double (&rpf)[3], int st) {
    const int lim[3] = {g.sm4, g.sn4, g.so4};
    int comm[3];
    for (int f = 0; f < 3; f++) {
        double *val = st == 0 ? &rpf[f] : &rp0[f];
        if (!isfinite(*val)) return false;
        // a tracer moves less than a cell per step; the bound only keeps a
        // wild value from looping (the reference would loop on)
        for (int it = 0; *val <= -0.5; it++) {
            if (it >= 1024) return false;
            rp0[f] += 1.0;
            rpf[f] += 1.0;
            pc[f]--;
        }
        for (int it = 0; *val > 0.5; it++) {
            if (it >= 1024) return false;
            rp0[f] -= 1.0;
            rpf[f] -= 1.0;
            pc[f]++;
        }
        const bool low = pc[f] < 0 || (pc[f] == 0 && *val < 0);
        const bool high = pc[f] > lim[f] - 4 || (pc[f] == lim[f] - 4 && *val >= 0);
        if (low) {
            comm[f] = 0;
        } else if (high) {
            comm[f] = 2;
            pc[f] -= lim[f] - 4;
        } else {
            comm[f] = 1;
        }
    }
    if (comm[0] == 1 && comm[1] == 1 && comm[2] == 1) return true;
    for (int f = 0; f < 3; f++)
        if (comm[f] != 1 && !g.prd[f]) return false;
    for (int f = 0; f < 3; f++) {
        const double val = st == 0 ? rpf[f] : rp0[f];
        if (pc[f] < 0 || (pc[f] == 0 && val < 0)) pc[f] += lim[f] - 4;
    }
    return true;
}

__device__ inline double tracer_loc(const tracer_args &A, int f, int pc, double rp) {
    return A.low[f] + (1.5 + rp + pc) * A.h[f];
}

// tracers::predict (tracers.hh:222-290): forward Euler from rp0 with the
// velocity at the start of the step, into rpf
__global__ void k_tracer_predict(grid_dev g, const fields_dev *__restrict__ F, tracer_args A, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !A.alive[t]) return;
    int pc[3];
    double rp0[3], rpf[3], v0[3];
    for (int f = 0; f < 3; f++) {
        pc[f] = A.pc[f * n + t];
        rp0[f] = A.rp[f * n + t];
    }
    tracer_interp(g, F, pc[0], pc[1], pc[2], rp0, v0);
    for (int f = 0; f < 3; f++) rpf[f] = rp0[f] + tracer_dx(A, f, v0[f], tracer_loc(A, f, pc[f], rp0[f])) / A.h[f];
    if (!tracer_adjust(g, A, pc, rp0, rpf, 0)) {
        A.alive[t] = 0;
        return;
    }
    for (int f = 0; f < 3; f++) {
        A.pc[f * n + t] = pc[f];
        A.rp[f * n + t] = rp0[f];
        A.rp[(3 + f) * n + t] = rpf[f];
    }
}

// tracers::imp_euler (tracers.hh:292-318): the improved Euler corrector with
// the velocity at the end of the step, interpolated at rpf
__global__ void k_tracer_advect(grid_dev g, const fields_dev *__restrict__ F, tracer_args A, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !A.alive[t]) return;
    int pc[3];
    double rp0[3], rpf[3], vf[3];
    for (int f = 0; f < 3; f++) {
        pc[f] = A.pc[f * n + t];
        rp0[f] = A.rp[f * n + t];
        rpf[f] = A.rp[(3 + f) * n + t];
    }
    tracer_interp(g, F, pc[0], pc[1], pc[2], rpf, vf);
    for (int f = 0; f < 3; f++) {
        const double dr0 = rpf[f] - rp0[f];
        const double drf = tracer_dx(A, f, vf[f], tracer_loc(A, f, pc[f], rpf[f])) / A.h[f];
        rp0[f] += 0.5 * (dr0 + drf);
    }
    if (!tracer_adjust(g, A, pc, rp0, rpf, 1)) {
        A.alive[t] = 0;
        return;
    }
    for (int f = 0; f < 3; f++) {
        A.pc[f * n + t] = pc[f];
        A.rp[f * n + t] = rp0[f];
        A.rp[(3 + f) * n + t] = rpf[f];
    }
}

// tracers::set (tracers.hh:158-168) for tracer t at (x, y, z): a position
// outside the box leaves the tracer out (the reference does not add it)
__global__ void k_tracer_place(grid_dev g, tracer_args A, int n, const double *xyz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int lim[3] = {g.sm4, g.sn4, g.so4};
    bool in = true;
    for (int f = 0; f < 3; f++) {
        const double t_ind = (xyz[3 * t + f] - A.low[f]) / A.h[f] - 1;
        const int p = (int)t_ind;
        const double rp = t_ind - p - 0.5;
        A.pc[f * n + t] = p;
        A.rp[f * n + t] = rp;
        A.rp[(3 + f) * n + t] = 0;
        const bool low = p < 0 || (p == 0 && rp < 0);
        const bool high = p > lim[f] - 4 || (p == lim[f] - 4 && rp >= 0);
        if (low || high || !isfinite(t_ind)) in = false;
    }
    A.alive[t] = in ? 1 : 0;
}

// tracers::print's coordinates (tracers.cc:105-133): loc0 of every tracer
// by id as float, zeros for a tracer that is gone
__global__ void k_tracer_positions(tracer_args A, int n, float *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    for (int f = 0; f < 3; f++)
        out[3 * t + f] = A.alive[t] ? (float)tracer_loc(A, f, A.pc[f * n + t], A.rp[f * n + t]) : 0.f;
}

}  // namespace rmt3d
