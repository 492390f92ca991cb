// Fluid-side kernels of the FSI step: ghost frames, stress, Godunov edge
// states and upwinding, the explicit momentum update and the two projection
// right-hand sides / corrections.  Each kernel cites the reference loop it
// replaces; floating-point expressions keep the reference's association order
// so that, built without FMA contraction, results track the reference's CPU
// run to rounding.
#include <cuda.h>

#include "dev_common.cuh"
#include "kernels.h"

namespace rmt3d {

// -------------------------------------------------------------------------
// Periodic ghost copy: replaces fluid_3d::communicate<flags> on one rank
// (fluid_3d_comm.cc:76-198), where each ghost region whose direction has only
// periodic components receives the interior slab from the opposite side.
// corner != 0 selects the nodal table (fluid_3d_comm.cc:55-58), whose extent
// along a non-periodic axis is one node longer.
// -------------------------------------------------------------------------
__global__ void k_periodic_copy(grid_dev g, ptr_list pl, int corner) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.sm4 || j >= g.sn4 || k >= g.so4) return;
    const int c[3] = {i, j, k};
    const int s[3] = {g.sm, g.sn, g.so};
    int src[3];
    bool ghost = false;
    for (int d = 0; d < 3; d++) {
        int len = s[d] + ((corner && !g.prd[d]) ? 1 : 0);
        if (c[d] >= 2 && c[d] < 2 + len) {
            src[d] = c[d];
            continue;
        }
        if (!g.prd[d]) return;  // wall ghost: not filled by the exchange
        ghost = true;
        src[d] = (c[d] < 2) ? c[d] + s[d] : c[d] - s[d];
    }
    if (!ghost) return;
    int dst = gidx(g, i, j, k), from = gidx(g, src[0], src[1], src[2]);
    for (int a = 0; a < pl.n; a++) pl.p[a][dst] = pl.p[a][from];
    for (int a = 0; a < pl.nf; a++) pl.fp[a][dst] = pl.fp[a][from];
    for (int a = 0; a < pl.ni; a++) pl.ip[a][dst] = pl.ip[a][from];
}

// -------------------------------------------------------------------------
// Physical BC ghost fill of one face, face_gm::set_ghost_cc
// (fields.hh:765-800): both ghost layers, the whole tangential extent.
// -------------------------------------------------------------------------
__global__ void k_bc_cc(grid_dev g, int n, bc_face lo, bc_face hi, double *u, double *v, double *w) {
    // both faces of axis n in one launch: blockIdx.z = 2 * side + layer - 1.
    // The two faces write disjoint ghost layers and read only cells of their
    // own side, so they run together; the axes still run in order, x, y, z,
    // since a later axis reads the earlier axes' ghost values at edges.
    const int lower = (blockIdx.z < 2);
    const int face = 2 * n + (lower ? 0 : 1);
    const bc_face &bc = lower ? lo : hi;
    const int t0 = (n == 0) ? 1 : 0, t1 = (n == 2) ? 1 : 2;
    const int ext[3] = {g.sm4, g.sn4, g.so4};
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    int b = blockIdx.y * blockDim.y + threadIdx.y;
    int layer = (blockIdx.z & 1) + 1;  // 1 or 2
    if (a >= ext[t0] || b >= ext[t1]) return;
    (void)face;
    // flat indices from the strides of the three axes (no runtime-indexed
    // arrays, which would live in local memory)
    const int sa = t0 == 0 ? 1 : g.sm4, sb = t1 == 1 ? g.sm4 : g.smn4;
    const int sn_ = n == 0 ? 1 : (n == 1 ? g.sm4 : g.smn4);
    const int ln = n == 0 ? g.sm : (n == 1 ? g.sn : g.so);
    const int gn = lower ? 2 - layer : 2 + ln - 1 + layer;
    const int mn = lower ? 2 + layer - 1 : 2 + ln - layer;
    const int gi = a * sa + b * sb + gn * sn_;
    const int mi = a * sa + b * sb + mn * sn_;
    const double sgn = lower ? -1 : 1;
    const double dn = 2 * fabs(0.5 * bc.h * (2 * layer - 1));
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double *vc = c == 0 ? u : (c == 1 ? v : w);
        if (bc.bct[c] == 1) vc[gi] = 2 * bc.bcv[c] - vc[mi];
        else vc[gi] = sgn * dn * bc.bcv[c] + vc[mi];
    }
}

// -------------------------------------------------------------------------
// Face-velocity BC of one face, face_gm::set_ghost_cf / compute_ghost_cf
// (fields.hh:804-849): the boundary face of the outermost interior layer and
// the matching face of the inner ghost layer.
// -------------------------------------------------------------------------
// All wall faces in one launch (blockIdx.z = face; bit f of walls marks a
// wall): each face reads velocities only and writes its own face-velocity
// components, so the faces are independent.
__global__ void k_bc_cf(grid_dev g, int walls, bc_faces bcs, const fields_dev *F) {
    const int face = blockIdx.z;
    if (!((walls >> face) & 1)) return;
    const bc_face &bc = bcs.f[face];
    const int n = face / 2;
    const int lower = (face % 2 == 0);
    const int t0 = (n == 0) ? 1 : 0, t1 = (n == 2) ? 1 : 2;
    const int ext[3] = {g.sm4, g.sn4, g.so4};
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    int b = blockIdx.y * blockDim.y + threadIdx.y;
    if (a >= ext[t0] || b >= ext[t1]) return;
    const int sa = t0 == 0 ? 1 : g.sm4, sb = t1 == 1 ? g.sm4 : g.smn4;
    const int sn_ = n == 0 ? 1 : (n == 1 ? g.sm4 : g.smn4);
    const int ln = n == 0 ? g.sm : (n == 1 ? g.sn : g.so);
    const int base = a * sa + b * sb;
    const int gi = base + (lower ? 1 : 2 + ln) * sn_;
    const int i0 = base + (lower ? 2 : 1 + ln) * sn_;
    const int i1 = base + (lower ? 3 : ln) * sn_;
    const double sgn = lower ? -1 : 1;
    const int inner = 2 * n + (lower ? 1 : 0);
    for (int c = 0; c < 3; c++) {
        double f = bc.bcv[c];
        if (bc.bct[c] == 2) f = (3 * bc.h * bc.bcv[c] * sgn + 9 * F->vel[c][i0] - F->vel[c][i1]) * 0.125;
        face_st(g, F, 3 * face + c, i0, f);
        face_st(g, F, 3 * inner + c, gi, f);
    }
}

// -------------------------------------------------------------------------
// Stress on the three lower faces, fluid_3d::compute_stress
// (fluid_3d.cc:1360-1461) with solid_stress (:1777-1997), fluid_stress
// (:2001-2031) and collision_stress (:1465-1773).  One thread per cell over
// relative cells -1..s+1 inclusive, i.e. absolute 1..s+3.
// -------------------------------------------------------------------------
__device__ inline bool has_map(const objmap_dev &m, int ind) { return m.code[ind] >= 0; }

__device__ inline double map_phi(const grid_dev &g, const objmap_dev &m, int o, int ind) {
    return obj_phi(g, o, m.x[0][ind], m.x[1][ind], m.x[2][ind]);
}

// Collision stress between maps of different objects sharing a cell,
// fluid_3d::collision_stress (fluid_3d.cc:1465-1773).  The reference derives
// the neighbour positions from the cell's offset relative to the first
// interior cell (unpack_index(eid), :1476), so its box check runs on shifted
// coordinates; that is reproduced, including C++ truncating division.
template <int FF>
__device__ void collision_face(const grid_dev &g, const fields_dev *__restrict__ F, int i, int j, int k, int ind,
                               const int *order, int nmaps, double out[3]) {
    const int strides[3] = {1, g.sm4, g.smn4};
    const double facs[3] = {g.dxsp, g.dysp, g.dzsp};
    const int strd = strides[FF];
    const int ad1 = (FF + 1) % 3, ad2 = (FF + 2) % 3;
    const int ext[3] = {g.sm4, g.sn4, g.so4};
    const int G0 = gidx(g, 2, 2, 2);
    const int eid = ind - G0;
    int lp[3];
    lp[2] = eid / g.smn4;
    lp[1] = (eid % g.smn4) / g.sm4;
    lp[0] = eid % g.sm4;
    auto nbo = [&](const objmap_dev &m, int da, int sa, int db, int sb) -> int {
        int p[3] = {lp[0], lp[1], lp[2]};
        p[da] += sa;
        p[db] += sb;
        for (int d = 0; d < 3; d++)
            if (p[d] < 0 || p[d] >= ext[d]) return -1;
        int q = ind + sa * strides[da] + sb * strides[db];
        if (q < 0 || q >= g.ncell) return -1;
        return m.code[q] >= 0 ? q : -1;
    };
    auto grad = [&](const objmap_dev &m, int o, int rn, int q1p, int q1p1, int q1m, int q1m1, int q2p, int q2p1,
                    int q2m, int q2m1, double dph[3]) {
        dph[FF] = facs[FF] * (map_phi(g, m, o, ind) - map_phi(g, m, o, rn));
        dph[ad1] = 0.25 * facs[ad1] *
                   (map_phi(g, m, o, q1p) + map_phi(g, m, o, q1p1) - map_phi(g, m, o, q1m) - map_phi(g, m, o, q1m1));
        dph[ad2] = 0.25 * facs[ad2] *
                   (map_phi(g, m, o, q2p) + map_phi(g, m, o, q2p1) - map_phi(g, m, o, q2m) - map_phi(g, m, o, q2m1));
        double nrm = 0;
        for (int c = 0; c < 3; c++) nrm += dph[c] * dph[c];
        if (nrm > 0) {
            nrm = sqrt(nrm);
            for (int c = 0; c < 3; c++) dph[c] /= nrm;
        }
    };
    for (int ii = 0; ii < nmaps - 1; ii++) {
        const int o0 = order[ii];
        const objmap_dev &m0 = F->om[o0];
        const double G0m = g.obj[o0].G;
        int rn0 = nbo(m0, FF, -1, FF, 0);
        if (rn0 < 0) continue;
        double phiv0 = 0.5 * (map_phi(g, m0, o0, ind) + map_phi(g, m0, o0, rn0));
        if (phiv0 > g.eps) continue;
        int a1 = nbo(m0, ad1, 1, FF, 0), a2 = nbo(m0, ad1, 1, FF, -1), a3 = nbo(m0, ad1, -1, FF, 0),
            a4 = nbo(m0, ad1, -1, FF, -1);
        int b1 = nbo(m0, ad2, 1, FF, 0), b2 = nbo(m0, ad2, 1, FF, -1), b3 = nbo(m0, ad2, -1, FF, 0),
            b4 = nbo(m0, ad2, -1, FF, -1);
        if (a1 < 0 || a2 < 0 || a3 < 0 || a4 < 0 || b1 < 0 || b2 < 0 || b3 < 0 || b4 < 0) continue;
        double d0[3];
        grad(m0, o0, rn0, a1, a2, a3, a4, b1, b2, b3, b4, d0);
        for (int jj = ii + 1; jj < nmaps; jj++) {
            const int o1 = order[jj];
            const objmap_dev &m1 = F->om[o1];
            int rn1 = ind - strd;
            if (rn1 < 0 || m1.code[rn1] < 0) continue;
            double phiv1 = 0.5 * (map_phi(g, m1, o1, ind) + map_phi(g, m1, o1, rn1));
            if (phiv1 > g.eps || phiv0 + phiv1 > g.eps) continue;
            int c1 = nbo(m1, ad1, 1, FF, 0), c2 = nbo(m1, ad1, 1, FF, -1), c3 = nbo(m1, ad1, -1, FF, 0),
                c4 = nbo(m1, ad1, -1, FF, -1);
            int e1 = nbo(m1, ad2, 1, FF, 0), e2 = nbo(m1, ad2, 1, FF, -1), e3 = nbo(m1, ad2, -1, FF, 0),
                e4 = nbo(m1, ad2, -1, FF, -1);
            if (c1 < 0 || c2 < 0 || c3 < 0 || c4 < 0 || e1 < 0 || e2 < 0 || e3 < 0 || e4 < 0) continue;
            double d1[3];
            grad(m1, o1, rn1, c1, c2, c3, c4, e1, e2, e3, e4, d1);
            double nv[3], den = 0;
            for (int nn = 0; nn < 3; nn++) {
                nv[nn] = d1[nn] - d0[nn];
                den += nv[nn] * nv[nn];
            }
            den = sqrt(den);
            if (den < 100. * 2.220446049250313e-16) continue;
            for (int nn = 0; nn < 3; nn++) nv[nn] /= den;
            const double G1m = g.obj[o1].G;
            double cf = G0m * coll_func(g, phiv0) + G1m * coll_func(g, phiv1);
            double cs[3][3];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) cs[a][b] = -cf * nv[a] * nv[b];
            double avg = (cs[0][0] + cs[1][1] + cs[2][2]) / 3.;
            for (int b = 0; b < 3; b++) cs[b][b] -= avg;
            for (int a = 0; a < 3; a++) out[a] += cs[FF][a];
        }
    }
}

template <int FF>
__device__ void face_stress(const grid_dev &g, const fields_dev *__restrict__ F, int i, int j, int k, int ind,
                            bool collide) {
    const int strides[3] = {1, g.sm4, g.smn4};
    const double facs[3] = {g.dxsp, g.dysp, g.dzsp};
    const int strd = strides[FF];
    const int ad1 = (FF + 1) % 3, ad2 = (FF + 2) % 3;
    const int pos[3] = {i, j, k};
    const int ext[3] = {g.sm4, g.sn4, g.so4};
    double ss[3] = {0, 0, 0};
    double sfrac = 0;
    // maps in the reference's order: the primary first, then extrapolations
    int order[kMaxObj];
    int nmaps = 0, prim = -1;
    for (int o = 0; o < g.n_obj; o++) {
        int cd = F->om[o].code[ind];
        if (cd == 0) prim = o;
    }
    if (prim >= 0) order[nmaps++] = prim;
    for (int o = 0; o < g.n_obj; o++)
        if (o != prim && F->om[o].code[ind] > 0) order[nmaps++] = o;

    for (int mi = 0; mi < nmaps; mi++) {
        const int o = order[mi];
        const objmap_dev &m = F->om[o];
        for (int c = 0; c < 3; c++) m.gp[3 * FF + c][ind] = -kBig;
        m.det[FF][ind] = -kBig;
        m.el[FF][ind] = -kBig;
        // neighbour inside the local box (get_refmap with a position check)
        auto nb = [&](int da, int sa, int db, int sb) -> int {
            int p[3] = {pos[0], pos[1], pos[2]};
            p[da] += sa;
            p[db] += sb;
            for (int d = 0; d < 3; d++)
                if (p[d] < 0 || p[d] >= ext[d]) return -1;
            int q = gidx(g, p[0], p[1], p[2]);
            return has_map(m, q) ? q : -1;
        };
        int rn = nb(FF, -1, FF, 0);
        if (rn < 0) continue;
        const double ph = map_phi(g, m, o, ind);
        const double phn = map_phi(g, m, o, rn);
        double phiv = 0.5 * (ph + phn);
        if (phiv > g.eps) continue;
        double tf = heaviside(g, phiv);
        sfrac += tf;
        const obj_dev &ob = g.obj[o];
        double G = ob.G * tf;
        int r1p = nb(ad1, 1, FF, 0), r1p1 = nb(ad1, 1, FF, -1), r1m = nb(ad1, -1, FF, 0), r1m1 = nb(ad1, -1, FF, -1);
        int r2p = nb(ad2, 1, FF, 0), r2p1 = nb(ad2, 1, FF, -1), r2m = nb(ad2, -1, FF, 0), r2m1 = nb(ad2, -1, FF, -1);
        if (r1p < 0 || r1p1 < 0 || r1m < 0 || r1m1 < 0 || r2p < 0 || r2p1 < 0 || r2m < 0 || r2m1 < 0) continue;
        double gph[3];
        gph[FF] = facs[FF] * (ph - phn);
        gph[ad1] = 0.25 * facs[ad1] *
                   (map_phi(g, m, o, r1p) + map_phi(g, m, o, r1p1) - map_phi(g, m, o, r1m) - map_phi(g, m, o, r1m1));
        gph[ad2] = 0.25 * facs[ad2] *
                   (map_phi(g, m, o, r2p) + map_phi(g, m, o, r2p1) - map_phi(g, m, o, r2m) - map_phi(g, m, o, r2m1));
        {  // ref_map::normalize_grad_phi (fields.hh:382-394)
            double nrm = 0;
            for (int c = 0; c < 3; c++) nrm += gph[c] * gph[c];
            nrm = sqrt(nrm);
            if (nrm != 0.) {
                double ninv = 1. / nrm;
                for (int c = 0; c < 3; c++) gph[c] = ninv * gph[c];
            }
        }
        for (int c = 0; c < 3; c++) m.gp[3 * FF + c][ind] = gph[c];
        double dR[3][3];
        for (int nn = 0; nn < 3; nn++) {
            dR[FF][nn] = facs[FF] * (m.x[nn][ind] - m.x[nn][rn]);
            dR[ad1][nn] = 0.25 * facs[ad1] * (m.x[nn][r1p] + m.x[nn][r1p1] - m.x[nn][r1m] - m.x[nn][r1m1]);
            dR[ad2][nn] = 0.25 * facs[ad2] * (m.x[nn][r2p] + m.x[nn][r2p1] - m.x[nn][r2m] - m.x[nn][r2m1]);
        }
        // grad_xi(i,j) = dR[j][i], row-major (matlib.hh:160-175)
        double v[9] = {dR[0][0], dR[1][0], dR[2][0], dR[0][1], dR[1][1], dR[2][1], dR[0][2], dR[1][2], dR[2][2]};
        // matrix::inverse via the transposed cofactors (matlib.hh:303-329)
        double d = v[0] * (v[4] * v[8] - v[5] * v[7]) + v[3] * (v[2] * v[7] - v[1] * v[8]) + v[6] * (v[1] * v[5] - v[2] * v[4]);
        double Fm[9];
        for (int jj = 0; jj < 3; jj++)
            for (int ii = 0; ii < 3; ii++) {
                double cof = v[3 * ((ii + 1) % 3) + (jj + 1) % 3] * v[3 * ((ii + 2) % 3) + (jj + 2) % 3] -
                             v[3 * ((ii + 1) % 3) + (jj + 2) % 3] * v[3 * ((ii + 2) % 3) + (jj + 1) % 3];
                Fm[3 * jj + ii] = cof / d;
            }
        const double detF = Fm[0] * (Fm[4] * Fm[8] - Fm[5] * Fm[7]) + Fm[3] * (Fm[2] * Fm[7] - Fm[1] * Fm[8]) +
                            Fm[6] * (Fm[1] * Fm[5] - Fm[2] * Fm[4]);
        m.det[FF][ind] = detF;
        {  // strain energy 0.5 G (tr(F^T F) - 3 - 2 log det F) (fluid_3d.cc:1933-1938)
            double tr = 0;
            for (int a = 0; a < 3; a++) {
                double d = 0;
                for (int kk = 0; kk < 3; kk++) d += Fm[3 * kk + a] * Fm[3 * kk + a];
                tr += d;
            }
            m.el[FF][ind] = 0.5 * G * (tr - 3 - 2 * log(detF));
        }
        // left Cauchy-Green F F^T as a symmetric matrix (matlib.hh:214-229)
        double sg[3][3];
        for (int a = 0; a < 3; a++)
            for (int b = a; b < 3; b++) {
                double val = 0;
                for (int kk = 0; kk < 3; kk++) val += Fm[3 * a + kk] * Fm[3 * b + kk];
                sg[a][b] = sg[b][a] = val;
            }
        double avg = (sg[0][0] + sg[1][1] + sg[2][2]) / 3.0;
        for (int nn = 0; nn < 3; nn++) sg[nn][nn] -= avg;
        double ex_mu = ob.ex_mu * tf * (1 + ob.ev_trans_mult * tderiv_func_in(g, phiv));
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) sg[a][b] *= G;
        for (int nn = 0; nn < 3; nn++) {
            const double *vn = F->vel[nn];
            const double *vF = F->vel[FF];
            ss[nn] += sg[FF][nn];
            double tang;
            if (nn == FF) {
                tang = vn[ind] - vn[ind - strd];
            } else {
                int sn_ = strides[nn];
                tang = 0.25 * (vF[ind + sn_] + vF[ind + sn_ - strd] - vF[ind - sn_] - vF[ind - sn_ - strd]);
            }
            ss[nn] += ex_mu * facs[FF] * ((vn[ind] - vn[ind - strd]) + tang);
        }
    }
    double out[3];
    if (sfrac >= 1) {
        for (int s = 0; s < 3; s++) out[s] = ss[s] / sfrac;
    } else {
        double fs[3];
        for (int nn = 0; nn < 3; nn++) fs[nn] = g.mu * facs[FF] * (F->vel[nn][ind] - F->vel[nn][ind - strd]);
        for (int s = 0; s < 3; s++) out[s] = (1 - sfrac) * fs[s] + ss[s];
    }
    if (collide && nmaps > 1) collision_face<FF>(g, F, i, j, k, ind, order, nmaps, out);
    for (int s = 0; s < 3; s++) F->sigma[3 * FF + s][ind] = out[s];
}

// Cells that hold any reference map: the full stress (solid, fluid blend,
// collision).  Cells without maps are left to k_stress_fluid.
// The full stress of the listed cells, one thread per (cell, face): work
// item t is face t / n of cell list[t % n].  The three faces of a cell write
// disjoint outputs and read only what no face writes, so they run in any
// order; a thread holds one face's state instead of three, and every lane of
// a warp has a map cell to work on.
__global__ void __launch_bounds__(128) k_stress(grid_dev g, const fields_dev *__restrict__ F, const int *list,
                                                const int *cnt) {
    const int n = *cnt;
    const long total = 3L * n;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int FF = (int)(t / n), e = (int)(t - (long)FF * n);
        const int ind = list[e];
        const int i = ind % g.sm4, j = (ind / g.sm4) % g.sn4, k = ind / g.smn4;
        if (FF == 0) face_stress<0>(g, F, i, j, k, ind, true);
        else if (FF == 1) face_stress<1>(g, F, i, j, k, ind, true);
        else face_stress<2>(g, F, i, j, k, ind, true);
    }
}

// One pass over the box range of the stress faces (absolute indices 1..s+3
// on every axis).  Cells without reference maps (most of the box) get the
// pure fluid stress of their three lower faces: the nmaps = 0 path of
// face_stress written with the same expression ((1 - sfrac) * fs + ss with
// sfrac = ss = 0), in a small kernel that keeps many more threads resident
// than the full one.  Cells that hold any map are appended to list (when
// given) for the full stress kernel, one atomic per warp.
__global__ void k_stress_fluid(grid_dev g, const fields_dev *__restrict__ F, int *list, int *cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i > g.sm + 3 || j > g.sn + 3 || k > g.so + 3) return;
    const int ind = gidx(g, i, j, k);
    const bool any = map_mask(g, F, ind) != 0;
    if (list) {
        const unsigned act = __activemask();
        const unsigned maps = __ballot_sync(act, any);
        if (maps) {
            const int lane = threadIdx.x & 31;  // blockDim.x is a multiple of 32
            const int leader = __ffs(maps) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(cnt, __popc(maps));
            base = __shfl_sync(act, base, leader);
            if (any) list[base + __popc(maps & ((1u << lane) - 1))] = ind;
        }
    }
    if (any) return;
    const int strides[3] = {1, g.sm4, g.smn4};
    const double facs[3] = {g.dxsp, g.dysp, g.dzsp};
    const double sfrac = 0, ss = 0;
#pragma unroll
    for (int FF = 0; FF < 3; FF++) {
        const int strd = strides[FF];
        for (int nn = 0; nn < 3; nn++) {
            const double fs = g.mu * facs[FF] * (F->vel[nn][ind] - F->vel[nn][ind - strd]);
            F->sigma[3 * FF + nn][ind] = (1 - sfrac) * fs + ss;
        }
    }
}

// -------------------------------------------------------------------------
// Acceleration at a cell centre, fluid_3d::acceleration (fluid_3d.cc:980-1033)
// with neg_pres_grad (:2347-2361) and the sim_manager body/solid forces
// (Sim/sim_manager.cc:133-295).
// -------------------------------------------------------------------------
__device__ inline void solid_accel(const grid_dev &g, int o, const double rv[3], double x, double y, double z,
                                   double t, double &fx, double &fy, double &fz) {
    fx = fy = fz = 0;
    if (g.sim_type != 2) return;  // base sim_manager: no solid forces
    // sim_objects::solid_acceleration (sim_manager.cc:212-295) with the
    // average object velocities at their reset value 0 (no macro output)
    double krep = g.min_wall_acc;
    double phiv = obj_phi(g, o, rv[0], rv[1], rv[2]);
    const double h[3] = {g.dx, g.dy, g.dz};
    const double hs[3] = {g.dxsp, g.dysp, g.dzsp};
    const double pos[3] = {x, y, z};
    double f[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++) {
        // wall_trans_func(phiv, h, 1/h) (sim_manager.hh:281-285)
        double wt;
        if (phiv < -h[a]) wt = 1;
        else if (phiv < h[a]) wt = 0.5 * (1 - phiv * hs[a]);
        else wt = 0;
        if (g.walls[2 * a]) {
            double dist = pos[a] - g.wall_pos[2 * a];
            if (dist <= g.wall_dist) {
                double xx = dist * g.winv;
                double del = (xx <= 0) ? 100 : (1 - xx) / xx;
                f[a] += del * krep * wt;
            }
        }
        if (g.walls[2 * a + 1]) {
            double dist = g.wall_pos[2 * a + 1] - pos[a];
            if (dist <= g.wall_dist) {
                double xx = dist * g.winv;
                double del = (xx <= 0) ? 100 : (1 - xx) / xx;
                f[a] -= del * krep * wt;
            }
        }
    }
    fx = f[0];
    fy = f[1];
    fz = f[2];
    double f_norm = sqrt(fx * fx + fy * fy + fz * fz);
    if (f_norm >= g.K_stiff) {
        double nf = g.K_stiff / f_norm;
        fx *= nf;
        fy *= nf;
        fz *= nf;
    }
    // spheres have no anchors: dtoe1 = dtoe2 = 2 eps gives K = 0 (object.hh:62-64)
    double Kh = g.K_stiff * heaviside(g, 2 * g.eps) * heaviside(g, 2 * g.eps);
    fx -= Kh * 0;
    fy -= Kh * 0;
    fz -= Kh * 0;
    fz += g.gravity * heaviside(g, phiv);
}

__device__ inline void fluid_accel(const grid_dev &g, double x, double y, double z, double t, double &fx, double &fy,
                                   double &fz) {
    if (g.sim_type == 0) {  // sim_ftest::fluid_acceleration (sim_manager.cc:169-178)
        const double PI = 3.14159265358979323846;
        double mu = g.mu;
        fx = (12 * PI * cos(2 * PI * y) * cos(2 * PI * z) * (-6 * PI * mu * cos(2 * PI * t) + sin(2 * PI * t)) *
                  sin(2 * PI * x) +
              PI * cos(2 * PI * t) * cos(2 * PI * t) * (2 + cos(4 * PI * y) + cos(4 * PI * z)) * sin(4 * PI * x)) /
             4;
        fy = -(PI * cos(2 * PI * t) * cos(2 * PI * t) * (-1 + cos(4 * PI * x) - 2 * cos(4 * PI * z)) * sin(4 * PI * y)) * 0.125;
        fz = -(PI * cos(2 * PI * t) * cos(2 * PI * t) * (-1 + cos(4 * PI * x) - 2 * cos(4 * PI * y)) * sin(4 * PI * z)) * 0.125;
    } else if (g.sim_type == 2) {  // sim_objects: gravity (sim_manager.hh:400-404)
        fx = fy = 0;
        fz = 0;
        fz += g.gravity;
    } else {
        fx = fy = fz = 0;
    }
}

__device__ void acceleration(const grid_dev &g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                             const double *lz, int i, int j, int k, double t, bool var_den, double acc[3]) {
    const int ind = gidx(g, i, j, k);
    const int s1 = g.sm4, s2 = g.smn4;
    for (int c = 0; c < 3; c++) {
        const double *s0 = F->sigma[c], *sy = F->sigma[3 + c], *sz = F->sigma[6 + c];
        acc[c] += g.dxsp * (s0[ind + 1] - s0[ind]) + g.dysp * (sy[ind + s1] - sy[ind]) + g.dzsp * (sz[ind + s2] - sz[ind]);
    }
    // neg_pres_grad: -grad p from the 8 nodal pressures around the cell
    double pr[8];
    for (int n = 0; n < 8; n++) pr[n] = F->p[ind + n % 2 + s1 * ((n / 2) % 2) + (n / 4) * s2];
    double xa = 0, ya = 0, za = 0;
    for (int n = 0; n < 4; n++) {
        xa += pr[2 * n + 1] - pr[2 * n];
        int yi = (n / 2) * 4 + n % 2;
        ya += pr[yi + 2] - pr[yi];
        za += pr[n + 4] - pr[n];
    }
    xa *= -0.25 * g.dxsp;
    ya *= -0.25 * g.dysp;
    za *= -0.25 * g.dzsp;
    double tmp[3] = {xa, ya, za};
    for (int c = 0; c < 3; c++) {
        acc[c] += tmp[c];
        if (var_den) acc[c] /= F->rho[ind];
    }
    for (int c = 0; c < 3; c++) tmp[c] = 0.;
    double anc[3] = {0, 0, 0};
    double sfrac = 0;
    const double xx = lx[i], yy = ly[j], zz = lz[k];
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        if (m.code[ind] < 0) continue;
        double rv[3] = {m.x[0][ind], m.x[1][ind], m.x[2][ind]};
        double phiv = obj_phi(g, o, rv[0], rv[1], rv[2]);
        if (phiv < g.eps) {
            double lfrac = heaviside(g, phiv);
            solid_accel(g, o, rv, xx, yy, zz, t, anc[0], anc[1], anc[2]);
            for (int nn = 0; nn < 3; nn++) tmp[nn] += anc[nn];
            sfrac += lfrac;
        }
    }
    if (sfrac > 1.)
        for (int nn = 0; nn < 3; nn++) tmp[nn] /= sfrac;
    for (int nn = 0; nn < 3; nn++) acc[nn] += tmp[nn];
    if (sfrac < 1.) {
        fluid_accel(g, xx, yy, zz, t, anc[0], anc[1], anc[2]);
        for (int nn = 0; nn < 3; nn++) acc[nn] += anc[nn] * (1 - sfrac);
    }
}

// The six face states of a cell from its velocity, slopes and acceleration,
// FP64 in the reference's order of operations (fields.hh:147-177; halves as
// products, the same bits as the divisions).
__device__ __forceinline__ void edge_store_f64(const grid_dev &g, const fields_dev *__restrict__ F, int ind,
                                               const double (&vel)[3], const double (&nv)[3][3],
                                               const double (&acc)[3], double cdt) {
    const double dh2[3] = {g.dx * 0.5, g.dy * 0.5, g.dz * 0.5};
    const double dt2 = cdt * 0.5;
    double adv[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++) {
        for (int b = 0; b < 3; b++) adv[a] -= vel[b] * nv[b][a];
        adv[a] *= dt2;
    }
    for (int f = 0; f < 6; f++) {
        int dim = f / 2;
        double d = dh2[dim] * (2 * (f % 2) - 1);
        for (int c = 0; c < 3; c++) F->fvel[3 * f + c][ind] = vel[c] + d * nv[dim][c] + adv[c] + dt2 * acc[c];
    }
}
// The FP32 face states of the FP32-advection form (RMT3D_MIXED_BULK32): the
// same formula in FP32 with fused
// multiply-adds (the acceleration is formed in FP64 and rounded once).
__device__ __forceinline__ void edge_store_f32(const grid_dev &g, const fields_dev *__restrict__ F, int ind,
                                               const float (&vel)[3], const float (&nv)[3][3],
                                               const double (&acc)[3], double cdt) {
    const float dh2[3] = {(float)(g.dx * 0.5), (float)(g.dy * 0.5), (float)(g.dz * 0.5)};
    const float dt2 = (float)(cdt * 0.5);
    float base[3];
    for (int a = 0; a < 3; a++) {
        float adv = 0.f;
        for (int b = 0; b < 3; b++) adv = fmaf(-vel[b], nv[b][a], adv);
        base[a] = vel[a] + fmaf(adv, dt2, (float)(cdt * 0.5 * acc[a]));
    }
    for (int f = 0; f < 6; f++) {
        int dim = f / 2;
        float d = (f % 2) ? dh2[dim] : -dh2[dim];
        for (int c = 0; c < 3; c++) F->fvel32[3 * f + c][ind] = fmaf(d, nv[dim][c], base[c]);
    }
}

// -------------------------------------------------------------------------
// Limited slopes + half-step edge extrapolation of the velocity:
// normal_derivatives_velocity (fluid_3d.cc:582-617) fused with
// compute_half_time_edge_velocities (:1038-1066) and field::godunov_extrap
// (fields.hh:147-177, non-TANG branch).  Interior cells.
// -------------------------------------------------------------------------
template <typename FT>
__global__ void __launch_bounds__(256, 3) k_edge_vel(grid_dev g, const fields_dev *__restrict__ F, const double *lx,
                                                     const double *ly, const double *lz, double cdt,
                                                     const double *time_p, int var_den) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const double time = *time_p;  // device-resident simulation time
    const int ind = gidx(g, i, j, k);
    const int strides[3] = {1, g.sm4, g.smn4};
    if constexpr (sizeof(FT) == 8) {
        const double dhsp[3] = {g.dxsp, g.dysp, g.dzsp};
        double nv[3][3];
        double vel[3];
        for (int c = 0; c < 3; c++) vel[c] = F->vel[c][ind];
        for (int d = 0; d < 3; d++) {
            int s = strides[d];
            for (int c = 0; c < 3; c++) {
                const double *u = F->vel[c];
                nv[d][c] = dhsp[d] * mono_diff(u[ind - 2 * s], u[ind - s], u[ind], u[ind + s], u[ind + 2 * s]);
            }
        }
        double acc[3] = {0, 0, 0};
        acceleration(g, F, lx, ly, lz, i, j, k, time, var_den != 0, acc);
        edge_store_f64(g, F, ind, vel, nv, acc, cdt);
    } else {
        const float dhsp[3] = {(float)g.dxsp, (float)g.dysp, (float)g.dzsp};
        float nv[3][3];
        float vel[3];
        for (int c = 0; c < 3; c++) vel[c] = (float)F->vel[c][ind];
        for (int d = 0; d < 3; d++) {
            int s = strides[d];
            for (int c = 0; c < 3; c++) {
                const double *u = F->vel[c];
                nv[d][c] = dhsp[d] * mono_diff_f((float)u[ind - 2 * s], (float)u[ind - s], vel[c], (float)u[ind + s],
                                                 (float)u[ind + 2 * s]);
            }
        }
        double acc[3] = {0, 0, 0};
        acceleration(g, F, lx, ly, lz, i, j, k, time, var_den != 0, acc);
        edge_store_f32(g, F, ind, vel, nv, acc, cdt);
    }
}
template __global__ void k_edge_vel<double>(grid_dev, const fields_dev *__restrict__, const double *, const double *,
                                            const double *, double, const double *, int);
template __global__ void k_edge_vel<float>(grid_dev, const fields_dev *__restrict__, const double *, const double *,
                                           const double *, double, const double *, int);

// -------------------------------------------------------------------------
// The same computation with the velocity staged through TMA.  A block owns
// 32 x 8 cells in x, y and a chunk of planes in z; the planes of u, v, w with
// a halo of two cells in x and y stream through a ring of shared-memory
// planes, each plane brought in by three tiled bulk-tensor copies
// (cp.async.bulk.tensor, one per component) that complete on the plane's
// mbarrier.  Three planes ahead of the one being computed are in flight.
// Each cell's slopes read the five-point lines of the velocity from the ring
// -- the operands k_edge_vel reads from global memory, in the same order --
// so the face states are bit-identical.  The rest (stress divergence,
// pressure gradient, body and solid forces) reads global memory as before.
// The tensor maps cover the scene's own velocity arrays (no multicast).
// -------------------------------------------------------------------------
constexpr int kEvX = 32, kEvY = 8, kEvW = kEvX + 4, kEvH = kEvY + 4, kEvRing = 6;
constexpr unsigned kEvPlaneBytes = kEvW * kEvH * sizeof(double);  // one component of one plane

__device__ __forceinline__ void ev_mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"((unsigned)__cvta_generic_to_shared(bar)) : "memory");
}
// thread 0: expect the three copies of a plane and start them
__device__ __forceinline__ void ev_fetch(uint64_t *bar, double *dst, const CUtensorMap *tm0, const CUtensorMap *tm1,
                                         const CUtensorMap *tm2, int x, int y, int z) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(3 * kEvPlaneBytes) : "memory");
    const CUtensorMap *tms[3] = {tm0, tm1, tm2};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + c * kEvW * kEvH);
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
            ::"r"(d), "l"((unsigned long long)tms[c]), "r"(x), "r"(y), "r"(z), "r"(b)
            : "memory");
    }
}
// bounded wait for a phase of a plane's mbarrier: false if it did not
// complete within the limit (the copies are of valid global memory, so this
// does not happen; the bound keeps a fault from turning into a hang)
__device__ __forceinline__ bool ev_wait(uint64_t *bar, unsigned parity) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    for (int it = 0; it < (1 << 22); it++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(b), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

template <typename FT>
__global__ void __launch_bounds__(256, 2) k_edge_vel_tma(grid_dev g, const fields_dev *__restrict__ F,
                                                         const __grid_constant__ CUtensorMap tmu,
                                                         const __grid_constant__ CUtensorMap tmv,
                                                         const __grid_constant__ CUtensorMap tmw, const double *lx,
                                                         const double *ly, const double *lz, double cdt,
                                                         const double *time_p, int var_den, int tz, int *err) {
    extern __shared__ __align__(128) unsigned char ev_smem[];
    double *ring = reinterpret_cast<double *>(ev_smem);  // [kEvRing][3][kEvH][kEvW]
    uint64_t *bar = reinterpret_cast<uint64_t *>(ev_smem + (size_t)kEvRing * 3 * kEvPlaneBytes);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool lead = tx == 0 && ty == 0;
    const int i0 = 2 + kEvX * blockIdx.x, j0 = 2 + kEvY * blockIdx.y;
    const int k0 = 2 + tz * blockIdx.z, k1 = min(k0 + tz, g.so + 2);  // interior planes [k0, k1)
    const int p0 = k0 - 2, p1 = k1 + 1;                             // planes staged [p0, p1]
    if (lead) {
        for (int q = 0; q < kEvRing; q++) ev_mbar_init(bar + q);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    auto slot = [&](int p) { return (p - p0) % kEvRing; };
    auto fetch = [&](int p) {
        ev_fetch(bar + slot(p), ring + (size_t)slot(p) * 3 * kEvW * kEvH, &tmu, &tmv, &tmw, i0 - 2, j0 - 2, p);
    };
    // prologue: the five planes of the first cell plane and one more
    if (lead)
        for (int p = p0; p <= min(p0 + 5, p1); p++) fetch(p);
    const int i = i0 + tx, j = j0 + ty;
    const bool mine = i < g.sm + 2 && j < g.sn + 2;
    const double time = *time_p;  // device-resident simulation time
    bool ok = true;
    for (int k = k0; k < k1; k++) {
        // planes k-2 .. k+2 have landed (k+2 is the newest one needed)
        for (int p = (k == k0 ? p0 : k + 2); p <= k + 2 && ok; p++) ok = ev_wait(bar + slot(p), ((p - p0) / kEvRing) & 1);
        if (!ok) break;
        if (mine) {
            const int ind = gidx(g, i, j, k);
            const int o = (ty + 2) * kEvW + (tx + 2);
            const double *pl[5];
#pragma unroll
            for (int d = 0; d < 5; d++) pl[d] = ring + (size_t)slot(k - 2 + d) * 3 * kEvW * kEvH;
            if constexpr (sizeof(FT) == 8) {
                const double dhsp[3] = {g.dxsp, g.dysp, g.dzsp};
                double nv[3][3];
                double vel[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double *u2 = pl[2] + c * kEvW * kEvH;
                    vel[c] = u2[o];
                    nv[0][c] = dhsp[0] * mono_diff(u2[o - 2], u2[o - 1], u2[o], u2[o + 1], u2[o + 2]);
                    nv[1][c] = dhsp[1] * mono_diff(u2[o - 2 * kEvW], u2[o - kEvW], u2[o], u2[o + kEvW], u2[o + 2 * kEvW]);
                    nv[2][c] = dhsp[2] * mono_diff(pl[0][c * kEvW * kEvH + o], pl[1][c * kEvW * kEvH + o], u2[o],
                                                   pl[3][c * kEvW * kEvH + o], pl[4][c * kEvW * kEvH + o]);
                }
                double acc[3] = {0, 0, 0};
                acceleration(g, F, lx, ly, lz, i, j, k, time, var_den != 0, acc);
                edge_store_f64(g, F, ind, vel, nv, acc, cdt);
            } else {
                const float dhsp[3] = {(float)g.dxsp, (float)g.dysp, (float)g.dzsp};
                float nv[3][3];
                float vel[3];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const double *u2 = pl[2] + c * kEvW * kEvH;
                    vel[c] = (float)u2[o];
                    nv[0][c] = dhsp[0] * mono_diff_f((float)u2[o - 2], (float)u2[o - 1], vel[c], (float)u2[o + 1],
                                                     (float)u2[o + 2]);
                    nv[1][c] = dhsp[1] * mono_diff_f((float)u2[o - 2 * kEvW], (float)u2[o - kEvW], vel[c],
                                                     (float)u2[o + kEvW], (float)u2[o + 2 * kEvW]);
                    nv[2][c] = dhsp[2] * mono_diff_f((float)pl[0][c * kEvW * kEvH + o], (float)pl[1][c * kEvW * kEvH + o],
                                                     vel[c], (float)pl[3][c * kEvW * kEvH + o],
                                                     (float)pl[4][c * kEvW * kEvH + o]);
                }
                double acc[3] = {0, 0, 0};
                acceleration(g, F, lx, ly, lz, i, j, k, time, var_den != 0, acc);
                edge_store_f32(g, F, ind, vel, nv, acc, cdt);
            }
        }
        // every thread is done with plane k-2: its slot takes plane k+4
        __syncthreads();
        if (lead && k + 4 <= p1) fetch(k + 4);
    }
    if (!ok && tx == 0 && ty == 0) atomicAdd(err, 1);
    // no copy is left in flight: every fetched plane was waited for, or the
    // block gave up on a wait (recorded above); let outstanding copies land
    // before the shared memory goes away
    if (!ok)
        for (int p = p0; p <= p1; p++) ev_wait(bar + slot(p), ((p - p0) / kEvRing) & 1);
}

size_t edge_vel_tma_smem() { return (size_t)kEvRing * 3 * kEvPlaneBytes + kEvRing * sizeof(uint64_t); }

// Tiled tensor map of one velocity array (the ghosted box, FP64) for
// k_edge_vel_tma: box of kEvW x kEvH x 1 elements.  Needs 16-byte row
// strides (sm + 4 even).  Returns false if the map cannot be made.
bool edge_vel_tensor_map(const grid_dev &g, const double *base, CUtensorMap *out) {
    if ((g.sm4 * sizeof(double)) % 16 != 0 || ((uintptr_t)base) % 16 != 0) return false;
    typedef CUresult (*encode_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static encode_fn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            return false;
        fn = (encode_fn)p;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.sm4, (cuuint64_t)g.sn4, (cuuint64_t)g.so4};
    const cuuint64_t strides[2] = {(cuuint64_t)g.sm4 * sizeof(double), (cuuint64_t)g.smn4 * sizeof(double)};
    const cuuint32_t box[3] = {kEvW, kEvH, 1}, estr[3] = {1, 1, 1};
    return fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// launch of k_edge_vel_tma over the interior: z chunks of tz planes
void launch_edge_vel_tma(const grid_dev &g, const fields_dev *F, const CUtensorMap tm[3], const double *lx,
                         const double *ly, const double *lz, double cdt, const double *time_p, int var_den, int *err,
                         cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_edge_vel_tma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)edge_vel_tma_smem());
        cudaFuncSetAttribute(k_edge_vel_tma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)edge_vel_tma_smem());
        attr = true;
    }
    const int tx = (g.sm + kEvX - 1) / kEvX, ty = (g.sn + kEvY - 1) / kEvY;
    // z chunks for about 8 blocks per SM (two resident, four waves): a
    // block's planes are a serial pipeline, so many short chunks keep more
    // planes in flight than a few long ones; at least 2 planes each
    int nz = (8 * 148 + tx * ty - 1) / (tx * ty);
    nz = nz < 1 ? 1 : (nz > (g.so + 1) / 2 ? (g.so + 1) / 2 : nz);
    const int tz = (g.so + nz - 1) / nz;
    const dim3 grid(tx, ty, (g.so + tz - 1) / tz);
    if (g.f32face)
        k_edge_vel_tma<float><<<grid, dim3(kEvX, kEvY), edge_vel_tma_smem(), st>>>(g, F, tm[0], tm[1], tm[2], lx, ly,
                                                                                  lz, cdt, time_p, var_den, tz, err);
    else
        k_edge_vel_tma<double><<<grid, dim3(kEvX, kEvY), edge_vel_tma_smem(), st>>>(g, F, tm[0], tm[1], tm[2], lx, ly,
                                                                                   lz, cdt, time_p, var_den, tz, err);
}

// -------------------------------------------------------------------------
// Godunov upwinding on every upper face from relative index -1,
// fluid_3d::godunov_upwinding_set (fluid_3d.cc:811-944) with
// godunov_set_velocity (:2156-2176) and godunov_set_refmap (:2184-2204).
// The reference-map pairs are upwinded first, with the fluid states still
// unmodified, exactly as the reference's per-cell loop does.
// -------------------------------------------------------------------------
__device__ inline void set_refmap(double norml, double normr, double &ml, double &vl, double &wl, double &mr,
                                  double &vr, double &wr) {
    if (norml + normr > 0 && norml > 0) {
        mr = ml;
        vr = vl;
        wr = wl;
    } else if (norml + normr < 0 && normr < 0) {
        ml = mr;
        vl = vr;
        wl = wr;
    } else {
        double t = 0.5 * (ml + mr);
        ml = mr = t;
        t = 0.5 * (vl + vr);
        vl = vr = t;
        t = 0.5 * (wl + wr);
        wl = wr = t;
    }
}

template <typename FT>
__global__ void k_upwind(grid_dev g, const fields_dev *__restrict__ F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const int ind = gidx(g, i, j, k);
    const int strides[3] = {1, g.sm4, g.smn4};
    for (unsigned mk = map_mask(g, F, ind); mk; mk &= mk - 1) {
        const int o = __ffs(mk) - 1;
        const objmap_dev &m = F->om[o];
        bool go = (m.code[ind] == 0);
        if (!go) {  // an extrapolated map with a primary neighbour on its upper side (neigh_inside)
            for (int d = 0; d < 3 && !go; d++)
                if (m.code[ind + strides[d]] == 0) go = true;
        }
        if (!go) continue;
        for (int dir = 0; dir < 3; dir++) {
            const int nb = ind + strides[dir];
            const int ff = 2 * dir + 1, nf = ff ^ 1;
            const int a1 = (dir + 1) % 3, a2 = (dir + 2) % 3;
            const double norml = face_ptr<FT>(F, 3 * ff + dir)[ind], normr = face_ptr<FT>(F, 3 * nf + dir)[nb];
            double ml = m.fx[3 * ff + dir][ind], vl = m.fx[3 * ff + a1][ind], wl = m.fx[3 * ff + a2][ind];
            double mr = m.fx[3 * nf + dir][nb], vr = m.fx[3 * nf + a1][nb], wr = m.fx[3 * nf + a2][nb];
            set_refmap(norml, normr, ml, vl, wl, mr, vr, wr);
            m.fx[3 * ff + dir][ind] = ml;
            m.fx[3 * ff + a1][ind] = vl;
            m.fx[3 * ff + a2][ind] = wl;
            m.fx[3 * nf + dir][nb] = mr;
            m.fx[3 * nf + a1][nb] = vr;
            m.fx[3 * nf + a2][nb] = wr;
        }
    }
    for (int dir = 0; dir < 3; dir++) {
        const int nb = ind + strides[dir];
        const int ff = 2 * dir + 1, nf = ff ^ 1;
        const int a1 = (dir + 1) % 3, a2 = (dir + 2) % 3;
        FT *const fl[3] = {face_ptr<FT>(F, 3 * ff + dir), face_ptr<FT>(F, 3 * ff + a1), face_ptr<FT>(F, 3 * ff + a2)};
        FT *const fr[3] = {face_ptr<FT>(F, 3 * nf + dir), face_ptr<FT>(F, 3 * nf + a1), face_ptr<FT>(F, 3 * nf + a2)};
        FT nl = fl[0][ind], vl = fl[1][ind], wl = fl[2][ind];
        FT nr = fr[0][nb], vr = fr[1][nb], wr = fr[2][nb];
        if (nl + nr > 0 && nl > 0) {
            nr = nl;
            vr = vl;
            wr = wl;
        } else if (nl + nr < 0 && nr < 0) {
            nl = nr;
            vl = vr;
            wl = wr;
        } else {
            nl = nr = 0;
            FT t = (FT)0.5 * (vl + vr);
            vl = vr = t;
            t = (FT)0.5 * (wl + wr);
            wl = wr = t;
        }
        fl[0][ind] = nl;
        fl[1][ind] = vl;
        fl[2][ind] = wl;
        fr[0][nb] = nr;
        fr[1][nb] = vr;
        fr[2][nb] = wr;
    }
}
template __global__ void k_upwind<double>(grid_dev, const fields_dev *__restrict__);
template __global__ void k_upwind<float>(grid_dev, const fields_dev *__restrict__);

// -------------------------------------------------------------------------
// MAC projection: rhs (fill_mac_rhs, fluid_3d.cc:2244-2265), solution
// extraction (:2268-2281) and face correction (subtract_q_grad, :2284-2304).
// -------------------------------------------------------------------------
__global__ void k_mac_rhs(grid_dev g, const fields_dev *__restrict__ F, double *r, double cdt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.sm || j >= g.sn || k >= g.so) return;
    const int ind = gidx(g, i + 2, j + 2, k + 2);
    const double fac = g.dx / (2 * cdt);
    double s = 0;
    for (int f = 0; f < 3; f++) s += fac * (face_ld(g, F, 3 * (2 * f + 1) + f, ind) - face_ld(g, F, 3 * (2 * f) + f, ind));
    r[i + g.sm * (j + g.sn * k)] = s;
}

__global__ void k_mac_extract(grid_dev g, const fields_dev *__restrict__ F, const double *x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i >= g.sm || j >= g.sn || k >= g.so) return;
    F->q[gidx(g, i + 2, j + 2, k + 2)] = x[i + g.sm * (j + g.sn * k)];
}

__global__ void k_sub_qgrad(grid_dev g, const fields_dev *__restrict__ F, double cdt, int var_den) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const int ind = gidx(g, i, j, k);
    const int strides[3] = {1, g.sm4, g.smn4};
    const double fac = 2 * cdt * g.dxsp;
    const double *q = F->q;
    for (int f = 0; f < 3; f++) {
        int s = strides[f];
        double down, up;
        if (var_den) {
            const double *rho = F->rho;
            down = fac * (q[ind] - q[ind - s]) / (0.5 * (rho[ind] + rho[ind - s]));
            up = fac * (q[ind + s] - q[ind]) / (0.5 * (rho[ind + s] + rho[ind]));
        } else {
            down = fac * (q[ind] - q[ind - s]);
            up = fac * (q[ind + s] - q[ind]);
        }
        face_st(g, F, 3 * (2 * f) + f, ind, face_ld(g, F, 3 * (2 * f) + f, ind) - down);
        face_st(g, F, 3 * (2 * f + 1) + f, ind, face_ld(g, F, 3 * (2 * f + 1) + f, ind) - up);
    }
}

// -------------------------------------------------------------------------
// Explicit momentum update, fluid_3d::compute_ustar (fluid_3d.cc:1309-1352).
// -------------------------------------------------------------------------
template <typename FT>
__global__ void __launch_bounds__(256, 3) k_ustar(grid_dev g, const fields_dev *__restrict__ F, const double *lx,
                                                  const double *ly, const double *lz, double cdt,
                                                  const double *time_p, int var_den) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const double time = *time_p;  // device-resident simulation time
    const int ind = gidx(g, i, j, k);
    double acc[3] = {0, 0, 0};
    acceleration(g, F, lx, ly, lz, i, j, k, time, var_den != 0, acc);
    FT fv[18];
    for (int a = 0; a < 18; a++) fv[a] = face_ptr<FT>(F, a)[ind];
    double dv[3];
    if constexpr (sizeof(FT) == 8) {
        double avgs[3];
        avgs[0] = -0.5 * cdt * (fv[0] + fv[3]) * g.dxsp;
        avgs[1] = -0.5 * cdt * (fv[3 * 2 + 1] + fv[3 * 3 + 1]) * g.dysp;
        avgs[2] = -0.5 * cdt * (fv[3 * 4 + 2] + fv[3 * 5 + 2]) * g.dzsp;
        for (int d = 0; d < 3; d++) {
            dv[d] = avgs[0] * (fv[3 + d] - fv[d]) + avgs[1] * (fv[9 + d] - fv[6 + d]) + avgs[2] * (fv[15 + d] - fv[12 + d]);
            acc[d] *= cdt;
        }
        for (int d = 0; d < 3; d++) dv[d] += acc[d];
    } else {
        // the FP32-advection form: the advective increment in FP32 from the FP32 face
        // states, added to the FP64 velocity with the FP64 acceleration term
        const float hdt = (float)(-0.5 * cdt);
        const float avgs[3] = {hdt * (fv[0] + fv[3]) * (float)g.dxsp, hdt * (fv[3 * 2 + 1] + fv[3 * 3 + 1]) * (float)g.dysp,
                               hdt * (fv[3 * 4 + 2] + fv[3 * 5 + 2]) * (float)g.dzsp};
        for (int d = 0; d < 3; d++) {
            float t = avgs[0] * (fv[3 + d] - fv[d]);
            t = fmaf(avgs[1], fv[9 + d] - fv[6 + d], t);
            t = fmaf(avgs[2], fv[15 + d] - fv[12 + d], t);
            dv[d] = (double)t + acc[d] * cdt;
        }
    }
    for (int d = 0; d < 3; d++) {
        double dd = 0.;
        dd += dv[d];
        F->dvel[d][ind] = dd;
        F->vel[d][ind] += dd;
    }
}
template __global__ void k_ustar<double>(grid_dev, const fields_dev *__restrict__, const double *, const double *,
                                         const double *, double, const double *, int);
template __global__ void k_ustar<float>(grid_dev, const fields_dev *__restrict__, const double *, const double *,
                                        const double *, double, const double *, int);

// -------------------------------------------------------------------------
// FEM projection right-hand side, fluid_3d::fill_pp_rhs (fluid_3d.cc:
// 2554-2649), written as a gather over the (up to) eight elements around each
// node in the reference's element order, followed by the domain-face flux
// terms in face order.  One thread per FEM node.
// -------------------------------------------------------------------------
__device__ inline bool elem_in_domain(const grid_dev &g, int ei, int ej, int ek) {
    return (g.prd[0] || (ei >= 0 && ei <= g.sm - 1)) && (g.prd[1] || (ej >= 0 && ej <= g.sn - 1)) &&
           (g.prd[2] || (ek >= 0 && ek <= g.so - 1));
}

__global__ void k_fem_rhs(grid_dev g, const fields_dev *__restrict__ F, double *r, gradphi_t gp) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    int b = blockIdx.y * blockDim.y + threadIdx.y;
    int c = blockIdx.z * blockDim.z + threadIdx.z;
    if (a >= g.fm || b >= g.fn || c >= g.fo) return;
    double s = 0;
    // element (ei,ej,ek) touches node (a,b,c) as local node (a-ei)+2(b-ej)+4(c-ek)
    for (int ek = c - 1; ek <= c; ek++)
        for (int ej = b - 1; ej <= b; ej++)
            for (int ei = a - 1; ei <= a; ei++) {
                if (ei < -1 || ej < -1 || ek < -1) continue;
                if (ei > g.fm - 1 || ej > g.fn - 1 || ek > g.fo - 1) continue;
                if (!elem_in_domain(g, ei, ej, ek)) continue;
                const int n = (a - ei) + 2 * (b - ej) + 4 * (c - ek);
                const int ind = gidx(g, ei + 2, ej + 2, ek + 2);
                double val = 0;
                for (int l = 0; l < 3; l++) val += F->dvel[l][ind] * gp.v[n][l];
                s += val;
            }
    // domain-face flux terms of non-periodic faces (fluid_3d.cc:2585-2645)
    const int node[3] = {a, b, c};
    const int fdim[3] = {g.fm, g.fn, g.fo};
    for (int face = 0; face < 6; face++) {
        const int nd = face / 2;
        if (g.prd[nd]) continue;
        const int side = face % 2;
        // nodes on this face: node[nd] == 0 (lower) or == len (upper)
        if (node[nd] != (side ? fdim[nd] - 1 : 0)) continue;
        const int t0 = (nd == 0) ? 1 : 0, t1 = (nd == 2) ? 1 : 2;
        // boundary cells around the node in the reference's loop order
        for (int c1 = node[t1] - 1; c1 <= node[t1]; c1++)
            for (int c0 = node[t0] - 1; c0 <= node[t0]; c0++) {
                int e[3];
                e[nd] = side ? fdim[nd] - 2 : 0;
                e[t0] = c0;
                e[t1] = c1;
                if (e[t0] < -1 || e[t1] < -1) continue;
                const int lens[3] = {g.sm, g.sn, g.so};
                if (e[t0] > lens[t0] || e[t1] > lens[t1]) continue;
                if (!elem_in_domain(g, e[0], e[1], e[2])) continue;
                int inds[3];
                inds[nd] = side;
                inds[t0] = node[t0] - e[t0];
                inds[t1] = node[t1] - e[t1];
                // node validity as in map_ref_to_local
                bool ok = true;
                for (int d = 0; d < 3; d++) {
                    int nn = e[d] + inds[d];
                    if (nn > fdim[d] - 1) ok = false;
                    if (e[d] < 0 && inds[d] == 0) ok = false;
                }
                if (!ok) continue;
                const int lid = inds[0] + 2 * inds[1] + 4 * inds[2];
                const int cell = gidx(g, e[0] + 2, e[1] + 2, e[2] + 2);
                double val = -face_ld(g, F, 3 * face + nd, cell) * gp.v[lid][nd];
                s += val;
            }
    }
    r[a + g.fm * (b + g.fn * c)] = s;
}

// p += x - mean, dp = x - mean over FEM nodes (extract_pp_soln, :2685-2712)
__global__ void k_fem_extract(grid_dev g, const fields_dev *__restrict__ F, const double *x, const double *mean) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    int b = blockIdx.y * blockDim.y + threadIdx.y;
    int c = blockIdx.z * blockDim.z + threadIdx.z;
    if (a >= g.fm || b >= g.fn || c >= g.fo) return;
    const double m = *mean;
    const double v = x[a + g.fm * (b + g.fn * c)];
    const int ind = gidx(g, a + 2, b + 2, c + 2);
    F->p[ind] += (v - m);
    F->dp[ind] = (v - m);
}

// u, dvel -= dt grad(dp), subtract_pres_grad (:2717-2753) with neg_pres_dgrad
__global__ void k_sub_pgrad(grid_dev g, const fields_dev *__restrict__ F, double dt, int var_den) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const int ind = gidx(g, i, j, k);
    const int s1 = g.sm4, s2 = g.smn4;
    double pr[8];
    for (int n = 0; n < 8; n++) pr[n] = F->dp[ind + n % 2 + s1 * ((n / 2) % 2) + (n / 4) * s2];
    double xa = 0, ya = 0, za = 0;
    for (int n = 0; n < 4; n++) {
        xa += pr[2 * n + 1] - pr[2 * n];
        int yi = (n / 2) * 4 + n % 2;
        ya += pr[yi + 2] - pr[yi];
        za += pr[n + 4] - pr[n];
    }
    xa *= -0.25 * g.dxsp;
    ya *= -0.25 * g.dysp;
    za *= -0.25 * g.dzsp;
    double npg[3] = {xa, ya, za};
    for (int c = 0; c < 3; c++) {
        if (var_den) npg[c] *= dt / F->rho[ind];
        else npg[c] *= dt;
        F->vel[c][ind] += npg[c];
        F->dvel[c][ind] += npg[c];
    }
}

}  // namespace rmt3d
