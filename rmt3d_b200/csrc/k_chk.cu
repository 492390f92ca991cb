// Checkpoint slices (F3D_Source/fluid_3d_chk_pt.cc, fluid_3d_io.cc) packed
// and unpacked on the device.  A packed checkpoint is kChkFields blocks (vx,
// vy, vz, p, X, Y, Z, OID) of so slices of (sm+1)(sn+1) doubles each: the
// reference's per-slice buffer u_global, in file order.
#include "kernels.h"

namespace rmt3d {

// One thread per (slice k, buffer position). Cell fields fill positions
// i + sm*j (i < sm, j < sn), the pressure the nodal positions i + fm*j
// (i < fm, j < fn), as the reference's slice gather does (fluid_3d_io.cc:
// 98-255, 479-505).  Its one buffer is reused across slices and fields in
// the order vx, vy, vz, p, X, ..., so positions a field does not write keep
// what the previous writer left: zeros before the pressure, the last
// pressure slice after it.  Maps take the least level set among the
// primary and extrapolated maps of the cell (min_phi_id, :420-434; strict
// '<', extrapolated maps in object order); X/Y/Z are 100 and OID 0 where a
// cell has none, and OID is 0 where the least is an extrapolated map
// (:387-400).
__global__ void k_chk_pack(grid_dev g, const fields_dev *__restrict__ F, double *__restrict__ buf) {
    const int m = g.sm, n = g.sn, o = g.so;
    const long L = (long)(m + 1) * (n + 1);
    const long per = L * o;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < per; t += (long)gridDim.x * blockDim.x) {
        const int k = (int)(t / L);
        const int pos = (int)(t - (long)k * L);
        const bool in_c = pos < m * n;
        const bool in_p = pos < g.fm * g.fn;
        const int ip = pos % g.fm, jp = pos / g.fm;
        double v[8];
        v[3] = in_p ? F->p[gidx(g, ip + 2, jp + 2, k + 2)] : 0.;
        if (in_c) {
            const int ind = gidx(g, pos % m + 2, pos / m + 2, k + 2);
            for (int c = 0; c < 3; c++) v[c] = F->vel[c][ind];
            int prim = -1;
            for (int ob = 0; ob < g.n_obj; ob++)
                if (F->om[ob].code[ind] == 0) prim = ob;
            int best = prim;
            double mphi = 1e30;
            if (prim >= 0) {
                const objmap_dev &mp = F->om[prim];
                mphi = obj_phi(g, prim, mp.x[0][ind], mp.x[1][ind], mp.x[2][ind]);
            }
            for (int ob = 0; ob < g.n_obj; ob++) {
                const objmap_dev &me = F->om[ob];
                if (me.code[ind] <= 0) continue;
                const double tphi = obj_phi(g, ob, me.x[0][ind], me.x[1][ind], me.x[2][ind]);
                if (tphi < mphi) {
                    mphi = tphi;
                    best = ob;
                }
            }
            if (best < 0) {
                v[4] = v[5] = v[6] = 100.;
                v[7] = 0.;
            } else {
                const objmap_dev &mb = F->om[best];
                for (int a = 0; a < 3; a++) v[4 + a] = mb.x[a][ind];
                v[7] = (best == prim) ? (double)(prim + 1) : 0.;
            }
        } else {
            v[0] = v[1] = v[2] = 0.;
            const double tail = in_p ? F->p[gidx(g, ip + 2, jp + 2, o - 1 + 2)] : 0.;
            v[4] = v[5] = v[6] = v[7] = tail;
        }
        for (int f = 0; f < 8; f++) buf[f * per + t] = v[f];
    }
}

// One thread per cell of the ghosted box: the state of a freshly
// constructed fluid_3d after copy_chk_to_field (fluid_3d_chk_pt.cc:318-351).
// Interior cells take velocities and maps (x = xpred = X, owner = OID); the
// pressure takes the nodal points of slices k < so, each row read with the
// cell stride sm as the reference's copy_chk_slice_to_buf does (:303-316).
// Every other value is the constructor's: zero, no map, grad_phi unset.
// An OID that names no object is counted in *bad.
__global__ void k_chk_unpack(grid_dev g, const fields_dev *__restrict__ F, const double *__restrict__ buf, int *bad) {
    const int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    const int m = g.sm, n = g.sn, o = g.so;
    const long L = (long)(m + 1) * (n + 1);
    const long per = L * o;
    const int i = ind % g.sm4 - 2, j = (ind / g.sm4) % g.sn4 - 2, k = ind / g.smn4 - 2;
    const bool interior = i >= 0 && i < m && j >= 0 && j < n && k >= 0 && k < o;
    double X[3] = {0, 0, 0};
    int owner = -1;
    if (interior) {
        const long base = (long)k * L + i + (long)m * j;
        for (int c = 0; c < 3; c++) F->vel[c][ind] = buf[c * per + base];
        for (int a = 0; a < 3; a++) X[a] = buf[(4 + a) * per + base];
        const double id = buf[7 * per + base];
        if (id != 0.) {
            if (id >= 1. && id <= (double)g.n_obj && id == floor(id)) owner = (int)id - 1;
            else atomicAdd(bad, 1);
        }
    } else {
        for (int c = 0; c < 3; c++) F->vel[c][ind] = 0.;
    }
    const bool node = i >= 0 && i < g.fm && j >= 0 && j < g.fn && k >= 0 && k < o;
    F->p[ind] = node ? buf[3 * per + (long)k * L + i + (long)m * j] : 0.;
    for (int ob = 0; ob < g.n_obj; ob++) {
        const objmap_dev &mm = F->om[ob];
        mm.code[ind] = (owner == ob) ? 0 : -1;
        for (int a = 0; a < 3; a++) {
            mm.x[a][ind] = X[a];
            mm.xp[a][ind] = X[a];
            mm.det[a][ind] = 0.;
            mm.el[a][ind] = 0.;
        }
        for (int a = 0; a < 9; a++) mm.gp[a][ind] = -kBig;
        for (int a = 0; a < 18; a++) mm.fx[a][ind] = 0.;
    }
}

}  // namespace rmt3d
