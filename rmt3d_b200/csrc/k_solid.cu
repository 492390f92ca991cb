// Solid-side kernels: reference-map advection (slopes, half-step face states,
// predictor / corrector), the layer-by-layer least-squares extrapolation of
// the reference map across the interface, and the boundary redraw.
#include "dev_common.cuh"
#include "solid.h"

namespace rmt3d {

__device__ inline double mphi(const grid_dev &g, const objmap_dev &m, int o, int ind) {
    return obj_phi(g, o, m.x[0][ind], m.x[1][ind], m.x[2][ind]);
}

// -------------------------------------------------------------------------
// normal_derivatives_refmap (fluid_3d.cc:621-806) fused with
// compute_half_time_edge_refmap (:1071-1100) and ref_map::godunov_extrap
// (fields.hh:572-592, non-TANG): for the primary map of every interior cell
// and for extrapolated maps that abut a primary map orthogonally.
// -------------------------------------------------------------------------
__global__ void __launch_bounds__(256, 3) k_edge_refmap(grid_dev g, const fields_dev *__restrict__ F, double cdt, int *err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const int ind = gidx(g, i, j, k);
    const int strides[3] = {1, g.sm4, g.smn4};
    const double dhsp[3] = {g.dxsp, g.dysp, g.dzsp};
    // halves as products (the same bits as the divisions, far fewer instructions)
    const double dh2[3] = {g.dx * 0.5, g.dy * 0.5, g.dz * 0.5};
    const double dt2 = cdt * 0.5;
    double vel[3];
    for (int c = 0; c < 3; c++) vel[c] = F->vel[c][ind];
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        int cd = m.code[ind];
        if (cd < 0) continue;
        if (cd > 0) {  // ref_map::abut_primary (fields.hh:466-477)
            bool ab = false;
            for (int d = 0; d < 3 && !ab; d++)
                if (m.code[ind + strides[d]] == 0 || m.code[ind - strides[d]] == 0) ab = true;
            if (!ab) continue;
        }
        double nv[3][3];
        for (int d = 0; d < 3; d++) {
            int s = strides[d];
            int q[5] = {ind - 2 * s, ind - s, ind, ind + s, ind + 2 * s};
            if (m.code[q[0]] < 0 || m.code[q[1]] < 0 || m.code[q[3]] < 0 || m.code[q[4]] < 0) {
                atomicAdd(err, 1);  // missing cells for the finite differences (:668-676)
                return;
            }
            for (int c = 0; c < 3; c++) {
                const double *x = m.x[c];
                nv[d][c] = dhsp[d] * mono_diff(x[q[0]], x[q[1]], x[q[2]], x[q[3]], x[q[4]]);
            }
        }
        double x[3] = {m.x[0][ind], m.x[1][ind], m.x[2][ind]};
        for (int f = 0; f < 6; f++) {
            int dim = f / 2, a1 = (dim + 1) % 3, a2 = (dim + 2) % 3;
            double nvel = vel[dim];
            double d = dh2[dim] * (2 * (f % 2) - 1);
            double a1v = vel[a1], a2v = vel[a2];
            for (int c = 0; c < 3; c++)
                m.fx[3 * f + c][ind] = x[c] + (d - dt2 * nvel) * nv[dim][c] - dt2 * (a1v * nv[a1][c] + a2v * nv[a2][c]);
        }
    }
}

// -------------------------------------------------------------------------
// Predictor of update_reference_map (fluid_3d.cc:1149-1196): xpred = x +
// advective increment from the MAC-projected face velocities and the
// upwinded face maps.  Interior cells with a primary map.
// -------------------------------------------------------------------------
__global__ void k_refmap_predict(grid_dev g, const fields_dev *__restrict__ F, double cdt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    int j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    int k = blockIdx.z * blockDim.z + threadIdx.z + 2;
    if (i >= g.sm + 2 || j >= g.sn + 2 || k >= g.so + 2) return;
    const int ind = gidx(g, i, j, k);
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        if (m.code[ind] != 0) continue;
        double avgs[3];
        avgs[0] = -0.5 * cdt * (face_ld(g, F, 0, ind) + face_ld(g, F, 3, ind)) * g.dxsp;
        avgs[1] = -0.5 * cdt * (face_ld(g, F, 7, ind) + face_ld(g, F, 10, ind)) * g.dysp;
        avgs[2] = -0.5 * cdt * (face_ld(g, F, 14, ind) + face_ld(g, F, 17, ind)) * g.dzsp;
        for (int d = 0; d < 3; d++) {
            double dx = avgs[0] * (m.fx[3 + d][ind] - m.fx[d][ind]) + avgs[1] * (m.fx[9 + d][ind] - m.fx[6 + d][ind]) +
                        avgs[2] * (m.fx[15 + d][ind] - m.fx[12 + d][ind]);
            m.xp[d][ind] = m.x[d][ind] + dx;
        }
    }
}

// extraps.copy(temp_extraps); extraps.reset() (fluid_3d.cc:1202-1203)
// With lay given (no periodic axis: nothing changes the codes before the
// extrapolation starts), the pass also sets the extrapolation's layer tags
// and claims as k_lay_init would from the reset codes: primary cells 0,
// every other cell free.
__global__ void k_snapshot_reset(grid_dev g, const fields_dev *__restrict__ F, uint8_t *lay, int *inl) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        int cd = m.code[ind];
        m.code_prev[ind] = (cd > 0) ? cd : -1;
        if (cd > 0) {
            for (int c = 0; c < 3; c++) m.x_prev[c][ind] = m.x[c][ind];
            for (int c = 0; c < 9; c++) m.gp_prev[c][ind] = m.gp[c][ind];
            m.code[ind] = -1;
        }
        if (lay) {
            lay[(size_t)o * g.ncell + ind] = (cd == 0) ? 0 : 255;
            inl[(size_t)o * g.ncell + ind] = 0;
        }
    }
}

// extraps.reset() alone (init_iter, fluid_3d.cc:270)
__global__ void k_reset_extraps(grid_dev g, const fields_dev *__restrict__ F) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++)
        if (F->om[o].code[ind] > 0) F->om[o].code[ind] = -1;
}

// -------------------------------------------------------------------------
// Extrapolation frontier (Extrapolation/extrap_helper.{hh,cc}).
// lay[] holds, for the object being extrapolated, 0 on primary cells, L on
// cells listed for layer L, 255 on free cells -- the reference's mask values
// relative to cur_mask.
// -------------------------------------------------------------------------
__device__ inline bool image_backed(const grid_dev &g, int i, int j, int k) {
    const int c[3] = {i, j, k};
    const int s[3] = {g.sm, g.sn, g.so};
    bool ghost = false;
    for (int d = 0; d < 3; d++) {
        if (c[d] >= 2 && c[d] < 2 + s[d]) continue;
        if (!g.prd[d]) return false;
        ghost = true;
    }
    return ghost;
}
__device__ inline bool inner_ghost(const grid_dev &g, int i, int j, int k) {
    return i >= 1 && i <= g.sm4 - 2 && j >= 1 && j <= g.sn4 - 2 && k >= 1 && k <= g.so4 - 2;
}

// The frontier state of every object side by side: lay[o * ncell + cell]
// holds, for object o, 0 on primary cells, L on cells listed for layer L and
// 255 on free cells (the reference's mask values relative to cur_mask);
// front[o * ncell + t] lists object o's current frontier, cnt[o] its length.
// Objects are extrapolated independently of one another (each reads and
// writes only its own maps), so all of them advance one layer per launch.

// first_layer + mark_primary (fluid_3d_ex.cc:52-70): reset the layer tags
__global__ void k_lay_init(grid_dev g, const fields_dev *__restrict__ F, uint8_t *lay, int *inl) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        lay[(size_t)o * g.ncell + ind] = (F->om[o].code[ind] == 0) ? 0 : 255;
        inl[(size_t)o * g.ncell + ind] = 0;
    }
}

// Cell c joins the frontier of layer `next`: its tag becomes `next`, and the
// one thread whose claim on inl[c] succeeds appends it to the frontier list
// (add_to_next_list and update_list in one step; the list order is free,
// since the cells of one layer do not read one another).
// A slot at the end of list cnt for each calling thread: one atomic per
// group of converged threads that append to the same list (the threads of a
// warp may serve different objects' lists).  Blocks are one-dimensional.
__device__ inline int list_slot(int *cnt) {
    const unsigned act = __activemask();
    const unsigned same = __match_any_sync(act, (unsigned long long)cnt);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cnt, __popc(same));
    base = __shfl_sync(same, base, leader);
    return base + __popc(same & ((1u << lane) - 1));
}

__device__ inline void join_layer(int c, uint8_t *lay, int *inl, int next, int *front, int *cnt) {
    lay[c] = (uint8_t)next;
    if (atomicCAS(inl + c, 0, next) == 0) front[list_slot(cnt)] = c;
}

// the free orthogonal neighbours of cell ind join layer `next`
__device__ inline void push_from(const grid_dev &g, int ind, uint8_t *lay, int *inl, int next, int *front,
                                 int *cnt) {
    const int strides[3] = {1, g.sm4, g.smn4};
    int k = ind / g.smn4, j = (ind % g.smn4) / g.sm4, i = ind % g.sm4;
    if (!inner_ghost(g, i, j, k)) return;
    for (int d = 0; d < 3; d++)
        for (int sg = -1; sg <= 1; sg += 2) {
            int c = ind + sg * strides[d];
            if (lay[c] == 255) join_layer(c, lay, inl, next, front, cnt);
        }
}

// (object, index) of entry t of the concatenated frontiers; false past the end
__device__ inline bool front_entry(int n_obj, const int *cnt, int &t, int &o) {
    for (o = 0; o < n_obj; o++) {
        if (t < cnt[o]) return true;
        t -= cnt[o];
    }
    return false;
}

// neighbours of the primary cells (from_primary) or of the current
// frontiers (front, cnt) join the next layer, listed in nfront / ncnt
// (add_to_next_list with the orthogonal rule, extrap_helper.hh:166-255)
__global__ void k_lay_push(grid_dev g, const int *front, const int *cnt, int from_primary, uint8_t *lay, int *inl,
                           int next, int *nfront, int *ncnt) {
    if (from_primary) {
        int ind = blockIdx.x * blockDim.x + threadIdx.x;
        if (ind >= g.ncell) return;
        for (int o = 0; o < g.n_obj; o++) {
            const size_t off = (size_t)o * g.ncell;
            if (lay[off + ind] == 0) push_from(g, ind, lay + off, inl + off, next, nfront + off, ncnt + o);
        }
        return;
    }
    int total = 0;
    for (int o = 0; o < g.n_obj; o++) total += cnt[o];
    if (blockIdx.x * blockDim.x >= total) return;  // no frontier entry in any round
    for (int t0 = blockIdx.x * blockDim.x + threadIdx.x; t0 < total; t0 += gridDim.x * blockDim.x) {
        int t = t0, o;
        if (!front_entry(g.n_obj, cnt, t, o)) break;
        const size_t off = (size_t)o * g.ncell;
        push_from(g, front[off + t], lay + off, inl + off, next, nfront + off, ncnt + o);
    }
}

// image-backed ghost cells take their image's tag and join its layer
// (periodic domains only)
__global__ void k_lay_ghost(grid_dev g, uint8_t *lay, int *inl, int next, int *nfront, int *ncnt) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    int k = ind / g.smn4, j = (ind % g.smn4) / g.sm4, i = ind % g.sm4;
    if (!image_backed(g, i, j, k)) return;
    const int s[3] = {g.sm, g.sn, g.so};
    int c[3] = {i, j, k};
    for (int d = 0; d < 3; d++) {
        if (c[d] < 2) c[d] += s[d];
        else if (c[d] >= 2 + s[d]) c[d] -= s[d];
    }
    const int src = gidx(g, c[0], c[1], c[2]);
    for (int o = 0; o < g.n_obj; o++) {
        const size_t off = (size_t)o * g.ncell;
        uint8_t v = lay[off + src];
        lay[off + ind] = v;
        if (v == next && atomicCAS(inl + off + ind, 0, next) == 0) nfront[off + list_slot(ncnt + o)] = ind;
    }
}

// LANES lanes work on one frontier cell: an aligned group of a warp.  Fewer
// lanes per cell put more cells in flight at once but make each cell a
// longer chain; a layer's frontier is a few thousand cells per scene, which
// a warp per cell covers in about one round when the scene has the GPU to
// itself, while concurrent scenes fill the GPU better with 4 lanes per cell.
template <int LANES>
__device__ inline unsigned group_mask() {
    static_assert(LANES == 4 || LANES == 8 || LANES == 16 || LANES == 32, "lanes per frontier cell");
    if (LANES == 32) return 0xffffffffu;
    return ((1u << (LANES & 31)) - 1) << ((threadIdx.x & 31) & ~(LANES - 1));
}

template <int LANES>
__device__ inline double group_sum(double v, unsigned mask) {
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// -------------------------------------------------------------------------
// One layer of least-squares extrapolation, one lane group per frontier cell:
// gather_and_list (fluid_3d_ex.cc:86-272), extrap_helper::least_square
// (extrap_helper.cc:34-103) with lin_sys (:129-146), mat3::inverse
// (Utilities/mat3.hh:61-67) and transfer (fluid_3d_ex.cc:293-328).
// -------------------------------------------------------------------------
constexpr int kPowTab = 64;

// One radius R of the least-squares fit for the frontier cell (ii, jj, kk)
// of map m: false when no candidate is eligible or the normal matrix is
// singular (the caller then widens R).  W = 2R + 1 as a compile-time
// constant for the common radii, 0 for the general case.
template <int W, int LANES>
__device__ bool ls_radius(const grid_dev &g, const objmap_dev &m, int R, int L, int lane, int ii, int jj, int kk,
                          int ind, bool directional, const double (&gph)[3], double cx, double cy, double cz,
                          const double *lx, const double *ly, const double *lz, const double *wpow, double wt,
                          double (&val)[3]) {
    const int w = W ? W : 2 * R + 1, nc = w * w * w;
    auto wpw = [&](int e) { return e < kPowTab ? wpow[e] : pow(wt, (double)e); };
    // pass 1: weights and weighted sums of positions and values
    double sw = 0, sd[3] = {0, 0, 0}, sr[3] = {0, 0, 0};
    int cnt = 0;
    for (int s = lane; s < nc; s += LANES) {
        int p = s % w - R, q = (s / w) % w - R, r = s / (w * w) - R;
        if (ii + p > g.sm4 - 1 || ii + p < 0) continue;
        if (jj + q > g.sn4 - 1 || jj + q < 0) continue;
        if (kk + r > g.so4 - 1 || kk + r < 0) continue;
        int qi = ind + p + g.sm4 * q + g.smn4 * r;
        // the candidate's map values are loaded together with its code (qi is
        // inside the box), so the two loads do not wait on each other; they
        // are used only when the code makes the candidate eligible
        const int cd = m.code[qi];
        const double xv[3] = {m.xp[0][qi], m.xp[1][qi], m.xp[2][qi]};
        if (cd < 0 || cd >= L) continue;
        double d[3] = {lx[ii + p], ly[jj + q], lz[kk + r]};
        double wgt = wpw(abs(p) + abs(q) + abs(r));
        if (directional) {
            double ev[3] = {cx - d[0], cy - d[1], cz - d[2]};
            double dw = 0, en = 0;
            for (int pp = 0; pp < 3; pp++) {
                dw += ev[pp] * gph[pp];
                en += ev[pp] * ev[pp];
            }
            en = sqrt(en);
            dw /= en;
            dw *= wgt;
            if (!(dw > 0)) continue;
            wgt = dw;
        }
        sw += wgt;
        cnt++;
        for (int c = 0; c < 3; c++) {
            sd[c] += d[c] * wgt;
            sr[c] += xv[c] * wgt;
        }
    }
    const unsigned gm = group_mask<LANES>();
    sw = group_sum<LANES>(sw, gm);
    for (int c = 0; c < 3; c++) {
        sd[c] = group_sum<LANES>(sd[c], gm);
        sr[c] = group_sum<LANES>(sr[c], gm);
    }
    for (int off = LANES / 2; off > 0; off >>= 1) cnt += __shfl_xor_sync(gm, cnt, off);
    if (cnt == 0) return false;
    double davg[3], ravg[3];
    for (int c = 0; c < 3; c++) {
        ravg[c] = sr[c] / sw;
        davg[c] = sd[c] / sw;
    }
    // pass 2: weighted normal equations about the averages
    double a[6] = {0, 0, 0, 0, 0, 0}, rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int s = lane; s < nc; s += LANES) {
        int p = s % w - R, q = (s / w) % w - R, r = s / (w * w) - R;
        if (ii + p > g.sm4 - 1 || ii + p < 0) continue;
        if (jj + q > g.sn4 - 1 || jj + q < 0) continue;
        if (kk + r > g.so4 - 1 || kk + r < 0) continue;
        int qi = ind + p + g.sm4 * q + g.smn4 * r;
        const int cd = m.code[qi];
        const double xv[3] = {m.xp[0][qi], m.xp[1][qi], m.xp[2][qi]};
        if (cd < 0 || cd >= L) continue;
        double d[3] = {lx[ii + p], ly[jj + q], lz[kk + r]};
        double Q = wpw(abs(p) + abs(q) + abs(r));
        if (directional) {
            double ev[3] = {cx - d[0], cy - d[1], cz - d[2]};
            double dw = 0, en = 0;
            for (int pp = 0; pp < 3; pp++) {
                dw += ev[pp] * gph[pp];
                en += ev[pp] * ev[pp];
            }
            en = sqrt(en);
            dw /= en;
            dw *= Q;
            if (!(dw > 0)) continue;
            Q = dw;
        }
        double e0 = d[0] - davg[0], e1 = d[1] - davg[1], e2 = d[2] - davg[2];
        a[0] += Q * e0 * e0;
        a[1] += Q * e1 * e1;
        a[2] += Q * e2 * e2;
        a[3] += Q * e0 * e1;
        a[4] += Q * e0 * e2;
        a[5] += Q * e1 * e2;
        for (int c = 0; c < 3; c++) {
            double lr = Q * (xv[c] - ravg[c]);
            rhs[3 * c + 0] += e0 * lr;
            rhs[3 * c + 1] += e1 * lr;
            rhs[3 * c + 2] += e2 * lr;
        }
    }
    for (int c = 0; c < 6; c++) a[c] = group_sum<LANES>(a[c], gm);
    for (int c = 0; c < 9; c++) rhs[c] = group_sum<LANES>(rhs[c], gm);
    // mat3 A(XX, XY, XZ, XY, YY, YZ, XZ, YZ, ZZ) and its inverse
    const double a11 = a[0], a12 = a[3], a13 = a[4], a21 = a[3], a22 = a[1], a23 = a[5], a31 = a[4],
                 a32 = a[5], a33 = a[2];
    double det = a11 * (a22 * a33 - a23 * a32) + a21 * (a13 * a32 - a12 * a33) + a31 * (a12 * a23 - a13 * a22);
    if (fabs(det) < 1e-17) return false;
    double id = 1 / det;
    double inv[9] = {(a22 * a33 - a23 * a32) * id, (a13 * a32 - a12 * a33) * id, (a12 * a23 - a13 * a22) * id,
                     (a23 * a31 - a21 * a33) * id, (a11 * a33 - a13 * a31) * id, (a13 * a21 - a11 * a23) * id,
                     (a21 * a32 - a22 * a31) * id, (a12 * a31 - a11 * a32) * id, (a11 * a22 - a12 * a21) * id};
    double ps[3] = {cx - davg[0], cy - davg[1], cz - davg[2]};
    for (int c = 0; c < 3; c++) {
        double co0 = inv[0] * rhs[3 * c] + inv[1] * rhs[3 * c + 1] + inv[2] * rhs[3 * c + 2];
        double co1 = inv[3] * rhs[3 * c] + inv[4] * rhs[3 * c + 1] + inv[5] * rhs[3 * c + 2];
        double co2 = inv[6] * rhs[3 * c] + inv[7] * rhs[3 * c + 1] + inv[8] * rhs[3 * c + 2];
        double v = ravg[c];
        v += co0 * ps[0];
        v += co1 * ps[1];
        v += co2 * ps[2];
        val[c] = v;
    }
    return true;
}

// Every object's frontier in one launch: lane group w (LANES lanes)
// takes entry w of the concatenated frontiers.  The weights wt^n (n = |p|+|q|+|r|) come from a
// per-block table of the same pow() values.
template <int LANES>
__global__ void k_extrap_layer(grid_dev g, const fields_dev *__restrict__ F, const int *front, const int *cnt, int L,
                               int max_rs, double wt, const double *lx, const double *ly, const double *lz,
                               int *err) {
    __shared__ double wpow[kPowTab];
    int total = 0;
    for (int o = 0; o < g.n_obj; o++) total += cnt[o];
    // the grid is sized for the largest frontiers: a block whose first lane
    // group is past this layer's frontier has no cell in any round and leaves
    // before building its weight table (the whole block, so no barrier waits)
    if (blockIdx.x * (blockDim.x / LANES) >= total) return;
    const int npow = 3 * max_rs + 1;
    for (int q = threadIdx.x; q < kPowTab && q < npow; q += blockDim.x) wpow[q] = pow(wt, (double)q);
    __syncthreads();
    const int lane = threadIdx.x & (LANES - 1);
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / LANES;
    const int nwarps = (gridDim.x * blockDim.x) / LANES;
    for (int t0 = warp; t0 < total; t0 += nwarps) {
        int t = t0, o;
        if (!front_entry(g.n_obj, cnt, t, o)) break;
        const objmap_dev &m = F->om[o];
        const int ind = front[(size_t)o * g.ncell + t];
        const int kk = ind / g.smn4, jj = (ind % g.smn4) / g.sm4, ii = ind % g.sm4;
        if (image_backed(g, ii, jj, kk)) continue;  // within_extrapolation_domain
        // average of the previous step's interface normals over the six faces
        double gph[3] = {0, 0, 0};
        double gnorm = 0;
        if (ii >= 2 && ii <= g.sm4 - 3 && jj >= 2 && jj <= g.sn4 - 3 && kk >= 2 && kk <= g.so4 - 3) {
            const int pidx[4] = {ind, ind + 1, ind + g.sm4, ind + g.smn4};
            int nfaces = 0;
            for (int pp = 0; pp < 4; pp++) {
                int q = pidx[pp];
                const double *const *gsrc;
                if (m.code[q] == 0) gsrc = m.gp;            // primary: current values
                else if (m.code_prev[q] > 0) gsrc = m.gp_prev;  // previous extrapolation
                else continue;
                int d0 = (pp == 0) ? 0 : pp - 1, d1 = (pp == 0) ? 3 : pp;
                for (int dd = d0; dd < d1; dd++) {
                    if (gsrc[3 * dd + dd][q] != -kBig) {
                        bool add = false;
                        for (int ff = 0; ff < 3; ff++) {
                            double v = gsrc[3 * dd + ff][q];
                            if (v != 0.0) add = true;
                            gph[ff] += v;
                        }
                        if (add) nfaces++;
                    }
                }
            }
            if (nfaces == 6) {
                for (int pp = 0; pp < 3; pp++) {
                    gph[pp] /= nfaces;
                    gnorm += gph[pp] * gph[pp];
                }
                if (gnorm != 0) {
                    gnorm = sqrt(gnorm);
                    for (int pp = 0; pp < 3; pp++) gph[pp] /= gnorm;
                } else {
                    for (int pp = 0; pp < 3; pp++) gph[pp] = 0;
                }
            } else {
                for (int pp = 0; pp < 3; pp++) gph[pp] = 0;
            }
        }
        const bool directional = (gnorm != 0. && L <= 2);
        const double cx = lx[ii], cy = ly[jj], cz = lz[kk];
        bool success = false;
        double val[3] = {0, 0, 0};
        for (int R = 2; R <= max_rs && !success; R++) {
#define LS_ARGS g, m, R, L, lane, ii, jj, kk, ind, directional, gph, cx, cy, cz, lx, ly, lz, wpow, wt, val
            switch (R) {
                case 2: success = ls_radius<5, LANES>(LS_ARGS); break;
                case 3: success = ls_radius<7, LANES>(LS_ARGS); break;
                case 4: success = ls_radius<9, LANES>(LS_ARGS); break;
                case 5: success = ls_radius<11, LANES>(LS_ARGS); break;
                default: success = ls_radius<0, LANES>(LS_ARGS); break;
            }
#undef LS_ARGS
        }
        if (!success) {
            if (lane == 0) atomicAdd(err, 1);
            continue;
        }
        if (lane == 0 && !(isnan(val[0]) || isnan(val[1]) || isnan(val[2]))) {
            m.code[ind] = L;
            for (int c = 0; c < 3; c++) {
                m.x[c][ind] = val[c];
                m.xp[c][ind] = val[c];
            }
        }
    }
}

template __global__ void k_extrap_layer<4>(grid_dev, const fields_dev *__restrict__, const int *, const int *, int,
                                            int, double, const double *, const double *, const double *, int *);
template __global__ void k_extrap_layer<32>(grid_dev, const fields_dev *__restrict__, const int *, const int *, int,
                                             int, double, const double *, const double *, const double *, int *);

// communicate_a_layer on one rank (fluid_3d_comm.cc:203-280): image-backed
// ghosts receive the maps of the layer just made at their image (periodic
// domains only).
__global__ void k_layer_ghost_copy(grid_dev g, const fields_dev *__restrict__ F, int L) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    int k = ind / g.smn4, j = (ind % g.smn4) / g.sm4, i = ind % g.sm4;
    if (!image_backed(g, i, j, k)) return;
    const int s[3] = {g.sm, g.sn, g.so};
    int c[3] = {i, j, k};
    for (int d = 0; d < 3; d++) {
        if (c[d] < 2) c[d] += s[d];
        else if (c[d] >= 2 + s[d]) c[d] -= s[d];
    }
    const int src = gidx(g, c[0], c[1], c[2]);
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        if (m.code[src] != L) continue;
        m.code[ind] = L;
        for (int a = 0; a < 3; a++) {
            m.x[a][ind] = m.xp[a][src];
            m.xp[a][ind] = m.xp[a][src];
        }
    }
}

// -------------------------------------------------------------------------
// Corrector of update_reference_map (fluid_3d.cc:1205-1247) over every cell:
// primary x = (x + xpred)/2; extrapolated maps average with the previous
// extrapolation of the same object, or take xpred where none existed.
// -------------------------------------------------------------------------
__global__ void k_refmap_correct(grid_dev g, const fields_dev *__restrict__ F, int *prob, int var_den) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        int cd = m.code[ind];
        if (cd < 0) continue;
        if (cd == 0) {
            for (int c = 0; c < 3; c++) m.x[c][ind] = 0.5 * (m.x[c][ind] + m.xp[c][ind]);
        } else if (m.code_prev[ind] > 0) {
            for (int c = 0; c < 3; c++) m.x[c][ind] = 0.5 * (m.x_prev[c][ind] + m.xp[c][ind]);
        } else {
            double dist = obj_phi(g, o, m.xp[0][ind], m.xp[1][ind], m.xp[2][ind]);
            if (dist < g.eps && cd <= 3) atomicAdd(prob, 1);
            else
                for (int c = 0; c < 3; c++) m.x[c][ind] = m.xp[c][ind];
        }
    }
    // update_rho (fluid_3d.cc:1252) from this cell's corrected maps
    if (var_den) F->rho[ind] = cell_rho(g, F, ind);
}

// revert_reference_map_update (fluid_3d.cc:1257-1283)
__global__ void k_refmap_revert(grid_dev g, const fields_dev *__restrict__ F) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        int cd = m.code[ind];
        if (cd == 0) {
            for (int c = 0; c < 3; c++) m.x[c][ind] = 2 * m.x[c][ind] - m.xp[c][ind];
        } else if (cd > 0 && m.code_prev[ind] > 0) {
            for (int c = 0; c < 3; c++) m.x[c][ind] = m.x_prev[c][ind];
        }
    }
}

// update_reference_map_full (fluid_3d.cc:1285-1306): x = xpred everywhere,
// then its update_rho (:1304) from this cell's maps
__global__ void k_refmap_full(grid_dev g, const fields_dev *__restrict__ F, int var_den) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        if (m.code[ind] < 0) continue;
        for (int c = 0; c < 3; c++) m.x[c][ind] = m.xp[c][ind];
    }
    if (var_den) F->rho[ind] = cell_rho(g, F, ind);
}

// x = xpred for the maps of one extrapolation (init_extrapolate,
// fluid_3d_ex.cc:16-27)
__global__ void k_extraps_full(grid_dev g, const fields_dev *__restrict__ F) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    for (int o = 0; o < g.n_obj; o++) {
        const objmap_dev &m = F->om[o];
        if (m.code[ind] <= 0) continue;
        for (int c = 0; c < 3; c++) m.x[c][ind] = m.xp[c][ind];
    }
}

// -------------------------------------------------------------------------
// redraw_boundary (fluid_3d_ex.cc:336-394) over every cell: a primary map
// whose level set became positive leaves the body (kept as an extrapolated
// map of layer nlayers+1); a first-layer extrapolated map with negative level
// set enters it.
// -------------------------------------------------------------------------
__global__ void k_redraw(grid_dev g, const fields_dev *__restrict__ F, int nlayers, int *fatal) {
    int ind = blockIdx.x * blockDim.x + threadIdx.x;
    if (ind >= g.ncell) return;
    bool occupied = false;
    int prim = -1;
    for (int o = 0; o < g.n_obj; o++)
        if (F->om[o].code[ind] == 0) prim = o;
    int moved_out = -1;
    if (prim >= 0) {
        const objmap_dev &m = F->om[prim];
        double pphi = mphi(g, m, prim, ind);
        if (pphi > 0) {
            m.code[ind] = nlayers + 1;
            moved_out = prim;
            prim = -1;
        } else {
            occupied = true;
        }
    }
    // extrapolated maps in object order, the map that just moved out last
    for (int pass = 0; pass < 2; pass++) {
        for (int o = 0; o < g.n_obj; o++) {
            if ((pass == 0) == (o == moved_out)) continue;
            const objmap_dev &m = F->om[o];
            int cd = m.code[ind];
            if (cd <= 0) continue;
            double sp = mphi(g, m, o, ind);
            bool inside = (sp < 0 && cd == 1);
            if (!inside) continue;
            double pp = (prim >= 0) ? mphi(g, F->om[prim], prim, ind) : nan("");
            if ((occupied && sp < pp) || !occupied) {
                if (pp < -g.dx) atomicAdd(fatal, 1);
                if (prim >= 0) F->om[prim].code[ind] = -1;  // overwritten primary map
                m.code[ind] = 0;
                prim = o;
                occupied = true;
            }
        }
    }
}

}  // namespace rmt3d
