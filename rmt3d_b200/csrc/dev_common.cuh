// Device-side definitions shared by every kernel of the FSI step.
//
// Layout: every per-cell quantity is a separate FP64 array (SoA) over the
// reference's ghosted box of (sm+4)(sn+4)(so+4) cells, with the reference's
// index i + sm4*j + smn4*k on absolute (ghost-inclusive) coordinates
// (F3D_Source/fluid_3d.cc:21-24).  Interior cells have absolute indices
// 2..sm+1.  Keeping the reference's index space makes every ghost-frame rule
// (physical BCs, periodic wrap, extrapolation into ghosts) carry over
// one-to-one, and each array is contiguous along x for coalesced access.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rmt3d {

constexpr int kMaxObj = 16;
constexpr double kBig = 1.e200;  // "unset" marker for grad_phi (fields.hh:338)

// Object parameters consumed inside kernels (Sim/object.hh:76-123,
// Sim/sim_manager.hh:15-74).
struct obj_dev {
    int type;
    double c[3];
    double R;
    double eig[3];   // SPHERE initial-map scale per axis (object.hh:100-114)
    double omega[3]; // initial spin
    double G, rho, ex_mu, ev_trans_mult;
};

// Per-scene constants passed by value to kernels.
struct grid_dev {
    int sm, sn, so;       // interior cells
    int sm4, sn4, so4;    // ghosted extents
    int smn4;             // sm4*sn4
    int ncell;            // sm4*sn4*so4
    int prd[3];           // periodic flags
    int fm, fn, fo;       // FEM node grid (m+1 per non-periodic axis)
    double dx, dy, dz, dxsp, dysp, dzsp;
    double ax, ay, az;
    double mu;            // fluid dynamic viscosity
    double frho;
    double eps, tf1, tf2, tf3;  // transition zone constants (sim_manager.cc:37-47)
    int n_obj;
    int sim_type;
    int has_exact;
    int f32face;          // face states stored in FP32 (RMT3D_MIXED_BULK32), else FP64
    double gravity;
    double K_stiff, wall_dist, winv, min_wall_acc, wall_acc_mult;
    int walls[6];
    double wall_pos[6];
    obj_dev obj[kMaxObj];
};

__host__ __device__ inline int gidx(const grid_dev &g, int i, int j, int k) { return i + g.sm4 * j + g.smn4 * k; }

// ---- scalar helpers of the Godunov scheme (fluid_3d.cc:2310-2340) -------
__device__ inline double rmin(double x, double y) { return (x < y) ? x : y; }
__device__ inline double rsign(double x) { return (x >= 0) ? 1 : -1; }

__device__ inline double del_lim(double u0, double u1, double u2) {
    double t1 = 2 * (u1 - u0);
    double t2 = 2 * (u2 - u1);
    if (t1 * t2 > 0) return rmin(fabs(t1), fabs(t2));
    return 0;
}
__device__ inline double del_f(double u0, double u1, double u2) {
    double dlim = del_lim(u0, u1, u2);
    double cen = 0.5 * (u2 - u0);
    return rsign(cen) * rmin(fabs(cen), dlim);
}
// 4th-order monotonicity-limited slope, Yu (2003) Eq. 3.25-3.26
__device__ inline double mono_diff(double u0, double u1, double u2, double u3, double u4) {
    double dlim = del_lim(u1, u2, u3);
    double cen = 0.5 * (u3 - u1);
    double neigh_delf = (del_f(u0, u1, u2) + del_f(u2, u3, u4)) / 6.0;
    return rsign(cen) * rmin(dlim, fabs(4.0 / 3.0 * cen - neigh_delf));
}

// The same slope in FP32 (the FP32-advection form's stencil), written on the
// successive differences d0 = u1 - u0, ..., d3 = u4 - u3, of which every term
// of mono_diff is a sum.
__device__ __forceinline__ float del_lim_f(float a, float b) {
    const float t1 = 2 * a, t2 = 2 * b;
    return t1 * t2 > 0 ? fminf(fabsf(t1), fabsf(t2)) : 0.f;
}
__device__ __forceinline__ float del_f_f(float a, float b) {
    const float cen = 0.5f * (a + b);
    return (cen >= 0.f ? 1.f : -1.f) * fminf(fabsf(cen), del_lim_f(a, b));
}
__device__ __forceinline__ float mono_diff_f(float u0, float u1, float u2, float u3, float u4) {
    const float d0 = u1 - u0, d1 = u2 - u1, d2 = u3 - u2, d3 = u4 - u3;
    const float dlim = del_lim_f(d1, d2);
    const float cen = 0.5f * (d1 + d2);
    const float neigh = (del_f_f(d0, d1) + del_f_f(d2, d3)) * (1.f / 6.f);
    return (cen >= 0.f ? 1.f : -1.f) * fminf(dlim, fabsf(4.f / 3.f * cen - neigh));
}

// ---- transition-zone functions (sim_manager.hh:259-280) ------------------
__device__ inline double heaviside(const grid_dev &g, double phi) {
    if (phi >= g.eps) return 0;
    if (phi <= -g.eps) return 1;
    double tmp = 0.5 - phi * g.tf1 - sin(g.tf3 * phi) * g.tf2;
    if (tmp < 0) tmp = 0.;
    else if (tmp > 1) tmp = 1;
    return tmp;
}
__device__ inline double tderiv_func_in(const grid_dev &g, double x) {
    double tmp = 0;
    if (x > -g.eps && x < g.eps) tmp = 0.5 + 0.5 * cos(x * g.tf3);
    return tmp;
}
__device__ inline double coll_func(const grid_dev &g, double x) { return x > g.eps ? 0 : (0.5 - x * g.tf1); }

// level set of object o evaluated at reference-map value xi
// (basic_sphere::phi, Sim/object.cc:76-82; SPHERE inherits it)
__device__ inline double obj_phi(const grid_dev &g, int o, double x0, double x1, double x2) {
    const obj_dev &ob = g.obj[o];
    double sq = 0;
    sq += (x0 - ob.c[0]) * (x0 - ob.c[0]);
    sq += (x1 - ob.c[1]) * (x1 - ob.c[1]);
    sq += (x2 - ob.c[2]) * (x2 - ob.c[2]);
    return sqrt(sq) - ob.R;
}

// physical coordinate of absolute index i along an axis (fluid_3d.cc:137-139)
__device__ inline double coord(double a, int i, double h) { return a + ((double)(i - 2) + 0.5) * h; }

// Reference-map storage of one object slot: one map per (object, cell) at
// most, as in the reference where a cell holds either the primary map or one
// extrapolated map of each object (extrap_mmap.cc:60-200).
struct objmap_dev {
    int *code;       // -1 none, 0 primary, L >= 1 extrapolation layer L
    double *x[3];    // reference map
    double *xp[3];   // predicted reference map
    double *fx[18];  // face states fx[f][c] (fields.hh:296)
    double *gp[9];   // grad_phi[F][c] (fields.hh:310)
    double *det[3];  // detF per lower face (fields.hh:308)
    double *el[3];   // elastic energy density per lower face (fields.hh:307)
    // snapshot of the previous extrapolated maps (temp_extraps, fluid_3d.hh:122)
    int *code_prev;
    double *x_prev[3];
    double *gp_prev[9];
};

// All device arrays of a scene.
struct fields_dev {
    double *vel[3];
    double *p, *dp, *q;
    double *dvel[3];
    double *fvel[18];     // face states in FP64 (null when they are FP32)
    float *fvel32[18];    // face states in FP32 (RMT3D_MIXED_BULK32 only)
    double *sigma[9];
    double *rho;  // VAR_DEN density per cell (fluid_3d.hh:160)
    objmap_dev om[kMaxObj];
    unsigned int *flags;  // scratch per-cell flags (extrapolation frontier)
};

// Velocity face states fvel[f][c] (fields.hh:296), written by the edge
// extrapolation and read by the upwinding, both projections and the momentum
// update.  The FP64 and mixed forms keep them in FP64; the FP32-advection
// form (RMT3D_MIXED_BULK32) keeps them in FP32, as intermediate values of the
// advection stencils (the velocity, the pressure and the reference maps stay
// FP64).  face_ptr picks the array of a kernel instantiated for one storage
// type; face_ld / face_st serve kernels that run with either and read
// g.f32face, which is uniform over the launch.
template <typename FT>
__device__ __forceinline__ FT *face_ptr(const fields_dev *__restrict__ F, int a);
template <>
__device__ __forceinline__ double *face_ptr<double>(const fields_dev *__restrict__ F, int a) {
    return F->fvel[a];
}
template <>
__device__ __forceinline__ float *face_ptr<float>(const fields_dev *__restrict__ F, int a) {
    return F->fvel32[a];
}
__device__ __forceinline__ double face_ld(const grid_dev &g, const fields_dev *__restrict__ F, int a, int ind) {
    return g.f32face ? (double)F->fvel32[a][ind] : F->fvel[a][ind];
}
__device__ __forceinline__ void face_st(const grid_dev &g, const fields_dev *__restrict__ F, int a, int ind,
                                        double v) {
    if (g.f32face) F->fvel32[a][ind] = (float)v;
    else F->fvel[a][ind] = v;
}

// Bit o set when object o holds a map (code >= 0) at cell ind.  The codes are
// loaded four objects at a time, so a cell costs one memory round trip per
// four objects instead of one per object; loops over the set bits visit the
// objects in increasing order, as loops over o do.
__device__ inline unsigned map_mask(const grid_dev &g, const fields_dev *__restrict__ F, int ind) {
    unsigned m = 0;
    for (int base = 0; base < g.n_obj; base += 4) {
        int c[4];
#pragma unroll
        for (int u = 0; u < 4; u++) c[u] = base + u < g.n_obj ? F->om[base + u].code[ind] : -1;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (c[u] >= 0) m |= 1u << (base + u);
    }
    return m;
}

// update_rho at one cell (fluid_3d.cc:1104-1143, VAR_DEN): the solid fractions of the
// primary map, then of every extrapolated map, blended with the fluid density
__device__ inline double cell_rho(const grid_dev &g, const fields_dev *__restrict__ F, int ind) {
    double sfrac = 0, srho = 0;
    int prim = -1;
    unsigned ext = 0;  // objects with an extrapolated map here
    for (unsigned mk = map_mask(g, F, ind); mk; mk &= mk - 1) {
        const int o = __ffs(mk) - 1;
        if (F->om[o].code[ind] == 0) prim = o;
        else ext |= 1u << o;
    }
    if (prim >= 0) {
        const objmap_dev &m = F->om[prim];
        double t = heaviside(g, obj_phi(g, prim, m.x[0][ind], m.x[1][ind], m.x[2][ind]));
        srho += t * g.obj[prim].rho;
        sfrac += t;
    }
    for (; ext; ext &= ext - 1) {
        const int o = __ffs(ext) - 1;
        const objmap_dev &m = F->om[o];
        double t = heaviside(g, obj_phi(g, o, m.x[0][ind], m.x[1][ind], m.x[2][ind]));
        srho += t * g.obj[o].rho;
        sfrac += t;
    }
    if (sfrac > 1.) srho /= sfrac;
    else srho += (1 - sfrac) * g.frho;
    return srho;
}

}  // namespace rmt3d
