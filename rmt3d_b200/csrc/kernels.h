// Kernel declarations and small by-value argument structs shared between the
// kernel translation units and the host orchestration (scene.cu).
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "dev_common.cuh"

namespace rmt3d {

// arrays touched by one periodic ghost exchange
struct ptr_list {
    double *p[40];
    int *ip[4];
    float *fp[18];
    int n, ni, nf;
};

// one physical boundary face (face_gm, fields.hh:661-850)
struct bc_face {
    int bct[3];
    double bcv[3];
    double h;
};
// the tracers of a scene and the constants their kernels read
struct tracer_args {
    int *pc;         // [3][n] corner cell of each tracer's 4x4x4 cube
    double *rp;      // [6][n] rp0 (x, y, z) then rpf (x, y, z), in cell units
    uint8_t *alive;  // [n] 0 for a tracer that left through a wall
    double low[3];   // coordinate of ghost cell 0 on each axis (tracers.cc:18-20)
    double h[3];
    double lo[3], hi[3];  // the domain's walls (tracers.hh:370-375)
    double dt;
    int homog[3][2];  // [axis][low/high face]: homogeneous Dirichlet wall for that velocity component
};

struct bc_faces {
    bc_face f[6];
};

// FEM element-integrated basis gradients (fluid_3d.cc:2506-2517)
struct gradphi_t {
    double v[8][3];
};

__global__ void k_periodic_copy(grid_dev g, ptr_list pl, int corner);
__global__ void k_bc_cc(grid_dev g, int n, bc_face lo, bc_face hi, double *u, double *v, double *w);
__global__ void k_bc_cf(grid_dev g, int walls, bc_faces bcs, const fields_dev *F);
__global__ void k_stress(grid_dev g, const fields_dev *__restrict__ F, const int *list, const int *cnt);
__global__ void k_stress_fluid(grid_dev g, const fields_dev *__restrict__ F, int *list, int *cnt);
// FT: the face states' type: float in the FP32-advection form (RMT3D_MIXED_BULK32), else double
template <typename FT>
__global__ void k_edge_vel(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                           const double *lz, double cdt, const double *time_p, int var_den);
// the velocity edge states with TMA-staged velocity tiles (k_fluid.cu)
bool edge_vel_tensor_map(const grid_dev &g, const double *base, CUtensorMap *out);
void launch_edge_vel_tma(const grid_dev &g, const fields_dev *F, const CUtensorMap tm[3], const double *lx,
                         const double *ly, const double *lz, double cdt, const double *time_p, int var_den, int *err,
                         cudaStream_t st);
template <typename FT>
__global__ void k_upwind(grid_dev g, const fields_dev *__restrict__ F);
__global__ void k_mac_rhs(grid_dev g, const fields_dev *__restrict__ F, double *r, double cdt);
__global__ void k_mac_extract(grid_dev g, const fields_dev *__restrict__ F, const double *x);
__global__ void k_sub_qgrad(grid_dev g, const fields_dev *__restrict__ F, double cdt, int var_den);
template <typename FT>
__global__ void k_ustar(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                        const double *lz, double cdt, const double *time_p, int var_den);
__global__ void k_fem_rhs(grid_dev g, const fields_dev *__restrict__ F, double *r, gradphi_t gp);
__global__ void k_fem_extract(grid_dev g, const fields_dev *__restrict__ F, const double *x, const double *mean);
__global__ void k_sub_pgrad(grid_dev g, const fields_dev *__restrict__ F, double dt, int var_den);
__global__ void k_chk_pack(grid_dev g, const fields_dev *__restrict__ F, double *__restrict__ buf);
__global__ void k_macro_cells(grid_dev g, const fields_dev *__restrict__ F, const double *lz, int var_den,
                              double *out, unsigned *ticket);
__global__ void k_macro_obj(grid_dev g, const fields_dev *__restrict__ F, const double *lx, const double *ly,
                            const double *lz, int o, double *out, unsigned *ticket);
__global__ void k_divu_l2(grid_dev g, const double *r, double *out, unsigned *ticket);
__global__ void k_checksum(grid_dev g, const fields_dev *__restrict__ F, double *out, unsigned *ticket);
__global__ void k_slice(grid_dev g, const fields_dev *__restrict__ F, const double *r, int type, int dim, int point,
                        int obj_id, int var_den, int d1, int d2, double *out);
__global__ void k_tracer_predict(grid_dev g, const fields_dev *__restrict__ F, tracer_args A, int n);
__global__ void k_tracer_advect(grid_dev g, const fields_dev *__restrict__ F, tracer_args A, int n);
__global__ void k_tracer_place(grid_dev g, tracer_args A, int n, const double *xyz);
__global__ void k_tracer_positions(tracer_args A, int n, float *out);
__global__ void k_chk_unpack(grid_dev g, const fields_dev *__restrict__ F, const double *__restrict__ buf, int *bad);

}  // namespace rmt3d
