// Solid-side kernel declarations (k_solid.cu).
#pragma once
#include <stdint.h>
#include "dev_common.cuh"

namespace rmt3d {

__global__ void k_edge_refmap(grid_dev g, const fields_dev *__restrict__ F, double cdt, int *err);
__global__ void k_refmap_predict(grid_dev g, const fields_dev *__restrict__ F, double cdt);
__global__ void k_snapshot_reset(grid_dev g, const fields_dev *__restrict__ F, uint8_t *lay, int *inl);
__global__ void k_reset_extraps(grid_dev g, const fields_dev *__restrict__ F);
__global__ void k_lay_init(grid_dev g, const fields_dev *__restrict__ F, uint8_t *lay, int *inl);
__global__ void k_lay_push(grid_dev g, const int *front, const int *cnt, int from_primary, uint8_t *lay, int *inl,
                           int next, int *nfront, int *ncnt);
__global__ void k_lay_ghost(grid_dev g, uint8_t *lay, int *inl, int next, int *nfront, int *ncnt);
// LANES lanes per frontier cell; instantiated for 4 and 32
template <int LANES>
__global__ void k_extrap_layer(grid_dev g, const fields_dev *__restrict__ F, const int *front, const int *cnt, int L,
                               int max_rs, double wt, const double *lx, const double *ly, const double *lz,
                               int *err);
__global__ void k_layer_ghost_copy(grid_dev g, const fields_dev *__restrict__ F, int L);
__global__ void k_refmap_correct(grid_dev g, const fields_dev *__restrict__ F, int *prob, int var_den);
__global__ void k_refmap_revert(grid_dev g, const fields_dev *__restrict__ F);
__global__ void k_refmap_full(grid_dev g, const fields_dev *__restrict__ F, int var_den);
__global__ void k_extraps_full(grid_dev g, const fields_dev *__restrict__ F);
__global__ void k_redraw(grid_dev g, const fields_dev *__restrict__ F, int nlayers, int *fatal);

}  // namespace rmt3d
