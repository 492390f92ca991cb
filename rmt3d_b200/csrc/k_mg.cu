// Multigrid kernels and V-cycle driver (see mg.h).
//
// Operators (rediscretised on every level, nothing stored):
//  * MAC, cell centred: 7-point [1 ... -6]; at a wall the missing face
//    neighbour moves onto the centre (Neumann fix of stencil_set::set_partials
//    with macfix, mg_probs.hh:281-343).  Coarsening pairs cells; restriction
//    sums the 8 children with weight 1/2 (the (2h)^2 scaling of the coarse
//    operator); prolongation is cell-centred trilinear (3/4, 1/4 per axis,
//    constant extension at walls).  Red-black Gauss-Seidel smoothing.
//  * FEM, nodal: 27-point Q1 stencil 32/-2/-1 (faces 0); each entry is halved
//    once per non-periodic axis on which the node lies on the boundary and the
//    offset along that axis is zero (set_partials(false)).  Vertex coarsening
//    (coarse node I on fine node 2I), trilinear prolongation P and restriction
//    P^T/2, which equals the Galerkin operator P^T A P of this stencil.
//    Four-colour Gauss-Seidel (exact GS ordering: the face entries are zero).
//  * Coarsest level: a dense inverse of A + (alpha/n) 1 1^T, precomputed on the
//    host; for the singular Neumann/periodic operators (null space = the
//    constants) it returns the solution orthogonal to the constants.
// Residual max norms are reduced with warp shuffles and one atomic per warp.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "host_common.h"
#include "mg.h"
#include "graph_build.h"
#include "mg_ops.cuh"
#include "mg_body.cuh"
#include "mg_tile.cuh"
#include "rmt3d_gpu.h"

namespace rmt3d {

// ---- single-scene phase kernels (bodies in mg_body.cuh) ---------------------
template <typename T>
__global__ void k_mac_rb(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int colour, const T *__restrict__ ri) {
    body_mac_rb<T>(L, x, r, colour, ri, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T>
__global__ void k_fem_gs(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int colour, const T *__restrict__ ri) {
    body_fem_gs<T>(L, x, r, colour, ri, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T, int KIND>
__global__ void k_resid(lvl_dev L, const T *__restrict__ x, const T *__restrict__ r, T *__restrict__ res,
                        unsigned long long *mx, const T *__restrict__ ri) {
    const double a = body_resid<T, KIND>(L, x, r, res, ri, blockIdx.x, blockIdx.y, blockIdx.z);
    if (mx) warp_max_into(a, mx);
}
// the control's max-norm residual, computed only when the control will read it
template <int KIND>
__global__ void k_resid_ctl(lvl_dev L, const double *__restrict__ x, const double *__restrict__ r,
                            unsigned long long *mx, const double *__restrict__ ri, const mg_ctl *c) {
    if (!c->need_res) return;
    const double a = body_resid<double, KIND>(L, x, r, nullptr, ri, blockIdx.x, blockIdx.y, blockIdx.z);
    warp_max_into(a, mx);
}
template <typename T>
__global__ void k_mac_restrict(lvl_dev F, lvl_dev C, const T *__restrict__ res, T *__restrict__ rc,
                               T *__restrict__ xc0) {
    body_mac_restrict<T>(F, C, res, rc, xc0, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int KIND>
__global__ void k_resid_to_f32(lvl_dev L, const double *__restrict__ x, const double *__restrict__ r,
                               const double *__restrict__ ri, float *__restrict__ rs, float *__restrict__ xs) {
    body_resid_to_f32<KIND>(L, x, r, ri, rs, xs, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T>
__global__ void k_mac_prolong(lvl_dev F, lvl_dev C, T *__restrict__ x, const T *__restrict__ xc) {
    body_mac_prolong<T>(F, C, x, xc, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T>
__global__ void k_fem_restrict(lvl_dev F, lvl_dev C, const T *__restrict__ res, T *__restrict__ rc,
                               T *__restrict__ xc0) {
    body_fem_restrict<T>(F, C, res, rc, xc0, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T>
__global__ void k_fem_prolong(lvl_dev F, lvl_dev C, T *__restrict__ x, const T *__restrict__ xc) {
    body_fem_prolong<T>(F, C, x, xc, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename T>
__global__ void k_coarse_dense(int np, const double *__restrict__ B, T *__restrict__ x, const T *__restrict__ r) {
    body_coarse_dense<T>(np, B, x, r, blockIdx.x, gridDim.x);
}

// one whole sweep of a level on shared-memory tiles (mg_tile.cuh), one block
// per output box
template <typename T, int KIND, bool VD>
__global__ void __launch_bounds__(512) k_tile_sweep(lvl_dev L, const T *__restrict__ xin, T *__restrict__ xout,
                                                    const T *__restrict__ r, const T *__restrict__ ri) {
    extern __shared__ __align__(16) unsigned char tile_smem[];
    using S = tile_shape<T, KIND, VD>;
    body_tile_sweep<T, KIND, VD>(L, xin, xout, r, ri, blockIdx.x * S::TX, blockIdx.y * S::TY, blockIdx.z * S::TZ,
                                 tile_smem);
}

template <typename T>
__global__ void k_copy(const T *__restrict__ a, T *__restrict__ b, size_t n) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// coarsest grid fallback: many Gauss-Seidel sweeps inside one thread block
template <typename T, int KIND>
__global__ void k_coarse_solve(lvl_dev L, T *__restrict__ x, const T *__restrict__ r, int sweeps) {
    body_coarse_solve<T, KIND>(L, x, r, sweeps);
}

// The coarse-level part of a V-cycle (levels cf..nlev-1) in one CTA, with
// those levels' x, r and residual arrays held in shared memory for the whole
// sub-cycle: every phase reads and writes shared memory and only
// __syncthreads separates phases.  x and r of level cf come in from global
// memory and x of level cf goes back; the coarser levels live only here (the
// restriction zeroes their x on the way down).
constexpr int kCoarseThreads = 512;

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads) k_mg_coarse(pmg_args A, int cf) {
    extern __shared__ __align__(16) unsigned char coarse_smem[];
    __shared__ pmg_args S;
    T *sm = reinterpret_cast<T *>(coarse_smem);
    if (threadIdx.x == 0) {
        S = A;
        size_t off = 0;
        for (int l = cf; l < A.nlev; l++) {
            pmg_level &L = S.lv[l];
            const size_t np = (size_t)L.n[0] * L.n[1] * L.n[2];
            set_level_ptrs<T>(L, sm + off, sm + off + np, sm + off + 2 * np);
            off += 3 * np;
        }
    }
    __syncthreads();
    const pmg_level &G = A.lv[cf];
    const int n0 = G.n[0] * G.n[1] * G.n[2];
    const T *gx = LX<T>(G), *gr = LR<T>(G);
    T *sx = LX<T>(S.lv[cf]), *sr = LR<T>(S.lv[cf]);
    for (int p = threadIdx.x; p < n0; p += blockDim.x) {
        sx[p] = gx[p];
        sr[p] = gr[p];
    }
    __syncthreads();
    coarse_cycle<T>(S, cf);
    __syncthreads();
    T *ox = LX<T>(G);
    for (int p = threadIdx.x; p < n0; p += blockDim.x) ox[p] = sx[p];
}

constexpr size_t kCoarseSmemMax = 200 * 1024;

// shared-memory bytes of k_mg_coarse from level cf down
static size_t coarse_smem_bytes(const std::vector<mg_level> &lv, int cf, size_t elem) {
    size_t b = 0;
    for (size_t l = cf; l < lv.size(); l++) b += 3 * lv[l].npts() * elem;
    return b;
}

// FP64 <-> FP32 helpers of the mixed form
__global__ void k_to_f32(const double *__restrict__ a, float *__restrict__ b, size_t n) { body_to_f32(a, b, n, blockIdx.x); }
__global__ void k_add_f32(double *__restrict__ a, const float *__restrict__ b, size_t n) { body_add_f32(a, b, n, blockIdx.x); }
template <typename T>
__global__ void k_zero(T *a, size_t n) {
    body_zero<T>(a, n, blockIdx.x);
}

// ---- host side -----------------------------------------------------------
static lvl_dev dev_of(const mg_level &l) { return lvl_dev{l.n[0], l.n[1], l.n[2], l.prd[0], l.prd[1], l.prd[2]}; }

static dim3 blk3() { return dim3(32, 4, 2); }
static dim3 grid3(int a, int b, int c) { return dim3((a + 31) / 32, (b + 3) / 4, (c + 1) / 2); }

template <typename T, int KIND, bool VD>
static int tile_attr(const void *fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem_bytes<T, KIND, VD>()) !=
           cudaSuccess;
}

int tile_setup_batched();  // k_mgb.cu

int tile_setup() {
    static std::once_flag once;
    static int err = 0;
    std::call_once(once, []() {
        err |= tile_attr<double, 0, false>((const void *)k_tile_sweep<double, 0, false>);
        err |= tile_attr<double, 0, true>((const void *)k_tile_sweep<double, 0, true>);
        err |= tile_attr<double, 1, false>((const void *)k_tile_sweep<double, 1, false>);
        err |= tile_attr<double, 1, true>((const void *)k_tile_sweep<double, 1, true>);
        err |= tile_attr<float, 0, false>((const void *)k_tile_sweep<float, 0, false>);
        err |= tile_attr<float, 0, true>((const void *)k_tile_sweep<float, 0, true>);
        err |= tile_attr<float, 1, false>((const void *)k_tile_sweep<float, 1, false>);
        err |= tile_attr<float, 1, true>((const void *)k_tile_sweep<float, 1, true>);
        err |= tile_setup_batched();
    });
    return err;
}

// one tiled sweep xin -> xout of level L
template <typename T, int KIND, bool VD>
static void tile_sweep_k(const mg_level &L, const T *xin, T *xout, const T *r, const T *ri, cudaStream_t st) {
    using S = tile_shape<T, KIND, VD>;
    const dim3 g((L.n[0] + S::TX - 1) / S::TX, (L.n[1] + S::TY - 1) / S::TY, (L.n[2] + S::TZ - 1) / S::TZ);
    const lvl_dev d{L.n[0], L.n[1], L.n[2], L.prd[0], L.prd[1], L.prd[2]};
    k_tile_sweep<T, KIND, VD><<<g, S::NT, tile_smem_bytes<T, KIND, VD>(), st>>>(d, xin, xout, r, ri);
}

template <typename T>
static void tile_sweep(mg_kind kind, const mg_level &L, const T *xin, T *xout, const T *r, const T *ri,
                       cudaStream_t st) {
    if (kind == MG_MAC) {
        if (ri) tile_sweep_k<T, 0, true>(L, xin, xout, r, ri, st);
        else tile_sweep_k<T, 0, false>(L, xin, xout, r, ri, st);
    } else {
        if (ri) tile_sweep_k<T, 1, true>(L, xin, xout, r, ri, st);
        else tile_sweep_k<T, 1, false>(L, xin, xout, r, ri, st);
    }
}

// Host copy of the level operator, for the coarsest-grid inverse.
static void host_stencil_row(mg_kind kind, const mg_level &L, int i, int j, int k, std::vector<double> &row) {
    const int n[3] = {L.n[0], L.n[1], L.n[2]};
    const int c[3] = {i, j, k};
    auto wrap = [&](int v, int d) -> int {
        if (v < 0) return L.prd[d] ? v + n[d] : -1;
        if (v >= n[d]) return L.prd[d] ? v - n[d] : -1;
        return v;
    };
    const int me = i + n[0] * (j + n[1] * k);
    if (kind == MG_MAC) {
        int missing = 0;
        for (int d = 0; d < 3; d++)
            for (int sg = -1; sg <= 1; sg += 2) {
                int q[3] = {i, j, k};
                q[d] = wrap(c[d] + sg, d);
                if (q[d] < 0) {
                    missing++;
                    continue;
                }
                row[q[0] + n[0] * (q[1] + n[1] * q[2])] += 1;
            }
        row[me] += -6 + missing;
        return;
    }
    bool bd[3];
    for (int d = 0; d < 3; d++) bd[d] = !L.prd[d] && (c[d] == 0 || c[d] == n[d] - 1);
    for (int oc = -1; oc <= 1; oc++)
        for (int ob = -1; ob <= 1; ob++)
            for (int oa = -1; oa <= 1; oa++) {
                int q[3] = {wrap(i + oa, 0), wrap(j + ob, 1), wrap(k + oc, 2)};
                if (q[0] < 0 || q[1] < 0 || q[2] < 0) continue;
                int nz = (oa != 0) + (ob != 0) + (oc != 0);
                double co = (nz == 0) ? 32 : (nz == 1 ? 0 : (nz == 2 ? -2 : -1));
                int halve = (bd[0] && oa == 0) + (bd[1] && ob == 0) + (bd[2] && oc == 0);
                co /= (double)(1 << halve);
                row[q[0] + n[0] * (q[1] + n[1] * q[2])] += co;
            }
}

// Dense inverse of the coarsest operator.  The operators here are singular
// with the constants as null space (Neumann walls or periodic wrap); adding
// (alpha/n) 1 1^T with alpha = mean diagonal makes the matrix SPD and its
// inverse maps every right-hand side to the solution of the projected system
// that is orthogonal to the constants.
// Process-wide cache of coarsest-level inverses: every solver whose coarsest
// level has the same kind, shape and periodicity on the same device shares
// one device copy (they are read-only), so creating many scenes of a few
// grid sizes inverts each matrix once.
namespace {
struct dense_key {
    int dev, kind, n0, n1, n2, p0, p1, p2;
    bool operator<(const dense_key &o) const {
        return std::tie(dev, kind, n0, n1, n2, p0, p1, p2) < std::tie(o.dev, o.kind, o.n0, o.n1, o.n2, o.p0, o.p1, o.p2);
    }
};
std::mutex g_dense_mu;
std::map<dense_key, double *> g_dense;
}  // namespace

int mg_solver::build_dense(cudaStream_t st) {
    const mg_level &L = lv.back();
    const int np = (int)L.npts();
    if (np > kDenseMax) return 0;  // Gauss-Seidel fallback
    int dev = 0;
    cudaGetDevice(&dev);
    const dense_key key{dev, (int)kind, L.n[0], L.n[1], L.n[2], L.prd[0], L.prd[1], L.prd[2]};
    std::lock_guard<std::mutex> lk(g_dense_mu);
    auto it = g_dense.find(key);
    if (it != g_dense.end()) {
        dense = it->second;
        return 0;
    }
    std::vector<double> A((size_t)np * np, 0.0), row(np);
    double dsum = 0, rsum_max = 0;
    for (int k = 0; k < L.n[2]; k++)
        for (int j = 0; j < L.n[1]; j++)
            for (int i = 0; i < L.n[0]; i++) {
                std::fill(row.begin(), row.end(), 0.0);
                host_stencil_row(kind, L, i, j, k, row);
                int me = i + L.n[0] * (j + L.n[1] * k);
                double rs = 0;
                for (int c = 0; c < np; c++) {
                    A[(size_t)me * np + c] = row[c];
                    rs += row[c];
                }
                dsum += row[me];
                rsum_max = std::max(rsum_max, std::fabs(rs));
            }
    if (rsum_max < 1e-12) {
        double alpha = dsum / np;
        for (size_t e = 0; e < A.size(); e++) A[e] += alpha / np;
    }
    // Gauss-Jordan with partial pivoting
    std::vector<double> B((size_t)np * np, 0.0);
    for (int r = 0; r < np; r++) B[(size_t)r * np + r] = 1;
    for (int col = 0; col < np; col++) {
        int piv = col;
        for (int r = col + 1; r < np; r++)
            if (std::fabs(A[(size_t)r * np + col]) > std::fabs(A[(size_t)piv * np + col])) piv = r;
        if (piv != col)
            for (int c = 0; c < np; c++) {
                std::swap(A[(size_t)piv * np + c], A[(size_t)col * np + c]);
                std::swap(B[(size_t)piv * np + c], B[(size_t)col * np + c]);
            }
        double d = A[(size_t)col * np + col];
        if (d == 0) return 0;  // keep the Gauss-Seidel fallback
        double inv = 1 / d;
        // columns left of col are already unit vectors in A
        for (int c = col; c < np; c++) A[(size_t)col * np + c] *= inv;
        for (int c = 0; c < np; c++) B[(size_t)col * np + c] *= inv;
        for (int r = 0; r < np; r++) {
            if (r == col) continue;
            double f = A[(size_t)r * np + col];
            if (f == 0) continue;
            for (int c = col; c < np; c++) A[(size_t)r * np + c] -= f * A[(size_t)col * np + c];
            for (int c = 0; c < np; c++) B[(size_t)r * np + c] -= f * B[(size_t)col * np + c];
        }
    }
    if (cudaMalloc(&dense, B.size() * sizeof(double)) != cudaSuccess) return 1;
    cudaMemcpyAsync(dense, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    g_dense[key] = dense;
    return 0;
}

// Choose the first level of the one-CTA coarse sub-cycle: the finest level
// with at most `pts` points whose sub-hierarchy fits the shared-memory cap.
int mg_solver::set_coarse(int pts) {
    coarse_pts = vd ? 0 : pts;
    pts = coarse_pts;
    invalidate();
    cf = (int)lv.size() - 1;
    for (int l = 0; l < (int)lv.size(); l++)
        if (lv[l].npts() <= (size_t)pts && coarse_smem_bytes(lv, l, 8) <= kCoarseSmemMax) {
            cf = l;
            break;
        }
    // the attribute is per kernel and process-wide: always the cap, so that
    // every solver's launch fits whatever other solvers set
    if (cudaFuncSetAttribute(k_mg_coarse<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax) !=
        cudaSuccess)
        return 1;
    if (cudaFuncSetAttribute(k_mg_coarse<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoarseSmemMax) !=
        cudaSuccess)
        return 1;
    return 0;
}

// Device memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// scene's stream): creating and destroying scenes does not synchronise the
// device, so scenes that come and go do not stall the others.
void mg_solver::release() {
    if (!alloc_stream) return;
    if (slab) cudaFreeAsync(slab, alloc_stream);
    slab = nullptr;
    for (auto &l : lv) {
        l.x = l.r = l.res = nullptr;
        l.xs = l.rs = l.ress = nullptr;
    }
    if (d_max) cudaFreeAsync(d_max, alloc_stream);
    d_max = nullptr;
    alloc_stream = nullptr;
}

mg_solver::~mg_solver() {
    release();
    invalidate();
    if (own_gb) {
        own_gb->release();
        delete own_gb;
    }
    if (cap_main) cudaStreamDestroy(cap_main);
}

int mg_solver::plan(mg_kind k, const int n[3], const int prd[3], std::vector<mg_level> &lv) {
    lv.clear();
    mg_level L0;
    for (int d = 0; d < 3; d++) {
        L0.n[d] = n[d];
        L0.prd[d] = prd[d];
    }
    lv.push_back(L0);
    while (true) {
        const mg_level &f = lv.back();
        if (f.npts() <= (size_t)kDensePts) break;  // solved exactly by the dense inverse
        mg_level c;
        bool ok = true;
        for (int d = 0; d < 3; d++) {
            c.prd[d] = f.prd[d];
            int len = f.n[d];
            if (k == MG_MAC) {
                if (len % 2 != 0 || len < 4) ok = false;
                c.n[d] = len / 2;
            } else if (f.prd[d]) {
                if (len % 2 != 0 || len < 4) ok = false;
                c.n[d] = len / 2;
            } else {
                if ((len - 1) % 2 != 0 || len < 3) ok = false;
                c.n[d] = (len - 1) / 2 + 1;
            }
        }
        if (!ok) break;
        lv.push_back(c);
    }
    if (lv.back().npts() > 4096) return fail(RMT3D_ERR_UNSUPPORTED, "grid does not coarsen to a small enough level");
    if ((int)lv.size() > kMaxLev) return fail(RMT3D_ERR_UNSUPPORTED, "too many multigrid levels");
    return 0;
}

size_t mg_solver::footprint(mg_kind k, const int n[3], const int prd[3], bool mixed_form) {
    std::vector<mg_level> v;
    if (plan(k, n, prd, v)) return 0;
    size_t b = 0;
    for (auto &l : v)
        b += 3 * slab_pad(l.npts() * sizeof(double)) + (mixed_form ? 3 * slab_pad(l.npts() * sizeof(float)) : 0);
    // the coarsest-level inverse is shared by all solvers with that level
    // (one copy per distinct level shape in the process) and not counted here
    return b + 2 * sizeof(double);
}

int mg_solver::setup(mg_kind k, const int n[3], const int prd[3], bool mixed_form, cudaStream_t st) {
    kind = k;
    mixed = mixed_form;
    const double eps = 2.220446049250313e-16;
    // tolerances of simp_fem / simp_mac (mg_probs.hh:483-485, :516-518)
    max_norm_tol = (k == MG_FEM) ? 32 * eps * 1e2 : 6 * eps * 1e2;
    int pe = plan(k, n, prd, lv);
    if (pe) return pe;
    alloc_stream = st;
    // all levels in one allocation, level by level, each array on a 256-byte
    // boundary: the arrays' relative placement is the same for every solver
    // whatever the state of the memory pool
    size_t total = 0;
    for (auto &l : lv)
        total += 3 * slab_pad(l.npts() * sizeof(double)) + (mixed ? 3 * slab_pad(l.npts() * sizeof(float)) : 0);
    if (cudaMallocAsync((void **)&slab, total, st) != cudaSuccess) return fail(RMT3D_ERR_OOM, "multigrid allocation failed");
    bytes_alloc += total;
    cudaMemsetAsync(slab, 0, total, st);
    size_t off = 0;
    auto carve = [&](size_t bytes) {
        unsigned char *p = slab + off;
        off += slab_pad(bytes);
        return (void *)p;
    };
    for (auto &l : lv) {
        const size_t b = l.npts() * sizeof(double);
        l.x = (double *)carve(b);
        l.r = (double *)carve(b);
        l.res = (double *)carve(b);
        if (mixed) {
            const size_t bf = l.npts() * sizeof(float);
            l.xs = (float *)carve(bf);
            l.rs = (float *)carve(bf);
            l.ress = (float *)carve(bf);
        }
    }
    if (build_dense(st)) return fail(RMT3D_ERR_OOM, "coarse inverse allocation failed");
    if (set_coarse(coarse_pts)) return fail(RMT3D_ERR_CUDA, "coarse multigrid kernel configuration failed");
    if (tile_setup()) return fail(RMT3D_ERR_CUDA, "tiled sweep kernel configuration failed");

    setup_cluster();
    {
        const char *e = getenv("RMT3D_MG_CLUSTER");
        if (e && e[0] == '1') use_cluster = true;
    }
    if (cudaMallocAsync((void **)&d_max, 2 * sizeof(unsigned long long), st) != cudaSuccess)
        return fail(RMT3D_ERR_OOM, "multigrid allocation failed");
    bytes_alloc += 2 * sizeof(unsigned long long);
    cudaMemsetAsync(d_max, 0, 2 * sizeof(unsigned long long), st);
    return 0;
}

#define LAUNCH(...)                           \
    do {                                      \
        __VA_ARGS__;                          \
        if (launches) (*launches)++;          \
    } while (0)

int mg_solver::smooth(int l, int sweeps, int cur, cudaStream_t st) {
    mg_level &L = lv[l];
    lvl_dev d = dev_of(L);
    // algorithmic bytes of one colour pass: read x of the whole level, read r
    // and write x of the updated colour; of one tiled sweep: read x and r and
    // write x of the whole level (and read 1/rho with variable density)
    const double npts = (double)L.npts();
    const bool timed = prof && l == 0 && prof->target == (kind == MG_FEM ? 0 : 1);
    double *xb[2] = {L.x, L.res};
    for (int s = 0; s < sweeps; s++) {
        if (smoother == 1) {
            if (timed) prof->begin(st);
            LAUNCH(tile_sweep<double>(kind, L, xb[cur], xb[cur ^ 1], L.r, L.ri, st));
            if (timed) prof->end(st, npts, 8.0 * npts * (L.ri ? 4 : 3));
            cur ^= 1;
        } else if (kind == MG_MAC) {
            dim3 g((L.n[0] / 2 + 1 + 31) / 32, (L.n[1] + 3) / 4, (L.n[2] + 1) / 2);
            for (int c = 0; c < 2; c++) {
                if (timed) prof->begin(st);
                LAUNCH(k_mac_rb<double><<<g, blk3(), 0, st>>>(d, xb[cur], L.r, c, L.ri));
                if (timed) prof->end(st, npts / 2, 8.0 * (npts + npts / 2 + npts / 2));
            }
        } else {
            dim3 g(((L.n[0] + 1) / 2 + 31) / 32, ((L.n[1] + 1) / 2 + 3) / 4, (L.n[2] + 1) / 2);
            for (int c = 0; c < 4; c++) {
                if (timed) prof->begin(st);
                LAUNCH(k_fem_gs<double><<<g, blk3(), 0, st>>>(d, xb[cur], L.r, c, L.ri));
                if (timed) prof->end(st, npts / 4, 8.0 * (npts + npts / 4 + npts / 4));
            }
        }
    }
    return cur;
}

int mg_solver::smooth_f32(int l, int sweeps, int cur, cudaStream_t st) {
    mg_level &L = lv[l];
    lvl_dev d = dev_of(L);
    const double npts = (double)L.npts();
    const bool timed = prof && l == 0 && prof->target == (kind == MG_FEM ? 0 : 1);
    float *xb[2] = {L.xs, L.ress};
    for (int s = 0; s < sweeps; s++) {
        if (smoother == 1) {
            if (timed) prof->begin(st);
            LAUNCH(tile_sweep<float>(kind, L, xb[cur], xb[cur ^ 1], L.rs, L.ris, st));
            if (timed) prof->end(st, npts, 4.0 * npts * (L.ris ? 4 : 3));
            cur ^= 1;
        } else if (kind == MG_MAC) {
            dim3 g((L.n[0] / 2 + 1 + 31) / 32, (L.n[1] + 3) / 4, (L.n[2] + 1) / 2);
            for (int c = 0; c < 2; c++) {
                if (timed) prof->begin(st);
                LAUNCH(k_mac_rb<float><<<g, blk3(), 0, st>>>(d, xb[cur], L.rs, c, L.ris));
                if (timed) prof->end(st, npts / 2, 4.0 * (npts + npts / 2 + npts / 2));
            }
        } else {
            dim3 g(((L.n[0] + 1) / 2 + 31) / 32, ((L.n[1] + 1) / 2 + 3) / 4, (L.n[2] + 1) / 2);
            for (int c = 0; c < 4; c++) {
                if (timed) prof->begin(st);
                LAUNCH(k_fem_gs<float><<<g, blk3(), 0, st>>>(d, xb[cur], L.rs, c, L.ris));
                if (timed) prof->end(st, npts / 4, 4.0 * (npts + npts / 4 + npts / 4));
            }
        }
    }
    return cur;
}

// level table of the coarse sub-cycle kernel
static pmg_args coarse_args(const mg_solver &m) {
    pmg_args A;
    memset(&A, 0, sizeof(A));
    A.kind = (m.kind == MG_MAC) ? 0 : 1;
    A.nlev = (int)m.lv.size();
    for (int l = 0; l < A.nlev && l < kMaxLev; l++) {
        pmg_level &P = A.lv[l];
        for (int d = 0; d < 3; d++) {
            P.n[d] = m.lv[l].n[d];
            P.prd[d] = m.lv[l].prd[d];
        }
        P.x = m.lv[l].x;
        P.r = m.lv[l].r;
        P.res = m.lv[l].res;
        P.xs = m.lv[l].xs;
        P.rs = m.lv[l].rs;
        P.ress = m.lv[l].ress;
        P.ri = m.lv[l].ri;
        P.ris = m.lv[l].ris;
    }
    A.dense = m.dense;
    A.v_up = m.v_up;
    A.v_down = m.v_down;
    return A;
}

int mg_solver::set_cluster_coarse(int pts) {
    cluster_coarse_pts = pts;
    ccl = -1;
    if (pts > 0 && cluster_size > 0)
        for (int l = 1; l + 1 < (int)lv.size(); l++)
            if (lv[l].npts() <= (size_t)pts) {
                ccl = l;
                break;
            }
    invalidate();
    return 0;
}

int mg_solver::cycle(int l, cudaStream_t st) {
    mg_level &F = lv[l];
    lvl_dev fd = dev_of(F);
    if (l == ccl) {
        LAUNCH(coarse_cluster(*this, l, false, st));
        return 0;
    }
    if (l == cf && l < (int)lv.size() - 1) {
        LAUNCH(k_mg_coarse<double><<<1, kCoarseThreads, coarse_smem_bytes(lv, l, 8), st>>>(coarse_args(*this), l));
        return 0;
    }
    if (l == (int)lv.size() - 1) {
        if (dense) LAUNCH(k_coarse_dense<double><<<((int)F.npts() + 7) / 8, 256, 0, st>>>((int)F.npts(), dense, F.x, F.r));
        else if (kind == MG_MAC) LAUNCH(k_coarse_solve<double, 0><<<1, 512, 0, st>>>(fd, F.x, F.r, 80));
        else LAUNCH(k_coarse_solve<double, 1><<<1, 512, 0, st>>>(fd, F.x, F.r, 80));
        return 0;
    }
    // the level's solution moves between its x and residual arrays with the
    // tiled sweeps; the residual goes to whichever of the two is free
    int cur = smooth(l, v_down, 0, st);
    double *xb[2] = {F.x, F.res};
    mg_level &C = lv[l + 1];
    lvl_dev cd = dev_of(C);
    dim3 gf = grid3(F.n[0], F.n[1], F.n[2]), gc = grid3(C.n[0], C.n[1], C.n[2]);
    if (kind == MG_MAC) {
        LAUNCH((k_resid<double, 0><<<gf, blk3(), 0, st>>>(fd, xb[cur], F.r, xb[cur ^ 1], nullptr, F.ri)));
        LAUNCH(k_mac_restrict<double><<<gc, blk3(), 0, st>>>(fd, cd, xb[cur ^ 1], C.r, C.x));
    } else {
        LAUNCH((k_resid<double, 1><<<gf, blk3(), 0, st>>>(fd, xb[cur], F.r, xb[cur ^ 1], nullptr, F.ri)));
        LAUNCH(k_fem_restrict<double><<<gc, blk3(), 0, st>>>(fd, cd, xb[cur ^ 1], C.r, C.x));
    }
    const int cc = cycle(l + 1, st);
    const double *xc = cc ? C.res : C.x;
    if (kind == MG_MAC) LAUNCH(k_mac_prolong<double><<<gf, blk3(), 0, st>>>(fd, cd, xb[cur], xc));
    else LAUNCH(k_fem_prolong<double><<<gf, blk3(), 0, st>>>(fd, cd, xb[cur], xc));
    return smooth(l, v_up, cur, st);
}

int mg_solver::cycle_f32(int l, cudaStream_t st) {
    mg_level &F = lv[l];
    lvl_dev fd = dev_of(F);
    if (l == ccl) {
        LAUNCH(coarse_cluster(*this, l, true, st));
        return 0;
    }
    if (l == cf && l < (int)lv.size() - 1) {
        LAUNCH(k_mg_coarse<float><<<1, kCoarseThreads, coarse_smem_bytes(lv, l, 4), st>>>(coarse_args(*this), l));
        return 0;
    }
    if (l == (int)lv.size() - 1) {
        if (dense) LAUNCH(k_coarse_dense<float><<<((int)F.npts() + 7) / 8, 256, 0, st>>>((int)F.npts(), dense, F.xs, F.rs));
        else if (kind == MG_MAC) LAUNCH(k_coarse_solve<float, 0><<<1, 512, 0, st>>>(fd, F.xs, F.rs, 80));
        else LAUNCH(k_coarse_solve<float, 1><<<1, 512, 0, st>>>(fd, F.xs, F.rs, 80));
        return 0;
    }
    int cur = smooth_f32(l, v_down, 0, st);
    float *xb[2] = {F.xs, F.ress};
    mg_level &C = lv[l + 1];
    lvl_dev cd = dev_of(C);
    dim3 gf = grid3(F.n[0], F.n[1], F.n[2]), gc = grid3(C.n[0], C.n[1], C.n[2]);
    if (kind == MG_MAC) {
        LAUNCH((k_resid<float, 0><<<gf, blk3(), 0, st>>>(fd, xb[cur], F.rs, xb[cur ^ 1], nullptr, F.ris)));
        LAUNCH(k_mac_restrict<float><<<gc, blk3(), 0, st>>>(fd, cd, xb[cur ^ 1], C.rs, C.xs));
    } else {
        LAUNCH((k_resid<float, 1><<<gf, blk3(), 0, st>>>(fd, xb[cur], F.rs, xb[cur ^ 1], nullptr, F.ris)));
        LAUNCH(k_fem_restrict<float><<<gc, blk3(), 0, st>>>(fd, cd, xb[cur ^ 1], C.rs, C.xs));
    }
    const int cc = cycle_f32(l + 1, st);
    const float *xc = cc ? C.ress : C.xs;
    if (kind == MG_MAC) LAUNCH(k_mac_prolong<float><<<gf, blk3(), 0, st>>>(fd, cd, xb[cur], xc));
    else LAUNCH(k_fem_prolong<float><<<gf, blk3(), 0, st>>>(fd, cd, xb[cur], xc));
    return smooth_f32(l, v_up, cur, st);
}

// One refinement step of the mixed form: FP64 residual, FP32 V-cycle on the
// correction, FP64 update.
void mg_solver::refine_step(cudaStream_t st) {
    mg_level &F = lv[0];
    lvl_dev fd = dev_of(F);
    dim3 gf = grid3(F.n[0], F.n[1], F.n[2]);
    size_t n = F.npts();
    unsigned nb = (unsigned)((n + 255) / 256);
    // FP64 residual -> FP32 right-hand side, FP32 start value zero (one pass)
    if (kind == MG_MAC) LAUNCH((k_resid_to_f32<0><<<gf, blk3(), 0, st>>>(fd, F.x, F.r, F.ri, F.rs, F.xs)));
    else LAUNCH((k_resid_to_f32<1><<<gf, blk3(), 0, st>>>(fd, F.x, F.r, F.ri, F.rs, F.xs)));
    const int cur = cycle_f32(0, st);
    LAUNCH(k_add_f32<<<nb, 256, 0, st>>>(F.x, cur ? F.ress : F.xs, n));
}

void mg_solver::iterate(cudaStream_t st) {
    if (mixed) {
        refine_step(st);
    } else if (cycle(0, st)) {
        // the fine level's solution ended in its residual array
        const size_t n = lv[0].npts();
        LAUNCH(k_copy<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(lv[0].res, lv[0].x, n));
    }
}

// ---- device-side control of one solve ---------------------------------------
// k_mg_begin arms a solve; k_mg_ctl runs after every iteration with the
// max-norm residual of the fine level and follows mg_prob::run
// (Utilities/mg_probs.cc:3-83):
//   iV/iP predicted cycles; then, while the residual is above the tolerance
//   (at most 20 times), rounds of 1, 2, 3, ... extra cycles; then two
//   insurance cycles; the reported residual is the last one measured before
//   the insurance cycles; mg_pred::update(extras) (mg_probs.hh:51-66).
// In the exact mode cycles continue after the insurance cycles while the
// residual keeps falling by 30% per cycle (at most 60), and the reported
// residual is the last one.  The residual is measured after every cycle; the
// measurements the reference does not take change nothing.
__global__ void k_mg_begin(mg_ctl *c, unsigned long long *mx, cudaGraphConditionalHandle h, int armed) {
    mg_begin_state(c, mx);
    if (armed) cudaGraphSetConditional(h, 1u);
}

// max |r| of the right-hand side into mx[1] (ordered bits), for the mixed
// form's relative tolerance
__global__ void k_absmax(const double *__restrict__ r, size_t n, unsigned long long *mx) {
    double a = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = fabs(r[i]);
        if (v != v || v > a) a = (v != v) ? __longlong_as_double(0x7ff8000000000000LL) : v;
    }
    unsigned long long b = (unsigned long long)__double_as_longlong(a);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
        b = t > b ? t : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(mx + 1, b);
}

__global__ void k_mg_ctl(mg_ctl *c, unsigned long long *mx, double tol, double rtol, int exact,
                         cudaGraphConditionalHandle h, int armed) {
    const bool done = mg_ctl_step(c, mx, tol, rtol, exact);
    if (armed) cudaGraphSetConditional(h, done ? 0u : 1u);
}

// one loop iteration: an iteration of the solver, the fine-level residual
// max-norm and the control kernel
void mg_solver::launch_body(cudaStream_t st, bool armed, unsigned long long h) {
    iterate(st);
    mg_level &F = lv[0];
    lvl_dev fd = dev_of(F);
    dim3 gf = grid3(F.n[0], F.n[1], F.n[2]);
    if (kind == MG_MAC) LAUNCH((k_resid_ctl<0><<<gf, blk3(), 0, st>>>(fd, F.x, F.r, d_max, F.ri, ctl)));
    else LAUNCH((k_resid_ctl<1><<<gf, blk3(), 0, st>>>(fd, F.x, F.r, d_max, F.ri, ctl)));
    LAUNCH(k_mg_ctl<<<1, 1, 0, st>>>(ctl, d_max, max_norm_tol, rtol, exact ? 1 : 0, h, armed ? 1 : 0));
}

int mg_solver::capture_solve(cudaStream_t cur, graph_builder &gb) {
    if (cluster_mode()) {
        // the whole solve is one kernel node
        gb.note(launch_cluster(cur));
        body_kernels = 0;
        outside_kernels = 1;
        return gb.err == cudaSuccess ? 0 : -1;
    }
    outside_kernels = rtol > 0 ? 2 : 1;
    cudaGraphConditionalHandle h = gb.handle(cur);
    if (gb.err != cudaSuccess) return -1;
    k_mg_begin<<<1, 1, 0, cur>>>(ctl, d_max, h, 1);
    if (rtol > 0) k_absmax<<<148, 256, 0, cur>>>(lv[0].r, lv[0].npts(), d_max);
    cudaStream_t body = gb.open(cur, h, cudaGraphCondTypeWhile);
    if (!body) return -1;
    long long n = 0, *saved = launches;
    launches = &n;
    launch_body(body, true, h);
    launches = saved;
    gb.close(body);
    body_kernels = (int)n;
    return gb.err == cudaSuccess ? (int)n : -1;
}

void mg_solver::invalidate() {
    if (solve_exec) cudaGraphExecDestroy(solve_exec);
    solve_exec = nullptr;
}

int mg_solver::build_solve_graph() {
    if (!own_gb) {
        own_gb = new graph_builder();
        if (own_gb->init()) return 1;
    }
    if (!cap_main && cudaStreamCreateWithFlags(&cap_main, cudaStreamNonBlocking) != cudaSuccess) return 1;
    own_gb->err = cudaSuccess;
    if (cudaStreamBeginCapture(cap_main, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return 1;
    int r = capture_solve(cap_main, *own_gb);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap_main, &g);
    if (r < 0 || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return 1;
    }
    e = cudaGraphInstantiate(&solve_exec, g, 0);
    cudaGraphDestroy(g);
    return e != cudaSuccess;
}

void mg_solver::sync_host_mirror() {
    last_cycles = h_ctl->last_cycles;
    cycles_total = h_ctl->cycles_total;
}

double mg_solver::run(cudaStream_t st) {
    // the kernel profiler times the per-phase kernels one launch at a time
    const bool profiling = prof && prof->target >= 0;
    if (!profiling && cluster_mode()) {
        if (launch_cluster(st) != cudaSuccess) return NAN;
        if (launches) (*launches)++;
        cudaMemcpyAsync(h_ctl, ctl, sizeof(mg_ctl), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return NAN;
        sync_host_mirror();
        return h_ctl->res_out;
    }
    const bool host_loop = !use_graph || profiling;
    if (host_loop) {
        // launch by launch, so that the profiler's events bracket single kernels
        k_mg_begin<<<1, 1, 0, st>>>(ctl, d_max, 0, 0);
        if (launches) (*launches)++;
        if (rtol > 0) {
            k_absmax<<<148, 256, 0, st>>>(lv[0].r, lv[0].npts(), d_max);
            if (launches) (*launches)++;
        }
        for (int guard = 0; guard < kMgMaxCycles; guard++) {
            launch_body(st, false, 0);
            cudaMemcpyAsync(h_ctl, ctl, sizeof(mg_ctl), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return NAN;
            if (!h_ctl->active) break;
        }
    } else {
        if (!solve_exec && build_solve_graph()) {
            fail(RMT3D_ERR_CUDA, "multigrid solve graph could not be built");
            return NAN;
        }
        const long long before = h_ctl->cycles_total;
        if (cudaGraphLaunch(solve_exec, st) != cudaSuccess) return NAN;
        cudaMemcpyAsync(h_ctl, ctl, sizeof(mg_ctl), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return NAN;
        if (launches) *launches += outside_kernels + (h_ctl->cycles_total - before) * body_kernels;
    }
    sync_host_mirror();
    return h_ctl->res_out;
}

}  // namespace rmt3d
