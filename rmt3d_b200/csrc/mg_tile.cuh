// One whole Gauss-Seidel sweep (every colour) of a multigrid level in one
// launch, on shared-memory tiles.
//
// The colour passes of a sweep depend on each other: pass c reads the values
// pass c-1 wrote at distance one.  A block owns an output box of TX x TY x TZ
// points and copies the box with a halo of H = C points (C colours) on every
// side -- x, the right-hand side and, with variable density, 1/rho -- into
// shared memory with asynchronous copies (cp.async).  It then runs the C
// passes there, separated by barriers: pass c updates the colour-c points of
// the box shrunk by c + 1 points on every side, the region whose neighbours
// are exact after pass c - 1, so after C passes the output box is exact.  The
// halo's points are computed by the neighbouring blocks as well (overlapped
// tiling).  Walls end the halo: a point on a wall reads nothing beyond it, so
// the region does not shrink there.  Periodic axes load the wrapped points.
//
// Every point's update is the single-colour kernels' expression (mg_ops.cuh)
// with the same operands in the same order, read from the tile instead of
// global memory, so a tiled sweep gives exactly the bits of C colour passes.
// Blocks read the level's values from `xin` and write the swept values to
// `xout` (another array): a block's halo must see the values before the
// sweep, which an in-place update by neighbouring blocks would overwrite.
#pragma once
#include <cuda_runtime.h>

#include "mg_ops.cuh"

namespace rmt3d {

template <typename T, int KIND, bool VD>
struct tile_shape {
    static constexpr int C = KIND == 0 ? 2 : 4;  // colours of a sweep
    static constexpr int H = C;                  // halo on every side
    static constexpr int TX = 32;
    static constexpr int TY = KIND == 0 ? 16 : 8;
    // z depth: the box, its right-hand side and 1/rho fit the shared memory
    static constexpr int TZ = (KIND == 1 && VD && sizeof(T) == 8) ? 4 : 8;
    static constexpr int WX = TX + 2 * H, WY = TY + 2 * H, WZ = TZ + 2 * H;
    static constexpr int NT = 512;  // threads per block
    // variable density: 1/rho per cell.  MAC cells are the points; the FEM
    // box of cells is one wider per axis (node i uses cells i-1 and i)
    static constexpr int CX = KIND == 0 ? WX : WX + 1, CY = KIND == 0 ? WY : WY + 1,
                         CZ = KIND == 0 ? WZ : WZ + 1;
};

// x and right-hand-side boxes, and the 1/rho box with variable density
template <typename T, int KIND, bool VD>
constexpr size_t tile_smem_bytes() {
    using S = tile_shape<T, KIND, VD>;
    return 2 * (size_t)S::WX * S::WY * S::WZ * sizeof(T) + (VD ? (size_t)S::CX * S::CY * S::CZ * sizeof(T) : 0);
}

// asynchronous global -> shared copy of one element (LDGSTS), committed per plane
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N committed groups of this thread are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- stencils on the tile ---------------------------------------------------
// A point's neighbours are read through three plane pointers (z-1, z, z+1)
// and the offset o = lx + WX * ly of the point in its plane.

template <typename T, int WX>
struct tile_acc {
    const T *pm, *pc, *pp;
    int o;
    __device__ __forceinline__ T operator()(int a, int b, int c) const {
        const T *pl = c < 0 ? pm : (c > 0 ? pp : pc);
        return pl[o + a + WX * b];
    }
};

// mac_offdiag on the tile
template <typename T, int WX>
__device__ __forceinline__ T mac_offdiag_t(const lvl_dev L, const tile_acc<T, WX> &A, int i, int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        diag = (T)-6;
        return ((A(-1, 0, 0) + A(1, 0, 0)) + (A(0, -1, 0) + A(0, 1, 0))) + (A(0, 0, -1) + A(0, 0, 1));
    }
    T s = 0;
    int missing = 0;
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; d++) {
#pragma unroll
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            if (wrapi(c[d] + sgn, n[d], p[d]) < 0) {
                missing++;
                continue;
            }
            s += A(d == 0 ? sgn : 0, d == 1 ? sgn : 0, d == 2 ? sgn : 0);
        }
    }
    diag = (T)(-6 + missing);
    return s;
}

// mac_offdiag_vd on the tile (Rv: 1/rho of the points)
template <typename T, int WX>
__device__ __forceinline__ T mac_offdiag_vd_t(const lvl_dev L, const tile_acc<T, WX> &A, const tile_acc<T, WX> &Rv,
                                              int i, int j, int k, T &diag) {
    const T rc = Rv(0, 0, 0);
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        const T ax1 = (T)0.5 * (Rv(-1, 0, 0) + rc), ax2 = (T)0.5 * (rc + Rv(1, 0, 0));
        const T ay1 = (T)0.5 * (Rv(0, -1, 0) + rc), ay2 = (T)0.5 * (rc + Rv(0, 1, 0));
        const T az1 = (T)0.5 * (Rv(0, 0, -1) + rc), az2 = (T)0.5 * (rc + Rv(0, 0, 1));
        T s = 0, csum = 0;
        s += ax1 * A(-1, 0, 0) + ax2 * A(1, 0, 0);
        csum += ax1 + ax2;
        s += ay1 * A(0, -1, 0) + ay2 * A(0, 1, 0);
        csum += ay1 + ay2;
        s += az1 * A(0, 0, -1) + az2 * A(0, 0, 1);
        csum += az1 + az2;
        diag = (T)(-6) * (csum / (T)6);
        return s;
    }
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
    T s = 0, csum = 0;
    int cnt = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const bool lo = wrapi(c[d] - 1, n[d], p[d]) >= 0, hi = wrapi(c[d] + 1, n[d], p[d]) >= 0;
        const int da = d == 0, db = d == 1, dc = d == 2;
        if (lo && hi) {
            const T a1 = (T)0.5 * (Rv(-da, -db, -dc) + rc), a2 = (T)0.5 * (rc + Rv(da, db, dc));
            s += a1 * A(-da, -db, -dc) + a2 * A(da, db, dc);
            csum += a1 + a2;
            cnt += 2;
        } else if (lo) {
            const T a1 = (T)0.5 * (Rv(-da, -db, -dc) + rc);
            s += a1 * A(-da, -db, -dc);
            csum += a1;
            cnt += 1;
        } else if (hi) {
            const T a2 = (T)0.5 * (rc + Rv(da, db, dc));
            s += a2 * A(da, db, dc);
            csum += a2;
            cnt += 1;
        }
    }
    diag = (T)(-cnt) * (csum / (T)cnt);
    return s;
}

// fem_offdiag on the tile
template <typename T, int WX>
__device__ __forceinline__ T fem_offdiag_t(const lvl_dev L, const tile_acc<T, WX> &A, int i, int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        T e = (A(-1, -1, 0) + A(1, -1, 0)) + (A(-1, 1, 0) + A(1, 1, 0));
        e += (A(-1, 0, -1) + A(1, 0, -1)) + (A(0, -1, -1) + A(0, 1, -1));
        e += (A(-1, 0, 1) + A(1, 0, 1)) + (A(0, -1, 1) + A(0, 1, 1));
        T q = (A(-1, -1, -1) + A(1, -1, -1)) + (A(-1, 1, -1) + A(1, 1, -1));
        q += (A(-1, -1, 1) + A(1, -1, 1)) + (A(-1, 1, 1) + A(1, 1, 1));
        diag = (T)32;
        return (T)-2 * e - q;
    }
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int c[3] = {i, j, k};
    bool bd[3], ok[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bd[d] = !p[d] && (c[d] == 0 || c[d] == n[d] - 1);
#pragma unroll
        for (int o = -1; o <= 1; o++) ok[d][o + 1] = wrapi(c[d] + o, n[d], p[d]) >= 0;
    }
    T s = 0;
#pragma unroll
    for (int oc = 0; oc < 3; oc++) {
        if (!ok[2][oc]) continue;
#pragma unroll
        for (int ob = 0; ob < 3; ob++) {
            if (!ok[1][ob]) continue;
#pragma unroll
            for (int oa = 0; oa < 3; oa++) {
                if (!ok[0][oa]) continue;
                const int nz = (oa != 1) + (ob != 1) + (oc != 1);
                if (nz == 0 || nz == 1) continue;  // centre handled below, faces are 0
                T co = (nz == 2) ? (T)-2 : (T)-1;
                const int halve = (bd[0] && oa == 1) + (bd[1] && ob == 1) + (bd[2] && oc == 1);
                if (halve == 1) co *= (T)0.5;
                else if (halve == 2) co *= (T)0.25;
                s += co * A(oa - 1, ob - 1, oc - 1);
            }
        }
    }
    const int hc = bd[0] + bd[1] + bd[2];
    diag = (T)32 / (T)(1 << hc);
    return s;
}

// fem_offdiag_vd on the tile.  Rv reads the cells of the tile of cells: the
// cell below-left-front of the node is Rv(0, 0, 0) (its plane pointer pc is
// the cell plane k-1), the one above-right-back Rv(1, 1, 1).
template <typename T, int WX, int CX>
__device__ __forceinline__ T fem_offdiag_vd_t(const lvl_dev L, const tile_acc<T, WX> &A, const tile_acc<T, CX> &Rv,
                                              int i, int j, int k, T &diag) {
    if (i > 0 && i < L.n0 - 1 && j > 0 && j < L.n1 - 1 && k > 0 && k < L.n2 - 1) {
        T v[2][2][2];
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int e = 0; e < 2; e++) v[a][b][e] = Rv(e, b, a);
        T s = 0;
#pragma unroll
        for (int oc = 0; oc < 3; oc++)
#pragma unroll
            for (int ob = 0; ob < 3; ob++)
#pragma unroll
                for (int oa = 0; oa < 3; oa++) {
                    const int nz = (oa != 1) + (ob != 1) + (oc != 1);
                    if (nz <= 1) continue;
                    const T xv = A(oa - 1, ob - 1, oc - 1);
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
    const int n[3] = {L.n0, L.n1, L.n2}, p[3] = {L.p0, L.p1, L.p2};
    const int nc[3] = {p[0] ? n[0] : n[0] - 1, p[1] ? n[1] : n[1] - 1, p[2] ? n[2] : n[2] - 1};
    const int c[3] = {i, j, k};
    bool cell[3][2];  // the cells below / above the node on each axis exist
    bool bd[3], ok[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bd[d] = !p[d] && (c[d] == 0 || c[d] == n[d] - 1);
        cell[d][0] = (c[d] - 1 >= 0) || p[d];
        cell[d][1] = (c[d] < nc[d]) || p[d];
#pragma unroll
        for (int o = -1; o <= 1; o++) ok[d][o + 1] = wrapi(c[d] + o, n[d], p[d]) >= 0;
    }
    T v[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int e = 0; e < 2; e++) v[a][b][e] = (cell[0][e] && cell[1][b] && cell[2][a]) ? Rv(e, b, a) : (T)0;
    T s = 0;
#pragma unroll
    for (int oc = 0; oc < 3; oc++) {
#pragma unroll
        for (int ob = 0; ob < 3; ob++) {
#pragma unroll
            for (int oa = 0; oa < 3; oa++) {
                const int nz = (oa != 1) + (ob != 1) + (oc != 1);
                if (nz <= 1) continue;
                if (!ok[2][oc] || !ok[1][ob] || !ok[0][oa]) continue;
                T co = (nz == 2) ? (T)-2 : (T)-1;
                const int halve = (bd[0] && oa == 1) + (bd[1] && ob == 1) + (bd[2] && oc == 1);
                if (halve == 1) co *= (T)0.5;
                else if (halve == 2) co *= (T)0.25;
                T sum = 0;
                int num = 0;
#pragma unroll
                for (int a = (oc == 2 ? 1 : 0); a <= (oc == 0 ? 0 : 1); a++)
#pragma unroll
                    for (int b = (ob == 2 ? 1 : 0); b <= (ob == 0 ? 0 : 1); b++)
#pragma unroll
                        for (int e = (oa == 2 ? 1 : 0); e <= (oa == 0 ? 0 : 1); e++)
                            if (cell[2][a] && cell[1][b] && cell[0][e]) {
                                sum += v[a][b][e];
                                num++;
                            }
                s += co * div_pow2(sum, num) * A(oa - 1, ob - 1, oc - 1);
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
                if (cell[2][a] && cell[1][b] && cell[0][e]) {
                    sum += v[a][b][e];
                    num++;
                }
    const int hc = bd[0] + bd[1] + bd[2];
    diag = ((T)32 / (T)(1 << hc)) * div_pow2(sum, num);
    return s;
}

// ---- the sweep ----------------------------------------------------------------
// Global coordinate of local index l on an axis whose tile starts at u0:
// wrapped on a periodic axis, -1 outside a walled one.
__device__ __forceinline__ int tile_coord(int u, int n, int prd) {
    if (u < 0) return prd ? ((u % n) + n) % n : -1;
    if (u >= n) return prd ? u % n : -1;
    return u;
}

// One sweep of the level over the output box starting at (X0, Y0, Z0): reads
// xin, writes xout (both the level's layout).
template <typename T, int KIND, bool VD>
__device__ __forceinline__ void body_tile_sweep(const lvl_dev L, const T *__restrict__ xin, T *__restrict__ xout,
                                                const T *__restrict__ r, const T *__restrict__ ri, int X0, int Y0,
                                                int Z0, unsigned char *smem) {
    using S = tile_shape<T, KIND, VD>;
    constexpr int C = S::C, H = S::H, WX = S::WX, WY = S::WY, WZ = S::WZ, CX = S::CX, CY = S::CY, CZ = S::CZ;
    constexpr int WXY = WX * WY, WN = WXY * WZ;
    T *xs = reinterpret_cast<T *>(smem);
    T *rr = xs + WN;  // right-hand side
    T *rs = rr + WN;  // 1/rho (VD)
    const int tid = threadIdx.x;
    const int n0 = L.n0, n1 = L.n1, n2 = L.n2;
    const size_t sy = (size_t)n0, sz = (size_t)n0 * n1;
    // the box with its halo, copied asynchronously; points outside a walled
    // domain are zero (no point of the passes reads them)
    for (int e = tid; e < WN; e += S::NT) {
        const int lx = e % WX, ly = (e / WX) % WY, lz = e / WXY;
        const int gx = tile_coord(X0 - H + lx, n0, L.p0), gy = tile_coord(Y0 - H + ly, n1, L.p1),
                  gz = tile_coord(Z0 - H + lz, n2, L.p2);
        if (gx >= 0 && gy >= 0 && gz >= 0) {
            const size_t gi = gx + sy * gy + sz * gz;
            cp_async_elem(xs + e, xin + gi);
            cp_async_elem(rr + e, r + gi);
            if constexpr (VD && KIND == 0) cp_async_elem(rs + e, ri + gi);
        } else {
            xs[e] = (T)0;
            rr[e] = (T)0;
            if constexpr (VD && KIND == 0) rs[e] = (T)0;
        }
    }
    if constexpr (VD && KIND == 1) {
        // the cells around the box's nodes: cell c lies between nodes c and c+1
        const int nc0 = L.p0 ? n0 : n0 - 1, nc1 = L.p1 ? n1 : n1 - 1, nc2 = L.p2 ? n2 : n2 - 1;
        for (int e = tid; e < CX * CY * CZ; e += S::NT) {
            const int lx = e % CX, ly = (e / CX) % CY, lz = e / (CX * CY);
            const int cx = tile_coord(X0 - H - 1 + lx, nc0, L.p0), cy = tile_coord(Y0 - H - 1 + ly, nc1, L.p1),
                      cz = tile_coord(Z0 - H - 1 + lz, nc2, L.p2);
            if (cx >= 0 && cy >= 0 && cz >= 0) cp_async_elem(rs + e, ri + cx + (size_t)nc0 * (cy + (size_t)nc1 * cz));
            else rs[e] = (T)0;
        }
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const int T0[3] = {X0, Y0, Z0}, TT[3] = {S::TX, S::TY, S::TZ}, NN[3] = {n0, n1, n2}, PP[3] = {L.p0, L.p1, L.p2};
#pragma unroll
    for (int c = 0; c < C; c++) {
        // the range of pass c on each axis, in global (unwrapped) coordinates:
        // the box shrunk by c + 1, but not past a wall
        int lo[3], hi[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            lo[d] = T0[d] - H + c + 1;
            hi[d] = T0[d] + TT[d] + H - 2 - c;
            if (!PP[d]) {
                lo[d] = max(lo[d], 0);
                hi[d] = min(hi[d], NN[d] - 1);
            }
        }
        int px, py, nx, ny;
        const int nz = hi[2] - lo[2] + 1;
        if constexpr (KIND == 1) {  // colour c: (x, y) parities (c & 1, c >> 1), every z
            px = (lo[0] & 1) == (c & 1) ? lo[0] : lo[0] + 1;
            py = (lo[1] & 1) == ((c >> 1) & 1) ? lo[1] : lo[1] + 1;
            nx = hi[0] >= px ? (hi[0] - px) / 2 + 1 : 0;
            ny = hi[1] >= py ? (hi[1] - py) / 2 + 1 : 0;
        } else {  // colour c: parity of x + y + z; at most half a row each
            px = lo[0];
            py = lo[1];
            nx = (hi[0] - lo[0] + 2) / 2;
            ny = hi[1] - lo[1] + 1;
        }
        const int total = nx * ny * (nz > 0 ? nz : 0);
        for (int e = tid; e < total; e += S::NT) {
            int ux, uy;
            const int uz = lo[2] + e / (nx * ny);
            const int exy = e % (nx * ny);
            if constexpr (KIND == 1) {
                ux = px + 2 * (exy % nx);
                uy = py + 2 * (exy / nx);
            } else {
                uy = py + exy / nx;
                ux = lo[0] + (((lo[0] + uy + uz + c) & 1) ? 1 : 0) + 2 * (exy % nx);
                if (ux > hi[0]) continue;
            }
            const int lx = ux - (X0 - H), ly = uy - (Y0 - H), lz = uz - (Z0 - H);
            const int gx = tile_coord(ux, n0, L.p0), gy = tile_coord(uy, n1, L.p1), gz = tile_coord(uz, n2, L.p2);
            const int o = lx + WX * ly + WXY * lz;
            tile_acc<T, WX> A{xs - WXY, xs, xs + WXY, o};
            const T rv = rr[o];
            T diag, s;
            if constexpr (KIND == 0) {
                if constexpr (VD) {
                    tile_acc<T, WX> Rv{rs - WXY, rs, rs + WXY, o};
                    s = mac_offdiag_vd_t<T, WX>(L, A, Rv, gx, gy, gz, diag);
                } else {
                    s = mac_offdiag_t<T, WX>(L, A, gx, gy, gz, diag);
                }
                xs[o] = (rv - s) / diag;
            } else {
                if constexpr (VD) {
                    // the cell box is one wider: local cell (lx, ly, lz) is the
                    // cell below-left-front of local node (lx, ly, lz)
                    const T *cp = rs + CX * CY * lz;
                    tile_acc<T, CX> Rv{nullptr, cp, cp + CX * CY, lx + CX * ly};
                    s = fem_offdiag_vd_t<T, WX, CX>(L, A, Rv, gx, gy, gz, diag);
                    xs[o] = (rv - s) / diag;
                } else {
                    s = fem_offdiag_t<T, WX>(L, A, gx, gy, gz, diag);
                    xs[o] = (rv - s) * fem_inv_diag<T>(L, gx, gy, gz);
                }
            }
        }
        __syncthreads();
    }
    // the output box
    for (int e = tid; e < S::TX * S::TY * S::TZ; e += S::NT) {
        const int ux = X0 + e % S::TX, uy = Y0 + (e / S::TX) % S::TY, uz = Z0 + e / (S::TX * S::TY);
        if (ux < n0 && uy < n1 && uz < n2)
            xout[ux + sy * uy + sz * uz] = xs[(ux - X0 + H) + WX * (uy - Y0 + H) + WXY * (uz - Z0 + H)];
    }
}

}  // namespace rmt3d
