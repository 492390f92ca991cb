/* PGMG-compatible single-rank "geometry" for the CPU oracle build (test
 * infrastructure).  Semantics follow the reference's call sites:
 *  - the grid holds m x n x o points on one rank (ai=aj=ak=0, sm=m, ...);
 *  - copying a geometry gives the nodal (corner) grid used by the FEM pressure
 *    projection, one point longer in every non-periodic direction
 *    (F3D_Source/fluid_3d.cc:33 and :2524-2548 index nodes 0..m there);
 *  - set_up_neighbors fills the 27-entry neighbour table with rank 0 where the
 *    neighbour exists through periodic wrap and -1 where a wall cuts it off
 *    (as consumed at F3D_Source/fluid_3d_comm.cc:96 and
 *    Extrapolation/extrap_helper.hh:295-404). */
#ifndef RMT3D_ORACLE_PGMG_GEOMETRY_HH
#define RMT3D_ORACLE_PGMG_GEOMETRY_HH
#include <mpi.h>

class geometry {
  public:
    int m, n, o;
    int mp, np, op;
    int ip, jp, kp;
    int sm, sn, so;
    int ai, aj, ak, bi, bj, bk;
    bool x_prd, y_prd, z_prd;
    int rank, procs;
    MPI_Comm cart;

    geometry(int m_, int n_, int o_, bool xp, bool yp, bool zp)
        : m(m_), n(n_), o(o_), mp(1), np(1), op(1), ip(0), jp(0), kp(0),
          sm(m_), sn(n_), so(o_), ai(0), aj(0), ak(0), bi(m_), bj(n_), bk(o_),
          x_prd(xp), y_prd(yp), z_prd(zp), rank(0), procs(1), cart(MPI_COMM_WORLD) {}

    /* nodal copy: one extra point in each non-periodic direction */
    geometry(const geometry &g)
        : m(g.m + (g.x_prd ? 0 : 1)), n(g.n + (g.y_prd ? 0 : 1)), o(g.o + (g.z_prd ? 0 : 1)),
          mp(1), np(1), op(1), ip(0), jp(0), kp(0),
          sm(m), sn(n), so(o), ai(0), aj(0), ak(0), bi(m), bj(n), bk(o),
          x_prd(g.x_prd), y_prd(g.y_prd), z_prd(g.z_prd), rank(0), procs(1), cart(g.cart) {}

    void set_up_neighbors(int *neigh) const {
        const bool prd[3] = {x_prd, y_prd, z_prd};
        for (int tag = 0; tag < 27; tag++) {
            int t[3] = {tag % 3, (tag / 3) % 3, tag / 9};
            bool ok = true;
            for (int d = 0; d < 3; d++)
                if (t[d] != 1 && !prd[d]) ok = false;
            neigh[tag] = ok ? 0 : -1;
        }
    }
    void free() {}
};
#endif
