/* PGMG-compatible "common.hh" for the CPU oracle build (test infrastructure).
 * Provides the error helpers and the world communicator that the reference's
 * sources take from the PGMG library (absent here; see the call sites listed in
 * the oracle's README).  Written from the call sites, not from PGMG's source. */
#ifndef RMT3D_ORACLE_PGMG_COMMON_HH
#define RMT3D_ORACLE_PGMG_COMMON_HH
#include <cstdio>
#include <cstdlib>
#include <mpi.h>

#define PGMG_SETUP_ERROR 1
#define PGMG_INTERNAL_ERROR 2
#define PGMG_MATH_ERROR 3
#define PGMG_FILE_ERROR 4
#define PGMG_MEMORY_ERROR 5

static const MPI_Comm world = MPI_COMM_WORLD;

/* message tags used by the reference's slice/contour gathers */
const int msg_trans_dims = 1 << 14;
const int msg_contour1 = (1 << 14) + 1;
const int msg_contour2 = (1 << 14) + 2;
const int msg_contour3 = (1 << 14) + 3;
const int msg_contour4 = (1 << 14) + 4;

inline void fatal_error(const char *msg, int code) {
    fprintf(stderr, "Error: %s\n", msg);
    exit(code == 0 ? 1 : code);
}
inline void p_fatal_error(const char *msg, int code) { fatal_error(msg, code); }
inline void p_die() { fatal_error("internal error", PGMG_INTERNAL_ERROR); }
inline FILE *safe_fopen(const char *fn, const char *mode) {
    FILE *f = fopen(fn, mode);
    if (f == NULL) {
        fprintf(stderr, "Unable to open file '%s'\n", fn);
        exit(PGMG_FILE_ERROR);
    }
    return f;
}
inline FILE *p_safe_fopen(const char *fn, const char *mode) { return safe_fopen(fn, mode); }
#endif
