/* Minimal deterministic stand-in for the GSL random-number API used by the
 * reference's passive tracers (Utilities/tracers.cc:28-53).  Test
 * infrastructure for the CPU oracle build only; tracers are off (dump_code 0)
 * in every configuration the oracle runs, so the stream itself never matters. */
#ifndef RMT3D_ORACLE_GSL_RNG_SHIM_H
#define RMT3D_ORACLE_GSL_RNG_SHIM_H
#include <cstdint>

struct gsl_rng_type { int id; };
struct gsl_rng { uint64_t state; };
static const gsl_rng_type gsl_rng_taus_impl = {0};
static const gsl_rng_type *gsl_rng_taus = &gsl_rng_taus_impl;

inline void gsl_rng_env_setup() {}
inline gsl_rng *gsl_rng_alloc(const gsl_rng_type *) { gsl_rng *r = new gsl_rng; r->state = 1; return r; }
inline void gsl_rng_set(gsl_rng *r, unsigned long s) { r->state = s ? s : 1; }
inline double gsl_rng_uniform(gsl_rng *r) {
    /* xorshift64*, mapped to [0,1) */
    r->state ^= r->state >> 12; r->state ^= r->state << 25; r->state ^= r->state >> 27;
    return (double)((r->state * 2685821657736338717ULL) >> 11) * (1.0 / 9007199254740992.0);
}
inline void gsl_rng_free(gsl_rng *r) { delete r; }
#endif
