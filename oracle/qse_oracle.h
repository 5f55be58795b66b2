/*
 * qse_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference engine's FP64 algorithms, used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
 * checker.  The product (quantumsimevo_b200) never links or calls it.
 *
 * Parity is pinned two ways: (1) the QSETests known-answer vectors
 * (tests/golden/kat_qsetests.json) and (2) the reference's own sources
 * compiled here into oracle/_ref (oracle/Makefile, target `ref`), compared
 * amplitude by amplitude in tests/test_oracle_vs_reference.py.
 */
#ifndef QSE_ORACLE_H
#define QSE_ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include "../include/qse_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* state: 2^n complex128, interleaved */
void orc_init(double* st, unsigned n);
int  orc_apply(double* st, unsigned n, const qse_op* op, double theta);
int  orc_run(double* st, unsigned n, const qse_op* ops, size_t nops, const double* params);

/* sampling / measurement with injected uniforms */
void   orc_cdf(const double* st, unsigned n, double* cum);
size_t orc_lower_bound(const double* cum, size_t size, double target);
void   orc_sample(const double* st, unsigned n, const double* u, size_t nshots, uint64_t* out);
/* orc_sample plus the count of draws within `ulps` ulps of a cumulative boundary;
 * (size_t)-1 if the cumulative array cannot be allocated */
size_t orc_sample_margin(const double* st, unsigned n, const double* u, size_t nshots, uint64_t* out, double ulps);
uint64_t orc_measure(double* st, unsigned n, double u);
/* StateVector::measureQubit / resetQubit (StateVector.cpp:158-221), draw injected;
 * return the outcome, *prob1 = the probability of the qubit being 1 */
int orc_measure_qubit(double* st, unsigned n, unsigned q, double u, double* prob1);
int orc_reset_qubit(double* st, unsigned n, unsigned q, double u, double* prob1);

/* mt19937 + libstdc++ generate_canonical<double,53> */
typedef struct orc_mt { uint32_t mt[624]; int idx; } orc_mt;
void     orc_mt_seed(orc_mt* g, uint32_t seed);
uint32_t orc_mt_next(orc_mt* g);
double   orc_mt_canonical(orc_mt* g);

/* Philox4x32-10 (Salmon et al., SC'11) */
void   orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void   orc_philox_uniform_pair(uint64_t seed, uint64_t counter, double* u1, double* u2);

/* Noise.cpp restated: counts per qubit, decisions from a uniform source */
typedef struct orc_noise {
    unsigned n;
    int32_t bit[64];
    int32_t phase[64];
    double  rates[16];
    double  mult;
    int     mode;          /* qse_rng_mode */
    orc_mt  mt;
    uint64_t seed;
    uint64_t draws;        /* noisy gates so far (Philox counter) */
} orc_noise;
void orc_noise_init(orc_noise* nz, unsigned n, const qse_noise_config* cfg);
/* one gate: returns number of uniforms consumed from *inj (0 or 2) */
int  orc_noise_accumulate(orc_noise* nz, int type, unsigned target, const double* inj);
void orc_noise_apply(orc_noise* nz, double* st);
/* Circuit::execute with noise: accumulate before each gate, apply at the end */
int  orc_execute(double* st, unsigned n, const qse_op* ops, size_t nops, const double* params,
                 orc_noise* nz, const double* inj, size_t ninj);

/* diagonal Z-string observable */
double orc_expectation(const double* st, unsigned n, const qse_observable* obs);
double orc_obs_value(uint64_t x, const qse_observable* obs);
/* gradients: textbook adjoint and the two-term parameter-shift rule */
double orc_adjoint(unsigned n, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                   const qse_observable* obs, double* grad);
double orc_param_shift(unsigned n, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                       const qse_observable* obs, double* grad);

#ifdef __cplusplus
}
#endif
#endif
