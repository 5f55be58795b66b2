/*
 * qse_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Plain-C restatement of the reference engine's FP64 algorithms on the hot
 * path.  Each function cites the reference lines it follows (paths relative
 * to the QuantumSimEvo project).  Arithmetic is written in the same order as
 * the reference's std::complex<double> expressions compile to with GCC
 * (complex product re = ar*br - ai*bi, im = ar*bi + ai*br; scalar*complex
 * scales both parts), and this file is compiled with -ffp-contract=off, so the
 * gate results match the reference scalar backend bit for bit.
 *
 * Element-wise gate loops run under OpenMP (every iteration writes its own
 * amplitudes, so the results do not depend on the thread count); the
 * expectation and gradient sums use a fixed chunked order (the same bits for
 * any thread count); reductions that the reference performs in index order
 * (cumulative sums, measure's running sum, measureQubit's probability) stay
 * sequential.
 *
 * Pinning: tests/test_oracle_kat.py checks these functions against the
 * QSETests known answers; tests/test_oracle_vs_reference.py against the
 * reference sources compiled into oracle/_ref.
 */
#include "qse_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

static inline cplx cmk(double re, double im) { cplx z = {re, im}; return z; }
/* GCC expansion of a complex<double> product */
static inline cplx cmul(cplx a, cplx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cplx cadd(cplx a, cplx b) { return cmk(a.re + b.re, a.im + b.im); }
static inline cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
/* double * complex<double>: libstdc++ scales both parts */
static inline cplx cscl(double s, cplx a) { return cmk(a.re * s, a.im * s); }
/* std::exp(Complex(0, t)) == glibc cexp(0 + i t) == (cos t, sin t) */
static inline cplx cexpi(double t) { return cmk(cos(t), sin(t)); }
static inline double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }

#define AMP(st, i) (((cplx*)(st))[i])

/* Reductions under OpenMP in a fixed order: kChunks contiguous index ranges
 * summed in parallel, then the chunk sums in chunk order -- the same bits for
 * every thread count and every run. */
enum { kChunks = 256 };
static size_t chunk_len(size_t size) { return (size + kChunks - 1) / kChunks; }
static double sum_parts(const double* part)
{
    double acc = 0.0;
    for (int c = 0; c < kChunks; ++c) acc += part[c];
    return acc;
}

void orc_init(double* st, unsigned n)
{
    /* StateVector.cpp:14-27: zero fill, amplitude 0 = 1 */
    size_t size = (size_t)1 << n;
    memset(st, 0, size * 2 * sizeof(double));
    st[0] = 1.0;
}

/* CircuitUnitaryOperation.cpp:10-36 (applyGate) */
static void g_2x2(double* st, unsigned n, const cplx g[4], unsigned q)
{
    size_t size = (size_t)1 << n, sec = (size_t)1 << q;
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < (size >> 1); ++i) {
        size_t i0 = ((i >> q) << (q + 1)) | (i & (sec - 1));
        size_t i1 = i0 | sec;
        cplx lo = AMP(st, i0), hi = AMP(st, i1);
        AMP(st, i0) = cadd(cmul(g[0], lo), cmul(g[1], hi));
        AMP(st, i1) = cadd(cmul(g[2], lo), cmul(g[3], hi));
    }
}

/* CircuitUnitaryOperation.cpp:38-59 (applyCNOT) */
static void g_cnot(double* st, unsigned n, unsigned c, unsigned t)
{
    size_t size = (size_t)1 << n, cm = (size_t)1 << c, tm = (size_t)1 << t;
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if ((i & cm) && (i < (i ^ tm))) {
            cplx tmp = AMP(st, i);
            AMP(st, i) = AMP(st, i ^ tm);
            AMP(st, i ^ tm) = tmp;
        }
}

/* CircuitUnitaryOperation.cpp:61-79 (applyPauliX) */
static void g_x(double* st, unsigned n, unsigned q)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (!(i & m)) {
            cplx tmp = AMP(st, i);
            AMP(st, i) = AMP(st, i | m);
            AMP(st, i | m) = tmp;
        }
}

/* CircuitUnitaryOperation.cpp:81-110 (applyHadamard), s = 0.7071067811865475244 */
static void g_h(double* st, unsigned n, unsigned q)
{
    const double s = 0.7071067811865475244;
    size_t size = (size_t)1 << n, step = (size_t)1 << q;
    /* the reference's blocked double loop visits each pair (j, j + step) once;
     * the same pairs as one flat loop over pair indices */
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < (size >> 1); ++k) {
        size_t j = ((k >> q) << (q + 1)) | (k & (step - 1));
        cplx v0 = AMP(st, j), v1 = AMP(st, j + step);
        AMP(st, j) = cscl(s, cadd(v0, v1));
        AMP(st, j + step) = cscl(s, csub(v0, v1));
    }
}

/* CircuitUnitaryOperation.cpp:112-132 (applyPhase) */
static void g_phase(double* st, unsigned n, unsigned q, double theta)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    cplx ph = cexpi(theta);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (i & m) AMP(st, i) = cmul(AMP(st, i), ph);
}

/* CircuitUnitaryOperation.cpp:134-160 (applyPauliY): (-I*v1, I*v0) */
static void g_y(double* st, unsigned n, unsigned q)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    const cplx I = cmk(0.0, 1.0), mI = cmk(-0.0, -1.0);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (!(i & m)) {
            cplx v0 = AMP(st, i), v1 = AMP(st, i | m);
            AMP(st, i) = cmul(mI, v1);
            AMP(st, i | m) = cmul(I, v0);
        }
}

/* CircuitUnitaryOperation.cpp:162-179 (applyPauliZ) -- the scalar backend,
 * not the AVX2 one whose loop skips qubit 0 (CircuitUnitaryOperationAVX.cpp:131-138) */
static void g_z(double* st, unsigned n, unsigned q)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (i & m) AMP(st, i) = cmk(-AMP(st, i).re, -AMP(st, i).im);
}

/* CircuitUnitaryOperation.cpp:181-208 (applyRotateX) */
static void g_rx(double* st, unsigned n, unsigned q, double theta)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    double c = cos(theta / 2.0), s = sin(theta / 2.0);
    cplx miS = cmk(0.0, -s);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (!(i & m)) {
            cplx v0 = AMP(st, i), v1 = AMP(st, i | m);
            AMP(st, i) = cadd(cscl(c, v0), cmul(miS, v1));
            AMP(st, i | m) = cadd(cmul(miS, v0), cscl(c, v1));
        }
}

/* CircuitUnitaryOperation.cpp:210-236 (applyRotateY) */
static void g_ry(double* st, unsigned n, unsigned q, double theta)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    double c = cos(theta / 2.0), s = sin(theta / 2.0);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (!(i & m)) {
            cplx v0 = AMP(st, i), v1 = AMP(st, i | m);
            AMP(st, i) = csub(cscl(c, v0), cscl(s, v1));
            AMP(st, i | m) = cadd(cscl(s, v0), cscl(c, v1));
        }
}

/* CircuitUnitaryOperation.cpp:238-265 (applyRotateZ) */
static void g_rz(double* st, unsigned n, unsigned q, double theta)
{
    size_t size = (size_t)1 << n, m = (size_t)1 << q;
    cplx p0 = cexpi(-theta / 2.0), p1 = cexpi(theta / 2.0);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        AMP(st, i) = cmul(AMP(st, i), (i & m) ? p1 : p0);
}

/* CircuitUnitaryOperation.cpp:267-289 (applySwap) */
static void g_swap(double* st, unsigned n, unsigned q0, unsigned q1)
{
    size_t size = (size_t)1 << n, m0 = (size_t)1 << q0, m1 = (size_t)1 << q1;
    unsigned lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
    size_t low_mask = ((size_t)1 << lo) - 1;
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < size / 4; ++k) {
        size_t i = ((k >> lo) << (lo + 1)) | (k & low_mask);
        size_t idx = ((i >> hi) << (hi + 1)) | (i & (((size_t)1 << hi) - 1));
        cplx tmp = AMP(st, idx | m0);
        AMP(st, idx | m0) = AMP(st, idx | m1);
        AMP(st, idx | m1) = tmp;
    }
}

/* CircuitUnitaryOperation.cpp:291-312 (applyMCPhase) */
static void g_mcphase(double* st, unsigned n, uint64_t all_mask, double theta)
{
    size_t size = (size_t)1 << n;
    cplx ph = cexpi(theta);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if (((uint64_t)i & all_mask) == all_mask) AMP(st, i) = cmul(AMP(st, i), ph);
}

/* CircuitUnitaryOperation.cpp:314-339 (applyCPhase): explicit (re*c - im*s, re*s + im*c) */
static void g_cphase(double* st, unsigned n, unsigned c, unsigned t, double theta)
{
    size_t size = (size_t)1 << n, cm = (size_t)1 << c, tm = (size_t)1 << t;
    double co = cos(theta), si = sin(theta);
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i)
        if ((i & cm) && (i & tm)) {
            double re = AMP(st, i).re, im = AMP(st, i).im;
            AMP(st, i) = cmk(re * co - im * si, re * si + im * co);
        }
}

static int qubit_ok(unsigned q, unsigned n) { return q < n; }

/* One GateCommand, dispatched like Circuit::execute's switch (Circuit.cpp:73-112).
 * theta is the bound angle. Returns 0, or -1 for a bad qubit / unsupported type. */
int orc_apply(double* st, unsigned n, const qse_op* op, double theta)
{
    switch (op->type) {
    case QSE_GATE_IDENTITY: return 0;
    case QSE_GATE_H: if (!qubit_ok(op->target, n)) return -1; g_h(st, n, op->target); return 0;
    case QSE_GATE_X: if (!qubit_ok(op->target, n)) return -1; g_x(st, n, op->target); return 0;
    case QSE_GATE_Y: if (!qubit_ok(op->target, n)) return -1; g_y(st, n, op->target); return 0;
    case QSE_GATE_Z: if (!qubit_ok(op->target, n)) return -1; g_z(st, n, op->target); return 0;
    case QSE_GATE_PHASE: if (!qubit_ok(op->target, n)) return -1; g_phase(st, n, op->target, theta); return 0;
    case QSE_GATE_RX: if (!qubit_ok(op->target, n)) return -1; g_rx(st, n, op->target, theta); return 0;
    case QSE_GATE_RY: if (!qubit_ok(op->target, n)) return -1; g_ry(st, n, op->target, theta); return 0;
    case QSE_GATE_RZ: if (!qubit_ok(op->target, n)) return -1; g_rz(st, n, op->target, theta); return 0;
    case QSE_GATE_CNOT:
        if (!qubit_ok(op->target, n) || !qubit_ok(op->control, n)) return -1;
        g_cnot(st, n, op->control, op->target); return 0;
    case QSE_GATE_CPHASE:
        if (!qubit_ok(op->target, n) || !qubit_ok(op->control, n)) return -1;
        g_cphase(st, n, op->control, op->target, theta); return 0;
    case QSE_GATE_MCPHASE: {
        if (!qubit_ok(op->target, n)) return -1;
        if (n < 64 && (op->controls >> n) != 0) return -1;
        g_mcphase(st, n, op->controls | ((uint64_t)1 << op->target), theta); return 0;
    }
    case QSE_GATE_SWAP:
        if (!qubit_ok(op->target, n) || !qubit_ok(op->control, n)) return -1;
        g_swap(st, n, op->target, op->control); return 0;
    case QSE_GATE_2X2: {
        if (!qubit_ok(op->target, n)) return -1;
        cplx g[4] = {cmk(op->m[0], op->m[1]), cmk(op->m[2], op->m[3]),
                     cmk(op->m[4], op->m[5]), cmk(op->m[6], op->m[7])};
        g_2x2(st, n, g, op->target); return 0;
    }
    default: return -1;
    }
}

static double bound_angle(const qse_op* op, const double* params)
{
    if (op->param >= 0 && params) return op->theta + op->coeff * params[op->param];
    return op->theta;
}

int orc_run(double* st, unsigned n, const qse_op* ops, size_t nops, const double* params)
{
    for (size_t k = 0; k < nops; ++k)
        if (orc_apply(st, n, &ops[k], bound_angle(&ops[k], params)) != 0) return -1;
    return 0;
}

/* ---------------- sampling / measurement ---------------- */

/* StateVector.cpp:85-92: norms, then a sequential inclusive prefix sum */
void orc_cdf(const double* st, unsigned n, double* cum)
{
    size_t size = (size_t)1 << n;
    for (size_t i = 0; i < size; ++i) cum[i] = cnorm(AMP(st, i));
    for (size_t i = 1; i < size; ++i) cum[i] += cum[i - 1];
}

/* std::lower_bound: first i with !(cum[i] < target) (StateVector.cpp:106-107) */
size_t orc_lower_bound(const double* cum, size_t size, double target)
{
    size_t lo = 0, len = size;
    while (len > 0) {
        size_t half = len >> 1, mid = lo + half;
        if (cum[mid] < target) { lo = mid + 1; len = len - half - 1; }
        else len = half;
    }
    return lo;
}

/* StateVector.cpp:77-116 with the uniform draw injected:
 * target = uniform_real_distribution(0, total) = u * (total - 0) + 0 */
void orc_sample(const double* st, unsigned n, const double* u, size_t nshots, uint64_t* out)
{
    size_t size = (size_t)1 << n;
    double* cum = (double*)malloc(size * sizeof(double));
    orc_cdf(st, n, cum);
    double total = cum[size - 1];
    for (size_t s = 0; s < nshots; ++s) {
        double target = u[s] * (total - 0.0) + 0.0;
        out[s] = orc_lower_bound(cum, size, target);
    }
    free(cum);
}

/* orc_sample, and in the same cumulative array (one build: at 30 qubits it
 * is 8 GiB) the number of draws whose target lies within `ulps` units in the
 * last place of the cumulative value at or just below the chosen index --
 * the draws where a differently rounded prefix sum could pick a neighbour. */
size_t orc_sample_margin(const double* st, unsigned n, const double* u, size_t nshots, uint64_t* out, double ulps)
{
    size_t size = (size_t)1 << n;
    double* cum = (double*)malloc(size * sizeof(double));
    if (!cum) return (size_t)-1;
    orc_cdf(st, n, cum);
    double total = cum[size - 1];
    size_t near = 0;
    for (size_t s = 0; s < nshots; ++s) {
        double target = u[s] * (total - 0.0) + 0.0;
        size_t i = orc_lower_bound(cum, size, target);
        out[s] = i;
        double c_hi = i < size ? cum[i] : total;
        double c_lo = i > 0 ? cum[i - 1] : 0.0;
        double tol = ulps * (nextafter(target, INFINITY) - target);
        if (fabs(c_hi - target) <= tol || fabs(target - c_lo) <= tol) ++near;
    }
    free(cum);
    return near;
}

/* StateVector.cpp:118-156 with the draw injected.  The total is the
 * sequentially rounded sum (the reduction with one OpenMP thread). */
uint64_t orc_measure(double* st, unsigned n, double u)
{
    size_t size = (size_t)1 << n;
    double total = 0.0;
    for (size_t i = 0; i < size; ++i) total += cnorm(AMP(st, i));
    double target = u * (total - 0.0) + 0.0;
    size_t collapsed = 0;
    double running = 0.0;
    for (size_t i = 0; i < size; ++i) {
        running += cnorm(AMP(st, i));
        if (running >= target) { collapsed = i; break; }
    }
    memset(st, 0, size * 2 * sizeof(double));
    st[2 * collapsed] = 1.0;
    return collapsed;
}

/* StateVector.cpp:158-185 with the draw injected: prob1 summed in index order
 * (the reduction with one OpenMP thread), outcome = u < prob1, the other half
 * zeroed and the kept half divided by sqrt(probability of the outcome). */
static double prob_one(const double* st, unsigned n, unsigned q)
{
    size_t size = (size_t)1 << n, bit = (size_t)1 << q;
    double p1 = 0.0;
    for (size_t i = 0; i < size; ++i)
        if (i & bit) p1 += cnorm(AMP(st, i));
    return p1;
}

int orc_measure_qubit(double* st, unsigned n, unsigned q, double u, double* prob1)
{
    size_t size = (size_t)1 << n, bit = (size_t)1 << q;
    double p1 = prob_one(st, n, q);
    int outcome = (u < p1) ? 1 : 0;
    double norm = outcome ? sqrt(p1) : sqrt(1.0 - p1);
    for (size_t i = 0; i < size; ++i) {
        int one = (i & bit) != 0;
        if (one != outcome) {
            st[2 * i] = 0.0;
            st[2 * i + 1] = 0.0;
        } else {
            st[2 * i] /= norm;
            st[2 * i + 1] /= norm;
        }
    }
    if (prob1) *prob1 = p1;
    return outcome;
}

/* StateVector.cpp:187-221: the same draw; the outcome's amplitudes move to the
 * qubit-0 half, renormalised, and the qubit-1 half is zeroed. */
int orc_reset_qubit(double* st, unsigned n, unsigned q, double u, double* prob1)
{
    size_t size = (size_t)1 << n, bit = (size_t)1 << q, lower = bit - 1;
    double p1 = prob_one(st, n, q);
    int outcome = (u < p1) ? 1 : 0;
    double nf = sqrt(outcome ? p1 : 1.0 - p1);
    for (size_t i = 0; i < size / 2; ++i) {
        size_t i0 = ((i & ~lower) << 1) | (i & lower), i1 = i0 | bit;
        if (outcome == 0) {
            st[2 * i0] /= nf;
            st[2 * i0 + 1] /= nf;
        } else {
            st[2 * i0] = st[2 * i1] / nf;
            st[2 * i0 + 1] = st[2 * i1 + 1] / nf;
        }
        st[2 * i1] = 0.0;
        st[2 * i1 + 1] = 0.0;
    }
    if (prob1) *prob1 = p1;
    return outcome;
}

/* ---------------- mt19937 (Matsumoto & Nishimura 1998) ---------------- */
void orc_mt_seed(orc_mt* g, uint32_t seed)
{
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

uint32_t orc_mt_next(orc_mt* g)
{
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* libstdc++ generate_canonical<double, 53>(mt19937): two 32-bit draws,
 * sum = g1 + g2 * 2^32 rounded to double, divided by 2^64, clamped below 1. */
double orc_mt_canonical(orc_mt* g)
{
    double sum = 0.0, tmp = 1.0;
    sum += (double)orc_mt_next(g) * tmp; tmp *= 4294967296.0;
    sum += (double)orc_mt_next(g) * tmp; tmp *= 4294967296.0;
    double r = sum / tmp;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* ---------------- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ---------------- */
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 53-bit uniforms in [0,1) from one Philox block: the product's convention
 * (counter word 2 = 0x4E4F4953 tags the noise stream). */
void orc_philox_uniform_pair(uint64_t seed, uint64_t counter, double* u1, double* u2)
{
    uint32_t ctr[4] = {(uint32_t)counter, (uint32_t)(counter >> 32), 0x4E4F4953u, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    orc_philox4x32_10(ctr, key, w);
    uint64_t a = ((uint64_t)w[1] << 32) | w[0];
    uint64_t b = ((uint64_t)w[3] << 32) | w[2];
    *u1 = (double)(a >> 11) * 0x1.0p-53;
    *u2 = (double)(b >> 11) * 0x1.0p-53;
}

/* ---------------- Noise (Noise.cpp) ---------------- */
void orc_noise_init(orc_noise* nz, unsigned n, const qse_noise_config* cfg)
{
    memset(nz, 0, sizeof(*nz));
    nz->n = n;
    nz->mult = cfg->multiplier;
    nz->mode = cfg->rng_mode;
    nz->seed = cfg->seed;
    memcpy(nz->rates, cfg->rates, sizeof(nz->rates));
    orc_mt_seed(&nz->mt, (uint32_t)cfg->seed);   /* std::mt19937 gen(seed) (Noise.cpp:7) */
}

/* Noise.cpp:21-32.  rates[type] < 0 means `type` is not in errorRates. */
int orc_noise_accumulate(orc_noise* nz, int type, unsigned target, const double* inj)
{
    if (type < 0 || type >= 16 || nz->rates[type] < 0.0) return 0;
    double p = nz->rates[type] * nz->mult;
    double u1, u2;
    if (nz->mode == QSE_RNG_MT19937) {
        u1 = orc_mt_canonical(&nz->mt);
        u2 = orc_mt_canonical(&nz->mt);
    } else if (nz->mode == QSE_RNG_PHILOX) {
        orc_philox_uniform_pair(nz->seed, nz->draws, &u1, &u2);
    } else {
        u1 = inj[0];
        u2 = inj[1];
    }
    nz->draws++;
    if (u1 < p) nz->bit[target]++;
    if (u2 < p) nz->phase[target]++;
    return 2;
}

/* Noise.cpp:34-44 */
void orc_noise_apply(orc_noise* nz, double* st)
{
    for (unsigned q = 0; q < nz->n; ++q) {
        if (nz->bit[q] % 2 != 0) g_x(st, nz->n, q);
        if (nz->phase[q] % 2 != 0) g_z(st, nz->n, q);
    }
}

/* Circuit::execute (Circuit.cpp:64-120): draw before each gate, apply noise after the loop */
int orc_execute(double* st, unsigned n, const qse_op* ops, size_t nops, const double* params,
                orc_noise* nz, const double* inj, size_t ninj)
{
    size_t used = 0;
    for (size_t k = 0; k < nops; ++k) {
        if (nz) {
            if (nz->mode == QSE_RNG_INJECTED && used + 2 > ninj &&
                ops[k].type >= 0 && ops[k].type < 16 && nz->rates[ops[k].type] >= 0.0)
                return -2;
            used += (size_t)orc_noise_accumulate(nz, ops[k].type, ops[k].target, inj ? inj + used : NULL);
        }
        if (orc_apply(st, n, &ops[k], bound_angle(&ops[k], params)) != 0) return -1;
    }
    if (nz) orc_noise_apply(nz, st);
    return 0;
}

/* ---------------- observables and gradients ---------------- */
double orc_obs_value(uint64_t x, const qse_observable* obs)
{
    double v = obs->constant;
    for (size_t t = 0; t < obs->nterms; ++t)
        v += (__builtin_popcountll(x & obs->zmask[t]) & 1) ? -obs->weight[t] : obs->weight[t];
    return v;
}

double orc_expectation(const double* st, unsigned n, const qse_observable* obs)
{
    size_t size = (size_t)1 << n;
    double part[kChunks];
    const size_t len = chunk_len(size);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < kChunks; ++c) {
        double acc = 0.0;
        for (size_t i = (size_t)c * len; i < size && i < (size_t)(c + 1) * len; ++i)
            acc += cnorm(AMP(st, i)) * orc_obs_value(i, obs);
        part[c] = acc;
    }
    return sum_parts(part);
}

/* inverse of one gate (all gate types of the reference are unitary) */
static int apply_inverse(double* st, unsigned n, const qse_op* op, double theta)
{
    qse_op inv = *op;
    switch (op->type) {
    case QSE_GATE_PHASE: case QSE_GATE_RX: case QSE_GATE_RY: case QSE_GATE_RZ:
    case QSE_GATE_CPHASE: case QSE_GATE_MCPHASE:
        return orc_apply(st, n, &inv, -theta);
    case QSE_GATE_2X2:
        /* conjugate transpose */
        inv.m[0] = op->m[0]; inv.m[1] = -op->m[1];
        inv.m[2] = op->m[4]; inv.m[3] = -op->m[5];
        inv.m[4] = op->m[2]; inv.m[5] = -op->m[3];
        inv.m[6] = op->m[6]; inv.m[7] = -op->m[7];
        return orc_apply(st, n, &inv, theta);
    case QSE_GATE_Y: case QSE_GATE_X: case QSE_GATE_Z: case QSE_GATE_H:
    case QSE_GATE_CNOT: case QSE_GATE_SWAP: case QSE_GATE_IDENTITY:
        return orc_apply(st, n, op, theta);
    default: return -1;
    }
}

/* mu = dG/dtheta psi for the parameterised types (a18: derivatives of the
 * a4/a5/a7/a8 matrices) */
static int apply_derivative(double* mu, const double* psi, unsigned n, const qse_op* op, double theta)
{
    size_t size = (size_t)1 << n;
    memset(mu, 0, size * 2 * sizeof(double));
    size_t m = (size_t)1 << op->target;
    double c = cos(theta / 2.0), s = sin(theta / 2.0);
    switch (op->type) {
    case QSE_GATE_RX: case QSE_GATE_RY: {
        cplx d[4];
        if (op->type == QSE_GATE_RX) { d[0] = cmk(-s / 2, 0); d[1] = cmk(0, -c / 2); d[2] = cmk(0, -c / 2); d[3] = cmk(-s / 2, 0); }
        else { d[0] = cmk(-s / 2, 0); d[1] = cmk(-c / 2, 0); d[2] = cmk(c / 2, 0); d[3] = cmk(-s / 2, 0); }
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < size; ++i)
            if (!(i & m)) {
                cplx v0 = AMP(psi, i), v1 = AMP(psi, i | m);
                AMP(mu, i) = cadd(cmul(d[0], v0), cmul(d[1], v1));
                AMP(mu, i | m) = cadd(cmul(d[2], v0), cmul(d[3], v1));
            }
        return 0;
    }
    case QSE_GATE_RZ: {
        cplx d0 = cmul(cmk(0, -0.5), cexpi(-theta / 2)), d1 = cmul(cmk(0, 0.5), cexpi(theta / 2));
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < size; ++i) AMP(mu, i) = cmul(AMP(psi, i), (i & m) ? d1 : d0);
        return 0;
    }
    case QSE_GATE_PHASE: case QSE_GATE_CPHASE: case QSE_GATE_MCPHASE: {
        uint64_t all = (uint64_t)m;
        if (op->type == QSE_GATE_CPHASE) all |= (uint64_t)1 << op->control;
        if (op->type == QSE_GATE_MCPHASE) all |= op->controls;
        cplx d = cmul(cmk(0, 1), cexpi(theta));
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < size; ++i)
            if (((uint64_t)i & all) == all) AMP(mu, i) = cmul(AMP(psi, i), d);
        return 0;
    }
    default: return -1;
    }
}

/* Adjoint differentiation (Jones & Gacon 2020): psi = U|0>, lambda = O psi,
 * reverse sweep psi <- G^dag psi, grad += 2 Re<lambda|dG psi>, lambda <- G^dag lambda. */
double orc_adjoint(unsigned n, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                   const qse_observable* obs, double* grad)
{
    size_t size = (size_t)1 << n;
    double* psi = (double*)malloc(size * 2 * sizeof(double));
    double* lam = (double*)malloc(size * 2 * sizeof(double));
    double* mu = (double*)malloc(size * 2 * sizeof(double));
    for (size_t p = 0; p < nparams; ++p) grad[p] = 0.0;
    orc_init(psi, n);
    orc_run(psi, n, ops, nops, params);
    double part[kChunks];
    const size_t len = chunk_len(size);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < kChunks; ++c) {
        double acc = 0.0;
        for (size_t i = (size_t)c * len; i < size && i < (size_t)(c + 1) * len; ++i) {
            double o = orc_obs_value(i, obs);
            AMP(lam, i) = cscl(o, AMP(psi, i));
            acc += cnorm(AMP(psi, i)) * o;
        }
        part[c] = acc;
    }
    double value = sum_parts(part);
    for (size_t k = nops; k-- > 0;) {
        const qse_op* op = &ops[k];
        double th = bound_angle(op, params);
        apply_inverse(psi, n, op, th);
        if (op->param >= 0 && (size_t)op->param < nparams) {
            apply_derivative(mu, psi, n, op, th);
#pragma omp parallel for schedule(static)
            for (int c = 0; c < kChunks; ++c) {
                double acc = 0.0;
                for (size_t i = (size_t)c * len; i < size && i < (size_t)(c + 1) * len; ++i)
                    acc += AMP(lam, i).re * AMP(mu, i).re + AMP(lam, i).im * AMP(mu, i).im;
                part[c] = acc;
            }
            grad[op->param] += op->coeff * 2.0 * sum_parts(part);
        }
        apply_inverse(lam, n, op, th);
    }
    free(psi); free(lam); free(mu);
    return value;
}

/* Two-term parameter shift (a19): d/dtheta = [f(theta+pi/2) - f(theta-pi/2)]/2,
 * exact for RX/RY/RZ (generator eigenvalues +-1/2) and for phase-type gates
 * (projector generator, eigenvalues 0 and 1).  Two full executes per occurrence. */
double orc_param_shift(unsigned n, const qse_op* ops, size_t nops, const double* params, size_t nparams,
                       const qse_observable* obs, double* grad)
{
    size_t size = (size_t)1 << n;
    double* psi = (double*)malloc(size * 2 * sizeof(double));
    qse_op* work = (qse_op*)malloc(nops * sizeof(qse_op));
    for (size_t p = 0; p < nparams; ++p) grad[p] = 0.0;
    /* bind all angles once: work[k].theta holds the bound angle */
    for (size_t k = 0; k < nops; ++k) { work[k] = ops[k]; work[k].theta = bound_angle(&ops[k], params); work[k].param = -1; }
    orc_init(psi, n);
    orc_run(psi, n, work, nops, NULL);
    double value = orc_expectation(psi, n, obs);
    const double half_pi = 1.5707963267948966192;
    for (size_t k = 0; k < nops; ++k) {
        if (ops[k].param < 0 || (size_t)ops[k].param >= nparams) continue;
        double th = work[k].theta, f[2];
        for (int sgn = 0; sgn < 2; ++sgn) {
            work[k].theta = th + (sgn ? -half_pi : half_pi);
            orc_init(psi, n);
            orc_run(psi, n, work, nops, NULL);
            f[sgn] = orc_expectation(psi, n, obs);
        }
        work[k].theta = th;
        grad[ops[k].param] += ops[k].coeff * (f[0] - f[1]) / 2.0;
    }
    free(psi); free(work);
    return value;
}
