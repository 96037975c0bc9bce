/*
 * kt_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C restatement of the kettle reference algorithms on the
 * circuit-propagation path, used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  Nothing in the product links
 * or calls this file.  It is pinned against the reference library itself
 * (oracle/_ref, built from the reference sources by oracle/Makefile) and
 * against the known-answer cases of the reference's own tests (tests/golden).
 *
 * Built with -O2 -ffp-contract=off so every product and sum rounds like the
 * reference's plain C++ (no FMA contraction).
 *
 * Citations are to files of the kettle project.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "kettle_b200.h"

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b)
{
    /* std::complex<double> operator* for finite values: (ac - bd, ad + bc) */
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx cadd(cplx a, cplx b)
{
    cplx r = {a.re + b.re, a.im + b.im};
    return r;
}
static inline cplx cconj(cplx a)
{
    cplx r = {a.re, -a.im};
    return r;
}

/* ---------------------------------------------------------------------------
 * Pair enumeration, in the reference's order.
 * SingleQubitGatePairGenerator (simulation/gate_pair_generator.hpp:25-65):
 *   i0 in [0, 2^t), i1 in [0, 2^(n-t-1)), i1 varies fastest;
 *   state0 = i0 + 2*i1*2^t, state1 = state0 + 2^t.
 *   set_state(k): (i0, i1) = (k / 2^(n-t-1), k % 2^(n-t-1))  (common/mathtools.cpp:50-57)
 */
void kto_pairs_single(uint32_t n, uint32_t t, uint64_t k0, uint64_t count, uint64_t* out)
{
    const uint64_t i0_max = (uint64_t)1 << t;
    const uint64_t i1_max = (uint64_t)1 << (n - t - 1);
    uint64_t i0 = k0 / i1_max;
    uint64_t i1 = k0 - i0 * i1_max;
    for (uint64_t k = 0; k < count; ++k) {
        const uint64_t s0 = i0 + 2 * i1 * i0_max;
        out[2 * k] = s0;
        out[2 * k + 1] = s0 + i0_max;
        ++i1;
        if (i1 == i1_max) {
            ++i0;
            i1 = 0;
        }
    }
}

/* DoubleQubitGatePairGenerator (gate_pair_generator.hpp:81-160):
 *   lo = min(c,t), hi = max(c,t); i0 < 2^lo, i1 < 2^(hi-lo-1), i2 < 2^(n-hi-1),
 *   i2 fastest then i1 then i0;  base = i0 + i1*2^(lo+1) + i2*2^(hi+1).
 *   next():               (base + 2^c, base + 2^c + 2^t)
 *   next_unset_and_set(): (base, base + 2^t, base + 2^c, base + 2^c + 2^t)
 *   set_state(k) per flat_index_to_grid_indices_3d (mathtools.cpp:63-75). */
void kto_pairs_double(uint32_t n, uint32_t c, uint32_t t, int32_t quad, uint64_t k0, uint64_t count,
                      uint64_t* out)
{
    const uint32_t lo = c < t ? c : t;
    const uint32_t hi = c < t ? t : c;
    const uint64_t lo_shift = (uint64_t)1 << (lo + 1);
    const uint64_t hi_shift = (uint64_t)1 << (hi + 1);
    const uint64_t c_shift = (uint64_t)1 << c;
    const uint64_t t_shift = (uint64_t)1 << t;
    const uint64_t i1_max = (uint64_t)1 << (hi - lo - 1);
    const uint64_t i2_max = (uint64_t)1 << (n - hi - 1);
    uint64_t i0 = k0 / (i1_max * i2_max);
    uint64_t rem = k0 - i0 * i1_max * i2_max;
    uint64_t i1 = rem / i2_max;
    uint64_t i2 = rem - i1 * i2_max;
    for (uint64_t k = 0; k < count; ++k) {
        const uint64_t base = i0 + i1 * lo_shift + i2 * hi_shift;
        if (quad) {
            out[4 * k] = base;
            out[4 * k + 1] = base + t_shift;
            out[4 * k + 2] = base + c_shift;
            out[4 * k + 3] = base + c_shift + t_shift;
        } else {
            out[2 * k] = base + c_shift;
            out[2 * k + 1] = base + c_shift + t_shift;
        }
        ++i2;
        if (i2 == i2_max) {
            ++i1;
            i2 = 0;
            if (i1 == i1_max) {
                ++i0;
                i1 = 0;
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * Two-amplitude updates (simulation/operations.cpp:13-185), same arithmetic. */
#define SQ12 0.70710678118654752440 /* M_SQRT1_2 */

static void op_pair(int op, cplx* a, cplx* b, double theta, const double* u)
{
    const cplx s0 = *a;
    const cplx s1 = *b;
    switch (op) {
        case KT_OP_H:
        case KT_OP_CH: {
            a->re = SQ12 * (s0.re + s1.re);
            a->im = SQ12 * (s0.im + s1.im);
            b->re = SQ12 * (s0.re - s1.re);
            b->im = SQ12 * (s0.im - s1.im);
            return;
        }
        case KT_OP_X:
        case KT_OP_CX: *a = s1; *b = s0; return;
        case KT_OP_Y:
        case KT_OP_CY: {
            a->re = s1.im;
            a->im = -s1.re;
            b->re = -s0.im;
            b->im = s0.re;
            return;
        }
        case KT_OP_Z:
        case KT_OP_CZ: b->re = -1.0 * s1.re; b->im = -1.0 * s1.im; return;
        case KT_OP_S:
        case KT_OP_CS: b->re = -s1.im; b->im = s1.re; return;
        case KT_OP_SDAG:
        case KT_OP_CSDAG: b->re = s1.im; b->im = -s1.re; return;
        case KT_OP_T:
        case KT_OP_CT: {
            b->re = SQ12 * (s1.re - s1.im);
            b->im = SQ12 * (s1.re + s1.im);
            return;
        }
        case KT_OP_TDAG:
        case KT_OP_CTDAG: {
            b->re = SQ12 * (s1.re + s1.im);
            b->im = -SQ12 * (s1.re - s1.im);
            return;
        }
        case KT_OP_SX:
        case KT_OP_CSX: {
            a->re = 0.5 * (s0.re - s0.im + s1.re + s1.im);
            a->im = 0.5 * (s0.re + s0.im - s1.re + s1.im);
            b->re = 0.5 * (s0.re + s0.im + s1.re - s1.im);
            b->im = 0.5 * (-s0.re + s0.im + s1.re + s1.im);
            return;
        }
        case KT_OP_SXDAG:
        case KT_OP_CSXDAG: {
            a->re = 0.5 * (s0.re + s0.im + s1.re - s1.im);
            a->im = 0.5 * (-s0.re + s0.im + s1.re + s1.im);
            b->re = 0.5 * (s0.re - s0.im + s1.re + s1.im);
            b->im = 0.5 * (s0.re + s0.im - s1.re + s1.im);
            return;
        }
        case KT_OP_RX:
        case KT_OP_CRX: {
            const double c = cos(theta / 2.0), s = sin(theta / 2.0);
            a->re = (s0.re * c) + (s1.im * s);
            a->im = (s0.im * c) - (s1.re * s);
            b->re = (s1.re * c) + (s0.im * s);
            b->im = (s1.im * c) - (s0.re * s);
            return;
        }
        case KT_OP_RY:
        case KT_OP_CRY: {
            const double c = cos(theta / 2.0), s = sin(theta / 2.0);
            a->re = (s0.re * c) - (s1.re * s);
            a->im = (s0.im * c) - (s1.im * s);
            b->re = (s1.re * c) + (s0.re * s);
            b->im = (s1.im * c) + (s0.im * s);
            return;
        }
        case KT_OP_RZ:
        case KT_OP_CRZ: {
            const double c = cos(theta / 2.0), s = sin(theta / 2.0);
            a->re = (s0.re * c) + (s0.im * s);
            a->im = (s0.im * c) - (s0.re * s);
            b->re = (s1.re * c) - (s1.im * s);
            b->im = (s1.im * c) + (s1.re * s);
            return;
        }
        case KT_OP_P:
        case KT_OP_CP: {
            const double c = cos(theta), s = sin(theta);
            b->re = (s1.re * c) - (s1.im * s);
            b->im = (s1.im * c) + (s1.re * s);
            return;
        }
        case KT_OP_U:
        case KT_OP_CU: {
            const cplx m00 = {u[0], u[1]}, m01 = {u[2], u[3]}, m10 = {u[4], u[5]}, m11 = {u[6], u[7]};
            *a = cadd(cmul(s0, m00), cmul(s1, m01));
            *b = cadd(cmul(s0, m10), cmul(s1, m11));
            return;
        }
        default: return;
    }
}

static int is_controlled(int op)
{
    return (op >= KT_OP_CH && op <= KT_OP_CP) || op == KT_OP_CU;
}

static double gate_angle(const kt_gate* g, const double* params)
{
    return (g->param >= 0) ? params[g->param] : g->angle;
}

/* Gate matrices (gates/common_u_gates.cpp:7-178), row-major interleaved. */
void kto_gate_matrix(const kt_gate* g, const double* params, double* m)
{
    const double th = gate_angle(g, params);
    memset(m, 0, 8 * sizeof(double));
    switch (g->op) {
        case KT_OP_H: case KT_OP_CH: m[0] = SQ12; m[2] = SQ12; m[4] = SQ12; m[6] = -SQ12; return;
        case KT_OP_X: case KT_OP_CX: m[2] = 1.0; m[4] = 1.0; return;
        case KT_OP_Y: case KT_OP_CY: m[3] = -1.0; m[5] = 1.0; return;
        case KT_OP_Z: case KT_OP_CZ: m[0] = 1.0; m[6] = -1.0; return;
        case KT_OP_S: case KT_OP_CS: m[0] = 1.0; m[7] = 1.0; return;
        case KT_OP_SDAG: case KT_OP_CSDAG: m[0] = 1.0; m[7] = -1.0; return;
        case KT_OP_T: case KT_OP_CT: m[0] = 1.0; m[6] = SQ12; m[7] = SQ12; return;
        case KT_OP_TDAG: case KT_OP_CTDAG: m[0] = 1.0; m[6] = SQ12; m[7] = -SQ12; return;
        case KT_OP_SX: case KT_OP_CSX: m[0] = 0.5; m[1] = 0.5; m[2] = 0.5; m[3] = -0.5; m[4] = 0.5; m[5] = -0.5; m[6] = 0.5; m[7] = 0.5; return;
        case KT_OP_SXDAG: case KT_OP_CSXDAG: m[0] = 0.5; m[1] = -0.5; m[2] = 0.5; m[3] = 0.5; m[4] = 0.5; m[5] = 0.5; m[6] = 0.5; m[7] = -0.5; return;
        case KT_OP_RX: case KT_OP_CRX: { const double c = cos(th / 2.0), s = sin(th / 2.0); m[0] = c; m[3] = -s; m[5] = -s; m[6] = c; return; }
        case KT_OP_RY: case KT_OP_CRY: { const double c = cos(th / 2.0), s = sin(th / 2.0); m[0] = c; m[2] = -s; m[4] = s; m[6] = c; return; }
        case KT_OP_RZ: case KT_OP_CRZ: { const double c = cos(th / 2.0), s = sin(th / 2.0); m[0] = c; m[1] = -s; m[6] = c; m[7] = s; return; }
        case KT_OP_P: case KT_OP_CP: { m[0] = 1.0; m[6] = cos(th); m[7] = sin(th); return; }
        case KT_OP_U: case KT_OP_CU: memcpy(m, g->u, 8 * sizeof(double)); return;
        default: return;
    }
}

/* ---------------------------------------------------------------------------
 * Statevector simulation: one full sweep per gate, in circuit order
 * (simulation/simulate.cpp:40-262 and :265-415).  M gates are rejected here
 * (kto_measure restates them).  Returns 0, or -1 for a bad record. */
int32_t kto_apply(int32_t n, double* amps, const kt_gate* gates, int64_t n_gates, const double* params)
{
    cplx* st = (cplx*)amps;
    const uint64_t half = (uint64_t)1 << (n - 1);
    const uint64_t quarter = n >= 2 ? ((uint64_t)1 << (n - 2)) : 0;
    uint64_t* pr = (uint64_t*)malloc(2 * sizeof(uint64_t) * 4096);
    if (!pr) return -1;
    for (int64_t gi = 0; gi < n_gates; ++gi) {
        const kt_gate* g = &gates[gi];
        if (g->op > KT_OP_CU || g->target >= (uint32_t)n) { free(pr); return -1; }
        const double th = gate_angle(g, params);
        if (is_controlled(g->op)) {
            if (g->control >= (uint32_t)n || g->control == g->target) { free(pr); return -1; }
            for (uint64_t k0 = 0; k0 < quarter; k0 += 4096) {
                const uint64_t cnt = (quarter - k0) < 4096 ? (quarter - k0) : 4096;
                kto_pairs_double((uint32_t)n, g->control, g->target, 0, k0, cnt, pr);
                for (uint64_t k = 0; k < cnt; ++k) op_pair(g->op, &st[pr[2 * k]], &st[pr[2 * k + 1]], th, g->u);
            }
        } else {
            for (uint64_t k0 = 0; k0 < half; k0 += 4096) {
                const uint64_t cnt = (half - k0) < 4096 ? (half - k0) : 4096;
                kto_pairs_single((uint32_t)n, g->target, k0, cnt, pr);
                for (uint64_t k = 0; k < cnt; ++k) op_pair(g->op, &st[pr[2 * k]], &st[pr[2 * k + 1]], th, g->u);
            }
        }
    }
    free(pr);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Pauli expectation, as expectation_value does it (operator/pauli/pauli_operator.cpp:76-103):
 * copy the state, apply X / Y / Z per non-identity site with the same pair
 * sweeps (simulation/simulate_pauli.cpp:28-87), take inner_product(state, copy)
 * (state/state.cpp:159-172), multiply by the phase (sparse_pauli_string.hpp:32-37). */
static const cplx PHASES[4] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}, {0.0, -1.0}};

int32_t kto_expect(int32_t n, const double* amps, const kt_pauli* strings, int64_t n_strings,
                   const double* coeffs, double* out_terms, double* out_total)
{
    const uint64_t N = (uint64_t)1 << n;
    const cplx* st = (const cplx*)amps;
    cplx* ket = (cplx*)malloc(N * sizeof(cplx));
    uint64_t* pr = (uint64_t*)malloc(2 * sizeof(uint64_t) * 4096);
    if (!ket || !pr) { free(ket); free(pr); return -1; }
    cplx total = {0.0, 0.0};
    for (int64_t k = 0; k < n_strings; ++k) {
        memcpy(ket, st, N * sizeof(cplx));
        for (uint32_t q = 0; q < (uint32_t)n; ++q) {
            const int x = (int)((strings[k].x_mask >> q) & 1U);
            const int z = (int)((strings[k].z_mask >> q) & 1U);
            if (!x && !z) continue;
            const int op = (x && z) ? KT_OP_Y : (x ? KT_OP_X : KT_OP_Z);
            for (uint64_t k0 = 0; k0 < N / 2; k0 += 4096) {
                const uint64_t cnt = (N / 2 - k0) < 4096 ? (N / 2 - k0) : 4096;
                kto_pairs_single((uint32_t)n, q, k0, cnt, pr);
                for (uint64_t p = 0; p < cnt; ++p) op_pair(op, &ket[pr[2 * p]], &ket[pr[2 * p + 1]], 0.0, NULL);
            }
        }
        cplx inner = {0.0, 0.0};
        for (uint64_t i = 0; i < N; ++i) inner = cadd(inner, cmul(cconj(st[i]), ket[i]));
        const cplx phase = PHASES[strings[k].phase & 3];
        const cplx term = cmul(phase, inner);
        if (out_terms) { out_terms[2 * k] = term.re; out_terms[2 * k + 1] = term.im; }
        const cplx c = coeffs ? (cplx){coeffs[2 * k], coeffs[2 * k + 1]} : (cplx){1.0, 0.0};
        total = cadd(total, cmul(cmul(c, phase), inner));
    }
    if (out_total) { out_total[0] = total.re; out_total[1] = total.im; }
    free(ket);
    free(pr);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Probabilities and noise (calculations/probabilities.cpp:49-71, :110-124):
 * p_i = re*re + im*im (std::norm, no contraction), then for each qubit in
 * order the bit-flip mix over that qubit's pairs. */
int32_t kto_probabilities(int32_t n, const double* amps, const double* noise, double* out)
{
    const uint64_t N = (uint64_t)1 << n;
    for (uint64_t i = 0; i < N; ++i) {
        const double re = amps[2 * i], im = amps[2 * i + 1];
        out[i] = re * re + im * im;
    }
    if (noise) {
        uint64_t* pr = (uint64_t*)malloc(2 * sizeof(uint64_t) * 4096);
        if (!pr) return -1;
        for (uint32_t q = 0; q < (uint32_t)n; ++q) {
            const double e = noise[q];
            for (uint64_t k0 = 0; k0 < N / 2; k0 += 4096) {
                const uint64_t cnt = (N / 2 - k0) < 4096 ? (N / 2 - k0) : 4096;
                kto_pairs_single((uint32_t)n, q, k0, cnt, pr);
                for (uint64_t p = 0; p < cnt; ++p) {
                    const double p0 = out[pr[2 * p]], p1 = out[pr[2 * p + 1]];
                    out[pr[2 * p]] = ((1.0 - e) * p0) + (e * p1);
                    out[pr[2 * p + 1]] = ((1.0 - e) * p1) + (e * p0);
                }
            }
        }
        free(pr);
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * MT19937 (Matsumoto & Nishimura 1998; the parameters std::mt19937 fixes) and
 * generate_canonical<double, 53> for a 32-bit engine as libstdc++ implements
 * it: two draws, (g0 + g1 * 2^32) / 2^64, and a result that rounds up to 1.0 is
 * replaced by the largest double below 1. */
typedef struct { uint32_t mt[624]; int idx; } mt19937;

static void mt_seed(mt19937* s, uint32_t seed)
{
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i) s->mt[i] = 1812433253U * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t mt_next(mt19937* s)
{
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (s->mt[i] & 0x80000000U) | (s->mt[(i + 1) % 624] & 0x7fffffffU);
            s->mt[i] = s->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1U) ? 0x9908b0dfU : 0U);
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680U;
    y ^= (y << 15) & 0xefc60000U;
    y ^= y >> 18;
    return y;
}

int32_t kto_canonicals_mt19937(uint32_t seed, int64_t count, double* out)
{
    mt19937 s;
    mt_seed(&s, seed);
    for (int64_t i = 0; i < count; ++i) {
        const double g0 = (double)mt_next(&s);
        const double g1 = (double)mt_next(&s);
        const double r = 4294967296.0;
        double v = (g0 + g1 * r) / (r * r);
        if (v >= 1.0) v = nextafter(1.0, 0.0);
        out[i] = v;
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Sampling (calculations/measurements.cpp:235-311): cdf = sequential partial
 * sum; offset = (last - last strictly smaller cdf value) * 1e-4; a draw is
 * u = canonical * (last - offset) (+ 0.0, the distribution's lower bound) and
 * the outcome is lower_bound(cdf, u). */
int32_t kto_sample_raw(const double* probs, uint64_t N, const double* canonicals, int64_t n_shots, uint64_t* out)
{
    if (N == 0) return -1;
    double* cdf = (double*)malloc(N * sizeof(double));
    if (!cdf) return -1;
    double acc = 0.0;
    for (uint64_t i = 0; i < N; ++i) {
        acc = (i == 0) ? probs[0] : acc + probs[i];
        cdf[i] = acc;
    }
    const double last = cdf[N - 1];
    double second = 0.0;
    for (uint64_t i = N - 1; i > 0; --i) {
        if (cdf[i - 1] < last) { second = cdf[i - 1]; break; }
    }
    const double offset = (last - second) * 1.0e-4;
    const double bound = last - offset;
    for (int64_t s = 0; s < n_shots; ++s) {
        const double u = canonicals[s] * (bound - 0.0) + 0.0;
        uint64_t lo = 0, len = N;
        while (len > 0) {
            const uint64_t half = len / 2;
            if (cdf[lo + half] < u) { lo = lo + half + 1; len = len - half - 1; }
            else { len = half; }
        }
        if (lo >= N) { free(cdf); return -1; }
        out[s] = lo;
    }
    free(cdf);
    return 0;
}

/* the same on a state's 2^n probabilities */
int32_t kto_sample(int32_t n, const double* probs, const double* canonicals, int64_t n_shots, uint64_t* out)
{
    return kto_sample_raw(probs, (uint64_t)1 << n, canonicals, n_shots, out);
}

/* ---------------------------------------------------------------------------
 * M gate (simulation/measure.hpp:34-55, measure.cpp:22-68): P(0), P(1) as
 * sequential sums over the target's pairs; the outcome is what
 * std::discrete_distribution<int>{P0, P1} draws from one canonical c
 * (libstdc++: cumulative {P0/(P0+P1), 1.0}, outcome = lower_bound(c));
 * then the surviving half is scaled by sqrt(1/P(outcome)), the other zeroed. */
int32_t kto_measure(int32_t n, double* amps, uint32_t q, double canonical, int32_t* outcome, double* p0_out,
                    double* p1_out)
{
    cplx* st = (cplx*)amps;
    const uint64_t half = (uint64_t)1 << (n - 1);
    uint64_t* pr = (uint64_t*)malloc(2 * sizeof(uint64_t) * 4096);
    if (!pr) return -1;
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t k0 = 0; k0 < half; k0 += 4096) {
        const uint64_t cnt = (half - k0) < 4096 ? (half - k0) : 4096;
        kto_pairs_single((uint32_t)n, q, k0, cnt, pr);
        for (uint64_t k = 0; k < cnt; ++k) {
            const cplx a = st[pr[2 * k]], b = st[pr[2 * k + 1]];
            p0 += a.re * a.re + a.im * a.im;
            p1 += b.re * b.re + b.im * b.im;
        }
    }
    const double sum = p0 + p1;
    const double cp0 = p0 / sum;
    const int32_t res = (canonical <= cp0) ? 0 : 1;
    const double scale = sqrt(1.0 / (res == 0 ? p0 : p1));
    for (uint64_t k0 = 0; k0 < half; k0 += 4096) {
        const uint64_t cnt = (half - k0) < 4096 ? (half - k0) : 4096;
        kto_pairs_single((uint32_t)n, q, k0, cnt, pr);
        for (uint64_t k = 0; k < cnt; ++k) {
            cplx* a = &st[pr[2 * k]];
            cplx* b = &st[pr[2 * k + 1]];
            if (res == 0) { a->re *= scale; a->im *= scale; b->re = 0.0; b->im = 0.0; }
            else { a->re = 0.0; a->im = 0.0; b->re *= scale; b->im *= scale; }
        }
    }
    free(pr);
    if (outcome) *outcome = res;
    if (p0_out) *p0_out = p0;
    if (p1_out) *p1_out = p1;
    return 0;
}

/* ---------------------------------------------------------------------------
 * Density matrix: rho <- U rho U^dagger as two passes through a buffer
 * (simulation/simulate_density_matrix.cpp:42-180; operations_density_matrix.cpp:18-176):
 *   pass 1, buffer = U rho over row pairs (r0, r1) for every column;
 *   pass 2, rho = buffer U^dagger over column pairs (c0, c1) for every row.
 * Controlled gates act on the (control = 1) rows in pass 1 and columns in pass 2.
 * rho is column-major: (r, c) at r + c*N. */
int32_t kto_simulate_dm(int32_t n, double* rho_d, const kt_gate* gates, int64_t n_gates, const double* params)
{
    const uint64_t N = (uint64_t)1 << n;
    cplx* rho = (cplx*)rho_d;
    cplx* buf = (cplx*)malloc(N * N * sizeof(cplx));
    if (!buf) return -1;
    for (int64_t gi = 0; gi < n_gates; ++gi) {
        const kt_gate* g = &gates[gi];
        if (g->op > KT_OP_CU || g->target >= (uint32_t)n) { free(buf); return -1; }
        double m[8];
        kto_gate_matrix(g, params, m);
        const cplx u00 = {m[0], m[1]}, u01 = {m[2], m[3]}, u10 = {m[4], m[5]}, u11 = {m[6], m[7]};
        const cplx a00 = cconj(u00), a01 = cconj(u10), a10 = cconj(u01), a11 = cconj(u11); /* U^dagger */
        const uint64_t tb = (uint64_t)1 << g->target;
        const int ctl = is_controlled(g->op);
        const uint64_t cb = ctl ? ((uint64_t)1 << g->control) : 0;
        memcpy(buf, rho, N * N * sizeof(cplx));
        /* pass 1: buffer = U rho (acts on row index) */
        for (uint64_t c = 0; c < N; ++c) {
            for (uint64_t r0 = 0; r0 < N; ++r0) {
                if (r0 & tb) continue;
                if (ctl && !(r0 & cb)) continue;
                const uint64_t r1 = r0 | tb;
                const cplx x0 = rho[r0 + c * N], x1 = rho[r1 + c * N];
                buf[r0 + c * N] = cadd(cmul(x0, u00), cmul(x1, u01));
                buf[r1 + c * N] = cadd(cmul(x0, u10), cmul(x1, u11));
            }
        }
        memcpy(rho, buf, N * N * sizeof(cplx));
        /* pass 2: rho = buffer U^dagger (acts on column index) */
        for (uint64_t c0 = 0; c0 < N; ++c0) {
            if (c0 & tb) continue;
            if (ctl && !(c0 & cb)) continue;
            const uint64_t c1 = c0 | tb;
            for (uint64_t r = 0; r < N; ++r) {
                const cplx b0 = buf[r + c0 * N], b1 = buf[r + c1 * N];
                rho[r + c0 * N] = cadd(cmul(b0, a00), cmul(b1, a10));
                rho[r + c1 * N] = cadd(cmul(b0, a01), cmul(b1, a11));
            }
        }
    }
    free(buf);
    return 0;
}

/* Tr(P rho) for each string (new capability, pinned through the pure-state
 * identity Tr(P |psi><psi|) = <psi|P|psi>): sum_r <r|P|r^x> rho[r^x, r]. */
int32_t kto_dm_expect(int32_t n, const double* rho_d, const kt_pauli* strings, int64_t n_strings,
                      const double* coeffs, double* out_terms, double* out_total)
{
    const uint64_t N = (uint64_t)1 << n;
    const cplx* rho = (const cplx*)rho_d;
    cplx total = {0.0, 0.0};
    for (int64_t k = 0; k < n_strings; ++k) {
        const uint64_t x = strings[k].x_mask, z = strings[k].z_mask;
        const int ny = __builtin_popcountll(x & z);
        cplx acc = {0.0, 0.0};
        for (uint64_t j = 0; j < N; ++j) {
            /* P|j> = i^ny (-1)^{popcount(j & z)} |j ^ x>, so <j^x|P|j> is that factor */
            const uint64_t r = j ^ x;
            cplx f = PHASES[ny & 3];
            if (__builtin_popcountll(j & z) & 1) { f.re = -f.re; f.im = -f.im; }
            /* Tr(P rho) = sum_j <r|P|j> rho[j, r] with r = j ^ x */
            acc = cadd(acc, cmul(f, rho[j + r * N]));
        }
        const cplx phase = PHASES[strings[k].phase & 3];
        const cplx term = cmul(phase, acc);
        if (out_terms) { out_terms[2 * k] = term.re; out_terms[2 * k + 1] = term.im; }
        const cplx c = coeffs ? (cplx){coeffs[2 * k], coeffs[2 * k + 1]} : (cplx){1.0, 0.0};
        total = cadd(total, cmul(c, term));
    }
    if (out_total) { out_total[0] = total.re; out_total[1] = total.im; }
    return 0;
}

/*
 * Partial trace, restated from state/density_matrix.cpp:231-278: the indices
 * are sorted high to low and traced one at a time; tracing (current-matrix)
 * qubit q keeps, for every reduced row r' and column c' (column-major), the
 * sum current(r, c) + current(r + 2^q, c + 2^q) with r, c = r', c' with a 0
 * inserted at bit q (PartialTraceIndexGenerator_ order: blocks of 2^(q+1),
 * steps of 1 inside the low half).  `qubits` holds k indices, each < n
 * (duplicates allowed: each is an index into the matrix left by the traces
 * before it, as the reference reads them).  rho_out has 4^(n-k) entries.
 */
static int cmp_desc_size(const void* a, const void* b)
{
    const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x < y) - (x > y);
}

int32_t kto_dm_partial_trace(int32_t n, const double* rho_d, const int64_t* qubits, int32_t k, double* out_d)
{
    if (n < 0 || k < 0 || k > n) {
        return KT_ERR_INVALID;
    }
    int64_t* q = (int64_t*)malloc(sizeof(int64_t) * (size_t)(k > 0 ? k : 1));
    for (int32_t i = 0; i < k; ++i) {
        if (qubits[i] < 0 || qubits[i] >= n) {
            free(q);
            return KT_ERR_INVALID;
        }
        q[i] = qubits[i];
    }
    qsort(q, (size_t)k, sizeof(int64_t), cmp_desc_size);
    uint64_t N = (uint64_t)1 << n;
    cplx* cur = (cplx*)malloc(sizeof(cplx) * N * N);
    memcpy(cur, rho_d, sizeof(cplx) * N * N);
    for (int32_t i = 0; i < k; ++i) {
        const int64_t n_cur = n - i;
        if (q[i] >= n_cur) {
            free(cur);
            free(q);
            return KT_ERR_INVALID;
        }
        const uint64_t step = (uint64_t)1 << q[i];
        const uint64_t Nc = (uint64_t)1 << n_cur;
        const uint64_t Nr = Nc >> 1;
        cplx* red = (cplx*)malloc(sizeof(cplx) * (Nr > 0 ? Nr * Nr : 1));
        for (uint64_t ic = 0; ic < Nr; ++ic) {
            const uint64_t c = ((ic / step) * 2 * step) + (ic % step);
            for (uint64_t ir = 0; ir < Nr; ++ir) {
                const uint64_t r = ((ir / step) * 2 * step) + (ir % step);
                red[ir + ic * Nr] = cadd(cur[r + c * Nc], cur[(r + step) + (c + step) * Nc]);
            }
        }
        free(cur);
        cur = red;
        N = Nr;
    }
    memcpy(out_d, cur, sizeof(cplx) * N * N);
    free(cur);
    free(q);
    return KT_OK;
}

/* state/density_matrix.cpp:187-214: result(rR * A + rL, cR * A + cL) = L(rL, cL) R(rR, cR) */
int32_t kto_dm_tensor_product(int32_t nl, const double* left_d, int32_t nr, const double* right_d, double* out_d)
{
    const uint64_t A = (uint64_t)1 << nl, B = (uint64_t)1 << nr, D = A * B;
    const cplx* L = (const cplx*)left_d;
    const cplx* R = (const cplx*)right_d;
    cplx* out = (cplx*)out_d;
    for (uint64_t cl = 0; cl < A; ++cl) {
        for (uint64_t rl = 0; rl < A; ++rl) {
            const cplx lv = L[rl + cl * A];
            for (uint64_t cr = 0; cr < B; ++cr) {
                for (uint64_t rr = 0; rr < B; ++rr) {
                    out[(rr * A + rl) + (cr * A + cl) * D] = cmul(lv, R[rr + cr * B]);
                }
            }
        }
    }
    return KT_OK;
}

/* Tr(rho^2) = sum_i sum_j rho(i, j) rho(j, i), row by row */
int32_t kto_dm_trace_of_square(int32_t n, const double* rho_d, double* out)
{
    const uint64_t N = (uint64_t)1 << n;
    const cplx* rho = (const cplx*)rho_d;
    cplx s = {0.0, 0.0};
    for (uint64_t i = 0; i < N; ++i) {
        for (uint64_t j = 0; j < N; ++j) {
            s = cadd(s, cmul(rho[i + j * N], rho[j + i * N]));
        }
    }
    out[0] = s.re;
    out[1] = s.im;
    return KT_OK;
}
