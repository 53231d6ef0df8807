/*
 * lqcs_oracle.c — ORACLE (test infrastructure only; never part of the product path).
 *
 * A scalar CPU restatement of the reference's statevector kernels, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.  Each function
 * cites the reference function it restates (paths relative to the reference project).
 * Arithmetic follows the reference's std::complex<double> evaluation on x86-64 without
 * FMA: every product and sum is rounded separately (this file is compiled with
 * -ffp-contract=off), and |z|^2 is re*re + im*im as libstdc++'s std::norm computes it.
 *
 * State layout: 2^n complex128, interleaved (re, im), qubit 0 = least significant bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cx;

static inline cx cx_mul(cx a, cx b) {
    cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cx cx_add(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static inline double cx_norm(cx a) { return a.re * a.re + a.im * a.im; }

/* include/lqcs/core/bit_utils.hpp:9-12 */
static inline uint64_t insert_zero_bit(uint64_t v, unsigned pos) {
    const uint64_t low = (pos >= 64) ? ~0ull : ((1ull << pos) - 1);
    return ((v & ~low) << 1) | (v & low);
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return (x > y) - (x < y);
}

/* src/backend/kernels/gate_kernels.cpp:26-39 — a' = M a on every (i0, i1) pair. */
void orc_apply_single_qubit(double* s, uint64_t n_amps, uint32_t t, const double* m8) {
    cx* st = (cx*)s;
    const cx m0 = {m8[0], m8[1]}, m1 = {m8[2], m8[3]}, m2 = {m8[4], m8[5]}, m3 = {m8[6], m8[7]};
    for (uint64_t g = 0; g < n_amps / 2; ++g) {
        const uint64_t i0 = insert_zero_bit(g, t), i1 = i0 | (1ull << t);
        const cx a0 = st[i0], a1 = st[i1];
        st[i0] = cx_add(cx_mul(m0, a0), cx_mul(m1, a1));
        st[i1] = cx_add(cx_mul(m2, a0), cx_mul(m3, a1));
    }
}

/* src/backend/kernels/gate_kernels.cpp:41-47 — multiply by d0 or d1 by bit t. */
void orc_apply_diagonal(double* s, uint64_t n_amps, uint32_t t, const double* d4) {
    cx* st = (cx*)s;
    const cx d0 = {d4[0], d4[1]}, d1 = {d4[2], d4[3]};
    for (uint64_t i = 0; i < n_amps; ++i) st[i] = cx_mul(st[i], ((i >> t) & 1) ? d1 : d0);
}

/* src/backend/kernels/gate_kernels.cpp:49-69 — 2x2 on the control=1 subspace. */
void orc_apply_controlled_single(double* s, uint64_t n_amps, uint32_t c, uint32_t t,
                                 const double* m8) {
    cx* st = (cx*)s;
    const cx m0 = {m8[0], m8[1]}, m1 = {m8[2], m8[3]}, m2 = {m8[4], m8[5]}, m3 = {m8[6], m8[7]};
    const unsigned lo = c < t ? c : t, hi = c < t ? t : c;
    for (uint64_t g = 0; g < n_amps / 4; ++g) {
        const uint64_t base = insert_zero_bit(insert_zero_bit(g, lo), hi);
        const uint64_t i0 = base | (1ull << c), i1 = i0 | (1ull << t);
        const cx a0 = st[i0], a1 = st[i1];
        st[i0] = cx_add(cx_mul(m0, a0), cx_mul(m1, a1));
        st[i1] = cx_add(cx_mul(m2, a0), cx_mul(m3, a1));
    }
}

/* src/backend/kernels/gate_kernels.cpp:71-84 — swap |a=1,b=0> and |a=0,b=1>. */
void orc_apply_swap(double* s, uint64_t n_amps, uint32_t a, uint32_t b) {
    cx* st = (cx*)s;
    const unsigned lo = a < b ? a : b, hi = a < b ? b : a;
    for (uint64_t g = 0; g < n_amps / 4; ++g) {
        const uint64_t base = insert_zero_bit(insert_zero_bit(g, lo), hi);
        const cx tmp = st[base | (1ull << a)];
        st[base | (1ull << a)] = st[base | (1ull << b)];
        st[base | (1ull << b)] = tmp;
    }
}

/* src/backend/kernels/gate_kernels.cpp:86-106 — 4x4 on quads (local bit 0 <-> q0). */
void orc_apply_two_qubit(double* s, uint64_t n_amps, uint32_t q0, uint32_t q1,
                         const double* m32) {
    cx* st = (cx*)s;
    const unsigned lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
    for (uint64_t g = 0; g < n_amps / 4; ++g) {
        const uint64_t base = insert_zero_bit(insert_zero_bit(g, lo), hi);
        const uint64_t idx[4] = {base, base | (1ull << q0), base | (1ull << q1),
                                 base | (1ull << q0) | (1ull << q1)};
        cx a[4];
        for (int r = 0; r < 4; ++r) a[r] = st[idx[r]];
        for (int r = 0; r < 4; ++r) {
            cx acc = cx_mul((cx){m32[2 * (r * 4)], m32[2 * (r * 4) + 1]}, a[0]);
            for (int c = 1; c < 4; ++c)
                acc = cx_add(acc, cx_mul((cx){m32[2 * (r * 4 + c)], m32[2 * (r * 4 + c) + 1]}, a[c]));
            st[idx[r]] = acc;
        }
    }
}

/* Fixed-bit layout shared by the controlled-unitary and controlled-permutation loops:
 * src/backend/kernels/gate_kernels.cpp:111-141 (make_layout). */
typedef struct {
    uint32_t fixed[64];
    uint32_t n_fixed;
    uint64_t c_mask;
    uint64_t* offset;
    uint64_t n_groups;
} layout_t;

static void make_layout(layout_t* lay, uint64_t n_amps, const uint32_t* controls, uint32_t nc,
                        const uint32_t* targets, uint32_t k) {
    lay->n_fixed = nc + k;
    for (uint32_t i = 0; i < nc; ++i) lay->fixed[i] = controls[i];
    for (uint32_t i = 0; i < k; ++i) lay->fixed[nc + i] = targets[i];
    qsort(lay->fixed, lay->n_fixed, sizeof(uint32_t), cmp_u32);
    lay->c_mask = 0;
    for (uint32_t i = 0; i < nc; ++i) lay->c_mask |= 1ull << controls[i];
    const uint64_t dim = 1ull << k;
    lay->offset = (uint64_t*)calloc(dim, sizeof(uint64_t));
    for (uint64_t l = 0; l < dim; ++l)
        for (uint32_t j = 0; j < k; ++j)
            if ((l >> j) & 1) lay->offset[l] |= 1ull << targets[j];
    lay->n_groups = n_amps >> lay->n_fixed;
}

static inline uint64_t expand(uint64_t g, const layout_t* lay) {
    for (uint32_t i = 0; i < lay->n_fixed; ++i) g = insert_zero_bit(g, lay->fixed[i]);
    return g;
}

/* src/backend/kernels/gate_kernels.cpp:143-167 — dense 2^k block on the controls=1
 * subspace; sum starts at 0 and accumulates m[r][c]*a[c] in column order. */
void orc_apply_controlled_unitary(double* s, uint64_t n_amps, const uint32_t* controls,
                                  uint32_t nc, const uint32_t* targets, uint32_t k,
                                  const double* m) {
    cx* st = (cx*)s;
    layout_t lay;
    make_layout(&lay, n_amps, controls, nc, targets, k);
    const uint64_t dim = 1ull << k;
    cx* a = (cx*)malloc(dim * sizeof(cx));
    uint64_t* idx = (uint64_t*)malloc(dim * sizeof(uint64_t));
    for (uint64_t g = 0; g < lay.n_groups; ++g) {
        const uint64_t base = expand(g, &lay) | lay.c_mask;
        for (uint64_t l = 0; l < dim; ++l) { idx[l] = base | lay.offset[l]; a[l] = st[idx[l]]; }
        for (uint64_t r = 0; r < dim; ++r) {
            cx sum = {0.0, 0.0};
            for (uint64_t c = 0; c < dim; ++c) {
                const cx mm = {m[2 * (r * dim + c)], m[2 * (r * dim + c) + 1]};
                sum = cx_add(sum, cx_mul(mm, a[c]));
            }
            st[idx[r]] = sum;
        }
    }
    free(a); free(idx); free(lay.offset);
}

/* src/backend/kernels/gate_kernels.cpp:169-189 — |l> -> |perm[l]> on controls=1. */
void orc_apply_controlled_permutation(double* s, uint64_t n_amps, const uint32_t* controls,
                                      uint32_t nc, const uint32_t* targets, uint32_t k,
                                      const uint64_t* perm) {
    cx* st = (cx*)s;
    layout_t lay;
    make_layout(&lay, n_amps, controls, nc, targets, k);
    const uint64_t dim = 1ull << k;
    cx* a = (cx*)malloc(dim * sizeof(cx));
    for (uint64_t g = 0; g < lay.n_groups; ++g) {
        const uint64_t base = expand(g, &lay) | lay.c_mask;
        for (uint64_t l = 0; l < dim; ++l) a[l] = st[base | lay.offset[l]];
        for (uint64_t l = 0; l < dim; ++l) st[base | lay.offset[perm[l]]] = a[l];
    }
    free(a); free(lay.offset);
}

/* src/backend/kernels/gate_kernels.cpp:191-225 — exp(-i theta/2 P) from global masks.
 * cos/sin of theta/2 are passed in (c, s) so the caller controls libm. */
void orc_apply_pauli_rotation(double* s, uint64_t n_amps, uint64_t x, uint64_t zy,
                              uint32_t n_y, double cos_h, double sin_h) {
    cx* st = (cx*)s;
    const cx c = {cos_h, 0.0};
    const cx mis = {0.0, -sin_h};
    static const cx ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    const cx yphase = cx_mul(mis, ipow[n_y % 4]);
    if (x == 0) {
        for (uint64_t i = 0; i < n_amps; ++i) {
            const double sign = (__builtin_popcountll(i & zy) % 2 == 0) ? 1.0 : -1.0;
            const cx ys = {yphase.re * sign, yphase.im * sign};
            st[i] = cx_mul(st[i], cx_add(c, ys));
        }
        return;
    }
    const uint64_t lsb = x & (~x + 1);
    for (uint64_t i = 0; i < n_amps; ++i) {
        if (i & lsb) continue;
        const uint64_t j = i ^ x;
        const double si = (__builtin_popcountll(i & zy) % 2 == 0) ? 1.0 : -1.0;
        const double sj = (__builtin_popcountll(j & zy) % 2 == 0) ? 1.0 : -1.0;
        const cx ai = st[i], aj = st[j];
        const cx ysj = {yphase.re * sj, yphase.im * sj};
        const cx ysi = {yphase.re * si, yphase.im * si};
        st[i] = cx_add(cx_mul(c, ai), cx_mul(ysj, aj));
        st[j] = cx_add(cx_mul(ysi, ai), cx_mul(c, aj));
    }
}

/* src/backend/kernels/gate_kernels.cpp:227-247 — returns the outcome. */
int orc_collapse_qubit(double* s, uint64_t n_amps, uint32_t q, double u) {
    cx* st = (cx*)s;
    double p1 = 0.0;
    for (uint64_t i = 0; i < n_amps; ++i)
        if ((i >> q) & 1) p1 += cx_norm(st[i]);
    const int outcome = u < p1;
    const double keep = outcome ? p1 : 1.0 - p1;
    const double scale = 1.0 / sqrt(keep);
    for (uint64_t i = 0; i < n_amps; ++i) {
        if ((int)((i >> q) & 1) == outcome) { st[i].re *= scale; st[i].im *= scale; }
        else { st[i].re = 0.0; st[i].im = 0.0; }
    }
    return outcome;
}

/* src/backend/kernels/gate_kernels.cpp:249-260 */
void orc_reset_qubit(double* s, uint64_t n_amps, uint32_t q, double u) {
    cx* st = (cx*)s;
    if (!orc_collapse_qubit(s, n_amps, q, u)) return;
    const uint64_t mask = 1ull << q;
    for (uint64_t g = 0; g < n_amps / 2; ++g) {
        const uint64_t i0 = insert_zero_bit(g, q);
        st[i0] = st[i0 | mask];
        st[i0 | mask].re = 0.0; st[i0 | mask].im = 0.0;
    }
}

/* src/backend/kernels/gate_kernels.cpp:262-277 */
double orc_kraus_probability(const double* s, uint64_t n_amps, uint32_t t, const double* k8) {
    const cx* st = (const cx*)s;
    const cx k0 = {k8[0], k8[1]}, k1 = {k8[2], k8[3]}, k2 = {k8[4], k8[5]}, k3 = {k8[6], k8[7]};
    double p = 0.0;
    for (uint64_t g = 0; g < n_amps / 2; ++g) {
        const uint64_t i0 = insert_zero_bit(g, t), i1 = i0 | (1ull << t);
        const cx a0 = st[i0], a1 = st[i1];
        p += cx_norm(cx_add(cx_mul(k0, a0), cx_mul(k1, a1))) +
             cx_norm(cx_add(cx_mul(k2, a0), cx_mul(k3, a1)));
    }
    return p;
}

/* src/backend/statevector.cpp:39-78 — masks already mapped to global bits. */
double orc_expectation(const double* s, uint64_t n_amps, uint64_t x, uint64_t zy, uint32_t n_y) {
    const cx* st = (const cx*)s;
    double re = 0.0, im = 0.0;
    for (uint64_t i = 0; i < n_amps; ++i) {
        const double sign = (__builtin_popcountll(i & zy) % 2 == 0) ? 1.0 : -1.0;
        const cx a = st[i], b = st[i ^ x];
        const cx sa = {sign * a.re, sign * a.im};
        const cx t = cx_mul(sa, (cx){b.re, -b.im});
        re += t.re; im += t.im;
    }
    static const cx ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    return cx_mul(ipow[n_y % 4], (cx){re, im}).re;
}

/* src/backend/statevector.cpp:33-37 followed by std::partial_sum
 * (src/backend/statevector_simulator.cpp:98-100): sequential inclusive prefix sum. */
void orc_cumulative(const double* s, uint64_t n_amps, double* cum) {
    const cx* st = (const cx*)s;
    double acc = 0.0;
    for (uint64_t i = 0; i < n_amps; ++i) {
        acc = (i == 0) ? cx_norm(st[0]) : acc + cx_norm(st[i]);
        cum[i] = acc;
    }
}

/* std::upper_bound over cum (src/backend/statevector_simulator.cpp:105-109). */
uint64_t orc_upper_bound(const double* cum, uint64_t n, double r) {
    uint64_t lo = 0, len = n;
    while (len > 0) {
        const uint64_t half = len / 2;
        if (!(r < cum[lo + half])) { lo = lo + half + 1; len = len - half - 1; }
        else len = half;
    }
    return lo;
}

double orc_norm(const double* s, uint64_t n_amps) {
    const cx* st = (const cx*)s;
    double sum = 0.0;
    for (uint64_t i = 0; i < n_amps; ++i) sum += cx_norm(st[i]);
    return sqrt(sum);
}

/* ------------------------------------------------------------------ mt19937_64
 * The 64-bit Mersenne Twister (Nishimura 2000; the parameters std::mt19937_64 is
 * specified with: w=64 n=312 m=156 r=31 a=0xB5026F5AA96619E9 u=29 d=0x5555555555555555
 * s=17 b=0x71D67FFFEDA60000 t=37 c=0xFFF7EEE000000000 l=43 f=6364136223846793005),
 * restated so the oracle can draw the reference's uniforms (include/lqcs/core/random.hpp:
 * uniform_real_distribution<double>(0,1) over mt19937_64, which libstdc++ evaluates as one
 * 64-bit draw converted to double and divided by 2^64, clamped below 1). */
typedef struct { uint64_t mt[312]; int idx; } orc_mt64;

void orc_mt64_seed(orc_mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ull * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = 312;
}

uint64_t orc_mt64_next(orc_mt64* g) {
    const uint64_t upper = 0xFFFFFFFF80000000ull, lower = 0x7FFFFFFFull;
    if (g->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t y = (g->mt[i] & upper) | (g->mt[(i + 1) % 312] & lower);
            uint64_t v = g->mt[(i + 156) % 312] ^ (y >> 1);
            if (y & 1) v ^= 0xB5026F5AA96619E9ull;
            g->mt[i] = v;
        }
        g->idx = 0;
    }
    uint64_t z = g->mt[g->idx++];
    z ^= (z >> 29) & 0x5555555555555555ull;
    z ^= (z << 17) & 0x71D67FFFEDA60000ull;
    z ^= (z << 37) & 0xFFF7EEE000000000ull;
    z ^= z >> 43;
    return z;
}

double orc_mt64_uniform(orc_mt64* g) {
    const double r = (double)orc_mt64_next(g) / 18446744073709551616.0;
    return r >= 1.0 ? nextafter(1.0, 0.0) : r;
}

size_t orc_mt64_sizeof(void) { return sizeof(orc_mt64); }

void orc_mt64_uniforms(orc_mt64* g, uint64_t n, double* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = orc_mt64_uniform(g);
}
