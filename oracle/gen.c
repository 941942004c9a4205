/*
 * gen.c - CPU restatement of the engine's synthetic input generator, for the timed CPU baseline and
 * the reference arm of the benchmark. TEST/BASELINE INFRASTRUCTURE ONLY: it lets the reference's own
 * CPU join (run_sanity_check) be fed the benchmark's inputs without loading the engine library.
 *
 * Rows are computed independently from (seed, row), so the loops are OpenMP-parallel:
 *   R key of row i : 1 + A2 * (A1 * i + B1)^5 + B2 (mod p), p = 2^31 - 1 (x^5 is a bijection of Z_p
 *                    since gcd(5, p - 1) = 1), so the keys are distinct and lie in [1, 2^31);
 *   S rows          : a seeded permutation pi of [0, |S|) by cycle-walking a bijection of [0, 2^b)
 *                    (three odd-multiply / xor-shift rounds); row i matches iff pi(i) < m =
 *                    floor(match_frac * |S|) and then takes the key of R row u(i), u uniform on
 *                    [0, |R|) by multiply-shift range reduction (Lemire 2019) of a SplitMix64 hash;
 *                    a non-match row takes 2^31 + (A3 * (pi(i) - m) + B3 mod p);
 *   values          : the row index.
 * The constants come from SplitMix64 (Steele, Lea, Flood, OOPSLA 2014) of the seed. The test
 * tests/test_oracle.py checks this file row-for-row against the engine's own host generator.
 * Only uniform matches are restated (the Zipf form is not needed by the CPU baseline).
 */
#include "oracle.h"

#include <math.h>

#define P31 0x7fffffffu

static uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27; x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

static uint32_t modp31(uint64_t x) {
    x = (x & P31) + (x >> 31);
    x = (x & P31) + (x >> 31);
    return x >= P31 ? (uint32_t)(x - P31) : (uint32_t)x;
}

typedef struct {
    uint64_t seed;
    int64_t nr, ns, m;
    uint32_t a1, b1, a2, b2, a3, b3;
    int bits, sh;
    uint64_t mul[3], add[3];
} gen_t;

static uint64_t seeded(uint64_t seed, uint64_t c) { return mix64(seed * 0x9e3779b97f4a7c15ull + c); }

static void gen_setup(gen_t* g, uint64_t seed, int64_t nr, int64_t ns, double match_frac) {
    int64_t m = (int64_t)floor(match_frac * (double)ns);
    if (nr <= 0 || m < 0) m = 0;
    if (m > ns) m = ns;
    g->seed = seed;
    g->nr = nr;
    g->ns = ns;
    g->m = m;
    g->a1 = 1u + (uint32_t)(seeded(seed, 1) % (P31 - 1u));
    g->b1 = (uint32_t)(seeded(seed, 2) % P31);
    g->a2 = 1u + (uint32_t)(seeded(seed, 3) % (P31 - 1u));
    g->b2 = (uint32_t)(seeded(seed, 4) % P31);
    g->a3 = 1u + (uint32_t)(seeded(seed, 5) % (P31 - 1u));
    g->b3 = (uint32_t)(seeded(seed, 6) % P31);
    int b = 0;
    while (b < 62 && ((int64_t)1 << b) < ns) ++b;
    g->bits = b;
    g->sh = b / 2 > 0 ? b / 2 : 1;
    for (int i = 0; i < 3; ++i) {
        g->mul[i] = seeded(seed, 7 + (uint64_t)i) | 1ull;
        g->add[i] = seeded(seed, 10 + (uint64_t)i);
    }
}

static uint32_t r_key(const gen_t* g, int64_t i) {
    const uint32_t x = modp31((uint64_t)g->a1 * (uint64_t)i + g->b1);
    const uint32_t x2 = modp31((uint64_t)x * x);
    const uint32_t x4 = modp31((uint64_t)x2 * x2);
    const uint32_t x5 = modp31((uint64_t)x4 * x);
    return modp31((uint64_t)g->a2 * x5 + g->b2) + 1u;
}

/* One round of the bijection of [0, 2^bits) that the S permutation cycle-walks. */
static uint64_t perm_round(const gen_t* g, uint64_t x) {
    const uint64_t mask = ((uint64_t)1 << g->bits) - 1u;
    x = (x * g->mul[0] + g->add[0]) & mask;
    x ^= x >> g->sh;
    x = (x * g->mul[1] + g->add[1]) & mask;
    x ^= x >> g->sh;
    x = (x * g->mul[2] + g->add[2]) & mask;
    return x;
}

static uint32_t s_key(const gen_t* g, int64_t i) {
    uint64_t y = perm_round(g, (uint64_t)i);
    while (y >= (uint64_t)g->ns) y = perm_round(g, y);
    const int64_t pi = (int64_t)y;
    if (pi < g->m) {
        const uint64_t h = mix64(g->seed ^ 0x243f6a8885a308d3ull ^ ((uint64_t)i * 0x9e3779b97f4a7c15ull));
        const uint32_t row = (uint32_t)(((uint64_t)(uint32_t)(h >> 32) * (uint64_t)(uint32_t)g->nr) >> 32);
        return r_key(g, row);
    }
    return 0x80000000u + modp31((uint64_t)g->a3 * (uint64_t)(pi - g->m) + g->b3);
}

int oracle_gen(uint64_t seed, int64_t nr, int64_t ns, double match_frac, uint32_t* rk, uint32_t* rv,
               uint32_t* sk, uint32_t* sv) {
    if (nr < 0 || ns < 0 || nr >= ((int64_t)1 << 32) || ns >= ((int64_t)1 << 32) || !(match_frac >= 0.0) ||
        match_frac > 1.0)
        return -1;
    gen_t g;
    gen_setup(&g, seed, nr, ns, match_frac);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nr; ++i) {
        if (rk) rk[i] = r_key(&g, i);
        if (rv) rv[i] = (uint32_t)i;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ns; ++i) {
        if (sk) sk[i] = s_key(&g, i);
        if (sv) sv[i] = (uint32_t)i;
    }
    return 0;
}
