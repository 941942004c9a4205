// brig_gen.cuh - deterministic synthetic join inputs, identical on host and device.
//
// The reference generator (datagen/gen_dataset.cpp:79-263) writes R = shuffled [0, k) u [k, R)
// and S = shuffled [0, k) u [R, R+S-k) with std::mt19937_64 Fisher-Yates shuffles. That is
// sequential; this generator computes every row independently from (seed, row) so the device can
// produce 640M-row inputs in milliseconds and the host can reproduce any row:
//   R key of row i : 1 + F(i), F a seeded bijection of Z_p, p = 2^31 - 1 (affine map, x -> x^5,
//                    affine map; x^5 is a bijection because gcd(5, p-1) = 1). Keys are distinct and
//                    lie in [1, 2^31).
//   S rows          : a seeded permutation pi of [0, |S|) (cycle-walking over a bijection of
//                    [0, 2^b)); row i is a match row iff pi(i) < m = floor(match_frac * |S|).
//                    A match row takes the key of R row u(i), u uniform on [0, |R|) (or Zipf(s)
//                    ranked by R row order); a non-match row takes 2^31 + G(pi(i) - m), G another
//                    bijection of Z_p, so non-match keys are distinct and lie in [2^31, 2^32 - 1).
//   values          : the row index.
#pragma once

#include <cmath>
#include <cstdint>
#include "brig_common.cuh"

namespace brig {

constexpr uint32_t kP31 = 0x7fffffffu;  // 2^31 - 1, a Mersenne prime

BRIG_HD uint32_t modp31(uint64_t x) {
    x = (x & kP31) + (x >> 31);
    x = (x & kP31) + (x >> 31);
    return x >= kP31 ? (uint32_t)(x - kP31) : (uint32_t)x;
}

struct GenParams {
    uint64_t seed;
    int64_t nr, ns, m;
    uint32_t A1, B1, A2, B2, A3, B3;
    int32_t sbits, sh;
    uint64_t sm1, sm2, sm3, sc1, sc2, sc3;
    // Zipf rejection-inversion constants (Hoermann & Derflinger, "Rejection-inversion to generate
    // variates from monotone discrete distributions", ACM TOMACS 1996).
    double zs, hX1, hN, sVal;
};

BRIG_HD double zipf_helper1(double x) {  // expm1(x)/x, -> 1 as x -> 0
    return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
}
BRIG_HD double zipf_helper2(double x) {  // log1p(x)/x, -> 1 as x -> 0
    return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
}
// H(x) = integral_1^x t^-s dt ; h(x) = x^-s ; Hinv the inverse of H.
BRIG_HD double zipf_H(double x, double s) {
    const double lx = log(x);
    return zipf_helper1((1.0 - s) * lx) * lx;
}
BRIG_HD double zipf_h(double x, double s) { return exp(-s * log(x)); }
BRIG_HD double zipf_Hinv(double y, double s) {
    double t = y * (1.0 - s);
    if (t < -1.0) t = -1.0;  // guard rounding below the domain
    return exp(zipf_helper2(t) * y);
}

inline GenParams make_gen_params(uint64_t seed, int64_t nr, int64_t ns, double match_frac, double zipf_s) {
    GenParams g{};
    g.seed = seed;
    g.nr = nr;
    g.ns = ns;
    int64_t m = (int64_t)std::floor(match_frac * (double)ns);
    if (nr <= 0) m = 0;
    if (m < 0) m = 0;
    if (m > ns) m = ns;
    g.m = m;
    auto r = [&](uint64_t c) { return mix64(seed * 0x9e3779b97f4a7c15ull + c); };
    g.A1 = 1 + (uint32_t)(r(1) % (kP31 - 1));
    g.B1 = (uint32_t)(r(2) % kP31);
    g.A2 = 1 + (uint32_t)(r(3) % (kP31 - 1));
    g.B2 = (uint32_t)(r(4) % kP31);
    g.A3 = 1 + (uint32_t)(r(5) % (kP31 - 1));
    g.B3 = (uint32_t)(r(6) % kP31);
    int bits = 0;
    while (bits < 62 && ((int64_t)1 << bits) < ns) ++bits;
    g.sbits = bits;
    g.sh = bits / 2 > 0 ? bits / 2 : 1;
    g.sm1 = r(7) | 1ull; g.sm2 = r(8) | 1ull; g.sm3 = r(9) | 1ull;
    g.sc1 = r(10); g.sc2 = r(11); g.sc3 = r(12);
    g.zs = zipf_s;
    if (zipf_s > 0.0 && nr > 0) {
        g.hX1 = zipf_H(1.5, zipf_s) - 1.0;
        g.hN = zipf_H((double)nr + 0.5, zipf_s);
        g.sVal = 2.0 - zipf_Hinv(zipf_H(2.5, zipf_s) - zipf_h(2.0, zipf_s), zipf_s);
    }
    return g;
}

BRIG_HD uint32_t gen_r_key(const GenParams& g, int64_t i) {
    const uint32_t x = modp31((uint64_t)g.A1 * (uint64_t)i + g.B1);
    const uint32_t x2 = modp31((uint64_t)x * x);
    const uint32_t x4 = modp31((uint64_t)x2 * x2);
    const uint32_t x5 = modp31((uint64_t)x4 * x);
    return modp31((uint64_t)g.A2 * x5 + g.B2) + 1u;
}

BRIG_HD uint64_t gen_sperm_step(const GenParams& g, uint64_t x) {
    const uint64_t mask = g.sbits >= 64 ? ~0ull : ((1ull << g.sbits) - 1ull);
    x = (x * g.sm1 + g.sc1) & mask;
    x ^= x >> g.sh;
    x = (x * g.sm2 + g.sc2) & mask;
    x ^= x >> g.sh;
    x = (x * g.sm3 + g.sc3) & mask;
    return x;
}

BRIG_HD int64_t gen_sperm(const GenParams& g, int64_t i) {
    uint64_t y = gen_sperm_step(g, (uint64_t)i);
    while (y >= (uint64_t)g.ns) y = gen_sperm_step(g, y);
    return (int64_t)y;
}

// Zipf(s) rank in [1, nr] for S row i.
BRIG_HD int64_t gen_zipf_rank(const GenParams& g, int64_t i) {
    for (int t = 0; t < 64; ++t) {
        const uint64_t bits = mix64(g.seed ^ ((uint64_t)i * 0xd1b54a32d192ed03ull) ^ ((uint64_t)t << 56) ^ 0x5a5a);
        const double u01 = (double)(bits >> 11) * (1.0 / 9007199254740992.0);
        const double u = g.hN + u01 * (g.hX1 - g.hN);
        const double x = zipf_Hinv(u, g.zs);
        int64_t k = (int64_t)(x + 0.5);
        if (k < 1) k = 1;
        if (k > g.nr) k = g.nr;
        if ((double)k - x <= g.sVal || u >= zipf_H((double)k + 0.5, g.zs) - zipf_h((double)k, g.zs)) return k;
    }
    return 1;
}

BRIG_HD uint32_t gen_s_key(const GenParams& g, int64_t i) {
    const int64_t pi = gen_sperm(g, i);
    if (pi < g.m) {
        int64_t row;
        if (g.zs > 0.0) {
            row = gen_zipf_rank(g, i) - 1;
        } else {
            const uint64_t h = mix64(g.seed ^ 0x243f6a8885a308d3ull ^ ((uint64_t)i * 0x9e3779b97f4a7c15ull));
            row = (int64_t)fastrange32((uint32_t)(h >> 32), (uint32_t)g.nr);
        }
        return gen_r_key(g, row);
    }
    return 0x80000000u + modp31((uint64_t)g.A3 * (uint64_t)(pi - g.m) + g.B3);
}

}  // namespace brig
