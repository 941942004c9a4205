/*
 * oracle.h - CPU restatement of BRIG-Join's join semantics (test infrastructure only; see oracle.c).
 */
#ifndef BRIG_ORACLE_H_
#define BRIG_ORACLE_H_
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Number of key-equal (R, S) pairs; restates run_sanity_check (src/sanity_check.cpp:16-62). */
int64_t oracle_count(const uint32_t* rk, int64_t nr, const uint32_t* sk, int64_t ns);

/* Every key-equal pair (r_val, s_val[, key]) in S order; writes the first `cap`, returns the total.
 * The pair-emitting form of the same build/probe (src/sanity_check.cpp:28-62) with per-key chains
 * of R rows, matching the GPU hash path's emission of all R duplicates
 * (src/kernel_functions.cu:415-430). */
int64_t oracle_pairs(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk, const uint32_t* sv,
                     int64_t ns, uint32_t* out_r, uint32_t* out_s, uint32_t* out_k, int64_t cap);

/* Independent sort-merge join producing the same multiset (cross-check of oracle_pairs). */
int64_t oracle_sortmerge_pairs(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk,
                               const uint32_t* sv, int64_t ns, uint32_t* out_r, uint32_t* out_s, int64_t cap);

/* Sorts pairs lexicographically by (a, b) in place. */
int oracle_sort_pairs(uint32_t* a, uint32_t* b, int64_t n);

/* FNV-1a fingerprint of a sorted pair list. */
uint64_t oracle_pairs_digest(const uint32_t* a, const uint32_t* b, int64_t n);

/* The benchmark's synthetic inputs (gen.c): distinct R keys in [1, 2^31), a fraction match_frac of
 * S rows drawn uniformly from R's keys, the rest distinct in [2^31, 2^32 - 1), values = row index.
 * Any output pointer may be NULL. Returns 0, or -1 for bad arguments. */
int oracle_gen(uint64_t seed, int64_t nr, int64_t ns, double match_frac, uint32_t* rk, uint32_t* rv,
               uint32_t* sk, uint32_t* sv);

#ifdef __cplusplus
}
#endif
#endif
