/*
 * oracle.c - CPU restatement of BRIG-Join's join semantics. TEST INFRASTRUCTURE ONLY: the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the checker; the engine never
 * calls it, links it or falls back to it.
 *
 * Semantics pinned here (from the reference):
 *   - The join result is every (r_val, s_val) pair with r_key == s_key; duplicates on either side
 *     multiply (the hash path emits all R duplicates, src/kernel_functions.cu:415-430; the CPU
 *     check counts all of them, src/sanity_check.cpp:36-41,55-60).
 *   - The count is the number of such pairs (run_sanity_check's cpu_answer_num,
 *     src/sanity_check.cpp:50-62).
 * Deliberate difference: the reference uses INT_MIN (0x80000000) as its EMPTY slot marker
 * (src/sanity_check.cpp:16, src/kernel_functions.cu:352), so an R key equal to 0x80000000 never
 * matches there. The oracle and the engine treat every 32-bit key as valid.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

/* Table capacity 2^ceil(log2(2R)) and multiplicative hash key*2654435761 with linear probing,
 * as src/sanity_check.cpp:17-18,31,43. An occupancy byte replaces the INT_MIN sentinel. */
typedef struct {
    int64_t cap, mask;
    uint32_t* key;
    uint8_t* used;
    int64_t* cnt;   /* per-slot count of R tuples (count mode) */
    int64_t* head;  /* per-slot first R row in a chain (pair mode) */
} table_t;

static int64_t table_cap(int64_t nr) {
    int64_t cap = 1;
    while (cap < 2 * nr) cap <<= 1;
    return cap < 2 ? 2 : cap;
}

static int64_t slot0(uint32_t key, int64_t mask) {
    return (int64_t)(((uint64_t)key * 2654435761ull) & (uint64_t)mask);
}

static int table_init(table_t* t, int64_t nr, int want_cnt, int want_head) {
    memset(t, 0, sizeof(*t));
    t->cap = table_cap(nr);
    t->mask = t->cap - 1;
    t->key = (uint32_t*)malloc((size_t)t->cap * 4);
    t->used = (uint8_t*)calloc((size_t)t->cap, 1);
    if (want_cnt) t->cnt = (int64_t*)calloc((size_t)t->cap, 8);
    if (want_head) t->head = (int64_t*)malloc((size_t)t->cap * 8);
    if (!t->key || !t->used || (want_cnt && !t->cnt) || (want_head && !t->head)) return -1;
    return 0;
}

static void table_free(table_t* t) {
    free(t->key);
    free(t->used);
    free(t->cnt);
    free(t->head);
}

/* Returns the slot holding `key`, inserting it if absent. */
static int64_t table_upsert(table_t* t, uint32_t key, int* inserted) {
    int64_t h = slot0(key, t->mask);
    for (;;) {
        if (!t->used[h]) {
            t->used[h] = 1;
            t->key[h] = key;
            *inserted = 1;
            return h;
        }
        if (t->key[h] == key) {
            *inserted = 0;
            return h;
        }
        h = (h + 1) & t->mask;
    }
}

static int64_t table_find(const table_t* t, uint32_t key) {
    int64_t h = slot0(key, t->mask);
    while (t->used[h]) {
        if (t->key[h] == key) return h;
        h = (h + 1) & t->mask;
    }
    return -1;
}

int64_t oracle_count(const uint32_t* rk, int64_t nr, const uint32_t* sk, int64_t ns) {
    if (nr <= 0 || ns <= 0) return 0;
    table_t t;
    if (table_init(&t, nr, 1, 0) != 0) {
        table_free(&t);
        return -1;
    }
    for (int64_t i = 0; i < nr; ++i) {
        int ins;
        const int64_t h = table_upsert(&t, rk[i], &ins);
        t.cnt[h] += 1;
    }
    int64_t total = 0;
    for (int64_t j = 0; j < ns; ++j) {
        const int64_t h = table_find(&t, sk[j]);
        if (h >= 0) total += t.cnt[h];
    }
    table_free(&t);
    return total;
}

int64_t oracle_pairs(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk, const uint32_t* sv,
                     int64_t ns, uint32_t* out_r, uint32_t* out_s, uint32_t* out_k, int64_t cap) {
    if (nr <= 0 || ns <= 0) return 0;
    table_t t;
    int64_t* next = (int64_t*)malloc((size_t)nr * 8);
    if (!next || table_init(&t, nr, 0, 1) != 0) {
        free(next);
        table_free(&t);
        return -1;
    }
    for (int64_t i = 0; i < nr; ++i) {
        int ins;
        const int64_t h = table_upsert(&t, rk[i], &ins);
        next[i] = ins ? -1 : t.head[h];
        t.head[h] = i;
    }
    int64_t n = 0;
    for (int64_t j = 0; j < ns; ++j) {
        const int64_t h = table_find(&t, sk[j]);
        if (h < 0) continue;
        for (int64_t i = t.head[h]; i >= 0; i = next[i]) {
            if (n < cap) {
                if (out_r) out_r[n] = rv[i];
                if (out_s) out_s[n] = sv[j];
                if (out_k) out_k[n] = sk[j];
            }
            ++n;
        }
    }
    free(next);
    table_free(&t);
    return n;
}

/* LSD radix sort of 64-bit values, 16 bits per pass. */
static int radix_sort_u64(uint64_t* a, int64_t n) {
    if (n <= 1) return 0;
    uint64_t* b = (uint64_t*)malloc((size_t)n * 8);
    int64_t* cnt = (int64_t*)malloc(65536 * 8);
    if (!b || !cnt) {
        free(b);
        free(cnt);
        return -1;
    }
    for (int pass = 0; pass < 4; ++pass) {
        const int sh = pass * 16;
        memset(cnt, 0, 65536 * 8);
        for (int64_t i = 0; i < n; ++i) cnt[(a[i] >> sh) & 0xffff]++;
        int64_t run = 0;
        for (int d = 0; d < 65536; ++d) {
            const int64_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (int64_t i = 0; i < n; ++i) b[cnt[(a[i] >> sh) & 0xffff]++] = a[i];
        uint64_t* t = a;
        a = b;
        b = t;
    }
    /* four passes: the sorted data is back in the caller's array */
    free(b);
    free(cnt);
    return 0;
}

int oracle_sort_pairs(uint32_t* a, uint32_t* b, int64_t n) {
    if (n <= 1) return 0;
    uint64_t* v = (uint64_t*)malloc((size_t)n * 8);
    if (!v) return -1;
    for (int64_t i = 0; i < n; ++i) v[i] = ((uint64_t)a[i] << 32) | b[i];
    if (radix_sort_u64(v, n) != 0) {
        free(v);
        return -1;
    }
    for (int64_t i = 0; i < n; ++i) {
        a[i] = (uint32_t)(v[i] >> 32);
        b[i] = (uint32_t)v[i];
    }
    free(v);
    return 0;
}

/* Independent cross-check: sort both sides by key (key<<32 | row) and merge equal-key runs. */
int64_t oracle_sortmerge_pairs(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk,
                               const uint32_t* sv, int64_t ns, uint32_t* out_r, uint32_t* out_s, int64_t cap) {
    if (nr <= 0 || ns <= 0) return 0;
    uint64_t* r = (uint64_t*)malloc((size_t)nr * 8);
    uint64_t* s = (uint64_t*)malloc((size_t)ns * 8);
    if (!r || !s) {
        free(r);
        free(s);
        return -1;
    }
    for (int64_t i = 0; i < nr; ++i) r[i] = ((uint64_t)rk[i] << 32) | (uint64_t)(uint32_t)i;
    for (int64_t j = 0; j < ns; ++j) s[j] = ((uint64_t)sk[j] << 32) | (uint64_t)(uint32_t)j;
    if (nr >= ((int64_t)1 << 32) || ns >= ((int64_t)1 << 32) || radix_sort_u64(r, nr) || radix_sort_u64(s, ns)) {
        free(r);
        free(s);
        return -1;
    }
    int64_t i = 0, j = 0, n = 0;
    while (i < nr && j < ns) {
        const uint32_t kr = (uint32_t)(r[i] >> 32), ks = (uint32_t)(s[j] >> 32);
        if (kr < ks) { ++i; continue; }
        if (ks < kr) { ++j; continue; }
        int64_t i2 = i, j2 = j;
        while (i2 < nr && (uint32_t)(r[i2] >> 32) == kr) ++i2;
        while (j2 < ns && (uint32_t)(s[j2] >> 32) == ks) ++j2;
        for (int64_t a = i; a < i2; ++a)
            for (int64_t b = j; b < j2; ++b) {
                if (n < cap) {
                    if (out_r) out_r[n] = rv[(uint32_t)r[a]];
                    if (out_s) out_s[n] = sv[(uint32_t)s[b]];
                }
                ++n;
            }
        i = i2;
        j = j2;
    }
    free(r);
    free(s);
    return n;
}

/* FNV-1a over the (already sorted) pairs: a compact fingerprint of a pair multiset. */
uint64_t oracle_pairs_digest(const uint32_t* a, const uint32_t* b, int64_t n) {
    uint64_t h = 1469598103934665603ull;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t w[2] = {a[i], b[i]};
        const unsigned char* p = (const unsigned char*)w;
        for (int k = 0; k < 8; ++k) {
            h ^= p[k];
            h *= 1099511628211ull;
        }
    }
    return h;
}
