// shard.cu - key ownership across GPUs: the local steps of a join sharded over ranks (one process
// per GPU). The exchanges between them (all-to-all of tuples, all-gather of filters) are the
// caller's, over NCCL; brig_join/shard.py does them with torch.distributed.
//
// The reference sends R and the Bloom-prefiltered S to the PE that owns each first-level partition
// (partition p on PE p * D / P, src/r_shuffle.cu:33-191), merges the PEs' filters with an OR
// all-reduce (src/bf_allreduce.cu:236-284) and joins locally. For skewed inputs it rebalances S' and
// replicates hot R partitions (src/s_redistribute.cu:26-152, src/r_replicate.cu:13-100). Here:
//   - a key's owner is fastrange32(owner_mix(key), nranks). owner_mix is the partition mix on the
//     key xor a fixed seed, so ownership is independent of the partition and bucket bits. An owner's
//     keys still spread over all of its local partitions. Owning whole first-level partitions, as
//     the reference does, would leave each GPU's join with 1/nranks of its partitions;
//   - a filter is built after R's exchange, one per owner over the R tuples it owns. The owners'
//     filters cover disjoint keys, so gathering them gives every rank the whole filter without an
//     OR reduction (NCCL has none);
//   - S is prefiltered and grouped by owner in one pass over the keys for the counts and one for the
//     scatter, each key tested against its owner's filter;
//   - heavy keys (a short sorted list the caller picks from a sample of S) go to one extra bin,
//     untested: the caller replicates their R tuples to every rank and keeps their S tuples where
//     they are, so no rank receives a hot key's whole share of S.
// k_shard_split counts (kWrite false) or scatters (kWrite true) one relation's tuples into the
// bins. Each warp ranks its lanes of one bin together (one shared-memory atomic per bin and warp),
// so the stores of a warp's tuples of one bin are consecutive. k_shard_offsets turns the counts
// into bin starts. k_shard_bloom_build builds one owner's filter: the engine's blocked word-pair
// filter (brig_common.cuh) with a single segment, one 64-bit atomicOr per key.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include "../../include/brig_join.h"
#include "engine.h"
#include "launch.h"

namespace brig {
namespace {

constexpr int kShardThreads = 512;
constexpr int kShardItems = 8;  // tuples per thread and tile
constexpr int kShardTile = kShardThreads * kShardItems;
constexpr int kMaxBins = BRIG_SHARD_MAX_RANKS + 1;
constexpr uint32_t kOwnerSeed = 0x6a09e667u;  // the first 32 fractional bits of sqrt(2)

// CTAs of k_shard_split per SM: 32 registers a thread for the count without filters, 64 for the
// scatters (keys, values, bins and ranks of 8 tuples) and with filters (8 filter word pairs and
// masks in flight).
constexpr int shard_ctas(bool write, bool filter, bool cache = false) {
    return (filter || cache || write) ? 2 : 4;
}

BRIG_HD uint32_t owner_of(uint32_t key, uint32_t nranks) { return fastrange32(mix32(key ^ kOwnerSeed), nranks); }

struct ShardArgs {
    int32_t nranks, nbins;   // nbins = nranks + 1 with heavy keys (bin nranks), else nranks
    const uint32_t* filter;  // every owner's filter words, or nullptr
    const int64_t* floc;     // [2 * nranks]: word offset and word count of owner r's filter
    const uint32_t* heavy;   // sorted heavy keys
    int32_t n_heavy;
    int32_t k;               // hashes of the filters
    uint8_t* cache;          // [n] bin of every tuple (0xff: dropped), or nullptr
};

// Whether k is in the sorted array a[0, n).
__device__ __forceinline__ bool in_sorted(const uint32_t* a, int n, uint32_t k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && a[lo] == k;
}

// counts: [nbins] (kWrite false). start: [nbins + 1] bin starts in out_key/out_val, cursor: [nbins]
// tuples placed so far per bin, errors: tuples that found their bin full (kWrite true). kFilter:
// the spec has filters (K: their mask class); without them a thread needs fewer registers and
// more CTAs fit on an SM (shard_ctas), so more key loads are in flight. With a bin cache the count
// pass stores every tuple's bin and the scatter (kCache) reads it instead of testing the filters
// again.
template <bool kWrite, bool kFilter, int K, bool kCache = false>
__global__ void __launch_bounds__(kShardThreads, shard_ctas(kWrite, kFilter, kCache))
k_shard_split(ShardArgs a, const uint32_t* __restrict__ key, const uint32_t* __restrict__ val, int64_t n,
              unsigned long long* counts, const int64_t* __restrict__ start, unsigned long long* cursor,
              uint32_t* __restrict__ out_key, uint32_t* __restrict__ out_val, unsigned long long* errors) {
    __shared__ uint32_t s_cnt[kMaxBins];
    __shared__ int64_t s_base[kMaxBins];
    __shared__ int64_t s_end[kMaxBins];
    __shared__ int64_t s_floc[2 * BRIG_SHARD_MAX_RANKS];
    __shared__ uint32_t s_heavy[BRIG_SHARD_MAX_HEAVY];
    __shared__ uint2 s_pat[pat_entries<K>()];
    if (kFilter && K != kBloomFastK) fill_patterns(s_pat, a.k);
    for (int i = threadIdx.x; i < a.nbins; i += kShardThreads) {
        s_cnt[i] = 0;
        if (kWrite) s_end[i] = start[i + 1];
    }
    if (kFilter)
        for (int i = threadIdx.x; i < 2 * a.nranks; i += kShardThreads) s_floc[i] = a.floc[i];
    for (int i = threadIdx.x; i < a.n_heavy; i += kShardThreads) s_heavy[i] = a.heavy[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t nr = (uint32_t)a.nranks;
    const int64_t ntiles = (n + kShardTile - 1) / kShardTile;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t t0 = t * kShardTile;
        uint32_t kk[kShardItems], vv[kShardItems];
        int bin[kShardItems];
        // a scatter without filters keeps every tuple: its values load with its keys
        constexpr bool kAllKept = kWrite && !kFilter && !kCache;
#pragma unroll
        for (int u = 0; u < kShardItems; ++u) {
            const int64_t i = t0 + u * kShardThreads + threadIdx.x;
            kk[u] = i < n ? key[i] : 0u;
            vv[u] = (kAllKept && i < n) ? val[i] : 0u;
            bin[u] = i < n ? 0 : -1;
        }
        if constexpr (kCache) {
#pragma unroll
            for (int u = 0; u < kShardItems; ++u) {
                const int64_t i = t0 + u * kShardThreads + threadIdx.x;
                if (i < n) {
                    const uint32_t c = a.cache[i];
                    bin[u] = c == 0xffu ? -1 : (int)c;
                }
            }
        } else {
            // owners, and the filter words of every key in flight together
            uint2 w[kShardItems], mk[kShardItems];
#pragma unroll
            for (int u = 0; u < kShardItems; ++u) {
                w[u] = make_uint2(0u, 0u);
                mk[u] = make_uint2(0u, 0u);
                if (bin[u] < 0) continue;
                if (a.n_heavy > 0 && in_sorted(s_heavy, a.n_heavy, kk[u])) {
                    bin[u] = (int)nr;
                    continue;
                }
                const uint32_t o = owner_of(kk[u], nr);
                bin[u] = (int)o;
                if (kFilter) {
                    const int64_t off = s_floc[2 * o], words = s_floc[2 * o + 1];
                    if (words < 8 || off < 0 || (off & 1)) {  // no filter block (the owner holds no R
                        bin[u] = -1;                           // tuple), or no aligned word pair to read
                        continue;
                    }
                    const BloomSlot sl = bloom_slot(mix32(kk[u]), 0u, (uint32_t)(words >> 3));
                    mk[u] = slot_masks<K>(s_pat, sl);
                    w[u] = __ldg(reinterpret_cast<const uint2*>(a.filter + off + sl.widx));
                }
            }
            if constexpr (kFilter) {
#pragma unroll
                for (int u = 0; u < kShardItems; ++u)
                    if (bin[u] >= 0 && bin[u] < (int)nr && !bloom_pass(w[u], mk[u])) bin[u] = -1;
            }
            if (!kWrite && a.cache != nullptr) {
#pragma unroll
                for (int u = 0; u < kShardItems; ++u) {
                    const int64_t i = t0 + u * kShardThreads + threadIdx.x;
                    if (i < n) a.cache[i] = (uint8_t)(bin[u] < 0 ? 0xff : bin[u]);
                }
            }
        }
        if constexpr (kWrite && !kAllKept) {
            // the kept tuples' values, in flight while the tile is ranked and the bins reserved
#pragma unroll
            for (int u = 0; u < kShardItems; ++u)
                if (bin[u] >= 0) vv[u] = val[t0 + u * kShardThreads + threadIdx.x];
        }
        uint32_t rank[kShardItems];
#pragma unroll
        for (int u = 0; u < kShardItems; ++u) {
            const int b = bin[u];
            const uint32_t peers = __match_any_sync(0xffffffffu, b);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (b >= 0 && lane == leader) base = atomicAdd(&s_cnt[b], (uint32_t)__popc(peers));
            if (kWrite) rank[u] = __shfl_sync(0xffffffffu, base, leader) + (uint32_t)__popc(peers & below);
        }
        if constexpr (kWrite) {
            __syncthreads();
            if (threadIdx.x < a.nbins) {
                const uint32_t c = s_cnt[threadIdx.x];
                s_base[threadIdx.x] =
                    c ? start[threadIdx.x] + (int64_t)atomicAdd(&cursor[threadIdx.x], (unsigned long long)c) : 0;
                s_cnt[threadIdx.x] = 0;
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < kShardItems; ++u) {
                const int b = bin[u];
                if (b < 0) continue;
                const int64_t p = s_base[b] + rank[u];
                if (p < s_end[b]) {
                    out_key[p] = kk[u];
                    out_val[p] = vv[u];
                } else {
                    atomicAdd(errors, 1ull);
                }
            }
            __syncthreads();  // s_base is read before the next tile's reservations
        }
    }
    if constexpr (!kWrite) {
        __syncthreads();
        if (threadIdx.x < a.nbins && s_cnt[threadIdx.x])
            atomicAdd(&counts[threadIdx.x], (unsigned long long)s_cnt[threadIdx.x]);
    }
}

// start[b] = counts of the bins before b, start[nbins] = the total; cursors and the error word zeroed.
__global__ void k_shard_offsets(const int64_t* __restrict__ counts, int nbins, int64_t* start,
                                unsigned long long* cursor, unsigned long long* errors) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t s = 0;
    for (int b = 0; b < nbins; ++b) {
        start[b] = s;
        s += counts[b];
        cursor[b] = 0;
    }
    start[nbins] = s;
    *errors = 0;
}

template <int K>
__global__ void __launch_bounds__(kShardThreads)
k_shard_bloom_build(const uint32_t* __restrict__ key, int64_t n, uint32_t* words, uint32_t nblocks, int k) {
    __shared__ uint2 s_pat[pat_entries<K>()];
    if constexpr (K != kBloomFastK) {
        fill_patterns(s_pat, k);
        __syncthreads();
    }
    for (int64_t i = (int64_t)blockIdx.x * kShardThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kShardThreads) {
        const BloomSlot sl = bloom_slot(mix32(key[i]), 0u, nblocks);
        const uint2 mk = slot_masks<K>(s_pat, sl);
        // one 64-bit atomic on the word pair (even word low): the build is bound by the number of
        // atomics the L2 serves, not by their width
        atomicOr(reinterpret_cast<unsigned long long*>(words + sl.widx),
                 ((unsigned long long)mk.y << 32) | (unsigned long long)mk.x);
    }
}

int sm_count() {
    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    return std::max(sms, 1);
}

ShardArgs check_spec(const brig_shard_spec* sp, int64_t n, const uint32_t* key) {
    if (!sp) fail(BRIG_E_INVALID, "null shard spec");
    if (sp->nranks < 1 || sp->nranks > BRIG_SHARD_MAX_RANKS) fail(BRIG_E_INVALID, "nranks out of range");
    if (n < 0 || (n > 0 && !key)) fail(BRIG_E_INVALID, "bad key array");
    if (sp->n_heavy < 0 || sp->n_heavy > BRIG_SHARD_MAX_HEAVY || (sp->n_heavy > 0 && !sp->heavy))
        fail(BRIG_E_INVALID, "bad heavy-key list");
    if (sp->filter && (!sp->filter_loc || sp->bloom_num_hashes < 1 || sp->bloom_num_hashes > 16))
        fail(BRIG_E_INVALID, "a filter needs filter_loc and 1 <= bloom_num_hashes <= 16");
    if (sp->filter && (reinterpret_cast<uintptr_t>(sp->filter) & 7))
        fail(BRIG_E_INVALID, "filter words must be 8-byte aligned");
    ShardArgs a;
    a.nranks = sp->nranks;
    a.nbins = sp->nranks + (sp->n_heavy > 0 ? 1 : 0);
    a.filter = sp->filter;
    a.floc = sp->filter_loc;
    a.heavy = sp->heavy;
    a.n_heavy = sp->n_heavy;
    a.k = sp->bloom_num_hashes;
    a.cache = sp->bin_cache;
    return a;
}

template <bool kWrite>
void launch_split(const ShardArgs& a, const uint32_t* key, const uint32_t* val, int64_t n, unsigned long long* counts,
                  const int64_t* start, unsigned long long* cursor, uint32_t* ok, uint32_t* ov,
                  unsigned long long* errors, cudaStream_t st) {
    if (n == 0) return;
    const int64_t ntiles = (n + kShardTile - 1) / kShardTile;
    const int sms = sm_count();
    const int grid = (int)std::min<int64_t>(ntiles, (int64_t)sms * shard_ctas(kWrite, a.filter != nullptr));
    if constexpr (kWrite) {
        if (a.cache) {
            const int grid_c = (int)std::min<int64_t>(ntiles, (int64_t)sms * shard_ctas(true, false, true));
            k_shard_split<true, false, kBloomFastK, true><<<grid_c, kShardThreads, 0, st>>>(a, key, val, n, counts,
                                                                                           start, cursor, ok, ov,
                                                                                           errors);
            note_launches(1);
            cuda_check(cudaGetLastError(), "k_shard_split");
            return;
        }
    }
    if (!a.filter)
        k_shard_split<kWrite, false, kBloomFastK><<<grid, kShardThreads, 0, st>>>(a, key, val, n, counts, start, cursor,
                                                                                  ok, ov, errors);
    else if (a.k != kBloomFastK)
        k_shard_split<kWrite, true, 0><<<grid, kShardThreads, 0, st>>>(a, key, val, n, counts, start, cursor, ok, ov,
                                                                       errors);
    else
        k_shard_split<kWrite, true, kBloomFastK><<<grid, kShardThreads, 0, st>>>(a, key, val, n, counts, start, cursor,
                                                                                 ok, ov, errors);
    note_launches(1);
    cuda_check(cudaGetLastError(), "k_shard_split");
}

template <class F>
int shard_guard(F&& f) {
    try {
        f();
        return BRIG_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.status;
    }
}

}  // namespace
}  // namespace brig

extern "C" {

int32_t brig_shard_owner(uint32_t key, int32_t nranks) {
    if (nranks < 1 || nranks > BRIG_SHARD_MAX_RANKS) return -1;
    return (int32_t)brig::owner_of(key, (uint32_t)nranks);
}

int64_t brig_shard_filter_words(int64_t n_keys, double bits_per_key) {
    if (n_keys < 0 || !(bits_per_key > 0.0) || bits_per_key > 1024.0) return -1;
    const double blocks = std::ceil((double)n_keys * bits_per_key / 256.0);
    const int64_t words = std::max<int64_t>(1, (int64_t)blocks) * 8;
    return words < (int64_t(1) << 32) ? words : -1;
}

int brig_shard_count(const brig_shard_spec* sp, const uint32_t* key, int64_t n, int64_t* counts, void* stream) {
    using namespace brig;
    return shard_guard([&] {
        const ShardArgs a = check_spec(sp, n, key);
        if (!counts) fail(BRIG_E_INVALID, "null counts");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        cuda_check(cudaMemsetAsync(counts, 0, sizeof(int64_t) * a.nbins, st), "cudaMemsetAsync");
        launch_split<false>(a, key, nullptr, n, reinterpret_cast<unsigned long long*>(counts), nullptr, nullptr,
                            nullptr, nullptr, nullptr, st);
    });
}

int brig_shard_scatter(const brig_shard_spec* sp, const uint32_t* key, const uint32_t* val, int64_t n,
                       const int64_t* counts, int64_t* scratch, uint32_t* out_key, uint32_t* out_val, void* stream) {
    using namespace brig;
    return shard_guard([&] {
        const ShardArgs a = check_spec(sp, n, key);
        if (!counts || !scratch || (n > 0 && (!val || !out_key || !out_val)))
            fail(BRIG_E_INVALID, "null counts, scratch, values or outputs");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        int64_t* start = scratch;
        auto* cursor = reinterpret_cast<unsigned long long*>(scratch + a.nbins + 1);
        auto* errors = reinterpret_cast<unsigned long long*>(scratch + 2 * a.nbins + 1);
        k_shard_offsets<<<1, 32, 0, st>>>(counts, a.nbins, start, cursor, errors);
        note_launches(1);
        cuda_check(cudaGetLastError(), "k_shard_offsets");
        launch_split<true>(a, key, val, n, nullptr, start, cursor, out_key, out_val, errors, st);
    });
}

int brig_shard_bloom_build(const uint32_t* key, int64_t n, uint32_t* words, int64_t n_words, int32_t num_hashes,
                           void* stream) {
    using namespace brig;
    return shard_guard([&] {
        if (n < 0 || (n > 0 && !key) || !words || n_words < 8 || (n_words & 7) || n_words >= (int64_t(1) << 32) ||
            num_hashes < 1 || num_hashes > 16 || (reinterpret_cast<uintptr_t>(words) & 7))
            fail(BRIG_E_INVALID, "brig_shard_bloom_build: bad argument");
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        cuda_check(cudaMemsetAsync(words, 0, (size_t)n_words * 4, st), "cudaMemsetAsync");
        if (n == 0) return;
        const int grid = (int)std::min<int64_t>((n + kShardThreads - 1) / kShardThreads, (int64_t)sm_count() * 4);
        const uint32_t nblocks = (uint32_t)(n_words >> 3);
        if (num_hashes == kBloomFastK)
            k_shard_bloom_build<kBloomFastK><<<grid, kShardThreads, 0, st>>>(key, n, words, nblocks, num_hashes);
        else
            k_shard_bloom_build<0><<<grid, kShardThreads, 0, st>>>(key, n, words, nblocks, num_hashes);
        note_launches(1);
        cuda_check(cudaGetLastError(), "k_shard_bloom_build");
    });
}

}  // extern "C"
