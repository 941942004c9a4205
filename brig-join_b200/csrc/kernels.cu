// kernels.cu - the join pipeline for sm_100a.
//
// Stage map (reference kernel -> kernel here):
//   gpu_prefix_init + gpu_run_hist_for_both (src/kernel_functions.cu:22-90,141-159) -> k_l1_hist
//   queryAndCompactKernelPartitioned (src/bloom.cu:725-773), fused into S's histogram pass
//                                                                            -> k_l1_hist (Bloom)
//   gpu_make_simple_prefix (src/kernel_functions.cu:461-492)          -> k_scan_* (device-wide)
//   gpu_make_sorted_table_for_both (src/kernel_functions.cu:95-133)    -> k_l1_scatter
//   gpu_run_hist_second_pass + gpu_build_table_second_pass_kv (src/kernel_functions.cu:163-281)
//                                                                      -> k_l2_partition
//   insertKernelPartitioned (src/bloom.cu:698-722)                     -> k_bloom_build
//   gpu_probe_with_second_pass / gpu_fused_probe_transfer local part
//   (src/kernel_functions.cu:294-454, 612-789), including the split path (:356-395)
//                                                                      -> k_tasks_* + k_probe
//
// Design points that differ from the reference on purpose:
//   * The first-level scatter does no global atomics. Each CTA owns a contiguous slice of the
//     input, the histogram pass records a per-(partition, slice) count, and one exclusive scan of
//     the partition-major [P1][slices] matrix gives every slice a private output run per partition.
//     The reference takes one 64-bit global atomic per tuple on P counters (:122,129).
//   * Tiles are staged in shared memory and reordered by partition before they are written, so
//     consecutive threads store consecutive addresses of the same partition run.
//   * The probe is a persistent work-queue kernel over (join, partition-pair) tasks. An R partition
//     larger than one shared-memory table is cut into table-sized chunks, each probed by the whole
//     S partition, so duplicates are exact (the reference's split path stops at the first match,
//     :371). A large S partition is cut into chunks that run as separate tasks.
//   * Matches are staged per warp in shared memory and written with one global atomic per flush
//     (the reference takes one global atomic per output pair, :420).
//   * The shared-memory table is bucketised (counting sort by bucket) rather than open addressing,
//     so every 32-bit key is valid (the reference reserves 0x80000000 as EMPTY, :352).
//   * Every computed store position is checked against its buffer; a failure increments an error
//     word the host reads instead of writing out of bounds.
#include <cstdio>
#include <algorithm>
#include "launch.h"

namespace brig {

namespace {

__device__ __forceinline__ int64_t min_i64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Index j with prefix[j] <= g < prefix[j+1] (prefix is non-decreasing, prefix[0] == 0).
__device__ __forceinline__ int find_owner(const int64_t* __restrict__ prefix, int n, int64_t g) {
    int lo = 0, hi = n;  // answer in [lo, hi)
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// Block-wide exclusive scan of n uint32 values in shared memory, in place. Returns the total.
// blockDim.x must be kThreads; tmp holds kThreads/32 words.
__device__ uint32_t block_scan_excl(uint32_t* a, int n, uint32_t* tmp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int kWarps = kThreads / 32;
    const int per = (n + kThreads - 1) / kThreads;
    const int beg = min(n, (int)threadIdx.x * per);
    const int end = min(n, beg + per);
    uint32_t sum = 0;
    for (int i = beg; i < end; ++i) sum += a[i];
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < kWarps ? tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) tmp[lane] = w;
    }
    __syncthreads();
    uint32_t run = x - sum + (wid > 0 ? tmp[wid - 1] : 0u);
    const uint32_t total = tmp[kWarps - 1];
    for (int i = beg; i < end; ++i) {
        uint32_t v = a[i];
        a[i] = run;
        run += v;
    }
    __syncthreads();
    return total;
}

// Same for int64 values (one value per thread), returns the exclusive prefix of this thread.
__device__ int64_t block_scan_excl_i64(int64_t v, int64_t* tmp /* kThreads/32 */, int64_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int kWarps = kThreads / 32;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int64_t w = lane < kWarps ? tmp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) tmp[lane] = w;
    }
    __syncthreads();
    int64_t excl = x - v + (wid > 0 ? tmp[wid - 1] : 0);
    *total = tmp[kWarps - 1];
    __syncthreads();
    return excl;
}

__device__ __forceinline__ const uint2* final_buf(const JoinDesc& d, int rel) {
    return d.pf.P2 > 1 ? d.rel[rel].l2 : d.rel[rel].l1;
}

// Loads one tuple from separate key/value arrays.
struct SoASrc {
    const uint32_t* __restrict__ k;
    const uint32_t* __restrict__ v;
    __device__ __forceinline__ uint2 operator()(int64_t i) const {
        return make_uint2(__ldg(k + i), __ldg(v + i));
    }
};
// Loads one packed tuple.
struct AoSSrc {
    const uint2* __restrict__ p;
    __device__ __forceinline__ uint2 operator()(int64_t i) const { return __ldg(p + i); }
};
struct Bin1 {
    PartFn f;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return part1(f, key); }
};
struct Bin2 {
    PartFn f;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return part2(f, key); }
};

// Scatters tuples [begin, end) of `src` into `out`. cursor[b] is the next output position of bin
// b; it advances as tiles are written. Each tile of kTile tuples is counted, reordered by bin in
// shared memory (stage), and written so that consecutive threads store consecutive positions of
// one bin's run.
template <class Src, class Bin>
__device__ void scatter_tiles(const Src& src, int64_t begin, int64_t end, const Bin& bin, int nbins,
                              uint2* __restrict__ out, int64_t out_limit, int64_t* cursor,
                              uint32_t* cnt, uint32_t* tmp, uint2* stage,
                              unsigned long long* errors) {
    constexpr int kItems = kTile / kThreads;
    for (int64_t t0 = begin; t0 < end; t0 += kTile) {
        const int tn = (int)min_i64(kTile, end - t0);
        for (int b = threadIdx.x; b < nbins; b += kThreads) cnt[b] = 0;
        __syncthreads();
        uint2 v[kItems];
        uint32_t bb[kItems], rk[kItems];
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < tn) {
                v[k] = src(t0 + i);
                bb[k] = bin(v[k].x);
                rk[k] = atomicAdd(&cnt[bb[k]], 1u);
            }
        }
        __syncthreads();
        block_scan_excl(cnt, nbins, tmp);  // cnt[b] = first staged position of bin b
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < tn) stage[cnt[bb[k]] + rk[k]] = v[k];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < tn; i += kThreads) {
            const uint2 e = stage[i];
            const uint32_t b = bin(e.x);
            const int64_t dst = cursor[b] + (int64_t)(i - (int)cnt[b]);
            if (dst >= 0 && dst < out_limit) out[dst] = e;
            else atomicAdd(errors, 1ull);
        }
        __syncthreads();
        for (int b = threadIdx.x; b < nbins; b += kThreads) {
            const uint32_t nxt = (b + 1 < nbins) ? cnt[b + 1] : (uint32_t)tn;
            cursor[b] += (int64_t)(nxt - cnt[b]);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Level 1, pass 1: per-slice histogram over P1 partitions (R, or S without Bloom), or the fused
// Bloom probe + survivor compaction + histogram (S with Bloom).
// hist layout per relation: [p * nslices + s], plus one trailing zero (sentinel) so that the
// exclusive scan of entry P1*nslices is the relation's total.
__global__ void __launch_bounds__(kThreads)
k_l1_hist(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ slice_prefix,
          uint32_t* __restrict__ hist, unsigned long long* gwords) {
    extern __shared__ uint32_t sh_cnt[];  // [max P1]
    __shared__ uint32_t s_cursor;
    const int lane = threadIdx.x & 31;
    const int64_t total = slice_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(slice_prefix, nj, g);
        const JoinDesc& d = J[j];
        const RelPlan& R = d.rel[rel];
        const int s = (int)(g - slice_prefix[j]);
        const int64_t b = (int64_t)s * R.slice_len;
        const int64_t e = min(b + R.slice_len, R.n);
        const PartFn pf = d.pf;
        const uint32_t P1 = pf.P1;
        for (uint32_t i = threadIdx.x; i < P1; i += kThreads) sh_cnt[i] = 0;
        if (threadIdx.x == 0) s_cursor = 0;
        __syncthreads();
        const bool bloom = (rel == 1) && d.bloom != nullptr;
        if (!bloom) {
            const uint32_t* __restrict__ key = R.key;
            if ((((uintptr_t)(key + b)) & 15) == 0) {
                int64_t i = b + 4 * (int64_t)threadIdx.x;
                for (; i + 3 < e; i += 4 * kThreads) {
                    const uint4 k4 = __ldg(reinterpret_cast<const uint4*>(key + i));
                    atomicAdd(&sh_cnt[part1(pf, k4.x)], 1u);
                    atomicAdd(&sh_cnt[part1(pf, k4.y)], 1u);
                    atomicAdd(&sh_cnt[part1(pf, k4.z)], 1u);
                    atomicAdd(&sh_cnt[part1(pf, k4.w)], 1u);
                }
                // tail: at most 3 tuples past the last full vector
                const int64_t tail0 = b + ((e - b) & ~(int64_t)3);
                for (int64_t t = tail0 + threadIdx.x; t < e; t += kThreads)
                    atomicAdd(&sh_cnt[part1(pf, __ldg(key + t))], 1u);
            } else {
                for (int64_t t = b + threadIdx.x; t < e; t += kThreads)
                    atomicAdd(&sh_cnt[part1(pf, __ldg(key + t))], 1u);
            }
        } else {
            // Bloom probe of every S key against the segment of its finest partition; survivors are
            // compacted (key, value) into R.cmp[b, b + count) and counted per level-1 partition.
            const uint32_t* __restrict__ key = R.key;
            const uint32_t* __restrict__ val = R.val;
            const uint32_t* __restrict__ filt = d.bloom;
            const uint32_t seg_blocks = d.seg_blocks;
            const int k = d.bloom_k;
            for (int64_t i0 = b; i0 < e; i0 += kThreads) {
                const int64_t i = i0 + threadIdx.x;
                bool pass = false;
                uint32_t kk = 0, p = 0;
                if (i < e) {
                    kk = __ldg(key + i);
                    p = part1(pf, kk);
                    const uint32_t f = p * pf.P2 + part2(pf, kk);
                    BloomKey bk;
                    bloom_key(kk, seg_blocks, k, bk);
                    const uint4* blk = reinterpret_cast<const uint4*>(
                        filt + ((int64_t)f * seg_blocks + bk.block) * 8);
                    const uint4 w0 = __ldg(blk), w1 = __ldg(blk + 1);
                    pass = ((w0.x & bk.mask[0]) == bk.mask[0]) && ((w0.y & bk.mask[1]) == bk.mask[1]) &&
                           ((w0.z & bk.mask[2]) == bk.mask[2]) && ((w0.w & bk.mask[3]) == bk.mask[3]) &&
                           ((w1.x & bk.mask[4]) == bk.mask[4]) && ((w1.y & bk.mask[5]) == bk.mask[5]) &&
                           ((w1.z & bk.mask[6]) == bk.mask[6]) && ((w1.w & bk.mask[7]) == bk.mask[7]);
                }
                const uint32_t m = __ballot_sync(0xffffffffu, pass);
                if (m) {
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(&s_cursor, (uint32_t)__popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (pass) {
                        atomicAdd(&sh_cnt[p], 1u);
                        const int64_t dst = b + base + __popc(m & lanemask_lt());
                        if (dst < e) R.cmp[dst] = make_uint2(kk, __ldg(val + i));
                        else atomicAdd(&gwords[kGErrors], 1ull);
                    }
                }
            }
        }
        __syncthreads();
        uint32_t* H = hist + R.hist_base;
        for (uint32_t p = threadIdx.x; p < P1; p += kThreads) H[(int64_t)p * R.nslices + s] = sh_cnt[p];
        if (threadIdx.x == 0) {
            if (s == 0) H[(int64_t)P1 * R.nslices] = 0;
            if (bloom) {
                R.slice_cnt[s] = s_cursor;
                atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSurvivors]),
                          (unsigned long long)s_cursor);
            } else if (rel == 1) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSurvivors]),
                          (unsigned long long)(e - b));
            }
        }
        __syncthreads();
    }
}

// Level 1, pass 2: scatter each slice into its private runs. cursor[p] = scan[p][s] - scan[0][0]
// of this relation, i.e. the partition's start plus the counts of all earlier slices.
__global__ void __launch_bounds__(kThreads)
k_l1_scatter(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ slice_prefix,
             const int64_t* __restrict__ scan, unsigned long long* gwords) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* stage = reinterpret_cast<uint2*>(smem);                          // [kTile]
    int64_t* cursor = reinterpret_cast<int64_t*>(stage + kTile);            // [max P1]
    uint32_t* cnt = reinterpret_cast<uint32_t*>(cursor + kMaxP1);           // [max P1]
    __shared__ uint32_t tmp[kThreads / 32];
    const int64_t total = slice_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(slice_prefix, nj, g);
        const JoinDesc& d = J[j];
        const RelPlan& R = d.rel[rel];
        const int s = (int)(g - slice_prefix[j]);
        const int64_t b = (int64_t)s * R.slice_len;
        const bool bloom = (rel == 1) && d.bloom != nullptr;
        const int64_t e = bloom ? b + R.slice_cnt[s] : min(b + R.slice_len, R.n);
        const uint32_t P1 = d.pf.P1;
        const int64_t* S = scan + R.hist_base;
        const int64_t s0 = S[0];
        for (uint32_t p = threadIdx.x; p < P1; p += kThreads)
            cursor[p] = S[(int64_t)p * R.nslices + s] - s0;
        __syncthreads();
        const Bin1 bin{d.pf};
        if (bloom) {
            scatter_tiles(AoSSrc{R.cmp}, b, e, bin, (int)P1, R.l1, R.n, cursor, cnt, tmp, stage,
                          &gwords[kGErrors]);
        } else {
            scatter_tiles(SoASrc{R.key, R.val}, b, e, bin, (int)P1, R.l1, R.n, cursor, cnt, tmp, stage,
                          &gwords[kGErrors]);
        }
    }
}

// Level-1 partition starts of every join with P2 == 1, or the level-2 input ranges otherwise:
// b1[p] = start of partition p in l1, b1[P1] = relation total. One thread per entry.
__global__ void k_bounds_l1(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ scan) {
    for (int j = blockIdx.y; j < nj; j += gridDim.y) {
        const JoinDesc& d = J[j];
        const RelPlan& R = d.rel[rel];
        const uint32_t P1 = d.pf.P1;
        const int64_t* S = scan + R.hist_base;
        int64_t* b1 = R.b1;
        const int64_t s0 = S[0];
        for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p <= P1; p += gridDim.x * blockDim.x)
            b1[p] = S[(int64_t)p * R.nslices] - s0;
    }
}

// Level 2: one CTA per (join, level-1 partition). Counts the partition by its level-2 id, writes
// the finest-partition bounds, then scatters the partition from l1 into l2 in the same range.
__global__ void __launch_bounds__(kThreads)
k_l2_partition(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ seg_prefix,
               unsigned long long* gwords) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* stage = reinterpret_cast<uint2*>(smem);                 // [kTile]
    int64_t* cursor = reinterpret_cast<int64_t*>(stage + kTile);   // [max P2]
    uint32_t* cnt = reinterpret_cast<uint32_t*>(cursor + kMaxP2);  // [max P2]
    __shared__ uint32_t tmp[kThreads / 32];
    const int64_t total = seg_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(seg_prefix, nj, g);
        const JoinDesc& d = J[j];
        const RelPlan& R = d.rel[rel];
        const uint32_t p = (uint32_t)(g - seg_prefix[j]);
        const uint32_t P2 = d.pf.P2, P1 = d.pf.P1;
        const int64_t begin = R.b1[p], end = R.b1[p + 1];
        const Bin2 bin{d.pf};
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) cnt[q] = 0;
        __syncthreads();
        for (int64_t i = begin + threadIdx.x; i < end; i += kThreads)
            atomicAdd(&cnt[bin(__ldg(&R.l1[i].x))], 1u);
        __syncthreads();
        block_scan_excl(cnt, (int)P2, tmp);
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) {
            cursor[q] = begin + cnt[q];
            R.bounds[(int64_t)p * P2 + q] = begin + cnt[q];
        }
        if (threadIdx.x == 0 && p == P1 - 1) R.bounds[(int64_t)P1 * P2] = end;
        __syncthreads();
        scatter_tiles(AoSSrc{R.l1}, begin, end, bin, (int)P2, R.l2, end, cursor, cnt, tmp, stage,
                      &gwords[kGErrors]);
    }
}

// Bloom build: one CTA per finest partition of a Bloom-enabled join. The segment is built in shared
// memory with 32-bit atomicOr and written out whole (so the filter needs no clearing); segments too
// large for shared memory are built with global atomicOr.
__global__ void __launch_bounds__(kThreads)
k_bloom_build(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ bloom_prefix,
              int smem_words) {
    extern __shared__ uint32_t seg[];
    const int64_t total = bloom_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(bloom_prefix, nj, g);
        const JoinDesc& d = J[j];
        const int64_t f = g - bloom_prefix[j];
        const RelPlan& R = d.rel[0];
        const uint2* buf = final_buf(d, 0);
        const int64_t begin = R.bounds[f], end = R.bounds[f + 1];
        const uint32_t nw = d.seg_blocks * 8;
        uint32_t* gseg = d.bloom + f * (int64_t)nw;
        const int k = d.bloom_k;
        if ((int)nw <= smem_words) {
            for (uint32_t w = threadIdx.x; w < nw; w += kThreads) seg[w] = 0;
            __syncthreads();
            for (int64_t i = begin + threadIdx.x; i < end; i += kThreads) {
                BloomKey bk;
                bloom_key(__ldg(&buf[i].x), d.seg_blocks, k, bk);
                uint32_t* blk = seg + bk.block * 8;
#pragma unroll
                for (int w = 0; w < 8; ++w)
                    if (bk.mask[w]) atomicOr(blk + w, bk.mask[w]);
            }
            __syncthreads();
            for (uint32_t w = threadIdx.x; w < nw; w += kThreads) gseg[w] = seg[w];
            __syncthreads();
        } else {
            for (uint32_t w = threadIdx.x; w < nw; w += kThreads) gseg[w] = 0;
            __syncthreads();
            for (int64_t i = begin + threadIdx.x; i < end; i += kThreads) {
                BloomKey bk;
                bloom_key(__ldg(&buf[i].x), d.seg_blocks, k, bk);
                uint32_t* blk = gseg + (int64_t)bk.block * 8;
#pragma unroll
                for (int w = 0; w < 8; ++w)
                    if (bk.mask[w]) atomicOr(blk + w, bk.mask[w]);
            }
            __syncthreads();
        }
    }
}

// Probe tasks per finest partition. An R partition of at most table_cap tuples is built once per
// S chunk of s_chunk tuples; a larger one is cut into table_cap chunks, each probed by the whole S
// partition (the exact form of the reference's split path).
__device__ __forceinline__ void task_shape(int64_t nr, int64_t ns, int64_t T, int64_t C,
                                           int64_t& nrc, int64_t& nsc) {
    if (nr == 0 || ns == 0) { nrc = 0; nsc = 0; return; }
    nrc = (nr + T - 1) / T;
    nsc = nrc == 1 ? (ns + C - 1) / C : 1;
}

__global__ void k_tasks_count(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ fine_prefix,
                              uint32_t* __restrict__ tcount) {
    const int64_t total = fine_prefix[nj];
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= total;
         g += (int64_t)gridDim.x * blockDim.x) {
        if (g == total) { tcount[g] = 0; continue; }
        const int j = find_owner(fine_prefix, nj, g);
        const JoinDesc& d = J[j];
        const int64_t f = g - fine_prefix[j];
        const int64_t nr = d.rel[0].bounds[f + 1] - d.rel[0].bounds[f];
        const int64_t ns = d.rel[1].bounds[f + 1] - d.rel[1].bounds[f];
        int64_t nrc, nsc;
        task_shape(nr, ns, d.table_cap, d.s_chunk, nrc, nsc);
        tcount[g] = (uint32_t)(nrc * nsc);
    }
}

__global__ void k_tasks_write(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ fine_prefix,
                              const int64_t* __restrict__ toff, Task* __restrict__ tasks, int64_t task_cap,
                              unsigned long long* gwords) {
    const int64_t total = fine_prefix[nj];
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int j = find_owner(fine_prefix, nj, g);
        const JoinDesc& d = J[j];
        const int64_t f = g - fine_prefix[j];
        const int64_t r0 = d.rel[0].bounds[f], nr = d.rel[0].bounds[f + 1] - r0;
        const int64_t s0 = d.rel[1].bounds[f], ns = d.rel[1].bounds[f + 1] - s0;
        int64_t nrc, nsc;
        const int64_t T = d.table_cap, C = d.s_chunk;
        task_shape(nr, ns, T, C, nrc, nsc);
        const int64_t n = nrc * nsc;
        if (n == 0) continue;
        int64_t t = toff[g];
        if (t < 0 || t + n > task_cap) { atomicAdd(&gwords[kGErrors], 1ull); continue; }
        for (int64_t c = 0; c < n; ++c, ++t) {
            Task tk;
            tk.join = j;
            if (nrc == 1) {
                tk.r_begin = r0; tk.r_len = (uint32_t)nr;
                tk.s_begin = s0 + c * C; tk.s_len = (uint32_t)min_i64(C, ns - c * C);
                tk.split = 0;
            } else {
                tk.r_begin = r0 + c * T; tk.r_len = (uint32_t)min_i64(T, nr - c * T);
                tk.s_begin = s0; tk.s_len = (uint32_t)ns;
                tk.split = 1;
            }
            tasks[t] = tk;
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntTasks]), (unsigned long long)n);
        if (nrc > 1)
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSplitTasks]),
                      (unsigned long long)n);
    }
}

// Writes a warp's staged pairs to the join's output with one global atomic, respecting capacity.
__device__ __forceinline__ void warp_flush(const JoinDesc& d, const uint32_t* wr, const uint32_t* ws,
                                           const uint32_t* wk, int n, int lane) {
    __syncwarp();
    unsigned long long base = 0;
    if (lane == 0)
        base = atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntMatches]),
                         (unsigned long long)n);
    base = __shfl_sync(0xffffffffu, base, 0);
    const int64_t cap = d.cap;
    uint32_t* __restrict__ orr = d.out_r;
    uint32_t* __restrict__ oss = d.out_s;
    uint32_t* __restrict__ okk = d.out_k;
    for (int i = lane; i < n; i += 32) {
        const int64_t dst = (int64_t)base + i;
        if (dst < cap) {
            orr[dst] = wr[i];
            oss[dst] = ws[i];
            if (okk) okk[dst] = wk[i];
        }
    }
    __syncwarp();
}

// Persistent probe kernel. Each CTA repeatedly takes the next task, builds a bucketised table of
// the task's R chunk in shared memory (count per bucket, exclusive scan, place), then streams the
// S chunk: every S tuple scans its bucket and every key-equal entry is a match. After placement
// off[b] holds the end of bucket b, so bucket b spans [off[b-1], off[b]).
__global__ void __launch_bounds__(kThreads, 2)
k_probe(const JoinDesc* __restrict__ J, const Task* __restrict__ tasks, unsigned long long* gwords,
        int table_cap, int emit_key) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* table = reinterpret_cast<uint2*>(smem);                          // [table_cap]
    uint32_t* off = reinterpret_cast<uint32_t*>(table + table_cap);         // [table_cap] (+pad)
    uint32_t* wbuf = off + table_cap + 4;
    __shared__ uint32_t tmp[kThreads / 32];
    __shared__ long long s_task;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int words_per_warp = kWarpBuf * (emit_key ? 3 : 2);
    uint32_t* wr = wbuf + wid * words_per_warp;
    uint32_t* ws = wr + kWarpBuf;
    uint32_t* wk = ws + kWarpBuf;
    int wcount = 0;
    int cur = -1;
    const long long ntasks = (long long)gwords[kGTasks];
    for (;;) {
        if (threadIdx.x == 0) s_task = (long long)atomicAdd(&gwords[kGQueue], 1ull);
        __syncthreads();
        const long long t = s_task;
        if (t >= ntasks) break;
        const Task tk = tasks[t];
        if (tk.join != cur) {
            if (cur >= 0 && wcount > 0) warp_flush(J[cur], wr, ws, wk, wcount, lane);
            wcount = 0;
            cur = tk.join;
        }
        const JoinDesc& d = J[tk.join];
        const uint2* __restrict__ Rb = final_buf(d, 0) + tk.r_begin;
        const uint2* __restrict__ Sb = final_buf(d, 1) + tk.s_begin;
        const uint32_t nr = min(tk.r_len, (uint32_t)table_cap);
        if (tk.r_len > (uint32_t)table_cap && threadIdx.x == 0) atomicAdd(&gwords[kGErrors], 1ull);
        uint32_t nb = 32;
        while (nb < nr) nb <<= 1;
        const uint32_t mask = nb - 1;
        // build: count, scan, place
        for (uint32_t i = threadIdx.x; i < nb; i += kThreads) off[i] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nr; i += kThreads)
            atomicAdd(&off[bucket_of(__ldg(&Rb[i].x), mask)], 1u);
        __syncthreads();
        block_scan_excl(off, (int)nb, tmp);
        for (uint32_t i = threadIdx.x; i < nr; i += kThreads) {
            const uint2 e = __ldg(&Rb[i]);
            const uint32_t pos = atomicAdd(&off[bucket_of(e.x, mask)], 1u);
            table[pos] = e;
        }
        __syncthreads();
        // probe
        for (uint32_t base = 0; base < tk.s_len; base += kThreads) {
            const uint32_t i = base + threadIdx.x;
            uint2 e = make_uint2(0u, 0u);
            uint32_t lo = 0, hi = 0;
            if (i < tk.s_len) {
                e = __ldg(&Sb[i]);
                const uint32_t b = bucket_of(e.x, mask);
                lo = b ? off[b - 1] : 0u;
                hi = off[b];
            }
            while (__any_sync(0xffffffffu, lo < hi)) {
                bool m = false;
                uint32_t rv = 0;
                if (lo < hi) {
                    const uint2 c = table[lo];
                    m = (c.x == e.x);
                    rv = c.y;
                    ++lo;
                }
                const uint32_t mm = __ballot_sync(0xffffffffu, m);
                if (mm) {
                    const int n = __popc(mm);
                    if (wcount + n > kWarpBuf) {
                        warp_flush(d, wr, ws, wk, wcount, lane);
                        wcount = 0;
                    }
                    if (m) {
                        const int pos = wcount + __popc(mm & lanemask_lt());
                        wr[pos] = rv;
                        ws[pos] = e.y;
                        if (emit_key) wk[pos] = e.x;
                    }
                    wcount += n;
                    __syncwarp();
                }
            }
        }
        __syncthreads();
    }
    if (cur >= 0 && wcount > 0) warp_flush(J[cur], wr, ws, wk, wcount, lane);
}

// Copies each join's match count to the caller's device int64 (if requested).
__global__ void k_publish_counts(const JoinDesc* __restrict__ J, int nj) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        const JoinDesc& d = J[j];
        if (d.user_count) *d.user_count = d.counters[kCntMatches];
    }
}

// ---- device-wide exclusive scan (uint32 -> int64), three kernels -------------------------------
constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) k_scan_reduce(const uint32_t* __restrict__ in, int64_t n,
                                                          int64_t* __restrict__ sums) {
    __shared__ int64_t tmp[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile;
    int64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = t0 + (int64_t)k * kThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    int64_t total;
    block_scan_excl_i64(s, tmp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) k_scan_sums(int64_t* __restrict__ sums, int64_t nblk,
                                                        int64_t* __restrict__ grand) {
    __shared__ int64_t tmp[kThreads / 32];
    int64_t carry = 0;
    for (int64_t c0 = 0; c0 < nblk; c0 += kThreads) {
        const int64_t i = c0 + threadIdx.x;
        const int64_t v = i < nblk ? sums[i] : 0;
        int64_t total;
        const int64_t ex = block_scan_excl_i64(v, tmp, &total);
        if (i < nblk) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && grand) *grand = carry;
}

__global__ void __launch_bounds__(kThreads) k_scan_down(const uint32_t* __restrict__ in, int64_t n,
                                                        const int64_t* __restrict__ sums,
                                                        int64_t* __restrict__ out) {
    __shared__ int64_t tmp[kThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = t0 + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    int64_t total;
    int64_t run = block_scan_excl_i64(s, tmp, &total) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = t0 + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

__global__ void k_fill_word(unsigned long long* p, unsigned long long v) { *p = v; }

}  // namespace

// ---------------------------------------------------------------------------------------------
static thread_local int64_t g_launches = 0;
static thread_local bool g_capturing = false;
static thread_local int64_t g_capture_tally = 0;
void note_launches(int n) {
    if (g_capturing) g_capture_tally += n;
    else g_launches += n;
}
int64_t launches_so_far() { return g_launches; }
void set_capturing(bool on) {
    g_capturing = on;
    if (on) g_capture_tally = 0;
}
int64_t take_capture_tally() { return g_capture_tally; }

const char* stage_name(int i) {
    static const char* names[kNumStages] = {"r_hist", "r_scan", "r_scatter", "r_level2", "bloom_build",
                                            "s_hist_probe", "s_scan", "s_scatter", "s_level2", "tasks",
                                            "probe"};
    return (i >= 0 && i < kNumStages) ? names[i] : nullptr;
}

int64_t scan_tmp_words(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t enqueue_scan(const uint32_t* in, int64_t* out, int64_t n, int64_t* tmp, int64_t* total,
                         cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t nblk = (n + kScanTile - 1) / kScanTile;
    k_scan_reduce<<<(unsigned)nblk, kThreads, 0, st>>>(in, n, tmp);
    k_scan_sums<<<1, kThreads, 0, st>>>(tmp, nblk, total);
    k_scan_down<<<(unsigned)nblk, kThreads, 0, st>>>(in, n, tmp, out);
    note_launches(3);
    return cudaGetLastError();
}

size_t probe_smem_bytes(int table_cap, int emit_key) {
    return (size_t)table_cap * 8 + ((size_t)table_cap + 4) * 4 +
           (size_t)(kThreads / 32) * kWarpBuf * (emit_key ? 3 : 2) * 4;
}

static size_t l1_scatter_smem() { return (size_t)kTile * 8 + (size_t)kMaxP1 * 8 + (size_t)kMaxP1 * 4; }
static size_t l2_smem() { return (size_t)kTile * 8 + (size_t)kMaxP2 * 8 + (size_t)kMaxP2 * 4; }

static cudaError_t set_smem_attr(const void* fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static int grid_for(int64_t work, int num_sms, int per_sm) {
    int64_t g = std::min<int64_t>(work, (int64_t)num_sms * per_sm);
    return (int)std::max<int64_t>(g, 1);
}

cudaError_t enqueue_pipeline(const PipelineArgs& a, cudaStream_t st) {
    static thread_local bool attrs_done = false;
    cudaError_t err;
    if (!attrs_done) {
        if ((err = set_smem_attr((const void*)k_l1_scatter, l1_scatter_smem())) != cudaSuccess) return err;
        if ((err = set_smem_attr((const void*)k_l2_partition, l2_smem())) != cudaSuccess) return err;
        if ((err = set_smem_attr((const void*)k_bloom_build, 200 * 1024)) != cudaSuccess) return err;
        if ((err = set_smem_attr((const void*)k_probe, probe_smem_bytes(kMaxTable, 1))) != cudaSuccess)
            return err;
        attrs_done = true;
    }
    const int sms = a.num_sms;
    int launches = 0;
    auto mark = [&](int i) {
        if (a.stage_events) cudaEventRecord(a.stage_events[i], st);
    };
    mark(0);
    k_fill_word<<<1, 1, 0, st>>>(a.gwords + kGQueue, 0ull);
    k_fill_word<<<1, 1, 0, st>>>(a.gwords + kGErrors, 0ull);
    launches += 2;

    // ---- R: level 1 -------------------------------------------------------------------------
    for (int rel = 0; rel < 2; ++rel) {
        if (rel == 1 && a.any_bloom && a.total_bloom_fine > 0) {
            // Bloom filter over the final R partitions, before S's first pass probes it.
            const int smem_words = std::min(a.max_seg_words, 200 * 1024 / 4);
            k_bloom_build<<<grid_for(a.total_bloom_fine, sms, 4), kThreads,
                            (size_t)smem_words * 4, st>>>(a.J, a.nj, a.bloom_prefix, smem_words);
            ++launches;
        }
        if (rel == 1) mark(5);
        const int m0 = rel == 0 ? 1 : 6;  // first stage mark of this relation
        if (a.total_slices[rel] > 0) {
            k_l1_hist<<<grid_for(a.total_slices[rel], sms, 4), kThreads, (size_t)a.max_p1 * 4, st>>>(
                a.J, a.nj, rel, a.slice_prefix[rel], a.hist, a.gwords);
            ++launches;
        }
        mark(m0);
        if ((err = enqueue_scan(a.hist + a.hist_begin[rel], a.hist_scan + a.hist_begin[rel],
                                a.hist_len[rel], a.scan_tmp, nullptr, st)) != cudaSuccess)
            return err;
        mark(m0 + 1);
        if (a.total_slices[rel] > 0) {
            k_l1_scatter<<<grid_for(a.total_slices[rel], sms, 2), kThreads, l1_scatter_smem(), st>>>(
                a.J, a.nj, rel, a.slice_prefix[rel], a.hist_scan, a.gwords);
            ++launches;
        }
        mark(m0 + 2);
        {
            dim3 grid((unsigned)((a.max_p1 + 1 + 255) / 256), (unsigned)std::min(a.nj, 65535));
            k_bounds_l1<<<grid, 256, 0, st>>>(a.J, a.nj, rel, a.hist_scan);
            ++launches;
        }
        if (a.total_segs > 0) {
            k_l2_partition<<<grid_for(a.total_segs, sms, 2), kThreads, l2_smem(), st>>>(
                a.J, a.nj, rel, a.seg_prefix, a.gwords);
            ++launches;
        }
        mark(m0 + 3);
    }
    // ---- tasks --------------------------------------------------------------------------------
    {
        const int64_t n = a.total_fine + 1;
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8);
        k_tasks_count<<<blocks, 256, 0, st>>>(a.J, a.nj, a.fine_prefix, a.tcount);
        ++launches;
        if ((err = enqueue_scan(a.tcount, a.toff, n, a.scan_tmp,
                                reinterpret_cast<int64_t*>(a.gwords + kGTasks), st)) != cudaSuccess)
            return err;
        k_tasks_write<<<blocks, 256, 0, st>>>(a.J, a.nj, a.fine_prefix, a.toff, a.tasks, a.task_cap,
                                              a.gwords);
        ++launches;
    }
    mark(10);
    // ---- probe --------------------------------------------------------------------------------
    {
        const size_t smem = probe_smem_bytes(a.table_cap, a.emit_key);
        int occ = 0;
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_probe, kThreads, smem)) !=
            cudaSuccess)
            return err;
        occ = std::max(occ, 1);
        k_probe<<<sms * occ, kThreads, smem, st>>>(a.J, a.tasks, a.gwords, a.table_cap, a.emit_key);
        mark(11);
        k_publish_counts<<<1, 256, 0, st>>>(a.J, a.nj);
        launches += 2;
    }
    note_launches(launches);
    return cudaGetLastError();
}

}  // namespace brig
