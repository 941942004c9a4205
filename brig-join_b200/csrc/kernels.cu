// kernels.cu - the join pipeline for sm_100a.
//
// Stage map (reference kernel -> kernel here):
//   gpu_prefix_init + gpu_run_hist_for_both (src/kernel_functions.cu:22-90,141-159) -> k_l1_hist
//   queryAndCompactKernelPartitioned (src/bloom.cu:725-773), fused into S's histogram pass
//                                                                            -> k_l1_hist (Bloom)
//   gpu_make_simple_prefix (src/kernel_functions.cu:461-492)          -> k_scan_* (device-wide)
//   gpu_make_sorted_table_for_both (src/kernel_functions.cu:95-133)    -> k_l1_scatter
//   gpu_run_hist_second_pass + gpu_build_table_second_pass_kv (src/kernel_functions.cu:163-281)
//                                     -> k_l2_plan + k_l2_hist + k_l2_scatter + k_l2_bounds
//   queryAndCompactKernelPartitioned, alternatively as S's level-2 pass      -> k_l2_bloom
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
//   * Tiles are staged in shared memory and reordered by partition before they are written: up to
//     1024 partitions each partition's run of a tile goes out as one shared-to-global bulk copy
//     (its staging slots are placed so the run's source and destination share their 16-byte
//     alignment); above that consecutive threads store consecutive addresses of one run.
//   * The probe is a persistent work-queue kernel over (join, partition-pair) tasks. An R partition
//     larger than one shared-memory table is cut into table-sized chunks, each probed by the whole
//     S partition, so duplicates are exact (the reference's split path stops at the first match,
//     :371). A large S partition is cut into chunks that run as separate tasks. Buckets of
//     repeated build keys are walked by the whole warp, 32 entries per step.
//   * Matches are staged per warp in shared memory and written with one global atomic per flush
//     (the reference takes one global atomic per output pair, :420).
//   * The shared-memory table is bucketised (counting sort by bucket) rather than open addressing,
//     so every 32-bit key is valid (the reference reserves 0x80000000 as EMPTY, :352).
//   * Every computed store position is checked against its buffer; a failure increments an error
//     word the host reads instead of writing out of bounds.
#include <cstdio>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include "launch.h"

namespace brig {

namespace {

__device__ __forceinline__ int64_t min_i64(int64_t a, int64_t b) { return a < b ? a : b; }
__device__ __forceinline__ int64_t max_i64(int64_t a, int64_t b) { return a > b ? a : b; }

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
// blockDim.x must be NT; tmp holds NT/32 words.
template <int NT>
__device__ uint32_t block_scan_excl_n(uint32_t* a, int n, uint32_t* tmp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int kWarps = NT / 32;
    const int per = (n + NT - 1) / NT;
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
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t* a, int n, uint32_t* tmp) {
    return block_scan_excl_n<kThreads>(a, n, tmp);
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

// ---- TMA bulk copies (cp.async.bulk, no multicast) into shared memory ---------------------------
// A CTA double-buffers its input: while it processes tile t out of one buffer, the bulk-copy engine
// fills the other with tile t+1, so the load latency overlaps the shared-memory phases of the
// previous tile. Completion is tracked with one mbarrier per buffer (arrival count 1: the issuing
// thread's expect_tx). Every wait is bounded; a wait that runs out counts an error, waits once
// more (also bounded) and lets the kernel continue, so the host reports BRIG_E_INTERNAL instead of
// the GPU hanging.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Global -> shared bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// Asks the TMA unit to bring [p, p + bytes) into L2 (a hint; no data is returned). The range is
// shrunk to whole 16-byte units inside [lo, hi), so nothing outside the buffer is touched.
__device__ __forceinline__ void prefetch_l2_range(const void* lo, const void* hi) {
    const uintptr_t a = ((uintptr_t)lo + 15) & ~(uintptr_t)15, b = (uintptr_t)hi & ~(uintptr_t)15;
    if (b > a) {
        const uint32_t bytes = (uint32_t)min_i64((int64_t)(b - a), 1 << 20);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes) : "memory");
    }
}
// Orders this thread's earlier shared-memory accesses before later async-proxy (bulk copy) writes.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Shared -> global bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned), tracked
// in this thread's bulk async-group.
__device__ __forceinline__ void bulk_s2g(void* gdst, const void* ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until this thread's committed bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until this thread's committed bulk stores have completed their global writes.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Polls of the bounded waits. The first bound is a runtime value (the pipeline's state word
// kGWaitPolls, kDefaultPolls unless the caller's configuration sets it): when it runs out the wait
// counts an error, which the host reports as BRIG_E_INTERNAL, and then waits once more, at most
// kDefaultPolls polls, for the copy in flight, so that no copy is outstanding when the CTA moves on
// or exits. A first bound of 0 makes every wait count an error at once (the error path's test).
constexpr uint32_t kDefaultPolls = kDefaultWaitPolls;  // each poll may suspend for a bounded hardware interval
__device__ __forceinline__ void mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long* err,
                                          uint32_t polls) {
    for (uint32_t it = 0; it < polls; ++it)
        if (mbar_try_wait(bar, parity)) return;
    if (threadIdx.x == 0) atomicAdd(err, 1ull);
    for (uint32_t it = 0; it < kDefaultPolls; ++it)
        if (mbar_try_wait(bar, parity)) return;
}
__device__ __forceinline__ uint32_t wait_polls(const unsigned long long* gwords) {
    return (uint32_t)gwords[kGWaitPolls];
}

// Where the tuples of a tile come from. PackedTiles: (key, value) pairs in an engine buffer; a tile
// is copied from the 16-byte boundary at or below its first tuple (engine buffers are padded, so
// reading up to 8 bytes past either end stays inside the workspace). KvTiles<TILE>: the caller's
// separate key and value arrays, keys at the start of a tile buffer and values TILE * 4 bytes in;
// the 16-byte-aligned span of each array inside the tile is bulk-copied (the two arrays may be
// misaligned differently) and the up to 3 + 3 tuples at its edges are read with ordinary loads, so
// nothing outside the caller's arrays is read. mis(t0, tn) is the per-tile layout word, issue() is
// called by one thread and arms `bar` (with no bytes when nothing is copied), item() reads tuple i
// of the tile. fast(layout) says whether load_full() may read a whole tile of NITEMS tuples per
// thread straight from shared memory with 16-byte loads and no bounds tests (the tuples of thread
// x are its slots x, x + NT, ... of the load width; the scatter does not care which tuples a
// thread holds).
struct PackedTiles {
    const uint2* p;
    __device__ __forceinline__ uint32_t mis(int64_t t0, int = 0) const {
        return (((uintptr_t)(p + t0)) & 15) ? 1u : 0u;
    }
    __device__ __forceinline__ void issue(int64_t t0, int tn, unsigned char* buf, uint64_t* bar) const {
        fence_proxy_async();
        const uint32_t m = mis(t0);
        const uint32_t bytes = (((uint32_t)tn + m) * 8u + 15u) & ~15u;
        if (tn <= 0) {
            mbar_arrive(bar);
            return;
        }
        mbar_arrive_tx(bar, bytes);
        bulk_g2s(buf, p + t0 - m, bytes, bar);
    }
    using Layout = uint32_t;  // tuples before the first one in the buffer (0 or 1)
    __device__ __forceinline__ Layout layout(int64_t t0, int) const { return mis(t0); }
    __device__ __forceinline__ uint2 item(const unsigned char* buf, int64_t, int i, int, Layout m) const {
        return reinterpret_cast<const uint2*>(buf)[i + m];
    }
    __device__ __forceinline__ bool fast(Layout) const { return true; }
    template <int NITEMS, int NT>
    __device__ __forceinline__ void load_full(const unsigned char* buf, Layout m, uint2 (&it)[NITEMS]) const {
        const uint2* s = reinterpret_cast<const uint2*>(buf) + m;
#pragma unroll
        for (int j = 0; j < NITEMS; ++j) it[j] = s[j * NT + threadIdx.x];
    }
};

template <int TILE>
struct KvTiles {
    const uint32_t* k;
    const uint32_t* v;
    bool bulk;  // both arrays are 4-byte aligned (uint32 arrays always are, unless misused)
    static constexpr size_t kValOff = (size_t)TILE * 4;  // byte offset of the values in a tile buffer
    // Per tile: the 16-byte-aligned span of each array inside [t0, t0 + tn), packed as
    // hk | hv << 2 | nk << 4 | nv << 18 (h: first aligned offset from t0, n: aligned count).
    __device__ __forceinline__ static uint32_t span(const uint32_t* p, int64_t t0, int tn, uint32_t& n) {
        const uint32_t h = (4u - (uint32_t)(((uintptr_t)(p + t0) >> 2) & 3u)) & 3u;
        n = (int)h < tn ? (uint32_t)(tn - (int)h) & ~3u : 0u;
        return h;
    }
    __device__ __forceinline__ uint32_t mis(int64_t t0, int tn) const {
        if (!bulk) return 0u;
        uint32_t nk, nv;
        const uint32_t hk = span(k, t0, tn, nk), hv = span(v, t0, tn, nv);
        return hk | (hv << 2) | (nk << 4) | (nv << 18);
    }
    __device__ __forceinline__ void issue(int64_t t0, int tn, unsigned char* buf, uint64_t* bar) const {
        fence_proxy_async();
        const uint32_t m = mis(t0, tn);
        const uint32_t hk = m & 3u, hv = (m >> 2) & 3u, nk = (m >> 4) & 0x3fffu, nv = m >> 18;
        if (nk + nv == 0) {
            mbar_arrive(bar);
            return;
        }
        mbar_arrive_tx(bar, 4u * (nk + nv));
        if (nk) bulk_g2s(buf, k + t0 + hk, nk * 4u, bar);
        if (nv) bulk_g2s(buf + kValOff, v + t0 + hv, nv * 4u, bar);
    }
    // The tile layout word decoded once per tile.
    struct Layout {
        uint32_t hk, hv, nk, nv;
        bool whole;  // both spans cover the whole tile: every tuple from shared memory
    };
    __device__ __forceinline__ Layout layout(int64_t t0, int tn) const {
        const uint32_t m = mis(t0, tn);
        Layout l{m & 3u, (m >> 2) & 3u, (m >> 4) & 0x3fffu, m >> 18, false};
        l.whole = l.hk == 0 && l.hv == 0 && l.nk == (uint32_t)tn && l.nv == (uint32_t)tn;
        return l;
    }
    __device__ __forceinline__ uint2 item(const unsigned char* buf, int64_t t0, int i, int, const Layout& l) const {
        if (l.whole)  // tile-uniform
            return make_uint2(reinterpret_cast<const uint32_t*>(buf)[i],
                              reinterpret_cast<const uint32_t*>(buf + kValOff)[i]);
        const uint32_t ik = (uint32_t)i - l.hk, iv = (uint32_t)i - l.hv;  // wrap below the span
        const uint32_t key = ik < l.nk ? reinterpret_cast<const uint32_t*>(buf)[ik] : __ldcs(k + t0 + i);
        const uint32_t val = iv < l.nv ? reinterpret_cast<const uint32_t*>(buf + kValOff)[iv]
                                       : __ldcs(v + t0 + i);
        return make_uint2(key, val);
    }
    __device__ __forceinline__ bool fast(const Layout& l) const { return l.whole; }
    template <int NITEMS, int NT>
    __device__ __forceinline__ void load_full(const unsigned char* buf, const Layout&, uint2 (&it)[NITEMS]) const {
        static_assert(NITEMS % 4 == 0, "four tuples per 16-byte load");
        const uint4* ks = reinterpret_cast<const uint4*>(buf);
        const uint4* vs = reinterpret_cast<const uint4*>(buf + kValOff);
#pragma unroll
        for (int j = 0; j < NITEMS / 4; ++j) {
            const uint4 kk = ks[j * NT + threadIdx.x];
            const uint4 vv = vs[j * NT + threadIdx.x];
            it[4 * j] = make_uint2(kk.x, vv.x);
            it[4 * j + 1] = make_uint2(kk.y, vv.y);
            it[4 * j + 2] = make_uint2(kk.z, vv.z);
            it[4 * j + 3] = make_uint2(kk.w, vv.w);
        }
    }
};

template <int M>
struct Bin1 {
    PartFn f;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return part1_m<M>(f, key); }
};
template <int M>
struct Bin2 {
    PartFn f;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return part2_m<M>(f, key); }
};

// Tiles of the two scatter forms. The bulk-store form (up to kBulkMaxBins bins) takes 12288-tuple
// tiles, one third more than the write-pass form (whose staged-bin array and per-bin deltas leave
// room for 8192 at 4096 bins): longer runs per bin and tile, and the per-tile scan, barriers and
// run stores amortised over more tuples (level-1 scatter at 640M keys: 2.85 ms with 8192, 2.40 ms
// with 12288).
constexpr int kSTileW = 8192;    // write-pass form
constexpr int kSTileB = kSTile;  // bulk-store form
static_assert(kSTileB % (4 * kSThreads) == 0 && kSTileW % (4 * kSThreads) == 0, "whole 16-byte loads per thread");

// The three scatter forms a launch can take (ScatterForm). kFormBulkSmall is the bulk-store form in CTAs of 512
// threads with 6144-tuple tiles, two CTAs per SM: each CTA's barriers, scans and slice start-up
// overlap the other CTA's work, which pays where slices are short (a batch of small joins, the
// Bloom survivors of a level-2 slice) or bins few (long runs per tile even in half a tile); on long
// slices over many bins the full-size tile's longer runs win (640M keys, 512 bins: 2.40 ms for the
// level-1 scatter against 3.61 in the small form).
__host__ __device__ constexpr int form_threads(int f) { return f == kFormBulkSmall ? kSThreadsSmall : kSThreads; }
__host__ __device__ constexpr int form_tile(int f) {
    return f == kFormBulkSmall ? kSTile / 2 : (f == kFormBulk ? kSTileB : kSTileW);
}
__host__ __device__ constexpr int form_ctas_per_sm(int f) { return f == kFormBulkSmall ? 2 : 1; }
static_assert(form_tile(kFormBulkSmall) % (4 * kSThreadsSmall) == 0, "whole 16-byte loads per thread");
static_assert(kSTile % form_tile(kFormBulkSmall) == 0, "slices are whole small tiles");

// Scatters tuples [begin, end) of `in` into `out`. cursor[b] is the next output position of bin
// b; it advances as tiles are written. Each tile of kSTileW tuples arrives by bulk copy into one of
// the two input buffers while the previous tile is processed. Per tile every thread holds its
// kSTileW / kSThreads tuples in registers, takes a rank inside its tuple's bin with one
// shared-memory atomic, and after a scan of the bin counts writes the tuple to its bin-ordered
// position in `stage` (the tile's own input buffer, free once the tuples are in registers) with its
// bin in `sbin`. The write pass then stores consecutive staged positions from consecutive threads,
// i.e. runs of one bin to consecutive addresses; delta[b] = cursor[b] - (first staged position of b)
// turns a staged position into its output position with one add.
// `inbuf` holds two tile buffers, `bars` their mbarriers, `ph` the parity of each barrier.
constexpr size_t kTileBufW = (size_t)(kSTileW + 2) * 8;  // one write-pass input buffer

template <class In, class Bin>
__device__ void scatter_tiles(const In& in, int64_t begin, int64_t end, const Bin& bin, int nbins,
                              uint2* __restrict__ out, int64_t out_limit, int64_t* cursor, int64_t* delta,
                              uint32_t* cnt, uint16_t* sbin, uint32_t* tmp, unsigned char* inbuf, uint64_t* bars,
                              uint32_t& ph, unsigned long long* errors, uint32_t polls) {
    constexpr int kItems = kSTileW / kSThreads;
    const int64_t ntiles = (end - begin + kSTileW - 1) / kSTileW;
    if (ntiles <= 0) return;
    for (int x = threadIdx.x; x < nbins; x += kSThreads) cnt[x] = 0;
    if (threadIdx.x == 0) in.issue(begin, (int)min_i64(kSTileW, end - begin), inbuf, &bars[0]);
    for (int64_t t = 0; t < ntiles; ++t) {
        const int64_t t0 = begin + t * kSTileW;
        const int tn = (int)min_i64(kSTileW, end - t0);
        const int b = (int)(t & 1);
        mbar_wait(&bars[b], (ph >> b) & 1u, errors, polls);
        ph ^= 1u << b;
        // Every thread is past the previous tile's write pass, which read buffer b ^ 1 as `stage`
        // (and cnt is zero again): the next tile may now be copied into b ^ 1.
        __syncthreads();
        if (threadIdx.x == 0 && t + 1 < ntiles)
            in.issue(t0 + kSTileW, (int)min_i64(kSTileW, end - t0 - kSTileW), inbuf + (b ^ 1) * kTileBufW, &bars[b ^ 1]);
        unsigned char* buf = inbuf + b * kTileBufW;
        const auto lay = in.layout(t0, tn);
        const bool full = tn == kSTileW && in.fast(lay);  // block-uniform
        uint2 it[kItems];
        uint32_t br[kItems];  // bin << 16 | rank of the tuple within its bin in this tile
        if (full) {
            in.template load_full<kItems, kSThreads>(buf, lay, it);
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                const uint32_t bb = bin(it[k].x);
                br[k] = (bb << 16) | atomicAdd(&cnt[bb], 1u);
            }
        } else {
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                const int i = k * kSThreads + threadIdx.x;
                if (i < tn) {
                    it[k] = in.item(buf, t0, i, tn, lay);
                    const uint32_t bb = bin(it[k].x);
                    br[k] = (bb << 16) | atomicAdd(&cnt[bb], 1u);
                }
            }
        }
        __syncthreads();
        block_scan_excl_n<kSThreads>(cnt, nbins, tmp);  // cnt[b] = first staged position of bin b
        for (int x = threadIdx.x; x < nbins; x += kSThreads) {
            const uint32_t e0 = cnt[x];
            const uint32_t e1 = (x + 1 < nbins) ? cnt[x + 1] : (uint32_t)tn;
            const int64_t c = cursor[x];
            delta[x] = c - (int64_t)e0;
            cursor[x] = c + (int64_t)(e1 - e0);
        }
        uint2* stage = reinterpret_cast<uint2*>(buf);
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (full || k * kSThreads + (int)threadIdx.x < tn) {
                const uint32_t bb = br[k] >> 16;
                const uint32_t pos = cnt[bb] + (br[k] & 0xffffu);
                stage[pos] = it[k];
                sbin[pos] = (uint16_t)bb;
            }
        }
        __syncthreads();
        for (int x = threadIdx.x; x < nbins; x += kSThreads) cnt[x] = 0;  // for the next tile
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            const int i = k * kSThreads + threadIdx.x;
            if (i < tn) {
                const int64_t dst = delta[sbin[i]] + i;
                if ((uint64_t)dst < (uint64_t)out_limit) out[dst] = stage[i];
                else atomicAdd(errors, 1ull);
            }
        }
    }
    __syncthreads();  // the last write pass is done with the buffers, cursor and cnt
}

// The same scatter for at most kBulkMaxBins bins, with each bin's run of a tile written by the
// bulk-copy engine instead of a write pass over the tile. Thread x owns bin x. Per tile:
//   1. every thread takes its tuples from the tile buffer into registers and ranks them within
//      their bins (one shared-memory atomic each); a whole tile is read with 16-byte loads and no
//      bounds tests;
//   2. a scan of the bin counts gives each bin its staged start: bin b gets count + 1 slots, and
//      its run starts on the slot whose parity equals the parity of its output position, so the
//      run's source and destination are 16-byte aligned together;
//   3. every tuple is written to its staged slot (the tile's own buffer, free once the tuples are
//      in registers);
//   4. the owner of bin b stores the run [o, o + n) of b: a lone first tuple when o is odd and a
//      lone last tuple when the rest is odd, with plain 8-byte stores, and the pairs between them
//      with one shared -> global bulk copy.
// There is no pass that reads the staged tile back through the registers, so shared memory sees
// the staging stores and the bulk engine's reads only. The next tile's load goes into the other
// buffer once the bulk copies of the tile that used it have finished reading it (checked after
// step 1, by when they normally have).
static_assert(kBulkMaxBins <= kSThreads && kBulkSmallMaxBins <= kSThreadsSmall, "one bin per thread");
// A staging buffer of the bulk scatter: a tile of TILE tuples plus one slot per bin, a multiple of
// 16 bytes. The large form stages each tile in its own input buffer (two such buffers); the small
// form has one input buffer of a tile (plus the tuple before a misaligned start) and one staging
// buffer.
__host__ __device__ constexpr size_t bulk_tile_buf(int max_bins, int tile = kSTileB) {
    return (size_t)((tile + max_bins + 2 + 1) & ~1) * 8;
}
__host__ __device__ constexpr size_t bulk_in_buf(int tile) { return (size_t)(tile + 2) * 8; }
static_assert(bulk_in_buf(kSTile / 2) % 16 == 0, "the staging buffer after it starts on 16 bytes");

template <int F, class In, class Bin>
__device__ void scatter_tiles_bulk(const In& in, int64_t begin, int64_t end, const Bin& bin, int nbins,
                                   uint2* __restrict__ out, int64_t out_limit, int64_t* cursor, uint32_t* cnt,
                                   uint32_t* spos, uint32_t* tmp, unsigned char* inbuf, size_t buf_stride,
                                   uint64_t* bars, uint32_t& ph, unsigned long long* errors, uint32_t polls) {
    // kSplit: one input buffer and a separate staging buffer at inbuf + buf_stride (small form);
    // else two input buffers buf_stride apart, each tile staged in its own (large form).
    constexpr bool kSplit = F == kFormBulkSmall;
    constexpr int NT = form_threads(F), TILE = form_tile(F);
    constexpr int kItems = TILE / NT;
    constexpr int kWarps = NT / 32;
    const int64_t ntiles = (end - begin + TILE - 1) / TILE;
    if (ntiles <= 0) return;
    const int x = threadIdx.x, lane = x & 31, wid = x >> 5;
    const bool owner = x < nbins;
    if (owner) cnt[x] = 0;
    if (x == 0) in.issue(begin, (int)min_i64(TILE, end - begin), inbuf, &bars[0]);
    __syncthreads();  // cnt is zero
    for (int64_t t = 0; t < ntiles; ++t) {
        const int64_t t0 = begin + t * TILE;
        const int tn = (int)min_i64(TILE, end - t0);
        const int b = kSplit ? 0 : (int)(t & 1);
        mbar_wait(&bars[b], (ph >> b) & 1u, errors, polls);
        ph ^= 1u << b;
        unsigned char* buf = inbuf + b * buf_stride;
        uint2* stage = reinterpret_cast<uint2*>(kSplit ? inbuf + buf_stride : buf);
        const auto lay = in.layout(t0, tn);
        const bool full = tn == TILE && in.fast(lay);  // block-uniform
        uint2 it[kItems];
        uint32_t br[kItems];  // bin << 16 | rank of the tuple within its bin in this tile
        if (full) {
            in.template load_full<kItems, NT>(buf, lay, it);
        } else {
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                const int i = k * NT + x;
                if (i < tn) it[k] = in.item(buf, t0, i, tn, lay);
            }
        }
        if constexpr (kSplit) {
            // every thread holds its tuples: the input buffer takes the next tile, whose load then
            // overlaps this tile's ranking, scan, staging and stores
            __syncthreads();
            if (x == 0 && t + 1 < ntiles) in.issue(t0 + TILE, (int)min_i64(TILE, end - t0 - TILE), inbuf, &bars[0]);
        }
        if (full) {
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                const uint32_t bb = bin(it[k].x);
                br[k] = (bb << 16) | atomicAdd(&cnt[bb], 1u);
            }
        } else {
#pragma unroll
            for (int k = 0; k < kItems; ++k) {
                if (k * NT + x < tn) {
                    const uint32_t bb = bin(it[k].x);
                    br[k] = (bb << 16) | atomicAdd(&cnt[bb], 1u);
                }
            }
        }
        // this thread's bulk stores of the previous tile have read their staging slots (the other
        // input buffer, or the staging buffer)
        bulk_wait_read();
        __syncthreads();
        if (!kSplit && x == 0 && t + 1 < ntiles)
            in.issue(t0 + TILE, (int)min_i64(TILE, end - t0 - TILE), inbuf + (b ^ 1) * buf_stride, &bars[b ^ 1]);
        // exclusive scan of the counts, one bin per thread (every warp scans the warp totals itself);
        // cursor[x] is the next output position of bin x, spos[x] its staged start this tile
        const uint32_t n = owner ? cnt[x] : 0u;  // kept by the owner until it stores the run
        if (owner) cnt[x] = 0;  // for the next tile (its ranks may start before this tile's stores)
        uint32_t inc = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) tmp[wid] = inc;
        __syncthreads();
        uint32_t w = lane < kWarps ? tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        const uint32_t wbase = __shfl_sync(0xffffffffu, w, (wid + 31) & 31);
        const uint32_t e0 = inc - n + (wid > 0 ? wbase : 0u);
        uint32_t sx = 0;  // the owner's staged start, kept until it stores the run
        if (owner) {
            const uint32_t base = e0 + (uint32_t)x;                // bin x owns n + 1 slots
            sx = base + ((base ^ (uint32_t)cursor[x]) & 1u);       // same parity as its output
            spos[x] = sx;
        }
        __syncthreads();
        if (full) {
#pragma unroll
            for (int k = 0; k < kItems; ++k) stage[spos[br[k] >> 16] + (br[k] & 0xffffu)] = it[k];
        } else {
#pragma unroll
            for (int k = 0; k < kItems; ++k)
                if (k * NT + x < tn) stage[spos[br[k] >> 16] + (br[k] & 0xffffu)] = it[k];
        }
        fence_proxy_async();  // the staging stores before the bulk engine reads them
        __syncthreads();
        if (owner) {
            const uint32_t s = sx;
            const int64_t o = cursor[x];
            cursor[x] = o + n;
            if (n == 0) {
            } else if (o < 0 || o + (int64_t)n > out_limit) {
                atomicAdd(errors, 1ull);
            } else {
                const uint32_t h = (uint32_t)(o & 1);  // a lone first tuple
                const uint32_t m = n - h;
                const uint32_t pairs = m >> 1;
                const bool aligned = ((((uintptr_t)(out + o + h)) | (uintptr_t)smem_u32(stage + s + h)) & 15u) == 0;
                if (h) out[o] = stage[s];
                if (aligned) {
                    if (pairs) bulk_s2g(out + o + h, stage + s + h, pairs * 16u);
                } else {
                    for (uint32_t i = 0; i < 2 * pairs; ++i) out[o + h + i] = stage[s + h + i];
                }
                if (m & 1u) out[o + n - 1] = stage[s + n - 1];
            }
        }
        bulk_commit();
    }
    bulk_wait_read();
    __syncthreads();  // the bulk stores are done with the buffers; cnt is zero
}
static_assert(kSTileB + kBulkMaxBins + 2 < (1 << 16) && kSTileB < (1 << 16), "staged start and count in 16 bits");

// Shared-memory layout of the scatter kernels: two tile buffers, then cursor and delta (int64 per
// bin), the bin counts (uint32 per bin) and the staged bins (uint16 per tile position).
__device__ __forceinline__ void scatter_carve(unsigned char* smem, int max_bins, unsigned char*& inbuf,
                                              int64_t*& cursor, int64_t*& delta, uint32_t*& cnt,
                                              uint16_t*& sbin) {
    inbuf = smem;
    cursor = reinterpret_cast<int64_t*>(smem + 2 * kTileBufW);
    delta = cursor + max_bins;
    cnt = reinterpret_cast<uint32_t*>(delta + max_bins);
    sbin = reinterpret_cast<uint16_t*>(cnt + max_bins);
}

// Shared-memory layout of the bulk scatter: two tile buffers of bulk_tile_buf(max_bins) bytes, then
// the output cursors (int64 per bin), the bin counts and the staged starts (uint32 each).
__host__ __device__ constexpr size_t bulk_buf_stride(int form, int max_bins) {
    return form == kFormBulkSmall ? bulk_in_buf(kSTile / 2) : bulk_tile_buf(max_bins);
}
__host__ __device__ constexpr size_t bulk_bufs(int form, int max_bins) {
    return form == kFormBulkSmall ? bulk_in_buf(kSTile / 2) + bulk_tile_buf(max_bins, kSTile / 2)
                                  : 2 * bulk_tile_buf(max_bins);
}
__device__ __forceinline__ void bulk_carve(unsigned char* smem, int form, int max_bins, unsigned char*& inbuf,
                                           int64_t*& cursor, uint32_t*& cnt, uint32_t*& spos) {
    inbuf = smem;
    cursor = reinterpret_cast<int64_t*>(smem + bulk_bufs(form, max_bins));
    cnt = reinterpret_cast<uint32_t*>(cursor + max_bins);
    spos = cnt + max_bins;
}

__device__ __forceinline__ void init_bars(uint64_t* bars) {
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
}

// The mask class of a join (the K of the instantiation that handles it).
__device__ __forceinline__ int bloom_kclass(const JoinDesc& d) {
    return (d.bloom != nullptr && d.bloom_k == kBloomFastK) ? kBloomFastK : 0;
}
// Finest partition of a key with mix m (hash mode: the top b1 + b2 bits) or key (modulo mode).
template <int M>
__device__ __forceinline__ uint32_t fine_of(const PartFn& f, uint32_t key, uint32_t m) {
    if constexpr (M == 0) return top_bits(m, f.b1 + f.b2);
    else return fastmod(key, f.M1, f.P1) * f.P2 + fastmod(key, f.M2, f.P2);
}
constexpr int kProbeILP = 6;  // keys per thread with their filter words in flight together

// ---------------------------------------------------------------------------------------------
// Level 1, pass 1: per-slice histogram over P1 partitions (R, or S without Bloom), or the fused
// Bloom probe + survivor compaction + histogram (S with Bloom).
// hist layout per relation: [p * nslices + s], plus one trailing zero (sentinel) so that the
// exclusive scan of entry P1*nslices is the relation's total.
template <int M, int K>
__global__ void __launch_bounds__(kThreads, 2)
k_l1_hist(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ slice_prefix,
          uint32_t* __restrict__ hist, unsigned long long* gwords, int pat_k) {
    extern __shared__ uint32_t sh_cnt[];  // [max P1]
    __shared__ uint32_t s_cursor;
    __shared__ uint2 s_pat[pat_entries<K>()];  // pattern table (k != 7)
    if (K != kBloomFastK && rel == 1) fill_patterns(s_pat, pat_k);  // synchronised by the slice loop's first barrier
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
        if (pf.mode != M || bloom_kclass(d) != K) continue;  // another instantiation's join (block-uniform)
        const uint32_t P1 = pf.P1;
        for (uint32_t i = threadIdx.x; i < P1; i += kThreads) sh_cnt[i] = 0;
        if (threadIdx.x == 0) s_cursor = 0;
        __syncthreads();
        const bool bloom = (rel == 1) && d.bloom != nullptr && d.bloom_level == 1;
        if (!bloom) {
            const uint32_t* __restrict__ key = R.key;
            // the keys before the first 16-byte boundary (at most 3) one by one, then 16-byte loads
            const int64_t head = (((uintptr_t)key) & 3) ? (e - b)
                                 : min_i64(e - b, (4 - (int64_t)((((uintptr_t)(key + b)) >> 2) & 3)) & 3);
            if (head < e - b) {
                if ((int64_t)threadIdx.x < head) atomicAdd(&sh_cnt[part1_m<M>(pf, __ldcs(key + b + threadIdx.x))], 1u);
                const int64_t b4 = b + head;  // 16-byte aligned
                int64_t i = b4 + 4 * (int64_t)threadIdx.x;
                // four 16-byte loads in flight per thread
                for (; i + 12 * kThreads + 3 < e; i += 16 * kThreads) {
                    uint4 k4[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        k4[u] = __ldcs(reinterpret_cast<const uint4*>(key + i + 4 * u * kThreads));
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        atomicAdd(&sh_cnt[part1_m<M>(pf, k4[u].x)], 1u);
                        atomicAdd(&sh_cnt[part1_m<M>(pf, k4[u].y)], 1u);
                        atomicAdd(&sh_cnt[part1_m<M>(pf, k4[u].z)], 1u);
                        atomicAdd(&sh_cnt[part1_m<M>(pf, k4[u].w)], 1u);
                    }
                }
                for (; i + 3 < e; i += 4 * kThreads) {
                    const uint4 k4 = __ldcs(reinterpret_cast<const uint4*>(key + i));
                    atomicAdd(&sh_cnt[part1_m<M>(pf, k4.x)], 1u);
                    atomicAdd(&sh_cnt[part1_m<M>(pf, k4.y)], 1u);
                    atomicAdd(&sh_cnt[part1_m<M>(pf, k4.z)], 1u);
                    atomicAdd(&sh_cnt[part1_m<M>(pf, k4.w)], 1u);
                }
                // tail: at most 3 tuples past the last full vector
                const int64_t tail0 = b4 + ((e - b4) & ~(int64_t)3);
                for (int64_t t = tail0 + threadIdx.x; t < e; t += kThreads)
                    atomicAdd(&sh_cnt[part1_m<M>(pf, __ldcs(key + t))], 1u);
            } else {
                for (int64_t t = b + threadIdx.x; t < e; t += kThreads)
                    atomicAdd(&sh_cnt[part1_m<M>(pf, __ldcs(key + t))], 1u);
            }
        } else {
            // Bloom probe of every S key against the segment of its finest partition; survivors are
            // compacted (key, value) into R.cmp[b, b + count) and counted per level-1 partition.
            const uint32_t* __restrict__ key = R.key;
            const uint32_t* __restrict__ val = R.val;
            // descriptor fields in registers: the stores below could alias the descriptor, so
            // fields read through `d` inside the loop would be reloaded after every store
            const uint32_t seg_blocks = d.seg_blocks;
            const uint32_t* __restrict__ bloom = d.bloom;
            uint2* __restrict__ cmp = R.cmp;
            const int32_t len = (int32_t)(e - b);  // a slice is far below 2^31 tuples
            const uint32_t* __restrict__ skey = key + b;
            // each group loads the next group's keys before it reads its own filter words
            uint32_t kk[kProbeILP];
#pragma unroll
            for (int u = 0; u < kProbeILP; ++u) {
                const int32_t r = u * kThreads + (int32_t)threadIdx.x;
                kk[u] = r < len ? __ldcs(skey + r) : 0u;
            }
            for (int32_t r0 = 0; r0 < len; r0 += kProbeILP * kThreads) {
                uint32_t nk[kProbeILP];
                uint2 wv[kProbeILP], mk[kProbeILP];
#pragma unroll
                for (int u = 0; u < kProbeILP; ++u) {
                    const int32_t r = r0 + (kProbeILP + u) * kThreads + (int32_t)threadIdx.x;
                    nk[u] = r < len ? __ldcs(skey + r) : 0u;
                }
#pragma unroll
                for (int u = 0; u < kProbeILP; ++u) {
                    const int32_t r = r0 + u * kThreads + (int32_t)threadIdx.x;
                    const uint32_t m = mix32(kk[u]);
                    const BloomSlot sl = bloom_slot(m, fine_of<M>(pf, kk[u], m), seg_blocks);
                    wv[u] = make_uint2(0u, 0u);
                    if (r < len) wv[u] = __ldg(reinterpret_cast<const uint2*>(bloom + sl.widx));
                    mk[u] = slot_masks<K>(s_pat, sl);
                }
                uint32_t pm = 0;  // bit u: tuple u passed the filter
#pragma unroll
                for (int u = 0; u < kProbeILP; ++u) {
                    const int32_t r = r0 + u * kThreads + (int32_t)threadIdx.x;
                    if (r < len && bloom_pass(wv[u], mk[u])) pm |= 1u << u;
                }
                // survivors: one shared-memory atomic per warp for the whole group
                uint32_t bal[kProbeILP];
                uint32_t tot = 0;
#pragma unroll
                for (int u = 0; u < kProbeILP; ++u) {
                    bal[u] = __ballot_sync(0xffffffffu, (pm >> u) & 1u);
                    tot += __popc(bal[u]);
                }
                if (tot) {
                    uint32_t base = 0;
                    if (lane == 0) base = atomicAdd(&s_cursor, tot);
                    base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
                    for (int u = 0; u < kProbeILP; ++u) {
                        if ((pm >> u) & 1u) {
                            const int32_t r = r0 + u * kThreads + (int32_t)threadIdx.x;
                            atomicAdd(&sh_cnt[part1_m<M>(pf, kk[u])], 1u);
                            const int64_t dst = b + base + __popc(bal[u] & lanemask_lt());
                            if (dst < e) cmp[dst] = make_uint2(kk[u], __ldg(val + b + r));
                            else atomicAdd(&gwords[kGErrors], 1ull);
                        }
                        base += __popc(bal[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kProbeILP; ++u) kk[u] = nk[u];
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
            } else if (rel == 1 && d.bloom == nullptr) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSurvivors]),
                          (unsigned long long)(e - b));
            }
        }
        __syncthreads();
    }
}

// Level 1, pass 2: scatter each slice into its private runs. cursor[p] = scan[p][s] - scan[0][0]
// of this relation, i.e. the partition's start plus the counts of all earlier slices.
// kPacked selects the slices this launch handles: false = tuples from the caller's key/value arrays,
// true = S survivors of a level-1 Bloom probe, packed in cmp. One instantiation per input form keeps
// each kernel within 64 registers a thread. F is the scatter form (ScatterForm).
template <bool kPacked, int M, int F>
__global__ void __launch_bounds__(form_threads(F), form_ctas_per_sm(F))
k_l1_scatter(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ slice_prefix,
             const int64_t* __restrict__ scan, unsigned long long* gwords, int max_bins) {
    constexpr bool kBulk = F != kFormPass;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* inbuf;
    int64_t *cursor, *delta = nullptr;
    uint32_t *cnt, *spos = nullptr;
    uint16_t* sbin = nullptr;
    if constexpr (kBulk) bulk_carve(smem, F, max_bins, inbuf, cursor, cnt, spos);  // max_bins: at most the form's bins
    else scatter_carve(smem, max_bins, inbuf, cursor, delta, cnt, sbin);
    __shared__ uint32_t tmp[kSThreads / 32];
    __shared__ __align__(8) uint64_t bars[2];
    init_bars(bars);
    uint32_t ph = 0;
    const uint32_t polls = wait_polls(gwords);
    const int64_t total = slice_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(slice_prefix, nj, g);
        const JoinDesc& d = J[j];
        const RelPlan& R = d.rel[rel];
        const int s = (int)(g - slice_prefix[j]);
        const int64_t b = (int64_t)s * R.slice_len;
        const bool bloom = (rel == 1) && d.bloom != nullptr && d.bloom_level == 1;
        if (bloom != kPacked || d.pf.mode != M) continue;  // another instantiation's slice (block-uniform)
        const int64_t e = bloom ? b + R.slice_cnt[s] : min(b + R.slice_len, R.n);
        const uint32_t P1 = d.pf.P1;
        const int64_t* S = scan + R.hist_base;
        const int64_t s0 = S[0];
        for (uint32_t p = threadIdx.x; p < P1; p += form_threads(F))
            cursor[p] = S[(int64_t)p * R.nslices + s] - s0;
        __syncthreads();
        const Bin1<M> bin{d.pf};
        if constexpr (kPacked) {
            const PackedTiles in{R.cmp};
            if constexpr (kBulk)
                scatter_tiles_bulk<F>(in, b, e, bin, (int)P1, R.l1, R.n, cursor, cnt, spos, tmp, inbuf,
                                      bulk_buf_stride(F, max_bins), bars, ph, &gwords[kGErrors], polls);
            else
                scatter_tiles(in, b, e, bin, (int)P1, R.l1, R.n, cursor, delta, cnt, sbin, tmp, inbuf, bars, ph,
                              &gwords[kGErrors], polls);
        } else {
            const bool al = ((((uintptr_t)R.key) | ((uintptr_t)R.val)) & 3) == 0;
            if constexpr (kBulk) {
                const KvTiles<form_tile(F)> in{R.key, R.val, al};
                scatter_tiles_bulk<F>(in, b, e, bin, (int)P1, R.l1, R.n, cursor, cnt, spos, tmp, inbuf,
                                      bulk_buf_stride(F, max_bins), bars, ph, &gwords[kGErrors], polls);
            } else {
                const KvTiles<kSTileW> in{R.key, R.val, al};
                scatter_tiles(in, b, e, bin, (int)P1, R.l1, R.n, cursor, delta, cnt, sbin, tmp, inbuf, bars, ph,
                              &gwords[kGErrors], polls);
            }
        }
    }
    if constexpr (kBulk) bulk_wait_all();  // the bulk stores have written the output before the kernel ends
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

// ---- Level 2 ------------------------------------------------------------------------------------
// Every level-1 partition p is cut into slices of R.l2_slice tuples, planned on the device
// (k_l2_plan + a scan of the slice counts). Slices are handed to CTAs in (join, p, slice) order,
// so the CTAs running at any moment work on a few adjacent partitions: their output runs and, for
// a level-2 Bloom probe, their filter segments stay in L2. Per join the level-2 histogram is laid
// out [p][q][slice]; one exclusive scan of it gives every (p, q, slice) its output run, the same
// trick as level 1. Survivors of a level-2 Bloom probe are compacted per slice, so the level-2
// output is dense (survivors only) like the level-1 output.
// A global level-2 slice t decoded into its join, level-1 partition and slice within it.
struct L2Slice {
    int j;
    int64_t g;          // global segment index (seg_prefix[j] + p)
    uint32_t p;
    uint32_t ns;        // slices of this segment
    int64_t sl;         // slice within the segment
    int64_t local_off;  // slices of earlier segments of the same join
};

__device__ __forceinline__ L2Slice l2_decode(const int64_t* __restrict__ seg_prefix, int nj,
                                             const int64_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_ns,
                                             int64_t total_segs, int64_t t) {
    L2Slice x;
    // largest g with seg_off[g] <= t (seg_off is non-decreasing; empty segments have one slice)
    int64_t lo = 0, hi = total_segs;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (seg_off[mid] <= t) lo = mid; else hi = mid;
    }
    x.g = lo;
    x.j = find_owner(seg_prefix, nj, lo);
    x.p = (uint32_t)(lo - seg_prefix[x.j]);
    x.ns = seg_ns[lo];
    x.sl = t - seg_off[lo];
    x.local_off = seg_off[lo] - seg_off[seg_prefix[x.j]];
    return x;
}

// Slices per level-1 partition (at least one, so every partition owns a histogram region).
__global__ void k_l2_plan(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ seg_prefix,
                          uint32_t* __restrict__ seg_ns) {
    const int64_t total = seg_prefix[nj];
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= total; g += (int64_t)gridDim.x * blockDim.x) {
        if (g == total) { seg_ns[g] = 0; continue; }
        const int j = find_owner(seg_prefix, nj, g);
        const RelPlan& R = J[j].rel[rel];
        const int64_t p = g - seg_prefix[j];
        const int64_t len = R.b1[p + 1] - R.b1[p];
        seg_ns[g] = (uint32_t)max_i64(1, (len + R.l2_slice - 1) / R.l2_slice);
    }
}

// Level-2 histogram of one slice: counts by level-2 id. Handles every slice except those of S in
// joins that probe their filter at level 2 (k_l2_bloom does those).
template <int M>
__global__ void __launch_bounds__(kThreads, 2)
k_l2_hist(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ seg_prefix,
          const int64_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_ns, int64_t total_segs,
          uint32_t* __restrict__ hist2, unsigned long long* gwords) {
    extern __shared__ uint32_t cnt[];  // [max P2]
    const int64_t total = (int64_t)gwords[kGL2Slices + rel];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const L2Slice x = l2_decode(seg_prefix, nj, seg_off, seg_ns, total_segs, t);
        const JoinDesc& d = J[x.j];
        const RelPlan& R = d.rel[rel];
        const uint32_t P2 = d.pf.P2;
        const int64_t begin = R.b1[x.p] + x.sl * R.l2_slice;
        const int64_t end = min_i64(R.b1[x.p + 1], begin + R.l2_slice);
        const Bin2<M> bin{d.pf};
        const bool bloom = rel == 1 && d.bloom != nullptr && d.bloom_level == 2;
        if (bloom || d.pf.mode != M) continue;  // another kernel's slice (block-uniform)
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) cnt[q] = 0;
        __syncthreads();
        const uint2* __restrict__ l1 = R.l1;
        // each group of eight keys per thread loads the next group before it counts its own
        uint32_t kk[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t i = begin + threadIdx.x + u * kThreads;
            kk[u] = i < end ? __ldcs(&l1[i].x) : 0u;
        }
        for (int64_t i0 = begin + threadIdx.x; i0 < end; i0 += 8 * kThreads) {
            uint32_t nk[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int64_t i = i0 + (8 + u) * kThreads;
                nk[u] = i < end ? __ldcs(&l1[i].x) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (i0 + u * kThreads < end) atomicAdd(&cnt[bin(kk[u])], 1u);
#pragma unroll
            for (int u = 0; u < 8; ++u) kk[u] = nk[u];
        }
        __syncthreads();
        uint32_t* H = hist2 + R.h2_base + x.local_off * P2;
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) H[(int64_t)q * x.ns + x.sl] = cnt[q];
        __syncthreads();
    }
}

// Level-2 pass of S for joins that probe their filter at level 2: every key of the slice is tested
// against the filter segment of its finest partition, and the survivors are compacted into
// cmp[slice begin, + survivors) and counted by level-2 id. The filter segments of one level-1
// partition are contiguous (1.5 MB at 640M keys, 10 bits/key) and the slices of neighbouring
// partitions run together, so the filter words come from L2. One random filter read per key bounds
// the pass (the L1/texture pipeline looks up about one line per SM cycle), so the per-key work is
// kept to the minimum: one mix of the key from which its level-2 id, block, word pair (bloom_slot)
// and masks derive (compile-time shifts for k = 7, one 8-byte pattern look-up otherwise), one 8-byte
// filter load and a two-word test; full groups of U keys per thread run without bounds tests.
// Survivors are re-ranked per warp with one ballot per key and one shared atomic per warp group, and
// their level-2 ids recomputed (about one key in nine survives at 10% matches).
// Keys per thread with their filter words in flight. Each group also loads the next group's tuples
// before it reads its own filter words, so the stream's DRAM latency overlaps the filter reads (at
// 640M keys: 3.07 ms against 3.22 ms with six keys and no look-ahead).
constexpr int kL2BloomU = 4;

// One group of U keys per thread starting at slice offset r0; kTail: the group may end past len.
template <int M, int K, bool kTail>
__device__ __forceinline__ void l2_bloom_group(const uint2* __restrict__ src, int32_t r0, int32_t len,
                                               const uint32_t* __restrict__ bloom, uint32_t seg_blocks,
                                               uint32_t fine0, const PartFn& pf, const uint2* pat,
                                               uint2* __restrict__ cmp, uint32_t* cnt,
                                               uint32_t* s_surv, unsigned long long* errors, int lane,
                                               uint2 (&e)[kL2BloomU]) {
    constexpr int U = kL2BloomU;
    // the next group's tuples, loaded while this group's filter words are read
    uint2 ne[U];
    if constexpr (!kTail) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t r = r0 + (U + u) * kThreads + (int32_t)threadIdx.x;
            ne[u] = r < len ? __ldcs(src + r) : make_uint2(0u, 0u);
        }
    }
    uint2 wv[U], mk[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t r = r0 + u * kThreads + (int32_t)threadIdx.x;
        const uint32_t m = mix32(e[u].x);
        uint32_t q;
        if constexpr (M == 0) q = top_bits(m << pf.b1, pf.b2);
        else q = fastmod(e[u].x, pf.M2, pf.P2);
        const BloomSlot sl = bloom_slot(m, fine0 + q, seg_blocks);
        wv[u] = make_uint2(0u, 0u);
        if (!kTail || r < len) wv[u] = __ldg(reinterpret_cast<const uint2*>(bloom + sl.widx));
        mk[u] = slot_masks<K>(pat, sl);
    }
    uint32_t pm = 0;  // bit u: key u passed the filter
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int32_t r = r0 + u * kThreads + (int32_t)threadIdx.x;
        if ((!kTail || r < len) && bloom_pass(wv[u], mk[u])) pm |= 1u << u;
    }
    // survivors: one shared-memory atomic per warp for the whole group
    uint32_t bal[U];
    uint32_t tot = 0;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        bal[u] = __ballot_sync(0xffffffffu, (pm >> u) & 1u);
        tot += __popc(bal[u]);
    }
    if (tot) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(s_surv, tot);
        base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if ((pm >> u) & 1u) {
                atomicAdd(&cnt[part2_m<M>(pf, e[u].x)], 1u);
                const uint32_t dst = base + __popc(bal[u] & lanemask_lt());
                if ((int32_t)dst < len) cmp[dst] = e[u];
                else atomicAdd(errors, 1ull);
            }
            base += __popc(bal[u]);
        }
    }
    if constexpr (!kTail) {
#pragma unroll
        for (int u = 0; u < U; ++u) e[u] = ne[u];
    }
}

template <int M, int K>
__global__ void __launch_bounds__(kThreads, 2)
k_l2_bloom(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ seg_prefix,
           const int64_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_ns, int64_t total_segs,
           uint32_t* __restrict__ hist2, uint32_t* __restrict__ slice_cnt2, unsigned long long* gwords, int pat_k) {
    constexpr int U = kL2BloomU;
    extern __shared__ uint32_t cnt[];  // [max P2]
    __shared__ uint32_t s_surv;
    __shared__ uint2 s_pat[pat_entries<K>()];  // pattern table (k != 7)
    if (K != kBloomFastK) fill_patterns(s_pat, pat_k);  // synchronised by the slice loop's first barrier
    const int lane = threadIdx.x & 31;
    const int64_t total = (int64_t)gwords[kGL2Slices + 1];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const L2Slice x = l2_decode(seg_prefix, nj, seg_off, seg_ns, total_segs, t);
        const JoinDesc& d = J[x.j];
        if (d.bloom == nullptr || d.bloom_level != 2 || d.pf.mode != M || bloom_kclass(d) != K)
            continue;  // another kernel's slice (block-uniform)
        const RelPlan& R = d.rel[1];
        const PartFn pf = d.pf;
        const uint32_t P2 = pf.P2;
        const int64_t begin = R.b1[x.p] + x.sl * R.l2_slice;
        const int64_t end = min_i64(R.b1[x.p + 1], begin + R.l2_slice);
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) cnt[q] = 0;
        if (threadIdx.x == 0) s_surv = 0;
        __syncthreads();
        // descriptor fields in registers: the stores below could alias the descriptor
        const uint32_t seg_blocks = d.seg_blocks;
        const uint32_t* __restrict__ bloom = d.bloom;
        uint2* __restrict__ cmp = R.cmp + begin;
        const uint2* __restrict__ src = R.l1 + begin;
        const int32_t len = (int32_t)(end - begin);  // at most one level-2 slice
        const int32_t full = len - len % (U * kThreads);
        const uint32_t fine0 = x.p * P2;
        int32_t r0 = 0;
        uint2 e[U];  // the tuples of the group in hand; each group loads the next one's
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int32_t r = u * kThreads + (int32_t)threadIdx.x;
            e[u] = r < len ? __ldcs(src + r) : make_uint2(0u, 0u);
        }
        for (; r0 < full; r0 += U * kThreads)
            l2_bloom_group<M, K, false>(src, r0, len, bloom, seg_blocks, fine0, pf, s_pat, cmp, cnt,
                                     &s_surv, &gwords[kGErrors], lane, e);
        if (r0 < len)
            l2_bloom_group<M, K, true>(src, r0, len, bloom, seg_blocks, fine0, pf, s_pat, cmp, cnt,
                                    &s_surv, &gwords[kGErrors], lane, e);
        __syncthreads();
        uint32_t* H = hist2 + R.h2_base + x.local_off * P2;
        for (uint32_t q = threadIdx.x; q < P2; q += kThreads) H[(int64_t)q * x.ns + x.sl] = cnt[q];
        if (threadIdx.x == 0) {
            slice_cnt2[t] = s_surv;
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSurvivors]), (unsigned long long)s_surv);
        }
        __syncthreads();
    }
}

// Level-2 scatter of one slice into its private runs of the level-2 buffer (F: the scatter form).
template <int M, int F>
__global__ void __launch_bounds__(form_threads(F), form_ctas_per_sm(F))
k_l2_scatter(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ seg_prefix,
             const int64_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_ns, int64_t total_segs,
             const int64_t* __restrict__ scan2, const uint32_t* __restrict__ slice_cnt2, unsigned long long* gwords,
             int max_bins) {
    constexpr bool kBulk = F != kFormPass;
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* inbuf;
    int64_t *cursor, *delta = nullptr;
    uint32_t *cnt, *spos = nullptr;
    uint16_t* sbin = nullptr;
    if constexpr (kBulk) bulk_carve(smem, F, max_bins, inbuf, cursor, cnt, spos);  // max_bins: at most the form's bins
    else scatter_carve(smem, max_bins, inbuf, cursor, delta, cnt, sbin);
    __shared__ uint32_t tmp[kSThreads / 32];
    __shared__ __align__(8) uint64_t bars[2];
    init_bars(bars);
    uint32_t ph = 0;
    const uint32_t polls = wait_polls(gwords);
    const int64_t total = (int64_t)gwords[kGL2Slices + rel];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const L2Slice x = l2_decode(seg_prefix, nj, seg_off, seg_ns, total_segs, t);
        const JoinDesc& d = J[x.j];
        if (d.pf.mode != M) continue;  // the other instantiation's join (block-uniform)
        const RelPlan& R = d.rel[rel];
        const uint32_t P2 = d.pf.P2;
        const int64_t begin = R.b1[x.p] + x.sl * R.l2_slice;
        const bool bloom = rel == 1 && d.bloom != nullptr && d.bloom_level == 2;
        const int64_t end = bloom ? begin + slice_cnt2[t] : min_i64(R.b1[x.p + 1], begin + R.l2_slice);
        const int64_t* S2 = scan2 + R.h2_base;
        const int64_t s0 = S2[0];
        const int64_t* Sx = S2 + x.local_off * P2;
        for (uint32_t q = threadIdx.x; q < P2; q += form_threads(F)) cursor[q] = Sx[(int64_t)q * x.ns + x.sl] - s0;
        __syncthreads();
        const PackedTiles in{bloom ? R.cmp : R.l1};
        if constexpr (kBulk)
            scatter_tiles_bulk<F>(in, begin, end, Bin2<M>{d.pf}, (int)P2, R.l2, R.n, cursor, cnt, spos, tmp, inbuf,
                                  bulk_buf_stride(F, max_bins), bars, ph, &gwords[kGErrors], polls);
        else
            scatter_tiles(in, begin, end, Bin2<M>{d.pf}, (int)P2, R.l2, R.n, cursor, delta, cnt, sbin, tmp, inbuf,
                          bars, ph, &gwords[kGErrors], polls);
    }
    if constexpr (kBulk) bulk_wait_all();  // the bulk stores have written the output before the kernel ends
}

// Finest-partition starts from the level-2 scan: bounds[p*P2+q] = start of (p, q); bounds[P1*P2] =
// the relation's level-2 total. One grid row per join.
__global__ void k_l2_bounds(const JoinDesc* __restrict__ J, int nj, int rel, const int64_t* __restrict__ seg_prefix,
                            const int64_t* __restrict__ seg_off, const uint32_t* __restrict__ seg_ns,
                            const int64_t* __restrict__ scan2) {
    for (int j = blockIdx.y; j < nj; j += gridDim.y) {
        const JoinDesc& d = J[j];
        if (d.pf.P2 <= 1) continue;
        const RelPlan& R = d.rel[rel];
        const int64_t P2 = d.pf.P2, nf = (int64_t)d.pf.P1 * P2;
        const int64_t* S2 = scan2 + R.h2_base;
        const int64_t s0 = S2[0];
        const int64_t g0 = seg_prefix[j];
        for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f <= nf; f += (int64_t)gridDim.x * blockDim.x) {
            if (f == nf) {
                const int64_t local_total = seg_off[seg_prefix[j + 1]] - seg_off[g0];
                R.bounds[f] = S2[local_total * P2] - s0;
                continue;
            }
            const int64_t g = g0 + f / P2, q = f % P2;
            R.bounds[f] = S2[(seg_off[g] - seg_off[g0]) * P2 + q * (int64_t)seg_ns[g]] - s0;
        }
    }
}

// Bloom build: one CTA per group of G consecutive finest partitions of a Bloom-enabled join
// (G = JoinDesc::bloom_group, chosen so the group's segments fit in shared memory). The group's R
// tuples are contiguous in the final R buffer; every key sets its bits in its two words with two
// 32-bit atomicOr in the shared-memory copy of its segment, and the segments are written out
// whole, so the filter needs no clearing. A segment too large for shared memory (G = 1 then) is
// built with global atomicOr. The kernel is bound by the integer ALU pipe: per key one mix, the
// slot arithmetic of bloom_slot on the group-relative segment index, one pattern look-up and the two
// atomics, with 32-bit indices and no bounds tests in full groups.
template <int M, int K, bool kTail>
__device__ __forceinline__ void bloom_build_group(const uint2* __restrict__ buf, int32_t i0, int32_t n,
                                                  uint32_t* dst, uint32_t f0, uint32_t nf, const PartFn& pf,
                                                  uint32_t seg_blocks, const uint2* pat, unsigned long long* errors) {
    uint32_t kk[kProbeILP];
#pragma unroll
    for (int u = 0; u < kProbeILP; ++u) {
        const int32_t i = i0 + u * kThreads + (int32_t)threadIdx.x;
        kk[u] = (!kTail || i < n) ? __ldcs(&buf[i].x) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kProbeILP; ++u) {
        const int32_t i = i0 + u * kThreads + (int32_t)threadIdx.x;
        if (kTail && i >= n) continue;
        const uint32_t m = mix32(kk[u]);
        const uint32_t local = fine_of<M>(pf, kk[u], m) - f0;
        if (local >= nf) {  // a key outside the group's partitions: a partitioning fault
            atomicAdd(errors, 1ull);
            continue;
        }
        const BloomSlot sl = bloom_slot(m, local, seg_blocks);  // word index relative to the group
        const uint2 mk = slot_masks<K>(pat, sl);
        atomicOr(dst + sl.widx, mk.x);
        if (mk.y) atomicOr(dst + sl.widx + 1, mk.y);
    }
}

template <int M, int K>
__global__ void __launch_bounds__(kThreads)
k_bloom_build(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ bloom_prefix,
              int smem_words, unsigned long long* gwords, int pat_k) {
    extern __shared__ __align__(16) uint32_t seg[];
    __shared__ uint2 s_pat[pat_entries<K>()];  // pattern table (k != 7)
    if (K != kBloomFastK) fill_patterns(s_pat, pat_k);  // synchronised by the group loop's first barrier
    unsigned long long* errors = &gwords[kGErrors];
    const int64_t total = bloom_prefix[nj];
    for (int64_t g = blockIdx.x; g < total; g += gridDim.x) {
        const int j = find_owner(bloom_prefix, nj, g);
        const JoinDesc& d = J[j];
        if (d.pf.mode != M || bloom_kclass(d) != K) continue;  // another instantiation's join (block-uniform)
        const RelPlan& R = d.rel[0];
        const int64_t nfine = (int64_t)d.pf.P1 * d.pf.P2;
        const int64_t f0 = (g - bloom_prefix[j]) * d.bloom_group;
        const int64_t f1 = min_i64(f0 + d.bloom_group, nfine);
        const int64_t begin = R.bounds[f0], end = R.bounds[f1];
        const uint2* __restrict__ buf = final_buf(d, 0) + begin;
        const uint32_t nw = d.seg_blocks * 8;
        const int64_t words = (f1 - f0) * (int64_t)nw;
        uint32_t* gseg = d.bloom + f0 * (int64_t)nw;
        // descriptor fields in registers: the atomics below may write global memory (segments too
        // large for shared memory), so fields read through `d` would be reloaded after each one
        const PartFn pf = d.pf;
        const uint32_t seg_blocks = d.seg_blocks;
        const uint32_t nf = (uint32_t)(f1 - f0);
        const int32_t n = (int32_t)(end - begin);  // the group's R tuples
        const bool in_smem = words <= smem_words;
        uint32_t* dst = in_smem ? seg : gseg;
        for (int64_t w = threadIdx.x; w < words; w += kThreads) dst[w] = 0;
        __syncthreads();
        constexpr int32_t kStep = kProbeILP * kThreads;
        const int32_t full = n - n % kStep;
        if (threadIdx.x == 0) prefetch_l2_range(buf, buf + min_i64(n, 2 * kStep));
        int32_t i0 = 0;
        if (in_smem) {
            for (; i0 < full; i0 += kStep) {
                if (threadIdx.x == 0 && i0 + 2 * kStep < n)
                    prefetch_l2_range(buf + i0 + 2 * kStep, buf + min_i64(n, (int64_t)i0 + 3 * kStep));
                bloom_build_group<M, K, false>(buf, i0, n, seg, (uint32_t)f0, nf, pf, seg_blocks, s_pat, errors);
            }
            if (i0 < n)
                bloom_build_group<M, K, true>(buf, i0, n, seg, (uint32_t)f0, nf, pf, seg_blocks, s_pat, errors);
        } else {
            for (; i0 < n; i0 += kStep)
                bloom_build_group<M, K, true>(buf, i0, n, gseg, (uint32_t)f0, nf, pf, seg_blocks, s_pat, errors);
        }
        __syncthreads();
        if (in_smem) {
            for (int64_t w = threadIdx.x; w < words; w += kThreads) gseg[w] = seg[w];
            __syncthreads();
        }
    }
}

// Probe tasks. A task domain is one level-1 partition (two-level plans) or the whole join
// (one-level plans); inside a domain the finest partitions of each side are adjacent in memory.
// The smaller side of the domain is the build side. Consecutive finest partitions are grouped into
// one task until their build sides would exceed table_cap tuples: keys of different partitions
// never match, so one table over the group is exact, and fewer, larger tasks amortise the per-task
// table set-up. A group's streamed side is cut into chunks of s_chunk tuples, each a task of its
// own (a hot partition spreads over many CTAs). A single partition whose build side exceeds
// table_cap is cut into table_cap chunks, each streamed against the partition's whole other side:
// the exact form of the reference's split path, which stops at the first match
// (src/kernel_functions.cu:356-395).
__device__ __forceinline__ void fine_range(const RelPlan& R, int64_t f, int64_t& begin, int64_t& n) {
    begin = R.bounds[f];
    n = R.bounds[f + 1] - begin;
}

// Walks domain `dom` of join d with one warp and calls emit(b_begin, b_len, p_begin, p_len, split,
// build_s) for every task, in order, on every lane (the grouping state is warp-uniform). Lanes load
// 32 partitions' bounds at a time; the greedy grouping then steps through them with shuffles.
template <class Emit>
__device__ void walk_domain(const JoinDesc& d, int64_t dom, Emit&& emit) {
    const int lane = threadIdx.x & 31;
    const int64_t P2 = d.pf.P2;
    const int64_t f_first = P2 > 1 ? dom * P2 : 0;
    const int64_t f_last = P2 > 1 ? f_first + P2 : (int64_t)d.pf.P1;
    int64_t tot_r = 0, tot_s = 0;
    for (int64_t f = f_first + lane; f < f_last; f += 32) {
        int64_t b, n;
        fine_range(d.rel[0], f, b, n);
        tot_r += n;
        fine_range(d.rel[1], f, b, n);
        tot_s += n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tot_r += __shfl_xor_sync(0xffffffffu, tot_r, o);
        tot_s += __shfl_xor_sync(0xffffffffu, tot_s, o);
    }
    if (tot_r == 0 || tot_s == 0) return;
    const bool bs = tot_s < tot_r;
    const RelPlan& B = d.rel[bs ? 1 : 0];
    const RelPlan& P = d.rel[bs ? 0 : 1];
    const int64_t T = d.table_cap, C = d.s_chunk;
    int64_t gb0 = -1, gp0 = -1, nb = 0, np = 0;
    auto close = [&]() {
        if (nb > 0 && np > 0)
            for (int64_t c = 0; c * C < np; ++c) emit(gb0, nb, gp0 + c * C, min_i64(C, np - c * C), false, bs);
        gb0 = -1;
        nb = 0;
        np = 0;
    };
    for (int64_t f0 = f_first; f0 < f_last; f0 += 32) {
        int64_t mb = 0, mbn = 0, mp = 0, mpn = 0;
        if (f0 + lane < f_last) {
            fine_range(B, f0 + lane, mb, mbn);
            fine_range(P, f0 + lane, mp, mpn);
        }
        const int cnt = (int)min_i64(32, f_last - f0);
        for (int l = 0; l < cnt; ++l) {
            const int64_t bb = __shfl_sync(0xffffffffu, mb, l), bn = __shfl_sync(0xffffffffu, mbn, l);
            const int64_t pb = __shfl_sync(0xffffffffu, mp, l), pn = __shfl_sync(0xffffffffu, mpn, l);
            if (bn > T) {
                close();
                if (pn > 0)
                    for (int64_t c = 0; c * T < bn; ++c) emit(bb + c * T, min_i64(T, bn - c * T), pb, pn, true, bs);
                continue;
            }
            if (nb + bn > T) close();
            if (gb0 < 0) {
                gb0 = bb;
                gp0 = pb;
            }
            nb += bn;
            np += pn;
        }
    }
    close();
}

constexpr int kTaskWarps = 8;  // warps (domains) per task-builder CTA

__global__ void __launch_bounds__(kTaskWarps * 32)
k_tasks_count(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ dom_prefix,
              uint32_t* __restrict__ tcount) {
    const int64_t total = dom_prefix[nj];
    const int64_t warp0 = (int64_t)blockIdx.x * kTaskWarps + (threadIdx.x >> 5);
    for (int64_t g = warp0; g <= total; g += (int64_t)gridDim.x * kTaskWarps) {
        if (g == total) {
            if ((threadIdx.x & 31) == 0) tcount[g] = 0;
            continue;
        }
        const int j = find_owner(dom_prefix, nj, g);
        uint32_t n = 0;
        walk_domain(J[j], g - dom_prefix[j], [&](int64_t, int64_t, int64_t, int64_t, bool, bool) { ++n; });
        if ((threadIdx.x & 31) == 0) tcount[g] = n;
    }
}

__global__ void __launch_bounds__(kTaskWarps * 32)
k_tasks_write(const JoinDesc* __restrict__ J, int nj, const int64_t* __restrict__ dom_prefix,
              const int64_t* __restrict__ toff, Task* __restrict__ tasks, int64_t task_cap,
              unsigned long long* gwords) {
    const int64_t total = dom_prefix[nj];
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (int64_t)blockIdx.x * kTaskWarps + (threadIdx.x >> 5);
    for (int64_t g = warp0; g < total; g += (int64_t)gridDim.x * kTaskWarps) {
        const int j = find_owner(dom_prefix, nj, g);
        const JoinDesc& d = J[j];
        int64_t t = toff[g];
        int64_t n = 0, nsplit = 0;
        walk_domain(d, g - dom_prefix[j], [&](int64_t b0, int64_t bn, int64_t p0, int64_t pn, bool split, bool bs) {
            if (lane == 0) {
                if (t < 0 || t >= task_cap) {
                    atomicAdd(&gwords[kGErrors], 1ull);
                } else {
                    Task tk;
                    tk.join = j;
                    tk.flags = (bs ? kTaskBuildS : 0u) | (split ? kTaskSplit : 0u);
                    tk.b_begin = b0;
                    tk.b_len = (uint32_t)bn;
                    tk.p_begin = p0;
                    tk.p_len = (uint32_t)pn;
                    tasks[t] = tk;
                }
            }
            ++t;
            ++n;
            nsplit += split ? 1 : 0;
        });
        if (lane == 0) {
            if (n) atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntTasks]), (unsigned long long)n);
            if (nsplit)
                atomicAdd(reinterpret_cast<unsigned long long*>(&d.counters[kCntSplitTasks]),
                          (unsigned long long)nsplit);
        }
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

// Exclusive scan of the bucket directory off[0, nb) for nb = PER * kThreads (PER a multiple of 4):
// each thread scans PER consecutive entries with 16-byte
// shared-memory accesses. off[nb] is set to the total.
template <int PER>
__device__ __forceinline__ void scan_dir(uint32_t* off, uint32_t nb, uint32_t* tmp) {
    static_assert(PER % 4 == 0, "16-byte accesses");
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int kWarps = kThreads / 32;
    uint4 v[PER / 4];
    uint4* p = reinterpret_cast<uint4*>(off + threadIdx.x * PER);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < PER / 4; ++k) {
        v[k] = p[k];
        sum += v[k].x + v[k].y + v[k].z + v[k].w;
    }
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[wid] = x;
    __syncthreads();
    uint32_t w = lane < kWarps ? tmp[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, w, kWarps - 1);
    uint32_t run = x - sum + (wid > 0 ? __shfl_sync(0xffffffffu, w, wid - 1) : 0u);
#pragma unroll
    for (int k = 0; k < PER / 4; ++k) {
        uint4 o4;
        o4.x = run; run += v[k].x;
        o4.y = run; run += v[k].y;
        o4.z = run; run += v[k].z;
        o4.w = run; run += v[k].w;
        p[k] = o4;
    }
    if (threadIdx.x == 0) off[nb] = total;
    __syncthreads();
}

// Persistent probe kernel, two CTAs per SM. Each CTA takes tasks from the global queue (the next
// task index is fetched while the current task runs). Per task the CTA
//   * loads the build chunk (at most table_cap tuples) once, into registers, kBuildPer per thread,
//     counts it per bucket with one shared-memory atomic per tuple (the atomic's result is the
//     tuple's rank in its bucket), scans the counts into bucket starts (off[nb] = the chunk size)
//     and places every tuple at off[bucket] + rank: a bucketised table with at least as many
//     buckets as tuples, bucket b = [off[b], off[b+1]). Every build key also sets one bit of a
//     262144-bit presence bitmap;
//   * streams the other side from global memory with kProbeU coalesced tuples per thread in flight
//     (its first two iterations are prefetched into L2 while the table is built, and later the
//     range two iterations ahead). A streamed tuple whose bitmap bit is clear cannot match (at
//     most 4096 keys set at most 1.6% of the bits); the others are compacted with ballot/popc into
//     the warp's candidate queue in shared memory. Every 32 queued candidates the warp scans their
//     buckets in lock step, one candidate per lane, and compacts matches into the warp's output
//     staging buffer, which is written out with one global atomic per flush. So the bucket scans,
//     whose cost is the longest bucket among the lanes, run only on full warps of likely matches.
// The bitmap index is a multiplicative hash of the key, independent of the partition bits (the
// keys of one task share the top bits of mix32) and of the bucket bits.
constexpr int kProbeU = 4;                        // streamed tuples per thread in flight
constexpr int kBuildPer = kMaxTable / kThreads;   // build tuples per thread
// 262144-bit presence bitmap: 1.6% false candidates at 4096 keys, against 3% at 131072 bits and 6%
// at 65536 (probe at 640M x 640M: 2.02, 2.10 and 2.22 ms). Its 16 KB more shared memory come from the
// buffer that held the first 2048 streamed tuples of a task, which the L2 prefetch replaces.
constexpr int kBitmapWords = 8192;
constexpr int kQueue = 64;                        // candidates queued per warp

__device__ __forceinline__ uint32_t presence_bit(uint32_t key) { return (key * 0x9E3779B1u) >> 14; }

// Output staging of one warp: the pairs found so far for join `d`.
struct WarpOut {
    uint32_t* wr;
    uint32_t* ws;
    uint32_t* wk;
    int count;
};

// Stages one match per lane with m set (warp-wide; flushes first when the staging buffer is full).
__device__ __forceinline__ void stage_matches(const JoinDesc& d, bool m, uint32_t r_val, uint32_t s_val,
                                              uint32_t key, int emit_key, int lane, WarpOut& o) {
    const uint32_t mm = __ballot_sync(0xffffffffu, m);
    if (!mm) return;
    const int c = __popc(mm);
    if (o.count + c > kWarpBuf) {
        warp_flush(d, o.wr, o.ws, o.wk, o.count, lane);
        o.count = 0;
    }
    if (m) {
        const int pos = o.count + __popc(mm & lanemask_lt());
        o.wr[pos] = r_val;
        o.ws[pos] = s_val;
        if (emit_key) o.wk[pos] = key;
    }
    o.count += c;
    __syncwarp();
}

// Longest bucket the lanes scan in lock step; a warp with a longer one spreads the entries of all
// its buckets over the lanes instead (duplicate-heavy build keys, e.g. Zipf-skewed matches).
constexpr uint32_t kLockstepMax = 8;

// The spread walk: the warp walks the concatenation of its candidates' buckets 32 entries at a
// time, with a warp prefix sum of the bucket lengths and, per entry, a five-step shuffle binary
// search for the candidate that owns it. A key repeated k times on the build side then costs about
// k/32 steps instead of k. Lane l holds candidate e with bucket [lo, lo + len). Kept out of line
// (it runs only for warps with a long bucket), so its registers do not weigh on the common path;
// it takes and returns the warp's staging count by value. Returns the new count.
__device__ __noinline__ int probe_spread(const JoinDesc* d, uint2 e, uint32_t lo, uint32_t len,
                                         const uint2* table, bool bs, int emit_key, int lane, uint32_t* wr,
                                         uint32_t* ws, uint32_t* wk, int count) {
    WarpOut o{wr, ws, wk, count};
    uint32_t inc = len;  // inclusive prefix of the bucket lengths over the lanes
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, s);
        if (lane >= s) inc += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t g = base + (uint32_t)lane;
        // owner: the first lane c with inc[c] > g (lanes with empty buckets are skipped over)
        int c = 0;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const uint32_t v = __shfl_sync(0xffffffffu, inc, c + s - 1);
            if (v <= g) c += s;
        }
        const uint32_t c_lo = __shfl_sync(0xffffffffu, lo, c);
        const uint32_t c_start = __shfl_sync(0xffffffffu, inc - len, c);
        const uint32_t c_key = __shfl_sync(0xffffffffu, e.x, c);
        const uint32_t c_val = __shfl_sync(0xffffffffu, e.y, c);
        bool m = false;
        uint32_t rv = 0;
        if (g < total) {
            const uint2 cc = table[c_lo + (g - c_start)];
            m = (cc.x == c_key);
            rv = cc.y;
        }
        stage_matches(*d, m, bs ? c_val : rv, bs ? rv : c_val, c_key, emit_key, lane, o);
    }
    return o.count;
}

// The warp scans the buckets of candidates q[0, n) (n <= 32), one per lane, and stages every match.
// Buckets are scanned in lock step, one entry per lane per step, so the warp takes as many steps as
// its longest bucket; above kLockstepMax steps it takes the spread walk instead.
__device__ __forceinline__ void probe_candidates(const JoinDesc& d, const uint2* q, int n, const uint2* table,
                                                 const uint32_t* off, uint32_t mask, bool bs, int emit_key,
                                                 int lane, WarpOut& o) {
    uint2 e = make_uint2(0u, 0u);
    uint32_t lo = 0, hi = 0;
    if (lane < n) {
        e = q[lane];
        const uint32_t bk = bucket_of(e.x, mask);
        lo = off[bk];
        hi = off[bk + 1];
    }
    if (__reduce_max_sync(0xffffffffu, hi - lo) > kLockstepMax) {
        o.count = probe_spread(&d, e, lo, hi - lo, table, bs, emit_key, lane, o.wr, o.ws, o.wk, o.count);
        return;
    }
    while (__any_sync(0xffffffffu, lo < hi)) {
        bool m = false;
        uint32_t rv = 0;
        if (lo < hi) {
            const uint2 cc = table[lo];
            m = (cc.x == e.x);
            rv = cc.y;
            ++lo;
        }
        stage_matches(d, m, bs ? e.y : rv, bs ? rv : e.y, e.x, emit_key, lane, o);
    }
}

// Streams tuples [0, n) of `src` (global memory) through the filter and
// the warp's candidate queue; full warps of candidates are probed as they form.
template <int U, bool kGuard>
__device__ __forceinline__ void probe_step(const JoinDesc& d, const uint2* __restrict__ src, uint32_t base, uint32_t n,
                                           const uint32_t* bitmap, uint2* q, int& qn, const uint2* table,
                                           const uint32_t* off, uint32_t mask, bool bs, int emit_key, int lane,
                                           WarpOut& o) {
    uint2 e[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint32_t i = base + u * kThreads + threadIdx.x;
        e[u] = (!kGuard || i < n) ? __ldcs(src + i) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const uint32_t i = base + u * kThreads + threadIdx.x;
        const uint32_t pb = presence_bit(e[u].x);
        const bool cand = (!kGuard || i < n) && ((bitmap[pb >> 5] >> (pb & 31u)) & 1u);
        const uint32_t cm = __ballot_sync(0xffffffffu, cand);
        if (cm) {
            if (cand) q[qn + __popc(cm & lanemask_lt())] = e[u];
            qn += __popc(cm);
            __syncwarp();
            if (qn >= 32) {
                probe_candidates(d, q, 32, table, off, mask, bs, emit_key, lane, o);
                // move the overflow (fewer than 32) to the front of the queue
                const uint2 rest = lane < qn - 32 ? q[32 + lane] : make_uint2(0u, 0u);
                __syncwarp();
                if (lane < qn - 32) q[lane] = rest;
                qn -= 32;
                __syncwarp();
            }
        }
    }
}

template <int U>
__device__ __forceinline__ void probe_stream(const JoinDesc& d, const uint2* __restrict__ src, uint32_t n,
                                             const uint32_t* bitmap, uint2* q, int& qn, const uint2* table,
                                             const uint32_t* off, uint32_t mask, bool bs, int emit_key, int lane,
                                             WarpOut& o) {
    constexpr uint32_t kStep = (uint32_t)(U * kThreads);
    uint32_t base = 0;
    for (; base + kStep <= n; base += kStep) {
        // streamed from global memory: keep the range two iterations ahead on its way into L2
        if (threadIdx.x == 0 && base + 2 * kStep < n)
            prefetch_l2_range(src + base + 2 * kStep, src + min_i64((int64_t)n, (int64_t)base + 3 * kStep));
        probe_step<U, false>(d, src, base, n, bitmap, q, qn, table, off, mask, bs, emit_key, lane, o);
    }
    if (base < n) probe_step<U, true>(d, src, base, n, bitmap, q, qn, table, off, mask, bs, emit_key, lane, o);
}

// A task of the probe queue with its join's buffers resolved: the build and streamed ranges.
struct ProbeTask {
    const uint2* bsrc;
    const uint2* psrc;
    uint32_t b_len, p_len;
    int32_t join;
    int32_t bs;  // the build side is S
};

// Reads task t's record and its join's final buffers into `out` (t >= ntasks leaves it unset).
__device__ __forceinline__ void resolve_task(const JoinDesc* __restrict__ J, const Task* __restrict__ tasks,
                                             long long t, long long ntasks, ProbeTask& out) {
    if (t >= ntasks) return;
    const Task tk = tasks[t];
    const JoinDesc& d = J[tk.join];
    const bool bs = (tk.flags & kTaskBuildS) != 0;
    out.bsrc = final_buf(d, bs ? 1 : 0) + tk.b_begin;
    out.psrc = final_buf(d, bs ? 0 : 1) + tk.p_begin;
    out.b_len = tk.b_len;
    out.p_len = tk.p_len;
    out.join = tk.join;
    out.bs = bs ? 1 : 0;
}

__global__ void __launch_bounds__(kThreads, 2)
k_probe(const JoinDesc* __restrict__ J, const Task* __restrict__ tasks, unsigned long long* gwords,
        int table_cap, int emit_key) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* table = reinterpret_cast<uint2*>(smem);                              // [table_cap]
    uint2* queue = table + table_cap;                                           // [warps][kQueue]
    uint32_t* bitmap = reinterpret_cast<uint32_t*>(queue + (kThreads / 32) * kQueue);  // [kBitmapWords]
    uint32_t* off = bitmap + kBitmapWords;                                      // [table_cap + 1] (+pad)
    uint32_t* wbuf = off + table_cap + 4;
    __shared__ uint32_t tmp[kThreads / 32];
    __shared__ long long s_task[2];
    __shared__ ProbeTask s_info[2];  // the current task and the next one, resolved by thread 0
    unsigned long long* errors = &gwords[kGErrors];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int words_per_warp = kWarpBuf * (emit_key ? 3 : 2);
    WarpOut o;
    o.wr = wbuf + wid * words_per_warp;
    o.ws = o.wr + kWarpBuf;
    o.wk = o.ws + kWarpBuf;
    o.count = 0;
    uint2* q = queue + wid * kQueue;
    int cur = -1;
    const long long ntasks = (long long)gwords[kGTasks];
    if (threadIdx.x == 0) {
        const long long t0 = (long long)atomicAdd(&gwords[kGQueue], 1ull);
        s_task[0] = t0;
        resolve_task(J, tasks, t0, ntasks, s_info[0]);
    }
    __syncthreads();
    for (int slot = 0;; slot ^= 1) {
        const long long t = s_task[slot];
        if (t >= ntasks) break;
        const ProbeTask tk = s_info[slot];
        const JoinDesc& d = J[tk.join];
        const bool bs = tk.bs != 0;
        const uint2* __restrict__ bsrc = tk.bsrc;
        const uint2* __restrict__ psrc = tk.psrc;
        const uint32_t pn = tk.p_len;
        if (threadIdx.x == 0) {
            // the first two iterations of the probe side go to L2 while the table is built
            prefetch_l2_range(psrc, psrc + min_i64((int64_t)pn, (int64_t)2 * kProbeU * kThreads));
            s_task[slot ^ 1] = (long long)atomicAdd(&gwords[kGQueue], 1ull);  // resolved after the probe
        }
        if (tk.join != cur) {
            if (cur >= 0 && o.count > 0) warp_flush(J[cur], o.wr, o.ws, o.wk, o.count, lane);
            o.count = 0;
            cur = tk.join;
        }
        int nr = (int)tk.b_len;
        if (nr > table_cap) {
            if (threadIdx.x == 0) atomicAdd(errors, 1ull);
            nr = table_cap;
        }
        uint32_t nb = 32;
        while (nb < (uint32_t)nr) nb <<= 1;
        const uint32_t mask = nb - 1;
        // the previous task's probe is done with table, off and bitmap
        for (uint32_t i = threadIdx.x; i <= nb; i += kThreads) off[i] = 0;
        for (int i = threadIdx.x; i < kBitmapWords; i += kThreads) bitmap[i] = 0;
        // ---- build: count per bucket (the atomic's result is the rank), set the bitmap bits
        uint2 bt[kBuildPer];
#pragma unroll
        for (int k = 0; k < kBuildPer; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < nr) bt[k] = __ldg(bsrc + i);
        }
        __syncthreads();
        uint32_t br[kBuildPer];  // bucket << 16 | rank in bucket
#pragma unroll
        for (int k = 0; k < kBuildPer; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < nr) {
                const uint32_t bk = bucket_of(bt[k].x, mask);
                br[k] = (bk << 16) | atomicAdd(&off[bk], 1u);
                const uint32_t pb = presence_bit(bt[k].x);
                atomicOr(&bitmap[pb >> 5], 1u << (pb & 31u));
            }
        }
        __syncthreads();
        // off[b] = start of bucket b, off[nb] = nr
        if (nb == 8 * kThreads) scan_dir<8>(off, nb, tmp);
        else if (nb == 4 * kThreads) scan_dir<4>(off, nb, tmp);
        else block_scan_excl(off, (int)nb + 1, tmp);
        // the build tuples are read again (cache hits) rather than held in registers across the scan
#pragma unroll
        for (int k = 0; k < kBuildPer; ++k) {
            const int i = k * kThreads + threadIdx.x;
            if (i < nr) table[off[br[k] >> 16] + (br[k] & 0xffffu)] = __ldg(bsrc + i);
        }
        __syncthreads();
        // ---- probe: the other side streamed from global memory
        int qn = 0;  // candidates in this warp's queue (warp-uniform)
        probe_stream<kProbeU>(d, psrc, pn, bitmap, q, qn, table, off, mask, bs, emit_key, lane, o);
        if (qn > 0) probe_candidates(d, q, qn, table, off, mask, bs, emit_key, lane, o);
        // the next task's record and buffers, read while the other warps finish this task, and its
        // build chunk on its way into L2
        if (threadIdx.x == 0) {
            ProbeTask& nx = s_info[slot ^ 1];
            resolve_task(J, tasks, s_task[slot ^ 1], ntasks, nx);
            if (s_task[slot ^ 1] < ntasks) prefetch_l2_range(nx.bsrc, nx.bsrc + nx.b_len);
        }
        __syncwarp();
        __syncthreads();
    }
    if (cur >= 0 && o.count > 0) warp_flush(J[cur], o.wr, o.ws, o.wk, o.count, lane);
}

// Copies each join's match count to the caller's device int64 (if requested), or -1 when a
// device-side consistency check of this run failed (the host reports BRIG_E_INTERNAL), so that a
// caller that reads only the device count, without a host synchronisation, sees the failure too.
__global__ void k_publish_counts(const JoinDesc* __restrict__ J, int nj, const unsigned long long* gwords) {
    const bool failed = gwords[kGErrors] != 0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nj; j += gridDim.x * blockDim.x) {
        const JoinDesc& d = J[j];
        if (d.user_count) *d.user_count = failed ? -1 : d.counters[kCntMatches];
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

// Resets the run's state words: the task queue, the error count (unless the run continues an earlier
// launch's count) and the bound of the waits.
__global__ void k_init_words(unsigned long long* g, int keep_errors, uint32_t polls) {
    g[kGQueue] = 0ull;
    if (!keep_errors) g[kGErrors] = 0ull;
    g[kGWaitPolls] = polls;
}

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
    static const char* names[kNumStages] = {"r_hist", "r_scan", "r_scatter", "r_l2_hist", "r_l2_scatter",
                                            "bloom_build", "s_hist_probe", "s_scan", "s_scatter", "s_l2_hist",
                                            "s_l2_scatter", "tasks",
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
    return (size_t)table_cap * 8 + (size_t)(kThreads / 32) * kQueue * 8 +
           (size_t)kBitmapWords * 4 +
           ((size_t)table_cap + 4) * 4 +
           (size_t)(kThreads / 32) * kWarpBuf * (emit_key ? 3 : 2) * 4;
}

// Shared memory of the scatter kernels: two bulk-copy tile buffers, the reordered tile, and a
// cursor and a count per bin.
// Dynamic shared memory of a scatter kernel over at most max_bins bins: the bulk-store layout
// (bulk_carve) or the write-pass layout (scatter_carve).
static size_t scatter_smem(int max_bins, int form) {
    if (form != kFormPass) return bulk_bufs(form, max_bins) + (size_t)max_bins * (8 + 4 + 4);
    return 2 * kTileBufW + (size_t)max_bins * (8 + 8 + 4) + (size_t)kSTileW * 2;
}

static cudaError_t set_smem_attr(const void* fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Calls f(std::integral_constant<int, M>, std::integral_constant<int, K>) for every partition mode
// M and Bloom mask class K present in the batch.
template <class F>
static void for_mode_k(int modes, int kclasses, F&& f) {
    if ((modes & 1) && (kclasses & 1)) f(std::integral_constant<int, 0>{}, std::integral_constant<int, 0>{});
    if ((modes & 1) && (kclasses & 2)) f(std::integral_constant<int, 0>{}, std::integral_constant<int, kBloomFastK>{});
    if ((modes & 2) && (kclasses & 1)) f(std::integral_constant<int, 1>{}, std::integral_constant<int, 0>{});
    if ((modes & 2) && (kclasses & 2)) f(std::integral_constant<int, 1>{}, std::integral_constant<int, kBloomFastK>{});
}

// Calls f(std::integral_constant<int, M>) for every partition mode M present in the batch.
template <class F>
static void for_modes(int modes, F&& f) {
    if (modes & 1) f(std::integral_constant<int, 0>{});
    if (modes & 2) f(std::integral_constant<int, 1>{});
}

// Calls f(std::integral_constant<int, F>) for the scatter form F (ScatterForm).
template <class Fn>
static void for_form(int form, Fn&& f) {
    if (form == kFormBulkSmall) f(std::integral_constant<int, kFormBulkSmall>{});
    else if (form == kFormBulk) f(std::integral_constant<int, kFormBulk>{});
    else f(std::integral_constant<int, kFormPass>{});
}

static int grid_for(int64_t work, int num_sms, int per_sm) {
    int64_t g = std::min<int64_t>(work, (int64_t)num_sms * per_sm);
    return (int)std::max<int64_t>(g, 1);
}

static cudaError_t set_kernel_attrs() {
    cudaError_t err;
    const void* l1s[] = {(const void*)k_l1_scatter<false, 0, kFormPass>, (const void*)k_l1_scatter<false, 1, kFormPass>,
                         (const void*)k_l1_scatter<true, 0, kFormPass>, (const void*)k_l1_scatter<true, 1, kFormPass>};
    for (const void* f : l1s)
        if ((err = set_smem_attr(f, scatter_smem(kMaxP1, kFormPass))) != cudaSuccess) return err;
    const void* bulks[] = {(const void*)k_l1_scatter<false, 0, kFormBulk>, (const void*)k_l1_scatter<false, 1, kFormBulk>,
                           (const void*)k_l1_scatter<true, 0, kFormBulk>,  (const void*)k_l1_scatter<true, 1, kFormBulk>,
                           (const void*)k_l2_scatter<0, kFormBulk>,        (const void*)k_l2_scatter<1, kFormBulk>};
    for (const void* f : bulks)
        if ((err = set_smem_attr(f, scatter_smem(kBulkMaxBins, kFormBulk))) != cudaSuccess) return err;
    // the small form: two CTAs per SM, so shared memory takes the largest carve-out
    const void* smalls[] = {
        (const void*)k_l1_scatter<false, 0, kFormBulkSmall>, (const void*)k_l1_scatter<false, 1, kFormBulkSmall>,
        (const void*)k_l1_scatter<true, 0, kFormBulkSmall>,  (const void*)k_l1_scatter<true, 1, kFormBulkSmall>,
        (const void*)k_l2_scatter<0, kFormBulkSmall>,        (const void*)k_l2_scatter<1, kFormBulkSmall>};
    for (const void* f : smalls) {
        if ((err = set_smem_attr(f, scatter_smem(kBulkSmallMaxBins, kFormBulkSmall))) != cudaSuccess) return err;
        if ((err = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
            return err;
    }
    const void* l2s[] = {(const void*)k_l2_scatter<0, kFormPass>, (const void*)k_l2_scatter<1, kFormPass>};
    for (const void* f : l2s)
        if ((err = set_smem_attr(f, scatter_smem(kMaxP2, kFormPass))) != cudaSuccess) return err;
    const void* bbs[] = {(const void*)k_bloom_build<0, 0>, (const void*)k_bloom_build<1, 0>,
                         (const void*)k_bloom_build<0, kBloomFastK>, (const void*)k_bloom_build<1, kBloomFastK>};
    for (const void* f : bbs)
        if ((err = set_smem_attr(f, kBloomSmemWords * 4)) != cudaSuccess) return err;
    if ((err = set_smem_attr((const void*)k_probe, probe_smem_bytes(kMaxTable, 1))) != cudaSuccess)
        return err;
    return cudaSuccess;
}

// Kernel attributes (the dynamic shared-memory limits above 48 KB) hold per device: they are set once
// for every device the process launches on.
static std::mutex g_attr_mu;
static uint64_t g_attr_done = 0;  // bit d: attributes set on device d (ordinals 0..63)

cudaError_t enqueue_pipeline(const PipelineArgs& a, cudaStream_t st) {
    cudaError_t err;
    int dev = 0;
    if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
    {
        std::lock_guard<std::mutex> lk(g_attr_mu);
        const bool known = dev >= 0 && dev < 64;
        if (!known || !((g_attr_done >> dev) & 1u)) {
            if ((err = set_kernel_attrs()) != cudaSuccess) return err;
            if (known) g_attr_done |= 1ull << dev;
        }
    }
    const int sms = a.num_sms;

    int launches = 0;
    auto mark = [&](int i) {
        if (a.stage_events) cudaEventRecord(a.stage_events[i], st);
    };
    mark(0);
    k_init_words<<<1, 1, 0, st>>>(a.gwords, a.keep_errors, a.wait_polls);
    ++launches;

    // ---- R, then S: level 1 and level 2 (the Bloom build sits between them) -----------------
    for (int rel = 0; rel < 2; ++rel) {
        const bool part = (a.stages & (rel == 0 ? kRunPartR : kRunPartS)) != 0;
        if (rel == 1 && (a.stages & kRunBloom) && a.any_bloom && a.total_bloom_groups > 0) {
            // Bloom filter over the final R partitions, before S's first pass probes it.
            for_mode_k(a.modes, a.kclasses, [&](auto mt, auto kt) {
                constexpr int M = decltype(mt)::value, K = decltype(kt)::value;
                k_bloom_build<M, K><<<grid_for(a.total_bloom_groups, sms, 4), kThreads,
                                   (size_t)a.bloom_smem_words * 4, st>>>(a.J, a.nj, a.bloom_prefix,
                                                                         a.bloom_smem_words, a.gwords, a.pat_k);
                ++launches;
            });
        }
        if (rel == 1 && a.s_ready && (err = cudaStreamWaitEvent(st, a.s_ready, 0)) != cudaSuccess) return err;
        if (rel == 1) mark(6);
        const int m0 = rel == 0 ? 1 : 7;  // first stage mark of this relation
        if (!part) {
            for (int m = m0; m < m0 + 5; ++m) mark(m);
            continue;
        }
        if (a.total_slices[rel] > 0) {
            for_mode_k(a.modes, a.kclasses, [&](auto mt, auto kt) {
                constexpr int M = decltype(mt)::value, K = decltype(kt)::value;
                k_l1_hist<M, K><<<grid_for(a.total_slices[rel], sms, 4), kThreads, (size_t)a.max_p1 * 4, st>>>(
                    a.J, a.nj, rel, a.slice_prefix[rel], a.hist, a.gwords, a.pat_k);
                ++launches;
            });
        }
        mark(m0);
        if ((err = enqueue_scan(a.hist + a.hist_begin[rel], a.hist_scan + a.hist_begin[rel],
                                a.hist_len[rel], a.scan_tmp, nullptr, st)) != cudaSuccess)
            return err;
        mark(m0 + 1);
        if (a.total_slices[rel] > 0) {
            for_modes(a.modes, [&](auto mt) {
                constexpr int M = decltype(mt)::value;
                const int form = a.l1_form[rel];
                for_form(form, [&](auto ft) {
                    constexpr int F = decltype(ft)::value;
                    const dim3 grid(grid_for(a.total_slices[rel], sms, form_ctas_per_sm(F)));
                    const size_t smem = scatter_smem(a.max_p1, F);
                    k_l1_scatter<false, M, F><<<grid, form_threads(F), smem, st>>>(
                        a.J, a.nj, rel, a.slice_prefix[rel], a.hist_scan, a.gwords, a.max_p1);
                    ++launches;
                    if (rel == 1 && a.any_bloom_l1) {
                        k_l1_scatter<true, M, F><<<grid, form_threads(F), smem, st>>>(
                            a.J, a.nj, rel, a.slice_prefix[rel], a.hist_scan, a.gwords, a.max_p1);
                        ++launches;
                    }
                });
            });
        }
        mark(m0 + 2);
        {
            dim3 grid((unsigned)((a.max_p1 + 1 + 255) / 256), (unsigned)std::min(a.nj, 65535));
            k_bounds_l1<<<grid, 256, 0, st>>>(a.J, a.nj, rel, a.hist_scan);
            ++launches;
        }
        if (a.total_segs > 0) {
            const int pb = (int)std::min<int64_t>((a.total_segs + 1 + 255) / 256, (int64_t)sms * 8);
            k_l2_plan<<<pb, 256, 0, st>>>(a.J, a.nj, rel, a.seg_prefix, a.seg_ns);
            ++launches;
            if ((err = enqueue_scan(a.seg_ns, a.seg_off, a.total_segs + 1, a.scan_tmp,
                                    reinterpret_cast<int64_t*>(a.gwords + kGL2Slices + rel), st)) != cudaSuccess)
                return err;
            uint32_t* h2 = a.hist2 + a.h2_begin[rel];
            if ((err = cudaMemsetAsync(h2, 0, (size_t)a.h2_len[rel] * 4, st)) != cudaSuccess) return err;
            if (!(rel == 1 && a.all_bloom_l2)) {
                for_modes(a.modes, [&](auto mt) {
                    constexpr int M = decltype(mt)::value;
                    const dim3 grid(grid_for(a.l2_slice_cap[rel], sms, 4));
                    k_l2_hist<M><<<grid, kThreads, (size_t)a.max_p2 * 4, st>>>(
                        a.J, a.nj, rel, a.seg_prefix, a.seg_off, a.seg_ns, a.total_segs, a.hist2, a.gwords);
                    ++launches;
                });
            }
            if (rel == 1 && a.any_bloom_l2) {
                for_mode_k(a.modes, a.kclasses, [&](auto mt, auto kt) {
                    constexpr int M = decltype(mt)::value, K = decltype(kt)::value;
                    k_l2_bloom<M, K><<<grid_for(a.l2_slice_cap[rel], sms, 4), kThreads, (size_t)a.max_p2 * 4, st>>>(
                        a.J, a.nj, a.seg_prefix, a.seg_off, a.seg_ns, a.total_segs, a.hist2, a.slice_cnt2, a.gwords,
                        a.pat_k);
                    ++launches;
                });
            }
            mark(m0 + 3);
            if ((err = enqueue_scan(h2, a.hist2_scan + a.h2_begin[rel], a.h2_len[rel], a.scan_tmp, nullptr, st)) !=
                cudaSuccess)
                return err;
            for_modes(a.modes, [&](auto mt) {
                constexpr int M = decltype(mt)::value;
                for_form(a.l2_form[rel], [&](auto ft) {
                    constexpr int F = decltype(ft)::value;
                    k_l2_scatter<M, F><<<grid_for(a.l2_slice_cap[rel], sms, form_ctas_per_sm(F)), form_threads(F),
                                         scatter_smem(a.max_p2, F), st>>>(
                        a.J, a.nj, rel, a.seg_prefix, a.seg_off, a.seg_ns, a.total_segs, a.hist2_scan, a.slice_cnt2,
                        a.gwords, a.max_p2);
                    ++launches;
                });
            });
            dim3 grid((unsigned)std::min<int64_t>(((int64_t)a.max_p1 * a.max_p2 + 1 + 255) / 256, 4096),
                      (unsigned)std::min(a.nj, 65535));
            k_l2_bounds<<<grid, 256, 0, st>>>(a.J, a.nj, rel, a.seg_prefix, a.seg_off, a.seg_ns, a.hist2_scan);
            ++launches;
        } else {
            mark(m0 + 3);
        }
        mark(m0 + 4);
    }
    // ---- tasks --------------------------------------------------------------------------------
    if (!(a.stages & kRunProbe)) {
        mark(12);
        mark(13);
        note_launches(launches);
        return cudaGetLastError();
    }
    {
        const int64_t n = a.total_domains + 1;
        const int blocks = (int)std::min<int64_t>((n + kTaskWarps - 1) / kTaskWarps, (int64_t)sms * 16);
        k_tasks_count<<<blocks, kTaskWarps * 32, 0, st>>>(a.J, a.nj, a.dom_prefix, a.tcount);
        ++launches;
        if ((err = enqueue_scan(a.tcount, a.toff, n, a.scan_tmp,
                                reinterpret_cast<int64_t*>(a.gwords + kGTasks), st)) != cudaSuccess)
            return err;
        k_tasks_write<<<blocks, kTaskWarps * 32, 0, st>>>(a.J, a.nj, a.dom_prefix, a.toff, a.tasks, a.task_cap,
                                                          a.gwords);
        ++launches;
    }
    mark(12);
    // ---- probe --------------------------------------------------------------------------------
    {
        const size_t smem = probe_smem_bytes(a.table_cap, a.emit_key);
        int occ = 0;
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_probe, kThreads, smem)) !=
            cudaSuccess)
            return err;
        occ = std::max(occ, 1);
        k_probe<<<sms * occ, kThreads, smem, st>>>(a.J, a.tasks, a.gwords, a.table_cap, a.emit_key);
        mark(13);
        k_publish_counts<<<1, 256, 0, st>>>(a.J, a.nj, a.gwords);
        launches += 2;
    }
    note_launches(launches);
    return cudaGetLastError();
}

}  // namespace brig
