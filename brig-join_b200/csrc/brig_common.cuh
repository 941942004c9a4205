// brig_common.cuh - types and integer mixing shared by the host planner and the sm_100a kernels.
//
// Tuples are (uint32 key, uint32 value). Inputs arrive as separate key and value arrays (the
// reference's int* tableA / tableA_val, src/hash_kernel.cu:302-307). Every partitioned buffer the
// engine writes stores a tuple as one 8-byte uint2 {key, value}, so a tuple moves with one
// coalesced 8-byte access (the reference's int2 KV layout, src/kernel_functions.cu:251-281).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define BRIG_HD __host__ __device__ __forceinline__
#else
#define BRIG_HD inline
#endif

namespace brig {

// ---- limits -------------------------------------------------------------------------------------
constexpr int kMaxP1 = 4096;          // first-level fan-out (the reference caps at PARTITION_MAX=2048,
                                      // src/kernel_functions.h:15); at most 12 radix bits, which
                                      // part1_m relies on
constexpr int kMaxP2 = 1024;          // second-level fan-out (SECOND_PASS_MAX=4096, :14)
constexpr int kMaxTable = 4096;       // build-side tuples per shared-memory table (largest allowed)
constexpr int kDefaultTable = 4096;   // default table capacity
constexpr int kDefaultChunk = 65536;  // default streamed tuples per probe task
constexpr int kMinTable = 256;
constexpr int kMaxBloomK = 16;
constexpr int kThreads = 512;         // threads per CTA of every partition and probe kernel
constexpr int kTile = 4096;           // unit of the level-2 slice length
constexpr int kSThreads = 1024;       // threads per CTA of the scatter kernels (one CTA per SM)
constexpr int kSThreadsSmall = 512;   // threads per CTA of their small bulk-store form (two per SM)
constexpr int kSTile = 12288;         // tuples per tile of the bulk-store scatter (slice lengths are
                                      // multiples of it)
// Forms of a scatter launch: the write pass (any bin count up to the fan-out limits), the
// bulk-store form (up to kBulkMaxBins bins, 12288-tuple tiles, one 1024-thread CTA per SM) and its
// small form (up to kBulkSmallMaxBins bins, 6144-tuple tiles, two 512-thread CTAs per SM).
enum ScatterForm : int { kFormPass = 0, kFormBulk = 1, kFormBulkSmall = 2 };
constexpr int kBulkMaxBins = 1024;
constexpr int kBulkSmallMaxBins = 512;
constexpr int kWarpBuf = 128;         // output pairs staged per warp before a global flush
// Tuples per level-2 slice: 262144, or 131072 for S when its second pass probes the Bloom filter
// (the filter segments of the partitions in flight must stay in L2; with the longer slices twice
// as many partitions are in flight).
constexpr int64_t kL2Slice = 21 * kSTile;
constexpr uint32_t kDefaultWaitPolls = 1u << 22;  // polls of a bounded wait before it gives up
constexpr int64_t kL2SliceBloom = 32 * kTile;

// Per-join device counters (int64 each).
enum Counter : int {
    kCntMatches = 0,      // exact number of matches
    kCntSurvivors = 1,    // S tuples that passed the Bloom filter
    kCntTasks = 2,        // probe tasks generated
    kCntSplitTasks = 3,   // tasks whose build chunk is a piece of an oversized partition
    kCntErrors = 4,       // device-side consistency failures (must stay 0)
    kCntWords = 8
};

// ---- integer mixing -----------------------------------------------------------------------------
// MurmurHash3 32-bit finaliser (Austin Appleby, public domain). A bijection on uint32: the radix
// partition ids are its top bits, the shared-memory bucket its low bits. The reference's Bloom hash
// is a variant of the same finaliser (src/bloom.cu:24-31).
BRIG_HD uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x85ebca6bu;
    x ^= x >> 13; x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014). Used by the input generator and for Bloom hashes beyond the eighth.
BRIG_HD uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27; x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

// Maps a uniform 32-bit value onto [0, n) with one multiply (Lemire, "Fast random integer
// generation in an interval", 2019).
BRIG_HD uint32_t fastrange32(uint32_t x, uint32_t n) {
    return (uint32_t)(((uint64_t)x * (uint64_t)n) >> 32);
}

// a % d for a runtime divisor d >= 1 via a precomputed 64-bit magic M = floor((2^64-1)/d) + 1
// (Lemire, Kaser, Kurz, "Faster remainder by direct computation", 2019).
BRIG_HD uint64_t fastmod_magic(uint32_t d) { return ~0ull / d + 1; }
BRIG_HD uint32_t fastmod(uint32_t a, uint64_t M, uint32_t d) {
    uint64_t lowbits = M * a;
#if defined(__CUDA_ARCH__)
    return (uint32_t)__umul64hi(lowbits, (uint64_t)d);
#else
    return (uint32_t)(((unsigned __int128)lowbits * d) >> 64);
#endif
}

// ---- partition functions ------------------------------------------------------------------------
// Level-1 id p in [0, P1), level-2 id q in [0, P2). Hash mode: P1 = 2^b1, P2 = 2^b2 and the ids are
// the top b1 bits and the next b2 bits of mix32(key). Modulo mode: p = key % P1, q = key % P2, the
// reference's two modulo levels (src/kernel_functions.cu:66,187).
struct PartFn {
    int32_t mode;       // 0 hash, 1 modulo
    int32_t b1, b2;     // radix bits (hash mode)
    uint32_t P1, P2;    // fan-outs
    uint64_t M1, M2;    // fastmod magics (modulo mode)
};

// mix32 without its last xor-shift, which changes only the low 16 bits: the top 16 bits are those
// of mix32(key), so the level-1 id (b1 <= 12 bits) takes two fewer instructions from it.
BRIG_HD uint32_t mix32_hi(uint32_t x) {
    x ^= x >> 16; x *= 0x85ebca6bu;
    x ^= x >> 13; x *= 0xc2b2ae35u;
    return x;
}
// The top s bits of x (0 when s == 0): one clamped funnel shift on the device.
BRIG_HD uint32_t top_bits(uint32_t x, int s) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_rc(x, 0u, 32u - (uint32_t)s);
#else
    return (uint32_t)(((uint64_t)x << s) >> 32);
#endif
}

// Mode-specialised forms, M = 0 (hash) or 1 (modulo). The partition kernels are instantiated per
// mode and skip the joins of the other mode, so their per-key code carries no mode test. In hash
// mode p is the top b1 bits of mix32(key) and q the next b2 bits (both 0 when the bit count is 0).
template <int M>
BRIG_HD uint32_t part1_m(const PartFn& f, uint32_t key) {
    if constexpr (M == 0) return top_bits(mix32_hi(key), f.b1);  // b1 <= 12: equal to mix32's top bits
    else return fastmod(key, f.M1, f.P1);
}
template <int M>
BRIG_HD uint32_t part2_m(const PartFn& f, uint32_t key) {
    if constexpr (M == 0) return top_bits(mix32(key) << f.b1, f.b2);
    else return fastmod(key, f.M2, f.P2);
}
// Finest partition id p * P2 + q: the probe-task unit and the Bloom segment index.
template <int M>
BRIG_HD uint32_t part_fine_m(const PartFn& f, uint32_t key) {
    return part1_m<M>(f, key) * f.P2 + part2_m<M>(f, key);
}
BRIG_HD uint32_t part1(const PartFn& f, uint32_t key) { return f.mode == 0 ? part1_m<0>(f, key) : part1_m<1>(f, key); }
BRIG_HD uint32_t part2(const PartFn& f, uint32_t key) { return f.mode == 0 ? part2_m<0>(f, key) : part2_m<1>(f, key); }
BRIG_HD uint32_t part_fine(const PartFn& f, uint32_t key) {
    return f.mode == 0 ? part_fine_m<0>(f, key) : part_fine_m<1>(f, key);
}
// Shared-memory bucket of a key in a table of nb (power of two) buckets: the low bits of the mix.
BRIG_HD uint32_t bucket_of(uint32_t key, uint32_t nb_mask) { return mix32(key) & nb_mask; }

// ---- Bloom filter -------------------------------------------------------------------------------
// Cache-sectorized blocked Bloom filter (Lang, Neumann, Kemper, Boncz, "Performance-Optimal
// Filtering: Bloom overtakes Cuckoo at High Throughput", VLDB 2019). The filter is one segment per
// finest partition; a segment is seg_blocks blocks of 256 bits, one 32-byte DRAM sector of eight
// 32-bit words, i.e. four 8-byte word pairs. A key picks one word pair and sets its k bit positions
// in those two words: the first ceil(k/2) in the even word, the rest in the odd word. So a build
// is two 32-bit atomicOr per key and a probe one 8-byte load, with no search or dynamic indexing.
// The reference uses 256-bit blocks with k bit positions anywhere in the block and one segment
// per first-level partition (src/bloom.cu:698-722, src/hash_kernel.cu:555-582).
//
// Hash bits (g = bloom_hash(key)): bits 40..63 pick the block, bits 35..36 the word pair, bits 0..9
// the pattern pair (below).

// The Bloom hash is mix32(key) (which the partition functions compute anyway) times an odd 64-bit
// constant: multiplication by an odd constant is a bijection modulo every power of two, so each
// field of the product is uniform when mix32(key) is, and the top bits depend on every input bit.
BRIG_HD uint64_t bloom_hash(uint32_t key) { return (uint64_t)mix32(key) * 0x9e3779b97f4a7c15ull; }

// Masks. For k = 7 (10 bits per key, the default) the bit positions are seven 5-bit fields of g
// (bits 0..34): fields 0..3 in the even word, 4..6 in the odd word, one funnel shift each.
// Every other k takes pattern-blocked masks (Lang et al., as above): hash bits 0..9 pick one of
// 1024 pattern pairs, ceil(k/2) bits for the even word and floor(k/2) bits for the odd word;
// pattern i of word w is the OR of 1 << (5-bit fields of a SplitMix64 hash of (w, i)). The kernels
// keep the pairs (8 KB), filled for the launch's k, in shared memory, so those masks cost one 8-byte
// shared-memory load. Measured at 640M keys: the compile-time shifts take the level-2 probe from
// 3.45 to 3.19 ms (its random filter loads keep the L1 pipe busy, and the look-ups compete with
// them) and the build from 1.51 to 1.61 ms; two look-ups per key, or seven shifts recomputed from
// the key, cost more in both.
constexpr int kBloomFastK = 7;  // template tag of the compile-time k = 7 instantiations
BRIG_HD uint32_t bloom_bit(uint32_t p) {  // 1 << (p mod 32): one funnel shift on the device
#if defined(__CUDA_ARCH__)
    return __funnelshift_l(0u, 1u, p);
#else
    return 1u << (p & 31u);
#endif
}
BRIG_HD uint2 bloom_masks7(uint64_t g) {
    const uint32_t lo = (uint32_t)g, hi = (uint32_t)(g >> 32);
    uint2 r;
    r.x = bloom_bit(lo) | bloom_bit(lo >> 5) | bloom_bit(lo >> 10) | bloom_bit(lo >> 15);
    r.y = bloom_bit(lo >> 20) | bloom_bit(lo >> 25) | bloom_bit((lo >> 30) | (hi << 2));
    return r;
}
constexpr int kPatterns = 1024;
BRIG_HD uint32_t bloom_pattern(int word, uint32_t i, int k) {
    const uint64_t h = mix64(((uint64_t)(word + 1) << 32) ^ (uint64_t)i ^ 0x243f6a8885a308d3ull);
    const int nb = word == 0 ? (k + 1) / 2 : k / 2;  // at most 8 fields of 5 bits
    uint32_t m = 0;
    for (int b = 0; b < nb; ++b) m |= 1u << ((uint32_t)(h >> (5 * b)) & 31u);
    return m;
}

// Where a key's filter bits live: the word index of its word pair in the whole filter (32-bit: the
// planner keeps a filter below 2^32 words) and its pattern index. m = mix32(key), fine = the key's
// finest partition (its segment), or its index relative to a group of segments. Of g =
// bloom_hash(key): the block is ((g >> 40) * seg_blocks) >> 24 (a multiply-high), the word pair
// (g >> 35) & 3, the pattern pair g & 1023.
struct BloomSlot {
    uint32_t widx;  // index of the pair's even word
    uint32_t pidx;  // pattern pair (k != 7)
    uint64_t g;     // the Bloom hash (its low 35 bits place the k = 7 bits)
};
BRIG_HD BloomSlot bloom_slot(uint32_t m, uint32_t fine, uint32_t seg_blocks) {
    const uint64_t g = (uint64_t)m * 0x9e3779b97f4a7c15ull;  // bloom_hash
    const uint32_t lo = (uint32_t)g, hi = (uint32_t)(g >> 32);
#if defined(__CUDA_ARCH__)
    const uint32_t blk = __umulhi(hi & 0xffffff00u, seg_blocks);
#else
    const uint32_t blk = (uint32_t)(((uint64_t)(hi & 0xffffff00u) * seg_blocks) >> 32);
#endif
    BloomSlot s;
    s.widx = ((fine * seg_blocks + blk) << 3) + ((hi >> 2) & 6u);
    s.pidx = lo & (kPatterns - 1);
    s.g = g;
    return s;
}

#if defined(__CUDACC__)
// The Bloom kernels keep the launch's pattern table (one pair of masks per pattern index, filled for
// the launch's k, which every filtered join of a launch shares) in shared memory. Fill is
// block-wide; the caller synchronises. k == 0: no filter.
__device__ __forceinline__ void fill_patterns(uint2* pat, int k) {
    if (k == 0) return;
    for (int i = threadIdx.x; i < kPatterns; i += blockDim.x)
        pat[i] = make_uint2(bloom_pattern(0, (uint32_t)i, k), bloom_pattern(1, (uint32_t)i, k));
}
// Masks of a key at slot s: compile-time shifts (K == kBloomFastK) or the pattern table.
template <int K>
__device__ __forceinline__ uint2 slot_masks(const uint2* pat, const BloomSlot& s) {
    if constexpr (K == kBloomFastK) return bloom_masks7(s.g);
    else return pat[s.pidx];
}
// Shared-memory entries of the pattern table of a kernel of class K (none for k = 7).
template <int K>
constexpr int pat_entries() { return K == kBloomFastK ? 1 : kPatterns; }
// A word pair passes when it holds every bit of both masks.
__device__ __forceinline__ bool bloom_pass(uint2 w, uint2 mk) {
    return (((w.x & mk.x) ^ mk.x) | ((w.y & mk.y) ^ mk.y)) == 0u;
}
#endif

// ---- per-join descriptor (device resident) ------------------------------------------------------
struct RelPlan {
    const uint32_t* key;   // input keys
    const uint32_t* val;   // input values
    int64_t n;             // input tuples
    uint2* l1;             // level-1 partitioned tuples [n]
    uint2* l2;             // level-2 partitioned tuples [n] (nullptr when P2 == 1)
    uint2* cmp;            // Bloom survivors staged per slice [n] (S with Bloom only)
    int64_t slice_len;     // tuples per level-1 slice
    int32_t nslices;       // level-1 slices
    int32_t l2_slice;      // tuples per level-2 slice
    int64_t hist_base;     // offset of this relation's [P1][nslices]+1 histogram in the global array
    int64_t* b1;           // [P1 + 1] start of each level-1 partition in l1
    int64_t* bounds;       // [P1*P2 + 1] start of each finest partition in the final buffer
                           // (equal to b1 when P2 == 1)
    uint32_t* slice_cnt;   // [nslices] survivors per slice (S with a level-1 Bloom probe)
    int64_t h2_base;       // offset of this relation's [P1][P2][slices] level-2 histogram in hist2
};

struct JoinDesc {
    RelPlan rel[2];        // 0 = R (build side), 1 = S (probe side)
    PartFn pf;
    uint32_t* out_r;       // pair outputs
    uint32_t* out_s;
    uint32_t* out_k;       // may be nullptr
    int64_t cap;           // output capacity (pairs)
    int64_t* counters;     // [kCntWords]
    int64_t* user_count;   // optional user int64 receiving the match count
    uint32_t* bloom;       // filter words (nullptr when off)
    uint32_t seg_blocks;   // blocks per Bloom segment
    int32_t bloom_k;
    int32_t bloom_level;   // S pass that probes the filter: 1 first (fused with the histogram of
                           // S's level-1 pass), 2 second (fused with S's level-2 pass)
    int32_t bloom_group;   // consecutive finest partitions per Bloom build CTA
    int64_t dom_base;      // offset of this join's task domains in the global task-count array
    int64_t fine_base;     // unused (kept zero)
    int32_t table_cap;     // max build-side tuples per probe task
    int32_t s_chunk;       // max streamed tuples per probe task
};

// One probe task of one finest partition: build a shared-memory table from a chunk of the build
// side, then stream a chunk of the other side through it. The build side is the smaller of the
// two partitions (with the Bloom filter on, usually S's survivors), so the larger side is read
// once, as a coalesced stream. Both ranges index the join's final partitioned buffers.
enum TaskFlag : uint32_t {
    kTaskSplit = 1u,       // the build chunk is a piece of a build side larger than one table
    kTaskBuildS = 2u,      // build from S and stream R (otherwise build from R and stream S)
};
struct Task {
    int32_t join;
    uint32_t flags;
    int64_t b_begin;       // build-side chunk
    int64_t p_begin;       // streamed chunk
    uint32_t b_len;
    uint32_t p_len;
};
static_assert(sizeof(Task) == 32, "task layout");

// Global queue/state words of one pipeline run (int64 each).
enum GlobalWord : int {
    kGQueue = 0,           // next task index to hand out
    kGTasks = 1,           // total tasks (written by the task builder)
    kGErrors = 2,          // device-side consistency failures
    kGL2Slices = 3,        // level-2 slices of R (word 3) and of S (word 4)
    kGWaitPolls = 5,       // polls after which a bounded wait gives up and counts an error
    kGWords = 8
};

}  // namespace brig
