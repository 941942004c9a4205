/*
 * brig_join.h - C ABI of the B200 equi-join engine.
 *
 * The engine joins two relations R and S of (uint32 key, uint32 value) tuples on key equality and
 * materialises every matching (r_val, s_val) pair (optionally with the key). It is the single-GPU
 * local join of BRIG-Join re-designed for sm_100a:
 *
 *   two-level partitioning of R and S -> Bloom filter built on R, probed in S's first partition
 *   pass -> per-partition shared-memory hash build and probe (oversized partitions are split into
 *   table-sized chunks) -> match materialisation with an exact count.
 *
 * Every entry point returns a status code (BRIG_OK or a BRIG_E_* value) and never exits the
 * process. brig_join_last_error() returns a message for the last failure on the calling thread.
 * Device pointers are plain CUDA device addresses; `stream` is a cudaStream_t passed as void*
 * (NULL = the legacy default stream). A handle may be used by one host thread at a time; separate
 * handles are independent and may run concurrently on different streams.
 *
 * Each declaration names the reference interface it replaces (path:line in BRIG-Join).
 */
#ifndef BRIG_JOIN_H_
#define BRIG_JOIN_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BRIG_JOIN_ABI_VERSION 1

/* Status codes. Replace the reference's exit-on-error CUDACHECK (src/hash_kernel.cu:48-55) and its
 * printed-only overflow/truncation report (src/hash_kernel.cu:1550-1555). */
enum brig_status {
    BRIG_OK            = 0,
    BRIG_E_INVALID     = 1,  /* bad argument: null pointer, negative size, out-of-range config */
    BRIG_E_NOMEM       = 2,  /* device or pinned host allocation failed */
    BRIG_E_CUDA        = 3,  /* CUDA runtime error (message in brig_join_last_error) */
    BRIG_E_OVERFLOW    = 4,  /* more matches than output capacity; count is exact, pairs truncated */
    BRIG_E_UNSUPPORTED = 5,  /* configuration outside the supported range */
    BRIG_E_TIMEOUT     = 6,  /* a bounded wait expired */
    BRIG_E_INTERNAL    = 7,  /* device-side consistency check failed (bounds or count mismatch) */
    BRIG_E_REJECTED    = 8,  /* serving: request can never fit the HBM budget, or loop stopped */
    BRIG_E_NOT_READY   = 9   /* serving: poll timed out before the request finished */
};

/* Partition function of both levels.
 * BRIG_PART_HASH:   radix bits of a bijective 32-bit mix of the key (default, skew-robust).
 * BRIG_PART_MODULO: (uint32)key % P at each level, the reference's layout
 *                   (src/kernel_functions.cu:66,121 first level; :187,238 second level). */
enum brig_partition_mode { BRIG_PART_HASH = 0, BRIG_PART_MODULO = 1 };

/* use_bloom values beyond the reference's on/off (see brig_join_config.use_bloom). */
#define BRIG_BLOOM_ADAPTIVE 2

/* Join configuration. Fields map onto the reference's gpu_main arguments and CLI flags
 * (src/hash_kernel.h:21-34, src/driver.cpp:66-94); zero means "choose automatically". */
typedef struct brig_join_config {
    int32_t abi_version;            /* must be BRIG_JOIN_ABI_VERSION */
    int32_t partition_mode;         /* enum brig_partition_mode */
    int32_t partition_size;         /* first-level fan-out P1 (--partition_size); 0 = auto */
    int32_t second_partition_size;  /* second-level fan-out P2 (--second_partition_size); 0 = auto,
                                       1 = single level */
    int32_t use_bloom;              /* 0 = no prefilter (use_bf 0); 1 = partitioned Bloom filter on R
                                       probed in S's first partition pass (use_bf 10/14);
                                       BRIG_BLOOM_ADAPTIVE = as 1, but a handle whose filtered
                                       single join let more than 30% of S through runs its next joins
                                       without the filter (there it costs more than it saves),
                                       testing it again every 16th run */
    int32_t bloom_num_hashes;       /* k (--num_hashes); 0 = round(bits_per_key * ln 2), max 16 */
    double  bloom_bits_per_key;     /* filter size when bloom_num_bits == 0; default 10 */
    int64_t bloom_num_bits;         /* total filter bits (--num_bits); 0 = bits_per_key * |R| */
    int32_t table_capacity;         /* max build-side tuples per shared-memory table, power of two
                                       in [256, 4096]; 0 = 4096 (the reference's HT_SIZE is 10007,
                                       src/common.h:15) */
    int32_t s_chunk;                /* max streamed tuples per probe task; 0 = 65536 */
    int32_t emit_key;               /* 1 = also write the key of each pair (GPU_answer array,
                                       src/kernel_functions.cu:422) */
    int32_t device;                 /* CUDA device ordinal; -1 = current device */
    int32_t use_cuda_graph;         /* 1 = capture the pipeline in a CUDA graph and replay it while
                                       the join shape (sizes, fan-outs) stays the same */
    int32_t profile_stages;         /* 1 = record a CUDA event after every pipeline stage (read with
                                       brig_join_stage_times); replaces the reference's chrono timers
                                       with forced syncs (src/vlsplit_hash_kernel.cu:36-107) */
    int32_t bloom_probe_level;      /* S partition pass that probes the filter: 1 = the first pass
                                       (the reference's prefilter before S's partitioning,
                                       src/hash_kernel.cu:935-954), 2 = the second pass, where each
                                       level-1 partition's filter segments stay in L2 (needs two
                                       partition levels); 0 = auto: 1 while the whole filter fits
                                       comfortably in L2, else 2 */
    int32_t max_level1_bits;        /* largest automatic level-1 fan-out, as radix bits (hash mode);
                                       0 = 9 (512 partitions) */
    int32_t s_chunks;               /* brig_join_run_host only: S is copied and joined in this many
                                       chunks against R partitioned once (the reference's s_chunks
                                       loop, src/hash_kernel.cu:910-1131), so S may exceed device
                                       memory; 0 or 1 = S in one piece */
    int32_t wait_poll_limit;        /* polls after which a kernel's bounded wait for a bulk copy gives
                                       up, counts a device-side error (the run then reports
                                       BRIG_E_INTERNAL and d_count reads -1) and waits once more, at
                                       most the default bound, for the copy in flight; 0 = 2^22 (the
                                       default), -1 = none, so every such wait reports the error at
                                       once (a test of the error path; the results stay exact). The
                                       reference's waits are unbounded (src/join_executor.cu:49) */
    int32_t partition_fill;         /* build-side tuples the planner aims for per finest partition, in
                                       percent of table_capacity (sets the level-2 fan-out; the
                                       reference aims at 8000 of its 10007 slots,
                                       src/hash_kernel.cu:240-284); 0 = 75 */
    int32_t slices_per_sm;          /* level-1 slices per SM of each launch class (the CTA work unit
                                       of the partition passes); 0 = 4 for one join, 16 for a batch */
} brig_join_config;

/* Output of one join. Pairs are written in an unspecified order; the multiset is exact. When the
 * number of matches exceeds `capacity`, the first `capacity` reserved slots are written, the count
 * stays exact and the run reports BRIG_E_OVERFLOW through brig_join_get_stats (the reference
 * writes only below d_answer_capacity, src/kernel_functions.cu:421, and counts all matches). */
typedef struct brig_join_output {
    uint32_t* r_val;     /* device [capacity]: R value of each pair (GPU_answer_val) */
    uint32_t* s_val;     /* device [capacity]: S value of each pair (GPU_answer_s_val) */
    uint32_t* key;       /* device [capacity] or NULL: key of each pair (GPU_answer) */
    int64_t   capacity;  /* number of pair slots */
    int64_t*  d_count;   /* device int64 or NULL: receives the exact match count, stream-ordered, or
                            -1 when a device-side consistency check of the run failed */
} brig_join_output;

/* What the last run did, read after it completes. */
typedef struct brig_join_stats {
    int64_t count;               /* exact number of matching pairs (GPU_answer_num) */
    int64_t written;             /* min(count, capacity) */
    int64_t s_survivors;         /* S tuples that passed the Bloom filter (= |S| when off)
                                    (BF candidate rate, src/hash_kernel.cu:1176-1179) */
    int64_t tasks;               /* probe tasks executed */
    int64_t split_tasks;         /* tasks on the oversized-partition path (probe overflow blocks,
                                    src/kernel_functions.cu:356-358) */
    int32_t overflow;            /* 1 when count > capacity */
    int32_t partition_size;      /* P1 used */
    int32_t second_partition_size;/* P2 used */
    int32_t bloom_num_hashes;    /* k used (0 when off) */
    int64_t bloom_num_bits;      /* filter bits allocated (0 when off) */
    int64_t workspace_bytes;     /* device workspace held by the handle */
} brig_join_stats;

typedef struct brig_join_t brig_join_t;

/* Fills `cfg` with defaults (hash partitioning, auto fan-outs, Bloom off, 10 bits/key). */
void brig_join_config_init(brig_join_config* cfg);

/* Creates a join handle. Replaces the set-up half of gpu_main (src/hash_kernel.cu:103-651):
 * device selection, sizing heuristics (:173-284) and buffer allocation (:370-480); buffers are
 * allocated lazily on the first run and grow as needed. */
int brig_join_create(const brig_join_config* cfg, brig_join_t** out);

/* Releases the handle and its device workspace (src/hash_kernel.cu:1609-1652). */
int brig_join_destroy(brig_join_t* h);

/* Joins R (r_key/r_val, n_r tuples) with S (s_key/s_val, n_s tuples), all device arrays, and
 * writes the pairs into `out`. Stream-ordered and asynchronous: returns after enqueueing work on
 * `stream`; inputs must stay valid until it completes. Replaces the one-PE join path of gpu_main:
 * partial_jointable_gpu_partition_r_only (src/vlsplit_hash_kernel.cu:224-255), the partitioned
 * Bloom build (src/hash_kernel.cu:670-705), queryAndCompactKernelPartitioned
 * (src/bloom.cu:725-773), partial_jointable_gpu_partition_s_only (src/vlsplit_hash_kernel.cu:258-297)
 * and join_execute_host (src/join_executor.cu:14-515). n_r or n_s may be 0. */
int brig_join_run(brig_join_t* h,
                  const uint32_t* r_key, const uint32_t* r_val, int64_t n_r,
                  const uint32_t* s_key, const uint32_t* s_val, int64_t n_s,
                  const brig_join_output* out, void* stream);

/* End-to-end form over HOST arrays: copies R and S to the device (pinned host memory is fastest),
 * joins, copies the pairs back into host arrays out_r_val/out_s_val (and out_key if not NULL) of
 * `capacity` entries and stores the exact count in *count. Synchronous. This is the reference's
 * measured "Total" region, which starts at the host-to-device copies (src/hash_kernel.cu:637-641,
 * 923-926). Returns BRIG_E_OVERFLOW when the count exceeds capacity (pairs truncated). */
int brig_join_run_host(brig_join_t* h,
                       const uint32_t* r_key, const uint32_t* r_val, int64_t n_r,
                       const uint32_t* s_key, const uint32_t* s_val, int64_t n_s,
                       uint32_t* out_r_val, uint32_t* out_s_val, uint32_t* out_key,
                       int64_t capacity, int64_t* count, void* stream);

/* Waits for the handle's last run and reports its statistics (the PE0 summary of
 * src/hash_kernel.cu:1142-1156,1550-1555). Returns BRIG_E_OVERFLOW if that run overflowed and
 * BRIG_E_INTERNAL if a device-side consistency check failed. */
int brig_join_get_stats(brig_join_t* h, brig_join_stats* st);

/* Pipeline stages timed when profile_stages is set, in execution order. */
#define BRIG_NUM_STAGES 13
/* Name of stage i ("r_hist", "r_scan", "r_scatter", "r_l2_hist", "r_l2_scatter", "bloom_build",
 * "s_hist_probe", "s_scan", "s_scatter", "s_l2_hist", "s_l2_scatter", "tasks", "probe"), or NULL. */
const char* brig_join_stage_name(int32_t i);
/* Waits for the last run and writes the mean device time of each stage in milliseconds, over
 * the runs since the previous call (at most the last 64), into ms[BRIG_NUM_STAGES] (the
 * reference's per-stage timing table, src/hash_kernel.cu:1182-1358). Reading needs no
 * synchronisation between runs. A profiled handle launches its kernels directly instead of
 * replaying a CUDA graph. BRIG_E_INVALID if the handle was created without profile_stages or
 * no run happened since the previous call. */
int brig_join_stage_times(brig_join_t* h, double* ms, int32_t n);

/* Device workspace the engine needs for one join of this shape (the reference's allocation plan,
 * src/hash_kernel.cu:370-480), with the fan-outs the planner picks. */
int brig_join_plan(const brig_join_config* cfg, int64_t n_r, int64_t n_s,
                   int32_t* partition_size, int32_t* second_partition_size,
                   int64_t* workspace_bytes);

/* ---- Batched joins: many independent joins in one pipeline ------------------------------------
 * No reference counterpart (the nearest is the S chunk loop, src/hash_kernel.cu:910-1131). All
 * joins of a batch are partitioned by the same kernels and probed by one persistent work-queue
 * kernel over (join, partition-pair) tasks; the pipeline is captured in a CUDA graph and replayed
 * when a batch of the same shape runs again. */
typedef struct brig_join_batch_item {
    const uint32_t* r_key; const uint32_t* r_val; int64_t n_r;
    const uint32_t* s_key; const uint32_t* s_val; int64_t n_s;
    brig_join_output out;
} brig_join_batch_item;

/* Runs `n_items` joins, stream-ordered and asynchronous. */
int brig_join_run_batch(brig_join_t* h, const brig_join_batch_item* items, int32_t n_items,
                        void* stream);

/* Waits for the last batch and copies its per-join exact counts into counts[n_items]. Returns
 * BRIG_E_OVERFLOW if any join exceeded its capacity. */
int brig_join_batch_counts(brig_join_t* h, int64_t* counts, int32_t n_items);

/* Tunes the handle's configuration on the given batch and keeps the fastest: a coordinate search,
 * one dimension at a time from the handle's configuration, over the Bloom prefilter (off; 8 bits/key,
 * k = 6; 10 bits/key, k = 7, probe level chosen by the planner or in S's second pass), the
 * shared-memory table capacity, the largest level-1 radix bits, partition_fill (the level-2 fan-out)
 * and slices_per_sm, each candidate timed as the median of three runs after a warm-up, repeated while
 * a pass improves the time by more than 2% (at most three passes). The chosen configuration is copied
 * to *chosen when not NULL. Results of the timing runs are discarded (outputs are overwritten); no
 * candidate changes the result of a join, only its speed. The reference has no autotuner; its
 * sizing is fixed heuristics (src/hash_kernel.cu:198-284). */
int brig_join_autotune(brig_join_t* h, const brig_join_batch_item* items, int32_t n_items, void* stream,
                       brig_join_config* chosen);

/* The configurations the autotuner may try from `base` (each dimension's values with the others at
 * base): writes up to `max` of them to out and their number to *n. */
int brig_join_autotune_candidates(const brig_join_config* base, brig_join_config* out, int32_t max, int32_t* n);

/* ---- Served joins: continuous batching under an HBM budget ------------------------------------
 * No reference counterpart. Requests are admitted while their device footprint fits the budget;
 * admitted requests are grouped into waves that run on several streams, so a request that arrives
 * while others are on the GPU starts in the next wave without waiting for them to finish. */
typedef struct brig_serve_config {
    int64_t hbm_budget_bytes;  /* admission budget for request footprints; 0 = 120 GB */
    int32_t max_wave;          /* max joins per wave; 0 = 64 */
    int32_t streams;           /* concurrent waves; 0 = 2 */
    int32_t max_queue;         /* pending requests before submit rejects; 0 = 4096 */
    int32_t max_wave_mtuples;  /* a wave stops growing at this many million tuples (|R|+|S| summed);
                                  a larger request runs as a wave of its own; 0 = 256 */
    int32_t large_mtuples;     /* requests above this many million tuples are large: they run one at
                                  a time (never two on the GPU together) on the first stream, and
                                  smaller requests may pass one that waits; 0 = max_wave_mtuples */
    int32_t reserved[3];
} brig_serve_config;

/* One request. Inputs are HOST arrays (copied in by the server) or device arrays when
 * `inputs_on_device` is 1. The server allocates the device output; results are copied back to
 * host arrays out_r_val/out_s_val of `capacity` entries when they are not NULL. */
typedef struct brig_serve_request {
    const uint32_t* r_key; const uint32_t* r_val; int64_t n_r;
    const uint32_t* s_key; const uint32_t* s_val; int64_t n_s;
    int32_t  inputs_on_device;
    int32_t  reserved0;
    uint32_t* out_r_val;  /* host [capacity] or NULL */
    uint32_t* out_s_val;  /* host [capacity] or NULL */
    int64_t  capacity;    /* output capacity; 0 = n_s (every S tuple matches at most once) */
} brig_serve_request;

typedef struct brig_serve_result {
    int32_t status;        /* BRIG_OK, BRIG_E_OVERFLOW, ... for this request */
    int32_t wave;          /* wave index the request ran in */
    int64_t count;         /* exact match count */
    double  submit_to_done_ms;  /* latency: submit -> results available */
    double  queue_ms;           /* submit -> start of its wave */
    double  setup_ms;           /* start of its wave -> the wave's work enqueued (buffers, workspace) */
    double  join_ms;            /* work enqueued -> the join finished on the device */
} brig_serve_result;

typedef struct brig_serve_t brig_serve_t;

int brig_serve_create(const brig_join_config* jcfg, const brig_serve_config* scfg,
                      brig_serve_t** out);
/* Queues a request; returns a ticket. Input arrays must stay valid until the request completes.
 * BRIG_E_REJECTED when the request alone exceeds the budget or the queue is full. */
int brig_serve_submit(brig_serve_t* s, const brig_serve_request* req, int64_t* ticket);
/* Waits up to timeout_ms (-1 = forever) for a ticket; BRIG_E_NOT_READY on timeout. A ticket is
 * released after it is returned once. */
int brig_serve_poll(brig_serve_t* s, int64_t ticket, int32_t timeout_ms, brig_serve_result* res);
/* Drains in-flight waves, rejects queued requests and frees everything. */
int brig_serve_destroy(brig_serve_t* s);

/* ---- Synthetic inputs (the analogue of datagen/gen_dataset.cpp) -------------------------------
 * R keys: distinct pseudo-random values in [1, 2^31); S keys: a fraction `match_frac` of rows take
 * a key drawn uniformly (with replacement) from R's keys, the other rows take distinct keys in
 * [2^31, 2^32-1); values are row indices. Deterministic in (seed, row), identical on host and
 * device. zipf_s > 0 draws the matching S keys with Zipf(s) skew over R's row order instead. */
int brig_gen_device(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s,
                    uint32_t* r_key, uint32_t* r_val, uint32_t* s_key, uint32_t* s_val,
                    void* stream);
int brig_gen_host(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s,
                  uint32_t* r_key, uint32_t* r_val, uint32_t* s_key, uint32_t* s_val);

/* ---- Allocation-free join ----------------------------------------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device memory when they join:
 * host frameworks that own all device memory through their own pool and forbid their operators to
 * allocate outside it, and latency-critical callers that cannot afford the device-wide
 * synchronisation of cudaMalloc/cudaFree. Same kernels and result as brig_join_run, but every
 * intermediate buffer lives in one static device array of BRIG_NOALLOC_SCRATCH_BYTES that each GPU
 * loading the library holds until the process exits; no handle, no cudaMalloc/cudaFree/
 * cudaMallocHost. Limit: at most BRIG_NOALLOC_MAX_TUPLES tuples per relation, and the join's layout
 * must fit the array (the default planner and the modulo preset with partition_size 512 do);
 * larger requests return BRIG_E_UNSUPPORTED. The count is written to out->d_count (required), or -1
 * when a device-side consistency check failed (there is no handle to report BRIG_E_INTERNAL through).
 * The first call on a device looks up the array's address and sets the kernels' attributes on that
 * device. It must not be called under stream capture (it returns BRIG_E_UNSUPPORTED there): its
 * descriptor upload reads a stack buffer that a replayed graph could not reach. All calls on a
 * device share the array and it keeps the last call's contents (the pipeline clears what must start
 * at zero); calls whose work overlaps on the GPU race on it, so order them on one stream or with
 * events. */
#define BRIG_NOALLOC_MAX_TUPLES 262144
#define BRIG_NOALLOC_SCRATCH_BYTES (16u << 20)
int brig_join_run_noalloc(const brig_join_config* cfg,
                          const uint32_t* r_key, const uint32_t* r_val, int64_t n_r,
                          const uint32_t* s_key, const uint32_t* s_val, int64_t n_s,
                          const brig_join_output* out, void* stream);

/* ---- The reference's file formats (host arrays, no device work) -------------------------------
 * Reads one relation in the reference's input layout: headerless little-endian int32, the n keys
 * followed, when read_val is 1, by the n values (datagen/gen_dataset.cpp writes the key block;
 * gpu_main reads both blocks with --read_val 1, src/hash_kernel.cu:300-335). With read_val 0 and
 * vals not NULL, vals[i] = val_base + i: the reference's synthesised payloads are row + 1 for R
 * (val_base 1) and row + 100000001 for S. BRIG_E_INVALID when the file is shorter than asked. */
int brig_join_read_relation(const char* path, int64_t n, int32_t read_val, uint32_t val_base,
                            uint32_t* keys, uint32_t* vals);

/* Writes n pairs to `path` in the same headerless int32 block layout: the keys (when key is not
 * NULL), then the R values, then the S values. The reference parses an output path and never
 * writes it (src/driver.cpp:50,119); this is the writer it lacks. */
int brig_join_write_pairs(const char* path, const uint32_t* key, const uint32_t* r_val, const uint32_t* s_val,
                          int64_t n);

/* ---- Sharded joins across GPUs: key ownership ------------------------------------------------
 * The local steps of a join whose relations are spread over nranks GPUs, one process per GPU; the
 * exchanges between the steps are the caller's (NCCL all-to-all and all-gather; brig_join.shard in
 * the Python package is one such caller). Replaces the reference's multi-PE path: the ownership
 * shuffle of R and of the prefiltered S (src/r_shuffle.cu:33-191), the Bloom filter merge
 * (src/bf_allreduce.cu:236-284) and, for skewed inputs, S' rebalancing and R replication
 * (src/s_redistribute.cu:26-152, src/r_replicate.cu:13-100). Per rank:
 *   1. brig_shard_count + brig_shard_scatter on its R: R grouped into owner bins; bin r goes to rank
 *      r (all-to-all), the heavy bin (below) to every rank (all-gather);
 *   2. brig_shard_bloom_build over the R tuples it received: its owner's filter of
 *      brig_shard_filter_words words; the filters are gathered on every rank (they cover disjoint
 *      keys, so no OR reduction is needed) and located by filter_loc;
 *   3. brig_shard_count + brig_shard_scatter on its S with the gathered filters: only S tuples that
 *      pass their owner's filter are kept; bin r goes to rank r, the heavy bin stays;
 *   4. brig_join_run of its owned R with the S it received, and of the gathered heavy R with the
 *      heavy S it kept.
 * Each output pair comes out on exactly one rank. A key's owner is brig_shard_owner(key, nranks), a
 * hash independent of the engine's partition bits. Heavy keys are a sorted list of distinct keys
 * that every rank passes alike; their tuples go to bin nranks and skip the filter. */
#define BRIG_SHARD_MAX_RANKS 64
#define BRIG_SHARD_MAX_HEAVY 1024
typedef struct brig_shard_spec {
    int32_t nranks;              /* owners, 1..BRIG_SHARD_MAX_RANKS */
    int32_t bloom_num_hashes;    /* k of the owners' filters (1..16) when filter is not NULL */
    const uint32_t* filter;      /* device: every owner's filter words (8-byte aligned), or NULL */
    const int64_t* filter_loc;   /* device int64[2 * nranks]: word offset (even) and word count of
                                    owner r's filter in `filter`; a count below 8, or an odd or
                                    negative offset, drops the owner's tuples */
    const uint32_t* heavy;       /* device: sorted distinct heavy keys, or NULL */
    int32_t n_heavy;             /* 0..BRIG_SHARD_MAX_HEAVY */
    int32_t reserved;
    uint8_t* bin_cache;          /* device uint8[n] or NULL: brig_shard_count stores each tuple's bin
                                    (0xff: dropped) and brig_shard_scatter, given the same spec and
                                    inputs, reads it instead of testing the filters again */
} brig_shard_spec;

/* Owner of `key` among nranks ranks (host), or -1 when nranks is out of range. */
int32_t brig_shard_owner(uint32_t key, int32_t nranks);
/* Words of an owner's filter for n_keys R tuples at bits_per_key (a multiple of 8, at least 8), or
 * -1 for a bad argument or a filter of 2^32 words or more. */
int64_t brig_shard_filter_words(int64_t n_keys, double bits_per_key);
/* Counts the tuples of each bin: counts (device int64[nbins], nbins = nranks + (n_heavy > 0)) is
 * zeroed and filled, stream-ordered. */
int brig_shard_count(const brig_shard_spec* sp, const uint32_t* key, int64_t n, int64_t* counts, void* stream);
/* Writes the tuples grouped by bin, bin b at [start_b, start_b + counts[b]) of out_key/out_val
 * (start = exclusive scan of counts, which must come from brig_shard_count on the same inputs and
 * spec; the outputs hold their sum). scratch: device int64[2 * nbins + 2]; scratch[0..nbins] receives
 * the bin starts and the total, and scratch[2 * nbins + 1] the number of tuples that found their bin
 * full (0 unless the inputs changed since the count). Tuples keep no order inside a bin. */
int brig_shard_scatter(const brig_shard_spec* sp, const uint32_t* key, const uint32_t* val, int64_t n,
                       const int64_t* counts, int64_t* scratch, uint32_t* out_key, uint32_t* out_val, void* stream);
/* Builds an owner's filter over n keys into words[n_words] (device, 8-byte aligned, n_words a
 * multiple of 8; zeroed first): the engine's blocked filter of word pairs with one segment, k =
 * num_hashes (the per-partition build of the reference, src/bloom.cu:698-722, over the owned keys). */
int brig_shard_bloom_build(const uint32_t* key, int64_t n, uint32_t* words, int64_t n_words, int32_t num_hashes,
                           void* stream);

/* Message for the last failed call on this thread (empty string if none). */
const char* brig_join_last_error(void);

/* Number of kernel launches issued by this thread since process start (all handles). */
int64_t brig_join_kernel_launches(void);

/* Measurement helper, with no counterpart in the reference: enqueues on `stream` one kernel that
 * performs about `loads` independent 8-byte reads at pseudo-random positions of `table` (a device
 * array of `table_bytes` bytes, a power of two of at least 256, 8-byte aligned; small enough to stay
 * in L2, like one level-1 partition's Bloom segments) and nothing else, two 512-thread CTAs per SM.
 * The reads each touch their own cache line, as the level-2 Bloom probe's filter reads do, so the
 * kernel's rate (time it with events around the call) is the ceiling of that probe. *loads_issued
 * receives the exact number of reads enqueued; `sink` (one device word) is written only if the
 * reads' checksum hits one fixed value. */
int brig_join_gather_rate(const void* table, int64_t table_bytes, int64_t loads, uint32_t* sink,
                          int64_t* loads_issued, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BRIG_JOIN_H_ */
