// engine.h - host-side join engine: planner, workspace, pipeline enqueue, CUDA-graph cache.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/brig_join.h"
#include "brig_common.cuh"
#include "launch.h"

namespace brig {

// Thrown inside the engine; the C ABI turns it into a status code and a message.
struct Error {
    int status;
    std::string msg;
};
[[noreturn]] void fail(int status, const std::string& msg);
// Message returned by brig_join_last_error() on the calling thread.
void set_last_error(const std::string& msg);
void cuda_check(cudaError_t e, const char* what);

// Fan-outs and Bloom sizing of one join (the reference's sizing heuristics,
// src/hash_kernel.cu:188-284).
struct JoinPlan {
    int64_t nr = 0, ns = 0;
    PartFn pf{};
    int64_t nfine = 1;
    bool bloom = false;
    int bloom_level = 0;        // S pass that probes the filter (1 or 2)
    int bloom_group = 1;        // consecutive finest partitions per Bloom build CTA
    int k = 0;
    uint32_t seg_blocks = 0;
    int64_t bloom_bits = 0;     // allocated bits
};
JoinPlan plan_join(const brig_join_config& cfg, int64_t nr, int64_t ns);
// Plans of the joins of one pipeline run: plan_join for each, then (with bloom_probe_level 0, and
// more than one join or an L2 shared with other runs in flight) the largest two-level joins move
// their Bloom probe to S's second pass until the filters probed in the first pass fit the shared
// L2 budget together.
std::vector<JoinPlan> plan_batch(const brig_join_config& cfg, const int64_t* nr, const int64_t* ns, int nj,
                                 bool shared_l2 = false);

// One join of a pipeline run, as given by the caller.
struct JoinIO {
    const uint32_t *rk, *rv, *sk, *sv;
    int64_t nr, ns;
    brig_join_output out;
};

// Byte offsets of one relation's buffers inside a pipeline workspace.
struct RelOffs {
    size_t l1 = 0, l2 = 0, cmp = 0, b1 = 0, bounds = 0, slice_cnt = 0;
    int64_t h2_base = 0;
    int64_t slice_len = 0;
    int32_t nslices = 0;
    int64_t hist_base = 0;
    int64_t l2_slice = 0;  // tuples per level-2 slice
};
struct JoinOffs {
    RelOffs rel[2];
    size_t bloom = 0;
};

// Workspace layout of one pipeline run (all offsets relative to the workspace base).
struct Shape {
    JoinOffs* jo = nullptr;      // [nj], caller-owned
    int64_t slice_len = 0;
    int64_t hist_len[2] = {0, 0};
    int64_t total_slices[2] = {0, 0};
    int64_t total_segs = 0, total_fine = 0, total_bloom_groups = 0, total_domains = 0;
    int64_t task_cap = 0;
    size_t hist = 0, hist_scan = 0, tcount = 0, toff = 0, tasks = 0, scan_tmp = 0, gwords = 0,
           counters = 0, meta = 0;
    size_t seg_ns = 0, seg_off = 0, hist2 = 0, hist2_scan = 0, slice_cnt2 = 0;
    int64_t h2_len[2] = {0, 0};
    int64_t l2_slice_cap[2] = {0, 0};
    int64_t scan_tmp_len = 0;
    size_t meta_bytes = 0;      // descriptor image: nj JoinDesc + 5 prefix arrays of nj+1 int64
    size_t total = 0;           // workspace bytes
    int max_p1 = 1, max_p2 = 1, max_seg_words = 0, bloom_smem_words = 0;
    bool any_bloom = false;
    bool any_bloom_l1 = false;
    bool any_bloom_l2 = false;
};

// Lays out `nj` joins in one workspace; fills jo[0..nj) and sh. Allocates nothing.
void layout_for(const brig_join_config& cfg, const JoinPlan* plans, int nj, int num_sms, JoinOffs* jo,
                Shape& sh);

// Writes the descriptor image for the joins into meta_host (sh.meta_bytes bytes of host memory,
// to be copied to ws + sh.meta) and the launch arguments into `a`. Allocates nothing.
void fill_pipeline(const brig_join_config& cfg, const JoinPlan* plans, const JoinIO* joins, int nj,
                   const Shape& sh, char* ws, char* meta_host, int num_sms, PipelineArgs& a);

// The autotuner's search space (Engine::autotune): kTuneDims dimensions, each with tune_values(dim)
// values; tune_apply(base, dim, v) is base with dimension dim set to its v-th value.
constexpr int kTuneDims = 5;
int tune_values(int dim);
brig_join_config tune_apply(const brig_join_config& base, int dim, int v);
std::vector<brig_join_config> autotune_candidates(const brig_join_config& base);

class Engine {
public:
    explicit Engine(const brig_join_config& cfg);
    ~Engine();

    // Enqueues all joins on `stream` (asynchronous). With `s_ready`, the S passes wait for that
    // event while R's passes and the Bloom build run (no graph: the event lives outside it).
    void run(const std::vector<JoinIO>& joins, cudaStream_t stream, bool use_graph,
             cudaEvent_t s_ready = nullptr);
    // Times candidate configurations on `joins`, keeps the fastest in the handle and returns it.
    brig_join_config autotune(const std::vector<JoinIO>& joins, cudaStream_t stream);
    // Waits for the last run; copies per-join counters.
    void sync_counters(std::vector<int64_t>& counters, int64_t& errors);
    const std::vector<JoinPlan>& last_plans() const { return plans_; }
    int64_t workspace_bytes() const { return (int64_t)ws_bytes_; }
    // Grows the workspace to at least `bytes`, stream-ordered on `stream` (after the last run).
    void reserve_workspace(size_t bytes, cudaStream_t stream) {
        if (have_run_ && bytes > ws_bytes_) cuda_check(cudaStreamWaitEvent(stream, done_, 0), "cudaStreamWaitEvent");
        ensure_workspace(bytes, stream);
    }
    const brig_join_config& config() const { return cfg_; }
    // Runs of this engine share the GPU's L2 with other engines' runs in flight (the serving
    // loop's slots): first-pass Bloom probes keep to the shared budget even for one join.
    void set_shared_l2(bool on) { shared_l2_ = on; }
    bool shared_l2() const { return shared_l2_; }
    int device() const { return device_; }
    const std::vector<int64_t>& last_caps() const { return caps_; }
    // Mean milliseconds of each pipeline stage over the runs since the previous call (at most the
    // last kStageRing); returns the number of runs averaged (profile_stages only).
    int stage_times(double* ms, int n);

    // Device workspace needed for these joins (bytes).
    static int64_t workspace_needed(const brig_join_config& cfg, const std::vector<JoinPlan>& plans,
                                    int num_sms);

    // Buffers owned by the engine for the host-array entry point.
    struct HostIOBufs {
        uint32_t *rk = nullptr, *rv = nullptr, *sk = nullptr, *sv = nullptr;
        uint32_t *outr = nullptr, *outs = nullptr, *outk = nullptr;
        int64_t cap_in_r = 0, cap_in_s = 0, cap_out = 0;
        bool outk_alloc = false;
    } hio;
    void ensure_host_io(int64_t nr, int64_t ns, int64_t cap, bool key);
    // Stream and events of the host-array entry point: S's inputs are copied on copy_stream after
    // R's (r_copied) while R's passes run; s_copied marks their arrival. With S in chunks, chunk c
    // goes to buffer c % 2 (chunk_copied marks its arrival, chunk_free the end of its passes).
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t r_copied = nullptr, s_copied = nullptr;
    cudaEvent_t chunk_copied[2] = {}, chunk_free[2] = {};
    // With S in chunks: the match count after chunk c's probe (pinned, chunk_count[c]) and an event
    // after its read-back (chunk_done[c]), so each chunk's pairs can be copied back on d2h_stream
    // while later chunks are copied in and joined (the link carries both directions at once).
    std::vector<cudaEvent_t> chunk_done;
    int64_t* chunk_count = nullptr;
    int chunk_count_cap = 0;
    int chunks_run = 0;
    cudaStream_t d2h_stream = nullptr;

    // Host-array join with S in `chunks` pieces (brig_join_config.s_chunks): R is copied, partitioned
    // and filtered once; each S chunk is copied into one of two device buffers on copy_stream while
    // the previous chunk's S passes and probe run on `stream` against the resident R, appending its
    // pairs to the handle's host-io output buffers. Asynchronous; read the count with
    // sync_counters.
    void run_host_chunked(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk,
                          const uint32_t* sv, int64_t ns, int chunks, int64_t cap, bool emit_key,
                          cudaStream_t stream);

private:
    void ensure_workspace(size_t bytes, cudaStream_t stream);
    void ensure_staging(size_t bytes);

    brig_join_config cfg_;
    int device_ = 0;
    int num_sms_ = 148;
    char* ws_ = nullptr;
    size_t ws_bytes_ = 0;
    char* stage_ = nullptr;          // pinned staging for descriptors
    size_t stage_bytes_ = 0;
    cudaEvent_t stage_free_ = nullptr;  // recorded after the staging copy
    cudaEvent_t done_ = nullptr;        // recorded after the last run
    bool have_run_ = false;
    bool shared_l2_ = false;
    std::vector<JoinPlan> plans_;
    std::vector<int64_t> caps_;
    int64_t* d_counters_ = nullptr;  // [nj * kCntWords] of the last run
    unsigned long long* d_gwords_ = nullptr;
    int nj_ = 0;

    // The adaptive filter (use_bloom == BRIG_BLOOM_ADAPTIVE, single joins): the survivor count of
    // the last filtered run comes back into pinned memory behind the run; while the last measured
    // share of S passing the filter is above the break-even, runs plan without the filter, and every
    // kBloomRetest-th of them tests it again.
    int64_t* surv_host_ = nullptr;
    cudaEvent_t surv_ev_ = nullptr;
    bool surv_pending_ = false;
    int64_t surv_ns_ = 0;
    bool bloom_off_ = false;
    int runs_off_ = 0;
    // The configuration the next run of `nj` joins plans with.
    brig_join_config adapt_config(int nj);
    // Queues the read-back of a filtered single join's survivor count (adaptive filter only).
    void note_survivors(const std::vector<JoinPlan>& plans, const int64_t* counters, cudaStream_t stream);

    // Stage events of the last kStageRing runs (profile_stages): run i records into set i % ring.
    static constexpr int kStageRing = 64;
    cudaEvent_t stage_ev_[kStageRing][kNumStages + 1] = {};
    int64_t runs_recorded_ = 0, runs_read_ = 0;
    bool profiling_ = false;

    // CUDA graph of the last pipeline shape.
    int64_t graph_kernels_ = 0;      // kernel launches one replay performs
    cudaGraphExec_t graph_exec_ = nullptr;
    std::vector<int64_t> graph_key_;
    cudaStream_t graph_stream_ = nullptr;
};

}  // namespace brig
