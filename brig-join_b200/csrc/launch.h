// launch.h - host-side launch wrappers for the sm_100a kernels (defined in kernels.cu, gen.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "brig_common.cuh"

namespace brig {

// Launch-time description of one pipeline run over `nj` joins. Every pointer is a device address.
struct PipelineArgs {
    const JoinDesc* J;            // [nj]
    int nj;
    const int64_t* slice_prefix[2];   // [nj+1] per relation: level-1 slices of joins before j
    const int64_t* seg_prefix;        // [nj+1] level-1 partitions of joins with P2 > 1 (per relation
                                      // the same count)
    const int64_t* fine_prefix;       // [nj+1] finest partitions of joins before j
    const int64_t* bloom_prefix;      // [nj+1] Bloom build groups of joins before j
    const int64_t* dom_prefix;        // [nj+1] task domains of joins before j
    int64_t total_slices[2];
    int64_t total_segs;               // sum of P1 over joins with P2 > 1
    int64_t total_fine;               // sum of P1*P2
    int64_t total_bloom_groups;       // Bloom build groups over all joins
    int64_t total_domains;            // task domains over all joins
    int bloom_smem_words;             // shared-memory words of one Bloom build group
    int64_t hist_begin[2], hist_len[2];  // range of each relation in the global histogram array
    uint32_t* hist;                   // global level-1 histogram array (both relations)
    int64_t* hist_scan;               // exclusive scan of hist (same indexing)
    uint32_t* tcount;                 // [total_fine + 1] tasks per finest partition
    int64_t* toff;                    // exclusive scan of tcount
    Task* tasks;                      // task list
    int64_t task_cap;
    int64_t* scan_tmp;                // block sums for the device-wide scan
    int64_t scan_tmp_len;
    unsigned long long* gwords;       // [kGWords]
    int max_p1, max_p2;               // over the batch (shared-memory sizing)
    int max_seg_words;                // largest Bloom segment (words)
    int table_cap;                    // probe table capacity (tuples)
    int emit_key;
    int any_bloom;
    int any_bloom_l1;                 // some join probes its filter in S's first pass
    int any_bloom_l2;                 // some join probes its filter in S's second pass
    int all_bloom_l2;                 // every two-level join probes its filter in S's second pass
    int modes;                        // partition modes present: bit 0 hash, bit 1 modulo
    int kclasses;                     // Bloom mask classes present: bit 0 pattern table (or no filter),
                                      // bit 1 compile-time k = 7
    int pat_k;                        // k the Bloom kernels fill their pattern tables for (0: none)
    int num_sms;
    cudaEvent_t* stage_events;        // [kNumStages + 1] or nullptr
    cudaEvent_t s_ready;              // when set, S's passes wait for it (its inputs are still arriving)
    int keep_errors;                  // 1: the error word keeps the counts of earlier launches of the run
    uint32_t wait_polls;              // first bound of the kernels' bounded waits (polls)
    int stages;                       // kRunPartR | kRunBloom | kRunPartS | kRunProbe
    // level 2 (planned on the device)
    uint32_t* seg_ns;                 // [total_segs + 1] slices per level-1 partition
    int64_t* seg_off;                 // [total_segs + 1] their exclusive scan
    uint32_t* hist2;                  // level-2 histograms of both relations
    int64_t* hist2_scan;              // their exclusive scan
    int64_t h2_begin[2], h2_len[2];   // range of each relation in hist2
    uint32_t* slice_cnt2;             // [max slices] survivors per slice (level-2 Bloom probe)
    int64_t l2_slice_cap[2];          // upper bound of level-2 slices per relation
    int l1_form[2], l2_form[2];       // ScatterForm of each relation's level-1 and level-2 scatters
};

// Pipeline parts (a full join runs all four; the reference-named entry points run subsets).
enum RunPart : int { kRunPartR = 1, kRunBloom = 2, kRunPartS = 4, kRunProbe = 8, kRunAll = 15 };

constexpr int kNumStages = 13;
constexpr int kBloomSmemWords = 12288;  // 48 KB of Bloom segments per build CTA
const char* stage_name(int i);

// Enqueues the full join pipeline (partition, Bloom, tasks, probe) for all joins on `stream`.
cudaError_t enqueue_pipeline(const PipelineArgs& a, cudaStream_t stream);

// Shared memory the probe kernel needs for a table of `table_cap` tuples.
size_t probe_smem_bytes(int table_cap, int emit_key);

// Device-wide exclusive scan of n uint32 counts into int64 offsets; writes the sum to *total
// (device pointer, may be null). tmp must hold scan_tmp_words(n) int64.
int64_t scan_tmp_words(int64_t n);
cudaError_t enqueue_scan(const uint32_t* in, int64_t* out, int64_t n, int64_t* tmp,
                         int64_t* total, cudaStream_t stream);

// Input generator (gen.cu).
cudaError_t enqueue_gen(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s,
                        uint32_t* r_key, uint32_t* r_val, uint32_t* s_key, uint32_t* s_val,
                        cudaStream_t stream);

// Count of kernel launches issued by this library on the calling thread. Launches enqueued while a
// stream is being captured are not counted; each replay of a graph adds the kernels it holds.
void note_launches(int n);
int64_t launches_so_far();
void set_capturing(bool on);   // while on, note_launches adds to the capture tally instead
int64_t take_capture_tally();  // kernels noted since set_capturing(true)

}  // namespace brig
