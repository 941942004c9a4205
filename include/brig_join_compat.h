/*
 * brig_join_compat.h - C++ entry points with the reference's names and signatures, implemented by
 * libbrigjoin.so, so BRIG-Join's own host code (src/driver.cpp, or a hash_kernel.cu that keeps its
 * orchestration) can link against the engine in place of the reference's local join. Declarations
 * are re-typed from the reference headers, each cited. Semantics are those of one PE: every
 * multi-GPU argument is accepted and ignored (with a note on stderr), since exchanges across GPUs
 * are not part of this engine.
 *
 * Layout contract (as the reference): keys and values are separate int arrays; partitioning is
 * in place, by (unsigned)key % partition_size then (unsigned)key % second_partition_size; the
 * level-1 index d_block_index_split[p] is the inclusive end of bucket p, the level-2 index
 * d_second_index_split[p * sp + q] the inclusive end of sub-bucket q relative to bucket p's start.
 */
#ifndef BRIG_JOIN_COMPAT_H_
#define BRIG_JOIN_COMPAT_H_

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <string>
#include <vector>

/* Tuning globals of the reference (src/common.h:8-13, defaults src/hash_kernel.cu:38-43). The
 * partition entry points read partition_size and second_partition_size; thread_no, block_no,
 * block_size and chunk_size are accepted for source compatibility and not used. */
extern int partition_size;
extern int second_partition_size;
extern int thread_no;
extern int block_no;
extern int block_size;
extern int chunk_size;

/* Slices the host tables into one contiguous part per device (src/hash_kernel.h:12-19). */
void split_tables(int device_num, int* const tableA, int* const tableB, int* const tableA_val,
                  int* const tableB_val, long long* tableA_size, long long* tableB_size, int** tableA_split,
                  int** tableB_split, int** tableA_val_split, int** tableB_val_split, const long long R,
                  const long long S);

/* The whole local join from files (src/hash_kernel.h:21-34). Reads R and S (int32 keys, then a value
 * block when read_val != 0, else values row+1 and row+100000001 as src/hash_kernel.cu:330-336),
 * joins them on the current GPU in s_chunks chunks of S and prints the grand total the way the
 * reference does (src/hash_kernel.cu:1153). use_bf != 0 turns the Bloom prefilter on, sized from
 * true_false_ratio or override_num_bits / override_num_hashes (src/hash_kernel.cu:189-196);
 * override_partition_size / override_second_partition_size select the reference's modulo layout;
 * answer_scale sizes the pair buffer (src/hash_kernel.cu:471). When sanityCheck is set and the
 * program also links the reference's run_sanity_check, that CPU check runs first. */
void gpu_main(std::vector<int>* solution, std::vector<int>* solution_ref, const std::string& r_inputPath,
              const std::string& s_inputPath, long long R, long long S, int use_bf = 0, bool use_nvlink = false,
              bool use_warp_compact = false, double true_false_ratio = 0.5, int s_chunks = 1,
              bool sanityCheck = false, int kernel_fusion = 0, double redist_skew_threshold = 0.0,
              long long override_num_bits = -1, int override_num_hashes = -1, int override_partition_rs_split = -1,
              int override_partition_size = -1, int override_second_partition_size = -1,
              int fused_probe_breakdown = 0, int read_val = 0, int r_shuffle_enable = 0,
              double r_replicate_ratio = -1.0, double answer_scale = 1.0);

/* Two-level partition of R and S in place (src/vlsplit_hash_kernel.h:15-24). d_oa_data/d_ob_data and
 * their value arrays are scratch; d_b_kv_out, when not null, also receives S as (key, value) pairs.
 * d_a_prefix_data[p] gets bucket p's count and d_a_offset[p] its end (likewise for S). */
void partial_jointable_gpu_partition(
    const int* const d_adata, const int* const d_bdata, int* const d_oa_data, int* const d_ob_data,
    int* const d_a_val, int* const d_b_val, int* const d_oa_val, int* const d_ob_val, int2* const d_b_kv_out,
    long long* const d_a_prefix_data, long long* const d_b_prefix_data, long long* const d_block_index_split_r,
    long long* const d_block_index_split_s, long long* const d_a_offset, long long* const d_b_offset,
    long long* const d_second_index_split_r, long long* const d_second_index_split_s, int* const d_answer_num,
    const long long R, const long long S, cudaStream_t gpu_stream, cudaEvent_t gpu_event,
    double& out_partition_sec, double& out_hist_sec, bool skip_r_hist = false);

/* The same with R and S timed separately (src/vlsplit_hash_kernel.h:27-36). */
void partial_jointable_gpu_partition_rs_split(
    const int* const d_adata, const int* const d_bdata, int* const d_oa_data, int* const d_ob_data,
    int* const d_a_val, int* const d_b_val, int* const d_oa_val, int* const d_ob_val, int2* const d_b_kv_out,
    long long* const d_a_prefix_data, long long* const d_b_prefix_data, long long* const d_block_index_split_r,
    long long* const d_block_index_split_s, long long* const d_a_offset, long long* const d_b_offset,
    long long* const d_second_index_split_r, long long* const d_second_index_split_s, int* const d_answer_num,
    const long long R, const long long S, cudaStream_t gpu_stream, cudaEvent_t gpu_event,
    double& out_partition_sec, double& out_partition_r_sec, double& out_partition_s_sec, double& out_hist_r_sec,
    double& out_hist_s_sec, bool skip_r_hist = false);

/* R only, in place (src/vlsplit_hash_kernel.h:39-44). */
void partial_jointable_gpu_partition_r_only(int* const d_adata, int* const d_oa_data, int* const d_a_val,
                                            int* const d_oa_val, long long* const d_a_prefix_data,
                                            long long* const d_block_index_split_r, long long* const d_a_offset,
                                            long long* const d_second_index_split_r, const long long R,
                                            cudaStream_t gpu_stream);

/* S only, in place, optional (key, value) copy; d_answer_num is cleared (src/vlsplit_hash_kernel.h:47-53). */
void partial_jointable_gpu_partition_s_only(int* const d_bdata, int* const d_ob_data, int* const d_b_val,
                                            int* const d_ob_val, int2* const d_b_kv_out,
                                            long long* const d_b_prefix_data, long long* const d_block_index_split_s,
                                            long long* const d_b_offset, long long* const d_second_index_split_s,
                                            int* const d_answer_num, const long long S, cudaStream_t gpu_stream);

/* Probes partitioned R with partitioned S (src/vlsplit_hash_kernel.h:56-60). Pairs are appended at
 * *d_answer_write_idx (which advances, as in the reference) up to the capacity set by
 * brig_compat_set_answer_capacity; d_answer_num and *final_answer_number get this call's exact
 * match count. The reference takes the capacity from its __device__ d_answer_capacity
 * (src/kernel_functions.cu:19). max_int_number_for_shared_memory is ignored. */
void partial_jointable_gpu_run_only_s(const int* const d_adata, const int* const d_bdata, const int* const d_a_val,
                                      const int* const d_b_val, long long* const d_block_index_split_r,
                                      long long* const d_block_index_split_s, long long* const d_second_index_split_r,
                                      long long* const d_second_index_split_s, int* const d_answer,
                                      int* const d_answer_val, int* const d_answer_s_val, int* const d_answer_num,
                                      int max_int_number_for_shared_memory, int* final_answer_number,
                                      cudaStream_t gpu_stream, cudaEvent_t gpu_event, int* const d_answer_write_idx);

/* Pair capacity used by partial_jointable_gpu_run_only_s (total over appended calls). */
void brig_compat_set_answer_capacity(long long capacity);

/* ---- Bloom filter object (src/bloom.cuh:8-36) ------------------------------------------------
 * The reference's global filter with its members and bit layout, so a filter built here can be
 * queried by code written against the reference and the other way round: the bit count is rounded
 * up to a multiple of 256; a key v lives in block hash(v, 1) % (bits / 256) of eight 32-bit words
 * and sets bit hash(v, i + 1) % 256 of that block for i < num_hashes, with hash the reference's
 * seeded MurmurHash3-style finaliser (src/bloom.cu:24-31). The device buffer comes from cudaMalloc
 * instead of nvshmem_malloc (one GPU). The engine's own join uses its partitioned filter instead;
 * this object serves callers of the reference's interface. */
class BloomFilter {
private:
    uint32_t* d_filter;
    uint32_t* h_filter;
    size_t num_bits;
    size_t num_words;
    int num_hashes;

public:
    BloomFilter(size_t bits, int hashes);
    ~BloomFilter();
    BloomFilter(const BloomFilter&) = delete;
    BloomFilter& operator=(const BloomFilter&) = delete;

    /* Inserts every key of a device array (src/bloom.cu:460-492). */
    void buildFromTable(int* gpu_data, size_t num_elements);
    /* Queries every key of a device array and prints how many pass (declared at
     * src/bloom.cuh:21). */
    void queryFromTable(int* gpu_data, size_t num_elements);
    /* Prints the size, the number of hashes and the fraction of set bits (src/bloom.cuh:22). */
    void printStats();
    /* Builds nothing: reads the int32 keys of both files, queries the query file's keys and
     * reports the keys of the build file among them that the filter rejects (must be none;
     * src/bloom.cuh:23). */
    void verifyNoFalseNegatives(const char* build_file, const char* query_file);

    uint32_t* getDeviceFilter() const { return d_filter; }
    size_t getNumWords() const { return num_words; }
    size_t getNumBits() const { return num_bits; }
    int getNumHashes() const { return num_hashes; }

    /* Device query: writes 1 or 0 per key into results (device bytes) and returns the number of
     * keys that pass. Not in the reference's header; the engine's tests use it. */
    long long query(const int* gpu_data, size_t num_elements, unsigned char* results);
};

/* ---- Probe executor (src/join_executor.h:10-88) -----------------------------------------------
 * The reference's per-chunk context, field for field. At one PE join_execute_host reads R's
 * partitioned arrays and indexes (GPUA_split, GPUA_val_split, GPU_block_index_split_R,
 * GPU_second_index_split_R), S's indexes for this PE (GPU_block_index_split_S[me],
 * GPU_second_index_split_S[me]) with S's partitioned arrays passed as effective_s_ptr /
 * effective_s_val, the pair buffers and counters (GPU_answer*, answer_num_host), gpu_stream and the
 * accumulators total_answer_num, total_overflow_count and first_pass_probe_sec. The transfer and
 * timing fields of the multi-GPU modes are accepted and left alone. */
struct JoinChunkContext {
    int me;
    int device_num;

    int  use_bf;
    bool use_nvlink;
    int  kernel_fusion;
    bool fused_probe_breakdown;

    int*   GPUA_split;
    int*   GPUB_send_buffer;
    int*   GPU_buffer;
    int*   h_pcie_stage;
    int*   GPUA_val_split;
    int*   GPUB_send_buffer_val;
    int*   GPU_buffer_val;
    int*   h_pcie_stage_val;
    int2*  GPUB_send_buffer_kv;

    int*       GPU_OB_split;
    int*       GPU_OB_val_split;
    long long* GPU_B_prefix_split;
    long long* GPU_B_offset;

    long long*  GPU_block_index_split_R;
    long long** GPU_block_index_split_S;
    long long*  GPU_second_index_split_R;
    long long** GPU_second_index_split_S;

    int* GPU_answer;
    int* GPU_answer_val;
    int* GPU_answer_s_val;
    int* GPU_answer_num;
    int* GPU_answer_write_idx;
    int* answer_num_host;

    std::vector<BloomFilter>* bf;
    size_t    bf_words;
    uint32_t* d_bf_global;

    cudaStream_t gpu_stream;
    cudaEvent_t  gpu_event;
    cudaStream_t send_stream;

    int max_int_number_for_shared_memory;

    double* first_pass_probe_sec;
    double* cumulative_bf_exchange_sec;
    double* cumulative_bf_pipeline_sec;
    double* cumulative_pre_send_barrier_sec;
    double* cumulative_inner_barrier_sec;
    double* cumulative_transfer_sec;
    double* cumulative_second_pass_sec;
    double* cumulative_fused_ht_sec;
    double* cumulative_fused_local_sec;
    double* cumulative_fused_get_sec;
    double* cumulative_fused_remote_probe_sec;
    double* cumulative_fused_wall_sec;
    double* cumulative_fused_setup_sec;

    double* cumulative_fp_preamble_sec;
    double* cumulative_fp_memset_sec;
    double* cumulative_fp_initbar_sec;
    double* cumulative_fp_build_sec;
    double* cumulative_fp_local_sec;
    double* cumulative_fp_reduce_sec;

    long long** d_s_block_ptrs;
    long long** d_s_second_ptrs;
    long long*  d_phase_timers;
    long long   d_phase_timers_slots;

    int*    total_answer_num;
    int*    total_overflow_count;
};

/* The local probe of one S chunk (src/join_executor.h:87-88): the engine's task builder and
 * persistent probe over the caller's partitioned R and S, pairs appended at *GPU_answer_write_idx
 * up to the capacity of brig_compat_set_answer_capacity, the chunk's count into GPU_answer_num,
 * answer_num_host[0] and added to *total_answer_num. Synchronous, as the reference. The engine has
 * no overflow blocks (oversized partitions are probed exactly), so *total_overflow_count gains 0;
 * actual_b_size is the chunk's S size (informational: the indexes carry it). */
void join_execute_host(JoinChunkContext& ctx, int* effective_s_ptr, int* effective_s_val, long long actual_b_size);

#endif /* BRIG_JOIN_COMPAT_H_ */
