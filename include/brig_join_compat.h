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

#endif /* BRIG_JOIN_COMPAT_H_ */
