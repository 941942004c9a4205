// compat.cu - the reference-named C++ entry points (include/brig_join_compat.h) over the engine.
//
// The partition entry points run the engine's own partition kernels in the reference's modulo
// layout (partition_mode = BRIG_PART_MODULO with the global fan-outs) and then translate the
// result into the reference's contract: tuples back into the caller's key/value arrays in place,
// inclusive-end bucket indexes, local inclusive-end sub-bucket indexes. The probe entry point does
// the reverse: it reads the caller's partitioned arrays and indexes into the engine's layout and
// runs the engine's task builder and probe kernel. gpu_main is the whole local join over files.
// Every helper here synchronises with the host where the reference does (its entry points are
// blocking); failures print to stderr and leave outputs untouched instead of exiting.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include "../../include/brig_join.h"
#include "../../include/brig_join_compat.h"
#include "engine.h"

int partition_size = 128;
int second_partition_size = 67;
int thread_no = 1024;
int block_no = 31250;
int block_size = 0;
int chunk_size = 1024;

// The reference's CPU check, used by gpu_main when the program links it (weak: optional).
void run_sanity_check(const int* tableA, long long R, const int* tableB, long long S) __attribute__((weak));

namespace brig {
namespace {

long long g_answer_capacity = (1ll << 62);

// Workspace of the compat entry points (one per process; the reference's are not reentrant either).
std::mutex g_mu;
char* g_ws = nullptr;
size_t g_ws_bytes = 0;

char* compat_workspace(size_t bytes) {
    if (bytes > g_ws_bytes) {
        if (g_ws) cudaFree(g_ws);
        g_ws = nullptr;
        g_ws_bytes = 0;
        cuda_check(cudaMalloc(&g_ws, bytes), "compat workspace");
        g_ws_bytes = bytes;
    }
    return g_ws;
}

brig_join_config modulo_config() {
    brig_join_config c;
    brig_join_config_init(&c);
    c.partition_mode = BRIG_PART_MODULO;
    c.partition_size = partition_size;
    c.second_partition_size = second_partition_size;
    return c;
}

// A pipeline over one join laid out in the compat workspace; the descriptor image stays on the
// host so the caller can read every buffer address.
struct Prepared {
    JoinPlan plan;
    JoinOffs jo;
    Shape sh;
    std::vector<char> meta;
    PipelineArgs a;
    char* ws = nullptr;
    const JoinDesc& desc() const { return *reinterpret_cast<const JoinDesc*>(meta.data()); }
};

void prepare(Prepared& p, const brig_join_config& cfg, const JoinIO& io) {
    int dev = 0, sms = 148;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    p.plan = plan_join(cfg, io.nr, io.ns);
    layout_for(cfg, &p.plan, 1, sms, &p.jo, p.sh);
    p.ws = compat_workspace(p.sh.total);
    p.meta.assign(p.sh.meta_bytes, 0);
    fill_pipeline(cfg, &p.plan, &io, 1, p.sh, p.ws, p.meta.data(), sms, p.a);
}

void launch(Prepared& p, int stages, cudaStream_t st) {
    cuda_check(cudaMemcpyAsync(p.ws + p.sh.meta, p.meta.data(), p.sh.meta_bytes, cudaMemcpyHostToDevice, st),
               "descriptor upload");
    cuda_check(cudaMemsetAsync(p.ws + p.sh.counters, 0, (size_t)kCntWords * 8, st), "counter reset");
    p.a.stages = stages;
    cuda_check(enqueue_pipeline(p.a, st), "pipeline launch");
}

// ---- layout translation kernels ----------------------------------------------------------------
__global__ void k_unpack(const uint2* __restrict__ in, int* __restrict__ key, int* __restrict__ val, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint2 e = in[i];
        key[i] = (int)e.x;
        val[i] = (int)e.y;
    }
}
__global__ void k_pack(const int* __restrict__ key, const int* __restrict__ val, uint2* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_uint2((uint32_t)key[i], (uint32_t)val[i]);
}
// Engine bounds -> reference indexes: blk[p] inclusive end of bucket p; sec[p*P2+q] inclusive end of
// sub-bucket q relative to bucket p's start; prefix[p] bucket size; offset[p] bucket end.
__global__ void k_to_ref_index(const int64_t* __restrict__ b1, const int64_t* __restrict__ bounds, int P1, int P2,
                               long long* blk, long long* sec, long long* prefix, long long* offset) {
    const int64_t nf = (int64_t)P1 * P2;
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = f / P2;
        if (sec) sec[f] = bounds[f + 1] - b1[p];
        if (f % P2 == 0) {
            if (blk) blk[p] = b1[p + 1];
            if (prefix) prefix[p] = b1[p + 1] - b1[p];
            if (offset) offset[p] = b1[p + 1];
        }
    }
}
// Reference indexes -> engine bounds (start of every finest partition, plus the total).
__global__ void k_from_ref_index(const long long* __restrict__ blk, const long long* __restrict__ sec, int P1, int P2,
                                 int64_t* __restrict__ bounds) {
    const int64_t nf = (int64_t)P1 * P2;
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f <= nf; f += (int64_t)gridDim.x * blockDim.x) {
        if (f == nf) {
            bounds[f] = blk[P1 - 1];
            continue;
        }
        const int64_t p = f / P2, q = f % P2;
        bounds[f] = (p ? blk[p - 1] : 0) + (q ? sec[f - 1] : 0);
    }
}

constexpr int kCompatGrid = 1184;

// Partitions one relation (rel 0 = R from io.rk/rv, rel 1 = S from io.sk/sv) and translates the
// result into the reference's contract.
void partition_rel(int rel, int* d_data, int* d_val, int2* d_kv_out, long long* d_prefix, long long* d_block_index,
                   long long* d_offset, long long* d_second_index, long long n, cudaStream_t st) {
    if (partition_size <= 0 || second_partition_size <= 0) fail(BRIG_E_INVALID, "partition sizes must be positive");
    const brig_join_config cfg = modulo_config();
    JoinIO io{};
    if (rel == 0) {
        io.rk = reinterpret_cast<const uint32_t*>(d_data);
        io.rv = reinterpret_cast<const uint32_t*>(d_val);
        io.nr = n;
    } else {
        io.sk = reinterpret_cast<const uint32_t*>(d_data);
        io.sv = reinterpret_cast<const uint32_t*>(d_val);
        io.ns = n;
    }
    Prepared p;
    prepare(p, cfg, io);
    launch(p, rel == 0 ? kRunPartR : kRunPartS, st);
    const JoinDesc& d = p.desc();
    const RelPlan& R = d.rel[rel];
    const uint2* fin = d.pf.P2 > 1 ? R.l2 : R.l1;
    if (n > 0) {
        k_unpack<<<kCompatGrid, 256, 0, st>>>(fin, d_data, d_val, n);
        if (d_kv_out)
            cuda_check(cudaMemcpyAsync(d_kv_out, fin, (size_t)n * 8, cudaMemcpyDeviceToDevice, st), "kv copy");
    }
    k_to_ref_index<<<kCompatGrid, 256, 0, st>>>(R.b1, R.bounds, (int)d.pf.P1, (int)d.pf.P2, d_block_index, d_second_index,
                                                d_prefix, d_offset);
    note_launches(n > 0 ? 2 : 1);
    cuda_check(cudaGetLastError(), "translation launch");
}

void report(const Error& e, const char* where) { fprintf(stderr, "[brig compat] %s: %s\n", where, e.msg.c_str()); }

}  // namespace
}  // namespace brig

using namespace brig;

void brig_compat_set_answer_capacity(long long capacity) { g_answer_capacity = capacity < 0 ? 0 : capacity; }

void split_tables(int device_num, int* const tableA, int* const tableB, int* const tableA_val, int* const tableB_val,
                  long long* tableA_size, long long* tableB_size, int** tableA_split, int** tableB_split,
                  int** tableA_val_split, int** tableB_val_split, const long long R, const long long S) {
    const long long r = R / device_num, s = S / device_num;
    for (int i = 0; i < device_num; ++i) {
        tableA_split[i] = tableA + r * i;
        tableB_split[i] = tableB + s * i;
        tableA_val_split[i] = tableA_val + r * i;
        tableB_val_split[i] = tableB_val + s * i;
        tableA_size[i] = (i == device_num - 1) ? R - r * i : r;
        tableB_size[i] = (i == device_num - 1) ? S - s * i : s;
    }
}

void partial_jointable_gpu_partition_r_only(int* const d_adata, int* const, int* const d_a_val, int* const,
                                            long long* const d_a_prefix_data, long long* const d_block_index_split_r,
                                            long long* const d_a_offset, long long* const d_second_index_split_r,
                                            const long long R, cudaStream_t gpu_stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    try {
        partition_rel(0, d_adata, d_a_val, nullptr, d_a_prefix_data, d_block_index_split_r, d_a_offset,
                      d_second_index_split_r, R, gpu_stream);
        cuda_check(cudaStreamSynchronize(gpu_stream), "cudaStreamSynchronize");
    } catch (const Error& e) {
        report(e, "partial_jointable_gpu_partition_r_only");
    }
}

void partial_jointable_gpu_partition_s_only(int* const d_bdata, int* const, int* const d_b_val, int* const,
                                            int2* const d_b_kv_out, long long* const d_b_prefix_data,
                                            long long* const d_block_index_split_s, long long* const d_b_offset,
                                            long long* const d_second_index_split_s, int* const d_answer_num,
                                            const long long S, cudaStream_t gpu_stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    try {
        if (d_answer_num) cuda_check(cudaMemsetAsync(d_answer_num, 0, sizeof(int), gpu_stream), "memset");
        partition_rel(1, d_bdata, d_b_val, d_b_kv_out, d_b_prefix_data, d_block_index_split_s, d_b_offset,
                      d_second_index_split_s, S, gpu_stream);
        cuda_check(cudaStreamSynchronize(gpu_stream), "cudaStreamSynchronize");
    } catch (const Error& e) {
        report(e, "partial_jointable_gpu_partition_s_only");
    }
}

void partial_jointable_gpu_partition(const int* const d_adata, const int* const d_bdata, int* const d_oa_data,
                                     int* const d_ob_data, int* const d_a_val, int* const d_b_val, int* const d_oa_val,
                                     int* const d_ob_val, int2* const d_b_kv_out, long long* const d_a_prefix_data,
                                     long long* const d_b_prefix_data, long long* const d_block_index_split_r,
                                     long long* const d_block_index_split_s, long long* const d_a_offset,
                                     long long* const d_b_offset, long long* const d_second_index_split_r,
                                     long long* const d_second_index_split_s, int* const d_answer_num,
                                     const long long R, const long long S, cudaStream_t gpu_stream, cudaEvent_t,
                                     double& out_partition_sec, double& out_hist_sec, bool) {
    const auto t0 = std::chrono::steady_clock::now();
    // The reference partitions its (const-declared) input buffers in place as well.
    partial_jointable_gpu_partition_r_only(const_cast<int*>(d_adata), d_oa_data, d_a_val, d_oa_val, d_a_prefix_data,
                                           d_block_index_split_r, d_a_offset, d_second_index_split_r, R, gpu_stream);
    partial_jointable_gpu_partition_s_only(const_cast<int*>(d_bdata), d_ob_data, d_b_val, d_ob_val, d_b_kv_out,
                                           d_b_prefix_data, d_block_index_split_s, d_b_offset, d_second_index_split_s,
                                           d_answer_num, S, gpu_stream);
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out_partition_sec += sec;
    out_hist_sec += 0.0;  // the histogram passes are inside the partition time here
}

void partial_jointable_gpu_partition_rs_split(
    const int* const d_adata, const int* const d_bdata, int* const d_oa_data, int* const d_ob_data, int* const d_a_val,
    int* const d_b_val, int* const d_oa_val, int* const d_ob_val, int2* const d_b_kv_out,
    long long* const d_a_prefix_data, long long* const d_b_prefix_data, long long* const d_block_index_split_r,
    long long* const d_block_index_split_s, long long* const d_a_offset, long long* const d_b_offset,
    long long* const d_second_index_split_r, long long* const d_second_index_split_s, int* const d_answer_num,
    const long long R, const long long S, cudaStream_t gpu_stream, cudaEvent_t, double& out_partition_sec,
    double& out_partition_r_sec, double& out_partition_s_sec, double& out_hist_r_sec, double& out_hist_s_sec, bool) {
    const auto t0 = std::chrono::steady_clock::now();
    partial_jointable_gpu_partition_r_only(const_cast<int*>(d_adata), d_oa_data, d_a_val, d_oa_val, d_a_prefix_data,
                                           d_block_index_split_r, d_a_offset, d_second_index_split_r, R, gpu_stream);
    const auto t1 = std::chrono::steady_clock::now();
    partial_jointable_gpu_partition_s_only(const_cast<int*>(d_bdata), d_ob_data, d_b_val, d_ob_val, d_b_kv_out,
                                           d_b_prefix_data, d_block_index_split_s, d_b_offset, d_second_index_split_s,
                                           d_answer_num, S, gpu_stream);
    const auto t2 = std::chrono::steady_clock::now();
    out_partition_r_sec += std::chrono::duration<double>(t1 - t0).count();
    out_partition_s_sec += std::chrono::duration<double>(t2 - t1).count();
    out_partition_sec += std::chrono::duration<double>(t2 - t0).count();
    out_hist_r_sec += 0.0;
    out_hist_s_sec += 0.0;
}

void partial_jointable_gpu_run_only_s(const int* const d_adata, const int* const d_bdata, const int* const d_a_val,
                                      const int* const d_b_val, long long* const d_block_index_split_r,
                                      long long* const d_block_index_split_s, long long* const d_second_index_split_r,
                                      long long* const d_second_index_split_s, int* const d_answer,
                                      int* const d_answer_val, int* const d_answer_s_val, int* const d_answer_num, int,
                                      int* final_answer_number, cudaStream_t gpu_stream, cudaEvent_t,
                                      int* const d_answer_write_idx) {
    std::lock_guard<std::mutex> lk(g_mu);
    try {
        cudaStream_t st = gpu_stream;
        const int P1 = partition_size, P2 = second_partition_size;
        if (P1 <= 0 || P2 <= 0) fail(BRIG_E_INVALID, "partition sizes must be positive");
        long long nr = 0, ns = 0;
        cuda_check(cudaMemcpyAsync(&nr, d_block_index_split_r + (P1 - 1), 8, cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaMemcpyAsync(&ns, d_block_index_split_s + (P1 - 1), 8, cudaMemcpyDeviceToHost, st), "D2H");
        int wi = 0;
        if (d_answer_write_idx)
            cuda_check(cudaMemcpyAsync(&wi, d_answer_write_idx, 4, cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        brig_join_config cfg = modulo_config();
        // the caller's layout fixes the fan-outs; keep them even when the planner would choose
        // differently for these sizes
        cfg.partition_size = P1;
        cfg.second_partition_size = P2;
        const int64_t base = std::max(0, wi);
        const int64_t cap = std::max<int64_t>(0, g_answer_capacity - base);
        brig_join_output out{reinterpret_cast<uint32_t*>(d_answer_val) + base,
                             reinterpret_cast<uint32_t*>(d_answer_s_val) + base,
                             d_answer ? reinterpret_cast<uint32_t*>(d_answer) + base : nullptr, cap, nullptr};
        JoinIO io{reinterpret_cast<const uint32_t*>(d_adata), reinterpret_cast<const uint32_t*>(d_a_val),
                  reinterpret_cast<const uint32_t*>(d_bdata), reinterpret_cast<const uint32_t*>(d_b_val), nr, ns, out};
        Prepared p;
        prepare(p, cfg, io);
        const JoinDesc& d = p.desc();
        for (int rel = 0; rel < 2; ++rel) {
            const RelPlan& R = d.rel[rel];
            uint2* fin = d.pf.P2 > 1 ? R.l2 : R.l1;
            const int64_t n = rel ? ns : nr;
            if (n > 0)
                k_pack<<<kCompatGrid, 256, 0, st>>>(rel ? d_bdata : d_adata, rel ? d_b_val : d_a_val, fin, n);
            k_from_ref_index<<<kCompatGrid, 256, 0, st>>>(rel ? d_block_index_split_s : d_block_index_split_r,
                                                          rel ? d_second_index_split_s : d_second_index_split_r, P1, P2,
                                                          R.bounds);
            if (d.pf.P2 > 1)  // b1 is only read by level-2 kernels, which do not run here
                cuda_check(cudaMemsetAsync(R.b1, 0, ((size_t)P1 + 1) * 8, st), "memset");
            note_launches(n > 0 ? 2 : 1);
        }
        cuda_check(cudaGetLastError(), "translation launch");
        launch(p, kRunProbe, st);
        long long cnt = 0;
        cuda_check(cudaMemcpyAsync(&cnt, d.counters + kCntMatches, 8, cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        const int c32 = (int)cnt;
        if (d_answer_num) cuda_check(cudaMemcpy(d_answer_num, &c32, 4, cudaMemcpyHostToDevice), "H2D");
        if (d_answer_write_idx) {
            const int next = (int)(base + cnt);
            cuda_check(cudaMemcpy(d_answer_write_idx, &next, 4, cudaMemcpyHostToDevice), "H2D");
        }
        if (final_answer_number) *final_answer_number = c32;
    } catch (const Error& e) {
        report(e, "partial_jointable_gpu_run_only_s");
    }
}

void gpu_main(std::vector<int>*, std::vector<int>*, const std::string& r_inputPath, const std::string& s_inputPath,
              long long R, long long S, int use_bf, bool use_nvlink, bool, double true_false_ratio, int s_chunks,
              bool sanityCheck, int kernel_fusion, double redist_skew_threshold, long long override_num_bits,
              int override_num_hashes, int, int override_partition_size, int override_second_partition_size, int,
              int read_val, int r_shuffle_enable, double r_replicate_ratio, double answer_scale) {
    if (use_nvlink || kernel_fusion || redist_skew_threshold > 0.0 || r_shuffle_enable || r_replicate_ratio >= 0.0)
        fprintf(stderr, "[brig compat] one GPU: multi-GPU options (nvlink, fusion, redistribution, shuffle, "
                        "replication) have no effect\n");
    if (R < 0 || S < 0 || s_chunks < 1) {
        fprintf(stderr, "[brig compat] gpu_main: bad sizes\n");
        return;
    }
    std::vector<int> tk(R), tv(R), sk(S), sv(S);
    auto u32 = [](std::vector<int>& v) { return reinterpret_cast<uint32_t*>(v.data()); };
    if (brig_join_read_relation(r_inputPath.c_str(), R, read_val ? 1 : 0, 1u, u32(tk), u32(tv)) != BRIG_OK ||
        brig_join_read_relation(s_inputPath.c_str(), S, read_val ? 1 : 0, 100000001u, u32(sk), u32(sv)) != BRIG_OK) {
        fprintf(stderr, "[brig compat] gpu_main: %s\n", brig_join_last_error());
        return;
    }
    if (sanityCheck && run_sanity_check) run_sanity_check(tk.data(), R, sk.data(), S);
    brig_join_config cfg;
    brig_join_config_init(&cfg);
    if (use_bf) {
        cfg.use_bloom = 1;
        const double ln2 = std::log(2.0);
        const double bits = -(double)R * std::log(true_false_ratio) / (ln2 * ln2);
        cfg.bloom_num_bits = override_num_bits >= 0 ? override_num_bits : (int64_t)bits;
        cfg.bloom_num_hashes = override_num_hashes >= 0 ? override_num_hashes : std::max(1, (int)(bits / std::max<double>(R, 1) * ln2));
        if (cfg.bloom_num_hashes > kMaxBloomK) cfg.bloom_num_hashes = kMaxBloomK;
    }
    if (override_partition_size >= 0 || override_second_partition_size >= 0) {
        cfg.partition_mode = BRIG_PART_MODULO;
        cfg.partition_size = override_partition_size > 0 ? override_partition_size : partition_size;
        if (override_second_partition_size > 0) cfg.second_partition_size = override_second_partition_size;
    }
    // The reference's S chunk loop (src/hash_kernel.cu:910-1131): R is partitioned and filtered once
    // and S is copied and joined chunk by chunk (brig_join_config.s_chunks). The reference keeps its
    // answers on the device and reports the count; the count here is exact with no pairs written.
    (void)answer_scale;
    cfg.s_chunks = s_chunks;
    brig_join_t* h = nullptr;
    if (brig_join_create(&cfg, &h) != BRIG_OK) {
        fprintf(stderr, "[brig compat] gpu_main: %s\n", brig_join_last_error());
        return;
    }
    long long total = 0, overflow_tasks = 0;
    const auto t0 = std::chrono::steady_clock::now();
    int64_t cnt = 0;
    int rc = brig_join_run_host(h, reinterpret_cast<const uint32_t*>(tk.data()),
                                reinterpret_cast<const uint32_t*>(tv.data()), R,
                                reinterpret_cast<const uint32_t*>(sk.data()),
                                reinterpret_cast<const uint32_t*>(sv.data()), S, nullptr, nullptr, nullptr, 0, &cnt,
                                nullptr);
    brig_join_stats st;
    if (rc == BRIG_OK || rc == BRIG_E_OVERFLOW) rc = brig_join_get_stats(h, &st);
    const bool ok = rc == BRIG_OK || rc == BRIG_E_OVERFLOW;
    if (ok) {
        total = st.count;
        overflow_tasks = st.split_tasks;
    } else {
        fprintf(stderr, "[brig compat] gpu_main: %s\n", brig_join_last_error());
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (ok) {
        printf("[PE0] PE0 answer count: %lld\n", total);
        printf("=== Grand Total Answer Count (all PEs): %lld ===\n", total);
        printf("[PE0] Total (H2D + join) %.4f sec, split tasks %lld\n", sec, overflow_tasks);
    }
    brig_join_destroy(h);
}

// ---- BloomFilter (src/bloom.cuh:8-36) ------------------------------------------------------------
namespace brig {
namespace {

// The reference's Bloom hash (src/bloom.cu:24-31): the seed xor the key, then the two multiply /
// xor-shift rounds of the MurmurHash3 finaliser.
__host__ __device__ __forceinline__ uint32_t ref_bloom_hash(int32_t v, uint32_t seed) {
    uint32_t h = seed ^ (uint32_t)v;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// The eight words a key sets in its 256-bit block (bit hash(v, j + 1) % 256 for j < k).
__device__ __forceinline__ void ref_bloom_bits(int32_t v, int k, uint32_t (&w)[8]) {
#pragma unroll
    for (int x = 0; x < 8; ++x) w[x] = 0u;
    for (int j = 0; j < k; ++j) {
        const uint32_t pos = ref_bloom_hash(v, (uint32_t)j + 1u) & 255u;
        const uint32_t bit = 1u << (pos & 31u), word = pos >> 5;
#pragma unroll
        for (int x = 0; x < 8; ++x) w[x] |= word == (uint32_t)x ? bit : 0u;
    }
}

// One thread per key: the key's bits are gathered per word, then one atomicOr per touched word.
__global__ void k_refbf_insert(uint32_t* __restrict__ f, const int* __restrict__ data, int64_t n, int k,
                               uint64_t nblocks) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int v = data[i];
        uint32_t w[8];
        ref_bloom_bits(v, k, w);
        uint32_t* b = f + (ref_bloom_hash(v, 1u) % nblocks) * 8;
#pragma unroll
        for (int x = 0; x < 8; ++x)
            if (w[x]) atomicOr(b + x, w[x]);
    }
}

// One thread per key: the key's block is read as two 16-byte loads; a key passes when every one
// of its bits is set. Passing keys are counted with one atomic per warp.
__global__ void k_refbf_query(const uint32_t* __restrict__ f, const int* __restrict__ data, int64_t n, int k,
                              uint64_t nblocks, unsigned char* __restrict__ results,
                              unsigned long long* __restrict__ passed) {
    for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        bool ok = false;
        if (i < n) {
            const int v = data[i];
            uint32_t w[8];
            ref_bloom_bits(v, k, w);
            const uint4* b = reinterpret_cast<const uint4*>(f + (ref_bloom_hash(v, 1u) % nblocks) * 8);
            const uint4 a = __ldg(b), c = __ldg(b + 1);
            ok = ((a.x & w[0]) == w[0]) && ((a.y & w[1]) == w[1]) && ((a.z & w[2]) == w[2]) && ((a.w & w[3]) == w[3]) &&
                 ((c.x & w[4]) == w[4]) && ((c.y & w[5]) == w[5]) && ((c.z & w[6]) == w[6]) && ((c.w & w[7]) == w[7]);
            if (results) results[i] = ok ? 1 : 0;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(passed, (unsigned long long)__popc(m));
    }
}

std::vector<int> read_int_file(const char* path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f.is_open()) fail(BRIG_E_INVALID, std::string("cannot open ") + path);
    const std::streamsize bytes = f.tellg();
    std::vector<int> v((size_t)(bytes / 4));
    f.seekg(0);
    f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(v.size() * 4));
    return v;
}

}  // namespace
}  // namespace brig

BloomFilter::BloomFilter(size_t bits, int hashes) : d_filter(nullptr), h_filter(nullptr), num_bits(bits),
                                                    num_words(0), num_hashes(hashes) {
    num_bits = (num_bits + 255) / 256 * 256;  // whole 256-bit blocks (src/bloom.cu:428-431)
    if (num_bits == 0) num_bits = 256;
    num_words = num_bits / 32;
    h_filter = new uint32_t[num_words]();
    if (cudaMalloc(&d_filter, num_words * 4) != cudaSuccess || cudaMemset(d_filter, 0, num_words * 4) != cudaSuccess) {
        fprintf(stderr, "[brig compat] BloomFilter: device allocation of %zu bytes failed\n", num_words * 4);
        d_filter = nullptr;
    }
}

BloomFilter::~BloomFilter() {
    delete[] h_filter;
    if (d_filter) cudaFree(d_filter);
}

void BloomFilter::buildFromTable(int* gpu_data, size_t num_elements) {
    if (!d_filter || num_elements == 0) return;
    brig::k_refbf_insert<<<1184, 256>>>(d_filter, gpu_data, (int64_t)num_elements, num_hashes, num_bits / 256);
    brig::note_launches(1);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) fprintf(stderr, "[brig compat] BloomFilter::buildFromTable: %s\n", cudaGetErrorString(e));
}

long long BloomFilter::query(const int* gpu_data, size_t num_elements, unsigned char* results) {
    if (!d_filter || num_elements == 0) return 0;
    unsigned long long* d_passed = nullptr;
    if (cudaMalloc(&d_passed, 8) != cudaSuccess) return -1;
    cudaMemset(d_passed, 0, 8);
    brig::k_refbf_query<<<1184, 256>>>(d_filter, gpu_data, (int64_t)num_elements, num_hashes, num_bits / 256, results,
                                        d_passed);
    brig::note_launches(1);
    unsigned long long passed = 0;
    const cudaError_t e = cudaMemcpy(&passed, d_passed, 8, cudaMemcpyDeviceToHost);
    cudaFree(d_passed);
    if (e != cudaSuccess) {
        fprintf(stderr, "[brig compat] BloomFilter::query: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return (long long)passed;
}

void BloomFilter::queryFromTable(int* gpu_data, size_t num_elements) {
    const long long passed = query(gpu_data, num_elements, nullptr);
    printf("[BloomFilter] %lld of %zu keys pass\n", passed, num_elements);
}

void BloomFilter::printStats() {
    if (!d_filter) return;
    if (cudaMemcpy(h_filter, d_filter, num_words * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return;
    size_t set = 0;
    for (size_t i = 0; i < num_words; ++i) set += (size_t)__builtin_popcount(h_filter[i]);
    printf("[BloomFilter] bits: %zu, hash functions: %d, memory: %.2f MB, bits set: %.4f\n", num_bits, num_hashes,
           (double)num_words * 4 / (1024.0 * 1024.0), (double)set / (double)num_bits);
}

void BloomFilter::verifyNoFalseNegatives(const char* build_file, const char* query_file) {
    try {
        const std::vector<int> b = brig::read_int_file(build_file), q = brig::read_int_file(query_file);
        int* d_q = nullptr;
        unsigned char* d_res = nullptr;
        brig::cuda_check(cudaMalloc(&d_q, std::max<size_t>(q.size(), 1) * 4), "cudaMalloc");
        brig::cuda_check(cudaMalloc(&d_res, std::max<size_t>(q.size(), 1)), "cudaMalloc");
        brig::cuda_check(cudaMemcpy(d_q, q.data(), q.size() * 4, cudaMemcpyHostToDevice), "H2D");
        query(d_q, q.size(), d_res);
        std::vector<unsigned char> res(q.size());
        brig::cuda_check(cudaMemcpy(res.data(), d_res, res.size(), cudaMemcpyDeviceToHost), "D2H");
        cudaFree(d_q);
        cudaFree(d_res);
        std::vector<int> sorted(b);
        std::sort(sorted.begin(), sorted.end());
        long long members = 0, false_neg = 0, passed = 0;
        for (size_t i = 0; i < q.size(); ++i) {
            const bool in = std::binary_search(sorted.begin(), sorted.end(), q[i]);
            members += in;
            passed += res[i];
            false_neg += in && !res[i];
        }
        printf("[BloomFilter] verify: %zu queries, %lld members, %lld pass, %lld false negatives\n", q.size(), members,
               passed, false_neg);
    } catch (const brig::Error& e) {
        brig::report(e, "BloomFilter::verifyNoFalseNegatives");
    }
}

// ---- join_execute_host (src/join_executor.h:87-88) -------------------------------------------------
void join_execute_host(JoinChunkContext& ctx, int* effective_s_ptr, int* effective_s_val, long long) {
    if (ctx.device_num > 1 || ctx.kernel_fusion == 2)
        fprintf(stderr, "[brig compat] join_execute_host: one GPU: the cross-GPU transfer and probe have no effect\n");
    const auto t0 = std::chrono::steady_clock::now();
    int n = 0;
    partial_jointable_gpu_run_only_s(ctx.GPUA_split, effective_s_ptr, ctx.GPUA_val_split, effective_s_val,
                                     ctx.GPU_block_index_split_R,
                                     ctx.GPU_block_index_split_S ? ctx.GPU_block_index_split_S[ctx.me] : nullptr,
                                     ctx.GPU_second_index_split_R,
                                     ctx.GPU_second_index_split_S ? ctx.GPU_second_index_split_S[ctx.me] : nullptr,
                                     ctx.GPU_answer, ctx.GPU_answer_val, ctx.GPU_answer_s_val, ctx.GPU_answer_num,
                                     ctx.max_int_number_for_shared_memory, &n, ctx.gpu_stream, ctx.gpu_event,
                                     ctx.GPU_answer_write_idx);
    if (ctx.first_pass_probe_sec)
        *ctx.first_pass_probe_sec += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (ctx.answer_num_host) ctx.answer_num_host[0] = n;
    if (ctx.total_answer_num) *ctx.total_answer_num += n;
    // the engine probes oversized partitions exactly: no overflow blocks to report
}
