// engine.cu - planner, workspace layout and pipeline orchestration (host C++).
//
// Replaces gpu_main's one-PE slice (src/hash_kernel.cu:103-1131): sizing (:173-284), allocation
// (:370-480), the use_bf==10 partitioned filter (:555-582, :670-705), the S chunk prefilter
// (:935-954) and the partition/probe sequence (:1073-1130). The reference synchronises the host
// after nearly every stage (src/vlsplit_hash_kernel.cu:36-107, src/join_executor.cu:49); here the
// whole pipeline is enqueued on one stream with every size it needs computed on the device, so a
// run is a single stream-ordered unit that can be captured in a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>
#include "engine.h"

namespace brig {

[[noreturn]] void fail(int status, const std::string& msg) { throw Error{status, msg}; }

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int st = (e == cudaErrorMemoryAllocation) ? BRIG_E_NOMEM : BRIG_E_CUDA;
    fail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

static int ceil_log2(int64_t x) {
    int b = 0;
    while (((int64_t)1 << b) < x) ++b;
    return b;
}
static bool is_pow2(int64_t x) { return x > 0 && (x & (x - 1)) == 0; }

// Filter bytes up to which one join probes its filter in S's first pass: 96 MB. At |R| = 2^26,
// |S| = 2^30 an 80 MB filter probed there took 10.4 ms against 12.5 ms in the second pass at a 0.1%
// match rate (14.7 against 14.6 ms at 10%); 112 MB and up are faster in the second pass.
constexpr int64_t kL1FilterBytes = 96ll << 20;
// Filter bytes that the first-pass probes of one batch may touch together (they share L2).
constexpr int64_t kL2FilterBytes = 64ll << 20;

JoinPlan plan_join(const brig_join_config& cfg, int64_t nr, int64_t ns) {
    JoinPlan p;
    p.nr = nr;
    p.ns = ns;
    const int T = cfg.table_capacity > 0 ? cfg.table_capacity : kDefaultTable;
    if (cfg.partition_fill < 0 || cfg.partition_fill > 100) fail(BRIG_E_INVALID, "partition_fill must be in [0, 100]");
    const int fill = cfg.partition_fill > 0 ? cfg.partition_fill : 75;
    const int64_t target = std::max<int64_t>(1, (int64_t)T * fill / 100);  // R tuples per finest partition
    PartFn& f = p.pf;
    f.mode = cfg.partition_mode;
    if (f.mode == BRIG_PART_HASH) {
        const int bits = ceil_log2(std::max<int64_t>(1, (nr + target - 1) / target));
        int b1, b2;
        if (cfg.partition_size > 0) {
            if (!is_pow2(cfg.partition_size) || cfg.partition_size > kMaxP1)
                fail(BRIG_E_INVALID, "hash partitioning needs a power-of-two partition_size <= 4096 "
                                     "(use BRIG_PART_MODULO for other fan-outs)");
            b1 = ceil_log2(cfg.partition_size);
        } else {
            // At most 512 level-1 partitions: every CTA keeps one open output run per partition,
            // and at 512 the runs of all CTAs (148 x 512 lines) stay resident in L2 until they are
            // completed, so DRAM sees whole lines. Anything finer goes to level 2.
            const int cap = cfg.max_level1_bits > 0 ? std::min(cfg.max_level1_bits, 12) : 9;
            b1 = bits <= cap ? bits : cap;
        }
        if (cfg.second_partition_size > 0) {
            if (!is_pow2(cfg.second_partition_size) || cfg.second_partition_size > kMaxP2)
                fail(BRIG_E_INVALID, "hash partitioning needs a power-of-two second_partition_size <= 1024");
            b2 = ceil_log2(cfg.second_partition_size);
        } else {
            b2 = std::max(0, bits - b1);
            if (b2 > 10) fail(BRIG_E_UNSUPPORTED, "relation too large for two partition levels");
        }
        if (b1 + b2 > 24) fail(BRIG_E_UNSUPPORTED, "more than 2^24 finest partitions");
        f.b1 = b1;
        f.b2 = b2;
        f.P1 = 1u << b1;
        f.P2 = 1u << b2;
    } else if (f.mode == BRIG_PART_MODULO) {
        const int64_t P1 = cfg.partition_size > 0 ? cfg.partition_size : 512;
        if (P1 > kMaxP1) fail(BRIG_E_INVALID, "partition_size > 4096");
        int64_t P2 = cfg.second_partition_size;
        if (P2 <= 0) {
            // The reference starts at 67 and grows to the next odd value when the average
            // sub-bucket exceeds the table target (src/hash_kernel.cu:240-284).
            P2 = 67;
            const int64_t sub = (nr + P1 * P2 - 1) / (P1 * P2);
            if (sub > target) {
                P2 = (nr + P1 * target - 1) / (P1 * target);
                if (P2 % 2 == 0) ++P2;
            }
        }
        if (P2 > kMaxP2) fail(BRIG_E_UNSUPPORTED, "second_partition_size > 1024 (raise partition_size)");
        f.P1 = (uint32_t)P1;
        f.P2 = (uint32_t)P2;
        f.M1 = fastmod_magic(f.P1);
        f.M2 = fastmod_magic(f.P2);
    } else {
        fail(BRIG_E_INVALID, "unknown partition_mode");
    }
    p.nfine = (int64_t)f.P1 * f.P2;
    if (cfg.use_bloom) {
        const double bpk = cfg.bloom_bits_per_key > 0 ? cfg.bloom_bits_per_key : 10.0;
        int64_t bits = cfg.bloom_num_bits > 0 ? cfg.bloom_num_bits : (int64_t)std::llround(bpk * (double)nr);
        bits = std::max<int64_t>(bits, 256);
        int k = cfg.bloom_num_hashes > 0 ? cfg.bloom_num_hashes : (int)std::lround(bpk * std::log(2.0));
        k = std::min(std::max(k, 1), kMaxBloomK);
        const int64_t blocks = (bits + 255) / 256;
        p.seg_blocks = (uint32_t)std::max<int64_t>(1, (blocks + p.nfine - 1) / p.nfine);
        // the kernels index filter words with 32 bits
        if (p.nfine * (int64_t)p.seg_blocks * 8 >= (1ll << 32))
            fail(BRIG_E_UNSUPPORTED, "Bloom filter above 2^37 bits (16 GB)");
        p.bloom = true;
        p.k = k;
        p.bloom_bits = p.nfine * (int64_t)p.seg_blocks * 256;
        const int64_t nw = (int64_t)p.seg_blocks * 8;
        p.bloom_group = nw <= kBloomSmemWords ? (int)std::min<int64_t>(kBloomSmemWords / nw, p.nfine) : 1;
        // Probing in S's first pass reads one random 32-byte block per S tuple; that is cheap only
        // while the filter stays in the 126 MB L2. A larger filter is probed in S's second pass,
        // one level-1 partition (a contiguous run of segments) at a time.
        int lvl = cfg.bloom_probe_level;
        if (lvl == 0) lvl = (p.bloom_bits / 8 <= kL1FilterBytes) ? 1 : 2;
        if (lvl != 1 && lvl != 2) fail(BRIG_E_INVALID, "bloom_probe_level must be 0, 1 or 2");
        if (f.P2 == 1) lvl = 1;
        p.bloom_level = lvl;
    }
    return p;
}

std::vector<JoinPlan> plan_batch(const brig_join_config& cfg, const int64_t* nr, const int64_t* ns, int nj,
                                 bool shared_l2) {
    std::vector<JoinPlan> plans(nj);
    for (int j = 0; j < nj; ++j) plans[j] = plan_join(cfg, nr[j], ns[j]);
    if (cfg.bloom_probe_level != 0 || (nj <= 1 && !shared_l2)) return plans;
    // One first-pass probe launch covers every join of the batch, so their filters share L2.
    // While they do not fit, the largest joins that have a second pass probe there instead.
    int64_t l1 = 0;
    std::vector<int> movable;
    for (int j = 0; j < nj; ++j) {
        const JoinPlan& p = plans[j];
        if (!p.bloom || p.bloom_level != 1) continue;
        l1 += p.bloom_bits / 8;
        if (p.pf.P2 > 1) movable.push_back(j);
    }
    std::stable_sort(movable.begin(), movable.end(),
                     [&](int a, int b) { return plans[a].bloom_bits > plans[b].bloom_bits; });
    for (int j : movable) {
        if (l1 <= kL2FilterBytes) break;
        plans[j].bloom_level = 2;
        l1 -= plans[j].bloom_bits / 8;
    }
    return plans;
}

// ---- workspace layout ---------------------------------------------------------------------------
namespace {

struct Layout {
    size_t off = 0;
    size_t take(size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        const size_t o = off;
        off += bytes;
        return o;
    }
};

}  // namespace

void layout_for(const brig_join_config& cfg, const JoinPlan* plans, int nj, int num_sms, JoinOffs* jo,
                Shape& sh) {
    sh = Shape{};
    sh.jo = jo;
    for (int j = 0; j < nj; ++j) jo[j] = JoinOffs{};
    // Level-1 slice length per launch class: R; S probed by the Bloom filter in its first pass;
    // the other S. Each class is one launch over all joins of the run that deals slices to CTAs
    // round-robin, so a class of n tuples is cut into about W x SMs slices (a multiple of the
    // scatter tile, at least 2 tiles): W = 4 for one join, whose slices are then equal, and 16 for
    // a batch, where every join ends in a partial slice and finer slices keep the CTAs' shares even.
    int64_t class_tuples[3] = {0, 0, 0};
    auto slice_class = [](const JoinPlan& p, int r) { return r == 0 ? 0 : (p.bloom && p.bloom_level == 1 ? 1 : 2); };
    for (int j = 0; j < nj; ++j)
        for (int r = 0; r < 2; ++r) class_tuples[slice_class(plans[j], r)] += r == 0 ? plans[j].nr : plans[j].ns;
    if (cfg.slices_per_sm < 0) fail(BRIG_E_INVALID, "slices_per_sm must be >= 0");
    const int per_sm = cfg.slices_per_sm > 0 ? cfg.slices_per_sm : (nj > 1 ? 16 : 4);
    const int64_t target = (int64_t)std::max(num_sms, 1) * per_sm;
    int64_t class_sl[3];
    for (int c = 0; c < 3; ++c) {
        int64_t sl = (class_tuples[c] + target - 1) / target;
        sl = ((sl + kSTile - 1) / kSTile) * kSTile;
        class_sl[c] = std::max<int64_t>(sl, 2 * kSTile);
    }
    sh.slice_len = class_sl[0];
    const int T = cfg.table_capacity > 0 ? cfg.table_capacity : kDefaultTable;
    const int C = cfg.s_chunk > 0 ? cfg.s_chunk : kDefaultChunk;
    Layout L;
    for (int j = 0; j < nj; ++j) {
        const JoinPlan& p = plans[j];
        JoinOffs& o = sh.jo[j];
        const int64_t n[2] = {p.nr, p.ns};
        const bool two = p.pf.P2 > 1;
        sh.max_p1 = std::max<int>(sh.max_p1, (int)p.pf.P1);
        sh.max_p2 = std::max<int>(sh.max_p2, (int)p.pf.P2);
        for (int r = 0; r < 2; ++r) {
            RelOffs& ro = o.rel[r];
            const int64_t sl = class_sl[slice_class(p, r)];
            ro.slice_len = sl;
            ro.nslices = (int32_t)std::max<int64_t>(1, (n[r] + sl - 1) / sl);
            ro.l1 = L.take((size_t)std::max<int64_t>(n[r], 1) * 8);
            if (two) ro.l2 = L.take((size_t)std::max<int64_t>(n[r], 1) * 8);
            ro.b1 = L.take(((size_t)p.pf.P1 + 1) * 8);
            if (two) ro.bounds = L.take(((size_t)p.nfine + 1) * 8);
            if (r == 1 && p.bloom) {
                ro.cmp = L.take((size_t)std::max<int64_t>(n[r], 1) * 8);
                if (p.bloom_level == 1) ro.slice_cnt = L.take((size_t)ro.nslices * 4);
            }
            ro.l2_slice = (r == 1 && p.bloom && p.bloom_level == 2) ? kL2SliceBloom : kL2Slice;
            if (two) sh.l2_slice_cap[r] += (int64_t)p.pf.P1 + n[r] / ro.l2_slice + 1;
            ro.hist_base = sh.hist_len[0] + sh.hist_len[1];  // provisional, fixed below
            sh.total_slices[r] += ro.nslices;
        }
        if (p.bloom) {
            o.bloom = L.take((size_t)p.nfine * p.seg_blocks * 32);
            sh.any_bloom = true;
            if (p.bloom_level == 1) sh.any_bloom_l1 = true;
            if (p.bloom_level == 2) sh.any_bloom_l2 = true;
            sh.total_bloom_groups += (p.nfine + p.bloom_group - 1) / p.bloom_group;
            const int64_t nw = (int64_t)p.seg_blocks * 8;
            sh.max_seg_words = std::max<int>(sh.max_seg_words, (int)nw);
            if (nw <= kBloomSmemWords)
                sh.bloom_smem_words = std::max<int>(sh.bloom_smem_words, (int)(nw * p.bloom_group));
        }
        if (two) sh.total_segs += p.pf.P1;
        sh.total_fine += p.nfine;
        sh.total_domains += two ? p.pf.P1 : 1;
        // Grouped tasks per domain: at most one group per finest partition, plus one task per
        // streamed chunk, plus the split chunks of oversized partitions.
        sh.task_cap += 2 * p.nfine + (p.nr + p.ns) / C + (p.nr + p.ns) / T + 4;
    }
    // Histograms: all R regions, then all S regions (each scanned as one sequence).
    for (int r = 0; r < 2; ++r) {
        int64_t base = (r == 0) ? 0 : sh.hist_len[0];
        for (int j = 0; j < nj; ++j) {
            RelOffs& ro = sh.jo[j].rel[r];
            ro.hist_base = base;
            base += (int64_t)plans[j].pf.P1 * ro.nslices + 1;
        }
        sh.hist_len[r] = base - ((r == 0) ? 0 : sh.hist_len[0]);
    }
    // Level-2 histograms [p][q][slice] per join, sized by the slice bound P1 + n / l2_slice + 1.
    for (int r = 0; r < 2; ++r) {
        int64_t base = (r == 0) ? 0 : sh.h2_len[0];
        for (int j = 0; j < nj; ++j) {
            const JoinPlan& p = plans[j];
            RelOffs& ro = sh.jo[j].rel[r];
            ro.h2_base = base;
            if (p.pf.P2 > 1) {
                const int64_t n = r == 0 ? p.nr : p.ns;
                base += ((int64_t)p.pf.P1 + n / ro.l2_slice + 1) * p.pf.P2 + 1;
            }
        }
        sh.h2_len[r] = base - ((r == 0) ? 0 : sh.h2_len[0]);
    }
    const int64_t h2_total = std::max<int64_t>(1, sh.h2_len[0] + sh.h2_len[1]);
    sh.hist2 = L.take((size_t)h2_total * 4);
    sh.hist2_scan = L.take((size_t)h2_total * 8);
    sh.seg_ns = L.take(((size_t)sh.total_segs + 1) * 4);
    sh.seg_off = L.take(((size_t)sh.total_segs + 1) * 8);
    sh.slice_cnt2 = L.take((size_t)std::max<int64_t>(1, std::max(sh.l2_slice_cap[0], sh.l2_slice_cap[1])) * 4);
    const int64_t hist_total = sh.hist_len[0] + sh.hist_len[1];
    sh.hist = L.take((size_t)hist_total * 4);
    sh.hist_scan = L.take((size_t)hist_total * 8);
    sh.tcount = L.take(((size_t)sh.total_domains + 1) * 4);
    sh.toff = L.take(((size_t)sh.total_domains + 1) * 8);
    sh.tasks = L.take((size_t)sh.task_cap * sizeof(Task));
    sh.scan_tmp_len = std::max({scan_tmp_words(std::max(sh.hist_len[0], sh.hist_len[1])),
                                scan_tmp_words(sh.total_domains + 1), scan_tmp_words(sh.total_segs + 1),
                                scan_tmp_words(std::max(sh.h2_len[0], sh.h2_len[1]))});
    sh.scan_tmp = L.take((size_t)sh.scan_tmp_len * 8);
    sh.gwords = L.take(kGWords * 8);
    sh.counters = L.take((size_t)nj * kCntWords * 8);
    sh.meta_bytes = (size_t)nj * sizeof(JoinDesc) + 5 * ((size_t)nj + 1) * 8;
    sh.meta = L.take(sh.meta_bytes);
    sh.total = L.off + 256;
}

int64_t Engine::workspace_needed(const brig_join_config& cfg, const std::vector<JoinPlan>& plans,
                                 int num_sms) {
    std::vector<JoinOffs> jo(plans.size());
    Shape sh;
    layout_for(cfg, plans.data(), (int)plans.size(), num_sms, jo.data(), sh);
    return (int64_t)sh.total;
}

Engine::Engine(const brig_join_config& cfg) : cfg_(cfg) {
    if (cfg.device >= 0) cuda_check(cudaSetDevice(cfg.device), "cudaSetDevice");
    cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_),
               "cudaDeviceGetAttribute");
    int major = 0;
    cuda_check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device_),
               "cudaDeviceGetAttribute");
    if (major != 10) fail(BRIG_E_UNSUPPORTED, "this build targets sm_100a (B200)");
    cuda_check(cudaEventCreateWithFlags(&stage_free_, cudaEventDisableTiming), "cudaEventCreate");
    cuda_check(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming), "cudaEventCreate");
    if (cfg.profile_stages) {
        for (auto& set : stage_ev_)
            for (auto& e : set) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        profiling_ = true;
    }
}

int Engine::stage_times(double* ms, int n) {
    if (!profiling_) fail(BRIG_E_INVALID, "handle created without profile_stages");
    if (!have_run_) fail(BRIG_E_INVALID, "no run on this handle");
    cuda_check(cudaEventSynchronize(done_), "cudaEventSynchronize");
    const int64_t first = std::max(runs_read_, runs_recorded_ - kStageRing);
    const int runs = (int)(runs_recorded_ - first);
    for (int i = 0; i < n && i < kNumStages; ++i) ms[i] = 0.0;
    for (int64_t r = first; r < runs_recorded_; ++r) {
        cudaEvent_t* ev = stage_ev_[r % kStageRing];
        for (int i = 0; i < n && i < kNumStages; ++i) {
            float t = 0.f;
            cuda_check(cudaEventElapsedTime(&t, ev[i], ev[i + 1]), "cudaEventElapsedTime");
            ms[i] += t;
        }
    }
    if (runs > 0)
        for (int i = 0; i < n && i < kNumStages; ++i) ms[i] /= runs;
    runs_read_ = runs_recorded_;
    return runs;
}

Engine::~Engine() {
    if (have_run_) cudaEventSynchronize(done_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (ws_) cudaFree(ws_);
    if (stage_) cudaFreeHost(stage_);
    if (surv_host_) cudaFreeHost(surv_host_);
    if (surv_ev_) cudaEventDestroy(surv_ev_);
    if (hio.rk) cudaFree(hio.rk);
    if (hio.rv) cudaFree(hio.rv);
    if (hio.sk) cudaFree(hio.sk);
    if (hio.sv) cudaFree(hio.sv);
    if (hio.outr) cudaFree(hio.outr);
    if (hio.outs) cudaFree(hio.outs);
    if (hio.outk) cudaFree(hio.outk);
    for (auto& set : stage_ev_)
        for (auto& e : set)
            if (e) cudaEventDestroy(e);
    if (stage_free_) cudaEventDestroy(stage_free_);
    if (done_) cudaEventDestroy(done_);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (d2h_stream) cudaStreamDestroy(d2h_stream);
    for (cudaEvent_t ev : chunk_done) cudaEventDestroy(ev);
    if (chunk_count) cudaFreeHost(chunk_count);
    if (r_copied) cudaEventDestroy(r_copied);
    if (s_copied) cudaEventDestroy(s_copied);
    for (int b = 0; b < 2; ++b) {
        if (chunk_copied[b]) cudaEventDestroy(chunk_copied[b]);
        if (chunk_free[b]) cudaEventDestroy(chunk_free[b]);
    }
}

// Growing the workspace is stream-ordered (cudaFreeAsync / cudaMallocAsync on the run's stream,
// after the handle's previous run), so it never synchronises the device: other handles' work on
// other streams, e.g. the other slots of a server, keeps running.
void Engine::ensure_workspace(size_t bytes, cudaStream_t stream) {
    if (bytes <= ws_bytes_) return;
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
        graph_key_.clear();
    }
    if (ws_) cuda_check(cudaFreeAsync(ws_, stream), "workspace cudaFreeAsync");
    ws_ = nullptr;
    ws_bytes_ = 0;
    cuda_check(cudaMallocAsync(&ws_, bytes, stream), "workspace cudaMallocAsync");
    ws_bytes_ = bytes;
}

void Engine::ensure_staging(size_t bytes) {
    if (bytes <= stage_bytes_) return;
    if (have_run_) cuda_check(cudaEventSynchronize(done_), "cudaEventSynchronize");
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
        graph_key_.clear();
    }
    if (stage_) cudaFreeHost(stage_);
    stage_ = nullptr;
    stage_bytes_ = 0;
    const size_t b = std::max<size_t>(bytes, 64 * 1024);
    cuda_check(cudaMallocHost(&stage_, b), "pinned staging cudaMallocHost");
    stage_bytes_ = b;
}

static void grow(uint32_t*& p, int64_t& cap, int64_t need) {
    if (need <= cap && p) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cuda_check(cudaMalloc(&p, (size_t)std::max<int64_t>(need, 1) * 4), "io cudaMalloc");
    cap = need;
}

void Engine::ensure_host_io(int64_t nr, int64_t ns, int64_t cap, bool key) {
    if (have_run_) cuda_check(cudaEventSynchronize(done_), "cudaEventSynchronize");
    int64_t c = hio.cap_in_r;
    grow(hio.rk, c, nr);
    c = hio.cap_in_r;
    grow(hio.rv, c, nr);
    hio.cap_in_r = std::max(hio.cap_in_r, nr);
    c = hio.cap_in_s;
    grow(hio.sk, c, ns);
    c = hio.cap_in_s;
    grow(hio.sv, c, ns);
    hio.cap_in_s = std::max(hio.cap_in_s, ns);
    c = hio.cap_out;
    grow(hio.outr, c, cap);
    c = hio.cap_out;
    grow(hio.outs, c, cap);
    if (key) {
        c = hio.outk_alloc ? hio.cap_out : 0;
        grow(hio.outk, c, cap);
        hio.outk_alloc = true;
    }
    hio.cap_out = std::max(hio.cap_out, cap);
    if (!copy_stream) {
        cuda_check(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreateWithFlags(&r_copied, cudaEventDisableTiming), "cudaEventCreate");
        cuda_check(cudaEventCreateWithFlags(&s_copied, cudaEventDisableTiming), "cudaEventCreate");
        for (int b = 0; b < 2; ++b) {
            cuda_check(cudaEventCreateWithFlags(&chunk_copied[b], cudaEventDisableTiming), "cudaEventCreate");
            cuda_check(cudaEventCreateWithFlags(&chunk_free[b], cudaEventDisableTiming), "cudaEventCreate");
        }
    }
}

void Engine::run_host_chunked(const uint32_t* rk, const uint32_t* rv, int64_t nr, const uint32_t* sk,
                              const uint32_t* sv, int64_t ns, int chunks, int64_t cap, bool emit_key,
                              cudaStream_t st) {
    if (nr <= 0 || ns <= 0 || chunks < 2) fail(BRIG_E_INVALID, "chunked join needs R, S and at least 2 chunks");
    const int64_t chunk = (ns + chunks - 1) / chunks;
    const int64_t nc = (ns + chunk - 1) / chunk;
    ensure_host_io(nr, 2 * chunk, cap, emit_key);  // waits for the handle's previous run
    if (chunk_count_cap < nc) {
        if (chunk_count) cudaFreeHost(chunk_count);
        chunk_count = nullptr;
        chunk_count_cap = 0;
        cuda_check(cudaMallocHost(&chunk_count, (size_t)nc * sizeof(int64_t)), "cudaMallocHost");
        chunk_count_cap = (int)nc;
    }
    while ((int64_t)chunk_done.size() < nc) {
        cudaEvent_t ev;
        cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        chunk_done.push_back(ev);
    }
    if (!d2h_stream) cuda_check(cudaStreamCreateWithFlags(&d2h_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    // One plan and one workspace layout for every chunk, sized by the largest chunk: R's buffers and
    // the filter stay where they are, and a smaller last chunk only leaves trailing slices empty.
    std::vector<JoinPlan> plans{plan_join(cfg_, nr, chunk)};
    JoinOffs jo;
    Shape sh;
    layout_for(cfg_, plans.data(), 1, num_sms_, &jo, sh);
    ensure_workspace(sh.total, st);
    char* ws = ws_;
    int64_t* counters = reinterpret_cast<int64_t*>(ws + sh.counters);
    std::vector<char> meta(sh.meta_bytes);
    const brig_join_output out{hio.outr, hio.outs, emit_key ? hio.outk : nullptr, cap, nullptr};
    PipelineArgs a{};
    // the descriptors go up from pageable memory: the copy returns once they are staged
    auto launch = [&](const JoinIO& io, int stages, bool keep_errors) {
        fill_pipeline(cfg_, plans.data(), &io, 1, sh, ws, meta.data(), num_sms_, a);
        a.stages = stages;
        a.keep_errors = keep_errors ? 1 : 0;
        cuda_check(cudaMemcpyAsync(ws + sh.meta, meta.data(), sh.meta_bytes, cudaMemcpyHostToDevice, st),
                   "descriptor upload");
        cuda_check(enqueue_pipeline(a, st), "pipeline launch");
    };
    // R: copied once, then its two passes and the Bloom build
    cuda_check(cudaMemcpyAsync(hio.rk, rk, (size_t)nr * 4, cudaMemcpyHostToDevice, st), "H2D R keys");
    cuda_check(cudaMemcpyAsync(hio.rv, rv, (size_t)nr * 4, cudaMemcpyHostToDevice, st), "H2D R vals");
    cuda_check(cudaEventRecord(r_copied, st), "cudaEventRecord");
    cuda_check(cudaMemsetAsync(counters, 0, (size_t)kCntWords * 8, st), "counter reset");
    launch(JoinIO{hio.rk, hio.rv, hio.sk, hio.sv, nr, std::min(chunk, ns), out}, kRunPartR | kRunBloom, false);
    // S: chunk c into buffer c % 2; its copy waits for R's copy (first chunk) or for the end of the
    // passes of chunk c - 2 (same buffer); its passes wait for its copy
    for (int64_t c = 0; c < nc; ++c) {
        const int b = (int)(c & 1);
        const int64_t off = c * chunk, n = std::min(chunk, ns - off);
        uint32_t* dk = hio.sk + (size_t)b * chunk;
        uint32_t* dv = hio.sv + (size_t)b * chunk;
        if (c == 0) cuda_check(cudaStreamWaitEvent(copy_stream, r_copied, 0), "cudaStreamWaitEvent");
        if (c >= 2) cuda_check(cudaStreamWaitEvent(copy_stream, chunk_free[b], 0), "cudaStreamWaitEvent");
        cuda_check(cudaMemcpyAsync(dk, sk + off, (size_t)n * 4, cudaMemcpyHostToDevice, copy_stream), "H2D S keys");
        cuda_check(cudaMemcpyAsync(dv, sv + off, (size_t)n * 4, cudaMemcpyHostToDevice, copy_stream), "H2D S vals");
        cuda_check(cudaEventRecord(chunk_copied[b], copy_stream), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(st, chunk_copied[b], 0), "cudaStreamWaitEvent");
        launch(JoinIO{hio.rk, hio.rv, dk, dv, nr, n, out}, kRunPartS | kRunProbe, true);
        cuda_check(cudaEventRecord(chunk_free[b], st), "cudaEventRecord");
        // the pairs so far end at the match count (each chunk's probe appends after the previous one's)
        cuda_check(cudaMemcpyAsync(chunk_count + c, counters + kCntMatches, sizeof(int64_t), cudaMemcpyDeviceToHost, st),
                   "chunk count read-back");
        cuda_check(cudaEventRecord(chunk_done[c], st), "cudaEventRecord");
    }
    chunks_run = (int)nc;
    cuda_check(cudaEventRecord(done_, st), "cudaEventRecord");
    have_run_ = true;
    plans_ = plans;
    caps_.assign(1, cap);
    d_counters_ = counters;
    d_gwords_ = a.gwords;
    nj_ = 1;
}

void fill_pipeline(const brig_join_config& cfg, const JoinPlan* plans, const JoinIO* joins, int nj,
                   const Shape& sh, char* ws, char* meta_host, int num_sms, PipelineArgs& a) {
    const int T = cfg.table_capacity > 0 ? cfg.table_capacity : kDefaultTable;
    const int C = cfg.s_chunk > 0 ? cfg.s_chunk : kDefaultChunk;
    if (T < kMinTable || T > kMaxTable || !is_pow2(T))
        fail(BRIG_E_INVALID, "table_capacity must be a power of two in [256, 4096]");
    if (C < 1) fail(BRIG_E_INVALID, "s_chunk must be >= 1");
    // The Bloom kernels fill their pattern table for the k of the first filtered join; the joins of
    // one run share their configuration, so that is every filtered join's k (checked below).
    int run_k = 0;
    for (int j = 0; j < nj && !run_k; ++j)
        if (plans[j].bloom) run_k = plans[j].k;
    const int pat_k = run_k == kBloomFastK ? 0 : run_k;  // k = 7 masks need no table
    JoinDesc* hJ = reinterpret_cast<JoinDesc*>(meta_host);
    int64_t* hpre = reinterpret_cast<int64_t*>(meta_host + (size_t)nj * sizeof(JoinDesc));
    int64_t* sp0 = hpre;
    int64_t* sp1 = hpre + (nj + 1);
    int64_t* segp = hpre + 2 * (nj + 1);
    int64_t* finep = hpre + 3 * (nj + 1);
    int64_t* bloomp = hpre + 4 * (nj + 1);
    sp0[0] = sp1[0] = segp[0] = finep[0] = bloomp[0] = 0;  // finep: task domains
    int64_t* counters = reinterpret_cast<int64_t*>(ws + sh.counters);
    for (int j = 0; j < nj; ++j) {
        const JoinPlan& p = plans[j];
        const JoinOffs& o = sh.jo[j];
        const JoinIO& io = joins[j];
        JoinDesc d;
        std::memset(&d, 0, sizeof(d));
        const uint32_t* keys[2] = {io.rk, io.sk};
        const uint32_t* vals[2] = {io.rv, io.sv};
        const int64_t n[2] = {io.nr, io.ns};
        for (int r = 0; r < 2; ++r) {
            RelPlan& R = d.rel[r];
            const RelOffs& ro = o.rel[r];
            R.key = keys[r];
            R.val = vals[r];
            R.n = n[r];
            R.l1 = reinterpret_cast<uint2*>(ws + ro.l1);
            R.l2 = p.pf.P2 > 1 ? reinterpret_cast<uint2*>(ws + ro.l2) : nullptr;
            R.cmp = ro.cmp ? reinterpret_cast<uint2*>(ws + ro.cmp) : nullptr;
            R.slice_len = ro.slice_len;
            R.nslices = ro.nslices;
            R.l2_slice = (int32_t)ro.l2_slice;
            R.hist_base = ro.hist_base;
            R.b1 = reinterpret_cast<int64_t*>(ws + ro.b1);
            R.bounds = p.pf.P2 > 1 ? reinterpret_cast<int64_t*>(ws + ro.bounds) : R.b1;
            R.slice_cnt = ro.slice_cnt ? reinterpret_cast<uint32_t*>(ws + ro.slice_cnt) : nullptr;
            R.h2_base = ro.h2_base;
        }
        d.pf = p.pf;
        d.out_r = io.out.r_val;
        d.out_s = io.out.s_val;
        d.out_k = io.out.key;
        d.cap = io.out.capacity;
        d.counters = counters + (size_t)j * kCntWords;
        d.user_count = io.out.d_count;
        d.bloom = p.bloom ? reinterpret_cast<uint32_t*>(ws + o.bloom) : nullptr;
        d.seg_blocks = p.seg_blocks;
        d.bloom_k = p.k;
        d.bloom_level = p.bloom_level;
        d.fine_base = 0;
        d.dom_base = finep[j];
        d.bloom_group = p.bloom_group;
        if (p.bloom && p.k != run_k)
            fail(BRIG_E_INVALID, "the filtered joins of one run must share their number of Bloom hashes");
        d.table_cap = T;
        d.s_chunk = C;
        hJ[j] = d;
        sp0[j + 1] = sp0[j] + o.rel[0].nslices;
        sp1[j + 1] = sp1[j] + o.rel[1].nslices;
        segp[j + 1] = segp[j] + (p.pf.P2 > 1 ? p.pf.P1 : 0);
        finep[j + 1] = finep[j] + (p.pf.P2 > 1 ? p.pf.P1 : 1);
        bloomp[j + 1] = bloomp[j] + (p.bloom ? (p.nfine + p.bloom_group - 1) / p.bloom_group : 0);
    }
    char* meta = ws + sh.meta;
    const int64_t* dpre = reinterpret_cast<const int64_t*>(meta + (size_t)nj * sizeof(JoinDesc));
    a = PipelineArgs{};
    a.J = reinterpret_cast<const JoinDesc*>(meta);
    a.nj = nj;
    a.slice_prefix[0] = dpre;
    a.slice_prefix[1] = dpre + (nj + 1);
    a.seg_prefix = dpre + 2 * (nj + 1);
    a.fine_prefix = nullptr;
    a.dom_prefix = dpre + 3 * (nj + 1);
    a.bloom_prefix = dpre + 4 * (nj + 1);
    a.total_slices[0] = sh.total_slices[0];
    a.total_slices[1] = sh.total_slices[1];
    a.total_segs = sh.total_segs;
    a.total_fine = sh.total_fine;
    a.total_bloom_groups = sh.total_bloom_groups;
    a.total_domains = sh.total_domains;
    a.bloom_smem_words = sh.bloom_smem_words;
    a.hist_begin[0] = 0;
    a.hist_len[0] = sh.hist_len[0];
    a.hist_begin[1] = sh.hist_len[0];
    a.hist_len[1] = sh.hist_len[1];
    a.hist = reinterpret_cast<uint32_t*>(ws + sh.hist);
    a.hist_scan = reinterpret_cast<int64_t*>(ws + sh.hist_scan);
    a.tcount = reinterpret_cast<uint32_t*>(ws + sh.tcount);
    a.toff = reinterpret_cast<int64_t*>(ws + sh.toff);
    a.tasks = reinterpret_cast<Task*>(ws + sh.tasks);
    a.task_cap = sh.task_cap;
    a.scan_tmp = reinterpret_cast<int64_t*>(ws + sh.scan_tmp);
    a.scan_tmp_len = sh.scan_tmp_len;
    a.gwords = reinterpret_cast<unsigned long long*>(ws + sh.gwords);
    a.max_p1 = sh.max_p1;
    a.max_p2 = sh.max_p2;
    a.max_seg_words = sh.max_seg_words;
    a.table_cap = T;
    a.emit_key = 0;
    for (int j = 0; j < nj; ++j)
        if (joins[j].out.key) a.emit_key = 1;
    a.any_bloom = sh.any_bloom ? 1 : 0;
    a.any_bloom_l1 = sh.any_bloom_l1 ? 1 : 0;
    a.any_bloom_l2 = sh.any_bloom_l2 ? 1 : 0;
    a.modes = 0;
    for (int j = 0; j < nj; ++j) a.modes |= plans[j].pf.mode == 0 ? 1 : 2;
    a.pat_k = pat_k;
    a.kclasses = 0;
    for (int j = 0; j < nj; ++j) a.kclasses |= (plans[j].bloom && plans[j].k == kBloomFastK) ? 2 : 1;
    a.all_bloom_l2 = 1;
    for (int j = 0; j < nj; ++j)
        if (plans[j].pf.P2 > 1 && !(plans[j].bloom && plans[j].bloom_level == 2)) a.all_bloom_l2 = 0;
    a.num_sms = num_sms;
    if (cfg.wait_poll_limit < -1) fail(BRIG_E_INVALID, "wait_poll_limit must be >= -1");
    a.wait_polls = cfg.wait_poll_limit == 0 ? kDefaultWaitPolls
                   : cfg.wait_poll_limit < 0 ? 0u : (uint32_t)cfg.wait_poll_limit;
    a.stage_events = nullptr;
    a.stages = kRunAll;
    a.seg_ns = reinterpret_cast<uint32_t*>(ws + sh.seg_ns);
    a.seg_off = reinterpret_cast<int64_t*>(ws + sh.seg_off);
    a.hist2 = reinterpret_cast<uint32_t*>(ws + sh.hist2);
    a.hist2_scan = reinterpret_cast<int64_t*>(ws + sh.hist2_scan);
    a.h2_begin[0] = 0;
    a.h2_len[0] = sh.h2_len[0];
    a.h2_begin[1] = sh.h2_len[0];
    a.h2_len[1] = sh.h2_len[1];
    a.slice_cnt2 = reinterpret_cast<uint32_t*>(ws + sh.slice_cnt2);
    a.l2_slice_cap[0] = sh.l2_slice_cap[0];
    a.l2_slice_cap[1] = sh.l2_slice_cap[1];
    // Scatter forms. The small bulk-store form (two CTAs per SM, half-size tiles) hides the
    // per-slice start-up and the per-tile barriers of one CTA behind the other's work, which is what
    // short slices need; the full-size tiles' longer runs per bin win on long slices over many bins.
    // Slices are short below 64K tuples, or below 256K when there are at most 128 bins (runs of 48
    // or more tuples per half tile). S's level-2 input is the filter's survivors when its filter is
    // probed at level 2: a fraction of slices of 131072 tuples, short in any case. Measured at 640M
    // x 640M (512 x 512 bins): level-1 slices of 1M tuples, level-2 slices of R of 214K tuples in the
    // large form; survivors 0.52 ms in the small form against 0.69 in the large one.
    int64_t rel_n[2] = {0, 0};
    for (int j = 0; j < nj; ++j) {
        rel_n[0] += plans[j].nr;
        rel_n[1] += plans[j].ns;
    }
    auto form_for = [](int bins, int64_t avg_slice, bool short_slices) {
        if (bins > kBulkMaxBins) return (int)kFormPass;
        if (bins <= kBulkSmallMaxBins &&
            (short_slices || avg_slice < 65536 || (bins <= 128 && avg_slice < 262144)))
            return (int)kFormBulkSmall;
        return (int)kFormBulk;
    };
    for (int r = 0; r < 2; ++r) {
        a.l1_form[r] = form_for(sh.max_p1, rel_n[r] / std::max<int64_t>(1, sh.total_slices[r]), false);
        a.l2_form[r] = form_for(sh.max_p2, rel_n[r] / std::max<int64_t>(1, sh.l2_slice_cap[r]),
                                r == 1 && sh.any_bloom_l2);
    }
}

void Engine::run(const std::vector<JoinIO>& joins, cudaStream_t stream, bool use_graph, cudaEvent_t s_ready) {
    if (s_ready) use_graph = false;
    const int nj = (int)joins.size();
    if (nj <= 0) fail(BRIG_E_INVALID, "no joins");
    std::vector<int64_t> nr(nj), ns(nj);
    for (int j = 0; j < nj; ++j) {
        nr[j] = joins[j].nr;
        ns[j] = joins[j].ns;
    }
    std::vector<JoinPlan> plans = plan_batch(adapt_config(nj), nr.data(), ns.data(), nj, shared_l2_);
    std::vector<JoinOffs> jo(nj);
    Shape sh;
    layout_for(cfg_, plans.data(), nj, num_sms_, jo.data(), sh);
    // A handle's runs are ordered even across streams: this run's work (and a workspace growth)
    // starts after the previous run's last operation.
    if (have_run_) cuda_check(cudaStreamWaitEvent(stream, done_, 0), "cudaStreamWaitEvent");
    ensure_workspace(sh.total, stream);
    ensure_staging(sh.meta_bytes);
    // The staging buffer may still be read by the previous run's copy.
    if (have_run_) cuda_check(cudaEventSynchronize(stage_free_), "cudaEventSynchronize");

    char* ws = ws_;
    PipelineArgs a{};
    fill_pipeline(cfg_, plans.data(), joins.data(), nj, sh, ws, stage_, num_sms_, a);
    char* meta = ws + sh.meta;
    int64_t* counters = reinterpret_cast<int64_t*>(ws + sh.counters);
    // Stage events are plain stream records, so a profiled handle launches directly (a record
    // captured into a graph is only a dependency edge, not a timestamp).
    if (profiling_) use_graph = false;
    a.stage_events = profiling_ ? stage_ev_[runs_recorded_ % kStageRing] : nullptr;
    a.s_ready = s_ready;

    auto enqueue_all = [&](cudaStream_t st) {
        cuda_check(cudaMemcpyAsync(meta, stage_, sh.meta_bytes, cudaMemcpyHostToDevice, st),
                   "descriptor upload");
        // Outside capture the staging buffer is free once this copy has run, so the next run's
        // host work overlaps this run's kernels.
        if (!use_graph) cuda_check(cudaEventRecord(stage_free_, st), "cudaEventRecord");
        cuda_check(cudaMemsetAsync(counters, 0, (size_t)nj * kCntWords * 8, st), "counter reset");
        cuda_check(enqueue_pipeline(a, st), "pipeline launch");
    };

    // Graph key: everything that shapes the launch sequence (sizes, plans, workspace address).
    std::vector<int64_t> key;
    if (use_graph) {
        key.reserve(8 + (size_t)nj * 8);
        key.push_back((int64_t)(uintptr_t)ws_);
        key.push_back(nj);
        key.push_back(a.emit_key);
        for (int j = 0; j < nj; ++j) {
            key.push_back(plans[j].nr);
            key.push_back(plans[j].ns);
            key.push_back(plans[j].pf.P1);
            key.push_back(plans[j].pf.P2);
            key.push_back(plans[j].bloom ? (int64_t)plans[j].seg_blocks : (int64_t)-1);
            key.push_back(plans[j].bloom_level);
        }
    }
    if (use_graph) {
        if (!(graph_exec_ && key == graph_key_)) {
            if (graph_exec_) {
                cudaGraphExecDestroy(graph_exec_);
                graph_exec_ = nullptr;
            }
            // Kernel attributes are set on the first direct launch, outside capture.
            if (!have_run_) {
                enqueue_all(stream);
                cuda_check(cudaStreamSynchronize(stream), "warm-up run");
            }
            cudaStream_t cs;
            cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
            cudaGraph_t g;
            cuda_check(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
            set_capturing(true);
            try {
                enqueue_all(cs);
            } catch (...) {
                set_capturing(false);
                cudaStreamEndCapture(cs, &g);
                cudaStreamDestroy(cs);
                throw;
            }
            set_capturing(false);
            graph_kernels_ = take_capture_tally();
            cuda_check(cudaStreamEndCapture(cs, &g), "end capture");
            cudaStreamDestroy(cs);
            cudaError_t e = cudaGraphInstantiate(&graph_exec_, g, 0);
            cudaGraphDestroy(g);
            cuda_check(e, "cudaGraphInstantiate");
            graph_key_ = key;
        }
        cuda_check(cudaGraphLaunch(graph_exec_, stream), "cudaGraphLaunch");
        note_launches((int)graph_kernels_);
    } else {
        enqueue_all(stream);
    }
    if (use_graph) cuda_check(cudaEventRecord(stage_free_, stream), "cudaEventRecord");
    note_survivors(plans, counters, stream);
    cuda_check(cudaEventRecord(done_, stream), "cudaEventRecord");
    have_run_ = true;
    if (profiling_) ++runs_recorded_;
    plans_ = plans;
    caps_.resize(nj);
    for (int j = 0; j < nj; ++j) caps_[j] = joins[j].out.capacity;
    d_counters_ = counters;
    d_gwords_ = a.gwords;
    nj_ = nj;
}

// The adaptive filter's break-even: at |R| = 2^26, |S| = 2^30 and 10 bits/key the filtered join
// took 13.9 ms against 15.0 ms unfiltered at 22% survivors, 16.1 against 15.9 ms at 31% and 18.4
// against 16.8 ms at 41%; above this share of S passing the filter, a join runs faster without it.
constexpr double kBloomOffShare = 0.30;
constexpr int kBloomRetest = 16;  // while the filter is off, every 16th run tests it again

brig_join_config Engine::adapt_config(int nj) {
    brig_join_config c = cfg_;
    if (cfg_.use_bloom != BRIG_BLOOM_ADAPTIVE) return c;
    c.use_bloom = 1;
    // the last filtered run's survivor count, once it has arrived (never waits for it)
    if (surv_pending_ && cudaEventQuery(surv_ev_) == cudaSuccess) {
        surv_pending_ = false;
        const bool off = surv_ns_ > 0 && (double)*surv_host_ > kBloomOffShare * (double)surv_ns_;
        if (off != bloom_off_) runs_off_ = 0;
        bloom_off_ = off;
    }
    if (nj == 1 && bloom_off_) {
        if (++runs_off_ < kBloomRetest) c.use_bloom = 0;
        else runs_off_ = 0;  // this run tests the filter again
    }
    return c;
}

void Engine::note_survivors(const std::vector<JoinPlan>& plans, const int64_t* counters, cudaStream_t stream) {
    if (cfg_.use_bloom != BRIG_BLOOM_ADAPTIVE || plans.size() != 1 || !plans[0].bloom) return;
    if (!surv_host_) {
        cuda_check(cudaMallocHost(&surv_host_, sizeof(int64_t)), "cudaMallocHost");
        cuda_check(cudaEventCreateWithFlags(&surv_ev_, cudaEventDisableTiming), "cudaEventCreate");
    }
    // a newer copy replaces one still in flight: the event then marks the newer one
    cuda_check(cudaMemcpyAsync(surv_host_, counters + kCntSurvivors, sizeof(int64_t), cudaMemcpyDeviceToHost, stream),
               "survivor count read-back");
    cuda_check(cudaEventRecord(surv_ev_, stream), "cudaEventRecord");
    surv_pending_ = true;
    surv_ns_ = plans[0].ns;
}

std::vector<brig_join_config> autotune_candidates(const brig_join_config& base) {
    std::vector<brig_join_config> out;
    for (int dim = 0; dim < kTuneDims; ++dim)
        for (int v = 0; v < tune_values(dim); ++v) out.push_back(tune_apply(base, dim, v));
    return out;
}

int tune_values(int dim) {
    static const int n[kTuneDims] = {4, 3, 4, 3, 3};
    return (dim >= 0 && dim < kTuneDims) ? n[dim] : 0;
}

brig_join_config tune_apply(const brig_join_config& base, int dim, int v) {
    brig_join_config c = base;
    switch (dim) {
        case 0: {  // Bloom prefilter: off; 8 bits/key (k = 6); 10 bits/key (k = 7), auto or second pass
            static const int use[] = {0, 1, 1, 1}, k[] = {0, 6, 7, 7}, lvl[] = {0, 0, 0, 2};
            static const double bpk[] = {0.0, 8.0, 10.0, 10.0};
            c.use_bloom = use[v];
            c.bloom_bits_per_key = use[v] ? bpk[v] : 10.0;
            c.bloom_num_hashes = k[v];
            c.bloom_num_bits = 0;
            c.bloom_probe_level = lvl[v];
            break;
        }
        case 1: {
            static const int t[] = {1024, 2048, 4096};
            c.table_capacity = t[v];
            break;
        }
        case 2: {
            static const int b[] = {7, 8, 9, 10};
            c.max_level1_bits = b[v];
            break;
        }
        case 3: {
            static const int f[] = {50, 75, 100};
            c.partition_fill = f[v];
            break;
        }
        case 4: {
            static const int w[] = {8, 16, 32};
            c.slices_per_sm = w[v];
            break;
        }
    }
    return c;
}

brig_join_config Engine::autotune(const std::vector<JoinIO>& joins, cudaStream_t stream) {
    // Coordinate search: from the handle's configuration, each dimension in turn takes the value
    // whose median time over three runs (after a warm-up run that also sizes the workspace) is
    // lowest, the others held; passes repeat while one improves the time by more than 2%. No
    // candidate changes a join's result, only its speed.
    const brig_join_config base = cfg_;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    auto time_cfg = [&](const brig_join_config& c) {
        cfg_ = c;
        cfg_.profile_stages = 0;
        run(joins, stream, false);  // warm-up (sizes the workspace)
        float t[3];
        for (float& x : t) {
            cuda_check(cudaEventRecord(e0, stream), "cudaEventRecord");
            run(joins, stream, false);
            cuda_check(cudaEventRecord(e1, stream), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
            cuda_check(cudaEventElapsedTime(&x, e0, e1), "cudaEventElapsedTime");
        }
        std::sort(t, t + 3);
        return t[1];
    };
    brig_join_config best_cfg = base;
    try {
        float best = time_cfg(best_cfg);
        for (int pass = 0; pass < 3; ++pass) {
            const float start = best;
            for (int dim = 0; dim < kTuneDims; ++dim) {
                for (int v = 0; v < tune_values(dim); ++v) {
                    const brig_join_config c = tune_apply(best_cfg, dim, v);
                    if (std::memcmp(&c, &best_cfg, sizeof(c)) == 0) continue;
                    const float ms = time_cfg(c);
                    if (ms < best) {
                        best = ms;
                        best_cfg = c;
                    }
                }
            }
            if (best > start * 0.98f) break;
        }
    } catch (...) {
        cfg_ = base;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    best_cfg.profile_stages = base.profile_stages;
    cfg_ = best_cfg;
    if (graph_exec_) {
        cudaGraphExecDestroy(graph_exec_);
        graph_exec_ = nullptr;
        graph_key_.clear();
    }
    return cfg_;
}

void Engine::sync_counters(std::vector<int64_t>& counters, int64_t& errors) {
    if (!have_run_) fail(BRIG_E_INVALID, "no run on this handle");
    cuda_check(cudaEventSynchronize(done_), "cudaEventSynchronize");
    counters.assign((size_t)nj_ * kCntWords, 0);
    cuda_check(cudaMemcpy(counters.data(), d_counters_, counters.size() * 8, cudaMemcpyDeviceToHost),
               "counter readback");
    unsigned long long g[kGWords];
    cuda_check(cudaMemcpy(g, d_gwords_, sizeof(g), cudaMemcpyDeviceToHost), "state readback");
    errors = (int64_t)g[kGErrors];
}

}  // namespace brig
