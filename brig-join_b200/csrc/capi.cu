// capi.cu - the extern "C" boundary (include/brig_join.h). Every entry point catches engine errors
// and returns a status code; nothing here exits the process (the reference exits on any CUDA error,
// src/hash_kernel.cu:48-55).
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include "../../include/brig_join.h"
#include "brig_gen.cuh"
#include "engine.h"

using brig::Engine;
using brig::Error;
using brig::fail;

struct brig_join_t {
    Engine* eng = nullptr;
    int last_kind = 0;   // 1 single join, 2 batch
    int last_items = 0;
};

namespace {

thread_local std::string g_last_error;

int set_error(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <class F>
int guarded(F&& f) {
    try {
        g_last_error.clear();
        return f();
    } catch (const Error& e) {
        return (int)set_error(e.status, e.msg);
    } catch (const std::bad_alloc&) {
        return (int)set_error(BRIG_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return (int)set_error(BRIG_E_INTERNAL, e.what());
    } catch (...) {
        return (int)set_error(BRIG_E_INTERNAL, "unknown failure");
    }
}

void check_cfg(const brig_join_config* cfg) {
    if (!cfg) fail(BRIG_E_INVALID, "null config");
    if (cfg->abi_version != BRIG_JOIN_ABI_VERSION) fail(BRIG_E_INVALID, "config ABI version mismatch");
    if (cfg->partition_size < 0 || cfg->second_partition_size < 0 || cfg->table_capacity < 0 ||
        cfg->s_chunk < 0 || cfg->bloom_num_hashes < 0 || cfg->bloom_num_bits < 0 ||
        cfg->bloom_bits_per_key < 0 || cfg->s_chunks < 0)
        fail(BRIG_E_INVALID, "negative config field");
    if (cfg->bloom_num_hashes > brig::kMaxBloomK) fail(BRIG_E_INVALID, "bloom_num_hashes > 16");
}

void check_rel(const uint32_t* k, const uint32_t* v, int64_t n, const char* what) {
    if (n < 0) fail(BRIG_E_INVALID, std::string("negative size of ") + what);
    if (n > ((int64_t)1 << 33)) fail(BRIG_E_UNSUPPORTED, std::string(what) + " larger than 2^33 tuples");
    if (n > 0 && (!k || !v)) fail(BRIG_E_INVALID, std::string("null array for ") + what);
}

void check_out(const brig_join_output* out) {
    if (!out) fail(BRIG_E_INVALID, "null output");
    if (out->capacity < 0) fail(BRIG_E_INVALID, "negative output capacity");
    if (out->capacity > 0 && (!out->r_val || !out->s_val)) fail(BRIG_E_INVALID, "null output arrays");
}

}  // namespace

namespace brig {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace brig

extern "C" {

void brig_join_config_init(brig_join_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->abi_version = BRIG_JOIN_ABI_VERSION;
    cfg->partition_mode = BRIG_PART_HASH;
    cfg->bloom_bits_per_key = 10.0;
    cfg->device = -1;
}

int brig_join_create(const brig_join_config* cfg, brig_join_t** out) {
    return guarded([&] {
        check_cfg(cfg);
        if (!out) fail(BRIG_E_INVALID, "null handle pointer");
        *out = nullptr;
        auto* h = new brig_join_t;
        try {
            h->eng = new Engine(*cfg);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return (int)BRIG_OK;
    });
}

int brig_join_destroy(brig_join_t* h) {
    return guarded([&] {
        if (!h) return (int)BRIG_OK;
        delete h->eng;
        delete h;
        return (int)BRIG_OK;
    });
}

int brig_join_run(brig_join_t* h, const uint32_t* r_key, const uint32_t* r_val, int64_t n_r,
                  const uint32_t* s_key, const uint32_t* s_val, int64_t n_s, const brig_join_output* out,
                  void* stream) {
    return guarded([&] {
        if (!h) fail(BRIG_E_INVALID, "null handle");
        check_rel(r_key, r_val, n_r, "R");
        check_rel(s_key, s_val, n_s, "S");
        check_out(out);
        brig::JoinIO io{r_key, r_val, s_key, s_val, n_r, n_s, *out};
        h->eng->run({io}, static_cast<cudaStream_t>(stream), h->eng->config().use_cuda_graph != 0);
        h->last_kind = 1;
        h->last_items = 1;
        return (int)BRIG_OK;
    });
}

int brig_join_get_stats(brig_join_t* h, brig_join_stats* st) {
    return guarded([&] {
        if (!h || !st) fail(BRIG_E_INVALID, "null argument");
        std::memset(st, 0, sizeof(*st));
        std::vector<int64_t> c;
        int64_t errors = 0;
        h->eng->sync_counters(c, errors);
        const auto& plans = h->eng->last_plans();
        const auto& caps = h->eng->last_caps();
        int64_t count = 0, surv = 0, tasks = 0, split = 0, written = 0;
        bool overflow = false;
        for (size_t j = 0; j < plans.size(); ++j) {
            const int64_t* cj = c.data() + j * brig::kCntWords;
            count += cj[brig::kCntMatches];
            surv += cj[brig::kCntSurvivors];
            tasks += cj[brig::kCntTasks];
            split += cj[brig::kCntSplitTasks];
            written += std::min(cj[brig::kCntMatches], caps[j]);
            if (cj[brig::kCntMatches] > caps[j]) overflow = true;
        }
        st->count = count;
        st->written = written;
        st->s_survivors = surv;
        st->tasks = tasks;
        st->split_tasks = split;
        st->overflow = overflow ? 1 : 0;
        if (!plans.empty()) {
            st->partition_size = (int32_t)plans[0].pf.P1;
            st->second_partition_size = (int32_t)plans[0].pf.P2;
            st->bloom_num_hashes = plans[0].bloom ? plans[0].k : 0;
            st->bloom_num_bits = plans[0].bloom ? plans[0].bloom_bits : 0;
        }
        st->workspace_bytes = h->eng->workspace_bytes();
        if (errors != 0)
            fail(BRIG_E_INTERNAL, "device-side consistency check failed (" + std::to_string(errors) + ")");
        if (overflow) return (int)set_error(BRIG_E_OVERFLOW, "match count exceeds output capacity");
        return (int)BRIG_OK;
    });
}

// Inputs of at least this many tuples overlap S's host-to-device copy with R's passes.
static constexpr int64_t kSplitCopyTuples = 1 << 23;

// The end of a host-array join: waits for the counts, copies min(count, capacity) pairs back.
static int finish_host_run(brig_join_t* h, uint32_t* out_r_val, uint32_t* out_s_val, uint32_t* out_key,
                    int64_t capacity, int64_t* count, cudaStream_t st) {
    Engine& e = *h->eng;
    auto& b = e.hio;
    h->last_kind = 1;
    h->last_items = 1;
    std::vector<int64_t> c;
    int64_t errors = 0;
    e.sync_counters(c, errors);
    if (errors) fail(BRIG_E_INTERNAL, "device-side consistency check failed");
    const int64_t cnt = c[brig::kCntMatches];
    const int64_t n = std::min(cnt, capacity);
    if (n > 0) {
        brig::cuda_check(cudaMemcpyAsync(out_r_val, b.outr, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H r_val");
        brig::cuda_check(cudaMemcpyAsync(out_s_val, b.outs, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H s_val");
        if (out_key)
            brig::cuda_check(cudaMemcpyAsync(out_key, b.outk, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H key");
    }
    brig::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (count) *count = cnt;
    if (cnt > capacity) return (int)set_error(BRIG_E_OVERFLOW, "match count exceeds output capacity");
    return (int)BRIG_OK;
}

// The end of a host-array join with S in chunks: each chunk's pairs are copied back as soon as its
// probe has ended, on a stream of their own, while later chunks are still copied in and joined.
static int finish_chunked_run(brig_join_t* h, uint32_t* out_r_val, uint32_t* out_s_val, uint32_t* out_key,
                              int64_t capacity, int64_t* count, cudaStream_t st) {
    Engine& e = *h->eng;
    auto& b = e.hio;
    h->last_kind = 1;
    h->last_items = 1;
    int64_t done = 0;  // pairs whose copy is issued
    for (int c = 0; c < e.chunks_run; ++c) {
        brig::cuda_check(cudaEventSynchronize(e.chunk_done[c]), "cudaEventSynchronize");
        const int64_t upto = std::min(e.chunk_count[c], capacity);
        if (upto > done) {
            const size_t n = (size_t)(upto - done) * 4;
            brig::cuda_check(cudaMemcpyAsync(out_r_val + done, b.outr + done, n, cudaMemcpyDeviceToHost, e.d2h_stream),
                             "D2H r_val");
            brig::cuda_check(cudaMemcpyAsync(out_s_val + done, b.outs + done, n, cudaMemcpyDeviceToHost, e.d2h_stream),
                             "D2H s_val");
            if (out_key)
                brig::cuda_check(cudaMemcpyAsync(out_key + done, b.outk + done, n, cudaMemcpyDeviceToHost, e.d2h_stream),
                                 "D2H key");
            done = upto;
        }
    }
    std::vector<int64_t> c;
    int64_t errors = 0;
    e.sync_counters(c, errors);
    brig::cuda_check(cudaStreamSynchronize(e.d2h_stream), "cudaStreamSynchronize");
    brig::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (errors) fail(BRIG_E_INTERNAL, "device-side consistency check failed");
    const int64_t cnt = c[brig::kCntMatches];
    if (count) *count = cnt;
    if (cnt > capacity) return (int)set_error(BRIG_E_OVERFLOW, "match count exceeds output capacity");
    return (int)BRIG_OK;
}

int brig_join_run_host(brig_join_t* h, const uint32_t* r_key, const uint32_t* r_val, int64_t n_r,
                       const uint32_t* s_key, const uint32_t* s_val, int64_t n_s, uint32_t* out_r_val,
                       uint32_t* out_s_val, uint32_t* out_key, int64_t capacity, int64_t* count,
                       void* stream) {
    return guarded([&] {
        if (!h) fail(BRIG_E_INVALID, "null handle");
        check_rel(r_key, r_val, n_r, "R");
        check_rel(s_key, s_val, n_s, "S");
        if (capacity < 0) fail(BRIG_E_INVALID, "negative capacity");
        if (capacity > 0 && (!out_r_val || !out_s_val)) fail(BRIG_E_INVALID, "null output arrays");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        Engine& e = *h->eng;
        auto& b = e.hio;
        const int chunks = e.config().s_chunks;
        if (chunks > 1 && n_r > 0 && n_s > 0) {
            e.run_host_chunked(r_key, r_val, n_r, s_key, s_val, n_s, chunks, capacity, out_key != nullptr, st);
            return finish_chunked_run(h, out_r_val, out_s_val, out_key, capacity, count, st);
        }
        e.ensure_host_io(n_r, n_s, capacity, out_key != nullptr);
        // Large inputs: S is copied on the engine's copy stream after R, while R's passes and the
        // Bloom build run on `st`; S's passes wait for its copy. Small ones: all copies on `st`.
        const bool split = n_r > 0 && n_s > 0 && n_r + n_s >= kSplitCopyTuples;
        if (n_r > 0) {
            brig::cuda_check(cudaMemcpyAsync(b.rk, r_key, (size_t)n_r * 4, cudaMemcpyHostToDevice, st), "H2D R keys");
            brig::cuda_check(cudaMemcpyAsync(b.rv, r_val, (size_t)n_r * 4, cudaMemcpyHostToDevice, st), "H2D R vals");
        }
        cudaStream_t sst = st;
        if (split) {
            brig::cuda_check(cudaEventRecord(e.r_copied, st), "cudaEventRecord");
            brig::cuda_check(cudaStreamWaitEvent(e.copy_stream, e.r_copied, 0), "cudaStreamWaitEvent");
            sst = e.copy_stream;
        }
        if (n_s > 0) {
            brig::cuda_check(cudaMemcpyAsync(b.sk, s_key, (size_t)n_s * 4, cudaMemcpyHostToDevice, sst), "H2D S keys");
            brig::cuda_check(cudaMemcpyAsync(b.sv, s_val, (size_t)n_s * 4, cudaMemcpyHostToDevice, sst), "H2D S vals");
        }
        if (split) brig::cuda_check(cudaEventRecord(e.s_copied, sst), "cudaEventRecord");
        brig_join_output o{b.outr, b.outs, out_key ? b.outk : nullptr, capacity, nullptr};
        brig::JoinIO io{b.rk, b.rv, b.sk, b.sv, n_r, n_s, o};
        e.run({io}, st, e.config().use_cuda_graph != 0, split ? e.s_copied : nullptr);
        return finish_host_run(h, out_r_val, out_s_val, out_key, capacity, count, st);
    });
}

int brig_join_plan(const brig_join_config* cfg, int64_t n_r, int64_t n_s, int32_t* partition_size,
                   int32_t* second_partition_size, int64_t* workspace_bytes) {
    return guarded([&] {
        check_cfg(cfg);
        if (n_r < 0 || n_s < 0) fail(BRIG_E_INVALID, "negative size");
        const brig::JoinPlan p = brig::plan_join(*cfg, n_r, n_s);
        if (partition_size) *partition_size = (int32_t)p.pf.P1;
        if (second_partition_size) *second_partition_size = (int32_t)p.pf.P2;
        if (workspace_bytes) *workspace_bytes = Engine::workspace_needed(*cfg, {p}, 148);
        return (int)BRIG_OK;
    });
}

int brig_join_run_batch(brig_join_t* h, const brig_join_batch_item* items, int32_t n_items, void* stream) {
    return guarded([&] {
        if (!h || !items || n_items <= 0) fail(BRIG_E_INVALID, "bad batch arguments");
        std::vector<brig::JoinIO> io((size_t)n_items);
        for (int i = 0; i < n_items; ++i) {
            const auto& it = items[i];
            check_rel(it.r_key, it.r_val, it.n_r, "R");
            check_rel(it.s_key, it.s_val, it.n_s, "S");
            check_out(&it.out);
            io[i] = brig::JoinIO{it.r_key, it.r_val, it.s_key, it.s_val, it.n_r, it.n_s, it.out};
        }
        h->eng->run(io, static_cast<cudaStream_t>(stream), h->eng->config().use_cuda_graph != 0);
        h->last_kind = 2;
        h->last_items = n_items;
        return (int)BRIG_OK;
    });
}

int brig_join_autotune(brig_join_t* h, const brig_join_batch_item* items, int32_t n_items, void* stream,
                       brig_join_config* chosen) {
    return guarded([&] {
        if (!h || !items || n_items <= 0) fail(BRIG_E_INVALID, "bad autotune arguments");
        std::vector<brig::JoinIO> io((size_t)n_items);
        for (int i = 0; i < n_items; ++i) {
            const auto& it = items[i];
            check_rel(it.r_key, it.r_val, it.n_r, "R");
            check_rel(it.s_key, it.s_val, it.n_s, "S");
            check_out(&it.out);
            io[i] = brig::JoinIO{it.r_key, it.r_val, it.s_key, it.s_val, it.n_r, it.n_s, it.out};
        }
        const brig_join_config c = h->eng->autotune(io, static_cast<cudaStream_t>(stream));
        if (chosen) *chosen = c;
        h->last_kind = 2;
        h->last_items = n_items;
        return (int)BRIG_OK;
    });
}

int brig_join_autotune_candidates(const brig_join_config* base, brig_join_config* out, int32_t max, int32_t* n) {
    return guarded([&] {
        if (!base || !n || (max > 0 && !out)) fail(BRIG_E_INVALID, "null argument");
        const std::vector<brig_join_config> c = brig::autotune_candidates(*base);
        for (int32_t i = 0; i < max && i < (int32_t)c.size(); ++i) out[i] = c[i];
        *n = (int32_t)c.size();
        return (int)BRIG_OK;
    });
}

int brig_join_batch_counts(brig_join_t* h, int64_t* counts, int32_t n_items) {
    return guarded([&] {
        if (!h || !counts) fail(BRIG_E_INVALID, "null argument");
        if (n_items != h->last_items) fail(BRIG_E_INVALID, "n_items differs from the last batch");
        std::vector<int64_t> c;
        int64_t errors = 0;
        h->eng->sync_counters(c, errors);
        const auto& caps = h->eng->last_caps();
        bool overflow = false;
        for (int i = 0; i < n_items; ++i) {
            counts[i] = c[(size_t)i * brig::kCntWords + brig::kCntMatches];
            if (counts[i] > caps[i]) overflow = true;
        }
        if (errors) fail(BRIG_E_INTERNAL, "device-side consistency check failed");
        if (overflow) return (int)set_error(BRIG_E_OVERFLOW, "a join exceeded its output capacity");
        return (int)BRIG_OK;
    });
}

int brig_gen_device(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s,
                    uint32_t* r_key, uint32_t* r_val, uint32_t* s_key, uint32_t* s_val, void* stream) {
    return guarded([&] {
        if (n_r < 0 || n_s < 0) fail(BRIG_E_INVALID, "negative size");
        if (n_r > (int64_t)brig::kP31 || n_s > (int64_t)brig::kP31)
            fail(BRIG_E_UNSUPPORTED, "generator supports up to 2^31-1 rows");
        if (match_frac < 0 || match_frac > 1) fail(BRIG_E_INVALID, "match_frac outside [0, 1]");
        brig::cuda_check(brig::enqueue_gen(seed, n_r, n_s, match_frac, zipf_s, r_key, r_val, s_key, s_val,
                                           static_cast<cudaStream_t>(stream)),
                         "generator launch");
        return (int)BRIG_OK;
    });
}

int brig_gen_host(uint64_t seed, int64_t n_r, int64_t n_s, double match_frac, double zipf_s, uint32_t* r_key,
                  uint32_t* r_val, uint32_t* s_key, uint32_t* s_val) {
    return guarded([&] {
        if (n_r < 0 || n_s < 0) fail(BRIG_E_INVALID, "negative size");
        if (n_r > (int64_t)brig::kP31 || n_s > (int64_t)brig::kP31)
            fail(BRIG_E_UNSUPPORTED, "generator supports up to 2^31-1 rows");
        if (match_frac < 0 || match_frac > 1) fail(BRIG_E_INVALID, "match_frac outside [0, 1]");
        const brig::GenParams g = brig::make_gen_params(seed, n_r, n_s, match_frac, zipf_s);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n_r; ++i) {
            if (r_key) r_key[i] = brig::gen_r_key(g, i);
            if (r_val) r_val[i] = (uint32_t)i;
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n_s; ++i) {
            if (s_key) s_key[i] = brig::gen_s_key(g, i);
            if (s_val) s_val[i] = (uint32_t)i;
        }
        return (int)BRIG_OK;
    });
}

const char* brig_join_stage_name(int32_t i) { return brig::stage_name(i); }

int brig_join_stage_times(brig_join_t* h, double* ms, int32_t n) {
    return guarded([&] {
        if (!h || !ms || n < 0) fail(BRIG_E_INVALID, "bad arguments");
        if (h->eng->stage_times(ms, n) == 0) fail(BRIG_E_INVALID, "no profiled run since the last call");
        return (int)BRIG_OK;
    });
}

const char* brig_join_last_error(void) { return g_last_error.c_str(); }

int64_t brig_join_kernel_launches(void) { return brig::launches_so_far(); }

}  // extern "C"
