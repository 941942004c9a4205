// serve.cu - served joins: continuous batching under an HBM budget (no reference counterpart).
//
// A scheduler thread owns `streams` slots, each a CUDA stream with its own Engine (workspace).
// Loop:
//   1. completions: a slot whose wave finished its join reads the per-join counts and enqueues the
//      device-to-host copies of the pairs; when those land, each request is marked done and its
//      device memory returns to the budget;
//   2. admission: while a slot is idle and the oldest pending request's footprint fits the budget,
//      requests (up to max_wave) are admitted into one wave and launched on that slot: host inputs
//      are copied in, the wave runs as one batched pipeline, results follow in step 1.
// A request that arrives while other waves are on the GPU is admitted as soon as a slot and memory
// are free, so its work overlaps the waves already running; large requests (above large_mtuples
// tuples) run one at a time on slot 0 and small ones may pass them. Submit and poll are
// thread-safe.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>
#include "../../include/brig_join.h"
#include "engine.h"

namespace brig {
namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    int64_t ticket = 0;
    brig_serve_request in{};
    int64_t cap = 0;
    int64_t footprint = 0;
    Clock::time_point t_submit, t_start, t_enqueued, t_joined;
    // device buffers owned by the request (host-input copies and outputs)
    uint32_t *rk = nullptr, *rv = nullptr, *sk = nullptr, *sv = nullptr, *outr = nullptr, *outs = nullptr;
    int state = 0;  // 0 pending, 1 running, 2 done
    brig_serve_result res{};
};

struct Slot {
    cudaStream_t stream = nullptr;
    Engine* eng = nullptr;
    int64_t ws_target = 0;  // workspace the admitted wave runs in (accounted in the budget)
    std::vector<Req*> wave;
    int phase = 0;  // 0 idle, 1 joining, 2 copying results
    cudaEvent_t ev = nullptr;
    int wave_id = 0;
};

}  // namespace

struct Server {
    brig_join_config jcfg{};
    brig_serve_config scfg{};
    int num_sms = 148;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Req*> pending;
    std::map<int64_t, Req*> tickets;
    int64_t next_ticket = 1;
    int64_t used = 0;  // bytes of budget in use (request buffers + slot workspaces)
    bool stop = false;
    std::vector<Slot> slots;
    std::thread th;
    int next_wave = 0;
    int device = 0;
    std::string fatal;

    // Device bytes a request needs for itself: host-input copies and outputs.
    static int64_t io_bytes(const brig_serve_request& r, int64_t cap) {
        return 8 * cap + (r.inputs_on_device ? 0 : 8 * (r.n_r + r.n_s));
    }
    // io_bytes plus the workspace of the request joined alone (the admission bound).
    int64_t footprint(const brig_serve_request& r, int64_t cap) const {
        return Engine::workspace_needed(jcfg, plan_batch(jcfg, &r.n_r, &r.n_s, 1, true), num_sms) + io_bytes(r, cap);
    }
    int64_t wave_workspace(const std::vector<Req*>& w) const {
        std::vector<int64_t> nr, ns;
        for (Req* q : w) {
            nr.push_back(q->in.n_r);
            ns.push_back(q->in.n_s);
        }
        return Engine::workspace_needed(jcfg, plan_batch(jcfg, nr.data(), ns.data(), (int)w.size(), true), num_sms);
    }

    // Request buffers are stream-ordered allocations on the slot's stream, so allocating and
    // freeing them never waits for the waves running on other slots.
    void free_req_buffers(Req* q, cudaStream_t st) {
        for (uint32_t* p : {q->rk, q->rv, q->sk, q->sv, q->outr, q->outs})
            if (p) cudaFreeAsync(p, st);
        q->rk = q->rv = q->sk = q->sv = q->outr = q->outs = nullptr;
    }

    // Launches a wave on slot s (scheduler thread, without the lock).
    void launch(Slot& s) {
        std::vector<JoinIO> io;
        io.reserve(s.wave.size());
        for (Req* q : s.wave) {
            auto alloc = [&](uint32_t*& p, int64_t n) {
                cuda_check(cudaMallocAsync((void**)&p, (size_t)std::max<int64_t>(n, 1) * 4, s.stream),
                           "serve cudaMallocAsync");
            };
            const auto& r = q->in;
            const uint32_t *rk = r.r_key, *rv = r.r_val, *sk = r.s_key, *sv = r.s_val;
            if (!r.inputs_on_device) {
                alloc(q->rk, r.n_r);
                alloc(q->rv, r.n_r);
                alloc(q->sk, r.n_s);
                alloc(q->sv, r.n_s);
                if (r.n_r) {
                    cuda_check(cudaMemcpyAsync(q->rk, r.r_key, r.n_r * 4, cudaMemcpyHostToDevice, s.stream), "H2D");
                    cuda_check(cudaMemcpyAsync(q->rv, r.r_val, r.n_r * 4, cudaMemcpyHostToDevice, s.stream), "H2D");
                }
                if (r.n_s) {
                    cuda_check(cudaMemcpyAsync(q->sk, r.s_key, r.n_s * 4, cudaMemcpyHostToDevice, s.stream), "H2D");
                    cuda_check(cudaMemcpyAsync(q->sv, r.s_val, r.n_s * 4, cudaMemcpyHostToDevice, s.stream), "H2D");
                }
                rk = q->rk; rv = q->rv; sk = q->sk; sv = q->sv;
            }
            alloc(q->outr, q->cap);
            alloc(q->outs, q->cap);
            brig_join_output o{q->outr, q->outs, nullptr, q->cap, nullptr};
            io.push_back(JoinIO{rk, rv, sk, sv, r.n_r, r.n_s, o});
        }
        s.eng->reserve_workspace((size_t)s.ws_target, s.stream);
        s.eng->run(io, s.stream, false);
        cuda_check(cudaEventRecord(s.ev, s.stream), "cudaEventRecord");
        const auto now = Clock::now();
        for (Req* q : s.wave) q->t_enqueued = now;
        s.phase = 1;
    }

    // Slot s finished its join: copy pairs back (phase 1 -> 2) or finish requests (phase 2 -> 0).
    void advance(Slot& s) {
        if (s.phase == 1) {
            const auto joined = Clock::now();
            for (Req* q : s.wave) q->t_joined = joined;
            std::vector<int64_t> c;
            int64_t errors = 0;
            s.eng->sync_counters(c, errors);
            for (size_t i = 0; i < s.wave.size(); ++i) {
                Req* q = s.wave[i];
                const int64_t cnt = c[i * kCntWords + kCntMatches];
                q->res.count = cnt;
                q->res.status = errors ? BRIG_E_INTERNAL : (cnt > q->cap ? BRIG_E_OVERFLOW : BRIG_OK);
                const int64_t n = std::min(cnt, q->cap);
                if (n > 0 && q->in.out_r_val && q->in.out_s_val) {
                    cuda_check(cudaMemcpyAsync(q->in.out_r_val, q->outr, n * 4, cudaMemcpyDeviceToHost, s.stream), "D2H");
                    cuda_check(cudaMemcpyAsync(q->in.out_s_val, q->outs, n * 4, cudaMemcpyDeviceToHost, s.stream), "D2H");
                }
            }
            cuda_check(cudaEventRecord(s.ev, s.stream), "cudaEventRecord");
            s.phase = 2;
            return;
        }
        const auto now = Clock::now();
        for (Req* q : s.wave) free_req_buffers(q, s.stream);
        std::lock_guard<std::mutex> lk(mu);
        for (Req* q : s.wave) {
            used -= io_bytes(q->in, q->cap);
            q->res.submit_to_done_ms = std::chrono::duration<double, std::milli>(now - q->t_submit).count();
            q->res.queue_ms = std::chrono::duration<double, std::milli>(q->t_start - q->t_submit).count();
            q->res.setup_ms = std::chrono::duration<double, std::milli>(q->t_enqueued - q->t_start).count();
            q->res.join_ms = std::chrono::duration<double, std::milli>(q->t_joined - q->t_enqueued).count();
            q->state = 2;
        }
        s.wave.clear();
        s.phase = 0;
        cv_done.notify_all();
    }

    void loop() {
        cudaSetDevice(device);
        for (;;) {
            bool busy = false;
            for (auto& s : slots) {
                if (s.phase == 0) continue;
                busy = true;
                const cudaError_t q = cudaEventQuery(s.ev);
                if (q == cudaSuccess) {
                    try {
                        advance(s);
                    } catch (const Error& e) {
                        fail_wave(s, e.status, e.msg);
                    }
                } else if (q != cudaErrorNotReady) {
                    fail_wave(s, BRIG_E_CUDA, cudaGetErrorString(q));
                }
            }
            // admission. A request above large_mtuples tuples is large: large requests run one at a
            // time, each as a wave of its own, on slot 0, so two of them never share the GPU (which
            // would slow both and set the tail latency); the other slots batch and overlap the
            // small requests, which may pass a large one waiting for slot 0 instead of queueing
            // behind it. Slot 0 also takes small waves while no large request waits. So slot 0's
            // workspace grows to the largest request once (the warm-up), the others stay small,
            // and no slot has to map fresh device memory for a request later.
            for (size_t si = 0; si < slots.size(); ++si) {
                Slot& s = slots[(si + 1) % slots.size()];  // small-request slots first, then slot 0
                const bool large_slot = &s == &slots[0];
                if (s.phase != 0) continue;
                std::vector<Req*> wave;
                bool more = false;  // requests still pending after this slot's turn
                {
                    // Grow the wave while the budget holds: bytes in use (live request buffers and
                    // every slot's workspace) + this wave's request buffers + the growth of this
                    // slot's workspace. A wave of small requests also stops at max_wave_mtuples
                    // million tuples.
                    std::lock_guard<std::mutex> lk(mu);
                    const int64_t ws_have = s.eng->workspace_bytes();
                    const int64_t max_tuples = (int64_t)scfg.max_wave_mtuples * 1000000;
                    const int64_t large_tuples = (int64_t)scfg.large_mtuples * 1000000;
                    auto is_large = [&](const Req* q) { return q->in.n_r + q->in.n_s > large_tuples; };
                    int64_t io = 0, ws_new = ws_have, tuples = 0;
                    auto fits = [&](const std::vector<Req*>& w, int64_t io2, int64_t& ws2) {
                        ws2 = std::max(ws_have, wave_workspace(w));
                        return used + io2 + (ws2 - ws_have) <= scfg.hbm_budget_bytes;
                    };
                    // slot 0: the oldest large request, alone
                    if (large_slot) {
                        for (auto it = pending.begin(); it != pending.end(); ++it) {
                            if (!is_large(*it)) continue;
                            wave.push_back(*it);
                            int64_t ws2 = 0;
                            const int64_t io2 = io_bytes((*it)->in, (*it)->cap);
                            if (fits(wave, io2, ws2)) {
                                io = io2;
                                ws_new = ws2;
                                tuples = (*it)->in.n_r + (*it)->in.n_s;
                                pending.erase(it);
                            } else {
                                wave.clear();
                            }
                            break;
                        }
                    }
                    // otherwise small requests in arrival order, passing any large one
                    const bool large_waiting =
                        std::any_of(pending.begin(), pending.end(), [&](const Req* q) { return is_large(q); });
                    if (wave.empty() && !(large_slot && large_waiting)) {
                        for (auto it = pending.begin(); it != pending.end() && (int)wave.size() < scfg.max_wave;) {
                            Req* q = *it;
                            if (is_large(q)) {
                                ++it;
                                continue;
                            }
                            const int64_t t2 = tuples + q->in.n_r + q->in.n_s;
                            if (!wave.empty() && t2 > max_tuples) break;
                            wave.push_back(q);
                            int64_t ws2 = 0;
                            const int64_t io2 = io + io_bytes(q->in, q->cap);
                            if (!fits(wave, io2, ws2)) {
                                wave.pop_back();
                                break;
                            }
                            io = io2;
                            ws_new = ws2;
                            tuples = t2;
                            it = pending.erase(it);
                        }
                    }
                    for (Req* q : wave) {
                        q->state = 1;
                        q->t_start = Clock::now();
                        q->res.wave = next_wave;
                    }
                    // A small-request slot that must grow grows to at least the largest workspace of
                    // the small-request slots (when the budget allows), so after a warm-up none
                    // grows again: growing maps fresh device memory and blocks the scheduler.
                    if (!wave.empty() && ws_new > ws_have && !large_slot) {
                        int64_t widest = 0;
                        for (size_t o = 1; o < slots.size(); ++o) widest = std::max(widest, slots[o].ws_target);
                        const int64_t room = scfg.hbm_budget_bytes - (used + io + (ws_new - ws_have));
                        if (widest > ws_new) ws_new += std::min(widest - ws_new, std::max<int64_t>(room, 0));
                    }
                    if (!wave.empty()) {
                        used += io + (ws_new - ws_have);
                        s.ws_target = ws_new;
                        // the idle small-request slots grow with it (budget permitting), so that after
                        // a warm-up no small-request slot grows for a request later
                        if (!large_slot && ws_new > ws_have)
                            for (size_t o = 1; o < slots.size(); ++o) {
                                Slot& t = slots[o];
                                if (&t == &s || t.phase != 0 || t.ws_target >= ws_new) continue;
                                if (used + (ws_new - t.ws_target) > scfg.hbm_budget_bytes) continue;
                                used += ws_new - t.ws_target;
                                t.ws_target = ws_new;
                                t.eng->reserve_workspace((size_t)ws_new, t.stream);
                            }
                    }
                    more = !pending.empty();
                }
                if (wave.empty()) {
                    if (!more) break;
                    continue;  // what is pending waits for another slot (or for memory); try the next
                }
                s.wave = wave;
                s.wave_id = next_wave++;
                try {
                    launch(s);
                } catch (const Error& e) {
                    fail_wave(s, e.status, e.msg);
                }
                busy = true;
            }
            std::unique_lock<std::mutex> lk(mu);
            if (stop && pending.empty()) {
                bool idle = true;
                for (auto& s : slots) idle = idle && s.phase == 0;
                if (idle) return;
            }
            if (busy)
                cv_sched.wait_for(lk, std::chrono::microseconds(50));
            else
                cv_sched.wait_for(lk, std::chrono::milliseconds(5), [&] { return stop || !pending.empty(); });
        }
    }

    void fail_wave(Slot& s, int status, const std::string& msg) {
        cudaStreamSynchronize(s.stream);
        for (Req* q : s.wave) free_req_buffers(q, s.stream);
        cudaStreamSynchronize(s.stream);
        std::lock_guard<std::mutex> lk(mu);
        for (Req* q : s.wave) {
            used -= io_bytes(q->in, q->cap);
            q->res.status = status;
            q->state = 2;
        }
        fatal = msg;
        s.wave.clear();
        s.phase = 0;
        cv_done.notify_all();
    }
};

}  // namespace brig

struct brig_serve_t {
    brig::Server* srv = nullptr;
};

namespace {
template <class F>
int serve_guard(F&& f) {
    try {
        brig::set_last_error("");
        return f();
    } catch (const brig::Error& e) {
        brig::set_last_error(e.msg);
        return e.status;
    } catch (...) {
        brig::set_last_error("unknown failure");
        return (int)BRIG_E_INTERNAL;
    }
}
}  // namespace

extern "C" {

int brig_serve_create(const brig_join_config* jcfg, const brig_serve_config* scfg, brig_serve_t** out) {
    return serve_guard([&] {
        if (!jcfg || !out) brig::fail(BRIG_E_INVALID, "null argument");
        if (jcfg->abi_version != BRIG_JOIN_ABI_VERSION) brig::fail(BRIG_E_INVALID, "config ABI version mismatch");
        *out = nullptr;
        auto* s = new brig::Server;
        s->jcfg = *jcfg;
        s->jcfg.use_cuda_graph = 0;
        s->jcfg.profile_stages = 0;
        if (scfg) s->scfg = *scfg;
        if (s->scfg.hbm_budget_bytes <= 0) s->scfg.hbm_budget_bytes = 120ll * 1000 * 1000 * 1000;
        if (s->scfg.max_wave <= 0) s->scfg.max_wave = 64;
        if (s->scfg.streams <= 0) s->scfg.streams = 2;
        if (s->scfg.max_queue <= 0) s->scfg.max_queue = 4096;
        if (s->scfg.max_wave_mtuples <= 0) s->scfg.max_wave_mtuples = 256;
        if (s->scfg.large_mtuples <= 0) s->scfg.large_mtuples = s->scfg.max_wave_mtuples;
        try {
            if (jcfg->device >= 0) brig::cuda_check(cudaSetDevice(jcfg->device), "cudaSetDevice");
            brig::cuda_check(cudaGetDevice(&s->device), "cudaGetDevice");
            cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
            // Keep freed request buffers in the stream-ordered pool up to the budget instead of
            // returning them to the driver at every synchronisation.
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
                uint64_t thr = (uint64_t)s->scfg.hbm_budget_bytes;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
            }
            s->slots.resize(s->scfg.streams);
            for (auto& sl : s->slots) {
                brig::cuda_check(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate");
                brig::cuda_check(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming), "cudaEventCreate");
                sl.eng = new brig::Engine(s->jcfg);
                sl.eng->set_shared_l2(true);  // the slots' waves run side by side
            }
        } catch (...) {
            for (auto& sl : s->slots) {
                delete sl.eng;
                if (sl.stream) cudaStreamDestroy(sl.stream);
                if (sl.ev) cudaEventDestroy(sl.ev);
            }
            delete s;
            throw;
        }
        s->th = std::thread([s] { s->loop(); });
        auto* h = new brig_serve_t;
        h->srv = s;
        *out = h;
        return (int)BRIG_OK;
    });
}

int brig_serve_submit(brig_serve_t* h, const brig_serve_request* req, int64_t* ticket) {
    return serve_guard([&] {
        if (!h || !req || !ticket) brig::fail(BRIG_E_INVALID, "null argument");
        brig::Server* s = h->srv;
        if (req->n_r < 0 || req->n_s < 0 || req->capacity < 0) brig::fail(BRIG_E_INVALID, "negative size");
        if ((req->n_r > 0 && (!req->r_key || !req->r_val)) || (req->n_s > 0 && (!req->s_key || !req->s_val)))
            brig::fail(BRIG_E_INVALID, "null input array");
        auto* q = new brig::Req;
        q->in = *req;
        q->cap = req->capacity > 0 ? req->capacity : std::max<int64_t>(req->n_s, 1);
        try {
            q->footprint = s->footprint(*req, q->cap);
        } catch (...) {
            delete q;
            throw;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete q;
            brig::fail(BRIG_E_REJECTED, "server is stopping");
        }
        if (q->footprint > s->scfg.hbm_budget_bytes) {
            delete q;
            brig::fail(BRIG_E_REJECTED, "request footprint exceeds the HBM budget");
        }
        if ((int)s->pending.size() >= s->scfg.max_queue) {
            delete q;
            brig::fail(BRIG_E_REJECTED, "queue full");
        }
        q->ticket = s->next_ticket++;
        q->t_submit = brig::Clock::now();
        s->pending.push_back(q);
        s->tickets[q->ticket] = q;
        *ticket = q->ticket;
        s->cv_sched.notify_one();
        return (int)BRIG_OK;
    });
}

int brig_serve_poll(brig_serve_t* h, int64_t ticket, int32_t timeout_ms, brig_serve_result* res) {
    return serve_guard([&] {
        if (!h || !res) brig::fail(BRIG_E_INVALID, "null argument");
        brig::Server* s = h->srv;
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) brig::fail(BRIG_E_INVALID, "unknown ticket");
        brig::Req* q = it->second;
        auto done = [&] { return q->state == 2; };
        if (timeout_ms < 0)
            s->cv_done.wait(lk, done);
        else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
            return (int)BRIG_E_NOT_READY;
        *res = q->res;
        s->tickets.erase(it);
        delete q;
        return (int)BRIG_OK;
    });
}

int brig_serve_destroy(brig_serve_t* h) {
    return serve_guard([&] {
        if (!h) return (int)BRIG_OK;
        brig::Server* s = h->srv;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            for (brig::Req* q : s->pending) {
                q->res.status = BRIG_E_REJECTED;
                q->state = 2;
            }
            s->pending.clear();
            s->cv_sched.notify_all();
            s->cv_done.notify_all();
        }
        if (s->th.joinable()) s->th.join();
        for (auto& sl : s->slots) {
            delete sl.eng;
            cudaStreamDestroy(sl.stream);
            cudaEventDestroy(sl.ev);
        }
        for (auto& kv : s->tickets) delete kv.second;
        delete s;
        delete h;
        return (int)BRIG_OK;
    });
}

}  // extern "C"
