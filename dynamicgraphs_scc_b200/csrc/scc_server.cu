// Serving loop for streaming edge updates (the streaming configuration; the
// reference has no server: its dynamic methods 5-11 read one insert or delete
// file per process, src/common_main.h:500-732).
//
// Sessions are device-resident graphs with their decomposition (graph + state,
// each state on its own CUDA stream).  Clients submit edge batches; worker
// threads ("slots") run scc_update_batch.  Continuous batching: a request is
// admitted as soon as a slot is free, its session has no request running (a
// session's requests run in arrival order) and its device-memory estimate fits
// the HBM budget next to everything resident and in flight; requests of
// different sessions therefore overlap on the device.  A request that could
// never fit the budget is rejected with SCC_ERR_OOM.  Latency = completion -
// submission (host clock); p50/p99 and updates/s are kept.
//
// Backpressure (scc_server_set_admission, off by default): a submission that
// would take the backlog of queued edges above a limit is refused with
// SCC_ERR_BUSY, and a request that has waited longer than an age limit is
// dropped (status SCC_ERR_BUSY) when a slot reaches it, so under overload the
// queue and the latency of admitted requests stay bounded instead of growing
// for the whole run.  Offered, served, shed and expired counts are kept.
//
// Coalescing (scc_server_set_coalesce, off by default): when a session's turn
// comes with several of its requests queued, up to max_requests of them
// (max_edges edges in all) are composed into one batch and applied by one
// update, so one CSR merge and one recompute serve them all.  Composition keeps
// the sequential result exactly: a batch deletes every copy of its deleted
// pairs and then adds its inserts, so an insert survives the group unless a
// later batch of the group deletes that pair.  Every request of a group
// completes with the group's result (the session after the whole group).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <string.h>
#include "scc_internal.cuh"

struct ServerRequest {
    int64_t id = 0;
    int32_t session = 0;
    std::vector<int32_t> ins_src, ins_dst, del_src, del_dst;
    int64_t est_bytes = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int rc = SCC_OK;
    scc_update_stats st;
    bool done = false;
};

struct ServerSession {
    scc_graph* g = nullptr;
    scc_state* s = nullptr;
    bool busy = false;
    int64_t resident = 0;
};

struct scc_server {
    int device = 0;
    int64_t budget = 0;
    int64_t in_use = 0;          // resident sessions + admitted requests
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<ServerSession> sessions;
    std::unordered_map<int64_t, std::unique_ptr<ServerRequest>> reqs;
    std::deque<int64_t> queue;
    std::vector<std::thread> workers;
    bool stop = false;
    int64_t next_id = 1;
    std::vector<double> latencies;
    int64_t updates_done = 0, completed = 0, rejected = 0, max_inflight = 0, inflight = 0;
    int64_t groups = 0;          // updates applied (one per request, or per coalesced group)
    int32_t coalesce = 1;        // requests per group (1 = off)
    int64_t coalesce_edges = 0;  // edge cap of a group
    double t_first = -1.0, t_last = 0.0;
    int64_t max_queued = 0;      // admission: backlog limit in edges (0 = none)
    double max_age_ms = 0.0;     //            age limit of a queued request (0 = none)
    int64_t queued_edges = 0, max_queued_seen = 0;
    int64_t offered_edges = 0, shed = 0, shed_edges = 0, expired = 0;
    double t_last_submit = 0.0;
};

// ------------------------------------------------------------------ composition of queued batches
// Open-addressing map from an edge key (u << 32 | v) to the index of the last
// batch of the group that deletes it.
struct LastDelete {
    std::vector<unsigned long long> keys;
    std::vector<int32_t> vals;
    size_t mask = 0;
    explicit LastDelete(size_t n) {
        size_t cap = 16;
        while (cap < 2 * n + 16) cap <<= 1;
        keys.assign(cap, ~0ull);
        vals.assign(cap, -1);
        mask = cap - 1;
    }
    static size_t hash(unsigned long long k) {
        k ^= k >> 33; k *= 0xFF51AFD7ED558CCDull; k ^= k >> 33;
        return (size_t)k;
    }
    void put(unsigned long long k, int32_t v) {
        for (size_t i = hash(k) & mask;; i = (i + 1) & mask) {
            if (keys[i] == k || keys[i] == ~0ull) { keys[i] = k; vals[i] = v; return; }
        }
    }
    int32_t get(unsigned long long k) const {
        for (size_t i = hash(k) & mask;; i = (i + 1) & mask) {
            if (keys[i] == k) return vals[i];
            if (keys[i] == ~0ull) return -1;
        }
    }
};

static inline unsigned long long edge_key(int32_t u, int32_t v) {
    return ((unsigned long long)(uint32_t)u << 32) | (uint32_t)v;
}

// One batch equivalent to applying grp's batches in order (see the header).
static void compose_group(const std::vector<ServerRequest*>& grp, std::vector<int32_t>& is, std::vector<int32_t>& id,
                          std::vector<int32_t>& ds, std::vector<int32_t>& dd) {
    size_t nd = 0, ni = 0;
    for (auto* r : grp) { nd += r->del_src.size(); ni += r->ins_src.size(); }
    LastDelete last(nd);
    ds.reserve(nd); dd.reserve(nd);
    for (size_t j = 0; j < grp.size(); ++j) {
        const ServerRequest* r = grp[j];
        for (size_t e = 0; e < r->del_src.size(); ++e) {
            last.put(edge_key(r->del_src[e], r->del_dst[e]), (int32_t)j);
            ds.push_back(r->del_src[e]);
            dd.push_back(r->del_dst[e]);
        }
    }
    is.reserve(ni); id.reserve(ni);
    for (size_t j = 0; j < grp.size(); ++j) {
        const ServerRequest* r = grp[j];
        for (size_t e = 0; e < r->ins_src.size(); ++e) {
            if (nd && last.get(edge_key(r->ins_src[e], r->ins_dst[e])) > (int32_t)j) continue;   // deleted later
            is.push_back(r->ins_src[e]);
            id.push_back(r->ins_dst[e]);
        }
    }
}

static double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

static int64_t graph_bytes(int32_t n, int64_t m) { return 8LL * ((int64_t)n + 1) + 8LL * m; }
// state: per-vertex arrays, queues and per-colour slots (scc_state_create),
// plus the 8-byte counts within colours a later peel allocates at first use
static int64_t state_bytes(int32_t n) { return 148LL * (int64_t)n + 4096; }
// an update: new CSR + transpose, deleted flags, sorted keys, temporaries
static int64_t update_bytes(int32_t n, int64_t m, int64_t k_ins, int64_t k_del) {
    return 10LL * (m + k_ins) + 64LL * (k_ins + k_del) + 16LL * (int64_t)n + (1 << 20);
}

static void worker_main(scc_server* sv) {
    cudaSetDevice(sv->device);
    for (;;) {
        ServerRequest* r = nullptr;
        ServerSession* ses = nullptr;
        std::vector<ServerRequest*> grp;
        int64_t grp_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            for (;;) {
                if (sv->stop) return;
                bool rejected_one = false;
                std::vector<char> blocked(sv->sessions.size(), 0);
                for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
                    ServerRequest* c = sv->reqs[*it].get();
                    ServerSession& s = sv->sessions[(size_t)c->session];
                    if (blocked[(size_t)c->session] || s.busy) { blocked[(size_t)c->session] = 1; continue; }
                    if (sv->max_age_ms > 0 && now_ms() - c->t_submit > sv->max_age_ms) {
                        // waited past the age limit: dropped, the session unchanged
                        c->rc = SCC_ERR_BUSY;
                        c->done = true;
                        c->t_done = now_ms();
                        sv->expired++;
                        sv->completed++;
                        sv->queued_edges -= (int64_t)(c->ins_src.size() + c->del_src.size());
                        sv->queue.erase(it);
                        sv->cv_done.notify_all();
                        rejected_one = true;
                        break;
                    }
                    if (sv->in_use + c->est_bytes > sv->budget) {
                        if (sv->inflight == 0) {   // can never fit: reject
                            c->rc = SCC_ERR_OOM;
                            c->done = true;
                            c->t_done = now_ms();
                            sv->rejected++;
                            sv->completed++;
                            sv->queued_edges -= (int64_t)(c->ins_src.size() + c->del_src.size());
                            sv->queue.erase(it);
                            sv->cv_done.notify_all();
                            rejected_one = true;
                            break;
                        }
                        blocked[(size_t)c->session] = 1;
                        continue;
                    }
                    r = c;
                    ses = &s;
                    sv->queued_edges -= (int64_t)(c->ins_src.size() + c->del_src.size());
                    sv->queue.erase(it);
                    break;
                }
                if (r) break;
                if (rejected_one) continue;   // the queue changed: scan again
                sv->cv_work.wait(lk);
            }
            // the rest of the group: this session's next queued requests, in order
            grp.push_back(r);
            int64_t n_ins = (int64_t)r->ins_src.size(), n_del = (int64_t)r->del_src.size();
            grp_bytes = r->est_bytes;
            if (sv->coalesce > 1) {
                for (auto it = sv->queue.begin(); it != sv->queue.end() && (int32_t)grp.size() < sv->coalesce;) {
                    ServerRequest* c = sv->reqs[*it].get();
                    if (c->session != r->session) { ++it; continue; }
                    int64_t ni = n_ins + (int64_t)c->ins_src.size(), nd = n_del + (int64_t)c->del_src.size();
                    int64_t bytes = update_bytes(ses->g->n, ses->g->m, ni, nd);
                    if (ni + nd > sv->coalesce_edges || sv->in_use + bytes > sv->budget) break;
                    if (sv->max_age_ms > 0 && now_ms() - c->t_submit > sv->max_age_ms) break;
                    sv->queued_edges -= (int64_t)(c->ins_src.size() + c->del_src.size());
                    grp.push_back(c);
                    n_ins = ni; n_del = nd; grp_bytes = bytes;
                    it = sv->queue.erase(it);
                }
            }
            ses->busy = true;
            sv->in_use += grp_bytes;
            sv->inflight++;
            sv->max_inflight = std::max(sv->max_inflight, sv->inflight);
            double t0 = now_ms();
            for (auto* c : grp) c->t_start = t0;
        }
        int rc;
        scc_update_stats st;
        memset(&st, 0, sizeof(st));
        if (grp.size() == 1) {
            rc = scc_update_batch(ses->g, ses->s, (int64_t)r->ins_src.size(), r->ins_src.data(), r->ins_dst.data(),
                                  (int64_t)r->del_src.size(), r->del_src.data(), r->del_dst.data(), 0, &st);
        } else {
            std::vector<int32_t> is, id, ds, dd;
            compose_group(grp, is, id, ds, dd);
            rc = scc_update_batch(ses->g, ses->s, (int64_t)is.size(), is.data(), id.data(), (int64_t)ds.size(),
                                  ds.data(), dd.data(), 0, &st);
        }
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            double t1 = now_ms();
            ses->busy = false;
            sv->in_use -= grp_bytes;
            sv->in_use -= ses->resident;
            ses->resident = graph_bytes(ses->g->n, ses->g->m) + state_bytes(ses->g->n);
            sv->in_use += ses->resident;
            sv->inflight--;
            sv->groups++;
            for (auto* c : grp) {
                c->rc = rc;
                c->st = st;
                c->t_done = t1;
                c->done = true;
                sv->completed++;
                if (rc == SCC_OK) {
                    sv->latencies.push_back(c->t_done - c->t_submit);
                    sv->updates_done += (int64_t)(c->ins_src.size() + c->del_src.size());
                }
                c->ins_src.clear(); c->ins_src.shrink_to_fit(); c->ins_dst.clear(); c->ins_dst.shrink_to_fit();
                c->del_src.clear(); c->del_src.shrink_to_fit(); c->del_dst.clear(); c->del_dst.shrink_to_fit();
            }
            sv->t_last = std::max(sv->t_last, t1);
        }
        sv->cv_done.notify_all();
        sv->cv_work.notify_all();
    }
}

extern "C" int scc_server_set_coalesce(scc_server* sv, int32_t max_requests, int64_t max_edges) {
    SCC_REQUIRE(sv && max_requests >= 1 && max_edges >= 0, SCC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->coalesce = max_requests;
    sv->coalesce_edges = max_edges;
    return SCC_OK;
}

extern "C" int scc_server_set_admission(scc_server* sv, int64_t max_queued_edges, double max_queue_ms) {
    SCC_REQUIRE(sv && max_queued_edges >= 0 && max_queue_ms >= 0, SCC_ERR_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->max_queued = max_queued_edges;
    sv->max_age_ms = max_queue_ms;
    return SCC_OK;
}

extern "C" int scc_server_create(int device, int num_slots, int64_t hbm_budget_bytes, scc_server** out) {
    SCC_REQUIRE(out && num_slots >= 1 && num_slots <= 64 && hbm_budget_bytes > 0, SCC_ERR_INVALID, "bad argument");
    SCC_CUDA(cudaSetDevice(device));
    scc_server* sv = new scc_server();
    sv->device = device;
    sv->budget = hbm_budget_bytes;
    for (int i = 0; i < num_slots; ++i) sv->workers.emplace_back(worker_main, sv);
    *out = sv;
    return SCC_OK;
}

// Takes ownership of g; decomposes it (method 2) before the session serves.
extern "C" int scc_server_add_graph(scc_server* sv, scc_graph* g, int32_t* session) {
    SCC_REQUIRE(sv && g && session, SCC_ERR_INVALID, "NULL argument");
    int64_t need = graph_bytes(g->n, g->m) + state_bytes(g->n);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        SCC_REQUIRE(sv->in_use + need <= sv->budget, SCC_ERR_OOM, "graph needs %lld bytes, budget left %lld",
                    (long long)need, (long long)(sv->budget - sv->in_use));
        sv->in_use += need;
    }
    scc_state* s = nullptr;
    int rc = scc_state_create(g, &s);
    scc_run_stats st;
    if (rc == SCC_OK) rc = scc_run(g, s, SCC_METHOD_GLOBAL_WCC_FB, SCC_PIVOT_DEGREE, &st);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (rc != SCC_OK) {
        sv->in_use -= need;
        scc_state_free(s);
        return rc;
    }
    ServerSession ses;
    ses.g = g; ses.s = s; ses.resident = need;
    sv->sessions.push_back(ses);
    *session = (int32_t)sv->sessions.size() - 1;
    return SCC_OK;
}

extern "C" int scc_server_submit(scc_server* sv, int32_t session, int64_t n_ins, const int32_t* ins_src,
                                 const int32_t* ins_dst, int64_t n_del, const int32_t* del_src, const int32_t* del_dst,
                                 int64_t* request_id) {
    SCC_REQUIRE(sv && request_id, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(n_ins >= 0 && n_del >= 0 && (n_ins == 0 || (ins_src && ins_dst)) && (n_del == 0 || (del_src && del_dst)),
                SCC_ERR_INVALID, "bad batch");
    *request_id = -1;
    {
        // backpressure before the copy: a refused batch costs nothing
        std::lock_guard<std::mutex> lk(sv->mu);
        SCC_REQUIRE(session >= 0 && session < (int32_t)sv->sessions.size(), SCC_ERR_INVALID, "no session %d", session);
        double t = now_ms();
        if (sv->t_first < 0) sv->t_first = t;
        sv->t_last_submit = t;
        sv->offered_edges += n_ins + n_del;
        if (sv->max_queued > 0 && sv->queued_edges + n_ins + n_del > sv->max_queued) {
            sv->shed++;
            sv->shed_edges += n_ins + n_del;
            scc_set_error("serving queue holds %lld edges; limit %lld", (long long)sv->queued_edges,
                          (long long)sv->max_queued);
            return SCC_ERR_BUSY;
        }
    }
    auto r = std::make_unique<ServerRequest>();
    r->ins_src.assign(ins_src, ins_src + n_ins); r->ins_dst.assign(ins_dst, ins_dst + n_ins);
    r->del_src.assign(del_src, del_src + n_del); r->del_dst.assign(del_dst, del_dst + n_del);
    std::lock_guard<std::mutex> lk(sv->mu);
    const ServerSession& s = sv->sessions[(size_t)session];
    r->session = session;
    r->id = sv->next_id++;
    r->est_bytes = update_bytes(s.g->n, s.g->m, n_ins, n_del);
    r->t_submit = now_ms();
    sv->queued_edges += n_ins + n_del;
    sv->max_queued_seen = std::max(sv->max_queued_seen, sv->queued_edges);
    *request_id = r->id;
    sv->queue.push_back(r->id);
    sv->reqs[r->id] = std::move(r);
    sv->cv_work.notify_one();
    return SCC_OK;
}

extern "C" int scc_server_wait(scc_server* sv, int64_t request_id, scc_request_result* out) {
    SCC_REQUIRE(sv, SCC_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(request_id);
    SCC_REQUIRE(it != sv->reqs.end(), SCC_ERR_INVALID, "no request %lld", (long long)request_id);
    ServerRequest* r = it->second.get();
    sv->cv_done.wait(lk, [&] { return r->done; });
    if (out) {
        out->status = r->rc;
        out->session = r->session;
        out->latency_ms = r->t_done - r->t_submit;
        out->queue_ms = (r->t_start > 0 ? r->t_start : r->t_done) - r->t_submit;
        out->update = r->st;
    }
    return SCC_OK;
}

extern "C" int scc_server_drain(scc_server* sv) {
    SCC_REQUIRE(sv, SCC_ERR_INVALID, "NULL argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->cv_done.wait(lk, [&] { return sv->queue.empty() && sv->inflight == 0; });
    return SCC_OK;
}

extern "C" int scc_server_get_stats(scc_server* sv, scc_server_stats* out) {
    SCC_REQUIRE(sv && out, SCC_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    memset(out, 0, sizeof(*out));
    std::vector<double> l = sv->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l.empty() ? 0.0 : l[(size_t)std::min<double>(l.size() - 1, p * (l.size() - 1) + 0.5)]; };
    out->completed = sv->completed;
    out->rejected = sv->rejected;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = l.empty() ? 0.0 : l.back();
    out->updates = sv->updates_done;
    double span = sv->t_last - sv->t_first;
    out->updates_per_s = span > 0 ? sv->updates_done / (span * 1e-3) : 0.0;
    out->max_inflight = sv->max_inflight;
    out->bytes_in_use = sv->in_use;
    out->groups = sv->groups;
    out->offered_edges = sv->offered_edges;
    out->shed = sv->shed;
    out->shed_edges = sv->shed_edges;
    out->expired = sv->expired;
    out->max_queued_edges = sv->max_queued_seen;
    double offer_span = sv->t_last_submit - sv->t_first;
    out->offered_per_s = offer_span > 0 ? sv->offered_edges / (offer_span * 1e-3) : 0.0;
    return SCC_OK;
}

extern "C" int scc_server_labels(scc_server* sv, int32_t session, int32_t* labels) {
    SCC_REQUIRE(sv && labels, SCC_ERR_INVALID, "NULL argument");
    ServerSession* s = nullptr;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        SCC_REQUIRE(session >= 0 && session < (int32_t)sv->sessions.size(), SCC_ERR_INVALID, "no session %d", session);
        s = &sv->sessions[(size_t)session];
        SCC_REQUIRE(!s->busy, SCC_ERR_STATE, "session %d is busy", session);
    }
    return scc_canonical_labels(s->s, labels);
}

extern "C" int scc_server_session_graph(scc_server* sv, int32_t session, scc_graph** g) {
    SCC_REQUIRE(sv && g, SCC_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    SCC_REQUIRE(session >= 0 && session < (int32_t)sv->sessions.size(), SCC_ERR_INVALID, "no session %d", session);
    *g = sv->sessions[(size_t)session].g;
    return SCC_OK;
}

extern "C" int scc_server_free(scc_server* sv) {
    if (!sv) return SCC_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    for (auto& t : sv->workers) t.join();
    for (auto& s : sv->sessions) { scc_state_free(s.s); scc_graph_free(s.g); }
    delete sv;
    return SCC_OK;
}
