// The serving loop: queries over HBM-resident tables as they arrive.
//
// The reference runs one query at a time through its operators
// (compute/src/operator.rs); here a request loop keeps tables, vector
// indexes and join hash tables resident, admits work against a device-memory
// budget, and batches continuously: while work is on the GPU, new top-k
// requests queue, and the next free worker stacks every queued request that
// differs from the oldest one only in its query vector, k and its per-query
// literal into one tensor-core scan; queued join-aggregates of one shape
// (same table, group key, aggregates and comparisons) run as one launch of
// the fused kernel, each into its own table.  Workers own one CUDA stream each, so
// admitted work items overlap on the device.  Latencies (submit to result)
// give p50/p99 beside throughput.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "internal.h"

namespace oxb {

namespace {

using Clock = std::chrono::steady_clock;

enum : int { kReqTopk = 1, kReqJoinAggregate = 2 };

struct Request {
    uint64_t id = 0;
    int kind = 0;
    // top-k
    const oxb_vector_index* index = nullptr;
    const oxb_batch* input = nullptr;
    std::vector<oxb_leaf> leaves;  // shared WHERE (without the per-query leaf)
    bool has_qleaf = false;
    oxb_leaf qleaf{};
    std::vector<float> query;
    int k = 0, metric = 0;
    // join-aggregate
    oxb_join_aggregate_args ja{};
    std::vector<oxb_leaf> ja_leaves;
    // bookkeeping
    size_t est_bytes = 0;
    Clock::time_point t_submit, t_done;
    bool done = false;
    oxb_status status = OXB_OK;
    std::string error;
    std::vector<int64_t> ids;
    std::vector<float> dist;
    oxb_batch* batch = nullptr;
};

bool same_leaf(const oxb_leaf& a, const oxb_leaf& b) {
    return a.column == b.column && a.op == b.op && a.lit_type == b.lit_type && a.lit.i == b.lit.i;
}

// Requests one top-k scan can answer together: same index, batch, metric,
// shared WHERE and per-query leaf shape.
bool batchable(const Request& a, const Request& b) {
    if (a.kind != kReqTopk || b.kind != kReqTopk) return false;
    if (a.index != b.index || a.input != b.input || a.metric != b.metric || a.has_qleaf != b.has_qleaf) return false;
    if (a.has_qleaf && (a.qleaf.column != b.qleaf.column || a.qleaf.op != b.qleaf.op ||
                        a.qleaf.lit_type != b.qleaf.lit_type))
        return false;
    if (a.leaves.size() != b.leaves.size()) return false;
    for (size_t i = 0; i < a.leaves.size(); i++)
        if (!same_leaf(a.leaves[i], b.leaves[i])) return false;
    return true;
}

}  // namespace

struct Server {
    oxb_backend* backend;
    size_t budget;
    int max_batch;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    size_t in_use = 0, peak = 0;
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    // statistics since the last reset
    std::vector<double> latency_us;
    int64_t completed = 0, rejected = 0, dispatches = 0, batched = 0;
    Clock::time_point first_submit, last_done;
    bool any = false;

    // Device memory a top-k scan of nq queries may hold: candidate lists,
    // the merged pools, query copies and the exact path's per-row buffers.
    size_t estimate_topk(const Request& r, int nq, int k) const {
        return ((size_t)64 << 20) + (size_t)nq * ((size_t)r.index->dp * 6 + (size_t)k * 12) +
               (size_t)r.index->n * 12;
    }
    // A join-aggregate's table (at most two slots per group-side row, each
    // key plus up to two arrays per aggregate), its probe table and output.
    size_t estimate_join_aggregate(const oxb_join_aggregate_args& a) const {
        const long long g = a.group_side ? a.build->rows : a.probe->rows;
        const size_t slots = (size_t)next_pow2_host(2 * std::max<long long>(g, 1));
        return ((size_t)16 << 20) + slots * 8 * (2 + 2 * (size_t)a.naggregates) +
               (size_t)a.table->t.capacity * 20;
    }
    static long long next_pow2_host(long long v) {
        long long c = 4096;
        while (c < v) c <<= 1;
        return c;
    }

    void run_worker() {
        cudaSetDevice(backend->b.device);
        auto st = std::make_shared<StreamState>();
        st->device = backend->b.device;
        st->owned = true;
        if (cudaStreamCreateWithFlags(&st->stream, cudaStreamNonBlocking) != cudaSuccess) return;
        StreamRef s = st;
        for (;;) {
            std::vector<Request*> work;
            size_t est = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stop && pending.empty()) return;
                    if (!pending.empty()) {
                        Request* r = pending.front();
                        std::vector<Request*> pick{r};
                        if (r->kind == kReqTopk) {
                            for (Request* o : pending)
                                if (o != r && (int)pick.size() < max_batch && batchable(*r, *o)) pick.push_back(o);
                            int kmax = 0;
                            for (Request* o : pick) kmax = std::max(kmax, o->k);
                            est = estimate_topk(*r, (int)pick.size(), kmax);
                        } else {
                            // Join-aggregates of one shape share a launch, each
                            // with its own table: their estimates add.
                            est = r->est_bytes;
                            for (Request* o : pending)
                                if (o != r && (int)pick.size() < max_batch && o->kind == kReqJoinAggregate &&
                                    same_join_shape(r->ja, o->ja) && in_use + est + o->est_bytes <= budget) {
                                    pick.push_back(o);
                                    est += o->est_bytes;
                                }
                        }
                        // Admission: wait for memory to free up unless nothing
                        // else holds any (a request alone never exceeds the
                        // budget: submit refuses those).
                        if (in_use + est <= budget || running == 0) {
                            for (Request* o : pick)
                                pending.erase(std::find(pending.begin(), pending.end(), o));
                            work = std::move(pick);
                            in_use += est;
                            peak = std::max(peak, in_use);
                            running++;
                            dispatches++;
                            if (work.size() > 1) batched += (int64_t)work.size();
                            break;
                        }
                    }
                    cv.wait(lk);
                }
            }
            execute(s, work);
            {
                std::lock_guard<std::mutex> lk(mu);
                in_use -= est;
                running--;
                const Clock::time_point now = Clock::now();
                for (Request* r : work) {
                    r->t_done = now;
                    r->done = true;
                    latency_us.push_back(std::chrono::duration<double, std::micro>(now - r->t_submit).count());
                    completed++;
                }
                last_done = now;
            }
            cv.notify_all();
        }
    }

    void execute(const StreamRef& s, std::vector<Request*>& work) {
        const Backend& b = backend->b;
        try {
            if (work[0]->kind == kReqTopk) {
                const Request& r0 = *work[0];
                const int nq = (int)work.size();
                const int dim = r0.index->dim;
                int kmax = 0;
                for (Request* r : work) kmax = std::max(kmax, r->k);
                std::vector<float> q((size_t)nq * dim);
                std::vector<int64_t> lits(nq);
                for (int i = 0; i < nq; i++) {
                    std::copy(work[i]->query.begin(), work[i]->query.end(), q.begin() + (size_t)i * dim);
                    lits[i] = work[i]->qleaf.lit.i;
                }
                oxb_vector_topk_args a{};
                a.index = r0.index;
                a.input = r0.input;
                a.leaves = r0.leaves.empty() ? nullptr : r0.leaves.data();
                a.nleaves = (int)r0.leaves.size();
                a.nqueries = nq;
                a.queries = q.data();
                a.dim = dim;
                a.k = kmax;
                a.metric = r0.metric;
                a.qleaf_column = r0.has_qleaf ? r0.qleaf.column : -1;
                a.qleaf_op = r0.qleaf.op;
                a.qleaf_type = r0.qleaf.lit_type;
                a.qleaf_lits = lits.data();
                std::vector<int64_t> ids((size_t)nq * kmax);
                std::vector<float> dist((size_t)nq * kmax);
                vector_topk(s, b, a, ids.data(), dist.data(), nullptr);
                // Each request's own k: the prefix of the same total order.
                for (int i = 0; i < nq; i++) {
                    Request& r = *work[i];
                    r.ids.assign(ids.begin() + (size_t)i * kmax, ids.begin() + (size_t)i * kmax + r.k);
                    r.dist.assign(dist.begin() + (size_t)i * kmax, dist.begin() + (size_t)i * kmax + r.k);
                }
            } else if (work.size() == 1) {
                Request& r = *work[0];
                r.batch = join_aggregate(s, b, r.ja);
            } else {
                std::vector<oxb_join_aggregate_args> args;
                for (Request* r : work) args.push_back(r->ja);
                std::vector<oxb_batch*> res = join_aggregate_many(s, b, args.data(), (int)args.size());
                for (size_t i = 0; i < work.size(); i++) work[i]->batch = res[i];
            }
        } catch (const Error& e) {
            for (Request* r : work) {
                r->status = e.status;
                r->error = e.message;
            }
        } catch (const std::exception& e) {
            for (Request* r : work) {
                r->status = OXB_EXECUTION;
                r->error = e.what();
            }
        }
    }

    uint64_t submit(std::unique_ptr<Request> r) {
        std::lock_guard<std::mutex> lk(mu);
        if (r->est_bytes > budget) {
            rejected++;
            fail(OXB_OOM_ADMISSION, "the request's estimated " + std::to_string(r->est_bytes >> 20) +
                                        " MiB of device memory exceed the serving budget of " +
                                        std::to_string(budget >> 20) + " MiB");
        }
        r->id = next_id++;
        r->t_submit = Clock::now();
        if (!any) {
            first_submit = r->t_submit;
            any = true;
        }
        const uint64_t id = r->id;
        pending.push_back(r.get());
        requests[id] = std::move(r);
        cv.notify_all();
        return id;
    }

    std::unique_ptr<Request> wait(uint64_t id) {
        std::unique_lock<std::mutex> lk(mu);
        auto it = requests.find(id);
        if (it == requests.end()) fail(OXB_PLAN, "unknown ticket " + std::to_string(id));
        Request* r = it->second.get();
        cv.wait(lk, [&] { return r->done; });
        std::unique_ptr<Request> out = std::move(it->second);
        requests.erase(it);
        return out;
    }
};

}  // namespace oxb

struct oxb_server {
    std::unique_ptr<oxb::Server> s;
};

namespace oxb {

oxb_server* server_create(oxb_backend* backend, const oxb_server_config& cfg) {
    auto out = std::make_unique<oxb_server>();
    out->s = std::make_unique<Server>();
    Server& S = *out->s;
    S.backend = backend;
    S.budget = cfg.memory_budget ? cfg.memory_budget : (size_t)150 << 30;
    S.max_batch = cfg.max_batch > 0 ? cfg.max_batch : 256;
    const int nw = cfg.workers > 0 ? cfg.workers : 2;
    for (int i = 0; i < nw; i++) S.workers.emplace_back([&S] { S.run_worker(); });
    return out.release();
}

void server_destroy(oxb_server* srv) {
    if (!srv) return;
    Server& S = *srv->s;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        S.stop = true;
    }
    S.cv.notify_all();
    for (auto& t : S.workers) t.join();
    for (auto& kv : S.requests) delete kv.second->batch;
    delete srv;
}

uint64_t server_submit_topk(oxb_server* srv, const oxb_topk_request& q) {
    if (!q.index || !q.input) fail(OXB_PLAN, "top-k request without an index or batch");
    if (q.dim != q.index->dim) fail(OXB_PLAN, "query dimension differs from the index's");
    if (q.k < 1 || q.k > 4096) fail(OXB_UNSUPPORTED, "k must be between 1 and 4096");
    if (q.metric != OXB_METRIC_L2 && q.metric != OXB_METRIC_COSINE) fail(OXB_PLAN, "unknown metric");
    if (q.nleaves < 0 || (q.nleaves > 0 && !q.leaves) || !q.query) fail(OXB_PLAN, "null leaves or query");
    auto r = std::make_unique<Request>();
    r->kind = kReqTopk;
    r->index = q.index;
    r->input = q.input;
    r->metric = q.metric;
    r->k = q.k;
    r->query.assign(q.query, q.query + q.dim);
    int shared = q.nleaves;
    if (q.qleaf && q.nleaves > 0) {
        r->has_qleaf = true;
        r->qleaf = q.leaves[q.nleaves - 1];
        shared--;
    }
    r->leaves.assign(q.leaves, q.leaves + shared);
    r->est_bytes = srv->s->estimate_topk(*r, 1, q.k);
    return srv->s->submit(std::move(r));
}

uint64_t server_submit_join_aggregate(oxb_server* srv, const oxb_join_aggregate_args& a) {
    if (!a.probe || !a.table || !a.build) fail(OXB_PLAN, "join-aggregate request without probe, build or table");
    auto r = std::make_unique<Request>();
    r->kind = kReqJoinAggregate;
    r->ja = a;
    if (a.nleaves > 0) {
        if (!a.leaves) fail(OXB_PLAN, "null leaves");
        r->ja_leaves.assign(a.leaves, a.leaves + a.nleaves);
        r->ja.leaves = r->ja_leaves.data();
    }
    r->est_bytes = srv->s->estimate_join_aggregate(a);
    return srv->s->submit(std::move(r));
}

double server_wait(oxb_server* srv, uint64_t ticket, int64_t* ids, float* dist, oxb_batch** out) {
    std::unique_ptr<Request> r = srv->s->wait(ticket);
    if (r->status != OXB_OK) fail(r->status, r->error);
    if (r->kind == kReqTopk) {
        if (!ids || !dist) fail(OXB_PLAN, "null result buffers");
        std::copy(r->ids.begin(), r->ids.end(), ids);
        std::copy(r->dist.begin(), r->dist.end(), dist);
    } else {
        if (!out) {
            delete r->batch;
            fail(OXB_PLAN, "null result handle");
        }
        *out = r->batch;
        r->batch = nullptr;
    }
    return std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count();
}

void server_stats(oxb_server* srv, oxb_server_stats* out, bool reset) {
    Server& S = *srv->s;
    std::lock_guard<std::mutex> lk(S.mu);
    oxb_server_stats st{};
    st.completed = S.completed;
    st.rejected = S.rejected;
    st.dispatches = S.dispatches;
    st.batched_queries = S.batched;
    st.peak_bytes = (int64_t)S.peak;
    std::vector<double> l = S.latency_us;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (double)(l.size() - 1) + 0.5))]; };
        st.p50_us = pct(0.50);
        st.p99_us = pct(0.99);
        const double secs = std::chrono::duration<double>(S.last_done - S.first_submit).count();
        st.qps = secs > 0 ? (double)l.size() / secs : 0.0;
    }
    *out = st;
    if (reset) {
        S.latency_us.clear();
        S.completed = S.rejected = S.dispatches = S.batched = 0;
        S.peak = S.in_use;
        S.any = false;
    }
}

}  // namespace oxb
