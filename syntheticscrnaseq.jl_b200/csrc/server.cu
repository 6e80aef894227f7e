// Serving loop with continuous batching (scrna_server_*).
//
// A worker thread owns the device side.  Submitted requests queue FIFO; at every chunk
// boundary the worker admits queued requests while their device footprint fits the HBM
// budget, then advances every running request by chunk_steps Euler steps (small requests by
// a multiple of that, up to the largest request's work) with one
// persistent work-queue launch per register-path kernel group (the same kernels as
// scrna_cle_simulate).  State stays on the device between chunks, so a request's result
// does not depend on what else runs beside it.  Finished requests keep their outputs on
// the device until scrna_wait copies them out and releases the memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "capi_internal.h"
#include "nvtx_range.h"

namespace scrna {
void gene_tables_host(const scrna_net* n, const scrna_kinetics* kin, double dt, GeneRec* gr, GeneInit* gi,
                      uint8_t* qt);
}

using namespace scrna;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct SrvRequest {
    uint64_t ticket = 0;
    scrna_request req{};
    scrna_net* net = nullptr;
    int64_t N = 0, n_steps = 0, next = 1;
    scrna_state* st = nullptr;
    DevBuf genes, ginit, qtel;
    FusedArgs args{};
    KernelChoice kc{};
    int state = SCRNA_REQ_QUEUED;
    int64_t footprint = 0;
    double t_submit = 0, t_done = 0;
    std::string error;
    int64_t s0 = 0, s1 = 0;  // step range of the chunk in flight
    bool admitted = false;   // counted in the server's bytes in use
    bool cancel = false;     // cancellation requested while running (applied between chunks)
};

int64_t footprint_of(const scrna_net* n, int64_t N, int readout, bool cap) {
    const int64_t gn = (int64_t)n->G * N;
    int64_t b = gn * (4 + 4 + 1 + 4);                     // M, P, promoter, next switch
    b += gn * 8 * (readout == SCRNA_READOUT_BOTH ? 2 : 1);  // readout
    if (cap) b += gn * 4 + N * 8;
    return b + (1 << 16);
}

}  // namespace

struct scrna_server {
    scrna_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SrvRequest*> queue;
    std::vector<SrvRequest*> active;
    std::map<uint64_t, SrvRequest*> reqs;
    int64_t budget = 0, used = 0;
    int chunk_steps = 250;
    bool stop = false;
    uint64_t next_ticket = 1;
    scrna_server_stats stats{};
    DevBuf args_dev, items_dev, counters_dev;
    // the kernel groups of a chunk run side by side, one stream each, between two events
    static constexpr int kGroupStreams = 8;
    static constexpr int64_t kMaxChunkMultiple = 16;
    cudaStream_t gstream[kGroupStreams] = {};
    cudaEvent_t ev_inputs = nullptr, ev_group[kGroupStreams] = {};
    int n_group_streams = kGroupStreams;  // SCRNA_SERVER_GROUP_STREAMS=1: the groups one after another
    double t0 = 0.0;                      // creation time, origin of the trace clock
    static constexpr size_t kTrace = 4096;
    std::deque<scrna_chunk_record> trace;
    void run();
};

static void release(SrvRequest* r) {
    if (r->st) scrna_state_destroy(r->st);
    delete r;
}

// Device setup of an admitted request (worker thread).
static int setup_request(scrna_server* s, SrvRequest* r) {
    const scrna_net* n = r->net;
    if (int rr = scrna_state_create(s->ctx, n, r->N, r->req.opts.readout, r->req.with_capture, &r->st)) return rr;
    if (int rr = state_alloc(r->st, false, false)) return rr;
    r->st->have_counts = r->req.with_capture != 0;
    const int G = n->G;
    std::vector<GeneRec> gr(G);
    std::vector<GeneInit> gi(G);
    std::vector<uint8_t> qt((G + 3) / 4);
    gene_tables_host(n, &r->req.kin, r->req.opts.dt, gr.data(), gi.data(), qt.data());
    CU(r->genes.ensure(G * sizeof(GeneRec)));
    CU(r->ginit.ensure(G * sizeof(GeneInit)));
    CU(r->qtel.ensure(qt.size()));
    CU(cudaMemcpy(r->genes.p, gr.data(), G * sizeof(GeneRec), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(r->ginit.p, gi.data(), G * sizeof(GeneInit), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(r->qtel.p, qt.data(), qt.size(), cudaMemcpyHostToDevice));
    fill_fused_args(r->net, &r->req.kin, nullptr, r->req.with_capture ? &r->req.capture : nullptr, &r->req.opts,
                    r->st, &r->args);
    r->args.genes = r->genes.as<GeneRec>();  // this request's tables (the network's own are not uploaded here)
    r->args.ginit = r->ginit.as<GeneInit>();
    r->args.quad_tel = r->qtel.as<uint8_t>();
    // cached kernel choices only: a measurement here would stall every running request for
    // shapes that, in a request stream, mostly occur once
    if (int rr = choose_kernel_tuned(s->ctx, const_cast<scrna_net*>(n), &r->req.kin, &r->req.opts, r->st, &r->kc,
                                     &r->args, s->stream, false))
        return rr;
    r->args.lane_nw1 = r->kc.nw1;
    return SCRNA_OK;
}

void scrna_server::run() {
    cudaSetDevice(ctx->device);
    std::vector<FusedArgs> h_args;
    std::vector<TileWork> h_items;
    for (;;) {
        std::vector<SrvRequest*> admitted;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || !queue.empty() || !active.empty(); });
            if (stop) break;
            // cancellations of running requests take effect between chunks
            for (size_t i = 0; i < active.size();) {
                if (active[i]->cancel) {
                    active[i]->state = SCRNA_REQ_CANCELLED;
                    active.erase(active.begin() + i);
                    cv_done.notify_all();
                } else {
                    ++i;
                }
            }
            // FIFO admission by device footprint (a cancelled request has left the queue already)
            while (!queue.empty()) {
                SrvRequest* r = queue.front();
                if (r->footprint > budget) {
                    r->state = SCRNA_REQ_FAILED;
                    r->error = "request does not fit the device memory budget";
                    queue.pop_front();
                    stats.failed++;
                    cv_done.notify_all();
                    continue;
                }
                if (used + r->footprint > budget) break;
                used += r->footprint;
                r->admitted = true;
                // RUNNING from here: a cancellation during the set-up below becomes a flag honoured at
                // the next chunk boundary, so scrna_wait cannot free the request while it is set up
                r->state = SCRNA_REQ_RUNNING;
                queue.pop_front();
                admitted.push_back(r);
            }
        }
        for (SrvRequest* r : admitted) {
            const int rc = setup_request(this, r);
            std::lock_guard<std::mutex> lk(mu);
            if (rc != SCRNA_OK) {
                r->state = SCRNA_REQ_FAILED;
                r->error = scrna_last_error();
                stats.failed++;
                cv_done.notify_all();
            } else {
                active.push_back(r);
            }
        }
        std::vector<SrvRequest*> run_set;
        {
            std::lock_guard<std::mutex> lk(mu);
            run_set = active;
        }
        if (run_set.empty()) continue;
        const double t_chunk = now_s();
        NvtxRange nvtx_chunk_("scrna_server_chunk");
        // one persistent launch per kernel group over the running requests' tiles
        h_args.clear();
        std::map<std::tuple<int, int, int, int, int>, std::vector<TileWork>> groups;
        std::map<std::tuple<int, int, int, int, int>, std::pair<int, size_t>> shape;  // nw, smem
        // Steps of each request in this chunk: chunk_steps, or up to kMaxChunkMultiple times that
        // for a request whose work per step is that much smaller than the largest one's, so small
        // requests finish in few chunks while the chunk's length stays set by the largest
        // (results do not depend on the chunking).
        double w_max = 0.0;
        for (SrvRequest* r : run_set) w_max = std::max(w_max, (double)r->net->G * (double)r->N);
        for (size_t i = 0; i < run_set.size(); ++i) {
            SrvRequest* r = run_set[i];
            h_args.push_back(r->args);
            const double ups = (double)r->net->G * (double)r->N;
            const int64_t mult = std::min<int64_t>(kMaxChunkMultiple, std::max<int64_t>(1, (int64_t)(w_max / ups)));
            r->s0 = r->next;
            r->s1 = r->n_steps == 0 ? 0 : std::min<int64_t>(r->n_steps, r->next + chunk_steps * mult - 1);
            const KernelChoice& kc = r->kc;
            // (warp kernel, genes per lane, in-edges, warps per block or block-kernel quads per thread, terms)
            auto key = std::make_tuple((int)kc.warp, kc.warp ? kc.gpl : 0, kc.warp ? kc.emax : 0,
                                       kc.warp ? kc.nwarps : kc.block.upt, kc.warp ? kc.tmax : 0);
            int64_t cpt = 32;
            if (kc.warp) cpt = warpcell_cells_per_block_host(r->net->G, kc.gpl, kc.nw1);
            const int64_t tiles = (r->N + cpt - 1) / cpt;
            TileCtl ctl{(int32_t)r->s0, (int32_t)r->s1, r->s0 == 1 ? 1 : 0, r->s1 >= r->n_steps ? 1 : 0, 0, 0};
            auto& items = groups[key];
            for (int64_t t = 0; t < tiles; ++t) items.push_back(TileWork{(int32_t)i, (int32_t)t, ctl});
            auto& sh = shape[key];
            sh.first = std::max(sh.first, kc.warp ? 1 : kc.block.nw);
            sh.second = std::max(sh.second, kc.smem);
        }
        h_items.clear();
        std::vector<size_t> offsets;
        for (auto& kv : groups) {
            // longest step ranges first, so no long item starts at the end of the work queue
            std::stable_sort(kv.second.begin(), kv.second.end(), [](const TileWork& x, const TileWork& y) {
                return x.ctl.step_end - x.ctl.step_begin > y.ctl.step_end - y.ctl.step_begin;
            });
            offsets.push_back(h_items.size());
            h_items.insert(h_items.end(), kv.second.begin(), kv.second.end());
        }
        int rc = SCRNA_OK;
        cudaError_t e = cudaSuccess;
        if ((e = args_dev.ensure(h_args.size() * sizeof(FusedArgs))) != cudaSuccess ||
            (e = items_dev.ensure(h_items.size() * sizeof(TileWork))) != cudaSuccess ||
            (e = counters_dev.ensure(groups.size() * sizeof(int))) != cudaSuccess ||
            (e = cudaMemcpyAsync(args_dev.p, h_args.data(), h_args.size() * sizeof(FusedArgs), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(items_dev.p, h_items.data(), h_items.size() * sizeof(TileWork), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(counters_dev.p, 0, groups.size() * sizeof(int), stream)) != cudaSuccess)
            rc = SCRNA_ECUDA;
        // every group stream waits for this chunk's argument and work-item copies
        if (rc == SCRNA_OK && (e = cudaEventRecord(ev_inputs, stream)) != cudaSuccess) rc = SCRNA_ECUDA;
        for (int k = 0; rc == SCRNA_OK && k < n_group_streams && k < (int)groups.size(); ++k)
            if ((e = cudaStreamWaitEvent(gstream[k], ev_inputs, 0)) != cudaSuccess) rc = SCRNA_ECUDA;
        size_t gi = 0;
        for (auto& kv : groups) {
            if (rc != SCRNA_OK) break;
            cudaStream_t gs = gstream[gi % n_group_streams];
            const auto& key = kv.first;
            const int n_items = (int)kv.second.size();
            const TileWork* items = items_dev.as<TileWork>() + offsets[gi];
            int* counter = counters_dev.as<int>() + gi;
            const auto& sh = shape[key];
            const int per_sm = std::get<0>(key) ? std::max(1, 24 / std::get<3>(key)) : 8;
            const int grid = std::max(1, std::min(n_items, ctx->sm_count * per_sm));
            if (std::get<0>(key))
                e = warpcell_queue_launch(args_dev.as<FusedArgs>(), items, n_items, counter, std::get<1>(key),
                                          std::get<2>(key), std::get<4>(key), false, sh.second, grid,
                                          std::get<3>(key), TileCtl{}, 0, nullptr, gs);
            else
                e = fused_queue_launch(args_dev.as<FusedArgs>(), items, n_items, counter, std::get<3>(key), sh.first,
                                       sh.second, false, grid, TileCtl{}, 0, gs);
            if (e != cudaSuccess) rc = SCRNA_ECUDA;
            ++gi;
        }
        // the chunk ends when every group stream has finished
        for (int k = 0; k < n_group_streams && k < (int)groups.size(); ++k) {
            cudaError_t e2 = cudaEventRecord(ev_group[k], gstream[k]);
            if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(stream, ev_group[k], 0);
            if (e2 != cudaSuccess && rc == SCRNA_OK) { rc = SCRNA_ECUDA; e = e2; }
        }
        {
            cudaError_t e2 = cudaStreamSynchronize(stream);
            if (e2 != cudaSuccess && rc == SCRNA_OK) { rc = SCRNA_ECUDA; e = e2; }
        }
        const double t_end = now_s();
        std::lock_guard<std::mutex> lk(mu);
        {
            scrna_chunk_record rec{t_chunk - t0, t_end - t0, (int32_t)run_set.size(), (int32_t)groups.size(), 0};
            for (SrvRequest* r : run_set)
                if (r->s1 >= r->s0) rec.units += (int64_t)r->net->G * r->N * (r->s1 - r->s0 + 1);
            if (trace.size() == kTrace) trace.pop_front();
            trace.push_back(rec);
        }
        stats.busy_s += t_end - t_chunk;
        stats.chunks += (int64_t)groups.size();
        ctx->launches += (int64_t)groups.size();
        for (SrvRequest* r : run_set) {
            if (r->state != SCRNA_REQ_RUNNING) continue;
            if (rc != SCRNA_OK) {
                r->state = SCRNA_REQ_FAILED;
                r->error = std::string("kernel launch failed: ") + cudaGetErrorString(e);
                stats.failed++;
            } else {
                r->next = r->s1 + 1;
                if (r->s1 >= r->n_steps) {
                    r->state = SCRNA_REQ_DONE;
                    r->t_done = t_end;
                    stats.completed++;
                    stats.units_done += (int64_t)r->net->G * r->N * r->n_steps;
                }
            }
        }
        for (size_t i = 0; i < active.size();) {
            if (active[i]->state != SCRNA_REQ_RUNNING) active.erase(active.begin() + i);
            else ++i;
        }
        cv_done.notify_all();
    }
}

static void destroy_streams(scrna_server* s) {
    for (int k = 0; k < scrna_server::kGroupStreams; ++k) {
        if (s->ev_group[k]) cudaEventDestroy(s->ev_group[k]);
        if (s->gstream[k]) cudaStreamDestroy(s->gstream[k]);
    }
    if (s->ev_inputs) cudaEventDestroy(s->ev_inputs);
    if (s->stream) cudaStreamDestroy(s->stream);
}

extern "C" int scrna_server_create(scrna_ctx* ctx, int64_t budget, int32_t chunk_steps, scrna_server** out) {
    if (!ctx || !out) return fail(SCRNA_EINVAL, "ctx/out is NULL");
    if (chunk_steps <= 0) return fail(SCRNA_EINVAL, "chunk_steps must be positive");
    if (int r = set_device(ctx)) return r;
    auto* s = new scrna_server();
    s->ctx = ctx;
    s->chunk_steps = chunk_steps;
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        budget = (int64_t)(0.8 * (double)fr);
    }
    s->budget = budget;
    s->t0 = now_s();
    if (const char* g = std::getenv("SCRNA_SERVER_GROUP_STREAMS"))
        s->n_group_streams = std::min(std::max(std::atoi(g), 1), (int)scrna_server::kGroupStreams);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_inputs, cudaEventDisableTiming);
    for (int k = 0; k < scrna_server::kGroupStreams && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&s->gstream[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_group[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        destroy_streams(s);
        delete s;
        return fail(SCRNA_ECUDA, "stream/event creation: %s", cudaGetErrorString(e));
    }
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return SCRNA_OK;
}

extern "C" int scrna_server_destroy(scrna_server* s) {
    if (!s) return SCRNA_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->stream);
    for (int k = 0; k < scrna_server::kGroupStreams; ++k)
        if (s->gstream[k]) cudaStreamSynchronize(s->gstream[k]);
    for (auto& kv : s->reqs) release(kv.second);
    destroy_streams(s);
    delete s;
    return SCRNA_OK;
}

extern "C" int scrna_submit(scrna_server* s, const scrna_request* q, uint64_t* ticket) {
    if (!s || !q || !ticket) return fail(SCRNA_EINVAL, "bad arguments");
    const scrna_capture* cap = q->with_capture ? &q->capture : nullptr;
    if (int r = validate_run(q->net, &q->kin, nullptr, cap, &q->opts)) return r;
    if (q->opts.precision != SCRNA_PRECISION_FP32) return fail(SCRNA_ENOTSUP, "the server runs the FP32 path");
    const scrna_net* n = q->net;
    if (!register_path_holds(n->dev))
        return fail(SCRNA_ENOTSUP, "the server runs register-path networks (G <= 512, tables within shared memory)");
    if (q->opts.cell_num <= 0) return fail(SCRNA_EINVAL, "cell_num must be positive");
    if (q->opts.cell_offset < 0 || q->opts.cell_offset + q->opts.cell_num > (1ll << 32)) return fail(SCRNA_EINVAL, "cell indices must fit 32 bits");
    auto* r = new SrvRequest();
    r->req = *q;
    r->net = const_cast<scrna_net*>(n);
    r->N = q->opts.cell_num;
    r->n_steps = n_steps_of(&q->opts);
    if (r->n_steps >= (1ll << 31)) { delete r; return fail(SCRNA_EINVAL, "too many steps"); }
    r->footprint = footprint_of(n, r->N, q->opts.readout, cap != nullptr);
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->ticket = s->next_ticket++;
        s->reqs[r->ticket] = r;
        s->queue.push_back(r);
        s->stats.submitted++;
    }
    s->cv_work.notify_all();
    *ticket = r->ticket;
    return SCRNA_OK;
}

extern "C" int scrna_poll(scrna_server* s, uint64_t ticket, int32_t* state) {
    if (!s || !state) return fail(SCRNA_EINVAL, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(SCRNA_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
    *state = it->second->state;
    return SCRNA_OK;
}

extern "C" int scrna_wait(scrna_server* s, uint64_t ticket, int32_t timeout_ms, double* out, int32_t* counts,
                          double* eff, double* latency_s) {
    NvtxRange nvtx_range_("scrna_wait");
    if (!s) return fail(SCRNA_EINVAL, "server is NULL");
    SrvRequest* r = nullptr;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return fail(SCRNA_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
        r = it->second;
        auto finished = [&] { return r->state >= SCRNA_REQ_DONE; };
        if (timeout_ms < 0) s->cv_done.wait(lk, finished);
        else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished))
            return fail(SCRNA_ETIMEOUT, "request %llu not done within %d ms", (unsigned long long)ticket, timeout_ms);
        s->reqs.erase(it);
    }
    int rc = SCRNA_OK;
    if (r->state == SCRNA_REQ_DONE) {
        if (latency_s) *latency_s = r->t_done - r->t_submit;
        if (out || counts || eff)
            rc = scrna_state_read(s->ctx, r->st, out, r->req.with_capture ? counts : nullptr,
                                  r->req.with_capture ? eff : nullptr);
    } else if (r->state == SCRNA_REQ_CANCELLED) {
        rc = fail(SCRNA_ECANCELED, "request %llu was cancelled", (unsigned long long)ticket);
    } else {
        rc = fail(SCRNA_ECUDA, "request %llu failed: %s", (unsigned long long)ticket, r->error.c_str());
    }
    const bool admitted = r->admitted;
    const int64_t fp = r->footprint;
    release(r);
    if (admitted) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->used -= fp;
    }
    s->cv_work.notify_all();
    return rc;
}

extern "C" int scrna_cancel(scrna_server* s, uint64_t ticket) {
    if (!s) return fail(SCRNA_EINVAL, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(SCRNA_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
    SrvRequest* r = it->second;
    if (r->state == SCRNA_REQ_QUEUED) {  // never on the device: out of the queue before scrna_wait frees it
        s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), r), s->queue.end());
        r->state = SCRNA_REQ_CANCELLED;
        s->cv_done.notify_all();
    } else if (r->state == SCRNA_REQ_RUNNING) {
        r->cancel = true;  // dropped at the next chunk boundary (admitted requests are RUNNING)
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return SCRNA_OK;
}

extern "C" int scrna_server_trace(scrna_server* s, scrna_chunk_record* recs, int32_t capacity, int32_t* n) {
    if (!s || !n) return fail(SCRNA_EINVAL, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!recs) {
        *n = (int32_t)s->trace.size();
        return SCRNA_OK;
    }
    const int32_t k = std::min<int32_t>(std::max(capacity, 0), (int32_t)s->trace.size());
    for (int32_t i = 0; i < k; ++i) recs[i] = s->trace[i];
    *n = k;
    return SCRNA_OK;
}

extern "C" int scrna_server_get_stats(scrna_server* s, scrna_server_stats* out) {
    if (!s || !out) return fail(SCRNA_EINVAL, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->queued = (int64_t)s->queue.size();
    out->running = (int64_t)s->active.size();
    out->bytes_in_use = s->used;
    return SCRNA_OK;
}
