// Request server: continuous batching of bilateral, joint-bilateral and Gauss-transform
// requests onto the batched lattice.
//
// Workers are host threads, each with its own engine (CUDA stream, lattice workspace), so
// the batches of different workers overlap on the device.  An idle worker takes the
// oldest queued request that fits the memory budget, adds every queued request that can
// share its launches (same kind of output, position dimensions and value channels) while
// the batch stays within its share of the budget, runs the batch, and frees the budget.
// Requests that arrive meanwhile wait in the queue and are admitted as soon as a worker
// and memory are free.  The footprint that admission counts is the device memory a
// request needs: its images and its share of the hash table and vertex arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "engine.h"

namespace pgpu {
namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    long long id = 0;
    pgpu_request r;
    std::vector<float> sigmas;
    int d = 0, vd = 0, out_channels = 0;
    bool normalize = true;
    int key = 0;               // requests with equal keys can share a batch
    uint32_t n = 0;
    size_t footprint = 0;
    Clock::time_point t_submit, t_done;
    int status = -1;           // -1 while queued or running
    bool claimed = false;      // a thread is waiting for it (one waiter per ticket)
    std::string error;
};

// Device bytes of one request: staging images, hash-table slots (learned vertices per
// point x 1.3 / load, at most one vertex per point here as the conservative default) and
// per-point records.
size_t footprint(uint32_t n, int d, int vd, int in_ch, int ref_ch, int out_ch, int payload, float load) {
    const int vdp = vdp_for(vd);
    const size_t accb = accum_bytes(payload), payb = payload_bytes(payload);
    const int kw = key_words(d);
    const size_t per_slot = 16 * 2 + (size_t)(kw - 1) * 32 + vdp * accb * 2 + 12 + vdp * payb * 2 +
                            vdp * 4 + (size_t)(d + 1) * 8;
    const double slots = 1.3 * n / (load > 0.05f ? load : 0.5f) + 256;
    const size_t per_point = (size_t)(d + 1) * 4 + ((size_t)(d + 1) + 31) / 32 * 8 +
                             (size_t)(in_ch + ref_ch + out_ch) * 4;
    return (size_t)(slots * per_slot) + (size_t)n * per_point + 4096;
}

class Server {
public:
    pgpu_server_config cfg;
    size_t worker_cap = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> queue;
    std::unordered_map<long long, Req*> reqs;
    std::vector<std::thread> threads;
    std::vector<Engine*> engines;
    bool stopping = false;
    long long next_id = 1;
    size_t inflight = 0, peak = 0;
    long long running = 0;
    // measurement window
    std::vector<double> lat_ms;
    long long submitted = 0, completed = 0, failed = 0, rejected = 0, batches = 0, pixels = 0;
    bool have_t0 = false;
    Clock::time_point t0, t_last;

    bool head_fits() const {
        return !queue.empty() && inflight + queue.front()->footprint <= (size_t)cfg.memory_budget;
    }

    void worker(int w) {
        Engine& E = *engines[w];
        cudaSetDevice(cfg.device);
        set_call_stream(E.stream);   // this worker's workspace lives on its stream
        std::vector<Req*> batch;
        for (;;) {
            size_t fp = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stopping || head_fits(); });
                if (stopping && queue.empty()) return;
                batch.clear();
                for (auto it = queue.begin(); it != queue.end();) {
                    Req* q = *it;
                    const bool first = batch.empty();
                    if (first) {
                        if (inflight + q->footprint > (size_t)cfg.memory_budget) break;
                    } else if (q->key != batch[0]->key || (int)batch.size() >= cfg.max_batch ||
                               fp + q->footprint > worker_cap ||
                               inflight + fp + q->footprint > (size_t)cfg.memory_budget) {
                        ++it;
                        continue;
                    }
                    batch.push_back(q);
                    fp += q->footprint;
                    it = queue.erase(it);
                }
                if (batch.empty()) continue;
                inflight += fp;
                peak = std::max(peak, inflight);
                running += (long long)batch.size();
            }
            const int rc = run_and_drain(E, batch);
            const std::string err = rc ? std::string(last_error()) : std::string();
            {
                std::lock_guard<std::mutex> lk(mu);
                inflight -= fp;
                running -= (long long)batch.size();
                ++batches;
                const Clock::time_point now = Clock::now();
                t_last = now;
                for (Req* q : batch) {
                    q->t_done = now;
                    q->status = rc;
                    q->error = err;
                    if (rc == PGPU_OK) {
                        ++completed;
                        pixels += q->n;
                        lat_ms.push_back(std::chrono::duration<double, std::milli>(now - q->t_submit).count());
                    } else {
                        ++failed;
                    }
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    // run() and then wait for the worker's stream whatever run() returned: a failure can
    // leave copies from or to the requests' host buffers queued, and the caller may free
    // or reuse those buffers as soon as the request is published as finished
    int run_and_drain(Engine& E, const std::vector<Req*>& batch) {
        int rc = run(E, batch);
        const std::string err = rc ? std::string(last_error()) : std::string();
        const cudaError_t se = cudaStreamSynchronize(E.stream);
        if (rc) return fail(rc, "%s", err.c_str());
        if (se != cudaSuccess)
            return fail(PGPU_ERR_CUDA, "server stream: %s", cudaGetErrorString(se));
        return PGPU_OK;
    }

    // stage the batch's images, run the batched lattice, copy the results back
    int run(Engine& E, const std::vector<Req*>& batch) {
        clear_error();
        const cudaStream_t st = E.stream;
        size_t floats = 0;
        for (Req* q : batch) {
            const pgpu_request& r = q->r;
            floats += (size_t)q->n * (r.in.channels + q->out_channels +
                                      (r.kind == PGPU_REQ_BILATERAL ? 0 : r.ref.channels));
        }
        int rc;
        if ((rc = E.img_a.ensure(floats * sizeof(float)))) return rc;
        float* p = (float*)E.img_a.p;
        BatchJob B;
        B.d = batch[0]->d;
        B.vd = batch[0]->vd;
        B.payload = cfg.payload;
        B.load = cfg.load_factor;
        B.homog = batch[0]->normalize;
        B.replay = true;
        B.items.resize(batch.size());
        std::vector<pgpu_image> dout(batch.size());
        volatile float one = 1.0f;
        for (size_t k = 0; k < batch.size(); ++k) {
            const Req* q = batch[k];
            const pgpu_request& r = q->r;
            pgpu_image din = dense_like(r.in, p, r.in.channels);
            p += (size_t)q->n * r.in.channels;
            if ((rc = copy_view(r.in, din, r.in.channels, cudaMemcpyHostToDevice, st))) return rc;
            pgpu_image dpos = din;
            if (r.kind != PGPU_REQ_BILATERAL) {
                dpos = dense_like(r.ref, p, r.ref.channels);
                p += (size_t)q->n * r.ref.channels;
                if ((rc = copy_view(r.ref, dpos, r.ref.channels, cudaMemcpyHostToDevice, st))) return rc;
            }
            dout[k] = dense_like(r.out, p, q->out_channels);
            p += (size_t)q->n * q->out_channels;
            BatchItem& it = B.items[k];
            PointSource& s = it.splat;
            memset(&s, 0, sizeof(s));
            s.width = r.in.width;
            s.height = r.in.height;
            s.frames = r.in.frames;
            s.pos = planar(dpos);
            s.pos_channels = dpos.channels;
            s.val = planar(din);
            s.val_channels = din.channels;
            if (r.kind == PGPU_REQ_GAUSS_TRANSFORM) {
                for (int c = 0; c < dpos.channels; ++c) s.pos_scale[c] = one / q->sigmas[c];
                s.homogeneous = 0;
                it.out = outview(dout[k], q->out_channels, 0);
            } else {
                const float inv_r = one / r.color_sigma;
                for (int c = 0; c < dpos.channels; ++c) s.pos_scale[c] = inv_r;
                s.coord_mask = 3;
                s.coord_scale[0] = one / r.filter_width;
                s.coord_scale[1] = one / r.filter_width;
                s.homogeneous = 1;
                it.out = outview(dout[k], q->out_channels, 1);
            }
            it.n = q->n;
        }
        // The lattices follow the uploads on this worker's stream; the other workers'
        // copies and lattices run on theirs at the same time.
        if ((rc = run_batch(E, B, st))) return rc;
        for (size_t k = 0; k < batch.size(); ++k)
            if ((rc = copy_view(dout[k], batch[k]->r.out, batch[k]->out_channels, cudaMemcpyDeviceToHost, st)))
                return rc;
        CUDA_TRY(cudaStreamSynchronize(st));
        return PGPU_OK;
    }

    int validate(const pgpu_request& r, Req* q) {
        if (!view_ok(&r.in) || !view_ok(&r.out)) return fail(PGPU_ERR_ARGUMENT, "invalid image view");
        if (!points_fit(&r.in)) return fail(PGPU_ERR_UNSUPPORTED, "more than 2^32 - 1 points in one request");
        const pgpu_image& a = r.in;
        switch (r.kind) {
        case PGPU_REQ_BILATERAL:
        case PGPU_REQ_JOINT_BILATERAL: {
            const pgpu_image& g = r.kind == PGPU_REQ_BILATERAL ? r.in : r.ref;
            if (r.kind == PGPU_REQ_JOINT_BILATERAL &&
                (!view_ok(&r.ref) || r.ref.width != a.width || r.ref.height != a.height || r.ref.frames != 1))
                return fail(PGPU_ERR_ARGUMENT, "reference must be a single frame of the image's size");
            if (a.frames != 1 || a.width < 2 || a.height < 2 || !(r.filter_width > 0) ||
                !(r.filter_width < 10 * a.width) || !(r.filter_width < 10 * a.height) || !(r.color_sigma > 0))
                return fail(PGPU_ERR_UNSUPPORTED,
                            "bilateral requests: single frames larger than 1x1 with 0 < filter width < 10 x "
                            "their size (filter others with pgpu_bilateral)");
            if (a.channels + 1 > 8 || g.channels + 2 > kMaxD)
                return fail(PGPU_ERR_UNSUPPORTED, "too many channels");
            if (r.out.width != a.width || r.out.height != a.height || r.out.frames != 1 || r.out.channels < a.channels)
                return fail(PGPU_ERR_ARGUMENT, "output must have the image's size and channels");
            q->d = g.channels + 2;
            q->vd = a.channels + 1;
            q->out_channels = a.channels;
            q->normalize = true;
            q->key = (q->d << 8) | q->vd;
            break;
        }
        case PGPU_REQ_GAUSS_TRANSFORM: {
            if (!view_ok(&r.ref) || r.ref.width != a.width || r.ref.height != a.height || r.ref.frames != a.frames)
                return fail(PGPU_ERR_ARGUMENT, "Weights and locations of the Gaussians must be the same size");
            if (r.ref.channels > kMaxD || a.channels > 8)
                return fail(PGPU_ERR_UNSUPPORTED, "at most %d position and 8 value channels", kMaxD);
            if (!r.sigmas || r.n_sigmas < r.ref.channels)
                return fail(PGPU_ERR_ARGUMENT, "need one sigma per position channel");
            if (r.out.width != a.width || r.out.height != a.height || r.out.frames != a.frames ||
                r.out.channels < a.channels)
                return fail(PGPU_ERR_ARGUMENT, "output must have the positions' size and the values' channels");
            q->d = r.ref.channels;
            q->vd = a.channels;
            q->out_channels = a.channels;
            q->normalize = false;
            q->sigmas.assign(r.sigmas, r.sigmas + r.ref.channels);
            q->key = (1 << 16) | (q->d << 8) | q->vd;
            break;
        }
        default:
            return fail(PGPU_ERR_ARGUMENT, "unknown request kind %d", r.kind);
        }
        q->n = (uint32_t)((size_t)a.width * a.height * a.frames);
        q->footprint = footprint(q->n, q->d, q->vd, a.channels,
                                 r.kind == PGPU_REQ_BILATERAL ? 0 : r.ref.channels, q->out_channels,
                                 cfg.payload, cfg.load_factor);
        if (q->footprint > (size_t)cfg.memory_budget)
            return fail(PGPU_ERR_ADMISSION, "request needs about %zu bytes of device memory, more than the "
                        "budget of %lld", q->footprint, cfg.memory_budget);
        return PGPU_OK;
    }
};

}  // namespace
}  // namespace pgpu

using namespace pgpu;

extern "C" {

int pgpu_server_create(const pgpu_server_config* cfg_in, void** out) {
    clear_error();
    if (!out) return fail(PGPU_ERR_ARGUMENT, "null server pointer");
    pgpu_server_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    if (cfg_in) cfg = *cfg_in;
    // Two workers by default: measured on the served request mix at saturation, one worker
    // retires 2750 req/s, two 3450-3640, and three or more far fewer (1180-1440), their
    // lattices' tables competing for L2 while they overlap.
    if (cfg.workers <= 0) cfg.workers = 2;
    if (cfg.max_batch <= 0) cfg.max_batch = 64;
    if (!(cfg.load_factor > 0.05f && cfg.load_factor <= 0.9f)) cfg.load_factor = 0.5f;
    if (cfg.memory_budget <= 0) cfg.memory_budget = 40ll << 30;
    if (cfg.payload < 0 || cfg.payload > 3) return fail(PGPU_ERR_ARGUMENT, "unknown payload %d", cfg.payload);
    std::unique_ptr<Server> S(new Server());
    S->cfg = cfg;
    S->worker_cap = (size_t)cfg.memory_budget / (size_t)cfg.workers;
    for (int w = 0; w < cfg.workers; ++w) {
        Engine* e = new Engine();
        const int rc = e->init(cfg.device);
        if (rc) {
            delete e;
            for (Engine* x : S->engines) { x->shutdown(); delete x; }
            return rc;
        }
        S->engines.push_back(e);
    }
    // The workspaces of requests admitted under the budget come from memory the library's
    // pool already holds: reserving the budget now keeps their growth under load from
    // mapping new device memory in the middle of the stream (served outliers of 100-350 ms).
    {
        const int rc = reserve_pool_memory((size_t)cfg.memory_budget, S->engines[0]->stream);
        if (rc) {
            for (Engine* x : S->engines) { x->shutdown(); delete x; }
            return rc;
        }
    }
    Server* raw = S.get();
    for (int w = 0; w < cfg.workers; ++w) S->threads.emplace_back([raw, w] { raw->worker(w); });
    *out = S.release();
    return PGPU_OK;
}

int pgpu_server_submit(void* server, const pgpu_request* req, long long* ticket) {
    clear_error();
    Server* S = (Server*)server;
    if (!S || !req) return fail(PGPU_ERR_ARGUMENT, "null server or request");
    Req* q = new Req();
    q->r = *req;
    const int rc = S->validate(*req, q);
    std::lock_guard<std::mutex> lk(S->mu);
    if (rc) {
        ++S->rejected;
        delete q;
        return rc;
    }
    q->id = S->next_id++;
    q->t_submit = Clock::now();
    if (!S->have_t0) {
        S->have_t0 = true;
        S->t0 = q->t_submit;
    }
    ++S->submitted;
    S->reqs[q->id] = q;
    S->queue.push_back(q);
    if (ticket) *ticket = q->id;
    S->cv_work.notify_one();
    return PGPU_OK;
}

int pgpu_server_wait(void* server, long long ticket, int timeout_ms) {
    Server* S = (Server*)server;
    if (!S) return fail(PGPU_ERR_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(PGPU_ERR_ARGUMENT, "unknown ticket %lld", ticket);
    Req* q = it->second;
    // the first waiter to find the request done deletes it, so a second concurrent waiter
    // on the same ticket is refused rather than left reading freed memory
    if (q->claimed) return fail(PGPU_ERR_ARGUMENT, "ticket %lld is already being waited for", ticket);
    q->claimed = true;
    if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)),
                             [&] { return q->status >= 0; })) {
        q->claimed = false;   // a later wait may try again
        return fail(PGPU_ERR_TIMEOUT, "request %lld not done after %d ms", ticket, timeout_ms);
    }
    const int rc = q->status;
    if (rc) fail(rc, "%s", q->error.c_str());
    S->reqs.erase(it);
    delete q;
    return rc;
}

int pgpu_server_drain(void* server, int timeout_ms) {
    Server* S = (Server*)server;
    if (!S) return fail(PGPU_ERR_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)),
                             [&] { return S->queue.empty() && S->running == 0; }))
        return fail(PGPU_ERR_TIMEOUT, "server still busy after %d ms", timeout_ms);
    return PGPU_OK;
}

int pgpu_server_get_stats(void* server, pgpu_server_stats* out) {
    Server* S = (Server*)server;
    if (!S || !out) return fail(PGPU_ERR_ARGUMENT, "null server or stats");
    std::lock_guard<std::mutex> lk(S->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->failed = S->failed;
    out->rejected = S->rejected;
    out->queued = (long long)S->queue.size();
    out->in_flight = S->running;
    out->batches = S->batches;
    out->pixels = S->pixels;
    out->peak_bytes = (long long)S->peak;
    if (S->have_t0 && S->completed)
        out->seconds = std::chrono::duration<double>(S->t_last - S->t0).count();
    std::vector<double> l(S->lat_ms);
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = l.back();
        double s = 0;
        for (double x : l) s += x;
        out->mean_ms = s / l.size();
    }
    if (out->seconds > 0) {
        out->mpix_per_s = S->pixels / out->seconds / 1e6;
        out->req_per_s = S->completed / out->seconds;
    }
    return PGPU_OK;
}

int pgpu_server_reset_stats(void* server) {
    Server* S = (Server*)server;
    if (!S) return fail(PGPU_ERR_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    S->lat_ms.clear();
    S->submitted = S->completed = S->failed = S->rejected = S->batches = S->pixels = 0;
    S->have_t0 = false;
    S->peak = S->inflight;
    return PGPU_OK;
}

void pgpu_server_destroy(void* server) {
    Server* S = (Server*)server;
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto& t : S->threads) t.join();
    for (Engine* e : S->engines) {
        e->shutdown();
        delete e;
    }
    for (auto& kv : S->reqs) delete kv.second;
    delete S;
}

}  // extern "C"
