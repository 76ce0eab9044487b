// serve.cpp -- many independent GPLMR solves on one GPU: a request queue
// with admission by device footprint and a pool of worker threads, each on
// its own CUDA stream, so that the kernels of different solves overlap.
//
// The reference runs one GPLMR_EIG per MPI job (doublyexcited.F90:238-241)
// and has no serving layer; the solve itself is de_gplmr_eig unchanged.
//
// Scheduling: first come, first served.  A free worker takes the head of the
// queue once its footprint fits in the budget that the running solves leave;
// the head is never overtaken, so a large request waits for memory rather
// than starving.  Handles (operator tables) are cached per worker by
// operator key; each solve's workspace goes back to the stream-ordered pool
// when it ends, so the budget counts only running solves.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "de_internal.h"
#include "de_kernels.h"

using namespace de;

namespace {

using clk = std::chrono::steady_clock;

struct Job {
    uint64_t id;
    de_request req;
    int64_t footprint;
    de_result res;
    bool done = false;
    bool collected = false;
};

bool same_operator(const de_params &a, const de_params &b)
{
    return a.n == b.n && a.delta == b.delta && a.radius == b.radius && a.autodelta == b.autodelta &&
           a.theta == b.theta && a.charge == b.charge && a.nelec == b.nelec && a.nsmall == b.nsmall &&
           a.tfactor == b.tfactor && a.precision == b.precision;
}

}  // namespace

struct de_server_impl {
    de_server_opts opts{};
    clk::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::list<Job *> finished;  // done, not yet collected, in completion order
    std::vector<std::thread> workers;
    int64_t reserved = 0;
    int running = 0;
    uint64_t next_id = 1;
    bool stop = false;

    double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }

    void worker_main(int w)
    {
        cudaSetDevice(opts.device);
        struct Cached {
            de_params p;
            de_problem *h;
        };
        std::list<Cached> handles;  // most recent first, at most 4
        for (;;) {
            Job *j = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    return stop || (!queue.empty() && reserved + queue.front()->footprint <= opts.max_bytes);
                });
                if (stop) break;
                j = queue.front();
                queue.pop_front();
                reserved += j->footprint;
                ++running;
                j->res.t_start_s = now();
                j->res.worker = w;
            }
            // operator handle for this request (cached per worker)
            de_problem *h = nullptr;
            int s = DE_OK;
            for (auto it = handles.begin(); it != handles.end(); ++it)
                if (same_operator(it->p, j->req.params)) {
                    h = it->h;
                    handles.splice(handles.begin(), handles, it);
                    break;
                }
            if (!h) {
                de_params p = j->req.params;
                p.device = opts.device;
                s = de_problem_create(&p, &h);
                if (s == DE_OK) {
                    handles.push_front(Cached{j->req.params, h});
                    if (handles.size() > 4) {
                        de_problem_destroy(handles.back().h);
                        handles.pop_back();
                    }
                }
            }
            de_stats st{};
            if (s == DE_OK) {
                const de_request &r = j->req;
                s = de_gplmr_eig(h, r.x, r.e, h->m, h->dim / h->m, r.sigma, r.nev, r.ns, r.maxit, r.tol, &r.gm, 0,
                                 &st);
                {
                    std::lock_guard<std::mutex> hl(h->mu);
                    h->trim();  // the workspace goes back to the pool
                }
                cudaStreamSynchronize(h->stream);
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                j->res.status = s;
                j->res.stats = st;
                j->res.t_end_s = now();
                j->done = true;
                reserved -= j->footprint;
                --running;
                finished.push_back(j);
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
        for (auto &c : handles) de_problem_destroy(c.h);
    }
};

extern "C" {

DE_API int de_request_footprint(const de_request *r, int64_t *bytes)
{
    if (!r || !bytes) return set_error(DE_E_INVALID, "null argument");
    const de_params &p = r->params;
    if (p.n < 1 || p.nelec != 2) return set_error(DE_E_INVALID, "request: N >= 1 and nelec = 2 required");
    if (r->nev < 1 || r->ns < 0 || r->gm.max_inner_iter < 0) return set_error(DE_E_INVALID, "request: bad solver sizes");
    const int64_t nn = 2 * p.n + 1, m = nn * nn * nn, d = m * m, w = 2 * nn - 1;
    const int64_t nev = r->nev, order = r->gm.max_inner_iter;
    // X (staging) AX W AW P AP, S AS
    int64_t vec16 = 6 * nev + 2 * (int64_t)r->ns * nev;
    // inner-solve Krylov blocks LV LQ: complex64 in the mixed form
    int64_t inner_bytes = 2 * order * nev * d * ((p.precision == DE_PREC_MIXED && order > 1) ? 8 : 16);
    // the GMRES inner solve (usepetscflag = 0) keeps its own basis: restart + 4 vectors
    if (r->gm.usepetscflag == 0 && order > 1) inner_bytes = (std::min<int64_t>(order, 30) + 4) * d * 16;
    const int64_t work = (1 + std::max<int64_t>(296LL * 64 * 128, 296LL * 32)) * 16;
    const int64_t tables = m * 12 + w * w * w * 12 + 64 * 256 * 16 + 64 * 128 * 16 * 2;
    *bytes = vec16 * d * 16 + inner_bytes + work + tables + (8LL << 20);
    return DE_OK;
}

DE_API int de_server_create(const de_server_opts *o, void **server)
{
    if (!o || !server) return set_error(DE_E_INVALID, "null argument");
    *server = nullptr;
    if (o->workers < 1 || o->workers > 64) return set_error(DE_E_INVALID, "workers must be in 1..64");
    if (o->max_bytes < 0) return set_error(DE_E_INVALID, "max_bytes must be >= 0");
    DE_CUDA(cudaSetDevice(o->device));
    auto s = std::make_unique<de_server_impl>();
    s->opts = *o;
    if (s->opts.max_bytes == 0) {
        size_t fr = 0, tot = 0;
        DE_CUDA(cudaMemGetInfo(&fr, &tot));
        s->opts.max_bytes = (int64_t)(0.9 * (double)fr);
    }
    s->t0 = clk::now();
    for (int w = 0; w < o->workers; ++w) s->workers.emplace_back([p = s.get(), w] { p->worker_main(w); });
    *server = s.release();
    return DE_OK;
}

DE_API int de_server_submit(void *server, const de_request *r, uint64_t *id)
{
    auto *s = static_cast<de_server_impl *>(server);
    if (!s || !r) return set_error(DE_E_INVALID, "null argument");
    if (!r->x || !r->e) return set_error(DE_E_INVALID, "request: null x or e");
    if ((3 + r->ns) * r->nev > 64 || r->nev > 16) return set_error(DE_E_INVALID, "request: (3+NS)*NEV exceeds 64");
    int64_t fp = 0;
    DE_TRY(de_request_footprint(r, &fp));
    if (fp > s->opts.max_bytes)
        return set_error(DE_E_BUSY, "request needs %lld device bytes, more than the server's %lld", (long long)fp,
                         (long long)s->opts.max_bytes);
    auto j = std::make_unique<Job>();
    j->req = *r;
    j->footprint = fp;
    std::memset(&j->res, 0, sizeof j->res);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return set_error(DE_E_INVALID, "server is shutting down");
        j->id = s->next_id++;
        j->res.id = j->id;
        j->res.footprint_bytes = fp;
        j->res.t_submit_s = s->now();
        if (id) *id = j->id;
        s->queue.push_back(j.get());
        s->jobs[j->id] = std::move(j);
    }
    s->cv_work.notify_all();
    return DE_OK;
}

static int collect(de_server_impl *s, Job *j, de_result *out)
{
    if (out) *out = j->res;
    j->collected = true;
    s->finished.remove(j);
    s->jobs.erase(j->id);
    return DE_OK;
}

DE_API int de_server_wait(void *server, uint64_t id, double timeout_s, de_result *out)
{
    auto *s = static_cast<de_server_impl *>(server);
    if (!s) return set_error(DE_E_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return set_error(DE_E_INVALID, "unknown or already collected request %llu", (unsigned long long)id);
    Job *j = it->second.get();
    auto ready = [&] { return j->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return set_error(DE_E_BUSY, "request %llu still running", (unsigned long long)id);
    }
    return collect(s, j, out);
}

DE_API int de_server_wait_any(void *server, double timeout_s, de_result *out)
{
    auto *s = static_cast<de_server_impl *>(server);
    if (!s) return set_error(DE_E_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return !s->finished.empty(); };
    if (timeout_s < 0) {
        if (s->jobs.empty()) return set_error(DE_E_INVALID, "no requests outstanding");
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return set_error(DE_E_BUSY, "no request finished within %.3f s", timeout_s);
    }
    return collect(s, s->finished.front(), out);
}

DE_API double de_server_now(void *server)
{
    auto *s = static_cast<de_server_impl *>(server);
    return s ? s->now() : 0.0;
}

DE_API int de_server_load(void *server, int *queued, int *running, int64_t *bytes_reserved)
{
    auto *s = static_cast<de_server_impl *>(server);
    if (!s) return set_error(DE_E_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = (int)s->queue.size();
    if (running) *running = s->running;
    if (bytes_reserved) *bytes_reserved = s->reserved;
    return DE_OK;
}

DE_API int de_server_destroy(void *server)
{
    auto *s = static_cast<de_server_impl *>(server);
    if (!s) return DE_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->queue.clear();
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    delete s;
    return DE_OK;
}

}  // extern "C"
