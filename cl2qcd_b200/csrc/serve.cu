// serve.cu -- request loop for inversions on one GPU (continuous admission).
//
// A server owns N slots; each slot is a worker thread with its own context
// (and so its own CUDA stream).  Requests -- one gauge field, kappa, mu and
// 1..64 seeded sources on one lattice -- are queued by c2q_server_submit and
// admitted by the first free slot as soon as their HBM footprint fits the
// server's budget: requests that arrive while others run start at once when
// memory and a slot are free, and their kernels overlap on the device with the
// running ones (different streams).  Gauge fields are registered once, built
// in every storage the solvers read, and stay resident.  A request's sources
// are generated on the device and solved together by the multi-right-hand-
// side mixed-precision CG (c2q_cg_multi); the result reports the timestamps
// (submission, admission, completion) the latency statistics are made of.
//
// Admission: first fit in arrival order; once the oldest waiting request has
// waited longer than `fairness_s` seconds, nothing may overtake it, so large
// requests are not starved.  A request whose footprint exceeds the whole
// budget fails with C2Q_OOM without running.  A "heavy" request -- eo sites
// times sources at least `heavy_site_rhs`, enough slots for several waves of
// blocks on every SM -- saturates the GPU by itself: two of them side by side
// share SMs and L2 and finish later than one after the other, so at most
// `max_heavy` heavy requests run at a time, while light requests (launch- and
// latency-bound) are admitted beside them.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "c2q_host.h"

using namespace c2q;

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    long long ticket = 0;
    c2q_request req{};
    c2q_request_result res{};
    size_t footprint = 0;
    bool heavy       = false;
    bool done        = false;
};

struct GaugeEntry {
    c2q_gauge* g = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct c2q_server {
    int device = 0;
    int precision = 16;
    int rec12 = 1;
    size_t budget = 0;           // bytes for gauge fields + admitted requests
    size_t gauge_bytes = 0;      // resident gauge fields
    size_t reserved = 0;         // footprints of running requests
    double fairness_s = 2.0;
    long long heavy_site_rhs = 1LL << 19;  // eo sites x sources of a request that fills the GPU alone
    int max_heavy            = 1;          // heavy requests running at a time
    int running_heavy        = 0;
    Clock::time_point t0;
    c2q_ctx* loader = nullptr;   // builds the gauge fields
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Job>> queue;
    std::map<long long, std::shared_ptr<Job>> jobs;
    std::map<unsigned long long, GaugeEntry> gauges;
    std::vector<std::thread> workers;
    long long next_ticket = 1, completed = 0;
    int busy = 0;
    bool stop = false;
    std::string err;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// Device bytes a request holds while it runs: per source the FP64 solution and
// source, the FP32 residual and increment and four inner-precision fields, plus
// three FP64 fields per batch of up to 16 sources and the solver scratch.
size_t footprint_bytes(const c2q_lattice& lat, int nsrc, int precision)
{
    Geom g;
    if (!make_geom(lat, &g)) return 0;
    const size_t f64 = field_bytes(g, 64), f32 = field_bytes(g, 32), fin = field_bytes(g, precision);
    const size_t per_src = 2 * f64 + (precision == 64 ? 3 * f64 : 2 * f32 + 4 * fin);
    const size_t batch   = 3 * f64;
    return (size_t)nsrc * per_src + batch + (size_t)(4 << 20);
}

std::shared_ptr<Job> pick(c2q_server* s)
{
    const size_t avail = s->budget > s->gauge_bytes + s->reserved ? s->budget - s->gauge_bytes - s->reserved : 0;
    const double t     = s->now();
    for (size_t i = 0; i < s->queue.size(); ++i) {
        auto& j = s->queue[i];
        if (j->footprint <= avail && (!j->heavy || s->running_heavy < s->max_heavy)) {
            auto out = j;
            s->queue.erase(s->queue.begin() + (long)i);
            return out;
        }
        // the oldest request has waited long enough: nothing overtakes it
        if (i == 0 && t - j->res.t_submit > s->fairness_s) break;
    }
    return nullptr;
}

void run_job(c2q_server* s, c2q_ctx* ctx, Job& job)
{
    const c2q_request& r = job.req;
    c2q_request_result& out = job.res;
    GaugeEntry ge;
    {
        std::lock_guard<std::mutex> lk(s->m);
        auto it = s->gauges.find(r.gauge_id);
        if (it != s->gauges.end()) ge = it->second;
    }
    if (!ge.g) {
        out.status = C2Q_BAD_ARG;
        return;
    }
    const int n = r.nsrc;
    std::vector<c2q_spinor_eo*> x(n, nullptr), b(n, nullptr);
    std::vector<c2q_solve_report> reps(n);
    int rc = 0;
    for (int k = 0; k < n && !rc; ++k) {
        rc = c2q_spinor_eo_create(ctx, &r.lat, &x[k]);
        if (!rc) rc = c2q_spinor_eo_create(ctx, &r.lat, &b[k]);
        if (!rc) rc = c2q_spinor_eo_source(b[k], r.source_kind, r.source_seed + (unsigned long long)k);
    }
    if (!rc) {
        c2q_solver_params p = r.params;
        p.precision         = s->precision;
        p.use_rec12         = s->rec12;
        rc = c2q_cg_multi(x.data(), C2Q_OP_QPLUSQMINUS_EO, ge.g, b.data(), n, r.kappa, 2.0 * r.kappa * r.mu,
                          C2Q_ACTION_TWISTEDMASS, &p, reps.data());
    }
    double norm2 = 0;
    for (int k = 0; k < n && rc >= 0; ++k) {
        double q = 0;
        if (c2q_squarenorm(x[k], &q) == C2Q_OK) norm2 += q;
        if (r.solutions) {
            Geom g;
            make_geom(r.lat, &g);
            c2q_spinor_eo_download(x[k], r.solutions + (size_t)k * g.seo * 24);
        }
    }
    c2q_ctx_synchronize(ctx);
    int iters = 0;
    double worst = 0;
    for (int k = 0; k < n; ++k) {
        iters = std::max(iters, reps[k].iterations);
        worst = std::max(worst, reps[k].true_resid_rel);
    }
    for (int k = 0; k < n; ++k) {
        c2q_spinor_eo_destroy(x[k]);
        c2q_spinor_eo_destroy(b[k]);
    }
    c2q_ctx_synchronize(ctx);
    out.status             = rc;
    out.iterations_max     = iters;
    out.true_resid_rel_max = worst;
    out.solution_norm2     = norm2;
}

void worker_main(c2q_server* s)
{
    c2q_ctx* ctx = nullptr;
    const int rc = c2q_ctx_create(&ctx, s->device, nullptr);
    for (;;) {
        std::shared_ptr<Job> job;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return s->stop || (!s->queue.empty() && (job = pick(s)) != nullptr); });
            if (!job) break;  // stopping
            s->reserved += job->footprint;
            s->running_heavy += job->heavy ? 1 : 0;
            ++s->busy;
            job->res.t_admit = s->now();
        }
        if (rc)
            job->res.status = rc;
        else
            run_job(s, ctx, *job);
        {
            std::lock_guard<std::mutex> lk(s->m);
            job->res.t_done = s->now();
            job->done       = true;
            s->reserved -= job->footprint;
            s->running_heavy -= job->heavy ? 1 : 0;
            --s->busy;
            ++s->completed;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    if (ctx) c2q_ctx_destroy(ctx);
}

}  // namespace

extern "C" {

C2Q_EXPORT size_t c2q_request_footprint(const c2q_lattice* lat, int nsrc, int precision)
{
    if (!lat || nsrc < 1 || (precision != 64 && precision != 32 && precision != 16)) return 0;
    return footprint_bytes(*lat, nsrc, precision);
}

C2Q_EXPORT int c2q_server_create(c2q_server** out, int device, int slots, size_t hbm_budget, int precision,
                                 int rec12)
{
    if (!out || slots < 1 || slots > 64 || (precision != 32 && precision != 16)) return C2Q_BAD_ARG;
    *out = nullptr;
    c2q_ctx* loader = nullptr;
    int rc          = c2q_ctx_create(&loader, device, nullptr);
    if (rc) return rc;
    if (hbm_budget == 0) {  // 85% of what is free now
        size_t fr = 0, tot = 0;
        cudaSetDevice(device);
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            c2q_ctx_destroy(loader);
            return C2Q_CUDA_ERROR;
        }
        hbm_budget = (size_t)(0.85 * (double)fr);
    }
    c2q_server* s = new c2q_server();
    s->device     = device;
    s->precision  = precision;
    s->rec12      = rec12 ? 1 : 0;
    s->budget     = hbm_budget;
    s->t0         = Clock::now();
    s->loader     = loader;
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_main, s);
    *out = s;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_server_set_heavy_limit(c2q_server* s, long long heavy_site_rhs, int max_heavy)
{
    if (!s || heavy_site_rhs < 1 || max_heavy < 1) return C2Q_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->m);
    s->heavy_site_rhs = heavy_site_rhs;
    s->max_heavy      = max_heavy;
    s->cv_work.notify_all();
    return C2Q_OK;
}

C2Q_EXPORT int c2q_server_add_gauge(c2q_server* s, unsigned long long gauge_id, const c2q_lattice* lat,
                                    const double* aos)
{
    if (!s || !lat || !aos) return C2Q_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->gauges.count(gauge_id)) return C2Q_BAD_ARG;
    }
    c2q_gauge* g = nullptr;
    int rc       = c2q_gauge_create(s->loader, lat, &g);
    if (!rc) rc = c2q_gauge_upload(g, aos);
    // every storage the server's solvers read, built now so that the slots
    // only ever read the gauge object
    const int inner = gkind_for(s->precision, s->rec12);
    if (!rc) rc = gauge_ensure(g, inner);
    // the inner sweeps of the mixed-precision CG in the temporal gauge, built here
    // so that solves running side by side only read the gauge object
    if (!rc && gkind_tg(inner) >= 0 && tg_applicable(g->lat)) rc = gauge_ensure(g, gkind_tg(inner));
    if (!rc && s->rec12) rc = gauge_ensure(g, G64R12);
    // whether 12-real FP64 residuals are exact for this field, measured here
    // (once) rather than by the first solve that asks
    if (!rc && s->rec12) (void)rec12_exact(g);
    if (!rc) rc = c2q_ctx_synchronize(s->loader);
    if (rc) {
        if (g) c2q_gauge_destroy(g);
        return rc;
    }
    std::lock_guard<std::mutex> lk(s->m);
    GaugeEntry e{g, c2q_gauge_device_bytes(g)};
    s->gauges[gauge_id] = e;
    s->gauge_bytes += e.bytes;
    return C2Q_OK;
}

C2Q_EXPORT int c2q_server_submit(c2q_server* s, const c2q_request* req, long long* ticket)
{
    if (!s || !req || !ticket || req->nsrc < 1 || req->nsrc > 64) return C2Q_BAD_ARG;
    auto job       = std::make_shared<Job>();
    job->req       = *req;
    job->footprint = footprint_bytes(req->lat, req->nsrc, s->precision);
    {
        std::lock_guard<std::mutex> lk(s->m);
        job->ticket      = s->next_ticket++;
        job->res.nsrc    = req->nsrc;
        job->res.t_submit = s->now();
        job->res.footprint_bytes = (long long)job->footprint;
        {
            Geom g;
            job->heavy = make_geom(req->lat, &g) && (long long)g.seo * req->nsrc >= s->heavy_site_rhs;
        }
        auto it = s->gauges.find(req->gauge_id);
        const bool ok_gauge = it != s->gauges.end() && same_lattice(it->second.g->lat, req->lat);
        const bool fits     = s->gauge_bytes + job->footprint <= s->budget;
        s->jobs[job->ticket] = job;
        *ticket              = job->ticket;
        if (!ok_gauge || !fits) {  // fails without running
            job->res.status = ok_gauge ? C2Q_OOM : C2Q_BAD_ARG;
            job->res.t_admit = job->res.t_done = job->res.t_submit;
            job->done = true;
            ++s->completed;
        } else {
            s->queue.push_back(job);
        }
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    return C2Q_OK;
}

C2Q_EXPORT int c2q_server_wait(c2q_server* s, long long ticket, c2q_request_result* out)
{
    if (!s || !out) return C2Q_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return C2Q_BAD_ARG;
    auto job = it->second;
    s->cv_done.wait(lk, [&] { return job->done; });
    *out = job->res;
    s->jobs.erase(ticket);
    return C2Q_OK;
}

C2Q_EXPORT int c2q_server_get_stats(c2q_server* s, c2q_server_stats* out)
{
    if (!s || !out) return C2Q_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->m);
    out->budget_bytes   = (long long)s->budget;
    out->gauge_bytes    = (long long)s->gauge_bytes;
    out->reserved_bytes = (long long)s->reserved;
    out->queued         = (int)s->queue.size();
    out->running        = s->busy;
    out->slots          = (int)s->workers.size();
    out->completed      = s->completed;
    out->seconds        = s->now();
    return C2Q_OK;
}

// Stops after the running requests; queued ones are cancelled (C2Q_TIMEOUT).
C2Q_EXPORT int c2q_server_destroy(c2q_server* s)
{
    if (!s) return C2Q_OK;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
        for (auto& j : s->queue) {
            j->res.status = C2Q_TIMEOUT;
            j->done       = true;
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->gauges) c2q_gauge_destroy(kv.second.g);
    c2q_ctx_destroy(s->loader);
    delete s;
    return C2Q_OK;
}

}  // extern "C"
