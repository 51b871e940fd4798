// Serving loop: jobs (boxes + step counts) are admitted while their device footprint fits
// the HBM budget and stay resident until done.  Between chunks of steps the resident jobs with
// the least remaining work (particles x steps left) are picked, up to a particle cap, and stepped
// together by the batched graph (continuous batching, shortest remaining work first): a GPU step
// over that many particles already runs at full throughput, and a short job that arrives behind
// long ones finishes in its own time instead of theirs.  The others wait on the device.
// One driver thread issues all device work; submit/poll/cancel/preempt only touch the queue.
// A preempted job leaves with its x, v (tag order) and step count kept on the host: its
// checkpoint, from which a resubmitted box (start_step) continues the run.
//
// The reference's only form of many simulations is one LAMMPS instance per MPI rank
// group (main_ensemble, src/main.cpp:49-117); here they share one GPU and one launch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "../../include/mdpd.h"
#include "engine.h"
#include "script.h"

namespace mdpd {
void spec_from_box(const mdpd_box_spec &bs, Spec &s, Fill &fill);
}

using namespace mdpd;

namespace {

struct Job {
    int64_t id = 0;
    mdpd_job_spec spec{};
    std::vector<double> x0, v0;  // copies of caller-provided initial state
    int state = 0, error = 0;
    int64_t done = 0;
    double submit_s = 0, start_s = 0, end_s = 0;
    std::vector<float> step_ms;
    mdpd_thermo_t thermo{};
    std::vector<double> xf, vf;
    std::unique_ptr<Box> box;
    size_t bytes = 0;
    // set by the API threads, read by the driver thread between chunks
    std::atomic<bool> cancel{false};
    std::atomic<bool> preempt{false};
    bool set_up = false;  // its setup (rebuild, density and force passes) has run
    double remaining() const { return (double)spec.box.n * (double)(spec.nsteps - done); }
};

double pct(std::vector<float> v, double p)
{
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const size_t k = std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5));
    return v[k];
}

}  // namespace

struct mdpd_server_s {
    uint64_t budget = 0;
    int device = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::map<int64_t, std::shared_ptr<Job>> jobs;
    std::deque<int64_t> queue;
    int64_t next_id = 1;
    bool stop = false;
    std::thread th;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    // stats
    double particle_steps = 0, busy_s = 0;
    // host wall seconds of the loop's parts: box creation, batch formation (units and captured
    // graphs), setup of new boxes, stepping chunks (device time of the chunks is busy_s)
    double t_create = 0, t_form = 0, t_setup = 0, t_chunks = 0, t_wait = 0, t_retire = 0;
    int64_t n_forms = 0;
    std::vector<float> all_step_ms;
    std::vector<double> job_latency_s;
    uint64_t resident = 0, peak_resident = 0;
    int chunk = 50;
    // particles stepped together (0: every resident job); see mdpd_server_set_step_particles
    int64_t step_cap = 8ll << 20;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void loop();
    // a job leaves the device: result, checkpoint (kept x, v) and latency recorded, box freed
    void retire(Job &j, const Thermo &t, int error, bool finished);
    // active minus `gone`
    static void drop(std::vector<std::shared_ptr<Job>> &active, const std::vector<std::shared_ptr<Job>> &gone)
    {
        std::vector<std::shared_ptr<Job>> keep;
        for (auto &j : active)
            if (std::find(gone.begin(), gone.end(), j) == gone.end()) keep.push_back(j);
        active.swap(keep);
    }
};

void mdpd_server_s::retire(Job &j, const Thermo &t, int error, bool finished)
{
    const bool fail = error != 0;
    const bool preempted = j.preempt && !finished && !fail && !j.cancel;
    mdpd_thermo_t out{};
    out.step = t.step;
    out.natoms = t.n;
    out.nbuild = t.nbuild;
    out.temp = t.temp;
    out.press = t.press;
    out.ke = 0.5 * t.ke_all;
    for (int d = 0; d < 3; ++d) out.momentum[d] = t.mom[d];
    for (int d = 0; d < 6; ++d) out.ptensor[d] = t.ptensor[d];
    out.pe = t.pe;
    out.surface_tension = t.surface_tension;
    out.status = t.status;
    std::vector<double> xf, vf;
    if ((j.spec.keep_state || preempted) && !fail) {
        const int n = j.box->n;
        xf.resize(3 * (size_t)n);
        vf.resize(3 * (size_t)n);
        j.box->download_by_tag(xf.data(), vf.data());
    }
    // the device memory goes back to the pool before the job is reported done, outside the lock
    // (pollers and submitters are not held up by it)
    j.box.reset();
    std::lock_guard<std::mutex> lk(mu);
    j.thermo = out;
    j.xf.swap(xf);
    j.vf.swap(vf);
    j.state = fail ? 3 : j.cancel ? 4 : preempted ? 5 : 2;
    if (fail) j.error = error;
    j.end_s = now();
    if (!preempted && !j.cancel) job_latency_s.push_back(j.end_s - j.submit_s);  // a preempted job goes on elsewhere
    resident -= j.bytes;
    cv.notify_all();
}

// the kernels of a batch are chosen per batch (pair style, RNG mode): jobs step together only
// when they share both
static bool same_family(const Job &a, const Job &b)
{
    return a.spec.box.style == b.spec.box.style && (a.spec.box.exact_rng != 0) == (b.spec.box.exact_rng != 0);
}

void mdpd_server_s::loop()
{
    cudaSetDevice(device);
    std::vector<std::shared_ptr<Job>> active;    // resident jobs
    std::vector<std::shared_ptr<Job>> stepping;  // the jobs of `batch`, in id order
    std::unique_ptr<Batch> batch;
    StepConfig cfg;
    cfg.sms = sm_count();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (;;) {
        std::vector<std::shared_ptr<Job>> admitted;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty()) {
                const double tw0 = now();
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                t_wait += now() - tw0;
            }
            if (stop) break;
            // admission: FIFO while the next job fits the budget
            while (!queue.empty()) {
                std::shared_ptr<Job> j = jobs[queue.front()];
                if (j->cancel) {
                    j->state = 4;
                    queue.pop_front();
                    continue;
                }
                if (j->preempt) {  // never started: its checkpoint is what it was submitted with
                    j->state = 5;
                    j->thermo.step = j->spec.box.start_step;
                    j->xf = j->x0;
                    j->vf = j->v0.empty() && !j->x0.empty() ? std::vector<double>(j->x0.size(), 0.0) : j->v0;
                    j->end_s = now();
                    queue.pop_front();
                    continue;
                }
                if (resident + j->bytes > budget) break;
                // another pass family waits, in order, until the resident jobs have ended
                const Job *ref = !active.empty() ? active[0].get() : !admitted.empty() ? admitted[0].get() : nullptr;
                if (ref && !same_family(*j, *ref)) break;
                queue.pop_front();
                resident += j->bytes;
                admitted.push_back(j);
            }
        }
        // allocate admitted boxes (outside the lock)
        const double tc0 = now();
        for (auto &j : admitted) {
            try {
                Spec s;
                Fill fill;
                mdpd_box_spec bs = j->spec.box;
                if (!j->x0.empty()) {
                    bs.x = j->x0.data();
                    bs.v = j->v0.empty() ? nullptr : j->v0.data();
                }
                spec_from_box(bs, s, fill);
                if (bs.x)
                    j->box.reset(new Box(s, bs.n, bs.x, bs.v, nullptr, nullptr, nullptr, cfg.sms));
                else
                    j->box.reset(new Box(s, bs.n, fill, cfg.sms));
                std::lock_guard<std::mutex> lk(mu);
                j->state = 1;
                j->start_s = now();
                active.push_back(j);
            } catch (const std::exception &e) {
                std::lock_guard<std::mutex> lk(mu);
                j->state = 3;
                j->error = std::string(e.what()).rfind("OOM", 0) == 0 ? MDPD_ERR_OOM : MDPD_ERR_ARG;
                j->end_s = now();
                resident -= j->bytes;
            }
        }
        t_create += now() - tc0;
        peak_resident = std::max(peak_resident, resident);
        if (active.empty()) continue;
        // jobs cancelled or preempted while they wait leave at the step they reached
        std::vector<std::shared_ptr<Job>> leaving;
        for (auto &j : active)
            if ((j->cancel || j->preempt) &&
                std::find(stepping.begin(), stepping.end(), j) == stepping.end())
                leaving.push_back(j);
        if (!leaving.empty()) {
            std::vector<Box *> raw;
            for (auto &j : leaving)
                if (j->set_up) raw.push_back(j->box.get());
            std::vector<Thermo> th;
            if (!raw.empty()) {
                try {
                    Batch tb(raw, cfg);  // a batch over the leaving boxes that have stepped, for their thermo only
                    tb.thermo(th);
                } catch (const std::exception &) {
                    th.assign(raw.size(), Thermo{});
                }
            }
            size_t q = 0;
            for (auto &j : leaving) {
                Thermo t{};
                if (j->set_up) t = th[q++];
                else {  // never stepped: the state it was admitted with
                    t.step = j->spec.box.start_step;
                    t.n = j->spec.box.n;
                }
                retire(*j, t, 0, false);
            }
            drop(active, leaving);
        }
        if (active.empty()) continue;
        // the stepping set: least remaining work first, up to step_cap particles (at least one job).
        // It is picked again when it has lost a job, when a waiting job fits beside it, or when a
        // waiting job has less than half the remaining work of the longest stepping one; otherwise
        // it keeps stepping as it is (each new set costs a batch and its captured graphs)
        int64_t cap;
        {
            std::lock_guard<std::mutex> lk(mu);
            cap = step_cap;
        }
        bool repick = !batch || stepping.empty();
        if (!repick) {
            int64_t np = 0;
            double longest = 0;
            for (auto &j : stepping) {
                np += j->spec.box.n;
                longest = std::max(longest, j->remaining());
            }
            for (auto &j : active) {
                if (std::find(stepping.begin(), stepping.end(), j) != stepping.end()) continue;
                if (cap <= 0 || np + j->spec.box.n <= cap || j->remaining() < 0.5 * longest) {
                    repick = true;
                    break;
                }
            }
        }
        std::vector<std::shared_ptr<Job>> want = stepping;
        if (repick) {
            want.clear();
            std::vector<std::shared_ptr<Job>> order(active);
            std::sort(order.begin(), order.end(), [](const std::shared_ptr<Job> &a, const std::shared_ptr<Job> &b) {
                const double ra = a->remaining(), rb = b->remaining();
                return ra < rb || (ra == rb && a->id < b->id);
            });
            int64_t np = 0;
            for (auto &j : order) {
                if (!want.empty() && cap > 0 && np + j->spec.box.n > cap) continue;
                want.push_back(j);
                np += j->spec.box.n;
            }
            std::sort(want.begin(), want.end(),
                      [](const std::shared_ptr<Job> &a, const std::shared_ptr<Job> &b) { return a->id < b->id; });
        }
        if (!batch || want != stepping) {
            batch.reset();
            stepping = want;
            std::vector<Box *> raw;
            std::vector<int> fresh;
            for (size_t k = 0; k < stepping.size(); ++k) {
                raw.push_back(stepping[k]->box.get());
                if (!stepping[k]->set_up) fresh.push_back((int)k);
            }
            cfg.style = stepping[0]->spec.box.style;
            cfg.exact_rng = stepping[0]->spec.box.exact_rng != 0;
            try {
                const double tf0 = now();
                batch.reset(new Batch(raw, cfg));
                const double tf1 = now();
                batch->setup_boxes(fresh);
                for (int k : fresh) stepping[k]->set_up = true;
                t_form += tf1 - tf0;
                t_setup += now() - tf1;
                ++n_forms;
            } catch (const std::exception &e) {
                std::lock_guard<std::mutex> lk(mu);
                for (auto &j : active) {
                    j->state = 3;
                    j->error = MDPD_ERR_CUDA;
                    j->end_s = now();
                    j->box.reset();
                }
                active.clear();
                stepping.clear();
                batch.reset();
                resident = 0;
                continue;
            }
        }
        // run a chunk: until the first stepping job finishes, at most `chunk` steps
        int64_t k = chunk;
        for (auto &j : stepping) k = std::min<int64_t>(k, j->spec.nsteps - j->done);
        k = std::max<int64_t>(k, 1);
        Range chunk_range("mdpd::server_chunk");
        const double tk0 = now();
        cudaEventRecord(e0, batch->stream());
        batch->run(k, false, true);  // a retiring job's thermo reports its last step's energy and virial
        cudaEventRecord(e1, batch->stream());
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        long long nparts = 0;
        for (auto &j : stepping) nparts += j->box->n;
        t_chunks += now() - tk0;
        {
            std::lock_guard<std::mutex> lk(mu);
            particle_steps += (double)nparts * k;
            busy_s += ms * 1e-3;
            for (int64_t q = 0; q < k; ++q) all_step_ms.push_back(ms / k);
        }
        // retire finished / failed / cancelled / preempted stepping jobs
        const double tr0 = now();
        std::vector<std::shared_ptr<Job>> out;
        std::vector<Thermo> th;
        std::vector<BoxState> states;
        batch->read_states(states);  // every stepping box's scalars: one gather, one copy
        for (size_t q = 0; q < stepping.size(); ++q) {
            auto &j = stepping[q];
            const BoxState &bst = states[q];
            j->done += k;
            for (int64_t s = 0; s < k; ++s) j->step_ms.push_back(ms / k);
            const bool fail = bst.status != 0;
            const bool finished = j->done >= j->spec.nsteps;
            if (finished || fail || j->cancel || j->preempt) {
                if (th.empty()) batch->thermo(th);
                retire(*j, th[q], !fail ? 0 : (bst.status & kErrNonFinite) ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW,
                       finished);
                out.push_back(j);
            }
        }
        if (!out.empty()) {
            batch.reset();
            stepping.clear();
            drop(active, out);
        }
        t_retire += now() - tr0;
    }
    batch.reset();
    for (auto &j : active) j->box.reset();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

extern "C" {

int mdpd_box_bytes(const mdpd_box_spec *spec, uint64_t *bytes)
{
    if (!spec || !bytes || spec->n <= 0) return MDPD_ERR_ARG;
    try {
        Spec sp;
        Fill fill;
        mdpd_box_spec bs = *spec;
        bs.x = nullptr, bs.v = nullptr;
        bs.n = 1;
        spec_from_box(bs, sp, fill);
        *bytes = Box::estimate_bytes(sp, spec->n);
    } catch (const std::exception &) {
        return MDPD_ERR_ARG;
    }
    return MDPD_OK;
}

int mdpd_server_start(mdpd_server_t **out, uint64_t budget, const mdpd_opts *opts)
{
    if (!out || budget == 0) return MDPD_ERR_ARG;
    auto *s = new mdpd_server_s;
    s->budget = budget;
    s->device = opts ? opts->device : 0;
    // the budget's device memory is mapped into the box pool now, so an admission does not pay
    // for mapping fresh pages (the pool keeps it for the process's later boxes too)
    if (cudaSetDevice(s->device) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return MDPD_ERR_CUDA;
    }
    try {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
            reserve_box_pool((size_t)std::min<uint64_t>(budget, free_b > (2ull << 30) ? free_b - (2ull << 30) : 0));
    } catch (const std::exception &) {
        cudaGetLastError();
    }
    s->th = std::thread([s] { s->loop(); });
    *out = s;
    return MDPD_OK;
}

int mdpd_server_submit(mdpd_server_t *s, const mdpd_job_spec *job, int64_t *id)
{
    if (!s || !job || !id || job->nsteps <= 0 || job->box.n <= 0) return MDPD_ERR_ARG;
    auto j = std::make_shared<Job>();
    j->spec = *job;
    const int n = job->box.n;
    if (job->box.x) j->x0.assign(job->box.x, job->box.x + 3 * (size_t)n);
    if (job->box.v) j->v0.assign(job->box.v, job->box.v + 3 * (size_t)n);
    j->spec.box.x = nullptr;
    j->spec.box.v = nullptr;
    try {
        Spec sp;
        Fill fill;
        mdpd_box_spec bs = job->box;
        bs.x = nullptr, bs.v = nullptr;
        bs.n = 1;  // geometry/physics check only; the footprint uses the real n
        spec_from_box(bs, sp, fill);
        j->bytes = Box::estimate_bytes(sp, n);
    } catch (const std::exception &) {
        return MDPD_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (j->bytes > s->budget) return MDPD_ERR_BUDGET;
    j->id = s->next_id++;
    j->submit_s = s->now();
    s->jobs[j->id] = j;
    s->queue.push_back(j->id);
    *id = j->id;
    s->cv.notify_all();
    return MDPD_OK;
}

int mdpd_server_poll(mdpd_server_t *s, int64_t id, mdpd_job_result *out)
{
    if (!s || !out) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return MDPD_ERR_ARG;
    const Job &j = *it->second;
    std::memset(out, 0, sizeof(*out));
    out->state = j.state;
    out->error = j.error;
    out->steps_done = j.done;
    out->submit_s = j.submit_s;
    out->start_s = j.start_s;
    out->end_s = j.end_s;
    out->step_ms_p50 = pct(j.step_ms, 0.5);
    out->step_ms_p99 = pct(j.step_ms, 0.99);
    out->thermo = j.thermo;
    return MDPD_OK;
}

int mdpd_server_get_state(mdpd_server_t *s, int64_t id, double *x, double *v, int64_t n)
{
    if (!s) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return MDPD_ERR_ARG;
    const Job &j = *it->second;
    if ((j.state != 2 && j.state != 5) || j.xf.empty()) return MDPD_ERR_STATE;
    if ((int64_t)j.xf.size() != 3 * n) return MDPD_ERR_ARG;
    if (x) std::copy(j.xf.begin(), j.xf.end(), x);
    if (v) std::copy(j.vf.begin(), j.vf.end(), v);
    return MDPD_OK;
}

int mdpd_server_cancel(mdpd_server_t *s, int64_t id)
{
    if (!s) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return MDPD_ERR_ARG;
    it->second->cancel = true;
    s->cv.notify_all();
    return MDPD_OK;
}

int mdpd_server_preempt(mdpd_server_t *s, int64_t id)
{
    if (!s) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return MDPD_ERR_ARG;
    if (it->second->state >= 2) return MDPD_ERR_STATE;  // already ended
    it->second->preempt = true;
    s->cv.notify_all();
    return MDPD_OK;
}

int mdpd_server_drain(mdpd_server_t *s, double timeout_s)
{
    if (!s) return MDPD_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto pending = [&] {
        for (auto &kv : s->jobs)
            if (kv.second->state < 2) return true;
        return false;
    };
    if (timeout_s > 0) {
        if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return !pending(); }))
            return MDPD_ERR_TIMEOUT;
    } else
        s->cv.wait(lk, [&] { return !pending(); });
    return MDPD_OK;
}

int mdpd_server_set_step_particles(mdpd_server_t *s, int64_t n)
{
    if (!s || n < 0) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->step_cap = n;
    s->cv.notify_all();
    return MDPD_OK;
}

int mdpd_server_timing(mdpd_server_t *s, double *o)
{
    if (!s || !o) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    o[0] = s->t_create;
    o[1] = s->t_form;
    o[2] = s->t_setup;
    o[3] = s->t_chunks;
    o[4] = s->busy_s;
    o[5] = (double)s->n_forms;
    o[6] = s->t_wait;
    o[7] = s->t_retire;
    return MDPD_OK;
}

int mdpd_server_stats(mdpd_server_t *s, double *o)
{
    if (!s || !o) return MDPD_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    o[0] = s->busy_s > 0 ? s->particle_steps / s->busy_s : 0;
    o[1] = pct(s->all_step_ms, 0.5);
    o[2] = pct(s->all_step_ms, 0.99);
    std::vector<float> lat(s->job_latency_s.begin(), s->job_latency_s.end());
    o[3] = pct(lat, 0.5);
    o[4] = pct(lat, 0.99);
    o[5] = (double)s->job_latency_s.size();
    o[6] = (double)s->peak_resident;
    return MDPD_OK;
}

void mdpd_server_stop(mdpd_server_t *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    delete s;
}

}  // extern "C"
