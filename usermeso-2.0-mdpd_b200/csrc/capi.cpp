// extern "C" entry points of libmdpd.so (include/mdpd.h).  Exceptions never cross the
// boundary: each call maps them to an MDPD_* status and keeps the message for
// mdpd_last_error.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>

#include "../../include/mdpd.h"
#include "engine.h"
#include "jobs.h"
#include "script.h"
#include "tune_cache.h"

using namespace mdpd;

struct mdpd_s {
    std::unique_ptr<Script> script;
    std::string err;
    int verbose = 0;
};

struct mdpd_batch_s {
    std::vector<std::unique_ptr<Box>> boxes;
    std::unique_ptr<Batch> batch;
    std::string err;
    int device = 0;
    double *scratch = nullptr;  // device staging of state downloads, grown on demand
    size_t scratch_bytes = 0;
};

static thread_local std::string g_err;

static int code_of(const std::string &m)
{
    if (m.rfind("OOM", 0) == 0) return MDPD_ERR_OOM;
    if (m.rfind("ARG", 0) == 0) return MDPD_ERR_ARG;
    if (m.rfind("PARSE", 0) == 0) return MDPD_ERR_PARSE;
    if (m.rfind("CUDA", 0) == 0) return MDPD_ERR_CUDA;
    if (m.rfind("BUDGET", 0) == 0) return MDPD_ERR_BUDGET;
    return MDPD_ERR_STATE;
}

template <class F> static int guard(std::string &err, F &&f)
{
    try {
        f();
        err.clear();
        return MDPD_OK;
    } catch (const ScriptError &e) {
        err = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        err = "host allocation failed";
        return MDPD_ERR_OOM;
    } catch (const std::exception &e) {
        err = e.what();
        return code_of(err);
    }
}

static void fill_thermo(const Thermo &t, mdpd_thermo_t *o)
{
    std::memset(o, 0, sizeof(*o));
    o->step = t.step;
    o->natoms = t.n;
    o->nbuild = t.nbuild;
    o->temp = t.temp;
    o->press = t.press;
    o->pe = t.pe;
    o->ke = 0.5 * t.ke_all;
    for (int k = 0; k < 6; ++k) o->virial[k] = t.virial[k];
    for (int k = 0; k < 3; ++k) o->momentum[k] = t.mom[k];
    o->temp_group = t.n_group > 1 ? t.ke_group / (3.0 * t.n_group - 3.0) : 0.0;
    for (int k = 0; k < 6; ++k) o->ptensor[k] = t.ptensor[k];
    o->surface_tension = t.surface_tension;
    o->status = t.status;
}

extern "C" {

int mdpd_create(mdpd_t **h, const mdpd_opts *opts)
{
    if (!h) return MDPD_ERR_ARG;
    *h = nullptr;
    std::unique_ptr<mdpd_s> s(new mdpd_s);
    const int rc = guard(g_err, [&] { s->script.reset(new Script(opts ? opts->device : 0)); });
    if (rc) return rc;
    s->verbose = opts ? opts->verbose : 0;
    *h = s.release();
    return MDPD_OK;
}

int mdpd_command(mdpd_t *h, const char *line)
{
    if (!h || !line) return MDPD_ERR_ARG;
    return guard(h->err, [&] { h->script->command(line); });
}

int mdpd_file(mdpd_t *h, const char *path)
{
    if (!h || !path) return MDPD_ERR_ARG;
    return guard(h->err, [&] { h->script->file(path); });
}

int mdpd_run(mdpd_t *h, int64_t nsteps)
{
    if (!h || nsteps < 0) return MDPD_ERR_ARG;
    return guard(h->err, [&] { h->script->run(nsteps); });
}

int mdpd_setup(mdpd_t *h)
{
    if (!h) return MDPD_ERR_ARG;
    return guard(h->err, [&] { h->script->setup(); });
}

int mdpd_step(mdpd_t *h, int64_t nsteps)
{
    if (!h || nsteps < 0) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Batch *b = h->script->batch();
        if (!b || !h->script->box()) throw ScriptError(MDPD_ERR_STATE, "mdpd_step before mdpd_setup/mdpd_run");
        b->run(nsteps, true);
        std::string msg;
        if (int st = b->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_natoms(mdpd_t *h, int64_t *n)
{
    if (!h || !n) return MDPD_ERR_ARG;
    *n = (int64_t)h->script->particles().size();
    return MDPD_OK;
}

int mdpd_get_state(mdpd_t *h, double *x, double *v, int32_t *tag, int32_t *type, int64_t n)
{
    if (!h) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        h->script->sync_host();
        Particles &p = h->script->particles();
        if ((int64_t)p.size() != n) throw ScriptError(MDPD_ERR_ARG, "size mismatch");
        // parts_ is in tag order after setup; sort defensively
        std::vector<size_t> ord(p.size());
        for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
        std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return p.tag[a] < p.tag[b]; });
        for (size_t r = 0; r < ord.size(); ++r) {
            const size_t i = ord[r];
            for (int d = 0; d < 3; ++d) {
                if (x) x[3 * r + d] = p.x[3 * i + d];
                if (v) v[3 * r + d] = p.v[3 * i + d];
            }
            if (tag) tag[r] = p.tag[i];
            if (type) type[r] = p.type[i];
        }
    });
}

int mdpd_set_state(mdpd_t *h, const double *x, const double *v, int64_t n)
{
    if (!h) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        h->script->sync_host();
        Particles &p = h->script->particles();
        if ((int64_t)p.size() != n) throw ScriptError(MDPD_ERR_ARG, "size mismatch");
        for (size_t i = 0; i < p.size(); ++i) {
            const int64_t r = p.tag[i] - 1;
            if (r < 0 || r >= n) throw ScriptError(MDPD_ERR_ARG, "tags must be 1..n");
            for (int d = 0; d < 3; ++d) {
                if (x) p.x[3 * i + d] = x[3 * r + d];
                if (v) p.v[3 * i + d] = v[3 * r + d];
            }
        }
        h->script->invalidate();
    });
}

int mdpd_thermo(mdpd_t *h, mdpd_thermo_t *out)
{
    if (!h || !out) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Thermo t;
        h->script->thermo(t);
        fill_thermo(t, out);
    });
}

const char *mdpd_log(mdpd_t *h) { return h ? h->script->log.c_str() : ""; }
const char *mdpd_last_error(mdpd_t *h) { return h ? h->err.c_str() : g_err.c_str(); }

void mdpd_destroy(mdpd_t *h)
{
    if (!h) return;
    try {
        h->script.reset();
    } catch (...) {
    }
    delete h;
}

// --- internal arrays --------------------------------------------------------------------

static int64_t field_count(Box &b, const std::string &name)
{
    BoxState st = b.state();
    st.nghost = std::min(st.nghost, b.desc.ghost_cap);
    const int64_t n = b.n, na = (int64_t)b.n + st.nghost;
    if (name == "pos4" || name == "vel4") return 4 * na;
    if (name == "rho") return na;
    if (name == "force") return 4 * n;
    if (name == "count" || name == "tag" || name == "type" || name == "mask" || name == "phi") return n;
    if (name == "ghost_src" || name == "ghost_img") return st.nghost;
    if (name == "x" || name == "v") return 3 * n;
    if (name == "list") return (int64_t)b.desc.nrow * b.desc.n_col;
    throw ScriptError(MDPD_ERR_ARG, "unknown field " + name);
}

int mdpd_field_size(mdpd_t *h, const char *name, int64_t *count)
{
    if (!h || !name || !count) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Box *b = h->script->box();
        if (!b) throw ScriptError(MDPD_ERR_STATE, "no device state");
        *count = field_count(*b, name);
    });
}

int mdpd_get_field(mdpd_t *h, const char *name, void *out, int64_t nbytes)
{
    if (!h || !name || !out) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Box *b = h->script->box();
        if (!b) throw ScriptError(MDPD_ERR_STATE, "no device state");
        const std::string f = name;
        const int64_t cnt = field_count(*b, f);
        const BoxState st = b->state();
        const BoxDesc &B = b->desc;
        const int c = st.cur;
        auto get = [&](const void *src, size_t esz) {
            if ((int64_t)(cnt * esz) > nbytes) throw ScriptError(MDPD_ERR_ARG, "buffer too small");
            check_cuda(cudaMemcpy(out, src, cnt * esz, cudaMemcpyDeviceToHost), "get field");
        };
        if (f == "pos4") get(B.pos, 4);
        else if (f == "vel4") get(B.vel, 4);
        else if (f == "rho") get(B.rho, 4);
        else if (f == "force") {  // after post_force, as the reference: pair force + body force
            get(B.f[c], 4);
            if (B.body_bit) {
                std::vector<int> mask(cnt / 4);
                check_cuda(cudaMemcpy(mask.data(), B.mask[c], sizeof(int) * mask.size(), cudaMemcpyDeviceToHost),
                           "get field");
                float *fo = static_cast<float *>(out);
                for (size_t i = 0; i < mask.size(); ++i)
                    if (mask[i] & B.body_bit)
                        for (int d = 0; d < 3; ++d) fo[4 * i + d] = (float)((double)fo[4 * i + d] + B.body[d]);
            }
        }
        else if (f == "count") get(B.count, 4);
        else if (f == "tag") get(B.tag[c], 4);
        else if (f == "type") get(B.type[c], 4);
        else if (f == "mask") get(B.mask[c], 4);
        else if (f == "phi") get(B.phi[c], 4);
        else if (f == "ghost_src") get(B.gsrc, 4);
        else if (f == "ghost_img") get(B.gimg, 4);
        else if (f == "list") {  // indices only: the ownership flag of reduced rows is cleared
            get(B.table, 4);
            int32_t *o = static_cast<int32_t *>(out);
            for (size_t q = 0; q < cnt; ++q) o[q] &= kEntryIndexMask;
        }
        else if (f == "x" || f == "v") {
            if (cnt * 8 > nbytes) throw ScriptError(MDPD_ERR_ARG, "buffer too small");
            if (f == "x") b->download_state((double *)out, nullptr, nullptr, nullptr, nullptr, nullptr);
            else b->download_state(nullptr, (double *)out, nullptr, nullptr, nullptr, nullptr);
        }
    });
}

int mdpd_geometry(mdpd_t *h, double *o)
{
    if (!h || !o) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Box *b = h->script->box();
        if (!b) throw ScriptError(MDPD_ERR_STATE, "no device state");
        const BoxState st = b->state();
        const BoxDesc &B = b->desc;
        for (int d = 0; d < 3; ++d) {
            o[d] = B.lo[d];
            o[3 + d] = B.hi[d];
            o[6 + d] = B.cen[d];
            o[9 + d] = B.mbin[d];
        }
        o[12] = B.cutghost;
        o[13] = B.n_col;
        o[14] = st.nghost;
        // n_bulk and nbuild are readable through mdpd_thermo / fields
    });
}

int mdpd_get_pairs(mdpd_t *h, int32_t *ti, int32_t *tj, int64_t cap, int64_t *npairs)
{
    if (!h || !npairs) return MDPD_ERR_ARG;
    return guard(h->err, [&] {
        Box *b = h->script->box();
        if (!b) throw ScriptError(MDPD_ERR_STATE, "no device state");
        BoxState st = b->state();
        const BoxDesc &B = b->desc;
        st.nghost = std::min(st.nghost, B.ghost_cap);
        const int n = b->n, c = st.cur;
        std::vector<int> cnt(n), tag(n), gsrc(std::max(st.nghost, 1));
        std::vector<int> table((size_t)B.nrow * B.n_col);
        check_cuda(cudaMemcpy(cnt.data(), B.count, 4 * n, cudaMemcpyDeviceToHost), "pairs");
        check_cuda(cudaMemcpy(tag.data(), B.tag[c], 4 * n, cudaMemcpyDeviceToHost), "pairs");
        if (st.nghost) check_cuda(cudaMemcpy(gsrc.data(), B.gsrc, 4 * st.nghost, cudaMemcpyDeviceToHost), "pairs");
        check_cuda(cudaMemcpy(table.data(), B.table, 4 * table.size(), cudaMemcpyDeviceToHost), "pairs");
        int64_t np = 0;
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < cnt[i]; ++k) {
                const int j = table[(size_t)(i & ~31) * B.n_col + 32 * k + (i & 31)] & kEntryIndexMask;
                if (np < cap && ti && tj) {
                    ti[np] = tag[i];
                    tj[np] = j < n ? tag[j] : tag[gsrc[j - n]];
                }
                ++np;
            }
        *npairs = np;
    });
}

int mdpd_index_checks(void)
{
#ifdef MDPD_CHECK
    return 1;
#else
    return 0;
#endif
}

int mdpd_gaussian(const uint32_t *si, const uint32_t *sj, double *exact, float *fast, int64_t n)
{
    if (!si || !sj || n < 0) return MDPD_ERR_ARG;
    return guard(g_err, [&] {
        if (n == 0) return;
        uint32_t *d_i, *d_j;
        double *d_e = nullptr;
        float *d_f = nullptr;
        check_cuda(cudaMalloc(&d_i, 4 * n), "gaussian");
        check_cuda(cudaMalloc(&d_j, 4 * n), "gaussian");
        if (exact) check_cuda(cudaMalloc(&d_e, 8 * n), "gaussian");
        if (fast) check_cuda(cudaMalloc(&d_f, 4 * n), "gaussian");
        check_cuda(cudaMemcpy(d_i, si, 4 * n, cudaMemcpyHostToDevice), "gaussian");
        check_cuda(cudaMemcpy(d_j, sj, 4 * n, cudaMemcpyHostToDevice), "gaussian");
        launch_gaussian(0, d_i, d_j, d_e, d_f, (int)n);
        check_cuda(cudaGetLastError(), "gaussian launch");
        if (exact) check_cuda(cudaMemcpy(exact, d_e, 8 * n, cudaMemcpyDeviceToHost), "gaussian");
        if (fast) check_cuda(cudaMemcpy(fast, d_f, 4 * n, cudaMemcpyDeviceToHost), "gaussian");
        cudaFree(d_i);
        cudaFree(d_j);
        cudaFree(d_e);
        cudaFree(d_f);
    });
}

// --- batch ------------------------------------------------------------------------------

}  // extern "C"

namespace mdpd {

// synthetic box of a mdpd_box_spec: the physics and, if x is NULL, the seeded device fill (uniform
// positions in the fill region, Maxwell velocities at kT with zero net momentum)
void spec_from_box(const mdpd_box_spec &bs, Spec &s, Fill &fill)
{
    if (bs.n <= 0) throw std::runtime_error("ARG: box spec with n <= 0");
    s = Spec();
    s.style = bs.style;
    s.ntype = 1;
    for (int d = 0; d < 3; ++d) s.lo[d] = bs.lo[d], s.hi[d] = bs.hi[d];
    s.skin = bs.skin > 0 ? bs.skin : 0.3;
    s.every = bs.every > 0 ? bs.every : 1;
    s.delay = bs.delay;
    s.check = bs.check;
    s.dt = bs.dt > 0 ? bs.dt : 0.01;
    s.kT = bs.kT;
    s.seed = bs.seed;
    s.rho_est = bs.rho_est;
    s.mass[0] = bs.mass > 0 ? bs.mass : 1.0;
    s.cut_rho = bs.cut_rho > 0 ? bs.cut_rho : 0.75;
    s.exact_rng = bs.exact_rng;
    if (bs.start_step < 0) throw std::runtime_error("ARG: box spec with start_step < 0");
    s.step0 = bs.start_step;
    PairParam q;
    q.set = 1;
    q.A = bs.A, q.B = bs.B, q.gamma = bs.gamma, q.cut = bs.cut > 0 ? bs.cut : 1.0;
    q.cut_r = bs.cut_r > 0 ? bs.cut_r : 0.75;
    q.sigma = bs.sigma;
    q.expw = 1.0;
    if (q.cut < q.cut_r) throw std::runtime_error("PARSE: cutA should be larger than cutB.");
    s.pair[0][0] = q;
    for (int d = 0; d < 3; ++d) {
        const bool sub = bs.fill_hi[d] > bs.fill_lo[d];
        fill.lo[d] = sub ? std::max(bs.fill_lo[d], bs.lo[d]) : bs.lo[d];
        fill.hi[d] = sub ? std::min(bs.fill_hi[d], bs.hi[d]) : bs.hi[d];
    }
    fill.seed = bs.init_seed;
    fill.vscale = std::sqrt(bs.kT / s.mass[0]);
}

}  // namespace mdpd

extern "C" {

int mdpd_batch_create(mdpd_batch_t **out, const mdpd_box_spec *specs, int32_t nbox, const mdpd_opts *opts)
{
    if (!out || !specs || nbox <= 0) return MDPD_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<mdpd_batch_s> b(new mdpd_batch_s);
    const int rc = guard(g_err, [&] {
        b->device = opts ? opts->device : 0;
        check_cuda(cudaSetDevice(b->device), "set device");
        StepConfig cfg;
        cfg.sms = sm_count();
        cfg.style = specs[0].style;
        cfg.exact_rng = specs[0].exact_rng;
        std::vector<Box *> raw;
        try {
            for (int k = 0; k < nbox; ++k) {
                if (specs[k].style != cfg.style) throw std::runtime_error("ARG: a batch holds boxes of one pair style");
                if ((specs[k].exact_rng != 0) != (cfg.exact_rng != 0))
                    throw std::runtime_error("ARG: a batch holds boxes of one RNG mode (exact_rng)");
                Spec s;
                Fill fill;
                spec_from_box(specs[k], s, fill);
                if (specs[k].x)  // the caller's arrays go to the device directly, the copies queued
                    b->boxes.emplace_back(
                        new Box(s, specs[k].n, specs[k].x, specs[k].v, nullptr, nullptr, nullptr, cfg.sms, false));
                else
                    b->boxes.emplace_back(new Box(s, specs[k].n, fill, cfg.sms, false));
                raw.push_back(b->boxes.back().get());
            }
        } catch (...) {
            cudaDeviceSynchronize();  // no queued copy reads the caller's arrays after the call
            throw;
        }
        check_cuda(cudaStreamSynchronize(0), "upload");  // the caller's x, v are read by now
        b->batch.reset(new Batch(raw, cfg));
        // staging for state downloads, sized once for the largest box
        int nmax = 0;
        for (Box *x : raw) nmax = std::max(nmax, x->n);
        b->scratch_bytes = sizeof(double) * 6 * (size_t)nmax;
        check_cuda(cudaMalloc(&b->scratch, b->scratch_bytes), "download scratch");
    });
    if (rc) return rc;
    *out = b.release();
    return MDPD_OK;
}

int mdpd_batch_setup(mdpd_batch_t *b)
{
    if (!b) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        b->batch->setup();
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_batch_step(mdpd_batch_t *b, int64_t nsteps)
{
    if (!b || nsteps < 0) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        b->batch->run(nsteps, true, true);
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_batch_run_thermo(mdpd_batch_t *b, int64_t nsteps, mdpd_thermo_t *out, int64_t *d2h_bytes_per_step)
{
    if (!b || nsteps < 0 || (nsteps > 0 && !out)) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        const size_t nb = b->boxes.size();
        int bad = 0;
        b->batch->run_thermo(nsteps, [&](long long k, const std::vector<Thermo> &t) {
            for (size_t q = 0; q < nb; ++q) {
                fill_thermo(t[q], out + (size_t)k * nb + q);
                bad |= t[q].status;
            }
        });
        if (d2h_bytes_per_step) *d2h_bytes_per_step = (int64_t)b->batch->thermo_bytes_per_step();
        if (bad) throw ScriptError(bad & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, status_text(bad));
    });
}

int mdpd_batch_thermo(mdpd_batch_t *b, int32_t box, mdpd_thermo_t *out)
{
    if (!b || !out || box < 0 || box >= (int)b->boxes.size()) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        std::vector<Thermo> t;
        b->batch->thermo(t);
        fill_thermo(t[box], out);
    });
}

int mdpd_batch_thermo_all(mdpd_batch_t *b, mdpd_thermo_t *out, int32_t nbox)
{
    if (!b || !out || nbox != (int32_t)b->boxes.size()) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        std::vector<Thermo> t;
        b->batch->thermo(t);
        for (int k = 0; k < nbox; ++k) fill_thermo(t[k], out + k);
    });
}

int mdpd_batch_get_state(mdpd_batch_t *b, int32_t box, double *x, double *v, int64_t n)
{
    if (!b || box < 0 || box >= (int)b->boxes.size()) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        Box &bx = *b->boxes[box];
        if (n != bx.n) throw ScriptError(MDPD_ERR_ARG, "size mismatch");
        check_cuda(cudaSetDevice(b->device), "set device");  // the gather runs on the batch's device
        const size_t need = sizeof(double) * 6 * (size_t)n;
        if (b->scratch_bytes < need) {
            cudaFree(b->scratch);
            b->scratch = nullptr;
            b->scratch_bytes = 0;
            check_cuda(cudaMalloc(&b->scratch, need), "download scratch");
            b->scratch_bytes = need;
        }
        bx.download_by_tag(x, v, b->scratch);
    });
}

int mdpd_batch_get_states(mdpd_batch_t *b, double *const *x, double *const *v, int32_t nbox)
{
    if (!b || !x || !v || nbox != (int)b->boxes.size()) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        check_cuda(cudaSetDevice(b->device), "set device");
        b->batch->download_all(x, v);
    });
}

int mdpd_batch_time(mdpd_batch_t *b, int64_t nsteps, double *ms)
{
    if (!b || !ms || nsteps <= 0) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "event");
        check_cuda(cudaEventCreate(&e1), "event");
        cudaStream_t s = b->batch->stream();
        check_cuda(cudaEventRecord(e0, s), "event");
        b->batch->run(nsteps, false);
        check_cuda(cudaEventRecord(e1, s), "event");
        check_cuda(cudaEventSynchronize(e1), "event");
        float t = 0;
        check_cuda(cudaEventElapsedTime(&t, e0, e1), "event");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = t / nsteps;
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

// candidate shapes of the pair passes for the batch's pass family
static std::vector<StepConfig> tune_candidates(const StepConfig &base)
{
    std::vector<StepConfig> cands;
    if (base.half) {  // pair-once passes: the density pass's gathers in flight, the force
                      // pass's entries staged in shared memory or read from the table
        for (int g : {4, 6, 8})
            for (int st : {1, 0}) {
                StepConfig c = base;
                c.gather = g;
                c.stage_rows = st;
                cands.push_back(c);
            }
    } else {  // full-list passes: threads per particle of each pass
        for (int td : {1, 2, 4})
            for (int tf : {1, 2, 4}) {
                StepConfig c = base;
                c.tpp_density = td;
                c.tpp_force = tf;
                cands.push_back(c);
            }
    }
    return cands;
}

static TunePick pick_of(const StepConfig &c, double ms)
{
    TunePick p;
    p.density = c.half ? c.gather : c.tpp_density;
    p.force = c.half ? (c.stage_rows ? 32 : 0) : c.tpp_force;
    p.ms_per_step = ms;
    return p;
}

// time every candidate's pair passes on the batch's current state (one untimed and five timed
// evaluations; the same work for every candidate, and the boxes do not advance) and keep the
// fastest; the pick's ms is its pair passes' time per evaluation
static TunePick tune_by_timing(mdpd_batch_s *b)
{
    const StepConfig base = b->batch->cfg;
    double best = 1e30;
    StepConfig pick = base;
    for (const StepConfig &c : tune_candidates(base)) {
        b->batch->reconfigure(c);
        const double t = b->batch->time_pair_passes(5);
        if (t < best) best = t, pick = c;
    }
    b->batch->reconfigure(pick);
    return pick_of(pick, best);
}

// the workload class a stored pick applies to: GPU model and SM count, the pass family and
// its options, mean density (0.25 steps), neighbour cutoff (0.05 steps), total particles and
// box count (powers of two)
static std::string tune_key(mdpd_batch_s *b)
{
    const Batch &bt = *b->batch;
    const StepConfig &c = bt.cfg;
    cudaDeviceProp prop{};
    check_cuda(cudaGetDeviceProperties(&prop, b->device), "device properties");
    long long ntot = 0;
    double vol = 0.0, rc = 0.0;
    for (Box *x : bt.boxes()) {
        ntot += x->n;
        vol += x->desc.prd[0] * x->desc.prd[1] * x->desc.prd[2];
        rc = std::max(rc, x->desc.cutghost);
    }
    std::string fam = c.half ? "mdpd pair-once" : c.style ? "dpd full-list" : "mdpd full-list";
    if (c.wall_coupling) fam += " +wall-coupling";
    if (c.wall) fam += " +bounce-back";
    if (c.aboundary) fam += " +aboundary";
    if (c.exact_rng) fam += " +exact-rng";
    if (!c.uniform_types) fam += " +types";
    const int nb = (int)bt.boxes().size();
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s sm%d | %s | rho %.2f | rc %.2f | particles 2^%d | boxes 2^%d", prop.name,
                  prop.multiProcessorCount, fam.c_str(), std::round(4.0 * ntot / std::max(vol, 1e-300)) / 4.0,
                  std::round(20.0 * rc) / 20.0, ntot > 0 ? (int)std::floor(std::log2((double)ntot)) : 0,
                  (int)std::floor(std::log2((double)std::max(nb, 1))));
    return buf;
}

int mdpd_batch_tune(mdpd_batch_t *b, int32_t *shape_density, int32_t *shape_force)
{
    if (!b) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        const TunePick p = tune_by_timing(b);
        if (shape_density) *shape_density = p.density;
        if (shape_force) *shape_force = p.force;
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_batch_tune_cached(mdpd_batch_t *b, const char *path, int32_t *shape_density, int32_t *shape_force,
                           int32_t *cached)
{
    if (!b || !path || !*path) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        const std::string key = tune_key(b);
        const StepConfig base = b->batch->cfg;
        TunePick p;
        const bool hit = tune_cache_get(path, key, p);
        if (hit) {
            // the stored shapes must be ones this batch's family offers
            const StepConfig *use = nullptr;
            for (const StepConfig &c : tune_candidates(base)) {
                const TunePick q = pick_of(c, 0.0);
                if (q.density == p.density && q.force == p.force) {
                    b->batch->reconfigure(c);
                    use = &c;
                    break;
                }
            }
            if (!use)
                throw std::runtime_error("PARSE: tune cache " + std::string(path) + ": entry \"" + key +
                                         "\" holds shapes (" + std::to_string(p.density) + ", " +
                                         std::to_string(p.force) + ") this pass family does not offer");
        } else {
            p = tune_by_timing(b);
            tune_cache_put(path, key, p);
        }
        if (shape_density) *shape_density = p.density;
        if (shape_force) *shape_force = p.force;
        if (cached) *cached = hit ? 1 : 0;
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_batch_set_shapes(mdpd_batch_t *b, int32_t shape_density, int32_t shape_force)
{
    if (!b) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        for (const StepConfig &c : tune_candidates(b->batch->cfg)) {
            const TunePick q = pick_of(c, 0.0);
            if (q.density == shape_density && q.force == shape_force) {
                b->batch->reconfigure(c);
                return;
            }
        }
        throw std::runtime_error("ARG: shapes (" + std::to_string(shape_density) + ", " + std::to_string(shape_force) +
                                 ") are not offered for this batch's pass family");
    });
}

int mdpd_jobs_validate(const char *spec_path, int32_t *njobs, uint64_t *bytes)
{
    if (!spec_path) return MDPD_ERR_ARG;
    return guard(g_err, [&] {
        const JobFile jf = read_job_file(spec_path);
        uint64_t total = 0;
        for (const JobEntry &e : jf.jobs) {
            uint64_t b = 0;
            mdpd_box_bytes(&e.spec.box, &b);
            total += b;
        }
        if (njobs) *njobs = (int32_t)jf.jobs.size();
        if (bytes) *bytes = total;
    });
}

int mdpd_run_jobs(const char *spec_path, const char *out_path, const mdpd_opts *opts)
{
    if (!spec_path) return MDPD_ERR_ARG;
    return guard(g_err, [&] {
        const JobFile jf = read_job_file(spec_path);  // every job checked before the device is touched
        int rc;
        if (out_path && *out_path) {
            std::ofstream f(out_path, std::ios::binary | std::ios::trunc);
            if (!f) throw std::runtime_error("ARG: cannot write " + std::string(out_path));
            rc = run_job_file(jf, opts, f);
        } else {
            rc = run_job_file(jf, opts, std::cout);
        }
        if (rc) throw ScriptError(rc, "a job did not finish (MDPD_* code " + std::to_string(rc) + "): see its result line");
    });
}

int mdpd_batch_profile(mdpd_batch_t *b, int64_t nsteps, double *out5)
{
    if (!b || !out5 || nsteps <= 0) return MDPD_ERR_ARG;
    return guard(b->err, [&] {
        b->batch->profile(nsteps, out5);
        std::string msg;
        if (int st = b->batch->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    });
}

int mdpd_batch_rebuild_steps(mdpd_batch_t *b, int64_t *n)
{
    if (!b || !n) return MDPD_ERR_ARG;
    return guard(b->err, [&] { *n = b->batch->rebuild_steps(); });
}

const char *mdpd_batch_last_error(mdpd_batch_t *b) { return b ? b->err.c_str() : g_err.c_str(); }

void mdpd_batch_destroy(mdpd_batch_t *b)
{
    if (!b) return;
    b->batch.reset();
    b->boxes.clear();
    cudaFree(b->scratch);
    delete b;
}

}  // extern "C"
