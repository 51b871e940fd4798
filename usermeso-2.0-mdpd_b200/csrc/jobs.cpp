// JSON job specs (jobs.h).  The file names the boxes a server runs; every box field of
// mdpd_box_spec has a key, with the defaults of a deck's usual mdpd/meso settings, and a
// "defaults" object sets them for all jobs:
//
//   {"budget_gb": 150, "timeout_s": 0,
//    "defaults": {"A": -40, "B": 25, "gamma": 4.5, "kT": 1.0, "cut_r": 0.75},
//    "jobs": [{"name": "drop", "n": 20000, "box": 15.0, "steps": 5000, "seed": 7},
//             {"name": "slab", "n": 60000, "box": [40, 15, 15], "fill_hi": [20, 15, 15], ...}]}
//
// An unknown key, a value of the wrong kind, or a missing n, box or steps is an error that names
// the job and the key, like an unknown keyword in a LAMMPS input line (input.cpp).  Results:
// one JSON line per job (state, steps, latency percentiles, throughput, final thermo) and a
// summary line with the server's counters.
#include "jobs.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "engine.h"
#include "json.h"

namespace mdpd {

void spec_from_box(const mdpd_box_spec &bs, Spec &s, Fill &fill);  // capi.cpp

namespace {

[[noreturn]] void bad(const std::string &path, const std::string &where, const std::string &what)
{
    throw std::runtime_error("PARSE: job file " + path + ": " + where + ": " + what);
}

double num(const std::string &path, const std::string &where, const std::string &key, const Json &v)
{
    if (v.kind == Json::Bool) return v.b ? 1.0 : 0.0;
    if (v.kind != Json::Num) bad(path, where, "\"" + key + "\" must be a number");
    return v.num;
}

long long integer(const std::string &path, const std::string &where, const std::string &key, const Json &v,
                  double lo, double hi)
{
    const double x = num(path, where, key, v);
    if (x != std::floor(x) || x < lo || x > hi)
        bad(path, where, "\"" + key + "\" must be an integer in [" + std::to_string((long long)lo) + ", " +
                             std::to_string((long long)hi) + "]");
    return (long long)x;
}

void vec3(const std::string &path, const std::string &where, const std::string &key, const Json &v, double out[3],
          bool scalar_ok)
{
    if (scalar_ok && v.kind == Json::Num) {
        out[0] = out[1] = out[2] = v.num;
        return;
    }
    if (v.kind != Json::Arr || v.arr.size() != 3)
        bad(path, where, "\"" + key + "\" must be " + (scalar_ok ? "a number or " : "") + "a list of 3 numbers");
    for (int d = 0; d < 3; ++d) out[d] = num(path, where, key, v.arr[d]);
}

// set one box/job field from a key of a job (or of "defaults")
void apply(const std::string &path, const std::string &where, const std::string &key, const Json &v, JobEntry &e,
           double L[3], bool &have_n, bool &have_box, bool &have_steps)
{
    mdpd_box_spec &b = e.spec.box;
    const double i32 = 2147483647.0;
    if (key == "name") {
        if (v.kind != Json::Str) bad(path, where, "\"name\" must be a string");
        e.name = v.str;
    } else if (key == "style") {
        if (v.kind == Json::Str && (v.str == "mdpd" || v.str == "mdpd/meso")) b.style = 0;
        else if (v.kind == Json::Str && (v.str == "dpd" || v.str == "dpd/meso")) b.style = 1;
        else bad(path, where, "\"style\" must be \"mdpd\" or \"dpd\"");
    } else if (key == "n") {
        b.n = (int32_t)integer(path, where, key, v, 1, i32);
        have_n = true;
    } else if (key == "box") {
        vec3(path, where, key, v, L, true);
        have_box = true;
    } else if (key == "lo") {
        vec3(path, where, key, v, b.lo, false);
    } else if (key == "steps") {
        e.spec.nsteps = integer(path, where, key, v, 1, 9.0e15);
        have_steps = true;
    } else if (key == "A") b.A = num(path, where, key, v);
    else if (key == "B") b.B = num(path, where, key, v);
    else if (key == "gamma") b.gamma = num(path, where, key, v);
    else if (key == "kT") b.kT = num(path, where, key, v);
    else if (key == "cut") b.cut = num(path, where, key, v);
    else if (key == "cut_r") b.cut_r = num(path, where, key, v);
    else if (key == "cut_rho") b.cut_rho = num(path, where, key, v);
    else if (key == "sigma") b.sigma = num(path, where, key, v);
    else if (key == "dt") b.dt = num(path, where, key, v);
    else if (key == "skin") b.skin = num(path, where, key, v);
    else if (key == "rho_est") b.rho_est = num(path, where, key, v);
    else if (key == "mass") b.mass = num(path, where, key, v);
    else if (key == "seed") b.seed = (uint32_t)integer(path, where, key, v, 0, 4294967295.0);
    else if (key == "every") b.every = (int32_t)integer(path, where, key, v, 1, i32);
    else if (key == "delay") b.delay = (int32_t)integer(path, where, key, v, 0, i32);
    else if (key == "check") b.check = (int32_t)integer(path, where, key, v, 0, 1);
    else if (key == "exact_rng") b.exact_rng = (int32_t)integer(path, where, key, v, 0, 1);
    else if (key == "init_seed") b.init_seed = (uint64_t)integer(path, where, key, v, 0, 9.0e15);
    else if (key == "fill_lo") vec3(path, where, key, v, b.fill_lo, false);
    else if (key == "fill_hi") vec3(path, where, key, v, b.fill_hi, false);
    else if (key == "start_step") b.start_step = integer(path, where, key, v, 0, 9.0e15);
    else bad(path, where, "unknown key \"" + key + "\"");
}

const char *state_name(int s)
{
    static const char *names[] = {"queued", "running", "done", "failed", "cancelled", "preempted"};
    return s >= 0 && s < 6 ? names[s] : "unknown";
}

}  // namespace

JobFile read_job_file(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("ARG: job file " + path + ": cannot be read");
    std::stringstream ss;
    ss << f.rdbuf();
    Json doc;
    try {
        doc = json_parse(ss.str());
    } catch (const std::exception &e) {
        throw std::runtime_error("PARSE: job file " + path + ": " + e.what());
    }
    if (doc.kind != Json::Obj) bad(path, "top level", "not a JSON object");
    JobFile jf;
    double budget_gb = 150.0;
    const Json *defaults = nullptr, *jobs = nullptr;
    for (auto &kv : doc.obj) {
        if (kv.first == "version") continue;
        if (kv.first == "budget_gb") {
            budget_gb = num(path, "top level", kv.first, kv.second);
            if (!(budget_gb > 0 && budget_gb < 1e6)) bad(path, "top level", "\"budget_gb\" must be positive");
        } else if (kv.first == "timeout_s") {
            jf.timeout_s = num(path, "top level", kv.first, kv.second);
            if (!(jf.timeout_s >= 0)) bad(path, "top level", "\"timeout_s\" must be >= 0");
        } else if (kv.first == "defaults") {
            if (kv.second.kind != Json::Obj) bad(path, "top level", "\"defaults\" must be an object");
            defaults = &kv.second;
        } else if (kv.first == "jobs") {
            if (kv.second.kind != Json::Arr) bad(path, "top level", "\"jobs\" must be a list");
            jobs = &kv.second;
        } else
            bad(path, "top level", "unknown key \"" + kv.first + "\"");
    }
    if (!jobs || jobs->arr.empty()) bad(path, "top level", "\"jobs\" must list at least one job");
    jf.budget_bytes = (uint64_t)(budget_gb * 1073741824.0);
    for (size_t k = 0; k < jobs->arr.size(); ++k) {
        const Json &j = jobs->arr[k];
        JobEntry e;
        e.name = "job" + std::to_string(k);
        mdpd_box_spec &b = e.spec.box;
        // the usual mdpd/meso deck settings (the Python box_spec defaults)
        b.style = 0;
        b.A = -40.0, b.B = 25.0, b.gamma = 4.5, b.kT = 1.0;
        b.cut = 1.0, b.cut_r = 0.75, b.cut_rho = 0.75, b.sigma = 3.0;
        b.dt = 0.01, b.skin = 0.3, b.rho_est = 6.05, b.mass = 1.0;
        b.seed = 1234, b.every = 1, b.delay = 0, b.check = 1, b.exact_rng = 0, b.init_seed = 1;
        double L[3] = {0, 0, 0};
        bool have_n = false, have_box = false, have_steps = false;
        if (j.kind != Json::Obj) bad(path, "job " + std::to_string(k), "not an object");
        if (defaults)
            for (auto &kv : defaults->obj) {
                if (kv.first == "name") bad(path, "defaults", "\"name\" is per job");
                apply(path, "defaults", kv.first, kv.second, e, L, have_n, have_box, have_steps);
            }
        const Json *nm = j.get("name");
        const std::string where = "job " + std::to_string(k) + (nm && nm->kind == Json::Str ? " (" + nm->str + ")" : "");
        for (auto &kv : j.obj) apply(path, where, kv.first, kv.second, e, L, have_n, have_box, have_steps);
        if (!have_n) bad(path, where, "\"n\" is required");
        if (!have_box) bad(path, where, "\"box\" is required");
        if (!have_steps) bad(path, where, "\"steps\" is required");
        for (int d = 0; d < 3; ++d) {
            if (!(L[d] > 0)) bad(path, where, "\"box\" edges must be positive");
            b.hi[d] = b.lo[d] + L[d];
        }
        for (auto &o : jf.jobs)
            if (o.name == e.name) bad(path, where, "duplicate name \"" + e.name + "\"");
        uint64_t bytes = 0;
        try {  // the checks a box of this spec meets at creation, with their messages
            Spec sp;
            Fill fill;
            mdpd_box_spec one = b;
            one.n = 1;
            spec_from_box(one, sp, fill);
            bytes = Box::estimate_bytes(sp, b.n);
        } catch (const std::exception &ex) {
            bad(path, where, ex.what());
        }
        if (bytes > jf.budget_bytes)
            bad(path, where, "needs " + std::to_string(bytes) + " device bytes, above budget_gb");
        jf.jobs.push_back(e);
    }
    return jf;
}

int run_job_file(const JobFile &jf, const mdpd_opts *opts, std::ostream &out)
{
    mdpd_server_t *srv = nullptr;
    int rc = mdpd_server_start(&srv, jf.budget_bytes, opts);
    if (rc) return rc;
    std::vector<int64_t> ids(jf.jobs.size(), -1);
    std::vector<int> submit_rc(jf.jobs.size(), MDPD_OK);
    for (size_t k = 0; k < jf.jobs.size(); ++k) submit_rc[k] = mdpd_server_submit(srv, &jf.jobs[k].spec, &ids[k]);
    const int drained = mdpd_server_drain(srv, jf.timeout_s);
    int first = MDPD_OK;
    double start = 1e300, end = 0.0;
    long long done = 0;
    for (size_t k = 0; k < jf.jobs.size(); ++k) {
        const JobEntry &e = jf.jobs[k];
        Json line = Json::object();
        auto put = [&](const char *key, Json v) { line.obj.emplace_back(key, std::move(v)); };
        Json nm;
        nm.kind = Json::Str;
        nm.str = e.name;
        put("job", nm);
        put("n", Json::number(e.spec.box.n));
        put("steps", Json::number((double)e.spec.nsteps));
        mdpd_job_result r{};
        const int prc = submit_rc[k] ? submit_rc[k] : mdpd_server_poll(srv, ids[k], &r);
        Json st;
        st.kind = Json::Str;
        if (prc) {
            st.str = "rejected";
            put("state", st);
            put("error", Json::number(prc));
            if (!first) first = prc;
        } else {
            st.str = state_name(r.state);
            put("id", Json::number((double)ids[k]));
            put("state", st);
            put("error", Json::number(r.error));
            put("steps_done", Json::number((double)r.steps_done));
            const double run_s = r.end_s > r.start_s ? r.end_s - r.start_s : 0.0;
            put("queue_s", Json::number(r.start_s > r.submit_s ? r.start_s - r.submit_s : 0.0));
            put("run_s", Json::number(run_s));
            put("particle_steps_per_s",
                Json::number(run_s > 0 ? (double)e.spec.box.n * (double)r.steps_done / run_s : 0.0));
            put("step_ms_p50", Json::number(r.step_ms_p50));
            put("step_ms_p99", Json::number(r.step_ms_p99));
            put("nbuild", Json::number((double)r.thermo.nbuild));
            put("temp", Json::number(r.thermo.temp));
            put("pe", Json::number(r.thermo.pe));
            put("press", Json::number(r.thermo.press));
            put("status", Json::number(r.thermo.status));
            if (r.state == 2) {
                ++done;
                start = std::min(start, r.start_s);
                end = std::max(end, r.end_s);
            } else if (!first)
                first = r.state == 3 && r.error ? r.error : drained ? drained : MDPD_ERR_STATE;
        }
        out << json_line(line) << "\n";
    }
    double s7[7] = {0, 0, 0, 0, 0, 0, 0};
    mdpd_server_stats(srv, s7);
    Json sum = Json::object();
    sum.obj.emplace_back("jobs", Json::number((double)jf.jobs.size()));
    sum.obj.emplace_back("done", Json::number((double)done));
    sum.obj.emplace_back("particle_steps_per_s", Json::number(s7[0]));
    sum.obj.emplace_back("step_ms_p50", Json::number(s7[1]));
    sum.obj.emplace_back("step_ms_p99", Json::number(s7[2]));
    sum.obj.emplace_back("job_s_p50", Json::number(s7[3]));
    sum.obj.emplace_back("job_s_p99", Json::number(s7[4]));
    sum.obj.emplace_back("peak_resident_bytes", Json::number(s7[6]));
    sum.obj.emplace_back("span_s", Json::number(end > start ? end - start : 0.0));
    Json top = Json::object();
    top.obj.emplace_back("summary", sum);
    out << json_line(top) << "\n";
    out.flush();
    mdpd_server_stop(srv);
    return first;
}

}  // namespace mdpd
