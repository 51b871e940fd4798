// Persisted autotuner picks: a JSON file mapping a workload key to the pair-pass shapes the
// timing chose for it, so a later batch of the same kind (same GPU, pass family, density,
// cutoff and size class) takes the shapes without timing.  The reference's tuner learns online
// and forgets at exit (autotuner_meso.h:11-96); this one keeps what it learnt.
//
// File format (written by tune_cache_put, any other members are kept on rewrite):
//   {"version": 1, "entries": {"<key>": {"density": 6, "force": 32, "ms_per_step": 7.8}, ...}}
// Pure C++ (no CUDA), on the reader and writer of json.h; a malformed file is an error, never
// overwritten.
#include "tune_cache.h"

#include "json.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unistd.h>

namespace mdpd {

namespace {

// the file's document; an empty object when the file does not exist
bool load(const std::string &path, Json &doc)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        doc = Json();
        doc.kind = Json::Obj;
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    try {
        doc = json_parse(ss.str());
    } catch (const std::exception &e) {
        throw std::runtime_error("PARSE: tune cache " + path + ": " + e.what());
    }
    if (doc.kind != Json::Obj) throw std::runtime_error("PARSE: tune cache " + path + ": not a JSON object");
    const Json *en = doc.get("entries");
    if (en && en->kind != Json::Obj)
        throw std::runtime_error("PARSE: tune cache " + path + ": \"entries\" is not an object");
    return true;
}

}  // namespace

bool tune_cache_get(const std::string &path, const std::string &key, TunePick &out)
{
    Json doc;
    if (!load(path, doc)) return false;
    const Json *en = doc.get("entries");
    const Json *e = en ? en->get(key) : nullptr;
    if (!e) return false;
    const Json *d = e->kind == Json::Obj ? e->get("density") : nullptr;
    const Json *f = e->kind == Json::Obj ? e->get("force") : nullptr;
    if (!d || !f || d->kind != Json::Num || f->kind != Json::Num)
        throw std::runtime_error("PARSE: tune cache " + path + ": entry \"" + key +
                                 "\" lacks numeric \"density\" and \"force\"");
    out.density = (int)d->num;
    out.force = (int)f->num;
    const Json *ms = e->get("ms_per_step");
    out.ms_per_step = ms && ms->kind == Json::Num ? ms->num : 0.0;
    return true;
}

void tune_cache_put(const std::string &path, const std::string &key, const TunePick &pick)
{
    Json doc;
    load(path, doc);
    Json entry;
    entry.kind = Json::Obj;
    entry.obj.emplace_back("density", Json::number(pick.density));
    entry.obj.emplace_back("force", Json::number(pick.force));
    entry.obj.emplace_back("ms_per_step", Json::number(pick.ms_per_step));
    bool have_version = false, placed = false;
    for (auto &kv : doc.obj) {
        if (kv.first == "version") have_version = true;
        if (kv.first != "entries") continue;
        for (auto &e : kv.second.obj)
            if (e.first == key) e.second = entry, placed = true;
        if (!placed) kv.second.obj.emplace_back(key, entry), placed = true;
    }
    if (!have_version) doc.obj.insert(doc.obj.begin(), {"version", Json::number(1)});
    if (!placed) {
        Json en;
        en.kind = Json::Obj;
        en.obj.emplace_back(key, entry);
        doc.obj.emplace_back("entries", en);
    }
    // write beside the file and rename over it: a reader never sees half a file
    const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) throw std::runtime_error("ARG: tune cache " + path + ": cannot write " + tmp);
        json_emit(f, doc, 0);
        f << "\n";
        if (!f.good()) throw std::runtime_error("ARG: tune cache " + path + ": write failed");
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw std::runtime_error("ARG: tune cache " + path + ": cannot replace the file");
    }
}

}  // namespace mdpd
