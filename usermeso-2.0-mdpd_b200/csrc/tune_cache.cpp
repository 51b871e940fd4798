// Persisted autotuner picks: a JSON file mapping a workload key to the pair-pass shapes the
// timing chose for it, so a later batch of the same kind (same GPU, pass family, density,
// cutoff and size class) takes the shapes without timing.  The reference's tuner learns online
// and forgets at exit (autotuner_meso.h:11-96); this one keeps what it learnt.
//
// File format (written by tune_cache_put, any other members are kept on rewrite):
//   {"version": 1, "entries": {"<key>": {"density": 6, "force": 32, "ms_per_step": 7.8}, ...}}
// Pure C++ (no CUDA): the reader is a small JSON parser of objects, arrays, strings, numbers,
// true/false/null; a malformed file is an error, never overwritten.
#include "tune_cache.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unistd.h>

namespace mdpd {

namespace {

struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0;
    bool b = false;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;  // insertion order kept

    const Json *get(const std::string &k) const
    {
        for (auto &kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class Parser {
public:
    explicit Parser(const std::string &t) : s(t) {}
    Json document()
    {
        Json v = value();
        ws();
        if (p != s.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string &s;
    size_t p = 0;
    int depth = 0;

    [[noreturn]] void fail(const char *what)
    {
        throw std::runtime_error(std::string(what) + " at offset " + std::to_string(p));
    }
    void ws()
    {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) ++p;
    }
    bool lit(const char *w)
    {
        size_t n = 0;
        while (w[n]) ++n;
        if (s.compare(p, n, w) == 0) {
            p += n;
            return true;
        }
        return false;
    }
    std::string string()
    {
        if (p >= s.size() || s[p] != '"') fail("expected a string");
        ++p;
        std::string out;
        while (true) {
            if (p >= s.size()) fail("unterminated string");
            const char c = s[p++];
            if (c == '"') break;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (p >= s.size()) fail("unterminated escape");
            const char e = s[p++];
            switch (e) {
            case '"': out += '"'; break;
            case '\\': out += '\\'; break;
            case '/': out += '/'; break;
            case 'b': out += '\b'; break;
            case 'f': out += '\f'; break;
            case 'n': out += '\n'; break;
            case 'r': out += '\r'; break;
            case 't': out += '\t'; break;
            case 'u': {  // keys are ASCII; other code points are kept as UTF-8
                if (p + 4 > s.size()) fail("short \\u escape");
                unsigned cp = 0;
                for (int k = 0; k < 4; ++k) {
                    const char h = s[p++];
                    cp <<= 4;
                    if (h >= '0' && h <= '9') cp |= h - '0';
                    else if (h >= 'a' && h <= 'f') cp |= h - 'a' + 10;
                    else if (h >= 'A' && h <= 'F') cp |= h - 'A' + 10;
                    else fail("bad \\u escape");
                }
                if (cp < 0x80) out += (char)cp;
                else if (cp < 0x800) out += (char)(0xC0 | (cp >> 6)), out += (char)(0x80 | (cp & 0x3F));
                else
                    out += (char)(0xE0 | (cp >> 12)), out += (char)(0x80 | ((cp >> 6) & 0x3F)),
                        out += (char)(0x80 | (cp & 0x3F));
                break;
            }
            default: fail("bad escape");
            }
        }
        return out;
    }
    Json value()
    {
        if (++depth > 64) fail("nesting too deep");
        ws();
        Json v;
        if (p >= s.size()) fail("unexpected end");
        const char c = s[p];
        if (c == '{') {
            v.kind = Json::Obj;
            ++p;
            ws();
            if (p < s.size() && s[p] == '}') {
                ++p;
            } else {
                while (true) {
                    ws();
                    std::string k = string();
                    ws();
                    if (p >= s.size() || s[p] != ':') fail("expected ':'");
                    ++p;
                    v.obj.emplace_back(std::move(k), value());
                    ws();
                    if (p < s.size() && s[p] == ',') {
                        ++p;
                        continue;
                    }
                    if (p < s.size() && s[p] == '}') {
                        ++p;
                        break;
                    }
                    fail("expected ',' or '}'");
                }
            }
        } else if (c == '[') {
            v.kind = Json::Arr;
            ++p;
            ws();
            if (p < s.size() && s[p] == ']') {
                ++p;
            } else {
                while (true) {
                    v.arr.push_back(value());
                    ws();
                    if (p < s.size() && s[p] == ',') {
                        ++p;
                        continue;
                    }
                    if (p < s.size() && s[p] == ']') {
                        ++p;
                        break;
                    }
                    fail("expected ',' or ']'");
                }
            }
        } else if (c == '"') {
            v.kind = Json::Str;
            v.str = string();
        } else if (lit("true")) {
            v.kind = Json::Bool, v.b = true;
        } else if (lit("false")) {
            v.kind = Json::Bool;
        } else if (lit("null")) {
            v.kind = Json::Null;
        } else {
            const size_t q = p;
            if (p < s.size() && s[p] == '-') ++p;
            while (p < s.size() && ((s[p] >= '0' && s[p] <= '9') || s[p] == '.' || s[p] == 'e' || s[p] == 'E' ||
                                    s[p] == '+' || s[p] == '-'))
                ++p;
            if (p == q) fail("unexpected character");
            const std::string t = s.substr(q, p - q);
            char *end = nullptr;
            v.kind = Json::Num;
            v.num = std::strtod(t.c_str(), &end);
            if (!end || *end) fail("bad number");
        }
        --depth;
        return v;
    }
};

std::string quote(const std::string &k)
{
    std::string o = "\"";
    for (char c : k) {
        if (c == '"' || c == '\\') o += '\\', o += c;
        else if ((unsigned char)c < 0x20) {
            char b[8];
            std::snprintf(b, sizeof b, "\\u%04x", (unsigned char)c);
            o += b;
        } else
            o += c;
    }
    return o + "\"";
}

void emit(std::ostream &o, const Json &v, int ind)
{
    const std::string pad(ind + 2, ' ');
    switch (v.kind) {
    case Json::Null: o << "null"; break;
    case Json::Bool: o << (v.b ? "true" : "false"); break;
    case Json::Num: {
        char b[32];
        std::snprintf(b, sizeof b, "%.17g", v.num);
        o << b;
        break;
    }
    case Json::Str: o << quote(v.str); break;
    case Json::Arr:
        o << "[";
        for (size_t k = 0; k < v.arr.size(); ++k) {
            if (k) o << ", ";
            emit(o, v.arr[k], ind);
        }
        o << "]";
        break;
    case Json::Obj:
        if (v.obj.empty()) {
            o << "{}";
            break;
        }
        o << "{\n";
        for (size_t k = 0; k < v.obj.size(); ++k) {
            o << pad << quote(v.obj[k].first) << ": ";
            emit(o, v.obj[k].second, ind + 2);
            o << (k + 1 < v.obj.size() ? ",\n" : "\n");
        }
        o << std::string(ind, ' ') << "}";
        break;
    }
}

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
        doc = Parser(ss.str()).document();
    } catch (const std::exception &e) {
        throw std::runtime_error("PARSE: tune cache " + path + ": " + e.what());
    }
    if (doc.kind != Json::Obj) throw std::runtime_error("PARSE: tune cache " + path + ": not a JSON object");
    const Json *en = doc.get("entries");
    if (en && en->kind != Json::Obj)
        throw std::runtime_error("PARSE: tune cache " + path + ": \"entries\" is not an object");
    return true;
}

Json number(double x)
{
    Json v;
    v.kind = Json::Num;
    v.num = x;
    return v;
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
    entry.obj.emplace_back("density", number(pick.density));
    entry.obj.emplace_back("force", number(pick.force));
    entry.obj.emplace_back("ms_per_step", number(pick.ms_per_step));
    bool have_version = false, placed = false;
    for (auto &kv : doc.obj) {
        if (kv.first == "version") have_version = true;
        if (kv.first != "entries") continue;
        for (auto &e : kv.second.obj)
            if (e.first == key) e.second = entry, placed = true;
        if (!placed) kv.second.obj.emplace_back(key, entry), placed = true;
    }
    if (!have_version) doc.obj.insert(doc.obj.begin(), {"version", number(1)});
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
        emit(f, doc, 0);
        f << "\n";
        if (!f.good()) throw std::runtime_error("ARG: tune cache " + path + ": write failed");
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw std::runtime_error("ARG: tune cache " + path + ": cannot replace the file");
    }
}

}  // namespace mdpd
