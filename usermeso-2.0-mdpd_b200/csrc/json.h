// A small JSON reader and writer for the library's own files (persisted tuner picks, job
// specs): objects keep their members in file order, numbers are doubles.
#pragma once

#include <ostream>
#include <string>
#include <utility>
#include <vector>

namespace mdpd {

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
    static Json number(double x)
    {
        Json v;
        v.kind = Num;
        v.num = x;
        return v;
    }
    static Json object()
    {
        Json v;
        v.kind = Obj;
        return v;
    }
};

// the document in text; throws std::runtime_error("<what> at offset <k>") when malformed
Json json_parse(const std::string &text);
// the value as JSON text, objects one member per line indented by ind + 2 spaces
void json_emit(std::ostream &o, const Json &v, int ind = 0);
// the value on one line (JSON lines)
std::string json_line(const Json &v);
// k as a JSON string literal
std::string json_quote(const std::string &k);

}  // namespace mdpd
