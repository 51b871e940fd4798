// JSON reader and writer (json.h).
#include "json.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <stdexcept>

namespace mdpd {

namespace {

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

std::string quote_impl(const std::string &k)
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

void emit_impl(std::ostream &o, const Json &v, int ind, bool oneline)
{
    const std::string pad(ind + 2, ' ');
    switch (v.kind) {
    case Json::Null: o << "null"; break;
    case Json::Bool: o << (v.b ? "true" : "false"); break;
    case Json::Num: {
        if (!std::isfinite(v.num)) {  // JSON has no NaN or infinity
            o << "null";
            break;
        }
        // the shorter of 15 and 17 significant digits that reads back as the same double
        char b[32];
        std::snprintf(b, sizeof b, "%.15g", v.num);
        if (std::strtod(b, nullptr) != v.num) std::snprintf(b, sizeof b, "%.17g", v.num);
        o << b;
        break;
    }
    case Json::Str: o << quote_impl(v.str); break;
    case Json::Arr:
        o << "[";
        for (size_t k = 0; k < v.arr.size(); ++k) {
            if (k) o << ", ";
            emit_impl(o, v.arr[k], ind, oneline);
        }
        o << "]";
        break;
    case Json::Obj:
        if (v.obj.empty()) {
            o << "{}";
            break;
        }
        o << (oneline ? "{" : "{\n");
        for (size_t k = 0; k < v.obj.size(); ++k) {
            if (!oneline) o << pad;
            o << quote_impl(v.obj[k].first) << ": ";
            emit_impl(o, v.obj[k].second, ind + 2, oneline);
            if (k + 1 < v.obj.size()) o << (oneline ? ", " : ",\n");
            else if (!oneline) o << "\n";
        }
        if (!oneline) o << std::string(ind, ' ');
        o << "}";
        break;
    }
}

}  // namespace

Json json_parse(const std::string &text) { return Parser(text).document(); }

void json_emit(std::ostream &o, const Json &v, int ind) { emit_impl(o, v, ind, false); }

std::string json_line(const Json &v)
{
    std::ostringstream o;
    emit_impl(o, v, 0, true);
    return o.str();
}

std::string json_quote(const std::string &k) { return quote_impl(k); }

}  // namespace mdpd
