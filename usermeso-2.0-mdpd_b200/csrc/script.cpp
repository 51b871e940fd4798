// LAMMPS input-script front end (see script.h).  Argument order, defaults and error
// texts follow the reference styles cited beside each command.
#include "script.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <sstream>

#include "../../include/mdpd.h"

namespace mdpd {

static std::vector<std::string> split(const std::string &s)
{
    std::vector<std::string> out;
    std::istringstream is(s);
    std::string t;
    while (is >> t) out.push_back(t);
    return out;
}

[[noreturn]] static void parse_error(const std::string &m) { throw ScriptError(MDPD_ERR_PARSE, m); }

// Park-Miller minimal standard generator, as LAMMPS RanPark (random_park.cpp:33-63)
struct Park {
    int seed;
    bool save = false;
    double second = 0;
    explicit Park(int s) : seed(s)
    {
        if (s <= 0) parse_error("Invalid seed for Park random # generator");
    }
    double uniform()
    {
        const int k = seed / 127773;
        seed = 16807 * (seed - k * 127773) - 2836 * k;
        if (seed < 0) seed += 2147483647;
        return (1.0 / 2147483647) * seed;
    }
    double gaussian()
    {
        if (save) {
            save = false;
            return second;
        }
        double v1, v2, rsq;
        do {
            v1 = 2.0 * uniform() - 1.0;
            v2 = 2.0 * uniform() - 1.0;
            rsq = v1 * v1 + v2 * v2;
        } while (!(rsq < 1.0 && rsq != 0.0));
        const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
        second = v1 * fac;
        save = true;
        return v2 * fac;
    }
};

Script::Script(int device) : device_(device)
{
    // the device is first touched by the first run/setup, so scripts parse without a GPU
    groups_["all"] = 0;
    for (int a = 0; a < kMaxTypes; ++a)
        for (int b = 0; b < kMaxTypes; ++b) spec_.pair[a][b] = PairParam();
}

Script::~Script()
{
    // fix density/meso writes its open window at destruction (fix_density_profile_meso.cpp:85-96)
    for (DensityFix &d : dens_) {
        const long long n = (step_ + d.every / 2) / d.every, m = n * d.every;
        if (step_ - m >= -d.window && step_ - m < d.window && d.last_dump < step_ && d.frames > 0) {
            try {
                density_dump(d, m);
            } catch (...) {
            }
        }
        if (d.d_counts) cudaFree(d.d_counts);
    }
    batch_.reset();
    box_.reset();
}

// ---------------------------------------------------------------------------
// variables and expressions
// ---------------------------------------------------------------------------
namespace {
struct Expr {
    const std::string &s;
    size_t p = 0;
    std::map<std::string, std::string> &vars;
    std::function<double(const std::string &)> varval;
    void ws()
    {
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
    }
    double primary()
    {
        ws();
        if (p >= s.size()) parse_error("Invalid syntax in variable formula: " + s);
        if (s[p] == '(') {
            ++p;
            double v = add();
            ws();
            if (p >= s.size() || s[p] != ')') parse_error("Invalid syntax in variable formula: " + s);
            ++p;
            return v;
        }
        if (s[p] == '-') {
            ++p;
            return -power();
        }
        if (s[p] == '+') {
            ++p;
            return power();
        }
        if (std::isdigit((unsigned char)s[p]) || s[p] == '.') {
            size_t q = p;
            while (q < s.size() && (std::isdigit((unsigned char)s[q]) || s[q] == '.')) ++q;
            if (q < s.size() && (s[q] == 'e' || s[q] == 'E')) {
                ++q;
                if (q < s.size() && (s[q] == '+' || s[q] == '-')) ++q;
                while (q < s.size() && std::isdigit((unsigned char)s[q])) ++q;
            }
            double v = std::strtod(s.substr(p, q - p).c_str(), nullptr);
            p = q;
            return v;
        }
        if (std::isalpha((unsigned char)s[p]) || s[p] == '_') {
            size_t q = p;
            while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_')) ++q;
            std::string name = s.substr(p, q - p);
            p = q;
            ws();
            if (p < s.size() && s[p] == '(') {
                ++p;
                double a = add();
                ws();
                if (p >= s.size() || s[p] != ')') parse_error("Invalid math function in variable formula");
                ++p;
                if (name == "round") return std::round(a);
                if (name == "floor") return std::floor(a);
                if (name == "ceil") return std::ceil(a);
                if (name == "sqrt") return std::sqrt(a);
                if (name == "exp") return std::exp(a);
                if (name == "ln") return std::log(a);
                if (name == "log") return std::log10(a);
                if (name == "abs") return std::fabs(a);
                if (name == "sin") return std::sin(a);
                if (name == "cos") return std::cos(a);
                parse_error("Invalid math function in variable formula: " + name);
            }
            if (name == "PI") return M_PI;
            if (name.rfind("v_", 0) == 0) return varval(name.substr(2));
            parse_error("Invalid thermo keyword in variable formula: " + name);
        }
        parse_error("Invalid syntax in variable formula: " + s);
    }
    double power()
    {
        double v = primary();
        ws();
        if (p < s.size() && s[p] == '^') {
            ++p;
            return std::pow(v, power());
        }
        return v;
    }
    double mul()
    {
        double v = power();
        for (;;) {
            ws();
            if (p < s.size() && s[p] == '*') {
                ++p;
                v *= power();
            } else if (p < s.size() && s[p] == '/') {
                ++p;
                v /= power();
            } else
                return v;
        }
    }
    double add()
    {
        double v = mul();
        for (;;) {
            ws();
            if (p < s.size() && s[p] == '+') {
                ++p;
                v += mul();
            } else if (p < s.size() && s[p] == '-') {
                ++p;
                v -= mul();
            } else
                return v;
        }
    }
};
}  // namespace

double Script::eval(const std::string &expr)
{
    Expr e{expr, 0, vars_, [this](const std::string &n) {
               auto it = vars_.find(n);
               if (it == vars_.end()) parse_error("Invalid variable name in variable formula: " + n);
               return eval(it->second);
           }};
    double v = e.add();
    e.ws();
    if (e.p != expr.size()) parse_error("Invalid syntax in variable formula: " + expr);
    return v;
}

static std::string fmt15(double v)
{
    char b[64];
    std::snprintf(b, sizeof(b), "%.15g", v);
    return b;
}

std::string Script::substitute(const std::string &line)
{
    // strip comment, then replace ${name} and $c with equal-style values (input.cpp)
    std::string s;
    bool quote = false;
    for (char ch : line) {
        if (ch == '"') quote = !quote;
        if (ch == '#' && !quote) break;
        s += ch;
    }
    std::string out;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] == '$' && i + 1 < s.size()) {
            std::string name;
            if (s[i + 1] == '{') {
                size_t e = s.find('}', i + 2);
                if (e == std::string::npos) parse_error("Invalid variable name");
                name = s.substr(i + 2, e - i - 2);
                i = e;
            } else {
                name = s.substr(i + 1, 1);
                i += 1;
            }
            auto it = vars_.find(name);
            if (it == vars_.end()) parse_error("Substitution for illegal variable " + name);
            out += fmt15(eval(it->second));
        } else
            out += s[i];
    }
    return out;
}

double Script::num(const std::string &tok)
{
    char *end = nullptr;
    double v = std::strtod(tok.c_str(), &end);
    if (end == tok.c_str() || *end) parse_error("Expected floating point parameter instead of " + tok);
    return v;
}

int Script::inum(const std::string &tok)
{
    char *end = nullptr;
    long v = std::strtol(tok.c_str(), &end, 10);
    if (end == tok.c_str() || *end) parse_error("Expected integer parameter instead of " + tok);
    return (int)v;
}

int Script::group_bit(const std::string &name)
{
    auto it = groups_.find(name);
    if (it == groups_.end()) parse_error("Could not find group ID " + name);
    return 1 << it->second;
}

void Script::type_range(const std::string &tok, int &lo, int &hi)
{
    // Force::bounds: "*", "n", "n*", "*n", "m*n"
    const int nt = spec_.ntype;
    size_t st = tok.find('*');
    if (st == std::string::npos) {
        lo = hi = inum(tok);
    } else {
        lo = st == 0 ? 1 : inum(tok.substr(0, st));
        hi = st + 1 == tok.size() ? nt : inum(tok.substr(st + 1));
    }
    if (lo < 1 || hi > nt || lo > hi) parse_error("Numeric index is out of bounds");
}

void Script::add_atom(int type, const double *x)
{
    if (type < 1 || type > spec_.ntype) parse_error("Invalid atom type in create_atoms command");
    parts_.x.insert(parts_.x.end(), x, x + 3);
    for (int d = 0; d < 3; ++d) parts_.v.push_back(0.0);
    parts_.tag.push_back((int)parts_.tag.size() + 1);
    parts_.type.push_back(type);
    parts_.mask.push_back(1);
}

// ---------------------------------------------------------------------------
// commands
// ---------------------------------------------------------------------------
void Script::file(const std::string &path)
{
    std::ifstream in(path);
    if (!in) throw ScriptError(MDPD_ERR_ARG, "Cannot open input script " + path);
    std::string line, acc;
    while (std::getline(in, line)) {
        // continuation with a trailing '&'
        size_t e = line.find_last_not_of(" \t\r");
        if (e != std::string::npos && line[e] == '&') {
            acc += line.substr(0, e) + " ";
            continue;
        }
        acc += line;
        command(acc);
        acc.clear();
    }
    if (!acc.empty()) command(acc);
}

void Script::command(const std::string &raw)
{
    std::string line = substitute(raw);
    std::vector<std::string> a = split(line);
    if (a.empty()) return;
    if (echo) log += line + "\n";
    const std::string &c = a[0];
    const int narg = (int)a.size() - 1;
    static const char *readonly[] = {"variable", "echo", "thermo", "print", "run", "dump", "undump",
                                     "write_data", "units", "dimension", "boundary", "run_style"};
    bool ro = false;
    for (const char *r : readonly) ro = ro || c == r;
    if (!ro) sync_host();  // device state back to the host before it is modified

    if (c == "variable") {
        // variable name equal expr | index/string value
        if (narg < 3) parse_error("Illegal variable command");
        std::string expr;
        for (int k = 3; k <= narg; ++k) expr += (k > 3 ? " " : "") + a[k];
        if (a[2] == "equal" || a[2] == "index" || a[2] == "string") {
            if (!vars_.count(a[1]) || a[2] == "equal") vars_[a[1]] = expr;
        } else
            parse_error("Unsupported variable style " + a[2]);
    } else if (c == "echo") {
        echo = narg >= 1 && (a[1] == "screen" || a[1] == "both" || a[1] == "log");
    } else if (c == "units") {
        if (narg != 1 || a[1] != "lj") parse_error("Only units lj is supported by this path");
    } else if (c == "dimension") {
        if (narg != 1 || a[1] != "3") parse_error("Only dimension 3 is supported");
    } else if (c == "boundary") {
        if (narg != 3 || a[1] != "p" || a[2] != "p" || a[3] != "p")
            parse_error("Only boundary p p p is supported");
    } else if (c == "atom_style") {
        if (narg < 1) parse_error("Illegal atom_style command");
        if (a[1] == "mdpd/atomic/meso") {
            // atom_vec_mdpd_atomic_meso.cu:27-30
            if (narg < 2)
                parse_error("For atom_style mdpd/atomic/meso, an estimation to maximum local particle "
                            "density must be given. Or input 0 for default.");
            spec_.style = 0;
            spec_.rho_est = num(a[2]);
        } else if (a[1] == "dpd/atomic/meso") {
            spec_.style = 1;
            spec_.rho_est = 0;
        } else
            parse_error("Unsupported atom_style " + a[1]);
    } else if (c == "lattice") {
        if (narg < 2) parse_error("Illegal lattice command");
        if (a[1] == "fcc") {
            lattice_fcc_ = 1;
            lattice_a_ = std::pow(4.0 / num(a[2]), 1.0 / 3.0);  // lj: reduced density
        } else if (a[1] == "none") {
            lattice_fcc_ = 0;
            lattice_a_ = num(a[2]);
        } else
            parse_error("Unsupported lattice style " + a[1]);
    } else if (c == "region") {
        if (narg < 8 || a[2] != "block") parse_error("Only region block is supported");
        double scale = lattice_a_;
        for (int k = 9; k + 1 <= narg; ++k)
            if (a[k] == "units") scale = a[k + 1] == "box" ? 1.0 : lattice_a_;
        Region r;
        for (int d = 0; d < 3; ++d) {
            const std::string &lo = a[3 + 2 * d], &hi = a[4 + 2 * d];
            r.lo[d] = (lo == "INF" || lo == "EDGE") ? (box_defined_ ? spec_.lo[d] : -1e300) : num(lo) * scale;
            r.hi[d] = (hi == "INF" || hi == "EDGE") ? (box_defined_ ? spec_.hi[d] : 1e300) : num(hi) * scale;
        }
        regions_[a[1]] = r;
    } else if (c == "create_box") {
        if (narg < 2) parse_error("Illegal create_box command");
        auto it = regions_.find(a[2]);
        if (it == regions_.end()) parse_error("Create_box region ID does not exist");
        spec_.ntype = inum(a[1]);
        if (spec_.ntype < 1 || spec_.ntype > kMaxTypes) parse_error("1..8 atom types supported");
        for (int d = 0; d < 3; ++d) spec_.lo[d] = it->second.lo[d], spec_.hi[d] = it->second.hi[d];
        box_defined_ = true;
    } else if (c == "create_atoms") {
        if (!box_defined_) parse_error("Create_atoms command before simulation box is defined");
        if (narg < 2) parse_error("Illegal create_atoms command");
        const int type = inum(a[1]);
        if (a[2] == "random") {
            // CreateAtoms::add_random (create_atoms.cpp): RanPark(seed), bbox of the region
            if (narg < 5) parse_error("Illegal create_atoms command");
            const int nrand = inum(a[3]);
            Park rng(inum(a[4]));
            double lo[3], hi[3];
            const Region *reg = nullptr;
            if (a[5] != "NULL") {
                auto it = regions_.find(a[5]);
                if (it == regions_.end()) parse_error("Create_atoms region ID does not exist");
                reg = &it->second;
            }
            for (int d = 0; d < 3; ++d) {
                lo[d] = spec_.lo[d], hi[d] = spec_.hi[d];
                if (reg) lo[d] = std::max(lo[d], reg->lo[d]), hi[d] = std::min(hi[d], reg->hi[d]);
            }
            for (int i = 0; i < nrand; ++i) {
                double x[3];
                for (;;) {
                    for (int d = 0; d < 3; ++d) x[d] = lo[d] + rng.uniform() * (hi[d] - lo[d]);
                    bool ok = true;
                    if (reg)
                        for (int d = 0; d < 3; ++d) ok = ok && x[d] >= reg->lo[d] && x[d] <= reg->hi[d];
                    if (ok) break;
                }
                bool inside = true;
                for (int d = 0; d < 3; ++d) inside = inside && x[d] >= spec_.lo[d] && x[d] < spec_.hi[d];
                if (inside) add_atom(type, x);
            }
        } else if (a[2] == "region" || a[2] == "box") {
            if (!lattice_fcc_) parse_error("Cannot create atoms with undefined lattice");
            const Region *reg = nullptr;
            if (a[2] == "region") {
                auto it = regions_.find(a[3]);
                if (it == regions_.end()) parse_error("Create_atoms region ID does not exist");
                reg = &it->second;
            }
            static const double basis[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
            int lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
                lo[d] = (int)std::floor(spec_.lo[d] / lattice_a_) - 1;
                hi[d] = (int)std::ceil(spec_.hi[d] / lattice_a_) + 1;
            }
            for (int k = lo[2]; k <= hi[2]; ++k)
                for (int j = lo[1]; j <= hi[1]; ++j)
                    for (int i = lo[0]; i <= hi[0]; ++i)
                        for (int m = 0; m < 4; ++m) {
                            double x[3] = {(i + basis[m][0]) * lattice_a_, (j + basis[m][1]) * lattice_a_,
                                           (k + basis[m][2]) * lattice_a_};
                            bool ok = true;
                            for (int d = 0; d < 3; ++d) ok = ok && x[d] >= spec_.lo[d] && x[d] < spec_.hi[d];
                            if (reg)
                                for (int d = 0; d < 3; ++d) ok = ok && x[d] >= reg->lo[d] && x[d] <= reg->hi[d];
                            if (ok) add_atom(type, x);
                        }
        } else
            parse_error("Unsupported create_atoms style " + a[2]);
        dirty_ = true;
    } else if (c == "read_data") {
        if (narg < 1) parse_error("Illegal read_data command");
        read_data(a[1]);
        dirty_ = true;
    } else if (c == "mass") {
        if (narg != 2) parse_error("Illegal mass command");
        int lo, hi;
        type_range(a[1], lo, hi);
        for (int t = lo; t <= hi; ++t) spec_.mass[t - 1] = num(a[2]);
        dirty_ = true;
    } else if (c == "group") {
        if (narg < 2) parse_error("Illegal group command");
        sync_host();
        int idx;
        auto it = groups_.find(a[1]);
        if (it != groups_.end())
            idx = it->second;
        else {
            if (ngroup_ >= 32) parse_error("Too many groups");
            idx = ngroup_++;
            groups_[a[1]] = idx;
        }
        const int bit = 1 << idx;
        const size_t n = parts_.size();
        if (a[2] == "type") {
            std::vector<char> sel(kMaxTypes + 1, 0);
            for (int k = 3; k <= narg; ++k) {
                int lo, hi;
                if (a[k].find(':') != std::string::npos) {
                    lo = inum(a[k].substr(0, a[k].find(':')));
                    hi = inum(a[k].substr(a[k].find(':') + 1));
                } else
                    lo = hi = inum(a[k]);
                for (int t = lo; t <= hi && t <= kMaxTypes; ++t) sel[t] = 1;
            }
            for (size_t i = 0; i < n; ++i)
                if (sel[parts_.type[i]]) parts_.mask[i] |= bit;
        } else if (a[2] == "union" || a[2] == "intersect") {
            int m_or = 0;
            std::vector<int> bits;
            for (int k = 3; k <= narg; ++k) bits.push_back(group_bit(a[k]));
            for (int b : bits) m_or |= b;
            for (size_t i = 0; i < n; ++i) {
                bool hit;
                if (a[2] == "union")
                    hit = parts_.mask[i] & m_or;
                else {
                    hit = true;
                    for (int b : bits) hit = hit && (parts_.mask[i] & b);
                }
                if (hit) parts_.mask[i] |= bit;
            }
        } else if (a[2] == "region") {
            auto rt = regions_.find(a[3]);
            if (rt == regions_.end()) parse_error("Group region ID does not exist");
            for (size_t i = 0; i < n; ++i) {
                bool ok = true;
                for (int d = 0; d < 3; ++d)
                    ok = ok && parts_.x[3 * i + d] >= rt->second.lo[d] && parts_.x[3 * i + d] <= rt->second.hi[d];
                if (ok) parts_.mask[i] |= bit;
            }
        } else if (a[2] == "delete") {
            for (size_t i = 0; i < n; ++i) parts_.mask[i] &= ~bit;
        } else
            parse_error("Unsupported group style " + a[2]);
        dirty_ = true;
    } else if (c == "velocity") {
        if (narg < 2) parse_error("Illegal velocity command");
        sync_host();
        const int gb = group_bit(a[1]);
        const size_t n = parts_.size();
        if (a[2] == "create") {
            // Velocity::create, loop all (velocity.cpp:201-253), then zero momentum and rescale
            const double t_want = num(a[3]);
            const int seed = inum(a[4]);
            int dist = 0, mom = 1;
            for (int k = 5; k + 1 <= narg; k += 2) {
                if (a[k] == "dist") dist = a[k + 1] == "gaussian";
                else if (a[k] == "mom") mom = a[k + 1] == "yes";
                else if (a[k] == "loop" && a[k + 1] != "all") parse_error("Only velocity loop all is supported");
            }
            Park rng(seed);
            std::vector<int> idx(n + 1, -1);
            for (size_t i = 0; i < n; ++i)
                if (parts_.tag[i] >= 1 && (size_t)parts_.tag[i] <= n) idx[parts_.tag[i]] = (int)i;
            for (size_t t = 1; t <= n; ++t) {
                double v[3];
                for (int d = 0; d < 3; ++d) v[d] = dist ? rng.gaussian() : rng.uniform();
                const int m = idx[t];
                if (m >= 0 && (parts_.mask[m] & gb)) {
                    const double f = 1.0 / std::sqrt(spec_.mass[parts_.type[m] - 1]);
                    for (int d = 0; d < 3; ++d) parts_.v[3 * m + d] = v[d] * f;
                }
            }
            double mt = 0, p[3] = {0, 0, 0};
            int cnt = 0;
            for (size_t i = 0; i < n; ++i)
                if (parts_.mask[i] & gb) {
                    const double m = spec_.mass[parts_.type[i] - 1];
                    mt += m;
                    ++cnt;
                    for (int d = 0; d < 3; ++d) p[d] += m * parts_.v[3 * i + d];
                }
            if (mom && mt > 0)
                for (size_t i = 0; i < n; ++i)
                    if (parts_.mask[i] & gb)
                        for (int d = 0; d < 3; ++d) parts_.v[3 * i + d] -= p[d] / mt;
            double ke = 0;
            for (size_t i = 0; i < n; ++i)
                if (parts_.mask[i] & gb) {
                    const double m = spec_.mass[parts_.type[i] - 1];
                    for (int d = 0; d < 3; ++d) ke += m * parts_.v[3 * i + d] * parts_.v[3 * i + d];
                }
            const double t_now = ke / (3.0 * cnt - 3.0);
            if (t_now == 0.0) parse_error("Attempting to rescale a 0.0 temperature");
            const double f = std::sqrt(t_want / t_now);
            for (size_t i = 0; i < n; ++i)
                if (parts_.mask[i] & gb)
                    for (int d = 0; d < 3; ++d) parts_.v[3 * i + d] *= f;
        } else if (a[2] == "set") {
            for (size_t i = 0; i < n; ++i)
                if (parts_.mask[i] & gb)
                    for (int d = 0; d < 3; ++d)
                        if (a[3 + d] != "NULL") parts_.v[3 * i + d] = num(a[3 + d]);
        } else if (a[2] == "zero") {
            double mt = 0, p[3] = {0, 0, 0};
            for (size_t i = 0; i < n; ++i)
                if (parts_.mask[i] & gb) {
                    const double m = spec_.mass[parts_.type[i] - 1];
                    mt += m;
                    for (int d = 0; d < 3; ++d) p[d] += m * parts_.v[3 * i + d];
                }
            for (size_t i = 0; i < n; ++i)
                if ((parts_.mask[i] & gb) && mt > 0)
                    for (int d = 0; d < 3; ++d) parts_.v[3 * i + d] -= p[d] / mt;
        } else
            parse_error("Unsupported velocity style " + a[2]);
        dirty_ = true;
    } else if (c == "pair_style") {
        if (narg < 1) parse_error("Illegal pair_style command");
        if (a[1] == "mdpd/meso") {
            // MesoPairMDPD::settings (pair_mdpd_meso.cu:299-328)
            if (narg < 4)
                parse_error("Illegal pair_style command:\n temperature cut_global seed fluid_group wall_group, "
                            "or temperature cut_global seed ");
            if (spec_.style != 0) parse_error("pair_style mdpd/meso requires atom_style mdpd/atomic/meso");
            spec_.kT = num(a[2]);
            spec_.seed = (uint32_t)inum(a[4]);
            spec_.arb_bc = 0;
            if (narg > 4) {
                auto g1 = groups_.find(a[5]);
                if (g1 == groups_.end()) parse_error("<MESO> Undefined fluid group id in pairstyle mdpd/meso");
                if (narg < 5) parse_error("<MESO> Undefined wall group id in pairstyle mdpd/meso");
                auto g2 = groups_.find(a[6]);
                if (g2 == groups_.end()) parse_error("<MESO> Undefined wall group id in pairstyle mdpd/meso");
                spec_.arb_bc = 1;
                spec_.mobile_bit = 1 << g1->second;
                spec_.wall_bit = 1 << g2->second;
            }
        } else if (a[1] == "dpd/meso") {
            // MesoPairDPD::settings (pair_dpd_meso.cu:272-287)
            if (narg != 3) parse_error("Illegal pair_style command");
            if (spec_.style != 1) parse_error("pair_style dpd/meso requires atom_style dpd/atomic/meso");
            spec_.seed = (uint32_t)inum(a[3]);
            for (int i = 0; i < kMaxTypes; ++i)
                for (int j = 0; j < kMaxTypes; ++j) spec_.pair[i][j].cut = num(a[2]);
        } else
            parse_error("Unsupported pair_style " + a[1]);
        pair_set_ = 1;
        dirty_ = true;
    } else if (c == "pair_coeff") {
        if (!pair_set_) parse_error("Pair_coeff command before pair_style is defined");
        int ilo, ihi, jlo, jhi;
        if (narg < 2) parse_error("Incorrect args for pair coefficients");
        type_range(a[1], ilo, ihi);
        type_range(a[2], jlo, jhi);
        PairParam q;
        q.set = 1;
        if (spec_.style == 0) {
            // MesoPairMDPD::coeff (pair_mdpd_meso.cu:330-365)
            if (narg != 7)
                parse_error("Incorrect args for mdpd pair coefficients: \n itype jtype A B gamma cutA cutB");
            q.A = num(a[3]), q.B = num(a[4]), q.gamma = num(a[5]), q.cut = num(a[6]), q.cut_r = num(a[7]);
            if (q.cut < q.cut_r)
                parse_error("Incorrect args for pair coefficients:\n cutA should be larger than cutB.");
        } else {
            // MesoPairDPD::coeff (pair_dpd_meso.cu:289-327)
            if (narg < 6 || narg > 7) parse_error("Incorrect args for pair coefficients");
            q.A = num(a[3]), q.gamma = num(a[4]), q.sigma = num(a[5]), q.expw = num(a[6]);
            q.cut = narg == 7 ? num(a[7]) : spec_.pair[0][0].cut;
        }
        int count = 0;
        for (int i = ilo; i <= ihi; ++i)
            for (int j = std::max(jlo, i); j <= jhi; ++j) {
                spec_.pair[i - 1][j - 1] = q;
                spec_.pair[j - 1][i - 1] = q;
                ++count;
            }
        if (!count) parse_error("Incorrect args for pair coefficients");
        dirty_ = true;
    } else if (c == "pair_modify") {
        // extensions: pair_modify rng exact|fast (FP64 bit-exact gaussian or FP32 transform);
        // gather 4|6|8 pins the pair-once density pass's neighbour gathers in flight per lane;
        // stage yes|no stages each warp's compact rows in shared memory for the pair-once force
        // pass, or has its pair loop read them from the table
        for (int k = 1; k + 1 <= narg; k += 2) {
            if (a[k] == "rng") spec_.exact_rng = a[k + 1] == "exact";
            else if (a[k] == "gather") {
                const int g = inum(a[k + 1]);
                if (g != 4 && g != 6 && g != 8) parse_error("pair_modify gather must be 4, 6 or 8");
                cfg.gather = g;
            } else if (a[k] == "stage") {
                if (a[k + 1] != "yes" && a[k + 1] != "no") parse_error("pair_modify stage must be yes or no");
                cfg.stage_rows = a[k + 1] == "yes";
            }
        }
        dirty_ = true;
    } else if (c == "neighbor") {
        if (narg != 2) parse_error("Illegal neighbor command");
        spec_.skin = num(a[1]);
        if (a[2] != "bin") parse_error("Only neighbor style bin is supported");
        dirty_ = true;
    } else if (c == "neigh_modify") {
        for (int k = 1; k + 1 <= narg; k += 2) {
            if (a[k] == "every") spec_.every = inum(a[k + 1]);
            else if (a[k] == "delay") spec_.delay = inum(a[k + 1]);
            else if (a[k] == "check") spec_.check = a[k + 1] == "yes";
        }
        dirty_ = true;
    } else if (c == "fix") {
        if (narg < 3) parse_error("Illegal fix command");
        const std::string &id = a[1], &style = a[3];
        const int gb = group_bit(a[2]);
        if (style == "nve/meso") {
            spec_.nve_bit = gb;
            nve_fix_ = id;
        } else if (style == "aboundary/rho/meso") {
            // FixArbitraryBoundaryRho ctor (fix_aboundary_rho_meso.cu:30-104)
            double cut_rho = 0, cut_phi = 0, phi_c = 0, rho_wall = 0;
            int wall = 0, mobile = 0, arb = 0;
            for (int k = 4; k <= narg; ++k) {
                if (a[k] == "cut_rho" && k < narg) cut_rho = num(a[++k]);
                else if (a[k] == "cut_phi" && k < narg) cut_phi = num(a[++k]);
                else if (a[k] == "phi_c" && k < narg) phi_c = num(a[++k]);
                else if (a[k] == "rho_wall" && k < narg) rho_wall = num(a[++k]);
                else if (a[k] == "wall" && k < narg) {
                    auto g = groups_.find(a[++k]);
                    if (g == groups_.end()) parse_error("<MESO> Undefined wall group id in fix aboundary/rho/meso");
                    wall = 1 << g->second, arb = 1;
                } else if (a[k] == "mobile" && k < narg) {
                    auto g = groups_.find(a[++k]);
                    if (g == groups_.end()) parse_error("<MESO> Undefined fluid group id in fix aboundary/rho/meso");
                    mobile = 1 << g->second, arb = 1;
                }
            }
            if (!arb && cut_rho == 0) parse_error("<MESO> Fix aboundary/rho/meso parameters are not set properly.");
            if (arb && (cut_rho == 0 || cut_phi == 0 || phi_c == 0 || rho_wall == 0))
                parse_error("<MESO> Fix aboundary/rho/meso parameters are not set properly.");
            spec_.rho_bit = gb;
            spec_.cut_rho = cut_rho;
            spec_.wall_fix = arb;
            spec_.cut_phi = cut_phi;
            spec_.phi_c = phi_c;
            spec_.rho_wall = rho_wall;
            if (arb) {
                spec_.wall_bit = wall;
                spec_.mobile_bit = mobile;
            }
            rho_fix_ = id;
        } else if (style == "aboundary/meso") {
            // FixArbitraryBoundary ctor (fix_aboundary_meso.cu:31-82): keywords anywhere in the line
            int wall = 0;
            double rc = 0, rho0 = 0, sigma = 0;
            for (int k = 1; k <= narg; ++k) {
                if (a[k] == "wall" && k < narg) {
                    auto g = groups_.find(a[++k]);
                    if (g == groups_.end()) parse_error("<MESO> Undefined wall group id in fix aboundary/meso");
                    wall = 1 << g->second;
                    if (gb & wall) log += "WARNING: <MESO> fix aboundary/meso mobile and wall group overlapped\n";
                }
                if (a[k] == "rc" && k < narg) rc = num(a[++k]);
                else if (a[k] == "rho" && k < narg) rho0 = num(a[++k]);
                else if (a[k] == "sigma" && k < narg) sigma = num(a[++k]);
                else if (a[k] == "frac" && k < narg) ++k;  // read and unused by the reference
            }
            if (wall == 0 || rc == 0 || rho0 == 0)
                parse_error("<MESO> Fix aboundary/meso usage: " + style +
                            " <wall groupid> <rc double> <rho double> [sigma double]");
            spec_.ab_mobile_bit = gb;
            spec_.ab_wall_bit = wall;
            spec_.ab_rho0 = rho0;
            spec_.ab_sigma = sigma == 0 ? rc * rc / 4.0 / M_PI : sigma;
            ab_fix_ = id;
        } else if (style == "addforce/meso") {
            // fix ID group addforce/meso fx fy fz; extra words are ignored (fix_addforce_meso.cu:37-48)
            if (narg < 6) parse_error("Illegal fix addforce/meso command");
            spec_.body_bit = gb;
            for (int d = 0; d < 3; ++d) spec_.body[d] = num(a[4 + d]);
        } else if (style == "density/meso") {
            // MesoFixDensityProf ctor (fix_density_profile_meso.cpp:32-80)
            DensityFix d;
            d.id = id;
            d.group = gb;
            d.along = -1;
            for (int k = 4; k <= narg; ++k) {
                if (a[k] == "output" && k < narg) d.output = a[++k];
                else if (a[k] == "along" && k < narg) {
                    const char ch = a[++k][0];
                    d.along = ch == 'x' ? 0 : ch == 'y' ? 1 : ch == 'z' ? 2 : -1;
                } else if (a[k] == "nbin" && k < narg) d.nbin = inum(a[++k]);
                else if (a[k] == "every" && k < narg) d.every = inum(a[++k]);
                else if (a[k] == "window" && k < narg) d.window = inum(a[++k]);
            }
            if (d.output.empty() || d.along < 0 || d.nbin == 0 || d.every == 0 || d.window == 0)
                parse_error("Incomplete fix vprof command: insufficient arguments");
            d.counts.assign(d.nbin, 0);
            dens_.push_back(d);  // device counters are allocated at the first run
        } else
            parse_error("Unsupported fix style " + style);
        dirty_ = true;
    } else if (c == "unfix") {
        if (narg != 1) parse_error("Illegal unfix command");
        if (a[1] == nve_fix_) spec_.nve_bit = 0, nve_fix_.clear();
        if (a[1] == ab_fix_) spec_.ab_mobile_bit = spec_.ab_wall_bit = 0, ab_fix_.clear();
        for (size_t k = 0; k < dens_.size(); ++k)
            if (dens_[k].id == a[1]) {
                if (dens_[k].d_counts) cudaFree(dens_[k].d_counts);
                dens_.erase(dens_.begin() + k);
                break;
            }
        dirty_ = true;
    } else if (c == "timestep") {
        if (narg != 1) parse_error("Illegal timestep command");
        spec_.dt = num(a[1]);
        dirty_ = true;
    } else if (c == "run_style") {
        if (narg < 1 || a[1] != "mvv/meso") parse_error("Only run_style mvv/meso is supported by this path");
    } else if (c == "thermo") {
        if (narg != 1) parse_error("Illegal thermo command");
        thermo_every_ = inum(a[1]);
    } else if (c == "reset_timestep") {
        if (narg != 1) parse_error("Illegal reset_timestep command");
        sync_host();
        step_ = inum(a[1]);
        dirty_ = true;
    } else if (c == "run") {
        if (narg < 1) parse_error("Illegal run command");
        run(std::stoll(a[1]));
    } else if (c == "dump") {
        if (narg < 5 || a[3] != "custom") parse_error("Only dump custom is supported");
        DumpSpec d;
        d.id = a[1];
        d.group = group_bit(a[2]);
        d.every = inum(a[4]);
        d.file = a[5];
        for (int k = 6; k <= narg; ++k) d.cols.push_back(a[k]);
        dumps_.push_back(d);
    } else if (c == "undump") {
        for (size_t k = 0; k < dumps_.size(); ++k)
            if (dumps_[k].id == a[1]) {
                dumps_.erase(dumps_.begin() + k);
                break;
            }
    } else if (c == "write_data") {
        if (narg < 1) parse_error("Illegal write_data command");
        write_data(a[1]);
    } else if (c == "print") {
        for (int k = 1; k <= narg; ++k) log += (k > 1 ? " " : "") + a[k];
        log += "\n";
    } else if (c == "newton" || c == "comm_modify" || c == "atom_modify" || c == "thermo_style" ||
               c == "thermo_modify" || c == "log" || c == "processors" || c == "dump_modify" ||
               c == "special_bonds" || c == "package" || c == "suffix" || c == "clear") {
        // accepted: no effect on this path (newton is forced off by run_style mvv/meso)
    } else {
        parse_error("Unknown command: " + line);
    }
}

// ---------------------------------------------------------------------------
// device lifecycle and run
// ---------------------------------------------------------------------------
void Script::sync_host()
{
    if (!box_ || dirty_) return;
    const int n = box_->n;
    std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n);
    std::vector<int32_t> tag(n), type(n), mask(n);
    box_->download_state(x.data(), v.data(), nullptr, tag.data(), type.data(), mask.data());
    // back to tag order (tags 1..n)
    for (int i = 0; i < n; ++i) {
        const int t = tag[i] - 1;
        if (t < 0 || t >= n) continue;
        for (int d = 0; d < 3; ++d) {
            parts_.x[3 * t + d] = x[3 * i + d];
            parts_.v[3 * t + d] = v[3 * i + d];
        }
        parts_.tag[t] = tag[i];
        parts_.type[t] = type[i];
        parts_.mask[t] = mask[i];
    }
    step_ = box_->state().step;
}

void Script::ensure_device()
{
    if (!dirty_ && box_) return;
    if (!box_defined_) throw ScriptError(MDPD_ERR_STATE, "Run command before simulation box is defined");
    if (!pair_set_) throw ScriptError(MDPD_ERR_STATE, "Pair style is not defined");
    if (parts_.size() == 0) throw ScriptError(MDPD_ERR_STATE, "No atoms in the system");
    // tag order for deterministic layout
    std::vector<size_t> ord(parts_.size());
    for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](size_t p, size_t q) { return parts_.tag[p] < parts_.tag[q]; });
    Particles p;
    for (size_t k : ord) {
        p.x.insert(p.x.end(), &parts_.x[3 * k], &parts_.x[3 * k] + 3);
        p.v.insert(p.v.end(), &parts_.v[3 * k], &parts_.v[3 * k] + 3);
        p.tag.push_back(parts_.tag[k]);
        p.type.push_back(parts_.type[k]);
        p.mask.push_back(parts_.mask[k] | 1);
    }
    parts_ = p;
    batch_.reset();
    box_.reset();
    if (!device_ready_) {
        if (device_ >= 0) check_cuda(cudaSetDevice(device_), "set device");
        cfg.sms = sm_count();
        device_ready_ = true;
    }
    for (DensityFix &d : dens_)
        if (!d.d_counts) {
            check_cuda(cudaMalloc(&d.d_counts, sizeof(unsigned long long) * d.nbin), "density fix");
            check_cuda(cudaMemset(d.d_counts, 0, sizeof(unsigned long long) * d.nbin), "density fix");
        }
    cfg.style = spec_.style;
    cfg.exact_rng = spec_.exact_rng;
    cfg.wall = spec_.wall_fix;
    cfg.aboundary = spec_.ab_mobile_bit != 0;
    cfg.wall_coupling = spec_.arb_bc;
    box_.reset(new Box(spec_, parts_, cfg.sms));
    // device step counter starts at the script's current step
    BoxState st{};
    st.step = step_;
    check_cuda(cudaMemcpy(box_->d_state, &st, sizeof(st), cudaMemcpyHostToDevice), "state");
    batch_.reset(new Batch({box_.get()}, cfg));
    dirty_ = false;
}

void Script::setup()
{
    ensure_device();
    batch_->setup();
    std::string msg;
    const int st = batch_->status(msg);
    if (st) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
}

void Script::thermo(Thermo &t)
{
    ensure_device();
    std::vector<Thermo> v;
    batch_->thermo(v);
    t = v[0];
}

void Script::emit_thermo(bool header)
{
    Thermo t;
    thermo(t);
    char b[256];
    if (header) log += "Step Temp E_pair E_mol TotEng Press \n";
    const double n = t.n > 0 ? t.n : 1;
    const double ke = 0.5 * (3.0 * t.n - 3.0) * t.temp;
    std::snprintf(b, sizeof(b), "%8lld %12.8g %12.8g %12.8g %12.8g %12.8g \n", t.step, t.temp, t.pe / n, 0.0,
                  (t.pe + ke) / n, t.press);
    log += b;
}

void Script::density_sample(long long step)
{
    for (DensityFix &d : dens_) {
        const long long n = (step + d.every / 2) / d.every, m = n * d.every;
        if (step - m >= -d.window && step - m < d.window) {
            const double bs = (spec_.hi[d.along] - spec_.lo[d.along]) / d.nbin;
            launch_density_profile(batch_->stream(), batch_->d_boxes, 0, batch_->units.local.d,
                                   batch_->units.local.n, d.along, d.group, spec_.lo[d.along], 1.0 / bs, d.nbin,
                                   d.d_counts);
            d.frames++;
        } else if (step - m == d.window) {
            density_dump(d, m);
        }
    }
}

void Script::density_dump(DensityFix &d, long long stamp)
{
    // MesoFixDensityProf::dump (fix_density_profile_meso.cpp:190-219)
    d.last_dump = step_;
    check_cuda(cudaStreamSynchronize(batch_ ? batch_->stream() : 0), "density dump");
    check_cuda(cudaMemcpy(d.counts.data(), d.d_counts, sizeof(unsigned long long) * d.nbin, cudaMemcpyDeviceToHost),
               "density dump");
    check_cuda(cudaMemset(d.d_counts, 0, sizeof(unsigned long long) * d.nbin), "density dump");
    char fn[512];
    std::snprintf(fn, sizeof(fn), "%s.%09lld", d.output.c_str(), stamp);
    std::ofstream f(fn);
    f << std::setprecision(15);
    const double bs = (spec_.hi[d.along] - spec_.lo[d.along]) / d.nbin;
    for (int i = 0; i < d.nbin; ++i) f << (i + 0.5) * bs << '\t' << d.counts[i] / float(d.frames) << std::endl;
    d.frames = 0;
}

void Script::write_dump(const DumpSpec &d)
{
    sync_host();
    std::ofstream f(d.file, std::ios::app);
    const size_t n = parts_.size();
    size_t cnt = 0;
    for (size_t i = 0; i < n; ++i) cnt += (parts_.mask[i] & d.group) != 0;
    f << "ITEM: TIMESTEP\n" << step_ << "\nITEM: NUMBER OF ATOMS\n" << cnt << "\nITEM: BOX BOUNDS pp pp pp\n";
    f << std::setprecision(16);
    for (int k = 0; k < 3; ++k) f << spec_.lo[k] << " " << spec_.hi[k] << "\n";
    f << "ITEM: ATOMS";
    for (const std::string &col : d.cols) f << " " << col;
    f << "\n" << std::setprecision(8);
    for (size_t i = 0; i < n; ++i) {
        if (!(parts_.mask[i] & d.group)) continue;
        for (size_t k = 0; k < d.cols.size(); ++k) {
            const std::string &col = d.cols[k];
            if (k) f << " ";
            if (col == "id") f << parts_.tag[i];
            else if (col == "type") f << parts_.type[i];
            else if (col == "x" || col == "y" || col == "z") f << parts_.x[3 * i + (col[0] - 'x')];
            else if (col == "xs" || col == "ys" || col == "zs") {
                const int dd = col[0] - 'x';
                f << (parts_.x[3 * i + dd] - spec_.lo[dd]) / (spec_.hi[dd] - spec_.lo[dd]);
            } else if (col == "vx" || col == "vy" || col == "vz") f << parts_.v[3 * i + (col[1] - 'x')];
            else f << 0;
        }
        f << "\n";
    }
}

void Script::write_data(const std::string &path)
{
    // AtomVecMDPDAtomic::data_atom format (atom_vec_mdpd_atomic_meso.cu:609-637): id type x y z
    sync_host();
    std::ofstream f(path);
    if (!f) throw ScriptError(MDPD_ERR_ARG, "Cannot open data file " + path);
    f << "LAMMPS data file via write_data, timestep = " << step_ << "\n\n";
    f << parts_.size() << " atoms\n" << spec_.ntype << " atom types\n\n";
    f << std::setprecision(16) << std::scientific;
    const char *ax[3] = {"xlo xhi", "ylo yhi", "zlo zhi"};
    for (int d = 0; d < 3; ++d) f << spec_.lo[d] << " " << spec_.hi[d] << " " << ax[d] << "\n";
    f << "\nMasses\n\n";
    for (int t = 0; t < spec_.ntype; ++t) f << t + 1 << " " << spec_.mass[t] << "\n";
    f << "\nAtoms\n\n";
    for (size_t i = 0; i < parts_.size(); ++i)
        f << parts_.tag[i] << " " << parts_.type[i] << " " << parts_.x[3 * i] << " " << parts_.x[3 * i + 1] << " "
          << parts_.x[3 * i + 2] << "\n";
    f << "\nVelocities\n\n";
    for (size_t i = 0; i < parts_.size(); ++i)
        f << parts_.tag[i] << " " << parts_.v[3 * i] << " " << parts_.v[3 * i + 1] << " " << parts_.v[3 * i + 2]
          << "\n";
}

void Script::read_data(const std::string &path)
{
    std::ifstream f(path);
    if (!f) throw ScriptError(MDPD_ERR_ARG, "Cannot open file " + path);
    std::string line;
    std::getline(f, line);  // title
    long long natoms = 0;
    int ntypes = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    std::string section;
    // header
    while (std::getline(f, line)) {
        std::string t = line.substr(0, line.find('#'));
        std::vector<std::string> w = split(t);
        if (w.empty()) continue;
        if (w.size() >= 2 && w[1] == "atoms") natoms = std::stoll(w[0]);
        else if (w.size() >= 3 && w[1] == "atom" && w[2] == "types") ntypes = std::stoi(w[0]);
        else if (w.size() >= 4 && w[2] == "xlo") lo[0] = num(w[0]), hi[0] = num(w[1]);
        else if (w.size() >= 4 && w[2] == "ylo") lo[1] = num(w[0]), hi[1] = num(w[1]);
        else if (w.size() >= 4 && w[2] == "zlo") lo[2] = num(w[0]), hi[2] = num(w[1]);
        else {
            section = w[0];
            break;
        }
    }
    if (ntypes < 1 || ntypes > kMaxTypes) parse_error("read_data: 1..8 atom types supported");
    spec_.ntype = ntypes;
    for (int d = 0; d < 3; ++d) spec_.lo[d] = lo[d], spec_.hi[d] = hi[d];
    box_defined_ = true;
    parts_ = Particles();
    std::map<int, size_t> by_tag;
    while (!section.empty()) {
        std::string next;
        long long got = 0;
        while (std::getline(f, line)) {
            std::string t = line.substr(0, line.find('#'));
            std::vector<std::string> w = split(t);
            if (w.empty()) continue;
            if (std::isalpha((unsigned char)w[0][0])) {
                next = w[0];
                break;
            }
            if (section == "Masses") {
                spec_.mass[inum(w[0]) - 1] = num(w[1]);
            } else if (section == "Atoms") {
                // atomic: id type x y z [ix iy iz]
                if (w.size() < 5) parse_error("Incorrect atom format in data file");
                const int tag = inum(w[0]), type = inum(w[1]);
                double x[3] = {num(w[2]), num(w[3]), num(w[4])};
                if (w.size() >= 8)
                    for (int d = 0; d < 3; ++d) x[d] += inum(w[5 + d]) * (hi[d] - lo[d]);
                by_tag[tag] = parts_.size();
                parts_.x.insert(parts_.x.end(), x, x + 3);
                for (int d = 0; d < 3; ++d) parts_.v.push_back(0);
                parts_.tag.push_back(tag);
                parts_.type.push_back(type);
                parts_.mask.push_back(1);
                ++got;
            } else if (section == "Velocities") {
                auto it = by_tag.find(inum(w[0]));
                if (it == by_tag.end()) parse_error("Invalid atom ID in Velocities section of data file");
                for (int d = 0; d < 3; ++d) parts_.v[3 * it->second + d] = num(w[1 + d]);
            }
        }
        if (section == "Atoms" && got != natoms) parse_error("Did not assign all atoms correctly");
        section = next;
    }
}

void Script::run(long long nsteps)
{
    ensure_device();
    // setup (ModifiedVerlet::setup): rebuild, density, forces with energy/virial
    batch_->setup();
    step_ = box_->state().step;
    std::string msg;
    if (int st = batch_->status(msg)) throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
    if (thermo_every_ >= 0) emit_thermo(true);
    for (const DumpSpec &d : dumps_)
        if (step_ % d.every == 0) write_dump(d);
    const long long end = step_ + nsteps;
    const bool per_step = !dens_.empty();
    while (step_ < end) {
        long long next = end;
        if (thermo_every_ > 0) next = std::min(next, (step_ / thermo_every_ + 1) * thermo_every_);
        for (const DumpSpec &d : dumps_) next = std::min(next, (step_ / d.every + 1) * d.every);
        const long long k = next - step_;
        const bool ev_last = (thermo_every_ > 0 && next % thermo_every_ == 0) || next == end;
        if (per_step) {
            for (long long q = 0; q < k; ++q) {
                if (q == k - 1 && ev_last) batch_->step_ev();
                else batch_->run(1, false);
                density_sample(step_ + q + 1);
            }
        } else {
            batch_->run(ev_last ? k - 1 : k, false);
            if (ev_last) batch_->step_ev();
        }
        check_cuda(cudaStreamSynchronize(batch_->stream()), "run");
        step_ = next;
        if (int st = batch_->status(msg))
            throw ScriptError(st & kErrNonFinite ? MDPD_ERR_NAN : MDPD_ERR_OVERFLOW, msg);
        if (ev_last) emit_thermo(false);
        for (const DumpSpec &d : dumps_)
            if (step_ % d.every == 0) write_dump(d);
    }
}

}  // namespace mdpd
