// rc_host.cpp -- parameters, multigrid geometry and spectral tables on the
// host.  Everything here follows the reference's host code:
//   parameters   src/param/param.h, src/param/NarrowBand.h
//   geometry     src/montecarlo/definitions.h:68-136 (Gridn::mk_grid)
//   tables       src/montecarlo/read_tables.cpp:21-96 (readT) and the
//                writers nbcorrk/write_tables.cpp:18-109, CDF formulas of
//                nbcorrk/calc_prob.cpp:68-116.
#include "rc_host.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <sstream>

#include "radchan_math.h"

namespace rc {

// ---------------------------------------------------------------------------
// parameters
// ---------------------------------------------------------------------------

int params_default(rc_params &p) {
    memset(&p, 0, sizeof(p));
    // param.h:8-20 (num_gpu/p_col reduced to the single-GPU drop-in)
    p.num_gpu = 1;
    p.p_col = 1;
    p.imax = 406;
    p.jmax = 576;
    p.kmax = 2304;
    p.Lx = 2.f;
    p.Ly = 6.283185307179586f;
    p.Lz = 37.69911184307751f;
    p.fact_mesh = 1.6;
    p.nVar = 1;
    p.photmax = 6000;
    p.chanHeight = 0.5;
    // param.h:24-49
    p.grid_num = 9;
    const int mi[9] = {406, 406, 406, 406, 406, 406 / 29, 406 / 29, 406 / 29, 406 / 203};
    const int mj[9] = {576, 576 / 3, 576 / 6, 576 / 12, 576 / 24, 576 / 48, 576 / 96, 576 / 96, 576 / 192};
    const int mk[9] = {2304, 2304 / 2, 2304 / 4, 2304 / 8, 2304 / 16, 2304 / 32, 2304 / 64, 2304 / 128, 2304 / 256};
    for (int l = 0; l < 9; ++l) {
        p.maxi[l] = mi[l];
        p.maxj[l] = mj[l];
        p.maxk[l] = mk[l];
        p.maxs[l] = (l == 8) ? 100000 : 5;
    }
    // param.h:52-65
    p.num_streams = 2;
    p.blockdim = 128;
    p.nblocks = 4096;
    p.srt = 1;
    p.grey = 0;
    p.calcwalls = 0;
    p.random = 1;
    p.floatpoint = 0;
    // param.h:68-100
    for (int w = 0; w < 6; ++w) {
        p.eps[w] = 1.f;
        p.Tw[w] = 0.f;
    }
    p.adiabw = 1;
    p.adiabe = 1;
    p.stefan = 5.670373e-08;
    p.toll = 1.0e-3f;
    p.tollS = 1.0e-3f;
    p.bd[RC_WEST] = 2;
    p.bd[RC_EAST] = 2;
    p.bd[RC_SOUTH] = 1;
    p.bd[RC_NORTH] = 1;
    p.bd[RC_BOT] = 4;
    p.bd[RC_TOP] = 4;
    // NarrowBand.h:189-191, 214-219
    p.nT = 135;
    p.nQ = 16;
    p.nB = 999;
    p.grey_nT = 65;
    p.grey_nB = 1000;
    p.abscoeff = 1.f;
    p.Tmins = 490.f;
    p.wvmax = 5000.f;
    p.seed = 1234;
    return RC_OK;
}

int params_validate(const rc_params &p, std::string &err) {
    auto bad = [&](const std::string &m) {
        err = m;
        return RC_E_INVALID;
    };
    if (p.imax < 1 || p.jmax < 1 || p.kmax < 1) return bad("imax, jmax, kmax must be >= 1");
    if (p.num_gpu != 1) return bad("num_gpu must be 1: one solve runs on one GPU");
    if (p.p_col < 1 || p.kmax % p.p_col != 0) return bad("p_col must divide kmax");
    if (p.grid_num < 1 || p.grid_num > RC_MAX_LEVELS) return bad("grid_num must be in [1, 9]");
    if (p.maxi[0] != p.imax || p.maxj[0] != p.jmax || p.maxk[0] != p.kmax)
        return bad("level 0 must be the full grid (maxi[0]=imax, maxj[0]=jmax, maxk[0]=kmax)");
    for (int l = 0; l < p.grid_num; ++l) {
        if (p.maxi[l] < 1 || p.maxj[l] < 1 || p.maxk[l] < 1) return bad("grid level sizes must be >= 1");
        if (p.imax % p.maxi[l] || p.jmax % p.maxj[l] || p.kmax % p.maxk[l])
            return bad("every level must divide the fine grid (param.h:26)");
        if (l > 0 && (p.maxi[l - 1] % p.maxi[l] || p.maxj[l - 1] % p.maxj[l] || p.maxk[l - 1] % p.maxk[l]))
            return bad("each level must divide the previous one (param.h:26)");
        if (p.maxs[l] < 0) return bad("maxs must be >= 0");
    }
    if (p.maxs[p.grid_num - 1] < 1) return bad("the last level needs maxs >= 1");
    if (p.nVar < 1) return bad("nVar must be >= 1");
    if (p.photmax < 1) return bad("photmax must be >= 1");
    if (!(p.Lx > 0 && p.Ly > 0 && p.Lz > 0)) return bad("Lx, Ly, Lz must be > 0");
    for (int w = 0; w < 6; ++w)
        if (p.bd[w] < 1 || p.bd[w] > 5) return bad("bd values must be in 1..5");
    if (!(p.toll > 0 && p.toll < 1) || !(p.tollS > 0 && p.tollS < 1)) return bad("toll, tollS must be in (0,1)");
    if (p.grey) {
        if (p.grey_nT < 2 || p.grey_nB < 1) return bad("grey_nT >= 2 and grey_nB >= 1 required");
        if (!(p.abscoeff >= 0)) return bad("abscoeff must be >= 0");
    } else {
        if (p.nT < 2 || p.nB < 1 || p.nQ < 1) return bad("nT >= 2, nB >= 1, nQ >= 1 required");
    }
    if (p.floatpoint != 0 && p.floatpoint != 1) return bad("floatpoint must be 0 or 1");
    // 2 * 1 bits of kind and 24 bits of replicate in the Philox counter
    if (p.nVar > (1 << 24)) return bad("nVar too large");
    return RC_OK;
}

void wall_types(const rc_params &p, int wt[6]) {
    for (int w = 0; w < 6; ++w) {
        int b = p.bd[w];
        int adiab = (w == RC_WEST) ? p.adiabw : (w == RC_EAST) ? p.adiabe : 0;
        if (b == 2)
            wt[w] = adiab ? WT_BLACK_FACE : WT_BLACK_FIXED;
        else
            wt[w] = b;
    }
}

// ---------------------------------------------------------------------------
// param.h / NarrowBand.h parser: #define, #if/#elif/#else/#endif and the
// brace initialisers of maxi/maxj/maxk/maxs/gq/wq.
// ---------------------------------------------------------------------------
namespace {

struct Val {
    double v = 0;
    bool isint = true;
};

struct Expr {
    std::vector<std::string> tok;
    size_t pos = 0;
    const std::map<std::string, std::string> *defs;
    int depth = 0;
    bool ok = true;

    static std::vector<std::string> lex(const std::string &s) {
        std::vector<std::string> t;
        size_t i = 0;
        while (i < s.size()) {
            char c = s[i];
            if (isspace((unsigned char)c)) {
                ++i;
                continue;
            }
            if (isdigit((unsigned char)c) || (c == '.' && i + 1 < s.size() && isdigit((unsigned char)s[i + 1]))) {
                size_t j = i;
                while (j < s.size() && (isalnum((unsigned char)s[j]) || s[j] == '.' ||
                                        ((s[j] == '-' || s[j] == '+') && (s[j - 1] == 'e' || s[j - 1] == 'E'))))
                    ++j;
                t.push_back(s.substr(i, j - i));
                i = j;
                continue;
            }
            if (isalpha((unsigned char)c) || c == '_') {
                size_t j = i;
                while (j < s.size() && (isalnum((unsigned char)s[j]) || s[j] == '_')) ++j;
                t.push_back(s.substr(i, j - i));
                i = j;
                continue;
            }
            if (i + 1 < s.size()) {
                std::string two = s.substr(i, 2);
                if (two == "==" || two == "!=" || two == "<=" || two == ">=" || two == "&&" || two == "||") {
                    t.push_back(two);
                    i += 2;
                    continue;
                }
            }
            t.push_back(std::string(1, c));
            ++i;
        }
        return t;
    }
    const std::string &peek() {
        static const std::string end;
        return pos < tok.size() ? tok[pos] : end;
    }
    Val number(const std::string &s) {
        Val r;
        std::string t = s;
        bool flt = false;
        while (!t.empty() && (t.back() == 'f' || t.back() == 'F' || t.back() == 'u' || t.back() == 'U' ||
                              t.back() == 'l' || t.back() == 'L')) {
            if (t.back() == 'f' || t.back() == 'F') flt = true;
            t.pop_back();
        }
        if (t.find_first_of(".eE") != std::string::npos) flt = true;
        r.v = strtod(t.c_str(), nullptr);
        r.isint = !flt;
        return r;
    }
    Val eval_ident(const std::string &name) {
        auto it = defs->find(name);
        if (it == defs->end() || depth > 32) {
            ok = false;
            return Val{0, true};
        }
        Expr sub;
        sub.tok = lex(it->second);
        sub.defs = defs;
        sub.depth = depth + 1;
        Val r = sub.parse_or();
        if (!sub.ok) ok = false;
        return r;
    }
    Val primary() {
        std::string t = peek();
        if (t.empty()) {
            ok = false;
            return Val{};
        }
        ++pos;
        if (t == "(") {
            Val r = parse_or();
            if (peek() == ")") ++pos;
            else ok = false;
            return r;
        }
        if (t == "-") {
            Val r = primary();
            r.v = -r.v;
            return r;
        }
        if (t == "+") return primary();
        if (t == "!") {
            Val r = primary();
            return Val{r.v == 0 ? 1.0 : 0.0, true};
        }
        if (isdigit((unsigned char)t[0]) || t[0] == '.') return number(t);
        if (t == "defined") {
            bool par = peek() == "(";
            if (par) ++pos;
            std::string n = peek();
            ++pos;
            if (par && peek() == ")") ++pos;
            return Val{defs->count(n) ? 1.0 : 0.0, true};
        }
        return eval_ident(t);
    }
    Val mul() {
        Val a = primary();
        while (peek() == "*" || peek() == "/") {
            std::string op = peek();
            ++pos;
            Val b = primary();
            if (op == "*") {
                a.v *= b.v;
                a.isint = a.isint && b.isint;
            } else {
                if (a.isint && b.isint) {
                    if ((long long)b.v == 0) {
                        ok = false;
                        return a;
                    }
                    a.v = (double)((long long)a.v / (long long)b.v);
                } else {
                    a.v /= b.v;
                    a.isint = false;
                }
            }
        }
        return a;
    }
    Val add() {
        Val a = mul();
        while (peek() == "+" || peek() == "-") {
            std::string op = peek();
            ++pos;
            Val b = mul();
            a.v = (op == "+") ? a.v + b.v : a.v - b.v;
            a.isint = a.isint && b.isint;
        }
        return a;
    }
    Val cmp() {
        Val a = add();
        while (peek() == "==" || peek() == "!=" || peek() == "<" || peek() == ">" || peek() == "<=" ||
               peek() == ">=") {
            std::string op = peek();
            ++pos;
            Val b = add();
            bool r = op == "==" ? a.v == b.v : op == "!=" ? a.v != b.v : op == "<" ? a.v < b.v
                     : op == ">"  ? a.v > b.v : op == "<=" ? a.v <= b.v : a.v >= b.v;
            a = Val{r ? 1.0 : 0.0, true};
        }
        return a;
    }
    Val land() {
        Val a = cmp();
        while (peek() == "&&") {
            ++pos;
            Val b = cmp();
            a = Val{(a.v != 0 && b.v != 0) ? 1.0 : 0.0, true};
        }
        return a;
    }
    Val parse_or() {
        Val a = land();
        while (peek() == "||") {
            ++pos;
            Val b = land();
            a = Val{(a.v != 0 || b.v != 0) ? 1.0 : 0.0, true};
        }
        return a;
    }
};

std::string strip_comments(const std::string &src) {
    std::string out;
    out.reserve(src.size());
    size_t i = 0;
    while (i < src.size()) {
        if (src.compare(i, 2, "/*") == 0) {
            size_t e = src.find("*/", i + 2);
            i = (e == std::string::npos) ? src.size() : e + 2;
            out += ' ';
            continue;
        }
        if (src.compare(i, 2, "//") == 0) {
            size_t e = src.find('\n', i);
            i = (e == std::string::npos) ? src.size() : e;
            continue;
        }
        out += src[i++];
    }
    return out;
}

struct Preproc {
    std::map<std::string, std::string> defs;
    std::map<std::string, std::vector<std::string>> arrays;  // name -> element expressions
    std::string err;

    bool eval(const std::string &e, Val &v) {
        Expr x;
        x.tok = Expr::lex(e);
        x.defs = &defs;
        v = x.parse_or();
        return x.ok && x.pos == x.tok.size();
    }

    bool run(const std::string &raw) {
        std::string src = strip_comments(raw);
        // join continuation lines
        std::string joined;
        for (size_t i = 0; i < src.size(); ++i) {
            if (src[i] == '\\' && i + 1 < src.size() && src[i + 1] == '\n') {
                ++i;
                continue;
            }
            joined += src[i];
        }
        std::istringstream in(joined);
        std::string line;
        struct Cond {
            bool active, taken, parent;
        };
        std::vector<Cond> st;
        auto active = [&]() { return st.empty() || st.back().active; };
        std::string pending;  // accumulates a brace initialiser across lines
        while (std::getline(in, line)) {
            std::string s = line;
            size_t a = s.find_first_not_of(" \t\r");
            if (a == std::string::npos) continue;
            s = s.substr(a);
            if (s[0] == '#') {
                std::string d = s.substr(1);
                size_t b = d.find_first_not_of(" \t");
                d = (b == std::string::npos) ? "" : d.substr(b);
                auto word = [&](const std::string &w) {
                    return d.compare(0, w.size(), w) == 0 &&
                           (d.size() == w.size() || isspace((unsigned char)d[w.size()]) || d[w.size()] == '(');
                };
                if (word("ifdef") || word("ifndef")) {
                    std::string n = d.substr(word("ifdef") ? 5 : 6);
                    n.erase(0, n.find_first_not_of(" \t"));
                    n = n.substr(0, n.find_first_of(" \t\r"));
                    bool c = defs.count(n) > 0;
                    if (word("ifndef")) c = !c;
                    bool par = active();
                    st.push_back({par && c, c, par});
                } else if (word("if")) {
                    Val v;
                    bool par = active();
                    bool c = false;
                    if (par) {
                        if (!eval(d.substr(2), v)) {
                            err = "cannot evaluate #if " + d.substr(2);
                            return false;
                        }
                        c = v.v != 0;
                    }
                    st.push_back({par && c, c, par});
                } else if (word("elif")) {
                    if (st.empty()) {
                        err = "#elif without #if";
                        return false;
                    }
                    Cond &c = st.back();
                    if (c.parent && !c.taken) {
                        Val v;
                        if (!eval(d.substr(4), v)) {
                            err = "cannot evaluate #elif " + d.substr(4);
                            return false;
                        }
                        c.active = v.v != 0;
                        c.taken = c.active;
                    } else {
                        c.active = false;
                    }
                } else if (word("else")) {
                    if (st.empty()) {
                        err = "#else without #if";
                        return false;
                    }
                    Cond &c = st.back();
                    c.active = c.parent && !c.taken;
                    c.taken = true;
                } else if (word("endif")) {
                    if (st.empty()) {
                        err = "#endif without #if";
                        return false;
                    }
                    st.pop_back();
                } else if (word("define") && active()) {
                    std::string r = d.substr(6);
                    r.erase(0, r.find_first_not_of(" \t"));
                    size_t e = 0;
                    while (e < r.size() && (isalnum((unsigned char)r[e]) || r[e] == '_')) ++e;
                    std::string name = r.substr(0, e);
                    if (e < r.size() && r[e] == '(') continue;  // function-like macro: ignored
                    std::string val = r.substr(e);
                    val.erase(0, val.find_first_not_of(" \t"));
                    while (!val.empty() && isspace((unsigned char)val.back())) val.pop_back();
                    defs[name] = val;
                } else if (word("undef") && active()) {
                    std::string n = d.substr(5);
                    n.erase(0, n.find_first_not_of(" \t"));
                    n = n.substr(0, n.find_first_of(" \t\r"));
                    defs.erase(n);
                }
                continue;
            }
            if (!active()) continue;
            // array initialisers: "... name[...] = { e1, e2, ... };" possibly over lines
            if (!pending.empty() || s.find('{') != std::string::npos) {
                pending += " " + s;
                if (pending.find('}') == std::string::npos) continue;
                size_t eq = pending.find('=');
                size_t lb = pending.find('{'), rb = pending.find('}');
                if (eq != std::string::npos && lb != std::string::npos && eq < lb) {
                    std::string lhs = pending.substr(0, eq);
                    size_t br = lhs.find('[');
                    std::string head = lhs.substr(0, br == std::string::npos ? lhs.size() : br);
                    while (!head.empty() && isspace((unsigned char)head.back())) head.pop_back();
                    size_t ns = head.find_last_of(" \t");
                    std::string name = (ns == std::string::npos) ? head : head.substr(ns + 1);
                    std::string body = pending.substr(lb + 1, rb - lb - 1);
                    std::vector<std::string> items;
                    std::string cur;
                    for (char c : body) {
                        if (c == ',') {
                            items.push_back(cur);
                            cur.clear();
                        } else {
                            cur += c;
                        }
                    }
                    if (cur.find_first_not_of(" \t\r\n") != std::string::npos) items.push_back(cur);
                    arrays[name] = items;
                }
                pending.clear();
            }
        }
        if (!st.empty()) {
            err = "unterminated #if";
            return false;
        }
        return true;
    }
};

template <typename T>
bool get_num(Preproc &pp, const char *name, T &out) {
    if (!pp.defs.count(name)) return false;
    Val v;
    if (!pp.eval(name, v)) return false;
    out = (T)v.v;
    return true;
}

bool read_file(const std::string &path, std::string &out) {
    std::ifstream f(path);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

}  // namespace

int params_from_headers(const std::string &param_h, const std::string &nb_h, rc_params &p, std::string &err) {
    params_default(p);
    std::string src;
    if (!read_file(param_h, src)) {
        err = "cannot read " + param_h;
        return RC_E_IO;
    }
    std::string nb;
    if (!nb_h.empty()) {
        if (!read_file(nb_h, nb)) {
            err = "cannot read " + nb_h;
            return RC_E_IO;
        }
    }
    // param.h includes NarrowBand.h only through definitions.h; evaluating
    // param.h first and NarrowBand.h second matches the include order of
    // the reference translation units.
    Preproc pp;
    pp.defs["myfloat"] = "float";
    if (!pp.run(src)) {
        err = param_h + ": " + pp.err;
        return RC_E_INVALID;
    }
    if (!nb.empty() && !pp.run(nb)) {
        err = nb_h + ": " + pp.err;
        return RC_E_INVALID;
    }
    int num_gpu = 1;
    get_num(pp, "num_gpu", num_gpu);
    get_num(pp, "p_col", p.p_col);
    get_num(pp, "imax", p.imax);
    get_num(pp, "jmax", p.jmax);
    get_num(pp, "kmax", p.kmax);
    get_num(pp, "Lx", p.Lx);
    get_num(pp, "Ly", p.Ly);
    get_num(pp, "Lz", p.Lz);
    get_num(pp, "fact_mesh", p.fact_mesh);
    get_num(pp, "nVar", p.nVar);
    get_num(pp, "photmax", p.photmax);
    get_num(pp, "chanHeight", p.chanHeight);
    get_num(pp, "grid_num", p.grid_num);
    get_num(pp, "num_streams", p.num_streams);
    get_num(pp, "blockdim", p.blockdim);
    get_num(pp, "nblocks", p.nblocks);
    get_num(pp, "srt", p.srt);
    get_num(pp, "grey", p.grey);
    get_num(pp, "calcwalls", p.calcwalls);
    get_num(pp, "random", p.random);
    get_num(pp, "floatpoint", p.floatpoint);
    const char *en[6] = {"epsw", "epse", "epss", "epsn", "epsb", "epst"};
    const char *tn[6] = {"Tww", "Twe", "Tws", "Twn", "Twb", "Twt"};
    const char *bn[6] = {"bdw", "bde", "bds", "bdn", "bdb", "bdt"};
    for (int w = 0; w < 6; ++w) {
        get_num(pp, en[w], p.eps[w]);
        get_num(pp, tn[w], p.Tw[w]);
        get_num(pp, bn[w], p.bd[w]);
    }
    get_num(pp, "adiabw", p.adiabw);
    get_num(pp, "adiabe", p.adiabe);
    get_num(pp, "stefan", p.stefan);
    get_num(pp, "toll", p.toll);
    get_num(pp, "tollS", p.tollS);
    if (p.grey) {
        get_num(pp, "nT", p.grey_nT);
        get_num(pp, "nB", p.grey_nB);
        get_num(pp, "abscoeff", p.abscoeff);
        get_num(pp, "Tmins", p.Tmins);
        get_num(pp, "wvmax", p.wvmax);
    } else {
        get_num(pp, "nT", p.nT);
        get_num(pp, "nQ", p.nQ);
        get_num(pp, "nB", p.nB);
    }
    // the parser keeps the one maxs initialiser of the active #if branch
    const char *an[4] = {"maxi", "maxj", "maxk", "maxs"};
    int *dst[4] = {p.maxi, p.maxj, p.maxk, p.maxs};
    for (int a = 0; a < 4; ++a) {
        auto it = pp.arrays.find(an[a]);
        if (it == pp.arrays.end()) continue;
        for (size_t l = 0; l < it->second.size() && l < RC_MAX_LEVELS; ++l) {
            Val v;
            if (!pp.eval(it->second[l], v)) {
                err = std::string("cannot evaluate ") + an[a] + "[" + std::to_string(l) + "]";
                return RC_E_INVALID;
            }
            dst[a][l] = (int)v.v;
        }
    }
    if (num_gpu != 1) {
        // the drop-in runs the whole domain on one GPU (one solve per GPU)
        p.num_gpu = 1;
    }
    return RC_OK;
}

// ---------------------------------------------------------------------------
// geometry: restatement of Gridn::mk_grid (definitions.h:68-136), keeping
// its mix of float storage and double intermediate arithmetic.
// ---------------------------------------------------------------------------
void build_grid_level(const rc_params &p, int level, GridLevel &g) {
    const int im = p.maxi[level], jm = p.maxj[level], km = p.maxk[level], im0 = p.maxi[0];
    g.im = im;
    g.jm = jm;
    g.km = km;
    g.maxs = p.maxs[level];
    g.x.assign(im + 2, 0.f);
    g.xu.assign(im + 1, 0.f);
    g.y.assign(jm + 2, 0.f);
    g.z.assign(km + 2, 0.f);
    g.yu.assign(jm + 1, 0.f);
    g.zu.assign(km + 1, 0.f);
    std::vector<float> xu0(im0 + 1, 0.f);

    const float dy = p.Ly * 1.0f / jm;  // definitions.h:85-86
    const float dz = p.Lz * 1.0f / km;
    for (int i = 0; i < jm + 1; i++) g.yu[i] = i * dy;
    for (int i = 0; i < km + 1; i++) g.zu[i] = i * dz;
    g.y[0] = -dy / 2;
    g.z[0] = -dz / 2;
    for (int i = 1; i < jm + 1; i++) g.y[i] = (g.yu[i - 1] + g.yu[i]) / 2;
    for (int i = 1; i < km + 1; i++) g.z[i] = (g.zu[i - 1] + g.zu[i]) / 2;
    g.y[jm + 1] = g.y[jm] + dy;
    g.z[km + 1] = g.z[km] + dz;

    // parabolic face spacing dx = 0.5 - fact_mesh (r - 0.5)^2 (definitions.h:108-123)
    xu0[0] = 0;
    for (int i = 1; i < im0 / 2 + 1; i++) {
        float r = (1.f * i) / im0;
        float dx = (float)(0.5 - p.fact_mesh * ((double)r - 0.5) * ((double)r - 0.5));
        xu0[i] = xu0[i - 1] + dx;
    }
    const float xnorm = xu0[im0 / 2];
    for (int i = 1; i < im0 / 2 + 1; i++) xu0[i] = (float)((double)p.Lx / 2. * (double)xu0[i] / (double)xnorm);
    for (int i = im0; i > im0 / 2; i--) xu0[i] = p.Lx - xu0[im0 - i];

    g.xu[0] = 0;
    for (int i = 1; i < im + 1; i++) g.xu[i] = xu0[(long long)i * im0 / im];
    for (int i = 1; i < im + 1; i++) g.x[i] = (float)(0.5 * (double)(g.xu[i] + g.xu[i - 1]));
    g.x[0] = -g.x[1];
    g.x[im + 1] = g.xu[im] + (g.xu[im] - g.x[im]);
}

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------
void TableSet::view(rc_tables *t) const {
    t->nT = nT;
    t->nB = nB;
    t->nQ = nQ;
    t->Tnb = Tnb.data();
    t->kP = kP.data();
    t->wvl = wvl.data();
    t->wvr = wvr.data();
    t->wvc = wvc.data();
    t->kavg = kavg.data();
    t->kq = kq.data();
    t->prob = prob.data();
    t->probg = probg.data();
    t->wq = wq.data();
}

void TableSet::from_view(const rc_tables *t) {
    nT = t->nT;
    nB = t->nB;
    nQ = t->nQ;
    auto cp = [](std::vector<float> &v, const float *s, size_t n) {
        if (s) v.assign(s, s + n);
        else v.assign(n, 0.f);
    };
    cp(Tnb, t->Tnb, nT);
    cp(kP, t->kP, nT);
    kR.assign(nT, 0.f);
    kM.assign(nT, 0.f);
    cp(wvl, t->wvl, nB);
    cp(wvr, t->wvr, nB);
    cp(wvc, t->wvc, nB);
    cp(kavg, t->kavg, nB);
    cp(kq, t->kq, (size_t)nB * nT * nQ);
    cp(prob, t->prob, (size_t)nT * nB);
    cp(probg, t->probg, (size_t)nT * nB * nQ);
    cp(wq, t->wq, nQ);
    gq.assign(nQ, 0.f);
    kavg_t.assign((size_t)nT * nB, 0.f);
    for (int b = 0; b < nB; ++b) kavg_t[(size_t)(nT - 1) * nB + b] = kavg[b];
}

double synth_uniform(uint64_t seed, uint32_t stream, uint32_t idx) {
    rc_u32x4 c = {idx, stream, 0x5eedu, 0u};
    rc_u32x4 r = rc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t hi = r.x >> 5, lo = r.y >> 6;  // 27 + 26 = 53 bits
    return (double)(hi * 67108864ull + lo) * (1.0 / 9007199254740992.0);
}

void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = cos(RC_PI_D * (i + 0.75) / (n + 0.5));
        double pp = 0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-15) break;
        }
        x[n - 1 - i] = z;  // ascending
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

int tables_synthetic(const rc_synth_spec &s, TableSet &t, std::string &err) {
    if (s.nB < 1 || s.nQ < 1 || s.nT < 2 || !(s.T_hi > s.T_lo) || !(s.T_lo > 0) || !(s.nu_hi > s.nu_lo) ||
        !(s.nu_lo > 0)) {
        err = "invalid synthetic table spec";
        return RC_E_INVALID;
    }
    const int nB = s.nB, nQ = s.nQ, nT = s.nT;
    t.nB = nB;
    t.nQ = nQ;
    t.nT = nT;
    std::vector<double> xi, wgl;
    gauss_legendre(nQ, xi, wgl);
    t.wq.resize(nQ);
    t.gq.resize(nQ);
    std::vector<double> wqd(nQ);
    for (int g = 0; g < nQ; ++g) {
        wqd[g] = wgl[g] / 2.0;
        t.wq[g] = (float)wqd[g];
        t.gq[g] = (float)((xi[g] + 1.0) / 2.0);
    }
    // band centres ~ U[nu_lo, nu_hi], sorted; edges at the midpoints
    std::vector<double> nu(nB), k0(nB), nexp(nB);
    for (int b = 0; b < nB; ++b) nu[b] = s.nu_lo + (s.nu_hi - s.nu_lo) * synth_uniform(s.seed, 1, b);
    std::sort(nu.begin(), nu.end());
    for (int b = 0; b < nB; ++b) {
        k0[b] = pow(10.0, s.logk_lo + (s.logk_hi - s.logk_lo) * synth_uniform(s.seed, 2, b));
        nexp[b] = -s.nexp + 2.0 * s.nexp * synth_uniform(s.seed, 3, b);
    }
    std::vector<double> el(nB), er(nB);
    for (int b = 0; b < nB; ++b) {
        el[b] = (b == 0) ? s.nu_lo : 0.5 * (nu[b - 1] + nu[b]);
        er[b] = (b == nB - 1) ? s.nu_hi : 0.5 * (nu[b] + nu[b + 1]);
    }
    t.wvl.resize(nB);
    t.wvr.resize(nB);
    t.wvc.resize(nB);
    for (int b = 0; b < nB; ++b) {
        t.wvl[b] = (float)el[b];
        t.wvr[b] = (float)er[b];
        t.wvc[b] = (float)nu[b];
    }
    t.Tnb.resize(nT);
    std::vector<double> Td(nT);
    for (int i = 0; i < nT; ++i) {
        Td[i] = s.T_lo + (s.T_hi - s.T_lo) * i / (double)(nT - 1);
        t.Tnb[i] = (float)Td[i];
    }
    const double stefan = 5.670373e-08;
    t.kq.assign((size_t)nB * nT * nQ, 0.f);
    t.prob.assign((size_t)nT * nB, 0.f);
    t.probg.assign((size_t)nT * nB * nQ, 0.f);
    t.kP.assign(nT, 0.f);
    t.kR.assign(nT, 0.f);
    t.kM.assign(nT, 0.f);
    t.kavg.assign(nB, 0.f);
    t.kavg_t.assign((size_t)nT * nB, 0.f);
    std::vector<double> kqd((size_t)nB * nQ), bandp(nB);
    for (int i = 0; i < nT; ++i) {
        const double T = Td[i];
        double total = 0.0;
        for (int b = 0; b < nB; ++b) {
            double ib = rc_planck(T, nu[b]);
            double dnu = (er[b] - el[b]) * 100.0;
            double kav = 0.0, pb = 0.0;
            for (int g = 0; g < nQ; ++g) {
                double k = k0[b] * exp(s.kexp * xi[g]) * pow(T / 1000.0, nexp[b]);
                kqd[(size_t)b * nQ + g] = k;
                t.kq[((size_t)b * nT + i) * nQ + g] = (float)k;
                kav += wqd[g] * k;
                pb += wqd[g] * k * ib * dnu;
            }
            t.kavg_t[(size_t)i * nB + b] = (float)kav;
            bandp[b] = pb;
            total += pb;
            // g cumulative probability ~ k_g w_g (calc_prob.cpp:97-116)
            double cg = 0.0, sg = 0.0;
            for (int g = 0; g < nQ; ++g) sg += kqd[(size_t)b * nQ + g] * wqd[g];
            for (int g = 0; g < nQ; ++g) {
                cg += kqd[(size_t)b * nQ + g] * wqd[g];
                t.probg[((size_t)i * nB + b) * nQ + g] = (g == nQ - 1) ? 1.0f : (float)(cg / sg);
            }
        }
        // Planck-mean coefficient and band cumulative probability
        // (calc_prob.cpp:54-86): pi sum k I_b dnu / (sigma T^4)
        t.kP[i] = (float)(RC_PI_D * total / (stefan * T * T * T * T));
        double c = 0.0;
        for (int b = 0; b < nB; ++b) {
            c += bandp[b];
            t.prob[(size_t)i * nB + b] = (b == nB - 1) ? 1.0f : (float)(c / total);
        }
    }
    // the reference reader keeps the k_avg of the last temperature row
    // (read_tables.cpp:52 overwrites it on every row)
    for (int b = 0; b < nB; ++b) t.kavg[b] = t.kavg_t[(size_t)(nT - 1) * nB + b];
    return RC_OK;
}

int tables_check(const TableSet &t, std::string &err) {
    auto bad = [&](const std::string &m) {
        err = m;
        return RC_E_INVALID;
    };
    if (t.nT < 2 || t.nB < 1 || t.nQ < 1) return bad("table dimensions must be nT >= 2, nB >= 1, nQ >= 1");
    if (t.nT > 256) return bad("at most 256 table temperatures");
    const size_t nT = t.nT, nB = t.nB, nQ = t.nQ;
    if (t.Tnb.size() < nT || t.kP.size() < nT || t.kq.size() < nB * nT * nQ || t.prob.size() < nT * nB ||
        t.probg.size() < nT * nB * nQ)
        return bad("table arrays shorter than their dimensions");
    if (!(t.Tnb[1] > t.Tnb[0]) || !std::isfinite(t.Tnb[0]) || !std::isfinite(t.Tnb[1]))
        return bad("table temperatures must be increasing");
    const double d0 = (double)t.Tnb[1] - t.Tnb[0];
    for (size_t i = 2; i < nT; ++i) {
        // the lookups assume uniform spacing (pos = (T - T0)/dT)
        const double di = (double)t.Tnb[i] - t.Tnb[i - 1];
        if (!(fabs(di - d0) <= 1e-3 * fabs(d0))) return bad("table temperatures must be uniformly spaced");
    }
    // the band and g searches assume non-decreasing cumulative
    // probabilities in [0, 1] (a NaN fails every comparison below)
    const float one = 1.0f + 1e-5f;
    for (size_t i = 0; i < nT; ++i) {
        for (size_t b = 0; b < nB; ++b) {
            const float v = t.prob[i * nB + b], prev = b ? t.prob[i * nB + b - 1] : 0.0f;
            if (!(v >= prev && v <= one)) return bad("band cumulative probability not non-decreasing in [0, 1] (prob_new2)");
            for (size_t g = 0; g < nQ; ++g) {
                const float u = t.probg[(i * nB + b) * nQ + g], pu = g ? t.probg[(i * nB + b) * nQ + g - 1] : 0.0f;
                if (!(u >= pu && u <= one)) return bad("g cumulative probability not non-decreasing in [0, 1] (prob_new2)");
            }
        }
        if (!(t.kP[i] >= 0.0f) || !std::isfinite(t.kP[i])) return bad("Planck-mean coefficient not finite and >= 0");
    }
    for (size_t q = 0; q < nB * nT * nQ; ++q)
        if (!(t.kq[q] >= 0.0f) || !std::isfinite(t.kq[q])) return bad("absorption coefficient not finite and >= 0 (NarrBand)");
    return RC_OK;
}

namespace {
bool read_numbers(const std::string &path, std::vector<double> &v) {
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return false;
    char buf[128];
    v.clear();
    int c;
    std::string tok;
    while ((c = fgetc(f)) != EOF) {
        if (isspace(c)) {
            if (!tok.empty()) {
                v.push_back(strtod(tok.c_str(), nullptr));
                tok.clear();
            }
        } else {
            tok += (char)c;
        }
    }
    if (!tok.empty()) v.push_back(strtod(tok.c_str(), nullptr));
    (void)buf;
    fclose(f);
    return true;
}
}  // namespace

int tables_read_dir(const std::string &dir, int nT, int nB, int nQ, TableSet &t, std::string &err) {
    if (nT < 2 || nB < 1 || nQ < 1) {
        err = "invalid table dimensions";
        return RC_E_INVALID;
    }
    t.nT = nT;
    t.nB = nB;
    t.nQ = nQ;
    std::vector<double> v;
    // planck-mean.txt: "T kPr kR kM" per row (write_tables.cpp:23-26)
    std::string f = dir + "/planck-mean.txt";
    if (!read_numbers(f, v) || v.size() < (size_t)4 * nT) {
        err = "missing or short " + f;
        return RC_E_IO;
    }
    t.Tnb.resize(nT);
    t.kP.resize(nT);
    t.kR.resize(nT);
    t.kM.resize(nT);
    for (int i = 0; i < nT; ++i) {
        t.Tnb[i] = (float)v[4 * i];
        t.kP[i] = (float)v[4 * i + 1];
        t.kR[i] = (float)v[4 * i + 2];
        t.kM[i] = (float)v[4 * i + 3];
    }
    // NarrBand%d.txt: "wvl wvr wvc" then per row "T cuprob k_avg kq[nQ]"
    t.wvl.resize(nB);
    t.wvr.resize(nB);
    t.wvc.resize(nB);
    t.kavg.resize(nB);
    t.kavg_t.assign((size_t)nT * nB, 0.f);
    t.kq.assign((size_t)nB * nT * nQ, 0.f);
    for (int b = 0; b < nB; ++b) {
        std::string fb = dir + "/NarrBand" + std::to_string(b) + ".txt";
        if (!read_numbers(fb, v) || v.size() < (size_t)3 + (size_t)nT * (3 + nQ)) {
            err = "missing or short " + fb;
            return RC_E_IO;
        }
        t.wvl[b] = (float)v[0];
        t.wvr[b] = (float)v[1];
        t.wvc[b] = (float)v[2];
        for (int i = 0; i < nT; ++i) {
            const double *r = &v[3 + (size_t)i * (3 + nQ)];
            t.kavg_t[(size_t)i * nB + b] = (float)r[2];
            for (int g = 0; g < nQ; ++g) t.kq[((size_t)b * nT + i) * nQ + g] = (float)r[3 + g];
        }
        t.kavg[b] = t.kavg_t[(size_t)(nT - 1) * nB + b];
    }
    // prob_new2.txt: "T j cuprob cuprob_new2[nQ]" per (T, band) (write_tables.cpp:40-53)
    f = dir + "/prob_new2.txt";
    if (!read_numbers(f, v) || v.size() < (size_t)nT * nB * (3 + nQ)) {
        err = "missing or short " + f;
        return RC_E_IO;
    }
    t.prob.assign((size_t)nT * nB, 0.f);
    t.probg.assign((size_t)nT * nB * nQ, 0.f);
    for (int i = 0; i < nT; ++i)
        for (int b = 0; b < nB; ++b) {
            const double *r = &v[((size_t)i * nB + b) * (3 + nQ)];
            t.prob[(size_t)i * nB + b] = (float)r[2];
            for (int g = 0; g < nQ; ++g) t.probg[((size_t)i * nB + b) * nQ + g] = (float)r[3 + g];
        }
    // g weights: NarrowBand.h:194-209 for the shipped sizes, else Gauss-Legendre/2
    static const float w16[16] = {0.09654009f, 0.09563872f, 0.09384440f, 0.09117387f, 0.08765209f, 0.08331193f,
                                  0.07819389f, 0.07234580f, 0.06582222f, 0.05868409f, 0.05099806f, 0.04283589f,
                                  0.03427387f, 0.02539207f, 0.01627439f, 0.00701862f};
    static const float w7[7] = {0.04500f, 0.24500f, 0.32000f, 0.24500f, 0.05611f, 0.05125f, 0.03764f};
    static const float w17[17] = {0.045f,  0.245f,   0.32f,    0.245f,  0.0495f,    0.0245f,
                                  0.032f,  0.0245f,  0.00495f, 0.00245f, 0.0032f,   0.00245f,
                                  0.0005f, 0.0002722f, 0.00035556f, 0.000272222f, 0.00005f};
    t.wq.resize(nQ);
    t.gq.assign(nQ, 0.f);
    if (nQ == 16) t.wq.assign(w16, w16 + 16);
    else if (nQ == 7) t.wq.assign(w7, w7 + 7);
    else if (nQ == 17) t.wq.assign(w17, w17 + 17);
    else {
        std::vector<double> x, w;
        gauss_legendre(nQ, x, w);
        for (int g = 0; g < nQ; ++g) t.wq[g] = (float)(w[g] / 2);
    }
    return RC_OK;
}

int tables_write_dir(const TableSet &t, const std::string &dir, std::string &err) {
    std::string f = dir + "/planck-mean.txt";
    FILE *fp = fopen(f.c_str(), "wt");
    if (!fp) {
        err = "cannot write " + f;
        return RC_E_IO;
    }
    for (int i = 0; i < t.nT; i++)
        fprintf(fp, "%lf %le %le %le\n", (double)t.Tnb[i], (double)t.kP[i], t.kR.empty() ? 0.0 : (double)t.kR[i],
                t.kM.empty() ? 0.0 : (double)t.kM[i]);
    fclose(fp);
    f = dir + "/prob_new2.txt";
    fp = fopen(f.c_str(), "wt");
    if (!fp) {
        err = "cannot write " + f;
        return RC_E_IO;
    }
    for (int i = 0; i < t.nT; i++)
        for (int j = 0; j < t.nB; j++) {
            fprintf(fp, "%lf \t %-5d \t%30.20le \t", (double)t.Tnb[i], j, (double)t.prob[(size_t)i * t.nB + j]);
            for (int g = 0; g < t.nQ; g++) fprintf(fp, "%30.20le\t", (double)t.probg[((size_t)i * t.nB + j) * t.nQ + g]);
            fprintf(fp, "\n");
        }
    fclose(fp);
    for (int j = 0; j < t.nB; j++) {
        f = dir + "/NarrBand" + std::to_string(j) + ".txt";
        fp = fopen(f.c_str(), "wt");
        if (!fp) {
            err = "cannot write " + f;
            return RC_E_IO;
        }
        fprintf(fp, "%le\t%le\t%le \n", (double)t.wvl[j], (double)t.wvr[j], (double)t.wvc[j]);
        for (int i = 0; i < t.nT; i++) {
            fprintf(fp, " %lf\t", (double)t.Tnb[i]);
            fprintf(fp, " %le\t", (double)t.prob[(size_t)i * t.nB + j]);
            float ka = t.kavg_t.empty() ? t.kavg[j] : t.kavg_t[(size_t)i * t.nB + j];
            fprintf(fp, " %le\t", (double)ka);
            for (int h = 0; h < t.nQ; h++) fprintf(fp, " %le\t", (double)t.kq[((size_t)j * t.nT + i) * t.nQ + h]);
            fprintf(fp, "\n");
        }
        fclose(fp);
    }
    return RC_OK;
}

}  // namespace rc
