// ldp_inp.cpp -- the .inp keyword-file reader and default-file writer.
//
// Restates INPUTPARSER::InputParser (src/inputParser.cpp:45-520) as the two
// mains configure it (src/langevinDynamicsSingleBarrier.cpp:64-188,
// src/langevinDynamicsDoubleBarrier.cpp:68-210): the same keys, defaults,
// value counts and "must appear once" rules; '#' comments; '\' line
// continuation; DEFINE a b; variable lines `a = b`; INCLUDE files;
// FOR start end step format symbol line...; FORn nested loops.  Values are
// converted with the reference's rules (text::to_boolean, stod/stoi/stoul).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ldp.h"

namespace {

enum class Kind { Input, Output, Parameter };

struct Opt {
    const char* key;
    const char* help;
    const char* def;
    int nval;
    bool multiple;
    Kind kind;
};

// Option tables in AddOption order.
const Opt kSingle[] = {
    {"OUTPUTBASE", "Output base", "langevinDynamicsSingleBarrier", 1, false, Kind::Output},
    {"OVERDAMPED", "Whether use overdamped equation", "false", 1, false, Kind::Parameter},
    {"X0", "Initial position (x0)", "0.0", 1, false, Kind::Parameter},
    {"V0", "Initial velocity (v0)", "1.0", 1, false, Kind::Parameter},
    {"GAMMA", "Friction coefficient (Gamma)", "1.0", 1, false, Kind::Parameter},
    {"KB", "Boltzman factor", "1.0", 1, false, Kind::Parameter},
    {"TEMPERATURE", "Temperature", "1.0", 1, false, Kind::Parameter},
    {"MASS", "Mass", "1.0", 1, false, Kind::Parameter},
    {"RANDOMIZEV", "Whether randomize initial velocity", "true", 1, false, Kind::Parameter},
    {"PERIODICLENGTH", "Periodic length", "10.0", 1, false, Kind::Parameter},
    {"BARRIERHEIGHTS", "Barrier heights (two)", "2.0 6.0", 2, false, Kind::Parameter},
    {"BARRIERHALFWIDTH", "Barrier half width", "1.0", 1, false, Kind::Parameter},
    {"TIMESTEP", "Timestep (dt)", "0.1", 1, false, Kind::Parameter},
    {"NUMBEROFSTEPS", "Number of steps", "10000", 1, false, Kind::Parameter},
    {"NUMBEROFPREVIOUSSTEPS", "Number of previous steps", "0", 1, false, Kind::Parameter},
    {"NUMBEROFRUNS", "Number of runs", "1", 1, false, Kind::Parameter},
    {"FREQSAVE", "Save frequency", "1", 1, false, Kind::Parameter},
    {"FREQSTAT", "Statistics frequency", "1", 1, false, Kind::Parameter},
    {"DISTRIBUTIONV0", "Whether calculate V0 distribution", "false", 1, false, Kind::Parameter},
    {"DISTRIBUTIONS0", "Whether calculate state0 distribution", "false", 1, false, Kind::Parameter},
    {"TAU", "Tau of bichotomic noise eta", "0.1", 1, false, Kind::Parameter},
    {"INITIALSTATE", "Initial barrier state (0 or 1)", "0", 1, false, Kind::Parameter},
    {"RANDOMIZESTATES", "Whether randomize initial states", "true", 1, false, Kind::Parameter},
    {"UNIFORMINITALSTATES", "Uniform initial states", "false", 1, false, Kind::Parameter},
    {"EQ", "Whether equal prob, constant forward K", "true 1.0", 2, false, Kind::Parameter},
    {"WAITINGTIME", "Whether calculate waiting time", "false", 1, false, Kind::Parameter},
    {"FPT", "Whether calculate first passage time", "false", 1, false, Kind::Parameter},
    {"TPT", "Whether calculate transition path time", "false", 1, false, Kind::Parameter},
    {"FPTCG", "Whether calculate coarse grained first passage time", "false 10", 2, true, Kind::Parameter},
    {"READRESTART", "Whether read restart", "false", 1, false, Kind::Parameter},
    {"WRITERESTART", "Whether write restart", "false", 1, false, Kind::Parameter},
    {"INPUTRESTART", "Input restart file base", "inputRestart", 1, false, Kind::Input},
    {"OUTPUTRESTART", "Output restart file base", "outputRestart", 1, false, Kind::Output},
    {"WRITEX", "Whether write x trajectory", "false", 1, false, Kind::Parameter},
    {"NUMBEROFLOGSAMPLES", "Number of samples point per order", "20", 1, false, Kind::Parameter},
    {"RANDOMSEED", "Random number seed", "-1", 1, false, Kind::Parameter},
    {"PRINTTIMER", "Whether print timer", "false", 1, false, Kind::Parameter},
};

const Opt kDouble[] = {
    {"OUTPUTBASE", "Output base", "langevinDynamicsSingleBarrier", 1, false, Kind::Output},
    {"OVERDAMPED", "Whether use overdamped equation", "false", 1, false, Kind::Parameter},
    {"X0", "Initial position (x0)", "0.0", 1, false, Kind::Parameter},
    {"V0", "Initial velocity (v0)", "1.0", 1, false, Kind::Parameter},
    {"GAMMA", "Friction coefficient (Gamma)", "1.0", 1, false, Kind::Parameter},
    {"KB", "Boltzman factor", "1.0", 1, false, Kind::Parameter},
    {"TEMPERATURE", "Temperature", "1.0", 1, false, Kind::Parameter},
    {"MASS", "Mass", "1.0", 1, false, Kind::Parameter},
    {"RANDOMIZEV", "Whether randomize initial velocity", "true", 1, false, Kind::Parameter},
    {"PERIODICLENGTH", "Periodic length", "10.0", 1, false, Kind::Parameter},
    {"BARRIERHEIGHTS0", "Barrier heights 0 (two)", "2.0 6.0", 2, false, Kind::Parameter},
    {"BARRIERHEIGHTS1", "Barrier heights 1 (two)", "2.0 6.0", 2, false, Kind::Parameter},
    {"BARRIERHALFWIDTH0", "Barrier half width 0", "1.0", 1, false, Kind::Parameter},
    {"BARRIERHALFWIDTH1", "Barrier half width 1", "1.0", 1, false, Kind::Parameter},
    {"BARRIERPOSITION0", "Barrier position 0", "1.0", 1, false, Kind::Parameter},
    {"BARRIERPOSITION1", "Barrier position 1", "2.0", 1, false, Kind::Parameter},
    {"TIMESTEP", "Timestep (dt)", "0.1", 1, false, Kind::Parameter},
    {"NUMBEROFSTEPS", "Number of steps", "10000", 1, false, Kind::Parameter},
    {"NUMBEROFPREVIOUSSTEPS", "Number of previous steps", "0", 1, false, Kind::Parameter},
    {"NUMBEROFRUNS", "Number of runs", "1", 1, false, Kind::Parameter},
    {"FREQSAVE", "Save frequency", "1", 1, false, Kind::Parameter},
    {"FREQSTAT", "Statistics frequency", "1", 1, false, Kind::Parameter},
    {"DISTRIBUTIONV0", "Whether calculate V0 distribution", "false", 1, false, Kind::Parameter},
    {"DISTRIBUTIONS0", "Whether calculate state0 distribution", "false", 1, false, Kind::Parameter},
    {"TAU", "Tau of bichotomic noise eta", "0.1", 1, false, Kind::Parameter},
    {"INITIALSTATE", "Initial barrier state (0 or 1)", "0", 1, false, Kind::Parameter},
    {"RANDOMIZESTATES", "Whether randomize initial states", "true", 1, false, Kind::Parameter},
    {"UNIFORMINITALSTATES", "Uniform initial states", "false", 1, false, Kind::Parameter},
    {"EQ", "Whether equal prob, constant forward K", "true 1.0", 2, false, Kind::Parameter},
    {"WAITINGTIME", "Whether calculate waiting time", "false", 1, false, Kind::Parameter},
    {"FPT", "Whether calculate first passage time", "false", 1, false, Kind::Parameter},
    {"TPT", "Whether calculate transition path time", "false", 1, false, Kind::Parameter},
    {"FPTCG", "Whether calculate coarse grained first passage time", "false 10", 2, true, Kind::Parameter},
    {"READRESTART", "Whether read restart", "false", 1, false, Kind::Parameter},
    {"WRITERESTART", "Whether write restart", "false", 1, false, Kind::Parameter},
    {"INPUTRESTART", "Input restart file base", "inputRestart", 1, false, Kind::Input},
    {"OUTPUTRESTART", "Output restart file base", "outputRestart", 1, false, Kind::Output},
    {"WRITEX", "Whether write x trajectory", "false", 1, false, Kind::Parameter},
    {"NUMBEROFLOGSAMPLES", "Number of samples point per order", "20", 1, false, Kind::Parameter},
    {"RANDOMSEED", "Random number seed", "-1", 1, false, Kind::Parameter},
    {"PRINTTIMER", "Whether print timer", "false", 1, false, Kind::Parameter},
};

struct Table {
    const Opt* opts;
    int n;
};

Table table_for(int model) {
    if (model == LDP_MODEL_DOUBLE) return {kDouble, (int)(sizeof(kDouble) / sizeof(kDouble[0]))};
    return {kSingle, (int)(sizeof(kSingle) / sizeof(kSingle[0]))};
}

std::vector<std::string> split_ws(const std::string& s, const char* mask = " \t\r\n") {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && std::strchr(mask, s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !std::strchr(mask, s[j])) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

std::string join(const std::vector<std::string>& w, size_t first) {
    std::string r;
    for (size_t i = first; i < w.size(); ++i) {
        if (i > first) r += " ";
        r += w[i];
    }
    return r;
}

bool is_blank(const std::string& s) { return s.find_first_not_of(" \t\r\n") == std::string::npos; }

std::string replace_all(std::string s, const std::string& a, const std::string& b) {
    if (a.empty()) return s;
    size_t pos = 0;
    while ((pos = s.find(a, pos)) != std::string::npos) {
        s.replace(pos, a.size(), b);
        pos += b.size();
    }
    return s;
}

bool iequals(const std::string& a, const char* b) {
    size_t n = std::strlen(b);
    if (a.size() != n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
    return true;
}

bool parse_int(const std::string& s, long long* v) {
    try {
        size_t pos = 0;
        *v = std::stoll(s, &pos);
        return true;
    } catch (...) {
        return false;
    }
}

bool parse_double(const std::string& s, double* v) {
    try {
        *v = std::stod(s);
        return true;
    } catch (...) {
        return false;
    }
}

// text::to_boolean, src/text.cpp:278-285.
bool to_boolean(const std::string& s) {
    if (s == "TRUE" || s == "True" || s == "true") return true;
    long long i;
    if (parse_int(s, &i) && i != 0) return true;
    double d;
    if (parse_double(s, &d) && d != 0.0) return true;
    return false;
}

struct Parser {
    std::map<std::string, std::string> defines, vars;
    std::vector<std::string> content;
    std::string err;

    std::string resolve(const std::string& base, const std::string& path) {
        if (path.empty() || path[0] == '/' || base.empty()) return path;
        return base + "/" + path;
    }

    void for_loops(const std::vector<long long>& a, const std::vector<long long>& b, const std::vector<long long>& c,
                   const std::vector<std::string>& fmt, const std::vector<std::string>& sym, size_t lvl,
                   const std::string& line) {
        for (long long i = a[lvl]; i < b[lvl]; i += c[lvl]) {
            char buf[256];
            std::snprintf(buf, sizeof(buf), fmt[lvl].c_str(), (int)i);
            std::string nl = replace_all(line, sym[lvl], buf);
            if (lvl + 1 == a.size()) content.push_back(nl);
            else for_loops(a, b, c, fmt, sym, lvl + 1, nl);
            if (c[lvl] <= 0) break;
        }
    }

    bool open_text(const std::string& text, const std::string& base_dir, int depth) {
        if (depth > 32) {
            err = "INCLUDE nesting too deep";
            return false;
        }
        std::vector<std::string> lines;
        bool append = false;
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            if (!line.empty() && line.back() == '\r') line.pop_back();
            size_t h = line.find('#');
            if (h != std::string::npos) line = line.substr(0, h);
            if (append) lines.back() += line;
            else lines.push_back(line);
            if (!line.empty() && line.back() == '\\') {
                lines.back().pop_back();
                append = true;
            } else {
                append = false;
            }
        }
        for (std::string l : lines) {
            if (is_blank(l)) continue;
            for (auto& kv : defines) l = replace_all(l, kv.first, kv.second);
            for (auto& kv : vars) l = replace_all(l, kv.first, kv.second);
            std::vector<std::string> w = split_ws(l);
            if (w.empty()) continue;
            // Variable assignment `a = b` (IsLineAssignment).
            if (l.find('=') != std::string::npos) {
                std::vector<std::string> we = split_ws(l, " \t=\r\n");
                if (we.size() == 2) {
                    vars[we[0]] = we[1];
                    continue;
                }
            }
            if (iequals(w[0], "include")) {
                if (w.size() < 2) {
                    err = "INCLUDE requires at least 1 argument";
                    return false;
                }
                for (size_t k = 1; k < w.size(); ++k) {
                    std::string path = resolve(base_dir, w[k]);
                    std::ifstream f(path);
                    if (!f) {
                        err = "can't open input file (" + path + ")";
                        return false;
                    }
                    std::stringstream ss;
                    ss << f.rdbuf();
                    // nested INCLUDEs resolve against the same base (the
                    // working directory unless the caller gave one)
                    if (!open_text(ss.str(), base_dir, depth + 1)) return false;
                }
            } else if (iequals(w[0], "define")) {
                if (w.size() != 3) {
                    err = "DEFINE requires 2 arguments";
                    return false;
                }
                defines[w[1]] = w[2];
            } else if (iequals(w[0], "for")) {
                if (w.size() >= 7) {
                    long long a = 0, b = 0, c = 1;
                    parse_int(w[1], &a);
                    parse_int(w[2], &b);
                    parse_int(w[3], &c);
                    for_loops({a}, {b}, {c}, {w[4]}, {w[5]}, 0, join(w, 6));
                }
            } else if (w[0].size() > 3 && iequals(w[0].substr(0, 3), "for")) {
                long long nloop = 0;
                if (!parse_int(w[0].substr(3), &nloop) || nloop < 1 || w.size() < (size_t)(nloop * 5 + 1)) {
                    err = "for is not followed by an integer (" + w[0].substr(3) + ")";
                    return false;
                }
                std::vector<long long> a(nloop), b(nloop), c(nloop);
                std::vector<std::string> fmt(nloop), sym(nloop);
                for (long long i = 0; i < nloop; ++i) {
                    parse_int(w[i * 5 + 1], &a[i]);
                    parse_int(w[i * 5 + 2], &b[i]);
                    parse_int(w[i * 5 + 3], &c[i]);
                    fmt[i] = w[i * 5 + 4];
                    sym[i] = w[i * 5 + 5];
                }
                for_loops(a, b, c, fmt, sym, 0, join(w, (size_t)(nloop * 5 + 1)));
            } else {
                content.push_back(l);
            }
        }
        return true;
    }
};

void set_str(char* dst, const std::string& s) { std::snprintf(dst, LDP_PATH_MAX, "%s", s.c_str()); }

}  // namespace

extern "C" void ldp_params_default(int model, ldp_params* p);

// Reads the .inp text into per-option value lists (option table order, one
// entry per occurrence, each the occurrence's values): OpenInput and
// ProcessInputLines, src/inputParser.cpp:269-330, 412-475.
static ldp_status parse_values(const char* text, const char* base_dir, int model, Table* tb,
                               std::vector<std::vector<std::vector<std::string>>>* vals, std::string* err) {
    Parser ps;
    if (!ps.open_text(text, base_dir ? base_dir : "", 0)) {
        *err = ps.err;
        return LDP_ERR_PARSE;
    }
    *tb = table_for(model);
    std::map<std::string, int> idx;
    for (int i = 0; i < tb->n; ++i) idx[tb->opts[i].key] = i;
    vals->assign(tb->n, {});
    for (const std::string& l : ps.content) {
        if (is_blank(l)) continue;
        std::vector<std::string> w = split_ws(l);
        auto it = idx.find(w[0]);
        if (it == idx.end()) {
            *err = "undefined option (" + w[0] + ")";
            return LDP_ERR_PARSE;
        }
        const Opt& o = tb->opts[it->second];
        std::vector<std::string> v(w.begin() + 1, w.end());
        if (!o.multiple && !(*vals)[it->second].empty()) {
            *err = "(" + w[0] + ") can be specified only once";
            return LDP_ERR_PARSE;
        }
        if ((int)v.size() != o.nval) {
            *err = "(" + w[0] + ") requires exactly " + std::to_string(o.nval) + " values but got " +
                   std::to_string(v.size()) + " (" + join(w, 1) + ")";
            return LDP_ERR_PARSE;
        }
        (*vals)[it->second].push_back(v);
    }
    for (int i = 0; i < tb->n; ++i)
        if ((*vals)[i].empty()) {
            *err = std::string("(") + tb->opts[i].key + ") must be specified at least once";
            return LDP_ERR_PARSE;
        }
    return LDP_OK;
}

extern "C" ldp_status ldp_params_from_inp_text(const char* text, const char* base_dir, int model, ldp_params* p,
                                               char* err, size_t errlen) {
    auto fail = [&](ldp_status st, const std::string& m) {
        if (err && errlen) std::snprintf(err, errlen, "Error (InputParser): %s", m.c_str());
        return st;
    };
    if (!text || !p) return fail(LDP_ERR_INVALID, "null argument");
    if (model != LDP_MODEL_SINGLE && model != LDP_MODEL_DOUBLE) return fail(LDP_ERR_INVALID, "unknown model");
    Table tb;
    std::vector<std::vector<std::vector<std::string>>> vals;
    std::string perr;
    const ldp_status pst = parse_values(text, base_dir, model, &tb, &vals, &perr);
    if (pst != LDP_OK) return fail(pst, perr);
    std::map<std::string, int> idx;
    for (int i = 0; i < tb.n; ++i) idx[tb.opts[i].key] = i;

    auto get = [&](const char* key, int j = 0, int k = 0) -> const std::string& { return vals[idx[key]][j][k]; };
    auto dbl = [&](const char* key, int k = 0) {
        double d = 0.0;
        parse_double(get(key, 0, k), &d);
        return d;
    };
    auto u64 = [&](const char* key) {
        try {
            return (uint64_t)std::stoull(get(key));
        } catch (...) {
            return (uint64_t)0;
        }
    };
    auto i64 = [&](const char* key) {
        long long v = 0;
        parse_int(get(key), &v);
        return (int64_t)v;
    };
    auto boolean = [&](const char* key, int k = 0) { return to_boolean(get(key, 0, k)) ? 1 : 0; };

    ldp_params_default(model, p);
    p->model = model;
    set_str(p->output_base, get("OUTPUTBASE"));
    p->overdamped = boolean("OVERDAMPED");
    p->x0 = dbl("X0");
    p->v0 = dbl("V0");
    p->gamma = dbl("GAMMA");
    p->kb = dbl("KB");
    p->temperature = dbl("TEMPERATURE");
    p->mass = dbl("MASS");
    p->randomize_v = boolean("RANDOMIZEV");
    p->periodic_length = dbl("PERIODICLENGTH");
    if (model == LDP_MODEL_SINGLE) {
        p->barrier_heights[0][0] = dbl("BARRIERHEIGHTS", 0);
        p->barrier_heights[0][1] = dbl("BARRIERHEIGHTS", 1);
        p->barrier_half_width[0] = dbl("BARRIERHALFWIDTH");
    } else {
        p->barrier_heights[0][0] = dbl("BARRIERHEIGHTS0", 0);
        p->barrier_heights[0][1] = dbl("BARRIERHEIGHTS0", 1);
        p->barrier_heights[1][0] = dbl("BARRIERHEIGHTS1", 0);
        p->barrier_heights[1][1] = dbl("BARRIERHEIGHTS1", 1);
        p->barrier_half_width[0] = dbl("BARRIERHALFWIDTH0");
        p->barrier_half_width[1] = dbl("BARRIERHALFWIDTH1");
        p->barrier_position[0] = dbl("BARRIERPOSITION0");
        p->barrier_position[1] = dbl("BARRIERPOSITION1");
    }
    p->timestep = dbl("TIMESTEP");
    p->number_of_steps = u64("NUMBEROFSTEPS");
    p->number_of_previous_steps = u64("NUMBEROFPREVIOUSSTEPS");
    p->number_of_runs = (int32_t)i64("NUMBEROFRUNS");
    p->freq_save = u64("FREQSAVE");
    p->freq_stat = u64("FREQSTAT");
    p->distribution_v0 = boolean("DISTRIBUTIONV0");
    p->distribution_s0 = boolean("DISTRIBUTIONS0");
    p->tau = dbl("TAU");
    p->initial_state = (int32_t)dbl("INITIALSTATE");   // read as double, used as int (S.cpp:143)
    p->randomize_states = boolean("RANDOMIZESTATES");
    p->uniform_initial_states = boolean("UNIFORMINITALSTATES");
    p->eq = boolean("EQ", 0);
    p->eq_constant = dbl("EQ", 1);
    p->waiting_time = boolean("WAITINGTIME");
    p->fpt = boolean("FPT");
    p->tpt = boolean("TPT");
    // FPTCG: the flag is the boolean of the last entry; every entry adds a
    // size (src/langevinDynamicsSingleBarrier.cpp:151-159).
    const auto& cg = vals[idx["FPTCG"]];
    if ((int)cg.size() > LDP_MAX_CG) return fail(LDP_ERR_UNSUPPORTED, "more than 16 FPTCG entries");
    p->n_cg = (int32_t)cg.size();
    for (size_t j = 0; j < cg.size(); ++j) {
        p->fptcg = to_boolean(cg[j][0]) ? 1 : 0;
        long long v = 0;
        parse_int(cg[j][1], &v);
        p->cg_sizes[j] = (int32_t)v;
    }
    p->read_restart = boolean("READRESTART");
    p->write_restart = boolean("WRITERESTART");
    set_str(p->input_restart, get("INPUTRESTART"));
    set_str(p->output_restart, get("OUTPUTRESTART"));
    p->write_x = boolean("WRITEX");
    p->number_of_log_samples = u64("NUMBEROFLOGSAMPLES");
    p->random_seed = i64("RANDOMSEED");
    p->print_timer = boolean("PRINTTIMER");
    if (p->freq_save == 0) return fail(LDP_ERR_INVALID, "FREQSAVE must be >= 1");
    if (p->number_of_log_samples == 0) return fail(LDP_ERR_INVALID, "NUMBEROFLOGSAMPLES must be >= 1");
    if (err && errlen) err[0] = 0;
    return LDP_OK;
}

extern "C" ldp_status ldp_params_from_inp(const char* path, int model, ldp_params* p, char* err, size_t errlen) {
    if (!path) return LDP_ERR_INVALID;
    std::ifstream f(path);
    if (!f) {
        if (err && errlen) std::snprintf(err, errlen, "Error (InputParser): can't open input file (%s)", path);
        return LDP_ERR_IO;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    // INCLUDE paths are opened as written, i.e. relative to the working
    // directory, as the reference's OpenInput does (src/inputParser.cpp:311).
    return ldp_params_from_inp_text(ss.str().c_str(), "", model, p, err, errlen);
}

// PrintAllValues (src/inputParser.cpp:188-196), the reference's `-p`: every
// option in table order, one line per occurrence, "%-20s %3d %s" with the
// occurrence's values joined by single spaces.
extern "C" ldp_status ldp_inp_print_values(const char* path, int model, char* buf, size_t buflen, size_t* needed) {
    if (!path || (!buf && buflen)) return LDP_ERR_INVALID;
    std::ifstream f(path);
    if (!f) {
        if (buf && buflen) std::snprintf(buf, buflen, "Error (InputParser): can't open input file (%s)\n", path);
        return LDP_ERR_IO;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    Table tb;
    std::vector<std::vector<std::vector<std::string>>> vals;
    std::string perr;
    const ldp_status st = parse_values(ss.str().c_str(), "", model, &tb, &vals, &perr);
    if (st != LDP_OK) {
        if (buf && buflen) std::snprintf(buf, buflen, "Error (InputParser): %s\n", perr.c_str());
        return st;
    }
    std::string out;
    char line[4096];
    for (int i = 0; i < tb.n; ++i)
        for (size_t j = 0; j < vals[i].size(); ++j) {
            std::snprintf(line, sizeof(line), "%-20s %3d %s\n", tb.opts[i].key, (int)j, join(vals[i][j], 0).c_str());
            out += line;
        }
    if (needed) *needed = out.size() + 1;
    if (out.size() + 1 > buflen) return LDP_ERR_NOMEM;
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return LDP_OK;
}

// PrintEmptyInputFile (src/inputParser.cpp:212-266): `# [Type] help` then
// `KEY default` for every option.
extern "C" ldp_status ldp_write_default_inp(const char* path, int model) {
    if (!path) return LDP_ERR_INVALID;
    FILE* f = std::fopen(path, "w");
    if (!f) return LDP_ERR_IO;
    Table tb = table_for(model);
    for (int i = 0; i < tb.n; ++i) {
        const char* kind = tb.opts[i].kind == Kind::Input ? "Input" : tb.opts[i].kind == Kind::Output ? "Output" : "Parameter";
        std::fprintf(f, "# [%s] %s\n", kind, tb.opts[i].help);
        std::fprintf(f, "%-20s %s\n", tb.opts[i].key, tb.opts[i].def);
    }
    std::fclose(f);
    return LDP_OK;
}
