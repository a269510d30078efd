// ldp_output.cpp -- the reference's output files, written from a finished job.
//
// Restates the post-processing and file output of
// LangevinEquationRunnerMPI::Run (src/langevinDynamicsSingleBarrier.h:
// 3452-3580 and 3594-4036; src/langevinDynamicsDoubleBarrier.h at the same
// places, +~630 lines) with the job's per-trajectory results: the same file
// names, PrintParameter header, number formats and reductions.  "Ranks" are
// the job's virtual ranks: per-rank partial sums are formed in trajectory
// order and then added over ranks, in rank order, as the reference's rank-0
// gathers do (src/mpiKernel.cpp:81-106, 139-170).
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ldp_internal.h"

namespace {

struct Hist {
    double min = 0, max = 0, step = 0, inv = 0;
    int size = 0;
    std::vector<double> count, percent;
    // HISTOGRAM::Allocate(min, max, int nbin), src/clsHistogram.cpp:158-166
    void alloc(double mn, double mx, int nbin) {
        min = mn;
        max = mx;
        size = nbin;
        step = (mx - mn) / nbin;
        inv = 1.0 / step;
        count.assign(nbin, 0.0);
        percent.assign(nbin, 0.0);
    }
    // AddValue: truncation toward zero (clsHistogram.cpp:257-265)
    void add_trunc(double v) {
        const int i = (int)((v - min) * inv);
        if (i >= 0 && i < size) count[i] += 1.0;
    }
    void normalize() {
        double s = 0.0;
        for (int i = 0; i < size; ++i) s += count[i];
        if (s != 0.0)
            for (int i = 0; i < size; ++i) percent[i] = count[i] / s;
    }
    void print(FILE* f) const {
        std::fprintf(f, "# HMin %23.16E\n", min);
        std::fprintf(f, "# HMax %23.16E\n", max);
        std::fprintf(f, "# HBin %23.16E\n", step);
        std::fprintf(f, "# NBin %23d\n", size);
        for (int i = 0; i < size; ++i)
            std::fprintf(f, "%23.16E %23.16E %23.16E %23.0f %23.16E\n", min + step * i, min + step * (i + 0.5),
                         min + step * (i + 1.0), count[i], percent[i]);
    }
};

bool exists(const std::string& p) { return access(p.c_str(), F_OK) != -1; }

// MOLUTILITY::findNextBackUpFileName (src/MOLUTILITY.cpp:6-22): an existing
// file is renamed to "#name_bk.N#" with the first free N.
void backup(const std::string& filename) {
    if (!exists(filename)) return;
    const size_t sl = filename.rfind('/');
    const std::string path = sl == std::string::npos ? "" : filename.substr(0, sl + 1);
    const std::string name = sl == std::string::npos ? filename : filename.substr(sl + 1);
    for (int c = 1;; ++c) {
        const std::string b = path + "#" + name + "_bk." + std::to_string(c) + "#";
        if (!exists(b)) {
            std::rename(filename.c_str(), b.c_str());
            return;
        }
    }
}

const char* tf(bool b) { return b ? "true" : "false"; }

// text::FromByte2Readable (src/text.cpp:893-904)
std::string readable_bytes(double v) {
    const char* unit[5] = {"B", "K", "M", "G", "T"};
    int u = 0;
    while (v > 1024.0 && u < 4) {
        v /= 1024.0;
        ++u;
    }
    char b[64];
    std::snprintf(b, sizeof(b), "%13.7f %s", v, unit[u]);
    return b;
}

// clsSystemTime::Print_Time_Diff (src/clsTime.cpp:28-47)
std::string time_diff(double seconds) {
    double t = seconds;
    const char* unit = "s";
    double in = t / 60.0;
    if (in > 1.0) {
        t = in;
        unit = "m";
        in = t / 60.0;
        if (in > 1.0) {
            t = in;
            unit = "h";
            in = t / 24.0;
            if (in > 1.0) {
                t = in;
                unit = "d";
            }
        }
    }
    char b[64];
    std::snprintf(b, sizeof(b), "%f %s", t, unit);
    return b;
}

double average(const std::vector<double>& v) {
    if (v.empty()) return 0.0;
    double s = 0.0;
    for (double x : v) s += x;
    return s / (double)v.size();
}

// STATISTICS::RMSD, population standard deviation (src/STATISTICS.cpp:122-134).
// The squares are accumulated with one rounding each (a fused multiply-add,
// as the reference's build evaluates `rmsd += d * d`): that is what
// reproduces the sd lines of its output files to the last digit.
double rmsd(const std::vector<double>& v) {
    if (v.empty()) return 0.0;
    const double a = average(v);
    double r = 0.0;
    for (double x : v) r = std::fma(x - a, x - a, r);
    return std::sqrt(r / (double)v.size());
}

struct Writer {
    const ldp_job* job;
    const ldp_params& p;
    std::string dir;
    int ranks, lanes, nruns;
    int64_t n;
    bool dbl;
    double xc = 0, yc = 0;

    std::string path(const std::string& name) const { return dir.empty() ? name : dir + "/" + name; }

    FILE* open(const std::string& name) const {
        const std::string f = path(name);
        backup(f);
        return std::fopen(f.c_str(), "w+");
    }

    // PrintParameter, S.h:3040-3124 / D.h:3671-3762.
    void header(FILE* f) const {
        const double ts = p.timestep * (double)p.freq_save;
        const bool wx = p.write_x != 0;
        const double ntset = 1.0 + (wx ? 6.0 : 0.0);
        const double mem = ntset * (double)(p.number_of_steps / p.freq_save + 1) * 8.0 * (double)lanes;
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Overdamped           = %13s\n", tf(p.overdamped));
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Number of node       = %13d\n", ranks);
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Time step            = %13.7f\n", p.timestep);
        std::fprintf(f, "# Save frequency       = %13zd\n", (size_t)p.freq_save);
        std::fprintf(f, "# Save time step       = %13.7f\n", ts);
        std::fprintf(f, "# Statistics freq      = %13zd\n", (size_t)p.freq_stat);
        std::fprintf(f, "# Number of step (pre) = %13zd\n", (size_t)p.number_of_previous_steps);
        std::fprintf(f, "# Number of step       = %13zd\n", (size_t)p.number_of_steps);
        std::fprintf(f, "# Simulation time      = %13.6E\n", p.timestep * (double)p.number_of_steps);
        std::fprintf(f, "# Number of trial      = %13d\n", nruns);
        std::fprintf(f, "# Number of run/trial  = %13d\n", lanes);
        std::fprintf(f, "# Number of run        = %13d\n", (int)n);
        std::fprintf(f, "# ==============================================\n");
        if (!dbl) {
            std::fprintf(f, "# Barrier height [0]   = %13.7f\n", p.barrier_heights[0][0]);
            std::fprintf(f, "# Barrier height [1]   = %13.7f\n", p.barrier_heights[0][1]);
            std::fprintf(f, "# Barrier periodicity  = %13.7f\n", p.periodic_length);
            std::fprintf(f, "# slope half length    = %13.7f\n", p.barrier_half_width[0]);
        } else {
            std::fprintf(f, "# Barrier height [0][0]= %13.7f\n", p.barrier_heights[0][0]);
            std::fprintf(f, "# Barrier height [0][1]= %13.7f\n", p.barrier_heights[0][1]);
            std::fprintf(f, "# Barrier height [1][0]= %13.7f\n", p.barrier_heights[1][0]);
            std::fprintf(f, "# Barrier height [1][1]= %13.7f\n", p.barrier_heights[1][1]);
            std::fprintf(f, "# Xc                   = %13.7f\n", xc);
            std::fprintf(f, "# Yc                   = %13.7f\n", yc);
            std::fprintf(f, "# Barrier periodicity  = %13.7f\n", p.periodic_length);
            std::fprintf(f, "# Slope half length[0] = %13.7f\n", p.barrier_half_width[0]);
            std::fprintf(f, "# Slope half length[1] = %13.7f\n", p.barrier_half_width[1]);
            std::fprintf(f, "# Barrier position [0] = %13.7f\n", p.barrier_position[0]);
            std::fprintf(f, "# Barrier position [1] = %13.7f\n", p.barrier_position[1]);
        }
        std::fprintf(f, "# Equal probability    = %13s\n", tf(p.eq));
        std::fprintf(f, "# Equilibrium constant = %13.7E\n", p.eq_constant);
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Mass                 = %13.7f\n", p.mass);
        std::fprintf(f, "# Gamma                = %13.7f\n", p.gamma);
        std::fprintf(f, "# Temperature          = %13.7f\n", p.temperature);
        std::fprintf(f, "# kB                   = %13.7f\n", p.kb);
        std::fprintf(f, "# Eta variance (Q)     = %13.7f\n", 0.2);      // hard-wired q (S.cpp:145)
        std::fprintf(f, "# Eta tau              = %13.7f\n", p.tau);
        std::fprintf(f, "# Sample per order     = %13d\n", (int)p.number_of_log_samples);
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# X0                   = %13.7f\n", p.x0);
        if (p.randomize_v) std::fprintf(f, "# V0                   = %13s\n", "Random");
        else std::fprintf(f, "# V0                   = %13.7f\n", p.v0);
        std::fprintf(f, "# Eta0                 = %13s\n", "Random");   // bEr hard-wired true
        if (p.randomize_states) std::fprintf(f, "# State0               = %13s\n", "Random");
        else std::fprintf(f, "# State0               = %13d\n", p.initial_state);
        std::fprintf(f, "# Same initial barrier = %13s\n", tf(p.uniform_initial_states));
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Random number seed0  = %13d\n", (int)p.random_seed);
        std::fprintf(f, "# Random number seed   = %13d\n", (int)job->seed);
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Number of traj(each) = %13.0f\n", ntset);
        std::fprintf(f, "# Memory usage (each)  = %13s\n", readable_bytes(mem).c_str());
        std::fprintf(f, "# Memory usage (total) = %13s\n", readable_bytes(mem * ranks).c_str());
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# MSD                  = %13s\n", "Mandatory");
        std::fprintf(f, "# Waiting time         = %13s\n", tf(p.waiting_time));
        std::fprintf(f, "# Write trajectories   = %13s\n", tf(p.write_x));
        std::fprintf(f, "# V0 Distribution      = %13s\n", tf(p.distribution_v0));
        std::fprintf(f, "# Eta0 Distribution    = %13s\n", "false");
        std::fprintf(f, "# State0 Distribution  = %13s\n", tf(p.distribution_s0));
        std::fprintf(f, "# Eta result           = %13s\n", "false");
        std::fprintf(f, "# First passage time   = %13s\n", tf(p.fpt));
        if (p.fpt) {
            std::fprintf(f, "# Barrier hist hmin    = %13.7f\n", 0.0);
            std::fprintf(f, "# Barrier hist hmax    = %13.7f\n", 10.0);
            std::fprintf(f, "# Barrier hist nbin    = %13d\n", 100);
        }
        std::fprintf(f, "# Transtion path time  = %13s\n", tf(p.tpt));
        std::fprintf(f, "# First passage time CG= %13s\n", tf(p.fptcg));
        if (p.fptcg)
            for (int j = 0; j < p.n_cg; ++j) std::fprintf(f, "# FFT CG size %4d     = %13d\n", j, p.cg_sizes[j]);
        std::fprintf(f, "# X correlation        = %13s\n", "false");
        std::fprintf(f, "# ==============================================\n");
        std::fprintf(f, "# Read restart         = %13s\n", tf(p.read_restart));
        std::fprintf(f, "# Write restart        = %13s\n", tf(p.write_restart));
        std::fprintf(f, "# Input restart (base) = %13s\n", p.input_restart);
        std::fprintf(f, "# Output restart (base)= %13s\n", p.output_restart);
        std::fprintf(f, "# ==============================================\n");
    }

    void stat_log(const std::string& name, const std::vector<double>& v) const {
        FILE* f = open(name);
        if (!f) return;
        header(f);
        std::fprintf(f, "# average %23.16E\n", average(v));
        std::fprintf(f, "# sd      %23.16E\n", rmsd(v));
        std::fprintf(f, "# count   %23zd\n", v.size());
        std::fclose(f);
    }

    void dat(const std::string& name, const std::vector<double>& v) const {
        const std::string fn = path(name);
        backup(fn);
        FILE* f = std::fopen(fn.c_str(), "wb");
        if (!f) return;
        if (!v.empty()) std::fwrite(v.data(), sizeof(double), v.size(), f);
        std::fclose(f);
    }
};

}  // namespace

static ldp_status write_outputs_timed(ldp_job* job, const char* dir, double t_total, double t_integrate,
                                      double t_analysis, double t_post);

extern "C" ldp_status ldp_job_write_outputs(ldp_job* job, const char* dir) {
    return write_outputs_timed(job, dir, -1.0, -1.0, -1.0, -1.0);
}

static ldp_status write_outputs_timed(ldp_job* job, const char* dir, double t_total, double t_integrate,
                                      double t_analysis, double t_post) {
    if (!job) return LDP_ERR_INVALID;
    if (job->o.mode != LDP_MODE_FIXED_STEPS) {
        ldp_set_error(job->ctx, "output files are written for fixed-step jobs");
        return LDP_ERR_UNSUPPORTED;
    }
    const auto t_start = std::chrono::steady_clock::now();
    const ldp_params& p = job->p;
    const int64_t n = job->ntraj;
    const int64_t nf = job->nframe;
    const int64_t tc = job->o.tick_cap;
    std::vector<int64_t> counts((size_t)LDP_NCOUNT * n);
    std::vector<double> sums((size_t)LDP_NSUM * n), v0(n);
    std::vector<int32_t> state0(n);
    std::vector<int64_t> ticks(tc > 0 ? (size_t)tc * n : 0);
    std::vector<double> fx, fv, ff, fb, fpe, fke, fst;
    ldp_traj_results r;
    std::memset(&r, 0, sizeof(r));
    r.counts = counts.data();
    r.sums = sums.data();
    r.v0 = v0.data();
    r.state0 = state0.data();
    if (tc > 0) r.ticks = ticks.data();
    if (p.write_x) {
        for (auto* v : {&fx, &fv, &ff, &fb, &fpe, &fke, &fst}) v->resize((size_t)nf * n);
        r.frames_x = fx.data(); r.frames_v = fv.data(); r.frames_f = ff.data(); r.frames_barrier = fb.data();
        r.frames_pe = fpe.data(); r.frames_ke = fke.data(); r.frames_state = fst.data();
    }
    ldp_status st = ldp_job_traj_results(job, &r);
    if (st != LDP_OK) return st;
    const int64_t nl = (int64_t)job->lags.size();
    std::vector<int64_t> lags(nl);
    std::vector<double> msd(nl);
    st = ldp_job_msd(job, lags.data(), msd.data(), nl);
    if (st != LDP_OK) return st;

    Writer W{job, p, dir ? dir : "", job->o.ranks, job->o.lanes, p.number_of_runs, n, p.model == LDP_MODEL_DOUBLE};
    W.xc = job->k.xc;
    if (W.dbl) {
        const double x1b = p.barrier_position[0], w1 = p.barrier_half_width[0], y1 = p.barrier_heights[0][0];
        W.yc = ((x1b + w1) - W.xc) / ((x1b + w1) - x1b) * y1;
    }
    if (!W.dir.empty()) mkdir(W.dir.c_str(), 0755);
    const std::string base = p.output_base;
    const int R = W.ranks;
    const int64_t per_rank = n / R;
    auto mean_of = [&](int cf, int sf, int64_t g) {
        const int64_t c = counts[(size_t)cf * n + g];
        return c ? sums[(size_t)sf * n + g] / (double)c : 0.0;   // AVERAGE of an empty list is 0
    };
    auto means = [&](int cf, int sf) {
        std::vector<double> v(n);
        for (int64_t g = 0; g < n; ++g) v[g] = mean_of(cf, sf, g);
        return v;
    };

    // ---- FPT (S.h:3594-3663) ----
    if (p.fpt) {
        W.dat(base + "_firstPassageTime.dat", means(LDP_C_FPT, LDP_S_FPT));
        W.dat(base + "_firstPassageTime2.dat", means(LDP_C_FPT2, LDP_S_FPT2));
        // The per-lane histograms of the initial / instantaneous barrier state
        // lists (S.h:2734-2753) are filled by HISTOGRAM::HistogramVector,
        // whose loop takes its bounds from the arguments before they are
        // clamped (src/clsHistogram.cpp:246-255): called with the default
        // last = -1 it visits no element, so the reference's files always
        // hold empty histograms.  They are written the same way; the counts
        // themselves are the LDP_C_INIT0/1 and LDP_C_INST0/1 results.
        Hist hi, hs;
        hi.alloc(0.0, 10.0, 100);
        hs.alloc(0.0, 10.0, 100);
        W.stat_log(base + "_firstPassageTime.log", means(LDP_C_FPT, LDP_S_FPT));
        W.stat_log(base + "_firstPassageTime2.log", means(LDP_C_FPT2, LDP_S_FPT2));
        if (FILE* f = W.open(base + "_initialBarrierHeightHistogram.log")) { W.header(f); hi.print(f); std::fclose(f); }
        if (FILE* f = W.open(base + "_instantBarrierHeightHistogram.log")) { W.header(f); hs.print(f); std::fclose(f); }
    }
    // ---- state count (S.h:3665-3679) ----
    {
        double sc[2] = {0.0, 0.0};
        for (int rk = 0; rk < R; ++rk) {
            double part[2] = {0.0, 0.0};
            for (int64_t g = rk * per_rank; g < (rk + 1) * per_rank; ++g) {
                part[0] += (double)counts[(size_t)LDP_C_STATE0 * n + g];
                part[1] += (double)counts[(size_t)LDP_C_STATE1 * n + g];
            }
            sc[0] += part[0];
            sc[1] += part[1];
        }
        if (FILE* f = W.open(base + "_stateCount.log")) {
            W.header(f);
            std::fprintf(f, "# state 0 %23.0f %13.7f\n", sc[0], sc[0] / (sc[0] + sc[1]));
            std::fprintf(f, "# state 1 %23.0f %13.7f\n", sc[1], sc[1] / (sc[0] + sc[1]));
            std::fclose(f);
        }
    }
    // ---- TPT (S.h:3681-3731) ----
    if (p.tpt) {
        W.dat(base + "_transitionPathTime.dat", means(LDP_C_TPT, LDP_S_TPT));
        W.dat(base + "_transitionPathTime2.dat", means(LDP_C_TPT2, LDP_S_TPT2));
        W.stat_log(base + "_transitionPathTime.log", means(LDP_C_TPT, LDP_S_TPT));
        W.stat_log(base + "_transitionPathTime2.log", means(LDP_C_TPT2, LDP_S_TPT2));
    }
    // ---- FPT CG (S.h:3733-3770) ----
    if (p.fptcg) {
        std::vector<std::vector<double>> cg(p.n_cg);
        for (int j = 0; j < p.n_cg; ++j) {
            cg[j] = means(LDP_C_CG0 + j, LDP_S_CG0 + j);
            char b[64];
            std::snprintf(b, sizeof(b), "_firstPassageTimeCG2_%04d_%04d.dat", j, p.cg_sizes[j]);
            W.dat(base + b, cg[j]);
        }
        if (FILE* f = W.open(base + "_firstPassageTimeCG2.log")) {
            W.header(f);
            for (int j = 0; j < p.n_cg; ++j) {
                std::fprintf(f, "# %4d %4d\n", j, p.cg_sizes[j]);
                std::fprintf(f, "# average %23.16E\n", average(cg[j]));
                std::fprintf(f, "# sd      %23.16E\n", rmsd(cg[j]));
                std::fprintf(f, "# count   %23zd\n", cg[j].size());
            }
            std::fclose(f);
        }
    }
    // ---- V0 / State0 distributions (S.h:3772-3825) ----
    if (p.distribution_v0) {
        const double s = std::sqrt(p.kb * p.temperature / p.mass);
        Hist h;
        h.alloc(-s * 5.0, s * 5.0, 200);
        for (int64_t g = 0; g < n; ++g) h.add_trunc(v0[g]);
        h.normalize();
        if (FILE* f = W.open(base + "_V0Distribution.log")) { W.header(f); h.print(f); std::fclose(f); }
    }
    if (p.distribution_s0) {
        Hist h;
        h.alloc(0.0, 2.0, 2);
        for (int64_t g = 0; g < n; ++g) h.add_trunc((double)state0[g]);
        h.normalize();
        if (FILE* f = W.open(base + "_State0Distribution.log")) { W.header(f); h.print(f); std::fclose(f); }
    }
    // ---- MSD (S.h:3892-3912; double D.h:4566-4582 prints %13.7f) ----
    if (FILE* f = W.open(base + "_msd.log")) {
        W.header(f);
        const double ts = p.timestep * (double)p.freq_save;
        for (int64_t i = 0; i < nl; ++i) {
            if (W.dbl) std::fprintf(f, "%13.7f %13.7f\n", ts * (double)lags[i], msd[i]);
            else std::fprintf(f, "%14.7E %14.7E\n", ts * (double)lags[i], msd[i]);
        }
        std::fclose(f);
    }
    // ---- waiting time (S.h:3914-3970) ----
    if (p.waiting_time) {
        std::vector<std::vector<double>> wl(R);
        double sum = 0, sum2 = 0, cnt = 0, mx = 0;
        bool any = false;
        for (int rk = 0; rk < R; ++rk) {
            for (int64_t g = rk * per_rank; g < (rk + 1) * per_rank; ++g) {
                const int64_t k = std::min<int64_t>(counts[(size_t)LDP_C_WT * n + g], tc);
                for (int64_t t = 1; t < k; ++t)
                    wl[rk].push_back((double)(ticks[(size_t)g * tc + t] - ticks[(size_t)g * tc + t - 1]) * p.timestep);
            }
            double s = 0, s2 = 0, m = -1.7976931348623157e308;
            for (double x : wl[rk]) { s += x; s2 += x * x; m = std::max(m, x); }
            if (wl[rk].empty()) m = 0.0;   // STATISTICS::MAX of an empty list
            sum += s;
            sum2 += s2;
            cnt += (double)wl[rk].size();
            mx = any ? std::max(mx, m) : m;
            any = true;
        }
        const double avg = sum / cnt, avg2 = sum2 / cnt;
        const double Rr = (avg2 - avg * avg) / avg / avg;
        int nbin = 100;
        if (cnt < 1000) nbin = std::max(10, (int)cnt / 100);
        // Filled by HISTOGRAM::HistogramVector (S.h:3952), which visits no
        // element (see the barrier histograms above): the reference writes
        // the bins of the waiting times' range with zero counts.
        Hist h;
        h.alloc(0.0, mx + 0.1, nbin);
        if (FILE* f = W.open(base + "_waitingTime.log")) {
            W.header(f);
            std::fprintf(f, "# R      = %13.7f\n", Rr);
            std::fprintf(f, "# Nwt    = %13zd\n", (size_t)cnt);
            h.print(f);
            std::fclose(f);
        }
    }
    // ---- trajectory logs (S.h:3514-3554) ----
    if (p.write_x) {
        const double ts = p.timestep * (double)p.freq_save;
        for (int64_t g = 0; g < n; ++g) {
            const int lane = (int)(g % W.lanes);
            const int trial = (int)((g / W.lanes) % W.nruns);
            const int rk = job->o.first_rank + (int)(g / ((int64_t)W.lanes * W.nruns));   // rank in the run
            char b[256];
            std::snprintf(b, sizeof(b), "%s_trajectory_%010d_%010d_%010d.log", base.c_str(), trial, lane, rk);
            FILE* f = W.open(b);
            if (!f) continue;
            W.header(f);
            for (int64_t t = 0; t < nf; ++t) {
                const size_t o = (size_t)t * n + g;
                std::fprintf(f, " %23.16f %13.7f %13.7f %13.7f %13.7f %13.7f %13.7f %13.7f\n", ts * (double)t, fx[o],
                             p.overdamped ? 0.0 : fv[o], ff[o], fb[o], fpe[o], p.overdamped ? 0.0 : fke[o], fst[o]);
            }
            if (p.waiting_time) {
                std::fprintf(f, "# event tick\n");
                const int64_t k = std::min<int64_t>(counts[(size_t)LDP_C_WT * n + g], tc);
                for (int64_t t = 0; t < k; ++t)
                    std::fprintf(f, "# %10zd %23.16E\n", (size_t)t, (double)ticks[(size_t)g * tc + t] * p.timestep);
            }
            std::fclose(f);
        }
    }
    // ---- time.log (S.h:3977-4036) ----
    {
        const double post = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        ldp_timing tm;
        double integ = t_integrate, analysis = t_analysis, total = t_total, post_s = t_post;
        if (ldp_job_timing_get(job, &tm) == LDP_OK) {
            if (integ < 0) integ = tm.integrate_ms * 1e-3;
            if (analysis < 0) analysis = tm.msd_ms * 1e-3;
        }
        if (integ < 0) integ = 0;
        if (analysis < 0) analysis = 0;
        if (post_s < 0) post_s = post;
        if (total < 0) total = integ + analysis + post_s;
        if (FILE* f = W.open(base + "_time.log")) {
            for (int rk = 0; rk < R; ++rk) std::fprintf(f, "Rank %10d Seed %10d\n", rk, (int)job->seed);
            // one process: the spread over ranks is zero
            std::fprintf(f, "Time consumed %s %s\n", time_diff(total).c_str(), time_diff(0.0).c_str());
            std::fprintf(f, "Integrate     %s %s\n", time_diff(integ).c_str(), time_diff(0.0).c_str());
            std::fprintf(f, "Analysis      %s %s\n", time_diff(analysis).c_str(), time_diff(0.0).c_str());
            std::fprintf(f, "Post          %s %s\n", time_diff(post_s).c_str(), time_diff(0.0).c_str());
            std::fclose(f);
        }
    }
    return LDP_OK;
}

// The drop-in for `mpirun -n ranks ./langevinDynamics*Barrier -i path`:
// parse, run on the device, write every output file (LangevinEquationRunnerMPI
// ::Run, S.h:3216-4039).
extern "C" ldp_status ldp_run_inp(ldp_ctx* ctx, const char* path, int model, const ldp_job_opts* o,
                                  const char* outdir) {
    if (!ctx || !path) return LDP_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    ldp_params p;
    char err[1024];
    ldp_status st = ldp_params_from_inp(path, model, &p, err, sizeof(err));
    if (st != LDP_OK) {
        ldp_set_error(ctx, "%s", err);
        return st;
    }
    std::fprintf(stderr, "LangevinEquationMultipleRunner\n");
    ldp_job* job = nullptr;
    st = ldp_job_create(ctx, &p, o, &job);
    if (st != LDP_OK) return st;
    std::fprintf(stderr, "Interval = %10zd\n", job->lags.size());
    // READRESTART: continue the runs saved under INPUTRESTART (Integrate ->
    // PreIntegrate -> ReadRestartFile, S.h:1344-1348).
    if (p.read_restart) st = ldp_job_restore(job, p.input_restart);
    if (st == LDP_OK) st = ldp_submit(ctx, job);
    if (st == LDP_OK) st = ldp_wait(ctx, job);
    if (st == LDP_OK) {
        ldp_timing tm;
        ldp_job_timing_get(job, &tm);
        const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        st = write_outputs_timed(job, outdir, total, tm.integrate_ms * 1e-3, tm.msd_ms * 1e-3, -1.0);
    }
    // WRITERESTART: OUTPUTRESTART files after the run (S.h:1513-1517).
    if (st == LDP_OK && p.write_restart) {
        const std::string base = (outdir && *outdir) ? std::string(outdir) + "/" + p.output_restart
                                                     : std::string(p.output_restart);
        st = ldp_job_save_restart(job, base.c_str());
    }
    ldp_job_destroy(job);
    return st;
}
