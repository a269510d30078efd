// ldp_cli.cpp -- drop-in for `mpirun -n N ./langevinDynamics{Single,Double}Barrier`.
//
// Same flags as the reference (src/inputParser.cpp:45-87): -i file.inp runs,
// -o file.inp writes the default input file, -p prints the parsed values.
// Extra flags: -n N virtual ranks (the reference's mpirun -n), --lanes W
// trajectories per rank and trial (default 8), --fp32 for the FP32 batched
// path, --device D.  Exit code is non-zero on error (the reference exits 0).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "ldp.h"

#ifndef LDP_CLI_MODEL
#define LDP_CLI_MODEL 0
#endif
#ifndef LDP_CLI_NAME
#define LDP_CLI_NAME "langevinDynamicsSingleBarrier"
#endif

static void usage() {
    std::fprintf(stderr,
                 "usage: %s -i input.inp [-n ranks] [--lanes W] [--fp32] [--device D]\n"
                 "       %s -o new.inp   (write default input file)\n"
                 "       %s -i input.inp -p   (print parsed values)\n",
                 LDP_CLI_NAME, LDP_CLI_NAME, LDP_CLI_NAME);
}

int main(int argc, char** argv) {
    const char* in = nullptr;
    const char* out = nullptr;
    bool print = false;
    ldp_job_opts o;
    ldp_job_opts_default(&o);
    int device = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char* what) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "Error: %s needs a value\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-i" || a == "--input") in = next("-i");
        else if (a == "-o" || a == "--output") out = next("-o");
        else if (a == "-p" || a == "--print") print = true;
        else if (a == "-n") o.ranks = std::atoi(next("-n"));
        else if (a == "--lanes") o.lanes = std::atoi(next("--lanes"));
        else if (a == "--fp32") o.precision = LDP_PREC_FP32_BATCHED;
        else if (a == "--device") device = std::atoi(next("--device"));
        else {
            usage();
            return 2;
        }
    }
    if (in && out) {
        std::fprintf(stderr, "Error (InputParser): only one of -i and -o can be specified\n");
        return 2;
    }
    if (out) {
        ldp_status st = ldp_write_default_inp(out, LDP_CLI_MODEL);
        if (st != LDP_OK) {
            std::fprintf(stderr, "Error (InputParser): Can't open empty input file (%s)\n", out);
            return 1;
        }
        return 0;
    }
    if (!in) {
        usage();
        return 2;
    }
    ldp_params p;
    char err[1024];
    ldp_status st = ldp_params_from_inp(in, LDP_CLI_MODEL, &p, err, sizeof(err));
    if (st != LDP_OK) {
        std::fprintf(stderr, "%s\n", err);
        return 1;
    }
    if (print) {
        // every parsed option, as the reference's PrintAllValues
        size_t need = 0;
        std::string buf(1 << 16, '\0');
        st = ldp_inp_print_values(in, LDP_CLI_MODEL, &buf[0], buf.size(), &need);
        if (st == LDP_ERR_NOMEM) {
            buf.assign(need, '\0');
            st = ldp_inp_print_values(in, LDP_CLI_MODEL, &buf[0], buf.size(), &need);
        }
        std::fputs(buf.c_str(), stderr);
        return st == LDP_OK ? 0 : 1;
    }
    ldp_ctx* ctx = nullptr;
    st = ldp_create(&ctx, device);
    if (st != LDP_OK) {
        std::fprintf(stderr, "Error: no CUDA device available (%s)\n", ldp_status_string(st));
        return 1;
    }
    st = ldp_run_inp(ctx, in, LDP_CLI_MODEL, &o, nullptr);
    if (st != LDP_OK) std::fprintf(stderr, "Error: %s: %s\n", ldp_status_string(st), ldp_last_error(ctx));
    ldp_destroy(ctx);
    return st == LDP_OK ? 0 : 1;
}
