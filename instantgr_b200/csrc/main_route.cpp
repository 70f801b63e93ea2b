// igr_route: command-line drop-in for `InstantGR -cap <f> -net <f> -out <f>`
// (src/main.cpp:91-102).  InstantGR reads argv[2], argv[4], argv[6]
// positionally; here the flags are parsed by name, and the positional form
// keeps working.  Extra flags: --rrr-iters N, --threads N, --mode M, --verbose.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/instantgr_b200.h"

int main(int argc, char **argv) {
    const char *cap = nullptr, *net = nullptr, *out = nullptr;
    igr_options o;
    igr_default_options(&o);
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&](const char *what) -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-cap") cap = val("-cap");
        else if (a == "-net") net = val("-net");
        else if (a == "-out") out = val("-out");
        else if (a == "--rrr-iters") o.rrr_iters = std::atoi(val("--rrr-iters"));
        else if (a == "--threads") o.threads = std::atoi(val("--threads"));
        else if (a == "--mode") o.mode = std::atoi(val("--mode"));
        else if (a == "--batched") o.batched = 1;
        else if (a == "--host-dags") o.host_dags = 1;
        else if (a == "--verbose") o.verbose = 1;
        else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 2;
        }
    }
    if (!cap || !net || !out) {
        std::fprintf(stderr, "usage: %s -cap <file> -net <file> -out <file> [--rrr-iters N] [--threads N] [--verbose]\n",
                     argv[0]);
        return 2;
    }
    const int rc = igr_route_files(cap, net, out, &o);
    if (rc) {
        std::fprintf(stderr, "igr_route: error %d: %s\n", rc, igr_last_error(nullptr));
        return 1;
    }
    return 0;
}
