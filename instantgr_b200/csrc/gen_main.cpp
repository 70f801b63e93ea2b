// igr_generate: writes a seeded synthetic ISPD2024-format design (.cap, .net).
// A stand-alone program (it links the generator alone, not the router), so that
// the inputs of a routing run can be made by a process that loads no router code.
//
//   igr_generate --config C [--seed S] [--scale F] --cap <file> --net <file>
//                [--window X0 Y0 W H]
//
// --window writes only the W x H GCell window at (X0, Y0) of the same design:
// its capacities, and the nets whose access points all lie inside it.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "host.hpp"

int main(int argc, char **argv) {
    int cfg = -1;
    unsigned long long seed = 1;
    double scale = 1.0;
    const char *cap = nullptr, *net = nullptr;
    int win[4] = {0, 0, 0, 0};
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        auto val = [&](const char *what) -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", what);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--config") cfg = std::atoi(val("--config"));
        else if (a == "--seed") seed = std::strtoull(val("--seed"), nullptr, 10);
        else if (a == "--scale") scale = std::atof(val("--scale"));
        else if (a == "--cap") cap = val("--cap");
        else if (a == "--net") net = val("--net");
        else if (a == "--window")
            for (int k = 0; k < 4; k++) win[k] = std::atoi(val("--window"));
        else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 2;
        }
    }
    if (cfg < 0 || !cap || !net) {
        std::fprintf(stderr,
                     "usage: %s --config C [--seed S] [--scale F] --cap <file> --net <file> [--window X0 Y0 W H]\n",
                     argv[0]);
        return 2;
    }
    try {
        igr::GenParams p = igr::config_params(cfg, seed, scale);
        p.win_x0 = win[0];
        p.win_y0 = win[1];
        p.win_w = win[2];
        p.win_h = win[3];
        igr::generate_design(p, cap, net);
    } catch (const igr::Error &e) {
        std::fprintf(stderr, "igr_generate: error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}
