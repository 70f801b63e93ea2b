// Reference front end — TEST INFRASTRUCTURE ONLY.
//
// Runs InstantGR's own .cap/.net reader and pin access-point selection
// (db::read and net::init, src/database.hpp:38-415, compiled unmodified from
// the reference tree by oracle/Makefile) and prints, per net, the chosen pins
// in ascending order, then '|', then the stacked-pin vias as pairs.  Runs on
// the CPU; its output pins the reader and pin selection of this project.
#include "database.hpp"

#include <algorithm>
#include <cstdio>

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s <cap> <net> <out>\n", argv[0]);
        return 2;
    }
    db::read(argv[1], argv[2]);
    FILE *f = fopen(argv[3], "w");
    if (!f) return 2;
    for (auto &n : db::nets) {
        std::vector<int> p(n.pins);
        std::sort(p.begin(), p.end());
        for (int v : p) fprintf(f, "%d ", v);
        fprintf(f, "|");
        std::vector<std::pair<int, int>> ex;
        for (size_t i = 0; i + 1 < n.extra_routes.size(); i += 2) ex.push_back({n.extra_routes[i], n.extra_routes[i + 1]});
        std::sort(ex.begin(), ex.end());
        for (auto &e : ex) fprintf(f, "%d %d ", e.first, e.second);
        fprintf(f, "\n");
    }
    fclose(f);
    return 0;
}
