// Reference front end — TEST INFRASTRUCTURE ONLY.
//
// Runs InstantGR's own .cap/.net reader and pin access-point selection
// (db::read and net::init, src/database.hpp:38-415, compiled unmodified from
// the reference tree by oracle/Makefile) and prints, per net, the chosen pins
// in the order net::init leaves them (the iteration order of its robin_hood
// sets), then '|', then the stacked-pin vias as pairs in their order.  Runs on
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
        for (int v : n.pins) fprintf(f, "%d ", v);
        fprintf(f, "|");
        for (size_t i = 0; i + 1 < n.extra_routes.size(); i += 2)
            fprintf(f, "%d %d ", n.extra_routes[i], n.extra_routes[i + 1]);
        fprintf(f, "\n");
    }
    fclose(f);
    return 0;
}
