// Reference route on the host cores — CPU BASELINE AND TEST INFRASTRUCTURE ONLY.
//
// The CPU implementation of the routing path that the reference arm of bench.py
// times.  It is built from two parts, neither of which is this project's router:
//   * InstantGR's own host code, compiled unmodified from the reference tree by
//     oracle/Makefile (FLUTE replaced by the shared Steiner provider, as for the
//     reference router build): the .cap/.net reader and pin selection
//     (db::read, src/database.hpp:247-415), the split into routing nets
//     (build_cuda_database, src/database_cuda.hpp:2096-2237), Steiner trees and
//     conflict shapes (net::construct_rsmt, :746-820), its host batch colouring
//     (generate_batches_rsmt, :634-693) and its detour-DAG builder
//     (net::generate_detours_reconstruct, :1429-2086);
//   * the oracle (oracle.c) for the stages the reference runs only as CUDA
//     kernels: cost refresh, tree DP, commits, rip-up marking, congestion view
//     and DAG DP, on all host cores (OpenMP).
// build_cuda_database also uploads the grid to the device, as the reference
// does; nothing runs on the device afterwards.
//
// One step is one complete route of the design, with the design read and its
// trees built beforehand (as the router's own timed step): HPWL order, host
// colouring, phase 1 batch by batch (cost refresh, tree DP, wire and via
// commit), then `rrr_iters` rip-up-and-reroute passes (overflow marking,
// congestion view, detour DAGs on all host threads, colouring, per batch:
// rip-up, cost refresh, DAG DP, commit).
//
//   ref_cpu <cap> <net> <steps> <warmup> <rrr_iters> <threads>
//   ref_cpu <cap> <net> trees <out>
//
// Output: lines starting with "REFCPU " followed by one JSON object, a setup
// record and then one record per step; everything else on stdout is the
// reference's own logging.  The `trees` form writes, for every routing net in
// the reference's order, its original design net, its pins and its tree in
// DFS preorder (little-endian int32: net count, then per net: design net,
// pin count, pins, node count, nodes, parents) and exits.
#include "Lshape_route.hpp"
#include "Lshape_route_detour.hpp"
#include "graph.hpp"
#include "database.hpp"
#include "database_cuda.hpp"

#include "oracle.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <string>
#include <thread>
#include <vector>

namespace refcpu {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Tree {
    std::vector<int> nodes, par;  // DFS preorder (Lshape_route.hpp:191-208)
};

// DFS flattening of a net's tree from node 0, children in adjacency order
// (the order of Lshape_route.hpp:198-205)
void dfs_tree(const cudb::net &nt, Tree &t) {
    const auto &graph = nt.rsmt;
    const int m = (int)graph.back().size();
    t.nodes.assign(m, 0);
    t.par.assign(m, -1);
    int cnt = 0;
    std::function<void(int, int, int)> dfs = [&](int x, int par, int par_idx) {
        const int idx = cnt++;
        t.nodes[idx] = graph.back()[x];
        t.par[idx] = par_idx;
        for (int e : graph[x])
            if (e != par) dfs(e, x, idx);
    };
    dfs(0, -1, -1);
}

struct Step {
    double seconds = 0;
    int batches1 = 0;
    std::vector<int> rerouted, batches2;
    long long wirelength = 0, vias = 0;
};

struct Route {
    orc_grid g{};
    int R = 0;
    std::vector<Tree> trees;
    std::vector<std::vector<int>> points0;  // phase-1 conflict points of every routing net
    std::vector<int> tree_cap;              // phase-1 record capacity
    std::vector<float> cap;
    int threads = 1;

    std::vector<float> dem;
    std::vector<int> pre, stamp;
    std::vector<int> routes;
    std::vector<int64_t> cur_off;
    std::vector<int> cur_cap;
    std::vector<float> xsum, ysum;
    std::vector<int> dag_touched;
    int gstamp = 0;

    void setup(int thr) {
        threads = thr;
        using namespace cudb;
        R = (int)nets.size();
        trees.resize(R);
        points0.resize(R);
        tree_cap.resize(R);
        for (int i = 0; i < R; i++) {
            nets[i].construct_rsmt(false, false);
            dfs_tree(nets[i], trees[i]);
            points0[i] = nets[i].points;
            tree_cap[i] = std::max(12 * (int)nets[i].pins.size(), 8 * (int)trees[i].nodes.size() + 1);
        }
        const size_t N = (size_t)L * X * Y;
        cap.resize(N);
        for (int l = 0; l < L; l++)
            for (int x = 0; x < X; x++)
                for (int y = 0; y < Y; y++) cap[((size_t)l * X + x) * Y + y] = (float)db::capacity[l + 1][x][y];
        static std::vector<double> shortc;
        shortc.resize(L);
        for (int l = 0; l < L; l++) shortc[l] = db::unit_length_short_costs[l + 1];
        g.L = L; g.X = X; g.Y = Y; g.DIR = DIR;
        g.xlen = db::x_edge_len.data();
        g.ylen = db::y_edge_len.data();
        g.unit_wire = db::unit_length_wire_cost;
        g.unit_via = db::unit_via_cost;
        g.short_cost = shortc.data();
        g.cap = cap.data();
        dem.assign(N, 0.f);
        pre.assign(N, 0);
        stamp.assign(N, 0);
        xsum.assign((size_t)X * Y, 0.f);
        ysum.assign((size_t)X * Y, 0.f);
    }

    void cost_refresh(std::vector<float> &wc, std::vector<float> &vc, std::vector<double> &ps) {
        orc_cost_refresh(&g, dem.data(), wc.data(), vc.data(), ps.data());
    }

    Step run(int rrr_iters) {
        using namespace cudb;
        Step st;
        const double t0 = now();
        const size_t N = (size_t)L * X * Y;
        // state of a fresh route; conflict points of the previous step's DAGs restored
        for (int i : dag_touched) nets[i].points = points0[i];
        dag_touched.clear();
        std::fill(dem.begin(), dem.end(), 0.f);
        std::fill(pre.begin(), pre.end(), 0);
        std::fill(stamp.begin(), stamp.end(), 0);
        gstamp = 0;
        std::vector<float> wc(N), vc(N);
        std::vector<double> ps(N);
        // phase 1 (Lshape_route.hpp:155-257): HPWL order, colouring, batches
        std::vector<int> order(R);
        for (int i = 0; i < R; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [](int l, int r) { return nets[l].hpwl > nets[r].hpwl; });
        auto batches = generate_batches_rsmt(order);
        std::reverse(batches.begin(), batches.end());
        st.batches1 = (int)batches.size();
        cur_off.assign(R, 0);
        cur_cap.assign(R, 0);
        int64_t total = 0;
        for (auto &b : batches)
            for (int id : b) {
                cur_off[id] = total;
                cur_cap[id] = tree_cap[id];
                total += tree_cap[id];
            }
        routes.assign((size_t)total + 1, 0);
        std::vector<int> node_off, nodes, par, rcap;
        std::vector<int64_t> roff;
        for (auto &b : batches) {
            const int n = (int)b.size();
            node_off.assign(n + 1, 0);
            nodes.clear();
            par.clear();
            roff.resize(n);
            rcap.resize(n);
            for (int k = 0; k < n; k++) {
                const Tree &t = trees[b[k]];
                nodes.insert(nodes.end(), t.nodes.begin(), t.nodes.end());
                par.insert(par.end(), t.par.begin(), t.par.end());
                node_off[k + 1] = (int)nodes.size();
                roff[k] = cur_off[b[k]];
                rcap[k] = cur_cap[b[k]];
            }
            const int s = ++gstamp;
            cost_refresh(wc, vc, ps);
            orc_pattern_route(&g, vc.data(), ps.data(), n, node_off.data(), nodes.data(), par.data(), roff.data(),
                              rcap.data(), routes.data(), pre.data(), stamp.data(), s);
            st.wirelength += orc_commit_wires(&g, pre.data(), dem.data(), stamp.data(), s);
            st.vias += orc_commit_vias(&g, n, roff.data(), routes.data(), dem.data(), stamp.data(), s, 1);
        }
        // rip-up and reroute (main.cpp:42-68, Lshape_route_detour.hpp:726-1112)
        std::vector<uint8_t> is_of(R);
        for (int it = 0; it < rrr_iters; it++) {
            orc_mark_overflow(&g, dem.data(), R, cur_off.data(), routes.data(), 0, 10, is_of.data());
            std::vector<int> of;
            for (int i = 0; i < R; i++)
                if (is_of[i]) of.push_back(i);
            st.rerouted.push_back((int)of.size());
            if (of.empty()) break;
            orc_congestion_view(&g, dem.data(), xsum.data(), ysum.data());
            std::sort(of.begin(), of.end(), [](int l, int r) { return nets[l].hpwl > nets[r].hpwl; });
            // detour DAGs on all host threads (the reference uses 8, Lshape_route_detour.hpp:702-724)
            {
                std::atomic<int> next(0);
                std::vector<std::thread> pool;
                float *xs = xsum.data(), *ys = ysum.data();
                for (int t = 0; t < threads; t++)
                    pool.emplace_back([&] {
                        for (;;) {
                            const int k = next.fetch_add(1);
                            if (k >= (int)of.size()) break;
                            nets[of[k]].generate_detours_reconstruct(nullptr, xs, ys, false, false);
                        }
                    });
                for (auto &th : pool) th.join();
            }
            for (int i : of) dag_touched.push_back(i);
            // the DP keeps at most 10 child slots per node (decimal slot digit):
            // larger DAGs keep their current route
            {
                std::vector<int> kept;
                for (int i : of) {
                    bool ok = true;
                    for (int v = 0; v < nets[i].node_index_cnt; v++) ok = ok && nets[i].child_num_cpu[v] <= 10;
                    if (ok) kept.push_back(i);
                }
                of.swap(kept);
            }
            auto b2 = generate_batches_rsmt(of, 300000);
            st.batches2.push_back((int)b2.size());
            std::vector<int> depth, par_off, child_slot, child_num;
            std::vector<int64_t> old_off;
            for (int ii = (int)b2.size() - 1; ii >= 0; ii--) {
                const auto &b = b2[ii];
                const int n = (int)b.size();
                node_off.assign(n + 1, 0);
                nodes.clear(); depth.clear(); par_off.assign(1, 0); par.clear(); child_slot.clear(); child_num.clear();
                roff.resize(n);
                rcap.resize(n);
                old_off.resize(n);
                for (int k = 0; k < n; k++) {
                    const cudb::net &nt = nets[b[k]];
                    const int m = nt.node_index_cnt, base = (int)nodes.size();
                    int q = 0;
                    for (int v = 0; v < m; v++) {
                        nodes.push_back(nt.nodes_cpu[v]);
                        depth.push_back(nt.node_depth_cpu[v]);
                        child_num.push_back(nt.child_num_cpu[v]);
                        for (int p = 0; p < nt.par_num_cpu[v]; p++, q++) {
                            par.push_back(base + nt.par_nodes_cpu[q]);
                            child_slot.push_back(nt.currentChildIDX_cpu[q]);
                        }
                        par_off.push_back((int)par.size());
                    }
                    node_off[k + 1] = (int)nodes.size();
                    old_off[k] = cur_off[b[k]];
                    rcap[k] = 8 * m + 1;
                    roff[k] = (int64_t)routes.size();
                    routes.resize(routes.size() + rcap[k], 0);
                }
                const int s1 = ++gstamp;
                orc_ripup_wires(&g, n, old_off.data(), routes.data(), dem.data(), stamp.data(), s1, -1);
                orc_commit_vias(&g, n, old_off.data(), routes.data(), dem.data(), stamp.data(), s1, -1);
                const int s2 = ++gstamp;
                cost_refresh(wc, vc, ps);
                orc_dag_route(&g, vc.data(), ps.data(), n, node_off.data(), nodes.data(), depth.data(), par_off.data(),
                              par.data(), child_slot.data(), child_num.data(), roff.data(), rcap.data(), routes.data(),
                              pre.data(), stamp.data(), s2);
                orc_commit_wires(&g, pre.data(), dem.data(), stamp.data(), s2);
                orc_commit_vias(&g, n, roff.data(), routes.data(), dem.data(), stamp.data(), s2, 1);
                for (int k = 0; k < n; k++) {
                    cur_off[b[k]] = roff[k];
                    cur_cap[b[k]] = rcap[k];
                }
            }
        }
        st.seconds = now() - t0;
        return st;
    }
};

void emit(const char *fmt_json) { std::printf("REFCPU %s\n", fmt_json); std::fflush(stdout); }

std::string ints(const std::vector<int> &v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); i++) s += (i ? "," : "") + std::to_string(v[i]);
    return s + "]";
}

}  // namespace refcpu

// routing nets and their trees as the reference builds them (build_cuda_database,
// construct_rsmt, the DFS of Lshape_route.hpp:191-208)
int dump_trees(const char *path) {
    using namespace cudb;
    FILE *f = std::fopen(path, "wb");
    if (!f) return 2;
    auto put = [&](int v) { std::fwrite(&v, 4, 1, f); };
    put((int)nets.size());
    for (auto &nt : nets) {
        nt.construct_rsmt(false, false);
        refcpu::Tree t;
        refcpu::dfs_tree(nt, t);
        put(nt.original_net_id);
        put((int)nt.pins.size());
        for (int p : nt.pins) put(p);
        put((int)t.nodes.size());
        for (int v : t.nodes) put(v);
        for (int v : t.par) put(v);
    }
    std::fclose(f);
    return 0;
}

int main(int argc, char **argv) {
    if (argc == 5 && std::string(argv[3]) == "trees") {
        program_start = std::chrono::high_resolution_clock::now();
        db::read(argv[1], argv[2]);
        build_cuda_database();
        const int rc = dump_trees(argv[4]);
        std::fflush(stdout);
        quick_exit(rc);
    }
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s <cap> <net> <steps> <warmup> <rrr_iters> <threads>\n", argv[0]);
        return 2;
    }
    const int steps = std::atoi(argv[3]), warmup = std::atoi(argv[4]), rrr = std::atoi(argv[5]);
    int threads = std::atoi(argv[6]);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    program_start = std::chrono::high_resolution_clock::now();
    const double t0 = refcpu::now();
    db::read(argv[1], argv[2]);
    const double t1 = refcpu::now();
    build_cuda_database();
    refcpu::Route r;
    r.setup(threads);
    const double t2 = refcpu::now();
    char buf[512];
    std::snprintf(buf, sizeof buf,
                  "{\"kind\": \"setup\", \"design_nets\": %zu, \"routing_nets\": %d, \"X\": %d, \"Y\": %d, "
                  "\"read_s\": %.3f, \"nets_trees_s\": %.3f, \"threads\": %d}",
                  db::nets.size(), r.R, cudb::X, cudb::Y, t1 - t0, t2 - t1, threads);
    refcpu::emit(buf);
    for (int i = 0; i < warmup + steps; i++) {
        refcpu::Step s = r.run(rrr);
        std::string js = "{\"kind\": \"step\", \"timed\": " + std::string(i >= warmup ? "true" : "false") +
                         ", \"seconds\": " + std::to_string(s.seconds) + ", \"batches1\": " +
                         std::to_string(s.batches1) + ", \"rerouted\": " + refcpu::ints(s.rerouted) +
                         ", \"batches2\": " + refcpu::ints(s.batches2) + ", \"wirelength1\": " +
                         std::to_string(s.wirelength) + ", \"vias1\": " + std::to_string(s.vias) + "}";
        refcpu::emit(js.c_str());
    }
    std::fflush(stdout);
    quick_exit(0);
}
