// Reference harness — TEST INFRASTRUCTURE ONLY.
//
// Compiled against InstantGR's own, unmodified sources (src/*.hpp, included
// from the reference tree by oracle/Makefile), it sets the reference's global
// device state from an input file and runs the reference's kernels and host
// routines on it, then writes their results.  The outputs are the golden
// vectors that pin the CPU oracle and the CUDA kernels of this project
// (tests/golden/make_golden.py drives it; it needs a GPU).
//
// Modes (all arrays little-endian, each prefixed by an int64 element count):
//   cost      grid, demand                     -> wcost, vcost, presum
//   pattern   grid, demand, cost map, trees    -> pre after the DP, routes, demand, stamps
//   ripup     grid, demand, routes             -> overflow nets, congestion view
//   dag       grid, demand, cost map, DAGs     -> pre after the DP, routes, demand, stamps
//   dagbuild  trees, congestion view           -> detour DAG CSR per net
#include "Lshape_route.hpp"
#include "Lshape_route_detour.hpp"
#include "graph.hpp"
#include "database.hpp"
#include "database_cuda.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace harness {

struct In {
    FILE *f;
    template <typename T>
    std::vector<T> arr() {
        long long n = 0;
        if (fread(&n, 8, 1, f) != 1) { fprintf(stderr, "short input\n"); exit(3); }
        std::vector<T> v((size_t)n);
        if (n && fread(v.data(), sizeof(T), (size_t)n, f) != (size_t)n) { fprintf(stderr, "short input\n"); exit(3); }
        return v;
    }
};
struct Out {
    FILE *f;
    template <typename T>
    void arr(const T *p, long long n) {
        fwrite(&n, 8, 1, f);
        if (n) fwrite(p, sizeof(T), (size_t)n, f);
    }
    template <typename T>
    void arr(const std::vector<T> &v) { arr(v.data(), (long long)v.size()); }
};

void check(const char *what) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e)); exit(4); }
}

template <typename T>
T *dev(const std::vector<T> &h, size_t extra = 0) {
    T *p = nullptr;
    cudaMalloc(&p, (h.size() + extra + 1) * sizeof(T));
    cudaMemset(p, 0, (h.size() + extra + 1) * sizeof(T));
    if (!h.empty()) cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
}
template <typename T>
std::vector<T> host(const T *p, size_t n) {
    std::vector<T> v(n);
    if (n) cudaMemcpy(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost);
    return v;
}

// grid: i32[L, X, Y, DIR], f64[unit_wire, unit_via], f64[L] short, i32 xlen, i32 ylen, f32 cap, f32 demand
void load_grid(In &in) {
    auto hd = in.arr<int>();
    auto uc = in.arr<double>();
    auto sc = in.arr<double>();
    auto xl = in.arr<int>();
    auto yl = in.arr<int>();
    auto cap = in.arr<float>();
    auto dem = in.arr<float>();
    cudb::L = hd[0]; cudb::X = hd[1]; cudb::Y = hd[2]; cudb::DIR = hd[3];
    cudb::XY = std::max(cudb::X, cudb::Y);
    cudb::unit_length_wire_cost = uc[0];
    cudb::unit_via_cost = uc[1];
    const size_t N = (size_t)cudb::L * cudb::X * cudb::Y;
    cudb::x_edge_len = dev(xl);
    cudb::y_edge_len = dev(yl);
    cudb::unit_length_short_costs = dev(sc);
    cudb::capacity = dev(cap);
    cudb::demand = dev(dem);
    cudaMalloc(&cudb::wcost, N * sizeof(float));
    cudaMalloc(&cudb::vcost, N * sizeof(float));
    cudaMalloc(&cudb::presum, N * sizeof(double));
    std::vector<int> zero_xy((size_t)cudb::X * cudb::Y, 0), zero_n(N, 0);
    cudb::cross_points = dev(zero_xy);
    cudb::pre_demand = dev(zero_n);
    cudb::timestamp = dev(zero_n);
    cudb::of_edge_sum = dev(zero_n);
    std::vector<int> tr;
    for (int l = 0; l < cudb::L; l++) {
        if ((l & 1 ^ cudb::DIR) == 0) for (int y = 0; y < cudb::Y; y++) tr.push_back(l * cudb::XY + y);
        if ((l & 1 ^ cudb::DIR) == 1) for (int x = 0; x < cudb::X; x++) tr.push_back(l * cudb::XY + x);
    }
    cudb::all_track_cnt = (int)tr.size();
    cudb::idx2track = dev(tr);
    cudaFuncSetAttribute(graph::compute_presum, cudaFuncAttributeMaxDynamicSharedMemorySize, 120 * 1024);
    cudaFuncSetAttribute(graph::compute_presum_general, cudaFuncAttributeMaxDynamicSharedMemorySize, 60 * 1024);
    check("grid");
}

size_t ncells() { return (size_t)cudb::L * cudb::X * cudb::Y; }

void load_costmap(In &in) {
    auto vc = in.arr<float>();
    auto ps = in.arr<double>();
    cudaMemcpy(cudb::vcost, vc.data(), vc.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(cudb::presum, ps.data(), ps.size() * 8, cudaMemcpyHostToDevice);
}

// per-net route slots: pins[k] "pins" of `per_pin` ints each (pin_acc_num layout)
void route_slots(const std::vector<int> &pins, int **acc, int &total) {
    std::vector<int> a(pins.size() + 1, 0);
    for (size_t k = 0; k < pins.size(); k++) a[k + 1] = a[k] + pins[k];
    total = a.back();
    *acc = dev(a);
}

int mode_cost(In &in, Out &out) {
    load_grid(in);
    graph::update_cost();
    graph::compute_presum<<<cudb::all_track_cnt, THREAD_NUM, sizeof(double) * cudb::XY>>>();
    check("cost");
    out.arr(host(cudb::wcost, ncells()));
    out.arr(host(cudb::vcost, ncells()));
    out.arr(host(cudb::presum, ncells()));
    return 0;
}

int mode_pattern(In &in, Out &out) {
    load_grid(in);
    load_costmap(in);
    const int stamp = in.arr<int>()[0];
    auto node_off = in.arr<int>();
    auto nodes = in.arr<int>();
    auto par = in.arr<int>();
    auto pins = in.arr<int>();
    const int n = (int)pins.size();
    int total = 0;
    route_slots(pins, &cudb::pin_acc_num, total);
    cudaMallocManaged(&cudb::routes, (ROUTE_PER_PIN * total + 1) * sizeof(int));
    cudaMemset(cudb::routes, 0, (ROUTE_PER_PIN * total + 1) * sizeof(int));
    std::vector<int> ids(n), zeros(n + 1, 0);
    for (int k = 0; k < n; k++) ids[k] = k;
    cudb::net_ids = dev(ids);
    cudb::ripup_flag = dev(zeros);
    cudb::NET_NUM = n;
    int max_nodes = 0;
    for (int k = 0; k < n; k++) max_nodes = std::max(max_nodes, node_off[k + 1] - node_off[k]);
    double *dist;
    int *from, *lr;
    cudaMalloc(&dist, (size_t)node_off[n] * 81 * sizeof(double));
    cudaMalloc(&from, (size_t)node_off[n] * 81 * sizeof(int));
    cudaMalloc(&lr, (size_t)node_off[n] * sizeof(int) + 4);
    int *d_off = dev(node_off), *d_nodes = dev(nodes), *d_par = dev(par);
    Lshape_route::Lshape_route_cuda<<<BLOCK_NUM(n), THREAD_NUM>>>(n, 0, d_off, d_nodes, d_par, dist, from, lr, stamp);
    check("Lshape_route_cuda");
    out.arr(host(cudb::pre_demand, ncells()));
    graph::batch_wire_update(stamp);
    graph::commit_via_demand<<<BLOCK_NUM(n), THREAD_NUM>>>(n, 0, stamp);
    check("commit");
    out.arr(host(cudb::routes, (size_t)ROUTE_PER_PIN * total + 1));
    out.arr(host(cudb::demand, ncells()));
    out.arr(host(cudb::timestamp, ncells()));
    return 0;
}

int mode_ripup(In &in, Out &out) {
    load_grid(in);
    auto pins = in.arr<int>();
    auto routes = in.arr<int>();
    const int n = (int)pins.size();
    int total = 0;
    route_slots(pins, &cudb::pin_acc_num, total);
    cudaMallocManaged(&cudb::routes, (ROUTE_PER_PIN * total + 1) * sizeof(int));
    cudaMemcpy(cudb::routes, routes.data(), routes.size() * 4, cudaMemcpyHostToDevice);
    std::vector<int> zeros(n + 1, 0);
    cudb::ripup_flag = dev(zeros);
    cudb::NET_NUM = n;
    cudaMalloc(&cudb::is_of_net, n + 1);
    cudaMalloc(&cudb::congestion, (size_t)cudb::X * cudb::Y);
    cudaMalloc(&cudb::congestion_xsum, (size_t)cudb::X * cudb::Y * 4);
    cudaMalloc(&cudb::congestion_ysum, (size_t)cudb::X * cudb::Y * 4);
    cudaMemset(cudb::congestion_xsum, 0, (size_t)cudb::X * cudb::Y * 4);
    cudaMemset(cudb::congestion_ysum, 0, (size_t)cudb::X * cudb::Y * 4);
    graph::extract_congestionView<<<BLOCK_NUM(cudb::L * cudb::X * cudb::Y), THREAD_NUM>>>();
    graph::extract_congestionView_xsum<<<cudb::Y, THREAD_NUM, sizeof(float) * cudb::X>>>();
    graph::extract_congestionView_ysum<<<cudb::X, THREAD_NUM, sizeof(float) * cudb::Y>>>();
    check("congestion view");
    auto of = graph::ripup(0);
    check("ripup");
    out.arr(of.first);
    out.arr(host(cudb::congestion_xsum, (size_t)cudb::X * cudb::Y));
    out.arr(host(cudb::congestion_ysum, (size_t)cudb::X * cudb::Y));
    return 0;
}

int mode_dag(In &in, Out &out) {
    load_grid(in);
    load_costmap(in);
    const int stamp = in.arr<int>()[0];
    auto node_off = in.arr<int>();
    auto nodes = in.arr<int>();
    auto depth = in.arr<int>();
    auto par_off = in.arr<int>();
    auto par = in.arr<int>();
    auto slot = in.arr<int>();
    auto child_num = in.arr<int>();
    auto pins = in.arr<int>();
    const int n = (int)pins.size(), N = node_off[n], E = par_off[N];
    int total = 0;
    route_slots(pins, &cudb::pin_acc_num_phase2, total);
    cudb::pin_acc_num = cudb::pin_acc_num_phase2;
    cudaMallocManaged(&cudb::routes_phase2, (ROUTE_PER_PIN_PHASE2 * total + 1) * sizeof(int));
    cudaMemset(cudb::routes_phase2, 0, (ROUTE_PER_PIN_PHASE2 * total + 1) * sizeof(int));
    cudaMallocManaged(&cudb::routes, 64);
    std::vector<int> ids(n), ones(n + 1, 1);
    for (int k = 0; k < n; k++) ids[k] = k;
    cudb::net_ids = dev(ids);
    cudb::ripup_flag = dev(ones);
    cudb::NET_NUM = n;
    std::vector<int> child_sum(N + 1, 0), cur_child(E), node_net(N), dn(N);
    for (int v = 0; v < N; v++) child_sum[v + 1] = child_sum[v] + child_num[v];
    for (int v = 0; v < N; v++)
        for (int e = par_off[v]; e < par_off[v + 1]; e++) cur_child[e] = v * 10 + slot[e];
    for (int k = 0; k < n; k++)
        for (int v = node_off[k]; v < node_off[k + 1]; v++) node_net[v] = k;
    int D = 0;
    for (int v = 0; v < N; v++) D = std::max(D, depth[v] + 1);
    std::vector<int> lev(D + 1, 0);
    for (int v = 0; v < N; v++) lev[depth[v] + 1]++;
    for (int d = 0; d < D; d++) lev[d + 1] += lev[d];
    std::vector<int> fill(lev.begin(), lev.end() - 1);
    for (int v = 0; v < N; v++) dn[fill[depth[v]]++] = v;
    using namespace Lshape_route_detour;
    Lshape_route_detour::nodes = dev(nodes);
    Lshape_route_detour::par_nodes = dev(par);
    Lshape_route_detour::par_num_sum = dev(par_off);
    Lshape_route_detour::child_num_sum = dev(child_sum);
    Lshape_route_detour::currentChildIDX = dev(cur_child);
    Lshape_route_detour::depth_node = dev(dn);
    Lshape_route_detour::node_net_idx = dev(node_net);
    const int slots = child_sum[N];
    cudaMalloc(&Lshape_route_detour::costs, (size_t)(N + 1) * MAX_LAYER * sizeof(double));
    cudaMalloc(&Lshape_route_detour::layer_output, (size_t)(N + 1) * sizeof(int));
    cudaMalloc(&Lshape_route_detour::best_path, (size_t)(slots + 1) * MAX_LAYER * 8);
    cudaMalloc(&Lshape_route_detour::packed_information, (size_t)(slots + 1) * MAX_LAYER * 8);
    cudaMalloc(&Lshape_route_detour::childCosts, (size_t)(slots + 1) * MAX_LAYER * 8);
    cudaMalloc(&Lshape_route_detour::childCosts_road, (size_t)(slots + 1) * MAX_LAYER * 4);
    cudaMalloc(&cost_edges, (size_t)(E + 1) * 81 * sizeof(double));
    cudaMalloc(&best_change, (size_t)(E + 1) * 81 * sizeof(int));
    cudaMemset(Lshape_route_detour::layer_output, 0xFF, (size_t)(N + 1) * sizeof(int));
    init_costs<<<N, 10>>>(N * MAX_LAYER);
    init_min_child_costs<<<(slots + 1) * MAX_LAYER, 1>>>((slots + 1) * MAX_LAYER);
    init_road<<<(slots + 1) * MAX_LAYER, 1>>>((slots + 1) * MAX_LAYER);
    check("init");
    precompute_cost_edge<<<BLOCK_NUM(E * 9), THREAD_NUM>>>(E);
    check("precompute_cost_edge");
    for (int d = D - 1; d >= 0; d--) {
        Lshape_route_node_layer_change_cuda<<<BLOCK_NUM(lev[d + 1] - lev[d] + 1), 512>>>(lev[d], lev[d + 1]);
        check("dp level");
    }
    for (int d = 0; d < D; d++) {
        get_routing_tree_layer_change_cuda<<<BLOCK_NUM(lev[d + 1] - lev[d] + 1), 512>>>(lev[d], lev[d + 1], d, stamp);
        check("trace level");
    }
    out.arr(host(cudb::pre_demand, ncells()));
    graph::batch_wire_update(stamp);
    graph::commit_via_demand<<<BLOCK_NUM(n), THREAD_NUM>>>(n, 0, stamp);
    check("commit");
    out.arr(host(cudb::routes_phase2, (size_t)ROUTE_PER_PIN_PHASE2 * total + 1));
    out.arr(host(cudb::demand, ncells()));
    out.arr(host(cudb::timestamp, ncells()));
    return 0;
}

int mode_dagbuild(In &in, Out &out) {
    auto hd = in.arr<int>();  // X, Y, mode
    cudb::X = hd[0];
    cudb::Y = hd[1];
    ::mode = hd[2];
    auto xs = in.arr<float>();
    auto ys = in.arr<float>();
    auto tree_off = in.arr<int>();  // per net node offsets
    auto pos = in.arr<int>();       // node positions (3-D, Steiner layer 9)
    auto adj_off = in.arr<int>();   // per node adjacency offsets (global)
    auto adj = in.arr<int>();       // neighbours (net-local)
    const int n = (int)tree_off.size() - 1;
    std::vector<int> res;
    for (int k = 0; k < n; k++) {
        cudb::net nt;
        const int a = tree_off[k], b = tree_off[k + 1];
        nt.rsmt.assign(b - a + 1, {});
        for (int v = a; v < b; v++)
            for (int q = adj_off[v]; q < adj_off[v + 1]; q++) nt.rsmt[v - a].push_back(adj[q]);
        nt.rsmt.back().assign(pos.begin() + a, pos.begin() + b);
        nt.generate_detours_reconstruct(nullptr, xs.data(), ys.data(), false, false, k);
        const int m = nt.node_index_cnt;
        res.push_back(m);
        res.insert(res.end(), nt.nodes_cpu.begin(), nt.nodes_cpu.begin() + m);
        res.insert(res.end(), nt.par_num_cpu.begin(), nt.par_num_cpu.begin() + m);
        res.insert(res.end(), nt.child_num_cpu.begin(), nt.child_num_cpu.begin() + m);
        res.insert(res.end(), nt.node_depth_cpu.begin(), nt.node_depth_cpu.begin() + m);
        const int E = nt.par_num_sum_cpu[m];
        res.push_back(E);
        res.insert(res.end(), nt.par_nodes_cpu.begin(), nt.par_nodes_cpu.begin() + E);
        res.insert(res.end(), nt.currentChildIDX_cpu.begin(), nt.currentChildIDX_cpu.begin() + E);
        res.push_back((int)nt.points.size());
        res.insert(res.end(), nt.points.begin(), nt.points.end());
    }
    out.arr(res);
    return 0;
}

}  // namespace harness

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s cost|pattern|ripup|dag|dagbuild <in> <out>\n", argv[0]);
        return 2;
    }
    harness::In in{fopen(argv[2], "rb")};
    harness::Out out{fopen(argv[3], "wb")};
    if (!in.f || !out.f) { fprintf(stderr, "cannot open files\n"); return 2; }
    std::string m = argv[1];
    int rc = 2;
    if (m == "cost") rc = harness::mode_cost(in, out);
    else if (m == "pattern") rc = harness::mode_pattern(in, out);
    else if (m == "ripup") rc = harness::mode_ripup(in, out);
    else if (m == "dag") rc = harness::mode_dag(in, out);
    else if (m == "dagbuild") rc = harness::mode_dagbuild(in, out);
    fclose(out.f);
    fclose(in.f);
    return rc;
}
