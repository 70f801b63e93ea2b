// Rip-up-and-reroute driver (src/main.cpp:22-73, src/Lshape_route.hpp:155-257,
// src/Lshape_route_detour.hpp:726-1112), restated for one GPU:
//
//   phase 1   HPWL order -> GPU colouring -> per batch: cost refresh, tree DP,
//             wire commit, via commit
//   pass i    overflow marking -> congestion view -> detour DAGs of the marked
//             nets (host threads) -> GPU colouring -> per batch: rip-up, cost
//             refresh, DAG DP, wire commit, via commit
//
// InstantGR runs one pass; rrr_iters > 1 repeats the pass on the nets that
// still overflow.  All per-batch work is stream-ordered with no host
// synchronisation between batches (the reference synchronises after every
// phase-2 launch).
#include "router.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

namespace igr {

void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw Error(ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ grid
void GridOwner::create(int L, int X, int Y, int DIR, const int *xl, const int *yl, double unit_wire,
                       double unit_via, const double *sc, const float *cap_ref, cudaStream_t s) {
    if (L != kRouteLayers) throw Error(ERR_INVALID, "the router handles 9 routing layers");
    if (X < 2 || Y < 2) throw Error(ERR_INVALID, "grid must be at least 2x2");
    if (X > 4096 || Y > 4096) throw Error(ERR_CAPACITY, "tracks longer than 4096 GCells are not supported");
    g = GridDev();
    g.L = L; g.X = X; g.Y = Y; g.DIR = DIR;
    g.N = (int64_t)L * X * Y;
    layer_first.assign(L + 1, 0);
    for (int l = 0; l < L; l++) layer_first[l + 1] = layer_first[l] + ((((l & 1) ^ DIR) != 0) ? X : Y);
    g.ntracks = layer_first[L];
    g.unit_wire = unit_wire;
    g.unit_via = unit_via;
    cap.alloc(g.N); demand.alloc(g.N); vcost.alloc(g.N); presum.alloc(g.N);
    pre.alloc(g.N); stamp.alloc(g.N);
    xlen.upload(xl, X - 1, s); ylen.upload(yl, Y - 1, s);
    short_cost.upload(sc, L, s);
    dirty_cost.alloc(g.ntracks); dirty_commit.alloc(g.ntracks);
    stats.alloc(4); err.alloc(1);
    score.alloc(g.ntracks + 1);
    g.cap = cap.p; g.demand = demand.p; g.vcost = vcost.p; g.presum = presum.p;
    g.pre = pre.p; g.stamp = stamp.p; g.xlen = xlen.p; g.ylen = ylen.p; g.short_cost = short_cost.p;
    g.dirty_cost = dirty_cost.p; g.dirty_commit = dirty_commit.p; g.stats = stats.p; g.err = err.p;
    // capacity: reference layout -> track layout through a staging buffer
    DevBuf<float> tmp;
    tmp.upload(cap_ref, g.N, s);
    launch_to_track_layout(g, tmp.p, cap.p, s);
    cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(vcost.p, 0, g.N * sizeof(float), s), "memset");
    cuda_check(cudaMemsetAsync(presum.p, 0, g.N * sizeof(double), s), "memset");
    reset_demand(s);
    cuda_check(cudaStreamSynchronize(s), "create");
}

void GridOwner::reset_demand(cudaStream_t s) {
    cuda_check(cudaMemsetAsync(demand.p, 0, g.N * sizeof(float), s), "memset");
    cuda_check(cudaMemsetAsync(pre.p, 0, g.N * sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(stamp.p, 0, g.N * sizeof(int), s), "memset");
    cuda_check(cudaMemsetAsync(stats.p, 0, 4 * sizeof(unsigned long long), s), "memset");
    cuda_check(cudaMemsetAsync(dirty_commit.p, 0, g.ntracks, s), "memset");
    mark_all_dirty(s);
}

void GridOwner::mark_all_dirty(cudaStream_t s) {
    cuda_check(cudaMemsetAsync(dirty_cost.p, 1, g.ntracks, s), "memset");
}

int GridOwner::check_error(cudaStream_t s) {
    int e = 0;
    cuda_check(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (e) cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    return e;
}

// ------------------------------------------------------------------ kernel timer
void KernelTimer::begin(int k) {
    if (!on) return;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    ev[k].push_back({a, b});
}
void KernelTimer::end(int k) {
    if (!on) return;
    cudaEventRecord(ev[k].back().second, s);
    launches[k]++;
}
void KernelTimer::collect() {
    for (int k = 0; k < KC_N; k++) {
        for (auto &p : ev[k]) {
            float t = 0;
            if (cudaEventElapsedTime(&t, p.first, p.second) == cudaSuccess) ms[k] += t;
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        ev[k].clear();
    }
}
void KernelTimer::reset() {
    collect();
    for (int k = 0; k < KC_N; k++) { ms[k] = 0; launches[k] = 0; }
}

// ------------------------------------------------------------------ router
Router::~Router() {
    kt.collect();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (s) cudaStreamDestroy(s);
}

void Router::open(const char *cap, const char *net) {
    const double t0 = now_s();
    read_design(d, cap, net, threads);
    build_netset(d, ns, threads);
    if (verbose) std::fprintf(stderr, "[igr] read+trees %.2fs: %d nets, %zu routing nets\n", now_s() - t0,
                              d.num_nets(), ns.nets.size());
}

// Device state is created on the first run, so that opening a design (parsing,
// pin selection, trees) needs no GPU.
void Router::ensure_device() {
    if (s) return;
    cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    cuda_check(cudaEventCreate(&ev0), "event");
    cuda_check(cudaEventCreate(&ev1), "event");
    const int L = d.L - 1, X = d.X, Y = d.Y;
    std::vector<float> capr((size_t)L * X * Y);
    std::memcpy(capr.data(), d.cap.data() + (size_t)X * Y, capr.size() * sizeof(float));
    std::vector<double> sc(L);
    for (int l = 0; l < L; l++) sc[l] = d.short_cost[l + 1];
    go.create(L, X, Y, d.layer_dir[1], d.x_edge_len.data(), d.y_edge_len.data(), d.unit_wire, d.unit_via, sc.data(),
              capr.data(), s);
}

void Router::grow_routes(int64_t need) {
    if ((int64_t)routes.n >= need) return;
    DevBuf<int> nb;
    nb.alloc((size_t)std::max<int64_t>(need, (int64_t)(routes.n * 3 / 2)));
    if (routes.p && route_end > 0)
        cuda_check(cudaMemcpyAsync(nb.p, routes.p, route_end * sizeof(int), cudaMemcpyDeviceToDevice, s), "D2D");
    std::swap(routes.p, nb.p);
    std::swap(routes.n, nb.n);
}

void Router::run() {
    ensure_device();
    const double t0 = now_s();
    st = RouterStats();
    kt.s = s;
    kt.reset();
    go.reset_demand(s);
    global_stamp = 0;
    const int R = (int)ns.nets.size();
    route_off.assign(R, 0);
    route_cap.assign(R, 0);
    route_end = 0;
    int m = mode;
    if (m < 0) m = R > 20000000 ? 2 : (R > 5000000 ? 1 : 0);
    mode_eff = m;
    phase1();
    for (int it = 0; it < rrr_iters; it++)
        if (!rrr_pass(it)) break;
    // host copy of all route records
    h_routes.resize(route_end);
    if (route_end)
        cuda_check(cudaMemcpyAsync(h_routes.data(), routes.p, route_end * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (int e = go.check_error(s)) throw Error(e, "device error during routing");
    st.wall = now_s() - t0;
    kt.collect();
    compute_score();
    if (verbose)
        std::fprintf(stderr, "[igr] route %.3fs  WL %.0f  via %.0f  OF %.0f  total %.0f\n", st.wall, score_wl,
                     score_via, score_of, score_wl + score_via + score_of);
}

// Phase 1 (Lshape_route.hpp:155-257)
void Router::phase1() {
    const int R = (int)ns.nets.size();
    const int X = ns.X, Y = ns.Y;
    std::vector<int> order(R);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int l, int r) { return ns.nets[l].hpwl > ns.nets[r].hpwl; });
    std::vector<std::vector<int>> batches;
    color_nets(order, false, 15, batches);
    std::reverse(batches.begin(), batches.end());
    st.batches1 = (int)batches.size();
    // routing order, tree CSR, route records
    std::vector<int> net_ids, batch_off{0}, node_off{0};
    net_ids.reserve(R);
    for (auto &b : batches) {
        net_ids.insert(net_ids.end(), b.begin(), b.end());
        batch_off.push_back((int)net_ids.size());
    }
    int64_t tot_nodes = 0;
    for (int id : net_ids) {
        tot_nodes += (int64_t)ns.nets[id].tnode.size();
        node_off.push_back((int)tot_nodes);
    }
    std::vector<int> nodes(tot_nodes), par(tot_nodes);
    parallel_for(R, threads, [&](int b, int e) {
        for (int k = b; k < e; k++) flatten_tree(ns.nets[net_ids[k]], nodes.data() + node_off[k], par.data() + node_off[k]);
    });
    for (int id = 0; id < R; id++) {
        const auto &n = ns.nets[id];
        route_cap[id] = (int)std::max<int64_t>(12 * (int64_t)n.pins.size(), 8 * (int64_t)n.tnode.size() + 1);
        route_off[id] = route_end;
        route_end += route_cap[id];
    }
    std::vector<int64_t> scratch_off(R, -1);
    int64_t scratch_nodes = 0;
    for (int k = 0; k < R; k++) {
        int cnt = node_off[k + 1] - node_off[k];
        if (cnt > kPatternNodeTile) { scratch_off[k] = scratch_nodes; scratch_nodes += cnt; }
    }
    grow_routes(route_end);
    DevBuf<int> d_ids, d_node_off, d_nodes, d_par;
    DevBuf<int64_t> d_scr_off;
    DevBuf<double> d_scr;
    d_ids.upload(net_ids, s); d_node_off.upload(node_off, s); d_nodes.upload(nodes, s); d_par.upload(par, s);
    d_route_off.upload(route_off, s); d_route_cap.upload(route_cap, s);
    d_scr_off.upload(scratch_off, s);
    d_scr.alloc((size_t)pattern_scratch_doubles(scratch_nodes));
    cuda_check(cudaEventRecord(ev0, s), "event");
    for (size_t bi = 0; bi + 1 < batch_off.size(); bi++) {
        const int off = batch_off[bi], n = batch_off[bi + 1] - off;
        const int stamp = ++global_stamp;
        kt.begin(KC_COST);
        launch_cost_refresh(go.g, true, s);
        kt.end(KC_COST);
        TreeBatchDev tb{d_ids.p + off, d_node_off.p + off, d_nodes.p, d_par.p, d_route_off.p, d_route_cap.p,
                        routes.p, d_scr.p, d_scr_off.p + off, scratch_nodes, n};
        kt.begin(KC_PATTERN);
        launch_pattern_route(go.g, tb, stamp, s);
        kt.end(KC_PATTERN);
        kt.begin(KC_WIRE_COMMIT);
        launch_wire_commit(go.g, stamp, true, s);
        kt.end(KC_WIRE_COMMIT);
        ViaBatchDev vb{d_ids.p + off, d_route_off.p, routes.p, n};
        kt.begin(KC_VIA_COMMIT);
        launch_via_commit(go.g, vb, stamp, 1, s);
        kt.end(KC_VIA_COMMIT);
        st.launches += 4;
    }
    cuda_check(cudaEventRecord(ev1, s), "event");
    cuda_check(cudaGetLastError(), "phase-1 launch");
    plan_ids = net_ids;
    plan_batch_off = batch_off;
    plan_node_off = node_off;
    plan_nodes.swap(nodes);
    plan_par.swap(par);
    plan_cap.resize(net_ids.size());
    for (size_t k = 0; k < net_ids.size(); k++) plan_cap[k] = route_cap[net_ids[k]];
    cuda_check(cudaEventSynchronize(ev1), "phase 1");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    st.p1_ms = ms;
    if (int e = go.check_error(s)) throw Error(e, "device error in phase 1");
    (void)X; (void)Y;
    if (verbose) std::fprintf(stderr, "[igr] phase 1: %zu batches, %.2f ms device\n", batches.size(), ms);
}

// Colours `order` (highest priority first) into batches of spatially disjoint
// nets (database_cuda.hpp:437-631); the colouring ranks the reversed list.
void Router::color_nets(const std::vector<int> &order, bool dag_points, int sparsity,
                        std::vector<std::vector<int>> &batches) {
    const int n = (int)order.size();
    batches.clear();
    if (n == 0) return;
    std::vector<int> list(order.rbegin(), order.rend());
    std::vector<int> pt_off{0}, pts, pt_net, h_off{0}, hs, v_off{0}, vs;
    for (int k = 0; k < n; k++) {
        const RNet &r = ns.nets[list[k]];
        const std::vector<int> &p = dag_points ? dag[list[k]].points : r.points;
        for (int q : p) { pts.push_back(q); pt_net.push_back(k); }
        pt_off.push_back((int)pts.size());
        for (auto &sg : r.hseg) { hs.push_back(sg.first); hs.push_back(sg.second); }
        h_off.push_back((int)(hs.size() / 2));
        for (auto &sg : r.vseg) { vs.push_back(sg.first); vs.push_back(sg.second); }
        v_off.push_back((int)(vs.size() / 2));
    }
    DevBuf<int> a, b, c, e, f, h, i, map, bat, sta, flags;
    a.upload(pt_off, s); b.upload(pts, s); c.upload(pt_net, s); e.upload(h_off, s); f.upload(hs, s);
    h.upload(v_off, s); i.upload(vs, s);
    map.alloc((size_t)ns.X * ns.Y); bat.alloc(n); sta.alloc(n); flags.alloc(8);
    ColorDev cd;
    cd.n = n; cd.X = ns.X; cd.Y = ns.Y; cd.sparsity = sparsity;
    cd.pt_off = a.p; cd.pts = b.p; cd.pt_net = c.p; cd.h_off = e.p; cd.hseg = f.p; cd.v_off = h.p; cd.vseg = i.p;
    cd.npts = (int)pts.size(); cd.map = map.p; cd.batch = bat.p; cd.status = sta.p; cd.flags = flags.p;
    kt.begin(KC_COLOR);
    int nb = run_coloring(cd, 0, s);
    kt.end(KC_COLOR);
    st.launches += 1;
    if (nb == -2) throw Error(ERR_TIMEOUT, "colouring barrier timed out");
    if (nb < 0) throw Error(ERR_CUDA, std::string("colouring failed: ") + cudaGetErrorString(cudaGetLastError()));
    std::vector<int> bid(n);
    cuda_check(cudaMemcpyAsync(bid.data(), bat.p, n * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    batches.assign(nb, {});
    for (int k = 0; k < n; k++) {
        if (bid[k] < 0 || bid[k] >= nb) throw Error(ERR_STATE, "a net was left without a batch");
        batches[bid[k]].push_back(list[k]);
    }
}

// One rip-up-and-reroute pass (main.cpp:37-68, Lshape_route_detour.hpp:726-1112).
// Returns false when no net overflows.
bool Router::rrr_pass(int iter) {
    const int R = (int)ns.nets.size();
    const int X = ns.X, Y = ns.Y;
    if (R == 0) return false;
    if (d_all_ids.n < (size_t)R) {
        std::vector<int> ids(R);
        std::iota(ids.begin(), ids.end(), 0);
        d_all_ids.upload(ids, s);
    }
    of_sum.alloc(go.g.N);
    d_is_of.alloc(R);
    d_xsum.alloc((size_t)X * Y);
    d_ysum.alloc((size_t)X * Y);
    d_bar.alloc(2);
    d_route_off.upload(route_off, s);
    d_route_cap.upload(route_cap, s);
    cuda_check(cudaEventRecord(ev0, s), "event");
    // overflow marking and congestion view (graph.hpp:588-601, main.cpp:42-45)
    ViaBatchDev all{d_all_ids.p, d_route_off.p, routes.p, R};
    kt.begin(KC_RIPUP);
    launch_mark_overflow(go.g, 0, of_sum.p, all, 10, d_is_of.p, s);
    launch_congestion_view(go.g, d_xsum.p, d_ysum.p, s);
    kt.end(KC_RIPUP);
    st.launches += 5;
    std::vector<uint8_t> is_of(R);
    CongestionView cv;
    cv.X = X; cv.Y = Y;
    cv.xsum.resize((size_t)X * Y);
    cv.ysum.resize((size_t)X * Y);
    cuda_check(cudaMemcpyAsync(is_of.data(), d_is_of.p, R, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(cv.xsum.data(), d_xsum.p, cv.xsum.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(cv.ysum.data(), d_ysum.p, cv.ysum.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    std::vector<int> of_nets;
    for (int i = 0; i < R; i++)
        if (is_of[i]) of_nets.push_back(i);
    st.rerouted = (int)of_nets.size();
    if (verbose) std::fprintf(stderr, "[igr] pass %d: %zu nets to reroute\n", iter, of_nets.size());
    if (of_nets.empty()) return false;
    std::sort(of_nets.begin(), of_nets.end(), [&](int l, int r) { return ns.nets[l].hpwl > ns.nets[r].hpwl; });
    // detour DAGs on host threads (Lshape_route_detour.hpp:702-748)
    const double th0 = now_s();
    dag.resize(R);
    parallel_for((int)of_nets.size(), threads, [&](int b, int e) {
        for (int k = b; k < e; k++) build_dag(ns, ns.nets[of_nets[k]], cv, mode_eff, dag[of_nets[k]]);
    });
    st.dag_host_ms += (now_s() - th0) * 1e3;
    std::vector<std::vector<int>> batches;
    color_nets(of_nets, true, mode_eff >= 1 ? 2 : 15, batches);
    std::reverse(batches.begin(), batches.end());
    // batch-local CSR of all batches, laid end to end
    struct BInfo { int nb, eb, pb, lb, nnb, nets, n, e, slots, depth, max_level; };
    std::vector<BInfo> bi;
    std::vector<int> nodes, par_off, par, cslot, echild, child_off, level_off, level_nodes, net_node_off, net_ids;
    std::vector<int64_t> old_off = route_off;
    for (size_t b = 0; b < batches.size(); b++) {
        BInfo f{};
        f.nb = (int)nodes.size(); f.eb = (int)par.size(); f.pb = (int)par_off.size();
        f.lb = (int)level_off.size(); f.nnb = (int)net_node_off.size(); f.nets = (int)net_ids.size();
        int n = 0, e = 0, sl = 0, depth = 0;
        for (int id : batches[b]) {
            const DagNet &dn = dag[id];
            n += (int)dn.nodes.size();
            for (int dv : dn.depth) depth = std::max(depth, dv + 1);
        }
        std::vector<int> dep(n);
        par_off.push_back(0);
        child_off.push_back(0);
        net_node_off.push_back(0);
        int base = 0;
        for (int id : batches[b]) {
            const DagNet &dn = dag[id];
            const int m = (int)dn.nodes.size();
            for (int v = 0; v < m; v++) {
                nodes.push_back(dn.nodes[v]);
                for (int q = dn.par_sum[v]; q < dn.par_sum[v + 1]; q++) {
                    par.push_back(base + dn.par_nodes[q]);
                    cslot.push_back(dn.child_idx[q]);
                    echild.push_back(base + v);
                    e++;
                }
                par_off.push_back(e);
                sl += dn.child_num[v];
                child_off.push_back(sl);
                dep[base + v] = dn.depth[v];
            }
            base += m;
            net_ids.push_back(id);
            net_node_off.push_back(base);
            // new route record of the net (appended)
            route_cap[id] = 8 * m + 1;
            route_off[id] = route_end;
            route_end += route_cap[id];
        }
        // counting sort of nodes by depth (stable in node order)
        std::vector<int> cnt(depth + 1, 0);
        for (int v = 0; v < n; v++) cnt[dep[v] + 1]++;
        for (int d = 0; d < depth; d++) cnt[d + 1] += cnt[d];
        int ml = 0;
        for (int d = 0; d <= depth; d++) level_off.push_back(cnt[d]);
        for (int d = 0; d < depth; d++) ml = std::max(ml, cnt[d + 1] - cnt[d]);
        std::vector<int> ln(n);
        for (int v = 0; v < n; v++) ln[cnt[dep[v]]++] = v;
        level_nodes.insert(level_nodes.end(), ln.begin(), ln.end());
        if ((int64_t)n * 100 + 99 > 0x7fffffffLL) throw Error(ERR_CAPACITY, "DAG batch too large for 32-bit node ids");
        f.n = n; f.e = e; f.slots = sl; f.depth = depth; f.max_level = ml;
        bi.push_back(f);
    }
    grow_routes(route_end);
    DevBuf<int> d_nodes, d_paroff, d_par, d_cslot, d_echild, d_childoff, d_leveloff, d_levelnodes, d_nno, d_ids;
    DevBuf<int64_t> d_old_off;
    d_nodes.upload(nodes, s); d_paroff.upload(par_off, s); d_par.upload(par, s); d_cslot.upload(cslot, s);
    d_echild.upload(echild, s); d_childoff.upload(child_off, s); d_leveloff.upload(level_off, s);
    d_levelnodes.upload(level_nodes, s); d_nno.upload(net_node_off, s); d_ids.upload(net_ids, s);
    d_old_off.upload(old_off, s);
    d_route_off.upload(route_off, s);
    d_route_cap.upload(route_cap, s);
    int mn = 1, me = 1, ms = 1;
    for (auto &f : bi) { mn = std::max(mn, f.n); me = std::max(me, f.e); ms = std::max(ms, f.slots); }
    DevBuf<double> costs, cedges;
    DevBuf<unsigned long long> best, packed;
    DevBuf<int> bchange, lout, stage, stage_cnt;
    costs.alloc((size_t)mn * 10); cedges.alloc((size_t)me * 81);
    best.alloc((size_t)ms * 10); packed.alloc((size_t)ms * 10);
    bchange.alloc((size_t)me * 81); lout.alloc(mn); stage.alloc((size_t)mn * 8); stage_cnt.alloc(mn);
    for (size_t b = 0; b < bi.size(); b++) {
        const BInfo &f = bi[b];
        const int nnet = (int)batches[b].size();
        ViaBatchDev old{d_ids.p + f.nets, d_old_off.p, routes.p, nnet};
        const int s1 = ++global_stamp;
        kt.begin(KC_RIPUP);
        launch_wire_ripup(go.g, old, s1, -1, s);
        launch_via_commit(go.g, old, s1, -1, s);
        kt.end(KC_RIPUP);
        const int s2 = ++global_stamp;
        kt.begin(KC_COST);
        launch_cost_refresh(go.g, true, s);
        kt.end(KC_COST);
        DagBatchDev db;
        db.n_nodes = f.n; db.n_edges = f.e; db.n_slots = f.slots; db.depth = f.depth; db.n_nets = nnet;
        db.max_level = f.max_level;
        db.nodes = d_nodes.p + f.nb; db.par_off = d_paroff.p + f.pb; db.par = d_par.p + f.eb;
        db.child_slot = d_cslot.p + f.eb; db.edge_child = d_echild.p + f.eb; db.child_off = d_childoff.p + f.pb;
        db.level_off = d_leveloff.p + f.lb; db.level_nodes = d_levelnodes.p + f.nb;
        db.h_level_off = level_off.data() + f.lb;
        db.net_node_off = d_nno.p + f.nnb; db.net_ids = d_ids.p + f.nets;
        db.costs = costs.p; db.best_path = best.p; db.packed = packed.p; db.cost_edges = cedges.p;
        db.best_change = bchange.p; db.layer_out = lout.p; db.stage = stage.p; db.stage_cnt = stage_cnt.p;
        db.route_off = d_route_off.p; db.route_cap = d_route_cap.p; db.routes = routes.p;
        kt.begin(KC_DAG);
        int nl = launch_dag_route(go.g, db, s2, d_bar.p, cooperative, s);
        if (nl < 0) {
            cudaGetLastError();
            cooperative = false;
            nl = launch_dag_route(go.g, db, s2, d_bar.p, false, s);
        }
        kt.end(KC_DAG);
        kt.begin(KC_WIRE_COMMIT);
        launch_wire_commit(go.g, s2, true, s);
        kt.end(KC_WIRE_COMMIT);
        ViaBatchDev nw{d_ids.p + f.nets, d_route_off.p, routes.p, nnet};
        kt.begin(KC_VIA_COMMIT);
        launch_via_commit(go.g, nw, s2, 1, s);
        kt.end(KC_VIA_COMMIT);
        st.launches += 5 + nl;
    }
    cuda_check(cudaEventRecord(ev1, s), "event");
    cuda_check(cudaGetLastError(), "reroute launch");
    cuda_check(cudaEventSynchronize(ev1), "reroute");
    float ms_ = 0;
    cudaEventElapsedTime(&ms_, ev0, ev1);
    st.rrr_ms += ms_;
    if (int e = go.check_error(s)) throw Error(e, "device error in rip-up and reroute");
    return true;
}

void Router::compute_score() {
    unsigned long long h[4] = {0, 0, 0, 0};
    double of = 0;
    launch_overflow_cost(go.g, go.score.p, s);
    cuda_check(cudaMemcpyAsync(h, go.stats.p, sizeof h, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(&of, go.score.p, sizeof of, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "sync");
    int64_t pin_vias = 0;
    for (size_t i = 0; i < d.sel.size(); i++) pin_vias += d.sel[i] < d.X * d.Y;
    cost_cells = h[2];
    score_wl = (double)(int64_t)h[0] * d.unit_wire;
    score_via = (double)((int64_t)h[1] + pin_vias) * d.unit_via;
    score_of = of;
}

void Router::write(const char *out) {
    RouteSource rs;
    rs.routes_of = [&](int net) -> const int * { return h_routes.empty() ? nullptr : route_of(net); };
    write_guides(d, ns, rs, out, threads);
}

}  // namespace igr
