// Host side of the device DAG builder: work-area size classes, the size and
// write passes, and the layout of the per-DAG arrays.
#include <algorithm>

#include "router.hpp"

namespace igr {

namespace {

// Work-area slices per size class and the most builders a class runs;
// most DAGs fit the first class (nets of up to 12 pins give trees of at most
// 22 nodes), the few larger ones the second, whose builders keep their work
// area in shared memory, one per SM; the third is for split nets whose trees
// kept growing.
struct DagClass {
    DagCaps caps;
    int threads;
    bool solo;  // one builder per block
};
const DagClass kClasses[] = {
    {{32, 256, 256, 256, 512, 1024}, 148 * 512, false},
    {{128, 1024, 1024, 1536, 3072, 6144}, 148, true},
    {{2048, 16384, 16384, 16384, 32768, 65536}, 512, true},
};
constexpr int kNumClasses = 3;

int round_threads(int n, int cap) {
    const int t = std::min(cap, std::max(n, 1));
    return (t + 127) / 128 * 128;
}

void run_class(DeviceDags &d, DagBuildArgs a, int cls, const std::vector<int> &members, cudaStream_t s) {
    const DagClass &c = kClasses[cls];
    const int n = (int)members.size();
    if (n == 0) return;
    const long long per = dag_work_ints(c.caps);
    const bool in_smem = c.solo && per * 4 <= dag_solo_smem_limit();
    const int threads = c.solo ? std::min(n, c.threads) : round_threads(n, c.threads);
    a.caps = c.caps;
    if (in_smem) {
        a.work = nullptr;
    } else {
        d.work.alloc((size_t)threads * (size_t)per);
        a.work = d.work.p;
    }
    a.n_list = n;
    bool identity = true;  // 0 .. n-1 in order
    for (int i = 0; i < n && identity; i++) identity = members[i] == i;
    if (identity) {
        a.list = nullptr;
    } else {
        d.list.upload(members, s);
        a.list = d.list.p;
    }
    if (c.solo)
        launch_dag_build_solo(a, threads, s);
    else
        launch_dag_build(a, threads, s);
    cuda_check(cudaGetLastError(), "DAG build launch");
}

// grows a pool to `count` entries, keeping its first `keep`
void grow_keep(DevBuf<int> &b, size_t count, size_t keep, cudaStream_t s) {
    if (count <= b.n && b.p) return;
    int *np = static_cast<int *>(dev_alloc(count * sizeof(int)));
    if (keep && b.p) cuda_check(cudaMemcpyAsync(np, b.p, keep * sizeof(int), cudaMemcpyDeviceToDevice, s), "D2D");
    b.release();  // synchronises the device first
    b.p = np;
    b.n = count;
}

}  // namespace

void DeviceDags::build(DagBuildArgs a, cudaStream_t s, const std::vector<int> *order_key) {
    const int n = a.n_list;
    hs.assign((size_t)n * kDagSizeFields, 0);
    tier.assign(n, 0);
    if (n == 0) return;
    sizes.alloc((size_t)n * kDagSizeFields);
    node_at.alloc(n); edge_at.alloc(n); point_at.alloc(n);
    used.alloc(3);
    cuda_check(cudaMemsetAsync(used.p, 0, 3 * sizeof(unsigned long long), s), "memset");
    // pools sized from the last build's entries per DAG, with a margin
    auto want = [&](double per) { return (size_t)(per * 1.25 * n) + 4096; };
    const size_t cn = want(per_node), ce = want(per_edge), cp = want(per_point);
    grow_keep(nodes, cn, 0, s); grow_keep(par_num, cn, 0, s); grow_keep(child_num, cn, 0, s);
    grow_keep(depth, cn, 0, s); grow_keep(par, ce, 0, s); grow_keep(child_idx, ce, 0, s); grow_keep(points, cp, 0, s);
    a.sizes = sizes.p;
    a.node_at = node_at.p; a.edge_at = edge_at.p; a.point_at = point_at.p;
    a.used = used.p;
    auto set_pools = [&]() {
        a.cap_nodes = (long long)nodes.n; a.cap_edges = (long long)par.n; a.cap_points = (long long)points.n;
        a.out_nodes = nodes.p; a.out_par_num = par_num.p; a.out_child_num = child_num.p; a.out_depth = depth.p;
        a.out_par = par.p; a.out_child_idx = child_idx.p; a.out_points = points.p;
    };
    set_pools();
    std::vector<int> members(n), next;  // DAGs to build in this class; for the next class
    for (int k = 0; k < n; k++) members[k] = k;
    // builders of nets alike in size side by side: a warp's 32 builders then
    // walk loops of similar lengths and diverge less (c2: 21/18/18 -> 18/13/13
    // ms per pass); each DAG is built alone, so the DAGs do not change
    if (order_key)
        std::stable_sort(members.begin(), members.end(),
                         [&](int l, int r) { return (*order_key)[l] > (*order_key)[r]; });
    int cls = 0, regrow = 0;
    while (true) {
        run_class(*this, a, cls, members, s);
        unsigned long long u[3];
        cuda_check(cudaMemcpyAsync(hs.data(), sizes.p, hs.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(u, used.p, sizeof u, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "DAG build");
        std::vector<int> full;
        for (int k : members) {
            const int status = sz(k, 6);
            if (status == 2) throw Error(ERR_STATE, "malformed tree or detour DAG");
            if (status == 1) next.push_back(k);
            if (status == 3) full.push_back(k);
            tier[k] = cls;
        }
        if (!full.empty()) {  // grow the pools past what was asked for and build those DAGs again
            if (++regrow > 8) throw Error(ERR_CAPACITY, "detour DAG pools keep overflowing");
            const double f = 2.0 * (double)full.size() + 4096;
            grow_keep(nodes, (size_t)(u[0] + f * per_node), nodes.n, s);
            grow_keep(par_num, nodes.n, par_num.n, s);
            grow_keep(child_num, nodes.n, child_num.n, s);
            grow_keep(depth, nodes.n, depth.n, s);
            grow_keep(par, (size_t)(u[1] + f * per_edge), par.n, s);
            grow_keep(child_idx, par.n, child_idx.n, s);
            grow_keep(points, (size_t)(u[2] + f * per_point), points.n, s);
            set_pools();
            members.swap(full);
            continue;  // same class
        }
        if (next.empty()) break;
        if (++cls >= kNumClasses) throw Error(ERR_CAPACITY, "a detour DAG outgrows the largest work area");
        std::sort(next.begin(), next.end());
        members.swap(next);
        next.clear();
    }
    for (int k = 0; k < n; k++)
        if (sz(k, 6) != 0) throw Error(ERR_STATE, "a detour DAG was left unbuilt");
    double tn = 0, te = 0, tp = 0;
    for (int k = 0; k < n; k++) { tn += sz(k, 0); te += sz(k, 1); tp += sz(k, 2); }
    per_node = std::max(8.0, tn / n);
    per_edge = std::max(8.0, te / n);
    per_point = std::max(8.0, tp / n);
}

}  // namespace igr
