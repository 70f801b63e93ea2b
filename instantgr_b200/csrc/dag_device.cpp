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
    if (members.back() == n - 1) {  // ascending and complete: 0 .. n-1
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

}  // namespace

void DeviceDags::measure(DagBuildArgs a, cudaStream_t s) {
    const int n = a.n_list;
    hs.assign((size_t)n * kDagSizeFields, 0);
    tier.assign(n, 0);
    if (n == 0) return;
    sizes.alloc((size_t)n * kDagSizeFields);
    a.sizes = sizes.p;
    a.out_nodes = nullptr;
    std::vector<int> members(n);
    for (int k = 0; k < n; k++) members[k] = k;
    for (int cls = 0; cls < kNumClasses && !members.empty(); cls++) {
        run_class(*this, a, cls, members, s);
        cuda_check(cudaMemcpyAsync(hs.data(), sizes.p, hs.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "DAG sizes");
        std::vector<int> again;
        for (int k : members) {
            const int status = sz(k, 6);
            if (status == 2) throw Error(ERR_STATE, "malformed tree or detour DAG");
            if (status == 1) again.push_back(k);
            tier[k] = cls;
        }
        members.swap(again);
    }
    if (!members.empty()) throw Error(ERR_CAPACITY, "a detour DAG outgrows the largest work area");
}

void DeviceDags::write(DagBuildArgs a, const std::vector<int> &kept, cudaStream_t s) {
    const int n = (int)kept.size();
    h_node_at.assign((size_t)n + 1, 0);
    h_edge_at.assign((size_t)n + 1, 0);
    h_point_at.assign((size_t)n + 1, 0);
    for (int i = 0; i < n; i++) {
        const int k = kept[i];
        h_node_at[i + 1] = h_node_at[i] + sz(k, 0);
        h_edge_at[i + 1] = h_edge_at[i] + sz(k, 1);
        h_point_at[i + 1] = h_point_at[i] + sz(k, 2);
    }
    if (n == 0) return;
    node_at.upload(h_node_at, s);
    edge_at.upload(h_edge_at, s);
    point_at.upload(h_point_at, s);
    const size_t nn = (size_t)std::max<long long>(1, h_node_at[n]), ne = (size_t)std::max<long long>(1, h_edge_at[n]),
                 np = (size_t)std::max<long long>(1, h_point_at[n]);
    nodes.alloc(nn); par_num.alloc(nn); child_num.alloc(nn); depth.alloc(nn);
    par.alloc(ne); child_idx.alloc(ne); points.alloc(np);
    err.alloc(1);
    cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    a.sizes = nullptr;
    a.node_at = node_at.p; a.edge_at = edge_at.p; a.point_at = point_at.p;
    a.out_nodes = nodes.p; a.out_par_num = par_num.p; a.out_child_num = child_num.p; a.out_depth = depth.p;
    a.out_par = par.p; a.out_child_idx = child_idx.p; a.out_points = points.p;
    a.err = err.p;
    a.n_list = n;
    for (int cls = 0; cls < kNumClasses; cls++) {
        std::vector<int> members;
        for (int i = 0; i < n; i++)
            if (tier[kept[i]] == cls) members.push_back(i);
        run_class(*this, a, cls, members, s);
    }
    int h_err = 0;
    cuda_check(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "DAG write");
    if (h_err) throw Error(ERR_STATE, "a detour DAG changed between the size and write passes");
}

}  // namespace igr
