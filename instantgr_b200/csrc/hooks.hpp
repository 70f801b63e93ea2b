// Test hooks: process-wide settings through which tests reach paths that the
// default sizes do not, and make bounded device waits run out without a fault.
// The defaults are normal operation; igr_test_hook (C ABI) changes them.
#pragma once
#include <atomic>

namespace igr {

struct TestHooks {
    std::atomic<long long> wait_ns{2000000000LL};  // limit of grid-barrier and mbarrier waits
    std::atomic<int> barrier_phantom{0};  // arrivals the colouring's grid barriers wait for and never get
    std::atomic<int> mbar_probe{0};       // seed GEMM: first waits on an mbarrier that nothing arrives on
    std::atomic<int> color_keep_map{1};   // igr_color_batches: keep the round-0 map (1) or re-claim (0)
    std::atomic<int> dag_split_nets{4096};  // DAG DP: batches of this many nets or more run split by DAG size
    std::atomic<int> color_keep_min_nets{2000000};  // router: colourings of this many nets or more keep the map
    std::atomic<int> shape_dedupe{1};  // router: each shape's conflict points and claims kept once
    std::atomic<int> dag_stage_nodes{1024};  // DAG DP: nets of at most this many nodes staged in shared memory
    void reset() {
        wait_ns = 2000000000LL;
        barrier_phantom = 0;
        mbar_probe = 0;
        color_keep_map = 1;
        dag_split_nets = 4096;
        color_keep_min_nets = 2000000;
        shape_dedupe = 1;
        dag_stage_nodes = 1024;
    }
};
TestHooks &test_hooks();

}  // namespace igr
