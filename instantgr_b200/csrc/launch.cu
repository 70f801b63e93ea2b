// Per-device launch set-up of kernels (see kernel_setup in device.hpp) and
// the process's test hooks (hooks.hpp).
#include "device.hpp"
#include "hooks.hpp"
#include "router.hpp"

#include <map>
#include <mutex>
#include <string>
#include <tuple>

namespace igr {

TestHooks &test_hooks() {
    static TestHooks h;
    return h;
}

KernelShape kernel_setup(const void *kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, size_t>, KernelShape> shapes;
    static std::map<std::pair<const void *, int>, size_t> smem_limit;  // attribute set per (kernel, device)
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(kernel, dev, smem);
    auto it = shapes.find(key);
    if (it != shapes.end()) return it->second;
    size_t &lim = smem_limit[std::make_pair(kernel, dev)];
    if (smem > lim) {
        cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                   "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
        lim = smem;
    }
    KernelShape k;
    cuda_check(cudaDeviceGetAttribute(&k.sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k.blocks_per_sm, kernel, threads, smem), "occupancy");
    if (k.blocks_per_sm < 1) k.blocks_per_sm = 1;
    shapes[key] = k;
    return k;
}

}  // namespace igr
