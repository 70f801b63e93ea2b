// Batch colouring: greedy independent sets of spatially disjoint nets.
//
// Semantics of generate_batches_rsmt_gpu (src/database_cuda.hpp:288-434,
// :437-631): nets are ranked by their position in the colouring order (higher
// rank wins a cell by atomicMax); in every round each unassigned, unblocked
// net claims the 4-neighbourhood of its conflict points and every
// `sparsity`-th cell of its tree segments; a net joins the batch when it still
// owns all of its points; nets whose points are owned by a net that joined are
// blocked for this batch and release their cells.  At most 30 rounds per
// batch; a batch with no new member ends the colouring.
//
// The reference is nondeterministic (a claiming thread re-reads the cell right
// after its atomicMax while others are still writing, and returns early).
// Here claiming, committing, blocking and releasing are separate phases
// separated by grid barriers, so the batches depend only on the input.
//
// Work layout: the cells a net claims are precomputed once (claim lists, CSR
// per shape), one warp handles one net with its lanes over the net's claims
// or points, and only nets still without a batch are visited: the list of
// active nets is compacted after every batch.  The whole colouring is one
// persistent cooperative kernel; the grid barrier gives up after two seconds
// and reports ERR_TIMEOUT instead of waiting forever.
#include "kcommon.cuh"

namespace igr {

namespace {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct Bar {
    unsigned *count;
    unsigned *gen;
};

// returns false when the barrier timed out or another block reported an error
__device__ bool grid_barrier(Bar b, int *err) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        s_ok = 1;
        volatile unsigned *vgen = b.gen;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(b.count, 1u);
        if (arrived == gridDim.x - 1) {
            *b.count = 0;
            __threadfence();
            atomicAdd(b.gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*vgen == g) {
                if (*(volatile int *)err) { s_ok = 0; break; }
                if (global_ns() - t0 > 2000000000ull) { set_error(err, ERR_TIMEOUT); s_ok = 0; break; }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*(volatile int *)err) s_ok = 0;
    }
    __syncthreads();
    return s_ok != 0;
}

// flags: [0] commit in batch, [1] commit in round, [2] batches, [3] active count,
//        [4..5] barrier, [6] error, [7] next active count
__global__ void coloring_kernel(ColorDev c, Bar bar, int *err, int max_batches) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int gw = tid >> 5, nw = nth >> 5;
    const int XY = c.X * c.Y;
    volatile int *flags = c.flags;
    int *act = c.active, *act2 = c.active2;
    for (int i = tid; i < c.n; i += nth) act[i] = i;
    if (tid == 0) flags[3] = c.n;
    if (!grid_barrier(bar, err)) return;
    for (int cur = 0; cur < max_batches; cur++) {
        const int na = flags[3];
        for (int i = tid; i < XY; i += nth) c.map[i] = -1;
        for (int i = tid; i < na; i += nth) c.status[act[i]] = 0;
        if (tid == 0) { flags[0] = 0; flags[7] = 0; }
        if (!grid_barrier(bar, err)) return;
        for (int round = 0; round < 30; round++) {
            if (tid == 0) { flags[1] = 0; flags[8]++; }
            // claim
            for (int w = gw; w < na; w += nw) {
                const int k = act[w];
                if (c.status[k] == 2 || c.batch[k] != -1) continue;  // blocked, or already a member
                if (lane == 0) c.status[k] = 1;
                const int sh = c.perm ? c.perm[k] : k;
                for (int i = c.claim_off[sh] + lane; i < c.claim_off[sh + 1]; i += 32) atomicMax(&c.map[c.claim[i]], k);
            }
            if (!grid_barrier(bar, err)) return;
            // commit: owns every point
            for (int w = gw; w < na; w += nw) {
                const int k = act[w];
                if (c.status[k] != 1 || c.batch[k] != -1) continue;
                const int sh = c.perm ? c.perm[k] : k;
                bool ok = true;
                for (int i = c.pt_off[sh] + lane; i < c.pt_off[sh + 1]; i += 32) ok &= c.map[c.pts[i]] == k;
                ok = __all_sync(0xffffffffu, ok);
                if (ok && lane == 0) {
                    c.batch[k] = cur;
                    flags[0] = 1;
                    flags[1] = 1;
                }
            }
            if (!grid_barrier(bar, err)) return;
            if (!flags[1]) break;
            // block candidates whose points belong to a member of this batch
            for (int w = gw; w < na; w += nw) {
                const int k = act[w];
                if (c.status[k] != 1 || c.batch[k] != -1) continue;
                const int sh = c.perm ? c.perm[k] : k;
                bool hit = false;
                for (int i = c.pt_off[sh] + lane; i < c.pt_off[sh + 1]; i += 32) {
                    const int pre = c.map[c.pts[i]];
                    hit |= (pre != -1 && c.batch[pre] != -1);
                }
                hit = __any_sync(0xffffffffu, hit);
                if (hit && lane == 0) c.status[k] = 2;
            }
            if (!grid_barrier(bar, err)) return;
            // blocked nets release the cells they own
            for (int w = gw; w < na; w += nw) {
                const int k = act[w];
                if (c.status[k] != 2) continue;
                const int sh = c.perm ? c.perm[k] : k;
                for (int i = c.claim_off[sh] + lane; i < c.claim_off[sh + 1]; i += 32)
                    if (c.map[c.claim[i]] == k) c.map[c.claim[i]] = -1;
            }
            if (!grid_barrier(bar, err)) return;
        }
        if (!flags[0]) {
            if (tid == 0) flags[2] = cur;
            return;
        }
        // nets still without a batch stay active (their order in the list does not matter)
        for (int i = tid; i < na; i += nth) {
            const int k = act[i];
            if (c.batch[k] == -1) act2[atomicAdd((int *)&flags[7], 1)] = k;
        }
        if (!grid_barrier(bar, err)) return;
        if (tid == 0) flags[3] = flags[7];
        int *t = act; act = act2; act2 = t;
        if (!grid_barrier(bar, err)) return;
        if (flags[3] == 0) {
            if (tid == 0) flags[2] = cur + 1;
            return;
        }
    }
    if (tid == 0) flags[2] = max_batches;
}

}  // namespace

void build_claims(int nshapes, const int *pt_off, const int *pts, const int *h_off, const int *hseg,
                  const int *v_off, const int *vseg, int X, int Y, int sparsity, std::vector<int> &off,
                  std::vector<int> &cells, int /*threads*/) {
    static const int dx[4] = {0, 0, -1, 1}, dy[4] = {0, -1, 0, 0};
    off.assign(nshapes + 1, 0);
    cells.clear();
    for (int k = 0; k < nshapes; k++) {
        for (int i = pt_off[k]; i < pt_off[k + 1]; i++) {
            const int x = pts[i] / Y, y = pts[i] % Y;
            for (int j = 0; j < 4; j++) {
                const int nx = x + dx[j], ny = y + dy[j];
                if (nx >= 0 && nx < X && ny >= 0 && ny < Y) cells.push_back(nx * Y + ny);
            }
        }
        for (int i = h_off[k]; i < h_off[k + 1]; i++) {
            const int s = hseg[2 * i], e = hseg[2 * i + 1], y = s % Y;
            for (int x = s / Y; x <= e / Y; x += sparsity) cells.push_back(x * Y + y);
        }
        for (int i = v_off[k]; i < v_off[k + 1]; i++) {
            const int s = vseg[2 * i], e = vseg[2 * i + 1], x = s / Y;
            for (int y = s % Y; y <= e % Y; y += sparsity) cells.push_back(x * Y + y);
        }
        off[k + 1] = (int)cells.size();
    }
}

int run_coloring(ColorDev &c, int max_batch, cudaStream_t s) {
    (void)max_batch;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 512;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coloring_kernel, threads, 0);
    int blocks = sms * (per < 2 ? per : 2);
    if (blocks < 1) blocks = 1;
    Bar bar{reinterpret_cast<unsigned *>(c.flags + 4), reinterpret_cast<unsigned *>(c.flags + 5)};
    int *err = c.flags + 6;
    cudaMemsetAsync(c.flags, 0, 16 * sizeof(int), s);
    cudaMemsetAsync(c.batch, 0xff, sizeof(int) * (size_t)c.n, s);
    int max_batches = c.n + 1;
    void *args[] = {&c, &bar, &err, &max_batches};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)coloring_kernel, dim3(blocks), dim3(threads), args, 0, s);
    if (e != cudaSuccess) return -1;
    int h[16];
    if (cudaMemcpyAsync(h, c.flags, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (h[6] != 0) return -2;
    c.rounds = h[8];
    return h[2];
}

}  // namespace igr
