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
// separated by grid barriers, so the batches depend only on the input.  The
// whole colouring is one persistent cooperative kernel: no host round trip per
// round.  The grid barrier gives up after two seconds and reports
// ERR_TIMEOUT instead of waiting forever.
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
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*(volatile int *)err) s_ok = 0;
    }
    __syncthreads();
    return s_ok != 0;
}

__global__ void coloring_kernel(ColorDev c, Bar bar, int *err, int max_batches) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const int XY = c.X * c.Y, X = c.X, Y = c.Y;
    volatile int *flags = c.flags;  // [0] commit in batch, [1] commit in round, [2] batches
    for (int cur = 0; cur < max_batches; cur++) {
        for (int i = tid; i < XY; i += nth) c.map[i] = -1;
        for (int i = tid; i < c.n; i += nth) c.status[i] = 0;
        if (tid == 0) flags[0] = 0;
        if (!grid_barrier(bar, err)) return;
        for (int round = 0; round < 30; round++) {
            if (tid == 0) flags[1] = 0;
            // claim
            for (int k = tid; k < c.n; k += nth) {
                if (c.status[k] == 2 || c.batch[k] != -1) continue;
                c.status[k] = 1;
                const int sh = c.perm ? c.perm[k] : k;
                for (int i = c.pt_off[sh]; i < c.pt_off[sh + 1]; i++) {
                    const int p = c.pts[i], x = p / Y, y = p % Y;
                    const int dx[4] = {0, 0, -1, 1}, dy[4] = {0, -1, 0, 0};
                    for (int j = 0; j < 4; j++) {
                        const int nx = x + dx[j], ny = y + dy[j];
                        if (nx >= 0 && nx < X && ny >= 0 && ny < Y) atomicMax(&c.map[nx * Y + ny], k);
                    }
                }
                for (int i = c.h_off[sh]; i < c.h_off[sh + 1]; i++) {
                    const int s = c.hseg[2 * i], e = c.hseg[2 * i + 1];
                    const int y = s % Y;
                    for (int x = s / Y; x <= e / Y; x += c.sparsity) atomicMax(&c.map[x * Y + y], k);
                }
                for (int i = c.v_off[sh]; i < c.v_off[sh + 1]; i++) {
                    const int s = c.vseg[2 * i], e = c.vseg[2 * i + 1];
                    const int x = s / Y;
                    for (int y = s % Y; y <= e % Y; y += c.sparsity) atomicMax(&c.map[x * Y + y], k);
                }
            }
            if (!grid_barrier(bar, err)) return;
            // commit: owns every point
            for (int k = tid; k < c.n; k += nth) {
                if (c.status[k] == 2 || c.batch[k] != -1) continue;
                bool ok = true;
                const int sh = c.perm ? c.perm[k] : k;
                for (int i = c.pt_off[sh]; i < c.pt_off[sh + 1] && ok; i++) ok = c.map[c.pts[i]] == k;
                if (ok) {
                    c.batch[k] = cur;
                    flags[0] = 1;
                    flags[1] = 1;
                }
            }
            if (!grid_barrier(bar, err)) return;
            if (!flags[1]) break;
            // block nets whose points belong to a member of this batch
            for (int i = tid; i < c.npts; i += nth) {
                const int k = c.rank ? c.rank[c.pt_net[i]] : c.pt_net[i];
                if (k < 0) continue;  // shape not in this colouring
                if (c.status[k] != 1 || c.batch[k] != -1) continue;
                const int pre = c.map[c.pts[i]];
                if (pre != -1 && c.batch[pre] != -1 && c.status[k] != 2) c.status[k] = 2;
            }
            if (!grid_barrier(bar, err)) return;
            // release the cells of blocked nets
            for (int i = tid; i < XY; i += nth) {
                const int k = c.map[i];
                if (k >= 0 && c.status[k] == 2) c.map[i] = -1;
            }
            if (!grid_barrier(bar, err)) return;
        }
        if (!flags[0]) {
            if (tid == 0) flags[2] = cur;
            return;
        }
        if (!grid_barrier(bar, err)) return;
    }
    if (tid == 0) flags[2] = max_batches;
}

}  // namespace

int run_coloring(ColorDev &c, int max_batch, cudaStream_t s) {
    (void)max_batch;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coloring_kernel, threads, 0);
    int blocks = sms * (per < 4 ? per : 4);
    if (blocks < 1) blocks = 1;
    // barrier words and error word live after the four flags
    Bar bar{reinterpret_cast<unsigned *>(c.flags + 4), reinterpret_cast<unsigned *>(c.flags + 5)};
    int *err = c.flags + 6;
    cudaMemsetAsync(c.flags, 0, 8 * sizeof(int), s);
    cudaMemsetAsync(c.batch, 0xff, sizeof(int) * (size_t)c.n, s);
    int max_batches = c.n + 1;
    void *args[] = {&c, &bar, &err, &max_batches};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)coloring_kernel, dim3(blocks), dim3(threads), args, 0, s);
    if (e != cudaSuccess) return -1;
    int h[8];
    if (cudaMemcpyAsync(h, c.flags, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (h[6] != 0) return -2;
    return h[2];
}

}  // namespace igr
