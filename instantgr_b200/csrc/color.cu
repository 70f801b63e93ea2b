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

constexpr int kG = 8;                 // lanes per net
constexpr int kNetsPerWarp = 32 / kG;
constexpr unsigned kGroupMask = (1u << kG) - 1;

// flags (ints): [0..1] commit seen in a round (by round parity), [2] batches,
// [4..5] barrier, [6] error, [8] rounds run, [9] lost count, [10] next
// candidate count, [11..12] nets left after a batch (by batch parity)
enum : int { F_ROUND = 0, F_NB = 2, F_ERR = 6, F_ROUNDS = 8, F_LOST = 9, F_CAND = 10, F_LEFT = 11 };

// Appends `k` of every group leader with `want` set to list[*count++]; called
// by all 32 lanes of the warp with the same control flow.
__device__ __forceinline__ void warp_append(int *list, int *count, bool want, int k, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (want) list[base + __popc(m & ((1u << lane) - 1))] = k;
}

// Per batch: candidates claim (atomicMax of their rank on their claim cells),
// candidates owning all their points join, the others are blocked when a
// member owns one of their points (and release their cells at once; a blocked
// net's cells are no member's points, so the release cannot change another
// net's check), else they stay candidates.  Three grid barriers per round.
// The lists are unordered: every phase is order-independent.
__global__ void __launch_bounds__(1024, 1) coloring_kernel(ColorDev c, Bar bar, int *err, int max_batches) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, grp = lane / kG, gl = lane % kG;
    const int gw = tid >> 5, nw = nth >> 5;
    const int XY = c.X * c.Y;
    int *flags = c.flags;
    volatile int *vflags = c.flags;
    int *act = c.active, *act2 = c.active2;
    for (int i = tid; i < c.n; i += nth) act[i] = i;
    for (int i = tid; i < XY; i += nth) c.map[i] = -1;
    if (!grid_barrier(bar, err)) return;
    int na = c.n;
    for (int cur = 0; cur < max_batches; cur++) {
        const int *cand = act;  // round 0: every net without a batch
        int nc = na;
        for (int round = 0; round < 30; round++) {
            // claim
            if (tid == 0) {
                flags[F_ROUNDS]++;
                flags[F_LOST] = 0;
                flags[F_ROUND + ((round + 1) & 1)] = 0;
            }
            for (int base = gw * kNetsPerWarp; base < nc; base += nw * kNetsPerWarp) {
                const int idx = base + grp;
                if (idx >= nc) continue;
                const int k = cand[idx];
                const int sh = c.perm ? c.perm[k] : k;
                const int e = c.claim_off[sh + 1];
                for (int i = c.claim_off[sh] + gl; i < e; i += kG) atomicMax(&c.map[c.claim[i]], k);
            }
            if (!grid_barrier(bar, err)) return;
            // commit: members own every point; the others go to the lost list
            if (tid == 0) {
                flags[F_CAND] = 0;
                if (round == 0) flags[F_LEFT + ((cur + 1) & 1)] = 0;
            }
            for (int base = gw * kNetsPerWarp; base < nc; base += nw * kNetsPerWarp) {
                const int idx = base + grp;
                const bool valid = idx < nc;
                const int k = valid ? cand[idx] : -1;
                bool ok = true;
                if (valid) {
                    const int sh = c.perm ? c.perm[k] : k;
                    const int e = c.pt_off[sh + 1];
                    for (int i = c.pt_off[sh] + gl; i < e; i += kG) ok &= c.map[c.pts[i]] == k;
                }
                const unsigned bad = (__ballot_sync(0xffffffffu, !ok) >> (grp * kG)) & kGroupMask;
                if (valid && bad == 0 && gl == 0) {
                    c.batch[k] = cur;
                    flags[F_ROUND + (round & 1)] = 1;
                }
                warp_append(c.lost, flags + F_LOST, valid && bad != 0 && gl == 0, k, lane);
            }
            if (!grid_barrier(bar, err)) return;
            if (!vflags[F_ROUND + (round & 1)]) break;
            // block (and release) or stay a candidate
            const int nl = vflags[F_LOST];
            for (int base = gw * kNetsPerWarp; base < nl; base += nw * kNetsPerWarp) {
                const int idx = base + grp;
                const bool valid = idx < nl;
                const int k = valid ? c.lost[idx] : -1;
                const int sh = valid ? (c.perm ? c.perm[k] : k) : 0;
                bool hit = false;
                if (valid) {
                    const int e = c.pt_off[sh + 1];
                    for (int i = c.pt_off[sh] + gl; i < e; i += kG) {
                        const int pre = c.map[c.pts[i]];
                        hit |= (pre != -1 && c.batch[pre] != -1);
                    }
                }
                const bool blocked = ((__ballot_sync(0xffffffffu, hit) >> (grp * kG)) & kGroupMask) != 0;
                if (valid && blocked) {
                    const int e = c.claim_off[sh + 1];
                    for (int i = c.claim_off[sh] + gl; i < e; i += kG)
                        if (c.map[c.claim[i]] == k) c.map[c.claim[i]] = -1;
                }
                warp_append(c.cand, flags + F_CAND, valid && !blocked && gl == 0, k, lane);
            }
            if (!grid_barrier(bar, err)) return;
            cand = c.cand;
            nc = vflags[F_CAND];
            if (nc == 0) break;
        }
        // nets still without a batch stay active; the map is cleared for the next batch
        for (int i = tid; i < XY; i += nth) c.map[i] = -1;
        if (tid == 0) flags[F_ROUND] = flags[F_ROUND + 1] = 0;
        for (int base = gw * 32; base < na; base += nw * 32) {
            const int i = base + lane;
            const int k = i < na ? act[i] : -1;
            warp_append(act2, flags + F_LEFT + (cur & 1), k >= 0 && c.batch[k] == -1, k, lane);
        }
        if (!grid_barrier(bar, err)) return;
        na = vflags[F_LEFT + (cur & 1)];
        int *t = act; act = act2; act2 = t;
        if (na == 0) {
            if (tid == 0) flags[F_NB] = cur + 1;
            return;
        }
    }
    if (tid == 0) flags[F_NB] = max_batches;
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
    const int threads = 1024;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coloring_kernel, threads, 0);
    int blocks = sms * (per < 1 ? per : 1);
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
