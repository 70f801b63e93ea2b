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
// Here claiming, committing and blocking are separate phases separated by
// grid barriers, so the batches depend only on the input.
//
// Work layout: the cells a net claims are precomputed once (claim lists, CSR
// per shape) and gathered per rank into one 16-byte header; a group of 8 lanes
// handles one net.  Each round walks only the nets it concerns: the
// candidates (claim, commit) and the nets that lost a point (block); the lists
// are rebuilt every phase with one global atomic per block (appends are staged
// in shared memory).  The whole colouring is one persistent cooperative
// kernel; the last rounds of a batch, which have few candidates, run in one
// block with block barriers.  Every grid barrier gives up after two seconds
// and reports ERR_TIMEOUT instead of waiting forever.
//
// Optionally (ColorDev::rev set) the round-0 map of every batch is kept up to
// date instead of being cleared and re-claimed by every net without a batch:
// the claimers of each cell are grouped by cell once; after a batch, each cell
// whose round-0 owner joined gets as new owner its highest claimer still
// without a batch (one warp per such cell, assigned claimers dropped from the
// list), which is the max the re-claim would give, since every other cell's
// owner is still without a batch and still the highest of a smaller set.
#include "gridsync.cuh"
#include "hooks.hpp"
#include "host.hpp"

namespace igr {

namespace {

constexpr int kThreads = 1024;
constexpr int kG = 8;                          // lanes per net
constexpr int kGroups = kThreads / kG;         // groups per block
constexpr unsigned kGroupMask = (1u << kG) - 1;
constexpr int kBuf = 4096;                     // staged list entries per block
// rounds with at most this many candidates run in block 0 alone (two nets per
// group and phase at most)
constexpr int kBlockRounds = 2 * kGroups;

// flags (ints): [2] batches, [4] barrier counter, [6] error, [8] rounds run,
// [9] lost count, [10] next candidate count, [11..12] nets left after a batch
// (by batch parity)
enum : int { F_NB = 2, F_BAR = 4, F_ERR = 6, F_ROUNDS = 8, F_LOST = 9, F_CAND = 10, F_LEFT = 11, F_DIRTY = 13 };

// memory operations of this thread, summed into c.ops at the end (roofline
// accounting): claimed cells, points checked for commit, points checked for
// blocking, cells checked for release, list entries scanned
struct Ops {
    unsigned long long claims = 0, points = 0, bpoints = 0, releases = 0, scans = 0;
};

struct Stage {
    int buf[kBuf];
    int n, base;
};

// Stages `k` of every lane with `want` set; called by all 32 lanes of a warp.
__device__ __forceinline__ void stage(Stage &st, bool want, int k, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(&st.n, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (want) st.buf[base + __popc(m & ((1u << lane) - 1))] = k;
}

// Appends the staged entries to list[*count ...]; every thread of the block calls it.
__device__ __forceinline__ void flush(Stage &st, int *list, int *count) {
    __syncthreads();
    const int m = st.n;
    if (threadIdx.x == 0 && m > 0) st.base = atomicAdd(count, m);
    __syncthreads();
    if (m > 0) {
        const int b = st.base;
        for (int i = threadIdx.x; i < m; i += blockDim.x) list[b + i] = st.buf[i];
    }
    if (threadIdx.x == 0) st.n = 0;
    __syncthreads();
}

// exclusive prefix of v over the block's threads (all threads call it); *total
// receives the block's sum
__device__ int block_exclusive(int v, int *total) {
    __shared__ int warp_sum[kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int t = lane < kThreads / 32 ? warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kThreads / 32) warp_sum[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const int before = (wid ? warp_sum[wid - 1] : 0) + x - v;
    *total = warp_sum[kThreads / 32 - 1];
    __syncthreads();
    return before;
}

// map and batch change during the kernel: read them from L2
__device__ __forceinline__ int owner(const ColorDev &c, int cell) { return __ldcg(c.map + cell); }

// Candidates claim their cells, four cells in flight per lane.  Blocks blk,
// blk+nblk, ... of the workers; group j of a block takes list entry j.
__device__ __forceinline__ void claim_phase(const ColorDev &c, const int *list, int n, int blk, int nblk, Ops &ops) {
    const int gl = threadIdx.x % kG;
    for (int idx = blk * kGroups + threadIdx.x / kG; idx < n; idx += nblk * kGroups) {
        const int k = list[idx];
        const int4 h = c.hdr[k];
        if (gl == 0) ops.claims += h.y - h.x;
        for (int i = h.x + gl; i < h.y; i += 4 * kG) {
            const int c0 = __ldg(c.claim + i);
            const int c1 = i + kG < h.y ? __ldg(c.claim + i + kG) : -1;
            const int c2 = i + 2 * kG < h.y ? __ldg(c.claim + i + 2 * kG) : -1;
            const int c3 = i + 3 * kG < h.y ? __ldg(c.claim + i + 3 * kG) : -1;
            atomicMax(c.map + c0, k);
            if (c1 >= 0) atomicMax(c.map + c1, k);
            if (c2 >= 0) atomicMax(c.map + c2, k);
            if (c3 >= 0) atomicMax(c.map + c3, k);
        }
    }
}

// Candidates owning all their points join batch `cur`; the others go to the
// lost list.  Block-uniform loop (staging and flushes).
__device__ __forceinline__ void commit_phase(const ColorDev &c, Stage &st, const int *list, int n, int cur,
                                             int *lost_cnt, int blk, int nblk, Ops &ops) {
    const int lane = threadIdx.x & 31, grp = lane / kG, gl = lane % kG;
    int it = 0;
    for (int b0 = blk * kGroups; b0 < n; b0 += nblk * kGroups, it++) {
        const int idx = b0 + threadIdx.x / kG;
        const bool valid = idx < n;
        const int k = valid ? list[idx] : -1;
        bool ok = true;
        if (valid) {
            const int4 h = c.hdr[k];
            if (gl == 0) ops.points += h.w - h.z;
            for (int i = h.z + gl; i < h.w; i += 2 * kG) {
                const int p0 = __ldg(c.pts + i);
                const int p1 = i + kG < h.w ? __ldg(c.pts + i + kG) : -1;
                const int o0 = owner(c, p0);
                const int o1 = p1 >= 0 ? owner(c, p1) : k;
                ok &= (o0 == k) & (o1 == k);
            }
        }
        const unsigned bad = (__ballot_sync(0xffffffffu, !ok) >> (grp * kG)) & kGroupMask;
        if (valid && bad == 0 && gl == 0) c.batch[k] = cur;
        stage(st, valid && bad != 0 && gl == 0, k, lane);
        if ((it + 1) % (kBuf / kGroups) == 0) flush(st, c.lost, lost_cnt);
    }
    flush(st, c.lost, lost_cnt);
}

// Lost nets with a point owned by a member are blocked and release their
// cells at once (a blocked net's cells are no member's points, so the release
// cannot change another net's check); the others stay candidates.
__device__ __forceinline__ void block_phase(const ColorDev &c, Stage &st, int n, int *cand_cnt, int blk, int nblk,
                                            Ops &ops) {
    const int lane = threadIdx.x & 31, grp = lane / kG, gl = lane % kG;
    int it = 0;
    for (int b0 = blk * kGroups; b0 < n; b0 += nblk * kGroups, it++) {
        const int idx = b0 + threadIdx.x / kG;
        const bool valid = idx < n;
        const int k = valid ? c.lost[idx] : -1;
        int4 h = make_int4(0, 0, 0, 0);
        bool hit = false;
        if (valid) {
            h = c.hdr[k];
            if (gl == 0) ops.bpoints += h.w - h.z;
            for (int i = h.z + gl; i < h.w; i += 2 * kG) {
                const int p0 = __ldg(c.pts + i);
                const int p1 = i + kG < h.w ? __ldg(c.pts + i + kG) : -1;
                const int o0 = owner(c, p0);
                const int o1 = p1 >= 0 ? owner(c, p1) : -1;
                const int b0v = o0 != -1 ? __ldcg(c.batch + o0) : -1;
                const int b1v = o1 != -1 ? __ldcg(c.batch + o1) : -1;
                hit |= (b0v != -1) | (b1v != -1);
            }
        }
        const bool blocked = ((__ballot_sync(0xffffffffu, hit) >> (grp * kG)) & kGroupMask) != 0;
        if (valid && blocked) {
            if (gl == 0) ops.releases += h.y - h.x;
            for (int i = h.x + gl; i < h.y; i += 4 * kG) {
                int cl[4], ow[4];
#pragma unroll
                for (int u = 0; u < 4; u++) cl[u] = i + u * kG < h.y ? __ldg(c.claim + i + u * kG) : -1;
#pragma unroll
                for (int u = 0; u < 4; u++) ow[u] = cl[u] >= 0 ? owner(c, cl[u]) : -1;
#pragma unroll
                for (int u = 0; u < 4; u++)
                    if (ow[u] == k) c.map[cl[u]] = -1;
            }
        }
        stage(st, valid && !blocked && gl == 0, k, lane);
        if ((it + 1) % (kBuf / kGroups) == 0) flush(st, c.cand, cand_cnt);
    }
    flush(st, c.cand, cand_cnt);
}

// Rounds `round`.. of batch `cur` in this block alone, over the nc candidates
// in c.cand.  Every thread of the block calls it.
__device__ void block_rounds(const ColorDev &c, Stage &st, int round, int nc, int cur, int *rounds_ctr, Ops &ops) {
    __shared__ int s_lost, s_cand;
    for (; round < 30; round++) {
        if (threadIdx.x == 0) {
            s_lost = 0;
            s_cand = 0;
            (*rounds_ctr)++;
        }
        __syncthreads();
        claim_phase(c, c.cand, nc, 0, 1, ops);
        __syncthreads();
        commit_phase(c, st, c.cand, nc, cur, &s_lost, 0, 1, ops);
        const int nl = s_lost;  // flush ends with a block barrier
        if (nl == nc) break;    // no net joined in this round
        block_phase(c, st, nl, &s_cand, 0, 1, ops);
        nc = s_cand;
        __syncthreads();  // every thread has read the counters before they are reset
        if (nc == 0) break;
    }
}

// Per batch: candidates claim (atomicMax of their rank on their claim cells),
// candidates owning all their points join, lost nets are blocked or stay
// candidates.  Three grid barriers per round; the last rounds of a batch,
// with few candidates, run in block 0 alone.  The lists are unordered: every
// phase is order-independent.
__global__ void __launch_bounds__(kThreads, 1) coloring_kernel(ColorDev c, int max_batches) {
    __shared__ Stage st;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int XY = c.X * c.Y;
    int *flags = c.flags;
    volatile int *vflags = c.flags;
    unsigned *bar = reinterpret_cast<unsigned *>(c.flags + F_BAR);
    int *err = c.flags + F_ERR;
    unsigned epoch = 0;
    Ops ops;
    auto sum_ops = [&]() {
        if (!c.ops) return;
        unsigned long long v[5] = {ops.claims, ops.points, ops.bpoints, ops.releases, ops.scans};
#pragma unroll
        for (int j = 0; j < 5; j++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
            if (lane == 0 && v[j]) atomicAdd(c.ops + j, v[j]);
        }
    };
    if (threadIdx.x == 0) st.n = 0;
    int *act = c.active, *act2 = c.active2;
    for (int k = tid; k < c.n; k += nth) {
        const int sh = c.perm ? c.perm[k] : k;
        const int c0 = c.claim_off[sh], p0 = c.pt_off[sh];
        c.hdr[k] = make_int4(c0, c.claim_n ? c0 + c.claim_n[sh] : c.claim_off[sh + 1], p0,
                             c.pt_n ? p0 + c.pt_n[sh] : c.pt_off[sh + 1]);
        act[k] = k;
    }
    const bool inc = c.rev != nullptr;
    for (int i = tid; i < XY; i += nth) {
        c.map[i] = -1;
        if (inc) c.rev_cnt[i] = 0;
    }
    if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
    if (inc) {
        // claimers of every cell (ranks), grouped by cell: counts, an exclusive
        // scan over the cells (a chunk per block), then the entries
        for (int k = tid; k < c.n; k += nth) {
            const int4 h = c.hdr[k];
            for (int i = h.x; i < h.y; i++) atomicAdd(c.rev_cnt + __ldg(c.claim + i), 1);
        }
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        const int chunk = (XY + gridDim.x - 1) / gridDim.x;
        const int lo = min(XY, blockIdx.x * chunk), hi = min(XY, lo + chunk);
        const int per = (hi - lo + kThreads - 1) / kThreads;
        const int a0 = min(hi, lo + threadIdx.x * per), a1 = min(hi, a0 + per);
        int mine = 0, total = 0;
        for (int i = a0; i < a1; i++) mine += c.rev_cnt[i];
        int run = block_exclusive(mine, &total);
        if (threadIdx.x == 0) c.part[blockIdx.x] = total;
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        if (tid == 0) {
            int acc = 0;
            for (int b = 0; b < (int)gridDim.x; b++) {
                const int t = c.part[b];
                c.part[b] = acc;
                acc += t;
            }
        }
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        run += c.part[blockIdx.x];
        for (int i = a0; i < a1; i++) {
            c.rev_off[i] = run;
            run += c.rev_cnt[i];
            c.rev_cnt[i] = 0;
        }
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        for (int k = tid; k < c.n; k += nth) {
            const int4 h = c.hdr[k];
            for (int i = h.x; i < h.y; i++) {
                const int cell = __ldg(c.claim + i);
                c.rev[c.rev_off[cell] + atomicAdd(c.rev_cnt + cell, 1)] = k;
            }
        }
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
    }
    int na = c.n;
    for (int cur = 0; cur < max_batches; cur++) {
        const int *cand = act;  // round 0: every net without a batch
        int nc = na;
        int round = 0;
        bool tail = false;
        for (; round < 30; round++) {
            if (round > 0 && nc <= kBlockRounds) {
                tail = true;
                break;
            }
            // with the round-0 map kept up to date, round 0 of a later batch
            // starts from it (its counters were reset before the last barrier)
            const bool kept = inc && round == 0 && cur > 0;
            if (tid == 0) {
                flags[F_ROUNDS]++;
                if (!kept) flags[F_LOST] = 0;
            }
            if (!kept) {
                claim_phase(c, cand, nc, blockIdx.x, gridDim.x, ops);
                if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
                if (tid == 0) {
                    flags[F_CAND] = 0;
                    if (round == 0) flags[F_LEFT + ((cur + 1) & 1)] = 0;
                }
            }
            if (inc && round == 0 && cur == 0)  // the first round-0 map, before any release
                for (int i = tid; i < XY; i += nth) c.snap[i] = __ldcg(c.map + i);
            commit_phase(c, st, cand, nc, cur, flags + F_LOST, blockIdx.x, gridDim.x, ops);
            if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
            const int nl = vflags[F_LOST];
            if (nl == nc) break;  // no net joined in this round
            block_phase(c, st, nl, flags + F_CAND, blockIdx.x, gridDim.x, ops);
            if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
            cand = c.cand;
            nc = vflags[F_CAND];
            if (nc == 0) break;
        }
        if (tail) {
            if (blockIdx.x == 0) block_rounds(c, st, round, nc, cur, flags + F_ROUNDS, ops);
            if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        }
        // nets still without a batch stay active; the map is cleared for the
        // next batch, or, when the round-0 map is kept, the cells whose
        // round-0 owner joined this batch are marked for recomputation
        if (!inc)
            for (int i = tid; i < XY; i += nth) c.map[i] = -1;
        int it = 0;
        for (int b0 = blockIdx.x * kThreads; b0 < na; b0 += nth, it++) {
            const int i = b0 + threadIdx.x;
            const int k = i < na ? act[i] : -1;
            const int bk = k >= 0 ? __ldcg(c.batch + k) : -2;
            if (k >= 0) ops.scans++;
            if (inc && bk == cur) {
                const int4 h = c.hdr[k];
                ops.releases += h.y - h.x;
                for (int q = h.x; q < h.y; q++) {
                    const int cell = __ldg(c.claim + q);
                    if (c.snap[cell] == k) {
                        c.snap[cell] = -1;
                        c.dirty[atomicAdd(flags + F_DIRTY, 1)] = cell;
                    }
                }
            }
            stage(st, bk == -1, k, lane);
            if ((it + 1) % (kBuf / kThreads) == 0) flush(st, act2, flags + F_LEFT + (cur & 1));
        }
        flush(st, act2, flags + F_LEFT + (cur & 1));
        if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        na = vflags[F_LEFT + (cur & 1)];
        int *t = act; act = act2; act2 = t;
        if (na == 0) {
            if (tid == 0) flags[F_NB] = cur + 1;
            sum_ops();
            return;
        }
        if (inc) {
            // new round-0 owner of every marked cell: its highest claimer
            // still without a batch (claimers with a batch leave the list)
            // one warp per marked cell: 32 claimers per step, compacted in place
            // (a step writes only below the entries it has read)
            const int nd = vflags[F_DIRTY];
            for (int i = tid >> 5; i < nd; i += nth >> 5) {
                const int cell = c.dirty[i];
                const int base = c.rev_off[cell], len = c.rev_cnt[cell];
                int best = -1, w = 0;
                for (int q0 = 0; q0 < len; q0 += 32) {
                    const int q = q0 + lane;
                    const int k = q < len ? c.rev[base + q] : -1;
                    const bool live = k >= 0 && __ldcg(c.batch + k) == -1;
                    const unsigned m = __ballot_sync(0xffffffffu, live);
                    if (live) {
                        c.rev[base + w + __popc(m & ((1u << lane) - 1))] = k;
                        best = max(best, k);
                    }
                    w += __popc(m);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
                if (lane == 0) {
                    ops.scans += len;
                    c.rev_cnt[cell] = w;
                    c.snap[cell] = best;
                }
            }
            if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
            for (int i = tid; i < XY; i += nth) c.map[i] = c.snap[i];
            if (tid == 0) {  // counters of round 0 of the next batch
                flags[F_DIRTY] = 0;
                flags[F_LOST] = 0;
                flags[F_CAND] = 0;
                flags[F_LEFT + ((cur + 2) & 1)] = 0;
            }
            if (!grid_sync(bar, err, epoch, c.wait_ns, c.phantom)) return;
        }
    }
    if (tid == 0) flags[F_NB] = max_batches;
    sum_ops();
}

}  // namespace

void build_claims(int nshapes, const int *pt_off, const int *pts, const int *h_off, const int *hseg,
                  const int *v_off, const int *vseg, int X, int Y, int sparsity, std::vector<int> &off,
                  std::vector<int> &cells, int threads) {
    static const int dx[4] = {0, 0, -1, 1}, dy[4] = {0, -1, 0, 0};
    // cells of shape k in claim order; emit(cell) is called for each
    auto walk = [&](int k, auto &&emit) {
        for (int i = pt_off[k]; i < pt_off[k + 1]; i++) {
            const int x = pts[i] / Y, y = pts[i] % Y;
            for (int j = 0; j < 4; j++) {
                const int nx = x + dx[j], ny = y + dy[j];
                if (nx >= 0 && nx < X && ny >= 0 && ny < Y) emit(nx * Y + ny);
            }
        }
        for (int i = h_off[k]; i < h_off[k + 1]; i++) {
            const int s0 = hseg[2 * i], e0 = hseg[2 * i + 1], y = s0 % Y;
            for (int x = s0 / Y; x <= e0 / Y; x += sparsity) emit(x * Y + y);
        }
        for (int i = v_off[k]; i < v_off[k + 1]; i++) {
            const int s0 = vseg[2 * i], e0 = vseg[2 * i + 1], x = s0 / Y;
            for (int y = s0 % Y; y <= e0 % Y; y += sparsity) emit(x * Y + y);
        }
    };
    off.assign(nshapes + 1, 0);
    parallel_for(nshapes, threads, [&](int b, int e) {
        for (int k = b; k < e; k++) {
            int n = 0;
            walk(k, [&](int) { n++; });
            off[k + 1] = n;
        }
    });
    for (int k = 0; k < nshapes; k++) off[k + 1] += off[k];
    cells.resize(off[nshapes]);
    parallel_for(nshapes, threads, [&](int b, int e) {
        for (int k = b; k < e; k++) {
            int *o = cells.data() + off[k];
            walk(k, [&](int c) { *o++ = c; });
        }
    });
}

int run_coloring(ColorDev &c, int max_batch, cudaStream_t s) {
    (void)max_batch;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, coloring_kernel, kThreads, 0);
    int blocks = sms * (per < 1 ? per : 1);
    if (blocks < 1) blocks = 1;
    c.wait_ns = (unsigned long long)test_hooks().wait_ns.load();
    c.phantom = (unsigned)test_hooks().barrier_phantom.load();
    cudaMemsetAsync(c.flags, 0, 16 * sizeof(int), s);
    cudaMemsetAsync(c.batch, 0xff, sizeof(int) * (size_t)c.n, s);
    int max_batches = c.n + 1;
    void *args[] = {&c, &max_batches};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)coloring_kernel, dim3(blocks), dim3(kThreads), args, 0, s);
    if (e != cudaSuccess) return -1;
    int h[16];
    if (cudaMemcpyAsync(h, c.flags, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (h[F_ERR] != 0) return -2;
    c.rounds = h[F_ROUNDS];
    return h[F_NB];
}

}  // namespace igr
