// Evaluation of a routing result on the device with the rules of the ISPD2024
// evaluator (run/evaluator.cpp:462-633, NVR_DB::read_gr_solution), without
// writing or reading a guide file.
//
// The evaluator reads the guides net by net: a via segment adds one via per
// crossed layer and a via location per layer; a wire marks its cells (both
// ends) with the net and counts one wire on every cell but the last.  At the
// end of a net every via location not yet marked by the same net (by one of
// its wires, or by an earlier via location) adds the stacked-via demand of
// its layer (half a unit on both track edges beside the cell, a full unit at
// the grid boundary).  Per routing layer the cell demand is 2 wires + stacked
// vias (kept in 16 bits as in the evaluator), the overflow loss is
// exp(0.5 * (demand - 2 cap) / 2) where cap > 0.001, else exp(0.5 * 1.5 demand)
// where the demand is positive, and the costs are summed per layer.
//
// Marks only ever compare with the net's own index, so every net is
// independent: the marks of a net are kept in two hash sets keyed by
// (net, layer, x, y) — the cells its wires cover, and its via locations with
// the first position in the net's guide order — and all nets run at once.
// The segments of a design net are the evaluator's guide lines of the route
// writer, in its order: pin vias from layer 0, stacked-pin pairs, then the
// route records of its routing nets.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ unsigned long long hash64(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// (net, layer, x, y) as one key: 28 + 4 + 16 + 16 bits
__device__ __forceinline__ unsigned long long cell_key(int net, int z, int x, int y) {
    return ((unsigned long long)net << 36) | ((unsigned long long)z << 32) | ((unsigned long long)x << 16) |
           (unsigned long long)y;
}

// inserts k; returns its slot (every probe sequence ends: the table is never full)
__device__ __forceinline__ unsigned long long set_insert(unsigned long long *keys, unsigned long long mask,
                                                         unsigned long long k) {
    unsigned long long s = hash64(k) & mask;
    for (unsigned long long n = 0; n <= mask; n++, s = (s + 1) & mask) {
        const unsigned long long prev = atomicCAS(keys + s, kEmpty, k);
        if (prev == kEmpty || prev == k) return s;
    }
    return kEmpty;
}

__device__ __forceinline__ bool set_contains(const unsigned long long *keys, unsigned long long mask,
                                             unsigned long long k) {
    unsigned long long s = hash64(k) & mask;
    for (unsigned long long n = 0; n <= mask; n++, s = (s + 1) & mask) {
        const unsigned long long v = keys[s];
        if (v == k) return true;
        if (v == kEmpty) return false;
    }
    return false;
}

// 3-D file-layer position of a route entry, and of a routing layer's cell in the
// track layout (file layer z >= 1 is routing layer z - 1)
__device__ __forceinline__ int64_t cell_at_file(const EvalDev &e, int z, int x, int y) {
    const int l = z - 1;
    const int64_t b = (int64_t)l * e.X * e.Y;
    return (((l & 1) ^ e.DIR) != 0) ? b + (int64_t)x * e.Y + y : b + (int64_t)y * e.X + x;
}

// Calls f(p, q) for every guide line of design net n, in the route writer's
// order, with p <= q (write_guides: pin vias, stacked-pin pairs, records).
template <class F>
__device__ __forceinline__ void for_each_line(const EvalDev &e, int n, F &&f) {
    const int XY = e.X * e.Y;
    for (int64_t i = e.sel_off[n]; i < e.sel_off[n + 1]; i++)
        if (e.sel[i] < XY) f(e.sel[i], e.sel[i] + XY);
    for (int64_t i = e.extra_off[n]; i + 1 < e.extra_off[n + 1]; i += 2) {
        const int a = e.extra[i], b = e.extra[i + 1];
        f(a < b ? a : b, a < b ? b : a);
    }
    for (int s = e.sub_off[n]; s < e.sub_off[n + 1]; s++) {
        const int *r = e.routes + e.route_off[s];
        for (int j = 1; j < r[0]; j += 2) {
            const int a = r[j] + XY, b = r[j + 1] + XY;
            f(a < b ? a : b, a < b ? b : a);
        }
    }
}

// counts per design net: via locations and wire cells (ends included)
__global__ void eval_count_kernel(EvalDev e, long long *via_cnt, long long *cell_cnt) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= e.n) return;
    const int X = e.X, Y = e.Y, XY = X * Y;
    long long vias = 0, cells = 0;
    for_each_line(e, n, [&](int p, int q) {
        const int zl = p / XY, zh = q / XY;
        if (zl != zh) {
            vias += zh - zl;
        } else {
            const int xl = p / Y % X, yl = p % Y, xh = q / Y % X, yh = q % Y;
            cells += (xh - xl) + (yh - yl) + 1;
        }
    });
    via_cnt[n] = vias;
    cell_cnt[n] = cells;
}

// One guide line of design net n at position t of the net's order; its via
// locations go to vloc[at ..].
__device__ __forceinline__ void eval_line(const EvalDev &e, int n, int p, int q, int t, long long at,
                                          unsigned long long *vias) {
    const int X = e.X, Y = e.Y, XY = X * Y;
    const int zl = p / XY, zh = q / XY;
    const int xl = p / Y % X, yl = p % Y, xh = q / Y % X, yh = q % Y;
    if (zl != zh) {
        const bool bad = xl != xh || yl != yh;  // a via must be vertical
        if (bad) set_error(e.err, ERR_STATE);
        for (int z = zl; z < zh; z++) {
            vias[z < kEvalLayers ? z : kEvalLayers - 1]++;
            const unsigned long long k = bad ? cell_key(n, 0, 0, 0) : cell_key(n, z, xl, yl);
            e.vloc[at] = k;
            e.vord[at] = (unsigned)t;
            at++;
            if (bad) continue;
            const unsigned long long s = set_insert(e.vkeys, e.vmask, k);
            if (s == kEmpty) set_error(e.err, ERR_CAPACITY);
            else atomicMin(e.vfirst + s, (unsigned)t);
        }
        return;
    }
    // a wire along its layer: horizontal layers run along x
    const bool hor = zl >= 1 && ((((zl - 1) & 1) ^ e.DIR) == 0);
    if (zl < 1 || (hor && !(xh > xl && yh == yl)) || (!hor && !(yh > yl && xh == xl))) {
        set_error(e.err, ERR_STATE);
        return;
    }
    const int len = hor ? xh - xl : yh - yl;
    for (int c = 0; c <= len; c++) {
        const int x = hor ? xl + c : xl, y = hor ? yl : yl + c;
        if (set_insert(e.wkeys, e.wmask, cell_key(n, zl, x, y)) == kEmpty) set_error(e.err, ERR_CAPACITY);
        if (c < len) atomicAdd(e.wire + cell_at_file(e, zl, x, y), 1);
    }
}

// one warp per design net, one lane per guide line: wires mark their cells
// and count wires; vias count per layer and record their locations (in the
// net's order, placed by prefix sums over the lanes)
__global__ void eval_lines_kernel(EvalDev e, const long long *via_off) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1;
    const int XY = e.X * e.Y;
    for (int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < e.n; n += (gridDim.x * blockDim.x) >> 5) {
        int tbase = 0;
        long long vbase = via_off[n];
        unsigned long long vias[kEvalLayers];
        for (int z = 0; z < kEvalLayers; z++) vias[z] = 0;
        // a round of up to 32 lines, line `lane` valid when `ok`
        auto round = [&](bool ok, int p, int q) {
            const int nv = ok ? q / XY - p / XY : 0;
            int inc = nv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += v;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) eval_line(e, n, p, q, tbase + __popc(m & lt), vbase + inc - nv, vias);
            tbase += __popc(m);
            vbase += __shfl_sync(0xffffffffu, inc, 31);
        };
        for (int64_t i0 = e.sel_off[n]; i0 < e.sel_off[n + 1]; i0 += 32) {
            const int64_t i = i0 + lane;
            const bool ok = i < e.sel_off[n + 1] && e.sel[i] < XY;
            const int p = ok ? e.sel[i] : 0;
            round(ok, p, p + XY);
        }
        const int64_t x0 = e.extra_off[n];
        const int ne = (int)((e.extra_off[n + 1] - x0) / 2);
        for (int k0 = 0; k0 < ne; k0 += 32) {
            const int k = k0 + lane;
            const bool ok = k < ne;
            const int a = ok ? e.extra[x0 + 2 * k] : 0, b = ok ? e.extra[x0 + 2 * k + 1] : 0;
            round(ok, a < b ? a : b, a < b ? b : a);
        }
        for (int s = e.sub_off[n]; s < e.sub_off[n + 1]; s++) {
            const int *r = e.routes + e.route_off[s];
            const int m = r[0] / 2;  // lines j = 1, 3, .. < r[0]
            for (int k0 = 0; k0 < m; k0 += 32) {
                const int k = k0 + lane;
                const bool ok = k < m;
                const int a = ok ? r[1 + 2 * k] + XY : 0, b = ok ? r[2 + 2 * k] + XY : 0;
                round(ok, a < b ? a : b, a < b ? b : a);
            }
        }
        for (int z = 0; z < kEvalLayers; z++) {
            unsigned long long v = vias[z];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0 && v) atomicAdd(e.total_vias + z, v);
        }
    }
}

// stacked vias: the first via location of its key in the net's order that no
// wire of the net covers (update_stacked_via_counter, evaluator.cpp:636-672)
__global__ void eval_stacked_kernel(EvalDev e, long long nloc) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nloc) return;
    const unsigned long long k = e.vloc[i];
    const int z = (int)((k >> 32) & 15), x = (int)((k >> 16) & 0xffff), y = (int)(k & 0xffff);
    if (z < 1) return;  // the pin layer is not a routing layer: its demand is not scored
    if (set_contains(e.wkeys, e.wmask, k)) return;
    // the key's slot holds the first position; find it
    unsigned long long s = hash64(k) & e.vmask;
    for (unsigned long long n = 0; n <= e.vmask; n++, s = (s + 1) & e.vmask)
        if (e.vkeys[s] == k) break;
    if (e.vfirst[s] != e.vord[i]) return;
    const bool hor = (((z - 1) & 1) ^ e.DIR) == 0;
    if (hor) {
        if (x > 0 && x < e.X - 1) {
            atomicAdd(e.stacked + cell_at_file(e, z, x - 1, y), 1);
            atomicAdd(e.stacked + cell_at_file(e, z, x, y), 1);
        } else if (x > 0) {
            atomicAdd(e.stacked + cell_at_file(e, z, x - 1, y), 2);
        } else if (x < e.X - 1) {
            atomicAdd(e.stacked + cell_at_file(e, z, x, y), 2);
        }
    } else {
        if (y > 0 && y < e.Y - 1) {
            atomicAdd(e.stacked + cell_at_file(e, z, x, y - 1), 1);
            atomicAdd(e.stacked + cell_at_file(e, z, x, y), 1);
        } else if (y > 0) {
            atomicAdd(e.stacked + cell_at_file(e, z, x, y - 1), 2);
        } else if (y < e.Y - 1) {
            atomicAdd(e.stacked + cell_at_file(e, z, x, y), 2);
        }
    }
}

constexpr int kCellThreads = 256;

// per routing layer and block of cells: the overflow loss in a fixed order
// (a fixed tree inside the block) and the wire length; the layer sums are
// then taken over the blocks in order, so the result does not depend on
// scheduling
__global__ void __launch_bounds__(kCellThreads) eval_cells_kernel(EvalDev e, int blocks_per_layer, double *part) {
    __shared__ double s[kCellThreads];
    const int l = blockIdx.x / blocks_per_layer, b = blockIdx.x % blocks_per_layer;
    const int z = l + 1;
    const int64_t XY = (int64_t)e.X * e.Y;
    const int64_t per = (XY + blocks_per_layer - 1) / blocks_per_layer;
    const int64_t c0 = b * per, c1 = c0 + per < XY ? c0 + per : XY;
    double loss = 0;
    unsigned long long wl = 0;
    const bool hor = ((l & 1) ^ e.DIR) == 0;
    for (int64_t c = c0 + threadIdx.x; c < c1; c += kCellThreads) {
        const int x = (int)(c / e.Y), y = (int)(c % e.Y);
        const int64_t i = cell_at_file(e, z, x, y);
        const int w = e.wire[i];
        const unsigned demand = (unsigned)(2 * w + e.stacked[i]) & 0xffffu;  // a 16-bit field in the evaluator
        const double cap = e.cap_d ? e.cap_d[i] : (double)e.cap[i];
        if (cap > 0.001) {
            const double overflow = double(demand) - 2 * cap;
            loss += exp((overflow / 2) * 0.5);
        } else if (cap >= 0 && demand > 0) {
            loss += exp((1.5 * double(demand)) * 0.5);
        }
        if (w) wl += (unsigned long long)w * (unsigned long long)(hor ? e.xlen[x] : e.ylen[y]);
    }
    s[threadIdx.x] = loss;
    __syncthreads();
    for (int o = kCellThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wl += __shfl_down_sync(0xffffffffu, wl, o);
    if ((threadIdx.x & 31) == 0 && wl) atomicAdd(e.wl + l, wl);
}

}  // namespace

int eval_blocks_per_layer(int64_t XY) {
    int64_t b = (XY + 4 * kCellThreads - 1) / (4 * kCellThreads);
    return (int)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

void launch_eval_count(const EvalDev &e, long long *via_cnt, long long *cell_cnt, cudaStream_t s) {
    if (e.n > 0) eval_count_kernel<<<(e.n + 255) / 256, 256, 0, s>>>(e, via_cnt, cell_cnt);
}

void launch_eval_marks(const EvalDev &e, const long long *via_off, long long nloc, cudaStream_t s) {
    if (e.n > 0) {
        const int warps = 8;
        int blocks = (e.n + warps - 1) / warps;
        if (blocks > 148 * 32) blocks = 148 * 32;
        eval_lines_kernel<<<blocks, 32 * warps, 0, s>>>(e, via_off);
    }
    if (nloc > 0) eval_stacked_kernel<<<(unsigned)((nloc + 255) / 256), 256, 0, s>>>(e, nloc);
}

void launch_eval_cells(const EvalDev &e, int blocks_per_layer, double *part, cudaStream_t s) {
    eval_cells_kernel<<<blocks_per_layer * e.L, kCellThreads, 0, s>>>(e, blocks_per_layer, part);
}

}  // namespace igr
