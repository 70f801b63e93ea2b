// Phase-1 conflict shapes and claim lists of the batch colouring, built on the
// device from the flattened trees already resident there.
//
// The shapes of a routing net (net::construct_rsmt, src/database_cuda.hpp:
// 746-820) are its tree nodes as points and, per tree edge, its segments and
// end or corner points; the claims (generate_batches_rsmt_gpu,
// src/database_cuda.hpp:288-434) are the cell, left, right and lower cells of
// every point and every `sparsity`-th cell of every segment.  They depend only
// on the set of tree edges, so they are generated here from the (node,
// parent) pairs of the DFS-ordered trees; the colouring treats points and
// claims as sets, so the order inside a net is free.  Two passes: counts per
// net with an exclusive scan (one block), then the fill.  The rip-up passes
// use the same kernels for the rerouted nets, with the DAG points given and
// the segments of their trees.
#include "kcommon.cuh"

namespace igr {

namespace {

constexpr int kScanThreads = 1024;

template <class Pt, class Hs, class Vs>
__device__ __forceinline__ void net_shapes(const int *nodes, const int *par, int m, int X, int Y, Pt &&point,
                                           Hs &&hseg, Vs &&vseg) {
    const int XY = X * Y;
    for (int i = 0; i < m; i++) {
        const int p = nodes[i] % XY;
        point(p / Y, p % Y);
    }
    for (int i = 1; i < m; i++) {
        const int j = par[i];
        if (j < 0) continue;
        const int pi = nodes[i] % XY, pj = nodes[j] % XY;
        const int xi = pi / Y, yi = pi % Y, xj = pj / Y, yj = pj % Y;
        const int mnx = min(xi, xj), mxx = max(xi, xj), mny = min(yi, yj), mxy = max(yi, yj);
        if (xi != xj && yi != yj) {
            hseg(mnx, mxx, mny);
            hseg(mnx, mxx, mxy);
            vseg(mny, mxy, mnx);
            vseg(mny, mxy, mxx);
            point(xi, yj);
            point(xj, yi);
        } else if (xi != xj) {
            hseg(mnx, mxx, mny);
            point(mnx, mny);
            point(mxx, mny);
        } else if (yi != yj) {
            vseg(mny, mxy, mnx);
            point(mnx, mny);
            point(mnx, mxy);
        }
    }
}

// claimed cells of a point: the cell, the one below, left and right (in the grid)
__device__ __forceinline__ int point_claims(int x, int y, int X, int Y) {
    return 1 + (y > 0) + (x > 0) + (x + 1 < X);
}

// shape k: routing net ids[k] (k when ids is null); its points are the tree's
// (nodes and edge points) or, when ext_off is given, ext_pts[ext_off[k] ..
// ext_off[k+1]); its segments are always the tree's
struct ShapeSrc {
    const int *tree_off, *tree_nodes, *tree_par, *ids, *ext_off, *ext_pts;
    const long long *ext_at;
    const int *ext_cnt;
    int ext_stride, n, X, Y, sp;
};

template <class Pt, class Hs, class Vs>
__device__ __forceinline__ void shape_of(const ShapeSrc &a, int k, Pt &&point, Hs &&hseg, Vs &&vseg) {
    const int net = a.ids ? a.ids[k] : k;
    const int t = a.tree_off[net], m = a.tree_off[net + 1] - t;
    if (a.ext_off || a.ext_at) {
        const long long q0 = a.ext_at ? a.ext_at[k] : a.ext_off[k];
        const long long q1 = a.ext_at ? q0 + a.ext_cnt[(size_t)k * a.ext_stride] : a.ext_off[k + 1];
        for (long long q = q0; q < q1; q++) point(a.ext_pts[q] / a.Y, a.ext_pts[q] % a.Y);
        net_shapes(a.tree_nodes + t, a.tree_par + t, m, a.X, a.Y, [](int, int) {}, hseg, vseg);
    } else {
        net_shapes(a.tree_nodes + t, a.tree_par + t, m, a.X, a.Y, point, hseg, vseg);
    }
}

__global__ void shape_count_kernel(ShapeSrc a, int *pt_cnt, int *claim_cnt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const int X = a.X, Y = a.Y, sp = a.sp;
    int np = 0, nc = 0;
    shape_of(
        a, k,
        [&](int x, int y) {
            np++;
            nc += point_claims(x, y, X, Y);
        },
        [&](int lo, int hi, int) { nc += (hi - lo) / sp + 1; }, [&](int lo, int hi, int) { nc += (hi - lo) / sp + 1; });
    pt_cnt[k + 1] = np;
    claim_cnt[k + 1] = nc;
}

// exclusive scan of a[1..n] into a[0..n] (a[0] = 0) in one block; the total
// goes to *total (64-bit, so that an overflow of the 32-bit offsets is seen)
__device__ void block_scan(int *a, int n, long long *total) {
    __shared__ long long part[kScanThreads];
    const int t = threadIdx.x;
    const int chunk = (n + kScanThreads - 1) / kScanThreads;
    const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
    long long sum = 0;
    for (int i = lo; i < hi; i++) sum += a[i + 1];
    part[t] = sum;
    __syncthreads();
    for (int d = 1; d < kScanThreads; d <<= 1) {
        const long long v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = part[t] - sum;
    for (int i = lo; i < hi; i++) {
        run += a[i + 1];
        a[i + 1] = (int)run;
    }
    if (t == 0) a[0] = 0;
    if (t == kScanThreads - 1) *total = part[t];
    __syncthreads();
}

__global__ void __launch_bounds__(kScanThreads) shape_scan_kernel(int R, int *pt_off, int *claim_off,
                                                                   long long *totals) {
    block_scan(pt_off, R, totals);
    block_scan(claim_off, R, totals + 1);
}

// Sorts a[0..n) (Shell's method, Ciura's gaps) and moves its distinct values
// to the front; returns their number.
__device__ int sort_unique(int *a, int n) {
    constexpr int kGaps[8] = {701, 301, 132, 57, 23, 10, 4, 1};
#pragma unroll 1
    for (int gi = 0; gi < 8; gi++) {
        const int gap = kGaps[gi];
        for (int i = gap; i < n; i++) {
            const int v = a[i];
            int j = i;
            while (j >= gap && a[j - gap] > v) {
                a[j] = a[j - gap];
                j -= gap;
            }
            a[j] = v;
        }
    }
    int m = 0;
    for (int i = 0; i < n; i++)
        if (m == 0 || a[i] != a[m - 1]) a[m++] = a[i];
    return m;
}

// pt_n / claim_n (optional): the number of distinct points and claimed cells of
// each shape, moved to the front of its range.  A node of a tree is a point
// once for itself and again for every straight edge it ends, and the claims of
// neighbouring points and of segment samples overlap; the colouring only asks
// whether a cell is claimed and whether a point is owned, so each is kept once.
__global__ void shape_fill_kernel(ShapeSrc a, const int *pt_off, const int *claim_off, int *pts, int *claim,
                                  int *pt_n, int *claim_n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const int X = a.X, Y = a.Y, sp = a.sp;
    int *pt = pts + pt_off[k];
    int *cl = claim + claim_off[k];
    shape_of(
        a, k,
        [&](int x, int y) {
            *pt++ = x * Y + y;
            *cl++ = x * Y + y;
            if (y > 0) *cl++ = x * Y + y - 1;
            if (x > 0) *cl++ = (x - 1) * Y + y;
            if (x + 1 < X) *cl++ = (x + 1) * Y + y;
        },
        [&](int lo, int hi, int y) {
            for (int x = lo; x <= hi; x += sp) *cl++ = x * Y + y;
        },
        [&](int lo, int hi, int x) {
            for (int y = lo; y <= hi; y += sp) *cl++ = x * Y + y;
        });
    if (pt_n) pt_n[k] = sort_unique(pts + pt_off[k], (int)(pt - (pts + pt_off[k])));
    if (claim_n) claim_n[k] = sort_unique(claim + claim_off[k], (int)(cl - (claim + claim_off[k])));
}

}  // namespace

void launch_shape_count(const ShapeArgs &a, int *pt_off, int *claim_off, long long *totals, cudaStream_t s) {
    const ShapeSrc src{a.tree_off, a.tree_nodes, a.tree_par, a.ids, a.ext_off, a.ext_pts, a.ext_at,
                       a.ext_cnt, a.ext_stride, a.n, a.X, a.Y, a.sparsity};
    if (a.n > 0) shape_count_kernel<<<(a.n + 255) / 256, 256, 0, s>>>(src, pt_off, claim_off);
    shape_scan_kernel<<<1, kScanThreads, 0, s>>>(a.n, pt_off, claim_off, totals);
}

void launch_shape_fill(const ShapeArgs &a, const int *pt_off, const int *claim_off, int *pts, int *claim,
                       int *pt_n, int *claim_n, cudaStream_t s) {
    const ShapeSrc src{a.tree_off, a.tree_nodes, a.tree_par, a.ids, a.ext_off, a.ext_pts, a.ext_at,
                       a.ext_cnt, a.ext_stride, a.n, a.X, a.Y, a.sparsity};
    if (a.n > 0)
        shape_fill_kernel<<<(a.n + 255) / 256, 256, 0, s>>>(src, pt_off, claim_off, pts, claim, pt_n, claim_n);
}

}  // namespace igr
