// Input features of the learned congestion seed, computed on the device from
// the resident trees of the routing nets and the capacities (the host
// restatement is seed_features in seed_model.cpp; the channels are the same):
//   0 pins per GCell (a quarter per pin), 1 RUDY-H, 2 RUDY-V (a net spreads
//   1/h of horizontal and 1/w of vertical wire density over its w x h
//   bounding box, halved), 3 fraction of blocked routing layers (capacity
//   below 0.5), 4..13 capacity of file layers 0..9 over 8, 14..15 zero.
// The RUDY difference arrays are accumulated in 2^-36 fixed point in 64-bit
// integers, so that the atomics add up to the same sums in any order; the
// host's double sums agree with them to about 1e-11, far below the features'
// BF16 rounding.
#include "kcommon.cuh"
#include "seed.hpp"

#include <cuda_bf16.h>

namespace igr {

namespace {

constexpr double kFix = 68719476736.0;  // 2^36

// One thread per routing net: its pins (tree nodes below the Steiner layer)
// counted per GCell, its bounding box's four corners added to the
// difference arrays ((X+1) x (Y+1), row-major by x).
__global__ void feat_net_kernel(int n, const int *tree_off, const int *nodes, int L, int X, int Y, int *pins,
                                long long *dh, long long *dv) {
    const int XY = X * Y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int minx = X, maxx = -1, miny = Y, maxy = -1;
        for (int i = tree_off[r]; i < tree_off[r + 1]; i++) {
            const int v = nodes[i];
            if (v >= L * XY) continue;  // Steiner point
            const int q = v % XY, x = q / Y, y = q - x * Y;
            atomicAdd(pins + q, 1);
            minx = min(minx, x); maxx = max(maxx, x);
            miny = min(miny, y); maxy = max(maxy, y);
        }
        if (maxx < 0) continue;
        const long long vh = __double2ll_rn(kFix / (double)(maxy - miny + 1));
        const long long vv = __double2ll_rn(kFix / (double)(maxx - minx + 1));
        const int W = Y + 1;
        auto add = [&](long long *a, int x, int y, long long v) {
            atomicAdd(reinterpret_cast<unsigned long long *>(a + (size_t)x * W + y), (unsigned long long)v);
        };
        add(dh, minx, miny, vh); add(dh, maxx + 1, miny, -vh); add(dh, minx, maxy + 1, -vh); add(dh, maxx + 1, maxy + 1, vh);
        add(dv, minx, miny, vv); add(dv, maxx + 1, miny, -vv); add(dv, minx, maxy + 1, -vv); add(dv, maxx + 1, maxy + 1, vv);
    }
}

// Prefix sums along y: one warp per row x of both arrays, 32 entries a step.
__global__ void feat_scan_y_kernel(int X, int Y, long long *dh, long long *dv) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp > X) return;
    const int W = Y + 1;
    for (int k = 0; k < 2; k++) {
        long long *row = (k ? dv : dh) + (size_t)warp * W;
        long long carry = 0;
        for (int y0 = 0; y0 < W; y0 += 32) {
            const int y = y0 + lane;
            long long v = y < W ? row[y] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += t;
            }
            v += carry;
            if (y < W) row[y] = v;
            carry = __shfl_sync(0xffffffffu, v, 31);
        }
    }
}

// Prefix sums along x: one thread per column y of both arrays.
__global__ void feat_scan_x_kernel(int X, int Y, long long *dh, long long *dv) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    const int W = Y + 1;
    if (y > Y) return;
    long long ch = 0, cv = 0;
    for (int x = 0; x <= X; x++) {
        const size_t i = (size_t)x * W + y;
        ch += dh[i];
        cv += dv[i];
        dh[i] = ch;
        dv[i] = cv;
    }
}

// One thread per GCell: the 16 channels (cap0: file layer 0's capacity in
// the reference layout; the routing layers' from the grid).
__global__ void feat_out_kernel(GridDev g, const float *cap0, int Lfile, const int *pins, const long long *dh,
                                const long long *dv, __nv_bfloat16 *out) {
    const int X = g.X, Y = g.Y;
    const int64_t XY = (int64_t)X * Y;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < XY; c += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(c / Y), y = (int)(c - (int64_t)x * Y);
        const size_t at = (size_t)x * (Y + 1) + y;
        __nv_bfloat16 o[16];
        o[0] = __float2bfloat16((float)pins[c] * 0.25f);
        o[1] = __float2bfloat16((float)(0.5 * ((double)dh[at] / kFix)));
        o[2] = __float2bfloat16((float)(0.5 * ((double)dv[at] / kFix)));
        int blocked = 0;
        for (int l = 0; l < 10; l++) {
            float cap = 0.f;
            if (l < Lfile) cap = l == 0 ? cap0[c] : g.cap[cell_at(g, l - 1, x, y)];
            o[4 + l] = __float2bfloat16(cap / 8.f);
            if (l > 0 && l < Lfile && cap < 0.5f) blocked++;
        }
        o[3] = __float2bfloat16(Lfile > 1 ? (float)blocked / (float)(Lfile - 1) : 0.f);
        o[14] = __float2bfloat16(0.f);
        o[15] = __float2bfloat16(0.f);
        uint4 *dst = reinterpret_cast<uint4 *>(out + c * 16);
        dst[0] = *reinterpret_cast<const uint4 *>(o);
        dst[1] = *reinterpret_cast<const uint4 *>(o + 8);
    }
}

}  // namespace

void launch_seed_features(const GridDev &g, int n, const int *tree_off, const int *tree_nodes, const float *cap0,
                          int file_layers, int *pins, long long *dh, long long *dv, __nv_bfloat16 *out,
                          cudaStream_t s) {
    const int X = g.X, Y = g.Y;
    const size_t XY = (size_t)X * Y, D = (size_t)(X + 1) * (Y + 1);
    cudaMemsetAsync(pins, 0, XY * sizeof(int), s);
    cudaMemsetAsync(dh, 0, D * sizeof(long long), s);
    cudaMemsetAsync(dv, 0, D * sizeof(long long), s);
    if (n > 0) feat_net_kernel<<<std::min((n + 255) / 256, 148 * 32), 256, 0, s>>>(n, tree_off, tree_nodes, g.L, X, Y,
                                                                                     pins, dh, dv);
    feat_scan_y_kernel<<<(X + 1 + 7) / 8, 256, 0, s>>>(X, Y, dh, dv);
    feat_scan_x_kernel<<<(Y + 1 + 255) / 256, 256, 0, s>>>(X, Y, dh, dv);
    feat_out_kernel<<<(int)std::min<size_t>((XY + 255) / 256, 148 * 32), 256, 0, s>>>(g, cap0, file_layers, pins, dh,
                                                                                          dv, out);
}

}  // namespace igr
