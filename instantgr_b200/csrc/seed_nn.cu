// Convolutions of the learned congestion seed as implicit GEMMs on the
// tcgen05 tensor cores.
//
// One kernel template drives every GEMM: a CTA of 128 threads owns a
// 128 x BN tile of the result in TMEM (f32), fills two shared-memory stages
// of 128 x 64 (A) and BN x 64 (B) BF16 operands in the canonical K-major
// layout with ordinary loads (the operand policy gathers the convolution
// window, so no im2col buffer exists), and one thread issues four
// tcgen05.mma (K = 16 each) per stage and commits them to the stage's
// mbarrier; the next fill of a stage waits for that commit.  The epilogue
// reads TMEM with tcgen05.ld.  Every wait is bounded (ERR_TIMEOUT in the
// error word) and the TMEM columns are freed on every path.
//
// Policies: forward (rows = output pixels, cols = output channels, K = 3x3
// taps x input channels), input gradient (rows = input pixels, cols = input
// channels, K = taps x output channels, the ReLU mask of the previous layer
// applied in the epilogue) and weight gradient (rows = taps x input channels,
// cols = output channels, K = output pixels split over CTAs, f32 atomics).
// Activations are channels-last BF16; channel counts are powers of two >= 16.
#include "kcommon.cuh"
#include "seed.hpp"
#include "umma.cuh"
#include "hooks.hpp"

#include <algorithm>

namespace igr {

namespace {

constexpr int kBK = 64;                           // K per stage (four MMAs)
constexpr int kRowPasses = 128 * kBK / 8 / 128;   // 16-byte A chunks per thread and stage
constexpr unsigned long long kWaitNs = 2000000000ull;

template <int BN>
constexpr size_t stage_bytes() { return (size_t)4 * (128 + BN) * 16 * 2; }

__device__ __forceinline__ void put8(__nv_bfloat16 *stage, int r, int kk, uint4 v) {
    *reinterpret_cast<uint4 *>(stage + (kk >> 4) * (128 * 16) + umma::sub_idx(r, kk & 15)) = v;
}
__device__ __forceinline__ void put8b(__nv_bfloat16 *stage, int bn, int r, int kk, uint4 v) {
    *reinterpret_cast<uint4 *>(stage + (kk >> 4) * (bn * 16) + umma::sub_idx(r, kk & 15)) = v;
}
__device__ __forceinline__ void put1(__nv_bfloat16 *stage, int rows, int r, int kk, __nv_bfloat16 v) {
    stage[(kk >> 4) * (rows * 16) + umma::sub_idx(r, kk & 15)] = v;
}

__device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

// input position of output pixel (oy, ox) under tap (dy, dx); false outside
__device__ __forceinline__ bool in_pos(const ConvSpec &c, int oy, int ox, int dy, int dx, int &iy, int &ix) {
    if (c.mode == 1) {
        iy = 2 * oy + dy - 1;
        ix = 2 * ox + dx - 1;
    } else if (c.mode == 2) {
        const int uy = oy + dy - 1, ux = ox + dx - 1;
        if (uy < 0 || ux < 0 || uy >= c.hout || ux >= c.wout) return false;
        iy = uy >> 1;
        ix = ux >> 1;
        return true;
    } else {
        iy = oy + dy - 1;
        ix = ox + dx - 1;
    }
    return iy >= 0 && ix >= 0 && iy < c.hin && ix < c.win;
}

struct FwdOp {
    ConvSpec c;
    const __nv_bfloat16 *X, *W;
    const float *bias;
    __nv_bfloat16 *Y;
    float *Y32;
    int M, K;
    __device__ void load_a(__nv_bfloat16 *sa, int m0, int k0, int ke) const {
        const int tid = threadIdx.x, kc = tid & 7, k = k0 + kc * 8;
        const int lc = ilog2(c.cin);
        const int tap = k >> lc, ci = k & (c.cin - 1), dy = tap / 3, dx = tap - 3 * (tap / 3);
        const int hw = c.hout * c.wout;
        // every load of the stage in flight before the first store
        uint4 v[kRowPasses];
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) {
            const int m = m0 + (tid >> 3) + 16 * it;
            v[it] = make_uint4(0, 0, 0, 0);
            if (m < M && k < ke) {
                const int t = m / hw, rem = m - t * hw, oy = rem / c.wout, ox = rem - oy * c.wout;
                int iy, ix;
                if (in_pos(c, oy, ox, dy, dx, iy, ix))
                    v[it] = *reinterpret_cast<const uint4 *>(X + (((size_t)t * c.hin + iy) * c.win + ix) * c.cin + ci);
            }
        }
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) put8(sa, (tid >> 3) + 16 * it, kc * 8, v[it]);
    }
    template <int BN>
    __device__ void load_b(__nv_bfloat16 *sb, int n0, int k0, int ke) const {
        uint4 v[BN / 16];
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it, r = q >> 3, kc = q & 7, k = k0 + kc * 8, n = n0 + r;
            v[it] = make_uint4(0, 0, 0, 0);
            if (n < c.cout && k < ke) v[it] = *reinterpret_cast<const uint4 *>(W + (size_t)n * K + k);
        }
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it;
            put8b(sb, BN, q >> 3, (q & 7) * 8, v[it]);
        }
    }
    __device__ void store(int row, int n0, const float *v) const {
        if (row >= M || n0 >= c.cout) return;
        __align__(16) __nv_bfloat16 o[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            float x = v[j] + bias[n0 + j];
            if (c.relu) x = fmaxf(x, 0.f);
            o[j] = __float2bfloat16(x);
            if (Y32) Y32[(size_t)row * c.cout + n0 + j] = x;
        }
        *reinterpret_cast<uint4 *>(Y + (size_t)row * c.cout + n0) = *reinterpret_cast<const uint4 *>(o);
    }
};

struct DgradOp {
    ConvSpec c;
    const __nv_bfloat16 *dY, *WT, *Aprev;
    __nv_bfloat16 *dX;
    int M, K;
    __device__ void load_a(__nv_bfloat16 *sa, int m0, int k0, int ke) const {
        const int tid = threadIdx.x, kc = tid & 7, k = k0 + kc * 8;
        const int lc = ilog2(c.cout), per = 9 * c.cout;
        const int sub = k / per, rem = k - sub * per;
        const int tap = rem >> lc, co = rem & (c.cout - 1), dy = tap / 3, dx = tap - 3 * (tap / 3);
        const int hw = c.hin * c.win;
        uint4 v[kRowPasses];
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) {
            const int m = m0 + (tid >> 3) + 16 * it;
            v[it] = make_uint4(0, 0, 0, 0);
            if (m < M && k < ke) {
                const int t = m / hw, q = m - t * hw, iy = q / c.win, ix = q - iy * c.win;
                int oy, ox;
                bool ok;
                if (c.mode == 1) {
                    const int ny = iy + 1 - dy, nx = ix + 1 - dx;
                    ok = ny >= 0 && nx >= 0 && !(ny & 1) && !(nx & 1);
                    oy = ny >> 1;
                    ox = nx >> 1;
                } else if (c.mode == 2) {
                    oy = 2 * iy + (sub >> 1) + 1 - dy;
                    ox = 2 * ix + (sub & 1) + 1 - dx;
                    ok = true;
                } else {
                    oy = iy + 1 - dy;
                    ox = ix + 1 - dx;
                    ok = true;
                }
                ok = ok && oy >= 0 && ox >= 0 && oy < c.hout && ox < c.wout;
                if (ok)
                    v[it] = *reinterpret_cast<const uint4 *>(dY + (((size_t)t * c.hout + oy) * c.wout + ox) * c.cout + co);
            }
        }
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) put8(sa, (tid >> 3) + 16 * it, kc * 8, v[it]);
    }
    template <int BN>
    __device__ void load_b(__nv_bfloat16 *sb, int n0, int k0, int ke) const {
        const int per = 9 * c.cout;
        uint4 v[BN / 16];
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it, r = q >> 3, kc = q & 7, k = k0 + kc * 8, n = n0 + r;
            v[it] = make_uint4(0, 0, 0, 0);
            if (n < c.cin && k < ke) v[it] = *reinterpret_cast<const uint4 *>(WT + (size_t)n * per + (k % per));
        }
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it;
            put8b(sb, BN, q >> 3, (q & 7) * 8, v[it]);
        }
    }
    __device__ void store(int row, int n0, const float *v) const {
        if (row >= M || n0 >= c.cin) return;
        __align__(16) __nv_bfloat16 o[8];
        __align__(16) __nv_bfloat16 a[8];
        if (Aprev) *reinterpret_cast<uint4 *>(a) = *reinterpret_cast<const uint4 *>(Aprev + (size_t)row * c.cin + n0);
#pragma unroll
        for (int j = 0; j < 8; j++) o[j] = __float2bfloat16((!Aprev || __bfloat162float(a[j]) > 0.f) ? v[j] : 0.f);
        *reinterpret_cast<uint4 *>(dX + (size_t)row * c.cin + n0) = *reinterpret_cast<const uint4 *>(o);
    }
};

struct WgradOp {
    ConvSpec c;
    const __nv_bfloat16 *X, *dY;
    float *dWT;
    int M, K;  // M = 9 * cin, K = output pixels
    __device__ void load_a(__nv_bfloat16 *sa, int m0, int k0, int ke) const {
        const int lc = ilog2(c.cin), hw = c.hout * c.wout;
        uint4 v[kRowPasses];
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) {
            const int q = threadIdx.x + 128 * it, kk = q & 63, r = (q >> 6) * 8, k = k0 + kk, m = m0 + r;
            v[it] = make_uint4(0, 0, 0, 0);
            if (m < M && k < ke) {
                const int tap = m >> lc, ci = m & (c.cin - 1), dy = tap / 3, dx = tap - 3 * (tap / 3);
                const int t = k / hw, rem = k - t * hw, oy = rem / c.wout, ox = rem - oy * c.wout;
                int iy, ix;
                if (in_pos(c, oy, ox, dy, dx, iy, ix))
                    v[it] = *reinterpret_cast<const uint4 *>(X + (((size_t)t * c.hin + iy) * c.win + ix) * c.cin + ci);
            }
        }
#pragma unroll
        for (int it = 0; it < kRowPasses; it++) {
            const int q = threadIdx.x + 128 * it, kk = q & 63, r = (q >> 6) * 8;
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v[it]);
#pragma unroll
            for (int j = 0; j < 8; j++) put1(sa, 128, r + j, kk, e[j]);
        }
    }
    template <int BN>
    __device__ void load_b(__nv_bfloat16 *sb, int n0, int k0, int ke) const {
        uint4 v[BN / 16];
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it, kk = q & 63, r = (q >> 6) * 8, k = k0 + kk, n = n0 + r;
            v[it] = make_uint4(0, 0, 0, 0);
            if (n < c.cout && k < ke) v[it] = *reinterpret_cast<const uint4 *>(dY + (size_t)k * c.cout + n);
        }
#pragma unroll
        for (int it = 0; it < BN / 16; it++) {
            const int q = threadIdx.x + 128 * it, kk = q & 63, r = (q >> 6) * 8;
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v[it]);
#pragma unroll
            for (int j = 0; j < 8; j++) put1(sb, BN, r + j, kk, e[j]);
        }
    }
    __device__ void store(int row, int n0, const float *v) const {
        if (row >= M || n0 >= c.cout) return;
#pragma unroll
        for (int j = 0; j < 8; j++) atomicAdd(dWT + (size_t)row * c.cout + n0 + j, v[j]);
    }
};

template <int BN, class Op>
__global__ void __launch_bounds__(128) umma_gemm_kernel(Op op, int kchunk, int *err, unsigned long long wait_ns,
                                                         int probe) {
    constexpr int kCols = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __nv_bfloat16 *sA = reinterpret_cast<__nv_bfloat16 *>(smem_raw);   // [2][4][128 * 16]
    __nv_bfloat16 *sB = sA + 2 * 4 * 128 * 16;                            // [2][4][BN * 16]
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tbase;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
    const int kb0 = blockIdx.z * kchunk, ke = min(op.K, kb0 + kchunk);
    if (warp == 0) umma::tmem_alloc(&tbase, kCols);
    if (tid == 0) {
        umma::mbar_init(&bar[0]);
        umma::mbar_init(&bar[1]);
        umma::mbar_init_fence();
    }
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t tmem = tbase;
    const int nk = ke > kb0 ? (ke - kb0 + kBK - 1) / kBK : 0;
    constexpr uint32_t idesc = umma::idesc_bf16(128, BN);
    int issued = 0;
    bool ok = true;
    if (probe) {  // test hook: a wait on a phase that nothing completes, before any MMA is issued
        bool w = true;
        if (tid == 0) w = umma::mbar_wait(&bar[0], 0, wait_ns);
        ok = __syncthreads_and(w) != 0;
    }
    for (int kb = 0; kb < nk && ok; kb++) {
        const int s = kb & 1;
        bool w = true;
        if (kb >= 2 && tid == 0) w = umma::mbar_wait(&bar[s], ((kb - 2) >> 1) & 1, wait_ns);
        ok = __syncthreads_and(w) != 0;
        if (!ok) break;
        __nv_bfloat16 *a = sA + s * 4 * 128 * 16, *b = sB + s * 4 * BN * 16;
        op.load_a(a, m0, kb0 + kb * kBK, ke);
        op.template load_b<BN>(b, n0, kb0 + kb * kBK, ke);
        umma::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            umma::fence_after();
#pragma unroll
            for (int j = 0; j < 4; j++)
                umma::mma_bf16(tmem, umma::smem_desc(umma::smem_u32(a + j * 128 * 16)),
                               umma::smem_desc(umma::smem_u32(b + j * BN * 16)), idesc, kb > 0 || j > 0);
            umma::mma_commit(&bar[s]);
        }
        issued = kb + 1;
    }
    // every issued MMA has completed once the last commit of each stage has
    bool drained = true;
    if (tid == 0)
        for (int s = 0; s < 2; s++)
            if (issued > s) {
                const int last = ((issued - 1 - s) / 2) * 2 + s;
                drained = umma::mbar_wait(&bar[s], (last >> 1) & 1, kWaitNs) && drained;
            }
    const bool good = __syncthreads_and(ok && drained) != 0;
    umma::fence_after();
    if (good && issued > 0) {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 8) {
            float v[8];
            umma::tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
            op.store(row, n0 + c0, v);
        }
    } else if (!good && tid == 0) {
        set_error(err, ERR_TIMEOUT);
    }
    umma::fence_before();
    __syncthreads();
    if (warp == 0) umma::tmem_free(tmem, kCols);
}

template <int BN, class Op>
void launch_gemm(const Op &op, int N, int kchunk, int *err, cudaStream_t s) {
    const size_t smem = 2 * stage_bytes<BN>();
    kernel_setup((const void *)umma_gemm_kernel<BN, Op>, 128, smem);
    if (kchunk <= 0) kchunk = op.K;
    dim3 grid((op.M + 127) / 128, (N + BN - 1) / BN, (op.K + kchunk - 1) / kchunk);
    umma_gemm_kernel<BN, Op><<<grid, 128, smem, s>>>(op, kchunk, err,
                                                      (unsigned long long)test_hooks().wait_ns.load(),
                                                      test_hooks().mbar_probe.load());
}

template <class Op>
void launch_by_n(const Op &op, int N, int kchunk, int *err, cudaStream_t s) {
    if (N <= 16) launch_gemm<16>(op, N, kchunk, err, s);
    else if (N <= 32) launch_gemm<32>(op, N, kchunk, err, s);
    else launch_gemm<64>(op, N, kchunk, err, s);
}

__global__ void bias_grad_kernel(int P, int cout, const __nv_bfloat16 *dY, float *db) {
    const int co = blockIdx.x;
    float s = 0;
    for (int p = threadIdx.x + blockIdx.y * blockDim.x; p < P; p += blockDim.x * gridDim.y)
        s += __bfloat162float(dY[(size_t)p * cout + co]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float w[8];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += w[i];
        atomicAdd(db + co, t);
    }
}

__global__ void seed_loss_kernel(int T, int S, int halo, const float *y, const float *tg, __nv_bfloat16 *dY,
                                 double *sums, double scale) {
    const long long n = (long long)T * S * S * kSeedOut;
    double se = 0, ae = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % kSeedOut);
        const long long p = i / kSeedOut;
        const int x = (int)(p % S), yy = (int)((p / S) % S);
        float g = 0;
        if (ch < kSeedLayersOut && x >= halo && x < S - halo && yy >= halo && yy < S - halo) {
            const float e = y[i] - tg[i];
            se += (double)e * e;
            ae += fabs((double)e);
            g = (float)(2.0 * e * scale);
        }
        dY[i] = __float2bfloat16(g);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        se += __shfl_down_sync(0xffffffffu, se, o);
        ae += __shfl_down_sync(0xffffffffu, ae, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(sums, se);
        atomicAdd(sums + 1, ae);
    }
}

__global__ void gather_tiles_kernel(int T, int S, int halo, const TileRef *tiles, const __nv_bfloat16 *pool,
                                    __nv_bfloat16 *out16, float *out32) {
    // one thread per (tile, pixel, 8-channel half)
    const long long n = (long long)T * S * S * 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(q & 1);
        const long long p = q >> 1;
        const int t = (int)(p / ((long long)S * S)), r = (int)(p % ((long long)S * S)), i = r / S, j = r % S;
        const TileRef tr = tiles[t];
        const int x = tr.x0 - halo + i, y = tr.y0 - halo + j;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (x >= 0 && y >= 0 && x < tr.X && y < tr.Y)
            v = *reinterpret_cast<const uint4 *>(pool + tr.base + ((long long)x * tr.Y + y) * kSeedIn + h * 8);
        if (out16) *reinterpret_cast<uint4 *>(out16 + p * kSeedIn + h * 8) = v;
        if (out32) {
            const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
            for (int c = 0; c < 8; c++) out32[p * kSeedIn + h * 8 + c] = __bfloat162float(e[c]);
        }
    }
}

__global__ void scatter_prediction_kernel(int T, int S, int halo, const TileRef *tiles, const float *y32, float *pred) {
    const int in = S - 2 * halo;
    const long long n = (long long)T * in * in * 4;  // (tile, cell, 4-channel quarter)
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int part = (int)(q & 3);
        const long long p = q >> 2;
        const int t = (int)(p / ((long long)in * in)), r = (int)(p % ((long long)in * in)), i = r / in, j = r % in;
        const TileRef tr = tiles[t];
        const int x = tr.x0 + i, y = tr.y0 + j;
        if (x >= tr.X || y >= tr.Y) continue;
        const float *src = y32 + (((long long)t * S + i + halo) * S + j + halo) * kSeedOut + part * 4;
        *reinterpret_cast<float4 *>(pred + ((long long)x * tr.Y + y) * kSeedOut + part * 4) =
            *reinterpret_cast<const float4 *>(src);
    }
}

__global__ void seed_demand_kernel(int X, int Y, int L, const float *pred, float alpha, int kind, const float *cap,
                                   float *out) {
    const long long n = (long long)L * X * Y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i / ((long long)X * Y));
        const long long c = i - (long long)l * X * Y;
        float v = 8.f * pred[c * kSeedOut + 1 + l];
        if (kind == 1) v -= cap[i];
        out[i] = v > 0.f ? alpha * v : 0.f;
    }
}

__global__ void seed_step_kernel(long long n, float *d, const float *base, float *cur, float frac) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float q = 0.5f * rintf(2.f * frac * base[i]);
        const float c = cur[i];
        if (q != c) {
            d[i] += q - c;
            cur[i] = q;
        }
    }
}

__global__ void seed_overflow_kernel(int X, int Y, int L, const float *pred, const float *cap, float *out) {
    const long long n = (long long)X * Y;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        float o = 0;
        for (int l = 0; l < L; l++) o += fmaxf(0.f, 8.f * pred[c * kSeedOut + 1 + l] - cap[(long long)l * n + c]);
        out[c] = o;
    }
}

__global__ void add_demand_kernel(long long n, float *d, const float *seed, float sign) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] += sign * seed[i];
}

__global__ void adam_kernel(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void seed_weights_kernel(int cin, int cout, const float *Wm, __nv_bfloat16 *W, __nv_bfloat16 *WT) {
    const int n = cout * 9 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int co = i / (9 * cin), r = i - co * 9 * cin, tap = r / cin, ci = r - tap * cin;
        const __nv_bfloat16 b = __float2bfloat16(Wm[i]);
        W[i] = b;
        WT[((size_t)ci * 9 + tap) * cout + co] = b;
    }
}

__global__ void seed_grad_layout_kernel(int cin, int cout, const float *dWT, float *dW) {
    const int n = cout * 9 * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int co = i / (9 * cin), r = i - co * 9 * cin;  // r = tap * cin + ci
        dW[i] = dWT[(size_t)r * cout + co];
    }
}

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>(148 * 8, (n + 255) / 256)); }

}  // namespace

void launch_conv_fwd(const ConvSpec &c, int T, const __nv_bfloat16 *X, const __nv_bfloat16 *W, const float *bias,
                     __nv_bfloat16 *Y, float *Y32, int *err, cudaStream_t s) {
    FwdOp op{c, X, W, bias, Y, Y32, T * c.hout * c.wout, 9 * c.cin};
    launch_by_n(op, c.cout, 0, err, s);
}

void launch_conv_dgrad(const ConvSpec &c, int T, const __nv_bfloat16 *dY, const __nv_bfloat16 *WT,
                       const __nv_bfloat16 *Aprev, __nv_bfloat16 *dXpre, int *err, cudaStream_t s) {
    DgradOp op{c, dY, WT, Aprev, dXpre, T * c.hin * c.win, (c.mode == 2 ? 4 : 1) * 9 * c.cout};
    launch_by_n(op, c.cin, 0, err, s);
}

void launch_conv_wgrad(const ConvSpec &c, int T, const __nv_bfloat16 *X, const __nv_bfloat16 *dY, float *dWT,
                       int *err, cudaStream_t s) {
    WgradOp op{c, X, dY, dWT, 9 * c.cin, T * c.hout * c.wout};
    // split the pixel reduction so that the grid covers the GPU (~2 CTAs per SM)
    const int mt = (op.M + 127) / 128, nt = (c.cout + 63) / 64;
    int splits = std::max(1, 296 / std::max(1, mt * nt));
    int kchunk = (op.K + splits - 1) / splits;
    kchunk = ((kchunk + kBK - 1) / kBK) * kBK;
    launch_by_n(op, c.cout, kchunk, err, s);
}

void launch_bias_grad(const ConvSpec &c, int T, const __nv_bfloat16 *dY, float *db, cudaStream_t s) {
    const int P = T * c.hout * c.wout;
    bias_grad_kernel<<<dim3(c.cout, 16), 256, 0, s>>>(P, c.cout, dY, db);
}

void launch_seed_loss(int T, int S, int halo, const float *y, const float *target, __nv_bfloat16 *dY, double *sums,
                      cudaStream_t s) {
    const long long n = (long long)T * S * S * kSeedOut;
    const double count = (double)T * (S - 2 * halo) * (S - 2 * halo) * kSeedLayersOut;
    seed_loss_kernel<<<blocks_for(n), 256, 0, s>>>(T, S, halo, y, target, dY, sums, 1.0 / count);
}

void launch_gather_tiles(int T, int S, int halo, const TileRef *tiles, const __nv_bfloat16 *pool, __nv_bfloat16 *out16,
                         float *out32, cudaStream_t s) {
    gather_tiles_kernel<<<blocks_for((long long)T * S * S * 2), 256, 0, s>>>(T, S, halo, tiles, pool, out16, out32);
}

void launch_scatter_prediction(int T, int S, int halo, const TileRef *tiles, const float *y32, float *pred,
                               cudaStream_t s) {
    const int in = S - 2 * halo;
    scatter_prediction_kernel<<<blocks_for((long long)T * in * in * 4), 256, 0, s>>>(T, S, halo, tiles, y32, pred);
}

void launch_seed_demand(int X, int Y, int L, const float *pred, float alpha, int kind, const float *cap_ref,
                        float *out_ref, cudaStream_t s) {
    seed_demand_kernel<<<blocks_for((long long)L * X * Y), 256, 0, s>>>(X, Y, L, pred, alpha, kind, cap_ref, out_ref);
}

void launch_seed_step(int64_t n, float *demand, const float *base, float *cur, float frac, cudaStream_t s) {
    seed_step_kernel<<<blocks_for(n), 256, 0, s>>>(n, demand, base, cur, frac);
}

void launch_seed_overflow(int X, int Y, int L, const float *pred, const float *cap_ref, float *out, cudaStream_t s) {
    seed_overflow_kernel<<<blocks_for((long long)X * Y), 256, 0, s>>>(X, Y, L, pred, cap_ref, out);
}

void launch_add_demand(int64_t n, float *demand, const float *seed, float sign, cudaStream_t s) {
    add_demand_kernel<<<blocks_for(n), 256, 0, s>>>(n, demand, seed, sign);
}

void launch_adam(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t s) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    adam_kernel<<<blocks_for(n), 256, 0, s>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
}

void launch_seed_weights(int cin, int cout, const float *Wm, __nv_bfloat16 *W, __nv_bfloat16 *WT, cudaStream_t s) {
    seed_weights_kernel<<<blocks_for((long long)cout * 9 * cin), 256, 0, s>>>(cin, cout, Wm, W, WT);
}

void launch_seed_grad_layout(int cin, int cout, const float *dWT, float *dW, cudaStream_t s) {
    seed_grad_layout_kernel<<<blocks_for((long long)cout * 9 * cin), 256, 0, s>>>(cin, cout, dWT, dW);
}

}  // namespace igr
