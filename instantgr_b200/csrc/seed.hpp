// Learned congestion seed: a small BF16 convolutional encoder-decoder that
// predicts per-layer routing demand from placement features, trained on the
// demand maps the plain router produces.  Device kernels in seed_nn.cu
// (tcgen05 implicit-GEMM convolutions, TMEM accumulators), host model in
// seed_model.cpp.  It has no counterpart in InstantGR.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace igr {

constexpr int kSeedIn = 16;    // 14 feature channels, padded
constexpr int kSeedOut = 16;   // 10 demand channels (file layers 0..9), padded
constexpr int kSeedFeat = 14;
constexpr int kSeedLayersOut = 10;
constexpr int kSeedTile = 256;  // predicted region per tile
constexpr int kSeedHalo = 16;
constexpr int kSeedS = kSeedTile + 2 * kSeedHalo;  // 288: tile with halo
constexpr int kSeedConvs = 6;

// one 3x3 convolution: mode 0 same size, 1 stride 2, 2 nearest upsample x2 then same
struct ConvSpec {
    int cin, cout, hin, win, hout, wout, mode, relu;
};

// Forward: Y[T][hout][wout][cout] = act(conv(X) + bias); Y32 (optional) gets f32 values.
void launch_conv_fwd(const ConvSpec &c, int T, const __nv_bfloat16 *X, const __nv_bfloat16 *W, const float *bias,
                     __nv_bfloat16 *Y, float *Y32, int *err, cudaStream_t s);
// Input gradient: dXpre[T][hin][win][cin] = (conv^T dY) * (Aprev > 0) (Aprev null: no mask);
// WT = weights as [cin][9][cout].
void launch_conv_dgrad(const ConvSpec &c, int T, const __nv_bfloat16 *dY, const __nv_bfloat16 *WT,
                       const __nv_bfloat16 *Aprev, __nv_bfloat16 *dXpre, int *err, cudaStream_t s);
// Weight gradient, accumulated: dWT[9*cin][cout] += sum over output pixels (f32 atomics).
void launch_conv_wgrad(const ConvSpec &c, int T, const __nv_bfloat16 *X, const __nv_bfloat16 *dY, float *dWT,
                       int *err, cudaStream_t s);
// Bias gradient: db[cout] += sum over pixels of dY.
void launch_bias_grad(const ConvSpec &c, int T, const __nv_bfloat16 *dY, float *db, cudaStream_t s);
// MSE loss over the central region [halo, S - halo)^2 of each S x S tile and the 10
// demand channels: dY = 2 (y - t) / count (bf16, zero elsewhere); sums[0] += sum of
// squared errors, sums[1] += sum of absolute errors (f64).
void launch_seed_loss(int T, int S, int halo, const float *y, const float *target, __nv_bfloat16 *dY, double *sums,
                      cudaStream_t s);
// Tiles from channels-last maps: out[t][i][j][c] = map_t[(x0_t - halo + i) * Y_t + (y0_t - halo + j)][c]
// (0 outside the map), for maps of bf16 (features) or bf16 -> f32 (targets).
struct TileRef {
    long long base;  // element offset of the map in the pool (cells x 16 channels)
    int X, Y, x0, y0;
};
void launch_gather_tiles(int T, int S, int halo, const TileRef *tiles, const __nv_bfloat16 *pool, __nv_bfloat16 *out16,
                         float *out32, cudaStream_t s);
// Writes the central (S - 2 halo)^2 region of each tile's output y32 into the
// channels-last prediction map pred [X][Y][16] (cells outside the map skipped).
void launch_scatter_prediction(int T, int S, int halo, const TileRef *tiles, const float *y32, float *pred,
                               cudaStream_t s);
// Seed demand of the routing layers in the reference layout [l][x][y]: alpha x the
// predicted demand of file layer l + 1 (pred in units of 8 GCell tracks), rounded
// to half units (exact in f32 and removable), clamped at 0.
// kind 1 seeds only the predicted overflow, alpha x max(0, predicted demand - capacity)
// (cap_ref: capacity of the routing layers, reference layout); kind 0 needs no cap_ref.
void launch_seed_demand(int X, int Y, int L, const float *pred, float alpha, int kind, const float *cap_ref,
                        float *out_ref, cudaStream_t s);
// Seed contribution at fraction `frac`: q = round_half(frac x base); demand += q - cur; cur = q
// (frac = 0 removes it); track layout, n cells.
void launch_seed_step(int64_t n, float *demand, const float *base, float *cur, float frac, cudaStream_t s);
// Predicted overflow per GCell: sum over routing layers of max(0, predicted demand - capacity);
// cap_ref is the capacity of the routing layers in the reference layout.
void launch_seed_overflow(int X, int Y, int L, const float *pred, const float *cap_ref, float *out, cudaStream_t s);
// demand[i] += sign * seed[i] over n cells
void launch_add_demand(int64_t n, float *demand, const float *seed, float sign, cudaStream_t s);
// Adam step over n parameters (f32 master, gradient, moments), bias-corrected.
void launch_adam(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t s);
// Working weights of a convolution from its master copy: W[cout][9][cin], WT[cin][9][cout] (bf16),
// and the gradient layout conversion dW[cout][9][cin] <- dWT[9*cin][cout].
void launch_seed_weights(int cin, int cout, const float *Wm, __nv_bfloat16 *W, __nv_bfloat16 *WT, cudaStream_t s);
void launch_seed_grad_layout(int cin, int cout, const float *dWT, float *dW, cudaStream_t s);
// The 16 input channels of a design ([X][Y][16] bf16, seed_feat.cu) from the
// resident trees of its n routing nets (positions l*X*Y + x*Y + y, Steiner
// points at layer g.L), the capacity of file layer 0 (cap0, [x][y]) and the
// grid's; pins ([X*Y]) and dh, dv ([(X+1)*(Y+1)]) are work arrays.
struct GridDev;
void launch_seed_features(const GridDev &g, int n, const int *tree_off, const int *tree_nodes, const float *cap0,
                          int file_layers, int *pins, long long *dh, long long *dv, __nv_bfloat16 *out,
                          cudaStream_t s);

}  // namespace igr
