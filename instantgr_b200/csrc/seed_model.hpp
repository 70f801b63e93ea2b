// Learned congestion seed: model state and host driver (seed_model.cpp).
#pragma once
#include "router.hpp"
#include "seed.hpp"

namespace igr {

struct SeedModel {
    int S = 0, halo = 0;
    ConvSpec spec[kSeedConvs] = {};
    cudaStream_t s = nullptr;
    // parameters: f32 master weights [cout][9][cin], biases, Adam moments,
    // gradients, and the BF16 working copies W and WT ([cin][9][cout])
    DevBuf<float> Wm[kSeedConvs], bias[kSeedConvs], mW[kSeedConvs], vW[kSeedConvs], dW[kSeedConvs],
        dWT[kSeedConvs], mb[kSeedConvs], vb[kSeedConvs], db[kSeedConvs];
    DevBuf<__nv_bfloat16> W[kSeedConvs], WT[kSeedConvs];
    int adam_t = 0;
    // activations of up to Tcap tiles: input, outputs of c1..c5, gradients of
    // the pre-activations of c1..c6, output (bf16 and f32) and target
    int Tcap = 0;
    DevBuf<__nv_bfloat16> x0, act[kSeedConvs - 1], grad[kSeedConvs], y16;
    DevBuf<float> y32, tgt32;
    DevBuf<double> sums;
    DevBuf<int> err;
    DevBuf<TileRef> tiles;
    // training maps (features and targets, [cells][16] bf16) kept on the device
    DevBuf<__nv_bfloat16> fpool, tpool;
    size_t pool_used = 0;
    std::vector<TileRef> maps;

    ~SeedModel();
    void set_tile(int S, int halo);   // tile size with halo (even), halo
    void init(uint64_t seed);         // He-normal weights, zero biases
    int params() const;               // weights then bias of each layer
    void get_params(std::vector<float> &out);
    void set_params(const float *p, size_t n);
    void ensure(int T);
    void forward(int T);              // x0 -> y32
    // device time of `reps` forward passes over T tiles, per convolution
    // (ms per pass, CUDA events on the model's stream) and its multiply-add
    // FLOPs per pass (2 x output pixels x 9 x cin x cout)
    void time_forward(int T, int reps, double *layer_ms, double *layer_flops);
    double backward(int T, double *mae);  // loss of y32 vs tgt32 and every gradient
    void adam(float lr);
    void grads(std::vector<float> &out);  // dW (as [cout][9][cin]) and db of each layer
    int add_map(int X, int Y, const __nv_bfloat16 *feat, const __nv_bfloat16 *target);  // host maps
    // Adam steps on random tiles of training maps [0, nmaps) (0: every map)
    double train(int steps, int T, float lr, uint64_t seed, std::vector<double> *curve, int nmaps = 0);
    // predicted channels-last map [X][Y][16] (f32) of a feature map on the device
    void predict(int X, int Y, const __nv_bfloat16 *feat_dev, float *pred_dev);
    // errors of a stored map's prediction: out[0] MSE, [1] MAE, [2] MAE of predicting 0,
    // [3] MAE of predicting each layer's mean demand over the map
    void evaluate(int map, double *out);
    void check(const char *what);

   private:
    void set_layer(int i, const float *w, const float *b);
};

// 16-channel features of a design, [X][Y][16]: pins, RUDY-H, RUDY-V, blocked
// routing-layer fraction, capacity of file layers 0..9 (scaled), 0, 0
void seed_features(const Design &d, const NetSet &ns, std::vector<__nv_bfloat16> &out);
// training target [X][Y][16] from the routed demand of the routing layers ([l][x][y])
void seed_targets(int X, int Y, int routing_layers, const float *demand_ref, std::vector<__nv_bfloat16> &out);

}  // namespace igr
