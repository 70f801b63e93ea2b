// Host side of the learned congestion seed: parameters and Adam state, the
// forward and backward schedule of the six convolutions, the training set
// kept in device memory, tiled inference over a whole grid, and the input
// features of a design.  It has no counterpart in InstantGR.
//
// Network (per tile of S x S GCells, S = 256 + 2 x 16 halo, channels-last BF16):
//   c1 3x3 16->32 ReLU | c2 3x3 stride 2 32->64 ReLU | c3, c4 3x3 64->64 ReLU |
//   c5 nearest x2 + 3x3 64->32 ReLU | c6 3x3 32->16 (channels 0..9 = predicted
//   demand of file layers 0..9, the rest unused).
// The loss is the mean squared error over the central 256 x 256 GCells of
// each tile and the 10 demand channels.
#include "seed_model.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace igr {

namespace {

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uni01(uint64_t &s) { return (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }
double normal(uint64_t &s) {
    const double u = std::max(uni01(s), 1e-300), v = uni01(s);
    return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * v);
}

const int kCin[kSeedConvs] = {16, 32, 64, 64, 64, 32};
const int kCout[kSeedConvs] = {32, 64, 64, 64, 32, 16};

}  // namespace

void SeedModel::set_tile(int S_, int halo_) {
    if (S_ < 8 || (S_ & 1) || halo_ < 0 || 2 * halo_ >= S_) throw Error(ERR_INVALID, "bad seed tile size");
    S = S_;
    halo = halo_;
    const int h = S / 2;
    spec[0] = {16, 32, S, S, S, S, 0, 1};
    spec[1] = {32, 64, S, S, h, h, 1, 1};
    spec[2] = {64, 64, h, h, h, h, 0, 1};
    spec[3] = {64, 64, h, h, h, h, 0, 1};
    spec[4] = {64, 32, h, h, S, S, 2, 1};
    spec[5] = {32, 16, S, S, S, S, 0, 0};
    Tcap = 0;
}

void SeedModel::init(uint64_t seed) {
    if (!s) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    if (spec[0].cin == 0) set_tile(kSeedS, kSeedHalo);
    uint64_t r = seed * 0x2545F4914F6CDD1Dull + 17;
    std::vector<float> w;
    for (int i = 0; i < kSeedConvs; i++) {
        const int n = kCout[i] * 9 * kCin[i];
        w.assign(n, 0.f);
        const double sd = std::sqrt(2.0 / (9.0 * (i == 0 ? kSeedFeat : kCin[i]))) * (i == kSeedConvs - 1 ? 0.1 : 1.0);
        for (int co = 0; co < kCout[i]; co++)
            for (int k = 0; k < 9 * kCin[i]; k++) {
                const int ci = k % kCin[i];
                const bool used = (i > 0 || ci < kSeedFeat) && (i < kSeedConvs - 1 || co < kSeedLayersOut);
                w[(size_t)co * 9 * kCin[i] + k] = used ? (float)(normal(r) * sd) : 0.f;
            }
        std::vector<float> z(kCout[i], 0.f);
        set_layer(i, w.data(), z.data());
    }
    adam_t = 0;
}

void SeedModel::set_layer(int i, const float *w, const float *b) {
    const int n = kCout[i] * 9 * kCin[i];
    Wm[i].upload(w, n, s);
    bias[i].upload(b, kCout[i], s);
    W[i].alloc(n);
    WT[i].alloc(n);
    for (auto *buf : {&mW[i], &vW[i], &dW[i], &dWT[i]}) {
        buf->alloc(n);
        cuda_check(cudaMemsetAsync(buf->p, 0, n * sizeof(float), s), "memset");
    }
    for (auto *buf : {&mb[i], &vb[i], &db[i]}) {
        buf->alloc(kCout[i]);
        cuda_check(cudaMemsetAsync(buf->p, 0, kCout[i] * sizeof(float), s), "memset");
    }
    launch_seed_weights(kCin[i], kCout[i], Wm[i].p, W[i].p, WT[i].p, s);
    cuda_check(cudaStreamSynchronize(s), "seed weights");
}

int SeedModel::params() const {
    int n = 0;
    for (int i = 0; i < kSeedConvs; i++) n += kCout[i] * 9 * kCin[i] + kCout[i];
    return n;
}

void SeedModel::get_params(std::vector<float> &out) {
    out.clear();
    for (int i = 0; i < kSeedConvs; i++) {
        const int n = kCout[i] * 9 * kCin[i];
        std::vector<float> w(n), b(kCout[i]);
        cuda_check(cudaMemcpyAsync(w.data(), Wm[i].p, n * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(b.data(), bias[i].p, kCout[i] * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "params");
        out.insert(out.end(), w.begin(), w.end());
        out.insert(out.end(), b.begin(), b.end());
    }
}

void SeedModel::set_params(const float *p, size_t n) {
    if ((int)n != params()) throw Error(ERR_FORMAT, "seed parameter count mismatch");
    if (!s) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    if (spec[0].cin == 0) set_tile(kSeedS, kSeedHalo);
    size_t o = 0;
    for (int i = 0; i < kSeedConvs; i++) {
        const int nw = kCout[i] * 9 * kCin[i];
        set_layer(i, p + o, p + o + nw);
        o += nw + kCout[i];
    }
    adam_t = 0;
}

void SeedModel::ensure(int T) {
    if (T <= Tcap) return;
    const size_t SS = (size_t)S * S, hh = (size_t)(S / 2) * (S / 2);
    x0.alloc(T * SS * 16);
    act[0].alloc(T * SS * 32);
    act[1].alloc(T * hh * 64);
    act[2].alloc(T * hh * 64);
    act[3].alloc(T * hh * 64);
    act[4].alloc(T * SS * 32);
    y16.alloc(T * SS * 16);
    y32.alloc(T * SS * 16);
    tgt32.alloc(T * SS * 16);
    grad[5].alloc(T * SS * 16);
    grad[4].alloc(T * SS * 32);
    grad[3].alloc(T * hh * 64);
    grad[2].alloc(T * hh * 64);
    grad[1].alloc(T * hh * 64);
    grad[0].alloc(T * SS * 32);
    tiles.alloc(T);
    sums.alloc(2);
    err.alloc(1);
    cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
    Tcap = T;
}

void SeedModel::check(const char *what) {
    cuda_check(cudaGetLastError(), what);
    int e = 0;
    cuda_check(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), what);
    if (e) {
        cuda_check(cudaMemsetAsync(err.p, 0, sizeof(int), s), "memset");
        throw Error(e, std::string("device error in the congestion seed: ") + what);
    }
}

void SeedModel::forward(int T) {
    const __nv_bfloat16 *in = x0.p;
    for (int i = 0; i < kSeedConvs; i++) {
        const bool last = i == kSeedConvs - 1;
        launch_conv_fwd(spec[i], T, in, W[i].p, bias[i].p, last ? y16.p : act[i].p, last ? y32.p : nullptr, err.p, s);
        if (!last) in = act[i].p;
    }
}

void SeedModel::time_forward(int T, int reps, double *layer_ms, double *layer_flops) {
    if (T < 1 || reps < 1) throw Error(ERR_INVALID, "tiles and repetitions must be positive");
    ensure(T);
    cudaEvent_t ev[kSeedConvs + 1];
    for (auto &e : ev) cuda_check(cudaEventCreate(&e), "event");
    double ms[kSeedConvs] = {0};
    for (int r = 0; r < reps; r++) {
        const __nv_bfloat16 *in = x0.p;
        cuda_check(cudaEventRecord(ev[0], s), "event");
        for (int i = 0; i < kSeedConvs; i++) {
            const bool last = i == kSeedConvs - 1;
            launch_conv_fwd(spec[i], T, in, W[i].p, bias[i].p, last ? y16.p : act[i].p, last ? y32.p : nullptr,
                            err.p, s);
            if (!last) in = act[i].p;
            cuda_check(cudaEventRecord(ev[i + 1], s), "event");
        }
        cuda_check(cudaEventSynchronize(ev[kSeedConvs]), "sync");
        for (int i = 0; i < kSeedConvs; i++) {
            float t = 0;
            cuda_check(cudaEventElapsedTime(&t, ev[i], ev[i + 1]), "event time");
            ms[i] += t;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    check("timed forward");
    for (int i = 0; i < kSeedConvs; i++) {
        layer_ms[i] = ms[i] / reps;
        layer_flops[i] = 2.0 * T * spec[i].hout * spec[i].wout * 9.0 * spec[i].cin * spec[i].cout;
    }
}

double SeedModel::backward(int T, double *mae) {
    cuda_check(cudaMemsetAsync(sums.p, 0, 2 * sizeof(double), s), "memset");
    launch_seed_loss(T, S, halo, y32.p, tgt32.p, grad[5].p, sums.p, s);
    for (int i = 0; i < kSeedConvs; i++) {
        const int n = kCout[i] * 9 * kCin[i];
        cuda_check(cudaMemsetAsync(dWT[i].p, 0, n * sizeof(float), s), "memset");
        cuda_check(cudaMemsetAsync(db[i].p, 0, kCout[i] * sizeof(float), s), "memset");
    }
    for (int i = kSeedConvs - 1; i >= 0; i--) {
        const __nv_bfloat16 *X = i == 0 ? x0.p : act[i - 1].p;
        launch_conv_wgrad(spec[i], T, X, grad[i].p, dWT[i].p, err.p, s);
        launch_bias_grad(spec[i], T, grad[i].p, db[i].p, s);
        if (i > 0) launch_conv_dgrad(spec[i], T, grad[i].p, WT[i].p, act[i - 1].p, grad[i - 1].p, err.p, s);
    }
    for (int i = 0; i < kSeedConvs; i++) launch_seed_grad_layout(kCin[i], kCout[i], dWT[i].p, dW[i].p, s);
    double h[2] = {0, 0};
    cuda_check(cudaMemcpyAsync(h, sums.p, sizeof h, cudaMemcpyDeviceToHost, s), "D2H");
    check("backward");
    const double count = (double)T * (S - 2 * halo) * (S - 2 * halo) * kSeedLayersOut;
    if (mae) *mae = h[1] / count;
    return h[0] / count;
}

void SeedModel::adam(float lr) {
    adam_t++;
    for (int i = 0; i < kSeedConvs; i++) {
        const int n = kCout[i] * 9 * kCin[i];
        launch_adam(n, Wm[i].p, dW[i].p, mW[i].p, vW[i].p, lr, 0.9f, 0.999f, 1e-8f, adam_t, s);
        launch_adam(kCout[i], bias[i].p, db[i].p, mb[i].p, vb[i].p, lr, 0.9f, 0.999f, 1e-8f, adam_t, s);
        launch_seed_weights(kCin[i], kCout[i], Wm[i].p, W[i].p, WT[i].p, s);
    }
}

void SeedModel::grads(std::vector<float> &out) {
    out.clear();
    for (int i = 0; i < kSeedConvs; i++) {
        const int n = kCout[i] * 9 * kCin[i];
        std::vector<float> w(n), b(kCout[i]);
        cuda_check(cudaMemcpyAsync(w.data(), dW[i].p, n * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaMemcpyAsync(b.data(), db[i].p, kCout[i] * 4, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "grads");
        out.insert(out.end(), w.begin(), w.end());
        out.insert(out.end(), b.begin(), b.end());
    }
}

// ---------------------------------------------------------------- data
int SeedModel::add_map(int X, int Y, const __nv_bfloat16 *feat, const __nv_bfloat16 *target) {
    const size_t cells = (size_t)X * Y * 16;
    const size_t need = pool_used + cells;
    if (need > fpool.n) {  // grow both pools, keeping what they hold
        const size_t cap = std::max(need, fpool.n * 3 / 2 + cells);
        DevBuf<__nv_bfloat16> nf, nt;
        nf.alloc(cap);
        nt.alloc(cap);
        if (pool_used) {
            cuda_check(cudaMemcpyAsync(nf.p, fpool.p, pool_used * 2, cudaMemcpyDeviceToDevice, s), "D2D");
            cuda_check(cudaMemcpyAsync(nt.p, tpool.p, pool_used * 2, cudaMemcpyDeviceToDevice, s), "D2D");
        }
        cuda_check(cudaStreamSynchronize(s), "pool");
        std::swap(fpool.p, nf.p);
        std::swap(fpool.n, nf.n);
        std::swap(tpool.p, nt.p);
        std::swap(tpool.n, nt.n);
    }
    cuda_check(cudaMemcpyAsync(fpool.p + pool_used, feat, cells * 2, cudaMemcpyHostToDevice, s), "H2D");
    cuda_check(cudaMemcpyAsync(tpool.p + pool_used, target, cells * 2, cudaMemcpyHostToDevice, s), "H2D");
    cuda_check(cudaStreamSynchronize(s), "pool");
    maps.push_back({(long long)pool_used, X, Y, 0, 0});
    pool_used = need;
    return (int)maps.size() - 1;
}

double SeedModel::train(int steps, int T, float lr, uint64_t seed, std::vector<double> *curve, int nmaps) {
    if (maps.empty()) throw Error(ERR_STATE, "no training maps");
    const size_t nm = nmaps > 0 ? std::min<size_t>((size_t)nmaps, maps.size()) : maps.size();
    ensure(T);
    uint64_t r = seed * 0x9E3779B97F4A7C15ull + 3;
    const int inner = S - 2 * halo;
    double last = 0;
    std::vector<TileRef> tr(T);
    for (int st = 0; st < steps; st++) {
        for (int t = 0; t < T; t++) {
            const TileRef &m = maps[splitmix(r) % nm];
            tr[t] = m;
            tr[t].x0 = m.X > inner ? (int)(splitmix(r) % (uint64_t)(m.X - inner + 1)) : 0;
            tr[t].y0 = m.Y > inner ? (int)(splitmix(r) % (uint64_t)(m.Y - inner + 1)) : 0;
        }
        cuda_check(cudaMemcpyAsync(tiles.p, tr.data(), T * sizeof(TileRef), cudaMemcpyHostToDevice, s), "H2D");
        launch_gather_tiles(T, S, halo, tiles.p, fpool.p, x0.p, nullptr, s);
        launch_gather_tiles(T, S, halo, tiles.p, tpool.p, nullptr, tgt32.p, s);
        forward(T);
        last = backward(T, nullptr);
        adam(lr);
        if (curve) curve->push_back(last);
    }
    check("train");
    return last;
}

void SeedModel::predict(int X, int Y, const __nv_bfloat16 *feat_dev, float *pred_dev) {
    const int inner = S - 2 * halo;
    const int tx = (X + inner - 1) / inner, ty = (Y + inner - 1) / inner;
    const int nt = tx * ty;
    const int T = std::min(nt, 16);
    ensure(T);
    std::vector<TileRef> tr;
    for (int a = 0; a < tx; a++)
        for (int b = 0; b < ty; b++) tr.push_back({0, X, Y, a * inner, b * inner});
    for (int t0 = 0; t0 < nt; t0 += T) {
        const int n = std::min(T, nt - t0);
        cuda_check(cudaMemcpyAsync(tiles.p, tr.data() + t0, n * sizeof(TileRef), cudaMemcpyHostToDevice, s), "H2D");
        launch_gather_tiles(n, S, halo, tiles.p, feat_dev, x0.p, nullptr, s);
        forward(n);
        launch_scatter_prediction(n, S, halo, tiles.p, y32.p, pred_dev, s);
    }
    check("predict");
}

void SeedModel::evaluate(int map, double *out) {
    const TileRef &m = maps.at(map);
    DevBuf<float> pred;
    pred.alloc((size_t)m.X * m.Y * 16);
    predict(m.X, m.Y, fpool.p + m.base, pred.p);
    std::vector<float> p((size_t)m.X * m.Y * 16);
    std::vector<__nv_bfloat16> t(p.size());
    cuda_check(cudaMemcpyAsync(p.data(), pred.p, p.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaMemcpyAsync(t.data(), tpool.p + m.base, t.size() * 2, cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "evaluate");
    const size_t cells = (size_t)m.X * m.Y;
    double mean[kSeedLayersOut] = {0};
    for (size_t c = 0; c < cells; c++)
        for (int ch = 0; ch < kSeedLayersOut; ch++) mean[ch] += __bfloat162float(t[c * 16 + ch]);
    for (int ch = 0; ch < kSeedLayersOut; ch++) mean[ch] /= (double)cells;
    double se = 0, ae = 0, az = 0, am = 0;
    for (size_t c = 0; c < cells; c++)
        for (int ch = 0; ch < kSeedLayersOut; ch++) {
            const double tv = __bfloat162float(t[c * 16 + ch]);
            const double e = p[c * 16 + ch] - tv;
            se += e * e;
            ae += std::fabs(e);
            az += std::fabs(tv);
            am += std::fabs(tv - mean[ch]);
        }
    const double cnt = (double)cells * kSeedLayersOut;
    out[0] = se / cnt;
    out[1] = ae / cnt;
    out[2] = az / cnt;
    out[3] = am / cnt;
}

SeedModel::~SeedModel() {
    if (s) cudaStreamDestroy(s);
}

// ---------------------------------------------------------------- features
void seed_features(const Design &d, const NetSet &ns, std::vector<__nv_bfloat16> &out) {
    const int X = d.X, Y = d.Y, L = d.L;
    const size_t XY = (size_t)X * Y;
    // pins per GCell, and RUDY: a net spreads w/(w h) of horizontal and h/(w h)
    // of vertical wire density over its bounding box (2-D difference arrays)
    std::vector<float> pins(XY, 0.f);
    std::vector<double> dh((X + 1) * (size_t)(Y + 1), 0.0), dv(dh.size(), 0.0);
    auto at = [&](int x, int y) { return (size_t)x * (Y + 1) + y; };
    for (const RNet &n : ns.nets) {
        for (int p : n.pins) pins[(size_t)(p % (int)XY)] += 0.25f;
        const double vh = 1.0 / (n.maxy - n.miny + 1), vv = 1.0 / (n.maxx - n.minx + 1);
        dh[at(n.minx, n.miny)] += vh;
        dh[at(n.maxx + 1, n.miny)] -= vh;
        dh[at(n.minx, n.maxy + 1)] -= vh;
        dh[at(n.maxx + 1, n.maxy + 1)] += vh;
        dv[at(n.minx, n.miny)] += vv;
        dv[at(n.maxx + 1, n.miny)] -= vv;
        dv[at(n.minx, n.maxy + 1)] -= vv;
        dv[at(n.maxx + 1, n.maxy + 1)] += vv;
    }
    // prefix sums: along y per row (parallel over x), then along x per column (parallel over y)
    parallel_for(X + 1, 0, [&](int b, int e) {
        for (int x = b; x < e; x++)
            for (int y = 1; y <= Y; y++) {
                dh[at(x, y)] += dh[at(x, y - 1)];
                dv[at(x, y)] += dv[at(x, y - 1)];
            }
    });
    parallel_for(Y + 1, 0, [&](int b, int e) {
        for (int x = 1; x <= X; x++)
            for (int y = b; y < e; y++) {
                dh[at(x, y)] += dh[at(x - 1, y)];
                dv[at(x, y)] += dv[at(x - 1, y)];
            }
    });
    out.resize(XY * 16);
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    parallel_for(X, 0, [&](int b, int e) {
        for (int x = b; x < e; x++)
            for (int y = 0; y < Y; y++) {
                const size_t c = (size_t)x * Y + y;
                __nv_bfloat16 *o = out.data() + c * 16;
                o[0] = __float2bfloat16(pins[c]);
                o[1] = __float2bfloat16((float)(0.5 * dh[at(x, y)]));
                o[2] = __float2bfloat16((float)(0.5 * dv[at(x, y)]));
                int blocked = 0;
                for (int l = 0; l < 10; l++) {
                    const float cap = l < L ? d.cap[(size_t)l * XY + c] : 0.f;
                    o[4 + l] = __float2bfloat16(cap / 8.f);
                    if (l > 0 && l < L && cap < 0.5f) blocked++;
                }
                o[3] = __float2bfloat16(L > 1 ? (float)blocked / (float)(L - 1) : 0.f);
                o[14] = zero;
                o[15] = zero;
            }
    });
}

void seed_targets(int X, int Y, int routing_layers, const float *demand_ref, std::vector<__nv_bfloat16> &out) {
    const size_t XY = (size_t)X * Y;
    out.assign(XY * 16, __float2bfloat16(0.f));
    for (int l = 0; l < routing_layers && l + 1 < kSeedLayersOut; l++)
        for (size_t c = 0; c < XY; c++) out[c * 16 + 1 + l] = __float2bfloat16(demand_ref[(size_t)l * XY + c] / 8.f);
}

}  // namespace igr
