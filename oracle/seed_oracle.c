/* CPU oracle of the learned congestion seed (test infrastructure only).
 *
 * Forward and backward pass of the six-convolution network of
 * instantgr_b200/csrc/seed_model.cpp in double precision, on channels-last
 * tiles [T][S][S][16].  With `round` set, values are rounded to BF16 where the
 * GPU stores BF16 (weights, activations after ReLU, the loss gradient and the
 * masked input gradients), so that the GPU's gradients can be compared with
 * it; with `round` clear it is the exact f64 function, which the tests pin
 * with finite differences.  This network has no counterpart in InstantGR. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const int CIN[6] = {16, 32, 64, 64, 64, 32};
static const int COUT[6] = {32, 64, 64, 64, 32, 16};
static const int MODE[6] = {0, 1, 0, 0, 2, 0};

/* round to nearest even BF16 */
static double bf16r(double v) {
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return f;
}

/* input position of output (oy, ox) under tap (dy, dx) for layer spec; 0 outside */
static int in_pos(int mode, int hin, int win, int hout, int wout, int oy, int ox, int dy, int dx, int *iy, int *ix) {
    if (mode == 1) {
        *iy = 2 * oy + dy - 1;
        *ix = 2 * ox + dx - 1;
    } else if (mode == 2) {
        int uy = oy + dy - 1, ux = ox + dx - 1;
        if (uy < 0 || ux < 0 || uy >= hout || ux >= wout) return 0;
        *iy = uy >> 1;
        *ix = ux >> 1;
        return 1;
    } else {
        *iy = oy + dy - 1;
        *ix = ox + dx - 1;
    }
    return *iy >= 0 && *ix >= 0 && *iy < hin && *ix < win;
}

int orc_seed_params(void) {
    int n = 0;
    for (int i = 0; i < 6; i++) n += COUT[i] * 9 * CIN[i] + COUT[i];
    return n;
}

/* loss (mean squared error over the central region and channels 0..9) and the
 * gradient of every parameter; params/grads: per layer w[cout][9][cin], b[cout] */
double orc_seed_grad(int T, int S, int halo, const float *x, const float *target, const float *params, float *grads,
                     int round) {
    int H[7], Wd[7];
    H[0] = Wd[0] = S;
    for (int i = 0; i < 6; i++) {
        H[i + 1] = MODE[i] == 1 ? H[i] / 2 : (MODE[i] == 2 ? H[i] * 2 : H[i]);
        Wd[i + 1] = H[i + 1];
    }
    double *act[7], *gr[7];
    const float *pw[6], *pb[6];
    float *gw[6], *gb[6];
    size_t o = 0;
    for (int i = 0; i < 6; i++) {
        pw[i] = params + o;
        gw[i] = grads + o;
        o += (size_t)COUT[i] * 9 * CIN[i];
        pb[i] = params + o;
        gb[i] = grads + o;
        o += COUT[i];
    }
    for (int i = 0; i <= 6; i++) {
        const int c = i == 0 ? CIN[0] : COUT[i - 1];
        act[i] = (double *)calloc((size_t)T * H[i] * Wd[i] * c, sizeof(double));
        gr[i] = (double *)calloc((size_t)T * H[i] * Wd[i] * c, sizeof(double));
    }
    for (size_t i = 0; i < (size_t)T * S * S * 16; i++) act[0][i] = round ? bf16r(x[i]) : x[i];
    /* forward */
    for (int L = 0; L < 6; L++) {
        const int ci_n = CIN[L], co_n = COUT[L], hi = H[L], wi = Wd[L], ho = H[L + 1], wo = Wd[L + 1];
        for (int t = 0; t < T; t++)
            for (int oy = 0; oy < ho; oy++)
                for (int ox = 0; ox < wo; ox++)
                    for (int co = 0; co < co_n; co++) {
                        double s = 0;
                        for (int tap = 0; tap < 9; tap++) {
                            int iy, ix;
                            if (!in_pos(MODE[L], hi, wi, ho, wo, oy, ox, tap / 3, tap % 3, &iy, &ix)) continue;
                            const double *a = act[L] + (((size_t)t * hi + iy) * wi + ix) * ci_n;
                            const float *w = pw[L] + ((size_t)co * 9 + tap) * ci_n;
                            for (int ci = 0; ci < ci_n; ci++) s += (round ? bf16r(w[ci]) : w[ci]) * a[ci];
                        }
                        s += pb[L][co];
                        if (L < 5) {
                            if (s < 0) s = 0;
                            if (round) s = bf16r(s);
                        }
                        act[L + 1][(((size_t)t * ho + oy) * wo + ox) * co_n + co] = s;
                    }
    }
    /* loss */
    const double count = (double)T * (S - 2 * halo) * (S - 2 * halo) * 10;
    double loss = 0;
    for (int t = 0; t < T; t++)
        for (int yy = 0; yy < S; yy++)
            for (int xx = 0; xx < S; xx++)
                for (int ch = 0; ch < 16; ch++) {
                    const size_t i = (((size_t)t * S + yy) * S + xx) * 16 + ch;
                    double g = 0;
                    if (ch < 10 && xx >= halo && xx < S - halo && yy >= halo && yy < S - halo) {
                        const double e = act[6][i] - target[i];
                        loss += e * e;
                        g = 2.0 * e / count;
                    }
                    gr[6][i] = round ? bf16r(g) : g;
                }
    loss /= count;
    /* backward */
    for (int L = 5; L >= 0; L--) {
        const int ci_n = CIN[L], co_n = COUT[L], hi = H[L], wi = Wd[L], ho = H[L + 1], wo = Wd[L + 1];
        double *dw = (double *)calloc((size_t)co_n * 9 * ci_n, sizeof(double));
        double *db = (double *)calloc(co_n, sizeof(double));
        double *dx = (double *)calloc((size_t)T * hi * wi * ci_n, sizeof(double));
        for (int t = 0; t < T; t++)
            for (int oy = 0; oy < ho; oy++)
                for (int ox = 0; ox < wo; ox++)
                    for (int co = 0; co < co_n; co++) {
                        const double g = gr[L + 1][(((size_t)t * ho + oy) * wo + ox) * co_n + co];
                        if (g == 0) continue;
                        db[co] += g;
                        for (int tap = 0; tap < 9; tap++) {
                            int iy, ix;
                            if (!in_pos(MODE[L], hi, wi, ho, wo, oy, ox, tap / 3, tap % 3, &iy, &ix)) continue;
                            const size_t q = (((size_t)t * hi + iy) * wi + ix) * ci_n;
                            const float *w = pw[L] + ((size_t)co * 9 + tap) * ci_n;
                            double *dwr = dw + ((size_t)co * 9 + tap) * ci_n;
                            for (int ci = 0; ci < ci_n; ci++) {
                                dwr[ci] += g * act[L][q + ci];
                                dx[q + ci] += g * (round ? bf16r(w[ci]) : w[ci]);
                            }
                        }
                    }
        for (size_t i = 0; i < (size_t)co_n * 9 * ci_n; i++) gw[L][i] = (float)dw[i];
        for (int co = 0; co < co_n; co++) gb[L][co] = (float)db[co];
        if (L > 0)
            for (size_t i = 0; i < (size_t)T * hi * wi * ci_n; i++) {
                const double v = act[L][i] > 0 ? dx[i] : 0.0;  /* ReLU of the layer below */
                gr[L][i] = round ? bf16r(v) : v;
            }
        free(dw);
        free(db);
        free(dx);
    }
    for (int i = 0; i <= 6; i++) {
        free(act[i]);
        free(gr[i]);
    }
    return loss;
}
