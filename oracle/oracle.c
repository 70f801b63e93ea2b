/*
 * CPU oracle for the routing hot path — TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Each function names the reference lines it restates.  Layout: [l][x][y],
 * IDX(l, x, y) = l*X*Y + x*Y + y, as in src/database_cuda.hpp:49.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(l, x, y) ((int64_t)(l) * g->X * g->Y + (int64_t)(x) * g->Y + (y))
#define ORC_INF 1e22
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))

static int dir_of(const orc_grid *g, int l) { return (l & 1) ^ g->DIR; }

/* of_cost_scaled with of_cost_scale = 1 (graph.hpp:23-27); exp() replaces __expf */
static double of_cost(float c, float d) {
    if (c > 0.001) {
        float t = d - c;
        return (double)(float)exp((double)(float)(0.5 * (double)t));
    }
    if (d > 0) return (double)(float)exp((double)(float)(1.5 * (double)d));
    return 0;
}

/* incremental_of_cost with incre_base = 0 (graph.hpp:34-38) */
static double incr(const orc_grid *g, const float *dem, int l, int x, int y, double inc) {
    int64_t i = IDX(l, x, y);
    double a = of_cost(g->cap[i], (float)((double)dem[i] + inc));
    double b = of_cost(g->cap[i], dem[i]);
    double v = (a - b) * g->short_cost[l];
    return v < 1e12 ? v : 1e12;
}

/* Sklansky in-place scan of compute_presum (graph.hpp:405-430) */
static void sklansky_d(double *s, int n) {
    for (int d = 0; (1 << d) < n; d++)
        for (int i = 0; i < n; i++)
            if ((i >> d) & 1) s[i] += s[((i >> d) << d) - 1];
}

void orc_cost_refresh(const orc_grid *g, const float *dem, float *wcost, float *vcost, double *presum) {
    const int L = g->L, X = g->X, Y = g->Y;
    /* update_wcost_cuda_ispd24 (graph.hpp:40-47) */
#pragma omp parallel for collapse(2) schedule(static)
    for (int l = 0; l < L; l++)
        for (int x = 0; x < X; x++)
            for (int y = 0; y < Y; y++) {
                float w = (float)incr(g, dem, l, x, y, 1.0);
                if (dir_of(g, l) == 0 && x < X - 1) w = (float)fma(g->unit_wire, (double)g->xlen[x], (double)w);
                if (dir_of(g, l) == 1 && y < Y - 1) w = (float)fma(g->unit_wire, (double)g->ylen[y], (double)w);
                wcost[IDX(l, x, y)] = w;
            }
    /* update_single_vcost_ispd24 (graph.hpp:52-71), cross_points = 0 */
#pragma omp parallel for collapse(2) schedule(static)
    for (int l = 0; l < L; l++)
        for (int x = 0; x < X; x++)
            for (int y = 0; y < Y; y++) {
                float v;
                if (dir_of(g, l)) {
                    if (y == 0) v = (float)incr(g, dem, l, x, y, 1);
                    else if (y == Y - 1) v = (float)incr(g, dem, l, x, y - 1, 1);
                    else v = (float)(incr(g, dem, l, x, y, 0.5) + incr(g, dem, l, x, y - 1, 0.5));
                } else {
                    if (x == 0) v = (float)incr(g, dem, l, x, y, 1);
                    else if (x == X - 1) v = (float)incr(g, dem, l, x - 1, y, 1);
                    else v = (float)(incr(g, dem, l, x, y, 0.5) + incr(g, dem, l, x - 1, y, 0.5));
                }
                vcost[IDX(l, x, y)] = (float)((double)v + g->unit_via);
            }
    /* compute_presum */
    int n = X > Y ? X : Y;
    /* one track per iteration: (l, t) with t < X on vertical layers, t < Y on horizontal ones */
#pragma omp parallel
    {
        double *s = (double *)malloc(sizeof(double) * (size_t)n);
#pragma omp for collapse(2) schedule(static)
        for (int l = 0; l < L; l++)
            for (int t = 0; t < n; t++) {
                if (dir_of(g, l)) {
                    if (t >= X) continue;
                    s[0] = 0;
                    for (int y = 0; y < Y - 1; y++) s[y + 1] = wcost[IDX(l, t, y)];
                    sklansky_d(s, Y);
                    for (int y = 0; y < Y; y++) presum[IDX(l, t, y)] = s[y];
                } else {
                    if (t >= Y) continue;
                    s[0] = 0;
                    for (int x = 0; x < X - 1; x++) s[x + 1] = wcost[IDX(l, x, t)];
                    sklansky_d(s, X);
                    for (int x = 0; x < X; x++) presum[IDX(l, x, t)] = s[x];
                }
            }
        free(s);
    }
}

static double wseg(const orc_grid *g, const double *presum, int l, int xa, int xb, int ya, int yb) {
    return presum[IDX(l, xb, yb)] - presum[IDX(l, xa, ya)];
}

/* atomic_add_unit_demand_wire_segment (graph.hpp:105-117), K = 1 */
static void add_seg(const orc_grid *g, int *pre, int *st, int l, int xa, int xb, int ya, int yb, int stamp) {
#pragma omp atomic
    pre[IDX(l, xa, ya)] += 1;
    if (xa == xb) {
#pragma omp atomic
        pre[IDX(l, xa, yb)] -= 1;
#pragma omp atomic write
        st[IDX(l, xa, yb)] = stamp;
    }
    if (ya == yb) {
#pragma omp atomic
        pre[IDX(l, xb, ya)] -= 1;
#pragma omp atomic write
        st[IDX(l, xb, ya)] = stamp;
    }
}

int orc_pattern_route(const orc_grid *g, const float *vcost, const double *presum, int n, const int *node_off,
                      const int *nodes, const int *par, const int64_t *route_off, const int *route_cap, int *routes,
                      int *pre, int *st, int stamp) {
    const int L = g->L, X = g->X, Y = g->Y, XY = X * Y, LL = L * L;
    int status = 0;
    /* the nets of a batch are independent: one net per iteration, on all cores */
#pragma omp parallel for schedule(dynamic, 64) reduction(min : status)
    for (int k = 0; k < n; k++) {
        const int nb = node_off[k], cnt = node_off[k + 1] - nb;
        const int *nd = nodes + nb, *pa = par + nb;
        double *dist = (double *)malloc(sizeof(double) * (size_t)cnt * LL);
        int *from = (int *)malloc(sizeof(int) * (size_t)cnt * LL);
        int *lr = (int *)malloc(sizeof(int) * (size_t)cnt);
        for (int i = 0; i < cnt * LL; i++) { dist[i] = 0; from[i] = 0; }
        /* via-stack costs (Lshape_route.hpp:22-32) */
        for (int i = 0; i < cnt; i++) {
            int l = nd[i] / XY, x = nd[i] / Y % X, y = nd[i] % Y;
            double *d = dist + i * LL;
            for (int mn = 0; mn < L; mn++) {
                d[mn * L + mn] = 0;
                for (int mx = mn + 1; mx < L; mx++) d[mn * L + mx] = d[mn * L + mx - 1] + vcost[IDX(mx - 1, x, y)];
                for (int mx = mn; mx < L; mx++)
                    if (l < L && (mn > l || mx < l)) d[mn * L + mx] = ORC_INF;
            }
        }
        /* bottom-up (Lshape_route.hpp:33-97) */
        for (int i = cnt - 1; i >= 1; i--) {
            int x = nd[i] / Y % X, y = nd[i] % Y;
            int px = nd[pa[i]] / Y % X, py = nd[pa[i]] % Y;
            int minx = MIN(x, px), maxx = MAX(x, px), miny = MIN(y, py), maxy = MAX(y, py);
            double *d = dist + i * LL, *pd = dist + pa[i] * LL;
            int *prev = from + i * LL, cf[16];
            double mcc[16], mcp[128];
            for (int l = 0; l < L; l++) {
                mcc[l] = mcp[l * L + l] = ORC_INF;
                cf[l] = 0;
                for (int mn = 0; mn <= l; mn++)
                    for (int mx = l; mx < L; mx++)
                        if (d[mn * L + mx] < mcc[l]) { mcc[l] = d[mn * L + mx]; cf[l] = mn * L + mx; }
            }
            if (x == px || y == py) {
                for (int l = 0; l < L; l++) {
                    if (dir_of(g, l) == 0 && y != py) continue;
                    if (dir_of(g, l) == 1 && x != px) continue;
                    mcp[l * L + l] = mcc[l] + wseg(g, presum, l, minx, maxx, miny, maxy);
                    prev[l * L + l] = cf[l] * LL + l * L + l;
                }
            } else {
                for (int cl = 0; cl < L; cl++) {
                    double cost = mcc[cl];
                    if (dir_of(g, cl)) cost += wseg(g, presum, cl, x, x, miny, maxy);
                    else cost += wseg(g, presum, cl, minx, maxx, y, y);
                    for (int pl = (cl & 1) ^ 1; pl < L; pl += 2) {
                        double c2 = 0;
                        for (int l = MIN(cl, pl) + 1; l < MAX(cl, pl); l++)
                            c2 += dir_of(g, cl) ? vcost[IDX(l, x, py)] : vcost[IDX(l, px, y)];
                        if (dir_of(g, pl)) c2 += wseg(g, presum, pl, px, px, miny, maxy);
                        else c2 += wseg(g, presum, pl, minx, maxx, py, py);
                        if (cost + c2 < mcp[pl * L + pl]) {
                            mcp[pl * L + pl] = cost + c2;
                            prev[pl * L + pl] = cf[cl] * LL + cl * L + pl;
                        }
                    }
                }
            }
            for (int mn = 0; mn < L; mn++) {
                for (int mx = mn + 1; mx < L; mx++) {
                    if (mcp[mn * L + mx - 1] <= mcp[mx * L + mx]) {
                        mcp[mn * L + mx] = mcp[mn * L + mx - 1];
                        prev[mn * L + mx] = prev[mn * L + mx - 1];
                    } else {
                        mcp[mn * L + mx] = mcp[mx * L + mx];
                        prev[mn * L + mx] = prev[mx * L + mx];
                    }
                }
                for (int mx = mn; mx < L; mx++) pd[mn * L + mx] += mcp[mn * L + mx];
            }
        }
        /* backtrace (Lshape_route.hpp:99-152) */
        int *r = routes + route_off[k];
        const int cap = route_cap[k];
        int c = 1;
#define EMIT(a, b)                           \
    do {                                     \
        if (c + 2 > cap) { status = -1; goto done; } \
        r[c++] = (a);                        \
        r[c++] = (b);                        \
    } while (0)
        lr[0] = 0;
        for (int mn = 0; mn < L; mn++)
            for (int mx = mn; mx < L; mx++)
                if (dist[mn * L + mx] < dist[lr[0]]) lr[0] = mn * L + mx;
        for (int i = 0; i < cnt; i++) {
            int *prev = from + i * LL;
            if (i > 0) lr[i] = prev[lr[pa[i]]] / LL;
            int mn = lr[i] / L, mx = lr[i] % L, x = nd[i] / Y % X, y = nd[i] % Y;
            if (mn < mx) EMIT((int)IDX(mn, x, y), (int)IDX(mx, x, y));
            if (i == 0) continue;
            int px = nd[pa[i]] / Y % X, py = nd[pa[i]] % Y;
            int minx = MIN(x, px), maxx = MAX(x, px), miny = MIN(y, py), maxy = MAX(y, py);
            int cl = prev[lr[pa[i]]] / L % L, pl = prev[lr[pa[i]]] % L;
            if (px == x || py == y) {
                EMIT((int)IDX(cl, minx, miny), (int)IDX(cl, maxx, maxy));
                add_seg(g, pre, st, cl, minx, maxx, miny, maxy, stamp);
            } else if (dir_of(g, cl)) {
                EMIT((int)IDX(cl, x, y), (int)IDX(cl, x, py));
                add_seg(g, pre, st, cl, x, x, miny, maxy, stamp);
                EMIT((int)IDX(cl, x, py), (int)IDX(pl, x, py));
                EMIT((int)IDX(pl, x, py), (int)IDX(pl, px, py));
                add_seg(g, pre, st, pl, minx, maxx, py, py, stamp);
            } else {
                EMIT((int)IDX(cl, x, y), (int)IDX(cl, px, y));
                add_seg(g, pre, st, cl, minx, maxx, y, y, stamp);
                EMIT((int)IDX(cl, px, y), (int)IDX(pl, px, y));
                EMIT((int)IDX(pl, px, y), (int)IDX(pl, px, py));
                add_seg(g, pre, st, pl, px, px, miny, maxy, stamp);
            }
        }
    done:
#undef EMIT
        r[0] = c;
        free(dist);
        free(from);
        free(lr);
    }
    return status;
}

int64_t orc_commit_wires(const orc_grid *g, int *pre, float *dem, int *st, int stamp) {
    const int L = g->L, X = g->X, Y = g->Y;
    int64_t wl = 0;
    const int n = X > Y ? X : Y;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : wl)
    for (int l = 0; l < L; l++)
        for (int t = 0; t < n; t++) {
        if (dir_of(g, l) == 0) {
            if (t < Y) {
                const int y = t;
                int acc = 0;
                for (int x = 0; x < X - 1; x++) {
                    acc += pre[IDX(l, x, y)];
                    if (acc > 0) {
                        dem[IDX(l, x, y)] += (float)acc;
                        st[IDX(l, x, y)] = stamp;
                        wl += (int64_t)acc * g->xlen[x];
                    }
                }
            }
        } else {
            if (t < X) {
                const int x = t;
                int acc = 0;
                for (int y = 0; y < Y - 1; y++) {
                    acc += pre[IDX(l, x, y)];
                    if (acc > 0) {
                        dem[IDX(l, x, y)] += (float)acc;
                        st[IDX(l, x, y)] = stamp;
                        wl += (int64_t)acc * g->ylen[y];
                    }
                }
            }
        }
        }
    memset(pre, 0, sizeof(int) * (size_t)L * X * Y);
    return wl;
}

/* demand values are multiples of 0.5: concurrent additions are exact in any order */
static inline void addf(float *p, float v) {
#pragma omp atomic
    *p += v;
}
static inline void setst(int *p, int v) {
#pragma omp atomic write
    *p = v;
}

int64_t orc_commit_vias(const orc_grid *g, int n, const int64_t *off, const int *routes, float *dem, const int *st,
                        int stamp, int K) {
    const int X = g->X, Y = g->Y, XY = X * Y;
    int64_t vias = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : vias)
    for (int k = 0; k < n; k++) {
        const int *r = routes + off[k];
        for (int i = 1; i < r[0]; i += 2) {
            if (r[i] / XY == r[i + 1] / XY) continue;
            int x = r[i] / Y % X, y = r[i] % Y, l0 = r[i] / XY, l1 = r[i + 1] / XY;
            int mn = MIN(l0, l1), mx = MAX(l0, l1);
            vias += mx - mn;
            for (int l = mn; l < mx; l++) {
                if (st[IDX(l, x, y)] >= stamp) continue;
                if (dir_of(g, l)) {
                    if (y == 0) addf(&dem[IDX(l, x, y)], (float)K);
                    else if (y == Y - 1) addf(&dem[IDX(l, x, y - 1)], (float)K);
                    else { addf(&dem[IDX(l, x, y - 1)], (float)(0.5 * K)); addf(&dem[IDX(l, x, y)], (float)(0.5 * K)); }
                } else {
                    if (x == 0) addf(&dem[IDX(l, x, y)], (float)K);
                    else if (x == X - 1) addf(&dem[IDX(l, x - 1, y)], (float)K);
                    else { addf(&dem[IDX(l, x - 1, y)], (float)(0.5 * K)); addf(&dem[IDX(l, x, y)], (float)(0.5 * K)); }
                }
            }
        }
    }
    return vias * K;
}

int64_t orc_ripup_wires(const orc_grid *g, int n, const int64_t *off, const int *routes, float *dem, int *st,
                        int stamp, int K) {
    const int X = g->X, Y = g->Y, XY = X * Y;
    int64_t wl = 0;
    /* demand changes by whole units and every writer stores the same stamp:
     * nets in any order give the same arrays */
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : wl)
    for (int k = 0; k < n; k++) {
        const int *r = routes + off[k];
        for (int i = 1; i < r[0]; i += 2) {
            if (r[i] / XY != r[i + 1] / XY) continue;
            int l = r[i] / XY, x0 = r[i] / Y % X, y0 = r[i] % Y, x1 = r[i + 1] / Y % X, y1 = r[i + 1] % Y;
            for (int x = MIN(x0, x1); x < MAX(x0, x1); x++) { addf(&dem[IDX(l, x, y0)], (float)K); wl += g->xlen[x]; setst(&st[IDX(l, x, y0)], stamp); }
            for (int y = MIN(y0, y1); y < MAX(y0, y1); y++) { addf(&dem[IDX(l, x0, y)], (float)K); wl += g->ylen[y]; setst(&st[IDX(l, x0, y)], stamp); }
            setst(&st[IDX(l, x0, y0)], stamp);
            setst(&st[IDX(l, x0, y1)], stamp);
            setst(&st[IDX(l, x1, y0)], stamp);
            setst(&st[IDX(l, x1, y1)], stamp);
        }
    }
    return wl * K;
}

void orc_mark_overflow(const orc_grid *g, const float *dem, int n, const int64_t *off, const int *routes,
                       int threshold, int min_edges, uint8_t *is_of) {
    const int L = g->L, X = g->X, Y = g->Y, XY = X * Y;
    int *of = (int *)calloc((size_t)L * XY, sizeof(int));
    for (int l = 0; l < L; l++) {
        if (dir_of(g, l) == 0) {
#pragma omp parallel for schedule(static)
            for (int y = 0; y < Y; y++) {
                int acc = 0;
                for (int x = 0; x < X; x++) {
                    of[IDX(l, x, y)] = acc;
                    if (x < X - 1) acc += (g->cap[IDX(l, x, y)] + (float)threshold <= dem[IDX(l, x, y)]) ? 1 : 0;
                }
            }
        } else {
#pragma omp parallel for schedule(static)
            for (int x = 0; x < X; x++) {
                int acc = 0;
                for (int y = 0; y < Y; y++) {
                    of[IDX(l, x, y)] = acc;
                    if (y < Y - 1) acc += (g->cap[IDX(l, x, y)] + (float)threshold <= dem[IDX(l, x, y)]) ? 1 : 0;
                }
            }
        }
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int k = 0; k < n; k++) {
        const int *r = routes + off[k];
        int c = 0;
        is_of[k] = 0;
        for (int i = 1; i < r[0]; i += 2) {
            int l = r[i] / XY, x0 = r[i] / Y % X, y0 = r[i] % Y, x1 = r[i + 1] / Y % X, y1 = r[i + 1] % Y;
            if (x0 != x1) c += of[IDX(l, MAX(x0, x1), y0)] - of[IDX(l, MIN(x0, x1), y0)];
            if (y0 != y1) c += of[IDX(l, x0, MAX(y0, y1))] - of[IDX(l, x0, MIN(y0, y1))];
            if (c > min_edges) { is_of[k] = 1; break; }
        }
    }
    free(of);
}

void orc_congestion_view(const orc_grid *g, const float *dem, float *xsum, float *ysum) {
    const int L = g->L, X = g->X, Y = g->Y;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < X; x++)
        for (int y = 0; y < Y; y++) {
            float m = 0;
            for (int l = 0; l < L; l++) {
                double res = (double)(g->cap[IDX(l, x, y)] - dem[IDX(l, x, y)]);
                if (res < 0 && (float)(-res) > m) m = (float)(-res);
            }
            xsum[x * Y + y] = m;
            ysum[x * Y + y] = m;
        }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < Y; y++) {
        float acc = 0;
        for (int x = 0; x < X; x++) {
            float v = xsum[x * Y + y];
            xsum[x * Y + y] = acc;
            if (x < X - 1) acc += v;
        }
    }
#pragma omp parallel for schedule(static)
    for (int x = 0; x < X; x++) {
        float acc = 0;
        for (int y = 0; y < Y; y++) {
            float v = ysum[x * Y + y];
            ysum[x * Y + y] = acc;
            if (y < Y - 1) acc += v;
        }
    }
}

double orc_overflow_cost(const orc_grid *g, const float *dem) {
    const int L = g->L, X = g->X, Y = g->Y;
    double tot = 0;
    for (int l = 0; l < L; l++)
        for (int x = 0; x < X; x++)
            for (int y = 0; y < Y; y++) {
                if ((dir_of(g, l) == 0 && x + 1 < X) || (dir_of(g, l) == 1 && y + 1 < Y))
                    tot += g->short_cost[l] * of_cost(g->cap[IDX(l, x, y)], dem[IDX(l, x, y)]);
            }
    return tot;
}

int orc_color(int X, int Y, int n, const int *pt_off, const int *pts, const int *h_off, const int *hseg,
              const int *v_off, const int *vseg, int sparsity, int *batch) {
    int *map = (int *)malloc(sizeof(int) * (size_t)X * Y);
    int *status = (int *)malloc(sizeof(int) * (size_t)(n ? n : 1));
    static const int dx[4] = {0, 0, -1, 1}, dy[4] = {0, -1, 0, 0};
    for (int k = 0; k < n; k++) batch[k] = -1;
    int cur;
    for (cur = 0; cur <= n; cur++) {
        int any = 0;
        for (int i = 0; i < X * Y; i++) map[i] = -1;
        for (int k = 0; k < n; k++) status[k] = 0;
        for (int round = 0; round < 30; round++) {
            int rc = 0;
            for (int k = 0; k < n; k++) {
                if (status[k] == 2 || batch[k] != -1) continue;
                status[k] = 1;
                for (int i = pt_off[k]; i < pt_off[k + 1]; i++) {
                    int x = pts[i] / Y, y = pts[i] % Y;
                    for (int j = 0; j < 4; j++) {
                        int nx = x + dx[j], ny = y + dy[j];
                        if (nx >= 0 && nx < X && ny >= 0 && ny < Y && map[nx * Y + ny] < k) map[nx * Y + ny] = k;
                    }
                }
                for (int i = h_off[k]; i < h_off[k + 1]; i++) {
                    int s = hseg[2 * i], e = hseg[2 * i + 1], y = s % Y;
                    for (int x = s / Y; x <= e / Y; x += sparsity)
                        if (map[x * Y + y] < k) map[x * Y + y] = k;
                }
                for (int i = v_off[k]; i < v_off[k + 1]; i++) {
                    int s = vseg[2 * i], e = vseg[2 * i + 1], x = s / Y;
                    for (int y = s % Y; y <= e % Y; y += sparsity)
                        if (map[x * Y + y] < k) map[x * Y + y] = k;
                }
            }
            for (int k = 0; k < n; k++) {
                if (status[k] == 2 || batch[k] != -1) continue;
                int ok = 1;
                for (int i = pt_off[k]; i < pt_off[k + 1] && ok; i++) ok = map[pts[i]] == k;
                if (ok) { batch[k] = cur; any = 1; rc = 1; }
            }
            if (!rc) break;
            for (int k = 0; k < n; k++)
                for (int i = pt_off[k]; i < pt_off[k + 1]; i++) {
                    if (status[k] != 1 || batch[k] != -1) continue;
                    int pre = map[pts[i]];
                    if (pre != -1 && batch[pre] != -1) status[k] = 2;
                }
            for (int i = 0; i < X * Y; i++)
                if (map[i] >= 0 && status[map[i]] == 2) map[i] = -1;
        }
        if (!any) break;
    }
    free(map);
    free(status);
    return cur;
}

/* ---------------------------------------------------------------- phase 2 */
static int32_t f2o(float f) {
    int32_t i;
    memcpy(&i, &f, 4);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
static float o2f(int32_t i) {
    int32_t j = i >= 0 ? i : i ^ 0x7FFFFFFF;
    float f;
    memcpy(&f, &j, 4);
    return f;
}
static uint64_t pack(float c, int id) { return ((uint64_t)(uint32_t)f2o(c) << 32) | (uint32_t)id; }

int orc_dag_route(const orc_grid *g, const float *vcost, const double *presum, int n, const int *node_off,
                  const int *nodes, const int *depth, const int *par_off, const int *par, const int *child_slot,
                  const int *child_num, const int64_t *route_off, const int *route_cap, int *routes, int *pre,
                  int *st, int stamp) {
    const int X = g->X, Y = g->Y, XY = X * Y, ML = 10;
    const int N = node_off[n], E = par_off[N];
    int *coff = (int *)malloc(sizeof(int) * (size_t)(N + 1));
    coff[0] = 0;
    for (int v = 0; v < N; v++) coff[v + 1] = coff[v] + child_num[v];
    double *costs = (double *)malloc(sizeof(double) * ((size_t)N * ML + 1));
    uint64_t *best = (uint64_t *)calloc((size_t)coff[N] * ML + 1, 8);
    uint64_t *pk = (uint64_t *)malloc(8 * ((size_t)coff[N] * ML + 1));
    double *ce = (double *)malloc(sizeof(double) * ((size_t)E * 81 + 1));
    int *bc = (int *)malloc(sizeof(int) * ((size_t)E * 81 + 1));
    int *lo = (int *)malloc(sizeof(int) * ((size_t)N + 1));
    int *stage = (int *)malloc(sizeof(int) * ((size_t)N * 8 + 1));
    int *scnt = (int *)calloc((size_t)N + 1, sizeof(int));
    int status = 0;
    /* The nets of a batch share no DAG node (each node's parents and children
     * belong to its own net), so the nets are routed one per iteration on all
     * cores.  Within a net the nodes are visited level by level, deepest level
     * first, as the reference's per-level launches do; the offers to a parent
     * are minima and the backtrace reads only earlier levels, so the order of
     * the nodes inside a level does not change the result. */
#pragma omp parallel for schedule(dynamic, 1) reduction(min : status)
    for (int k = 0; k < n; k++) {
        const int a = node_off[k], b = node_off[k + 1];
        int sk = 0, D = 0;
        for (int v = a; v < b; v++) {
            if (depth[v] + 1 > D) D = depth[v] + 1;
            lo[v] = -1;
            for (int j = 0; j < ML; j++) costs[(int64_t)v * ML + j] = ORC_INF;
        }
        for (int64_t i = (int64_t)coff[a] * ML; i < (int64_t)coff[b] * ML; i++) pk[i] = 7208259049189261824ULL;
        for (int64_t i = (int64_t)par_off[a] * 81; i < (int64_t)par_off[b] * 81; i++) { ce[i] = 0; bc[i] = -1; }
        /* nodes of the net by level (ascending node index inside a level) */
        int *lv_off = (int *)calloc((size_t)D + 1, sizeof(int));
        int *lv = (int *)malloc(sizeof(int) * (size_t)(b - a + 1));
        for (int v = a; v < b; v++) lv_off[depth[v] + 1]++;
        for (int d = 0; d < D; d++) lv_off[d + 1] += lv_off[d];
        {
            int *fill = (int *)malloc(sizeof(int) * (size_t)(D + 1));
            for (int d = 0; d <= D; d++) fill[d] = lv_off[d];
            for (int v = a; v < b; v++) lv[fill[depth[v]]++] = v;
            free(fill);
        }
        /* precompute_cost_edge (Lshape_route_detour.hpp:123-195) */
        for (int v = a; v < b; v++)
            for (int e = par_off[v]; e < par_off[v + 1]; e++)
                for (int f = 0; f < 9; f++) {
                    int tn = par[e];
                    int tox = nodes[tn] / Y % X, toy = nodes[tn] % Y, fx = nodes[v] / Y % X, fy = nodes[v] % Y;
                    if ((dir_of(g, f) == 0 && fy != toy) || (dir_of(g, f) == 1 && fx != tox)) {
                        for (int t = 0; t < 9; t++) ce[(int64_t)e * 81 + f * 9 + t] = ORC_INF;
                        continue;
                    }
                    int dist = abs(tox - fx) + abs(toy - fy);
                    if (dist == 0) continue;
                    int dd = dist / MIN(dist, 20);
                    int vert = fx == tox;
                    int s0 = vert ? MIN(fy, toy) : MIN(fx, tox), s1 = vert ? MAX(fy, toy) : MAX(fx, tox);
                    for (int t = 0; t < 9; t++) {
                        if (t % 2 != f % 2) continue;
                        double bestc = ORC_INF;
                        int pos = -1;
                        for (int sp = s0 + dd; sp < s1; sp += dd) {
                            int sx = vert ? fx : sp, sy = vert ? sp : fy;
                            double via = 0;
                            for (int ll = MIN(f, t); ll < MAX(f, t); ll++) via += vcost[IDX(ll, sx, sy)];
                            double c = via;
                            if (vert)
                                c += (wseg(g, presum, f, fx, fx, MIN(fy, sy), MAX(fy, sy)) + wseg(g, presum, t, tox, tox, MIN(toy, sy), MAX(toy, sy)));
                            else
                                c += (wseg(g, presum, f, MIN(fx, sx), MAX(fx, sx), fy, fy) + wseg(g, presum, t, MIN(tox, sx), MAX(tox, sx), toy, toy));
                            if (c < bestc) { bestc = c; pos = sp; }
                        }
                        ce[(int64_t)e * 81 + f * 9 + t] = bestc;
                        bc[(int64_t)e * 81 + f * 9 + t] = pos;
                    }
                }
        /* bottom-up (Lshape_route_detour.hpp:281-406) */
        for (int d = D - 1; d >= 0; d--)
            for (int q = lv_off[d]; q < lv_off[d + 1]; q++) {
                const int v = lv[q];
                int fl = 1 + nodes[v] / XY, x = nodes[v] / Y % X, y = nodes[v] % Y;
                int fh = fl == 10 ? 0 : fl, cb = coff[v], cn = coff[v + 1] - cb;
                double minc[10];
                uint64_t bp[10] = {0};
                for (int low = 1; low <= fl; low++) {
                    for (int c = 0; c < cn; c++) minc[c] = ORC_INF;
                    double via = 0;
                    for (int layer = low; layer < g->L + 1; layer++) {
                        if (layer > low) via += vcost[IDX(layer - 2, x, y)];
                        for (int c = 0; c < cn; c++) {
                            uint64_t p = pk[(int64_t)(cb + c) * ML + layer];
                            double cc = (double)o2f((int32_t)(p >> 32));
                            int id = (int)(p & 0xFFFFFFFFu);
                            if (cc < minc[c]) { minc[c] = cc; bp[c] = (uint64_t)id * ML + layer; }
                        }
                        if (layer >= fh) {
                            double t = via;
                            for (int c = 0; c < cn; c++) t += minc[c];
                            if (t < ORC_INF && t < costs[(int64_t)v * ML + layer]) {
                                costs[(int64_t)v * ML + layer] = t;
                                for (int c = 0; c < cn; c++) best[(int64_t)(cb + c) * ML + layer] = bp[c];
                            }
                        }
                    }
                    for (int layer = g->L - 1; layer >= low; layer--)
                        if (costs[(int64_t)v * ML + layer + 1] < costs[(int64_t)v * ML + layer]) {
                            costs[(int64_t)v * ML + layer] = costs[(int64_t)v * ML + layer + 1];
                            for (int c = 0; c < cn; c++) best[(int64_t)(cb + c) * ML + layer] = best[(int64_t)(cb + c) * ML + layer + 1];
                        }
                }
                for (int e = par_off[v]; e < par_off[v + 1]; e++) {
                    int p = par[e], sl = child_slot[e];
                    uint64_t *pp = pk + (int64_t)(coff[p] + sl) * ML;
                    int px = nodes[p] / Y % X, py = nodes[p] % Y;
                    int minx = MIN(x, px), maxx = MAX(x, px), miny = MIN(y, py), maxy = MAX(y, py);
                    for (int layer = 1; layer < ML; layer++) {
                        int dl = (layer & 1) ^ g->DIR;
                        if (dl == 1 && y != py) continue;
                        if (dl == 0 && x != px) continue;
                        double base = costs[(int64_t)v * ML + layer];
                        for (int t = 1 + (1 - layer % 2); t < ML; t += 2) {
                            double c2;
                            int ch = 82;
                            if (t == layer) c2 = base + wseg(g, presum, layer - 1, minx, maxx, miny, maxy);
                            else if (abs(x - px) + abs(y - py) > 4) {
                                int seq = (layer - 1) * 9 + (t - 1);
                                double c = ce[(int64_t)e * 81 + seq];
                                if (c < ORC_INF) { c2 = base + c; ch = seq; }
                                else continue;
                            } else continue;
                            uint64_t nv = pack((float)c2, v * 100 + ch);
                            if (nv < pp[t]) pp[t] = nv;
                        }
                    }
                }
            }
        /* top-down (Lshape_route_detour.hpp:520-694) */
#define STAGE(a, b)                                                    \
    do {                                                               \
        if (scnt[v] + 2 > 8) { sk = -1; } else {                       \
            stage[(int64_t)v * 8 + scnt[v]] = (a);                     \
            stage[(int64_t)v * 8 + scnt[v] + 1] = (b);                 \
            scnt[v] += 2; }                                            \
    } while (0)
        for (int d = 0; d < D; d++)
            for (int q = lv_off[d]; q < lv_off[d + 1]; q++) {
                const int v = lv[q];
                int l = nodes[v] / XY, cx = nodes[v] / Y % X, cy = nodes[v] % Y;
                int pn = par_off[v + 1] - par_off[v];
                if (pn == 0) {
                    int ml = 0;
                    double mc = costs[(int64_t)v * ML];
                    for (int layer = 1; layer < ML; layer++)
                        if (costs[(int64_t)v * ML + layer] < mc) { mc = costs[(int64_t)v * ML + layer]; ml = layer; }
                    lo[v] = ml;
                } else {
                    int pl = -1, pidx = -1, pseq = -1;
                    for (int pi = 0; pi < pn; pi++) {
                        int e = par_off[v] + pi, pnode = par[e];
                        if (lo[pnode] <= 0) continue;
                        pidx = pnode; pseq = pi; pl = lo[pnode];
                        uint64_t path = best[(int64_t)(coff[pidx] + child_slot[par_off[v] + pseq]) * ML + pl];
                        uint64_t cid = path / ML / 100, ch = (path / ML) % 100;
                        if (cid == (uint64_t)v) {
                            lo[v] = ch == 82 ? (int)(path % ML) : (int)(ch / 9 + 1);
                            int px = nodes[pidx] / Y % X, py = nodes[pidx] % Y, L1 = lo[v] - 1;
                            if (px == cx && cy != py) {
                                if (ch == 82) {
                                    add_seg(g, pre, st, L1, px, px, MIN(py, cy), MAX(py, cy), stamp);
                                    STAGE((int)IDX(L1, px, MIN(py, cy)), (int)IDX(L1, px, MAX(py, cy)));
                                } else {
                                    int f = (int)(ch / 9), t = (int)(ch % 9), cp = bc[(int64_t)e * 81 + f * 9 + t];
                                    add_seg(g, pre, st, f, cx, cx, MIN(cy, cp), MAX(cy, cp), stamp);
                                    add_seg(g, pre, st, t, cx, cx, MIN(py, cp), MAX(py, cp), stamp);
                                    STAGE((int)IDX(f, cx, MIN(cy, cp)), (int)IDX(f, cx, MAX(cy, cp)));
                                    STAGE((int)IDX(MIN(f, t), cx, cp), (int)IDX(MAX(f, t), cx, cp));
                                    STAGE((int)IDX(t, cx, MIN(py, cp)), (int)IDX(t, cx, MAX(py, cp)));
                                }
                            } else if (py == cy && cx != px) {
                                if (ch == 82) {
                                    add_seg(g, pre, st, L1, MIN(px, cx), MAX(px, cx), py, py, stamp);
                                    STAGE((int)IDX(L1, MIN(px, cx), py), (int)IDX(L1, MAX(px, cx), py));
                                } else {
                                    int f = (int)(ch / 9), t = (int)(ch % 9), cp = bc[(int64_t)e * 81 + f * 9 + t];
                                    add_seg(g, pre, st, f, MIN(cx, cp), MAX(cx, cp), cy, cy, stamp);
                                    add_seg(g, pre, st, t, MIN(px, cp), MAX(px, cp), cy, cy, stamp);
                                    STAGE((int)IDX(f, MIN(cx, cp), cy), (int)IDX(f, MAX(cx, cp), cy));
                                    STAGE((int)IDX(MIN(f, t), cp, cy), (int)IDX(MAX(f, t), cp, cy));
                                    STAGE((int)IDX(t, MIN(px, cp), cy), (int)IDX(t, MAX(px, cp), cy));
                                }
                            }
                            break;
                        } else {
                            lo[v] = -1;
                        }
                    }
                    if (pl == -1) { lo[v] = -1; continue; }
                    uint64_t path = best[(int64_t)(coff[pidx] + child_slot[par_off[v] + pseq]) * ML + pl];
                    if (path / ML / 100 != (uint64_t)v) { lo[v] = -1; continue; }
                }
                int cn = coff[v + 1] - coff[v];
                int mnl = l + 1, mxl = (l + 1) == ML ? 1 : l + 1;
                mnl = MIN(mnl, lo[v]);
                mxl = MAX(mxl, lo[v]);
                for (int c = 0; c < cn; c++) {
                    int lc = (int)(best[(int64_t)(coff[v] + c) * ML + lo[v]] % ML);
                    mnl = MIN(lc, mnl);
                    mxl = MAX(lc, mxl);
                }
                if (mnl < mxl) STAGE((int)IDX(mnl - 1, cx, cy), (int)IDX(mxl - 1, cx, cy));
            }
#undef STAGE
        /* route record in node order */
        {
            int *r = routes + route_off[k];
            int c = 1, full = 0;
            for (int v = a; v < b && !full; v++)
                for (int j = 0; j < scnt[v]; j++) {
                    if (c + 1 > route_cap[k]) { full = 1; sk = -1; break; }
                    r[c++] = stage[(int64_t)v * 8 + j];
                }
            r[0] = c;
        }
        free(lv_off);
        free(lv);
        if (sk < status) status = sk;
    }
    free(coff); free(costs); free(best); free(pk); free(ce); free(bc); free(lo); free(stage); free(scnt);
    return status;
}
