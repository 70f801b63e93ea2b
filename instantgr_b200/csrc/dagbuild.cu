// Detour DAGs of the rerouted nets, built on the device: one thread per net.
//
// The construction is the host builder's (dag_build.cpp), which restates
// net::generate_detours_reconstruct (src/database_cuda.hpp:1429-2086) with
// construct_segments = false; that file lists the steps and the reference's
// quirks, all kept here in the same order of node creation:
//   root by leaf-peeling BFS (:826-856); congestion regions, stems and trunk
//   ranges by a DFS from the root (:1494-1637); DAG nodes by a second DFS
//   (mirrors placed by the stem displacement rule :1734-1772, L and Z shapes,
//   long edges split at 50/150 GCells :1671-1724); renumbering so that parents
//   come first, with each node's depth its longest distance from the root
//   (:2027-2085).
// The recursions become explicit stacks and the growing containers become
// slices of a per-thread work area.  A net whose DAG does not fit its slices
// reports so and is built again with larger ones.  A finished DAG reserves its
// ranges of the node, edge and point pools with one atomic add each and is
// written there; a DAG that finds a pool full is built again once the pools
// have grown.  A second kernel gathers the DAGs of each colour batch into the
// batch-local arrays of the DAG router.
#include "kcommon.cuh"

namespace igr {

namespace {

// work area of one thread, carved from consecutive ints
struct Work {
    int *region, *rlo, *rhi, *shead;           // [2][tc] union-find parent, trunk range, stem list head
    int *sval, *snext, *ss;                    // [sc] stem pool; one region's stems, sorted
    int *qn, *qf;                              // [3tc+4] root BFS queue (node, from)
    int *mx, *mp, *mq;                         // [tc] region DFS stack (node, parent, next neighbour)
    int *pe, *pp, *ppn, *ps;                   // [tc] DAG DFS pending nodes (node, parent, parent DAG node, slot)
    int *pl_off, *pl_cnt, *nm_off, *nm_cnt;    // [2][tc] mirror places and mirror DAG nodes per tree node
    int *mpool;                                // [mc]
    int *nodes, *child_pre;                    // [nc]
    int *lc, *lp;                              // [ec] links: child, parent*10 + slot
    int *pts;                                  // [pc]
    int *poff;                                 // [nc+1]
    int *pcode;                                // [ec]
    int *at, *visit, *newid, *ord, *stn, *stq; // [nc]
    int *dep, *cn, *pn, *onode;                // [nc] depth, child slots, parents, position by new id
};

__host__ __device__ inline long long work_ints(const DagCaps &c) {
    return 29LL * c.tc + 3LL * c.sc + c.mc + 13LL * c.nc + 3LL * c.ec + c.pc + 16;
}

__device__ Work carve(int *p, const DagCaps &c) {
    Work w;
    auto take = [&](long long n) {
        int *r = p;
        p += n;
        return r;
    };
    w.region = take(2 * c.tc); w.rlo = take(2 * c.tc); w.rhi = take(2 * c.tc); w.shead = take(2 * c.tc);
    w.sval = take(c.sc); w.snext = take(c.sc); w.ss = take(c.sc);
    w.qn = take(3 * c.tc + 4); w.qf = take(3 * c.tc + 4);
    w.mx = take(c.tc); w.mp = take(c.tc); w.mq = take(c.tc);
    w.pe = take(c.tc); w.pp = take(c.tc); w.ppn = take(c.tc); w.ps = take(c.tc);
    w.pl_off = take(2 * c.tc); w.pl_cnt = take(2 * c.tc); w.nm_off = take(2 * c.tc); w.nm_cnt = take(2 * c.tc);
    w.mpool = take(c.mc);
    w.nodes = take(c.nc); w.child_pre = take(c.nc);
    w.lc = take(c.ec); w.lp = take(c.ec);
    w.pts = take(c.pc);
    w.poff = take(c.nc + 1);
    w.pcode = take(c.ec);
    w.at = take(c.nc); w.visit = take(c.nc); w.newid = take(c.nc); w.ord = take(c.nc); w.stn = take(c.nc);
    w.stq = take(c.nc);
    w.dep = take(c.nc); w.cn = take(c.nc); w.pn = take(c.nc); w.onode = take(c.nc);
    return w;
}

enum : int { kOk = 0, kTooLarge = 1, kMalformed = 2, kPoolFull = 3 };

// in-place ascending heap sort of a[0..n)
__device__ void heap_sort(int *a, int n) {
    auto sift = [&](int i, int m) {
        while (true) {
            int l = 2 * i + 1;
            if (l >= m) return;
            if (l + 1 < m && a[l + 1] > a[l]) l++;
            if (a[l] <= a[i]) return;
            const int t = a[i]; a[i] = a[l]; a[l] = t;
            i = l;
        }
    };
    for (int i = n / 2 - 1; i >= 0; i--) sift(i, n);
    for (int m = n - 1; m > 0; m--) {
        const int t = a[0]; a[0] = a[m]; a[m] = t;
        sift(0, m);
    }
}

struct Builder {
    const Work &w;
    const DagCaps &c;
    const int *P, *ao, *nb;  // tree positions, adjacency offsets (global), neighbours (net-local)
    const float *xsum, *ysum;
    int T, X, Y, XY;
    float ratio;
    int num_tracks, zs, sel;
    int root = -1;
    int nn = 0, nl = 0, np = 0, nsu = 0, nmu = 0;
    int bad = kOk;

    __device__ int px(int v) const { return v / Y % X; }
    __device__ int py(int v) const { return v % Y; }
    __device__ float ys(int x, int y) const { return __ldg(ysum + (size_t)x * Y + y); }
    __device__ float xs(int x, int y) const { return __ldg(xsum + (size_t)x * Y + y); }
    __device__ int deg(int x) const { return ao[x + 1] - ao[x]; }
    __device__ int nbr(int q) const { return nb[q]; }

    __device__ int create(int l, int x, int y) {
        if (nn >= c.nc) {
            bad = bad ? bad : kTooLarge;
            return 0;
        }
        w.nodes[nn] = l * XY + x * Y + y;
        w.child_pre[nn] = 0;
        return nn++;
    }

    __device__ void connect_pre(int p, int ch, int slot) {
        if (bad) return;
        if (nl >= c.ec || np + 2 > c.pc) {
            bad = kTooLarge;
            return;
        }
        w.pts[np++] = px(w.nodes[ch]) * Y + py(w.nodes[ch]);
        w.pts[np++] = px(w.nodes[p]) * Y + py(w.nodes[p]);
        w.lc[nl] = ch;
        w.lp[nl] = p * 10 + slot;
        nl++;
        w.child_pre[p]++;
    }

    // long edges get one or two intermediate nodes (connect_node, :1671-1724)
    __device__ void connect(int p, int ch, int slot) {
        if (bad) return;
        const int ax = px(w.nodes[p]), ay = py(w.nodes[p]), bx = px(w.nodes[ch]), by = py(w.nodes[ch]);
        const int len = abs(ax - bx) + abs(ay - by);
        if (len < 50) {
            connect_pre(p, ch, slot);
            return;
        }
        if (len < 150) {
            const int m = create(9, (ax + bx) / 2, (ay + by) / 2);
            connect_pre(p, m, slot);
            connect_pre(m, ch, 0);
            return;
        }
        int m1, m2;
        if (ay == by) {
            m1 = create(9, ax * 2 / 3 + bx / 3, ay);
            m2 = create(9, ax * 1 / 3 + bx * 2 / 3, ay);
        } else if (ax == bx) {
            m1 = create(9, ax, ay * 2 / 3 + by / 3);
            m2 = create(9, ax, ay * 1 / 3 + by * 2 / 3);
        } else {
            bad = kMalformed;  // a detour DAG edge that is not straight
            return;
        }
        connect_pre(p, m1, slot);
        connect_pre(m1, m2, 0);
        connect_pre(m2, ch, 0);
    }

    // union-find root with path compression; a chain that meets -1 gives -1
    // and every entry on it becomes -1, as the recursive form does
    __device__ int region_of(int x, int dir) {
        if (x < 0) return -1;
        int *r = w.region + dir * c.tc;
        int y = x, res, steps = 0;
        while (true) {
            const int ry = r[y];
            if (ry == -1) { res = -1; break; }
            if (ry == y) { res = y; break; }
            y = ry;
            if (++steps > T) {
                bad = kMalformed;
                return -1;
            }
        }
        y = x;
        while (r[y] != -1 && r[y] != y) {
            const int nx = r[y];
            r[y] = res;
            y = nx;
        }
        return res;
    }

    __device__ void stem_push(int dir, int node, int v) {
        if (nsu >= c.sc) {
            bad = bad ? bad : kTooLarge;
            return;
        }
        int &h = w.shead[dir * c.tc + node];
        w.sval[nsu] = v;
        w.snext[nsu] = h;
        h = nsu++;
    }

    // appends a copy of src's stems to dst's (the multiset is what matters)
    __device__ void stem_copy(int dir, int dst, int src) {
        for (int i = w.shead[dir * c.tc + src]; i != -1 && !bad; i = w.snext[i]) stem_push(dir, dst, w.sval[i]);
    }

    __device__ void range_merge(int dir, int dst, int lo, int hi) {
        int &a = w.rlo[dir * c.tc + dst], &b = w.rhi[dir * c.tc + dst];
        a = min(a, lo);
        b = max(b, hi);
    }

    // leaf-peeling BFS; the root is the last node taken from the queue
    __device__ int select_root() {
        int head = 0, tail = 0, sel = -1;
        const int qcap = 3 * c.tc + 4;
        for (int i = 0; i < T; i++) w.visit[i] = 0;
        for (int i = 0; i < T; i++)
            if (deg(i) == 1) {
                w.qn[tail] = i;
                w.qf[tail] = -1;
                tail++;
            }
        while (head < tail) {
            const int f = w.qn[head], from = w.qf[head];
            head++;
            sel = f;
            if (w.visit[f]) continue;
            w.visit[f] = 1;
            for (int q = ao[f]; q < ao[f + 1]; q++) {
                const int j = nbr(q);
                if (j == from) continue;
                if (tail >= qcap) {
                    bad = kMalformed;
                    return -1;
                }
                w.qn[tail] = j;
                w.qf[tail] = f;
                tail++;
            }
        }
        return sel;
    }

    // congestion of tree edge (x, e) and the region bookkeeping before the DFS
    // descends into e (:1494-1637)
    __device__ void mark_edge(int x, int e) {
        const int cx = px(P[x]), cy = py(P[x]);
        const int ex = px(P[e]), ey = py(P[e]);
        int dir = -1, cong = -1;
        if (ex == cx) {
            if (__fsub_rn(ys(cx, max(ey, cy)), ys(cx, min(ey, cy))) > 0) { dir = 1; cong = 1; }
        } else if (ey == cy) {
            if (__fsub_rn(xs(max(ex, cx), cy), xs(min(ex, cx), cy)) > 0) { dir = 0; cong = 1; }
        } else {
            const bool cyy = __fsub_rn(ys(cx, max(ey, cy)), ys(cx, min(ey, cy))) > 0 ||
                             __fsub_rn(ys(ex, max(ey, cy)), ys(ex, min(ey, cy))) > 0;
            if (cyy) { dir = 1; cong = 2; }
            if (cong == -1) {
                const bool cxx = __fsub_rn(xs(max(ex, cx), cy), xs(min(ex, cx), cy)) > 0 ||
                                 __fsub_rn(xs(max(ex, cx), ey), xs(min(ex, cx), ey)) > 0;
                if (cxx) { dir = 0; cong = 2; }
            }
        }
        int *r = w.region + (dir < 0 ? 0 : dir) * c.tc;
        if (cong == 1) {
            int target;
            if (x != root) {
                if (r[x] == -1) r[x] = x;
                target = region_of(x, dir);
            } else {
                if (r[e] == -1) r[e] = e;
                target = region_of(e, dir);
            }
            if (target < 0) {  // cannot happen for a tree: the entry was just set
                bad = kMalformed;
                return;
            }
            r[e] = target;
            if (x != root) stem_copy(dir, target, e);
            range_merge(dir, target, w.rlo[dir * c.tc + e], w.rhi[dir * c.tc + e]);
        } else if (cong == 2) {
            if (x != root && r[x] == -1) r[x] = x;
            if (r[e] == -1) r[e] = e;
        }
    }

    // stems across region borders once all children of x are done
    __device__ void mark_post(int x, int par) {
        const int cx = px(P[x]), cy = py(P[x]);
        for (int dir = 0; dir < 2; dir++) {
            const int xr = region_of(x, dir);
            for (int q = ao[x]; q < ao[x + 1] && !bad; q++) {
                const int e = nbr(q);
                if (e == par) continue;
                const int ex = px(P[e]), ey = py(P[e]);
                const int er = region_of(e, dir);
                if (xr != er) {
                    if (xr >= 0) {
                        stem_push(dir, xr, dir ? ex : ey);
                        range_merge(dir, xr, dir ? ey : ex, dir ? ey : ex);
                    }
                    if (er >= 0) {
                        stem_push(dir, er, dir ? cx : cy);
                        range_merge(dir, er, dir ? cy : cx, dir ? cy : cx);
                    }
                }
            }
        }
    }

    __device__ void mark_all() {
        int top = 0;
        w.mx[0] = root; w.mp[0] = -1; w.mq[0] = ao[root];
        top = 1;
        while (top > 0 && !bad) {
            const int f = top - 1;
            const int x = w.mx[f];
            if (w.mq[f] < ao[x + 1]) {
                const int e = nbr(w.mq[f]++);
                if (e == w.mp[f]) continue;
                mark_edge(x, e);
                if (top >= c.tc) {  // deeper than the tree has nodes: not a tree
                    bad = kMalformed;
                    return;
                }
                w.mx[top] = e; w.mp[top] = x; w.mq[top] = ao[e];
                top++;
            } else {
                mark_post(x, w.mp[f]);
                top--;
            }
        }
    }

    // mirror positions of region root t (get_mirror_places, :1734-1772),
    // appended to the mirror pool
    __device__ void mirror_places(int t, int dir, int &off, int &cnt) {
        const int v = P[t];
        const int reg = w.region[dir * c.tc + t];
        const int cx = px(v), cy = py(v);
        const int trunk = w.rhi[dir * c.tc + reg] - w.rlo[dir * c.tc + reg];
        const int maxd = (int)__fmul_rn(ratio, (float)trunk);
        const int orig = dir ? cx : cy;
        // The displacement D(q) = sum of |stem - q| over the region's stems is
        // walked incrementally over its sorted stems:
        //   D(q-1) = D(q) + n - 2 #{s < q},  D(q+1) = D(q) + 2 #{s <= q} - n,
        // which gives exactly the sums the reference recomputes at every step.
        int n = 0;
        for (int i = w.shead[dir * c.tc + reg]; i != -1; i = w.snext[i]) w.ss[n++] = w.sval[i];  // n <= nsu <= sc
        heap_sort(w.ss, n);
        int od = 0;
        for (int j = 0; j < n; j++) od += abs(w.ss[j] - orig);
        int lt = 0;  // #{s < orig}
        while (lt < n && w.ss[lt] < orig) lt++;
        int lo = orig, hi = orig;
        const int bound = dir ? X : Y;
        {   // lo: while D(lo - 1) - od <= maxd
            int D = od, below = lt;  // below = #{s < lo}
            while (lo - 1 >= 0) {
                const int Dm = D + n - 2 * below;
                if (Dm - od > maxd) break;
                lo--;
                D = Dm;
                while (below > 0 && w.ss[below - 1] >= lo) below--;
            }
        }
        {   // hi: while D(hi - 1) - od <= maxd (hi - 1: kept from :1750)
            int t = orig - 1, D = od + n - 2 * lt;  // D(orig - 1)
            int le = 0;                              // #{s <= t}
            while (le < n && w.ss[le] <= t) le++;
            while (hi + 1 < bound && D - od <= maxd) {
                hi++;
                D += 2 * le - n;  // D(t + 1)
                t++;
                while (le < n && w.ss[le] <= t) le++;
            }
        }
        int step = 1;
        while ((orig - lo) / (step + 1) + (hi - orig) / (step + 1) >= num_tracks) step++;
        lo = orig - (orig - lo) / step * step;
        hi = orig + (hi - orig) / step * step;
        off = nmu;
        cnt = 0;
        for (int pos = lo; pos <= hi; pos += step) {
            if (pos == orig) continue;
            if (nmu >= c.mc) {
                bad = bad ? bad : kTooLarge;
                return;
            }
            w.mpool[nmu++] = pos;
            cnt++;
        }
    }

    // Z-shape candidate k of leg pi between parent position (ppx, ppy) and
    // (cx, cy) with mz steps; false when it leaves the grid or meets an end
    __device__ bool mids(int k, int pi, int mz, int ppx, int ppy, int cx, int cy, int &x1, int &y1, int &x2,
                         int &y2) const {
        x1 = pi ? ppx : (ppx * k + cx * (mz - k)) / mz;
        y1 = pi ? (ppy * k + cy * (mz - k)) / mz : ppy;
        x2 = pi ? cx : (ppx * k + cx * (mz - k)) / mz;
        y2 = pi ? (ppy * k + cy * (mz - k)) / mz : cy;
        if (x1 < 0 || y1 < 0 || x1 >= X || y1 >= Y) return false;
        if (x1 == ppx && y1 == ppy) return false;
        if (x1 == cx && y1 == cy) return false;
        if (x2 < 0 || y2 < 0 || x2 >= X || y2 >= Y) return false;
        if (x2 == cx && y2 == cy) return false;
        if (x2 == ppx && y2 == ppy) return false;
        return true;
    }

    // DAG nodes of tree node x (one call of the reference's recursive DFS)
    __device__ int visit(int x, int par, int par_node, int slot) {
        const int v = P[x];
        const int cl = v / XY, cx = px(v), cy = py(v);
        const int me = create(cl, cx, cy);
        for (int dir = 0; dir < 2; dir++) {
            w.pl_off[dir * c.tc + x] = 0; w.pl_cnt[dir * c.tc + x] = 0;
            w.nm_off[dir * c.tc + x] = 0; w.nm_cnt[dir * c.tc + x] = 0;
        }
        if (par != -1) {  // every call but the root's receives the parent's places
            for (int dir = 0; dir < 2 && !bad; dir++) {
                const int rid = region_of(w.region[dir * c.tc + x], dir);
                if (rid < 0) continue;
                (void)region_of(w.region[dir * c.tc + par], dir);  // compression only, as the reference's depth test
                int poff, pcnt;
                if (x == rid) {
                    mirror_places(x, dir, poff, pcnt);
                    if (bad) return me;
                } else {
                    poff = w.pl_off[dir * c.tc + par];
                    pcnt = w.pl_cnt[dir * c.tc + par];
                }
                w.pl_off[dir * c.tc + x] = poff;
                w.pl_cnt[dir * c.tc + x] = pcnt;
                const int moff = w.nm_off[dir * c.tc + par], mcnt = w.nm_cnt[dir * c.tc + par];
                if (rid != x && pcnt != mcnt) {  // mirror count mismatch
                    bad = kMalformed;
                    return me;
                }
                if (nmu + pcnt > c.mc) {
                    bad = kTooLarge;
                    return me;
                }
                const int noff = nmu;
                nmu += pcnt;
                w.nm_off[dir * c.tc + x] = noff;
                w.nm_cnt[dir * c.tc + x] = pcnt;
                for (int m = 0; m < pcnt && !bad; m++) {
                    const int place = w.mpool[poff + m];
                    const int nx = dir ? place : cx, ny = dir ? cy : place;
                    int nm;
                    if (rid != x) {
                        nm = create(9, nx, ny);
                        connect(w.mpool[moff + m], nm, slot);
                    } else if (x != root) {
                        const int pxx = px(w.nodes[par_node]), pyy = py(w.nodes[par_node]);
                        if (nx != pxx && ny != pyy) {
                            int tmp[2];
                            for (int pi = 0; pi <= 1; pi++) {
                                const int mx_ = pi ? nx : pxx, my_ = pi ? pyy : ny;
                                tmp[pi] = create(9, mx_, my_);
                                connect(par_node, tmp[pi], slot);
                            }
                            nm = create(9, nx, ny);
                            connect(tmp[0], nm, 0);
                            connect(tmp[1], nm, 0);
                        } else {
                            nm = create(9, nx, ny);
                            connect(par_node, nm, slot);
                        }
                    } else {
                        nm = create(9, nx, ny);
                    }
                    w.mpool[noff + m] = nm;
                }
            }
        }
        if (bad) return me;
        if (par_node != -1) {
            const int ppx = px(w.nodes[par_node]), ppy = py(w.nodes[par_node]);
            if (ppx != cx && ppy != cy) {
                for (int pi = 0; pi <= 1; pi++) {
                    const int mx_ = pi ? cx : ppx, my_ = pi ? ppy : cy;
                    const int pre = create(9, mx_, my_);
                    connect(par_node, pre, slot);
                    connect(pre, me, 0);
                }
                for (int pi = 0; pi <= 1 && !bad; pi++) {
                    const int len = pi ? abs(ppy - cy) : abs(ppx - cx);
                    const int mz = min(zs, len);
                    float rv[10];
                    int rk[10];
#pragma unroll
                    for (int i = 0; i < 10; i++) { rv[i] = 0.f; rk[i] = 0; }  // value-initialised pairs
                    for (int k = 1; k < mz; k++) {
                        int x1, y1, x2, y2;
                        if (!mids(k, pi, mz, ppx, ppy, cx, cy, x1, y1, x2, y2)) continue;
                        int of = 0;  // int += float: the sum is taken in float and truncated
                        of = (int)__fadd_rn((float)of, __fsub_rn(ys(max(x1, x2), max(y1, y2)), ys(min(x1, x2), min(y1, y2))));
                        of = (int)__fadd_rn((float)of, __fsub_rn(ys(max(x1, ppx), max(y1, ppy)), ys(min(x1, ppx), min(y1, ppy))));
                        of = (int)__fadd_rn((float)of, __fsub_rn(ys(max(cx, x2), max(cy, y2)), ys(min(cx, x2), min(cy, y2))));
                        rv[k - 1] = (float)of;
                        rk[k - 1] = k;
                    }
                    // ascending (value, k) over the first mz - 1 entries
                    for (int a2 = 1; a2 < mz - 1; a2++)
                        for (int b2 = a2; b2 > 0 && (rv[b2] < rv[b2 - 1] || (rv[b2] == rv[b2 - 1] && rk[b2] < rk[b2 - 1]));
                             b2--) {
                            const float tv = rv[b2]; rv[b2] = rv[b2 - 1]; rv[b2 - 1] = tv;
                            const int tk = rk[b2]; rk[b2] = rk[b2 - 1]; rk[b2 - 1] = tk;
                        }
                    for (int ii = 0; ii < sel && !bad; ii++) {
                        const int k = rk[ii];
                        int x1, y1, x2, y2;
                        if (mz == 0 || !mids(k, pi, mz, ppx, ppy, cx, cy, x1, y1, x2, y2)) continue;
                        const int p1 = create(9, x1, y1);
                        connect(par_node, p1, slot);
                        if (np >= c.pc) {
                            bad = kTooLarge;
                            return me;
                        }
                        w.pts[np++] = (x1 + x2) / 2 * Y + (y1 + y2) / 2;
                        const int p2 = create(9, x2, y2);
                        connect(p1, p2, 0);
                        connect(p2, me, 0);
                    }
                }
            }
            for (int dir = 0; dir < 2 && !bad; dir++) {
                const int rid = region_of(w.region[dir * c.tc + x], dir);
                const int prid = region_of(w.region[dir * c.tc + par], dir);
                if (prid >= 0 && rid != prid) {
                    const int moff = w.nm_off[dir * c.tc + par], mcnt = w.nm_cnt[dir * c.tc + par];
                    for (int m = 0; m < mcnt && !bad; m++) {
                        const int pm = w.mpool[moff + m];
                        const int mx0 = px(w.nodes[pm]), my0 = py(w.nodes[pm]);
                        if (mx0 != cx && my0 != cy) {
                            for (int pi = 0; pi <= 1; pi++) {
                                const int mx_ = pi ? cx : mx0, my_ = pi ? my0 : cy;
                                const int ni = create(9, mx_, my_);
                                connect(pm, ni, slot);
                                connect(ni, me, 0);
                            }
                        } else {
                            connect(pm, me, slot);
                        }
                    }
                }
            }
            if (ppx == cx || ppy == cy) connect(par_node, me, slot);
        }
        for (int dir = 0; dir < 2 && !bad; dir++) {
            const int rid = region_of(x, dir);
            if (rid < 0) continue;
            if (x != root && cl < 9) {
                const int moff = w.nm_off[dir * c.tc + x], mcnt = w.nm_cnt[dir * c.tc + x];
                for (int m = 0; m < mcnt && !bad; m++) {
                    const int dup = create(cl, cx, cy);
                    connect(w.mpool[moff + m], dup, deg(x) - 1);
                }
            }
        }
        return me;
    }

    __device__ void dfs_all() {
        int top = 0;
        w.pe[0] = root; w.pp[0] = -1; w.ppn[0] = -1; w.ps[0] = -1;
        top = 1;
        while (top > 0 && !bad) {
            top--;
            const int x = w.pe[top], par = w.pp[top], par_node = w.ppn[top], slot = w.ps[top];
            const int me = visit(x, par, par_node, slot);
            if (bad) return;
            int cnt = 0;
            for (int q = ao[x]; q < ao[x + 1]; q++) cnt += nbr(q) != par;
            if (top + cnt > c.tc) {  // each tree node is pending once: not a tree
                bad = kMalformed;
                return;
            }
            // children in adjacency order: pushed last to first
            for (int q = ao[x + 1] - 1; q >= ao[x]; q--) {
                const int e = nbr(q);
                if (e == par) continue;
                cnt--;
                w.pe[top] = e; w.pp[top] = x; w.ppn[top] = me; w.ps[top] = cnt;
                top++;
            }
        }
    }

    // parents-first renumbering (:2027-2085); par/cidx (when given) receive
    // each node's parent slots in the new numbering
    __device__ void renumber(int *par, int *cidx) {
        const int cnt = nn;
        for (int i = 0; i <= cnt; i++) w.poff[i] = 0;
        for (int l = 0; l < nl; l++) w.poff[w.lc[l] + 1]++;
        for (int i = 0; i < cnt; i++) w.poff[i + 1] += w.poff[i];
        for (int i = 0; i < cnt; i++) w.at[i] = w.poff[i];
        for (int l = 0; l < nl; l++) w.pcode[w.at[w.lc[l]]++] = w.lp[l];
        for (int i = 0; i < cnt; i++) { w.visit[i] = 0; w.newid[i] = 0; w.dep[i] = 0; w.cn[i] = 0; }
        int otop = 0;
        for (int i = 0; i < cnt && !bad; i++) {
            if (w.child_pre[i] != 0) continue;
            if (otop >= cnt) { bad = kMalformed; return; }
            w.ord[otop++] = i;
            int stop = 0;
            w.stn[0] = i; w.stq[0] = w.poff[i];
            stop = 1;
            while (stop > 0) {
                const int f = stop - 1;
                if (w.stq[f] >= w.poff[w.stn[f] + 1]) { stop--; continue; }
                const int p = w.pcode[w.stq[f]++] / 10;
                if (p < 0 || p >= cnt) { bad = kMalformed; return; }
                if (++w.visit[p] == w.child_pre[p]) {
                    if (otop >= cnt || stop >= cnt) { bad = kMalformed; return; }
                    w.ord[otop++] = p;
                    w.stn[stop] = p; w.stq[stop] = w.poff[p];
                    stop++;
                }
            }
        }
        if (otop != cnt) {  // not acyclic
            bad = kMalformed;
            return;
        }
        int k = 0, e = 0;
        while (otop > 0) {
            const int idx = w.ord[--otop];
            for (int q = w.poff[idx]; q < w.poff[idx + 1]; q++) {
                const int code = w.pcode[q];
                const int p = code / 10, sl = code % 10;
                const int sp = w.newid[p];
                w.cn[sp] = max(w.cn[sp], sl + 1);
                if (par) { par[e] = sp; cidx[e] = sl; }
                e++;
                w.dep[k] = max(w.dep[k], w.dep[sp] + 1);
            }
            w.newid[idx] = k;
            w.pn[k] = w.poff[idx + 1] - w.poff[idx];
            w.onode[k] = w.nodes[idx];
            k++;
        }
    }
};

// Builds DAGs i = t, t + nt, ... of the list with work area w.
__device__ void build_dags(const DagBuildArgs &a, const Work &w, int t, int nt) {
    const DagCaps c = a.caps;
    const int XY = a.X * a.Y;
    for (int i = t; i < a.n_list; i += nt) {
        const int k = a.list ? a.list[i] : i;
        const int id = a.ids[k];
        const int b = a.tree_off[id], T = a.tree_off[id + 1] - b;
        Builder B{w, c, a.pos + b, a.adj_off + b, a.adj, a.xsum, a.ysum, T, a.X, a.Y, XY};
        B.ratio = 0.15f;
        B.num_tracks = 9;
        B.zs = 10;
        B.sel = 10;
        if (a.mode == 0 || a.mode == 1) {
            B.ratio = 0.1f;
            B.num_tracks = 6;
            B.zs = 7;
            B.sel = 2;
        }
        if (T > c.tc) B.bad = kTooLarge;
        if (!B.bad && T < 2) B.bad = kMalformed;
        for (int q = B.ao[0]; q < B.ao[T] && !B.bad; q++)
            if (a.adj[q] < 0 || a.adj[q] >= T) B.bad = kMalformed;
        if (!B.bad) {
            B.root = B.select_root();
            if (B.root < 0 && !B.bad) B.bad = kMalformed;  // a tree without leaves
        }
        if (!B.bad) {
            for (int dir = 0; dir < 2; dir++)
                for (int x = 0; x < T; x++) {
                    w.region[dir * c.tc + x] = -1;
                    w.shead[dir * c.tc + x] = -1;
                }
            for (int x = 0; x < T && !B.bad; x++) {
                const int v = B.P[x], cl = v / XY, cx = B.px(v), cy = B.py(v);
                for (int dir = 0; dir < 2; dir++) {
                    if (cl < 9) B.stem_push(dir, x, dir ? cx : cy);
                    const int tt = dir ? cy : cx;
                    w.rlo[dir * c.tc + x] = tt;
                    w.rhi[dir * c.tc + x] = tt;
                }
            }
        }
        if (!B.bad) B.mark_all();
        if (!B.bad) B.dfs_all();
        int npu = 0;
        if (!B.bad) {
            heap_sort(w.pts, B.np);
            for (int q = 0; q < B.np; q++)
                if (npu == 0 || w.pts[q] != w.pts[npu - 1]) w.pts[npu++] = w.pts[q];
        }
        // place the DAG: node, edge and point ranges reserved in the pools
        // (their order varies from run to run; every reader goes through the
        // per-DAG offsets, so results do not)
        long long no = 0, eo = 0, po = 0;
        if (!B.bad) {
            no = (long long)atomicAdd(a.used + 0, (unsigned long long)B.nn);
            eo = (long long)atomicAdd(a.used + 1, (unsigned long long)B.nl);
            po = (long long)atomicAdd(a.used + 2, (unsigned long long)npu);
            if (no + B.nn > a.cap_nodes || eo + B.nl > a.cap_edges || po + npu > a.cap_points) B.bad = kPoolFull;
        }
        if (!B.bad) B.renumber(a.out_par + eo, a.out_child_idx + eo);
        int D = 0, S = 0, mc = 0;
        if (!B.bad) {
            for (int v = 0; v < B.nn; v++) {
                a.out_nodes[no + v] = w.onode[v];
                a.out_par_num[no + v] = w.pn[v];
                a.out_child_num[no + v] = w.cn[v];
                a.out_depth[no + v] = w.dep[v];
                D = max(D, w.dep[v] + 1);
                S += w.cn[v];
                mc = max(mc, w.cn[v]);
            }
            for (int q = 0; q < npu; q++) a.out_points[po + q] = w.pts[q];
        }
        int *sz = a.sizes + (size_t)k * kDagSizeFields;
        sz[0] = B.bad ? 0 : B.nn;
        sz[1] = B.bad ? 0 : B.nl;
        sz[2] = B.bad ? 0 : npu;
        sz[3] = D;
        sz[4] = S;
        sz[5] = mc;
        sz[6] = B.bad;
        a.node_at[k] = no;
        a.edge_at[k] = eo;
        a.point_at[k] = po;
    }
}

// one builder per thread, work areas in global memory
__global__ void __launch_bounds__(128) dag_build_kernel(DagBuildArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    build_dags(a, carve(a.work + (long long)t * work_ints(a.caps), a.caps), t, gridDim.x * blockDim.x);
}

// one builder per block (its first thread) for the large DAGs: the work area
// in shared memory when a.work is null, else in global memory; few builders
// run per SM, so that their dependent accesses stay on chip
__global__ void __launch_bounds__(32) dag_build_solo_kernel(DagBuildArgs a) {
    extern __shared__ int smem[];
    if (threadIdx.x != 0) return;
    const int t = blockIdx.x;
    build_dags(a, carve(a.work ? a.work + (long long)t * work_ints(a.caps) : smem, a.caps), t, gridDim.x);
}

// One thread per net of the batch layout: copies its DAG from the per-net
// arrays into the batch-local arrays of the DAG router (the layout the host
// builds in the reference-order path: nodes, parent CSR with child slots and
// edge children, child-slot offsets, per-depth node lists).
__global__ void dag_gather_kernel(DagGatherArgs a) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n) return;
    const int *d = a.desc + (size_t)j * kDagDescFields;
    const int k = d[0], base = d[1], ebl = d[2], sl0 = d[3], lvb = d[4], jl = d[5], b = d[6];
    const int *bi = a.batch + (size_t)b * kDagBatchFields;  // nb, eb, pb, lb, nnb, nets
    const long long no = a.node_at[k], eo = a.edge_at[k];
    const int m = a.sizes[(size_t)k * kDagSizeFields];
    const int nb0 = bi[0] + base, eb0 = bi[1] + ebl, pb0 = bi[2] + base, lb0 = bi[3] + lvb, nnb0 = bi[4] + jl;
    if (jl == 0) {
        a.par_off[bi[2]] = 0;
        a.child_off[bi[2]] = 0;
        a.net_node_off[bi[4]] = 0;
        a.net_level_off[bi[4]] = 0;
    }
    int e = 0, sl = sl0, D = 0;
    for (int v = 0; v < m; v++) {
        a.nodes[nb0 + v] = a.src_nodes[no + v];
        const int pn = a.src_par_num[no + v];
        for (int q = 0; q < pn; q++) {
            a.par[eb0 + e] = base + a.src_par[eo + e];
            a.child_slot[eb0 + e] = a.src_child_idx[eo + e];
            a.edge_child[eb0 + e] = base + v;
            e++;
        }
        a.par_off[pb0 + v + 1] = ebl + e;
        sl += a.src_child_num[no + v];
        a.child_off[pb0 + v + 1] = sl;
        D = max(D, a.src_depth[no + v] + 1);
    }
    // per-depth lists: level_off[d] = first position of depth d, nodes of
    // one depth in node order
    int pos = base;
    for (int dd = 0; dd < D; dd++) {
        a.level_off[lb0 + dd] = pos;
        for (int v = 0; v < m; v++)
            if (a.src_depth[no + v] == dd) a.level_nodes[bi[0] + pos++] = base + v;
    }
    a.level_off[lb0 + D] = pos;
    a.net_node_off[nnb0 + 1] = base + m;
    a.net_ids[bi[5] + jl] = a.ids[k];
    a.net_level_off[nnb0 + 1] = lvb + D + 1;
}

}  // namespace

long long dag_work_ints(const DagCaps &c) { return work_ints(c); }

void launch_dag_build(const DagBuildArgs &a, int threads, cudaStream_t s) {
    if (a.n_list <= 0) return;
    // the work area holds `threads` slices (a multiple of 128)
    const int blocks = std::min(threads / 128, (a.n_list + 127) / 128);
    if (blocks < 1) return;
    dag_build_kernel<<<blocks, 128, 0, s>>>(a);
}

int dag_solo_smem_limit() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

void launch_dag_build_solo(const DagBuildArgs &a, int builders, cudaStream_t s) {
    if (a.n_list <= 0 || builders <= 0) return;
    const int blocks = std::min(builders, a.n_list);
    size_t smem = 0;
    if (!a.work) {
        smem = (size_t)work_ints(a.caps) * sizeof(int);
        kernel_setup((const void *)dag_build_solo_kernel, 32, smem);
    }
    dag_build_solo_kernel<<<blocks, 32, smem, s>>>(a);
}

void launch_dag_gather(const DagGatherArgs &a, cudaStream_t s) {
    if (a.n <= 0) return;
    dag_gather_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(a);
}

}  // namespace igr
