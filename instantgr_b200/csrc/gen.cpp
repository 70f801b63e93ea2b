// Seeded synthetic ISPD2024-format designs.
//
// The ISPD2024 suite and the reference's bundled example are not available, so
// designs with the stated shapes and distributions are generated from a seed:
// 10 layers, file layer 0 pin-only (capacity 0), layers 1..9 alternate H/V
// starting with H, GCell edges of length 1, unit wire cost 1, via cost 2,
// overflow weight 1 per layer.  Every random draw comes from SplitMix64 on a
// counter (state += 0x9E3779B97F4A7C15, then the SplitMix64 finaliser).
#include "host.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace igr {

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x2545F4914F6CDD1DULL + 0x9E3779B97F4A7C15ULL) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    int range(int lo, int hi) { return lo + (int)(next() % (uint64_t)(hi - lo + 1)); }  // [lo,hi]
    double normal() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct Out {
    FILE *f;
    std::vector<char> buf;
    explicit Out(const char *path) : f(std::fopen(path, "wb")) {
        if (!f) throw Error(ERR_IO, std::string("cannot open ") + path);
        buf.reserve(1 << 22);
    }
    ~Out() { flush(); if (f) std::fclose(f); }
    void flush() {
        if (!buf.empty()) std::fwrite(buf.data(), 1, buf.size(), f);
        buf.clear();
    }
    void s(const char *t) { buf.insert(buf.end(), t, t + std::strlen(t)); if (buf.size() > (1 << 22)) flush(); }
    void i(long long v) {
        char t[24];
        int n = std::snprintf(t, sizeof t, "%lld", v);
        buf.insert(buf.end(), t, t + n);
    }
    void c(char ch) { buf.push_back(ch); }
};

int pin_count(const GenParams &p, Rng &r) {
    if (p.pin_mode == 1) {
        double u = r.uni();
        if (u < 0.70) return 2;
        if (u < 0.90) return r.range(3, 8);
        if (u < 0.995) return r.range(9, 64);
        return r.range(65, 1000);
    }
    if (p.hifanout_frac > 0 && r.uni() < p.hifanout_frac) return -r.range(65, 500);  // negative: high fanout
    int k = 2;
    while (k < 64 && r.uni() < 0.5) k++;
    return k;
}

}  // namespace

void generate_design(const GenParams &p, const char *cap_path, const char *net_path) {
    const int X = p.X, Y = p.Y, L = 10;
    if (X < 2 || Y < 2) throw Error(ERR_INVALID, "grid must be at least 2x2");
    Rng rng(p.seed);
    // ---------------- capacities [l][x][y]
    std::vector<int> cap((size_t)L * X * Y, 0);
    for (int l = 1; l < L; l++) {
        int *c = cap.data() + (size_t)l * X * Y;
        for (size_t i = 0; i < (size_t)X * Y; i++) {
            if (p.cap_mode == 0) c[i] = rng.range(4, 12);
            else {
                int mean = (int)std::lround(10.0 - 6.0 * (l - 1) / 8.0);
                c[i] = std::max(0, mean + rng.range(-2, 2));
            }
        }
    }
    if (p.block_frac > 0) {
        const double target = p.block_frac * 9.0 * X * Y;
        double zeroed = 0;
        int guard = 0;
        while (zeroed < target && guard++ < 10000000) {
            int l = rng.range(1, L - 1), w = rng.range(4, 32), h = rng.range(4, 32);
            int x0 = rng.range(0, std::max(0, X - w)), y0 = rng.range(0, std::max(0, Y - h));
            int *c = cap.data() + (size_t)l * X * Y;
            for (int x = x0; x < std::min(X, x0 + w); x++)
                for (int y = y0; y < std::min(Y, y0 + h); y++)
                    if (c[(size_t)x * Y + y] != 0) { c[(size_t)x * Y + y] = 0; zeroed += 1; }
        }
    }
    // window written (the whole grid by default)
    const bool win = p.win_w > 0 && p.win_h > 0;
    const int wx0 = win ? p.win_x0 : 0, wy0 = win ? p.win_y0 : 0, WX = win ? p.win_w : X, WY = win ? p.win_h : Y;
    if (wx0 < 0 || wy0 < 0 || WX < 2 || WY < 2 || wx0 + WX > X || wy0 + WY > Y)
        throw Error(ERR_INVALID, "window must lie inside the grid and be at least 2x2");
    {
        Out o(cap_path);
        o.i(L); o.c(' '); o.i(WX); o.c(' '); o.i(WY); o.c('\n');
        o.s("1 2");
        for (int l = 0; l < L; l++) o.s(" 1");
        o.c('\n');
        for (int x = 0; x < WX - 1; x++) { if (x) o.c(' '); o.c('1'); }
        o.c('\n');
        for (int y = 0; y < WY - 1; y++) { if (y) o.c(' '); o.c('1'); }
        o.c('\n');
        for (int l = 0; l < L; l++) {
            o.s("metal"); o.i(l + 1); o.c(' ');
            o.i(l == 0 ? 1 : ((l - 1) & 1));  // layer 1 horizontal, alternate; layer 0 opposite of layer 1
            o.s(" 0\n");
            const int *c = cap.data() + (size_t)l * X * Y;
            for (int y = wy0; y < wy0 + WY; y++) {
                for (int x = wx0; x < wx0 + WX; x++) { if (x > wx0) o.c(' '); o.i(c[(size_t)x * Y + y]); }
                o.c('\n');
            }
        }
    }
    // ---------------- nets
    std::vector<double> hx, hy;
    for (int h = 0; h < p.hotspots; h++) { hx.push_back(rng.uni() * X); hy.push_back(rng.uni() * Y); }
    Out o(net_path);
    std::vector<std::pair<int, int>> used;
    std::vector<std::array<int, 3>> aps;  // access points (layer, x, y) of the net being drawn
    std::vector<int> pin_end;             // end of each pin's access points in aps
    for (int n = 0; n < p.nets; n++) {
        int k = pin_count(p, rng);
        bool hf = k < 0;
        if (hf) k = -k;
        double cx, cy;
        if (!hx.empty() && rng.uni() < p.hotspot_frac) {
            int h = (int)(rng.next() % hx.size());
            // centres off the grid are drawn again (clamping them would pile
            // the boxes of a hotspot near a corner onto the grid boundary)
            int tries = 0;
            do {
                cx = hx[h] + rng.normal() * p.hotspot_sigma;
                cy = hy[h] + rng.normal() * p.hotspot_sigma;
            } while ((cx < 0 || cx >= X || cy < 0 || cy >= Y) && ++tries < 16);
            if (tries == 16) {
                cx = rng.uni() * X;
                cy = rng.uni() * Y;
            }
        } else {
            cx = rng.uni() * X;
            cy = rng.uni() * Y;
        }
        int w, h;
        if (hf) {
            w = rng.range(std::min(50, p.hifanout_bbox), p.hifanout_bbox);
            h = rng.range(std::min(50, p.hifanout_bbox), p.hifanout_bbox);
        } else {
            w = (int)std::lround(p.bbox_median * std::exp(p.bbox_sigma * rng.normal()));
            h = (int)std::lround(p.bbox_median * std::exp(p.bbox_sigma * rng.normal()));
        }
        w = std::max(1, std::min(X, w));
        h = std::max(1, std::min(Y, h));
        // room for every pin on a GCell of its own (access points of different
        // pins never share a GCell, as in ISPD2024 designs)
        while ((int64_t)w * h < 4LL * k && (w < X || h < Y)) {
            if (w < X) w++;
            if (h < Y) h++;
        }
        int x0 = std::max(0, std::min(X - w, (int)std::lround(cx - w / 2.0)));
        int y0 = std::max(0, std::min(Y - h, (int)std::lround(cy - h / 2.0)));
        used.clear();
        aps.clear();
        pin_end.clear();
        auto taken = [&](int x, int y) { return std::find(used.begin(), used.end(), std::make_pair(x, y)) != used.end(); };
        for (int q = 0; q < k; q++) {
            int px = -1, py = -1;
            for (int t = 0; t < 64; t++) {
                int cx2 = x0 + rng.range(0, w - 1), cy2 = y0 + rng.range(0, h - 1);
                if (!taken(cx2, cy2)) { px = cx2; py = cy2; break; }
            }
            if (px < 0)  // dense box: first free GCell in scan order
                for (int x = x0; x < x0 + w && px < 0; x++)
                    for (int y = y0; y < y0 + h; y++)
                        if (!taken(x, y)) { px = x; py = y; break; }
            if (px < 0) break;  // the whole box is used: fewer pins
            int nap = rng.range(1, 3);
            static const int dx[4] = {1, -1, 0, 0}, dy[4] = {0, 0, 1, -1};
            int ax = px, ay = py;
            for (int a = 0; a < nap; a++) {
                if (a > 0) {  // a neighbouring GCell not used by any pin of the net yet
                    bool ok = false;
                    for (int t = 0; t < 8 && !ok; t++) {
                        int dd = rng.range(0, 3);
                        int nx = px + dx[dd], ny = py + dy[dd];
                        if (nx < 0 || ny < 0 || nx >= X || ny >= Y) continue;
                        if (taken(nx, ny)) continue;
                        ax = nx; ay = ny; ok = true;
                    }
                    if (!ok) break;
                }
                used.push_back({ax, ay});
                aps.push_back({rng.range(0, 1), ax, ay});
            }
            pin_end.push_back((int)aps.size());
        }
        bool inside = true;
        for (auto &a : aps)
            inside = inside && a[1] >= wx0 && a[1] < wx0 + WX && a[2] >= wy0 && a[2] < wy0 + WY;
        if (!inside) continue;
        o.s("net"); o.i(n); o.s("\n(\n");
        for (size_t q = 0, a = 0; q < pin_end.size(); q++) {
            o.c('[');
            for (size_t b = a; b < (size_t)pin_end[q]; b++) {
                if (b > a) o.s(", ");
                o.c('('); o.i(aps[b][0]); o.s(", "); o.i(aps[b][1] - wx0); o.s(", "); o.i(aps[b][2] - wy0); o.c(')');
            }
            o.s("]\n");
            a = (size_t)pin_end[q];
        }
        o.s(")\n");
    }
}

GenParams custom_params(int X, int Y, int nets, uint64_t seed, int cap_mode, double block_frac, int pin_mode,
                        double hifanout_frac, double bbox_median, double bbox_sigma, int hotspots, double hotspot_frac) {
    GenParams p;
    p.X = X; p.Y = Y; p.nets = nets; p.seed = seed; p.cap_mode = cap_mode; p.block_frac = block_frac;
    p.pin_mode = pin_mode; p.hifanout_frac = hifanout_frac; p.bbox_median = bbox_median;
    p.bbox_sigma = bbox_sigma; p.hotspots = hotspots; p.hotspot_frac = hotspot_frac;
    p.hotspot_sigma = 0.1 * std::max(X, Y);
    return p;
}

GenParams config_params(int cfg, uint64_t seed, double scale) {
    if (scale <= 0 || scale > 1) throw Error(ERR_INVALID, "scale must be in (0, 1]");
    auto nn = [&](int n) { return std::max(2, (int)(n * scale)); };
    switch (cfg) {
        case 0: return custom_params(256, 256, nn(20000), seed, 0, 0.05, 0, 0, 8, 1.0, 0, 0);
        case 1: return custom_params(840, 1140, nn(130000), seed, 1, 0, 0, 0.01, 8, 1.0, 0, 0);
        case 2: return custom_params(1600, 1600, nn(800000), seed, 1, 0, 1, 0, 10, 1.2, 6, 0.35);
        case 3: return custom_params(512, 512, nn(40000), seed, 1, 0, 1, 0, 10, 1.2, 6, 0.35);
        case 4: return custom_params(3000, 3000, nn(10000000), seed, 1, 0, 1, 0, 10, 1.2, 4, 0.40);
        default: throw Error(ERR_INVALID, "unknown configuration");
    }
}

}  // namespace igr
