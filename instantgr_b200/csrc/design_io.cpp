// ISPD2024 .cap/.net reader and route-guide writer.
//
// The reader follows the scanner of InstantGR (src/database.hpp:247-409) token
// for token: integers are runs of digits (anything else is skipped, so signs
// are ignored), reals are runs of digits and '.', names run up to the next
// space or newline.  The .net file is cut at net boundaries ("\n)\n") and the
// pieces are parsed on several threads, then concatenated in file order.
//
// The writer emits guides in the line format of src/graph.hpp:179-235
// ("x0 y0 l0 x1 y1 l1", the lower 3-D position first); nets are written in
// design order by a parallel formatter followed by one fwrite per chunk.
#include "host.hpp"

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <thread>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <memory>

namespace igr {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int hw_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)n : 1;
}

void parallel_for(int n, int threads, const std::function<void(int, int)> &fn) {
    if (n <= 0) return;
    if (threads <= 0) threads = hw_threads();
    threads = std::min(threads, n);
    if (threads <= 1) { fn(0, n); return; }
    // ranges are handed out dynamically, about eight per thread, so that items
    // of very different cost (a 500-pin net beside two-pin nets) balance
    const int chunk = std::max(1, n / (threads * 8));
    std::atomic<int> next{0};
    std::vector<std::exception_ptr> errs(threads);
    auto work = [&](int t) {
        try {
            for (int b; (b = next.fetch_add(chunk)) < n;) fn(b, std::min(n, b + chunk));
        } catch (...) {
            errs[t] = std::current_exception();
            next.store(n);
        }
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < threads; t++) ts.emplace_back(work, t);
    work(0);
    for (auto &t : ts) t.join();
    for (auto &e : errs) if (e) std::rethrow_exception(e);
}

namespace {

std::vector<char> slurp(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) throw Error(ERR_IO, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)sz + 1);
    if (sz > 0 && std::fread(buf.data(), 1, (size_t)sz, f) != (size_t)sz) {
        std::fclose(f);
        throw Error(ERR_IO, std::string("short read on ") + path);
    }
    std::fclose(f);
    buf[(size_t)sz] = 0;
    buf.resize((size_t)sz + 1);
    return buf;
}

inline bool is_dig(char c) { return c >= '0' && c <= '9'; }

struct Scanner {
    const char *b;
    size_t n, p = 0;
    Scanner(const char *buf, size_t len) : b(buf), n(len) {}
    void need() {
        if (p >= n) throw Error(ERR_FORMAT, "unexpected end of input");
    }
    int read_int() {
        while (p < n && !is_dig(b[p])) p++;
        need();
        long long v = 0;
        for (; p < n && is_dig(b[p]); p++) v = v * 10 + (b[p] - '0');
        return (int)v;
    }
    double read_double() {
        while (p < n && !is_dig(b[p])) p++;
        need();
        double ans = 0, scale = 0;
        for (; p < n && (is_dig(b[p]) || b[p] == '.'); p++) {
            if (b[p] == '.') scale = 1;
            else scale *= 10, ans = ans * 10 + (b[p] - '0');
        }
        return scale == 0 ? ans : ans / scale;
    }
    void read_token(size_t &beg, size_t &end) {
        while (p < n && (b[p] == ' ' || b[p] == '\n')) p++;
        need();
        beg = p;
        while (p < n && b[p] != ' ' && b[p] != '\n') p++;
        end = p;
    }
};

inline bool in_run(char c) { return is_dig(c) || c == '.'; }

// The capacity values of all layers, parsed on several threads.  The layer
// headers are read in order; a layer's values run up to the next layer name.
// Each value section is cut into pieces at blanks (a blank never lies inside
// a number, which is a digit followed by digits and dots); the numbers of
// every piece are counted, then parsed with the scanner's arithmetic into
// their places.  Returns false, having stored nothing that the sequential
// reader would not, unless every section holds exactly X*Y numbers and only
// blanks follow the last one before the next name: the caller then reads the
// layers sequentially, which also produces the errors of malformed files.
bool cap_layers_parallel(Design &d, const char *buf, size_t n, size_t p0, int threads) {
    const int L = d.L;
    const size_t XY = (size_t)d.X * d.Y;
    std::vector<size_t> beg(L), end(L);
    std::vector<int> dir(L);
    std::vector<double> minlen(L);
    Scanner t(buf, n);
    t.p = p0;
    try {
        for (int l = 0; l < L; l++) {
            size_t b, e;
            t.read_token(b, e);
            if (std::string(buf + b, buf + e) != "metal" + std::to_string(l + 1)) return false;
            dir[l] = t.read_int();
            minlen[l] = t.read_double();
            if (l && dir[l] == dir[l - 1]) return false;
            beg[l] = t.p;
            if (l + 1 < L) {
                const std::string next = "metal" + std::to_string(l + 2);
                const void *f = memmem(buf + beg[l], n - beg[l], next.data(), next.size());
                if (!f) return false;
                end[l] = (size_t)((const char *)f - buf);
                t.p = end[l];
            } else {
                end[l] = n;
            }
        }
    } catch (const Error &) {
        return false;
    }
    // pieces of 4 KB to 1 MB (about four per thread and section), cut at a blank
    struct Piece { int l; size_t a, e; int64_t first, count; size_t last; };
    std::vector<Piece> pc;
    const size_t T = (size_t)(threads > 0 ? threads : hw_threads());
    for (int l = 0; l < L; l++) {
        const size_t len = std::min<size_t>((size_t)1 << 20, std::max<size_t>(4096, (end[l] - beg[l]) / (4 * T)));
        size_t a = beg[l];
        while (a < end[l]) {
            size_t e = std::min(end[l], a + len);
            while (e < end[l] && buf[e] != ' ' && buf[e] != '\n') e++;
            pc.push_back({l, a, e, 0, 0, a});
            a = e;
        }
    }
    const int P = (int)pc.size();
    parallel_for(P, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) {
            Piece &q = pc[i];
            int64_t c = 0;
            bool run = false;
            for (size_t k = q.a; k < q.e; k++) {
                const char ch = buf[k];
                if (run) {
                    run = in_run(ch);
                } else if (is_dig(ch)) {
                    run = true;
                    c++;
                }
            }
            q.count = c;
        }
    });
    for (int l = 0, i = 0; l < L; l++) {
        int64_t c = 0;
        for (; i < P && pc[i].l == l; i++) {
            pc[i].first = c;
            c += pc[i].count;
        }
        if (c != (int64_t)XY) return false;
    }
    const int X = d.X, Y = d.Y;
    std::atomic<bool> inexact{false};
    parallel_for(P, threads, [&](int b, int e) {
        for (int i = b; i < e; i++) {
            Piece &q = pc[i];
            float *cap = d.cap.data() + (size_t)q.l * XY;
            int64_t idx = q.first;
            size_t k = q.a;
            while (k < q.e) {
                if (!is_dig(buf[k])) { k++; continue; }
                double ans = 0, scale = 0;
                for (; k < q.e && in_run(buf[k]); k++) {
                    if (buf[k] == '.') scale = 1;
                    else scale *= 10, ans = ans * 10 + (buf[k] - '0');
                }
                const int y = (int)(idx / X), x = (int)(idx % X);
                const double v = scale == 0 ? ans : ans / scale;
                cap[(size_t)x * Y + y] = (float)v;
                if ((double)(float)v != v) inexact = true;
                idx++;
                q.last = k;
            }
        }
    });
    // only blanks between a section's last number and the next layer name
    for (int l = 0, i = 0; l + 1 < L; l++) {
        size_t last = beg[l];
        for (; i < P && pc[i].l == l; i++)
            if (pc[i].count) last = pc[i].last;
        for (size_t k = last; k < end[l]; k++)
            if (buf[k] != ' ' && buf[k] != '\n') {
                std::fill(d.cap.begin(), d.cap.end(), 0.f);
                return false;
            }
    }
    for (int l = 0; l < L; l++) {
        d.layer_dir[l] = dir[l];
        d.layer_min_len[l] = minlen[l];
    }
    if (inexact) {  // rare: the exact values as well
        d.cap_d.assign(d.cap.size(), 0.0);
        parallel_for(P, threads, [&](int b, int e) {
            for (int i = b; i < e; i++) {
                const Piece &q = pc[i];
                double *cap = d.cap_d.data() + (size_t)q.l * XY;
                int64_t idx = q.first;
                for (size_t k = q.a; k < q.e;) {
                    if (!is_dig(buf[k])) { k++; continue; }
                    double ans = 0, scale = 0;
                    for (; k < q.e && in_run(buf[k]); k++) {
                        if (buf[k] == '.') scale = 1;
                        else scale *= 10, ans = ans * 10 + (buf[k] - '0');
                    }
                    cap[(size_t)(idx % X) * Y + (size_t)(idx / X)] = scale == 0 ? ans : ans / scale;
                    idx++;
                }
            }
        });
    }
    return true;
}

}  // namespace

void read_cap_buffer(Design &d, const char *buf, size_t n, int threads) {
    Scanner s(buf, n);
    d.L = s.read_int();
    d.X = s.read_int();
    d.Y = s.read_int();
    if (d.L != 10) throw Error(ERR_FORMAT, "the .cap file must have 10 layers");
    if (d.X < 2 || d.Y < 2) throw Error(ERR_FORMAT, "grid must be at least 2x2");
    if ((int64_t)d.L * d.X * d.Y > (int64_t)2000000000) throw Error(ERR_CAPACITY, "grid too large for 32-bit positions");
    d.unit_wire = s.read_double();
    d.unit_via = s.read_double();
    d.short_cost.resize(d.L);
    for (int i = 0; i < d.L; i++) d.short_cost[i] = s.read_double();
    d.x_edge_len.resize(d.X - 1);
    d.y_edge_len.resize(d.Y - 1);
    for (int i = 0; i < d.X - 1; i++) d.x_edge_len[i] = s.read_int();
    for (int i = 0; i < d.Y - 1; i++) d.y_edge_len[i] = s.read_int();
    d.dr_x.assign(d.X, 0);
    d.dr_y.assign(d.Y, 0);
    for (int i = 0; i < d.X - 1; i++) d.dr_x[i + 1] = d.dr_x[i] + d.x_edge_len[i];
    for (int i = 0; i < d.Y - 1; i++) d.dr_y[i + 1] = d.dr_y[i] + d.y_edge_len[i];
    d.dr2gr_x.assign(d.dr_x.back() + 1, -1);
    d.dr2gr_y.assign(d.dr_y.back() + 1, -1);
    for (int i = 0; i < d.X; i++) d.dr2gr_x[d.dr_x[i]] = i;
    for (int i = 0; i < d.Y; i++) d.dr2gr_y[d.dr_y[i]] = i;
    d.layer_dir.resize(d.L);
    d.layer_min_len.resize(d.L);
    d.cap.assign((size_t)d.L * d.X * d.Y, 0.f);
    d.cap_d.clear();
    if (cap_layers_parallel(d, buf, n, s.p, threads)) return;
    for (int l = 0; l < d.L; l++) {
        size_t b, e;
        s.read_token(b, e);
        std::string name(buf + b, buf + e), want = "metal" + std::to_string(l + 1);
        if (name != want) throw Error(ERR_FORMAT, "expected layer " + want + ", got " + name);
        d.layer_dir[l] = s.read_int();
        d.layer_min_len[l] = s.read_double();
        float *c = d.cap.data() + (size_t)l * d.X * d.Y;
        for (int y = 0; y < d.Y; y++)
            for (int x = 0; x < d.X; x++) {
                const double v = s.read_double();
                c[(size_t)x * d.Y + y] = (float)v;
                if ((double)(float)v != v) {
                    if (d.cap_d.empty()) {  // rare: keep the exact values as well
                        d.cap_d.resize(d.cap.size());
                        for (size_t i = 0; i < d.cap.size(); i++) d.cap_d[i] = d.cap[i];
                    }
                }
                if (!d.cap_d.empty()) d.cap_d[(size_t)l * d.X * d.Y + (size_t)x * d.Y + y] = v;
            }
        if (l && d.layer_dir[l] == d.layer_dir[l - 1])
            throw Error(ERR_FORMAT, "layer directions must alternate");
    }
}

namespace {

struct NetChunk {
    std::vector<char> names;
    std::vector<int64_t> name_len;
    std::vector<int> pins_per_net;
    std::vector<int> aps_per_pin;
    std::vector<int> ap;
    std::vector<int> bb;  // minx maxx miny maxy per net
};

void parse_net_chunk(const Design &d, const char *buf, size_t n, NetChunk &c) {
    Scanner s(buf, n);
    const int X = d.X, Y = d.Y, L = d.L;
    while (s.p < n && (buf[s.p] == ' ' || buf[s.p] == '\n')) s.p++;
    while (s.p < n) {
        size_t b, e;
        s.read_token(b, e);
        c.names.insert(c.names.end(), buf + b, buf + e);
        c.name_len.push_back((int64_t)(e - b));
        int minx = X, maxx = 0, miny = Y, maxy = 0, npin = 0;
        while (true) {  // pins
            int nap = 0;
            while (true) {  // access points
                int l = s.read_int(), x = s.read_int(), y = s.read_int();
                if (l >= L || x >= X || y >= Y) throw Error(ERR_FORMAT, "access point outside the grid");
                minx = std::min(minx, x); maxx = std::max(maxx, x);
                miny = std::min(miny, y); maxy = std::max(maxy, y);
                c.ap.push_back(l * X * Y + x * Y + y);
                if (++nap >= 20) throw Error(ERR_FORMAT, "more than 19 access points in a pin");
                bool pin_end = false;
                while (s.p < n && !is_dig(buf[s.p]))
                    if (buf[s.p++] == ']') { pin_end = true; break; }
                if (pin_end) break;
                s.need();
            }
            c.aps_per_pin.push_back(nap);
            npin++;
            bool net_end = false;
            while (s.p < n && !is_dig(buf[s.p]))
                if (buf[s.p++] == ')') { net_end = true; break; }
            if (net_end) break;
            s.need();
        }
        c.pins_per_net.push_back(npin);
        c.bb.insert(c.bb.end(), {minx, maxx, miny, maxy});
        while (s.p < n && (buf[s.p] == ' ' || buf[s.p] == '\n')) s.p++;
    }
}

}  // namespace

void read_net_buffer(Design &d, const char *buf, size_t n) {
    // Cut at "\n)\n" boundaries so that every piece holds whole nets.
    int T = std::max(1, std::min(hw_threads(), (int)(n / (1 << 20)) + 1));
    std::vector<size_t> cut{0};
    for (int t = 1; t < T; t++) {
        size_t g = std::max(cut.back(), n * t / T);
        const char *hit = nullptr;
        for (size_t p = g; p + 2 < n; p++)
            if (buf[p] == '\n' && buf[p + 1] == ')' && buf[p + 2] == '\n') { hit = buf + p + 3; break; }
        if (!hit) break;
        cut.push_back((size_t)(hit - buf));
    }
    cut.push_back(n);
    int parts = (int)cut.size() - 1;
    std::vector<NetChunk> ch(parts);
    parallel_for(parts, parts, [&](int b, int e) {
        for (int i = b; i < e; i++) parse_net_chunk(d, buf + cut[i], cut[i + 1] - cut[i], ch[i]);
    });
    // the chunks' arrays concatenated: each chunk copies into its own slice
    struct Base { size_t name = 0, net = 0, pin = 0, ap = 0; };
    std::vector<Base> base(parts + 1);
    for (int i = 0; i < parts; i++) {
        base[i + 1].name = base[i].name + ch[i].names.size();
        base[i + 1].net = base[i].net + ch[i].pins_per_net.size();
        base[i + 1].pin = base[i].pin + ch[i].aps_per_pin.size();
        base[i + 1].ap = base[i].ap + ch[i].ap.size();
    }
    const Base &tot = base[parts];
    d.name_pool.resize(tot.name);
    d.name_off.assign(tot.net + 1, 0);
    d.pin_off.assign(tot.net + 1, 0);
    d.ap_off.assign(tot.pin + 1, 0);
    d.ap.resize(tot.ap);
    d.bminx.resize(tot.net); d.bmaxx.resize(tot.net); d.bminy.resize(tot.net); d.bmaxy.resize(tot.net);
    parallel_for(parts, parts, [&](int b, int e) {
        for (int i = b; i < e; i++) {
            NetChunk &c = ch[i];
            const Base &o = base[i];
            std::copy(c.names.begin(), c.names.end(), d.name_pool.begin() + o.name);
            int64_t at = (int64_t)o.name, pin = (int64_t)o.pin, ap = (int64_t)o.ap;
            for (size_t k = 0; k < c.pins_per_net.size(); k++) {
                at += c.name_len[k];
                pin += c.pins_per_net[k];
                d.name_off[o.net + k + 1] = at;
                d.pin_off[o.net + k + 1] = pin;
                d.bminx[o.net + k] = c.bb[4 * k]; d.bmaxx[o.net + k] = c.bb[4 * k + 1];
                d.bminy[o.net + k] = c.bb[4 * k + 2]; d.bmaxy[o.net + k] = c.bb[4 * k + 3];
            }
            for (size_t k = 0; k < c.aps_per_pin.size(); k++) {
                ap += c.aps_per_pin[k];
                d.ap_off[o.pin + k + 1] = ap;
            }
            std::copy(c.ap.begin(), c.ap.end(), d.ap.begin() + o.ap);
            c = NetChunk();
        }
    });
}

namespace {

// read-only view of a whole file: a private mapping, or a copy where mapping fails
struct FileView {
    const char *data = nullptr;
    size_t size = 0;
    void *map = nullptr;
    std::vector<char> copy;
    explicit FileView(const char *path) {
        const int fd = ::open(path, O_RDONLY);
        if (fd < 0) throw Error(ERR_IO, std::string("cannot open ") + path);
        struct stat st;
        if (::fstat(fd, &st) == 0 && st.st_size > 0) {
            void *m = ::mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, fd, 0);
            if (m != MAP_FAILED) {
                map = m;
                data = static_cast<const char *>(m);
                size = (size_t)st.st_size;
            }
        }
        ::close(fd);
        if (!map) {
            copy = slurp(path);
            data = copy.data();
            size = copy.size() - 1;
        }
    }
    ~FileView() {
        if (map) ::munmap(map, size);
    }
    FileView(const FileView &) = delete;
    FileView &operator=(const FileView &) = delete;
};

}  // namespace

void read_design(Design &d, const char *cap_path, const char *net_path, int threads) {
    // the .net file is mapped while the capacities are parsed
    std::unique_ptr<FileView> net;
    std::exception_ptr net_err;
    std::thread loader([&] {
        try {
            net.reset(new FileView(net_path));
        } catch (...) {
            net_err = std::current_exception();
        }
    });
    try {
        FileView cap(cap_path);
        read_cap_buffer(d, cap.data, cap.size, threads);
    } catch (...) {
        loader.join();
        throw;
    }
    loader.join();
    if (net_err) std::rethrow_exception(net_err);
    read_net_buffer(d, net->data, net->size);
    net.reset();
    select_pins(d, threads);
}

// ------------------------------------------------------------------ writer
namespace {

// decimal digits of a non-negative value, two at a time
inline char *put_int(char *o, int v) {
    static const char kPairs[] =
        "00010203040506070809101112131415161718192021222324252627282930313233343536373839"
        "40414243444546474849505152535455565758596061626364656667686970717273747576777879"
        "8081828384858687888990919293949596979899";
    char t[12];
    char *e = t + sizeof t, *p = e;
    unsigned u = (unsigned)v;
    while (u >= 100) {
        const unsigned r = u % 100;
        u /= 100;
        p -= 2;
        std::memcpy(p, kPairs + 2 * r, 2);
    }
    if (u >= 10) {
        p -= 2;
        std::memcpy(p, kPairs + 2 * u, 2);
    } else {
        *--p = (char)('0' + u);
    }
    std::memcpy(o, p, (size_t)(e - p));
    return o + (e - p);
}

}  // namespace

namespace {

// writes all of buf at file offset `at`
bool pwrite_all(int fd, const char *buf, size_t n, off_t at) {
    while (n > 0) {
        const ssize_t w = ::pwrite(fd, buf, n, at);
        if (w < 0) {
            if (errno == EINTR) continue;
            return false;
        }
        buf += w;
        n -= (size_t)w;
        at += w;
    }
    return true;
}

}  // namespace

void write_guides(const Design &d, const NetSet &ns, const RouteSource &rs, const char *path, int threads) {
    const int fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0666);
    if (fd < 0) throw Error(ERR_IO, std::string("cannot open ") + path + " for writing");
    struct Closer {
        int fd;
        ~Closer() { if (fd >= 0) ::close(fd); }
    } closer{fd};
    const int X = d.X, Y = d.Y, XY = X * Y;
    const int N = d.num_nets();
    if (threads <= 0) threads = hw_threads();
    // Windows of chunks of nets: the chunks of a window are formatted in
    // parallel into private buffers, then written in parallel at their offsets.
    const int CH = 2048;
    int nch = (N + CH - 1) / CH;
    // a line of six values of at most 10 digits
    constexpr size_t kSegBytes = 6 * 11;
    struct Buf {
        std::unique_ptr<char[]> p;
        size_t cap = 0, size = 0;
    };
    auto fmt = [&](int c, Buf &out) {
        const int n0 = c * CH, n1 = std::min(N, (c + 1) * CH);
        // bytes of the chunk at most, so that the lines go straight into the buffer
        size_t ub = 0;
        for (int n = n0; n < n1; n++) {
            size_t segs = (size_t)(d.sel_off[n + 1] - d.sel_off[n]) + (size_t)(d.extra_off[n + 1] - d.extra_off[n]) / 2;
            if (n + 1 < (int)ns.sub_off.size())
                for (int s = ns.sub_off[n]; s < ns.sub_off[n + 1]; s++)
                    if (const int *r = rs.routes_of(s)) segs += (size_t)(r[0] > 1 ? r[0] / 2 : 0);
            ub += (size_t)(d.name_off[n + 1] - d.name_off[n]) + 5 + segs * kSegBytes;
        }
        if (out.cap < ub) {
            out.p.reset(new char[ub]);  // uninitialised: only the written part is touched
            out.cap = ub;
        }
        char *q = out.p.get();
        auto seg = [&](int p0, int p1) {
            if (p0 > p1) std::swap(p0, p1);
            q = put_int(q, p0 / Y % X); *q++ = ' ';
            q = put_int(q, p0 % Y); *q++ = ' ';
            q = put_int(q, p0 / XY); *q++ = ' ';
            q = put_int(q, p1 / Y % X); *q++ = ' ';
            q = put_int(q, p1 % Y); *q++ = ' ';
            q = put_int(q, p1 / XY); *q++ = '\n';
        };
        for (int n = n0; n < n1; n++) {
            const size_t nl = (size_t)(d.name_off[n + 1] - d.name_off[n]);
            std::memcpy(q, d.name_pool.data() + d.name_off[n], nl);
            q += nl;
            *q++ = '\n'; *q++ = '('; *q++ = '\n';
            for (int64_t i = d.sel_off[n]; i < d.sel_off[n + 1]; i++)
                if (d.sel[i] < XY) seg(d.sel[i], d.sel[i] + XY);
            for (int64_t i = d.extra_off[n]; i < d.extra_off[n + 1]; i += 2) seg(d.extra[i], d.extra[i + 1]);
            if (n + 1 < (int)ns.sub_off.size())
                for (int s = ns.sub_off[n]; s < ns.sub_off[n + 1]; s++) {
                    const int *r = rs.routes_of(s);
                    if (!r) continue;
                    for (int j = 1; j < r[0]; j += 2) seg(r[j] + XY, r[j + 1] + XY);
                }
            *q++ = ')'; *q++ = '\n';
        }
        out.size = (size_t)(q - out.p.get());
    };
    const int W = 8 * std::max(1, threads);
    std::vector<Buf> bufs(W);
    std::vector<off_t> at(W + 1);
    off_t pos = 0;
    for (int c0 = 0; c0 < nch; c0 += W) {
        const int k = std::min(W, nch - c0);
        parallel_for(k, threads, [&](int b, int e) {
            for (int i = b; i < e; i++) fmt(c0 + i, bufs[i]);
        });
        at[0] = pos;
        for (int i = 0; i < k; i++) at[i + 1] = at[i] + (off_t)bufs[i].size;
        std::atomic<bool> ok{true};
        parallel_for(k, threads, [&](int b, int e) {
            for (int i = b; i < e; i++)
                if (!pwrite_all(fd, bufs[i].p.get(), bufs[i].size, at[i])) ok = false;
        });
        if (!ok) throw Error(ERR_IO, std::string("write failed on ") + path);
        pos = at[k];
    }
    closer.fd = -1;
    if (::close(fd) != 0) throw Error(ERR_IO, std::string("write failed on ") + path);
}

}  // namespace igr
