// extern "C" entry points of include/instantgr_b200.h.
//
// Every entry point catches all exceptions and returns a status code with the
// message kept for igr_last_error(); nothing here exits the process.
#include "../../include/instantgr_b200.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>

#include "hooks.hpp"
#include "router.hpp"
#include "seed_model.hpp"

using namespace igr;

namespace {

thread_local std::string g_last_error;

int fail(std::string *slot, int code, const std::string &msg) {
    if (slot) *slot = msg;
    g_last_error = msg;
    return code;
}

template <typename F>
int guard(std::string *slot, F &&f) {
    try {
        f();
        return IGR_OK;
    } catch (const Error &e) {
        return fail(slot, e.code, e.what());
    } catch (const std::bad_alloc &) {
        return fail(slot, IGR_ERR_CAPACITY, "out of host memory");
    } catch (const std::exception &e) {
        return fail(slot, IGR_ERR_INVALID, e.what());
    }
}

}  // namespace

struct igr_router {
    Router r;
    std::string err;
};

struct igr_seed {
    SeedModel m;
    std::string err;
};

struct igr_ctx {
    GridOwner go;
    cudaStream_t s = nullptr;
    // side stream and its fork/join events for the split DAG DP (made on first use)
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    std::string err;
    // staging buffers reused across calls
    DevBuf<int> a, b, c, d, e, f, h, i, routes;
    DevBuf<int64_t> off;
    DevBuf<double> scr;
    DevBuf<uint8_t> u8;
    DevBuf<float> f1, f2;
    DevBuf<double> d1;
};

extern "C" {

void igr_default_options(igr_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->rrr_iters = 1;
    o->threads = 0;
    o->mode = -1;
    o->verbose = 0;
    o->batched = 0;
}

static void apply_options(Router &r, const igr_options *o) {
    igr_options def;
    igr_default_options(&def);
    if (!o) o = &def;
    if (o->rrr_iters < 0) throw Error(ERR_INVALID, "rrr_iters must be >= 0");
    r.rrr_iters = o->rrr_iters;
    r.threads = o->threads;
    r.mode = o->mode;
    r.verbose = o->verbose;
    r.batched = o->batched;
    r.split_commit = o->split_commit;
    r.host_dags = o->host_dags;
    r.kt.on = o->profile != 0;
}

int igr_router_open(const char *cap, const char *net, const igr_options *opt, igr_router **out) {
    if (!cap || !net || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    *out = nullptr;
    auto *h = new igr_router();
    int rc = guard(&h->err, [&] {
        apply_options(h->r, opt);
        h->r.open(cap, net);
    });
    if (rc) { delete h; return rc; }
    *out = h;
    return IGR_OK;
}

int igr_router_run(igr_router *h) {
    if (!h) return fail(nullptr, IGR_ERR_INVALID, "null router");
    return guard(&h->err, [&] { h->r.run(); });
}

int igr_router_write(igr_router *h, const char *out) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        if (!h->r.ran && !h->r.ns.nets.empty()) throw Error(ERR_STATE, "route before writing");
        h->r.write(out);
    });
}

int igr_router_evaluate(igr_router *h, double *out, double *layer_loss) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] { h->r.evaluate(out, layer_loss); });
}

int igr_router_stats(igr_router *h, double *o, int n) {
    if (!h || !o) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    const auto &r = h->r;
    double v[16] = {(double)r.ns.nets.size(), (double)r.st.rerouted, r.score_wl, r.score_via, r.score_of,
                    r.st.wall, (double)r.st.batches1, r.st.p1_ms, r.st.rrr_ms, r.st.dag_host_ms,
                    (double)r.st.launches, (double)r.d.num_nets(), (double)r.st.color_rounds,
                    (double)r.st.h2d_bytes, (double)r.st.d2h_bytes, (double)r.setup_h2d};
    for (int k = 0; k < n && k < 16; k++) o[k] = v[k];
    return IGR_OK;
}

int igr_router_kstats(igr_router *h, double *o, int n) {
    if (!h || !o) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    const auto &r = h->r;
    for (int k = 0; k < KC_N; k++) {
        double v[3] = {(double)r.kt.launches[k], r.kt.ms[k],
                       k == KC_COST             ? 20.0 * (double)r.cost_cells
                       : k == KC_COMMIT_REFRESH ? 20.0 * (double)r.commit_refresh_cells + 12.0 * (double)r.commit_cells
                       : k == KC_COLOR          ? r.color_bytes
                       : k == KC_PATTERN        ? r.dp_bytes
                                                : 0.0};
        for (int j = 0; j < 3; j++)
            if (3 * k + j < n) o[3 * k + j] = v[j];
    }
    return IGR_OK;
}

int igr_router_plan(igr_router *h, int64_t *sizes, int32_t *net_ids, int32_t *batch_off, int32_t *node_off,
                    int32_t *nodes, int32_t *par, int32_t *route_cap) {
    if (!h || !sizes) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        auto &r = h->r;
        if (!r.ran) throw Error(ERR_STATE, "route before reading the plan");
        r.build_plan();
        sizes[0] = (int64_t)r.plan_ids.size();
        sizes[1] = (int64_t)r.plan_batch_off.size() - 1;
        sizes[2] = (int64_t)r.plan_nodes.size();
        auto cp = [](int32_t *o, const std::vector<int> &v) {
            if (o && !v.empty()) std::memcpy(o, v.data(), v.size() * 4);
        };
        cp(net_ids, r.plan_ids);
        cp(batch_off, r.plan_batch_off);
        cp(node_off, r.plan_node_off);
        cp(nodes, r.plan_nodes);
        cp(par, r.plan_par);
        if (route_cap)
            for (size_t i = 0; i < r.plan_ids.size(); i++) route_cap[i] = r.plan_cap[i];
    });
}

int igr_router_grid(igr_router *h, int32_t *hdr, double *costs, int32_t *xl, int32_t *yl, float *cap) {
    if (!h) return fail(nullptr, IGR_ERR_INVALID, "null router");
    return guard(&h->err, [&] {
        const auto &d = h->r.d;
        const int L = d.L - 1, X = d.X, Y = d.Y;
        if (hdr) { hdr[0] = L; hdr[1] = X; hdr[2] = Y; hdr[3] = d.layer_dir[1]; }
        if (costs) {
            costs[0] = d.unit_wire;
            costs[1] = d.unit_via;
            for (int l = 0; l < L; l++) costs[2 + l] = d.short_cost[l + 1];
        }
        if (xl) std::memcpy(xl, d.x_edge_len.data(), 4 * (size_t)(X - 1));
        if (yl) std::memcpy(yl, d.y_edge_len.data(), 4 * (size_t)(Y - 1));
        if (cap) std::memcpy(cap, d.cap.data() + (size_t)X * Y, 4 * (size_t)L * X * Y);
    });
}

int igr_set_device(int device) {
    return guard(nullptr, [&] { cuda_check(cudaSetDevice(device), "cudaSetDevice"); });
}

int igr_router_sizes(igr_router *h, int64_t *dn, int64_t *rn) {
    if (!h) return fail(nullptr, IGR_ERR_INVALID, "null router");
    if (dn) *dn = h->r.d.num_nets();
    if (rn) *rn = (int64_t)h->r.ns.nets.size();
    return IGR_OK;
}

int igr_router_route(igr_router *h, int net, int32_t *out, int cap, int *len) {
    if (!h || !len) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        auto &r = h->r;
        if (net < 0 || net >= (int)r.ns.nets.size()) throw Error(ERR_INVALID, "net id out of range");
        if (!r.ran) throw Error(ERR_STATE, "route before reading routes");
        r.fetch_routes();
        const int *rec = r.route_of(net);
        *len = rec[0];
        if (out) {
            if (cap < rec[0]) throw Error(ERR_CAPACITY, "output buffer too small");
            std::memcpy(out, rec, sizeof(int) * rec[0]);
        }
    });
}

int igr_router_pins(igr_router *h, int net, int32_t *out, int cap, int *len) {
    if (!h || !len) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        const auto &d = h->r.d;
        if (net < 0 || net >= d.num_nets()) throw Error(ERR_INVALID, "net id out of range");
        std::vector<int> p(d.sel.begin() + d.sel_off[net], d.sel.begin() + d.sel_off[net + 1]);
        std::vector<int> v{(int)p.size()};
        v.insert(v.end(), p.begin(), p.end());
        v.push_back((int)(d.extra_off[net + 1] - d.extra_off[net]) / 2);
        v.insert(v.end(), d.extra.begin() + d.extra_off[net], d.extra.begin() + d.extra_off[net + 1]);
        *len = (int)v.size();
        if (out) {
            if (cap < *len) throw Error(ERR_CAPACITY, "output buffer too small");
            std::memcpy(out, v.data(), v.size() * 4);
        }
    });
}

int igr_router_demand(igr_router *h, float *out) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        auto &r = h->r;
        DevBuf<float> t;
        t.alloc(r.go.g.N);
        launch_from_track_layout_f(r.go.g, r.go.demand.p, t.p, r.s);
        cuda_check(cudaMemcpyAsync(out, t.p, r.go.g.N * sizeof(float), cudaMemcpyDeviceToHost, r.s), "D2H");
        cuda_check(cudaStreamSynchronize(r.s), "sync");
    });
}

void igr_router_close(igr_router *h) { delete h; }

int igr_route_files(const char *cap, const char *net, const char *out, const igr_options *opt) {
    igr_router *h = nullptr;
    int rc = igr_router_open(cap, net, opt, &h);
    if (rc) return rc;
    rc = igr_router_run(h);
    if (!rc) rc = igr_router_write(h, out);
    if (rc) g_last_error = h->err;
    igr_router_close(h);
    return rc;
}

int igr_generate_custom(int X, int Y, int nets, uint64_t seed, int cap_mode, double block_frac, int pin_mode,
                        double hifanout_frac, double bbox_median, double bbox_sigma, int hotspots,
                        double hotspot_frac, const char *cap_path, const char *net_path) {
    if (!cap_path || !net_path) return fail(nullptr, IGR_ERR_INVALID, "null path");
    return guard(nullptr, [&] {
        generate_design(custom_params(X, Y, nets, seed, cap_mode, block_frac, pin_mode, hifanout_frac, bbox_median,
                                      bbox_sigma, hotspots, hotspot_frac),
                        cap_path, net_path);
    });
}

int igr_generate(int cfg, uint64_t seed, double scale, const char *cap_path, const char *net_path) {
    if (!cap_path || !net_path) return fail(nullptr, IGR_ERR_INVALID, "null path");
    return guard(nullptr, [&] { generate_design(config_params(cfg, seed, scale), cap_path, net_path); });
}

// ------------------------------------------------------------------ device operators
int igr_create(const igr_grid_desc *g, igr_ctx **out) {
    if (!g || !out || !g->x_edge_len || !g->y_edge_len || !g->short_cost || !g->capacity)
        return fail(nullptr, IGR_ERR_INVALID, "null argument");
    *out = nullptr;
    auto *c = new igr_ctx();
    int rc = guard(&c->err, [&] {
        cuda_check(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking), "stream");
        c->go.create(g->L, g->X, g->Y, g->dir0, g->x_edge_len, g->y_edge_len, g->unit_wire, g->unit_via,
                     g->short_cost, g->capacity, c->s);
    });
    if (rc) {
        if (c->s) cudaStreamDestroy(c->s);
        delete c;
        return rc;
    }
    *out = c;
    return IGR_OK;
}

int igr_destroy(igr_ctx *c) {
    if (!c) return IGR_OK;
    cudaStreamSynchronize(c->s);
    cudaStream_t s = c->s, aux = c->aux;
    cudaEvent_t fork = c->fork, join = c->join;
    delete c;
    if (aux) cudaStreamDestroy(aux);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (s) cudaStreamDestroy(s);
    return IGR_OK;
}

const char *igr_last_error(const igr_ctx *c) { return c ? c->err.c_str() : g_last_error.c_str(); }

int igr_test_hook(int key, int64_t value) {
    TestHooks &h = test_hooks();
    switch (key) {
        case IGR_HOOK_RESET: h.reset(); return IGR_OK;
        case IGR_HOOK_WAIT_NS:
            if (value < 0) return fail(nullptr, IGR_ERR_INVALID, "negative wait limit");
            h.wait_ns = (long long)value;
            return IGR_OK;
        case IGR_HOOK_BARRIER_PHANTOM:
            if (value < 0 || value > 1024) return fail(nullptr, IGR_ERR_INVALID, "phantom arrivals in 0..1024");
            h.barrier_phantom = (int)value;
            return IGR_OK;
        case IGR_HOOK_MBAR_PROBE: h.mbar_probe = value != 0; return IGR_OK;
        case IGR_HOOK_COLOR_KEEP_MAP: h.color_keep_map = value != 0; return IGR_OK;
        case IGR_HOOK_COLOR_KEEP_MIN_NETS:
            if (value < 1) return fail(nullptr, IGR_ERR_INVALID, "threshold must be at least 1");
            h.color_keep_min_nets = (int)std::min<int64_t>(value, INT32_MAX);
            return IGR_OK;
        case IGR_HOOK_SHAPE_DEDUPE: h.shape_dedupe = value != 0; return IGR_OK;
        case IGR_HOOK_DAG_SPLIT_NETS:
            if (value < 1) return fail(nullptr, IGR_ERR_INVALID, "split threshold must be at least 1");
            h.dag_split_nets = (int)std::min<int64_t>(value, INT32_MAX);
            return IGR_OK;
        case IGR_HOOK_DAG_STAGE_NODES:
            if (value < 0 || value > 4096) return fail(nullptr, IGR_ERR_INVALID, "staging limit in 0..4096 nodes");
            h.dag_stage_nodes = (int)value;
            return IGR_OK;
        default: return fail(nullptr, IGR_ERR_INVALID, "unknown test hook");
    }
}

#define CTX_GUARD(c, ...)                                                       \
    do {                                                                        \
        if (!(c)) return fail(nullptr, IGR_ERR_INVALID, "null context");        \
        return guard(&(c)->err, [&] { __VA_ARGS__; });                          \
    } while (0)

static void sync_check(igr_ctx *c) {
    cuda_check(cudaGetLastError(), "launch");
    cuda_check(cudaStreamSynchronize(c->s), "sync");
    if (int e = c->go.check_error(c->s)) throw Error(e, "device reported an error");
}

int igr_set_demand(igr_ctx *c, const float *dem) {
    CTX_GUARD(c, {
        if (!dem) throw Error(ERR_INVALID, "null demand");
        c->f1.upload(dem, c->go.g.N, c->s);
        launch_to_track_layout(c->go.g, c->f1.p, c->go.demand.p, c->s);
        c->go.mark_all_dirty(c->s);
        sync_check(c);
    });
}

int igr_get_demand(igr_ctx *c, float *dem) {
    CTX_GUARD(c, {
        if (!dem) throw Error(ERR_INVALID, "null demand");
        c->f1.alloc(c->go.g.N);
        launch_from_track_layout_f(c->go.g, c->go.demand.p, c->f1.p, c->s);
        cuda_check(cudaMemcpyAsync(dem, c->f1.p, c->go.g.N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_get_stamp(igr_ctx *c, int32_t *o) {
    CTX_GUARD(c, {
        c->a.alloc(c->go.g.N);
        launch_from_track_layout_i(c->go.g, c->go.stamp.p, c->a.p, c->s);
        cuda_check(cudaMemcpyAsync(o, c->a.p, c->go.g.N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_get_pre(igr_ctx *c, int32_t *o) {
    CTX_GUARD(c, {
        c->a.alloc(c->go.g.N);
        launch_from_track_layout_i(c->go.g, c->go.pre.p, c->a.p, c->s);
        cuda_check(cudaMemcpyAsync(o, c->a.p, c->go.g.N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_cost_refresh(igr_ctx *c, int only_dirty) {
    CTX_GUARD(c, {
        launch_cost_refresh(c->go.g, only_dirty != 0, c->s);
        sync_check(c);
    });
}

int igr_get_costs(igr_ctx *c, float *vcost, double *presum) {
    CTX_GUARD(c, {
        if (vcost) {
            c->f1.alloc(c->go.g.N);
            launch_from_track_layout_f(c->go.g, c->go.vcost.p, c->f1.p, c->s);
            cuda_check(cudaMemcpyAsync(vcost, c->f1.p, c->go.g.N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        }
        if (presum) {
            c->d1.alloc(c->go.g.N);
            launch_from_track_layout_d(c->go.g, c->go.presum.p, c->d1.p, c->s);
            cuda_check(cudaMemcpyAsync(presum, c->d1.p, c->go.g.N * 8, cudaMemcpyDeviceToHost, c->s), "D2H");
        }
        sync_check(c);
    });
}

int igr_set_costs(igr_ctx *c, const float *vcost, const double *presum) {
    CTX_GUARD(c, {
        if (!vcost || !presum) throw Error(ERR_INVALID, "null cost table");
        c->f1.upload(vcost, c->go.g.N, c->s);
        launch_to_track_layout(c->go.g, c->f1.p, c->go.vcost.p, c->s);
        c->d1.upload(presum, c->go.g.N, c->s);
        launch_to_track_layout_d(c->go.g, c->d1.p, c->go.presum.p, c->s);
        cuda_check(cudaMemsetAsync(c->go.dirty_cost.p, 0, c->go.g.ntracks, c->s), "memset");
        sync_check(c);
    });
}

namespace {
constexpr char kStateMagic[8] = {'I', 'G', 'R', 'S', 'T', 'A', 'T', '1'};
}

int igr_dump_state(igr_ctx *c, const char *path) {
    CTX_GUARD(c, {
        if (!path) throw Error(ERR_INVALID, "null path");
        const GridDev &g = c->go.g;
        const size_t N = (size_t)g.N;
        std::vector<float> dem(N), vc(N);
        std::vector<double> ps(N);
        std::vector<int32_t> st(N), pre(N);
        c->f1.alloc(N);
        c->d1.alloc(N);
        c->a.alloc(N);
        launch_from_track_layout_f(g, c->go.demand.p, c->f1.p, c->s);
        cuda_check(cudaMemcpyAsync(dem.data(), c->f1.p, N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        launch_from_track_layout_f(g, c->go.vcost.p, c->f1.p, c->s);
        cuda_check(cudaMemcpyAsync(vc.data(), c->f1.p, N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        launch_from_track_layout_d(g, c->go.presum.p, c->d1.p, c->s);
        cuda_check(cudaMemcpyAsync(ps.data(), c->d1.p, N * 8, cudaMemcpyDeviceToHost, c->s), "D2H");
        launch_from_track_layout_i(g, c->go.stamp.p, c->a.p, c->s);
        cuda_check(cudaMemcpyAsync(st.data(), c->a.p, N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        cuda_check(cudaStreamSynchronize(c->s), "sync");  // c->a is reused below
        launch_from_track_layout_i(g, c->go.pre.p, c->a.p, c->s);
        cuda_check(cudaMemcpyAsync(pre.data(), c->a.p, N * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
        FILE *f = std::fopen(path, "wb");
        if (!f) throw Error(ERR_IO, std::string("cannot open ") + path + " for writing");
        const int32_t dims[3] = {g.L, g.X, g.Y};
        bool ok = std::fwrite(kStateMagic, 1, 8, f) == 8 && std::fwrite(dims, 4, 3, f) == 3 &&
                  std::fwrite(dem.data(), 4, N, f) == N && std::fwrite(vc.data(), 4, N, f) == N &&
                  std::fwrite(ps.data(), 8, N, f) == N && std::fwrite(st.data(), 4, N, f) == N &&
                  std::fwrite(pre.data(), 4, N, f) == N;
        ok = std::fclose(f) == 0 && ok;
        if (!ok) throw Error(ERR_IO, std::string("write failed on ") + path);
    });
}

int igr_load_state(igr_ctx *c, const char *path) {
    CTX_GUARD(c, {
        if (!path) throw Error(ERR_INVALID, "null path");
        const GridDev &g = c->go.g;
        const size_t N = (size_t)g.N;
        FILE *f = std::fopen(path, "rb");
        if (!f) throw Error(ERR_IO, std::string("cannot open ") + path);
        struct Closer {
            FILE *f;
            ~Closer() { std::fclose(f); }
        } closer{f};
        char magic[8];
        int32_t dims[3];
        if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kStateMagic, 8) != 0 || std::fread(dims, 4, 3, f) != 3)
            throw Error(ERR_FORMAT, std::string(path) + " is not a grid state file");
        if (dims[0] != g.L || dims[1] != g.X || dims[2] != g.Y)
            throw Error(ERR_INVALID, "the state file's grid differs from the context's");
        std::vector<float> dem(N), vc(N);
        std::vector<double> ps(N);
        std::vector<int32_t> st(N), pre(N);
        if (std::fread(dem.data(), 4, N, f) != N || std::fread(vc.data(), 4, N, f) != N ||
            std::fread(ps.data(), 8, N, f) != N || std::fread(st.data(), 4, N, f) != N ||
            std::fread(pre.data(), 4, N, f) != N)
            throw Error(ERR_FORMAT, std::string(path) + " is shorter than its grid");
        c->f1.upload(dem.data(), N, c->s);
        launch_to_track_layout(g, c->f1.p, c->go.demand.p, c->s);
        c->f2.upload(vc.data(), N, c->s);
        launch_to_track_layout(g, c->f2.p, c->go.vcost.p, c->s);
        c->d1.upload(ps.data(), N, c->s);
        launch_to_track_layout_d(g, c->d1.p, c->go.presum.p, c->s);
        c->a.upload(st.data(), N, c->s);
        launch_to_track_layout_i(g, c->a.p, c->go.stamp.p, c->s);
        c->b.upload(pre.data(), N, c->s);
        launch_to_track_layout_i(g, c->b.p, c->go.pre.p, c->s);
        cuda_check(cudaMemsetAsync(c->go.dirty_cost.p, 0, g.ntracks, c->s), "memset");
        cuda_check(cudaMemsetAsync(c->go.dirty_commit.p, 1, g.ntracks, c->s), "memset");
        sync_check(c);
    });
}

// length of a route-record array given offsets (records must already hold their counts)
static int64_t records_extent(int n, const int64_t *off, const int32_t *cap_or_null, const int32_t *routes) {
    int64_t m = 0;
    for (int k = 0; k < n; k++) {
        if (off[k] < 0) throw Error(ERR_INVALID, "negative route offset");
        const int64_t len = cap_or_null ? cap_or_null[k] : (routes ? routes[off[k]] : 1);
        if (len < 1) throw Error(ERR_INVALID, "route record without a count slot");
        m = std::max(m, off[k] + len);
    }
    return m;
}

static void check_tree(int n, const int32_t *node_off, const int32_t *nodes, const int32_t *par, int L, int X, int Y) {
    if (node_off[0] != 0) throw Error(ERR_INVALID, "node_off[0] must be 0");
    for (int k = 0; k < n; k++) {
        if (node_off[k + 1] < node_off[k] + 1) throw Error(ERR_INVALID, "every tree needs at least one node");
        for (int i = node_off[k]; i < node_off[k + 1]; i++) {
            const int loc = i - node_off[k];
            if (nodes[i] < 0 || nodes[i] >= (L + 1) * X * Y) throw Error(ERR_INVALID, "node position out of range");
            if (loc == 0 ? par[i] != -1 : (par[i] < 0 || par[i] >= loc))
                throw Error(ERR_STATE, "tree nodes must be in preorder with par[i] < i");
        }
    }
}

int igr_pattern_route(igr_ctx *c, int n, const int32_t *node_off, const int32_t *nodes, const int32_t *par,
                      const int64_t *route_off, const int32_t *route_cap, int32_t *routes_out, int32_t stamp) {
    CTX_GUARD(c, {
        if (n < 0 || (n && (!node_off || !nodes || !par || !route_off || !route_cap || !routes_out)))
            throw Error(ERR_INVALID, "bad arguments");
        if (n == 0) return;
        const auto &g = c->go.g;
        check_tree(n, node_off, nodes, par, g.L, g.X, g.Y);
        const int64_t ext = records_extent(n, route_off, route_cap, nullptr);
        const int total = node_off[n];
        std::vector<int> ids(n);
        std::iota(ids.begin(), ids.end(), 0);
        std::vector<int64_t> so(n, -1);
        int64_t sn = 0;
        for (int k = 0; k < n; k++) {
            const int cnt = node_off[k + 1] - node_off[k];
            if (cnt > kPatternNodeTile) { so[k] = sn; sn += cnt; }
        }
        c->a.upload(ids, c->s);
        c->b.upload(node_off, n + 1, c->s);
        c->d.upload(nodes, total, c->s);
        c->e.upload(par, total, c->s);
        c->f.upload(route_cap, n, c->s);
        c->off.upload(route_off, n, c->s);
        DevBuf<int64_t> d_so;
        d_so.upload(so, c->s);
        c->scr.alloc((size_t)pattern_scratch_doubles(sn));
        c->routes.upload(routes_out, (size_t)ext, c->s);
        TreeBatchDev tb{c->a.p, c->b.p, c->d.p, c->e.p, c->off.p, c->f.p, c->routes.p, c->scr.p, d_so.p, sn, n};
        c->h.alloc(1);
        cuda_check(cudaMemsetAsync(c->h.p, 0, sizeof(int), c->s), "memset");
        tb.queue = c->h.p;
        tb.tile = kPatternNodeTile;
        launch_pattern_route(g, tb, stamp, c->s);
        cuda_check(cudaMemcpyAsync(routes_out, c->routes.p, ext * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

static_assert(IGR_STATIC_SCRATCH_BYTES == kStaticScratchBytes, "static scratch size");
static_assert(IGR_STATIC_MAX_NETS == kStaticMaxNets, "static scratch net limit");

int igr_pattern_route_static(igr_ctx *c, int n, const int32_t *node_off, int64_t total_nodes, const int32_t *nodes,
                             const int32_t *par, const int64_t *route_off, const int32_t *route_cap, int32_t *routes,
                             int64_t routes_len, int32_t stamp) {
    CTX_GUARD(c, {
        pattern_route_static(c->go.g, n, node_off, total_nodes, nodes, par, route_off, route_cap, routes, routes_len,
                             stamp, c->s);
        sync_check(c);
    });
}

int igr_commit_wires(igr_ctx *c, int32_t stamp) {
    CTX_GUARD(c, {
        launch_wire_commit(c->go.g, stamp, true, c->s);
        sync_check(c);
    });
}

static void upload_records(igr_ctx *c, int n, const int64_t *off, const int32_t *routes) {
    const int64_t ext = records_extent(n, off, nullptr, routes);
    const int64_t cells = c->go.g.N;
    const int X = c->go.g.X, Y = c->go.g.Y;
    for (int k = 0; k < n; k++) {
        const int32_t *r = routes + off[k];
        if (r[0] < 1 || (r[0] & 1) == 0) throw Error(ERR_INVALID, "route record count must be odd and >= 1");
        for (int j = 1; j < r[0]; j += 2) {
            const int a = r[j], b = r[j + 1];
            if (a < 0 || b < 0 || a >= cells || b >= cells) throw Error(ERR_INVALID, "route position out of range");
            const int la = a / (X * Y), lb = b / (X * Y);
            const int xa = a / Y % X, ya = a % Y, xb = b / Y % X, yb = b % Y;
            if (la != lb && (xa != xb || ya != yb)) throw Error(ERR_INVALID, "a via must stay on one GCell");
            if (la == lb && xa != xb && ya != yb) throw Error(ERR_INVALID, "a wire must be straight");
        }
    }
    std::vector<int> ids(n);
    std::iota(ids.begin(), ids.end(), 0);
    c->a.upload(ids, c->s);
    c->off.upload(off, n, c->s);
    c->routes.upload(routes, (size_t)ext, c->s);
}

int igr_commit_vias(igr_ctx *c, int n, const int64_t *off, const int32_t *routes, int32_t stamp, int32_t K) {
    CTX_GUARD(c, {
        if (n < 0 || (n && (!off || !routes))) throw Error(ERR_INVALID, "bad arguments");
        if (n == 0) return;
        upload_records(c, n, off, routes);
        launch_via_commit(c->go.g, ViaBatchDev{c->a.p, c->off.p, c->routes.p, n}, stamp, K, c->s);
        sync_check(c);
    });
}

int igr_ripup_wires(igr_ctx *c, int n, const int64_t *off, const int32_t *routes, int32_t stamp, int32_t K) {
    CTX_GUARD(c, {
        if (n < 0 || (n && (!off || !routes))) throw Error(ERR_INVALID, "bad arguments");
        if (n == 0) return;
        upload_records(c, n, off, routes);
        launch_wire_ripup(c->go.g, ViaBatchDev{c->a.p, c->off.p, c->routes.p, n}, stamp, K, c->s);
        sync_check(c);
    });
}

int igr_mark_overflow(igr_ctx *c, int n, const int64_t *off, const int32_t *routes, int32_t threshold,
                      int32_t min_edges, uint8_t *is_of) {
    CTX_GUARD(c, {
        if (n < 0 || (n && (!off || !routes || !is_of))) throw Error(ERR_INVALID, "bad arguments");
        if (n == 0) return;
        upload_records(c, n, off, routes);
        c->h.alloc(c->go.g.N);
        c->u8.alloc(n);
        launch_mark_overflow(c->go.g, threshold, c->h.p, ViaBatchDev{c->a.p, c->off.p, c->routes.p, n}, min_edges,
                             c->u8.p, c->s);
        cuda_check(cudaMemcpyAsync(is_of, c->u8.p, n, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_congestion_view(igr_ctx *c, float *xsum, float *ysum) {
    CTX_GUARD(c, {
        if (!xsum || !ysum) throw Error(ERR_INVALID, "null output");
        const size_t xy = (size_t)c->go.g.X * c->go.g.Y;
        c->f1.alloc(xy);
        c->f2.alloc(xy);
        launch_congestion_view(c->go.g, c->f1.p, c->f2.p, c->s);
        cuda_check(cudaMemcpyAsync(xsum, c->f1.p, xy * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        cuda_check(cudaMemcpyAsync(ysum, c->f2.p, xy * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_score(igr_ctx *c, double *wl, double *vias, double *of) {
    CTX_GUARD(c, {
        unsigned long long h[4];
        double o = 0;
        launch_overflow_cost(c->go.g, c->go.score.p, c->s);
        cuda_check(cudaMemcpyAsync(h, c->go.stats.p, sizeof h, cudaMemcpyDeviceToHost, c->s), "D2H");
        cuda_check(cudaMemcpyAsync(&o, c->go.score.p, sizeof o, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
        if (wl) *wl = (double)(int64_t)h[0];
        if (vias) *vias = (double)(int64_t)h[1];
        if (of) *of = o;
    });
}

int igr_color_batches(igr_ctx *c, int n, const int32_t *pt_off, const int32_t *pts, const int32_t *h_off,
                      const int32_t *hseg, const int32_t *v_off, const int32_t *vseg, int32_t sparsity,
                      int32_t *batch_out, int32_t *n_batches) {
    CTX_GUARD(c, {
        if (n < 0 || !n_batches || (n && (!pt_off || !pts || !h_off || !v_off || !batch_out)))
            throw Error(ERR_INVALID, "bad arguments");
        if (sparsity < 1) throw Error(ERR_INVALID, "sparsity must be >= 1");
        *n_batches = 0;
        if (n == 0) return;
        const int XY = c->go.g.X * c->go.g.Y;
        std::vector<int> pt_net;
        for (int k = 0; k < n; k++) {
            if (pt_off[k + 1] <= pt_off[k]) throw Error(ERR_INVALID, "every net needs a conflict point");
            for (int i = pt_off[k]; i < pt_off[k + 1]; i++) {
                if (pts[i] < 0 || pts[i] >= XY) throw Error(ERR_INVALID, "conflict point outside the grid");
                pt_net.push_back(k);
            }
        }
        for (int i = 0; i < 2 * h_off[n]; i++)
            if (hseg[i] < 0 || hseg[i] >= XY) throw Error(ERR_INVALID, "segment outside the grid");
        for (int i = 0; i < 2 * v_off[n]; i++)
            if (vseg[i] < 0 || vseg[i] >= XY) throw Error(ERR_INVALID, "segment outside the grid");
        for (int k = 0; k < n; k++) {
            for (int i = h_off[k]; i < h_off[k + 1]; i++)
                if (hseg[2 * i] / c->go.g.Y > hseg[2 * i + 1] / c->go.g.Y || hseg[2 * i] % c->go.g.Y != hseg[2 * i + 1] % c->go.g.Y)
                    throw Error(ERR_INVALID, "horizontal segment must run along x from low to high");
            for (int i = v_off[k]; i < v_off[k + 1]; i++)
                if (vseg[2 * i] / c->go.g.Y != vseg[2 * i + 1] / c->go.g.Y || vseg[2 * i] % c->go.g.Y > vseg[2 * i + 1] % c->go.g.Y)
                    throw Error(ERR_INVALID, "vertical segment must run along y from low to high");
        }
        std::vector<int> co, cl;
        build_claims(n, pt_off, pts, h_off, hseg, v_off, vseg, c->go.g.X, c->go.g.Y, sparsity, co, cl, 0);
        DevBuf<int> po, p, pn, ho, hs, vo, vs, map, bat, flags, dco, dcl, act;
        po.upload(pt_off, n + 1, c->s); p.upload(pts, pt_off[n], c->s); pn.upload(pt_net, c->s);
        ho.upload(h_off, n + 1, c->s); hs.upload(hseg, 2 * (size_t)h_off[n], c->s);
        vo.upload(v_off, n + 1, c->s); vs.upload(vseg, 2 * (size_t)v_off[n], c->s);
        dco.upload(co, c->s); dcl.upload(cl, c->s);
        DevBuf<int4> hdr;
        map.alloc(XY); bat.alloc(n); flags.alloc(16); act.alloc(4 * (size_t)n); hdr.alloc(n);
        ColorDev cd;
        cd.n = n; cd.X = c->go.g.X; cd.Y = c->go.g.Y; cd.sparsity = sparsity;
        cd.pt_off = po.p; cd.pts = p.p; cd.pt_net = pn.p; cd.h_off = ho.p; cd.hseg = hs.p; cd.v_off = vo.p;
        cd.vseg = vs.p; cd.npts = pt_off[n]; cd.map = map.p; cd.batch = bat.p; cd.flags = flags.p;
        cd.claim_off = dco.p; cd.claim = dcl.p;
        cd.active = act.p; cd.active2 = act.p + n; cd.cand = act.p + 2 * (size_t)n; cd.lost = act.p + 3 * (size_t)n;
        cd.hdr = hdr.p;
        DevBuf<int> rev_off, rev_cnt, rev, snap, dirty, part;
        if (cl.size() < (size_t)INT32_MAX && test_hooks().color_keep_map.load()) {  // round-0 map kept up to date
            rev_off.alloc(XY); rev_cnt.alloc(XY); rev.alloc(std::max<size_t>(1, cl.size()));
            snap.alloc(XY); dirty.alloc(XY); part.alloc(1024);
            cd.rev_off = rev_off.p; cd.rev_cnt = rev_cnt.p; cd.rev = rev.p; cd.snap = snap.p; cd.dirty = dirty.p;
            cd.part = part.p;
        }
        const int nb = run_coloring(cd, 0, c->s);
        if (nb == -2) throw Error(ERR_TIMEOUT, "colouring barrier timed out");
        if (nb < 0) throw Error(ERR_CUDA, std::string("colouring launch failed: ") + cudaGetErrorString(cudaGetLastError()));
        cuda_check(cudaMemcpyAsync(batch_out, bat.p, n * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
        *n_batches = nb;
    });
}

int igr_dag_route(igr_ctx *c, int n, const int32_t *node_off, const int32_t *nodes, const int32_t *depth,
                  const int32_t *par_off, const int32_t *par, const int32_t *child_slot, const int32_t *child_num,
                  const int64_t *route_off, const int32_t *route_cap, int32_t *routes_out, int32_t stamp) {
    CTX_GUARD(c, {
        if (n < 0 || (n && (!node_off || !nodes || !depth || !par_off || !par || !child_slot || !child_num ||
                            !route_off || !route_cap || !routes_out)))
            throw Error(ERR_INVALID, "bad arguments");
        if (n == 0) return;
        const auto &g = c->go.g;
        if (g.L != kRouteLayers) throw Error(ERR_INVALID, "the DAG DP handles 9 routing layers");
        const int N = node_off[n], E = par_off[N];
        if (node_off[0] != 0 || par_off[0] != 0) throw Error(ERR_INVALID, "CSR offsets must start at 0");
        for (int k = 0; k < n; k++)
            if (node_off[k + 1] < node_off[k]) throw Error(ERR_INVALID, "node offsets must not decrease");
        for (int v = 0; v < N; v++) {
            if (depth[v] < 0) throw Error(ERR_INVALID, "negative depth");
            if (child_num[v] < 0 || child_num[v] > 10) throw Error(ERR_INVALID, "at most 10 child slots per node");
            if (nodes[v] < 0 || nodes[v] >= (g.L + 1) * g.X * g.Y) throw Error(ERR_INVALID, "node out of range");
        }
        for (int e = 0; e < E; e++) {
            if (par[e] < 0 || par[e] >= N) throw Error(ERR_INVALID, "parent out of range");
            if (child_slot[e] < 0 || child_slot[e] >= child_num[par[e]]) throw Error(ERR_INVALID, "child slot out of range");
        }
        std::vector<int> echild(E), child_off(N + 1, 0), ids(n);
        for (int k = 0; k < n; k++)
            for (int v = node_off[k]; v < node_off[k + 1]; v++) {
                for (int e = par_off[v]; e < par_off[v + 1]; e++) {
                    echild[e] = v;
                    if (par[e] < node_off[k] || par[e] >= node_off[k + 1])
                        throw Error(ERR_INVALID, "a parent must belong to the same net");
                    if (depth[par[e]] >= depth[v]) throw Error(ERR_STATE, "a parent must be shallower than its child");
                }
                child_off[v + 1] = child_off[v] + child_num[v];
            }
        std::iota(ids.begin(), ids.end(), 0);
        std::vector<int> ln, level_off, net_level_off;
        dag_levels(n, node_off, depth, ln, level_off, net_level_off);
        if ((int64_t)N * 100 + 99 > 0x7fffffffLL) throw Error(ERR_CAPACITY, "too many DAG nodes in one batch");
        const int64_t ext = records_extent(n, route_off, route_cap, nullptr);
        DevBuf<int> dn, dpo, dp, dcs, dec, dco, dlo, dln, dnl, dno, dids, dcap, dlout, dstage, dscnt, dbc;
        DevBuf<int64_t> droff;
        DevBuf<double> dcost, dce, doff;
        DevBuf<unsigned long long> dbest, dpk;
        dn.upload(nodes, N, c->s); dpo.upload(par_off, N + 1, c->s); dp.upload(par, E, c->s);
        dcs.upload(child_slot, E, c->s); dec.upload(echild, c->s); dco.upload(child_off, c->s);
        dlo.upload(level_off, c->s); dln.upload(ln, c->s); dnl.upload(net_level_off, c->s);
        dno.upload(node_off, n + 1, c->s);
        dids.upload(ids, c->s); dcap.upload(route_cap, n, c->s); droff.upload(route_off, n, c->s);
        dcost.alloc((size_t)N * 10); dce.alloc((size_t)std::max(E, 1) * 81); dbc.alloc((size_t)std::max(E, 1) * 81);
        doff.alloc((size_t)std::max(E, 1) * 54);
        dbest.alloc((size_t)std::max(child_off[N], 1) * 10); dpk.alloc((size_t)std::max(child_off[N], 1) * 10);
        dlout.alloc(N); dstage.alloc((size_t)N * 8); dscnt.alloc(N);
        c->routes.upload(routes_out, (size_t)ext, c->s);
        DagBatchDev db;
        db.n_nodes = N; db.n_edges = E; db.n_nets = n;
        db.nodes = dn.p; db.par_off = dpo.p; db.par = dp.p; db.child_slot = dcs.p; db.edge_child = dec.p;
        db.child_off = dco.p; db.level_off = dlo.p; db.level_nodes = dln.p; db.net_level_off = dnl.p;
        db.net_node_off = dno.p; db.net_ids = dids.p; db.costs = dcost.p; db.best_path = dbest.p; db.packed = dpk.p;
        db.cost_edges = dce.p; db.best_change = dbc.p; db.layer_out = dlout.p; db.stage = dstage.p; db.offers = doff.p;
        db.stage_cnt = dscnt.p; db.route_off = droff.p; db.route_cap = dcap.p; db.routes = c->routes.p;
        if (!c->aux) {
            cuda_check(cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking), "stream");
            cuda_check(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming), "event");
            cuda_check(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming), "event");
        }
        for (int k = 0; k < n; k++) {
            db.max_net_nodes = std::max(db.max_net_nodes, node_off[k + 1] - node_off[k]);
            db.max_net_edges = std::max(db.max_net_edges, par_off[node_off[k + 1]] - par_off[node_off[k]]);
        }
        launch_dag_route(g, db, stamp, c->s, c->aux, c->fork, c->join, test_hooks().dag_split_nets.load(),
                         test_hooks().dag_stage_nodes.load());
        cuda_check(cudaGetLastError(), "DAG launch");
        cuda_check(cudaMemcpyAsync(routes_out, c->routes.p, ext * 4, cudaMemcpyDeviceToHost, c->s), "D2H");
        sync_check(c);
    });
}

int igr_build_dag(int X, int Y, int mode, int ntree, const int32_t *pos, const int32_t *adj_off, const int32_t *adj,
                  const float *xsum, const float *ysum, int32_t *out, int64_t cap, int64_t *len) {
    if (!pos || !adj_off || !adj || !xsum || !ysum || !len || ntree < 2 || X < 2 || Y < 2)
        return fail(nullptr, IGR_ERR_INVALID, "bad arguments");
    return guard(nullptr, [&] {
        NetSet ns;
        ns.L = 9; ns.X = X; ns.Y = Y;
        RNet r;
        r.tnode.assign(pos, pos + ntree);
        r.adj.off.assign(1, 0);
        r.adj.nb.clear();
        for (int v = 0; v < ntree; v++) {
            if (pos[v] < 0 || pos[v] >= 10 * X * Y) throw Error(ERR_INVALID, "node position out of range");
            if (adj_off[v + 1] < adj_off[v]) throw Error(ERR_INVALID, "adjacency offsets must not decrease");
            for (int q = adj_off[v]; q < adj_off[v + 1]; q++) {
                if (adj[q] < 0 || adj[q] >= ntree) throw Error(ERR_INVALID, "adjacency out of range");
                r.adj.nb.push_back(adj[q]);
            }
            r.adj.off.push_back((int)r.adj.nb.size());
        }
        CongestionView cv;
        cv.X = X; cv.Y = Y;
        cv.xsum.assign(xsum, xsum + (size_t)X * Y);
        cv.ysum.assign(ysum, ysum + (size_t)X * Y);
        DagNet dn;
        build_dag(ns, r, cv, mode, dn);
        std::vector<int> v;
        const int m = (int)dn.nodes.size(), E = (int)dn.par_nodes.size();
        v.push_back(m);
        v.insert(v.end(), dn.nodes.begin(), dn.nodes.end());
        v.insert(v.end(), dn.par_num.begin(), dn.par_num.end());
        v.insert(v.end(), dn.child_num.begin(), dn.child_num.end());
        v.insert(v.end(), dn.depth.begin(), dn.depth.end());
        v.push_back(E);
        v.insert(v.end(), dn.par_nodes.begin(), dn.par_nodes.end());
        v.insert(v.end(), dn.child_idx.begin(), dn.child_idx.end());
        v.push_back((int)dn.points.size());
        v.insert(v.end(), dn.points.begin(), dn.points.end());
        *len = (int64_t)v.size();
        if (out && cap >= *len) std::memcpy(out, v.data(), v.size() * 4);
    });
}

int igr_build_dags(int X, int Y, int mode, int n, const int32_t *tree_off, const int32_t *pos,
                   const int32_t *adj_off, const int32_t *adj, const float *xsum, const float *ysum, int32_t *out,
                   int64_t cap, int64_t *rec_off, int64_t *len) {
    if (n < 0 || !tree_off || !xsum || !ysum || !len || !rec_off || X < 2 || Y < 2 || (n > 0 && (!pos || !adj_off || !adj)))
        return fail(nullptr, IGR_ERR_INVALID, "bad arguments");
    return guard(nullptr, [&] {
        if (tree_off[0] != 0) throw Error(ERR_INVALID, "tree offsets must start at 0");
        for (int k = 0; k < n; k++) {
            const int a = tree_off[k], b = tree_off[k + 1];
            if (b - a < 2) throw Error(ERR_INVALID, "a tree needs at least two nodes");
            for (int v = a; v < b; v++) {
                if (pos[v] < 0 || pos[v] >= 10 * X * Y) throw Error(ERR_INVALID, "node position out of range");
                if (adj_off[v + 1] < adj_off[v]) throw Error(ERR_INVALID, "adjacency offsets must not decrease");
                for (int q = adj_off[v]; q < adj_off[v + 1]; q++)
                    if (adj[q] < 0 || adj[q] >= b - a) throw Error(ERR_INVALID, "adjacency out of range");
            }
        }
        const int total = n ? tree_off[n] : 0;
        cudaStream_t s = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
        } sg{s};
        DevBuf<int> d_off, d_pos, d_aoff, d_adj, d_ids;
        DevBuf<float> d_xs, d_ys;
        std::vector<int> ids(n);
        std::iota(ids.begin(), ids.end(), 0);
        d_off.upload(tree_off, (size_t)n + 1, s);
        d_pos.upload(pos, (size_t)std::max(total, 1), s);
        d_aoff.upload(adj_off, (size_t)total + 1, s);
        d_adj.upload(adj, (size_t)std::max(adj_off[total], 1), s);
        d_ids.upload(ids, s);
        d_xs.upload(xsum, (size_t)X * Y, s);
        d_ys.upload(ysum, (size_t)X * Y, s);
        DagBuildArgs a;
        a.tree_off = d_off.p; a.pos = d_pos.p; a.adj_off = d_aoff.p; a.adj = d_adj.p;
        a.xsum = d_xs.p; a.ysum = d_ys.p; a.X = X; a.Y = Y; a.mode = mode;
        a.ids = d_ids.p; a.n_list = n;
        DeviceDags dd;
        dd.build(a, s);
        std::vector<long long> nat(n), eat(n), pat(n);
        unsigned long long u[3];
        auto down64 = [&](std::vector<long long> &h, const DevBuf<long long> &d) {
            if (!h.empty()) cuda_check(cudaMemcpyAsync(h.data(), d.p, h.size() * 8, cudaMemcpyDeviceToHost, s), "D2H");
        };
        down64(nat, dd.node_at); down64(eat, dd.edge_at); down64(pat, dd.point_at);
        cuda_check(cudaMemcpyAsync(u, dd.used.p, sizeof u, cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "sync");
        // the pools up to what was used (holes left by rebuilt DAGs included)
        const size_t nn = std::min<size_t>(u[0], dd.nodes.n), ne = std::min<size_t>(u[1], dd.par.n),
                     np = std::min<size_t>(u[2], dd.points.n);
        std::vector<int> nodes(nn), pnum(nn), cnum(nn), dep(nn), par(ne), cidx(ne), pts(np);
        auto down = [&](std::vector<int> &h, const DevBuf<int> &d) {
            if (!h.empty()) cuda_check(cudaMemcpyAsync(h.data(), d.p, h.size() * 4, cudaMemcpyDeviceToHost, s), "D2H");
        };
        down(nodes, dd.nodes); down(pnum, dd.par_num); down(cnum, dd.child_num); down(dep, dd.depth);
        down(par, dd.par); down(cidx, dd.child_idx); down(pts, dd.points);
        cuda_check(cudaStreamSynchronize(s), "sync");
        int64_t L = 0;
        for (int k = 0; k < n; k++) {
            rec_off[k] = L;
            L += 3 + 4 * (int64_t)dd.sz(k, 0) + 2 * (int64_t)dd.sz(k, 1) + dd.sz(k, 2);
        }
        rec_off[n] = L;
        *len = L;
        if (!out || cap < L) return;
        for (int k = 0; k < n; k++) {
            int32_t *o = out + rec_off[k];
            const int64_t a0 = nat[k], m = dd.sz(k, 0), e0 = eat[k], E = dd.sz(k, 1), p0 = pat[k], P = dd.sz(k, 2);
            *o++ = (int32_t)m;
            for (auto *v : {&nodes, &pnum, &cnum, &dep}) o = std::copy(v->begin() + a0, v->begin() + a0 + m, o);
            *o++ = (int32_t)E;
            for (auto *v : {&par, &cidx}) o = std::copy(v->begin() + e0, v->begin() + e0 + E, o);
            *o++ = (int32_t)P;
            o = std::copy(pts.begin() + p0, pts.begin() + p0 + P, o);
        }
    });
}

int igr_steiner(int n, const int32_t *x, const int32_t *y, int32_t *nx, int32_t *ny, int cap_nodes, int *n_nodes,
                int32_t *edges, int cap_edges, int *n_edges) {
    if (n < 0 || (n && (!x || !y)) || !n_nodes || !n_edges) return fail(nullptr, IGR_ERR_INVALID, "bad arguments");
    return guard(nullptr, [&] {
        std::vector<int> xs(x, x + n), ys(y, y + n);
        SteinerTree t;
        steiner_tree(xs, ys, t);
        *n_nodes = (int)t.x.size();
        *n_edges = (int)t.edges.size();
        if (*n_nodes > cap_nodes || *n_edges > cap_edges) throw Error(ERR_CAPACITY, "output buffers too small");
        for (int i = 0; i < *n_nodes; i++) { nx[i] = t.x[i]; ny[i] = t.y[i]; }
        for (int i = 0; i < *n_edges; i++) { edges[2 * i] = t.edges[i].first; edges[2 * i + 1] = t.edges[i].second; }
    });
}

// ------------------------------------------------------------------ learned congestion seed
int igr_router_set_seed(igr_router *h, igr_seed *m, double alpha, int mode, int kind, int levels) {
    if (!h) return fail(nullptr, IGR_ERR_INVALID, "null router");
    return guard(&h->err, [&] {
        if (mode < 0 || mode > 2 || !(alpha >= 0) || kind < 0 || kind > 3 || levels < 0)
            throw Error(ERR_INVALID, "bad seed mode, kind, levels or weight");
        if (mode && !m) throw Error(ERR_INVALID, "null model");
        auto &r = h->r;
        r.seed = mode ? &m->m : nullptr;
        r.seed_mode = mode;
        r.seed_alpha = alpha;
        r.seed_kind = kind & 1;
        r.seed_order = (kind & 2) != 0;
        r.seed_levels = levels;
        r.seed_ready = false;
        r.seed_used = false;
        r.seed_score_due = false;
    });
}

int igr_router_seed_stats(igr_router *h, double *out, int n) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        double v[4];
        h->r.seed_stats(v);
        for (int k = 0; k < n && k < 4; k++) out[k] = v[k];
    });
}

#define SEED_GUARD(m, ...)                                                      \
    do {                                                                        \
        if (!(m)) return fail(nullptr, IGR_ERR_INVALID, "null model");          \
        return guard(&(m)->err, [&] { __VA_ARGS__; });                          \
    } while (0)

static std::vector<__nv_bfloat16> to_bf16(const float *p, size_t n) {
    std::vector<__nv_bfloat16> v(n);
    for (size_t i = 0; i < n; i++) v[i] = __float2bfloat16(p[i]);
    return v;
}

int igr_seed_create(uint64_t init_seed, igr_seed **out) {
    if (!out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    *out = nullptr;
    auto *m = new igr_seed();
    const int rc = guard(&m->err, [&] { m->m.init(init_seed); });
    if (rc) { delete m; return rc; }
    *out = m;
    return IGR_OK;
}

int igr_seed_destroy(igr_seed *m) {
    delete m;
    return IGR_OK;
}

const char *igr_seed_last_error(const igr_seed *m) { return m ? m->err.c_str() : g_last_error.c_str(); }

int igr_seed_set_tile(igr_seed *m, int size, int halo) {
    SEED_GUARD(m, {
        std::vector<float> p;
        m->m.get_params(p);
        m->m.set_tile(size, halo);
        m->m.set_params(p.data(), p.size());
    });
}

int igr_seed_params(igr_seed *m, float *out, int64_t cap, int64_t *n) {
    SEED_GUARD(m, {
        if (!n) throw Error(ERR_INVALID, "null count");
        *n = m->m.params();
        if (out) {
            if (cap < *n) throw Error(ERR_CAPACITY, "output buffer too small");
            std::vector<float> p;
            m->m.get_params(p);
            std::memcpy(out, p.data(), p.size() * 4);
        }
    });
}

int igr_seed_set_params(igr_seed *m, const float *p, int64_t n) {
    SEED_GUARD(m, {
        if (!p) throw Error(ERR_INVALID, "null parameters");
        m->m.set_params(p, (size_t)n);
    });
}

int igr_seed_features(igr_router *h, float *out) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        std::vector<__nv_bfloat16> f;
        seed_features(h->r.d, h->r.ns, f);
        for (size_t i = 0; i < f.size(); i++) out[i] = __bfloat162float(f[i]);
    });
}

int igr_seed_features_device(igr_router *h, float *out) {
    if (!h || !out) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&h->err, [&] {
        auto &r = h->r;
        DevBuf<__nv_bfloat16> feat;
        r.device_seed_features(feat, r.s);
        std::vector<__nv_bfloat16> f((size_t)r.go.g.X * r.go.g.Y * 16);
        cuda_check(cudaMemcpyAsync(f.data(), feat.p, f.size() * 2, cudaMemcpyDeviceToHost, r.s), "D2H");
        cuda_check(cudaStreamSynchronize(r.s), "sync");
        for (size_t i = 0; i < f.size(); i++) out[i] = __bfloat162float(f[i]);
    });
}

int igr_seed_add_map(igr_seed *m, int X, int Y, const float *feat, const float *target, int32_t *map_id) {
    SEED_GUARD(m, {
        if (X < 1 || Y < 1 || !feat || !target) throw Error(ERR_INVALID, "bad map");
        const size_t n = (size_t)X * Y * 16;
        const auto f = to_bf16(feat, n), t = to_bf16(target, n);
        const int id = m->m.add_map(X, Y, f.data(), t.data());
        if (map_id) *map_id = id;
    });
}

int igr_seed_add_routed(igr_seed *m, igr_router *h, int32_t *map_id) {
    if (!m || !h) return fail(nullptr, IGR_ERR_INVALID, "null argument");
    return guard(&m->err, [&] {
        auto &r = h->r;
        if (!r.ran) throw Error(ERR_STATE, "route before taking the demand");
        std::vector<__nv_bfloat16> f, t;
        seed_features(r.d, r.ns, f);
        const int L = r.go.g.L, X = r.go.g.X, Y = r.go.g.Y;
        std::vector<float> dem((size_t)L * X * Y);
        DevBuf<float> tmp;
        tmp.alloc(dem.size());
        launch_from_track_layout_f(r.go.g, r.go.demand.p, tmp.p, r.s);
        cuda_check(cudaMemcpyAsync(dem.data(), tmp.p, dem.size() * 4, cudaMemcpyDeviceToHost, r.s), "D2H");
        cuda_check(cudaStreamSynchronize(r.s), "sync");
        seed_targets(X, Y, L, dem.data(), t);
        const int id = m->m.add_map(X, Y, f.data(), t.data());
        if (map_id) *map_id = id;
    });
}

int igr_seed_train(igr_seed *m, int steps, int tiles, float lr, uint64_t seed, int nmaps, double *loss_curve) {
    SEED_GUARD(m, {
        if (steps < 0 || tiles < 1 || tiles > 256 || nmaps < 0) throw Error(ERR_INVALID, "bad training arguments");
        std::vector<double> c;
        m->m.train(steps, tiles, lr, seed, &c, nmaps);
        if (loss_curve) std::memcpy(loss_curve, c.data(), c.size() * sizeof(double));
    });
}

int igr_seed_eval(igr_seed *m, int map, double *out, int n) {
    SEED_GUARD(m, {
        if (map < 0 || map >= (int)m->m.maps.size()) throw Error(ERR_INVALID, "no such map");
        if (!out) throw Error(ERR_INVALID, "null output");
        double v[4];
        m->m.evaluate(map, v);
        for (int k = 0; k < n && k < 4; k++) out[k] = v[k];
    });
}

int igr_seed_time_forward(igr_seed *m, int tiles, int reps, double *layer_ms, double *layer_flops) {
    SEED_GUARD(m, {
        if (!layer_ms || !layer_flops) throw Error(ERR_INVALID, "null output");
        static_assert(IGR_SEED_CONVS == kSeedConvs, "convolution count of the header");
        double f[kSeedConvs];
        m->m.time_forward(tiles, 1, layer_ms, f);  // untimed first pass (set-up, first launch)
        m->m.time_forward(tiles, reps, layer_ms, layer_flops);
    });
}

int igr_seed_predict(igr_seed *m, int X, int Y, const float *feat, float *pred) {
    SEED_GUARD(m, {
        if (X < 1 || Y < 1 || !feat || !pred) throw Error(ERR_INVALID, "bad map");
        const size_t n = (size_t)X * Y * 16;
        const auto f = to_bf16(feat, n);
        DevBuf<__nv_bfloat16> fd;
        DevBuf<float> pd;
        fd.upload(f.data(), n, m->m.s);
        pd.alloc(n);
        cuda_check(cudaMemsetAsync(pd.p, 0, n * 4, m->m.s), "memset");
        m->m.predict(X, Y, fd.p, pd.p);
        cuda_check(cudaMemcpyAsync(pred, pd.p, n * 4, cudaMemcpyDeviceToHost, m->m.s), "D2H");
        cuda_check(cudaStreamSynchronize(m->m.s), "sync");
    });
}

int igr_seed_grad(igr_seed *m, int T, const float *x, const float *target, double *loss, float *grads) {
    SEED_GUARD(m, {
        if (T < 1 || !x || !target) throw Error(ERR_INVALID, "bad arguments");
        auto &M = m->m;
        M.ensure(T);
        const size_t n = (size_t)T * M.S * M.S * 16;
        const auto xb = to_bf16(x, n);
        cuda_check(cudaMemcpyAsync(M.x0.p, xb.data(), n * 2, cudaMemcpyHostToDevice, M.s), "H2D");
        cuda_check(cudaMemcpyAsync(M.tgt32.p, target, n * 4, cudaMemcpyHostToDevice, M.s), "H2D");
        M.forward(T);
        const double l = M.backward(T, nullptr);
        if (loss) *loss = l;
        if (grads) {
            std::vector<float> g;
            M.grads(g);
            std::memcpy(grads, g.data(), g.size() * 4);
        }
    });
}

}  // extern "C"
