// Batched multi-scene forward + adjoint: the wos_batch_* entry points.
//
// A plan holds many (scene, query set) items.  Items are grouped by
// dimension, and within a group ordered by tree depth; each group runs its
// phases (forward walks, per-point reduction, loss, adjoint) over the
// concatenation of its items' walks: the walk phases as one persistent
// work-queue launch per run of items of equal depth (each compiled for that
// depth), the reductions as one launch per group.  The whole sequence is
// captured once into a CUDA graph that later runs replay with a single
// launch.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "scene_impl.h"
#include "walk.h"

namespace wosd {

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// Consecutive items of a group whose trees have the same depth.
struct BatchRun {
    int wl = 0;  // specialised_depth of the items' trees
    int first = 0, count = 0;
    long long base = 0, walks = 0;
};

struct BatchGroup {
    int dim = 0;
    std::vector<BatchRun> runs;
    std::vector<int> user_index;  // item index in the caller's list
    std::vector<BatchItemDev> items;
    std::vector<SceneView> views;
    std::vector<WalkCfg> cfgs;
    std::vector<wos_scene_t> scenes;
    std::vector<unsigned long long> gens;  // each scene's generation when `views` was read
    long long walks = 0;
    int points = 0;
    bool has_src = false;
    long long acc_len = 0;  // doubles
    // device
    BatchItemDev *d_items = nullptr;
    SceneView *d_views = nullptr;
    WalkCfg *d_cfgs = nullptr;
    float *vals = nullptr;
    int *wrec = nullptr;
    float *wds = nullptr;
    double *mean = nullptr, *var = nullptr, *loss = nullptr;
    float *dLdu = nullptr;
    double *acc = nullptr;
    float *grad = nullptr;  // float copy of acc
    unsigned long long *counters = nullptr;
    // adjoint sample order (launch_batch_order): sort keys, workspace, and
    // the sorted indices of the last enqueued step (inside order_ws)
    long long nkeys = 0;
    void *order_ws = nullptr;
    size_t order_bytes = 0;
    const unsigned *order = nullptr;
};

}  // namespace wosd

struct wos_batch_s {
    std::vector<wosd::BatchGroup> groups;
    wos_adjoint_params adj{};
    int want_adjoint = 1;
    // launch shape per (dimension - 2, phase 0 walk / 1 adjoint); count_work
    // is kept in every slot alike
    wosd::BatchLaunch slot[2][2] = {{{256, 0, 64, 0}, {256, 0, 64, 0}}, {{256, 0, 64, 0}, {256, 0, 64, 0}}};
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int n_items = 0;
    std::vector<std::pair<int, int>> where;  // caller item -> (group, index in group)
};

namespace wosd {

#define BT(x)                                          \
    do {                                               \
        cudaError_t _e = (x);                          \
        if (_e != cudaSuccess) return fail_cuda(_e, #x); \
    } while (0)

static void free_group(BatchGroup &g, cudaStream_t st) {
    void *ptrs[] = {g.d_items, g.d_views, g.d_cfgs, g.vals, g.wrec,     g.wds,     g.mean,
                    g.var,     g.loss,    g.dLdu,   g.acc,  g.grad, g.counters, g.order_ws};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, st);
}

static void drop_graph(wos_batch_s *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

static int upload_views(wos_batch_s *b, cudaStream_t st) {
    for (BatchGroup &g : b->groups) {
        g.gens.resize(g.scenes.size());
        for (size_t i = 0; i < g.scenes.size(); ++i) {
            g.views[i] = g.scenes[i]->impl.view();
            g.gens[i] = g.scenes[i]->impl.generation;
        }
        BT(cudaMemcpyAsync(g.d_views, g.views.data(), sizeof(SceneView) * g.views.size(), cudaMemcpyHostToDevice, st));
    }
    BT(cudaStreamSynchronize(st));
    return 0;
}

// True when a scene of the plan was rebuilt (wos_scene_update_vertices) or
// given a new source since its view was read: the view's by-value fields
// (bounding box, extents, source) are then out of date.
static bool stale_views(const wos_batch_s *b) {
    for (const BatchGroup &g : b->groups)
        for (size_t i = 0; i < g.scenes.size(); ++i)
            if (i >= g.gens.size() || g.gens[i] != g.scenes[i]->impl.generation) return true;
    return false;
}

static void set_count_work(wos_batch_s *b, int count) {
    for (auto &d : b->slot)
        for (auto &ph : d) ph.count_work = count;
}

// Enqueue one full step on stream st.
static int enqueue(wos_batch_s *b, cudaStream_t st) {
    const AdjCfg a = make_adj_cfg(b->adj);
    for (BatchGroup &g : b->groups) {
        const int n_items = (int)g.items.size();
        if (b->want_adjoint) BT(cudaMemsetAsync(g.acc, 0, sizeof(double) * g.acc_len, st));
        WalkOut o{g.vals, nullptr, b->want_adjoint ? g.wrec : nullptr, b->want_adjoint ? g.wds : nullptr,
                  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        for (const BatchRun &r : g.runs)
            if (int rc = launch_walk_batch(g.dim, r.wl, g.d_views + r.first, g.d_cfgs + r.first, g.d_items + r.first,
                                           r.count, r.base, r.walks, b->slot[g.dim - 2][0], o, g.counters, st))
                return rc;
        if (int rc = launch_reduce_batch(g.vals, g.d_items, n_items, g.points, g.mean, g.var, st)) return rc;
        if (int rc = launch_loss_batch(g.mean, g.d_items, n_items, g.dLdu, g.loss, st)) return rc;
        if (b->want_adjoint) {
            if (int rc = launch_batch_order(g.dim, g.d_views, g.d_items, n_items, g.nkeys, g.wrec, g.walks,
                                            g.order_ws, g.order_bytes, &g.order, st))
                return rc;
            for (const BatchRun &r : g.runs)
                if (int rc = launch_adjoint_batch(g.dim, r.wl, g.d_views + r.first, g.d_cfgs + r.first, a,
                                                  g.d_items + r.first, r.count, r.base, r.walks, g.dLdu, g.wrec,
                                                  g.wds, g.acc, b->slot[g.dim - 2][1], g.counters + 1, g.order, st))
                    return rc;
            if (int rc = launch_acc_to_f32(g.acc, g.grad, g.acc_len, st)) return rc;
        }
    }
    return 0;
}

// One phase (0 walks, 1 adjoint) of the dimension-dim group alone, over the
// first `frac` of every run's walks (a prefix of the run's walk range), for
// the slot tuner.  Needs a full step before it (the adjoint reads the walk
// phase's records and dL/du); the accumulators it fills are overwritten by
// the next full step.
static int enqueue_slot(wos_batch_s *b, int dim, int phase, double frac, cudaStream_t st) {
    const AdjCfg a = make_adj_cfg(b->adj);
    for (BatchGroup &g : b->groups) {
        if (g.dim != dim) continue;
        WalkOut o{g.vals, nullptr, b->want_adjoint ? g.wrec : nullptr, b->want_adjoint ? g.wds : nullptr,
                  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        for (const BatchRun &r : g.runs) {
            const long long w = std::max(1LL, std::min(r.walks, (long long)(frac * (double)r.walks)));
            if (phase == 0) {
                if (int rc = launch_walk_batch(g.dim, r.wl, g.d_views + r.first, g.d_cfgs + r.first,
                                               g.d_items + r.first, r.count, r.base, w, b->slot[dim - 2][0], o,
                                               g.counters, st))
                    return rc;
            } else if (b->want_adjoint) {
                if (int rc = launch_adjoint_batch(g.dim, r.wl, g.d_views + r.first, g.d_cfgs + r.first, a,
                                                  g.d_items + r.first, r.count, r.base, w, g.dLdu, g.wrec, g.wds,
                                                  g.acc, b->slot[dim - 2][1], g.counters + 1, g.order, st))
                    return rc;
            }
        }
    }
    return 0;
}

static int capture(wos_batch_s *b) {
    drop_graph(b);
    BT(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue(b, b->cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture");
    b->graph = graph;
    BT(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return 0;
}

}  // namespace wosd

using namespace wosd;

extern "C" {

int wos_batch_create(const wos_batch_item *items, int n_items, const wos_adjoint_params *a, int want_adjoint,
                     wos_stream_t stream, wos_batch_t *out) {
    if (out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (items == nullptr || n_items < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "a batch needs at least one item");
    if (want_adjoint && a == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "adjoint params are NULL");
    cudaStream_t st = (cudaStream_t)stream;
    wos_batch_s *b = new wos_batch_s();
    b->n_items = n_items;
    b->want_adjoint = want_adjoint ? 1 : 0;
    if (a) b->adj = *a;
    b->where.resize(n_items);
    BatchGroup g2, g3;
    g2.dim = 2;
    g3.dim = 3;
    for (int i = 0; i < n_items; ++i)
        if (items[i].scene == nullptr) {
            delete b;
            return fail(WOS_ERR_INVALID_ARGUMENT, "item " + std::to_string(i) + ": scene is NULL");
        }
    // within a dimension, items in order of tree depth (then caller order), so
    // that each depth is one contiguous run of walks
    std::vector<int> order(n_items);
    for (int i = 0; i < n_items; ++i) order[i] = i;
    auto depth = [&](int i) { return specialised_depth(items[i].scene->impl.wt_levels); };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return depth(x) < depth(y); });
    for (int i : order) {
        const wos_batch_item &it = items[i];
        const wos_params &p = it.params;
        if (p.nwalks < 1 || p.nsteps < 0 || !(p.epsilon >= 0.0f) || it.n < 0 || it.loss_kind < 0 ||
            it.loss_kind > 2 || (it.loss_kind != 1 && it.target_or_dLdu == nullptr && it.n > 0) ||
            (it.n > 0 && it.P == nullptr)) {
            delete b;
            return fail(WOS_ERR_INVALID_ARGUMENT, "item " + std::to_string(i) + ": invalid sizes or params");
        }
        const SceneImpl &S = it.scene->impl;
        BatchGroup &g = S.dim == 2 ? g2 : g3;
        b->where[i] = {S.dim == 2 ? 0 : 1, (int)g.items.size()};
        BatchItemDev d{};
        d.P = it.P;
        d.walk_begin = g.walks;
        d.n = it.n;
        d.nwalks = p.nwalks;
        d.point_begin = g.points;
        d.loss_kind = it.loss_kind;
        d.target = it.target_or_dLdu;
        d.dV_off = g.acc_len;
        g.acc_len += (long long)S.nV * S.dim;
        d.dg_off = g.acc_len;
        g.acc_len += S.nV;
        d.ds_off = g.acc_len;
        g.acc_len += 5;
        d.prim_off = g.nkeys;
        g.nkeys += (long long)S.nF + 1;
        const int wl = specialised_depth(S.wt_levels);
        if (g.runs.empty() || g.runs.back().wl != wl) {
            BatchRun r;
            r.wl = wl;
            r.first = (int)g.items.size();
            r.base = g.walks;
            g.runs.push_back(r);
        }
        g.runs.back().count += 1;
        g.runs.back().walks += (long long)it.n * p.nwalks;
        g.items.push_back(d);
        g.scenes.push_back(it.scene);
        g.views.push_back(S.view());
        g.cfgs.push_back(make_cfg(p));
        g.user_index.push_back(i);
        g.walks += (long long)it.n * p.nwalks;
        g.points += it.n;
        if (p.include_source && S.src_type != 0 && S.dim == 2) g.has_src = true;
    }
    // groups keep a fixed order: 2D then 3D; an empty group is dropped
    std::vector<BatchGroup> gs;
    if (!g2.items.empty()) gs.push_back(std::move(g2));
    if (!g3.items.empty()) gs.push_back(std::move(g3));
    for (int i = 0; i < n_items; ++i)
        if (b->where[i].first == 1 && gs.size() == 1) b->where[i].first = 0;
    b->groups = std::move(gs);
    int rc = 0;
    for (BatchGroup &g : b->groups) {
        const size_t W = (size_t)g.walks, Pn = (size_t)g.points, NI = g.items.size();
        const size_t rb = g.dim == 3 ? 16 : 8;
        cudaError_t e = cudaSuccess;
        auto A = [&](auto **p, size_t bytes) {
            if (e == cudaSuccess) e = cudaMallocAsync((void **)p, al256(std::max<size_t>(bytes, 1)), st);
        };
        A(&g.d_items, sizeof(BatchItemDev) * NI);
        A(&g.d_views, sizeof(SceneView) * NI);
        A(&g.d_cfgs, sizeof(WalkCfg) * NI);
        A(&g.vals, sizeof(float) * W);
        A(&g.mean, sizeof(double) * Pn);
        A(&g.var, sizeof(double) * Pn);
        A(&g.loss, sizeof(double) * NI);
        A(&g.dLdu, sizeof(float) * Pn);
        A(&g.counters, sizeof(unsigned long long) * 2);
        if (b->want_adjoint) {
            A(&g.wrec, rb * W);
            if (g.has_src && b->adj.want_dsrc) A(&g.wds, sizeof(float) * 5 * W);
            A(&g.acc, sizeof(double) * g.acc_len);
            A(&g.grad, sizeof(float) * g.acc_len);
            g.order_bytes = batch_order_bytes(g.nkeys, g.walks);
            if (g.order_bytes) A(&g.order_ws, g.order_bytes);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g.d_items, g.items.data(), sizeof(BatchItemDev) * NI, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g.d_cfgs, g.cfgs.data(), sizeof(WalkCfg) * NI, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            rc = fail_cuda(e, "batch buffers");
            break;
        }
    }
    if (!rc) rc = upload_views(b, st);
    if (!rc) {
        const cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = fail_cuda(e, "cudaStreamCreateWithFlags");
    }
    if (rc) {
        for (BatchGroup &g : b->groups) free_group(g, st);
        cudaStreamSynchronize(st);
        if (b->cap) cudaStreamDestroy(b->cap);
        delete b;
        return rc;
    }
    *out = b;
    return 0;
}

int wos_batch_set_launch(wos_batch_t b, int block_threads, int blocks_per_sm, int chunk) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (block_threads % 32 || block_threads < 32 || block_threads > 512)
        return fail(WOS_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 in [32, 512]");
    if (chunk < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "chunk must be >= 1");
    for (auto &d : b->slot)
        for (auto &ph : d) {
            ph.block = block_threads;
            ph.blocks_per_sm = std::max(0, blocks_per_sm);
            ph.chunk = chunk;
        }
    drop_graph(b);
    return 0;
}

int wos_batch_autotune(wos_batch_t b, const int32_t *block_threads, const int32_t *chunk, int n_candidates,
                       int repeats, wos_stream_t stream, float *ms, int32_t *best) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (block_threads == nullptr || chunk == nullptr || n_candidates < 1 || repeats < 1)
        return fail(WOS_ERR_INVALID_ARGUMENT, "autotune needs candidates and repeats >= 1");
    for (int i = 0; i < n_candidates; ++i)
        if (block_threads[i] % 32 || block_threads[i] < 32 || block_threads[i] > 512 || chunk[i] < 1)
            return fail(WOS_ERR_INVALID_ARGUMENT, "candidate " + std::to_string(i) + ": invalid launch shape");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    BT(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fail(WOS_ERR_INVALID_ARGUMENT, "autotune during stream capture");
    BatchLaunch keep[2][2];
    std::copy(&b->slot[0][0], &b->slot[0][0] + 4, &keep[0][0]);
    set_count_work(b, 0);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BT(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail_cuda(e, "cudaEventCreate");
    }
    int rc = 0, arg = -1;
    float best_ms = INFINITY;
    for (int i = 0; i < n_candidates && !rc; ++i) {
        for (auto &d : b->slot)
            for (auto &ph : d) {
                ph.block = block_threads[i];
                ph.chunk = chunk[i];
            }
        float t = INFINITY;
        for (int r = 0; r <= repeats && !rc; ++r) {
            if ((e = cudaEventRecord(e0, st)) != cudaSuccess) rc = fail_cuda(e, "cudaEventRecord");
            if (!rc) rc = enqueue(b, st);
            if (!rc && (e = cudaEventRecord(e1, st)) != cudaSuccess) rc = fail_cuda(e, "cudaEventRecord");
            if (!rc && (e = cudaEventSynchronize(e1)) != cudaSuccess) rc = fail_cuda(e, "cudaEventSynchronize");
            float x = 0.0f;
            if (!rc && (e = cudaEventElapsedTime(&x, e0, e1)) != cudaSuccess) rc = fail_cuda(e, "cudaEventElapsedTime");
            if (!rc && r > 0) t = std::min(t, x);  // r = 0 is the untimed step
        }
        if (ms) ms[i] = t;
        if (!rc && t < best_ms) {
            best_ms = t;
            arg = i;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::copy(&keep[0][0], &keep[0][0] + 4, &b->slot[0][0]);
    if (rc) return rc;
    for (auto &d : b->slot)
        for (auto &ph : d) {
            ph.block = block_threads[arg];
            ph.chunk = chunk[arg];
        }
    drop_graph(b);
    if (best) *best = arg;
    return 0;
}

int wos_batch_autotune_slots(wos_batch_t b, const int32_t *block_threads, const int32_t *blocks_per_sm,
                             const int32_t *chunk, int n_candidates, int repeats, double sample, wos_stream_t stream,
                             float *ms, int32_t *best) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (block_threads == nullptr || blocks_per_sm == nullptr || chunk == nullptr || n_candidates < 1 ||
        repeats < 1)
        return fail(WOS_ERR_INVALID_ARGUMENT, "autotune needs candidates and repeats >= 1");
    if (!(sample > 0.0 && sample <= 1.0)) return fail(WOS_ERR_INVALID_ARGUMENT, "sample must be in (0, 1]");
    for (int i = 0; i < n_candidates; ++i)
        if (block_threads[i] % 32 || block_threads[i] < 32 || block_threads[i] > 512 || chunk[i] < 1 ||
            blocks_per_sm[i] < 0)
            return fail(WOS_ERR_INVALID_ARGUMENT, "candidate " + std::to_string(i) + ": invalid launch shape");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    BT(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fail(WOS_ERR_INVALID_ARGUMENT, "autotune during stream capture");
    const int count = b->slot[0][0].count_work;
    set_count_work(b, 0);
    for (int k = 0; k < 4; ++k) {
        if (ms)
            for (int i = 0; i < n_candidates; ++i) ms[k * n_candidates + i] = NAN;
        if (best) best[k] = -1;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BT(cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail_cuda(e, "cudaEventCreate");
    }
    // one full step first: the adjoint slots read the walk phase's outputs
    int rc = enqueue(b, st);
    for (int dim = 2; dim <= 3 && !rc; ++dim) {
        bool present = false;
        for (const BatchGroup &g : b->groups) present = present || g.dim == dim;
        if (!present) continue;
        for (int phase = 0; phase < (b->want_adjoint ? 2 : 1) && !rc; ++phase) {
            BatchLaunch &L = b->slot[dim - 2][phase];
            const int k = (dim - 2) * 2 + phase;
            int arg = -1;
            float best_ms = INFINITY;
            for (int i = 0; i < n_candidates && !rc; ++i) {
                L.block = block_threads[i];
                L.blocks_per_sm = blocks_per_sm[i];
                L.chunk = chunk[i];
                float t = INFINITY;
                for (int r = 0; r < repeats && !rc; ++r) {
                    if ((e = cudaEventRecord(e0, st)) != cudaSuccess) rc = fail_cuda(e, "cudaEventRecord");
                    if (!rc) rc = enqueue_slot(b, dim, phase, sample, st);
                    if (!rc && (e = cudaEventRecord(e1, st)) != cudaSuccess) rc = fail_cuda(e, "cudaEventRecord");
                    if (!rc && (e = cudaEventSynchronize(e1)) != cudaSuccess) rc = fail_cuda(e, "cudaEventSynchronize");
                    float x = 0.0f;
                    if (!rc && (e = cudaEventElapsedTime(&x, e0, e1)) != cudaSuccess)
                        rc = fail_cuda(e, "cudaEventElapsedTime");
                    if (!rc) t = std::min(t, x);
                }
                if (ms) ms[k * n_candidates + i] = t;
                if (!rc && t < best_ms) {
                    best_ms = t;
                    arg = i;
                }
            }
            if (arg >= 0) {
                L.block = block_threads[arg];
                L.blocks_per_sm = blocks_per_sm[arg];
                L.chunk = chunk[arg];
            }
            if (best) best[k] = arg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    set_count_work(b, count);
    drop_graph(b);
    return rc;
}

int wos_batch_set_launch_slot(wos_batch_t b, int dim, int phase, int block_threads, int blocks_per_sm, int chunk) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (dim < 2 || dim > 3 || phase < 0 || phase > 1) return fail(WOS_ERR_INVALID_ARGUMENT, "dim 2-3, phase 0-1");
    if (block_threads % 32 || block_threads < 32 || block_threads > 512)
        return fail(WOS_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 in [32, 512]");
    if (chunk < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "chunk must be >= 1");
    BatchLaunch &L = b->slot[dim - 2][phase];
    L.block = block_threads;
    L.blocks_per_sm = std::max(0, blocks_per_sm);
    L.chunk = chunk;
    drop_graph(b);
    return 0;
}

int wos_batch_get_launch(wos_batch_t b, int dim, int phase, int32_t *out) {
    if (b == nullptr || out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch or out is NULL");
    if (dim < 2 || dim > 3 || phase < 0 || phase > 1) return fail(WOS_ERR_INVALID_ARGUMENT, "dim 2-3, phase 0-1");
    const BatchLaunch &L = b->slot[dim - 2][phase];
    out[0] = L.block;
    out[1] = L.blocks_per_sm;
    out[2] = L.chunk;
    return 0;
}

int wos_batch_refresh(wos_batch_t b, wos_stream_t stream) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    drop_graph(b);
    return upload_views(b, (cudaStream_t)stream);
}

int wos_batch_run(wos_batch_t b, int use_graph, wos_stream_t stream) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    // scenes changed since their views were read are read again, and the
    // graph that holds the old views is captured anew
    if (stale_views(b)) {
        drop_graph(b);
        if (int rc = upload_views(b, st)) return rc;
    }
    // the work-counting flag is a kernel argument: a captured graph keeps the
    // value it was captured with, so a change forces a new capture
    const int count = work_counting_enabled();
    if (!use_graph) {
        set_count_work(b, count);
        return enqueue(b, st);
    }
    if (b->exec == nullptr || b->slot[0][0].count_work != count) {
        set_count_work(b, count);
        if (int rc = capture(b)) return rc;
    }
    const cudaError_t e = cudaGraphLaunch(b->exec, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGraphLaunch");
    return 0;
}

int wos_batch_outputs(wos_batch_t b, int item, const double **mean, const double **var, const double **loss,
                      const float **dV, const float **dg, const float **dsrc) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (item < 0 || item >= b->n_items) return fail(WOS_ERR_INVALID_ARGUMENT, "item out of range");
    const BatchGroup &g = b->groups[b->where[item].first];
    const BatchItemDev &d = g.items[b->where[item].second];
    if (mean) *mean = g.mean + d.point_begin;
    if (var) *var = g.var + d.point_begin;
    if (loss) *loss = g.loss + b->where[item].second;
    if (dV) *dV = g.grad ? g.grad + d.dV_off : nullptr;
    if (dg) *dg = g.grad ? g.grad + d.dg_off : nullptr;
    if (dsrc) *dsrc = g.grad ? g.grad + d.ds_off : nullptr;
    return 0;
}

int wos_batch_copy_outputs(wos_batch_t b, int item, double *mean, double *var, double *loss, float *dV, float *dg,
                           float *dsrc, wos_stream_t stream) {
    const double *m, *v, *l;
    const float *gV, *gg, *gs;
    if (int rc = wos_batch_outputs(b, item, &m, &v, &l, &gV, &gg, &gs)) return rc;
    const BatchGroup &g = b->groups[b->where[item].first];
    const BatchItemDev &d = g.items[b->where[item].second];
    const SceneImpl &S = g.scenes[b->where[item].second]->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const cudaMemcpyKind K = cudaMemcpyDeviceToDevice;
    if (mean) BT(cudaMemcpyAsync(mean, m, sizeof(double) * d.n, K, st));
    if (var) BT(cudaMemcpyAsync(var, v, sizeof(double) * d.n, K, st));
    if (loss) BT(cudaMemcpyAsync(loss, l, sizeof(double), K, st));
    if (gV && dV) BT(cudaMemcpyAsync(dV, gV, sizeof(float) * S.nV * S.dim, K, st));
    if (gg && dg) BT(cudaMemcpyAsync(dg, gg, sizeof(float) * S.nV, K, st));
    if (gs && dsrc) BT(cudaMemcpyAsync(dsrc, gs, sizeof(float) * 5, K, st));
    return 0;
}

int wos_batch_info(wos_batch_t b, int64_t *total_walks, int64_t *total_points, int32_t *n_groups) {
    if (b == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "batch is NULL");
    long long w = 0, p = 0;
    for (const BatchGroup &g : b->groups) {
        w += g.walks;
        p += g.points;
    }
    if (total_walks) *total_walks = w;
    if (total_points) *total_points = p;
    if (n_groups) *n_groups = (int32_t)b->groups.size();
    return 0;
}

int wos_batch_destroy(wos_batch_t b, wos_stream_t stream) {
    if (b == nullptr) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    drop_graph(b);
    for (BatchGroup &g : b->groups) free_group(g, st);
    if (b->cap) {
        cudaStreamSynchronize(b->cap);
        cudaStreamDestroy(b->cap);
    }
    delete b;
    return 0;
}

}  // extern "C"
