// extern "C" entry points of libwos_b200.so (declared in include/wos_b200.h).
#include <cstring>
#include <string>

#include "../../include/wos_b200.h"
#include "scene_impl.h"
#include "walk.h"

namespace wosd {

static thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int fail_cuda(cudaError_t e, const char *where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return WOS_ERR_CUDA;
}

static bool is_device_ptr(const void *p) {
    if (p == nullptr) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

#define WOS_CHECK_DEV(ptr, name)                                                              \
    do {                                                                                      \
        if (!is_device_ptr(ptr))                                                              \
            return fail(WOS_ERR_INVALID_ARGUMENT, std::string(name) + " must be a device pointer"); \
    } while (0)

#define WOS_CHECK_DEV_OPT(ptr, name)            \
    do {                                        \
        if ((ptr) != nullptr) WOS_CHECK_DEV(ptr, name); \
    } while (0)

static int check_params(const wos_params *p) {
    if (p == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "params is NULL");
    if (p->nwalks < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "nwalks must be >= 1");
    if (p->nsteps < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "nsteps must be >= 0");
    if (!(p->epsilon >= 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "epsilon must be >= 0");
    return 0;
}

static int check_adj(const wos_adjoint_params *a) {
    if (a == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "adjoint params is NULL");
    if (!(a->epsilon2 >= 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "epsilon2 must be >= 0");
    if (!(a->clamping >= 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "clamping must be >= 0");
    return 0;
}

static AdjCfg make_adj(const wos_adjoint_params &a) {
    AdjCfg c;
    c.epsilon2 = a.epsilon2;
    c.clamping = a.clamping;
    c.control_variates = a.control_variates;
    c.source_in_nd = a.source_in_normal_derivative;
    c.ball_eps = a.ball_epsilon;
    c.want_dV = a.want_dV;
    c.want_dg = a.want_dg;
    c.want_dsrc = a.want_dsrc;
    return c;
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Stream-ordered scratch that is either carved from the caller's workspace
// or allocated (and freed) on the stream.
struct Scratch {
    char *base = nullptr;
    bool owned = false;
    cudaStream_t st = nullptr;
    int init(void *ws, size_t ws_bytes, size_t need, cudaStream_t s) {
        st = s;
        if (ws != nullptr) {
            if (ws_bytes < need) return fail(WOS_ERR_WORKSPACE, "workspace too small");
            if (!is_device_ptr(ws)) return fail(WOS_ERR_INVALID_ARGUMENT, "workspace must be a device pointer");
            base = (char *)ws;
            return 0;
        }
        const cudaError_t e = cudaMallocAsync((void **)&base, need ? need : 256, s);
        if (e != cudaSuccess) return fail_cuda(e, "cudaMallocAsync(workspace)");
        owned = true;
        return 0;
    }
    ~Scratch() {
        if (owned && base) cudaFreeAsync(base, st);
    }
};

}  // namespace wosd

using namespace wosd;

extern "C" {

int wos_version(void) { return 100; }

const char *wos_last_error_string(void) { return g_last_error.c_str(); }

int wos_device_status(int reset, int32_t *out) {
    if (out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "out is NULL");
    int v = 0;
    const int rc = read_status(reset, &v);
    *out = v;
    return rc;
}

int wos_scene_create(int dim, const float *V, int nV, const int *F, int nF, const float *g, int source_type,
                     const float *source_params, wos_stream_t stream, wos_scene_t *out) {
    if (out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (dim != 2 && dim != 3) return fail(WOS_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
    if (nV < 1 || nF < 1) return fail(WOS_ERR_EMPTY_SCENE, "scene needs at least one vertex and one face");
    if (source_type < 0 || source_type > 2) return fail(WOS_ERR_INVALID_ARGUMENT, "source_type must be 0, 1 or 2");
    if (dim == 3 && source_type != 0) return fail(WOS_ERR_UNSUPPORTED, "3D scenes have no source term");
    if (source_type != 0 && source_params == nullptr)
        return fail(WOS_ERR_INVALID_ARGUMENT, "source_params is NULL for a source");
    WOS_CHECK_DEV(V, "V");
    WOS_CHECK_DEV(F, "F");
    WOS_CHECK_DEV(g, "g");
    cudaStream_t st = (cudaStream_t)stream;
    wos_scene_s *s = new wos_scene_s();
    SceneImpl &S = s->impl;
    S.dim = dim;
    S.nV = nV;
    S.nF = nF;
    cudaGetDevice(&S.device);
    S.src_type = source_type;
    for (int k = 0; k < 5; ++k) S.src[k] = source_type ? source_params[k] : 0.0f;
    int rc = S.allocate(st);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(S.V, V, sizeof(float) * nV * dim, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(S.F, F, sizeof(int) * nF * dim, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(S.g, g, sizeof(float) * nV, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) rc = fail_cuda(e, "cudaMemcpyAsync(scene inputs)");
    }
    if (!rc) rc = S.check_indices(st);
    if (!rc) rc = S.build(st);
    if (rc) {
        S.release(st);
        cudaStreamSynchronize(st);
        delete s;
        return rc;
    }
    *out = s;
    return 0;
}

int wos_scene_destroy(wos_scene_t scene, wos_stream_t stream) {
    if (scene == nullptr) return 0;
    scene->impl.release((cudaStream_t)stream);
    delete scene;
    return 0;
}

int wos_scene_update_values(wos_scene_t scene, const float *g, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    WOS_CHECK_DEV(g, "g");
    SceneImpl &S = scene->impl;
    const cudaError_t e =
        cudaMemcpyAsync(S.g, g, sizeof(float) * S.nV, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync(values)");
    return 0;
}

int wos_scene_update_vertices(wos_scene_t scene, const float *V, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    WOS_CHECK_DEV(V, "V");
    SceneImpl &S = scene->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const cudaError_t e = cudaMemcpyAsync(S.V, V, sizeof(float) * S.nV * S.dim, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync(vertices)");
    return S.build(st);
}

int wos_scene_set_source(wos_scene_t scene, int source_type, const float *params) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (source_type < 0 || source_type > 2) return fail(WOS_ERR_INVALID_ARGUMENT, "source_type must be 0, 1 or 2");
    SceneImpl &S = scene->impl;
    if (S.dim == 3 && source_type != 0) return fail(WOS_ERR_UNSUPPORTED, "3D scenes have no source term");
    if (source_type != 0 && params == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "params is NULL");
    S.src_type = source_type;
    for (int k = 0; k < 5; ++k) S.src[k] = source_type ? params[k] : 0.0f;
    ++S.generation;
    return 0;
}

int wos_scene_get_info(wos_scene_t scene, wos_scene_info *out) {
    if (scene == nullptr || out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "NULL argument");
    const SceneImpl &S = scene->impl;
    out->dim = S.dim;
    out->n_vertices = S.nV;
    out->n_faces = S.nF;
    out->n_nodes = S.nNodes;
    out->bvh_depth = S.depth;
    out->source_type = S.src_type;
    for (int k = 0; k < 3; ++k) {
        out->aabb_min[k] = S.lo[k];
        out->aabb_max[k] = S.hi[k];
    }
    for (int k = 0; k < 5; ++k) out->source_params[k] = S.src[k];
    return 0;
}

int wos_scene_get_normals(wos_scene_t scene, float *out, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    WOS_CHECK_DEV(out, "out");
    const SceneImpl &S = scene->impl;
    const cudaError_t e =
        cudaMemcpyAsync(out, S.N, sizeof(float) * S.nV * S.dim, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyAsync(normals)");
    return 0;
}

int wos_closest_point(wos_scene_t scene, const float *P, int n, int use_bvh, int32_t *prim, float *dist,
                      float *t_or_uv, float *pt, float *normal, float *sdf, uint8_t *inside, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV_OPT(prim, "prim");
    WOS_CHECK_DEV_OPT(dist, "dist");
    WOS_CHECK_DEV_OPT(t_or_uv, "t_or_uv");
    WOS_CHECK_DEV_OPT(pt, "pt");
    WOS_CHECK_DEV_OPT(normal, "normal");
    WOS_CHECK_DEV_OPT(sdf, "sdf");
    WOS_CHECK_DEV_OPT(inside, "inside");
    QueryOut o{prim, dist, t_or_uv, pt, normal, sdf, inside};
    return launch_closest(scene->impl, P, n, use_bvh != 0, o, (cudaStream_t)stream);
}

int wos_sdf(wos_scene_t scene, const float *P, int n, int use_bvh, float *sdf, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(sdf, "sdf");
    QueryOut o{nullptr, nullptr, nullptr, nullptr, nullptr, sdf, nullptr};
    return launch_closest(scene->impl, P, n, use_bvh != 0, o, (cudaStream_t)stream);
}

int wos_largest_inscribed_ball(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal, int n,
                               float epsilon, int use_bvh, float *R, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(valid, "valid");
    WOS_CHECK_DEV(pt, "pt");
    WOS_CHECK_DEV(normal, "normal");
    WOS_CHECK_DEV(R, "R");
    return launch_ball(scene->impl, valid, pt, normal, n, epsilon, use_bvh != 0, R, (cudaStream_t)stream);
}

int wos_walk_records(wos_scene_t scene, const float *P, int n, const wos_params *p, uint8_t *valid, float *pt,
                     float *normal, float *t_or_uv, int32_t *prim, float *contrib, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(valid, "valid");
    WOS_CHECK_DEV_OPT(pt, "pt");
    WOS_CHECK_DEV_OPT(normal, "normal");
    WOS_CHECK_DEV_OPT(t_or_uv, "t_or_uv");
    WOS_CHECK_DEV_OPT(prim, "prim");
    WOS_CHECK_DEV_OPT(contrib, "contrib");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(nullptr, 0, 256, st)) return rc;
    WalkOut o{nullptr, nullptr, nullptr, nullptr, valid, pt, normal, t_or_uv, prim, contrib};
    return launch_walk(scene->impl, P, n, *p, true, o, (unsigned long long *)s.base, st);
}

int wos_walk_values(wos_scene_t scene, const float *P, int n, const wos_params *p, float *values, int32_t *steps,
                    wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(values, "values");
    WOS_CHECK_DEV_OPT(steps, "steps");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(nullptr, 0, 256, st)) return rc;
    WalkOut o{values, steps, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    return launch_walk(scene->impl, P, (long long)n * p->nwalks, *p, false, o, (unsigned long long *)s.base, st);
}

int wos_walk_values_plain(wos_scene_t scene, const float *P, int n, const wos_params *p, float *values,
                          wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(values, "values");
    return launch_walk_plain(scene->impl, P, (long long)n * p->nwalks, *p, values, (cudaStream_t)stream);
}

size_t wos_solve_workspace_size(int n, const wos_params *p) {
    if (p == nullptr || n < 0 || p->nwalks < 1) return 0;
    return 256 + align256(sizeof(float) * (size_t)n * (size_t)p->nwalks);
}

int wos_solve(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean, double *var,
              void *workspace, size_t workspace_bytes, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(mean, "mean");
    WOS_CHECK_DEV_OPT(var, "var");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, wos_solve_workspace_size(n, p), st)) return rc;
    unsigned long long *counter = (unsigned long long *)s.base;
    float *vals = (float *)(s.base + 256);
    WalkOut o{vals, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (int rc = launch_walk(scene->impl, P, (long long)n * p->nwalks, *p, false, o, counter, st)) return rc;
    return launch_reduce(vals, n, p->nwalks, mean, var, st);
}

static int normal_derivative_impl(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal,
                                  const float *t_or_uv, const int32_t *prim, const float *R, int n, const wos_params *p,
                                  const wos_adjoint_params *a, float *out, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (int rc = check_adj(a)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(valid, "valid");
    WOS_CHECK_DEV(pt, "pt");
    WOS_CHECK_DEV(normal, "normal");
    WOS_CHECK_DEV(t_or_uv, "t_or_uv");
    WOS_CHECK_DEV(prim, "prim");
    WOS_CHECK_DEV_OPT(R, "R");
    WOS_CHECK_DEV(out, "out");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(nullptr, 0, 256, st)) return rc;
    AdjOut o{};
    o.rvalid = valid;
    o.rpt = pt;
    o.rnrm = normal;
    o.rtuv = t_or_uv;
    o.rprim = prim;
    o.rR = R;
    o.nd = out;
    return launch_adjoint(scene->impl, nullptr, n, *p, make_adj(*a), nullptr, ADJ_ND_ONLY, o, (unsigned long long *)s.base,
                          st);
}

int wos_normal_derivative(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal,
                          const float *t_or_uv, const int32_t *prim, int n, const wos_params *p,
                          const wos_adjoint_params *a, float *out, wos_stream_t stream) {
    return normal_derivative_impl(scene, valid, pt, normal, t_or_uv, prim, nullptr, n, p, a, out, stream);
}

int wos_normal_derivative_radius(wos_scene_t scene, const uint8_t *valid, const float *pt, const float *normal,
                                 const float *t_or_uv, const int32_t *prim, const float *R, int n,
                                 const wos_params *p, const wos_adjoint_params *a, float *out, wos_stream_t stream) {
    if (R == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "R is NULL");
    return normal_derivative_impl(scene, valid, pt, normal, t_or_uv, prim, R, n, p, a, out, stream);
}

size_t wos_adjoint_workspace_size(wos_scene_t scene) {
    if (scene == nullptr) return 0;
    const SceneImpl &S = scene->impl;
    return 256 + align256(sizeof(double) * (size_t)S.nV * S.dim) + align256(sizeof(double) * (size_t)S.nV) + 256;
}

int wos_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p, const wos_adjoint_params *a,
                const float *dLdu, float *dV, float *dg, float *dsrc, void *workspace, size_t workspace_bytes,
                wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (int rc = check_adj(a)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    if (a->want_dV && dV == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dV set but dV is NULL");
    if (a->want_dg && dg == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dg set but dg is NULL");
    if (a->want_dsrc && dsrc == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dsrc set but dsrc is NULL");
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(dLdu, "dLdu");
    WOS_CHECK_DEV_OPT(dV, "dV");
    WOS_CHECK_DEV_OPT(dg, "dg");
    WOS_CHECK_DEV_OPT(dsrc, "dsrc");
    const SceneImpl &S = scene->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = wos_adjoint_workspace_size(scene);
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, need, st)) return rc;
    unsigned long long *counter = (unsigned long long *)s.base;
    double *aV = (double *)(s.base + 256);
    double *ag = (double *)((char *)aV + align256(sizeof(double) * (size_t)S.nV * S.dim));
    double *as = (double *)((char *)ag + align256(sizeof(double) * (size_t)S.nV));
    cudaError_t e = cudaMemsetAsync(s.base, 0, need, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(adjoint workspace)");
    AdjOut o{};
    o.dV = aV;
    o.dg = ag;
    o.dsrc = as;
    if (int rc = launch_adjoint(S, P, (long long)n * p->nwalks, *p, make_adj(*a), dLdu, ADJ_RECOMPUTE, o, counter, st))
        return rc;
    if (a->want_dV)
        if (int rc = launch_add_f64(aV, dV, (long long)S.nV * S.dim, st)) return rc;
    if (a->want_dg)
        if (int rc = launch_add_f64(ag, dg, S.nV, st)) return rc;
    if (a->want_dsrc)
        if (int rc = launch_add_f64(as, dsrc, 5, st)) return rc;
    return 0;
}

size_t wos_walk_record_bytes(int dim) { return dim == 3 ? 16 : 8; }

static bool wants_wds(const SceneImpl &S, const wos_params &p, const wos_adjoint_params &a) {
    return a.want_dsrc && p.include_source && S.src_type != 0 && S.dim == 2;
}

// Adjoint accumulators (double) at the start of a workspace region.
struct AdjAcc {
    double *dV, *dg, *ds;
    size_t bytes;
};
static AdjAcc adj_acc(const SceneImpl &S, char *base) {
    AdjAcc r;
    r.dV = (double *)base;
    r.dg = (double *)((char *)r.dV + align256(sizeof(double) * (size_t)S.nV * S.dim));
    r.ds = (double *)((char *)r.dg + align256(sizeof(double) * (size_t)S.nV));
    r.bytes = align256(sizeof(double) * (size_t)S.nV * S.dim) + align256(sizeof(double) * (size_t)S.nV) + 256;
    return r;
}

static int finish_adjoint(const SceneImpl &S, const wos_adjoint_params *a, const AdjAcc &acc, float *dV, float *dg,
                          float *dsrc, cudaStream_t st) {
    if (a->want_dV)
        if (int rc = launch_add_f64(acc.dV, dV, (long long)S.nV * S.dim, st)) return rc;
    if (a->want_dg)
        if (int rc = launch_add_f64(acc.dg, dg, S.nV, st)) return rc;
    if (a->want_dsrc)
        if (int rc = launch_add_f64(acc.ds, dsrc, 5, st)) return rc;
    return 0;
}

size_t wos_solve_adjoint_workspace_size(wos_scene_t scene, int n, const wos_params *p, const wos_adjoint_params *a) {
    if (scene == nullptr || p == nullptr || a == nullptr || n < 0 || p->nwalks < 1) return 0;
    const SceneImpl &S = scene->impl;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    size_t b = 256;                                                   // queue counter
    b += align256(sizeof(float) * nw);                                // per-walk values
    b += align256(wos_walk_record_bytes(S.dim) * nw);                 // per-walk records
    if (wants_wds(S, *p, *a)) b += align256(sizeof(float) * 5 * nw);  // per-walk source derivatives
    b += align256(sizeof(float) * (size_t)n);                         // dL/du
    b += adj_acc(S, nullptr).bytes;                                   // gradient accumulators
    b += align256(record_order_bytes(S.nF, (long long)nw));           // sample order
    return b;
}

int wos_solve_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p, const wos_adjoint_params *a,
                      int loss_kind, const float *target_or_dLdu, double *mean, double *var, double *loss, float *dV,
                      float *dg, float *dsrc, void *workspace, size_t workspace_bytes, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (int rc = check_adj(a)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (loss_kind < 0 || loss_kind > 2) return fail(WOS_ERR_INVALID_ARGUMENT, "loss_kind must be 0, 1 or 2");
    if (loss_kind != 1 && target_or_dLdu == nullptr)
        return fail(WOS_ERR_INVALID_ARGUMENT, "target_or_dLdu is NULL for this loss_kind");
    if (n == 0) return 0;
    if (a->want_dV && dV == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dV set but dV is NULL");
    if (a->want_dg && dg == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dg set but dg is NULL");
    if (a->want_dsrc && dsrc == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dsrc set but dsrc is NULL");
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(mean, "mean");
    WOS_CHECK_DEV_OPT(var, "var");
    WOS_CHECK_DEV_OPT(loss, "loss");
    WOS_CHECK_DEV_OPT(target_or_dLdu, "target_or_dLdu");
    WOS_CHECK_DEV_OPT(dV, "dV");
    WOS_CHECK_DEV_OPT(dg, "dg");
    WOS_CHECK_DEV_OPT(dsrc, "dsrc");
    const SceneImpl &S = scene->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = wos_solve_adjoint_workspace_size(scene, n, p, a);
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, need, st)) return rc;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    char *b = s.base;
    unsigned long long *counter = (unsigned long long *)b;
    b += 256;
    float *vals = (float *)b;
    b += align256(sizeof(float) * nw);
    int *wrec = (int *)b;
    b += align256(wos_walk_record_bytes(S.dim) * nw);
    float *wds = nullptr;
    if (wants_wds(S, *p, *a)) {
        wds = (float *)b;
        b += align256(sizeof(float) * 5 * nw);
    }
    float *dLdu = (float *)b;
    b += align256(sizeof(float) * (size_t)n);
    const AdjAcc acc = adj_acc(S, b);
    cudaError_t e = cudaMemsetAsync(b, 0, acc.bytes, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(adjoint accumulators)");
    b += acc.bytes;
    WalkOut o{vals, nullptr, wrec, wds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (int rc = launch_walk(S, P, (long long)nw, *p, false, o, counter, st)) return rc;
    if (int rc = launch_reduce(vals, n, p->nwalks, mean, var, st)) return rc;
    if (int rc = launch_loss(mean, n, loss_kind, target_or_dLdu, dLdu, loss, st)) return rc;
    AdjOut ao{};
    ao.dV = acc.dV;
    ao.dg = acc.dg;
    ao.dsrc = acc.ds;
    ao.wrec = wrec;
    ao.wds = wds;
    if (int rc = launch_record_order(S, wrec, (long long)nw, b, need - (size_t)(b - s.base), &ao.order, st))
        return rc;
    if (int rc = launch_adjoint(S, P, (long long)nw, *p, make_adj(*a), dLdu, ADJ_FROM_RECORDS, ao, counter, st))
        return rc;
    return finish_adjoint(S, a, acc, dV, dg, dsrc, st);
}

size_t wos_solve_tangent_workspace_size(wos_scene_t scene, int n, const wos_params *p, const wos_adjoint_params *a) {
    if (scene == nullptr || p == nullptr || a == nullptr || n < 0 || p->nwalks < 1) return 0;
    const SceneImpl &S = scene->impl;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    size_t b = 256;                                                   // queue counter
    b += align256(sizeof(float) * nw);                                // per-walk values
    b += align256(wos_walk_record_bytes(S.dim) * nw);                 // per-walk records
    if (wants_wds(S, *p, *a)) b += align256(sizeof(float) * 5 * nw);  // per-walk source derivatives
    b += align256(sizeof(float) * nw);                                // per-walk tangents
    b += align256(record_order_bytes(S.nF, (long long)nw));           // sample order
    return b;
}

int wos_solve_tangent(wos_scene_t scene, const float *P, int n, const wos_params *p, const wos_adjoint_params *a,
                      const float *dV_dir, const float *dg_dir, const float *dsrc_dir, double *mean, double *var,
                      double *tangent, double *tangent_var, void *workspace, size_t workspace_bytes,
                      wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (int rc = check_adj(a)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(mean, "mean");
    WOS_CHECK_DEV_OPT(var, "var");
    WOS_CHECK_DEV(tangent, "tangent");
    WOS_CHECK_DEV_OPT(tangent_var, "tangent_var");
    WOS_CHECK_DEV_OPT(dV_dir, "dV_dir");
    WOS_CHECK_DEV_OPT(dg_dir, "dg_dir");
    WOS_CHECK_DEV_OPT(dsrc_dir, "dsrc_dir");
    const SceneImpl &S = scene->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = wos_solve_tangent_workspace_size(scene, n, p, a);
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, need, st)) return rc;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    char *b = s.base;
    unsigned long long *counter = (unsigned long long *)b;
    b += 256;
    float *vals = (float *)b;
    b += align256(sizeof(float) * nw);
    int *wrec = (int *)b;
    b += align256(wos_walk_record_bytes(S.dim) * nw);
    float *wds = nullptr;
    if (wants_wds(S, *p, *a)) {
        wds = (float *)b;
        b += align256(sizeof(float) * 5 * nw);
    }
    float *tan = (float *)b;
    b += align256(sizeof(float) * nw);
    cudaError_t e = cudaMemsetAsync(tan, 0, sizeof(float) * nw, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(tangents)");
    WalkOut o{vals, nullptr, wrec, wds, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (int rc = launch_walk(S, P, (long long)nw, *p, false, o, counter, st)) return rc;
    if (int rc = launch_reduce(vals, n, p->nwalks, mean, var, st)) return rc;
    AdjOut ao{};
    ao.wrec = wrec;
    ao.wds = wds;
    ao.tV = dV_dir;
    ao.tg = dg_dir;
    ao.ts = dsrc_dir;
    ao.tan = tan;
    if (int rc = launch_record_order(S, wrec, (long long)nw, b, need - (size_t)(b - s.base), &ao.order, st))
        return rc;
    if (int rc = launch_adjoint(S, P, (long long)nw, *p, make_adj(*a), nullptr, ADJ_TANGENT, ao, counter, st))
        return rc;
    return launch_reduce(tan, n, p->nwalks, tangent, tangent_var, st);
}

size_t wos_soft_walk_workspace_size(int n, const wos_params *p) {
    if (p == nullptr || n < 0 || p->nwalks < 1) return 0;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    return 256 + 2 * align256(sizeof(float) * nw);
}

int wos_soft_walk(wos_scene_t scene, const float *P, int n, const wos_params *p, const float *dV_dir,
                  const float *dg_dir, double *mean, double *var, double *tangent, double *tangent_var, void *workspace,
                  size_t workspace_bytes, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (p->nsteps < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "the soft-edge walk needs nsteps >= 1");
    if (!(p->epsilon > 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "the soft-edge walk needs epsilon > 0");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(mean, "mean");
    WOS_CHECK_DEV_OPT(var, "var");
    WOS_CHECK_DEV_OPT(tangent, "tangent");
    WOS_CHECK_DEV_OPT(tangent_var, "tangent_var");
    WOS_CHECK_DEV_OPT(dV_dir, "dV_dir");
    WOS_CHECK_DEV_OPT(dg_dir, "dg_dir");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, wos_soft_walk_workspace_size(n, p), st)) return rc;
    const size_t nw = (size_t)n * (size_t)p->nwalks;
    unsigned long long *counter = (unsigned long long *)s.base;
    float *vals = (float *)(s.base + 256);
    float *tans = tangent != nullptr ? (float *)(s.base + 256 + align256(sizeof(float) * nw)) : nullptr;
    if (int rc = launch_walk_soft(scene->impl, P, (long long)nw, *p, dV_dir, dg_dir, vals, tans, counter, st))
        return rc;
    if (int rc = launch_reduce(vals, n, p->nwalks, mean, var, st)) return rc;
    if (tans != nullptr) return launch_reduce(tans, n, p->nwalks, tangent, tangent_var, st);
    return 0;
}

int wos_soft_walk_adjoint(wos_scene_t scene, const float *P, int n, const wos_params *p, const float *dLdu, float *dV,
                          float *dg, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (p->nsteps < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "the soft-edge walk needs nsteps >= 1");
    if (!(p->epsilon > 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "the soft-edge walk needs epsilon > 0");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0 || (dV == nullptr && dg == nullptr)) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(dLdu, "dLdu");
    WOS_CHECK_DEV_OPT(dV, "dV");
    WOS_CHECK_DEV_OPT(dg, "dg");
    const SceneImpl &S = scene->impl;
    cudaStream_t st = (cudaStream_t)stream;
    const long long nvd = (long long)S.nV * S.dim;
    double *acc = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&acc, sizeof(double) * (size_t)(nvd + S.nV), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMallocAsync(soft adjoint accumulators)");
    e = cudaMemsetAsync(acc, 0, sizeof(double) * (size_t)(nvd + S.nV), st);
    int rc = e == cudaSuccess ? 0 : fail_cuda(e, "cudaMemsetAsync(soft adjoint accumulators)");
    if (rc == 0)
        rc = launch_soft_adjoint(S, P, (long long)n * p->nwalks, *p, dLdu, acc, dg != nullptr ? acc + nvd : nullptr,
                                 st);
    if (rc == 0 && dV != nullptr) rc = launch_add_f64(acc, dV, nvd, st);
    if (rc == 0 && dg != nullptr) rc = launch_add_f64(acc + nvd, dg, S.nV, st);
    cudaFreeAsync(acc, st);
    return rc;
}

int wos_boundary_term(wos_scene_t scene, const wos_detector *det, int nwalks, uint64_t seed, const float *dV_dir,
                      double *image_tangent, const float *dLdI, float *dV, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (det == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "detector is NULL");
    if (nwalks < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "nwalks must be >= 1");
    const SceneImpl &S = scene->impl;
    if (det->res[0] < 1 || det->res[1] < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "detector res must be >= 1");
    if (!(det->vmax[0] > det->vmin[0]) || !(det->vmax[1] > det->vmin[1]))
        return fail(WOS_ERR_INVALID_ARGUMENT, "detector vmax must exceed vmin");
    if (det->axis_u < 0 || det->axis_u >= S.dim || det->axis_v < 0 || det->axis_v >= S.dim ||
        det->slab_axis < -1 || det->slab_axis >= S.dim)
        return fail(WOS_ERR_INVALID_ARGUMENT, "detector axes out of range for the scene's dimension");
    if (!(det->size > 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "detector size must be > 0");
    if ((det->flags & ~WOS_DETECTOR_REFERENCE_AREA_PDF) != 0)
        return fail(WOS_ERR_INVALID_ARGUMENT, "unknown detector flags");
    if ((dV_dir == nullptr) != (image_tangent == nullptr))
        return fail(WOS_ERR_INVALID_ARGUMENT, "dV_dir and image_tangent go together");
    if ((dLdI == nullptr) != (dV == nullptr)) return fail(WOS_ERR_INVALID_ARGUMENT, "dLdI and dV go together");
    WOS_CHECK_DEV_OPT(dV_dir, "dV_dir");
    WOS_CHECK_DEV_OPT(image_tangent, "image_tangent");
    WOS_CHECK_DEV_OPT(dLdI, "dLdI");
    WOS_CHECK_DEV_OPT(dV, "dV");
    if (dV_dir == nullptr && dLdI == nullptr) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    double *acc = nullptr;
    const long long nvd = (long long)S.nV * S.dim;
    if (dV != nullptr) {
        cudaError_t e = cudaMallocAsync((void **)&acc, sizeof(double) * (size_t)std::max<long long>(nvd, 1), st);
        if (e != cudaSuccess) return fail_cuda(e, "cudaMallocAsync(boundary accumulators)");
        e = cudaMemsetAsync(acc, 0, sizeof(double) * (size_t)nvd, st);
        if (e != cudaSuccess) {
            cudaFreeAsync(acc, st);
            return fail_cuda(e, "cudaMemsetAsync(boundary accumulators)");
        }
    }
    int rc = launch_boundary(S, *det, nwalks, seed, dV_dir, image_tangent, dLdI, acc, st);
    if (rc == 0 && acc != nullptr) rc = launch_add_f64(acc, dV, nvd, st);
    if (acc != nullptr) cudaFreeAsync(acc, st);
    return rc;
}

int wos_solve_records(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean, double *var,
                      void *records, float *dcontrib, void *workspace, size_t workspace_bytes, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(mean, "mean");
    WOS_CHECK_DEV_OPT(var, "var");
    WOS_CHECK_DEV(records, "records");
    WOS_CHECK_DEV_OPT(dcontrib, "dcontrib");
    cudaStream_t st = (cudaStream_t)stream;
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, wos_solve_workspace_size(n, p), st)) return rc;
    unsigned long long *counter = (unsigned long long *)s.base;
    float *vals = (float *)(s.base + 256);
    WalkOut o{vals, nullptr, (int *)records, dcontrib, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (int rc = launch_walk(scene->impl, P, (long long)n * p->nwalks, *p, false, o, counter, st)) return rc;
    return launch_reduce(vals, n, p->nwalks, mean, var, st);
}

size_t wos_adjoint_records_workspace_size(wos_scene_t scene, int n, const wos_params *p) {
    if (scene == nullptr || p == nullptr || n < 0 || p->nwalks < 1) return 0;
    return wos_adjoint_workspace_size(scene) +
           align256(record_order_bytes(scene->impl.nF, (long long)n * (long long)p->nwalks));
}

int wos_adjoint_records(wos_scene_t scene, const float *P, int n, const wos_params *p, const wos_adjoint_params *a,
                        const float *dLdu, const void *records, const float *dcontrib, float *dV, float *dg,
                        float *dsrc, void *workspace, size_t workspace_bytes, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (int rc = check_params(p)) return rc;
    if (int rc = check_adj(a)) return rc;
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    if (n == 0) return 0;
    const SceneImpl &S = scene->impl;
    if (a->want_dV && dV == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dV set but dV is NULL");
    if (a->want_dg && dg == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dg set but dg is NULL");
    if (a->want_dsrc && dsrc == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "want_dsrc set but dsrc is NULL");
    if (wants_wds(S, *p, *a) && dcontrib == nullptr)
        return fail(WOS_ERR_INVALID_ARGUMENT, "source gradient requested but dcontrib is NULL");
    WOS_CHECK_DEV(P, "P");
    WOS_CHECK_DEV(dLdu, "dLdu");
    WOS_CHECK_DEV(records, "records");
    WOS_CHECK_DEV_OPT(dcontrib, "dcontrib");
    WOS_CHECK_DEV_OPT(dV, "dV");
    WOS_CHECK_DEV_OPT(dg, "dg");
    WOS_CHECK_DEV_OPT(dsrc, "dsrc");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t need = wos_adjoint_workspace_size(scene);
    const size_t need_ordered = wos_adjoint_records_workspace_size(scene, n, p);
    const bool ordered = workspace == nullptr || workspace_bytes >= need_ordered;
    Scratch s;
    if (int rc = s.init(workspace, workspace_bytes, ordered ? need_ordered : need, st)) return rc;
    unsigned long long *counter = (unsigned long long *)s.base;
    const AdjAcc acc = adj_acc(S, s.base + 256);
    cudaError_t e = cudaMemsetAsync(s.base, 0, need, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(adjoint workspace)");
    AdjOut ao{};
    ao.dV = acc.dV;
    ao.dg = acc.dg;
    ao.dsrc = acc.ds;
    ao.wrec = (const int *)records;
    ao.wds = dcontrib;
    if (ordered && need_ordered > need)
        if (int rc = launch_record_order(S, ao.wrec, (long long)n * p->nwalks, s.base + need, need_ordered - need,
                                         &ao.order, st))
            return rc;
    if (int rc = launch_adjoint(S, P, (long long)n * p->nwalks, *p, make_adj(*a), dLdu, ADJ_FROM_RECORDS, ao, counter,
                                st))
        return rc;
    return finish_adjoint(S, a, acc, dV, dg, dsrc, st);
}

int wos_set_work_counting(int enable) { return set_work_counting(enable); }

int wos_set_sample_order(int mode) { return set_sample_order(mode); }

int wos_work_counters(int reset, int64_t *out) {
    if (out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "out is NULL");
    unsigned long long v[3] = {0, 0, 0};
    const int rc = read_work(reset, v);
    for (int k = 0; k < 3; ++k) out[k] = (int64_t)v[k];
    return rc;
}

int wos_set_launch_config(int dim, const wos_launch_config *cfg) {
    if (cfg == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "cfg is NULL");
    return set_launch_config(dim, cfg);
}

int wos_get_launch_config(int dim, wos_launch_config *out) {
    if (out == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "out is NULL");
    return get_launch_config(dim, out);
}

}  // extern "C"
