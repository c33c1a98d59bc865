// Launch-side interface of the walk kernels (walk.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "scene_impl.h"
#include "wos_device.cuh"

namespace wosd {

// Device copy of wos_params.
struct WalkCfg {
    int nwalks, nsteps;
    float eps;
    int double_sided, prevent_fd, use_IS, include_source, project;
    uint32_t walk_offset;
    Rng rng;
    int count;  // accumulate LBVH work counters (wos_set_work_counting)
    float jitter[3];  // start-point jitter extent per axis (0: none)
};

// Device copy of wos_adjoint_params.
struct AdjCfg {
    float epsilon2, clamping;
    int control_variates, source_in_nd;
    float ball_eps;
    int want_dV, want_dg, want_dsrc;
};

struct WalkOut {
    float *values;
    int *steps;
    int *wrec;   // per-walk WalkRec (walkrec_words(D) ints each), may be null
    float *wds;  // per-walk source-parameter derivative (5 floats each), may be null
    uint8_t *valid;
    float *pt, *nrm, *tuv;
    int *prim;
    float *contrib;
};

struct QueryOut {
    int *prim;
    float *dist, *tuv, *pt, *nrm, *sdf;
    uint8_t *inside;
};

struct AdjOut {
    double *dV, *dg, *dsrc;
    // normal-derivative-only mode: input records and the output estimates
    const uint8_t *rvalid;
    const float *rpt, *rnrm, *rtuv;
    const int *rprim;
    const float *rR;  // given ball radii (override_R), or null: the inscribed ball
    float *nd;
    // records mode: per-walk WalkRec and source derivatives from the forward pass
    const int *wrec;
    const float *wds;
    // tangent mode: directions of vertices (nV x dim), values (nV) and source
    // parameters (5), each may be null; per-walk directional derivative out
    const float *tV, *tg, *ts;
    float *tan;
    // records and tangent modes: sample processed at queue position i, or
    // null for queue order (launch_record_order)
    const unsigned *order;
};

// ADJ_TANGENT: forward mode from records -- each walk's derivative along a
// direction of (vertices, values, source parameters) instead of the scatter
// of dL/du into their gradients.
enum AdjMode { ADJ_RECOMPUTE = 0, ADJ_ND_ONLY = 1, ADJ_FROM_RECORDS = 2, ADJ_TANGENT = 3 };

// One (scene, query set) item of a batched launch, in device memory.
struct BatchItemDev {
    const float *P;          // n x dim query points
    long long walk_begin;    // first index of this item in the concatenated walk space
    int n, nwalks;
    int point_begin;         // first index in the concatenated point space
    int loss_kind;           // 0: dL/du given, 1: mean(u^2), 2: mean((u - target)^2)
    const float *target;     // n floats (kinds 0 and 2)
    long long dV_off, dg_off, ds_off;  // offsets of its FP64 gradient accumulators
    long long prim_off;      // first sort key of its primitives (sum of nF + 1 over earlier items)
};

struct BatchLaunch {
    int block, blocks_per_sm, chunk, count_work;
};

WalkCfg make_cfg(const wos_params &p);
AdjCfg make_adj_cfg(const wos_adjoint_params &a);
// Tree depths with their own kernel instance; deeper trees use the
// any-depth instance (depth argument 0).
constexpr int WT_SPECIALISED_LEVELS = 3;
inline int specialised_depth(int wt_levels) { return wt_levels <= WT_SPECIALISED_LEVELS ? wt_levels : 0; }

// A batch launch covers items [0, n_items) of `items` / `views` / `cfgs`
// (callers pass pointers offset to a run of items) whose walks are
// [base, base + total) of the group's walk index space; wl: the run's
// common tree depth (specialised_depth), 0 for mixed or deep trees.
int launch_walk_batch(int D, int wl, const SceneView *views, const WalkCfg *cfgs, const BatchItemDev *items,
                      int n_items, long long base, long long total, const BatchLaunch &L, const WalkOut &out,
                      unsigned long long *counter, cudaStream_t st);
int launch_adjoint_batch(int D, int wl, const SceneView *views, const WalkCfg *cfgs, const AdjCfg &a,
                         const BatchItemDev *items, int n_items, long long base, long long total,
                         const float *dLdu, const int *wrec, const float *wds, double *acc, const BatchLaunch &L,
                         unsigned long long *counter, const unsigned *order, cudaStream_t st);
// Sample order of a batch group's adjoint (see launch_record_order): nkeys =
// sum of nF + 1 over the group's items; 0 bytes: no order for this size.
size_t batch_order_bytes(long long nkeys, long long total);
int launch_batch_order(int D, const SceneView *views, const BatchItemDev *items, int n_items, long long nkeys,
                       const int *wrec, long long total, void *ws, size_t ws_bytes, const unsigned **order,
                       cudaStream_t st);
int launch_reduce_batch(const float *vals, const BatchItemDev *items, int n_items, int n_points, double *mean,
                        double *var, cudaStream_t st);
int launch_loss_batch(const double *mean, const BatchItemDev *items, int n_items, float *dLdu, double *loss,
                      cudaStream_t st);
int launch_acc_to_f32(const double *acc, float *out, long long n, cudaStream_t st);
int read_status(int reset, int *out);
int read_work(int reset, unsigned long long *out);
int set_work_counting(int enable);
int work_counting_enabled();
int set_launch_config(int dim, const wos_launch_config *cfg);
int get_launch_config(int dim, wos_launch_config *out);

int launch_walk(const SceneImpl &S, const float *P, long long total, const wos_params &p, bool records,
                const WalkOut &out, unsigned long long *counter, cudaStream_t st);
// Soft-edge walk values (and, with tans, forward-mode tangents along tV / tg).
int launch_walk_soft(const SceneImpl &S, const float *P, long long total, const wos_params &p, const float *tV,
                     const float *tg, float *vals, float *tans, unsigned long long *counter, cudaStream_t st);
int launch_walk_plain(const SceneImpl &S, const float *P, long long total, const wos_params &p, float *values,
                      cudaStream_t st);
int launch_reduce(const float *vals, int n, int nw, double *mean, double *var, cudaStream_t st);
int launch_soft_adjoint(const SceneImpl &S, const float *P, long long total, const wos_params &p, const float *dLdu,
                        double *dV, double *dg, cudaStream_t st);
int launch_closest(const SceneImpl &S, const float *P, int n, bool bvh, const QueryOut &o, cudaStream_t st);
int launch_ball(const SceneImpl &S, const uint8_t *valid, const float *pt, const float *nrm, int n, float eps,
                bool bvh, float *R, cudaStream_t st);
int launch_adjoint(const SceneImpl &S, const float *P, long long total, const wos_params &p, const AdjCfg &a,
                   const float *dLdu, int mode, const AdjOut &out, unsigned long long *counter, cudaStream_t st);
// Processing order of adjoint samples that start from forward records: the
// sample indices [0, total) sorted by the position of their record's boundary
// primitive in the trees' primitive order (invalid records last).  Workspace
// bytes for `total` samples on a scene of nF primitives (0: no order for
// this size), and the launch writing the order into that workspace; *order
// receives the sorted indices (inside the workspace).
size_t record_order_bytes(int nF, long long total);
int launch_record_order(const SceneImpl &S, const int *wrec, long long total, void *ws, size_t ws_bytes,
                        const unsigned **order, cudaStream_t st);
// 1 (default): adjoint samples from records run in record order; 0: queue order.
int set_sample_order(int mode);
int sample_order_mode();
int launch_loss(const double *mean, int n, int kind, const float *target_or_dLdu, float *dLdu, double *loss,
                cudaStream_t st);
int launch_add_f64(const double *src, float *dst, long long n, cudaStream_t st);
// Image-space boundary term (boundary.cu): forward mode into img_tan
// (npixels doubles, added) for vertex motion tV, and / or reverse mode into
// dV_acc (nV x dim doubles, added) for pixel weights dLdI.
int launch_boundary(const SceneImpl &S, const wos_detector &d, int nwalks, uint64_t seed, const float *tV,
                    double *img_tan, const float *dLdI, double *dV_acc, cudaStream_t st);

}  // namespace wosd
