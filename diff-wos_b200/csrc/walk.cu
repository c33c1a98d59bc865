// Walk-on-spheres kernels for sm_100a.
//
// Forward: a persistent kernel in which every warp keeps 32 walks in flight.
// Each loop iteration runs exactly one nearest-primitive query per lane;
// when a lane's walk ends, the warp refills idle lanes from a grabbed chunk
// of the flattened (point, walk) index space (ballot + prefix rank), so
// warps stay full while walk lengths differ.  Results depend only on the
// Philox counters, never on which lane or block ran a walk.
//
// Adjoint: the same persistent loop over (point, walk) samples, each sample a
// small state machine -- primal walk, 10-step inscribed-ball bisection, two
// antithetic walks on the ball -- in which every state transition is again one
// nearest query, so lanes in different phases share the query code path.
//
// Reference functions restated: WoSDevice<N>::walk (include/wos.cuh:97-145),
// WoS<N>::solve / singleWalk launchers (:184-448), normal_derivative
// (wos/wos.py:59-107, wos/wos_with_source.py:154-232, wos/wos3d.py:97-135),
// tangent_derivative (wos/scene.py:451-460, wos/wos3d.py:137-156), OursCUDA /
// Ours3D (wos/wos_grad.py:130-151, wos/wos_grad_3d.py:117-137).
#include <algorithm>
#include <climits>
#include <type_traits>

#include <cub/cub.cuh>

#include "scene_impl.h"
#include "walk.h"

namespace wosd {

__device__ int g_status;
__device__ unsigned long long g_work[3];

int read_status(int reset, int *out) {
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_status, sizeof(int));
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyFromSymbol(g_status)");
    if (reset) {
        const int z = 0;
        e = cudaMemcpyToSymbol(g_status, &z, sizeof(int));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyToSymbol(g_status)");
    }
    *out = v;
    return 0;
}

int read_work(int reset, unsigned long long *out) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_work, sizeof(unsigned long long) * 3);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyFromSymbol(g_work)");
    if (reset) {
        const unsigned long long z[3] = {0, 0, 0};
        e = cudaMemcpyToSymbol(g_work, z, sizeof(z));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMemcpyToSymbol(g_work)");
    }
    return 0;
}

template <int D, bool BVH, class WK>
__device__ __forceinline__ Hit query(const SceneView &S, const float *p, const float4 *top, int n_top, WK &wk) {
    if (BVH) return nearest_bvh<D>(S, p, top, n_top, &g_status, wk);
    return nearest_brute<D>(S, p, wk);
}

// Add a warp's work counters to the global totals (counting launches only).
// Cooperative queries count once per warp (every lane holds the same totals).
template <bool COOP>
__device__ __forceinline__ void flush_work(const Work &wk) {
    unsigned long long v[3] = {wk.nq, wk.nb, wk.np};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!COOP) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
        if ((threadIdx.x & 31) == 0) atomicAdd(&g_work[k], v[k]);
    }
}

// Nearest query of every active lane.  With the LBVH the lanes take turns:
// the whole warp answers each lane's query cooperatively (wquery), starting
// from the warm candidate `warm` (that lane's previous nearest primitive, or
// -1).  A lane with ball_m > 0 asks instead for a primitive blocking the
// ball of radius ball_m centred at x (wball): it gets that primitive, or
// prim = -1 when none blocks.  Brute force runs per lane and always returns
// the nearest primitive.  Must be called by all 32 lanes.
template <int D, bool BVH, int WL = 0, class WK>
__device__ __forceinline__ Hit warp_queries(const SceneView &S, bool active, const float *x, int warm, WK &work,
                                            float ball_m = -1.0f) {
    Hit mine{-1, INFINITY};
    if (!BVH) {
        if (active) mine = nearest_brute<D>(S, x, work);
        return mine;
    }
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned act = __ballot_sync(FULL, active);
    // The per-point parts of each search -- the pruning tolerance (or the
    // ball's bound) and the warm candidate's distance -- are computed by every
    // lane for its own point at once, not by the whole warp once per query;
    // the values are the same bits either way.
    float lim = 0.0f, wd2 = INFINITY;
    if (active) {
        const float tol2 = prune_tol2<D>(S, x);
        if (ball_m > 0.0f) {
            lim = wball_bound(ball_m, tol2);
        } else {
            lim = tol2;
            if (warm >= 0) wd2 = prim_d2<D>(S, warm, x);
        }
    }
    while (act) {
        const int j = __ffs(act) - 1;
        act &= act - 1u;
        float q[3];
        q[0] = __shfl_sync(FULL, x[0], j);
        q[1] = __shfl_sync(FULL, x[1], j);
        q[2] = D == 3 ? __shfl_sync(FULL, x[2], j) : 0.0f;
        const int wp = __shfl_sync(FULL, warm, j);
        const float bm = __shfl_sync(FULL, ball_m, j);
        const float lj = __shfl_sync(FULL, lim, j);
        const float wj = __shfl_sync(FULL, wd2, j);
        Hit h{-1, INFINITY};
        if (bm > 0.0f) {
            wball_b<D, WL>(S, q, lj, bm, h, work);
        } else {
            if (wp >= 0) {
                h.prim = wp;
                h.d2 = wj;
            }
            h = wquery_tol<D, WL>(S, q, h, lj, work);
        }
        if (lane == j) mine = h;
    }
    return mine;
}

// ------------------------------------------------------------------ walker
enum { W_CONTINUE = 0, W_VALID = 1, W_INVALID = 2, W_TRUNC = 3 };

struct Walker {
    float p[3];
    float contrib;
    float ds[5];
    int i;
    int last;  // nearest primitive of the previous query (warm start), -1 if none
    bool fresh;
    __device__ __forceinline__ void start(const float *x, int D) {
        p[0] = x[0];
        p[1] = x[1];
        p[2] = D == 3 ? x[2] : 0.0f;
        contrib = 0.0f;
#pragma unroll
        for (int k = 0; k < 5; ++k) ds[k] = 0.0f;
        i = 0;
        last = -1;
        fresh = true;
    }
};

// Start point of the primal walk (pt, wk): the query point, moved inside its
// pixel when the settings carry a jitter (Detector.make_jittered_points,
// wos/scene.py:33-39): offset (u - 1/2) * jitter per axis, u from the walk's
// own Philox draw (role ROLE_JITTER, step 0).
template <int D>
__device__ __forceinline__ void walk_origin(const WalkCfg &c, const float *P, uint32_t pt, uint32_t wk, float *x) {
#pragma unroll
    for (int k = 0; k < 3; ++k) x[k] = k < D ? P[(size_t)pt * D + k] : 0.0f;
    if (c.jitter[0] != 0.0f || c.jitter[1] != 0.0f || c.jitter[2] != 0.0f) {
        const uint4 r = philox(c.rng, pt, wk, 0, ROLE_JITTER);
        x[0] = fmaf(wosm::u01(r.x) - 0.5f, c.jitter[0], x[0]);
        x[1] = fmaf(wosm::u01(r.y) - 0.5f, c.jitter[1], x[1]);
        if (D == 3) x[2] = fmaf(wosm::u01(r.z) - 0.5f, c.jitter[2], x[2]);
    }
}

// Process the query result at w.p: inside test on the first query, shell
// test, truncation, then the source term and one step (include/wos.cuh:97-145).
template <int D>
__device__ __forceinline__ int walker_advance(Walker &w, const SceneView &S, const Hit &hit, const WalkCfg &c,
                                              float eps, bool project, bool prevent_fd, uint32_t pt, uint32_t wk,
                                              uint32_t role, bool want_ds, const unsigned short *guide) {
    // no primitive at a finite distance (a NaN or overflowing point)
    if (hit.prim < 0) return W_INVALID;
    float d = sqrtf(hit.d2);
    if (w.fresh) {
        w.fresh = false;
        if (!c.double_sided && !inside_test<D>(S, w.p, hit, nullptr)) return W_INVALID;
        if (prevent_fd) d *= 0.5f;
    }
    if (w.i < c.nsteps) {
        if (d < eps) return W_VALID;
        if (!project && w.i == c.nsteps - 1) return W_TRUNC;
        const uint4 r = philox(c.rng, pt, wk, (uint32_t)w.i, role);
        if (D == 2 && S.src_type != 0) {
            float yx, yy;
            const float K = source_step(S, guide, c.use_IS != 0, w.p[0], w.p[1], d, r.z, r.w, yx, yy);
            float df[5];
            const float f = source(S, yx, yy, want_ds ? df : nullptr);
            w.contrib = fmaf(f, K, w.contrib);
            if (want_ds) {
#pragma unroll
                for (int k = 0; k < 5; ++k) w.ds[k] = fmaf(df[k], K, w.ds[k]);
            }
        }
        if (D == 2) {
            float s, cs;
            wosm::sincos_2pi(wosm::u01(r.x), &s, &cs);
            w.p[0] = fmaf(cs, d, w.p[0]);
            w.p[1] = fmaf(s, d, w.p[1]);
        } else {
            const float z = fmaf(-2.0f, wosm::u01(r.x), 1.0f);
            const float rr = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
            float s, cs;
            wosm::sincos_2pi(wosm::u01(r.y), &s, &cs);
            w.p[0] = fmaf(rr * cs, d, w.p[0]);
            w.p[1] = fmaf(rr * s, d, w.p[1]);
            w.p[2] = fmaf(z, d, w.p[2]);
        }
        w.i += 1;
        return W_CONTINUE;
    }
    return project ? W_VALID : W_TRUNC;
}

// Dynamic shared memory: [G-CDF guide table][`thread_bytes` of scratch per
// thread].  Sized to the byte: the carve-out the driver picks for the
// kernel's resident blocks comes in steps, and every byte of it is L1 lost to
// the tree.
__host__ __device__ inline size_t smem_bytes(int n_guide, int nthreads, int thread_bytes) {
    size_t b = ((size_t)(n_guide + 1) * sizeof(unsigned short) + 15) & ~(size_t)15;
    b += ((size_t)nthreads * thread_bytes + 15) & ~(size_t)15;
    return b;
}

struct Smem {
    const unsigned short *guide;
    double *scratch;  // this thread's words
};

__device__ __forceinline__ Smem stage_smem(const SceneView &S, bool stage_guide, int thread_words, float4 *smem) {
    Smem m;
    char *base = reinterpret_cast<char *>(smem);
    const int ng = stage_guide ? S.n_guide : -1;
    unsigned short *sg = reinterpret_cast<unsigned short *>(base);
    m.guide = S.guide;
    if (stage_guide) {
        for (int t = threadIdx.x; t <= S.n_guide; t += blockDim.x) sg[t] = S.guide[t];
        m.guide = sg;
    }
    base += ((size_t)(ng + 1) * sizeof(unsigned short) + 15) & ~(size_t)15;
    m.scratch = reinterpret_cast<double *>(base) + (size_t)threadIdx.x * thread_words;
    __syncthreads();
    return m;
}

// Warp-uniform refill of idle lanes from chunks of the global index space.
// Returns false once the warp has no work left.
struct Queue {
    long long cb, ce;
    bool drained;
};

__device__ __forceinline__ bool refill(Queue &q, bool &active, long long &idx, unsigned long long *counter,
                                       long long total, int chunk) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned idle = __ballot_sync(FULL, !active);
    while (idle != 0u && !q.drained) {
        if (q.cb >= q.ce) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)chunk);
            base = __shfl_sync(FULL, base, 0);
            if ((long long)base >= total) {
                q.drained = true;
                break;
            }
            q.cb = (long long)base;
            q.ce = min((long long)base + chunk, total);
        }
        const int nidle = __popc(idle);
        const long long avail = min((long long)nidle, q.ce - q.cb);
        const int rank = __popc(idle & ((1u << lane) - 1u));
        if (!active && rank < avail) {
            idx = q.cb + rank;
            active = true;
        }
        q.cb += avail;
        idle = __ballot_sync(FULL, !active);
    }
    return __ballot_sync(FULL, active) != 0u;
}

// ------------------------------------------------------------------ forward
// COUNT: the instance that keeps work counters (launched while work
// accounting is on); the others carry none.  The 3D instances are compiled
// for 3 resident blocks of 512 (a 40-register cap): 1 % faster than 2 blocks
// at 64 registers; the 2D ones stay at 64 registers.
template <int D, bool BVH, bool RECORDS, int WL, bool COUNT>
__global__ void __launch_bounds__(512, D == 3 ? 3 : 1) k_walk(SceneView S, WalkCfg c, const float *__restrict__ P, long long total,
                                             unsigned long long *counter, int chunk, int n_top, int stage_cdf,
                                             WalkOut out) {
    extern __shared__ float4 smem[];
    const Smem sm = stage_smem(S, stage_cdf != 0, 0, smem);
    Queue q{0, 0, false};
    bool active = false;
    long long idx = 0;
    uint32_t pt = 0, wk = 0;
    Walker w;
    w.last = -1;
    typename std::conditional<COUNT, Work, NoWork>::type work{};
    for (;;) {
        const bool was = active;
        if (!refill(q, active, idx, counter, total, chunk)) break;
        if (active && !was) {
            if (RECORDS) {
                pt = (uint32_t)idx;
                wk = c.walk_offset;
            } else {
                pt = (uint32_t)(idx / c.nwalks);
                wk = c.walk_offset + (uint32_t)(idx - (long long)pt * c.nwalks);
            }
            float x0[3];
            walk_origin<D>(c, P, pt, wk, x0);
            w.start(x0, D);
        }
        const Hit hit = warp_queries<D, BVH, WL>(S, active, w.p, w.last, work);
        if (!active) continue;
        w.last = hit.prim;
        const int r = walker_advance<D>(w, S, hit, c, c.eps, c.project != 0, c.prevent_fd != 0, pt, wk, ROLE_PRIMAL,
                                        out.wds != nullptr, sm.guide);
        if (r == W_CONTINUE) continue;
        active = false;
        if (RECORDS) {
            const bool ok = r == W_VALID;
            out.valid[pt] = ok ? 1 : 0;
            Rec rec;
            if (ok) rec = closest_record<D>(S, w.p, hit.prim);
#pragma unroll
            for (int k = 0; k < D; ++k) {
                if (out.pt) out.pt[(size_t)pt * D + k] = ok ? rec.p[k] : 0.0f;
                if (out.nrm) out.nrm[(size_t)pt * D + k] = ok ? rec.n[k] : 0.0f;
            }
            if (out.tuv) {
                out.tuv[2 * (size_t)pt] = ok ? rec.t0 : 0.0f;
                out.tuv[2 * (size_t)pt + 1] = (ok && D == 3) ? rec.t1 : 0.0f;
            }
            if (out.prim) out.prim[pt] = ok ? hit.prim : -1;
            if (out.contrib) out.contrib[pt] = ok ? w.contrib : 0.0f;
        } else {
            float v = 0.0f;
            Rec rec;
            if (r == W_VALID) {
                rec = closest_record<D>(S, w.p, hit.prim);
                v = dirichlet<D>(S, hit.prim, rec.t0, rec.t1, nullptr, nullptr);
                if (c.include_source) v += w.contrib;
                if (!isfinite(v)) atomicOr(&g_status, ST_NONFINITE);
            }
            out.values[idx] = v;
            if (out.wrec) {
                if (D == 2) {
                    const int2 wr = r == W_VALID ? make_int2(hit.prim | (rec.flip ? 0x40000000 : 0),
                                                             __float_as_int(rec.t0))
                                                 : make_int2(-1, 0);
                    reinterpret_cast<int2 *>(out.wrec)[idx] = wr;
                } else {
                    const int4 wr = r == W_VALID ? make_int4(hit.prim | (rec.flip ? 0x40000000 : 0),
                                                             __float_as_int(rec.t0), __float_as_int(rec.t1), 0)
                                                 : make_int4(-1, 0, 0, 0);
                    reinterpret_cast<int4 *>(out.wrec)[idx] = wr;
                }
            }
            if (out.wds) {
#pragma unroll
                for (int k = 0; k < 5; ++k) out.wds[(size_t)idx * 5 + k] = r == W_VALID ? w.ds[k] : 0.0f;
            }
            if (out.steps) out.steps[idx] = r == W_TRUNC ? c.nsteps : w.i;
        }
    }
    if constexpr (COUNT) {
        if (c.count) flush_work<BVH>(work);
    } else {
        // never taken (counting launches use the COUNT instance); with this
        // epilogue in place the kernel measured 2-5 % faster than without it
        if (c.count) flush_work<BVH>(Work{0, 0, 0});
    }
}

// Reference-shaped kernel: one thread per (point, walk), no regeneration.
template <int D, bool BVH>
__global__ void __launch_bounds__(256) k_walk_plain(SceneView S, WalkCfg c, const float *__restrict__ P,
                                                   long long total, float *values) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const uint32_t pt = (uint32_t)(idx / c.nwalks);
    const uint32_t wk = c.walk_offset + (uint32_t)(idx - (long long)pt * c.nwalks);
    Walker w;
    float x0[3];
    walk_origin<D>(c, P, pt, wk, x0);
    w.start(x0, D);
    Work work{0, 0, 0};
    float v = 0.0f;
    for (;;) {
        const Hit hit = query<D, BVH>(S, w.p, nullptr, 0, work);
        const int r = walker_advance<D>(w, S, hit, c, c.eps, c.project != 0, c.prevent_fd != 0, pt, wk, ROLE_PRIMAL,
                                        false, S.guide);
        if (r == W_CONTINUE) continue;
        if (r == W_VALID) {
            const Rec rec = closest_record<D>(S, w.p, hit.prim);
            v = dirichlet<D>(S, hit.prim, rec.t0, rec.t1, nullptr, nullptr);
            if (c.include_source) v += w.contrib;
        }
        break;
    }
    values[idx] = v;
}

// Per-point FP64 mean and sample variance, one warp per point, Neumaier
// compensated partial sums combined across lanes.
__device__ __forceinline__ void neumaier_add(double &s, double &c, double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
}

__device__ __forceinline__ double warp_sum_comp(double s, double c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_down_sync(0xffffffffu, s, o);
        const double c2 = __shfl_down_sync(0xffffffffu, c, o);
        c += c2;
        neumaier_add(s, c, s2);
    }
    return __shfl_sync(0xffffffffu, s + c, 0);
}

__global__ void k_reduce(const float *__restrict__ vals, int n, int nw, double *mean, double *var) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const float *v = vals + (size_t)warp * nw;
    double s = 0.0, cc = 0.0;
    for (int w = lane; w < nw; w += 32) neumaier_add(s, cc, (double)v[w]);
    const double m = warp_sum_comp(s, cc) / nw;
    if (var) {
        double q = 0.0, qc = 0.0;
        for (int w = lane; w < nw; w += 32) {
            const double e = (double)v[w] - m;
            neumaier_add(q, qc, e * e);
        }
        const double qq = warp_sum_comp(q, qc);
        if (lane == 0) var[warp] = nw > 1 ? qq / (nw - 1) : 0.0;
    }
    if (lane == 0) mean[warp] = m;
}

// ------------------------------------------------------------------ queries
template <int D, bool BVH>
__global__ void k_closest(SceneView S, const float *__restrict__ P, int n, QueryOut o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p[3] = {P[(size_t)i * D], P[(size_t)i * D + 1], D == 3 ? P[(size_t)i * D + 2] : 0.0f};
    Work work{0, 0, 0};
    const Hit hit = query<D, BVH>(S, p, nullptr, 0, work);
    if (o.prim) o.prim[i] = hit.prim;
    if (o.dist) o.dist[i] = sqrtf(hit.d2);
    if (hit.prim < 0) {
        atomicOr(&g_status, ST_BAD_PRIM);
        return;
    }
    const Rec r = closest_record<D>(S, p, hit.prim);
#pragma unroll
    for (int k = 0; k < D; ++k) {
        if (o.pt) o.pt[(size_t)i * D + k] = r.p[k];
        if (o.nrm) o.nrm[(size_t)i * D + k] = r.n[k];
    }
    if (o.tuv) {
        o.tuv[2 * (size_t)i] = r.t0;
        o.tuv[2 * (size_t)i + 1] = D == 3 ? r.t1 : 0.0f;
    }
    if (o.sdf || o.inside) {
        float sd;
        const bool in = inside_test<D>(S, p, hit, &sd);
        if (o.sdf) o.sdf[i] = sd;
        if (o.inside) o.inside[i] = in ? 1 : 0;
    }
}

// Largest inscribed ball (include/scene.cuh:225-249).
template <int D, bool BVH>
__device__ __forceinline__ float inscribed_ball(const SceneView &S, const float *p, const float *n, float eps,
                                                const float4 *top, int n_top) {
    float b = S.half_min_extent, a = eps;
    Work work{0, 0, 0};
    for (int i = 0; i < 10; ++i) {
        const float m = (a + b) * 0.5f;
        float q[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = fmaf(n[k], m, p[k]);
        const float d = sqrtf(query<D, BVH>(S, q, top, n_top, work).d2);
        if (wosm::ball_accepts(d, m))
            a = m;
        else
            b = m;
    }
    return a;
}

template <int D, bool BVH>
__global__ void k_ball(SceneView S, const uint8_t *valid, const float *pt, const float *nrm, int n, float eps,
                       float *R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!valid[i]) {
        R[i] = 0.0f;
        return;
    }
    float p[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
    for (int k = 0; k < D; ++k) {
        p[k] = pt[(size_t)i * D + k];
        nn[k] = nrm[(size_t)i * D + k];
    }
    R[i] = inscribed_ball<D, BVH>(S, p, nn, eps, nullptr, 0);
}

// ------------------------------------------------------------------ adjoint
template <int D>
__device__ __forceinline__ void tangent_derivative(const SceneView &S, int prim, float *out) {
    if (D == 2) {
        const float4 s = __ldg(&S.seg[prim]);
        const int ia = __ldg(&S.F[2 * prim]), ib = __ldg(&S.F[2 * prim + 1]);
        const float len = sqrtf(dot2(s.z, s.w, s.z, s.w));
        const float dv = (__ldg(&S.g[ib]) - __ldg(&S.g[ia])) / len;
        out[0] = dv * (s.z / len);
        out[1] = dv * (s.w / len);
    } else {
        const float4 t1 = __ldg(&S.tri[3 * prim + 1]), t2 = __ldg(&S.tri[3 * prim + 2]);
        const int ia = __ldg(&S.F[3 * prim]), ib = __ldg(&S.F[3 * prim + 1]), ic = __ldg(&S.F[3 * prim + 2]);
        const float ab[3] = {t1.x, t1.y, t1.z}, ac[3] = {t2.x, t2.y, t2.z};
        const float lab = sqrtf(dot3(ab[0], ab[1], ab[2], ab[0], ab[1], ab[2]));
        float t[3], fn[3], n[3];
        for (int k = 0; k < 3; ++k) t[k] = ab[k] / lab;
        cross3(ab[0], ab[1], ab[2], ac[0], ac[1], ac[2], fn[0], fn[1], fn[2]);
        const float lfn = sqrtf(dot3(fn[0], fn[1], fn[2], fn[0], fn[1], fn[2]));
        for (int k = 0; k < 3; ++k) fn[k] = fn[k] / lfn;
        cross3(fn[0], fn[1], fn[2], t[0], t[1], t[2], n[0], n[1], n[2]);
        const float ln = sqrtf(dot3(n[0], n[1], n[2], n[0], n[1], n[2]));
        for (int k = 0; k < 3; ++k) n[k] = n[k] / ln;
        const float va = __ldg(&S.g[ia]), vb = __ldg(&S.g[ib]), vc = __ldg(&S.g[ic]);
        const float gt = (vb - va) / lab;
        const float gn = ((vc - va) - gt * dot3(ac[0], ac[1], ac[2], t[0], t[1], t[2])) /
                         dot3(ac[0], ac[1], ac[2], n[0], n[1], n[2]);
        for (int k = 0; k < 3; ++k) out[k] = fmaf(gt, t[k], gn * n[k]);
    }
}

__device__ __forceinline__ float eval_P(const float *c, const float *y, const float *s, float R) {
    const float yy0 = y[0] - c[0], yy1 = y[1] - c[1];
    const float ss0 = s[0] - c[0], ss1 = s[1] - c[1];
    const float rr = dot2(yy0, yy1, yy0, yy1);
    const float cc = dot2(yy0, yy1, ss0, ss1) / sqrtf(dot2(ss0, ss1, ss0, ss1));
    const float RR = R * R;
    const float denom = fmaf(-2.0f * R, cc, RR) + rr;
    return (RR - rr) / fmaxf(denom, 1e-5f) / (wosm::kTwoPi * R);
}

// State of one normal-derivative sample on the inscribed ball of radius R
// centred at c = p + rn R (wos/wos.py:71-107, wos/wos3d.py:103-135).  The
// outward normal n = -rn, the centre and the second tangent are recomputed
// where needed (the same float operations as storing them), which keeps the
// per-thread state small.
template <int D>
struct NdExtra {};
template <>
struct NdExtra<3> {
    float cph, sph;  // cos / sin of the azimuth
    float pd[3];     // first tangent (in 2D it is recomputed from the normal)
};
template <int D>
struct NdState : NdExtra<D> {
    float p[D];   // boundary point
    float rn[D];  // record normal (towards the interior)
    float R;
    float uref;
    float cs, sn;  // 2D: cos/sin theta.  3D: cos theta, sqrt(1 - cos^2)
    float gsum;
    int which;
};

template <int D>
__device__ __forceinline__ void nd_centre(const NdState<D> &st, float *c) {
#pragma unroll
    for (int k = 0; k < D; ++k) c[k] = fmaf(st.rn[k], st.R, st.p[k]);
}

// First tangent of the ball frame at the boundary point: in 2D the record
// normal turned by a right angle, recomputed where it is used (a smaller
// per-sample slot leaves more of the SM's L1 to the tree); in 3D stored by
// nd_setup (recomputing it costs more than the L1 it frees).
template <int D>
__device__ __forceinline__ void nd_tangent(const NdState<D> &st, float *pd) {
    if constexpr (D == 2) {
        pd[0] = st.rn[1];
        pd[1] = -st.rn[0];
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) pd[k] = st.pd[k];
    }
}

template <int D>
__device__ __forceinline__ void nd_setup(NdState<D> &st, const SceneView &S, const WalkCfg &c, const AdjCfg &a,
                                         uint32_t pt, uint32_t wk) {
    const uint4 rx = philox(c.rng, pt, wk, 0, ROLE_EXTRA);
    if constexpr (D == 2) {
        const float cu = a.clamping * wosm::kInv2Pi;
        const float u = fminf(fmaxf(wosm::u01(rx.x), cu), 1.0f - cu);
        wosm::sincos_2pi(u, &st.sn, &st.cs);
    } else {
        st.cs = fminf(fmaxf(fmaf(-2.0f, wosm::u01(rx.x), 1.0f), -1.0f), 1.0f - a.clamping);
        wosm::sincos_2pi(wosm::u01(rx.y), &st.sph, &st.cph);
        const float n[3] = {-st.rn[0], -st.rn[1], -st.rn[2]};
        const bool zu = fabsf(n[2]) < 0.9f;
        const float up0 = zu ? 0.0f : 1.0f, up2 = zu ? 1.0f : 0.0f;
        cross3(n[0], n[1], n[2], up0, 0.0f, up2, st.pd[0], st.pd[1], st.pd[2]);
        const float l = sqrtf(dot3(st.pd[0], st.pd[1], st.pd[2], st.pd[0], st.pd[1], st.pd[2]));
        for (int k = 0; k < 3; ++k) st.pd[k] = st.pd[k] / l;
        st.sn = sqrtf(fmaxf(0.0f, fmaf(-st.cs, st.cs, 1.0f)));
    }
    st.gsum = 0.0f;
    st.which = 0;
}

// Query point of antithetic sample st.which.
template <int D>
__device__ __forceinline__ void nd_point(const NdState<D> &st, float *q) {
    float c[3], pd[3];
    nd_centre<D>(st, c);
    nd_tangent<D>(st, pd);
    if constexpr (D == 2) {
        const float si = st.which == 0 ? st.sn : -st.sn;
#pragma unroll
        for (int k = 0; k < 2; ++k) q[k] = fmaf(st.R, fmaf(-st.rn[k], st.cs, pd[k] * si), c[k]);
        q[2] = 0.0f;
    } else {
        const float n[3] = {-st.rn[0], -st.rn[1], -st.rn[2]};
        float pd2[3];
        cross3(n[0], n[1], n[2], pd[0], pd[1], pd[2], pd2[0], pd2[1], pd2[2]);
        const float cp = st.which == 0 ? st.cph : -st.cph, sp = st.which == 0 ? st.sph : -st.sph;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            q[k] = fmaf(st.R, fmaf(st.cs, n[k], st.sn * fmaf(cp, pd[k], sp * pd2[k])), c[k]);
    }
}

template <int D>
__device__ __forceinline__ void nd_accumulate(NdState<D> &st, const AdjCfg &a, float uq) {
    float P;
    if (D == 2) {
        P = 1.0f / (st.cs - 1.0f);
    } else {
        const float om = 1.0f - st.cs;
        P = -1.0f / (1.41421356f * (om * sqrtf(om)));
    }
    st.gsum += a.control_variates ? P * (uq - st.uref) / st.R : P * uq / st.R;
}

// grad * n_out, including the 2D interior source term.
template <int D>
__device__ __forceinline__ void nd_finish(const NdState<D> &st, const SceneView &S, const WalkCfg &c,
                                          const AdjCfg &a, uint32_t pt, uint32_t wk, bool with_src, float *out) {
    float grad = st.gsum * 0.5f;
    if constexpr (D == 2) {
        if (with_src) {
            float ctr[3];
            nd_centre<D>(st, ctr);
            const uint4 rx = philox(c.rng, pt, wk, 0, ROLE_EXTRA);
            float ds, dc;
            wosm::sincos_2pi(wosm::u01(rx.w), &ds, &dc);
            const float rr = sqrtf(wosm::u01(rx.z));
            const float y[2] = {fmaf(st.R, rr * dc, ctr[0]), fmaf(st.R, rr * ds, ctr[1])};
            const float f = source(S, y[0], y[1], nullptr);
            const float P = eval_P(ctr, y, st.p, st.R);
            const float area = wosm::kPi * st.R * st.R;
            float ci;
            if (a.control_variates) {
                const float fs = source(S, st.p[0], st.p[1], nullptr);
                ci = (f - fs) * P * area + fs * st.R * 0.5f;
            } else {
                ci = f * P * area;
            }
            grad = grad - ci;
        }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) out[k] = grad * -st.rn[k];
}

// Lane-local part of one inscribed-ball bisection step at radius m, centre q:
// the primitive that blocked the previous rejected radius decides a
// rejection without a query (need = false, pre = that primitive); otherwise,
// if the ball's own primitive rprim is within m + 1e-5f, the step is accepted
// unless some primitive blocks, and the warp only searches for one
// (ball_m = m; pre = rprim, the result when none blocks).  Else the step
// takes the full nearest query (the reference's test on the nearest distance).
template <int D>
__device__ __forceinline__ void ball_precheck(const SceneView &S, const float *q, float m, int bwarm, int rprim,
                                              bool &need, float &ball_m, Hit &pre) {
    if (bwarm >= 0) {
        const float d2 = prim_d2<D>(S, bwarm, q);
        if (ball_blocks(d2, m)) {
            pre = Hit{bwarm, d2};
            need = false;
            return;
        }
    }
    const float d2 = prim_d2<D>(S, rprim, q);
    if (sqrtf(d2) - m <= 1e-5f) {
        pre = Hit{rprim, d2};
        ball_m = m;
    }
}

enum { PH_IDLE = 0, PH_PRIMAL = 1, PH_BALL = 2, PH_ANTI_START = 3, PH_ANTI_WALK = 4, PH_ND_START = 5 };

// Per-thread adjoint state kept in shared memory: touched at phase changes,
// not in the query loop, so it does not occupy registers.  Only 4-byte
// fields, an odd number of them: thread t's slot starts t * ADJ_SLOT_WORDS
// words in, so a warp reading one field touches 32 distinct banks.
template <int D>
struct AdjSlot {
    NdState<D> st;
    float rt0, rt1;
    float ba, bb;  // bisection bracket
    int bk;
    int bwarm;     // primitive that blocked the last rejected radius, or -1
    float tacc;    // tangent mode: the sample's directional derivative so far
};
template <int D>
constexpr int adj_slot_words() {
    return (int)(sizeof(AdjSlot<D>) / 4) | 1;
}
static_assert(sizeof(AdjSlot<2>) % 4 == 0 && alignof(AdjSlot<2>) == 4 && sizeof(AdjSlot<3>) % 4 == 0 &&
                  alignof(AdjSlot<3>) == 4,
              "AdjSlot holds 4-byte fields only");

// Shared memory after the guide table: [5 source-gradient accumulators x
// blockDim doubles, field-major (when `acc`)][blockDim AdjSlot of
// adj_slot_words words].  Bytes per thread, for the launch's size.
template <int D>
__host__ __device__ constexpr int adj_thread_bytes(bool acc) {
    return adj_slot_words<D>() * 4 + (acc ? 40 : 0);
}

template <int D>
struct AdjSmem {
    double *acc;  // this thread's first accumulator; the k-th is acc[k * blockDim.x]
    AdjSlot<D> *slot;
};

template <int D>
__device__ __forceinline__ AdjSmem<D> adj_smem(double *base, bool acc) {
    AdjSmem<D> m;
    m.acc = acc ? base + threadIdx.x : nullptr;
    float *slots = reinterpret_cast<float *>(base + (acc ? 5 * blockDim.x : 0));
    m.slot = reinterpret_cast<AdjSlot<D> *>(slots + (size_t)threadIdx.x * adj_slot_words<D>());
    return m;
}

// The adjoint kernel runs at most 256 threads per block and is compiled for
// at least ADJ_MIN_BLOCKS resident blocks per SM: a 64-register cap.  The
// single-scene 3D kernel, whose leaf loads wait on L2, is compiled for
// ADJ_MIN_BLOCKS_3D (a 40-register cap): measured against 3, 4, 5, 7 and 8
// blocks it is the fastest despite its spills (4 -> 6: C3 step -3 %; 7 and 8
// spill far more and lose 10 %).  The 2D kernel is fastest at 4 and the
// batched kernels, which carry more per-lane state, at 4 in both dimensions.
#ifndef ADJ_MIN_BLOCKS
#define ADJ_MIN_BLOCKS 4
#endif
#ifndef ADJ_MIN_BLOCKS_3D
#define ADJ_MIN_BLOCKS_3D 6
#endif

// Persistent adjoint kernel.  ND_ONLY: the items are boundary records and the
// kernel writes one normal-derivative estimate per record (the
// wos_normal_derivative entry point); otherwise items are (point, walk)
// samples and gradients are accumulated into dV / dg / dsrc.
template <int D, bool BVH, int MODE, int WL, bool COUNT>
__global__ void __launch_bounds__(256, D == 3 ? ADJ_MIN_BLOCKS_3D : ADJ_MIN_BLOCKS) k_adjoint(SceneView S, WalkCfg c, AdjCfg a, const float *__restrict__ P,
                                                long long total, const float *__restrict__ dLdu,
                                                unsigned long long *counter, int chunk, int n_top, int stage_cdf,
                                                AdjOut out) {
    extern __shared__ float4 smem[];
    const Smem sm = stage_smem(S, stage_cdf != 0, 0, smem);
    const unsigned short *cdf = sm.guide;
    const bool src2 = D == 2 && S.src_type != 0;
    constexpr bool ND_ONLY = MODE == ADJ_ND_ONLY;
    const bool want_src = !ND_ONLY && a.want_dsrc && c.include_source && src2;
    const AdjSmem<D> am = adj_smem<D>(sm.scratch, want_src);
    AdjSlot<D> &slot = *am.slot;
    double *acc_src = am.acc;  // k-th accumulator at acc_src[k * blockDim.x]
    const int AS = blockDim.x;
    if (want_src) {
#pragma unroll
        for (int k = 0; k < 5; ++k) acc_src[k * AS] = 0.0;
    }
    NdState<D> &st = slot.st;
    float *rn = st.rn;
    float &rt0 = slot.rt0, &rt1 = slot.rt1;
    float &ba = slot.ba, &bb = slot.bb;
    int &bk = slot.bk;
    int &bwarm = slot.bwarm;
    constexpr bool TAN = MODE == ADJ_TANGENT;
    constexpr bool FROM_REC = MODE == ADJ_FROM_RECORDS || TAN;
    float &tacc = slot.tacc;
    const bool with_src = a.source_in_nd && src2;
    Queue q{0, 0, false};
    bool active = false;
    long long idx = 0;
    uint32_t pt = 0, wk = 0;
    int phase = PH_IDLE;
    double W = 0.0;
    Walker w;
    int rprim = 0;
    float qpos[3] = {0, 0, 0};
    typename std::conditional<COUNT, Work, NoWork>::type work{};
    w.last = -1;

    // Every lane reaches warp_queries once per iteration: no `continue`
    // between refill() and the query.
    for (;;) {
        const bool was = active;
        if (!refill(q, active, idx, counter, total, chunk)) break;
        if (active && !was) {
            if (ND_ONLY) {
                pt = (uint32_t)idx;
                wk = c.walk_offset;
                const int rp = out.rprim[pt];
                if (!out.rvalid[pt] || rp < 0 || rp >= S.nF) {
                    if (out.rvalid[pt]) atomicOr(&g_status, ST_BAD_PRIM);
#pragma unroll
                    for (int k = 0; k < D; ++k) out.nd[(size_t)pt * D + k] = 0.0f;
                    active = false;
                }
                rprim = active ? rp : 0;
                rt0 = out.rtuv[2 * (size_t)pt];
                rt1 = out.rtuv[2 * (size_t)pt + 1];
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    st.p[k] = out.rpt[(size_t)pt * D + k];
                    rn[k] = out.rnrm[(size_t)pt * D + k];
                }
                phase = PH_ND_START;
            } else {
                if (FROM_REC && out.order != nullptr) idx = (long long)__ldg(&out.order[idx]);
                pt = (uint32_t)(idx / c.nwalks);
                wk = c.walk_offset + (uint32_t)(idx - (long long)pt * c.nwalks);
                W = TAN ? 1.0 : (double)__ldg(&dLdu[pt]) / c.nwalks;
                float x0[3];
                walk_origin<D>(c, P, pt, wk, x0);
                w.start(x0, D);
                phase = PH_PRIMAL;
                tacc = 0.0f;
                if (W == 0.0) active = false;
                if (FROM_REC && active) {
                    // the primal walk ran in the forward pass: start from its record
                    int code;
                    if (D == 2) {
                        const int2 wr = __ldg(reinterpret_cast<const int2 *>(out.wrec) + idx);
                        code = wr.x;
                        rt0 = __int_as_float(wr.y);
                        rt1 = 0.0f;
                    } else {
                        const int4 wr = __ldg(reinterpret_cast<const int4 *>(out.wrec) + idx);
                        code = wr.x;
                        rt0 = __int_as_float(wr.y);
                        rt1 = __int_as_float(wr.z);
                    }
                    if (code < 0) {
                        active = false;
                    } else {
                        rprim = code & 0x3fffffff;
                        const Rec rec = record_from<D>(S, rprim, rt0, rt1, (code & 0x40000000) != 0);
                        int vid[3];
                        float wts[3];
                        st.uref = dirichlet<D>(S, rprim, rt0, rt1, vid, wts);
                        if (TAN) {
                            if (a.want_dg && out.tg != nullptr) {
#pragma unroll
                                for (int s2 = 0; s2 < D; ++s2) tacc = fmaf(wts[s2], __ldg(&out.tg[vid[s2]]), tacc);
                            }
                            if (want_src && out.ts != nullptr) {
#pragma unroll
                                for (int k = 0; k < 5; ++k)
                                    tacc = fmaf(__ldg(&out.wds[(size_t)idx * 5 + k]), __ldg(&out.ts[k]), tacc);
                            }
                        } else {
                            if (a.want_dg) {
#pragma unroll
                                for (int s2 = 0; s2 < D; ++s2) atomicAdd(&out.dg[vid[s2]], W * (double)wts[s2]);
                            }
                            if (want_src) {
#pragma unroll
                                for (int k = 0; k < 5; ++k)
                                    acc_src[k * AS] += W * (double)__ldg(&out.wds[(size_t)idx * 5 + k]);
                            }
                        }
                        if (!a.want_dV || (TAN && out.tV == nullptr)) {
                            if (TAN) out.tan[idx] = tacc;
                            active = false;
                        } else {
#pragma unroll
                            for (int k = 0; k < D; ++k) {
                                st.p[k] = rec.p[k];
                                rn[k] = rec.n[k];
                            }
                            ba = a.ball_eps;
                            bb = S.half_min_extent;
                            bk = 0;
                            bwarm = -1;
                            const float m = (ba + bb) * 0.5f;
#pragma unroll
                            for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m, st.p[k]);
                            phase = PH_BALL;
                        }
                    }
                }
            }
        }
        if (ND_ONLY && active && phase == PH_ND_START && out.rR != nullptr) {
            // a given ball radius (override_R, wos/wos.py:71-74): no bisection
            st.uref = dirichlet<D>(S, rprim, rt0, rt1, nullptr, nullptr);
            st.R = out.rR[pt];
            nd_setup<D>(st, S, c, a, pt, wk);
            nd_point<D>(st, qpos);
            phase = PH_ANTI_START;
        }
        if (ND_ONLY && active && phase == PH_ND_START) {
            // no query needed to start: set up the bisection
            st.uref = dirichlet<D>(S, rprim, rt0, rt1, nullptr, nullptr);
            ba = a.ball_eps;
            bb = S.half_min_extent;
            bk = 0;
            bwarm = -1;
            const float m = (ba + bb) * 0.5f;
#pragma unroll
            for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m, st.p[k]);
            phase = PH_BALL;
        }
        // PH_PRIMAL and PH_ND_START occur only in their own modes: testing the
        // mode too compiles the other phases' code out of each instance, which
        // lowers register pressure (records mode: C2 adjoint 8 % faster)
        constexpr bool HAS_PRIMAL = MODE == ADJ_RECOMPUTE;
        const bool walking = (HAS_PRIMAL && phase == PH_PRIMAL) || phase == PH_ANTI_WALK;
        float x[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) x[k] = walking ? w.p[k] : qpos[k];
        bool need = active;
        float ball_m = -1.0f;
        Hit pre{-1, INFINITY};
        if (active && phase == PH_BALL) ball_precheck<D>(S, qpos, (ba + bb) * 0.5f, bwarm, rprim, need, ball_m, pre);
        Hit hit = warp_queries<D, BVH, WL>(S, need, x, walking ? w.last : rprim, work, ball_m);
        if (!active) continue;
        if (phase == PH_BALL && (!need || (ball_m > 0.0f && hit.prim < 0))) hit = pre;
        if (walking) w.last = hit.prim;
        bool finish_anti = false;
        float uq = 0.0f;
        if (HAS_PRIMAL && phase == PH_PRIMAL) {
            const int r = walker_advance<D>(w, S, hit, c, c.eps, c.project != 0, c.prevent_fd != 0, pt, wk,
                                            ROLE_PRIMAL, want_src, cdf);
            if (r == W_CONTINUE) continue;
            if (r != W_VALID) {
                active = false;
                continue;
            }
            const Rec rec = closest_record<D>(S, w.p, hit.prim);
            rprim = hit.prim;
            rt0 = rec.t0;
            rt1 = rec.t1;
            int vid[3];
            float wts[3];
            st.uref = dirichlet<D>(S, rprim, rt0, rt1, vid, wts);
            if (a.want_dg) {
#pragma unroll
                for (int s = 0; s < D; ++s) atomicAdd(&out.dg[vid[s]], W * (double)wts[s]);
            }
            if (want_src) {
#pragma unroll
                for (int k = 0; k < 5; ++k) acc_src[k * AS] += W * (double)w.ds[k];
            }
            if (!a.want_dV) {
                active = false;
                continue;
            }
#pragma unroll
            for (int k = 0; k < D; ++k) {
                st.p[k] = rec.p[k];
                rn[k] = rec.n[k];
            }
            ba = a.ball_eps;
            bb = S.half_min_extent;
            bk = 0;
            bwarm = -1;
            const float m = (ba + bb) * 0.5f;
#pragma unroll
            for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m, st.p[k]);
            phase = PH_BALL;
            continue;
        }
        if (phase == PH_BALL) {
            const float d = sqrtf(hit.d2);
            const float m = (ba + bb) * 0.5f;
            if (wosm::ball_accepts(d, m)) {
                ba = m;
            } else {
                bb = m;
                bwarm = hit.prim;
            }
            ++bk;
            if (bk < 10) {
                const float m2 = (ba + bb) * 0.5f;
#pragma unroll
                for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m2, st.p[k]);
                continue;
            }
            st.R = ba;
            nd_setup<D>(st, S, c, a, pt, wk);
            nd_point<D>(st, qpos);
            phase = PH_ANTI_START;
            continue;
        }
        const uint32_t role = st.which == 0 ? ROLE_ANTI_A : ROLE_ANTI_B;
        // the ball walk's first query (PH_ANTI_START) either ends it inside the
        // epsilon2 shell or starts the walk; both walk phases then share one
        // walker_advance (one inlined copy keeps the kernel's code small)
        bool advance = phase == PH_ANTI_WALK;
        if (phase == PH_ANTI_START) {
            const float d = sqrtf(hit.d2);
            if (d < a.epsilon2) {
                const Rec r2 = closest_record<D>(S, qpos, hit.prim);
                uq = dirichlet<D>(S, hit.prim, r2.t0, r2.t1, nullptr, nullptr);
                finish_anti = true;
            } else {
                w.start(qpos, D);
                w.last = hit.prim;
                phase = PH_ANTI_WALK;
                advance = true;
            }
        }
        if (advance) {
            const int r = walker_advance<D>(w, S, hit, c, a.epsilon2, c.project != 0, false, pt, wk, role, false, cdf);
            if (r == W_CONTINUE) continue;
            if (r == W_VALID) {
                const Rec r2 = closest_record<D>(S, w.p, hit.prim);
                uq = dirichlet<D>(S, hit.prim, r2.t0, r2.t1, nullptr, nullptr);
                if (with_src) uq += w.contrib;
            }
            finish_anti = true;
        }
        if (finish_anti) {
            nd_accumulate<D>(st, a, uq);
            st.which += 1;
            if (st.which == 1) {
                nd_point<D>(st, qpos);
                phase = PH_ANTI_START;
                continue;
            }
            float gn[3];
            nd_finish<D>(st, S, c, a, pt, wk, with_src, gn);
            if (ND_ONLY) {
#pragma unroll
                for (int k = 0; k < D; ++k) out.nd[(size_t)pt * D + k] = gn[k];
            } else {
                float gt[3];
                tangent_derivative<D>(S, rprim, gt);
                int vid[3];
                float wts[3];
                dirichlet<D>(S, rprim, rt0, rt1, vid, wts);
                if (TAN) {
                    // d(sample) = -(grad_n + grad_t) . dx, dx = sum_s wts_s dV[vid_s]
#pragma unroll
                    for (int s = 0; s < D; ++s)
#pragma unroll
                        for (int k = 0; k < D; ++k)
                            tacc = fmaf(-(wts[s] * (gn[k] + gt[k])), __ldg(&out.tV[(size_t)vid[s] * D + k]), tacc);
                    out.tan[idx] = tacc;
                } else {
#pragma unroll
                    for (int s = 0; s < D; ++s)
#pragma unroll
                        for (int k = 0; k < D; ++k)
                            atomicAdd(&out.dV[(size_t)vid[s] * D + k], W * (double)(-(wts[s] * (gn[k] + gt[k]))));
                }
            }
            active = false;
            phase = PH_IDLE;
        }
    }
    if constexpr (COUNT) {
        if (c.count) flush_work<BVH>(work);
    } else {
        // never taken (counting launches use the COUNT instance); with this
        // epilogue in place the kernel measured 2-5 % faster than without it
        if (c.count) flush_work<BVH>(Work{0, 0, 0});
    }
    if (want_src && !TAN) {
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            double v = acc_src[k * AS];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&out.dsrc[k], v);
        }
    }
}

// dL/du per point for a pointwise loss of the per-point means, and the loss
// (one block, fixed reduction order).  kind 1: mean(u^2); kind 2:
// mean((u - target)^2); kind 0: dL/du given.
__global__ void k_loss(const double *mean, int n, int kind, const float *tg, float *dLdu, double *loss) {
    __shared__ double red[1024];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double u = mean[i];
        double e = u;
        if (kind == 2) e = u - (double)tg[i];
        if (kind == 0) {
            dLdu[i] = tg[i];
        } else {
            dLdu[i] = (float)(2.0 * e / n);
            acc += e * e / n;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) *loss = red[0];
}

int launch_loss(const double *mean, int n, int kind, const float *target_or_dLdu, float *dLdu, double *loss,
                cudaStream_t st) {
    k_loss<<<1, 1024, 0, st>>>(mean, n, kind, target_or_dLdu, dLdu, loss);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_loss launch");
    return 0;
}

__global__ void k_add_f64_to_f32(const double *src, float *dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] += (float)src[i];
}

// ------------------------------------------------------------------ host
static wos_launch_config g_cfg[2] = {{256, 0, 64, 1024}, {256, 0, 16, 768}};

int set_launch_config(int dim, const wos_launch_config *cfg) {
    if (dim != 2 && dim != 3) return fail(WOS_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
    wos_launch_config &c = g_cfg[dim - 2];
    if (cfg->block_threads) {
        if (cfg->block_threads % 32 || cfg->block_threads < 32 || cfg->block_threads > 512)
            return fail(WOS_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32 in [32, 512]");
        c.block_threads = cfg->block_threads;
    }
    if (cfg->blocks_per_sm >= 0) c.blocks_per_sm = cfg->blocks_per_sm;
    if (cfg->chunk) {
        if (cfg->chunk < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "chunk must be >= 1");
        c.chunk = cfg->chunk;
    }
    if (cfg->smem_nodes >= 0) c.smem_nodes = cfg->smem_nodes;
    return 0;
}

int get_launch_config(int dim, wos_launch_config *out) {
    if (dim != 2 && dim != 3) return fail(WOS_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
    *out = g_cfg[dim - 2];
    return 0;
}

static int g_count_work = 0;

int set_work_counting(int enable) {
    g_count_work = enable ? 1 : 0;
    return 0;
}

int work_counting_enabled() { return g_count_work; }

AdjCfg make_adj_cfg(const wos_adjoint_params &a) {
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

WalkCfg make_cfg(const wos_params &p) {
    WalkCfg c;
    c.count = g_count_work;
    c.nwalks = p.nwalks;
    c.nsteps = p.nsteps;
    c.eps = p.epsilon;
    c.double_sided = p.double_sided;
    c.prevent_fd = p.prevent_fd_artifacts;
    c.use_IS = p.use_IS_for_greens;
    c.include_source = p.include_source;
    c.project = p.project_unterminated;
    c.walk_offset = p.walk_offset;
    c.rng = make_rng(p.seed);
    for (int k = 0; k < 3; ++k) c.jitter[k] = p.jitter[k];
    return c;
}

struct Shape {
    int grid, block, n_top, stage_cdf;
    size_t smem;
};

template <typename Kern>
static int shape_for(Kern kern, const SceneImpl &S, int D, bool bvh, bool want_cdf, Shape &sh,
                     int thread_bytes = 0, int max_block = 512) {
    const wos_launch_config &cfg = g_cfg[D - 2];
    sh.block = std::min(cfg.block_threads, max_block);
    // the persistent kernels query the wide tree cooperatively; no binary-LBVH
    // nodes are staged
    sh.n_top = 0;
    sh.stage_cdf = want_cdf ? 1 : 0;
    sh.smem = smem_bytes(want_cdf ? S.n_guide : -1, sh.block, thread_bytes);
    (void)bvh;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem);
    if (e != cudaSuccess) return fail_cuda(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, sh.block, sh.smem);
    if (e != cudaSuccess) return fail_cuda(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) return fail(WOS_ERR_UNSUPPORTED, "walk kernel does not fit on an SM with this launch config");
    const int per_sm = cfg.blocks_per_sm > 0 ? std::min(cfg.blocks_per_sm, occ) : occ;
    sh.grid = sms * per_sm;
    return 0;
}


template <int D, bool BVH, int WL, bool COUNT>
static int launch_walk_t(const SceneImpl &S, const float *P, long long total, const wos_params &p, bool records,
                         const WalkOut &out, unsigned long long *counter, cudaStream_t st) {
    const SceneView v = S.view();
    const WalkCfg c = make_cfg(p);
    const bool want_cdf = D == 2 && S.src_type != 0 && p.use_IS_for_greens;
    Shape sh;
    int rc;
    if (records)
        rc = shape_for(k_walk<D, BVH, true, WL, COUNT>, S, D, BVH, want_cdf, sh);
    else
        rc = shape_for(k_walk<D, BVH, false, WL, COUNT>, S, D, BVH, want_cdf, sh);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counter)");
    const int chunk = g_cfg[D - 2].chunk;
    if (records)
        k_walk<D, BVH, true, WL, COUNT><<<sh.grid, sh.block, sh.smem, st>>>(v, c, P, total, counter, chunk,
                                                                             sh.n_top, sh.stage_cdf, out);
    else
        k_walk<D, BVH, false, WL, COUNT><<<sh.grid, sh.block, sh.smem, st>>>(v, c, P, total, counter, chunk,
                                                                              sh.n_top, sh.stage_cdf, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_walk launch");
    return 0;
}

int launch_walk(const SceneImpl &S, const float *P, long long total, const wos_params &p, bool records,
                const WalkOut &out, unsigned long long *counter, cudaStream_t st) {
    if (total == 0) return 0;
    const bool bvh = p.use_bvh != 0;
    const int wl = specialised_depth(S.wt_levels);
    // work accounting runs the any-depth instance that keeps counters
    const bool count = work_counting_enabled() != 0;
#define WOS_WALK(D_)                                                                                      \
    if (count) {                                                                                          \
        if (!bvh) return launch_walk_t<D_, false, 0, true>(S, P, total, p, records, out, counter, st);    \
        return launch_walk_t<D_, true, 0, true>(S, P, total, p, records, out, counter, st);               \
    }                                                                                                     \
    if (!bvh) return launch_walk_t<D_, false, 0, false>(S, P, total, p, records, out, counter, st);       \
    switch (wl) {                                                                                         \
        case 1: return launch_walk_t<D_, true, 1, false>(S, P, total, p, records, out, counter, st);      \
        case 2: return launch_walk_t<D_, true, 2, false>(S, P, total, p, records, out, counter, st);      \
        case 3: return launch_walk_t<D_, true, 3, false>(S, P, total, p, records, out, counter, st);      \
        default: return launch_walk_t<D_, true, 0, false>(S, P, total, p, records, out, counter, st);     \
    }
    if (S.dim == 2) {
        WOS_WALK(2)
    }
    WOS_WALK(3)
#undef WOS_WALK
}

// ------------------------------------------------------------------ soft-edge walk
// The soft-edge walk of the reference's Baseline / Baseline3D
// (wos/wos.py:158-187, wos/wos_grad_3d.py:24-57): nsteps steps, each adding
// beta (1 - w) g(closest point) with w = min(d, eps) / eps and then
// beta *= w; it never stops early.  Forward mode carries the tangents of the
// position, the distance, beta and the result along a vertex / value motion.

// Barycentric region of the closest point on a triangle, by the cascade of
// tri_closest: 0 vertex a, 1 b, 2 c, 3 edge ab, 4 ac, 5 bc, 6 face, 7 degenerate.
__device__ __forceinline__ int tri_region(float4 t0, float4 t1, float4 t2, const float *x) {
    const float axx = x[0] - t0.x, axy = x[1] - t0.y, axz = x[2] - t0.z;
    const float ab2 = t0.w, abac = t1.w, ac2 = t2.w;
    const float d1 = dot3(t1.x, t1.y, t1.z, axx, axy, axz);
    const float d2 = dot3(t2.x, t2.y, t2.z, axx, axy, axz);
    if (d1 <= 0.0f && d2 <= 0.0f) return 0;
    const float d3 = d1 - ab2, d4 = d2 - abac;
    if (d3 >= 0.0f && d4 <= d3) return 1;
    const float d5 = d1 - abac, d6 = d2 - ac2;
    if (d6 >= 0.0f && d5 <= d6) return 2;
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return 3;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return 4;
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f) return 5;
    return va + vb + vc > 0.0f ? 6 : 7;
}

// Derivative of the projection parameter t = (x - a).e / (e.e) of x onto
// the line a + t e, for motions xd, ad, ed.
__device__ __forceinline__ float proj_dot(const float *x, const float *a, const float *e, const float *xd,
                                          const float *ad, const float *ed, int D, float t) {
    float ee = 0.0f, num = 0.0f, eed = 0.0f;
    for (int k = 0; k < D; ++k) {
        ee += e[k] * e[k];
        num += (xd[k] - ad[k]) * e[k] + (x[k] - a[k]) * ed[k];
        eed += e[k] * ed[k];
    }
    return ee > 0.0f ? (num - 2.0f * t * eed) / ee : 0.0f;
}

// Tangents at a soft-walk step: of the nearest distance d (> 0) to primitive
// prim at x, dd = n.(xd - cd) with n = (x - c)/d and cd the motion of the
// closest point at fixed barycentrics (n is normal to the feature, so the
// barycentrics' own motion drops out); and of the boundary value there, gd
// (barycentric motion through the projection plus value motion).  tV / tg:
// vertex and value directions, either may be null.
template <int D>
__device__ void soft_tangents(const SceneView &S, const float *x, const float *xd, float d, const Rec &r, int prim,
                              const float *tV, const float *tg, float &dd, float &gd) {
    int vid[3];
    float wts[3];
    dirichlet<D>(S, prim, r.t0, r.t1, vid, wts);
    float V[3][3], Vd[3][3];
    for (int j = 0; j < D; ++j)
        for (int k = 0; k < 3; ++k) {
            V[j][k] = k < D ? __ldg(&S.V[(size_t)vid[j] * D + k]) : 0.0f;
            Vd[j][k] = (tV != nullptr && k < D) ? __ldg(&tV[(size_t)vid[j] * D + k]) : 0.0f;
        }
    float cd[3] = {0.0f, 0.0f, 0.0f};
    for (int j = 0; j < D; ++j)
        for (int k = 0; k < D; ++k) cd[k] = fmaf(wts[j], Vd[j][k], cd[k]);
    dd = 0.0f;
    if (d > 0.0f)
        for (int k = 0; k < D; ++k) dd += (x[k] - r.p[k]) / d * (xd[k] - cd[k]);
    // barycentric motion
    float bd[3] = {0.0f, 0.0f, 0.0f};  // d(wts)/dt
    if (D == 2) {
        if (r.t0 > 0.0f && r.t0 < 1.0f) {
            const float e[2] = {V[1][0] - V[0][0], V[1][1] - V[0][1]};
            const float ed[2] = {Vd[1][0] - Vd[0][0], Vd[1][1] - Vd[0][1]};
            const float td = proj_dot(x, V[0], e, xd, Vd[0], ed, 2, r.t0);
            bd[0] = -td;
            bd[1] = td;
        }
    } else {
        const float4 t0 = __ldg(&S.tri[3 * prim]), t1 = __ldg(&S.tri[3 * prim + 1]), t2 = __ldg(&S.tri[3 * prim + 2]);
        const int reg = tri_region(t0, t1, t2, x);
        float ab[3], ac[3], abd[3], acd[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = V[1][k] - V[0][k];
            ac[k] = V[2][k] - V[0][k];
            abd[k] = Vd[1][k] - Vd[0][k];
            acd[k] = Vd[2][k] - Vd[0][k];
        }
        if (reg == 3) {
            const float vd = proj_dot(x, V[0], ab, xd, Vd[0], abd, 3, r.t0);
            bd[1] = vd;
            bd[0] = -vd;
        } else if (reg == 4) {
            const float wd = proj_dot(x, V[0], ac, xd, Vd[0], acd, 3, r.t1);
            bd[2] = wd;
            bd[0] = -wd;
        } else if (reg == 5) {
            float bc[3], bcd[3];
            for (int k = 0; k < 3; ++k) {
                bc[k] = V[2][k] - V[1][k];
                bcd[k] = Vd[2][k] - Vd[1][k];
            }
            const float wd = proj_dot(x, V[1], bc, xd, Vd[1], bcd, 3, r.t1);
            bd[2] = wd;
            bd[1] = -wd;
        } else if (reg == 6) {
            // G [v w]^T = rhs: G = [[ab.ab, ab.ac], [ab.ac, ac.ac]], rhs = [ab.(x-a), ac.(x-a)]
            float G00 = 0, G01 = 0, G11 = 0, Gd00 = 0, Gd01 = 0, Gd11 = 0, rd0 = 0, rd1 = 0;
            for (int k = 0; k < 3; ++k) {
                const float xa = x[k] - V[0][k], xad = xd[k] - Vd[0][k];
                G00 += ab[k] * ab[k];
                G01 += ab[k] * ac[k];
                G11 += ac[k] * ac[k];
                Gd00 += 2.0f * ab[k] * abd[k];
                Gd01 += abd[k] * ac[k] + ab[k] * acd[k];
                Gd11 += 2.0f * ac[k] * acd[k];
                rd0 += abd[k] * xa + ab[k] * xad;
                rd1 += acd[k] * xa + ac[k] * xad;
            }
            const float q0 = rd0 - (Gd00 * r.t0 + Gd01 * r.t1), q1 = rd1 - (Gd01 * r.t0 + Gd11 * r.t1);
            const float det = G00 * G11 - G01 * G01;
            if (det != 0.0f) {
                const float vd = (G11 * q0 - G01 * q1) / det, wd = (G00 * q1 - G01 * q0) / det;
                bd[1] = vd;
                bd[2] = wd;
                bd[0] = -vd - wd;
            }
        }
    }
    gd = 0.0f;
    for (int j = 0; j < D; ++j) {
        const float gj = __ldg(&S.g[vid[j]]);
        gd = fmaf(bd[j], gj, gd);
        if (tg != nullptr) gd = fmaf(wts[j], __ldg(&tg[vid[j]]), gd);
    }
}

template <int D, bool BVH, int WL>
__global__ void __launch_bounds__(256) k_walk_soft(SceneView S, WalkCfg c, const float *__restrict__ P,
                                                   long long total, unsigned long long *counter, int chunk,
                                                   const float *__restrict__ tV, const float *__restrict__ tg,
                                                   float *vals, float *tans) {
    Queue q{0, 0, false};
    bool active = false;
    long long idx = 0;
    uint32_t pt = 0, wk = 0;
    float p[3] = {0, 0, 0}, pd[3] = {0, 0, 0};
    float beta = 0.0f, betad = 0.0f, res = 0.0f, resd = 0.0f;
    int i = 0, last = -1;
    bool fresh = false;
    const float eps = c.eps;
    const bool want_tan = tans != nullptr;
    Work work{0, 0, 0};
    for (;;) {
        const bool was = active;
        if (!refill(q, active, idx, counter, total, chunk)) break;
        if (active && !was) {
            pt = (uint32_t)(idx / c.nwalks);
            wk = c.walk_offset + (uint32_t)(idx - (long long)pt * c.nwalks);
            walk_origin<D>(c, P, pt, wk, p);
            pd[0] = pd[1] = pd[2] = 0.0f;
            beta = 1.0f;
            betad = res = resd = 0.0f;
            i = 0;
            last = -1;
            fresh = true;
        }
        const Hit hit = warp_queries<D, BVH, WL>(S, active, p, last, work);
        if (!active) continue;
        last = hit.prim;
        bool done = hit.prim < 0;
        if (!done && fresh) {
            fresh = false;
            if (!c.double_sided && !inside_test<D>(S, p, hit, nullptr)) done = true;
        }
        if (done) {
            vals[idx] = 0.0f;
            if (want_tan) tans[idx] = 0.0f;
            active = false;
            continue;
        }
        const float d = sqrtf(hit.d2);
        const Rec r = closest_record<D>(S, p, hit.prim);
        const float g = dirichlet<D>(S, hit.prim, r.t0, r.t1, nullptr, nullptr);
        float dd = 0.0f, gd = 0.0f;
        if (want_tan) soft_tangents<D>(S, p, pd, d, r, hit.prim, tV, tg, dd, gd);
        const float w = fminf(d, eps) / eps;
        const float wd = d < eps ? dd / eps : 0.0f;
        if (d > 0.0f) {
            res = fmaf(beta * (1.0f - w), g, res);
            if (want_tan) resd += betad * (1.0f - w) * g - beta * wd * g + beta * (1.0f - w) * gd;
        }
        betad = betad * w + beta * wd;
        beta = beta * w;
        if (i >= c.nsteps - 1) {
            vals[idx] = res;
            if (want_tan) tans[idx] = resd;
            active = false;
            continue;
        }
        const uint4 rr = philox(c.rng, pt, wk, (uint32_t)i, ROLE_PRIMAL);
        float dir[3];
        if (D == 2) {
            float s, cs;
            wosm::sincos_2pi(wosm::u01(rr.x), &s, &cs);
            dir[0] = cs;
            dir[1] = s;
            dir[2] = 0.0f;
        } else {
            const float z = fmaf(-2.0f, wosm::u01(rr.x), 1.0f);
            const float rad = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
            float s, cs;
            wosm::sincos_2pi(wosm::u01(rr.y), &s, &cs);
            dir[0] = rad * cs;
            dir[1] = rad * s;
            dir[2] = z;
        }
        for (int k = 0; k < D; ++k) {
            p[k] = fmaf(dir[k], d, p[k]);
            pd[k] = fmaf(dir[k], dd, pd[k]);
        }
        ++i;
    }
    if (c.count) flush_work<BVH>(work);
}

// ------------------------------------------------------------------ soft-edge walk, reverse mode
// Transposed step of the soft walk's tangent recurrence (k_walk_soft): given
// the adjoint gbar of the step's boundary-value tangent gd, add the adjoints
// of the position tangent (pbar) and of the vertex motion (dV, FP64 atomics)
// that enter gd through the motion of the closest point's barycentrics
// (soft_tangents: proj_dot along an edge, the 2 x 2 normal equations on a
// face).
template <int D>
__device__ void soft_bary_adjoint(const SceneView &S, const float *x, const Rec &r, int prim, const int *vid,
                                  float gbar, float *pbar, double *dV) {
    float V[3][3], gv[3];
    for (int j = 0; j < D; ++j) {
        gv[j] = __ldg(&S.g[vid[j]]);
        for (int k = 0; k < 3; ++k) V[j][k] = k < D ? __ldg(&S.V[(size_t)vid[j] * D + k]) : 0.0f;
    }
    // an edge (i0 -> i1) at parameter t: bd[i1] = td, bd[i0] = -td
    auto edge = [&](int i0, int i1, float t) {
        const float tbar = gbar * (gv[i1] - gv[i0]);
        float e[3], xa[3], ee = 0.0f;
        for (int k = 0; k < D; ++k) {
            e[k] = V[i1][k] - V[i0][k];
            xa[k] = x[k] - V[i0][k];
            ee += e[k] * e[k];
        }
        if (!(ee > 0.0f) || tbar == 0.0f) return;
        for (int k = 0; k < D; ++k) {
            const float ce = tbar * e[k] / ee;                        // d td / d xd, -d td / d ad
            const float ced = tbar * (xa[k] - 2.0f * t * e[k]) / ee;  // d td / d ed
            pbar[k] += ce;
            atomicAdd(&dV[(size_t)vid[i0] * D + k], (double)(-ce - ced));
            atomicAdd(&dV[(size_t)vid[i1] * D + k], (double)ced);
        }
    };
    if (D == 2) {
        if (r.t0 > 0.0f && r.t0 < 1.0f) edge(0, 1, r.t0);
        return;
    }
    const float4 t0 = __ldg(&S.tri[3 * prim]), t1 = __ldg(&S.tri[3 * prim + 1]), t2 = __ldg(&S.tri[3 * prim + 2]);
    const int reg = tri_region(t0, t1, t2, x);
    if (reg == 3) {
        edge(0, 1, r.t0);
    } else if (reg == 4) {
        edge(0, 2, r.t1);
    } else if (reg == 5) {
        edge(1, 2, r.t1);
    } else if (reg == 6) {
        float ab[3], ac[3], xa[3], G00 = 0, G01 = 0, G11 = 0;
        for (int k = 0; k < 3; ++k) {
            ab[k] = V[1][k] - V[0][k];
            ac[k] = V[2][k] - V[0][k];
            xa[k] = x[k] - V[0][k];
            G00 += ab[k] * ab[k];
            G01 += ab[k] * ac[k];
            G11 += ac[k] * ac[k];
        }
        const float det = G00 * G11 - G01 * G01;
        if (det == 0.0f) return;
        // gd = vd (g1 - g0) + wd (g2 - g0), [vd wd] = G^-1 [q0 q1]
        const float vbar = gbar * (gv[1] - gv[0]), wbar = gbar * (gv[2] - gv[0]);
        const float q0 = (G11 * vbar - G01 * wbar) / det, q1 = (G00 * wbar - G01 * vbar) / det;
        const float v = r.t0, w = r.t1;
        for (int k = 0; k < 3; ++k) {
            const float cx = q0 * ab[k] + q1 * ac[k];  // via xd - ad
            const float cab = q0 * (xa[k] - 2.0f * v * ab[k] - w * ac[k]) - q1 * v * ac[k];
            const float cac = -q0 * w * ab[k] + q1 * (xa[k] - v * ab[k] - 2.0f * w * ac[k]);
            pbar[k] += cx;
            atomicAdd(&dV[(size_t)vid[0] * 3 + k], (double)(-cx - cab - cac));
            atomicAdd(&dV[(size_t)vid[1] * 3 + k], (double)cab);
            atomicAdd(&dV[(size_t)vid[2] * 3 + k], (double)cac);
        }
    }
}

// Direction of step i of the soft walk (pt, wk), as k_walk_soft draws it.
template <int D>
__device__ __forceinline__ void soft_dir(const WalkCfg &c, uint32_t pt, uint32_t wk, int i, float *dir) {
    const uint4 rr = philox(c.rng, pt, wk, (uint32_t)i, ROLE_PRIMAL);
    dir[2] = 0.0f;
    if (D == 2) {
        float sn, cs;
        wosm::sincos_2pi(wosm::u01(rr.x), &sn, &cs);
        dir[0] = cs;
        dir[1] = sn;
    } else {
        const float z = fmaf(-2.0f, wosm::u01(rr.x), 1.0f);
        const float rad = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
        float sn, cs;
        wosm::sincos_2pi(wosm::u01(rr.y), &sn, &cs);
        dir[0] = rad * cs;
        dir[1] = rad * sn;
        dir[2] = z;
    }
}

// Reverse mode of the soft-edge walk: for walks [w0, w0 + nchunk) of the
// flattened (point, walk) space, add dL/du[point] / nwalks times the walk's
// derivative with respect to vertex positions (dV) and values (dg).  One
// thread per walk repeats the walk of k_walk_soft (same Philox draws, the
// same exact nearest primitives, so the same positions), keeping each step's
// position, primitive and throughput in `state` / `sbeta` (step-major, so a
// step's stores coalesce), then sweeps the steps backwards applying the
// transposes of the step relations of k_walk_soft's tangent recurrence:
//   res  += [d > 0] beta (1 - w) g,   beta *= w,   w = min(d, eps) / eps,
//   p    += dir d (before the next step),
// with the tangents dd = n.(pd - cd) and gd of soft_tangents.
template <int D, bool BVH>
__global__ void __launch_bounds__(128) k_soft_adjoint(SceneView S, WalkCfg c, const float *__restrict__ P,
                                                      long long w0, long long nchunk,
                                                      const float *__restrict__ dLdu, float4 *state, float *sbeta,
                                                      double *dV, double *dg) {
    const float eps = c.eps;
    for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nchunk;
         l += (long long)gridDim.x * blockDim.x) {
        const long long idx = w0 + l;
        const uint32_t pt = (uint32_t)(idx / c.nwalks);
        const uint32_t wk = c.walk_offset + (uint32_t)(idx - (long long)pt * c.nwalks);
        const float W = dLdu[pt] / (float)c.nwalks;
        if (W == 0.0f) continue;
        float p[3];
        walk_origin<D>(c, P, pt, wk, p);
        Work work{0, 0, 0};
        float beta = 1.0f;
        bool ok = true;
        for (int i = 0; i < c.nsteps; ++i) {
            const Hit hit = query<D, BVH>(S, p, nullptr, 0, work);
            if (hit.prim < 0 || (i == 0 && !c.double_sided && !inside_test<D>(S, p, hit, nullptr))) {
                ok = false;  // the walk's value is 0 (k_walk_soft): no derivative
                break;
            }
            state[(size_t)i * nchunk + l] = make_float4(p[0], p[1], D == 3 ? p[2] : 0.0f, __int_as_float(hit.prim));
            sbeta[(size_t)i * nchunk + l] = beta;
            const float d = sqrtf(hit.d2);
            beta = beta * (fminf(d, eps) / eps);
            if (i == c.nsteps - 1) break;
            float dir[3];
            soft_dir<D>(c, pt, wk, i, dir);
            for (int k = 0; k < D; ++k) p[k] = fmaf(dir[k], d, p[k]);
        }
        if (!ok) continue;
        float pbar[3] = {0.0f, 0.0f, 0.0f};  // adjoint of the position tangent entering the step
        float bbar = 0.0f;                   // adjoint of the throughput tangent entering the step
        for (int i = c.nsteps - 1; i >= 0; --i) {
            const float4 sv = state[(size_t)i * nchunk + l];
            const float x[3] = {sv.x, sv.y, sv.z};
            const int prim = __float_as_int(sv.w);
            const float bt = sbeta[(size_t)i * nchunk + l];
            const float d = sqrtf(prim_d2<D>(S, prim, x));
            const Rec r = closest_record<D>(S, x, prim);
            int vid[3];
            float wts[3];
            const float g = dirichlet<D>(S, prim, r.t0, r.t1, vid, wts);
            const float w = fminf(d, eps) / eps;
            float dbar = 0.0f;
            if (i < c.nsteps - 1) {
                // p_{i+1} = p_i + dir d: the next step's position adjoint flows into d
                float dir[3];
                soft_dir<D>(c, pt, wk, i, dir);
                for (int k = 0; k < D; ++k) dbar += pbar[k] * dir[k];
            }
            const bool contrib = d > 0.0f;
            const float gbar = contrib ? W * bt * (1.0f - w) : 0.0f;
            const float wbar = (contrib ? -W * bt * g : 0.0f) + bbar * bt;
            if (d < eps) dbar += wbar / eps;
            bbar = (contrib ? W * (1.0f - w) * g : 0.0f) + bbar * w;
            // dd = n.(pd - cd), n = (x - c) / d, cd = sum_j wts_j dV_j
            if (d > 0.0f && dbar != 0.0f) {
                for (int k = 0; k < D; ++k) {
                    const float nk = (x[k] - r.p[k]) / d;
                    pbar[k] += dbar * nk;
                    for (int j = 0; j < D; ++j)
                        atomicAdd(&dV[(size_t)vid[j] * D + k], (double)(-dbar * nk * wts[j]));
                }
            }
            // gd = sum_j bd_j g_j + sum_j wts_j dg_j
            if (gbar != 0.0f) {
                if (dg != nullptr)
                    for (int j = 0; j < D; ++j) atomicAdd(&dg[vid[j]], (double)(gbar * wts[j]));
                soft_bary_adjoint<D>(S, x, r, prim, vid, gbar, pbar, dV);
            }
        }
    }
}

template <int D, bool BVH>
static int launch_soft_adjoint_t(const SceneImpl &S, const float *P, long long total, const wos_params &p,
                                 const float *dLdu, double *dV, double *dg, cudaStream_t st) {
    const SceneView v = S.view();
    const WalkCfg c = make_cfg(p);
    // walks per chunk: the per-step state (20 B per walk and step) stays under 256 MB
    const long long per_walk = (long long)p.nsteps * (long long)(sizeof(float4) + sizeof(float));
    const long long chunk = std::max(1LL, std::min(total, (256LL << 20) / per_walk));
    float4 *state = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&state, (size_t)(chunk * per_walk), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMallocAsync(soft adjoint state)");
    float *sbeta = reinterpret_cast<float *>(state + (size_t)chunk * p.nsteps);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (long long w0 = 0; w0 < total && e == cudaSuccess; w0 += chunk) {
        const long long nc = std::min(chunk, total - w0);
        const int grid = (int)std::min<long long>((nc + 127) / 128, (long long)sms * 16);
        k_soft_adjoint<D, BVH><<<grid, 128, 0, st>>>(v, c, P, w0, nc, dLdu, state, sbeta, dV, dg);
        e = cudaGetLastError();
    }
    cudaFreeAsync(state, st);
    if (e != cudaSuccess) return fail_cuda(e, "k_soft_adjoint launch");
    return 0;
}

int launch_soft_adjoint(const SceneImpl &S, const float *P, long long total, const wos_params &p, const float *dLdu,
                        double *dV, double *dg, cudaStream_t st) {
    if (total == 0) return 0;
    const bool bvh = p.use_bvh != 0;
    if (S.dim == 2)
        return bvh ? launch_soft_adjoint_t<2, true>(S, P, total, p, dLdu, dV, dg, st)
                   : launch_soft_adjoint_t<2, false>(S, P, total, p, dLdu, dV, dg, st);
    return bvh ? launch_soft_adjoint_t<3, true>(S, P, total, p, dLdu, dV, dg, st)
               : launch_soft_adjoint_t<3, false>(S, P, total, p, dLdu, dV, dg, st);
}

template <int D, bool BVH, int WL>
static int launch_soft_t(const SceneImpl &S, const float *P, long long total, const wos_params &p, const float *tV,
                         const float *tg, float *vals, float *tans, unsigned long long *counter, cudaStream_t st) {
    const SceneView v = S.view();
    const WalkCfg c = make_cfg(p);
    int grid = 0;
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_walk_soft<D, BVH, WL>, 256, 0);
    if (e != cudaSuccess) return fail_cuda(e, "occupancy(k_walk_soft)");
    grid = std::max(1, per) * sms;
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counter)");
    k_walk_soft<D, BVH, WL><<<grid, 256, 0, st>>>(v, c, P, total, counter, 32, tV, tg, vals, tans);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_walk_soft launch");
    return 0;
}

int launch_walk_soft(const SceneImpl &S, const float *P, long long total, const wos_params &p, const float *tV,
                     const float *tg, float *vals, float *tans, unsigned long long *counter, cudaStream_t st) {
    if (total == 0) return 0;
    const bool bvh = p.use_bvh != 0;
    if (S.dim == 2)
        return bvh ? launch_soft_t<2, true, 0>(S, P, total, p, tV, tg, vals, tans, counter, st)
                   : launch_soft_t<2, false, 0>(S, P, total, p, tV, tg, vals, tans, counter, st);
    return bvh ? launch_soft_t<3, true, 0>(S, P, total, p, tV, tg, vals, tans, counter, st)
               : launch_soft_t<3, false, 0>(S, P, total, p, tV, tg, vals, tans, counter, st);
}

int launch_walk_plain(const SceneImpl &S, const float *P, long long total, const wos_params &p, float *values,
                      cudaStream_t st) {
    if (total == 0) return 0;
    const SceneView v = S.view();
    const WalkCfg c = make_cfg(p);
    const int B = 256;
    const long long G = (total + B - 1) / B;
    const bool bvh = p.use_bvh != 0;
    if (S.dim == 2) {
        if (bvh)
            k_walk_plain<2, true><<<(unsigned)G, B, 0, st>>>(v, c, P, total, values);
        else
            k_walk_plain<2, false><<<(unsigned)G, B, 0, st>>>(v, c, P, total, values);
    } else {
        if (bvh)
            k_walk_plain<3, true><<<(unsigned)G, B, 0, st>>>(v, c, P, total, values);
        else
            k_walk_plain<3, false><<<(unsigned)G, B, 0, st>>>(v, c, P, total, values);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_walk_plain launch");
    return 0;
}

int launch_reduce(const float *vals, int n, int nw, double *mean, double *var, cudaStream_t st) {
    if (n == 0) return 0;
    const int B = 256;
    const long long G = ((long long)n * 32 + B - 1) / B;
    k_reduce<<<(unsigned)G, B, 0, st>>>(vals, n, nw, mean, var);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_reduce launch");
    return 0;
}

int launch_closest(const SceneImpl &S, const float *P, int n, bool bvh, const QueryOut &o, cudaStream_t st) {
    if (n == 0) return 0;
    const SceneView v = S.view();
    const int B = 128, G = (n + B - 1) / B;
    if (S.dim == 2) {
        if (bvh)
            k_closest<2, true><<<G, B, 0, st>>>(v, P, n, o);
        else
            k_closest<2, false><<<G, B, 0, st>>>(v, P, n, o);
    } else {
        if (bvh)
            k_closest<3, true><<<G, B, 0, st>>>(v, P, n, o);
        else
            k_closest<3, false><<<G, B, 0, st>>>(v, P, n, o);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_closest launch");
    return 0;
}

int launch_ball(const SceneImpl &S, const uint8_t *valid, const float *pt, const float *nrm, int n, float eps,
                bool bvh, float *R, cudaStream_t st) {
    if (n == 0) return 0;
    const SceneView v = S.view();
    const int B = 128, G = (n + B - 1) / B;
    if (S.dim == 2) {
        if (bvh)
            k_ball<2, true><<<G, B, 0, st>>>(v, valid, pt, nrm, n, eps, R);
        else
            k_ball<2, false><<<G, B, 0, st>>>(v, valid, pt, nrm, n, eps, R);
    } else {
        if (bvh)
            k_ball<3, true><<<G, B, 0, st>>>(v, valid, pt, nrm, n, eps, R);
        else
            k_ball<3, false><<<G, B, 0, st>>>(v, valid, pt, nrm, n, eps, R);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_ball launch");
    return 0;
}

template <int D, bool BVH, int ND, int WL, bool COUNT>
static int launch_adjoint_t(const SceneImpl &S, const float *P, long long total, const wos_params &p,
                            const AdjCfg &a, const float *dLdu, const AdjOut &out, unsigned long long *counter,
                            cudaStream_t st) {
    const SceneView v = S.view();
    const WalkCfg c = make_cfg(p);
    const bool want_cdf = D == 2 && S.src_type != 0 && p.use_IS_for_greens;
    Shape sh;
    const bool want_acc = ND != ADJ_ND_ONLY && a.want_dsrc && p.include_source && S.src_type != 0 && D == 2;
    int rc = shape_for(k_adjoint<D, BVH, ND, WL, COUNT>, S, D, BVH, want_cdf, sh, adj_thread_bytes<D>(want_acc),
                       256);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counter)");
    const int chunk = std::max(1, g_cfg[D - 2].chunk / 2);
    k_adjoint<D, BVH, ND, WL, COUNT><<<sh.grid, sh.block, sh.smem, st>>>(v, c, a, P, total, dLdu, counter, chunk,
                                                                         sh.n_top, sh.stage_cdf, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_adjoint launch");
    return 0;
}

int launch_adjoint(const SceneImpl &S, const float *P, long long total, const wos_params &p, const AdjCfg &a,
                   const float *dLdu, int mode, const AdjOut &out, unsigned long long *counter, cudaStream_t st) {
    if (total == 0) return 0;
    const bool bvh = p.use_bvh != 0;
    const int wl = specialised_depth(S.wt_levels);
    // work accounting runs the any-depth instance that keeps counters
    const bool count = work_counting_enabled() != 0;
#define WOS_ADJ_M(D_, B_, W_, C_)                                                                                   \
    switch (mode) {                                                                                                 \
        case ADJ_ND_ONLY:                                                                                           \
            return launch_adjoint_t<D_, B_, ADJ_ND_ONLY, W_, C_>(S, P, total, p, a, dLdu, out, counter, st);        \
        case ADJ_FROM_RECORDS:                                                                                      \
            return launch_adjoint_t<D_, B_, ADJ_FROM_RECORDS, W_, C_>(S, P, total, p, a, dLdu, out, counter, st);   \
        case ADJ_TANGENT:                                                                                           \
            return launch_adjoint_t<D_, B_, ADJ_TANGENT, W_, C_>(S, P, total, p, a, dLdu, out, counter, st);        \
        default: return launch_adjoint_t<D_, B_, ADJ_RECOMPUTE, W_, C_>(S, P, total, p, a, dLdu, out, counter, st); \
    }
#define WOS_ADJ(D_)                          \
    if (count) {                             \
        if (!bvh) {                          \
            WOS_ADJ_M(D_, false, 0, true)    \
        }                                    \
        WOS_ADJ_M(D_, true, 0, true)         \
    }                                        \
    if (!bvh) {                              \
        WOS_ADJ_M(D_, false, 0, false)       \
    }                                        \
    switch (wl) {                            \
        case 1: WOS_ADJ_M(D_, true, 1, false) \
        case 2: WOS_ADJ_M(D_, true, 2, false) \
        case 3: WOS_ADJ_M(D_, true, 3, false) \
        default: WOS_ADJ_M(D_, true, 0, false) \
    }
    if (S.dim == 2) {
        WOS_ADJ(2)
    }
    WOS_ADJ(3)
#undef WOS_ADJ_M
#undef WOS_ADJ
}

// ------------------------------------------------------------------ sample order
// Adjoint samples that start from forward records run in the order of their
// boundary primitive along the trees' primitive order (curve order in 2D,
// Hilbert order in 3D).  Every sample begins with the inscribed-ball
// bisection around that primitive, so in this order the lanes of a warp --
// and the warps the GPU runs at the same time -- start next to each other and
// share cached tree nodes for those queries.  The gain is small (0.5-1 % of a
// step: the ball walks, most of a sample's queries, leave the neighbourhood
// at once), the sort costs ~0.3 ms per 20 M samples.  Results do not depend on
// the order: each sample draws from its own Philox counters; only the
// summation order of the FP64 gradient atomics changes.
static int g_sample_order = 1;

int set_sample_order(int mode) {
    g_sample_order = mode ? 1 : 0;
    return 0;
}

int sample_order_mode() { return g_sample_order; }

__global__ void k_prim_rank(const int *__restrict__ lorig, int nF, unsigned *rank) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nF) rank[__ldg(&lorig[s])] = (unsigned)s;
}

template <int D>
__global__ void k_record_keys(const int *__restrict__ wrec, long long total, const unsigned *__restrict__ rank, int nF,
                              unsigned *keys, unsigned *ids) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += stride) {
        const int code = __ldg(&wrec[i * walkrec_words(D)]);
        const int prim = code & 0x3fffffff;
        keys[i] = (code < 0 || prim >= nF) ? (unsigned)nF : __ldg(&rank[prim]);
        ids[i] = (unsigned)i;
    }
}

// Bits of a radix-sort key whose largest value is n.
static int key_bits_ll(long long n) {
    int b = 1;
    while (b < 32 && (1LL << b) <= n) ++b;
    return b;
}
static int key_bits(int nF) { return key_bits_ll(nF); }

size_t record_order_bytes(int nF, long long total) {
    if (!g_sample_order || total <= 1 || total > (long long)INT_MAX || nF <= 0) return 0;
    cub::DoubleBuffer<unsigned> k(nullptr, nullptr), v(nullptr, nullptr);
    size_t tmp = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, tmp, k, v, (int)total, 0, key_bits(nF)) != cudaSuccess) return 0;
    const auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(sizeof(unsigned) * (size_t)nF) + 4 * al(sizeof(unsigned) * (size_t)total) + al(tmp);
}

int launch_record_order(const SceneImpl &S, const int *wrec, long long total, void *ws, size_t ws_bytes,
                        const unsigned **order, cudaStream_t st) {
    *order = nullptr;
    const size_t need = record_order_bytes(S.nF, total);
    if (need == 0) return 0;
    if (ws == nullptr || ws_bytes < need) return fail(WOS_ERR_WORKSPACE, "record order: workspace too small");
    const auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char *b = (char *)ws;
    unsigned *rank = (unsigned *)b;
    b += al(sizeof(unsigned) * (size_t)S.nF);
    unsigned *buf[4];
    for (int i = 0; i < 4; ++i) {
        buf[i] = (unsigned *)b;
        b += al(sizeof(unsigned) * (size_t)total);
    }
    const size_t tmp_bytes = need - (size_t)(b - (char *)ws);
    k_prim_rank<<<(S.nF + 255) / 256, 256, 0, st>>>(S.lorig, S.nF, rank);
    const int G = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    if (S.dim == 2)
        k_record_keys<2><<<G, 256, 0, st>>>(wrec, total, rank, S.nF, buf[0], buf[2]);
    else
        k_record_keys<3><<<G, 256, 0, st>>>(wrec, total, rank, S.nF, buf[0], buf[2]);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_record_keys launch");
    cub::DoubleBuffer<unsigned> k(buf[0], buf[1]), v(buf[2], buf[3]);
    size_t tmp = tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(b, tmp, k, v, (int)total, 0, key_bits(S.nF), st);
    if (e != cudaSuccess) return fail_cuda(e, "record order sort");
    *order = v.Current();
    return 0;
}

int launch_add_f64(const double *src, float *dst, long long n, cudaStream_t st) {
    if (n == 0 || dst == nullptr) return 0;
    const int B = 256;
    const int G = (int)std::min<long long>((n + B - 1) / B, 4096);
    k_add_f64_to_f32<<<G, B, 0, st>>>(src, dst, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_add_f64_to_f32 launch");
    return 0;
}

// ------------------------------------------------------------------ batched launch
// Many (scene, query set) items in one persistent launch per dimension.  The
// walk index space is the concatenation of every item's n x nwalks walks in
// item order (scene-major), so warps move through the items together and each
// scene's trees stay resident in L2 while its walks run.  Each lane carries
// its item; the cooperative query serves one lane's item at a time.

__device__ __forceinline__ int find_item(const BatchItemDev *__restrict__ items, int n_items, long long idx) {
    int lo = 0, hi = n_items - 1;  // last item with walk_begin <= idx
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&items[mid].walk_begin) <= idx)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_item_point(const BatchItemDev *__restrict__ items, int n_items, int p) {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&items[mid].point_begin) <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int D, int WL = 0, class WK>
__device__ __forceinline__ Hit warp_queries_batch(const SceneView *__restrict__ views, bool active, int item,
                                                  const float *x, int warm, WK &work, float ball_m = -1.0f) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    Hit mine{-1, INFINITY};
    unsigned act = __ballot_sync(FULL, active);
    // per-point parts of each search, every lane for its own point at once
    // (as in warp_queries)
    float lim = 0.0f, wd2 = INFINITY;
    if (active) {
        const SceneView &Si = views[item];
        const float tol2 = prune_tol2<D>(Si, x);
        if (ball_m > 0.0f) {
            lim = wball_bound(ball_m, tol2);
        } else {
            lim = tol2;
            if (warm >= 0) wd2 = prim_d2<D>(Si, warm, x);
        }
    }
    while (act) {
        const int j = __ffs(act) - 1;
        act &= act - 1u;
        float q[3];
        q[0] = __shfl_sync(FULL, x[0], j);
        q[1] = __shfl_sync(FULL, x[1], j);
        q[2] = D == 3 ? __shfl_sync(FULL, x[2], j) : 0.0f;
        const int wp = __shfl_sync(FULL, warm, j);
        const int it = __shfl_sync(FULL, item, j);
        const float bm = __shfl_sync(FULL, ball_m, j);
        const float lj = __shfl_sync(FULL, lim, j);
        const float wj = __shfl_sync(FULL, wd2, j);
        const SceneView &Sj = views[it];
        Hit h{-1, INFINITY};
        if (bm > 0.0f) {
            wball_b<D, WL>(Sj, q, lj, bm, h, work);
        } else {
            if (wp >= 0) {
                h.prim = wp;
                h.d2 = wj;
            }
            h = wquery_tol<D, WL>(Sj, q, h, lj, work);
        }
        if (lane == j) mine = h;
    }
    return mine;
}

// One launch covers a run of items whose walks occupy [base, base + total)
// of the group's walk index space; WL > 0: every item's tree has WL levels.
template <int D, int WL, bool COUNT>
__global__ void __launch_bounds__(512) k_walk_batch(const SceneView *__restrict__ views,
                                                   const WalkCfg *__restrict__ cfgs,
                                                   const BatchItemDev *__restrict__ items, int n_items,
                                                   long long base, long long total, unsigned long long *counter,
                                                   int chunk, WalkOut out, int count_work) {
    Queue q{0, 0, false};
    bool active = false;
    long long idx = 0;
    int item = 0;
    uint32_t pt = 0, wk = 0;
    Walker w;
    w.last = -1;
    typename std::conditional<COUNT, Work, NoWork>::type work{};
    for (;;) {
        const bool was = active;
        if (!refill(q, active, idx, counter, total, chunk)) break;
        if (active && !was) {
            idx += base;
            item = find_item(items, n_items, idx);
            const BatchItemDev &it = items[item];
            const long long local = idx - it.walk_begin;
            pt = (uint32_t)(local / it.nwalks);
            wk = cfgs[item].walk_offset + (uint32_t)(local - (long long)pt * it.nwalks);
            float x0[3];
            walk_origin<D>(cfgs[item], it.P, pt, wk, x0);
            w.start(x0, D);
        }
        const Hit hit = warp_queries_batch<D, WL>(views, active, item, w.p, w.last, work);
        if (!active) continue;
        const SceneView &S = views[item];
        const WalkCfg &c = cfgs[item];
        w.last = hit.prim;
        const int r = walker_advance<D>(w, S, hit, c, c.eps, c.project != 0, c.prevent_fd != 0, pt, wk, ROLE_PRIMAL,
                                        out.wds != nullptr, S.guide);
        if (r == W_CONTINUE) continue;
        active = false;
        float v = 0.0f;
        Rec rec;
        if (r == W_VALID) {
            rec = closest_record<D>(S, w.p, hit.prim);
            v = dirichlet<D>(S, hit.prim, rec.t0, rec.t1, nullptr, nullptr);
            if (c.include_source) v += w.contrib;
            if (!isfinite(v)) atomicOr(&g_status, ST_NONFINITE);
        }
        out.values[idx] = v;
        if (out.wrec) {
            if (D == 2) {
                reinterpret_cast<int2 *>(out.wrec)[idx] =
                    r == W_VALID ? make_int2(hit.prim | (rec.flip ? 0x40000000 : 0), __float_as_int(rec.t0))
                                 : make_int2(-1, 0);
            } else {
                reinterpret_cast<int4 *>(out.wrec)[idx] =
                    r == W_VALID ? make_int4(hit.prim | (rec.flip ? 0x40000000 : 0), __float_as_int(rec.t0),
                                             __float_as_int(rec.t1), 0)
                                 : make_int4(-1, 0, 0, 0);
            }
        }
        if (out.wds) {
#pragma unroll
            for (int k = 0; k < 5; ++k) out.wds[(size_t)idx * 5 + k] = r == W_VALID ? w.ds[k] : 0.0f;
        }
    }
    if constexpr (COUNT) {
        if (count_work) flush_work<true>(work);
    } else {
        // never taken; kept for the same reason as in k_walk
        if (count_work) flush_work<true>(Work{0, 0, 0});
    }
}

// Per-point FP64 mean / variance over the concatenated point space.
__global__ void k_reduce_batch(const float *__restrict__ vals, const BatchItemDev *__restrict__ items, int n_items,
                               int n_points, double *mean, double *var) {
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= n_points) return;
    const int item = find_item_point(items, n_items, p);
    const BatchItemDev &it = items[item];
    const int nw = it.nwalks;
    const float *v = vals + it.walk_begin + (long long)(p - it.point_begin) * nw;
    double s = 0.0, cc = 0.0;
    for (int w = lane; w < nw; w += 32) neumaier_add(s, cc, (double)v[w]);
    const double m = warp_sum_comp(s, cc) / nw;
    double qq = 0.0, qc = 0.0;
    for (int w = lane; w < nw; w += 32) {
        const double e = (double)v[w] - m;
        neumaier_add(qq, qc, e * e);
    }
    const double q2 = warp_sum_comp(qq, qc);
    if (lane == 0) {
        mean[p] = m;
        if (var) var[p] = nw > 1 ? q2 / (nw - 1) : 0.0;
    }
}

// Per item: dL/du of its points and its loss (one block per item).
__global__ void k_loss_batch(const double *__restrict__ mean, const BatchItemDev *__restrict__ items, float *dLdu,
                             double *loss) {
    __shared__ double red[256];
    const BatchItemDev &it = items[blockIdx.x];
    double acc = 0.0;
    for (int i = threadIdx.x; i < it.n; i += blockDim.x) {
        const int p = it.point_begin + i;
        const double u = mean[p];
        double e = u;
        if (it.loss_kind == 2) e = u - (double)it.target[i];
        if (it.loss_kind == 0) {
            dLdu[p] = it.target[i];
        } else {
            dLdu[p] = (float)(2.0 * e / it.n);
            acc += e * e / it.n;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[blockIdx.x] = red[0];
}

// Adjoint of every item, starting from the forward records.  Gradients go to
// per-item FP64 accumulators (acc + it.dV_off / dg_off / ds_off).
template <int D, int WL, bool COUNT>
__global__ void __launch_bounds__(256, ADJ_MIN_BLOCKS) k_adjoint_batch(
    const SceneView *__restrict__ views, const WalkCfg *__restrict__ cfgs, AdjCfg a,
    const BatchItemDev *__restrict__ items, int n_items, long long base, long long total,
    const float *__restrict__ dLdu,
    unsigned long long *counter, int chunk, const int *__restrict__ wrec, const float *__restrict__ wds, double *acc,
    int count_work, const unsigned *__restrict__ order) {
    extern __shared__ float4 smem[];
    // source-gradient accumulators only when the launch has source derivatives
    // (the launcher sizes shared memory the same way)
    const bool acc_on = D == 2 && wds != nullptr;  // source derivatives exist in 2D only
    const AdjSmem<D> am = adj_smem<D>(reinterpret_cast<double *>(smem), acc_on);
    AdjSlot<D> &slot = *am.slot;
    double *acc_src = am.acc;  // k-th accumulator at acc_src[k * blockDim.x]
    const int AS = blockDim.x;
    if (acc_on) {
#pragma unroll
        for (int k = 0; k < 5; ++k) acc_src[k * AS] = 0.0;
    }
    int acc_item = -1;  // item whose source gradient acc_src holds
    NdState<D> &st = slot.st;
    float *rn = st.rn;
    float &rt0 = slot.rt0, &rt1 = slot.rt1;
    float &ba = slot.ba, &bb = slot.bb;
    int &bk = slot.bk;
    int &bwarm = slot.bwarm;
    Queue q{0, 0, false};
    bool active = false;
    long long idx = 0;
    int item = 0;
    uint32_t pt = 0, wk = 0;
    int phase = PH_IDLE;
    double W = 0.0;
    Walker w;
    int rprim = 0;
    float qpos[3] = {0, 0, 0};
    typename std::conditional<COUNT, Work, NoWork>::type work{};
    w.last = -1;
    for (;;) {
        const bool was = active;
        if (!refill(q, active, idx, counter, total, chunk)) break;
        if (active && !was) {
            idx += base;
            if (order != nullptr) idx = (long long)__ldg(&order[idx]);
            item = find_item(items, n_items, idx);
            const BatchItemDev &it = items[item];
            const SceneView &S = views[item];
            const WalkCfg &c = cfgs[item];
            const long long local = idx - it.walk_begin;
            pt = (uint32_t)(local / it.nwalks);
            wk = c.walk_offset + (uint32_t)(local - (long long)pt * it.nwalks);
            W = (double)__ldg(&dLdu[it.point_begin + pt]) / it.nwalks;
            phase = PH_BALL;
            int code = -1;
            if (D == 2) {
                const int2 wr = __ldg(reinterpret_cast<const int2 *>(wrec) + idx);
                code = wr.x;
                rt0 = __int_as_float(wr.y);
                rt1 = 0.0f;
            } else {
                const int4 wr = __ldg(reinterpret_cast<const int4 *>(wrec) + idx);
                code = wr.x;
                rt0 = __int_as_float(wr.y);
                rt1 = __int_as_float(wr.z);
            }
            if (W == 0.0 || code < 0) {
                active = false;
            } else {
                rprim = code & 0x3fffffff;
                const Rec rec = record_from<D>(S, rprim, rt0, rt1, (code & 0x40000000) != 0);
                int vid[3];
                float wts[3];
                st.uref = dirichlet<D>(S, rprim, rt0, rt1, vid, wts);
                if (a.want_dg) {
#pragma unroll
                    for (int s2 = 0; s2 < D; ++s2) atomicAdd(&acc[it.dg_off + vid[s2]], W * (double)wts[s2]);
                }
                if (acc_on && a.want_dsrc && c.include_source && S.src_type != 0) {
                    if (acc_item != item) {
                        if (acc_item >= 0) {
#pragma unroll
                            for (int k = 0; k < 5; ++k)
                                if (acc_src[k * AS] != 0.0)
                                    atomicAdd(&acc[items[acc_item].ds_off + k], acc_src[k * AS]);
                        }
#pragma unroll
                        for (int k = 0; k < 5; ++k) acc_src[k * AS] = 0.0;
                        acc_item = item;
                    }
#pragma unroll
                    for (int k = 0; k < 5; ++k) acc_src[k * AS] += W * (double)__ldg(&wds[(size_t)idx * 5 + k]);
                }
                if (!a.want_dV) {
                    active = false;
                } else {
#pragma unroll
                    for (int k = 0; k < D; ++k) {
                        st.p[k] = rec.p[k];
                        rn[k] = rec.n[k];
                    }
                    ba = a.ball_eps;
                    bb = S.half_min_extent;
                    bk = 0;
                    bwarm = -1;
                    const float m = (ba + bb) * 0.5f;
#pragma unroll
                    for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m, st.p[k]);
                }
            }
        }
        const bool walking = phase == PH_ANTI_WALK;
        float x[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) x[k] = walking ? w.p[k] : qpos[k];
        bool need = active;
        float ball_m = -1.0f;
        Hit pre{-1, INFINITY};
        if (active && phase == PH_BALL)
            ball_precheck<D>(views[item], qpos, (ba + bb) * 0.5f, bwarm, rprim, need, ball_m, pre);
        Hit hit = warp_queries_batch<D, WL>(views, need, item, x, walking ? w.last : rprim, work, ball_m);
        if (!active) continue;
        if (phase == PH_BALL && (!need || (ball_m > 0.0f && hit.prim < 0))) hit = pre;
        const SceneView &S = views[item];
        const WalkCfg &c = cfgs[item];
        const bool with_src = a.source_in_nd && D == 2 && S.src_type != 0;
        if (walking) w.last = hit.prim;
        bool finish_anti = false;
        float uq = 0.0f;
        if (phase == PH_BALL) {
            const float d = sqrtf(hit.d2);
            const float m = (ba + bb) * 0.5f;
            if (wosm::ball_accepts(d, m)) {
                ba = m;
            } else {
                bb = m;
                bwarm = hit.prim;
            }
            ++bk;
            if (bk < 10) {
                const float m2 = (ba + bb) * 0.5f;
#pragma unroll
                for (int k = 0; k < D; ++k) qpos[k] = fmaf(rn[k], m2, st.p[k]);
                continue;
            }
            st.R = ba;
            nd_setup<D>(st, S, c, a, pt, wk);
            nd_point<D>(st, qpos);
            phase = PH_ANTI_START;
            continue;
        }
        const uint32_t role = st.which == 0 ? ROLE_ANTI_A : ROLE_ANTI_B;
        // the ball walk's first query (PH_ANTI_START) either ends it inside the
        // epsilon2 shell or starts the walk; both walk phases then share one
        // walker_advance (one inlined copy keeps the kernel's code small)
        bool advance = phase == PH_ANTI_WALK;
        if (phase == PH_ANTI_START) {
            const float d = sqrtf(hit.d2);
            if (d < a.epsilon2) {
                const Rec r2 = closest_record<D>(S, qpos, hit.prim);
                uq = dirichlet<D>(S, hit.prim, r2.t0, r2.t1, nullptr, nullptr);
                finish_anti = true;
            } else {
                w.start(qpos, D);
                w.last = hit.prim;
                phase = PH_ANTI_WALK;
                advance = true;
            }
        }
        if (advance) {
            const int r = walker_advance<D>(w, S, hit, c, a.epsilon2, c.project != 0, false, pt, wk, role, false, S.guide);
            if (r == W_CONTINUE) continue;
            if (r == W_VALID) {
                const Rec r2 = closest_record<D>(S, w.p, hit.prim);
                uq = dirichlet<D>(S, hit.prim, r2.t0, r2.t1, nullptr, nullptr);
                if (with_src) uq += w.contrib;
            }
            finish_anti = true;
        }
        if (finish_anti) {
            nd_accumulate<D>(st, a, uq);
            st.which += 1;
            if (st.which == 1) {
                nd_point<D>(st, qpos);
                phase = PH_ANTI_START;
                continue;
            }
            float gn[3], gt[3];
            nd_finish<D>(st, S, c, a, pt, wk, with_src, gn);
            tangent_derivative<D>(S, rprim, gt);
            int vid[3];
            float wts[3];
            dirichlet<D>(S, rprim, rt0, rt1, vid, wts);
            const long long off = items[item].dV_off;
#pragma unroll
            for (int s2 = 0; s2 < D; ++s2)
#pragma unroll
                for (int k = 0; k < D; ++k)
                    atomicAdd(&acc[off + (long long)vid[s2] * D + k], W * (double)(-(wts[s2] * (gn[k] + gt[k]))));
            active = false;
            phase = PH_IDLE;
        }
    }
    if constexpr (COUNT) {
        if (count_work) flush_work<true>(work);
    } else {
        // never taken; kept for the same reason as in k_walk
        if (count_work) flush_work<true>(Work{0, 0, 0});
    }
    if (acc_item >= 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k)
            if (acc_src[k * AS] != 0.0) atomicAdd(&acc[items[acc_item].ds_off + k], acc_src[k * AS]);
    }
}

__global__ void k_acc_to_f32(const double *__restrict__ acc, float *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)acc[i];
}

template <typename Kern>
static int persistent_grid(Kern kern, int block, size_t smem, int blocks_per_sm, int &grid) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail_cuda(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, block, smem);
    if (e != cudaSuccess) return fail_cuda(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) return fail(WOS_ERR_UNSUPPORTED, "batch kernel does not fit on an SM with this launch config");
    grid = sms * (blocks_per_sm > 0 ? std::min(blocks_per_sm, occ) : occ);
    return 0;
}

template <int D, int WL, bool COUNT>
static int launch_walk_batch_t(const SceneView *views, const WalkCfg *cfgs, const BatchItemDev *items, int n_items,
                               long long base, long long total, const BatchLaunch &L, const WalkOut &out,
                               unsigned long long *counter, cudaStream_t st) {
    int grid = 0;
    if (int rc = persistent_grid(k_walk_batch<D, WL, COUNT>, L.block, 0, L.blocks_per_sm, grid)) return rc;
    k_walk_batch<D, WL, COUNT><<<grid, L.block, 0, st>>>(views, cfgs, items, n_items, base, total, counter, L.chunk,
                                                         out, L.count_work);
    return 0;
}

int launch_walk_batch(int D, int wl, const SceneView *views, const WalkCfg *cfgs, const BatchItemDev *items,
                      int n_items, long long base, long long total, const BatchLaunch &L, const WalkOut &out,
                      unsigned long long *counter, cudaStream_t st) {
    if (total == 0 || n_items == 0) return 0;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counter)");
    static_assert(WT_SPECIALISED_LEVELS == 3, "one instance per specialised depth");
    int rc = 0;
#define WOS_WB(DD, WW, CC) \
    rc = launch_walk_batch_t<DD, WW, CC>(views, cfgs, items, n_items, base, total, L, out, counter, st)
    // work accounting runs the any-depth instance that keeps counters
    if (L.count_work) {
        if (D == 2) WOS_WB(2, 0, true); else WOS_WB(3, 0, true);
    } else if (D == 2) {
        if (wl == 1) WOS_WB(2, 1, false); else if (wl == 2) WOS_WB(2, 2, false);
        else if (wl == 3) WOS_WB(2, 3, false); else WOS_WB(2, 0, false);
    } else {
        if (wl == 1) WOS_WB(3, 1, false); else if (wl == 2) WOS_WB(3, 2, false);
        else if (wl == 3) WOS_WB(3, 3, false); else WOS_WB(3, 0, false);
    }
#undef WOS_WB
    if (rc) return rc;
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_walk_batch launch");
    return 0;
}

template <int D, int WL, bool COUNT>
static int launch_adjoint_batch_t(const SceneView *views, const WalkCfg *cfgs, const AdjCfg &a,
                                  const BatchItemDev *items, int n_items, long long base, long long total,
                                  const float *dLdu, const int *wrec, const float *wds, double *acc,
                                  const BatchLaunch &L, unsigned long long *counter, const unsigned *order,
                                  cudaStream_t st) {
    const int block = std::min(L.block, 256);
    const size_t smem = (size_t)block * adj_thread_bytes<D>(wds != nullptr) + 16;
    const int chunk = std::max(1, L.chunk / 2);
    int grid = 0;
    if (int rc = persistent_grid(k_adjoint_batch<D, WL, COUNT>, block, smem, L.blocks_per_sm, grid)) return rc;
    k_adjoint_batch<D, WL, COUNT><<<grid, block, smem, st>>>(views, cfgs, a, items, n_items, base, total, dLdu,
                                                             counter, chunk, wrec, wds, acc, L.count_work, order);
    return 0;
}

// Sample order of a batch group's adjoint (the batched counterpart of
// launch_record_order): keys are item-major -- item i owns the key range
// [prim_off_i, prim_off_i + nF_i], its invalid records taking the last key --
// so the sorted order keeps every item's samples, and so every run's, in
// their own walk range, each sorted by boundary primitive.
__device__ __forceinline__ int find_item_prim(const BatchItemDev *__restrict__ items, int n_items, long long s) {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&items[mid].prim_off) <= s)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void k_batch_prim_rank(const SceneView *__restrict__ views, const BatchItemDev *__restrict__ items,
                                  int n_items, long long nprims, unsigned *rank) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nprims; s += stride) {
        const int i = find_item_prim(items, n_items, s);
        const long long off = __ldg(&items[i].prim_off);
        const long long local = s - off;
        if (local < views[i].nF) rank[off + __ldg(&views[i].lorig[local])] = (unsigned)s;
    }
}

template <int D>
__global__ void k_batch_record_keys(const SceneView *__restrict__ views, const BatchItemDev *__restrict__ items,
                                    int n_items, const int *__restrict__ wrec, long long total,
                                    const unsigned *__restrict__ rank, unsigned *keys, unsigned *ids) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += stride) {
        const int it = find_item(items, n_items, i);
        const long long off = __ldg(&items[it].prim_off);
        const int nF = views[it].nF;
        const int code = __ldg(&wrec[i * walkrec_words(D)]);
        const int prim = code & 0x3fffffff;
        keys[i] = (code < 0 || prim >= nF) ? (unsigned)(off + nF) : __ldg(&rank[off + prim]);
        ids[i] = (unsigned)i;
    }
}

static size_t batch_order_bytes_any_mode(long long nkeys, long long total) {
    if (total <= 1 || total > (long long)INT_MAX || nkeys <= 0 || nkeys > (long long)UINT_MAX) return 0;
    cub::DoubleBuffer<unsigned> k(nullptr, nullptr), v(nullptr, nullptr);
    size_t tmp = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, tmp, k, v, (int)total, 0, key_bits_ll(nkeys)) != cudaSuccess)
        return 0;
    const auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return al(sizeof(unsigned) * (size_t)nkeys) + 4 * al(sizeof(unsigned) * (size_t)total) + al(tmp);
}

size_t batch_order_bytes(long long nkeys, long long total) {
    return g_sample_order ? batch_order_bytes_any_mode(nkeys, total) : 0;
}

// A plan sized for an order (created in mode 1) keeps it.
int launch_batch_order(int D, const SceneView *views, const BatchItemDev *items, int n_items, long long nkeys,
                       const int *wrec, long long total, void *ws, size_t ws_bytes, const unsigned **order,
                       cudaStream_t st) {
    *order = nullptr;
    if (ws == nullptr || ws_bytes == 0 || total <= 1) return 0;
    const size_t need = batch_order_bytes_any_mode(nkeys, total);
    if (need == 0) return 0;
    if (ws_bytes < need) return fail(WOS_ERR_WORKSPACE, "batch order: workspace too small");
    const auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char *b = (char *)ws;
    unsigned *rank = (unsigned *)b;
    b += al(sizeof(unsigned) * (size_t)nkeys);
    unsigned *buf[4];
    for (int i = 0; i < 4; ++i) {
        buf[i] = (unsigned *)b;
        b += al(sizeof(unsigned) * (size_t)total);
    }
    const size_t tmp_bytes = need - (size_t)(b - (char *)ws);
    const int GP = (int)std::min<long long>((nkeys + 255) / 256, 148 * 16);
    k_batch_prim_rank<<<GP, 256, 0, st>>>(views, items, n_items, nkeys, rank);
    const int G = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    if (D == 2)
        k_batch_record_keys<2><<<G, 256, 0, st>>>(views, items, n_items, wrec, total, rank, buf[0], buf[2]);
    else
        k_batch_record_keys<3><<<G, 256, 0, st>>>(views, items, n_items, wrec, total, rank, buf[0], buf[2]);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_batch_record_keys launch");
    cub::DoubleBuffer<unsigned> k(buf[0], buf[1]), v(buf[2], buf[3]);
    size_t tmp = tmp_bytes;
    e = cub::DeviceRadixSort::SortPairs(b, tmp, k, v, (int)total, 0, key_bits_ll(nkeys), st);
    if (e != cudaSuccess) return fail_cuda(e, "batch order sort");
    *order = v.Current();
    return 0;
}

int launch_adjoint_batch(int D, int wl, const SceneView *views, const WalkCfg *cfgs, const AdjCfg &a,
                         const BatchItemDev *items, int n_items, long long base, long long total,
                         const float *dLdu, const int *wrec, const float *wds, double *acc, const BatchLaunch &L,
                         unsigned long long *counter, const unsigned *order, cudaStream_t st) {
    if (total == 0 || n_items == 0) return 0;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemsetAsync(counter)");
    int rc = 0;
#define WOS_AB(DD, WW, CC)                                                                                        \
    rc = launch_adjoint_batch_t<DD, WW, CC>(views, cfgs, a, items, n_items, base, total, dLdu, wrec, wds, acc, L, \
                                            counter, order, st)
    // work accounting runs the any-depth instance that keeps counters
    if (L.count_work) {
        if (D == 2) WOS_AB(2, 0, true); else WOS_AB(3, 0, true);
    } else if (D == 2) {
        if (wl == 1) WOS_AB(2, 1, false); else if (wl == 2) WOS_AB(2, 2, false);
        else if (wl == 3) WOS_AB(2, 3, false); else WOS_AB(2, 0, false);
    } else {
        if (wl == 1) WOS_AB(3, 1, false); else if (wl == 2) WOS_AB(3, 2, false);
        else if (wl == 3) WOS_AB(3, 3, false); else WOS_AB(3, 0, false);
    }
#undef WOS_AB
    if (rc) return rc;
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_adjoint_batch launch");
    return 0;
}

int launch_reduce_batch(const float *vals, const BatchItemDev *items, int n_items, int n_points, double *mean,
                        double *var, cudaStream_t st) {
    if (n_points == 0) return 0;
    const int B = 256;
    const long long G = ((long long)n_points * 32 + B - 1) / B;
    k_reduce_batch<<<(unsigned)G, B, 0, st>>>(vals, items, n_items, n_points, mean, var);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_reduce_batch launch");
    return 0;
}

int launch_loss_batch(const double *mean, const BatchItemDev *items, int n_items, float *dLdu, double *loss,
                      cudaStream_t st) {
    if (n_items == 0) return 0;
    k_loss_batch<<<n_items, 256, 0, st>>>(mean, items, dLdu, loss);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_loss_batch launch");
    return 0;
}

int launch_acc_to_f32(const double *acc, float *out, long long n, cudaStream_t st) {
    if (n == 0) return 0;
    const int B = 256;
    const int G = (int)std::min<long long>((n + B - 1) / B, 8192);
    k_acc_to_f32<<<G, B, 0, st>>>(acc, out, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "k_acc_to_f32 launch");
    return 0;
}

}  // namespace wosd
