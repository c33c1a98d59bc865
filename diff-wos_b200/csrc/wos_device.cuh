// Device-side scene view, geometry, nearest-primitive queries and samplers
// for the walk-on-spheres kernels (sm_100a).
//
// Arithmetic is written with explicit fmaf() and compiled with -fmad=false,
// so each function returns the same bits as the CPU oracle's restatement of
// the same reference function (cited per function).
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "wos_math.h"

namespace wosd {

// ------------------------------------------------------------------ status
// Bits of the device status word (OR-ed by kernels, read by the host).
enum StatusBits : int {
    ST_STACK_OVERFLOW = 1,   // BVH traversal stack ran out (result may be wrong)
    ST_BAD_PRIM       = 2,   // a query returned no primitive
    ST_NONFINITE      = 4,   // a walk produced a non-finite value
    ST_QUEUE_LIMIT    = 8,   // a persistent loop hit its iteration limit
};

// ------------------------------------------------------------------ layout
// Scene data in HBM.  Primitive data is precomputed once per scene:
//   2D segment f:   seg[f]  = (a.x, a.y, (b-a).x, (b-a).y), seginv[f] = 1/|b-a|^2
//   3D triangle f:  tri[3f] = (a.xyz, |ab|^2), tri[3f+1] = (ab.xyz, ab.ac),
//                   tri[3f+2] = (ac.xyz, |ac|^2)
// The LBVH (Karras, leaf size 1) is stored breadth-first; node k holds the
// boxes of both children and the two child references:
//   2D: node[3k] = (L.lo, L.hi), node[3k+1] = (R.lo, R.hi), node[3k+2].xy = refs
//   3D: node[4k..4k+2] = (L.lo.xyz, L.hi.xyz, R.lo.xyz, R.hi.xyz) packed,
//       node[4k+3].xy = refs
// A reference r >= 0 is an internal node, r < 0 is leaf ~r in Morton order;
// leaf data is copied into Morton order (lseg/lseginv/ltri) with the original
// primitive index in lorig.
struct SceneView {
    int dim, nV, nF;
    const float *V;    // nV x dim
    const int *F;      // nF x dim
    const float *N;    // vertex normals, nV x dim
    const float *g;    // Dirichlet values, nV
    const float4 *seg;
    const float *seginv;
    const float4 *tri;
    int nNodes;
    const float4 *node;
    const float4 *lseg;
    const float *lseginv;
    const float4 *ltri;
    const int *lorig;
    float lo[3], hi[3];
    float half_min_extent;  // min_k (hi_k - lo_k) / 2
    float max_extent;       // max_k (hi_k - lo_k)
    float centre[3];        // (lo + hi) / 2
    int src_type;
    float src[5];
    const float *cdf;  // G CDF table (n_cdf entries)
    int n_cdf;
    // guide[k] = first index l with cdf[l] > k / n_guide (k = 0..n_guide):
    // brackets the CDF search to a few entries
    const unsigned short *guide;
    int n_guide;
    // Wide tree for the warp-cooperative query: an implicit tree over the
    // Morton-ordered primitives.  Level 1 nodes are leaves, leaf i holding
    // primitives [WT_LEAF i, WT_LEAF i + WT_LEAF) (in Morton order); level k
    // node i bounds level k-1 nodes [32 i, 32 i + 32); level wt_levels has at
    // most 32 nodes.  Boxes: 2D one float4 (lo.x, lo.y, hi.x, hi.y) per node,
    // 3D two float4 (lo.xyz, w), (hi.xyz, 0); level k starts at
    // wt_box[wt_off[k]] (in nodes).  The queries bound a leaf by its oriented
    // box instead (wt_obb, built by k_wt_obb): principal axes u_k of its
    // vertices, a centre c and half-extents e_k with |u_k.(y - c)| <= e_k;
    // 2D two float4 (u0.xy, c.xy), (e0, e1, 0, 0) with u1 = (-u0.y, u0.x), 3D
    // three (u0, e0), (u1, e1), (c, e2) with u2 = u0 x u1.  A 3D level-2 node
    // also has a slab bound: unit normal n and [oc - oh, oc + oh] containing
    // n.(v - c) for every vertex v, c its box centre; wt_slab[i] = (n.xyz, oc)
    // with oh in the box's lo.w.  Any point y of the node is at least
    // |n.(x - c) - oc| - oh from x.
    int wt_levels;
    int wt_count[8];
    int wt_off[8];
    const float4 *wt_box;
    const float4 *wt_slab;
    const float4 *wt_obb;
};

constexpr int WT_MAX_LEVELS = 5;
// Primitives per leaf: one per lane.  (Leaves of 8 or 16 primitives, four or
// two tested per warp step, were measured slower on both the 2D and the 3D
// workloads: the extra pops cost more than the tighter leaves save.)
constexpr int WT_LEAF = 32;

template <int D>
struct NodeWords;
template <>
struct NodeWords<2> {
    static constexpr int K = 3;
};
template <>
struct NodeWords<3> {
    static constexpr int K = 4;
};

// ------------------------------------------------------------------ Philox
// Philox-4x32-10 (Salmon et al., SC 2011); counter = (point, walk, step, role).
struct Rng {
    uint32_t k0, k1;
};

__host__ __device__ inline Rng make_rng(uint64_t seed) {
    return Rng{(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5bd1e995u};
}

__device__ __forceinline__ uint4 philox(Rng key, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    uint32_t k0 = key.k0, k1 = key.k1;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return make_uint4(c0, c1, c2, c3);
}

enum { ROLE_PRIMAL = 0, ROLE_ANTI_A = 1, ROLE_ANTI_B = 2, ROLE_EXTRA = 3, ROLE_JITTER = 4, ROLE_BOUNDARY = 5 };

// ------------------------------------------------------------------ vectors
__device__ __forceinline__ float dot2(float ax, float ay, float bx, float by) { return fmaf(ax, bx, ay * by); }
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return fmaf(ax, bx, fmaf(ay, by, az * bz));
}
__device__ __forceinline__ void cross3(float ax, float ay, float az, float bx, float by, float bz, float &ox,
                                       float &oy, float &oz) {
    ox = ay * bz - az * by;
    oy = az * bx - ax * bz;
    oz = ax * by - ay * bx;
}

// ------------------------------------------------------------------ geometry
// Squared distance from p to a segment (include/util.cuh:108-114), with the
// clamped parameter h.
__device__ __forceinline__ float seg_d2(float4 s, float inv, float px, float py, float &h) {
    const float pax = px - s.x, pay = py - s.y;
    float t = dot2(pax, pay, s.z, s.w) * inv;
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    const float vx = fmaf(-s.z, t, pax), vy = fmaf(-s.w, t, pay);
    h = t;
    return dot2(vx, vy, vx, vy);
}

// Closest point on a triangle (include/util.cuh:22-106, Ericson's Voronoi
// regions), in terms of a, ab, ac and the precomputed dot products.
// Returns the squared distance; (v, w) weight b and c; (dx, dy, dz) = x - pt.
__device__ __forceinline__ float tri_closest(float4 t0, float4 t1, float4 t2, float x, float y, float z, float &v,
                                             float &w, float &dx, float &dy, float &dz) {
    const float axx = x - t0.x, axy = y - t0.y, axz = z - t0.z;
    const float ab2 = t0.w, abac = t1.w, ac2 = t2.w;
    const float d1 = dot3(t1.x, t1.y, t1.z, axx, axy, axz);
    const float d2 = dot3(t2.x, t2.y, t2.z, axx, axy, axz);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        v = 0.0f;
        w = 0.0f;
    } else {
        const float d3 = d1 - ab2, d4 = d2 - abac;
        if (d3 >= 0.0f && d4 <= d3) {
            v = 1.0f;
            w = 0.0f;
        } else {
            const float d5 = d1 - abac, d6 = d2 - ac2;
            if (d6 >= 0.0f && d5 <= d6) {
                v = 0.0f;
                w = 1.0f;
            } else {
                const float vc = d1 * d4 - d3 * d2;
                if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
                    v = d1 / (d1 - d3);
                    w = 0.0f;
                } else {
                    const float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
                        v = 0.0f;
                        w = d2 / (d2 - d6);
                    } else {
                        const float va = d3 * d6 - d5 * d4;
                        const float e43 = d4 - d3, e56 = d5 - d6;
                        if (va <= 0.0f && e43 >= 0.0f && e56 >= 0.0f) {
                            w = e43 / (e43 + e56);
                            v = 1.0f - w;
                        } else {
                            const float sum = va + vb + vc;
                            if (sum > 0.0f) {
                                const float denom = 1.0f / sum;
                                v = vb * denom;
                                w = vc * denom;
                            } else {
                                v = 0.0f;
                                w = 0.0f;
                            }
                        }
                    }
                }
            }
        }
    }
    dx = fmaf(-t2.x, w, fmaf(-t1.x, v, axx));
    dy = fmaf(-t2.y, w, fmaf(-t1.y, v, axy));
    dz = fmaf(-t2.z, w, fmaf(-t1.z, v, axz));
    return dot3(dx, dy, dz, dx, dy, dz);
}

// Squared distance to a triangle for warp-wide leaf tests: a branch-free
// form of tri_closest's region cascade.  Every region test is evaluated with
// the cascade's own expressions, the first region that holds
// picks the result, and the one division the edge and face regions need is
// issued once with the selected numerator and denominator.  Each value is the
// same IEEE operation on the same operands as in the cascade, so the results
// are identical to tri_closest's, but the lanes of a warp testing different
// triangles do not diverge (and run one division instead of up to four in
// turn).  Per-thread searches keep the cascade, which skips work per lane.
__device__ __forceinline__ float tri_d2_uniform(float4 t0, float4 t1, float4 t2, float x, float y, float z) {
    const float axx = x - t0.x, axy = y - t0.y, axz = z - t0.z;
    const float ab2 = t0.w, abac = t1.w, ac2 = t2.w;
    const float d1 = dot3(t1.x, t1.y, t1.z, axx, axy, axz);
    const float d2 = dot3(t2.x, t2.y, t2.z, axx, axy, axz);
    const float d3 = d1 - ab2, d4 = d2 - abac;
    const float d5 = d1 - abac, d6 = d2 - ac2;
    const float vc = d1 * d4 - d3 * d2;
    const float vb = d5 * d2 - d1 * d6;
    const float va = d3 * d6 - d5 * d4;
    const float e43 = d4 - d3, e56 = d5 - d6;
    const float sum = va + vb + vc;
    const bool rA = d1 <= 0.0f && d2 <= 0.0f;                  // vertex a
    const bool rB = d3 >= 0.0f && d4 <= d3;                    // vertex b
    const bool rC = d6 >= 0.0f && d5 <= d6;                    // vertex c
    const bool rAB = vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f;   // edge ab
    const bool rAC = vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f;   // edge ac
    const bool rBC = va <= 0.0f && e43 >= 0.0f && e56 >= 0.0f; // edge bc
    // numerator / denominator of the first edge region that holds, else the face
    float num = 1.0f, den = sum;
    if (rBC) {
        num = e43;
        den = e43 + e56;
    }
    if (rAC) {
        num = d2;
        den = d2 - d6;
    }
    if (rAB) {
        num = d1;
        den = d1 - d3;
    }
    const float q = num / den;
    float v = 0.0f, w = 0.0f;
    if (rA) {
    } else if (rB) {
        v = 1.0f;
    } else if (rC) {
        w = 1.0f;
    } else if (rAB) {
        v = q;
    } else if (rAC) {
        w = q;
    } else if (rBC) {
        w = q;
        v = 1.0f - q;
    } else if (sum > 0.0f) {
        v = vb * q;
        w = vc * q;
    }
    const float dx = fmaf(-t2.x, w, fmaf(-t1.x, v, axx));
    const float dy = fmaf(-t2.y, w, fmaf(-t1.y, v, axy));
    const float dz = fmaf(-t2.z, w, fmaf(-t1.z, v, axz));
    return dot3(dx, dy, dz, dx, dy, dz);
}

__device__ __forceinline__ float tri_d2(float4 t0, float4 t1, float4 t2, float x, float y, float z) {
    float v, w, dx, dy, dz;
    return tri_closest(t0, t1, t2, x, y, z, v, w, dx, dy, dz);
}

// ------------------------------------------------------------------ queries
struct Hit {
    int prim;
    float d2;
};

// Per-thread LBVH work counters: queries, node visits (two child boxes each),
// primitive distance evaluations.
struct Work {
    unsigned nq, nb, np;
};

// The same interface counting nothing: the query functions take either type,
// and the hot kernels run with NoWork unless work accounting is switched on
// (the counters' registers and adds cost 1-3 % of a step).
struct NoCount {
    __device__ __forceinline__ NoCount &operator+=(unsigned) { return *this; }
};
struct NoWork {
    NoCount nq, nb, np;
};

// Pruning slack (same rule as the oracle): a box is skipped only when its
// squared distance exceeds (1 + 2^-10) best + 1025 (s 2^-20)^2, where s
// bounds the coordinates' magnitude around the scene.
template <int D>
__device__ __forceinline__ float prune_tol2(const SceneView &S, const float *p) {
    float s = S.max_extent;
#pragma unroll
    for (int k = 0; k < D; ++k) s += fabsf(p[k] - S.centre[k]);
    const float e = s * 9.5367431640625e-07f;
    return 1025.0f * (e * e);
}
__device__ __forceinline__ float prune_bound(float best, float tol2) { return fmaf(best, 1.0009765625f, tol2); }

// Brute-force nearest over the original primitive order, ties to the lowest
// index (include/scene.cuh:102-128).
template <int D, class WK>
__device__ __forceinline__ Hit nearest_brute(const SceneView &S, const float *p, WK &wk) {
    Hit h{-1, INFINITY};
    wk.nq += 1;
    wk.np += (unsigned)S.nF;
    if (D == 2) {
        for (int f = 0; f < S.nF; ++f) {
            float t;
            const float d2 = seg_d2(__ldg(&S.seg[f]), __ldg(&S.seginv[f]), p[0], p[1], t);
            if (d2 < h.d2) {
                h.d2 = d2;
                h.prim = f;
            }
        }
    } else {
        for (int f = 0; f < S.nF; ++f) {
            const float d2 = tri_d2(__ldg(&S.tri[3 * f]), __ldg(&S.tri[3 * f + 1]), __ldg(&S.tri[3 * f + 2]), p[0],
                                    p[1], p[2]);
            if (d2 < h.d2) {
                h.d2 = d2;
                h.prim = f;
            }
        }
    }
    return h;
}

template <int D>
__device__ __forceinline__ float box_d2(const float *lo, const float *hi, const float *p) {
    float d[3];
#pragma unroll
    for (int k = 0; k < D; ++k) d[k] = fmaxf(fmaxf(lo[k] - p[k], p[k] - hi[k]), 0.0f);
    return D == 2 ? fmaf(d[0], d[0], d[1] * d[1]) : fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2]));
}

template <int D>
__device__ __forceinline__ void load_node(const float4 *base, int k, float (*lo)[3], float (*hi)[3], int &c0,
                                          int &c1) {
    if (D == 2) {
        const float4 a = base[3 * k], b = base[3 * k + 1], c = base[3 * k + 2];
        lo[0][0] = a.x;
        lo[0][1] = a.y;
        hi[0][0] = a.z;
        hi[0][1] = a.w;
        lo[1][0] = b.x;
        lo[1][1] = b.y;
        hi[1][0] = b.z;
        hi[1][1] = b.w;
        c0 = __float_as_int(c.x);
        c1 = __float_as_int(c.y);
    } else {
        const float4 a = base[4 * k], b = base[4 * k + 1], c = base[4 * k + 2], e = base[4 * k + 3];
        lo[0][0] = a.x;
        lo[0][1] = a.y;
        lo[0][2] = a.z;
        hi[0][0] = a.w;
        hi[0][1] = b.x;
        hi[0][2] = b.y;
        lo[1][0] = b.z;
        lo[1][1] = b.w;
        lo[1][2] = c.x;
        hi[1][0] = c.y;
        hi[1][1] = c.z;
        hi[1][2] = c.w;
        c0 = __float_as_int(e.x);
        c1 = __float_as_int(e.y);
    }
}

#ifndef WOS_STACK
#define WOS_STACK 64
#endif

// LBVH nearest: nearest-first descent with a per-thread stack, conservative
// pruning, ties to the lowest original index.  The first n_top nodes (the
// shallowest, breadth-first) are read from shared memory.
template <int D, class WK>
__device__ __forceinline__ Hit nearest_bvh(const SceneView &S, const float *p, const float4 *top, int n_top,
                                           int *status, WK &wk) {
    Hit h{-1, INFINITY};
    wk.nq += 1;
    if (S.nF == 1) {
        wk.np += 1;
        h.prim = 0;
        if (D == 2) {
            float t;
            h.d2 = seg_d2(__ldg(&S.seg[0]), __ldg(&S.seginv[0]), p[0], p[1], t);
        } else {
            h.d2 = tri_d2(__ldg(&S.tri[0]), __ldg(&S.tri[1]), __ldg(&S.tri[2]), p[0], p[1], p[2]);
        }
        return h;
    }
    const float tol2 = prune_tol2<D>(S, p);
    int stn[WOS_STACK];
    float std2[WOS_STACK];
    int sp = 1;
    stn[0] = 0;
    std2[0] = 0.0f;
    int best_leaf = -1;
    while (sp > 0) {
        --sp;
        const int v = stn[sp];
        if (std2[sp] > prune_bound(h.d2, tol2)) continue;
        wk.nb += 1;
        float lo[2][3], hi[2][3];
        int ch[2];
        if (v < n_top)
            load_node<D>(top, v, lo, hi, ch[0], ch[1]);
        else
            load_node<D>(S.node, v, lo, hi, ch[0], ch[1]);
        float bd[2];
        bd[0] = box_d2<D>(lo[0], hi[0], p);
        bd[1] = box_d2<D>(lo[1], hi[1], p);
        const int nr = bd[1] < bd[0] ? 1 : 0;
        const int cn = nr ? ch[1] : ch[0], cf = nr ? ch[0] : ch[1];
        const float dn = nr ? bd[1] : bd[0], df = nr ? bd[0] : bd[1];
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const int c = pass == 0 ? cn : cf;
            const float bdc = pass == 0 ? dn : df;
            if (c < 0 && bdc <= prune_bound(h.d2, tol2)) {
                const int leaf = ~c;
                wk.np += 1;
                float d2;
                if (D == 2) {
                    float t;
                    d2 = seg_d2(__ldg(&S.lseg[leaf]), __ldg(&S.lseginv[leaf]), p[0], p[1], t);
                } else {
                    d2 = tri_d2(__ldg(&S.ltri[3 * leaf]), __ldg(&S.ltri[3 * leaf + 1]), __ldg(&S.ltri[3 * leaf + 2]),
                                p[0], p[1], p[2]);
                }
                if (d2 <= h.d2) {
                    const int orig = __ldg(&S.lorig[leaf]);
                    if (d2 < h.d2 || orig < h.prim) {
                        h.d2 = d2;
                        h.prim = orig;
                        best_leaf = leaf;
                    }
                }
            }
        }
        if (cf >= 0 && df <= prune_bound(h.d2, tol2)) {
            if (sp < WOS_STACK) {
                stn[sp] = cf;
                std2[sp] = df;
                ++sp;
            } else {
                atomicOr(status, ST_STACK_OVERFLOW);
            }
        }
        if (cn >= 0 && dn <= prune_bound(h.d2, tol2)) {
            if (sp < WOS_STACK) {
                stn[sp] = cn;
                std2[sp] = dn;
                ++sp;
            } else {
                atomicOr(status, ST_STACK_OVERFLOW);
            }
        }
    }
    (void)best_leaf;
    return h;
}

// ------------------------------------------------------------------ wide tree
// Warp minimum of a non-negative float (or +inf): for such values the IEEE
// bit pattern orders like the value, so one redux.sync integer minimum does it.
__device__ __forceinline__ float warp_min(float v) {
    return __uint_as_float(__reduce_min_sync(0xffffffffu, __float_as_uint(v)));
}
__device__ __forceinline__ int warp_min_int(int v) { return __reduce_min_sync(0xffffffffu, v); }

// Frontier key of a lane: its child's distance with the low 5 mantissa bits
// replaced by the lane, so one redux.sync minimum gives both the nearest
// child and its lane.  The distance read back from a key (low bits cleared)
// is at most the true one, so pruning on it stays conservative; only the
// order of near-equal children (within 32 ulps) changes.
__device__ __forceinline__ unsigned frontier_key(float d, int lane) {
    return (__float_as_uint(d) & ~31u) | (unsigned)lane;
}
__device__ __forceinline__ float key_dist(unsigned k) { return __uint_as_float(k & ~31u); }
// A taken entry: the largest +inf key (a NaN pattern would never compare
// above the bound, so the loop could not end).
constexpr unsigned KEY_TAKEN = 0x7f80001fu;

template <int D>
__device__ __forceinline__ float wt_box_d2(const SceneView &S, int node, const float *q) {
    float lo[3], hi[3];
    if (D == 2) {
        const float4 b = __ldg(&S.wt_box[node]);
        lo[0] = b.x;
        lo[1] = b.y;
        hi[0] = b.z;
        hi[1] = b.w;
    } else {
        const float4 a = __ldg(&S.wt_box[2 * node]), b = __ldg(&S.wt_box[2 * node + 1]);
        lo[0] = a.x;
        lo[1] = a.y;
        lo[2] = a.z;
        hi[0] = b.x;
        hi[1] = b.y;
        hi[2] = b.z;
    }
    return box_d2<D>(lo, hi, q);
}

// Lower bound on the squared distance from q to leaf `leaf`: the distance to
// its oriented box, sum_k max(|u_k.(q - c)| - e_k, 0)^2, scaled by
// (1 - 2^-18).  With |u_k.(y - c)| <= e_k for every point y of the leaf and
// the axes' matrix of norm below 1, the exact value is at most |q - y|^2; the
// float roundings of q - c and of the dot products (relative 2^-22 of
// |q - c|) are covered by the 1e-6 |y - c| margin in e_k for the |y - c| part
// and by the final scale for the rest, so the result stays below |q - y|^2 --
// a bound as safe as the box distance, and tighter wherever a leaf's patch or
// arc is tilted against the axes.
template <int D>
__device__ __forceinline__ float leaf_obb_d2(const SceneView &S, int leaf, const float *q) {
    constexpr float SHRINK = 0.999996185302734375f;  // 1 - 2^-18
    if (D == 2) {
        const float4 a = __ldg(&S.wt_obb[2 * leaf]), e = __ldg(&S.wt_obb[2 * leaf + 1]);
        const float vx = q[0] - a.z, vy = q[1] - a.w;
        const float a0 = fmaxf(fabsf(dot2(a.x, a.y, vx, vy)) - e.x, 0.0f);
        const float a1 = fmaxf(fabsf(dot2(-a.y, a.x, vx, vy)) - e.y, 0.0f);
        return fmaf(a0, a0, a1 * a1) * SHRINK;
    }
    const float4 f0 = __ldg(&S.wt_obb[3 * leaf]), f1 = __ldg(&S.wt_obb[3 * leaf + 1]),
                 f2 = __ldg(&S.wt_obb[3 * leaf + 2]);
    float u2[3];
    cross3(f0.x, f0.y, f0.z, f1.x, f1.y, f1.z, u2[0], u2[1], u2[2]);
    const float vx = q[0] - f2.x, vy = q[1] - f2.y, vz = q[2] - f2.z;
    const float a0 = fmaxf(fabsf(dot3(f0.x, f0.y, f0.z, vx, vy, vz)) - f0.w, 0.0f);
    const float a1 = fmaxf(fabsf(dot3(f1.x, f1.y, f1.z, vx, vy, vz)) - f1.w, 0.0f);
    const float a2 = fmaxf(fabsf(dot3(u2[0], u2[1], u2[2], vx, vy, vz)) - f2.w, 0.0f);
    return fmaf(a0, a0, fmaf(a1, a1, a2 * a2)) * SHRINK;
}

// Lower bound on the squared distance from q to node `node` of level L: a
// leaf's oriented-box distance; for a 3D level-2 node (a patch of 1024
// triangles, whose box is loose wherever the surface is tilted against the
// axes) the larger of its box distance and its slab distance; otherwise the
// box distance.
template <int D, int L>
__device__ __forceinline__ float node_bound(const SceneView &S, int node, const float *q) {
    float lo[3], hi[3], n[3], c[3], oc, oh;
    if constexpr (L == 1) {
        return leaf_obb_d2<D>(S, node, q);
    } else if (D == 2 || L > 2) {
        return wt_box_d2<D>(S, S.wt_off[L] + node, q);
    } else {
        const int bi = S.wt_off[L] + node;
        const float4 a = __ldg(&S.wt_box[2 * bi]), b = __ldg(&S.wt_box[2 * bi + 1]);
        const float4 sl = __ldg(&S.wt_slab[node]);
        lo[0] = a.x;
        lo[1] = a.y;
        lo[2] = a.z;
        hi[0] = b.x;
        hi[1] = b.y;
        hi[2] = b.z;
        n[0] = sl.x;
        n[1] = sl.y;
        n[2] = sl.z;
        oc = sl.w;
        oh = a.w;
    }
    const float bd = box_d2<D>(lo, hi, q);
#pragma unroll
    for (int k = 0; k < D; ++k) c[k] = (lo[k] + hi[k]) * 0.5f;
    const float t = dot3(n[0], n[1], n[2], q[0] - c[0], q[1] - c[1], q[2] - c[2]);
    const float lb = fabsf(t - oc) - oh;
    return lb > 0.0f ? fmaxf(bd, lb * lb) : bd;
}

// Squared distance to the primitive at Morton position s.
template <int D>
__device__ __forceinline__ float leaf_d2(const SceneView &S, int s, const float *q) {
    if (D == 2) {
        float t;
        return seg_d2(__ldg(&S.lseg[s]), __ldg(&S.lseginv[s]), q[0], q[1], t);
    }
    return tri_d2_uniform(__ldg(&S.ltri[3 * s]), __ldg(&S.ltri[3 * s + 1]), __ldg(&S.ltri[3 * s + 2]), q[0], q[1],
                          q[2]);
}

// Squared distance to primitive f in the original order.
template <int D>
__device__ __forceinline__ float prim_d2(const SceneView &S, int f, const float *q) {
    if (D == 2) {
        float t;
        return seg_d2(__ldg(&S.seg[f]), __ldg(&S.seginv[f]), q[0], q[1], t);
    }
    return tri_d2(__ldg(&S.tri[3 * f]), __ldg(&S.tri[3 * f + 1]), __ldg(&S.tri[3 * f + 2]), q[0], q[1], q[2]);
}

// Pruning bound of the wide-tree descent, clamped to the largest float so
// that +inf frontier entries (no child) are never taken, even before a first
// candidate exists or when the query point is NaN or overflows.
__device__ __forceinline__ float wt_bound(float best, float tol2) { return fminf(prune_bound(best, tol2), FLT_MAX); }

// Warp-cooperative nearest primitive for one query point q (the same q in
// every lane; every lane returns the same Hit).  Best-first descent of the
// wide tree, one template instance per level: the level's frontier of up to
// 32 child distances is one register per lane, the nearest unexpanded child
// is a redux.sync minimum, and a node expansion is one coalesced load of 32
// boxes (leaf bounds at level 1) or 32 primitives.  `best` may hold a
// warm-start candidate (a real primitive with its distance); pruning is
// conservative, so the result is the exact minimum of (d2, primitive index)
// -- the same as the brute-force search.
template <int D, int L, class WK>
__device__ __forceinline__ void wdescend(const SceneView &S, const float *q, int first, float tol2, Hit &best,
                                         WK &wk) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int child = first + lane;
    float d = INFINITY;
    if (child < S.wt_count[L]) d = node_bound<D, L>(S, child, q);
    unsigned key = frontier_key(d, lane);
    wk.nb += 1;
    unsigned mk = __reduce_min_sync(FULL, key);
    for (;;) {
        if (key_dist(mk) > wt_bound(best.d2, tol2)) return;
        const int j = (int)(mk & 31u);
        if (lane == j) key = KEY_TAKEN;
        const int node = first + j;
        // the next frontier entry, reduced before this node's work (whose
        // pruning cannot change the frontier) so that its latency overlaps it
        mk = __reduce_min_sync(FULL, key);
        if constexpr (L == 1) {
            wk.np += 1;
            const int s = node * WT_LEAF + lane;
            float d2 = INFINITY;
            if (s < S.nF) d2 = leaf_d2<D>(S, s, q);
            const float m2 = warp_min(d2);
            if (m2 <= best.d2 && m2 < INFINITY) {
                const unsigned c2 = __ballot_sync(FULL, d2 == m2);
                int o = 0x7fffffff;
                if ((c2 >> lane) & 1u) o = __ldg(&S.lorig[s]);
                const int omin = (__popc(c2) == 1) ? __shfl_sync(FULL, o, __ffs(c2) - 1) : warp_min_int(o);
                if (m2 < best.d2 || omin < best.prim) {
                    best.d2 = m2;
                    best.prim = omin;
                }
            }
        } else {
            wdescend<D, L - 1>(S, q, node * 32, tol2, best, wk);
        }
    }
}

// WL > 0: the tree has exactly WL levels (a kernel compiled for one depth
// holds one descent, which keeps its code small); WL = 0: any depth.  tol2
// is prune_tol2<D>(S, q), passed in so that a warp can compute it for all its
// lanes' points at once.
template <int D, int WL = 0, class WK>
__device__ __forceinline__ Hit wquery_tol(const SceneView &S, const float *q, Hit best, float tol2, WK &wk) {
    wk.nq += 1;
    if constexpr (WL > 0) {
        wdescend<D, WL>(S, q, 0, tol2, best, wk);
        return best;
    }
    switch (S.wt_levels) {
        case 1: wdescend<D, 1>(S, q, 0, tol2, best, wk); break;
        case 2: wdescend<D, 2>(S, q, 0, tol2, best, wk); break;
        case 3: wdescend<D, 3>(S, q, 0, tol2, best, wk); break;
        case 4: wdescend<D, 4>(S, q, 0, tol2, best, wk); break;
        default: wdescend<D, 5>(S, q, 0, tol2, best, wk); break;
    }
    return best;
}

template <int D, int WL = 0, class WK>
__device__ __forceinline__ Hit wquery(const SceneView &S, const float *q, Hit best, WK &wk) {
    return wquery_tol<D, WL>(S, q, best, prune_tol2<D>(S, q), wk);
}

// ------------------------------------------------------------------ ball test
// One bisection step of the inscribed-ball search accepts the radius m when
// |d - m| <= 1e-5f for the nearest distance d from the candidate centre
// (wosm::ball_accepts).  Since fl(sqrtf(d2) - m) is non-decreasing in d2, the
// step rejects exactly when some primitive "blocks" the ball,
// sqrtf(d2) - m < -1e-5f, or when even the nearest distance is above
// m + 1e-5f; the caller rules the second case out with the ball's own
// primitive.  So a step needs no nearest search: it stops at the first
// blocking primitive.
__device__ __forceinline__ bool ball_blocks(float d2, float m) { return sqrtf(d2) - m < -1e-5f; }

template <int D, int L, class WK>
__device__ __forceinline__ bool wball_descend(const SceneView &S, const float *q, int first, float bound, float m,
                                              Hit &hit, WK &wk) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int child = first + lane;
    float d = INFINITY;
    if (child < S.wt_count[L]) d = node_bound<D, L>(S, child, q);
    unsigned key = frontier_key(d, lane);
    wk.nb += 1;
    unsigned mk = __reduce_min_sync(FULL, key);
    for (;;) {
        if (key_dist(mk) > bound) return false;
        const int j = (int)(mk & 31u);
        if (lane == j) key = KEY_TAKEN;
        const int node = first + j;
        mk = __reduce_min_sync(FULL, key);
        if constexpr (L == 1) {
            wk.np += 1;
            const int s = node * WT_LEAF + lane;
            float d2 = INFINITY;
            if (s < S.nF) d2 = leaf_d2<D>(S, s, q);
            const unsigned b = __ballot_sync(FULL, s < S.nF && ball_blocks(d2, m));
            if (b) {
                const int src = __ffs(b) - 1;
                int o = 0;
                if (lane == src) o = __ldg(&S.lorig[s]);
                hit.prim = __shfl_sync(FULL, o, src);
                hit.d2 = __shfl_sync(FULL, d2, src);
                return true;
            }
        } else {
            if (wball_descend<D, L - 1>(S, q, node * 32, bound, m, hit, wk)) return true;
        }
    }
}

// Warp-cooperative blocking-primitive search for a ball of radius m centred
// at q: returns true with a blocking primitive in `hit`, or false when no
// primitive blocks.  Boxes are pruned against m^2 with the nearest search's
// conservative tolerance, so no blocking primitive is missed.
__device__ __forceinline__ float wball_bound(float m, float tol2) {
    return wt_bound((m * m) * (1.0f + 0x1p-20f), tol2);
}

// wball with its pruning bound wball_bound(m, prune_tol2<D>(S, q)) passed in.
template <int D, int WL = 0, class WK>
__device__ __forceinline__ bool wball_b(const SceneView &S, const float *q, float bound, float m, Hit &hit, WK &wk) {
    wk.nq += 1;
    if constexpr (WL > 0) return wball_descend<D, WL>(S, q, 0, bound, m, hit, wk);
    switch (S.wt_levels) {
        case 1: return wball_descend<D, 1>(S, q, 0, bound, m, hit, wk);
        case 2: return wball_descend<D, 2>(S, q, 0, bound, m, hit, wk);
        case 3: return wball_descend<D, 3>(S, q, 0, bound, m, hit, wk);
        case 4: return wball_descend<D, 4>(S, q, 0, bound, m, hit, wk);
        default: return wball_descend<D, 5>(S, q, 0, bound, m, hit, wk);
    }
}

template <int D, int WL = 0, class WK>
__device__ __forceinline__ bool wball(const SceneView &S, const float *q, float m, Hit &hit, WK &wk) {
    return wball_b<D, WL>(S, q, wball_bound(m, prune_tol2<D>(S, q)), m, hit, wk);
}

// ------------------------------------------------------------------ records
// Closest-point record at x for primitive prim (include/scene.cuh:180-223).
struct Rec {
    float p[3];
    float n[3];
    float t0, t1;  // 2D: (h, 0); 3D: (w_b, w_c)
    bool flip;     // the normal was negated to face the query point
};

// Per-walk boundary record stored by the forward pass for the adjoint:
// code = -1 (invalid walk) or prim | (flip << 30); t0, t1 as float bits.
struct WalkRec {
    int code;
    float t0, t1;
};
__host__ __device__ constexpr int walkrec_words(int D) { return D == 2 ? 2 : 4; }

template <int D>
__device__ __forceinline__ Rec closest_record(const SceneView &S, const float *x, int prim) {
    Rec r;
    if (D == 2) {
        const float4 s = __ldg(&S.seg[prim]);
        float h;
        seg_d2(s, __ldg(&S.seginv[prim]), x[0], x[1], h);
        const float pax = x[0] - s.x, pay = x[1] - s.y;
        r.p[0] = fmaf(s.z, h, s.x);
        r.p[1] = fmaf(s.w, h, s.y);
        float nx = s.w, ny = -s.z;
        const float len = sqrtf(dot2(nx, ny, nx, ny));
        nx = nx / len;
        ny = ny / len;
        r.flip = !(dot2(nx, ny, pax, pay) > 0.0f);
        if (r.flip) {
            nx = -nx;
            ny = -ny;
        }
        r.n[0] = nx;
        r.n[1] = ny;
        r.n[2] = 0.0f;
        r.p[2] = 0.0f;
        r.t0 = h;
        r.t1 = 0.0f;
    } else {
        const float4 t0 = __ldg(&S.tri[3 * prim]), t1 = __ldg(&S.tri[3 * prim + 1]), t2 = __ldg(&S.tri[3 * prim + 2]);
        float v, w, dx, dy, dz;
        tri_closest(t0, t1, t2, x[0], x[1], x[2], v, w, dx, dy, dz);
        r.p[0] = fmaf(t2.x, w, fmaf(t1.x, v, t0.x));
        r.p[1] = fmaf(t2.y, w, fmaf(t1.y, v, t0.y));
        r.p[2] = fmaf(t2.z, w, fmaf(t1.z, v, t0.z));
        float nx, ny, nz;
        cross3(t1.x, t1.y, t1.z, t2.x, t2.y, t2.z, nx, ny, nz);
        const float len = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
        nx = nx / len;
        ny = ny / len;
        nz = nz / len;
        const float axx = x[0] - t0.x, axy = x[1] - t0.y, axz = x[2] - t0.z;
        r.flip = !(dot3(nx, ny, nz, axx, axy, axz) > 0.0f);
        const float sg = r.flip ? -1.0f : 1.0f;
        r.n[0] = sg * nx;
        r.n[1] = sg * ny;
        r.n[2] = sg * nz;
        r.t0 = v;
        r.t1 = w;
    }
    return r;
}

// The record of closest_record() rebuilt from (prim, t0, t1, flip): the same
// operations on the same inputs, so the same bits.
template <int D>
__device__ __forceinline__ Rec record_from(const SceneView &S, int prim, float t0, float t1, bool flip) {
    Rec r;
    r.flip = flip;
    r.t0 = t0;
    r.t1 = t1;
    if (D == 2) {
        const float4 s = __ldg(&S.seg[prim]);
        r.p[0] = fmaf(s.z, t0, s.x);
        r.p[1] = fmaf(s.w, t0, s.y);
        r.p[2] = 0.0f;
        float nx = s.w, ny = -s.z;
        const float len = sqrtf(dot2(nx, ny, nx, ny));
        nx = nx / len;
        ny = ny / len;
        r.n[0] = flip ? -nx : nx;
        r.n[1] = flip ? -ny : ny;
        r.n[2] = 0.0f;
    } else {
        const float4 a = __ldg(&S.tri[3 * prim]), b = __ldg(&S.tri[3 * prim + 1]), c = __ldg(&S.tri[3 * prim + 2]);
        r.p[0] = fmaf(c.x, t1, fmaf(b.x, t0, a.x));
        r.p[1] = fmaf(c.y, t1, fmaf(b.y, t0, a.y));
        r.p[2] = fmaf(c.z, t1, fmaf(b.z, t0, a.z));
        float nx, ny, nz;
        cross3(b.x, b.y, b.z, c.x, c.y, c.z, nx, ny, nz);
        const float len = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
        const float sg = flip ? -1.0f : 1.0f;
        r.n[0] = sg * (nx / len);
        r.n[1] = sg * (ny / len);
        r.n[2] = sg * (nz / len);
    }
    return r;
}

// Signed distance and inside test (same composition as the oracle:
// include/scene.cuh:148-178 with wos/scene.py:325-339 and
// wos/scene3d.py:201-214).
template <int D>
__device__ __forceinline__ bool inside_test(const SceneView &S, const float *p, const Hit &hit, float *sd) {
    if (hit.prim < 0) {
        if (sd) *sd = INFINITY;
        return false;
    }
    const float d = sqrtf(hit.d2);
    if (D == 2) {
        const float4 s = __ldg(&S.seg[hit.prim]);
        float h;
        seg_d2(s, __ldg(&S.seginv[hit.prim]), p[0], p[1], h);
        const float pax = p[0] - s.x, pay = p[1] - s.y;
        const float vx = fmaf(-s.z, h, pax), vy = fmaf(-s.w, h, pay);
        const int ia = __ldg(&S.F[2 * hit.prim]), ib = __ldg(&S.F[2 * hit.prim + 1]);
        const float nax = __ldg(&S.N[2 * ia]), nay = __ldg(&S.N[2 * ia + 1]);
        const float nbx = __ldg(&S.N[2 * ib]), nby = __ldg(&S.N[2 * ib + 1]);
        const float nx = fmaf(nbx - nax, h, nax), ny = fmaf(nby - nay, h, nay);
        const float s2 = dot2(nx, ny, vx, vy);
        if (sd) *sd = s2 > 0.0f ? d : -d;
        return (s2 < 0.0f) && (hit.d2 > 0.0f);
    } else {
        const float4 t0 = __ldg(&S.tri[3 * hit.prim]), t1 = __ldg(&S.tri[3 * hit.prim + 1]),
                     t2 = __ldg(&S.tri[3 * hit.prim + 2]);
        float v, w, dx, dy, dz;
        tri_closest(t0, t1, t2, p[0], p[1], p[2], v, w, dx, dy, dz);
        float fx, fy, fz;
        cross3(t1.x, t1.y, t1.z, t2.x, t2.y, t2.z, fx, fy, fz);
        const float sf = dot3(fx, fy, fz, dx, dy, dz);
        const int ia = __ldg(&S.F[3 * hit.prim]), ib = __ldg(&S.F[3 * hit.prim + 1]),
                  ic = __ldg(&S.F[3 * hit.prim + 2]);
        const float w0 = (1.0f - v) - w;
        float nv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            nv[k] = fmaf(__ldg(&S.N[3 * ia + k]), w0, fmaf(__ldg(&S.N[3 * ib + k]), v, __ldg(&S.N[3 * ic + k]) * w));
        const float sv = dot3(nv[0], nv[1], nv[2], dx, dy, dz);
        if (sd) *sd = sf > 0.0f ? d : -d;
        return (hit.d2 > 0.0f) && (sv < 0.0f) && (sf <= 0.0f);
    }
}

// Dirichlet value (include/scene.cuh:251-264) and the vertex weights.
template <int D>
__device__ __forceinline__ float dirichlet(const SceneView &S, int prim, float t0, float t1, int *vid, float *wts) {
    if (D == 2) {
        const int ia = __ldg(&S.F[2 * prim]), ib = __ldg(&S.F[2 * prim + 1]);
        const float va = __ldg(&S.g[ia]), vb = __ldg(&S.g[ib]);
        if (vid) {
            vid[0] = ia;
            vid[1] = ib;
            wts[0] = 1.0f - t0;
            wts[1] = t0;
        }
        return fmaf(t0, vb - va, va);
    } else {
        const int ia = __ldg(&S.F[3 * prim]), ib = __ldg(&S.F[3 * prim + 1]), ic = __ldg(&S.F[3 * prim + 2]);
        const float va = __ldg(&S.g[ia]), vb = __ldg(&S.g[ib]), vc = __ldg(&S.g[ic]);
        const float w0 = (1.0f - t0) - t1;
        if (vid) {
            vid[0] = ia;
            vid[1] = ib;
            vid[2] = ic;
            wts[0] = w0;
            wts[1] = t0;
            wts[2] = t1;
        }
        return fmaf(va, w0, fmaf(vb, t0, vc * t1));
    }
}

// Source function and its parameter derivatives (include/scene.cuh:278-301).
__device__ __forceinline__ float source(const SceneView &S, float x, float y, float *df) {
    const float *q = S.src;
    if (S.src_type == 1) {
        const float tx = x - q[0], ty = y - q[1];
        const float sx2 = q[2] * q[2], sy2 = q[3] * q[3];
        const float dx = tx * tx / (2.0f * sx2);
        const float dy = ty * ty / (2.0f * sy2);
        const float E = wosm::exp_(-dx - dy);
        const float f = q[4] * E;
        if (df) {
            df[0] = f * (tx / sx2);
            df[1] = f * (ty / sy2);
            df[2] = f * (tx * tx / (sx2 * q[2]));
            df[3] = f * (ty * ty / (sy2 * q[3]));
            df[4] = E;
        }
        return f;
    }
    if (S.src_type == 2) {
        const float phi = fmaf(q[0], x, fmaf(q[1], y, q[2]));
        const float s = wosm::sin_(phi);
        if (df) {
            const float c = wosm::cos_(phi);
            df[0] = q[3] * c * x;
            df[1] = q[3] * c * y;
            df[2] = q[3] * c;
            df[3] = s;
            df[4] = 1.0f;
        }
        return fmaf(q[3], s, q[4]);
    }
    if (df) {
#pragma unroll
        for (int k = 0; k < 5; ++k) df[k] = 0.0f;
    }
    return 0.0f;
}

// Radius sample from the G CDF (include/wos.cuh:49-75).  The guide table
// (usually in shared memory) brackets the search; the bracket is checked and
// widened when it does not hold, so the result is always the first l with
// u < cdf[l], as a search over the whole table gives.
__device__ __forceinline__ float sample_G_radius(const float *cdf, int n, const unsigned short *guide, int ng,
                                                 float u, float R, float &pdf) {
    int k = (int)(u * (float)ng);
    k = min(max(k, 0), ng - 1);
    int l = guide[k], r = guide[k + 1];
    if (l > 0 && !(u >= __ldg(&cdf[l - 1]))) l = 0;
    if (!(u < __ldg(&cdf[r]))) r = n - 1;
    while (l < r) {
        const int mid = (l + r) >> 1;
        if (u < __ldg(&cdf[mid]))
            r = mid;
        else
            l = mid + 1;
    }
    const float pmf = l == 0 ? __ldg(&cdf[0]) : __ldg(&cdf[l]) - __ldg(&cdf[l - 1]);
    const float prev = l == 0 ? 0.0f : __ldg(&cdf[l - 1]);
    u = (u - prev) / pmf;
    pdf = pmf * (float)n / R;
    return R * ((float)l + u) / (float)n;
}

// Interior source term of one step (include/wos.cuh:115-139 with the
// importance-sampled branch of :121-130): returns the factor K with
// contrib += f(y) * K, and y.
__device__ __forceinline__ float source_step(const SceneView &S, const unsigned short *guide, bool use_IS, float px,
                                             float py, float d, uint32_t ra, uint32_t rb, float &yx, float &yy) {
    float dx, dy, pdf, weight;
    if (use_IS) {
        const float rad = sample_G_radius(S.cdf, S.n_cdf, guide, S.n_guide, wosm::u01(ra), d, pdf);
        float s, c;
        wosm::sincos_2pi(wosm::u01(rb), &s, &c);
        pdf = pdf / wosm::kTwoPi;
        dx = rad * c;
        dy = rad * s;
        weight = sqrtf(dot2(dx, dy, dx, dy));
    } else {
        float s, c;
        wosm::sincos_2pi(wosm::u01(ra), &s, &c);
        const float rr = sqrtf(wosm::u01(rb));
        dx = rr * c * d;
        dy = rr * s * d;
        pdf = 1.0f / (wosm::kPi * d * d);
        weight = 1.0f;
    }
    const float rn = sqrtf(dot2(dx, dy, dx, dy));
    const float G = wosm::log_(d / fmaxf(rn, 1e-4f)) * wosm::kInv2Pi;
    yx = px + dx;
    yy = py + dy;
    return pdf > 1e-5f ? G * weight / pdf : 0.0f;
}

}  // namespace wosd
