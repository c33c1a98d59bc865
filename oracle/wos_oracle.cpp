// CPU oracle for the walk-on-spheres hot path of diff-wos.
//
// TEST INFRASTRUCTURE ONLY.  This file is a C++17 restatement of the
// reference algorithm, used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker and the timed CPU baseline.
// The product (diff-wos_b200/) never links, loads or calls it.
//
// It follows, function by function (paths relative to the reference repo):
//   walk                  include/wos.cuh:97-145      (WoSDevice<N>::walk)
//   u()                   include/wos.cuh:90-95
//   uniform sphere/ball   include/wos.cuh:14-42
//   Green's fn / G-IS     include/wos.cuh:44-88, wos/wos_with_source.py:17-54
//   brute nearest         include/scene.cuh:102-128
//   sdf                   include/scene.cuh:148-178, wos/scene.py:325-339,
//                         wos/scene3d.py:201-214
//   closestPoint          include/scene.cuh:180-223
//   largestInscribedBall  include/scene.cuh:225-249
//   dirichlet             include/scene.cuh:251-264, wos/scene.py:353-357
//   source_function       include/scene.cuh:278-301
//   vertex normals        include/scene.cuh:368-409
//   scene AABB            include/scene.cuh:428-435
//   point-triangle        include/util.cuh:22-106 (Ericson, Real-Time
//                         Collision Detection, sec. 5.1.5)
//   normal derivative     wos/wos.py:59-107 (2D), wos/wos_with_source.py:
//                         154-232 (2D with source), wos/wos3d.py:97-135 (3D)
//   tangent derivative    wos/scene.py:451-460, wos/wos3d.py:137-156
//   boundary-shape term   wos/wos_grad.py:113-151 (OursCUDA), :57-86 (Ours),
//                         wos/wos_grad_3d.py:104-137 (Ours3D)
//   image boundary term   wos/wos_boundary.py:11-31 with sample_boundary,
//                         wos/scene.py:435-449, wos/scene3d.py:241-262
//   get_point / AD glue   wos/scene.py:416-433, wos/scene3d.py:225-239,
//                         wos/solver.py:49-65, 90-125
//   LBVH                  Karras, "Maximizing parallelism in the construction
//                         of BVHs, octrees and k-d trees", HPG 2012 (the
//                         reference uses the third-party lbvh library, whose
//                         source is not vendored; scene.cuh:130-146, 452).
//
// Deliberate, documented differences from the reference (same in the CUDA
// path): counter-based Philox-4x32-10 per (point, walk, step, role) instead
// of PCG32 streams; own sin/cos/log/exp polynomials (wos_math.h) so CPU and
// GPU agree bit for bit; nearest search compares squared distances (ties to
// the lowest primitive index); zero-length segments get h = 0.
//
// Parity pins: the reference ships no golden vectors.  The oracle is pinned
// by analytic harmonic / Poisson solutions, the reference's Green's-function
// CDF table, and the reference's point-triangle routine run on a numpy shim
// (tests/golden/).
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -mfma -fopenmp).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <omp.h>

#include "../diff-wos_b200/csrc/wos_math.h"

using wosm::fabs_;

namespace orc {

// ---------------------------------------------------------------- Philox
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011).
struct U4 {
    uint32_t x, y, z, w;
};

static inline U4 philox(uint32_t k0, uint32_t k1, U4 c) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

struct Rng {
    uint32_t k0, k1;
    U4 draw(uint32_t pt, uint32_t walk, uint32_t step, uint32_t role) const {
        return philox(k0, k1, U4{pt, walk, step, role});
    }
};

static inline Rng make_rng(uint64_t seed) {
    return Rng{(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x5bd1e995u};
}

// ---------------------------------------------------------------- params
// Must match wos_params in include/wos_b200.h.
struct Params {
    int32_t nwalks;
    int32_t nsteps;
    float epsilon;
    int32_t double_sided;
    int32_t prevent_fd_artifacts;
    int32_t use_IS_for_greens;
    int32_t include_source;
    int32_t project_unterminated;
    int32_t use_bvh;
    uint32_t walk_offset;
    uint64_t seed;
    float jitter[3];
};

// Must match wos_adjoint_params in include/wos_b200.h.
struct AdjParams {
    float epsilon2;
    float clamping;
    int32_t control_variates;
    int32_t source_in_normal_derivative;
    float ball_epsilon;
    int32_t want_dV;
    int32_t want_dg;
    int32_t want_dsrc;
};

enum { ROLE_PRIMAL = 0, ROLE_ANTI_A = 1, ROLE_ANTI_B = 2, ROLE_EXTRA = 3, ROLE_JITTER = 4 };

// ---------------------------------------------------------------- scene
struct Node {
    int child[2];  // >= 0 internal node, < 0: ~sorted leaf position
    float lo[2][3], hi[2][3];
};

struct Scene {
    int D;
    int nV, nF;
    std::vector<float> V, N, g;
    std::vector<int> F;
    int src_type;
    float src[5];
    float lo[3], hi[3];
    // LBVH
    std::vector<uint64_t> keys;  // sorted (morton << 32 | prim)
    std::vector<Node> nodes;
    std::vector<float> plo, phi;  // primitive boxes
    // G CDF
    std::vector<float> cdf;
};

static inline float dot2(const float *a, const float *b) { return fmaf(a[0], b[0], a[1] * b[1]); }
static inline float dot3(const float *a, const float *b) {
    return fmaf(a[0], b[0], fmaf(a[1], b[1], a[2] * b[2]));
}
static inline void cross3(const float *a, const float *b, float *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// Normalised CDF of pmf_i ~ r_i log(1/r_i), r_i = (i + 0.5)/n
// (include/tabulated_G_cdf.cuh:5-8, wos/wos_with_source.py:17-23).
static void build_cdf(std::vector<float> &cdf, int n) {
    std::vector<double> pmf(n);
    double total = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = (i + 0.5) / n;
        pmf[i] = r * std::log(1.0 / r) / (2.0 * 3.14159265358979323846);
        total += pmf[i];
    }
    cdf.resize(n);
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        acc += pmf[i];
        cdf[i] = (float)(acc / total);
    }
    cdf[n - 1] = 1.0f;
}

// Vertex normals (include/scene.cuh:368-409): 2D normalised sum of the two
// adjacent edge normals; 3D angle-weighted face normals.  Contributions are
// summed per vertex in face order, then slot order.
static void build_normals(Scene &S) {
    const int D = S.D;
    S.N.assign((size_t)S.nV * D, 0.0f);
    for (int f = 0; f < S.nF; ++f) {
        const int *I = &S.F[(size_t)f * D];
        if (D == 2) {
            const float *p0 = &S.V[2 * I[0]], *p1 = &S.V[2 * I[1]];
            float d[2] = {p1[0] - p0[0], p1[1] - p0[1]};
            float n[2] = {d[1], -d[0]};
            const float len = sqrtf(dot2(n, n));
            if (len > 0.0f) {
                n[0] = n[0] / len;
                n[1] = n[1] / len;
            } else {
                n[0] = n[1] = 0.0f;
            }
            for (int s = 0; s < 2; ++s) {
                S.N[2 * I[s]] += n[0];
                S.N[2 * I[s] + 1] += n[1];
            }
        } else {
            const float *p0 = &S.V[3 * I[0]], *p1 = &S.V[3 * I[1]], *p2 = &S.V[3 * I[2]];
            float e10[3], e20[3], e21[3], e01[3], e02[3], e12[3];
            for (int k = 0; k < 3; ++k) {
                e10[k] = p1[k] - p0[k];
                e20[k] = p2[k] - p0[k];
                e21[k] = p2[k] - p1[k];
                e01[k] = p0[k] - p1[k];
                e02[k] = p0[k] - p2[k];
                e12[k] = p1[k] - p2[k];
            }
            float n[3];
            cross3(e10, e20, n);
            const float len = sqrtf(dot3(n, n));
            if (len > 0.0f) {
                for (int k = 0; k < 3; ++k) n[k] = n[k] / len;
            } else {
                n[0] = n[1] = n[2] = 0.0f;
            }
            auto angle = [](const float *a, const float *b) {
                float c[3];
                cross3(a, b, c);
                return wosm::atan2_(sqrtf(dot3(c, c)), dot3(a, b));
            };
            const float ang[3] = {angle(e10, e20), angle(e21, e01), angle(e02, e12)};
            for (int s = 0; s < 3; ++s)
                for (int k = 0; k < 3; ++k) S.N[3 * I[s] + k] += ang[s] * n[k];
        }
    }
    for (int v = 0; v < S.nV; ++v) {
        float *n = &S.N[(size_t)v * D];
        const float len = sqrtf(D == 2 ? dot2(n, n) : dot3(n, n));
        for (int k = 0; k < D; ++k) n[k] = len > 0.0f ? n[k] / len : 0.0f;
    }
}

// ---------------------------------------------------------------- LBVH
static inline uint32_t spread2(uint32_t x) {  // 16 bits -> even bits
    x &= 0xffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
static inline uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

static void prim_box(const Scene &S, int f, float *lo, float *hi) {
    const int D = S.D;
    const int *I = &S.F[(size_t)f * D];
    for (int k = 0; k < D; ++k) {
        float a = S.V[(size_t)I[0] * D + k], b = S.V[(size_t)I[1] * D + k];
        lo[k] = fminf(a, b);
        hi[k] = fmaxf(a, b);
        if (D == 3) {
            float c = S.V[(size_t)I[2] * D + k];
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    }
}

static int delta(const std::vector<uint64_t> &k, int i, int j) {
    const int n = (int)k.size();
    if (j < 0 || j >= n) return -1;
    return __builtin_clzll(k[i] ^ k[j]);  // keys are unique
}

static void build_bvh(Scene &S) {
    const int D = S.D, n = S.nF;
    S.plo.resize((size_t)n * D);
    S.phi.resize((size_t)n * D);
    for (int f = 0; f < n; ++f) prim_box(S, f, &S.plo[(size_t)f * D], &S.phi[(size_t)f * D]);
    S.keys.resize(n);
    for (int f = 0; f < n; ++f) {
        uint32_t q[3];
        const float scale = D == 2 ? 65536.0f : 1024.0f;
        for (int k = 0; k < D; ++k) {
            const float c = (S.plo[(size_t)f * D + k] + S.phi[(size_t)f * D + k]) * 0.5f;
            const float ext = S.hi[k] - S.lo[k];
            const float u = ext > 0.0f ? (c - S.lo[k]) / ext : 0.0f;
            q[k] = (uint32_t)fminf(fmaxf(u * scale, 0.0f), scale - 1.0f);
        }
        const uint32_t m = D == 2 ? (spread2(q[0]) | (spread2(q[1]) << 1))
                                  : (spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2));
        S.keys[f] = ((uint64_t)m << 32) | (uint32_t)f;
    }
    std::sort(S.keys.begin(), S.keys.end());
    S.nodes.clear();
    if (n < 2) return;
    S.nodes.resize(n - 1);
    std::vector<int> parent_internal(n - 1, -1), parent_leaf(n, -1);
    for (int i = 0; i < n - 1; ++i) {
        const int d = (delta(S.keys, i, i + 1) - delta(S.keys, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(S.keys, i, i - d);
        int lmax = 2;
        while (delta(S.keys, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (delta(S.keys, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(S.keys, i, j);
        int s = 0;
        for (int div = 2;; div *= 2) {
            const int t = (l + div - 1) / div;
            if (delta(S.keys, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int gamma = i + s * d + std::min(d, 0);
        Node &nd = S.nodes[i];
        nd.child[0] = (std::min(i, j) == gamma) ? ~gamma : gamma;
        nd.child[1] = (std::max(i, j) == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    }
    // child boxes, post-order
    std::vector<float> nlo((size_t)(n - 1) * D), nhi((size_t)(n - 1) * D);
    std::vector<int> order;
    order.reserve(n - 1);
    std::vector<int> st{0};
    while (!st.empty()) {
        int v = st.back();
        st.pop_back();
        order.push_back(v);
        for (int c = 0; c < 2; ++c)
            if (S.nodes[v].child[c] >= 0) st.push_back(S.nodes[v].child[c]);
    }
    for (int oi = (int)order.size() - 1; oi >= 0; --oi) {
        const int v = order[oi];
        Node &nd = S.nodes[v];
        for (int c = 0; c < 2; ++c) {
            const int ch = nd.child[c];
            for (int k = 0; k < D; ++k) {
                if (ch < 0) {
                    const int prim = (int)(uint32_t)S.keys[~ch];
                    nd.lo[c][k] = S.plo[(size_t)prim * D + k];
                    nd.hi[c][k] = S.phi[(size_t)prim * D + k];
                } else {
                    nd.lo[c][k] = nlo[(size_t)ch * D + k];
                    nd.hi[c][k] = nhi[(size_t)ch * D + k];
                }
            }
        }
        for (int k = 0; k < D; ++k) {
            nlo[(size_t)v * D + k] = fminf(nd.lo[0][k], nd.lo[1][k]);
            nhi[(size_t)v * D + k] = fmaxf(nd.hi[0][k], nd.hi[1][k]);
        }
    }
}

// ---------------------------------------------------------------- geometry
// Squared distance to segment f; h = clamped projection parameter.
static inline float seg_d2(const Scene &S, int f, const float *p, float *h_out) {
    const int *I = &S.F[(size_t)f * 2];
    const float *a = &S.V[2 * I[0]], *b = &S.V[2 * I[1]];
    const float ba[2] = {b[0] - a[0], b[1] - a[1]};
    const float pa[2] = {p[0] - a[0], p[1] - a[1]};
    const float len2 = dot2(ba, ba);
    const float inv = len2 > 0.0f ? 1.0f / len2 : 0.0f;
    float h = dot2(pa, ba) * inv;
    h = fminf(fmaxf(h, 0.0f), 1.0f);
    const float v[2] = {fmaf(-ba[0], h, pa[0]), fmaf(-ba[1], h, pa[1])};
    if (h_out) *h_out = h;
    return dot2(v, v);
}

// Closest point on triangle f (Ericson's Voronoi-region walk), written with
// the precomputed products |ab|^2, ab.ac, |ac|^2.  Returns squared distance;
// (v, w) are the barycentric weights of b and c; diff = x - closest point.
static inline float tri_closest_raw(const float *a, const float *b, const float *c, const float *x, float *v_out,
                                    float *w_out, float *diff) {
    float ab[3], ac[3], ax[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        ac[k] = c[k] - a[k];
        ax[k] = x[k] - a[k];
    }
    const float ab2 = dot3(ab, ab), abac = dot3(ab, ac), ac2 = dot3(ac, ac);
    float v, w;
    const float d1 = dot3(ab, ax), d2 = dot3(ac, ax);
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
    float dd[3];
    for (int k = 0; k < 3; ++k) dd[k] = fmaf(-ac[k], w, fmaf(-ab[k], v, ax[k]));
    if (v_out) *v_out = v;
    if (w_out) *w_out = w;
    if (diff)
        for (int k = 0; k < 3; ++k) diff[k] = dd[k];
    return dot3(dd, dd);
}

static inline float tri_closest(const Scene &S, int f, const float *x, float *v_out, float *w_out, float *diff) {
    const int *I = &S.F[(size_t)f * 3];
    return tri_closest_raw(&S.V[3 * I[0]], &S.V[3 * I[1]], &S.V[3 * I[2]], x, v_out, w_out, diff);
}

static inline float prim_d2(const Scene &S, int f, const float *p) {
    return S.D == 2 ? seg_d2(S, f, p, nullptr) : tri_closest(S, f, p, nullptr, nullptr, nullptr);
}

struct Hit {
    int prim;
    float d2;
};

// Brute-force nearest primitive, lowest index on ties
// (include/scene.cuh:102-128).
static Hit nearest_brute(const Scene &S, const float *p) {
    Hit h{-1, INFINITY};
    for (int f = 0; f < S.nF; ++f) {
        const float d2 = prim_d2(S, f, p);
        if (d2 < h.d2) {
            h.d2 = d2;
            h.prim = f;
        }
    }
    return h;
}

static inline float box_d2(const float *lo, const float *hi, const float *p, int D) {
    float d[3];
    for (int k = 0; k < D; ++k) d[k] = fmaxf(fmaxf(lo[k] - p[k], p[k] - hi[k]), 0.0f);
    return D == 2 ? fmaf(d[0], d[0], d[1] * d[1]) : fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2]));
}

// Pruning slack: a box is skipped only when its distance exceeds the best
// primitive distance by more than the float rounding either can carry.
static inline float prune_tol2(const Scene &S, const float *p) {
    float s = 0.0f;
    for (int k = 0; k < S.D; ++k) {
        s = fmaxf(s, S.hi[k] - S.lo[k]);
    }
    for (int k = 0; k < S.D; ++k) s += fabsf(p[k] - (S.lo[k] + S.hi[k]) * 0.5f);
    const float e = s * 9.5367431640625e-07f;  // 2^-20
    return 1025.0f * (e * e);
}
static inline float prune_bound(float best, float tol2) { return fmaf(best, 1.0009765625f, tol2); }

// Per-thread traversal counters (node visits, primitive tests, queries) for
// the algorithmic-work figures of the benchmark.
static thread_local long long t_nbox = 0, t_nprim = 0, t_nquery = 0;

// LBVH nearest (replaces lbvh::query_device, include/scene.cuh:130-146):
// nearest-first descent, conservative pruning, ties to the lowest index.
static Hit nearest_bvh(const Scene &S, const float *p, int *nbox, int *nprim) {
    Hit h{-1, INFINITY};
    int cb = 0, cp = 0;
    if (S.nF == 1) {
        h.prim = 0;
        h.d2 = prim_d2(S, 0, p);
        cp = 1;
    } else if (S.nF > 1) {
        const float tol2 = prune_tol2(S, p);
        int stn[96];
        float std2[96];
        int sp = 0;
        stn[sp] = 0;
        std2[sp] = 0.0f;
        ++sp;
        auto test = [&](int leaf) {
            const int prim = (int)(uint32_t)S.keys[leaf];
            const float d2 = prim_d2(S, prim, p);
            ++cp;
            if (d2 < h.d2 || (d2 == h.d2 && prim < h.prim)) {
                h.d2 = d2;
                h.prim = prim;
            }
        };
        while (sp > 0) {
            --sp;
            const int v = stn[sp];
            if (std2[sp] > prune_bound(h.d2, tol2)) continue;
            ++cb;
            const Node &nd = S.nodes[v];
            float bd[2];
            for (int c = 0; c < 2; ++c) bd[c] = box_d2(nd.lo[c], nd.hi[c], p, S.D);
            const int nr = bd[1] < bd[0] ? 1 : 0, fr = 1 - nr;
            const int cn = nd.child[nr], cf = nd.child[fr];
            if (cn < 0 && bd[nr] <= prune_bound(h.d2, tol2)) test(~cn);
            if (cf < 0 && bd[fr] <= prune_bound(h.d2, tol2)) test(~cf);
            if (cf >= 0 && bd[fr] <= prune_bound(h.d2, tol2)) {
                stn[sp] = cf;
                std2[sp] = bd[fr];
                ++sp;
            }
            if (cn >= 0 && bd[nr] <= prune_bound(h.d2, tol2)) {
                stn[sp] = cn;
                std2[sp] = bd[nr];
                ++sp;
            }
        }
    }
    if (nbox) *nbox = cb;
    if (nprim) *nprim = cp;
    t_nbox += cb;
    t_nprim += cp;
    t_nquery += 1;
    return h;
}

static inline Hit nearest(const Scene &S, const float *p, bool bvh) {
    return bvh ? nearest_bvh(S, p, nullptr, nullptr) : nearest_brute(S, p);
}

// Closest-point record (include/scene.cuh:180-223).
struct Rec {
    bool valid;
    float p[3];
    float n[3];
    float t[2];  // 2D: t[0] = segment parameter; 3D: (w_b, w_c)
    int prim;
    float contrib;
    float dsrc[5];
};

static Rec closest_record(const Scene &S, const float *x, int prim) {
    Rec r{};
    r.valid = prim >= 0;
    r.prim = prim;
    if (prim < 0) return r;
    if (S.D == 2) {
        const int *I = &S.F[(size_t)prim * 2];
        const float *a = &S.V[2 * I[0]], *b = &S.V[2 * I[1]];
        float h;
        seg_d2(S, prim, x, &h);
        const float ba[2] = {b[0] - a[0], b[1] - a[1]};
        const float pa[2] = {x[0] - a[0], x[1] - a[1]};
        r.p[0] = fmaf(ba[0], h, a[0]);
        r.p[1] = fmaf(ba[1], h, a[1]);
        float n[2] = {ba[1], -ba[0]};
        const float len = sqrtf(dot2(n, n));
        n[0] = n[0] / len;
        n[1] = n[1] / len;
        if (!(dot2(n, pa) > 0.0f)) {  // sign(0) = -1 (include/fwd.cuh:122-128)
            n[0] = -n[0];
            n[1] = -n[1];
        }
        r.n[0] = n[0];
        r.n[1] = n[1];
        r.t[0] = h;
    } else {
        const int *I = &S.F[(size_t)prim * 3];
        const float *a = &S.V[3 * I[0]], *b = &S.V[3 * I[1]], *c = &S.V[3 * I[2]];
        float v, w;
        tri_closest(S, prim, x, &v, &w, nullptr);
        float ab[3], ac[3], ax[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = b[k] - a[k];
            ac[k] = c[k] - a[k];
            ax[k] = x[k] - a[k];
        }
        for (int k = 0; k < 3; ++k) r.p[k] = fmaf(ac[k], w, fmaf(ab[k], v, a[k]));
        float n[3];
        cross3(ab, ac, n);
        const float len = sqrtf(dot3(n, n));
        for (int k = 0; k < 3; ++k) n[k] = n[k] / len;
        const float sgn = dot3(n, ax) > 0.0f ? 1.0f : -1.0f;
        for (int k = 0; k < 3; ++k) r.n[k] = sgn * n[k];
        r.t[0] = v;
        r.t[1] = w;
    }
    return r;
}

// Signed distance and the inside test.  2D: sign of the lerped vertex
// pseudo-normal (scene.cuh:155-166 and scene.py:325-339 agree).  3D: the
// CUDA walk tests the face normal (scene.cuh:167-177) and the Python caller
// tests interpolated vertex normals (scene3d.py:201-214); a point is inside
// only when both say so, as in WoS3DCUDA.single_walk.
struct SdfOut {
    float sd;
    bool inside;
};

static SdfOut sdf_from_hit(const Scene &S, const float *p, const Hit &hit) {
    SdfOut o{};
    const float d = sqrtf(hit.d2);
    if (hit.prim < 0) {
        o.sd = INFINITY;
        o.inside = false;
        return o;
    }
    if (S.D == 2) {
        const int *I = &S.F[(size_t)hit.prim * 2];
        const float *a = &S.V[2 * I[0]], *b = &S.V[2 * I[1]];
        float h;
        seg_d2(S, hit.prim, p, &h);
        const float ba[2] = {b[0] - a[0], b[1] - a[1]};
        const float pa[2] = {p[0] - a[0], p[1] - a[1]};
        const float v[2] = {fmaf(-ba[0], h, pa[0]), fmaf(-ba[1], h, pa[1])};
        const float *na = &S.N[2 * I[0]], *nb = &S.N[2 * I[1]];
        const float n[2] = {fmaf(nb[0] - na[0], h, na[0]), fmaf(nb[1] - na[1], h, na[1])};
        const float s = dot2(n, v);
        o.inside = (s < 0.0f) && (hit.d2 > 0.0f);
        o.sd = s > 0.0f ? d : -d;
    } else {
        const int *I = &S.F[(size_t)hit.prim * 3];
        const float *a = &S.V[3 * I[0]], *b = &S.V[3 * I[1]], *c = &S.V[3 * I[2]];
        float v, w, diff[3];
        tri_closest(S, hit.prim, p, &v, &w, diff);
        float ab[3], ac[3], fn[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = b[k] - a[k];
            ac[k] = c[k] - a[k];
        }
        cross3(ab, ac, fn);
        const float sf = dot3(fn, diff);
        const float *na = &S.N[3 * I[0]], *nb = &S.N[3 * I[1]], *nc = &S.N[3 * I[2]];
        const float w0 = (1.0f - v) - w;
        float nv[3];
        for (int k = 0; k < 3; ++k) nv[k] = fmaf(na[k], w0, fmaf(nb[k], v, nc[k] * w));
        const float sv = dot3(nv, diff);
        o.inside = (hit.d2 > 0.0f) && (sv < 0.0f) && (sf <= 0.0f);
        o.sd = sf > 0.0f ? d : -d;
    }
    return o;
}

// Dirichlet value at a record (include/scene.cuh:251-264).
static inline float dirichlet(const Scene &S, const Rec &r) {
    if (!r.valid) return 0.0f;
    if (S.D == 2) {
        const int *I = &S.F[(size_t)r.prim * 2];
        const float va = S.g[I[0]], vb = S.g[I[1]];
        return fmaf(r.t[0], vb - va, va);
    }
    const int *I = &S.F[(size_t)r.prim * 3];
    const float va = S.g[I[0]], vb = S.g[I[1]], vc = S.g[I[2]];
    const float w0 = (1.0f - r.t[0]) - r.t[1];
    return fmaf(va, w0, fmaf(vb, r.t[0], vc * r.t[1]));
}

// Source function f and its parameter derivatives (include/scene.cuh:278-301).
static inline float source(const Scene &S, const float *p, float *df) {
    const float *q = S.src;
    if (S.src_type == 1) {
        const float tx = p[0] - q[0], ty = p[1] - q[1];
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
        const float phi = fmaf(q[0], p[0], fmaf(q[1], p[1], q[2]));
        const float s = wosm::sin_(phi);
        if (df) {
            const float c = wosm::cos_(phi);
            df[0] = q[3] * c * p[0];
            df[1] = q[3] * c * p[1];
            df[2] = q[3] * c;
            df[3] = s;
            df[4] = 1.0f;
        }
        return fmaf(q[3], s, q[4]);
    }
    if (df)
        for (int k = 0; k < 5; ++k) df[k] = 0.0f;
    return 0.0f;
}

// Radius sample from the tabulated G CDF, reusing the uniform
// (include/wos.cuh:49-75).
static inline float sample_G_radius(const Scene &S, float u, float R, float *pdf) {
    const int n = (int)S.cdf.size();
    int l = 0, r = n - 1;
    while (l < r) {
        const int mid = (l + r) / 2;
        if (u < S.cdf[mid])
            r = mid;
        else
            l = mid + 1;
    }
    const float pmf = l == 0 ? S.cdf[0] : S.cdf[l] - S.cdf[l - 1];
    const float prev = l == 0 ? 0.0f : S.cdf[l - 1];
    u = (u - prev) / pmf;
    *pdf = pmf * (float)n / R;
    return R * ((float)l + u) / (float)n;
}

// ---------------------------------------------------------------- the walk
// One walk from p0 (include/wos.cuh:97-145).  rng draws are indexed by
// (pt, walk, step, role).  steps_out counts the walk's steps.
static Rec walk(const Scene &S, const float *p0, const Params &prm, float eps, const Rng &rng, uint32_t pt,
                uint32_t wk, uint32_t role, bool want_dsrc, int *steps_out) {
    const int D = S.D;
    const bool bvh = prm.use_bvh != 0;
    Rec dead{};
    dead.valid = false;
    dead.prim = -1;
    float p[3] = {p0[0], p0[1], D == 3 ? p0[2] : 0.0f};
    // pixel jitter of the primal walk's start (wos/scene.py:33-39)
    if (role == ROLE_PRIMAL && (prm.jitter[0] != 0.0f || prm.jitter[1] != 0.0f || prm.jitter[2] != 0.0f)) {
        const U4 r = rng.draw(pt, wk, 0, ROLE_JITTER);
        p[0] = fmaf(wosm::u01(r.x) - 0.5f, prm.jitter[0], p[0]);
        p[1] = fmaf(wosm::u01(r.y) - 0.5f, prm.jitter[1], p[1]);
        if (D == 3) p[2] = fmaf(wosm::u01(r.z) - 0.5f, prm.jitter[2], p[2]);
    }
    Hit hit = nearest(S, p, bvh);
    if (steps_out) *steps_out = 0;
    if (!prm.double_sided) {
        const SdfOut so = sdf_from_hit(S, p, hit);
        if (!so.inside) return dead;
    }
    float d = sqrtf(hit.d2);
    if (prm.prevent_fd_artifacts) d *= 0.5f;
    float contrib = 0.0f, dsrc[5] = {0, 0, 0, 0, 0};
    const bool has_src = S.src_type != 0;
    for (int i = 0; i < prm.nsteps; ++i) {
        // no primitive at a finite distance (a NaN or overflowing point)
        if (hit.prim < 0) {
            if (steps_out) *steps_out = i;
            return dead;
        }
        if (d < eps) {
            Rec r = closest_record(S, p, hit.prim);
            r.contrib = contrib;
            for (int k = 0; k < 5; ++k) r.dsrc[k] = dsrc[k];
            if (steps_out) *steps_out = i;
            return r;
        }
        if (!prm.project_unterminated && i == prm.nsteps - 1) {
            if (steps_out) *steps_out = prm.nsteps;
            return dead;
        }
        const U4 r = rng.draw(pt, wk, (uint32_t)i, role);
        if (has_src && D == 2) {
            float dy[2], pdf, weight;
            if (prm.use_IS_for_greens) {
                const float rad = sample_G_radius(S, wosm::u01(r.z), d, &pdf);
                float s, c;
                wosm::sincos_2pi(wosm::u01(r.w), &s, &c);
                pdf = pdf / wosm::kTwoPi;
                dy[0] = rad * c;
                dy[1] = rad * s;
                weight = sqrtf(dot2(dy, dy));
            } else {
                float s, c;
                wosm::sincos_2pi(wosm::u01(r.z), &s, &c);
                const float rr = sqrtf(wosm::u01(r.w));
                dy[0] = rr * c * d;
                dy[1] = rr * s * d;
                pdf = 1.0f / (wosm::kPi * d * d);
                weight = 1.0f;
            }
            const float rn = sqrtf(dot2(dy, dy));
            const float G = wosm::log_(d / fmaxf(rn, 1e-4f)) * wosm::kInv2Pi;
            const float y[2] = {p[0] + dy[0], p[1] + dy[1]};
            float df[5];
            const float f = source(S, y, want_dsrc ? df : nullptr);
            if (pdf > 1e-5f) {
                const float K = G * weight / pdf;
                contrib = fmaf(f, K, contrib);
                if (want_dsrc)
                    for (int k = 0; k < 5; ++k) dsrc[k] = fmaf(df[k], K, dsrc[k]);
            }
        }
        if (D == 2) {
            float s, c;
            wosm::sincos_2pi(wosm::u01(r.x), &s, &c);
            p[0] = fmaf(c, d, p[0]);
            p[1] = fmaf(s, d, p[1]);
        } else {
            const float z = fmaf(-2.0f, wosm::u01(r.x), 1.0f);
            const float rr = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
            float s, c;
            wosm::sincos_2pi(wosm::u01(r.y), &s, &c);
            p[0] = fmaf(rr * c, d, p[0]);
            p[1] = fmaf(rr * s, d, p[1]);
            p[2] = fmaf(z, d, p[2]);
        }
        hit = nearest(S, p, bvh);
        d = sqrtf(hit.d2);
    }
    // the loop ran out (nsteps == 0 or projection of an unterminated walk,
    // wos/wos.py:43); without projection the walk is invalid
    if (!prm.project_unterminated || hit.prim < 0) {
        if (steps_out) *steps_out = prm.nsteps;
        return dead;
    }
    Rec r = closest_record(S, p, hit.prim);
    r.contrib = contrib;
    for (int k = 0; k < 5; ++k) r.dsrc[k] = dsrc[k];
    if (steps_out) *steps_out = prm.nsteps;
    return r;
}

static inline float walk_value(const Scene &S, const Rec &r, bool include_source) {
    if (!r.valid) return 0.0f;
    const float g = dirichlet(S, r);
    return include_source ? g + r.contrib : g;
}

// Largest inscribed ball by bisection (include/scene.cuh:225-249).
static float inscribed_ball(const Scene &S, const Rec &r, float eps, bool bvh) {
    if (!r.valid) return 0.0f;
    float ext = INFINITY;
    for (int k = 0; k < S.D; ++k) ext = fminf(ext, fabsf(S.hi[k] - S.lo[k]));
    float b = ext * 0.5f, a = eps;
    for (int i = 0; i < 10; ++i) {
        const float m = (a + b) * 0.5f;
        float q[3];
        for (int k = 0; k < S.D; ++k) q[k] = fmaf(r.n[k], m, r.p[k]);
        const float d = sqrtf(nearest(S, q, bvh).d2);
        if (wosm::ball_accepts(d, m))
            a = m;
        else
            b = m;
    }
    return a;
}

// u at a point on the inscribed ball: boundary value when within eps2,
// otherwise a full walk (wos/wos.py:94-98, wos/wos3d.py:124-129).
static float ball_u(const Scene &S, const float *q, const Params &prm, float eps2, const Rng &rng,
                    uint32_t pt, uint32_t wk, uint32_t role, bool with_src) {
    const Hit hit = nearest(S, q, prm.use_bvh != 0);
    const float d = sqrtf(hit.d2);
    if (d < eps2) return dirichlet(S, closest_record(S, q, hit.prim));
    // the ball walks end like the primal walk: projected (the Dr.Jit WoS,
    // wos/wos.py:43) or invalid (the CUDA walk, include/wos.cuh:144)
    Params p2 = prm;
    p2.prevent_fd_artifacts = 0;
    const Rec r = walk(S, q, p2, eps2, rng, pt, wk, role, false, nullptr);
    return walk_value(S, r, with_src);
}

static inline float eval_P(const float *c, const float *y, const float *s, float R) {
    const float yy[2] = {y[0] - c[0], y[1] - c[1]};
    const float ss[2] = {s[0] - c[0], s[1] - c[1]};
    const float rr = dot2(yy, yy);
    const float cc = dot2(yy, ss) / sqrtf(dot2(ss, ss));
    const float RR = R * R;
    const float denom = fmaf(-2.0f * R, cc, RR) + rr;
    return (RR - rr) / fmaxf(denom, 1e-5f) / (wosm::kTwoPi * R);
}

// Normal-derivative estimate at a boundary record; returns grad * n_out.
static void normal_derivative(const Scene &S, const Rec &rec, const Params &prm, const AdjParams &ap,
                              const Rng &rng, uint32_t pt, uint32_t wk, float *out, const float *R_given = nullptr) {
    const int D = S.D;
    const bool bvh = prm.use_bvh != 0;
    const bool with_src = ap.source_in_normal_derivative && S.src_type != 0 && D == 2;
    float n[3], p[3];
    for (int k = 0; k < D; ++k) {
        n[k] = -rec.n[k];
        p[k] = rec.p[k];
    }
    const float u_ref = dirichlet(S, rec);
    // the largest inscribed ball, or a given radius (override_R, wos/wos.py:71-74)
    const float R = R_given != nullptr ? *R_given : inscribed_ball(S, rec, ap.ball_epsilon, bvh);
    float c[3];
    for (int k = 0; k < D; ++k) c[k] = fmaf(-n[k], R, p[k]);
    const U4 rx = rng.draw(pt, wk, 0, ROLE_EXTRA);
    float grad = 0.0f;
    if (D == 2) {
        // theta = clamp(2 pi u, clamping, 2 pi - clamping), done in u-space
        const float cu = ap.clamping * wosm::kInv2Pi;
        const float u = fminf(fmaxf(wosm::u01(rx.x), cu), 1.0f - cu);
        float s, cs;
        wosm::sincos_2pi(u, &s, &cs);
        const float pd[2] = {-n[1], n[0]};
        for (int i = 0; i < 2; ++i) {
            const float si = i == 0 ? s : -s;
            float q[2];
            for (int k = 0; k < 2; ++k) q[k] = fmaf(R, fmaf(n[k], cs, pd[k] * si), c[k]);
            const float uq = ball_u(S, q, prm, ap.epsilon2, rng, pt, wk, i == 0 ? ROLE_ANTI_A : ROLE_ANTI_B, with_src);
            const float P = 1.0f / (cs - 1.0f);
            grad += ap.control_variates ? P * (uq - u_ref) / R : P * uq / R;
        }
        grad = grad * 0.5f;
        if (with_src) {
            // interior term (wos/wos_with_source.py:209-230)
            float ds, dc;
            wosm::sincos_2pi(wosm::u01(rx.w), &ds, &dc);
            const float rr = sqrtf(wosm::u01(rx.z));
            const float y[2] = {fmaf(R, rr * dc, c[0]), fmaf(R, rr * ds, c[1])};
            const float f = source(S, y, nullptr);
            const float P = eval_P(c, y, p, R);
            const float area = wosm::kPi * R * R;
            float ci;
            if (ap.control_variates) {
                const float fs = source(S, p, nullptr);
                ci = (f - fs) * P * area + fs * R * 0.5f;
            } else {
                ci = f * P * area;
            }
            grad = grad - ci;
        }
    } else {
        const float ct = fminf(fmaxf(fmaf(-2.0f, wosm::u01(rx.x), 1.0f), -1.0f), 1.0f - ap.clamping);
        float sp, cp;
        wosm::sincos_2pi(wosm::u01(rx.y), &sp, &cp);
        const float up[3] = {fabsf(n[2]) < 0.9f ? 0.0f : 1.0f, 0.0f, fabsf(n[2]) < 0.9f ? 1.0f : 0.0f};
        float pd[3], pd2[3];
        cross3(n, up, pd);
        const float l = sqrtf(dot3(pd, pd));
        for (int k = 0; k < 3; ++k) pd[k] = pd[k] / l;
        cross3(n, pd, pd2);
        const float r = sqrtf(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
        for (int i = 0; i < 2; ++i) {
            const float cphi = i == 0 ? cp : -cp, sphi = i == 0 ? sp : -sp;
            float q[3];
            for (int k = 0; k < 3; ++k) q[k] = fmaf(R, fmaf(ct, n[k], r * fmaf(cphi, pd[k], sphi * pd2[k])), c[k]);
            const float uq = ball_u(S, q, prm, ap.epsilon2, rng, pt, wk, i == 0 ? ROLE_ANTI_A : ROLE_ANTI_B, false);
            const float om = 1.0f - ct;
            const float P = -1.0f / (1.41421356f * (om * sqrtf(om)));
            grad += ap.control_variates ? P * (uq - u_ref) / R : P * uq / R;
        }
        grad = grad * 0.5f;
    }
    for (int k = 0; k < D; ++k) out[k] = grad * n[k];
}

// Tangential gradient of the Dirichlet data (wos/scene.py:451-460,
// wos/wos3d.py:137-156).
static void tangent_derivative(const Scene &S, const Rec &rec, float *out) {
    if (S.D == 2) {
        const int *I = &S.F[(size_t)rec.prim * 2];
        const float *a = &S.V[2 * I[0]], *b = &S.V[2 * I[1]];
        const float e[2] = {b[0] - a[0], b[1] - a[1]};
        const float len = sqrtf(dot2(e, e));
        const float dv = (S.g[I[1]] - S.g[I[0]]) / len;
        out[0] = dv * (e[0] / len);
        out[1] = dv * (e[1] / len);
    } else {
        const int *I = &S.F[(size_t)rec.prim * 3];
        const float *a = &S.V[3 * I[0]], *b = &S.V[3 * I[1]], *c = &S.V[3 * I[2]];
        float ab[3], ac[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = b[k] - a[k];
            ac[k] = c[k] - a[k];
        }
        const float lab = sqrtf(dot3(ab, ab));
        float t[3], fn[3], n[3];
        for (int k = 0; k < 3; ++k) t[k] = ab[k] / lab;
        cross3(ab, ac, fn);
        const float lfn = sqrtf(dot3(fn, fn));
        for (int k = 0; k < 3; ++k) fn[k] = fn[k] / lfn;
        cross3(fn, t, n);
        const float ln = sqrtf(dot3(n, n));
        for (int k = 0; k < 3; ++k) n[k] = n[k] / ln;
        const float va = S.g[I[0]], vb = S.g[I[1]], vc = S.g[I[2]];
        const float gt = (vb - va) / lab;
        const float gn = ((vc - va) - gt * dot3(ac, t)) / dot3(ac, n);
        for (int k = 0; k < 3; ++k) out[k] = fmaf(gt, t[k], gn * n[k]);
    }
}

// One adjoint sample (wos/wos_grad.py:130-151 plus the attached dirichlet
// and source gathers): adds W * d(sample)/d(theta) into dV, dg, dsrc.
static void adjoint_sample(const Scene &S, const float *p0, const Params &prm, const AdjParams &ap, const Rng &rng,
                           uint32_t pt, uint32_t wk, double W, double *dV, double *dg, double *dsrc) {
    const int D = S.D;
    const bool want_src = ap.want_dsrc && prm.include_source && S.src_type != 0;
    const Rec rec = walk(S, p0, prm, prm.epsilon, rng, pt, wk, ROLE_PRIMAL, want_src, nullptr);
    if (!rec.valid) return;
    const int *I = &S.F[(size_t)rec.prim * D];
    float wts[3];
    if (D == 2) {
        wts[0] = 1.0f - rec.t[0];
        wts[1] = rec.t[0];
    } else {
        wts[0] = (1.0f - rec.t[0]) - rec.t[1];
        wts[1] = rec.t[0];
        wts[2] = rec.t[1];
    }
    if (ap.want_dg)
        for (int s = 0; s < D; ++s) dg[I[s]] += W * (double)wts[s];
    if (want_src)
        for (int k = 0; k < 5; ++k) dsrc[k] += W * (double)rec.dsrc[k];
    if (ap.want_dV) {
        float gn[3], gt[3];
        normal_derivative(S, rec, prm, ap, rng, pt, wk, gn);
        tangent_derivative(S, rec, gt);
        for (int s = 0; s < D; ++s)
            for (int k = 0; k < D; ++k)
                dV[(size_t)I[s] * D + k] += W * (double)(-(wts[s] * (gn[k] + gt[k])));
    }
}

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------- C ABI
extern "C" {

void *orc_scene_create(int dim, const float *V, int nV, const int *F, int nF, const float *g, int src_type,
                       const float *src_params) {
    Scene *S = new Scene();
    S->D = dim;
    S->nV = nV;
    S->nF = nF;
    S->V.assign(V, V + (size_t)nV * dim);
    S->F.assign(F, F + (size_t)nF * dim);
    S->g.assign(g, g + nV);
    S->src_type = src_type;
    for (int k = 0; k < 5; ++k) S->src[k] = src_params ? src_params[k] : 0.0f;
    for (int k = 0; k < 3; ++k) {
        S->lo[k] = INFINITY;
        S->hi[k] = -INFINITY;
    }
    for (int v = 0; v < nV; ++v)
        for (int k = 0; k < dim; ++k) {
            S->lo[k] = fminf(S->lo[k], V[(size_t)v * dim + k]);
            S->hi[k] = fmaxf(S->hi[k], V[(size_t)v * dim + k]);
        }
    build_normals(*S);
    build_bvh(*S);
    build_cdf(S->cdf, 10000);
    return S;
}

void orc_scene_destroy(void *s) { delete (Scene *)s; }

void orc_scene_normals(void *s, float *out) {
    Scene *S = (Scene *)s;
    std::copy(S->N.begin(), S->N.end(), out);
}

void orc_scene_aabb(void *s, float *out) {
    Scene *S = (Scene *)s;
    for (int k = 0; k < S->D; ++k) {
        out[k] = S->lo[k];
        out[S->D + k] = S->hi[k];
    }
}

void orc_g_cdf(float *out, int n) {
    std::vector<float> c;
    build_cdf(c, n);
    std::copy(c.begin(), c.end(), out);
}

// child refs of the LBVH in Karras numbering; leaves as ~sorted_pos
int orc_bvh_export(void *s, int *children, uint64_t *keys) {
    Scene *S = (Scene *)s;
    for (size_t i = 0; i < S->nodes.size(); ++i) {
        children[2 * i] = S->nodes[i].child[0];
        children[2 * i + 1] = S->nodes[i].child[1];
    }
    std::copy(S->keys.begin(), S->keys.end(), keys);
    return (int)S->nodes.size();
}

void orc_closest(void *s, const float *P, int n, int use_bvh, int *prim, float *dist, float *tuv, float *pt,
                 float *nrm, float *sd, unsigned char *inside, int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        const float *p = &P[(size_t)i * D];
        const Hit h = nearest(*S, p, use_bvh != 0);
        const Rec r = closest_record(*S, p, h.prim);
        const SdfOut so = sdf_from_hit(*S, p, h);
        if (prim) prim[i] = h.prim;
        if (dist) dist[i] = sqrtf(h.d2);
        for (int k = 0; k < D; ++k) {
            if (pt) pt[(size_t)i * D + k] = r.p[k];
            if (nrm) nrm[(size_t)i * D + k] = r.n[k];
        }
        if (tuv) {
            tuv[(size_t)i * 2] = r.t[0];
            tuv[(size_t)i * 2 + 1] = D == 3 ? r.t[1] : 0.0f;
        }
        if (sd) sd[i] = so.sd;
        if (inside) inside[i] = so.inside ? 1 : 0;
    }
}

void orc_bvh_counts(void *s, const float *P, int n, int *nbox, int *nprim, int nthreads) {
    Scene *S = (Scene *)s;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) nearest_bvh(*S, &P[(size_t)i * S->D], &nbox[i], &nprim[i]);
}

void orc_inscribed_ball(void *s, const float *pt, const float *nrm, const unsigned char *valid, int n, float eps,
                        int use_bvh, float *R, int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        Rec r{};
        r.valid = valid[i] != 0;
        for (int k = 0; k < D; ++k) {
            r.p[k] = pt[(size_t)i * D + k];
            r.n[k] = nrm[(size_t)i * D + k];
        }
        R[i] = inscribed_ball(*S, r, eps, use_bvh != 0);
    }
}

// Soft-edge walk of Baseline / Baseline3D (wos/wos.py:158-187,
// wos/wos_grad_3d.py:24-57): exactly nsteps steps, each adding
// beta (1 - w) g with w = min(d, eps) / eps, then beta *= w.
static float soft_walk(const Scene &S, const float *p0, const Params &prm, const Rng &rng, uint32_t pt, uint32_t wk) {
    const int D = S.D;
    const bool bvh = prm.use_bvh != 0;
    float p[3] = {p0[0], p0[1], D == 3 ? p0[2] : 0.0f};
    if (prm.jitter[0] != 0.0f || prm.jitter[1] != 0.0f || prm.jitter[2] != 0.0f) {
        const U4 r = rng.draw(pt, wk, 0, ROLE_JITTER);
        p[0] = fmaf(wosm::u01(r.x) - 0.5f, prm.jitter[0], p[0]);
        p[1] = fmaf(wosm::u01(r.y) - 0.5f, prm.jitter[1], p[1]);
        if (D == 3) p[2] = fmaf(wosm::u01(r.z) - 0.5f, prm.jitter[2], p[2]);
    }
    Hit hit = nearest(S, p, bvh);
    if (hit.prim < 0) return 0.0f;
    if (!prm.double_sided && !sdf_from_hit(S, p, hit).inside) return 0.0f;
    const float eps = prm.epsilon;
    float beta = 1.0f, res = 0.0f;
    for (int i = 0; i < prm.nsteps; ++i) {
        const float d = sqrtf(hit.d2);
        const Rec r = closest_record(S, p, hit.prim);
        const float g = dirichlet(S, r);
        const float w = fminf(d, eps) / eps;
        if (d > 0.0f) res = fmaf(beta * (1.0f - w), g, res);
        beta = beta * w;
        if (i == prm.nsteps - 1) break;
        const U4 rr = rng.draw(pt, wk, (uint32_t)i, ROLE_PRIMAL);
        float dir[3] = {0.0f, 0.0f, 0.0f};
        if (D == 2) {
            float s, c;
            wosm::sincos_2pi(wosm::u01(rr.x), &s, &c);
            dir[0] = c;
            dir[1] = s;
        } else {
            const float z = fmaf(-2.0f, wosm::u01(rr.x), 1.0f);
            const float rad = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
            float s, c;
            wosm::sincos_2pi(wosm::u01(rr.y), &s, &c);
            dir[0] = rad * c;
            dir[1] = rad * s;
            dir[2] = z;
        }
        for (int k = 0; k < D; ++k) p[k] = fmaf(dir[k], d, p[k]);
        hit = nearest(S, p, bvh);
        if (hit.prim < 0) return 0.0f;
    }
    return res;
}

void orc_soft_walk(void *s, const float *P, int n, const Params *prm, float *vals, int nthreads) {
    Scene *S = (Scene *)s;
    const Rng rng = make_rng(prm->seed);
    const int nw = prm->nwalks;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long t = 0; t < (long long)n * nw; ++t) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        vals[t] = soft_walk(*S, &P[(size_t)i * S->D], *prm, rng, (uint32_t)i, prm->walk_offset + (uint32_t)w);
    }
}

// Must match wos_detector in include/wos_b200.h.
struct Detector {
    float vmin[2], vmax[2];
    int32_t res[2];
    int32_t axis_u, axis_v, slab_axis;
    float slab_center, slab_half_width;
    float size;
    int32_t flags;
};

// Image-space boundary term of WoSBoundary (wos/wos_boundary.py:11-31):
// res[0] * res[1] * nwalks boundary samples.  Sample s draws a primitive with
// probability proportional to its measure (segment length, triangle area;
// wos/scene.py:275-279, wos/scene3d.py:150-155) by inverse CDF over the
// running sums, reusing the uniform inside the primitive's interval as the
// segment parameter (Mitsuba's sample_reuse_pmf, wos/scene.py:435-449); a
// triangle point is (sqrt r1 (1 - r2), sqrt r1 r2) in barycentrics
// (wos/scene3d.py:253-257).  n is the detached normal (-ab.y, ab.x) / |ab| or
// -(ab x ac) / |ab x ac|, val the interpolated Dirichlet value.  The term
// -val (x . n - detach(x . n)) / pdf has derivative -val (n . dx) / pdf for a
// motion dx of the sample, the lerp / barycentric mix of its vertices'
// motion; it goes to the sample's pixel (Detector.index, wos/scene.py:18-24,
// wos/scene3d.py:35-43), divided by the detector size and nwalks
// (wos/wos_boundary.py:13-21).  pdf = 1 / total measure, or in 3D with
// flags & 1 the reference's pmf / |ab x ac| = 1 / (2 total area)
// (wos/scene3d.py:262).  Random numbers: Philox(seed; s mod 2^32, s / 2^32,
// 0, role 5).  Forward mode adds the derivative image for vertex motion tV to
// img; reverse mode adds the vertex gradient of pixel weights dLdI to dV.
static void boundary_sample(const Scene &S, const Detector &det, const std::vector<double> &cdf, double pdf_scale,
                            int nwalks, const Rng &rng, long long s, const float *tV, double *img,
                            const float *dLdI, double *dV) {
    const int D = S.D;
    const int nF = S.nF;
    const double total = cdf[nF - 1];
    const U4 r = rng.draw((uint32_t)s, (uint32_t)(s >> 32), 0, 5);
    const double target = (double)wosm::u01(r.x) * total;
    const int f = (int)(std::upper_bound(cdf.begin(), cdf.end() - 1, target) - cdf.begin());
    const double base = f > 0 ? cdf[f - 1] : 0.0;
    const double wdt = cdf[f] - base;
    float t = wdt > 0.0 ? (float)((target - base) / wdt) : 0.0f;
    t = fminf(fmaxf(t, 0.0f), 0x1.fffffep-1f);
    int vid[3] = {0, 0, 0};
    float wts[3] = {0.0f, 0.0f, 0.0f}, x[3] = {0.0f, 0.0f, 0.0f}, n[3] = {0.0f, 0.0f, 0.0f};
    float val;
    if (D == 2) {
        vid[0] = S.F[2 * f];
        vid[1] = S.F[2 * f + 1];
        const float ax = S.V[2 * vid[0]], ay = S.V[2 * vid[0] + 1];
        const float abx = S.V[2 * vid[1]] - ax, aby = S.V[2 * vid[1] + 1] - ay;
        x[0] = fmaf(t, abx, ax);
        x[1] = fmaf(t, aby, ay);
        wts[0] = 1.0f - t;
        wts[1] = t;
        val = fmaf(t, S.g[vid[1]] - S.g[vid[0]], S.g[vid[0]]);
        const float l = sqrtf(fmaf(abx, abx, aby * aby));
        n[0] = -aby / l;
        n[1] = abx / l;
    } else {
        for (int k = 0; k < 3; ++k) vid[k] = S.F[3 * f + k];
        const float su = sqrtf(wosm::u01(r.y)), r2 = wosm::u01(r.z);
        const float u = su * (1.0f - r2), v = su * r2;
        wts[0] = 1.0f - u - v;
        wts[1] = u;
        wts[2] = v;
        float ab[3], ac[3];
        for (int k = 0; k < 3; ++k) {
            const float a = S.V[3 * vid[0] + k];
            ab[k] = S.V[3 * vid[1] + k] - a;
            ac[k] = S.V[3 * vid[2] + k] - a;
            x[k] = fmaf(u, ab[k], fmaf(v, ac[k], a));
        }
        val = fmaf(wts[0], S.g[vid[0]], fmaf(u, S.g[vid[1]], v * S.g[vid[2]]));
        float c[3];
        cross3(ab, ac, c);
        const float l = sqrtf(dot3(c, c));
        for (int k = 0; k < 3; ++k) n[k] = -c[k] / l;
    }
    const int iu = (int)fmaf((x[det.axis_u] - det.vmin[0]) / (det.vmax[0] - det.vmin[0]), (float)det.res[0], 0.5f);
    const int iv = (int)fmaf((x[det.axis_v] - det.vmin[1]) / (det.vmax[1] - det.vmin[1]), (float)det.res[1], 0.5f);
    bool ok = iu >= 0 && iu < det.res[0] && iv >= 0 && iv < det.res[1];
    if (det.slab_axis >= 0) ok = ok && fabsf(x[det.slab_axis] - det.slab_center) < det.slab_half_width;
    const long long npix = (long long)det.res[0] * det.res[1];
    const long long idx = (long long)iu + (long long)(det.res[1] - iv) * det.res[0];
    if (!ok || idx < 0 || idx >= npix) return;
    const double w = -(double)val * total * pdf_scale / ((double)det.size * nwalks);
    if (tV != nullptr) {
        double nd = 0.0;
        for (int j = 0; j < D; ++j)
            for (int k = 0; k < D; ++k) nd += (double)n[k] * wts[j] * tV[(size_t)vid[j] * D + k];
        img[idx] += w * nd;
    }
    if (dLdI != nullptr) {
        const double cw = (double)dLdI[idx] * w;
        for (int j = 0; j < D; ++j)
            for (int k = 0; k < D; ++k) dV[(size_t)vid[j] * D + k] += cw * n[k] * wts[j];
    }
}

void orc_boundary_term(void *s, const Detector *det, int nwalks, uint64_t seed, const float *tV, double *img,
                       const float *dLdI, double *dV, int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    const int nF = S->nF;
    std::vector<double> cdf(nF);
    double run = 0.0;
    for (int f = 0; f < nF; ++f) {
        double m;
        if (D == 2) {
            const float *a = &S->V[2 * S->F[2 * f]], *b = &S->V[2 * S->F[2 * f + 1]];
            const double dx = (double)b[0] - a[0], dy = (double)b[1] - a[1];
            m = sqrt(dx * dx + dy * dy);
        } else {
            const float *a = &S->V[3 * S->F[3 * f]], *b = &S->V[3 * S->F[3 * f + 1]], *c = &S->V[3 * S->F[3 * f + 2]];
            const double u[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
            const double v[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
            const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
            m = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        }
        run += m;
        cdf[f] = run;
    }
    const double pdf_scale = (D == 3 && (det->flags & 1)) ? 2.0 : 1.0;
    const long long npix = (long long)det->res[0] * det->res[1];
    const long long ns = npix * nwalks;
    const Rng rng = make_rng(seed);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const size_t nvd = (size_t)S->nV * D;
#pragma omp parallel
    {
        std::vector<double> im(tV ? npix : 0, 0.0), dv(dLdI ? nvd : 0, 0.0);
#pragma omp for schedule(static)
        for (long long i = 0; i < ns; ++i)
            boundary_sample(*S, *det, cdf, pdf_scale, nwalks, rng, i, tV, im.data(), dLdI, dv.data());
#pragma omp critical
        {
            for (size_t k = 0; k < im.size(); ++k) img[k] += im[k];
            for (size_t k = 0; k < dv.size(); ++k) dV[k] += dv[k];
        }
    }
}

// FP64 reference solution of -lap u = f (f constant) with Dirichlet data g
// on a 2D polyline scene, for scoring the FP32 solvers against an FP64
// solution where no closed form exists (the star with f = 1).  The walk of
// include/wos.cuh:97-145 in double precision: nearest distance to the float
// geometry (exact in double) through the LBVH, whose float boxes bound the
// float segments exactly; a uniform direction on the circle from 53 random
// bits; termination in the eps-shell with g interpolated at the closest
// point.  Each step's source term is its expectation, f R^2 / 4 (the integral
// over the disk of its Green's function log(R / r) / 2 pi), so the estimator
// is unbiased for the same problem and samples no source point.  A walk still
// inside after max_steps steps takes the value at its closest boundary point
// (counted in *truncated).  Random numbers: Philox role 6, independent of the
// FP32 walks.  Per-point mean and unbiased variance.
static double seg_d2_f64(const Scene &S, int f, const double *p, double *h_out) {
    const int *I = &S.F[(size_t)f * 2];
    const double a[2] = {S.V[2 * I[0]], S.V[2 * I[0] + 1]}, b[2] = {S.V[2 * I[1]], S.V[2 * I[1] + 1]};
    const double ba[2] = {b[0] - a[0], b[1] - a[1]}, pa[2] = {p[0] - a[0], p[1] - a[1]};
    const double len2 = ba[0] * ba[0] + ba[1] * ba[1];
    double h = len2 > 0.0 ? (pa[0] * ba[0] + pa[1] * ba[1]) / len2 : 0.0;
    h = std::min(std::max(h, 0.0), 1.0);
    const double v[2] = {pa[0] - h * ba[0], pa[1] - h * ba[1]};
    *h_out = h;
    return v[0] * v[0] + v[1] * v[1];
}

static inline double box_d2_f64(const float *lo, const float *hi, const double *p) {
    double s = 0.0;
    for (int k = 0; k < 2; ++k) {
        const double d = std::max(std::max((double)lo[k] - p[k], p[k] - (double)hi[k]), 0.0);
        s += d * d;
    }
    return s;
}

static int nearest_f64(const Scene &S, const double *p, double &best, double &hbest) {
    int prim = -1;
    best = std::numeric_limits<double>::infinity();
    auto test = [&](int f) {
        double h;
        const double d2 = seg_d2_f64(S, f, p, &h);
        if (d2 < best) {
            best = d2;
            hbest = h;
            prim = f;
        }
    };
    if (S.nF == 1) {
        test(0);
        return prim;
    }
    int stn[96];
    double std2[96];
    int sp = 0;
    stn[sp] = 0;
    std2[sp++] = 0.0;
    while (sp > 0) {
        --sp;
        if (std2[sp] > best) continue;
        const Node &nd = S.nodes[stn[sp]];
        const double bd[2] = {box_d2_f64(nd.lo[0], nd.hi[0], p), box_d2_f64(nd.lo[1], nd.hi[1], p)};
        const int nr = bd[1] < bd[0] ? 1 : 0, fr = 1 - nr;
        const int order[2] = {fr, nr};  // push the far child first
        for (int c : order) {
            if (bd[c] > best) continue;
            const int ch = nd.child[c];
            if (ch < 0) {
                test((int)(uint32_t)S.keys[~ch]);
            } else if (sp < 96) {
                stn[sp] = ch;
                std2[sp++] = bd[c];
            }
        }
    }
    return prim;
}

static inline double g_f64(const Scene &S, int f, double h) {
    const int *I = &S.F[(size_t)f * 2];
    return (1.0 - h) * (double)S.g[I[0]] + h * (double)S.g[I[1]];
}

void orc_solve_f64_2d(void *s, const double *P, int n, int nwalks, int max_steps, double eps, double fconst,
                      uint64_t seed, int nthreads, double *mean, double *var, long long *truncated) {
    Scene *S = (Scene *)s;
    const Rng rng = make_rng(seed);
    const double two_pi = 6.283185307179586476925286766559;
    long long trunc = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : trunc)
    for (int i = 0; i < n; ++i) {
        double sum = 0.0, sum2 = 0.0;
        for (int w = 0; w < nwalks; ++w) {
            double x[2] = {P[2 * i], P[2 * i + 1]}, acc = 0.0, val = 0.0, d2, h;
            bool done = false;
            for (int k = 0; k < max_steps && !done; ++k) {
                const int f = nearest_f64(*S, x, d2, h);
                const double d = std::sqrt(d2);
                if (f < 0) {
                    done = true;  // no geometry: scored 0
                } else if (d < eps) {
                    val = g_f64(*S, f, h) + acc;
                    done = true;
                } else {
                    acc += fconst * d2 * 0.25;
                    const U4 r = rng.draw((uint32_t)i, (uint32_t)w, (uint32_t)k, 6u);
                    const double u = (double)(((uint64_t)r.x << 21) ^ (uint64_t)(r.y >> 11)) * 0x1p-53;
                    x[0] += d * std::cos(two_pi * u);
                    x[1] += d * std::sin(two_pi * u);
                }
            }
            if (!done) {
                const int f = nearest_f64(*S, x, d2, h);
                val = (f >= 0 ? g_f64(*S, f, h) : 0.0) + acc;
                ++trunc;
            }
            sum += val;
            sum2 += val * val;
        }
        const double m = sum / nwalks;
        mean[i] = m;
        var[i] = nwalks > 1 ? std::max(0.0, (sum2 - nwalks * m * m) / (nwalks - 1)) : 0.0;
    }
    if (truncated) *truncated = trunc;
}

// Per-walk values for points x walks; vals[i * nwalks + w].
void orc_walk_values(void *s, const float *P, int n, const Params *prm, float *vals, unsigned char *valid,
                     int *steps, int nthreads) {
    Scene *S = (Scene *)s;
    const Rng rng = make_rng(prm->seed);
    const int nw = prm->nwalks;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long t = 0; t < (long long)n * nw; ++t) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        int st = 0;
        const Rec r = walk(*S, &P[(size_t)i * S->D], *prm, prm->epsilon, rng, (uint32_t)i,
                           prm->walk_offset + (uint32_t)w, ROLE_PRIMAL, false, &st);
        vals[t] = walk_value(*S, r, prm->include_source != 0);
        if (valid) valid[t] = r.valid ? 1 : 0;
        if (steps) steps[t] = st;
    }
}

// One walk per point with walk index prm->walk_offset; full records.
void orc_walk_records(void *s, const float *P, int n, const Params *prm, unsigned char *valid, float *pt,
                      float *nrm, float *tuv, int *prim, float *contrib, int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    const Rng rng = make_rng(prm->seed);
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        const Rec r = walk(*S, &P[(size_t)i * D], *prm, prm->epsilon, rng, (uint32_t)i, prm->walk_offset,
                           ROLE_PRIMAL, false, nullptr);
        valid[i] = r.valid ? 1 : 0;
        for (int k = 0; k < D; ++k) {
            pt[(size_t)i * D + k] = r.valid ? r.p[k] : 0.0f;
            nrm[(size_t)i * D + k] = r.valid ? r.n[k] : 0.0f;
        }
        tuv[(size_t)i * 2] = r.valid ? r.t[0] : 0.0f;
        tuv[(size_t)i * 2 + 1] = (r.valid && D == 3) ? r.t[1] : 0.0f;
        prim[i] = r.valid ? r.prim : -1;
        contrib[i] = r.valid ? r.contrib : 0.0f;
    }
}

// Per-point FP64 mean and sample variance of per-walk values, with
// Neumaier-compensated sums, in walk order.
void orc_reduce(const float *vals, int n, int nwalks, double *mean, double *var) {
    for (int i = 0; i < n; ++i) {
        double s = 0.0, c = 0.0;
        for (int w = 0; w < nwalks; ++w) {
            const double x = vals[(size_t)i * nwalks + w];
            const double t = s + x;
            c += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
            s = t;
        }
        const double m = (s + c) / nwalks;
        double q = 0.0, qc = 0.0;
        for (int w = 0; w < nwalks; ++w) {
            const double e = vals[(size_t)i * nwalks + w] - m;
            const double x = e * e;
            const double t = q + x;
            qc += std::fabs(q) >= std::fabs(x) ? (q - t) + x : (x - t) + q;
            q = t;
        }
        mean[i] = m;
        if (var) var[i] = nwalks > 1 ? (q + qc) / (nwalks - 1) : 0.0;
    }
}

// Normal-derivative estimates at records (one sample per record, walk index
// prm->walk_offset); out = grad * n_out, n x dim.
void orc_normal_derivative_r(void *s, const unsigned char *valid, const float *pt, const float *nrm, const float *tuv,
                             const int *prim, const float *R, int n, const Params *prm, const AdjParams *ap, float *out,
                             int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    const Rng rng = make_rng(prm->seed);
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
        Rec r{};
        r.valid = valid[i] != 0;
        r.prim = prim[i];
        for (int k = 0; k < D; ++k) {
            r.p[k] = pt[(size_t)i * D + k];
            r.n[k] = nrm[(size_t)i * D + k];
        }
        r.t[0] = tuv[(size_t)i * 2];
        r.t[1] = tuv[(size_t)i * 2 + 1];
        float g[3] = {0, 0, 0};
        if (r.valid) normal_derivative(*S, r, *prm, *ap, rng, (uint32_t)i, prm->walk_offset, g, R ? &R[i] : nullptr);
        for (int k = 0; k < D; ++k) out[(size_t)i * D + k] = g[k];
    }
}

void orc_normal_derivative(void *s, const unsigned char *valid, const float *pt, const float *nrm, const float *tuv,
                           const int *prim, int n, const Params *prm, const AdjParams *ap, float *out, int nthreads) {
    orc_normal_derivative_r(s, valid, pt, nrm, tuv, prim, nullptr, n, prm, ap, out, nthreads);
}

// Adjoint of the per-point means: dL/dtheta = sum_i dLdu[i] * du_i/dtheta,
// one adjoint sample per (point, walk), weight dLdu[i] / nwalks.
void orc_adjoint(void *s, const float *P, int n, const Params *prm, const AdjParams *ap, const float *dLdu,
                 double *dV, double *dg, double *dsrc, int nthreads) {
    Scene *S = (Scene *)s;
    const int D = S->D;
    const Rng rng = make_rng(prm->seed);
    const int nw = prm->nwalks;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int T = omp_get_max_threads();
    std::vector<std::vector<double>> bV(T, std::vector<double>((size_t)S->nV * D, 0.0)),
        bg(T, std::vector<double>(S->nV, 0.0)), bs(T, std::vector<double>(5, 0.0));
#pragma omp parallel for schedule(dynamic, 1)
    for (long long t = 0; t < (long long)n * nw; ++t) {
        const int tid = omp_get_thread_num();
        const int i = (int)(t / nw), w = (int)(t % nw);
        const double W = (double)dLdu[i] / nw;
        if (W == 0.0) continue;
        adjoint_sample(*S, &P[(size_t)i * D], *prm, *ap, rng, (uint32_t)i, prm->walk_offset + (uint32_t)w, W,
                       bV[tid].data(), bg[tid].data(), bs[tid].data());
    }
    for (int t = 0; t < T; ++t) {
        for (size_t k = 0; k < bV[t].size(); ++k) dV[k] += bV[t][k];
        for (size_t k = 0; k < bg[t].size(); ++k) dg[k] += bg[t][k];
        for (int k = 0; k < 5; ++k) dsrc[k] += bs[t][k];
    }
}

// Totals of the traversal counters over all threads of the last
// orc_adjoint_counted / orc_walk_counted call: {queries, node visits, prims}.
static long long g_counts[3] = {0, 0, 0};

static void count_begin() {
#pragma omp parallel
    {
        t_nbox = 0;
        t_nprim = 0;
        t_nquery = 0;
    }
}
static void count_end() {
    long long a = 0, b = 0, c = 0;
#pragma omp parallel reduction(+ : a, b, c)
    {
        a += t_nquery;
        b += t_nbox;
        c += t_nprim;
    }
    g_counts[0] = a;
    g_counts[1] = b;
    g_counts[2] = c;
}

void orc_walk_counted(void *s, const float *P, int n, const Params *prm, float *vals, int nthreads, long long *counts) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    count_begin();
    orc_walk_values(s, P, n, prm, vals, nullptr, nullptr, nthreads);
    count_end();
    for (int k = 0; k < 3; ++k) counts[k] = g_counts[k];
}

void orc_adjoint_counted(void *s, const float *P, int n, const Params *prm, const AdjParams *ap, const float *dLdu,
                         double *dV, double *dg, double *dsrc, int nthreads, long long *counts) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    count_begin();
    orc_adjoint(s, P, n, prm, ap, dLdu, dV, dg, dsrc, nthreads);
    count_end();
    for (int k = 0; k < 3; ++k) counts[k] = g_counts[k];
}

// Test hooks for the elementary functions.
void orc_math(int which, const float *x, const float *y, float *out, int n) {
    for (int i = 0; i < n; ++i) {
        switch (which) {
            case 0: {
                float s, c;
                wosm::sincos_2pi(x[i], &s, &c);
                out[2 * i] = s;
                out[2 * i + 1] = c;
                break;
            }
            case 1: out[i] = wosm::sin_(x[i]); break;
            case 2: out[i] = wosm::cos_(x[i]); break;
            case 3: out[i] = wosm::log_(x[i]); break;
            case 4: out[i] = wosm::exp_(x[i]); break;
            case 5: out[i] = wosm::atan2_(x[i], y[i]); break;
        }
    }
}

// Point-triangle closest point on raw triangles: uv = (w_b, w_c), distance.
void orc_tri_closest(const float *A, const float *B, const float *C, const float *P, int n, float *uv, float *d) {
    for (int i = 0; i < n; ++i) {
        float v, w;
        const float d2 = tri_closest_raw(&A[3 * i], &B[3 * i], &C[3 * i], &P[3 * i], &v, &w, nullptr);
        uv[2 * i] = v;
        uv[2 * i + 1] = w;
        d[i] = sqrtf(d2);
    }
}

void orc_philox(uint64_t seed, const uint32_t *ctr, uint32_t *out, int n) {
    const Rng r = make_rng(seed);
    for (int i = 0; i < n; ++i) {
        const U4 v = r.draw(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]);
        out[4 * i] = v.x;
        out[4 * i + 1] = v.y;
        out[4 * i + 2] = v.z;
        out[4 * i + 3] = v.w;
    }
}

}  // extern "C"
