// Scene construction on the GPU: vertex normals, scene AABB, primitive
// precomputation and the LBVH (Morton codes, radix sort, Karras hierarchy,
// bottom-up refit, breadth-first node order).
//
// Replaces the reference's host Scene<N>::configure_normal / configure
// (include/scene.cuh:368-453), which did the AABB on the host and the BVH in
// the third-party lbvh library.  Everything here is deterministic: vertex
// normals are summed per vertex in (face, slot) order, the tree is a pure
// function of the sorted (morton << 32 | prim) keys, and boxes are min/max.
#include <cub/cub.cuh>

#include <vector>

#include "scene_impl.h"
#include "wos_device.cuh"

namespace wosd {

#define WOS_TRY(x)                                    \
    do {                                              \
        cudaError_t _e = (x);                         \
        if (_e != cudaSuccess) return fail_cuda(_e, #x); \
    } while (0)

// ------------------------------------------------------------------ kernels
__device__ __forceinline__ int ordered_int(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float from_ordered_int(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_check_indices(const int *F, long long n, int nV, int *bad) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int v = F[i];
        if (v < 0 || v >= nV) atomicOr(bad, 1);
    }
}

__global__ void k_aabb(const float *V, int nV, int dim, int *lohi) {
    // lohi[0..2] = ordered min, lohi[3..5] = ordered max
    __shared__ int smin[3], smax[3];
    if (threadIdx.x < 3) {
        smin[threadIdx.x] = 0x7fffffff;
        smax[threadIdx.x] = (int)0x80000000;
    }
    __syncthreads();
    int lmin[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, lmax[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nV; v += gridDim.x * blockDim.x)
        for (int k = 0; k < dim; ++k) {
            const int o = ordered_int(V[(size_t)v * dim + k]);
            lmin[k] = min(lmin[k], o);
            lmax[k] = max(lmax[k], o);
        }
    for (int k = 0; k < dim; ++k) {
        atomicMin(&smin[k], lmin[k]);
        atomicMax(&smax[k], lmax[k]);
    }
    __syncthreads();
    if (threadIdx.x < dim) {
        atomicMin(&lohi[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&lohi[3 + threadIdx.x], smax[threadIdx.x]);
    }
}

// Per (face, slot) normal contribution and its sort key (vertex << 32 | slot id).
template <int D>
__global__ void k_face_normals(const float *V, const int *F, int nF, float *contrib, unsigned long long *keys) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    if (D == 2) {
        const int i0 = F[2 * f], i1 = F[2 * f + 1];
        const float dx = V[2 * i1] - V[2 * i0], dy = V[2 * i1 + 1] - V[2 * i0 + 1];
        float nx = dy, ny = -dx;
        const float len = sqrtf(dot2(nx, ny, nx, ny));
        if (len > 0.0f) {
            nx = nx / len;
            ny = ny / len;
        } else {
            nx = ny = 0.0f;
        }
        for (int s = 0; s < 2; ++s) {
            contrib[(size_t)(2 * f + s) * 2] = nx;
            contrib[(size_t)(2 * f + s) * 2 + 1] = ny;
            keys[2 * f + s] = ((unsigned long long)(unsigned)F[2 * f + s] << 32) | (unsigned)(2 * f + s);
        }
    } else {
        const int i0 = F[3 * f], i1 = F[3 * f + 1], i2 = F[3 * f + 2];
        const float *p0 = V + 3 * (size_t)i0, *p1 = V + 3 * (size_t)i1, *p2 = V + 3 * (size_t)i2;
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
        cross3(e10[0], e10[1], e10[2], e20[0], e20[1], e20[2], n[0], n[1], n[2]);
        const float len = sqrtf(dot3(n[0], n[1], n[2], n[0], n[1], n[2]));
        if (len > 0.0f) {
            for (int k = 0; k < 3; ++k) n[k] = n[k] / len;
        } else {
            n[0] = n[1] = n[2] = 0.0f;
        }
        auto angle = [](const float *a, const float *b) {
            float c[3];
            cross3(a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]);
            return wosm::atan2_(sqrtf(dot3(c[0], c[1], c[2], c[0], c[1], c[2])), dot3(a[0], a[1], a[2], b[0], b[1], b[2]));
        };
        const float ang[3] = {angle(e10, e20), angle(e21, e01), angle(e02, e12)};
        for (int s = 0; s < 3; ++s) {
            for (int k = 0; k < 3; ++k) contrib[(size_t)(3 * f + s) * 3 + k] = ang[s] * n[k];
            keys[3 * f + s] = ((unsigned long long)(unsigned)F[3 * f + s] << 32) | (unsigned)(3 * f + s);
        }
    }
}

__global__ void k_segments(const unsigned long long *keys, int n, int *beg, int *end) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned v = (unsigned)(keys[i] >> 32);
    if (i == 0 || (unsigned)(keys[i - 1] >> 32) != v) beg[v] = i;
    if (i == n - 1 || (unsigned)(keys[i + 1] >> 32) != v) end[v] = i + 1;
}

template <int D>
__global__ void k_vertex_normals(const unsigned long long *keys, const float *contrib, const int *beg, const int *end,
                                 int nV, float *N) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nV) return;
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (int i = beg[v]; i < end[v]; ++i) {
        const unsigned slot = (unsigned)keys[i];
        for (int k = 0; k < D; ++k) s[k] += contrib[(size_t)slot * D + k];
    }
    const float len = sqrtf(D == 2 ? dot2(s[0], s[1], s[0], s[1]) : dot3(s[0], s[1], s[2], s[0], s[1], s[2]));
    for (int k = 0; k < D; ++k) N[(size_t)v * D + k] = len > 0.0f ? s[k] / len : 0.0f;
}

__device__ __forceinline__ uint32_t spread2(uint32_t x) {
    x &= 0xffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
__device__ __forceinline__ uint32_t spread3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// Hilbert index of a 3D cell (10 bits per axis), by Skilling's transpose
// method ("Programming the Hilbert curve", AIP Conf. Proc. 707, 2004): undo
// the excess work of the axes, Gray-encode, then interleave the transposed
// bits, axis 0 most significant.  Consecutive indices are face-adjacent
// cells, so runs of primitives sorted by it are more compact than Morton
// runs, whose curve jumps between octants.
__device__ __forceinline__ uint32_t hilbert3(uint32_t x0, uint32_t x1, uint32_t x2) {
    uint32_t X[3] = {x0, x1, x2};
    const uint32_t M = 1u << 9;
    for (uint32_t Q = M; Q > 1; Q >>= 1) {
        const uint32_t P = Q - 1;
        for (int i = 0; i < 3; ++i) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                const uint32_t t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    uint32_t t = 0;
    for (uint32_t Q = M; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    for (int i = 0; i < 3; ++i) X[i] ^= t;
    return (spread3(X[0]) << 2) | (spread3(X[1]) << 1) | spread3(X[2]);
}

// Number of segments f whose end vertex starts segment f + 1 (cyclically).
__global__ void k_chain_count(const int *F, int nF, int *count) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const int next = f + 1 < nF ? f + 1 : 0;
    if (F[2 * f + 1] == F[2 * next]) atomicAdd(count, 1);
}

// Primitive precomputation, primitive boxes and sort keys: Morton (order 0),
// the input index (order 1) or Hilbert (order 2) of the box centre.
template <int D>
__global__ void k_prims(const float *V, const int *F, int nF, float lo0, float lo1, float lo2, float hi0, float hi1,
                        float hi2, float4 *seg, float *seginv, float4 *tri, float *pbox, unsigned long long *keys,
                        int order) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const float slo[3] = {lo0, lo1, lo2}, shi[3] = {hi0, hi1, hi2};
    float bl[3], bh[3];
    if (D == 2) {
        const int i0 = F[2 * f], i1 = F[2 * f + 1];
        const float ax = V[2 * i0], ay = V[2 * i0 + 1], bx = V[2 * i1], by = V[2 * i1 + 1];
        const float bax = bx - ax, bay = by - ay;
        const float len2 = dot2(bax, bay, bax, bay);
        seg[f] = make_float4(ax, ay, bax, bay);
        seginv[f] = len2 > 0.0f ? 1.0f / len2 : 0.0f;
        bl[0] = fminf(ax, bx);
        bh[0] = fmaxf(ax, bx);
        bl[1] = fminf(ay, by);
        bh[1] = fmaxf(ay, by);
    } else {
        const int i0 = F[3 * f], i1 = F[3 * f + 1], i2 = F[3 * f + 2];
        float a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = V[3 * (size_t)i0 + k];
            b[k] = V[3 * (size_t)i1 + k];
            c[k] = V[3 * (size_t)i2 + k];
        }
        float ab[3], ac[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = b[k] - a[k];
            ac[k] = c[k] - a[k];
        }
        tri[3 * f] = make_float4(a[0], a[1], a[2], dot3(ab[0], ab[1], ab[2], ab[0], ab[1], ab[2]));
        tri[3 * f + 1] = make_float4(ab[0], ab[1], ab[2], dot3(ab[0], ab[1], ab[2], ac[0], ac[1], ac[2]));
        tri[3 * f + 2] = make_float4(ac[0], ac[1], ac[2], dot3(ac[0], ac[1], ac[2], ac[0], ac[1], ac[2]));
        for (int k = 0; k < 3; ++k) {
            bl[k] = fminf(fminf(a[k], b[k]), c[k]);
            bh[k] = fmaxf(fmaxf(a[k], b[k]), c[k]);
        }
    }
    uint32_t q[3];
    const float scale = D == 2 ? 65536.0f : 1024.0f;
    for (int k = 0; k < D; ++k) {
        pbox[(size_t)f * 2 * D + k] = bl[k];
        pbox[(size_t)f * 2 * D + D + k] = bh[k];
        const float c = (bl[k] + bh[k]) * 0.5f;
        const float ext = shi[k] - slo[k];
        const float u = ext > 0.0f ? (c - slo[k]) / ext : 0.0f;
        q[k] = (uint32_t)fminf(fmaxf(u * scale, 0.0f), scale - 1.0f);
    }
    uint32_t m;
    if (order == 1)
        m = (uint32_t)f;
    else if (D == 3 && order == 2)
        m = hilbert3(q[0], q[1], q[2]);
    else
        m = D == 2 ? (spread2(q[0]) | (spread2(q[1]) << 1))
                   : (spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2));
    keys[f] = ((unsigned long long)m << 32) | (unsigned)f;
}

__device__ __forceinline__ int kdelta(const unsigned long long *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);
}

// Karras 2012, one thread per internal node.
__global__ void k_karras(const unsigned long long *k, int n, int2 *child, int *parent_int, int *parent_leaf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (kdelta(k, n, i, i + 1) - kdelta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(k, n, i, i - d);
    int lmax = 2;
    while (kdelta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (kdelta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(k, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        const int t = (l + div - 1) / div;
        if (kdelta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    int2 c;
    if (min(i, j) == gamma) {
        c.x = ~gamma;
        parent_leaf[gamma] = i;
    } else {
        c.x = gamma;
        parent_int[gamma] = i;
    }
    if (max(i, j) == gamma + 1) {
        c.y = ~(gamma + 1);
        parent_leaf[gamma + 1] = i;
    } else {
        c.y = gamma + 1;
        parent_int[gamma + 1] = i;
    }
    child[i] = c;
}

// Bottom-up boxes: the second thread to reach a node merges its children.
template <int D>
__global__ void k_refit(const unsigned long long *keys, int n, const float *pbox, const int2 *child,
                        const int *parent_int, const int *parent_leaf, int *flags, float *nbox) {
    const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    int v = parent_leaf[leaf];
    while (v >= 0) {
        __threadfence();
        if (atomicAdd(&flags[v], 1) == 0) return;
        __threadfence();
        const int2 c = child[v];
        float lo[3], hi[3];
        for (int side = 0; side < 2; ++side) {
            const int r = side == 0 ? c.x : c.y;
            const float *b;
            if (r < 0) {
                const unsigned prim = (unsigned)keys[~r];
                b = pbox + (size_t)prim * 2 * D;
            } else {
                b = nbox + (size_t)r * 2 * D;
            }
            for (int k = 0; k < D; ++k) {
                const float l = __ldcg(b + k), h = __ldcg(b + D + k);
                lo[k] = side == 0 ? l : fminf(lo[k], l);
                hi[k] = side == 0 ? h : fmaxf(hi[k], h);
            }
        }
        for (int k = 0; k < D; ++k) {
            __stcg(nbox + (size_t)v * 2 * D + k, lo[k]);
            __stcg(nbox + (size_t)v * 2 * D + D + k, hi[k]);
        }
        v = parent_int[v];
    }
}

__global__ void k_depth(const int *parent_int, int nInt, unsigned long long *dkeys, int *maxdepth) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInt) return;
    int d = 0, v = i;
    while (v > 0 && d < 4096) {
        v = parent_int[v];
        ++d;
    }
    dkeys[i] = ((unsigned long long)d << 32) | (unsigned)i;
    atomicMax(maxdepth, d);
}

__global__ void k_bfs_rank(const unsigned long long *sorted, int nInt, int *new_of_old) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nInt) return;
    new_of_old[(unsigned)sorted[r]] = r;
}

template <int D>
__global__ void k_write_nodes(const unsigned long long *keys, int nInt, const float *pbox, const float *nbox,
                              const int2 *child, const int *new_of_old, float4 *node) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInt) return;
    const int2 c = child[i];
    float lo[2][3], hi[2][3];
    int ref[2];
    for (int side = 0; side < 2; ++side) {
        const int r = side == 0 ? c.x : c.y;
        const float *b;
        if (r < 0) {
            b = pbox + (size_t)(unsigned)keys[~r] * 2 * D;
            ref[side] = r;
        } else {
            b = nbox + (size_t)r * 2 * D;
            ref[side] = new_of_old[r];
        }
        for (int k = 0; k < D; ++k) {
            lo[side][k] = b[k];
            hi[side][k] = b[D + k];
        }
    }
    const int o = new_of_old[i];
    if (D == 2) {
        node[3 * o] = make_float4(lo[0][0], lo[0][1], hi[0][0], hi[0][1]);
        node[3 * o + 1] = make_float4(lo[1][0], lo[1][1], hi[1][0], hi[1][1]);
        node[3 * o + 2] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), 0.0f, 0.0f);
    } else {
        node[4 * o] = make_float4(lo[0][0], lo[0][1], lo[0][2], hi[0][0]);
        node[4 * o + 1] = make_float4(hi[0][1], hi[0][2], lo[1][0], lo[1][1]);
        node[4 * o + 2] = make_float4(lo[1][2], hi[1][0], hi[1][1], hi[1][2]);
        node[4 * o + 3] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), 0.0f, 0.0f);
    }
}

template <int D>
__global__ void k_leaf_data(const unsigned long long *keys, int n, const float4 *seg, const float *seginv,
                            const float4 *tri, float4 *lseg, float *lseginv, float4 *ltri, int *lorig) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int f = (int)(unsigned)keys[s];
    lorig[s] = f;
    if (D == 2) {
        lseg[s] = seg[f];
        lseginv[s] = seginv[f];
    } else {
        ltri[3 * s] = tri[3 * f];
        ltri[3 * s + 1] = tri[3 * f + 1];
        ltri[3 * s + 2] = tri[3 * f + 2];
    }
}

// Wide-tree leaf boxes.  Leaf i holds sorted positions [WT_LEAF i, WT_LEAF i
// + WT_LEAF); its box is the union of its primitives' boxes and bounds it in
// the level above.
template <int D>
__global__ void k_wt_level1(const unsigned long long *keys, int nF, const float *pbox, float4 *out, int n1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n1) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int b0 = WT_LEAF * i, e = min(b0 + WT_LEAF, nF);
    for (int s = b0; s < e; ++s) {
        const float *b = pbox + (size_t)(unsigned)keys[s] * 2 * D;
        for (int k = 0; k < D; ++k) {
            lo[k] = fminf(lo[k], b[k]);
            hi[k] = fmaxf(hi[k], b[D + k]);
        }
    }
    if (D == 2) {
        out[i] = make_float4(lo[0], lo[1], hi[0], hi[1]);
    } else {
        out[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        out[2 * i + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
}

// Eigenvectors of a symmetric 3 x 3 matrix by cyclic Jacobi rotations in
// double: on return the columns of v are orthonormal and a is (nearly)
// diagonal, a[k][k] the eigenvalue of column k.
__device__ void sym3_eigen(double a[3][3], double v[3][3]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) v[r][c] = r == c ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (!(off > 1e-30 * dia)) break;
        for (int p = 0; p < 2; ++p) {
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                // rotation in the (p, q) plane that zeroes a[p][q]: A <- J^T A J
                const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = c * vkp - s * vkq;
                    v[k][q] = s * vkp + c * vkq;
                }
            }
        }
    }
}

// Oriented box of each wide-tree leaf, the bound the queries test leaves by.
// Its axes are the principal axes of the leaf's vertices as the distance code
// sees them (a and a + d for a segment; a, a + ab, a + ac for a triangle):
// the eigenvectors of their covariance, rounded to float and shrunk by 2^-20
// so that the float axes, with the third 3D axis u2 = u0 x u1 evaluated in
// float exactly as the query does (cross3), form a matrix of norm below 1.
// The centre c is rounded to float, and e_k bounds |u_k.(y - c)| over the
// vertices y, evaluated in double with the float axes and centre and widened
// by 1e-6 |y - c|max, which covers the query's float rounding of q - c and of
// the dot products (relative 2^-22 of |q - c| <= |q - y| + |y - c|).  Layout:
// 2D (u0.x, u0.y, c.x, c.y), (e0, e1, 0, 0) with u1 = (-u0.y, u0.x); 3D
// (u0, e0), (u1, e1), (c, e2).
template <int D>
__global__ void k_wt_obb(const float4 *lseg, const float4 *ltri, int nF, float4 *obb, int n1) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n1) return;
    const int b0 = WT_LEAF * i, e = min(b0 + WT_LEAF, nF);
    constexpr int NV = D == 2 ? 2 : 3;
    auto vertex = [&](int s, int j, double *y) {
        if (D == 2) {
            const float4 g = lseg[s];
            y[0] = j == 0 ? (double)g.x : (double)g.x + g.z;
            y[1] = j == 0 ? (double)g.y : (double)g.y + g.w;
            y[2] = 0.0;
        } else {
            const float4 a = ltri[3 * s], ab = ltri[3 * s + 1], ac = ltri[3 * s + 2];
            y[0] = j == 0 ? (double)a.x : (double)a.x + (j == 1 ? ab.x : ac.x);
            y[1] = j == 0 ? (double)a.y : (double)a.y + (j == 1 ? ab.y : ac.y);
            y[2] = j == 0 ? (double)a.z : (double)a.z + (j == 1 ? ab.z : ac.z);
        }
    };
    double m[3] = {0.0, 0.0, 0.0}, y[3];
    for (int s = b0; s < e; ++s)
        for (int j = 0; j < NV; ++j) {
            vertex(s, j, y);
            for (int k = 0; k < D; ++k) m[k] += y[k];
        }
    const double nv = (double)((e - b0) * NV);
    for (int k = 0; k < D; ++k) m[k] /= nv;
    double cov[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int s = b0; s < e; ++s)
        for (int j = 0; j < NV; ++j) {
            vertex(s, j, y);
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) cov[r][c] += (y[r] - m[r]) * (y[c] - m[c]);
        }
    // float axes u[k][*]
    float u[3][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
    const double shrink = 1.0 - 0x1p-20;
    if (D == 2) {
        const double th = 0.5 * atan2(2.0 * cov[0][1], cov[0][0] - cov[1][1]);
        u[0][0] = (float)(cos(th) * shrink);
        u[0][1] = (float)(sin(th) * shrink);
        u[1][0] = -u[0][1];
        u[1][1] = u[0][0];
    } else {
        double vec[3][3];
        sym3_eigen(cov, vec);
        // u0, u1: the two largest-variance axes; u2 = u0 x u1 (the normal)
        int o[3] = {0, 1, 2};
        for (int a = 0; a < 2; ++a)
            for (int b = a + 1; b < 3; ++b)
                if (cov[o[b]][o[b]] > cov[o[a]][o[a]]) {
                    const int t = o[a];
                    o[a] = o[b];
                    o[b] = t;
                }
        for (int k = 0; k < 3; ++k) {
            u[0][k] = (float)(vec[k][o[0]] * shrink);
            u[1][k] = (float)(vec[k][o[1]] * shrink);
        }
        cross3(u[0][0], u[0][1], u[0][2], u[1][0], u[1][1], u[1][2], u[2][0], u[2][1], u[2][2]);
    }
    // centre: the middle of the projection ranges about the mean
    double pmin[3] = {INFINITY, INFINITY, INFINITY}, pmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int s = b0; s < e; ++s)
        for (int j = 0; j < NV; ++j) {
            vertex(s, j, y);
            for (int k = 0; k < D; ++k) {
                double p = 0.0;
                for (int c = 0; c < D; ++c) p += (double)u[k][c] * (y[c] - m[c]);
                pmin[k] = fmin(pmin[k], p);
                pmax[k] = fmax(pmax[k], p);
            }
        }
    float cf[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < D; ++c) {
        double x = m[c];
        for (int k = 0; k < D; ++k) x += 0.5 * (pmin[k] + pmax[k]) * (double)u[k][c];
        cf[c] = (float)x;
    }
    double ext[3] = {0.0, 0.0, 0.0}, r2 = 0.0;
    for (int s = b0; s < e; ++s)
        for (int j = 0; j < NV; ++j) {
            vertex(s, j, y);
            double d2 = 0.0;
            for (int c = 0; c < D; ++c) d2 += (y[c] - cf[c]) * (y[c] - cf[c]);
            r2 = fmax(r2, d2);
            for (int k = 0; k < D; ++k) {
                double p = 0.0;
                for (int c = 0; c < D; ++c) p += (double)u[k][c] * (y[c] - (double)cf[c]);
                ext[k] = fmax(ext[k], fabs(p));
            }
        }
    const double pad = 1e-6 * sqrt(r2);
    float ef[3];
    for (int k = 0; k < D; ++k) ef[k] = __double2float_ru(ext[k] + pad);
    if (D == 2) {
        obb[2 * i] = make_float4(u[0][0], u[0][1], cf[0], cf[1]);
        obb[2 * i + 1] = make_float4(ef[0], ef[1], 0.0f, 0.0f);
    } else {
        obb[3 * i] = make_float4(u[0][0], u[0][1], u[0][2], ef[0]);
        obb[3 * i + 1] = make_float4(u[1][0], u[1][1], u[1][2], ef[1]);
        obb[3 * i + 2] = make_float4(cf[0], cf[1], cf[2], ef[2]);
    }
}

template <int D>
__global__ void k_wt_level(const float4 *in, int n_in, float4 *out, int n_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int e = min(32 * i + 32, n_in);
    for (int c = 32 * i; c < e; ++c) {
        if (D == 2) {
            const float4 b = in[c];
            lo[0] = fminf(lo[0], b.x);
            lo[1] = fminf(lo[1], b.y);
            hi[0] = fmaxf(hi[0], b.z);
            hi[1] = fmaxf(hi[1], b.w);
        } else {
            const float4 a = in[2 * c], b = in[2 * c + 1];
            lo[0] = fminf(lo[0], a.x);
            lo[1] = fminf(lo[1], a.y);
            lo[2] = fminf(lo[2], a.z);
            hi[0] = fmaxf(hi[0], b.x);
            hi[1] = fmaxf(hi[1], b.y);
            hi[2] = fmaxf(hi[2], b.z);
        }
    }
    if (D == 2) {
        out[i] = make_float4(lo[0], lo[1], hi[0], hi[1]);
    } else {
        out[2 * i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        out[2 * i + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
}

// Slab bounds of the level-2 nodes of a 3D wide tree (patches of up to 1024
// triangles): n = the normalised sum of the unit face normals, and the
// interval [oc - oh, oc + oh] of n.(v - c) over the vertices v as the distance
// code sees them, c the node's box centre computed exactly as the query does,
// evaluated in double and widened by the float roundings plus a relative
// margin.  A node whose normals cancel gets n = 0 and oh = inf (no slab).  One block of
// SLAB_THREADS per node; fixed-order reductions.  The half-thickness goes to
// the box's first .w, the normal and the interval's centre to slab[node].
constexpr int SLAB_THREADS = 256;
__global__ void __launch_bounds__(SLAB_THREADS) k_wt_slab2(const float4 *ltri, int nF, float4 *box, float4 *slab,
                                                            int n2) {
    __shared__ double red[3][SLAB_THREADS];
    const int i = blockIdx.x, t = threadIdx.x;
    if (i >= n2) return;
    const int b0 = WT_LEAF * 32 * i, e = min(b0 + WT_LEAF * 32, nF);
    double ns[3] = {0.0, 0.0, 0.0};
    for (int s = b0 + t; s < e; s += SLAB_THREADS) {
        const float4 ab = ltri[3 * s + 1], ac = ltri[3 * s + 2];
        double nn[3];
        nn[0] = (double)ab.y * ac.z - (double)ab.z * ac.y;
        nn[1] = (double)ab.z * ac.x - (double)ab.x * ac.z;
        nn[2] = (double)ab.x * ac.y - (double)ab.y * ac.x;
        const double l = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
        if (l > 0.0)
            for (int k = 0; k < 3; ++k) ns[k] += nn[k] / l;
    }
    for (int k = 0; k < 3; ++k) red[k][t] = ns[k];
    __syncthreads();
    for (int h = SLAB_THREADS / 2; h > 0; h >>= 1) {
        if (t < h)
            for (int k = 0; k < 3; ++k) red[k][t] += red[k][t + h];
        __syncthreads();
    }
    for (int k = 0; k < 3; ++k) ns[k] = red[k][0];
    __syncthreads();
    const float4 ba = box[2 * i], bb = box[2 * i + 1];
    const float lo[3] = {ba.x, ba.y, ba.z}, hi[3] = {bb.x, bb.y, bb.z};
    float c[3];
    for (int k = 0; k < 3; ++k) c[k] = (lo[k] + hi[k]) * 0.5f;
    const double ln = sqrt(ns[0] * ns[0] + ns[1] * ns[1] + ns[2] * ns[2]);
    float nf[3] = {0.0f, 0.0f, 0.0f};
    float ocf = 0.0f, ohf = INFINITY;
    if (ln > 1e-6) {
        // unit normal, shrunk by 2^-20 so that |n| <= 1 after rounding
        for (int k = 0; k < 3; ++k) nf[k] = (float)(ns[k] / ln * (1.0 - 0x1p-20));
        double omin = INFINITY, omax = -INFINITY, diag2 = 0.0;
        for (int k = 0; k < 3; ++k) diag2 += ((double)hi[k] - lo[k]) * ((double)hi[k] - lo[k]);
        for (int s = b0 + t; s < e; s += SLAB_THREADS) {
            const float4 a = ltri[3 * s], ab = ltri[3 * s + 1], ac = ltri[3 * s + 2];
            const double av[3] = {a.x, a.y, a.z}, abv[3] = {ab.x, ab.y, ab.z}, acv[3] = {ac.x, ac.y, ac.z};
            for (int j = 0; j < 3; ++j) {
                double o = 0.0;
                for (int k = 0; k < 3; ++k) {
                    const double v = av[k] + (j == 1 ? abv[k] : j == 2 ? acv[k] : 0.0);
                    o += (double)nf[k] * (v - (double)c[k]);
                }
                omin = fmin(omin, o);
                omax = fmax(omax, o);
            }
        }
        red[0][t] = omin;
        red[1][t] = omax;
        __syncthreads();
        for (int h = SLAB_THREADS / 2; h > 0; h >>= 1) {
            if (t < h) {
                red[0][t] = fmin(red[0][t], red[0][t + h]);
                red[1][t] = fmax(red[1][t], red[1][t + h]);
            }
            __syncthreads();
        }
        omin = red[0][0];
        omax = red[1][0];
        const double oc = 0.5 * (omin + omax);
        ocf = (float)oc;
        const double oh = 0.5 * (omax - omin) + fabs(oc - (double)ocf) + 1e-6 * sqrt(diag2);
        ohf = __double2float_ru(oh);
    }
    if (t == 0) {
        box[2 * i].w = ohf;
        slab[i] = make_float4(nf[0], nf[1], nf[2], ocf);
    }
}

// ------------------------------------------------------------------ host
static inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

template <typename T>
static cudaError_t dalloc(T **p, size_t count, cudaStream_t st) {
    if (count == 0) count = 1;
    return cudaMallocAsync((void **)p, count * sizeof(T), st);
}

void SceneImpl::release(cudaStream_t st) {
    void *ptrs[] = {V, F, N, g, seg, seginv, tri, node, lseg, lseginv, ltri, lorig, cdf, wt_box, wt_slab, wt_obb, guide};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, st);
    V = nullptr;
    F = nullptr;
    N = nullptr;
    g = nullptr;
    seg = nullptr;
    seginv = nullptr;
    tri = nullptr;
    node = nullptr;
    lseg = nullptr;
    lseginv = nullptr;
    ltri = nullptr;
    lorig = nullptr;
    cdf = nullptr;
    wt_box = nullptr;
    wt_slab = nullptr;
    wt_obb = nullptr;
    wt_n[0] = wt_n[1] = wt_n[2] = 0;
    guide = nullptr;
}

// Normalised CDF of pmf_i ~ r_i log(1/r_i), r_i = (i + 0.5)/n, built in
// double on the host (include/tabulated_G_cdf.cuh:5-8 regenerated from its
// formula, wos/wos_with_source.py:17-23).
void build_g_cdf(std::vector<float> &cdf, int n) {
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

void build_g_guide(const std::vector<float> &cdf, int ng, std::vector<unsigned short> &guide) {
    const int n = (int)cdf.size();
    guide.resize(ng + 1);
    int l = 0;
    for (int k = 0; k <= ng; ++k) {
        const float u = (float)k / (float)ng;
        while (l < n - 1 && !(u < cdf[l])) ++l;
        guide[k] = (unsigned short)l;
    }
}

template <int D>
static int build_geometry(SceneImpl &S, cudaStream_t st) {
    const int nV = S.nV, nF = S.nF;
    const int TB = 256;
    // ---- AABB
    int *lohi = nullptr;
    WOS_TRY(dalloc(&lohi, 6, st));
    {
        int init[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, (int)0x80000000, (int)0x80000000, (int)0x80000000};
        WOS_TRY(cudaMemcpyAsync(lohi, init, sizeof(init), cudaMemcpyHostToDevice, st));
        WOS_TRY(cudaStreamSynchronize(st));
    }
    k_aabb<<<std::min(nblk(nV, TB), 1024), TB, 0, st>>>(S.V, nV, D, lohi);
    int lohi_h[6];
    WOS_TRY(cudaMemcpyAsync(lohi_h, lohi, sizeof(lohi_h), cudaMemcpyDeviceToHost, st));
    WOS_TRY(cudaStreamSynchronize(st));
    cudaFreeAsync(lohi, st);
    auto from_ord = [](int i) {
        int b = i >= 0 ? i : i ^ 0x7fffffff;
        float f;
        memcpy(&f, &b, 4);
        return f;
    };
    for (int k = 0; k < 3; ++k) {
        S.lo[k] = k < D ? from_ord(lohi_h[k]) : 0.0f;
        S.hi[k] = k < D ? from_ord(lohi_h[3 + k]) : 0.0f;
    }
    float ext = INFINITY;
    for (int k = 0; k < D; ++k) ext = fminf(ext, fabsf(S.hi[k] - S.lo[k]));
    S.half_min_extent = ext * 0.5f;

    // ---- vertex normals
    {
        const int ns = nF * D;
        float *contrib = nullptr;
        unsigned long long *keys = nullptr, *keys2 = nullptr;
        int *beg = nullptr, *end = nullptr;
        WOS_TRY(dalloc(&contrib, (size_t)ns * D, st));
        WOS_TRY(dalloc(&keys, ns, st));
        WOS_TRY(dalloc(&keys2, ns, st));
        WOS_TRY(dalloc(&beg, nV, st));
        WOS_TRY(dalloc(&end, nV, st));
        WOS_TRY(cudaMemsetAsync(beg, 0, sizeof(int) * nV, st));
        WOS_TRY(cudaMemsetAsync(end, 0, sizeof(int) * nV, st));
        k_face_normals<D><<<nblk(nF, TB), TB, 0, st>>>(S.V, S.F, nF, contrib, keys);
        size_t tmp_bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys, keys2, ns, 0, 64, st);
        void *tmp = nullptr;
        WOS_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
        WOS_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, keys2, ns, 0, 64, st));
        k_segments<<<nblk(ns, TB), TB, 0, st>>>(keys2, ns, beg, end);
        k_vertex_normals<D><<<nblk(nV, TB), TB, 0, st>>>(keys2, contrib, beg, end, nV, S.N);
        WOS_TRY(cudaGetLastError());
        cudaFreeAsync(tmp, st);
        cudaFreeAsync(contrib, st);
        cudaFreeAsync(keys, st);
        cudaFreeAsync(keys2, st);
        cudaFreeAsync(beg, st);
        cudaFreeAsync(end, st);
    }

    // ---- primitive order: a polyline whose segments follow each other keeps
    // its input order (its leaves are then arcs of the curve, the most
    // compact runs); other polylines sort by Morton code, meshes by Hilbert
    // index.  Decided once: moving vertices keeps the order.
    if (S.prim_order < 0) {
        S.prim_order = D == 3 ? 2 : 0;
        if (D == 2 && nF >= 2) {
            int *cnt = nullptr;
            WOS_TRY(dalloc(&cnt, 1, st));
            WOS_TRY(cudaMemsetAsync(cnt, 0, sizeof(int), st));
            k_chain_count<<<nblk(nF, TB), TB, 0, st>>>(S.F, nF, cnt);
            int cnt_h = 0;
            WOS_TRY(cudaMemcpyAsync(&cnt_h, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
            WOS_TRY(cudaStreamSynchronize(st));
            cudaFreeAsync(cnt, st);
            if (cnt_h >= nF - nF / 10) S.prim_order = 1;
        }
    }

    // ---- primitives + sort keys
    float *pbox = nullptr;
    unsigned long long *mkeys = nullptr, *skeys = nullptr;
    WOS_TRY(dalloc(&pbox, (size_t)nF * 2 * D, st));
    WOS_TRY(dalloc(&mkeys, nF, st));
    WOS_TRY(dalloc(&skeys, nF, st));
    k_prims<D><<<nblk(nF, TB), TB, 0, st>>>(S.V, S.F, nF, S.lo[0], S.lo[1], S.lo[2], S.hi[0], S.hi[1], S.hi[2], S.seg,
                                           S.seginv, S.tri, pbox, mkeys, S.prim_order);
    {
        size_t tmp_bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, mkeys, skeys, nF, 0, 64, st);
        void *tmp = nullptr;
        WOS_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
        WOS_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, mkeys, skeys, nF, 0, 64, st));
        cudaFreeAsync(tmp, st);
    }
    k_leaf_data<D><<<nblk(nF, TB), TB, 0, st>>>(skeys, nF, S.seg, S.seginv, S.tri, S.lseg, S.lseginv, S.ltri, S.lorig);

    // ---- wide tree (levels 1..wt_levels, the top one with <= 32 nodes)
    {
        const int W = D == 2 ? 1 : 2;  // float4 per box
        int count = (nF + WT_LEAF - 1) / WT_LEAF, level = 1, off = 0;
        S.wt_count[0] = nF;
        for (;;) {
            if (level > WT_MAX_LEVELS) return fail(WOS_ERR_UNSUPPORTED, "scene too large for the wide tree");
            S.wt_count[level] = count;
            S.wt_off[level] = off;
            off += count;
            if (count <= 32) break;
            count = (count + 31) / 32;
            ++level;
        }
        S.wt_levels = level;
        // The level sizes depend on nF alone, so a rebuild after the vertices
        // move (wos_scene_update_vertices) refills the buffers of the first
        // build in place: device views held elsewhere (batch plans, captured
        // graphs, launches on other streams) keep pointing at live memory.
        const bool slab2 = D == 3 && S.wt_levels >= 2;
        const size_t n_box = (size_t)off * W, n_slab = slab2 ? (size_t)S.wt_count[2] : 0,
                     n_obb = (size_t)S.wt_count[1] * (D == 2 ? 2 : 3);
        if (S.wt_box == nullptr || S.wt_n[0] != n_box || S.wt_n[1] != n_slab || S.wt_n[2] != n_obb) {
            if (S.wt_box) cudaFreeAsync(S.wt_box, st);
            if (S.wt_slab) cudaFreeAsync(S.wt_slab, st);
            if (S.wt_obb) cudaFreeAsync(S.wt_obb, st);
            S.wt_box = S.wt_slab = S.wt_obb = nullptr;
            WOS_TRY(dalloc(&S.wt_box, n_box, st));
            WOS_TRY(dalloc(&S.wt_slab, n_slab, st));
            WOS_TRY(dalloc(&S.wt_obb, n_obb, st));
            S.wt_n[0] = n_box;
            S.wt_n[1] = n_slab;
            S.wt_n[2] = n_obb;
        }
        k_wt_level1<D><<<nblk(S.wt_count[1], TB), TB, 0, st>>>(skeys, nF, pbox, S.wt_box, S.wt_count[1]);
        k_wt_obb<D><<<nblk(S.wt_count[1], 64), 64, 0, st>>>(S.lseg, S.ltri, nF, S.wt_obb, S.wt_count[1]);
        for (int l = 2; l <= S.wt_levels; ++l)
            k_wt_level<D><<<nblk(S.wt_count[l], TB), TB, 0, st>>>(S.wt_box + (size_t)S.wt_off[l - 1] * W,
                                                                S.wt_count[l - 1], S.wt_box + (size_t)S.wt_off[l] * W,
                                                                S.wt_count[l]);
        if (slab2)
            k_wt_slab2<<<S.wt_count[2], SLAB_THREADS, 0, st>>>(S.ltri, nF, S.wt_box + (size_t)S.wt_off[2] * W,
                                                               S.wt_slab, S.wt_count[2]);
        WOS_TRY(cudaGetLastError());
    }

    // ---- hierarchy
    const int nInt = nF - 1;
    S.nNodes = nInt;
    S.depth = 0;
    if (nInt > 0) {
        int2 *child = nullptr;
        int *pint = nullptr, *pleaf = nullptr, *flags = nullptr, *maxd = nullptr, *new_of_old = nullptr;
        float *nbox = nullptr;
        unsigned long long *dkeys = nullptr, *dkeys2 = nullptr;
        WOS_TRY(dalloc(&child, nInt, st));
        WOS_TRY(dalloc(&pint, nInt, st));
        WOS_TRY(dalloc(&pleaf, nF, st));
        WOS_TRY(dalloc(&flags, nInt, st));
        WOS_TRY(dalloc(&maxd, 1, st));
        WOS_TRY(dalloc(&new_of_old, nInt, st));
        WOS_TRY(dalloc(&nbox, (size_t)nInt * 2 * D, st));
        WOS_TRY(dalloc(&dkeys, nInt, st));
        WOS_TRY(dalloc(&dkeys2, nInt, st));
        WOS_TRY(cudaMemsetAsync(pint, 0xff, sizeof(int) * nInt, st));
        WOS_TRY(cudaMemsetAsync(pleaf, 0xff, sizeof(int) * nF, st));
        WOS_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * nInt, st));
        WOS_TRY(cudaMemsetAsync(maxd, 0, sizeof(int), st));
        k_karras<<<nblk(nInt, TB), TB, 0, st>>>(skeys, nF, child, pint, pleaf);
        k_refit<D><<<nblk(nF, TB), TB, 0, st>>>(skeys, nF, pbox, child, pint, pleaf, flags, nbox);
        k_depth<<<nblk(nInt, TB), TB, 0, st>>>(pint, nInt, dkeys, maxd);
        size_t tmp_bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, dkeys, dkeys2, nInt, 0, 64, st);
        void *tmp = nullptr;
        WOS_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
        WOS_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, dkeys, dkeys2, nInt, 0, 64, st));
        k_bfs_rank<<<nblk(nInt, TB), TB, 0, st>>>(dkeys2, nInt, new_of_old);
        k_write_nodes<D><<<nblk(nInt, TB), TB, 0, st>>>(skeys, nInt, pbox, nbox, child, new_of_old, S.node);
        WOS_TRY(cudaGetLastError());
        int maxd_h = 0;
        WOS_TRY(cudaMemcpyAsync(&maxd_h, maxd, sizeof(int), cudaMemcpyDeviceToHost, st));
        WOS_TRY(cudaStreamSynchronize(st));
        S.depth = maxd_h;
        cudaFreeAsync(tmp, st);
        cudaFreeAsync(child, st);
        cudaFreeAsync(pint, st);
        cudaFreeAsync(pleaf, st);
        cudaFreeAsync(flags, st);
        cudaFreeAsync(maxd, st);
        cudaFreeAsync(new_of_old, st);
        cudaFreeAsync(nbox, st);
        cudaFreeAsync(dkeys, st);
        cudaFreeAsync(dkeys2, st);
    }
    cudaFreeAsync(pbox, st);
    cudaFreeAsync(mkeys, st);
    cudaFreeAsync(skeys, st);
    WOS_TRY(cudaGetLastError());
    WOS_TRY(cudaStreamSynchronize(st));
    return 0;
}

int SceneImpl::allocate(cudaStream_t st) {
    const int D = dim;
    WOS_TRY(dalloc(&V, (size_t)nV * D, st));
    WOS_TRY(dalloc(&F, (size_t)nF * D, st));
    WOS_TRY(dalloc(&N, (size_t)nV * D, st));
    WOS_TRY(dalloc(&g, nV, st));
    if (D == 2) {
        WOS_TRY(dalloc(&seg, nF, st));
        WOS_TRY(dalloc(&seginv, nF, st));
        WOS_TRY(dalloc(&lseg, nF, st));
        WOS_TRY(dalloc(&lseginv, nF, st));
        WOS_TRY(dalloc(&node, (size_t)std::max(nF - 1, 1) * 3, st));
    } else {
        WOS_TRY(dalloc(&tri, (size_t)nF * 3, st));
        WOS_TRY(dalloc(&ltri, (size_t)nF * 3, st));
        WOS_TRY(dalloc(&node, (size_t)std::max(nF - 1, 1) * 4, st));
    }
    WOS_TRY(dalloc(&lorig, nF, st));
    std::vector<float> c;
    build_g_cdf(c, 10000);
    n_cdf = (int)c.size();
    std::vector<unsigned short> gd;
    n_guide = 2048;
    build_g_guide(c, n_guide, gd);
    WOS_TRY(dalloc(&cdf, c.size(), st));
    WOS_TRY(dalloc(&guide, gd.size(), st));
    WOS_TRY(cudaMemcpyAsync(cdf, c.data(), c.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    WOS_TRY(cudaMemcpyAsync(guide, gd.data(), gd.size() * sizeof(unsigned short), cudaMemcpyHostToDevice, st));
    WOS_TRY(cudaStreamSynchronize(st));
    return 0;
}

int SceneImpl::check_indices(cudaStream_t st) {
    int *bad = nullptr;
    WOS_TRY(dalloc(&bad, 1, st));
    WOS_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    const long long n = (long long)nF * dim;
    k_check_indices<<<std::min(nblk(n, 256), 4096), 256, 0, st>>>(F, n, nV, bad);
    int bad_h = 0;
    WOS_TRY(cudaMemcpyAsync(&bad_h, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    WOS_TRY(cudaStreamSynchronize(st));
    cudaFreeAsync(bad, st);
    if (bad_h) return fail(WOS_ERR_INVALID_ARGUMENT, "face index out of range [0, nV)");
    return 0;
}

int SceneImpl::build(cudaStream_t st) {
    const int rc = dim == 2 ? build_geometry<2>(*this, st) : build_geometry<3>(*this, st);
    ++generation;
    return rc;
}

SceneView SceneImpl::view() const {
    SceneView v{};
    v.dim = dim;
    v.nV = nV;
    v.nF = nF;
    v.V = V;
    v.F = F;
    v.N = N;
    v.g = g;
    v.seg = seg;
    v.seginv = seginv;
    v.tri = tri;
    v.nNodes = nNodes;
    v.node = node;
    // In input order the leaf-ordered copies equal the primitive arrays: point
    // the kernels at one copy so the tree's leaf tests and the warm-start /
    // record lookups share cache lines.
    v.lseg = prim_order == 1 ? seg : lseg;
    v.lseginv = prim_order == 1 ? seginv : lseginv;
    v.ltri = prim_order == 1 ? tri : ltri;
    v.lorig = lorig;
    for (int k = 0; k < 3; ++k) {
        v.lo[k] = lo[k];
        v.hi[k] = hi[k];
    }
    v.half_min_extent = half_min_extent;
    v.max_extent = 0.0f;
    for (int k = 0; k < dim; ++k) {
        v.max_extent = fmaxf(v.max_extent, hi[k] - lo[k]);
        v.centre[k] = (lo[k] + hi[k]) * 0.5f;
    }
    for (int k = dim; k < 3; ++k) v.centre[k] = 0.0f;
    v.src_type = src_type;
    for (int k = 0; k < 5; ++k) v.src[k] = src[k];
    v.cdf = cdf;
    v.n_cdf = n_cdf;
    v.guide = guide;
    v.n_guide = n_guide;
    v.wt_levels = wt_levels;
    for (int k = 0; k < 8; ++k) {
        v.wt_count[k] = wt_count[k];
        v.wt_off[k] = wt_off[k];
    }
    v.wt_box = wt_box;
    v.wt_slab = wt_slab;
    v.wt_obb = wt_obb;
    return v;
}

}  // namespace wosd
