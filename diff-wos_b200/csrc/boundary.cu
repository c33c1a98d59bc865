// Image-space boundary term of shape derivatives (WoSBoundary,
// wos/wos_boundary.py:11-31).  Boundary points are drawn uniformly by length
// (2D) or area (3D) over the whole boundary, npixels x nwalks of them; each
// one that lands in a detector pixel contributes -g(x) (n . dx) / pdf to that
// pixel, divided by the detector measure and nwalks, where dx is the motion
// of the sampled point (the lerp / barycentric mix of its vertices' motion)
// and n the primitive's normal (wos/scene.py:435-449, wos/scene3d.py:241-262).
// Its value is zero; it exists for its derivative with respect to vertex
// positions, computed here in forward mode (a derivative image for a given
// vertex motion) and in reverse mode (the vertex gradient of a weighting of
// the pixels).
#include <cub/cub.cuh>

#include "../../include/wos_b200.h"
#include "scene_impl.h"
#include "walk.h"

namespace wosd {

// Primitive measure: segment length, or triangle area.
template <int D>
__global__ void k_prim_measure(const float *__restrict__ V, const int *__restrict__ F, int nF, double *m) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    if (D == 2) {
        const float *a = V + 2 * F[2 * f], *b = V + 2 * F[2 * f + 1];
        const double dx = (double)b[0] - a[0], dy = (double)b[1] - a[1];
        m[f] = sqrt(dx * dx + dy * dy);
    } else {
        const float *a = V + 3 * F[3 * f], *b = V + 3 * F[3 * f + 1], *c = V + 3 * F[3 * f + 2];
        const double u[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
        const double v[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
        const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
        m[f] = 0.5 * sqrt(x * x + y * y + z * z);
    }
}

struct DetectorCfg {
    float vmin[2], vmax[2];
    int res[2];
    int au, av, slab;
    float slab_c, slab_h;
    float size;
    double pdf_scale;  // 1 / pdf = total measure * pdf_scale
};

// A sample's primitive (from the inclusive prefix sums `cdf` of the
// measures) and the reused uniform inside that primitive's interval.
__device__ __forceinline__ int sample_prim(const double *__restrict__ cdf, int nF, double target, float &t) {
    int lo = 0, hi = nF - 1;  // first f with cdf[f] > target
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cdf[mid] > target)
            hi = mid;
        else
            lo = mid + 1;
    }
    const double base = lo > 0 ? cdf[lo - 1] : 0.0;
    const double w = cdf[lo] - base;
    t = w > 0.0 ? (float)((target - base) / w) : 0.0f;
    t = fminf(fmaxf(t, 0.0f), 0x1.fffffep-1f);
    return lo;
}

template <int D>
__global__ void k_boundary(const float *__restrict__ V, const int *__restrict__ F, const float *__restrict__ g, int nF,
                           const double *__restrict__ cdf, DetectorCfg det, long long nsamples, int nwalks, Rng rng,
                           const float *__restrict__ tV, double *img_tan, const float *__restrict__ dLdI,
                           double *dV_acc) {
    const double total = cdf[nF - 1];
    const long long npix = (long long)det.res[0] * det.res[1];
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nsamples;
         s += (long long)gridDim.x * blockDim.x) {
        const uint4 r = philox(rng, (uint32_t)s, (uint32_t)(s >> 32), 0, ROLE_BOUNDARY);
        float t;
        const int f = sample_prim(cdf, nF, (double)wosm::u01(r.x) * total, t);
        int vid[3] = {0, 0, 0};
        float wts[3] = {0.0f, 0.0f, 0.0f}, x[3] = {0.0f, 0.0f, 0.0f}, n[3] = {0.0f, 0.0f, 0.0f};
        float val;
        if (D == 2) {
            vid[0] = F[2 * f];
            vid[1] = F[2 * f + 1];
            const float ax = V[2 * vid[0]], ay = V[2 * vid[0] + 1];
            const float abx = V[2 * vid[1]] - ax, aby = V[2 * vid[1] + 1] - ay;
            x[0] = fmaf(t, abx, ax);
            x[1] = fmaf(t, aby, ay);
            wts[0] = 1.0f - t;
            wts[1] = t;
            val = fmaf(t, g[vid[1]] - g[vid[0]], g[vid[0]]);
            const float l = sqrtf(fmaf(abx, abx, aby * aby));
            n[0] = -aby / l;
            n[1] = abx / l;
        } else {
            for (int k = 0; k < 3; ++k) vid[k] = F[3 * f + k];
            const float su = sqrtf(wosm::u01(r.y)), r2 = wosm::u01(r.z);
            const float u = su * (1.0f - r2), v = su * r2;
            wts[0] = 1.0f - u - v;
            wts[1] = u;
            wts[2] = v;
            float ab[3], ac[3];
            for (int k = 0; k < 3; ++k) {
                const float a = V[3 * vid[0] + k];
                ab[k] = V[3 * vid[1] + k] - a;
                ac[k] = V[3 * vid[2] + k] - a;
                x[k] = fmaf(u, ab[k], fmaf(v, ac[k], a));
            }
            val = fmaf(wts[0], g[vid[0]], fmaf(u, g[vid[1]], v * g[vid[2]]));
            float c[3];
            cross3(ab[0], ab[1], ab[2], ac[0], ac[1], ac[2], c[0], c[1], c[2]);
            const float l = sqrtf(dot3(c[0], c[1], c[2], c[0], c[1], c[2]));
            for (int k = 0; k < 3; ++k) n[k] = -c[k] / l;
        }
        // Detector.index (wos/scene.py:18-24, wos/scene3d.py:35-46)
        const int iu = (int)(fmaf((x[det.au] - det.vmin[0]) / (det.vmax[0] - det.vmin[0]), (float)det.res[0], 0.5f));
        const int iv = (int)(fmaf((x[det.av] - det.vmin[1]) / (det.vmax[1] - det.vmin[1]), (float)det.res[1], 0.5f));
        bool ok = iu >= 0 && iu < det.res[0] && iv >= 0 && iv < det.res[1];
        if (det.slab >= 0) ok = ok && fabsf(x[det.slab] - det.slab_c) < det.slab_h;
        const long long idx = (long long)iu + (long long)(det.res[1] - iv) * det.res[0];
        if (!ok || idx < 0 || idx >= npix) continue;
        // -val / pdf / (size * nwalks), pdf = 1 / (total measure * pdf_scale)
        const double w = -(double)val * total * det.pdf_scale / ((double)det.size * nwalks);
        if (tV != nullptr && img_tan != nullptr) {
            double nd = 0.0;
            for (int j = 0; j < D; ++j)
                for (int k = 0; k < D; ++k) nd += (double)n[k] * wts[j] * tV[(size_t)vid[j] * D + k];
            atomicAdd(&img_tan[idx], w * nd);
        }
        if (dLdI != nullptr && dV_acc != nullptr) {
            const double cw = (double)dLdI[idx] * w;
            if (cw != 0.0)
                for (int j = 0; j < D; ++j)
                    for (int k = 0; k < D; ++k) atomicAdd(&dV_acc[(size_t)vid[j] * D + k], cw * n[k] * wts[j]);
        }
    }
}

int launch_boundary(const SceneImpl &S, const wos_detector &d, int nwalks, uint64_t seed, const float *tV,
                    double *img_tan, const float *dLdI, double *dV_acc, cudaStream_t st) {
    const int nF = S.nF;
    if (nF == 0) return 0;
    double *m = nullptr, *cdf = nullptr;
    size_t tmp_bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, m, cdf, nF, st);
    cudaError_t e = cudaMallocAsync((void **)&m, sizeof(double) * 2 * (size_t)nF + tmp_bytes + 256, st);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMallocAsync(boundary)");
    cdf = m + nF;
    void *tmp = (void *)(((uintptr_t)(cdf + nF) + 255) & ~(uintptr_t)255);
    const int TB = 256;
    if (S.dim == 2)
        k_prim_measure<2><<<(nF + TB - 1) / TB, TB, 0, st>>>(S.V, S.F, nF, m);
    else
        k_prim_measure<3><<<(nF + TB - 1) / TB, TB, 0, st>>>(S.V, S.F, nF, m);
    e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, m, cdf, nF, st);
    if (e == cudaSuccess) {
        DetectorCfg c;
        for (int k = 0; k < 2; ++k) {
            c.vmin[k] = d.vmin[k];
            c.vmax[k] = d.vmax[k];
            c.res[k] = d.res[k];
        }
        c.au = d.axis_u;
        c.av = d.axis_v;
        c.slab = d.slab_axis;
        c.slab_c = d.slab_center;
        c.slab_h = d.slab_half_width;
        c.size = d.size;
        // the reference's 3D pdf divides by |ab x ac| = 2 * area (wos/scene3d.py:262)
        c.pdf_scale = (S.dim == 3 && (d.flags & WOS_DETECTOR_REFERENCE_AREA_PDF)) ? 2.0 : 1.0;
        const long long ns = (long long)d.res[0] * d.res[1] * nwalks;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = (int)std::min<long long>((ns + TB - 1) / TB, (long long)sms * 16);
        const Rng rng = make_rng(seed);
        if (S.dim == 2)
            k_boundary<2><<<grid, TB, 0, st>>>(S.V, S.F, S.g, nF, cdf, c, ns, nwalks, rng, tV, img_tan, dLdI, dV_acc);
        else
            k_boundary<3><<<grid, TB, 0, st>>>(S.V, S.F, S.g, nF, cdf, c, ns, nwalks, rng, tV, img_tan, dLdI, dV_acc);
        e = cudaGetLastError();
    }
    cudaFreeAsync(m, st);
    if (e != cudaSuccess) return fail_cuda(e, "k_boundary");
    return 0;
}

}  // namespace wosd
