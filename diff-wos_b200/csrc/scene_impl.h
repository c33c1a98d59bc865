// Internal scene object behind the opaque wos_scene_t handle, and the
// library's error plumbing.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "wos_device.cuh"

namespace wosd {

// Records the message for wos_last_error_string() and returns code.
int fail(int code, const std::string &msg);
int fail_cuda(cudaError_t e, const char *where);

void build_g_cdf(std::vector<float> &cdf, int n);
void build_g_guide(const std::vector<float> &cdf, int ng, std::vector<unsigned short> &guide);

// Owns every device buffer of one scene.  Geometry buffers are immutable
// between wos_scene_update_* calls.
struct SceneImpl {
    int dim = 0, nV = 0, nF = 0;
    int device = 0;
    float *V = nullptr;
    int *F = nullptr;
    float *N = nullptr;
    float *g = nullptr;
    float4 *seg = nullptr;
    float *seginv = nullptr;
    float4 *tri = nullptr;
    int nNodes = 0;
    int depth = 0;
    // Primitive order of the trees (decided at the first build, kept when
    // vertices move): 0 Morton, 1 input order (a polyline whose segments
    // follow each other), 2 Hilbert.
    int prim_order = -1;
    float4 *node = nullptr;
    float4 *lseg = nullptr;
    float *lseginv = nullptr;
    float4 *ltri = nullptr;
    int *lorig = nullptr;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    float half_min_extent = 0;
    int src_type = 0;
    float src[5] = {0, 0, 0, 0, 0};
    float *cdf = nullptr;
    int n_cdf = 0;
    unsigned short *guide = nullptr;
    int n_guide = 0;
    int wt_levels = 0;
    int wt_count[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int wt_off[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float4 *wt_box = nullptr;
    float4 *wt_slab = nullptr;
    float4 *wt_obb = nullptr;
    size_t wt_n[3] = {0, 0, 0};  // float4 counts allocated for wt_box, wt_slab, wt_obb
    // Incremented by every build and source change: the by-value fields of
    // view() (bounding box, extents, source) may have changed since a view
    // was taken.
    unsigned long long generation = 0;

    int allocate(cudaStream_t st);
    int check_indices(cudaStream_t st);
    int build(cudaStream_t st);
    void release(cudaStream_t st);
    SceneView view() const;
};

}  // namespace wosd

struct wos_scene_s {
    wosd::SceneImpl impl;
};
