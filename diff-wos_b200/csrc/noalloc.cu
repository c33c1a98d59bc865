// wos_solve_noalloc: the per-point solve without any device allocation.
//
// Some callers may not allocate device memory at all: host applications that
// own the whole device through their own memory pool and forbid plug-ins from
// calling cudaMalloc (a raw allocation fragments their pool and synchronises
// the device), latency-critical loops that cannot afford the implicit
// synchronisation and unpredictable cost of cudaMalloc / cudaFree, and
// processes running under a hard device-memory quota that want the library's
// footprint fixed when it loads.  For them this entry point keeps its scratch
// (the walk-queue counter and the per-walk values) in a fixed array compiled
// into the library, so a call allocates nothing.
//
// The array costs every GPU that loads the library 16 MiB + 256 bytes until
// the process exits.  Its device address is looked up (cudaGetSymbolAddress)
// on every call, with the caller's device current: the lookup is a host-side
// table read, and a fresh lookup stays valid across a device reset or a
// re-created primary context, where a cached address would dangle.  All calls
// share the one array: calls that overlap on the GPU race on it.
#include "../../include/wos_b200.h"
#include "scene_impl.h"
#include "walk.h"

namespace wosd {

constexpr size_t NOALLOC_COUNTER_BYTES = 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_COUNTER_BYTES + (size_t)WOS_NOALLOC_MAX_WALKS * sizeof(float);

// [queue counter (256 B)][per-walk values (WOS_NOALLOC_MAX_WALKS floats)]
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of the array on the current device.  In host code the
// symbol g_noalloc_scratch is only a host-side stand-in, so kernels are given
// this address, never the symbol.
static int noalloc_scratch(char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(noalloc scratch)");
    *out = static_cast<char *>(p);
    return 0;
}

}  // namespace wosd

using namespace wosd;

extern "C" int wos_solve_noalloc(wos_scene_t scene, const float *P, int n, const wos_params *p, double *mean,
                                 double *var, wos_stream_t stream) {
    if (scene == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (p == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "params is NULL");
    if (p->nwalks < 1) return fail(WOS_ERR_INVALID_ARGUMENT, "nwalks must be >= 1");
    if (p->nsteps < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "nsteps must be >= 0");
    if (!(p->epsilon >= 0.0f)) return fail(WOS_ERR_INVALID_ARGUMENT, "epsilon must be >= 0");
    if (n < 0) return fail(WOS_ERR_INVALID_ARGUMENT, "n must be >= 0");
    const long long walks = (long long)n * (long long)p->nwalks;
    if (walks > (long long)WOS_NOALLOC_MAX_WALKS)
        return fail(WOS_ERR_WORKSPACE,
                    "wos_solve_noalloc: n * nwalks = " + std::to_string(walks) +
                        " exceeds the fixed scratch capacity of " + std::to_string((long long)WOS_NOALLOC_MAX_WALKS) +
                        " walks; split the points or use wos_solve");
    if (n == 0) return 0;
    for (const void *ptr : {(const void *)P, (const void *)mean, (const void *)var}) {
        if (ptr == nullptr) continue;
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();
            return fail(WOS_ERR_INVALID_ARGUMENT, "P, mean and var must be device pointers");
        }
    }
    if (P == nullptr || mean == nullptr) return fail(WOS_ERR_INVALID_ARGUMENT, "P and mean must not be NULL");
    char *base = nullptr;
    if (int rc = noalloc_scratch(&base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(base);
    float *vals = reinterpret_cast<float *>(base + NOALLOC_COUNTER_BYTES);
    // launch_walk zeroes the counter on the stream before the kernel; every
    // per-walk value is overwritten, so no other state carries over.
    WalkOut o{vals, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (int rc = launch_walk(scene->impl, P, walks, *p, false, o, counter, st)) return rc;
    return launch_reduce(vals, n, p->nwalks, mean, var, st);
}
