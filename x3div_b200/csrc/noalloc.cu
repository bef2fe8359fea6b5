// Allocation-free divergence: x3d_divergence_noalloc.
//
// Some hosts cannot allocate device memory once their time loop runs: a
// Fortran host that maps its whole device working set up front through
// OpenACC data regions and runs under a fixed device-memory budget, or a
// solver that shares the GPU with other work and must not take memory (or
// risk an allocation failure) in the middle of a step.  This entry point
// gives them the divergence stage without any allocation: its five
// intermediate fields live in one fixed array compiled into the library
// instead of in context scratch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "x3d_internal.h"

namespace {

// Largest grid (points per field) the fixed array holds: 64^3.
constexpr size_t kMaxPoints = X3D_NOALLOC_MAX_POINTS;
constexpr int kFields = 5;

// The intermediate fields, kFields * kMaxPoints doubles (10 MiB).  A GPU holds
// this array from the first x3d_divergence_noalloc call on it (when the
// library's module is loaded there) until the process exits.
static __device__ __align__(256) unsigned char g_div_scratch[kFields * kMaxPoints * sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
// Per device: the CUDA context the address was looked up in, and the address.
// A device reset (cudaDeviceReset, or a primary context released and made
// again) gives the device a new context in which the array sits elsewhere,
// so the address is looked up again whenever the current context differs.
CUcontext g_ctx[kMaxDevices] = {};
void *g_addr[kMaxDevices] = {};

using CtxGetCurrent = CUresult (*)(CUcontext *);

CtxGetCurrent ctx_get_current()
{
    static CtxGetCurrent fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrent>(p);
    }
    return fn;
}

// Device address of the array on the current device.  Host code must not use
// the array's name as an address (it names a host-side stand-in); the
// address comes from cudaGetSymbolAddress, looked up once per device and
// context.  The first lookup on a device also loads the library's module
// there (under lazy module loading), which reserves the array.
int scratch_address(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices) return X3D_EINVAL;
    std::lock_guard<std::mutex> lock(g_mutex);
    CUcontext cur = nullptr;
    const CtxGetCurrent get = ctx_get_current();
    if (!get || get(&cur) != CUDA_SUCCESS || !cur) return X3D_ECUDA;
    if (!g_addr[device] || g_ctx[device] != cur) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_div_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return X3D_ECUDA;
        }
        g_addr[device] = p;
        g_ctx[device] = cur;
    }
    *out = g_addr[device];
    return X3D_OK;
}

bool on_device(const void *p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int x3d_divergence_noalloc(x3d_ctx ctx, double *pp3, const void *ux1, const void *uy1,
                                      const void *uz1)
{
    using namespace x3d;
    if (!ctx) return X3D_EINVAL;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(ctx, X3D_ECUDA, "cudaSetDevice failed");
    if (!pp3 || !ux1 || !uy1 || !uz1) return set_error(ctx, X3D_EINVAL, "null field");
    if (!ctx->periodic_all)
        return set_error(ctx, X3D_EUNSUPPORTED, "the divergence needs periodic boundaries in every direction");
    if (!on_device(pp3) || !on_device(ux1) || !on_device(uy1) || !on_device(uz1))
        return set_error(ctx, X3D_EINVAL,
                         "x3d_divergence_noalloc takes device pointers only (staging host arrays would allocate)");
    if (ctx->npts() > kMaxPoints)
        return set_error(ctx, X3D_EINVAL,
                         "grid has " + std::to_string(ctx->npts()) + " points; x3d_divergence_noalloc holds at most " +
                             std::to_string(kMaxPoints) + " (X3D_NOALLOC_MAX_POINTS)");
    void *base = nullptr;
    int rc = scratch_address(ctx->device, &base);
    if (rc) return set_error(ctx, rc, "cudaGetSymbolAddress of the divergence scratch array failed");
    // five fields of the context precision, packed; each field's bytes are a
    // multiple of 16 whenever the fused kernels accept the grid
    void *s[kFields];
    for (int i = 0; i < kFields; ++i)
        s[i] = static_cast<unsigned char *>(base) + (size_t)i * ctx->npts() * ctx->elem();
    const void *u[3] = {ux1, uy1, uz1};
    rc = fused_divergence_scratch(ctx, pp3, u, s);
    if (rc == X3D_EUNSUPPORTED)
        return set_error(ctx, X3D_EUNSUPPORTED,
                         "x3d_divergence_noalloc needs a grid the fused stage kernels take (x extent times the "
                         "element size a multiple of 16 bytes); use x3d_divergence");
    return rc;
}
