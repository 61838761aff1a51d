// pge_static.cu -- the thermal pass without a caller workspace.
//
// pge_thermal needs a caller-allocated workspace.  Some callers cannot
// allocate device memory at all: a host application that owns the whole
// device heap through its own pool and forbids any other allocation, or a
// loop that must not pay cudaMalloc's latency and implicit device
// synchronisation.  pge_thermal_noalloc serves them: its scratch (five
// float64 values per cell) is a file-scope __device__ array of fixed size,
// PGE_NOALLOC_MAX_CELLS cells (10 MiB), which every GPU that loads the
// library holds until the process exits.
//
// Host code cannot pass that array's name to a kernel: in host code the
// name is only a host-side stand-in, not a device address.  So the first
// call on each device, with that device current, looks its device address
// up with cudaGetSymbolAddress (checked) and keeps it for later calls on the
// same device.  That first call should come before any stream capture.  The
// kept address belongs to the device's primary context: after
// cudaDeviceReset (or anything else that destroys that context) the module
// is loaded again and the array may move, so a process that resets a device
// must not call this entry point on it again.
//
// Every call shares the one array and it keeps the last call's contents;
// nothing in it needs to start at zero (each pass writes every scratch value
// it reads).  Calls whose work overlaps on the GPU -- on different streams,
// or from different host threads -- race on the array: order them.
#include <mutex>

#include "pge_internal.cuh"
#include "pge_maps.cuh"

namespace pge {
namespace {

__device__ __align__(256) double g_thermal_scratch[5 * (size_t)PGE_NOALLOC_MAX_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch[kMaxDevices] = {};

// device address of the static scratch on the current device (set up once per device)
cudaError_t scratch_address(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_thermal_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[dev] = static_cast<double *>(p);
    }
    *out = g_scratch[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace pge

extern "C" PGE_API int pge_thermal_noalloc(const PgeGrid *g, PgeState *s, double thermal_rate, double creep_rate,
                                           double thermal_max, double talus_soft, double talus_hard, double dep_floor, void *stream)
{
    using namespace pge;
    int r;
    if ((r = check_shape(g))) return r;  // the same grid rules as pge_thermal
    const long long NE = g->N + 2LL * g->H;
    const long long n = (long long)g->F * NE * NE;
    if (n > PGE_NOALLOC_MAX_CELLS)
        return pge_set_error(PGE_E_ARG, "thermal_noalloc: %lld cells exceed the static scratch of %d cells (use pge_thermal)", n,
                             PGE_NOALLOC_MAX_CELLS);
    if (!s || !s->height || !s->sediment || !s->hardness || !s->metric || !s->base)
        return pge_set_error(PGE_E_ARG, "thermal_noalloc: state has a NULL array");
    double *tb = nullptr;
    cudaError_t e = scratch_address(&tb);
    if (e != cudaSuccess) return pge_set_error(PGE_E_CUDA, "thermal_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    const float soft = (float)talus_soft, diff = (float)(talus_hard - talus_soft);
    thermal_on_scratch(*g, *s, tb, n, thermal_rate, creep_rate, thermal_max, soft, diff, dep_floor, (cudaStream_t)stream);
    e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : pge_set_error(PGE_E_CUDA, "thermal_noalloc: %s", cudaGetErrorString(e));
}
