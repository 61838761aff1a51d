// Float64 droplet trace: compiled with -fmad=false, so every operation rounds
// like the reference's float64 numba code (no fused multiply-add).
#define PGE_REAL double
#define PGE_VARIANT f64
#include "pge_droplets.cuh"

namespace pge {
cudaError_t launch_droplets_f64(const DropArgs &a, int blocks, int threads, cudaStream_t st)
{
    if (a.p.lateral_rate > 0.0) return launch_droplets_f64_lateral(a, blocks, threads, st);
    if (a.R) return launch_droplets_f64_route(a, blocks, threads, st);
    if (!a.ledger && a.minb >= 2)  // record only, at most 128 registers: a wave's droplets one per warp
        f64::droplet_kernel<2, false><<<blocks, threads, 0, st>>>(a);
    else if (!a.ledger)
        f64::droplet_kernel<1, false><<<blocks, threads, 0, st>>>(a);
    else if (a.minb >= 2)
        f64::droplet_kernel<2, true><<<blocks, threads, 0, st>>>(a);
    else
        f64::droplet_kernel<1, true><<<blocks, threads, 0, st>>>(a);
    return cudaPeekAtLastError();
}
cudaError_t launch_droplets_f64_route(const DropArgs &a, int blocks, int threads, cudaStream_t st)
{
    if (a.ledger)
        f64::droplet_kernel<1, true, false, true><<<blocks, threads, 0, st>>>(a);
    else
        f64::droplet_kernel<1, false, false, true><<<blocks, threads, 0, st>>>(a);
    return cudaPeekAtLastError();
}
int droplet_blocks_per_sm_f64_route(int threads, bool ledger)
{
    int n = 0;
    const cudaError_t e = ledger ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true, false, true>, threads, 0)
                                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, false, false, true>, threads, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
// the bank cut (erosion.lateral_rate > 0), with or without the route
cudaError_t launch_droplets_f64_lateral(const DropArgs &a, int blocks, int threads, cudaStream_t st)
{
    if (a.R && a.ledger)
        f64::droplet_kernel<1, true, false, true, true><<<blocks, threads, 0, st>>>(a);
    else if (a.R)
        f64::droplet_kernel<1, false, false, true, true><<<blocks, threads, 0, st>>>(a);
    else if (a.ledger)
        f64::droplet_kernel<1, true, false, false, true><<<blocks, threads, 0, st>>>(a);
    else
        f64::droplet_kernel<1, false, false, false, true><<<blocks, threads, 0, st>>>(a);
    return cudaPeekAtLastError();
}
int droplet_blocks_per_sm_f64_lateral(int threads, bool ledger, bool route)
{
    int n = 0;
    const cudaError_t e =
        route ? (ledger ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true, false, true, true>, threads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, false, false, true, true>, threads, 0))
              : (ledger ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true, false, false, true>, threads, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, false, false, false, true>, threads, 0));
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
cudaError_t launch_droplets_f64_tape(const DropArgs &a, int blocks, int threads, cudaStream_t st)
{
    f64::droplet_kernel<1, true, true><<<blocks, threads, 0, st>>>(a);
    return cudaPeekAtLastError();
}
int droplet_blocks_per_sm_f64_tape(int threads)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true, true>, threads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
int droplet_blocks_per_sm_f64(int threads, int minb, bool ledger)
{
    int n = 0;
    cudaError_t e = !ledger     ? (minb >= 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<2, false>, threads, 0)
                                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, false>, threads, 0))
                    : minb >= 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<2, true>, threads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true>, threads, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
}  // namespace pge

// ---------------------------------------------------------------------------
// parity hooks: the float64 droplet kernel's own face-crossing and trig code,
// run over arrays (pge_cubesphere_map, pge_crmath)
// ---------------------------------------------------------------------------
namespace pge {
namespace {
__global__ void crmath_kernel(int op, long long n, const double *x, double *y)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = x[i];
        switch (op) {
        case 0: y[i] = cr::d_tan(v); break;
        case 1: y[i] = cr::d_atan(v); break;
        case 2: y[i] = cr::d_sin(v); break;
        case 3: y[i] = cr::d_cos(v); break;
        // CUDA's own functions, for comparison only (the trace does not use them)
        case 4: y[i] = tan(v); break;
        case 5: y[i] = atan(v); break;
        case 6: y[i] = sin(v); break;
        default: y[i] = cos(v); break;
        }
    }
}

__global__ void cubesphere_kernel(int op, long long n, int32_t *face, double *uv, double *ab, double *xyz)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (op == 0) {
            double x, y, z;
            f64::to_sphere(face[i], uv[2 * i], uv[2 * i + 1], x, y, z);
            xyz[3 * i] = x;
            xyz[3 * i + 1] = y;
            xyz[3 * i + 2] = z;
        } else if (op == 1) {
            double u, v;
            face[i] = f64::from_sphere(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], u, v);
            uv[2 * i] = u;
            uv[2 * i + 1] = v;
        } else {
            double u = uv[2 * i], v = uv[2 * i + 1], a = ab[2 * i], b = ab[2 * i + 1];
            face[i] = f64::transfer_velocity(face[i], u, v, a, b);
            uv[2 * i] = u;
            uv[2 * i + 1] = v;
            ab[2 * i] = a;
            ab[2 * i + 1] = b;
        }
    }
}
}  // namespace

cudaError_t launch_crmath(int op, long long n, const double *x, double *y, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    crmath_kernel<<<(int)blocks, 256, 0, st>>>(op, n, x, y);
    return cudaPeekAtLastError();
}

cudaError_t launch_cubesphere(int op, long long n, int32_t *face, double *uv, double *ab, double *xyz, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    cubesphere_kernel<<<(int)blocks, 256, 0, st>>>(op, n, face, uv, ab, xyz);
    return cudaPeekAtLastError();
}

// the same evaluations on the host (this file's host code is compiled without contraction)
void crmath_host(int op, long long n, const double *x, double *y)
{
    for (long long i = 0; i < n; i++) {
        const double v = x[i];
        y[i] = op == 0 ? cr::cr_tan(v) : op == 1 ? cr::cr_atan(v) : op == 2 ? cr::cr_sin(v) : cr::cr_cos(v);
    }
}
}  // namespace pge
