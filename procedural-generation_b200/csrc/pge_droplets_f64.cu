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
    if (!a.ledger)
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
    cudaError_t e = !ledger     ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, false>, threads, 0)
                    : minb >= 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<2, true>, threads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f64::droplet_kernel<1, true>, threads, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
}  // namespace pge
