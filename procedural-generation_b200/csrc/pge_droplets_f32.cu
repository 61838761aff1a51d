// Float32 droplet trace (the fast path); the ledger stays float64.
#define PGE_REAL float
#define PGE_VARIANT f32
#include "pge_droplets.cuh"

namespace pge {
cudaError_t launch_droplets_f32(const DropArgs &a, int blocks, int threads, cudaStream_t st)
{
    if (!a.ledger)
        f32::droplet_kernel<1, false><<<blocks, threads, 0, st>>>(a);
    else if (a.minb >= 2)
        f32::droplet_kernel<2, true><<<blocks, threads, 0, st>>>(a);
    else
        f32::droplet_kernel<1, true><<<blocks, threads, 0, st>>>(a);
    return cudaPeekAtLastError();
}
int droplet_blocks_per_sm_f32(int threads, int minb, bool ledger)
{
    int n = 0;
    cudaError_t e = !ledger     ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f32::droplet_kernel<1, false>, threads, 0)
                    : minb >= 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f32::droplet_kernel<2, true>, threads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f32::droplet_kernel<1, true>, threads, 0);
    if (e != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}
}  // namespace pge
