// pge_ordered.cu -- the exact, droplet-ordered apply of one wave's change lists.
//
// The reference applies every particle's change list serially in particle
// order against the live terrain (bake/globe/erosion/particle.py:821-1042).
// Entry k of droplet p reads the live terrain of its own cell c_k, of the
// next entry's cell c_{k+1} (erosion floor, final-deposit ceiling) and of
// the previous step entry's cell c_{k-1} (step-deposit ceiling), and writes
// c_k.  So the apply of droplet p depends on earlier droplets only through
// the cells in its sliding window {c_{k-1}, c_k, c_{k+1}}.
//
// Here every droplet of a wave applies its own list on its own thread, and
// each cell is handed from droplet to droplet in droplet order:
//   * the entries of the wave are sorted by (cell, droplet, entry) and each
//     entry learns D = the number of distinct earlier droplets that visit
//     its cell, and whether it is its droplet's last visit there;
//   * a droplet acquires a cell (waits until done[cell] == epoch + D) one
//     entry before it writes there (the erosion floor and final-deposit
//     ceiling read the next entry's cell), and releases it (done[cell] =
//     epoch + D + 1) right after its last write there; the step-deposit
//     ceiling of the following entry uses the live surface snapshotted at
//     that write -- exactly what the serial order reads, since no other
//     droplet runs between two entries of one droplet; the stockpile (death)
//     cell is released after the stockpile update.
// Every read and write of a cell therefore happens in exactly the
// reference's serial order, and the float64 arithmetic is the reference's
// (this file is compiled without FMA contraction).  Waits are bounded: a
// wait that gives up sets an error flag the host reports.
#include <cub/cub.cuh>
#include <cuda/atomic>

#include "pge_internal.cuh"
#include "pge_ordered.cuh"

namespace pge {

namespace {
inline int grid_for(long long n, int threads = 256)
{
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}

constexpr long long kSpinLimit = 1LL << 22;  // ~ seconds of polling: far beyond any real hand-off

// wait until the D earlier droplets of this wave that visit cell c have released it
__device__ __forceinline__ bool acquire(unsigned long long *done, long long c, unsigned long long epoch, int D, int *error)
{
    if (D == 0) return true;  // the first visitor of the wave: every earlier wave has finished
    const unsigned long long want = epoch + (unsigned long long)D;
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(done[c]);
    // poll with relaxed loads; one acquire fence once the hand-off is seen
    for (long long i = 0; i < kSpinLimit; i++) {
        if (r.load(cuda::memory_order_relaxed) == want) {
            cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
            return true;
        }
        if ((i & 255) == 255) {
            if (*(volatile int *)error) return false;  // another wait gave up: stop waiting
            __nanosleep(32);
        }
    }
    atomicExch(error, 1);
    return false;
}

__device__ __forceinline__ void release(unsigned long long *done, long long c, unsigned long long value)
{
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(done[c]);
    r.store(value, cuda::memory_order_release);
}

enum { OS_CLAMPED, OS_TOPEND, OS_DEFICIT, OS_LOSTOFF, OS_ERODED, OS_DEPOSITED, OS_N };
}  // namespace

// ---------------------------------------------------------------------------
// ranks
// ---------------------------------------------------------------------------
__global__ void ordered_keys_kernel(long long nslots, int cap, const int32_t *cell, const int64_t *count, int kbits, int pbits,
                                    unsigned long long invalid, unsigned long long *keys, int32_t *vals)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nslots; s += (long long)gridDim.x * blockDim.x) {
        const long long q = s / cap, k = s - q * cap;
        if (k < count[q])
            keys[s] = ((unsigned long long)cell[s] << (pbits + kbits)) | ((unsigned long long)q << kbits) | (unsigned long long)k;
        else
            keys[s] = invalid;
        vals[s] = (int32_t)s;
    }
}

__global__ void ordered_flags_kernel(long long nslots, const unsigned long long *keys, int kbits, int pbits,
                                     unsigned long long invalid, int32_t *runstart, int32_t *segpos)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        int rs = 0, sp = 0;
        if (k != invalid) {
            const unsigned long long run = k >> kbits, seg = k >> (kbits + pbits);
            if (i == 0) {
                rs = 1;
                sp = 0;
            } else {
                const unsigned long long kp = keys[i - 1];
                rs = (kp >> kbits) != run;
                sp = (kp >> (kbits + pbits)) != seg ? (int)i : 0;
            }
        }
        runstart[i] = rs;
        segpos[i] = sp;
    }
}

__global__ void ordered_rank_kernel(long long nslots, const unsigned long long *keys, const int32_t *vals, unsigned long long invalid,
                                    int kbits, const int32_t *runscan, const int32_t *segscan, int32_t *D, uint8_t *last)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k == invalid) continue;
        const int32_t s = vals[i];
        D[s] = runscan[i] - runscan[segscan[i]];
        bool lst = true;
        if (i + 1 < nslots) {
            const unsigned long long kn = keys[i + 1];
            lst = kn == invalid || (kn >> kbits) != (k >> kbits);
        }
        last[s] = lst ? 1 : 0;
    }
}

struct MaxOp {
    __device__ __forceinline__ int32_t operator()(const int32_t a, const int32_t b) const { return a > b ? a : b; }
};

size_t ordered_temp_bytes(long long nslots)
{
    size_t a = 0, b = 0, c = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long *)nullptr, (unsigned long long *)nullptr, (int32_t *)nullptr,
                                    (int32_t *)nullptr, (int)nslots);
    cub::DeviceScan::InclusiveSum(nullptr, b, (int32_t *)nullptr, (int32_t *)nullptr, (int)nslots);
    cub::DeviceScan::InclusiveScan(nullptr, c, (int32_t *)nullptr, (int32_t *)nullptr, MaxOp{}, (int)nslots);
    size_t m = a > b ? a : b;
    return m > c ? m : c;
}

// ---------------------------------------------------------------------------
// the ordered apply
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) ordered_apply_kernel(const OrderedArgs a)
{
    __shared__ unsigned long long sstat[OS_N];
    for (int k = threadIdx.x; k < OS_N; k += blockDim.x) sstat[k] = 0ull;
    __syncthreads();
    const PgeParams &p = a.p;
    // one droplet per warp (its lane 0): a droplet waits on earlier droplets' hand-offs, and lanes of
    // one warp waiting on each other would serialise the warp
    const long long T = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const bool lane0 = (threadIdx.x & 31) == 0;
    for (long long q = w0; lane0 && q < a.nw; q += T) {
        const int K = (int)a.count[q];
        if (K <= 0) continue;
        const long long b0 = q * a.cap;
        double deficit = 0.0, surplus = 0.0;
        long long death = -1;
        bool has_prev = false;
        double prev_live = 0.0;  // the previous step entry's cell right after its write (the step-deposit ceiling)
        long long clamped = 0, eroded_fx = 0, deposited_fx = 0;
        // entry descriptors: the current one and the next, loaded before any wait
        long long c = a.cell[b0];
        int Dc = a.D[b0];
        bool lastc = a.last[b0];
        double dlt = a.delta[b0];
        float vv = a.vol[b0];
        float m0 = a.mom[2 * b0], m1 = a.mom[2 * b0 + 1];
        long long nc = -1;
        int Dn = 0;
        if (K > 1) {
            nc = a.cell[b0 + 1];
            Dn = a.D[b0 + 1];
        }
        bool ok = true;
        bool have_c = false;       // the current entry's cell is acquired
        bool acc_known = false;    // acc_c holds its net change (read when it was acquired as the next cell)
        double acc_c = 0.0;
        for (int k = 0; k < K && ok; k++) {
            const long long e = b0 + k;
            const bool has_next = k + 1 < K;
            // read-only data of this entry's cell, loaded before any wait
            const double hs = a.L[c].x;
            const float b_c = a.B[c].w;
            const double sed_c = a.sediment[c];
            if (!have_c) {
                ok = acquire(a.done, c, a.epoch, Dc, a.error);
                if (!ok) break;
                have_c = true;
            }
            // an erosion entry (floor) and a final deposit (ceiling) read the next entry's cell
            // live: acquire it now; a step deposit does not, and acquires it only before writing it
            const bool is_step = vv >= 0.0f;
            const bool reads_next = has_next && (dlt < 0.0 || !is_step);
            double hs_n = 0.0, acc_n = 0.0;
            if (reads_next) {
                hs_n = a.L[nc].x;
                ok = acquire(a.done, nc, a.epoch, Dn, a.error);
                if (!ok) break;
                acc_n = a.acc4[4 * nc];
            }
            if (!acc_known) acc_c = a.acc4[4 * c];
            // prefetch the descriptor after next
            long long nnc = -1;
            int Dnn = 0;
            if (k + 2 < K) {
                nnc = a.cell[e + 2];
                Dnn = a.D[e + 2];
            }
            bool lastn = false;
            double dltn = 0.0;
            float vn = 0.0f, mn0 = 0.0f, mn1 = 0.0f;
            if (has_next) {
                lastn = a.last[e + 1];
                dltn = a.delta[e + 1];
                vn = a.vol[e + 1];
                mn0 = a.mom[2 * (e + 1)];
                mn1 = a.mom[2 * (e + 1) + 1];
            }
            double acc_new = acc_c;
            if (!(a.mask && a.mask[c] != PGE_MASK_ACTIVE)) {
                double *accp = a.acc4 + 4 * c;
                const double acc = acc_c;
                const double s_c = hs + acc;
                const double nlive = hs_n + acc_n;
                if (dlt < 0.0) {
                    const double ew = -dlt;
                    double e_act = ew;
                    double room = p.iter_erode + acc;
                    if (a.ecap) {
                        const double r2 = a.ecap[c] + acc;
                        if (r2 < room) room = r2;
                    }
                    if (e_act > room) e_act = room;
                    double floor_ = s_c >= (double)b_c ? (double)b_c : s_c;
                    if (has_next && nlive > floor_) floor_ = nlive;
                    if (e_act > s_c - floor_) e_act = s_c - floor_;
                    if (e_act < 0.0) e_act = 0.0;
                    if (e_act < ew) {
                        clamped++;
                        deficit += ew - e_act;
                    }
                    acc_new = acc - e_act;
                    eroded_fx += fx_mass(e_act);
                } else {
                    double want = dlt + surplus;
                    surplus = 0.0;
                    if (deficit > 0.0) {
                        const double t = want < deficit ? want : deficit;
                        want -= t;
                        deficit -= t;
                    }
                    double d_act = want;
                    const double room = p.iter_deposit - acc;
                    if (d_act > room) d_act = room;
                    bool has_ref = false;
                    double ref_live = 0.0;
                    if (is_step) {
                        has_ref = has_prev;
                        ref_live = prev_live;
                    } else if (has_next) {
                        has_ref = true;
                        ref_live = nlive;
                    }
                    if (has_ref) {
                        double ceil_ = ref_live + p.dep_floor;
                        if (s_c < (double)b_c && is_step) ceil_ -= p.dep_floor + p.fan_slope;
                        const double lim = ceil_ - s_c;
                        if (d_act > lim) d_act = lim;
                    }
                    if (s_c < (double)b_c) {
                        const double lim = (double)b_c - p.dep_floor - s_c;
                        if (d_act > lim) d_act = lim;
                    }
                    if (d_act < 0.0) d_act = 0.0;
                    if (d_act < want) clamped++;
                    surplus = want - d_act;
                    acc_new = acc + d_act;
                    deposited_fx += fx_mass(d_act);
                    if (!is_step && death < 0) death = c;
                }
                accp[0] = acc_new;
                // the packed samples follow the live terrain (particle.py:1005-1009)
                a.A[c].x = (float)(hs + acc_new);
                const double sd = sed_c + acc_new;
                a.B[c].z = (float)(sd > 0.0 ? sd : 0.0);
                if (is_step) {
                    if (vv > 0.0f) {
                        accp[1] += (double)vv;
                        accp[2] += (double)m0;
                        accp[3] += (double)m1;
                    }
                    has_prev = true;
                    prev_live = hs + acc_new;
                }
            }
            // a cell is handed on right after the droplet's last write there; the stockpile (death)
            // cell waits for the stockpile update
            if (lastc && c != death) release(a.done, c, a.epoch + (unsigned)Dc + 1ull);
            // the next entry's cell: acquired (and its net change known) if this entry read it;
            // the same cell again keeps its acquisition and its updated net change
            if (has_next && nc == c) {
                have_c = true;
                acc_known = true;
                acc_c = acc_new;
            } else {
                have_c = reads_next;
                acc_known = reads_next;
                acc_c = acc_n;
            }
            c = nc;
            Dc = Dn;
            lastc = lastn;
            dlt = dltn;
            vv = vn;
            m0 = mn0;
            m1 = mn1;
            nc = nnc;
            Dn = Dnn;
        }
        if (!ok) break;
        long long topend = 0, lostoff = 0;
        if (surplus > 0.0 && death >= 0) {
            if (a.L[death].x + a.acc4[4 * death] < (double)a.B[death].w) {
                double keep = surplus * (1.0 - p.offshore_writeoff);
                if (keep < 1e-4) keep = 0.0;
                a.pend[death] += keep;
                topend = fx_mass(keep);
                lostoff = fx_mass(surplus) - topend;
            } else {
                a.pend[death] += surplus;
                topend = fx_mass(surplus);
            }
        }
        if (death >= 0) {
            // the death cell's last visit is among the final deposits: find it and hand the cell on
            for (int k = K - 1; k >= 0; k--) {
                const long long e = b0 + k;
                if (a.cell[e] == death) {
                    release(a.done, death, a.epoch + (unsigned)a.D[e] + 1ull);
                    break;
                }
            }
        }
        if (clamped) atomicAdd(&sstat[OS_CLAMPED], (unsigned long long)clamped);
        if (topend) atomicAdd(&sstat[OS_TOPEND], (unsigned long long)topend);
        if (deficit > 0.0) atomicAdd(&sstat[OS_DEFICIT], (unsigned long long)fx_mass(deficit));
        if (lostoff) atomicAdd(&sstat[OS_LOSTOFF], (unsigned long long)lostoff);
        if (eroded_fx) atomicAdd(&sstat[OS_ERODED], (unsigned long long)eroded_fx);
        if (deposited_fx) atomicAdd(&sstat[OS_DEPOSITED], (unsigned long long)deposited_fx);
    }
    __syncthreads();
    if (threadIdx.x < OS_N && sstat[threadIdx.x]) {
        PgeStats *st = a.stats;
        int64_t *dst = threadIdx.x == OS_CLAMPED ? &st->clamped
                     : threadIdx.x == OS_TOPEND ? &st->to_pending_fx
                     : threadIdx.x == OS_DEFICIT ? &st->deficit_out_fx
                     : threadIdx.x == OS_LOSTOFF ? &st->lost_offshore_fx
                     : threadIdx.x == OS_ERODED ? &st->eroded_fx
                                                : &st->deposited_fx;
        red_add(reinterpret_cast<long long *>(dst), (long long)sstat[threadIdx.x]);
    }
}

int ordered_blocks_per_sm(int threads)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ordered_apply_kernel, threads, 0) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t ordered_wave(const OrderedWave &w, cudaStream_t st)
{
    const long long nslots = w.nw * w.cap;
    ordered_keys_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.cap, w.a.cell, w.a.count, w.kbits, w.pbits, w.invalid,
                                                          w.keys_in, w.vals_in);
    size_t tb = w.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(w.temp, tb, w.keys_in, w.keys_out, w.vals_in, w.vals_out, (int)nslots, 0,
                                                    w.end_bit, st);
    if (e != cudaSuccess) return e;
    ordered_flags_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.kbits, w.pbits, w.invalid, w.runstart, w.segpos);
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveSum(w.temp, tb, w.runstart, w.runscan, (int)nslots, st)) != cudaSuccess) return e;
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveScan(w.temp, tb, w.segpos, w.segscan, MaxOp{}, (int)nslots, st)) != cudaSuccess) return e;
    ordered_rank_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.vals_out, w.invalid, w.kbits, w.runscan, w.segscan,
                                                          const_cast<int32_t *>(w.a.D), const_cast<uint8_t *>(w.a.last));
    long long blocks = (w.nw * 32 + 255) / 256;  // a warp per droplet
    if (blocks > w.max_blocks) blocks = w.max_blocks;
    ordered_apply_kernel<<<(int)blocks, 256, 0, st>>>(w.a);
    return cudaPeekAtLastError();
}

}  // namespace pge
