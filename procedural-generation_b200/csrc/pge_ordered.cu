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
// Here every droplet of a wave applies its own list on its own warp, and
// each cell is handed from droplet to droplet in droplet order:
//   * the entries of the wave are sorted by (cell, droplet, entry) and each
//     entry learns D = the number of distinct earlier droplets that visit
//     its cell, and whether it is its droplet's last visit there;
//   * a cell's live net change and its hand-off counter share one 16-byte
//     word, read and written as single 128-bit accesses: a droplet acquires
//     a cell (polls until the counter is epoch + D, and has the net change
//     from the same load) one entry before it writes there (the erosion
//     floor and final-deposit ceiling read the next entry's cell), and
//     hands it on with one store of (net change, epoch + D + 1) right after
//     its last write there; the step-deposit ceiling of the following entry
//     uses the live surface snapshotted at that write -- exactly what the
//     serial order reads, since no other droplet runs between two entries of
//     one droplet; the stockpile (death) cell is handed on last.
//   * The order-dependent float64 sums that nothing in the wave reads back
//     -- the discharge and momentum tracks and the stockpile -- are summed
//     after the apply, per cell, walking the sorted entries: (droplet,
//     entry) order within a cell is the serial order.  The packed samples of
//     the touched cells are refreshed in the same walk.
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

// a cell's hand-off word: x = live net change, y = hand-off counter (bits), one 128-bit access
__device__ __forceinline__ void hand_load(const double2 *p, double &acc, unsigned long long &count)
{
    unsigned long long lo, hi;
    asm volatile(
        "{\n\t.reg .b128 t;\n\t"
        "ld.relaxed.gpu.global.b128 t, [%2];\n\t"
        "mov.b128 {%0, %1}, t;\n\t}"
        : "=l"(lo), "=l"(hi)
        : "l"(p)
        : "memory");
    acc = __longlong_as_double((long long)lo);
    count = hi;
}

__device__ __forceinline__ void hand_store(double2 *p, double acc, unsigned long long count)
{
    const unsigned long long lo = (unsigned long long)__double_as_longlong(acc);
    asm volatile(
        "{\n\t.reg .b128 t;\n\t"
        "mov.b128 t, {%1, %2};\n\t"
        "st.relaxed.gpu.global.b128 [%0], t;\n\t}"
        :
        : "l"(p), "l"(lo), "l"(count)
        : "memory");
}

// wait until the D earlier droplets of this wave that visit cell c have handed it on; acc = its net change
__device__ __forceinline__ bool acquire(const double2 *hand, long long c, unsigned long long epoch, int D, int *error, double &acc)
{
    unsigned long long n;
    hand_load(hand + c, acc, n);
    if (D == 0) return true;  // the first visitor of the wave: every earlier wave has finished
    const unsigned long long want = epoch + (unsigned long long)D;
    for (long long i = 0; i < kSpinLimit; i++) {
        if (n == want) return true;
        if ((i & 255) == 255) {
            if (*(volatile int *)error) return false;  // another wait gave up: stop waiting
            __nanosleep(32);
        }
        hand_load(hand + c, acc, n);
    }
    atomicExch(error, 1);
    return false;
}

enum { OS_CLAMPED, OS_TOPEND, OS_DEFICIT, OS_LOSTOFF, OS_ERODED, OS_DEPOSITED, OS_N };
}  // namespace

// ---------------------------------------------------------------------------
// ranks
// ---------------------------------------------------------------------------
// key = the slot's cell (invalid past a list's end); the slots enter the stable sort in (droplet,
// entry) order, so equal cells keep the serial order
__global__ void ordered_keys_kernel(long long nslots, int cap, const int32_t *cell, const int64_t *count,
                                    unsigned long long invalid, unsigned long long *keys, int32_t *vals)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nslots; s += (long long)gridDim.x * blockDim.x) {
        const long long q = s / cap, k = s - q * cap;
        keys[s] = k < count[q] ? (unsigned long long)cell[s] : invalid;
        vals[s] = (int32_t)s;
    }
}

// runstart: first slot of a (cell, droplet) run; segpos: position of a cell segment's first slot
__global__ void ordered_flags_kernel(long long nslots, const unsigned long long *keys, const int32_t *vals, int cap,
                                     unsigned long long invalid, int32_t *runstart, int32_t *segpos)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        int rs = 0, sp = 0;
        if (k != invalid) {
            if (i == 0) {
                rs = 1;
            } else {
                const bool newseg = keys[i - 1] != k;
                rs = newseg || vals[i - 1] / cap != vals[i] / cap;
                sp = newseg ? (int)i : 0;
            }
        }
        runstart[i] = rs;
        segpos[i] = sp;
    }
}

__global__ void ordered_rank_kernel(long long nslots, const unsigned long long *keys, const int32_t *vals, int cap,
                                    unsigned long long invalid, const int32_t *runscan, const int32_t *segscan, int32_t *D,
                                    uint8_t *last)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k == invalid) continue;
        const int32_t s = vals[i];
        D[s] = runscan[i] - runscan[segscan[i]];
        bool lst = true;
        if (i + 1 < nslots) lst = keys[i + 1] != k || vals[i + 1] / cap != s / cap;
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
        if (K <= 0) {
            a.dth[q] = -1;
            continue;
        }
        const long long b0 = q * a.cap;
        double deficit = 0.0, surplus = 0.0;
        long long death = -1;
        int Ddeath = 0;
        bool has_prev = false;
        double prev_live = 0.0;  // the previous step entry's cell right after its write (the step-deposit ceiling)
        long long clamped = 0, eroded_fx = 0, deposited_fx = 0;
        // the current entry: descriptor and read-only terrain; the next entry's cell and rank
        long long c = a.cell[b0];
        int Dc = a.D[b0];
        bool lastc = a.last[b0];
        double dlt = a.delta[b0];
        float vv = a.vol[b0];
        double hs = a.L[c].x;
        float b_c = a.B[c].w;
        bool act_c = !a.mask || a.mask[c] == PGE_MASK_ACTIVE;
        double cap_c = a.ecap ? a.ecap[c] : 0.0;
        long long nc = -1;
        int Dn = 0;
        if (K > 1) {
            nc = a.cell[b0 + 1];
            Dn = a.D[b0 + 1];
        }
        bool ok = true;
        bool have_c = false;  // the current entry's cell is acquired and acc_c holds its net change
        double acc_c = 0.0;
        for (int k = 0; k < K; k++) {
            const long long e = b0 + k;
            const bool has_next = k + 1 < K;
            // everything read-only the next entry needs, loaded before any wait
            double hs_n = 0.0, cap_n = 0.0, dltn = 0.0;
            float b_n = 0.0f, vn = 0.0f;
            bool act_n = true, lastn = false;
            long long nnc = -1;
            int Dnn = 0;
            if (has_next) {
                hs_n = a.L[nc].x;
                b_n = a.B[nc].w;
                if (a.mask) act_n = a.mask[nc] == PGE_MASK_ACTIVE;
                if (a.ecap) cap_n = a.ecap[nc];
                lastn = a.last[e + 1];
                dltn = a.delta[e + 1];
                vn = a.vol[e + 1];
                if (k + 2 < K) {
                    nnc = a.cell[e + 2];
                    Dnn = a.D[e + 2];
                }
            }
            if (!have_c && !(ok = acquire(a.hand, c, a.epoch, Dc, a.error, acc_c))) break;
            // an erosion entry (floor) and a final deposit (ceiling) read the next entry's cell live:
            // acquire it now; a step deposit does not, and acquires it only before writing it
            const bool is_step = vv >= 0.0f;
            const bool reads_next = has_next && (dlt < 0.0 || !is_step);
            double acc_n = 0.0;
            if (reads_next) {
                if (nc == c)
                    acc_n = acc_c;
                else if (!(ok = acquire(a.hand, nc, a.epoch, Dn, a.error, acc_n)))
                    break;
            }
            double acc_new = acc_c;
            if (act_c) {
                const double acc = acc_c;
                const double s_c = hs + acc;
                const double nlive = hs_n + acc_n;
                if (dlt < 0.0) {
                    const double ew = -dlt;
                    double e_act = ew;
                    double room = p.iter_erode + acc;
                    if (a.ecap) {
                        const double r2 = cap_c + acc;
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
                    if (!is_step && death < 0) {
                        death = c;
                        Ddeath = Dc;
                    }
                }
                if (is_step) {
                    has_prev = true;
                    prev_live = hs + acc_new;
                }
            }
            // publish the net change; a droplet's last write at a cell also hands the cell on, except
            // the stockpile (death) cell, which waits for the stockpile
            const bool handoff = lastc && c != death;
            if (act_c || handoff) hand_store(a.hand + c, acc_new, a.epoch + (unsigned long long)Dc + (handoff ? 1ull : 0ull));
            // the next entry's cell: acquired (with its net change) if this entry read it; the same
            // cell again keeps its acquisition and its updated net change
            if (has_next && nc == c) {
                have_c = true;
                acc_c = acc_new;
            } else {
                have_c = reads_next;
                acc_c = acc_n;
            }
            c = nc;
            Dc = Dn;
            lastc = lastn;
            dlt = dltn;
            vv = vn;
            hs = hs_n;
            b_c = b_n;
            act_c = act_n;
            cap_c = cap_n;
            nc = nnc;
            Dn = Dnn;
        }
        if (!ok) break;
        long long topend = 0, lostoff = 0;
        int32_t dth = -1;
        double add = 0.0;
        if (death >= 0) {
            double accd;
            unsigned long long nd;
            hand_load(a.hand + death, accd, nd);  // this droplet's own last write there
            if (surplus > 0.0) {
                if (a.L[death].x + accd < (double)a.B[death].w) {
                    double keep = surplus * (1.0 - p.offshore_writeoff);
                    if (keep < 1e-4) keep = 0.0;
                    add = keep;
                    topend = fx_mass(keep);
                    lostoff = fx_mass(surplus) - topend;
                } else {
                    add = surplus;
                    topend = fx_mass(surplus);
                }
                dth = (int32_t)death;
            }
            hand_store(a.hand + death, accd, a.epoch + (unsigned long long)Ddeath + 1ull);
        }
        a.dth[q] = dth;
        a.keep[q] = add;
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

// ---------------------------------------------------------------------------
// after the apply: per touched cell, in the serial (droplet, entry) order, the discharge and
// momentum tracks (particle.py:1013-1018) and the stockpile (:1019-1041); then the cell's net
// change to the accumulators and its packed samples (:1005-1009)
// ---------------------------------------------------------------------------
__global__ void ordered_finish_kernel(const OrderedArgs a, long long nslots, const unsigned long long *keys, const int32_t *vals,
                                      unsigned long long invalid)
{
    constexpr int U = 8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = keys[i];
        if (key == invalid || (i > 0 && keys[i - 1] == key)) continue;  // not the first slot of a cell
        const long long c = (long long)key;
        const bool active = !a.mask || a.mask[c] == PGE_MASK_ACTIVE;
        double *accp = a.acc4 + 4 * c;
        double tq = accp[1], ta = accp[2], tb = accp[3], pd = a.pend[c];
        bool more = true;
        for (long long j = i; more; j += U) {
            int32_t sl[U];
            bool in[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                in[u] = j + u < nslots && keys[j + u] == key;
                sl[u] = in[u] ? vals[j + u] : 0;
            }
            float v[U], m0[U], m1[U];
            bool stock[U];
            double kp[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                v[u] = 0.0f;
                m0[u] = m1[u] = 0.0f;
                stock[u] = false;
                kp[u] = 0.0;
                if (in[u]) {
                    const int32_t s = sl[u], q = s / a.cap;
                    v[u] = a.vol[s];
                    if (active && v[u] > 0.0f) {
                        m0[u] = a.mom[2 * (long long)s];
                        m1[u] = a.mom[2 * (long long)s + 1];
                    }
                    if (a.last[s] && a.dth[q] == (int32_t)c) {
                        stock[u] = true;
                        kp[u] = a.keep[q];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (!in[u]) continue;
                if (active && v[u] > 0.0f) {
                    tq += (double)v[u];
                    ta += (double)m0[u];
                    tb += (double)m1[u];
                }
                if (stock[u]) pd += kp[u];
            }
            more = in[U - 1];
        }
        accp[1] = tq;
        accp[2] = ta;
        accp[3] = tb;
        a.pend[c] = pd;
        const double acc = a.hand[c].x;
        accp[0] = acc;
        if (active) {
            a.A[c].x = (float)(a.L[c].x + acc);
            const double sd = a.sediment[c] + acc;
            a.B[c].z = (float)(sd > 0.0 ? sd : 0.0);
        }
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
    ordered_keys_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.cap, w.a.cell, w.a.count, w.invalid, w.keys_in, w.vals_in);
    size_t tb = w.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(w.temp, tb, w.keys_in, w.keys_out, w.vals_in, w.vals_out, (int)nslots, 0,
                                                    w.end_bit, st);
    if (e != cudaSuccess) return e;
    ordered_flags_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.vals_out, w.cap, w.invalid, w.runstart, w.segpos);
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveSum(w.temp, tb, w.runstart, w.runscan, (int)nslots, st)) != cudaSuccess) return e;
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveScan(w.temp, tb, w.segpos, w.segscan, MaxOp{}, (int)nslots, st)) != cudaSuccess) return e;
    ordered_rank_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.vals_out, w.cap, w.invalid, w.runscan, w.segscan,
                                                          const_cast<int32_t *>(w.a.D), const_cast<uint8_t *>(w.a.last));
    long long blocks = (w.nw * 32 + 255) / 256;  // a warp per droplet
    if (blocks > w.max_blocks) blocks = w.max_blocks;
    ordered_apply_kernel<<<(int)blocks, 256, 0, st>>>(w.a);
    ordered_finish_kernel<<<grid_for(nslots), 256, 0, st>>>(w.a, nslots, w.keys_out, w.vals_out, w.invalid);
    return cudaPeekAtLastError();
}

}  // namespace pge
