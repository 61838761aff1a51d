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
//     its cell, whether it is its droplet's first visit there, and whether
//     it is the last;
//   * a cell's live net change and its hand-off counter share one 16-byte
//     word: a droplet acquires a cell (the counter reads epoch + D; the net
//     change comes with it) one entry before it writes there (the erosion
//     floor and final-deposit ceiling read the next entry's cell), and hands
//     it on with one store of (net change, epoch + D + 1) right after its
//     last write there; the step-deposit ceiling of the following entry uses
//     the live surface snapshotted at that write -- exactly what the serial
//     order reads, since no other droplet runs between two entries of one
//     droplet.  The stockpile test (is the death cell submerged?) reads the
//     death cell as the droplet's own last write there left it, so it is
//     taken at that write and the death cell is handed on like any other;
//   * a droplet's path through the wave is mostly its own entries one after
//     another, so each entry's packed 16-byte descriptor, its cell's packed
//     16-byte terrain and the cell's hand-off word are copied into a ring in
//     shared memory several entries ahead (asynchronous copies, waited for
//     by group count);
//   * the order-dependent float64 sums that nothing in the wave reads back
//     -- the discharge and momentum tracks and the stockpile -- are summed
//     after the apply, per cell, walking the sorted entries: (droplet,
//     entry) order within a cell is the serial order.  The packed samples of
//     the touched cells are refreshed in the same walk.
// Every read and write of a cell therefore happens in exactly the
// reference's serial order, and the float64 arithmetic is the reference's
// (this file is compiled without FMA contraction).  Waits are bounded: a
// wait that gives up sets an error flag the host reports.
#include <cub/cub.cuh>

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
// a waiting warp sleeps PGE_POLL_SLEEP_NS after every PGE_POLL_EVERY polls (a power of two)
#ifndef PGE_POLL_EVERY
#define PGE_POLL_EVERY 256
#endif
#ifndef PGE_POLL_SLEEP_NS
#define PGE_POLL_SLEEP_NS 32
#endif
static_assert((PGE_POLL_EVERY & (PGE_POLL_EVERY - 1)) == 0, "poll interval: a power of two");

// A cell's hand-off word: 16 bytes, two 8-byte halves (acc low 32 bits | count << 32) and (acc high
// 32 bits | count << 32), where acc is the live net change and count the hand-off counter.  Each
// half is one single-copy-atomic 64-bit access, so a reader that sees the same count in both halves
// holds a consistent word, however the 16 bytes were read.
__device__ __forceinline__ void hand_pack(double acc, uint32_t count, unsigned long long &w0, unsigned long long &w1)
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(acc);
    w0 = ((unsigned long long)count << 32) | (bits & 0xffffffffull);
    w1 = ((unsigned long long)count << 32) | (bits >> 32);
}

__device__ __forceinline__ double hand_acc(unsigned long long w0, unsigned long long w1)
{
    return __longlong_as_double((long long)((w1 << 32) | (w0 & 0xffffffffull)));
}

__device__ __forceinline__ bool hand_ready(unsigned long long w0, unsigned long long w1, uint32_t want)
{
    return (uint32_t)(w0 >> 32) == want && (uint32_t)(w1 >> 32) == want;
}

__device__ __forceinline__ void hand_load(const double2 *p, unsigned long long &w0, unsigned long long &w1)
{
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(p) : "memory");
}

// the same read issued ahead of its use: no compiler barrier, the thread waits only where it uses the word
__device__ __forceinline__ void hand_load_ahead(const double2 *p, unsigned long long &w0, unsigned long long &w1)
{
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(p));
}

__device__ __forceinline__ void hand_store(double2 *p, double acc, uint32_t count)
{
    unsigned long long w0, w1;
    hand_pack(acc, count, w0, w1);
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" : : "l"(p), "l"(w0), "l"(w1));
}

// wait until the D earlier droplets of this wave that visit cell c have handed it on; acc = its net change
__device__ __forceinline__ bool acquire(const double2 *hand, long long c, uint32_t epoch, int D, int *error, double &acc)
{
    const uint32_t want = epoch + (uint32_t)D;
    unsigned long long w0, w1;
    for (long long i = 0; i < kSpinLimit; i++) {
        hand_load(hand + c, w0, w1);
        if (D == 0 || hand_ready(w0, w1, want)) {  // D == 0: the wave's first visitor, no earlier writer
            acc = hand_acc(w0, w1);
            return true;
        }
        if ((i & (PGE_POLL_EVERY - 1)) == PGE_POLL_EVERY - 1) {
            if (*(volatile int *)error) return false;  // another wait gave up: stop waiting
            __nanosleep(PGE_POLL_SLEEP_NS);
        }
    }
    atomicExch(error, 1);
    return false;
}

// a cell this droplet holds and has written before: its own last write (coherent for the same thread)
__device__ __forceinline__ double own_value(const double2 *hand, long long c)
{
    unsigned long long w0, w1;
    hand_load(hand + c, w0, w1);
    return hand_acc(w0, w1);
}

// asynchronous copies into shared memory: the waits count copy groups, so waiting for an old
// entry's data never waits for the copies issued after it
__device__ __forceinline__ uint32_t sm_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// (the copies and the commit carry no memory clobber: a ring slot is only read after the group wait that
// covers its copy, and that wait is the compiler barrier; the compiler may then overlap a copy's issue
// with the arithmetic around it)
__device__ __forceinline__ void cp_ca8(void *d, const void *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sm_addr(d)), "l"(__cvta_generic_to_global(g)));
}
__device__ __forceinline__ void cp_cg16(void *d, const void *g)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sm_addr(d)), "l"(__cvta_generic_to_global(g)));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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

// the entries of a wave's lists compacted in (droplet, entry) order: entry k of droplet q goes to offsets[q] + k
__global__ void ordered_compact_keys_kernel(long long nslots, int cap, const int32_t *cell, const int64_t *count,
                                            const long long *offsets, unsigned long long *keys, int32_t *vals)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nslots; s += (long long)gridDim.x * blockDim.x) {
        const long long q = s / cap, k = s - q * cap;
        if (k < count[q]) {
            const long long e = offsets[q] + k;
            keys[e] = (unsigned long long)cell[s];
            vals[e] = (int32_t)s;
        }
    }
}

__global__ void entry_total_kernel(const int64_t *count, const long long *offsets, long long nw, long long *total)
{
    *total = nw > 0 ? offsets[nw - 1] + count[nw - 1] : 0;
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
                                    unsigned long long invalid, const int32_t *runscan, const int32_t *segscan,
                                    const double *delta, const float *vol, EntryDesc *desc)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        if (k == invalid) continue;
        const int32_t s = vals[i];
        const uint32_t D = (uint32_t)(runscan[i] - runscan[segscan[i]]);
        bool lst = true;
        if (i + 1 < nslots) lst = keys[i + 1] != k || vals[i + 1] / cap != s / cap;
        const bool fst = i == 0 || keys[i - 1] != k || vals[i - 1] / cap != s / cap;
        EntryDesc d;
        d.cell = (int32_t)k;
        d.dflags = D | (lst ? ENTRY_LAST : 0u) | (fst ? ENTRY_FIRST : 0u) | (vol[s] >= 0.0f ? ENTRY_STEP : 0u) |
                   (vol[s] == -3.0f ? ENTRY_PARK : 0u);
        d.delta = delta[s];
        desc[s] = d;
    }
}

// the ordered apply's read-only terrain record of every cell
__global__ void ordered_terrain_kernel(long long ncell, const double2 *L, const float4 *B, const uint8_t *mask, CellTerr *terr)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        CellTerr t;
        t.hs = L[c].x;
        t.base = B[c].w;
        t.active = !mask || mask[c] == PGE_MASK_ACTIVE ? 1u : 0u;
        terr[c] = t;
    }
}

struct MaxOp {
    __device__ __forceinline__ int32_t operator()(const int32_t a, const int32_t b) const { return a > b ? a : b; }
};

size_t ordered_temp_bytes(long long nslots, long long max_wave)
{
    size_t a = 0, b = 0, c = 0, d = 0, x = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, x, (int64_t *)nullptr, (long long *)nullptr, (int)max_wave);
    cub::DeviceRadixSort::SortPairs(nullptr, a, (unsigned long long *)nullptr, (unsigned long long *)nullptr, (int32_t *)nullptr,
                                    (int32_t *)nullptr, (int)nslots);
    cub::DeviceScan::InclusiveSum(nullptr, b, (int32_t *)nullptr, (int32_t *)nullptr, (int)nslots);
    cub::DeviceScan::InclusiveScan(nullptr, c, (int32_t *)nullptr, (int32_t *)nullptr, MaxOp{}, (int)nslots);
    cub::DeviceRadixSort::SortPairs(nullptr, d, (uint32_t *)nullptr, (uint32_t *)nullptr, (int32_t *)nullptr, (int32_t *)nullptr,
                                    (int)(max_wave * LAKE_PARKS));
    size_t m = a > b ? a : b;
    m = m > c ? m : c;
    m = m > d ? m : d;
    return m > x ? m : x;
}

// ---------------------------------------------------------------------------
// lake parks: each lake's room counted down in droplet order (particle.py:912-933)
// ---------------------------------------------------------------------------
// one item per (droplet, park slot): key = the lake of the park's cell (all ones: no lake, or past the
// droplet's parks); the items enter the stable sort in (droplet, park) order, which is the serial order
__global__ void park_keys_kernel(long long nitems, int cap, const int32_t *cell, const double *delta, const int32_t *park_n,
                                 const int32_t *park_k, const int32_t *lake_id, long long lakes, uint32_t *keys, int32_t *vals,
                                 double *rest)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nitems; i += (long long)gridDim.x * blockDim.x) {
        const long long q = i / LAKE_PARKS;
        const int j = (int)(i - q * LAKE_PARKS);
        uint32_t key = 0xffffffffu;
        double r = 0.0;
        if (j < park_n[q] && park_k[i] >= 0 && park_k[i] < cap) {  // (an entry past the list's room was not recorded)
            const long long s = q * cap + park_k[i];
            const int32_t lk = lake_id[cell[s]];
            if (lk >= 0 && lk < lakes)
                key = (uint32_t)lk;
            else
                r = delta[s];  // no lake to take it: all of it is refused
        }
        keys[i] = key;
        vals[i] = (int32_t)i;
        rest[i] = r;
    }
}

// the first item of each lake walks its lake's parks in the serial order: the lake takes what it still has
// room for, the rest is refused
__global__ void park_walk_kernel(long long nitems, int cap, const uint32_t *keys, const int32_t *vals, const int32_t *cell,
                                 const double *delta, const int32_t *park_k, double *lake_room, double *lake_load, double *rest)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nitems; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t key = keys[i];
        if (key == 0xffffffffu || (i > 0 && keys[i - 1] == key)) continue;
        double room = lake_room[key];
        for (long long t = i; t < nitems && keys[t] == key; t++) {
            const int32_t v = vals[t];  // a park with a lake (its entry index checked by park_keys_kernel)
            const long long s = (long long)(v / LAKE_PARKS) * cap + park_k[v];
            double take = delta[s], r = 0.0;
            if (take > room) {
                r = take - room;
                take = room;
            }
            if (take > 0.0) {
                lake_load[cell[s]] += take;
                room -= take;
            }
            rest[v] = r;
        }
        lake_room[key] = room;
    }
}

cudaError_t park_wave(const ParkWave &pw, cudaStream_t st)
{
    const long long n = pw.nw * LAKE_PARKS;
    park_keys_kernel<<<grid_for(n), 256, 0, st>>>(n, pw.cap, pw.cell, pw.delta, pw.park_n, pw.park_k, pw.lake_id, pw.lakes, pw.keys_in,
                                                  pw.vals_in, pw.rest);
    size_t tb = pw.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(pw.temp, tb, pw.keys_in, pw.keys_out, pw.vals_in, pw.vals_out, (int)n, 0, 32, st);
    if (e != cudaSuccess) return e;
    park_walk_kernel<<<grid_for(n), 256, 0, st>>>(n, pw.cap, pw.keys_out, pw.vals_out, pw.cell, pw.delta, pw.park_k, pw.lake_room,
                                                  pw.lake_load, pw.rest);
    return cudaPeekAtLastError();
}

// ---------------------------------------------------------------------------
// the ordered apply
// ---------------------------------------------------------------------------
namespace {
// prefetch depth: at entry k the copies of the last LOOKAHEAD entries may still be in flight; the cell data of
// entry k + CELL_AHEAD and the descriptor of entry k + DESC_AHEAD are issued (the descriptor lands before its
// cell data is issued, the cell data before its entry and the one before it are applied)
#ifndef PGE_APPLY_LOOKAHEAD
#define PGE_APPLY_LOOKAHEAD 1
#endif
constexpr int LOOKAHEAD = PGE_APPLY_LOOKAHEAD;
constexpr int CELL_AHEAD = LOOKAHEAD + 2;
constexpr int DESC_AHEAD = CELL_AHEAD + LOOKAHEAD + 1;
constexpr int RING = DESC_AHEAD < 8 ? 8 : (DESC_AHEAD < 16 ? 16 : 32);  // entry slots per droplet (a power of two)
static_assert(RING > DESC_AHEAD, "the ring holds every entry in flight");
// two droplets per block: a block's warp slots free up as soon as its two droplets are done, so
// concurrent passes (other worlds' waves on other streams) pack around the long-lived droplets
constexpr int APPLY_THREADS = 64;
// resident blocks asked of the register allocator: 8 gives the plain variant 70 registers without spills (its
// own choice, 48 registers and 12 spilled bytes, was 2.5 % slower)
#ifndef PGE_APPLY_MINB
#define PGE_APPLY_MINB 8
#endif

// one entry of a droplet's list as the apply reads it, filled by asynchronous copies
struct alignas(16) Slot {
    EntryDesc d;                // descriptor
    unsigned long long spare[2];  // (the hand-off word is read into registers instead)
    CellTerr t;                 // the cell's read-only terrain
    double cap;                 // the slope erode cap (when on)
    float2 route;               // the cell's packed routing surface and flag (with lakes)
};
static_assert(sizeof(Slot) == 64, "slot layout");

__device__ __forceinline__ void stage_desc(const OrderedArgs &a, Slot &s, long long e) { cp_cg16(&s.d, a.desc + e); }

template <bool ECAP, bool LAKE>
__device__ __forceinline__ void stage_cell(const OrderedArgs &a, Slot &s)
{
    const long long c = s.d.cell;
    cp_cg16(&s.t, a.terr + c);
    if (ECAP) cp_ca8(&s.cap, a.ecap + c);
    if (LAKE) cp_ca8(&s.route, a.R + c);
}

// one entry's slot as registers: read one entry before it is applied, while the entry before it
// computes, so that the apply's chain from entry to entry holds only its arithmetic
struct Ent {
    int32_t c;
    uint32_t df;
    double dlt, hs, cap;
    float base;
    uint32_t active;
    unsigned long long h0, h1;
    float2 route;
};

template <bool ECAP, bool LAKE>
__device__ __forceinline__ Ent load_ent(const Slot &s)
{
    Ent e;
    e.c = s.d.cell;
    e.df = s.d.dflags;
    e.dlt = s.d.delta;
    e.hs = s.t.hs;
    e.base = s.t.base;
    e.active = s.t.active;
    e.h0 = e.h1 = 0ull;  // read separately, one entry ahead
    e.cap = ECAP ? s.cap : 0.0;
    e.route = LAKE ? s.route : make_float2(0.f, 0.f);
    return e;
}

// per droplet state carried from entry to entry
struct Walk {
    double deficit, surplus, prev_live, acc_c;
    int clamped;
    int32_t death;
    // this droplet's last three writes (cell, net change after it)
    int32_t w1c, w2c, w3c;
    double w1v, w2v, w3v;
    bool sub_death, has_prev, have_c, ok;
};

// the net change of a cell this droplet is about to read: a recent write of its own, its own
// earlier write (a revisit), the prefetched word once the D earlier droplets have handed the cell
// on, or a wait for them
__device__ __forceinline__ bool cell_value(const OrderedArgs &a, const Walk &w, int32_t c, uint32_t df,
                                           unsigned long long h0, unsigned long long h1, double &acc)
{
    if (c == w.w1c) {
        acc = w.w1v;
        return true;
    }
    if (c == w.w2c) {
        acc = w.w2v;
        return true;
    }
    if (c == w.w3c) {
        acc = w.w3v;
        return true;
    }
    if (!(df & ENTRY_FIRST)) {
        acc = own_value(a.hand, c);
        return true;
    }
    const uint32_t D = df & ENTRY_D_MASK;
    if (D == 0 || hand_ready(h0, h1, a.epoch + D)) {
        acc = hand_acc(h0, h1);
        return true;
    }
    return acquire(a.hand, c, a.epoch, (int)D, a.error, acc);
}
}  // namespace

// One change-list entry against the live terrain (particle.py:934-1002): the erosion floor (the
// base level or the cell itself, the next path cell's live surface nlive), the deposit ceilings (the
// previous step's live surface, or for a final deposit the next, older path cell), the deficit and
// surplus carried along the droplet's list.  acc is the cell's live net change; writes the new one
// and the amount actually moved.
template <bool ECAP, bool LAKE>
__device__ __forceinline__ void entry_arith(const PgeParams &p, Walk &w, int32_t c, double dlt, bool is_step, bool act, double hs,
                                            double b_c, double acc, bool has_next, double nlive, double capv, float2 route,
                                            double &acc_new, double &amount)
{
    if (act) {
        const double s_c = hs + acc;
        if (dlt < 0.0) {
            const double ew = -dlt;
            double e_act = ew;
            double room = p.iter_erode + acc;
            if (ECAP) {
                const double r2 = capv + acc;
                if (r2 < room) room = r2;
            }
            if (e_act > room) e_act = room;
            double floor_ = s_c >= b_c ? b_c : s_c;
            // a lake bed is never eroded below its water level (particle.py:952-956)
            if (LAKE && route.y >= 1.5f && (double)route.x > floor_) floor_ = (double)route.x;
            if (has_next && nlive > floor_) floor_ = nlive;
            if (e_act > s_c - floor_) e_act = s_c - floor_;
            if (e_act < 0.0) e_act = 0.0;
            if (e_act < ew) {
                w.clamped++;
                w.deficit += ew - e_act;
            }
            acc_new = acc - e_act;
            amount = e_act;
        } else {
            double want = dlt + w.surplus;
            w.surplus = 0.0;
            if (w.deficit > 0.0) {
                const double t = want < w.deficit ? want : w.deficit;
                want -= t;
                w.deficit -= t;
            }
            double d_act = want;
            const double room = p.iter_deposit - acc;
            if (d_act > room) d_act = room;
            bool has_ref = false;
            double ref_live = 0.0;
            if (is_step) {
                has_ref = w.has_prev;
                ref_live = w.prev_live;
            } else if (has_next) {
                has_ref = true;
                ref_live = nlive;
            }
            if (has_ref) {
                double ceil_ = ref_live + p.dep_floor;
                if (s_c < b_c && is_step) ceil_ -= p.dep_floor + p.fan_slope;
                const double lim = ceil_ - s_c;
                if (d_act > lim) d_act = lim;
            }
            if (s_c < b_c) {
                const double lim = b_c - p.dep_floor - s_c;
                if (d_act > lim) d_act = lim;
            }
            if (d_act < 0.0) d_act = 0.0;
            if (d_act < want) w.clamped++;
            w.surplus = want - d_act;
            acc_new = acc + d_act;
            amount = d_act;
            if (!is_step && w.death < 0) w.death = c;
        }
        if (c == w.death) w.sub_death = hs + acc_new < b_c;
        if (is_step) {
            w.has_prev = true;
            w.prev_live = hs + acc_new;
        }
    }
}

// a droplet's stockpile (particle.py:1019-1041) and its statistics, once its list is applied
__device__ __forceinline__ void droplet_end(const OrderedArgs &a, const Walk &w, long long q, unsigned long long *sstat)
{
    const PgeParams &p = a.p;
    long long topend = 0, lostoff = 0;
    int32_t dth = -1;
    double add = 0.0;
    double surplus = w.surplus;
    if (a.park_n) {  // the loads its lakes had no room for join what it could not place (particle.py:1019)
        double refused = 0.0;
        const int np = a.park_n[q];
        for (int j = 0; j < np; j++) refused += a.park_rest[q * LAKE_PARKS + j];
        surplus += refused;
    }
    if (w.death >= 0 && surplus > 0.0) {
        if (w.sub_death) {
            double keep = surplus * (1.0 - p.offshore_writeoff);
            if (keep < 1e-4) keep = 0.0;
            add = keep;
            topend = fx_mass(keep);
            lostoff = fx_mass(surplus) - topend;
        } else {
            add = surplus;
            topend = fx_mass(surplus);
        }
        dth = w.death;
    }
    a.dth[q] = dth;
    a.keep[q] = add;
    if (w.clamped) atomicAdd(&sstat[OS_CLAMPED], (unsigned long long)w.clamped);
    if (topend) atomicAdd(&sstat[OS_TOPEND], (unsigned long long)topend);
    if (w.deficit > 0.0) atomicAdd(&sstat[OS_DEFICIT], (unsigned long long)fx_mass(w.deficit));
    if (lostoff) atomicAdd(&sstat[OS_LOSTOFF], (unsigned long long)lostoff);
}

// the block's statistics to the pass totals (after a __syncthreads)
__device__ __forceinline__ void flush_stats(const OrderedArgs &a, const unsigned long long *sstat)
{
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

template <bool ECAP, bool LAKE>
__global__ void __launch_bounds__(APPLY_THREADS, PGE_APPLY_MINB) ordered_apply_kernel(const OrderedArgs a)
{
    __shared__ unsigned long long sstat[OS_N];
    extern __shared__ Slot ring[];  // per droplet lane: RING slots
    for (int k = threadIdx.x; k < OS_N; k += blockDim.x) sstat[k] = 0ull;
    __syncthreads();
    const PgeParams &p = a.p;
    // a.lanes droplets per warp, one per lane (1 when a pass runs alone: lanes of one warp that wait
    // on different hand-offs take turns; more when other passes share the GPU, to hold fewer warps).
    // A lane only ever waits for earlier droplets, which independent thread scheduling lets run.
    const int lane = threadIdx.x & 31, lanes = a.lanes;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    Slot *R = ring + ((size_t)(threadIdx.x >> 5) * lanes + lane) * RING;
    bool failed = false;
    for (long long q = gw * lanes + lane; lane < lanes && !failed && q < a.nw; q += nwarps * lanes) {
        const int K = (int)a.count[q];
        if (K <= 0) {
            a.dth[q] = -1;
            continue;
        }
        const long long b0 = q * a.cap;
        // prologue: the descriptors of the first DESC_AHEAD entries, then the cell data of the first CELL_AHEAD
        for (int j = 0; j < DESC_AHEAD && j < K; j++) stage_desc(a, R[j], b0 + j);
        cp_commit();
        cp_wait<0>();
        for (int j = 0; j < CELL_AHEAD && j < K; j++) stage_cell<ECAP, LAKE>(a, R[j]);
        cp_commit();
        cp_wait<0>();
        Walk w;
        w.deficit = w.surplus = w.prev_live = w.acc_c = 0.0;
        w.clamped = 0;
        w.death = -1;
        w.w1c = w.w2c = w.w3c = -1;
        w.w1v = w.w2v = w.w3v = 0.0;
        w.sub_death = w.has_prev = w.have_c = false;
        w.ok = true;
        // the hand-off words are read into registers one entry ahead of the entry that first reads them
        // (the terrain three ahead, through the ring): a word read later is less often stale
        unsigned long long p0 = 0ull, p1 = 0ull;
        Ent cur = load_ent<ECAP, LAKE>(R[0]);
        hand_load_ahead(a.hand + cur.c, cur.h0, cur.h1);
        if (K > 1) hand_load_ahead(a.hand + R[1].d.cell, p0, p1);
        for (int k = 0; k < K; k++) {
            // the copies issued LOOKAHEAD + 1 or more entries ago have landed: the descriptor of entry
            // k + CELL_AHEAD and the cell data of entries k and k + 1
            cp_wait<LOOKAHEAD>();
            const bool has_next = k + 1 < K;
            Ent nx;
            nx.c = -1;
            if (has_next) {
                nx = load_ent<ECAP, LAKE>(R[(k + 1) & (RING - 1)]);
                nx.h0 = p0;
                nx.h1 = p1;
            }
            // entry k + 2's descriptor landed with the group waited for above
            if (k + 2 < K) hand_load_ahead(a.hand + R[(k + 2) & (RING - 1)].d.cell, p0, p1);
            if (k + CELL_AHEAD < K) stage_cell<ECAP, LAKE>(a, R[(k + CELL_AHEAD) & (RING - 1)]);
            if (k + DESC_AHEAD < K) stage_desc(a, R[(k + DESC_AHEAD) & (RING - 1)], b0 + k + DESC_AHEAD);
            cp_commit();
            const int32_t c = cur.c;
            const uint32_t df = cur.df;
            const double dlt = cur.dlt;
            const double hs = cur.hs;
            const double b_c = (double)cur.base;
            const bool park = (df & ENTRY_PARK) != 0;  // a lake park changes no terrain (particle.py:912-933)
            const bool act = cur.active != 0 && !park;
            if (!w.have_c && !(w.ok = cell_value(a, w, c, df, cur.h0, cur.h1, w.acc_c))) break;
            // an erosion entry (floor) and a final deposit (ceiling) read the next entry's cell live:
            // acquire it now; a step deposit does not, and acquires it only before writing it
            const bool is_step = (df & ENTRY_STEP) != 0;
            const bool reads_next = has_next && !park && (dlt < 0.0 || !is_step);
            const int32_t ncell = nx.c;
            double acc_n = 0.0, hs_n = 0.0;
            if (reads_next) {
                hs_n = nx.hs;
                if (ncell == c)
                    acc_n = w.acc_c;
                else if (!(w.ok = cell_value(a, w, ncell, nx.df, nx.h0, nx.h1, acc_n)))
                    break;
            }
            const double acc = w.acc_c;
            double acc_new = acc, amount = 0.0;
            entry_arith<ECAP, LAKE>(p, w, c, dlt, is_step, act, hs, b_c, acc, has_next, hs_n + acc_n, cur.cap, cur.route, acc_new,
                                    amount);
            // publish the net change; a droplet's last write at a cell also hands the cell on
            const bool lastv = (df & ENTRY_LAST) != 0;
            if (act || lastv) hand_store(a.hand + c, acc_new, a.epoch + (df & ENTRY_D_MASK) + (lastv ? 1u : 0u));
            a.act[b0 + k] = amount;
            w.w3c = w.w2c;
            w.w3v = w.w2v;
            w.w2c = w.w1c;
            w.w2v = w.w1v;
            w.w1c = c;
            w.w1v = acc_new;
            // the next entry's cell: acquired (with its net change) if this entry read it; the same
            // cell again keeps its acquisition and its updated net change
            if (has_next && ncell == c) {
                w.have_c = true;
                w.acc_c = acc_new;
            } else {
                w.have_c = reads_next;
                w.acc_c = acc_n;
            }
            cur = nx;
        }
        cp_wait<0>();
        if (!w.ok) {
            failed = true;
            break;
        }
        droplet_end(a, w, q, sstat);
    }
    __syncthreads();
    flush_stats(a, sstat);
}

// ---------------------------------------------------------------------------
// after the apply: per touched cell, in the serial (droplet, entry) order, the discharge and
// momentum tracks (particle.py:1013-1018) and the stockpile (:1019-1041); then the cell's net
// change to the accumulators and its packed samples (:1005-1009); and the wave's eroded and
// deposited totals (integer fixed point, so their order does not matter).  First every sorted slot
// gathers what its entry adds into arrays in sorted order (one thread a slot, all loads in flight at
// once); then one thread a cell sums its run of those arrays in order (contiguous reads).
// ---------------------------------------------------------------------------
__global__ void ordered_gather_kernel(const OrderedArgs a, long long nslots, const unsigned long long *keys, const int32_t *vals,
                                      unsigned long long invalid, FinishRows g)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long key = keys[i];
        if (key == invalid) continue;
        const int32_t s = vals[i], q = s / a.cap;
        const bool active = !a.mask || a.mask[key] == PGE_MASK_ACTIVE;
        const float v = a.vol[s];
        const bool track = active && v > 0.0f;
        g.v[i] = track ? v : 0.0f;
        g.m0[i] = track ? a.mom[2 * (long long)s] : 0.0f;
        g.m1[i] = track ? a.mom[2 * (long long)s + 1] : 0.0f;
        const double amt = a.act[s];
        g.amt[i] = a.delta[s] < 0.0 ? -amt : amt;  // the sign says erosion (an eroded 0 is -0)
        g.kp[i] = (a.desc[s].dflags & ENTRY_LAST) && a.dth[q] == (int32_t)key ? a.keep[q] : -1.0;  // keep >= 0
    }
}

// One warp per 32 consecutive sorted slots; the warp walks every cell run that starts in its slots, 32
// entries at a time: the lanes load a step's rows at once, then every lane adds them in lane order (the
// float64 sums in the serial order, the additions shuffled out of the lanes), the integer totals per lane
constexpr int FINISH_THREADS = 256, FINISH_WARPS = FINISH_THREADS / 32;

__global__ void __launch_bounds__(FINISH_THREADS) ordered_finish_kernel(const OrderedArgs a, long long nslots, const unsigned long long *keys,
                                      unsigned long long invalid, FinishRows g)
{
    __shared__ unsigned long long sfx[2];
    // each warp's window of its run, read in order by every lane (broadcast reads: the loads of later slots
    // go out ahead of the float64 sums, which keep the serial order)
    __shared__ float sv[FINISH_WARPS][32], sa[FINISH_WARPS][32], sb[FINISH_WARPS][32];
    __shared__ double sk[FINISH_WARPS][32];
    if (threadIdx.x < 2) sfx[threadIdx.x] = 0ull;
    __syncthreads();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    long long eroded = 0, deposited = 0;
    for (long long base = warp * 32; base < nslots; base += nwarps * 32) {
        const long long i = base + lane;
        const unsigned long long ki = i < nslots ? keys[i] : invalid;
        const bool head = ki != invalid && (i == 0 || keys[i - 1] != ki);
        unsigned heads = __ballot_sync(full, head);
        while (heads) {
            const int hl = __ffs(heads) - 1;
            heads &= heads - 1;
            const unsigned long long key = __shfl_sync(full, ki, hl);
            const long long c = (long long)key;
            double *accp = a.acc4 + 4 * c;
            double tq = accp[1], ta = accp[2], tb = accp[3], pd = a.pend[c];
            for (long long j0 = base + hl;; j0 += 32) {
                const long long j = j0 + lane;
                const bool in = j < nslots && keys[j] == key;
                float v = 0.0f, m0 = 0.0f, m1 = 0.0f;
                double kp = -1.0;
                if (in) {
                    v = g.v[j];
                    m0 = g.m0[j];
                    m1 = g.m1[j];
                    kp = g.kp[j];
                    const double x = g.amt[j];
                    if (signbit(x))
                        eroded += fx_mass(-x);
                    else
                        deposited += fx_mass(x);
                }
                // the run covers a prefix of the lanes (keys are sorted)
                const int n = __popc(__ballot_sync(full, in));
                sv[wib][lane] = v;
                sa[wib][lane] = m0;
                sb[wib][lane] = m1;
                sk[wib][lane] = kp;
                __syncwarp();
#pragma unroll 4
                for (int t = 0; t < n; t++) {
                    const float vt = sv[wib][t];
                    const float at = sa[wib][t];
                    const float bt = sb[wib][t];
                    const double kt = sk[wib][t];
                    if (vt > 0.0f) {  // a step of volume > 0 on an active cell (gathered as 0 otherwise)
                        tq += (double)vt;
                        ta += (double)at;
                        tb += (double)bt;
                    }
                    if (kt >= 0.0) pd += kt;
                }
                __syncwarp();  // every lane has read the window before the next one is written
                if (n < 32) break;
            }
            if (lane == 0) {
                accp[1] = tq;
                accp[2] = ta;
                accp[3] = tb;
                a.pend[c] = pd;
                const unsigned long long *hw = reinterpret_cast<const unsigned long long *>(a.hand + c);
                const double acc = hand_acc(hw[0], hw[1]);
                accp[0] = acc;
                if (!a.mask || a.mask[c] == PGE_MASK_ACTIVE) {
                    const float surf = (float)(a.L[c].x + acc);
                    a.A[c].x = surf;
                    const double sd = a.sediment[c] + acc;
                    a.B[c].z = (float)(sd > 0.0 ? sd : 0.0);
                    // the route flag follows the live surface; a lake cell stays a lake cell (particle.py:1010-1012)
                    if (a.R && a.R[c].y < 1.5f) a.R[c].y = a.R[c].x != surf ? 1.0f : 0.0f;
                }
            }
        }
    }
    if (eroded) atomicAdd(&sfx[0], (unsigned long long)eroded);
    if (deposited) atomicAdd(&sfx[1], (unsigned long long)deposited);
    __syncthreads();
    if (threadIdx.x == 0 && sfx[0]) red_add(reinterpret_cast<long long *>(&a.stats->eroded_fx), (long long)sfx[0]);
    if (threadIdx.x == 1 && sfx[1]) red_add(reinterpret_cast<long long *>(&a.stats->deposited_fx), (long long)sfx[1]);
}

// zero the hand-off counters (the live net changes stay), so the 32-bit epochs can start over
__global__ void hand_reset_kernel(long long ncell, double2 *hand)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        unsigned long long *hw = reinterpret_cast<unsigned long long *>(hand + c);
        hw[0] &= 0xffffffffull;
        hw[1] &= 0xffffffffull;
    }
}

cudaError_t hand_reset(long long ncell, double2 *hand, cudaStream_t st)
{
    hand_reset_kernel<<<grid_for(ncell), 256, 0, st>>>(ncell, hand);
    return cudaPeekAtLastError();
}

cudaError_t ordered_terrain(long long ncell, const double2 *L, const float4 *B, const uint8_t *mask, CellTerr *terr, cudaStream_t st)
{
    ordered_terrain_kernel<<<grid_for(ncell), 256, 0, st>>>(ncell, L, B, mask, terr);
    return cudaPeekAtLastError();
}

int ordered_blocks_per_sm(int lanes)
{
    int n = 0;
    const size_t smem = (size_t)(APPLY_THREADS / 32) * lanes * RING * sizeof(Slot);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ordered_apply_kernel<false, false>, APPLY_THREADS, smem) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t ordered_wave(const OrderedWave &w, cudaStream_t st)
{
    long long nslots = w.nw * w.cap;
    size_t tb = w.temp_bytes;
    cudaError_t e;
    if (w.offsets) {
        // long lists (a lifetime of thousands of steps, most of it unused): only the recorded entries go through
        // the ranks, in (droplet, entry) order; their count comes back to the host for the library sorts
        if ((e = cub::DeviceScan::ExclusiveSum(w.temp, tb, w.a.count, w.offsets, (int)w.nw, st)) != cudaSuccess) return e;
        entry_total_kernel<<<1, 1, 0, st>>>(w.a.count, w.offsets, w.nw, w.offsets + w.nw);
        long long total = 0;
        if ((e = cudaMemcpyAsync(&total, w.offsets + w.nw, sizeof(long long), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        ordered_compact_keys_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.cap, w.a.cell, w.a.count, w.offsets, w.keys_in,
                                                                      w.vals_in);
        nslots = total;
    } else {
        ordered_keys_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.cap, w.a.cell, w.a.count, w.invalid, w.keys_in, w.vals_in);
    }
    tb = w.temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(w.temp, tb, w.keys_in, w.keys_out, w.vals_in, w.vals_out, (int)nslots, 0, w.end_bit, st);
    if (e != cudaSuccess) return e;
    ordered_flags_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.vals_out, w.cap, w.invalid, w.runstart, w.segpos);
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveSum(w.temp, tb, w.runstart, w.runscan, (int)nslots, st)) != cudaSuccess) return e;
    tb = w.temp_bytes;
    if ((e = cub::DeviceScan::InclusiveScan(w.temp, tb, w.segpos, w.segscan, MaxOp{}, (int)nslots, st)) != cudaSuccess) return e;
    ordered_rank_kernel<<<grid_for(nslots), 256, 0, st>>>(nslots, w.keys_out, w.vals_out, w.cap, w.invalid, w.runscan, w.segscan,
                                                          w.a.delta, w.a.vol, const_cast<EntryDesc *>(w.a.desc));
    const bool lake = w.a.lakes && w.a.R;
    const long long warps = (w.nw + w.a.lanes - 1) / w.a.lanes;  // a lane per droplet
    long long blocks = (warps * 32 + APPLY_THREADS - 1) / APPLY_THREADS;
    if (blocks > w.max_blocks) blocks = w.max_blocks;
    const size_t smem = (size_t)(APPLY_THREADS / 32) * w.a.lanes * RING * sizeof(Slot);
    if (w.a.ecap && lake)
        ordered_apply_kernel<true, true><<<(int)blocks, APPLY_THREADS, smem, st>>>(w.a);
    else if (w.a.ecap)
        ordered_apply_kernel<true, false><<<(int)blocks, APPLY_THREADS, smem, st>>>(w.a);
    else if (lake)
        ordered_apply_kernel<false, true><<<(int)blocks, APPLY_THREADS, smem, st>>>(w.a);
    else
        ordered_apply_kernel<false, false><<<(int)blocks, APPLY_THREADS, smem, st>>>(w.a);
    // the sort's input keys and the scans' buffers are free again: the gathered rows live there
    FinishRows g;
    g.v = reinterpret_cast<float *>(w.runstart);
    g.m0 = reinterpret_cast<float *>(w.segpos);
    g.m1 = reinterpret_cast<float *>(w.runscan);
    g.amt = reinterpret_cast<double *>(w.keys_in);
    g.kp = w.fin_kp;
    ordered_gather_kernel<<<grid_for(nslots), 256, 0, st>>>(w.a, nslots, w.keys_out, w.vals_out, w.invalid, g);
    ordered_finish_kernel<<<grid_for(nslots, FINISH_THREADS), FINISH_THREADS, 0, st>>>(w.a, nslots, w.keys_out, w.invalid, g);
    return cudaPeekAtLastError();
}

}  // namespace pge
