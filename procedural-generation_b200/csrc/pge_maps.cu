// pge_maps.cu -- the per-iteration map passes around the droplet pass.
//
// Compiled with -fmad=false like the float64 droplet trace, so the float64
// stencils round like the reference's numba / numpy code.
//
//   pack / refresh / fold+EMA   particle.py:164-191, 1005-1012, 1079-1101, 1230-1242
//   thermal passes a / r / b    particle.py:1107-1227, maps.py:1050-1085
//   uplift                      maps.py:1088-1147
//   datum order statistic       maps.py:1446-1508 (radix select instead of np.partition)
//   halo gather                 field.py:104-125
//   spawn weights / inverse CDF maps.py:793-833, particle.py:1245-1260
#include <cstring>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "pge_internal.cuh"
#include "pge_maps.cuh"

namespace pge {

namespace {
__constant__ int kD8[8][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, -1}};

__device__ __forceinline__ bool interior(long long c, int NE, int H, int N)
{
    const long long r = c % ((long long)NE * NE);
    const int i = (int)(r / NE), j = (int)(r % NE);
    return i >= H && i < H + N && j >= H && j < H + N;
}

inline int grid_for(long long n, int threads = 256)
{
    long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}
// a grid-stride launch for kernels that end in a few global atomics a block: 8 blocks a multiprocessor
inline int grid_reduce(long long n, int threads = 256)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
    }
    const int b = grid_for(n, threads);
    return b < 8 * sms ? b : 8 * sms;
}
}  // namespace

// ---------------------------------------------------------------------------
// pack / refresh / fold + EMA
// ---------------------------------------------------------------------------
__global__ void pack_kernel(long long ncell, const double *__restrict__ h, const double *__restrict__ s,
                            const double *__restrict__ q, const double *__restrict__ mom, const float *__restrict__ evap,
                            const float *__restrict__ hard, const double *__restrict__ base, float4 *A, float4 *B, double2 *L)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const double sd = s[c];
        const double hs = h[c] + sd;
        A[c] = make_float4((float)hs, (float)q[c], (float)mom[2 * c], (float)mom[2 * c + 1]);
        B[c] = make_float4(evap[c], hard[c], (float)sd, (float)base[c]);
        L[c] = make_double2(hs, 0.0);
    }
}

__global__ void pack_metric_kernel(long long n, const float *__restrict__ g, const float *__restrict__ gi, float4 *G)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        G[2 * c] = make_float4(g[3 * c], g[3 * c + 1], g[3 * c + 2], gi[3 * c]);
        G[2 * c + 1] = make_float4(gi[3 * c + 1], gi[3 * c + 2], 0.f, 0.f);
    }
}

// between waves: the packed surface / sediment and the ledger's wave-start
// change follow the net change so far (apply_changes' samp sync, particle.py:1005-1009)
__global__ void refresh_kernel(long long ncell, const double *__restrict__ s, const long long *__restrict__ acc4, float4 *A,
                               float4 *B, double2 *L, float2 *R)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const double a = (double)acc4[4 * c] * INV_FX_MASS;
        double2 l = L[c];
        if (l.y == a) continue;  // unchanged since the last refresh
        l.y = a;
        L[c] = l;
        const float surf = (float)(l.x + a);
        A[c].x = surf;
        const double sd = s[c] + a;
        B[c].z = (float)(sd > 0.0 ? sd : 0.0);
        // the route flag follows the live surface; a lake cell stays a lake cell (particle.py:1010-1012)
        if (R && R[c].y < 1.5f) R[c].y = R[c].x != surf ? 1.0f : 0.0f;
    }
}

// the routing surface and its flag, beside the packed surface (particle.py:165-190): 2 on an
// overflowing lake, 3 on one with room for its rivers' load, else 1 where the route is not the surface
__global__ void pack_route_kernel(long long ncell, const double *__restrict__ h, const double *__restrict__ s,
                                  const double *__restrict__ route, const uint8_t *__restrict__ lake, float2 *R)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const float r = (float)route[c], surf = (float)(h[c] + s[c]);
        const uint8_t lk = lake ? lake[c] : (uint8_t)0;
        R[c] = make_float2(r, lk > 0 ? (lk > 1 ? 3.0f : 2.0f) : (r != surf ? 1.0f : 0.0f));
    }
}

// the lakes of a window (maps.py:662-672): interior active cells the routing surface covers more
// than min_depth deep
__global__ void window_lakes_kernel(long long ncell, int N, int H, const double *__restrict__ h, const double *__restrict__ s,
                                    const double *__restrict__ route, const uint8_t *__restrict__ mask, double min_depth,
                                    uint8_t *flag, unsigned long long *count)
{
    const int NE = N + 2 * H;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(c % NE), i = (int)((c / NE) % NE);
        const bool inner = i >= H && i < H + N && j >= H && j < H + N;
        const bool lake = inner && (!mask || mask[c] == PGE_MASK_ACTIVE) && route[c] - (h[c] + s[c]) > min_depth;
        flag[c] = lake ? 1 : 0;
        const unsigned ballot = __ballot_sync(__activemask(), lake);
        if (count && ballot && (threadIdx.x & 31) == __ffs(ballot) - 1) atomicAdd(count, (unsigned long long)__popc(ballot));
    }
}

// the accumulators as float64: fixed point (wave apply) or plain float64 (ordered apply)
__device__ __forceinline__ void acc_values(const long long *acc4, const long long *pend, long long c, int exact, double &a,
                                           double &q, double &ma, double &mb, double &pd)
{
    if (exact) {
        const double *d4 = reinterpret_cast<const double *>(acc4);
        a = d4[4 * c];
        q = d4[4 * c + 1];
        ma = d4[4 * c + 2];
        mb = d4[4 * c + 3];
        pd = reinterpret_cast<const double *>(pend)[c];
    } else {
        a = (double)acc4[4 * c] * INV_FX_MASS;
        q = (double)acc4[4 * c + 1] * INV_FX_TRACK;
        ma = (double)acc4[4 * c + 2] * INV_FX_TRACK;
        mb = (double)acc4[4 * c + 3] * INV_FX_TRACK;
        pd = (double)pend[c] * INV_FX_MASS;
    }
}

__global__ void fold_ema_kernel(long long ncell, double *h, double *s, double *q, double *mom, double *pending,
                                const uint8_t *__restrict__ mask, const long long *__restrict__ acc4,
                                const long long *__restrict__ pend, double ema, int exact)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const bool act = mask ? mask[c] == PGE_MASK_ACTIVE : true;
        double a, tq, tma, tmb, pd;
        acc_values(acc4, pend, c, exact, a, tq, tma, tmb, pd);
        if (a != 0.0 && act) {
            if (a > 0.0) {
                s[c] += a;
            } else {
                const double take = -a, sd = s[c];
                if (sd >= take) {
                    s[c] = sd - take;
                } else {
                    h[c] -= take - sd;
                    s[c] = 0.0;
                }
            }
        }
        if (act) {
            q[c] = (1.0 - ema) * q[c] + ema * tq;
            mom[2 * c] = (1.0 - ema) * mom[2 * c] + ema * tma;
            mom[2 * c + 1] = (1.0 - ema) * mom[2 * c + 1] + ema * tmb;
        }
        if (pd != 0.0) pending[c] += pd;
    }
}

__global__ void read_acc_kernel(long long ncell, const long long *__restrict__ acc4, const long long *__restrict__ pend,
                                const unsigned long long *mode, double *acc, double *dtr, double *mtr, double *pending)
{
    const int exact = (int)*mode;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        double a, q, ma, mb, pd;
        acc_values(acc4, pend, c, exact, a, q, ma, mb, pd);
        if (acc) acc[c] = a;
        if (dtr) dtr[c] = q;
        if (mtr) {
            mtr[2 * c] = ma;
            mtr[2 * c + 1] = mb;
        }
        if (pending) pending[c] = pd;
    }
}

void pack(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, cudaStream_t st)
{
    const long long n = lay.ncell;
    pack_kernel<<<grid_for(n), 256, 0, st>>>(n, s.height, s.sediment, s.discharge, s.momentum, s.evap, s.hardness, s.base,
                                             ws_ptr<float4>(ws, lay.cellA), ws_ptr<float4>(ws, lay.cellB),
                                             ws_ptr<double2>(ws, lay.live));
    pack_metric_kernel<<<grid_for(lay.nmetric), 256, 0, st>>>(lay.nmetric, s.metric, s.metric_inv, ws_ptr<float4>(ws, lay.metric8));
    if (s.route)
        pack_route_kernel<<<grid_for(n), 256, 0, st>>>(n, s.height, s.sediment, s.route, s.lake_flag, ws_ptr<float2>(ws, lay.route2));
}

void refresh(const PgeState &s, const Layout &lay, void *ws, cudaStream_t st)
{
    refresh_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, s.sediment, ws_ptr<long long>(ws, lay.acc4),
                                                       ws_ptr<float4>(ws, lay.cellA), ws_ptr<float4>(ws, lay.cellB),
                                                       ws_ptr<double2>(ws, lay.live), s.route ? ws_ptr<float2>(ws, lay.route2) : nullptr);
}

void fold_ema(PgeState &s, const Layout &lay, void *ws, double ema, int exact, cudaStream_t st)
{
    fold_ema_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, s.height, s.sediment, s.discharge, s.momentum, s.pending,
                                                        s.mask, ws_ptr<long long>(ws, lay.acc4), ws_ptr<long long>(ws, lay.pend),
                                                        ema, exact);
}

void read_accumulators(const Layout &lay, void *ws, double *acc, double *dtr, double *mtr, double *pending, cudaStream_t st)
{
    read_acc_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, ws_ptr<long long>(ws, lay.acc4),
                                                        ws_ptr<long long>(ws, lay.pend),
                                                        ws_ptr<unsigned long long>(ws, lay.counters) + 4, acc, dtr, mtr, pending);
}

// ---------------------------------------------------------------------------
// the erode / deposit brush: the change each cell received since the last spread (the wave apply adds
// every entry's applied change to its own cell) is shared out over the active cells of its face within
// distance < r + 1 (the interior ones on the sphere), weights r + 1 - distance in integers of
// 1/PGE_BRUSH_SCALE renormalised over the footprint; each share is truncated toward zero and the rest
// stays on the cell, so the total is kept exactly.  A gather: each cell adds the shares its neighbours
// send it, computed by the same expression the sender uses for its rest, so no atomics are needed and the
// result is the same whatever the order.
// ---------------------------------------------------------------------------
struct BrushGeo {
    int NE, lo, hi, r;
    const uint8_t *mask;
};

__device__ __forceinline__ int brush_weight(int r, int di, int dj)
{
    const double v = (double)(r + 1) - sqrt((double)(di * di + dj * dj));
    return v > 0.0 ? (int)llround(PGE_BRUSH_SCALE * v) : 0;
}

__device__ __forceinline__ bool brush_valid(const BrushGeo &g, long long fb, int i, int j)
{
    if (i < g.lo || i >= g.hi || j < g.lo || j >= g.hi) return false;
    return !g.mask || g.mask[fb + (long long)i * g.NE + j] == PGE_MASK_ACTIVE;
}

__device__ __forceinline__ long long brush_share(long long d, int q, int Q) { return (long long)((double)d * (double)q / (double)Q); }

// pass 1: each cell's change since the last spread and, where it has one, its footprint's total weight
__global__ void brush_delta_kernel(long long ncell, BrushGeo g, const long long *acc4, const long long *prev, long long *delta, int *Q)
{
    const long long plane = (long long)g.NE * g.NE;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const long long d = acc4[4 * c] - prev[c];
        delta[c] = d;
        int q = 0;
        if (d != 0) {
            const long long fb = c / plane * plane;
            const int ei = (int)((c - fb) / g.NE), ej = (int)((c - fb) % g.NE);
            for (int di = -g.r; di <= g.r; di++)
                for (int dj = -g.r; dj <= g.r; dj++) {
                    const int w = brush_weight(g.r, di, dj);
                    if (w && ((di == 0 && dj == 0) || brush_valid(g, fb, ei + di, ej + dj))) q += w;
                }
        }
        Q[c] = q;
    }
}

// pass 2: the shares the footprint sends each cell, plus the rest of its own change; net change = the last spread + that
__global__ void brush_gather_kernel(long long ncell, BrushGeo g, const long long *delta, const int *Q, long long *acc4, long long *prev)
{
    const long long plane = (long long)g.NE * g.NE;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const long long fb = c / plane * plane;
        const int ei = (int)((c - fb) / g.NE), ej = (int)((c - fb) % g.NE);
        long long sum = 0;
        if (brush_valid(g, fb, ei, ej))
            for (int di = -g.r; di <= g.r; di++) {
                const int i = ei + di;
                if (i < 0 || i >= g.NE) continue;
                for (int dj = -g.r; dj <= g.r; dj++) {
                    const int j = ej + dj;
                    const int w = brush_weight(g.r, di, dj);
                    if (!w || (di == 0 && dj == 0) || j < 0 || j >= g.NE) continue;
                    const long long s = fb + (long long)i * g.NE + j;
                    const long long d = delta[s];
                    if (d != 0) sum += brush_share(d, w, Q[s]);
                }
            }
        const long long d = delta[c];
        if (d != 0) {
            long long kept = d;
            for (int di = -g.r; di <= g.r; di++)
                for (int dj = -g.r; dj <= g.r; dj++) {
                    const int w = brush_weight(g.r, di, dj);
                    if (!w || (di == 0 && dj == 0) || !brush_valid(g, fb, ei + di, ej + dj)) continue;
                    kept -= brush_share(d, w, Q[c]);
                }
            sum += kept;
        }
        if (sum != 0 || d != 0) {
            const long long v = prev[c] + sum;
            acc4[4 * c] = v;
            prev[c] = v;
        }
    }
}

void brush_spread(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, int r, cudaStream_t st)
{
    const int NE = g.N + 2 * g.H;
    BrushGeo bg{NE, g.spherical ? g.H : 0, g.spherical ? g.H + g.N : NE, r, s.mask};
    long long *acc4 = ws_ptr<long long>(ws, lay.acc4);
    long long *prev = ws_ptr<long long>(ws, lay.spread);
    long long *delta = ws_ptr<long long>(ws, lay.pwv);
    int *Q = ws_ptr<int>(ws, lay.flags);
    brush_delta_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, bg, acc4, prev, delta, Q);
    brush_gather_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, bg, delta, Q, acc4, prev);
}

// ---------------------------------------------------------------------------
// thermal erosion (talus / creep mass wasting)
// ---------------------------------------------------------------------------
struct ThermalArgs {
    int F, NE;
    const double *h, *s;
    const float *metric;  // (NE,NE,3) shared or (F,NE,NE,3)
    int metric_shared;
    const float *hard;    // talus = soft + (hard - soft) * hardness, in float32; nullptr: talus 0
    float talus_soft, talus_diff;
    const uint8_t *mask;  // nullptr: all active
    const double *base;   // creep: submerged cells (h + s < base) are frozen
    int creep;
    double rate, cap, dep_floor;
    double *out_total, *scale, *rscale, *new_h, *new_s;
};

__device__ __forceinline__ int tmask(const ThermalArgs &t, long long c)
{
    int m = t.mask ? t.mask[c] : PGE_MASK_ACTIVE;
    if (t.creep && t.h[c] + t.s[c] < t.base[c]) m = PGE_MASK_FROZEN;
    return m;
}

__device__ __forceinline__ double tout(const ThermalArgs &t, long long c, int k)
{
    const int di = kD8[k][0], dj = kD8[k][1];
    const long long nc = c + (long long)di * t.NE + dj;
    const double d = (t.h[c] + t.s[c]) - (t.h[nc] + t.s[nc]);
    if (d <= 0.0) return 0.0;
    const long long mc = t.metric_shared ? c % ((long long)t.NE * t.NE) : c;
    const double g0 = t.metric[3 * mc], g1 = t.metric[3 * mc + 1], g2 = t.metric[3 * mc + 2];
    const double dist = sqrt(g0 * di * di + 2.0 * g1 * di * dj + g2 * dj * dj);
    double talus = 0.0;
    if (t.hard) talus = (double)__fadd_rn(t.talus_soft, __fmul_rn(t.talus_diff, t.hard[c]));
    const double ex = d - talus * dist;
    if (ex <= 0.0) return 0.0;
    return 0.5 * t.rate * ex;
}

#define THERMAL_LOOP                                                                                            \
    const long long total = (long long)t.F * t.NE * t.NE;                                                       \
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x)

__global__ void thermal_a_kernel(const ThermalArgs t)
{
    THERMAL_LOOP
    {
        const int i = (int)((c / t.NE) % t.NE), j = (int)(c % t.NE);
        double ot = 0.0, sc_out = 0.0;
        if (i >= 1 && i < t.NE - 1 && j >= 1 && j < t.NE - 1 && tmask(t, c) == PGE_MASK_ACTIVE) {
            double S = 0.0, mx = 0.0;
            for (int k = 0; k < 8; k++) {
                if (tmask(t, c + (long long)kD8[k][0] * t.NE + kD8[k][1]) != PGE_MASK_ACTIVE) continue;
                const double o = tout(t, c, k);
                S += o;
                if (o > mx) mx = o;
            }
            if (S > 0.0) {
                double sc = 1.0;
                if (S > 2.0 * mx) sc = 2.0 * mx / S;
                if (t.cap > 0.0 && S * sc > t.cap) sc = t.cap / S;
                ot = S * sc;
                sc_out = sc;
            }
        }
        t.out_total[c] = ot;
        t.scale[c] = sc_out;
    }
}

__global__ void thermal_r_kernel(const ThermalArgs t)
{
    THERMAL_LOOP
    {
        const int i = (int)((c / t.NE) % t.NE), j = (int)(c % t.NE);
        double rs = 1.0;
        if (i >= 1 && i < t.NE - 1 && j >= 1 && j < t.NE - 1) {
            const double surf = t.h[c] + t.s[c];
            if (!(surf >= 0.0 || tmask(t, c) != PGE_MASK_ACTIVE)) {
                double inflow = 0.0;
                for (int k = 0; k < 8; k++) {
                    const long long nc = c + (long long)kD8[k][0] * t.NE + kD8[k][1];
                    const double sc = t.scale[nc];
                    if (sc <= 0.0 || tmask(t, nc) == PGE_MASK_OUTSIDE) continue;
                    inflow += sc * tout(t, nc, (k + 4) % 8);
                }
                double room = -t.dep_floor - surf;
                if (room < 0.0) room = 0.0;
                if (inflow > room) rs = room / inflow;
            }
        }
        t.rscale[c] = rs;
    }
}

__global__ void thermal_b_kernel(const ThermalArgs t)
{
    THERMAL_LOOP
    {
        const int i = (int)((c / t.NE) % t.NE), j = (int)(c % t.NE);
        double h = t.h[c], s = t.s[c];
        if (i >= 1 && i < t.NE - 1 && j >= 1 && j < t.NE - 1 && tmask(t, c) == PGE_MASK_ACTIVE) {
            double inflow = 0.0, out = 0.0;
            const double sc_self = t.scale[c];
            for (int k = 0; k < 8; k++) {
                const long long nc = c + (long long)kD8[k][0] * t.NE + kD8[k][1];
                const int mn = tmask(t, nc);
                if (mn == PGE_MASK_OUTSIDE) continue;
                if (sc_self > 0.0 && mn == PGE_MASK_ACTIVE) out += sc_self * t.rscale[nc] * tout(t, c, k);
                const double sc = t.scale[nc];
                if (sc <= 0.0) continue;
                inflow += sc * tout(t, nc, (k + 4) % 8);
            }
            inflow *= t.rscale[c];
            if (out > 0.0) {
                if (s >= out) {
                    s -= out;
                } else {
                    h -= out - s;
                    s = 0.0;
                }
            }
            s = s + inflow;
        }
        t.new_h[c] = h;
        t.new_s[c] = s;
    }
}

__global__ void copy2_kernel(long long n, const double *a, const double *b, double *da, double *db)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        da[c] = a[c];
        db[c] = b[c];
    }
}

void thermal(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double rate, double creep_rate, double cap,
             float soft, float diff, double dep_floor, cudaStream_t st)
{
    double *tb = ws_ptr<double>(ws, lay.thermal);
    const long long n = lay.ncell;
    ThermalArgs t;
    t.F = g.F;
    t.NE = g.N + 2 * g.H;
    t.h = s.height;
    t.s = s.sediment;
    t.metric = s.metric;
    t.metric_shared = g.metric_shared;
    t.talus_soft = soft;
    t.talus_diff = diff;
    t.mask = s.mask;
    t.base = s.base;
    t.dep_floor = dep_floor;
    t.cap = cap;
    t.out_total = tb;
    t.scale = tb + n;
    t.rscale = tb + 2 * n;
    t.new_h = tb + 3 * n;
    t.new_s = tb + 4 * n;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1 && !(creep_rate > 0.0)) break;
        t.hard = pass == 0 ? s.hardness : nullptr;
        t.creep = pass;
        t.rate = pass == 0 ? rate : creep_rate;
        thermal_a_kernel<<<grid_for(n), 256, 0, st>>>(t);
        thermal_r_kernel<<<grid_for(n), 256, 0, st>>>(t);
        thermal_b_kernel<<<grid_for(n), 256, 0, st>>>(t);
        copy2_kernel<<<grid_for(n), 256, 0, st>>>(n, t.new_h, t.new_s, s.height, s.sediment);
    }
}

// the same passes on caller-provided scratch (5 * ncell doubles), for the
// entry point that allocates nothing (pge_static.cu)
void thermal_on_scratch(const PgeGrid &g, PgeState &s, double *tb, long long n, double rate, double creep_rate, double cap,
                        float soft, float diff, double dep_floor, cudaStream_t st)
{
    ThermalArgs t;
    t.F = g.F;
    t.NE = g.N + 2 * g.H;
    t.h = s.height;
    t.s = s.sediment;
    t.metric = s.metric;
    t.metric_shared = g.metric_shared;
    t.talus_soft = soft;
    t.talus_diff = diff;
    t.mask = s.mask;
    t.base = s.base;
    t.dep_floor = dep_floor;
    t.cap = cap;
    t.out_total = tb;
    t.scale = tb + n;
    t.rscale = tb + 2 * n;
    t.new_h = tb + 3 * n;
    t.new_s = tb + 4 * n;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1 && !(creep_rate > 0.0)) break;
        t.hard = pass == 0 ? s.hardness : nullptr;
        t.creep = pass;
        t.rate = pass == 0 ? rate : creep_rate;
        thermal_a_kernel<<<grid_for(n), 256, 0, st>>>(t);
        thermal_r_kernel<<<grid_for(n), 256, 0, st>>>(t);
        thermal_b_kernel<<<grid_for(n), 256, 0, st>>>(t);
        copy2_kernel<<<grid_for(n), 256, 0, st>>>(n, t.new_h, t.new_s, s.height, s.sediment);
    }
}

struct UpliftValue {
    const double *u;
    double cap;
    int use_cap;
    __device__ __forceinline__ double operator()(const long long c) const
    {
        const double v = u[c];
        return use_cap && v > cap ? cap : v;
    }
};

struct InteriorActive {
    int NE, H, N;
    const uint8_t *mask;
    __device__ __forceinline__ bool operator()(const long long c) const
    {
        return interior(c, NE, H, N) && (!mask || mask[c] == PGE_MASK_ACTIVE);
    }
};

struct Positive {
    __device__ __forceinline__ bool operator()(const double x) const { return x > 0.0; }
};

// ---------------------------------------------------------------------------
// numpy's pairwise summation, so that a float64 sum the reference takes with
// numpy (ndarray.sum / mean of a contiguous float64 array) is reproduced bit for
// bit: n < 8 values are added one by one to 0; up to 128 values are added as
// eight running sums over the leading multiple of 8, combined as
// ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), and the rest added one by
// one; a longer range is split at n2 = n/2 rounded down to a multiple of 8 and
// the two halves' sums added.  (numpy's pairwise_sum, the reduction loop of
// np.add; checked against np.sum on ranges of 1..5000 values of mixed
// magnitudes.)  The top of the tree is expanded breadth-first into at most
// PW_MAX_LEVEL_NODES nodes a level (one block, a level at a time); the bottom
// nodes are summed one per thread and the tree is folded back up in order (one
// block, a level at a time).
// ---------------------------------------------------------------------------
constexpr int PW_LEAF = 128;
constexpr int PW_MAX_LEVELS = 24;
constexpr int PW_MAX_LEVEL_NODES = 32768;
constexpr int PW_THREADS = 1024;

struct PwNode {
    long long lo, n;
    int child, nchild;  // children in the next level
    double sum;
};

__device__ double pw_leaf(const double *a, long long n)
{
    if (n < 8) {
        double res = 0.0;
        for (long long i = 0; i < n; i++) res += a[i];
        return res;
    }
    double r0 = a[0], r1 = a[1], r2 = a[2], r3 = a[3], r4 = a[4], r5 = a[5], r6 = a[6], r7 = a[7];
    long long i = 8;
    for (; i < n - (n % 8); i += 8) {
        r0 += a[i];
        r1 += a[i + 1];
        r2 += a[i + 2];
        r3 += a[i + 3];
        r4 += a[i + 4];
        r5 += a[i + 5];
        r6 += a[i + 6];
        r7 += a[i + 7];
    }
    double res = ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7));
    for (; i < n; i++) res += a[i];
    return res;
}

__device__ __forceinline__ long long pw_split(long long n)
{
    const long long n2 = n / 2;
    return n2 - n2 % 8;
}

// the pairwise sum of a[0, n) by an explicit post-order walk (depth <= 40 for any n < 2^40)
__device__ double pw_sum(const double *a, long long n)
{
    if (n <= PW_LEAF) return pw_leaf(a, n);
    long long lo[40], len[40];
    double left[40];
    int stage[40];
    int sp = 0;
    lo[0] = 0;
    len[0] = n;
    stage[0] = 0;
    double v = 0.0;
    while (true) {
        const int t = sp;
        if (len[t] <= PW_LEAF || stage[t] == 2) {
            // a finished node: a leaf, or both halves done (v holds the right half)
            v = len[t] <= PW_LEAF ? pw_leaf(a + lo[t], len[t]) : left[t] + v;
            if (sp == 0) return v;
            sp--;
            if (stage[sp] == 1) {  // the left half just finished: keep it, descend into the right half
                left[sp] = v;
                const long long n2 = pw_split(len[sp]);
                stage[sp] = 2;
                sp++;
                lo[sp] = lo[sp - 1] + n2;
                len[sp] = len[sp - 1] - n2;
                stage[sp] = 0;
            }
            continue;
        }
        stage[t] = 1;  // descend into the left half
        sp++;
        lo[sp] = lo[t];
        len[sp] = pw_split(len[t]);
        stage[sp] = 0;
    }
}

// one block of PW_THREADS: a level's nodes split among the threads in order, each thread's children placed
// after those of the threads before it (a block scan of the counts)
__global__ void __launch_bounds__(PW_THREADS) pw_plan_kernel(const long long *count, PwNode *nodes, int *level_start)
{
    typedef cub::BlockScan<int, PW_THREADS> Scan;
    typedef cub::BlockReduce<long long, PW_THREADS> Reduce;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ typename Reduce::TempStorage red_tmp;
    __shared__ long long s_biggest;
    __shared__ int s_next;
    const int t = threadIdx.x;
    const long long M = *count;
    if (t == 0) {
        nodes[0] = PwNode{0, M, -1, 0, 0.0};
        level_start[0] = 0;
    }
    __syncthreads();
    int nl = 0, begin = 0, end = 1;
    while (nl + 1 < PW_MAX_LEVELS) {
        const int nnodes = end - begin;
        const int per = (nnodes + PW_THREADS - 1) / PW_THREADS;
        const int k0 = begin + t * per, k1 = min(k0 + per, end);
        long long big = 0;
        int nch = 0;
        for (int k = k0; k < k1; k++) {
            big = nodes[k].n > big ? nodes[k].n : big;
            nch += nodes[k].n > PW_LEAF ? 2 : 1;
        }
        const long long b = Reduce(red_tmp).Reduce(big, cub::Max());
        if (t == 0) s_biggest = b;
        __syncthreads();
        if (s_biggest <= 8 * PW_LEAF || 2 * nnodes > PW_MAX_LEVEL_NODES) break;
        int off, total;
        Scan(scan_tmp).ExclusiveSum(nch, off, total);
        int next = end + off;
        for (int k = k0; k < k1; k++) {
            PwNode &nd = nodes[k];
            nd.child = next;
            if (nd.n > PW_LEAF) {
                const long long n2 = pw_split(nd.n);
                nodes[next++] = PwNode{nd.lo, n2, -1, 0, 0.0};
                nodes[next++] = PwNode{nd.lo + n2, nd.n - n2, -1, 0, 0.0};
                nd.nchild = 2;
            } else {
                nodes[next++] = PwNode{nd.lo, nd.n, -1, 0, 0.0};  // a leaf passes down unchanged
                nd.nchild = 1;
            }
        }
        if (t == 0) s_next = end + total;
        __syncthreads();
        begin = end;
        end = s_next;
        nl++;
        if (t == 0) level_start[nl] = begin;
        __syncthreads();
    }
    if (t == 0) {
        level_start[nl + 1] = end;
        level_start[PW_MAX_LEVELS + 1] = nl;  // the bottom level's index
    }
}

__global__ void pw_bottom_kernel(const double *a, PwNode *nodes, const int *level_start)
{
    const int nl = level_start[PW_MAX_LEVELS + 1];
    const int begin = level_start[nl], end = level_start[nl + 1];
    for (int k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x)
        nodes[k].sum = pw_sum(a + nodes[k].lo, nodes[k].n);
}

// folds the levels back up, a level at a time (one block); out = the sum, or with mean_out the sum / count
__global__ void __launch_bounds__(PW_THREADS) pw_fold_kernel(PwNode *nodes, const int *level_start, const long long *count,
                                                             double *out, int mean_out)
{
    const int nl = level_start[PW_MAX_LEVELS + 1];
    for (int l = nl - 1; l >= 0; l--) {
        for (int k = level_start[l] + threadIdx.x; k < level_start[l + 1]; k += blockDim.x) {
            PwNode &nd = nodes[k];
            nd.sum = nd.nchild == 2 ? nodes[nd.child].sum + nodes[nd.child + 1].sum : nodes[nd.child].sum;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const long long M = *count;
        *out = mean_out ? (M > 0 ? nodes[0].sum / (double)M : 0.0) : nodes[0].sum;
    }
}

size_t pairwise_scratch_bytes() { return sizeof(PwNode) * (size_t)PW_MAX_LEVELS * PW_MAX_LEVEL_NODES + 256; }

// sum (or mean) of a[0, *count) in numpy's pairwise order, written to *out on the stream
void pairwise_sum(const double *a, const long long *count, void *scratch, double *out, int mean, cudaStream_t st)
{
    PwNode *nodes = static_cast<PwNode *>(scratch);
    int *level_start = reinterpret_cast<int *>(nodes + (size_t)PW_MAX_LEVELS * PW_MAX_LEVEL_NODES);
    pw_plan_kernel<<<1, PW_THREADS, 0, st>>>(count, nodes, level_start);
    pw_bottom_kernel<<<(PW_MAX_LEVEL_NODES + 127) / 128, 128, 0, st>>>(a, nodes, level_start);
    pw_fold_kernel<<<1, PW_THREADS, 0, st>>>(nodes, level_start, count, out, mean);
}

// ---------------------------------------------------------------------------
// uplift and the datum's order statistic
// ---------------------------------------------------------------------------
constexpr int RED_BLOCKS = 1024;  // the partial-result area of the workspace: scalars of the uplift and the select

__global__ void uplift_add_kernel(long long ncell, double *h, const double *u, const uint8_t *mask, double cap, int use_cap,
                                  const double *mean, double scale)
{
    const double m = mean ? *mean : 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        if (mask && mask[c] != PGE_MASK_ACTIVE) continue;
        double v = u[c];
        if (use_cap && v > cap) v = cap;
        h[c] += scale * (v - m);
    }
}

void uplift(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double cap, double scale, cudaStream_t st)
{
    // maps._applied_uplift (maps.py:1136-1147): the mean of the (capped) field over the interior active
    // cells, u[interior][active].mean() -- their values in cell order, summed in numpy's pairwise order
    const int NE = g.N + 2 * g.H;
    const int use_cap = cap >= 0.0;
    double *partial = ws_ptr<double>(ws, lay.partial);
    long long *pcount = reinterpret_cast<long long *>(partial + RED_BLOCKS);
    double *mean = partial + 2 * RED_BLOCKS;
    if (g.spherical) {
        double *vals = ws_ptr<double>(ws, lay.pwv);
        size_t tb = lay.cubtmp_bytes;
        const thrust::counting_iterator<long long> c0(0);
        cub::DeviceSelect::Flagged(ws_ptr<void>(ws, lay.cubtmp), tb,
                                   thrust::make_transform_iterator(c0, UpliftValue{s.uplift, cap, use_cap}),
                                   thrust::make_transform_iterator(c0, InteriorActive{NE, g.H, g.N, s.mask}), vals, pcount,
                                   (int)lay.ncell, st);
        pairwise_sum(vals, pcount, ws_ptr<void>(ws, lay.pwnode), mean, 1, st);
    }
    uplift_add_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, s.height, s.uplift, s.mask, cap, use_cap,
                                                           g.spherical ? mean : nullptr, scale);
}

// ---------------------------------------------------------------------------
// datum: k-th smallest interior surface by an 8-pass radix select on the
// order-preserving 64-bit image of the float64 keys
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long okey(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double unokey(unsigned long long k)
{
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

struct SelectState {
    unsigned long long prefix;  // digits found so far (high bits)
    long long k;                // rank still sought inside the prefix
    unsigned int hist[256];
};

__global__ void select_hist_kernel(long long ncell, int NE, int H, int N, const double *h, const double *s, SelectState *ss,
                                   int shift)
{
    __shared__ unsigned int sh[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const unsigned long long prefix = ss->prefix;
    const unsigned long long hmask = shift >= 56 ? 0ull : (~0ull << (shift + 8));
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        if (!interior(c, NE, H, N)) continue;
        const unsigned long long k = okey(h[c] + s[c]);
        if ((k & hmask) != (prefix & hmask)) continue;
        atomicAdd(&sh[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&ss->hist[i], sh[i]);
}

__global__ void select_pick_kernel(SelectState *ss, int shift)
{
    if (threadIdx.x == 0) {
        long long k = ss->k;
        int d = 0;
        for (; d < 255; d++) {
            const long long c = ss->hist[d];
            if (k < c) break;
            k -= c;
        }
        ss->k = k;
        ss->prefix |= (unsigned long long)d << shift;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x) ss->hist[i] = 0;
}

__global__ void select_init_kernel(SelectState *ss, long long k)
{
    for (int i = threadIdx.x; i < 256; i += blockDim.x) ss->hist[i] = 0;
    if (threadIdx.x == 0) {
        ss->prefix = 0;
        ss->k = k;
    }
}

__global__ void datum_shift_kernel(long long ncell, double *h, double *base, const SelectState *ss, double level, int plus_one,
                                   double *shift_out)
{
    double q = unokey(ss->prefix);
    if (plus_one) q += 1.0;
    q -= level;
    if (blockIdx.x == 0 && threadIdx.x == 0) *shift_out = q;
    if (q == 0.0) return;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        h[c] -= q;
        if (base[c] < 0.0) base[c] -= q;
    }
}

void hold_datum(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double land_fraction, double level,
                double *shift_dev, cudaStream_t st)
{
    const int NE = g.N + 2 * g.H;
    const long long M = (long long)g.F * g.N * g.N;
    long long n_land = (long long)llrint(land_fraction * (double)M);  // numpy round: half to even
    if (n_land < 0) n_land = 0;
    if (n_land > M) n_land = M;
    long long k;
    int plus_one = 0;
    if (n_land == 0) {
        k = M - 1;
        plus_one = 1;
    } else {
        k = M - n_land;
    }
    SelectState *ss = ws_ptr<SelectState>(ws, lay.partial + 4 * RED_BLOCKS * sizeof(double));
    select_init_kernel<<<1, 256, 0, st>>>(ss, k);
    for (int shift = 56; shift >= 0; shift -= 8) {
        select_hist_kernel<<<grid_reduce(lay.ncell), 256, 0, st>>>(lay.ncell, NE, g.H, g.N, s.height, s.sediment, ss, shift);
        select_pick_kernel<<<1, 256, 0, st>>>(ss, shift);
    }
    datum_shift_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, s.height, s.base, ss, level, plus_one, shift_dev);
}

// ---------------------------------------------------------------------------
// halo gather
// ---------------------------------------------------------------------------
__global__ void halo_scalar_kernel(long long K, const int32_t *dst, const int32_t *src, const double *w, double *f)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < K; k += (long long)gridDim.x * blockDim.x) {
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 16; q++) acc += w[16 * k + q] * f[src[16 * k + q]];
        f[dst[k]] = acc;
    }
}

__global__ void halo_vector_kernel(long long K, const int32_t *dst, const int32_t *src, const double *w, const double *rot,
                                   double *f)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < K; k += (long long)gridDim.x * blockDim.x) {
        double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
        for (int q = 0; q < 16; q++) {
            const long long sidx = src[16 * k + q];
            const double va = f[2 * sidx], vb = f[2 * sidx + 1];
            const double *R = rot + 4 * (16 * k + q);
            const double wq = w[16 * k + q];
            a0 += wq * (R[0] * va + R[1] * vb);
            a1 += wq * (R[2] * va + R[3] * vb);
        }
        f[2 * (long long)dst[k]] = a0;
        f[2 * (long long)dst[k] + 1] = a1;
    }
}

void halo_gather(const PgeHalo &h, double *field, int vector, cudaStream_t st)
{
    if (h.K <= 0) return;
    if (vector)
        halo_vector_kernel<<<grid_for(h.K), 256, 0, st>>>(h.K, h.dst, h.src, h.w, h.rot, field);
    else
        halo_scalar_kernel<<<grid_for(h.K), 256, 0, st>>>(h.K, h.dst, h.src, h.w, field);
}

// ---------------------------------------------------------------------------
// spawns
// ---------------------------------------------------------------------------
// a float32 x > 0 is m * 2^(e - 150) with m a 24-bit integer (e the biased exponent, 1 for subnormals)
__device__ __forceinline__ void f32_parts(float x, long long &m, int &e)
{
    const unsigned b = __float_as_uint(x);
    const unsigned E = (b >> 23) & 0xffu;
    m = (long long)((b & 0x7fffffu) | (E ? 0x800000u : 0u));
    e = E ? (int)E : 1;
}

__global__ void spawn_weight_kernel(long long ncell, int NE, int H, int N, const double *h, const double *s, const double *base,
                                    const uint8_t *mask, const float *precip, double *w, long long *lastc, long long *erange)
{
    long long last = -1;
    int emin = 1 << 20, emax = -1;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        const bool ok = interior(c, NE, H, N) && (!mask || mask[c] == PGE_MASK_ACTIVE) && (h[c] + s[c] >= base[c]) && precip[c] > 0.0f;
        w[c] = ok ? (double)precip[c] : 0.0;
        if (ok) {
            if (c > last) last = c;
            long long m;
            int e;
            f32_parts(precip[c], m, e);
            emin = e < emin ? e : emin;
            emax = e > emax ? e : emax;
        }
    }
    // the block's extremes first, then one atomic each a block
    typedef cub::BlockReduce<long long, 256> BR;
    typedef cub::BlockReduce<int, 256> BRi;
    __shared__ typename BR::TempStorage t0;
    __shared__ typename BRi::TempStorage t1, t2;
    last = BR(t0).Reduce(last, cub::Max());
    emin = BRi(t1).Reduce(emin, cub::Min());
    emax = BRi(t2).Reduce(emax, cub::Max());
    if (threadIdx.x == 0) {
        if (last >= 0) atomicMax(reinterpret_cast<unsigned long long *>(lastc), (unsigned long long)last);
        if (emax >= 0) {
            atomicMin(erange, (long long)emin);
            atomicMax(erange + 1, (long long)emax);
        }
    }
}

// The fixed-point unit of the weights' integer scan: 2^(base - 150), the smallest weight's
// last bit (so every weight is an integer of it and every prefix sum exact) unless the spread
// of exponents would overflow 62 bits over ncell weights.
__device__ __forceinline__ int spawn_fx_base(const long long *erange, long long ncell)
{
    int lg = 0;
    while ((1LL << lg) < ncell) lg++;
    const int emin = (int)erange[0], emax = (int)erange[1];
    const int need = emax + 24 + lg - 62;
    return emin > need ? emin : need;
}

__global__ void spawn_quant_kernel(long long ncell, const double *w, const long long *erange, long long *wq)
{
    const int base = spawn_fx_base(erange, ncell);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
        long long q = 0;
        if (w[c] > 0.0) {
            long long m;
            int e;
            f32_parts((float)w[c], m, e);
            const int sh = e - base;
            q = sh >= 0 ? m << sh : (sh > -40 ? (m + (1LL << (-sh - 1))) >> (-sh) : 0);
        }
        wq[c] = q;
    }
}

// the integer prefix sums back to float64, in place
__global__ void spawn_cdf_kernel(long long ncell, const long long *erange, double *cdf)
{
    const int base = spawn_fx_base(erange, ncell);
    long long *S = reinterpret_cast<long long *>(cdf);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        cdf[c] = ldexp((double)S[c], base - 150);
}

__global__ void spawn_count_kernel(long long ncell, const double *w, long long *count)
{
    long long n = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x)
        n += w[c] > 0.0;
    typedef cub::BlockReduce<long long, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    n = BR(tmp).Sum(n);
    if (threadIdx.x == 0 && n) atomicAdd(reinterpret_cast<unsigned long long *>(count), (unsigned long long)n);
}

__global__ void spawn_search_kernel(long long ncell, int NE, int H, const double *cdf, const long long *lastc, const double *u,
                                    const double *off, long long P, int32_t *face, double *x, double *y, double *sed, double *dir)
{
    const double total = cdf[ncell - 1];
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        const double target = u[p] * total;
        // first index with cdf > target (the reference walks its compacted cdf the same way)
        long long lo = 0, hi = ncell;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (cdf[mid] <= target) lo = mid + 1;
            else hi = mid;
        }
        long long c = lo < ncell ? lo : *lastc;
        const long long fa = c / ((long long)NE * NE);
        const long long rem = c - fa * NE * NE;
        const long long ei = rem / NE, ej = rem - ei * NE;
        face[p] = (int32_t)fa;
        x[p] = (double)(ei - H) + off[2 * p];
        y[p] = (double)(ej - H) + off[2 * p + 1];
        sed[p] = 0.0;
        dir[p] = 0.0;
    }
}

struct PendFlag {
    const double *pending;
    __device__ __forceinline__ bool operator()(const long long c) const { return pending[c] > 0.0; }
};

__global__ void pending_emit_kernel(const long long *idx, const long long *count, int NE, int H, double *pending, int32_t *face,
                                    double *x, double *y, double *sed, long long *released_fx)
{
    const long long n = *count;
    long long rel = 0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const long long c = idx[k];
        const long long fa = c / ((long long)NE * NE);
        const long long rem = c - fa * NE * NE;
        const long long ei = rem / NE, ej = rem - ei * NE;
        face[k] = (int32_t)fa;
        x[k] = (double)(ei - H) + 0.5;
        y[k] = (double)(ej - H) + 0.5;
        sed[k] = pending[c];
        rel += __double2ll_rn(pending[c] * FX_MASS);
        pending[c] = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) rel += __shfl_down_sync(0xffffffffu, rel, o);
    if ((threadIdx.x & 31) == 0 && rel) atomicAdd(reinterpret_cast<unsigned long long *>(released_fx), (unsigned long long)rel);
}

size_t cub_temp_bytes(int64_t ncell, int64_t max_droplets)
{
    size_t a = 0, b = 0, c = 0;
    cub::DeviceScan::InclusiveSum(nullptr, a, (double *)nullptr, (double *)nullptr, (int)ncell);
    cub::DeviceRadixSort::SortKeys(nullptr, b, (double *)nullptr, (double *)nullptr, (int)(max_droplets > 0 ? max_droplets : 1));
    cub::DeviceSelect::If(nullptr, c, thrust::counting_iterator<long long>(0), (long long *)nullptr, (long long *)nullptr,
                          (int)ncell, PendFlag{nullptr});
    size_t d = 0, f = 0, h = 0;
    cub::DeviceScan::InclusiveSum(nullptr, d, (long long *)nullptr, (long long *)nullptr, (int)ncell);
    cub::DeviceSelect::If(nullptr, f, (double *)nullptr, (double *)nullptr, (long long *)nullptr, (int)ncell, Positive{});
    cub::DeviceSelect::Flagged(nullptr, h, thrust::make_transform_iterator(thrust::counting_iterator<long long>(0), UpliftValue{}),
                               thrust::make_transform_iterator(thrust::counting_iterator<long long>(0), InteriorActive{}),
                               (double *)nullptr, (long long *)nullptr, (int)ncell);
    size_t m = a > b ? a : b;
    m = m > c ? m : c;
    m = m > d ? m : d;
    m = m > f ? m : f;
    return m > h ? m : h;
}

cudaError_t spawn_rain(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, const double *u, const double *off,
                       long long P, PgeSpawns &sp, double *total_dev, long long *nspawn_dev, cudaStream_t st)
{
    // maps.spawn_weights / spawn_particles (maps.py:793-833): w = precip on spawnable cells, their
    // cumulative sum (np.cumsum: sequential), total = w.sum() (numpy's pairwise order) and the inverse
    // CDF of the sorted uniforms (particle.spawn_cells).  The cumulative sum is an integer scan of the
    // weights in fixed point (their float32 bits), so it is order-free and equals the sequential float64
    // sum bit for bit whenever that sum is exact -- every prefix below 2^53 units of the smallest
    // weight's last bit (any float32 precip of 0.1 .. 3 over 6.3 M cells, or uniform rain).
    const int NE = g.N + 2 * g.H;
    double *w = ws_ptr<double>(ws, lay.cdf);
    double *cdf = w + lay.ncell;
    double *keys = ws_ptr<double>(ws, lay.sortkeys);
    long long *ctr = ws_ptr<long long>(ws, lay.counters);
    long long *lastc = ctr + 2, *erange = ctr + 24, *nsel = ctr + 26;  // slots 4 (the pass mode), 8, 12.. are taken
    long long *wq = ws_ptr<long long>(ws, lay.pwv);
    cudaError_t e = cudaMemsetAsync(lastc, 0, sizeof(long long), st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(erange, 0x7f, sizeof(long long), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(erange + 1, 0, sizeof(long long), st)) != cudaSuccess) return e;
    if (nspawn_dev && (e = cudaMemsetAsync(nspawn_dev, 0, sizeof(long long), st)) != cudaSuccess) return e;
    spawn_weight_kernel<<<grid_reduce(lay.ncell), 256, 0, st>>>(lay.ncell, NE, g.H, g.N, s.height, s.sediment, s.base, s.mask,
                                                             s.precip, w, lastc, erange);
    if (nspawn_dev) spawn_count_kernel<<<grid_reduce(lay.ncell), 256, 0, st>>>(lay.ncell, w, nspawn_dev);
    spawn_quant_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, w, erange, wq);
    size_t tb = lay.cubtmp_bytes;
    e = cub::DeviceScan::InclusiveSum(ws_ptr<void>(ws, lay.cubtmp), tb, wq, reinterpret_cast<long long *>(cdf), (int)lay.ncell, st);
    if (e != cudaSuccess) return e;
    spawn_cdf_kernel<<<grid_for(lay.ncell), 256, 0, st>>>(lay.ncell, erange, cdf);
    // the total weight in numpy's order: the spawnable weights compacted in cell order, summed pairwise
    double *wc = ws_ptr<double>(ws, lay.pwv);
    tb = lay.cubtmp_bytes;
    e = cub::DeviceSelect::If(ws_ptr<void>(ws, lay.cubtmp), tb, w, wc, nsel, (int)lay.ncell, Positive{}, st);
    if (e != cudaSuccess) return e;
    if (total_dev) pairwise_sum(wc, nsel, ws_ptr<void>(ws, lay.pwnode), total_dev, 0, st);
    tb = lay.cubtmp_bytes;
    e = cub::DeviceRadixSort::SortKeys(ws_ptr<void>(ws, lay.cubtmp), tb, u, keys, (int)P, 0, 64, st);
    if (e != cudaSuccess) return e;
    spawn_search_kernel<<<grid_for(P), 256, 0, st>>>(lay.ncell, NE, g.H, cdf, lastc, keys, off, P, sp.face, sp.x, sp.y, sp.sed,
                                                     sp.dir);
    return cudaPeekAtLastError();
}

cudaError_t count_pending(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, long long *count_dev, cudaStream_t st)
{
    long long *idx = ws_ptr<long long>(ws, lay.flags);
    long long *cnt = ws_ptr<long long>(ws, lay.counters) + 3;
    size_t tb = lay.cubtmp_bytes;
    cudaError_t e = cub::DeviceSelect::If(ws_ptr<void>(ws, lay.cubtmp), tb, thrust::counting_iterator<long long>(0), idx, cnt,
                                          (int)lay.ncell, PendFlag{s.pending}, st);
    if (e != cudaSuccess) return e;
    if (count_dev) e = cudaMemcpyAsync(count_dev, cnt, sizeof(long long), cudaMemcpyDeviceToDevice, st);
    return e;
}

cudaError_t collect_pending(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, PgeSpawns &sp, long long offset,
                            PgeStats *stats, cudaStream_t st)
{
    const int NE = g.N + 2 * g.H;
    long long *idx = ws_ptr<long long>(ws, lay.flags);
    const long long *count_dev = ws_ptr<long long>(ws, lay.counters) + 3;
    pending_emit_kernel<<<grid_for(lay.ncell / 64 + 1), 256, 0, st>>>(idx, count_dev, NE, g.H, s.pending, sp.face + offset,
                                                                     sp.x + offset, sp.y + offset, sp.sed + offset,
                                                                     reinterpret_cast<long long *>(&stats->released_fx));
    return cudaPeekAtLastError();
}

// ---------------------------------------------------------------------------
// soillib's pit-free erosion cap (particle.py:1046-1076): per active cell, k * |Godunov downhill
// gradient| of the surface, each axis the steeper of its two one-sided downhill differences
// (exit_slope off the array); float64 in the reference's operation order (no FMA in this file)
// ---------------------------------------------------------------------------
__global__ void slope_erode_cap_kernel(int F, int NE, const double *__restrict__ height, const double *__restrict__ sediment,
                                       const uint8_t *__restrict__ mask, double k, double exit_slope, double *__restrict__ out)
{
    const long long n = (long long)F * NE * NE;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        if (mask && mask[c] != PGE_MASK_ACTIVE) {
            out[c] = 0.0;
            continue;
        }
        const long long r = c % ((long long)NE * NE);
        const int i = (int)(r / NE), j = (int)(r - (long long)i * NE);
        const double h = height[c] + sediment[c];
        const double gxn = i == 0 ? exit_slope : h - (height[c - NE] + sediment[c - NE]);
        const double gxp = i == NE - 1 ? exit_slope : h - (height[c + NE] + sediment[c + NE]);
        const double gyn = j == 0 ? exit_slope : h - (height[c - 1] + sediment[c - 1]);
        const double gyp = j == NE - 1 ? exit_slope : h - (height[c + 1] + sediment[c + 1]);
        double gx = gxn > gxp ? gxn : gxp;
        double gy = gyn > gyp ? gyn : gyp;
        if (gx < 0.0) gx = 0.0;
        if (gy < 0.0) gy = 0.0;
        out[c] = k * sqrt(gx * gx + gy * gy);
    }
}

void slope_erode_cap(const PgeGrid &g, const PgeState &s, double k, double exit_slope, double *out, cudaStream_t st)
{
    const int NE = g.N + 2 * g.H;
    slope_erode_cap_kernel<<<grid_for((long long)g.F * NE * NE), 256, 0, st>>>(g.F, NE, s.height, s.sediment, s.mask, k, exit_slope,
                                                                             out);
}

// ---------------------------------------------------------------------------
// the isostasy smoother (maps.py:1331-1410): one explicit step of the metric-aware
// Laplace-Beltrami diffusion, FaceField.laplacian (field.py:179-188, 372-404) in flux form,
// (1/sqrt g) d_a(sqrt g g^ab d_b f), at extended indices 1..NE-2 of every face (0 on the outer
// ring), per m^2 and rounded to float32 as the reference's field is; then
//   out = a * in + (kappa * lap) * cell^2       (a = 1: a smoothing step; a = 0, kappa = 1: the
//                                                  Laplacian in cell units, for the step bound)
// float64 in the reference's operation order (no FMA in this file)
// ---------------------------------------------------------------------------
__global__ void smooth_step_kernel(int F, int NE, const double *__restrict__ d, const float *__restrict__ ginv_f,
                                   const float *__restrict__ sq_f, double c2, double kappa, int keep, double *__restrict__ out)
{
    const long long n = (long long)F * NE * NE;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long r = c % ((long long)NE * NE);
        const int i = (int)(r / NE), j = (int)(r - (long long)i * NE);
        double lap64 = 0.0;
        if (i >= 1 && i <= NE - 2 && j >= 1 && j <= NE - 2) {
            // the metric tables are the same on every face: index them by (i, j)
            auto G = [&](int ii, int jj, int k) { return (double)ginv_f[((long long)ii * NE + jj) * 3 + k]; };
            auto S = [&](int ii, int jj) { return (double)sq_f[(long long)ii * NE + jj]; };
            auto D = [&](int ii, int jj) { return d[c + (long long)(ii - i) * NE + (jj - j)]; };
            const double fj_c = 0.5 * (D(i, j + 1) - D(i, j - 1));
            const double fj_p = 0.5 * (D(i + 1, j + 1) - D(i + 1, j - 1));
            const double fj_m = 0.5 * (D(i - 1, j + 1) - D(i - 1, j - 1));
            const double fi_c = 0.5 * (D(i + 1, j) - D(i - 1, j));
            const double fi_p = 0.5 * (D(i + 1, j + 1) - D(i - 1, j + 1));
            const double fi_m = 0.5 * (D(i + 1, j - 1) - D(i - 1, j - 1));
            double gii = 0.5 * (G(i, j, 0) + G(i + 1, j, 0));
            double gij = 0.5 * (G(i, j, 1) + G(i + 1, j, 1));
            double sv = 0.5 * (S(i, j) + S(i + 1, j));
            const double Fi_p = sv * (gii * (D(i + 1, j) - D(i, j)) + gij * 0.5 * (fj_c + fj_p));
            gii = 0.5 * (G(i, j, 0) + G(i - 1, j, 0));
            gij = 0.5 * (G(i, j, 1) + G(i - 1, j, 1));
            sv = 0.5 * (S(i, j) + S(i - 1, j));
            const double Fi_m = sv * (gii * (D(i, j) - D(i - 1, j)) + gij * 0.5 * (fj_c + fj_m));
            double gjj = 0.5 * (G(i, j, 2) + G(i, j + 1, 2));
            gij = 0.5 * (G(i, j, 1) + G(i, j + 1, 1));
            sv = 0.5 * (S(i, j) + S(i, j + 1));
            const double Fj_p = sv * (gjj * (D(i, j + 1) - D(i, j)) + gij * 0.5 * (fi_c + fi_p));
            gjj = 0.5 * (G(i, j, 2) + G(i, j - 1, 2));
            gij = 0.5 * (G(i, j, 1) + G(i, j - 1, 1));
            sv = 0.5 * (S(i, j) + S(i, j - 1));
            const double Fj_m = sv * (gjj * (D(i, j) - D(i, j - 1)) + gij * 0.5 * (fi_c + fi_m));
            const double lap = (Fi_p - Fi_m + Fj_p - Fj_m) / S(i, j);
            lap64 = (double)(float)(lap / c2);  // per m^2, a float32 field
        }
        const double upd = kappa * lap64 * c2;
        out[c] = keep ? d[c] + upd : upd;
    }
}

void smooth_step(const PgeGrid &g, const double *in, const float *metric_inv, const float *sqrt_det, double kappa, int keep,
                 double cell_m, double *out, cudaStream_t st)
{
    const int NE = g.N + 2 * g.H;
    const double c2 = cell_m * cell_m;
    smooth_step_kernel<<<grid_for((long long)g.F * NE * NE), 256, 0, st>>>(g.F, NE, in, metric_inv, sqrt_det, c2, kappa, keep, out);
}

}  // namespace pge

namespace pge {

// ---------------------------------------------------------------------------
// routing surface: the epsilon-filled surface of a priority flood
// (globe/erosion/route.py:31-125), as the fixed point of a relaxation.  A cell
// reached from the seeds takes max(its surface, lowest reaching neighbour + eps);
// a heap flood reaches every cell first from its lowest reaching neighbour, so
// the fixed point is the heap flood's result value for value.  Neighbours are
// pushed to along the owner table (the reference's direction: from a popped cell
// to owner[its D8 neighbour]); values live as the datum select's order-preserving
// uint64 keys (okey) so a plain atomicMin keeps the lowest.
// ---------------------------------------------------------------------------
namespace {
enum : unsigned char { RF_EXCLUDED = 0, RF_FREE = 1, RF_SEED = 2 };
constexpr unsigned long long RF_UNREACHED = 0xFFFFFFFFFFFFFFFFull;
__constant__ int kRouteD8[8][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, -1}};

}  // namespace

__global__ void route_init_kernel(int F, int NE, int H, int N, const double *__restrict__ h, const double *__restrict__ s,
                                  const double *__restrict__ base, const uint8_t *__restrict__ mask, const int32_t *__restrict__ owner,
                                  unsigned long long *key, unsigned char *state)
{
    const long long total = (long long)F * NE * NE;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(c / ((long long)NE * NE));
        const int ei = (int)((c / NE) % NE), ej = (int)(c % NE);
        const double sv = h[c] + s[c];
        const bool outside = mask && mask[c] == PGE_MASK_OUTSIDE;
        if (outside || ei == 0 || ej == 0 || ei == NE - 1 || ej == NE - 1) {
            state[c] = RF_EXCLUDED;
            key[c] = okey(sv);
            continue;
        }
        bool seed = false;
        if (ei >= H && ei < H + N && ej >= H && ej < H + N) {
            seed = sv < 0.0 && sv <= base[c];
            for (int k = 0; k < 8 && !seed; k++) {
                const long long n = owner[((long long)f * NE + ei + kRouteD8[k][0]) * NE + ej + kRouteD8[k][1]];
                if (mask && mask[n] == PGE_MASK_OUTSIDE) {
                    seed = true;
                    break;
                }
                const long long rem = n % ((long long)NE * NE);
                const int nei = (int)(rem / NE), nej = (int)(rem % NE);
                if (nei < H || nei >= H + N || nej < H || nej >= H + N) seed = true;  // no real neighbour (window edge)
            }
        }
        state[c] = seed ? RF_SEED : RF_FREE;
        key[c] = seed ? okey(sv) : RF_UNREACHED;
    }
}

__global__ void route_push_kernel(int F, int NE, const double *__restrict__ h, const double *__restrict__ s, const int32_t *__restrict__ owner,
                                  double eps, unsigned long long *key, const unsigned char *__restrict__ state,
                                  unsigned long long *changed)
{
    const long long total = (long long)F * NE * NE;
    bool any = false;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x) {
        if (state[c] == RF_EXCLUDED) continue;
        const unsigned long long kc = ((volatile unsigned long long *)key)[c];
        if (kc == RF_UNREACHED) continue;
        const double v = unokey(kc) + eps;
        const int f = (int)(c / ((long long)NE * NE));
        const int ei = (int)((c / NE) % NE), ej = (int)(c % NE);
        for (int k = 0; k < 8; k++) {
            const long long n = owner[((long long)f * NE + ei + kRouteD8[k][0]) * NE + ej + kRouteD8[k][1]];
            if (state[n] != RF_FREE) continue;
            const double sn = h[n] + s[n];
            const unsigned long long kn = okey(sn > v ? sn : v);
            if (kn < ((volatile unsigned long long *)key)[n] && atomicMin(key + n, kn) > kn) any = true;
        }
    }
    if (any) *changed = 1ull;
}

__global__ void route_final_kernel(long long total, const double *__restrict__ h, const double *__restrict__ s,
                                   const unsigned long long *__restrict__ key, const unsigned char *__restrict__ state, double *route)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total; c += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = key[c];
        route[c] = (state[c] == RF_EXCLUDED || k == RF_UNREACHED) ? h[c] + s[c] : unokey(k);
    }
}

cudaError_t route_flood(const PgeGrid &g, const PgeState &st, const int32_t *owner, double eps, double *route, const Layout &lay,
                        void *ws, long long max_sweeps, long long *sweeps_out, cudaStream_t s)
{
    const int NE = g.N + 2 * g.H;
    const long long n = lay.ncell;
    unsigned long long *key = ws_ptr<unsigned long long>(ws, lay.cdf);
    unsigned char *state = ws_ptr<unsigned char>(ws, lay.flags);
    unsigned long long *changed = ws_ptr<unsigned long long>(ws, lay.counters) + 8;
    route_init_kernel<<<grid_for(n), 256, 0, s>>>(g.F, NE, g.H, g.N, st.height, st.sediment, st.base, st.mask, owner, key, state);
    unsigned long long host_changed = 1;
    long long sweeps = 0;
    const int batch = 32;  // sweeps between convergence checks (the check synchronises the stream)
    while (host_changed && sweeps < max_sweeps) {
        cudaError_t e = cudaMemsetAsync(changed, 0, 8, s);
        if (e != cudaSuccess) return e;
        for (int k = 0; k < batch; k++)
            route_push_kernel<<<grid_for(n), 256, 0, s>>>(g.F, NE, st.height, st.sediment, owner, eps, key, state, changed);
        sweeps += batch;
        if ((e = cudaMemcpyAsync(&host_changed, changed, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    }
    if (sweeps_out) *sweeps_out = host_changed ? -sweeps : sweeps;
    route_final_kernel<<<grid_for(n), 256, 0, s>>>(n, st.height, st.sediment, key, state, route);
    return cudaPeekAtLastError();
}

// ---------------------------------------------------------------------------
// sea mask: the base level (maps.py:360-420, hydro/run.py:64-83).  Interior
// cells under the waterline (float32 surface < 0) are joined into
// 8-connected components along the owner table (labels: the component's
// lowest cell id, by min-label propagation with pointer jumping); a component
// is open ocean when its area reaches min_area, and the largest always is;
// the others are closed basins, whose cells take the basin's lowest surface.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ long long sea_ext(long long c, int N, int H, int NE)
{
    const long long f = c / ((long long)N * N), rem = c % ((long long)N * N);
    return (f * NE + rem / N + H) * NE + rem % N + H;
}
__device__ __forceinline__ long long sea_nb(const int32_t *owner, long long c, int k, int N, int H, int NE)
{
    const long long f = c / ((long long)N * N), rem = c % ((long long)N * N);
    const long long o = owner[(f * NE + rem / N + H + kRouteD8[k][0]) * NE + rem % N + H + kRouteD8[k][1]];
    const long long f2 = o / ((long long)NE * NE), r2 = o % ((long long)NE * NE);
    return (f2 * N + r2 / NE - H) * N + r2 % NE - H;
}
}  // namespace

__global__ void sea_init_kernel(long long M, int N, int H, int NE, const double *__restrict__ h, const double *__restrict__ s,
                                int32_t *label, double *per, unsigned long long *floorkey)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        const long long e = sea_ext(c, N, H, NE);
        label[c] = (float)(h[e] + s[e]) < 0.0f ? (int32_t)c : -1;
        per[c] = 0.0;
        floorkey[c] = okey(0.0);  // the basin floor starts at 0 (maps.py: np.zeros, then np.minimum.at)
    }
}

__global__ void sea_join_kernel(long long M, int N, int H, int NE, const int32_t *__restrict__ owner, int32_t *label,
                                unsigned long long *changed)
{
    bool any = false;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        const int l = ((volatile int32_t *)label)[c];
        if (l < 0) continue;
        int m = l;
        const int ll = ((volatile int32_t *)label)[l];  // pointer jumping: the label of the label
        if (ll >= 0 && ll < m) m = ll;
        long long nb[8];
        for (int k = 0; k < 8; k++) {
            nb[k] = sea_nb(owner, c, k, N, H, NE);
            const int lq = ((volatile int32_t *)label)[nb[k]];
            if (lq >= 0 && lq < m) m = lq;
        }
        if (m < l && atomicMin(label + c, m) > m) any = true;
        for (int k = 0; k < 8; k++) {
            const int lq = ((volatile int32_t *)label)[nb[k]];
            if (lq > m && atomicMin(label + nb[k], m) > m) any = true;
        }
    }
    if (any) *changed = 1ull;
}

__global__ void sea_stats_kernel(long long M, int N, int H, int NE, const double *__restrict__ h, const double *__restrict__ s,
                                 const float *__restrict__ area, const int32_t *__restrict__ label, double *per,
                                 unsigned long long *floorkey)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        const int l = label[c];
        if (l < 0) continue;
        const long long e = sea_ext(c, N, H, NE);
        atomicAdd(per + l, (double)area[c]);
        atomicMin(floorkey + l, okey(h[e] + s[e]));
    }
}

__global__ void sea_largest_kernel(long long M, const int32_t *__restrict__ label, const double *__restrict__ per,
                                   unsigned long long *maxkey, unsigned long long *largest, int pass)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        if (label[c] != (int32_t)c) continue;  // one root per component
        const unsigned long long k = okey(per[c]);
        if (pass == 0) atomicMax(maxkey, k);
        else if (k == *maxkey) atomicMin(largest, (unsigned long long)c);  // np.argmax: the first (lowest) component
    }
}

__global__ void sea_base_kernel(long long total, int N, int H, int NE, const int32_t *__restrict__ label, const double *__restrict__ per,
                                const unsigned long long *__restrict__ floorkey, const unsigned long long *__restrict__ largest,
                                double min_area, double *base)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long f = e / ((long long)NE * NE), rem = e % ((long long)NE * NE);
        const int ei = (int)(rem / NE), ej = (int)(rem % NE);
        double b = 0.0;
        if (ei >= H && ei < H + N && ej >= H && ej < H + N) {
            const long long c = (f * N + ei - H) * N + ej - H;
            const int l = label[c];
            if (l >= 0 && (unsigned long long)l != *largest && !(per[l] >= min_area)) b = unokey(floorkey[l]);
        }
        base[e] = b;
    }
}

cudaError_t sea_base(const PgeGrid &g, const PgeState &st, const int32_t *owner, const float *area, double min_area, double *base,
                     int32_t *label_out, const Layout &lay, void *ws, long long max_sweeps, long long *sweeps_out, cudaStream_t s)
{
    const int N = g.N, H = g.H, NE = N + 2 * H;
    const long long M = (long long)g.F * N * N;
    int32_t *label = label_out ? label_out : ws_ptr<int32_t>(ws, lay.flags);
    double *per = ws_ptr<double>(ws, lay.cdf);
    unsigned long long *floorkey = reinterpret_cast<unsigned long long *>(per + M);
    unsigned long long *cnt = ws_ptr<unsigned long long>(ws, lay.counters);
    unsigned long long *changed = cnt + 9, *maxkey = cnt + 10, *largest = cnt + 11;
    sea_init_kernel<<<grid_for(M), 256, 0, s>>>(M, N, H, NE, st.height, st.sediment, label, per, floorkey);
    unsigned long long host_changed = 1;
    long long sweeps = 0;
    cudaError_t e;
    while (host_changed && sweeps < max_sweeps) {
        if ((e = cudaMemsetAsync(changed, 0, 8, s)) != cudaSuccess) return e;
        for (int k = 0; k < 16; k++) sea_join_kernel<<<grid_for(M), 256, 0, s>>>(M, N, H, NE, owner, label, changed);
        sweeps += 16;
        if ((e = cudaMemcpyAsync(&host_changed, changed, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    }
    if (sweeps_out) *sweeps_out = host_changed ? -sweeps : sweeps;
    sea_stats_kernel<<<grid_for(M), 256, 0, s>>>(M, N, H, NE, st.height, st.sediment, area, label, per, floorkey);
    if ((e = cudaMemsetAsync(maxkey, 0, 8, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(largest, 0xFF, 8, s)) != cudaSuccess) return e;
    sea_largest_kernel<<<grid_for(M), 256, 0, s>>>(M, label, per, maxkey, largest, 0);
    sea_largest_kernel<<<grid_for(M), 256, 0, s>>>(M, label, per, maxkey, largest, 1);
    sea_base_kernel<<<grid_for(lay.ncell), 256, 0, s>>>(lay.ncell, N, H, NE, label, per, floorkey, largest, min_area, base);
    return cudaPeekAtLastError();
}

// ---------------------------------------------------------------------------
// glacial pass (erosion/glacial.py:162-257; the ice line of the evaporation
// field).  Every per-cell rule runs on the whole extended array, neighbours
// wrapping at each face array's edges as numpy's roll does, so the interior
// comes out as the reference's; the sums are float64 atomics.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ long long glac_nb(long long e, int NE, int k)
{
    const long long f = e / ((long long)NE * NE), rem = e % ((long long)NE * NE);
    int i = (int)(rem / NE) + kRouteD8[k][0], j = (int)(rem % NE) + kRouteD8[k][1];
    i = i < 0 ? i + NE : (i >= NE ? i - NE : i);
    j = j < 0 ? j + NE : (j >= NE ? j - NE : j);
    return (f * NE + i) * NE + j;
}
__device__ __forceinline__ bool glac_interior(long long e, int NE, int H, int N)
{
    const long long rem = e % ((long long)NE * NE);
    const int i = (int)(rem / NE), j = (int)(rem % NE);
    return i >= H && i < H + N && j >= H && j < H + N;
}
struct GlacSums {
    unsigned long long ice_any, ice_interior, margin_any, margin_interior, max_key;
    double carved, wsum, parked;
};
}  // namespace

__global__ void glac_ice_kernel(long long n, int NE, int H, int N, const double *__restrict__ h, const double *__restrict__ s,
                                const float *__restrict__ evap, const uint8_t *__restrict__ mask, const uint8_t *__restrict__ prev,
                                float ice_evap, uint8_t *ice, double *depth, GlacSums *sums)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const bool active = mask ? mask[e] == PGE_MASK_ACTIVE : true;
        const bool cold = evap[e] <= ice_evap;
        bool v = active && cold && (h[e] + s[e] > 0.0);
        if (prev && prev[e] && active && cold) v = true;
        ice[e] = v;
        depth[e] = v ? 1.0 : 0.0;
        if (v) {
            atomicAdd(&sums->ice_any, 1ull);
            if (glac_interior(e, NE, H, N)) atomicAdd(&sums->ice_interior, 1ull);
        }
    }
}

// one ring: a cell stays inside while it and its eight neighbours are
__global__ void glac_ring_kernel(long long n, int NE, const uint8_t *__restrict__ inner, uint8_t *shrunk, double *depth)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        bool v = inner[e];
        for (int k = 0; k < 8 && v; k++) v = inner[glac_nb(e, NE, k)];
        shrunk[e] = v;
        if (v) depth[e] += 1.0;
    }
}

__global__ void glac_dz_kernel(long long n, int NE, int H, int N, const double *__restrict__ h, const double *__restrict__ s,
                               const double *__restrict__ q, const float *__restrict__ hard, const double *__restrict__ base,
                               const uint8_t *__restrict__ ice, const double *__restrict__ depth, int ramp, double rate, double cap,
                               double sat, double dep_floor, double *dz, GlacSums *sums)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double taper = depth[e];
        if (ramp > 0) {
            taper = taper / (double)(ramp + 1);
            taper = taper < 0.0 ? 0.0 : (taper > 1.0 ? 1.0 : taper);
        }
        const double qq = (q[e] > 0.0 ? q[e] : 0.0) / sat;
        const float hf = __fsub_rn(1.0f, __fmul_rn(0.5f, hard[e]));  // float32, as the reference's array arithmetic
        double d = rate * sqrt(qq) * (double)hf * taper;
        d = d < 0.0 ? 0.0 : (d > cap ? cap : d);
        if (!ice[e]) d = 0.0;
        double room = h[e] + s[e] + dep_floor - base[e];
        if (room < 0.0) room = 0.0;
        if (room < d) d = room;
        dz[e] = d;
        if (d != 0.0 && glac_interior(e, NE, H, N)) {
            atomicAdd(&sums->carved, d);
            atomicMax(&sums->max_key, okey(d));
        }
    }
}

__global__ void glac_carve_kernel(long long n, double *h, const double *__restrict__ dz)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        h[e] -= dz[e];
}

__global__ void glac_margin_kernel(long long n, int NE, int H, int N, const double *__restrict__ h, const double *__restrict__ s,
                                   const double *__restrict__ q, const double *__restrict__ base, const uint8_t *__restrict__ mask,
                                   const uint8_t *__restrict__ ice, double *w, GlacSums *sums)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        bool near = false;
        for (int k = 0; k < 8 && !near; k++) near = ice[glac_nb(e, NE, k)];
        const bool active = mask ? mask[e] == PGE_MASK_ACTIVE : true;
        const bool margin = near && !ice[e] && active && (h[e] + s[e] > base[e]);
        w[e] = margin ? (q[e] > 0.0 ? q[e] : 0.0) + 1e-6 : 0.0;
        if (margin) {
            atomicAdd(&sums->margin_any, 1ull);
            if (glac_interior(e, NE, H, N)) {
                atomicAdd(&sums->margin_interior, 1ull);
                atomicAdd(&sums->wsum, w[e]);
            }
        }
    }
}

__global__ void glac_moraine_kernel(long long n, int NE, int H, int N, const double *__restrict__ w, double wsum, double load, double cap,
                                    double *s, double *pending, GlacSums *sums)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double add = (w[e] / wsum) * load;
        const double placed = add < cap ? add : cap;
        s[e] += placed;
        pending[e] += add - placed;
        const double parked = add - placed;
        if (parked != 0.0 && glac_interior(e, NE, H, N)) atomicAdd(&sums->parked, parked);
    }
}

int glacial(const PgeGrid &g, PgeState &st, uint8_t *ice_prev, const GlacialArgs &ga, double stats[5], const Layout &lay, void *ws,
            cudaStream_t s)
{
    const int N = g.N, H = g.H, NE = N + 2 * H;
    const long long n = lay.ncell;
    stats[0] = stats[1] = stats[2] = stats[3] = stats[4] = 0.0;
    if (ga.rate <= 0.0) return 0;
    uint8_t *ice = ws_ptr<uint8_t>(ws, lay.flags), *ping = ice + n, *pong = ice + 2 * n;
    double *depth = ws_ptr<double>(ws, lay.thermal), *dz = depth + n, *w = depth + 2 * n;
    GlacSums *sums = reinterpret_cast<GlacSums *>(ws_ptr<unsigned long long>(ws, lay.counters) + 12);
    GlacSums hs;
    cudaError_t e;
    auto read = [&]() -> cudaError_t {
        cudaError_t r = cudaMemcpyAsync(&hs, sums, sizeof(GlacSums), cudaMemcpyDeviceToHost, s);
        return r == cudaSuccess ? cudaStreamSynchronize(s) : r;
    };
    if ((e = cudaMemsetAsync(sums, 0, sizeof(GlacSums), s)) != cudaSuccess) return -(int)e;
    glac_ice_kernel<<<grid_for(n), 256, 0, s>>>(n, NE, H, N, st.height, st.sediment, st.evap, st.mask, ice_prev, ga.ice_evap, ice,
                                                depth, sums);
    if ((e = read()) != cudaSuccess) return -(int)e;
    if (!hs.ice_any) return 0;  // no ice: nothing changes (and the last ice stays as it was)
    if (ice_prev && (e = cudaMemcpyAsync(ice_prev, ice, n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return -(int)e;
    if (ga.ramp > 0) {
        const uint8_t *inner = ice;
        for (int r = 0; r < ga.ramp; r++) {
            uint8_t *out = (r & 1) ? pong : ping;
            glac_ring_kernel<<<grid_for(n), 256, 0, s>>>(n, NE, inner, out, depth);
            inner = out;
        }
    }
    glac_dz_kernel<<<grid_for(n), 256, 0, s>>>(n, NE, H, N, st.height, st.sediment, st.discharge, st.hardness, st.base, ice, depth,
                                               ga.ramp, ga.rate, ga.cap, ga.sat, ga.dep_floor, dz, sums);
    if ((e = read()) != cudaSuccess) return -(int)e;
    if (!(hs.carved > 0.0)) return 0;  // nothing carved: the reference returns before any change (and empty statistics)
    glac_carve_kernel<<<grid_for(n), 256, 0, s>>>(n, st.height, dz);
    glac_margin_kernel<<<grid_for(n), 256, 0, s>>>(n, NE, H, N, st.height, st.sediment, st.discharge, st.base, st.mask, ice, w, sums);
    if ((e = read()) != cudaSuccess) return -(int)e;
    if (hs.margin_any && ga.moraine_frac > 0.0 && hs.wsum > 0.0) {
        glac_moraine_kernel<<<grid_for(n), 256, 0, s>>>(n, NE, H, N, w, hs.wsum, hs.carved * ga.moraine_frac, ga.iter_deposit,
                                                        st.sediment, st.pending, sums);
        if ((e = read()) != cudaSuccess) return -(int)e;
    }
    stats[0] = (double)hs.ice_interior;
    stats[1] = hs.carved;
    stats[2] = (double)hs.margin_interior;
    {  // the order-preserving key back to its double (host side of unokey)
        const unsigned long long k = hs.max_key;
        const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
        double v;
        memcpy(&v, &b, sizeof v);
        stats[3] = v;
    }
    stats[4] = hs.parked;
    return 0;
}

cudaError_t window_lakes(const PgeGrid &g, const PgeState &st, double min_depth, uint8_t *flag, int64_t *count, cudaStream_t stream)
{
    const long long NE = g.N + 2LL * g.H, n = (long long)g.F * NE * NE;
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(count);
    if (cnt) {
        const cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return e;
    }
    window_lakes_kernel<<<grid_for(n), 256, 0, stream>>>(n, g.N, g.H, st.height, st.sediment, st.route, st.mask, min_depth, flag, cnt);
    return cudaGetLastError();
}

}  // namespace pge

