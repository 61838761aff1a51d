// pge_droplets.cuh -- the persistent droplet kernel (trace + per-droplet ledger).
//
// Included by pge_droplets_f64.cu (PGE_REAL = double, compiled without FMA
// contraction: rounds like the reference's float64 numba code) and
// pge_droplets_f32.cu (PGE_REAL = float, the fast trace).
//
// One droplet per thread, persistent: a thread that finishes a droplet takes
// the next index of the wave from a warp-aggregated atomic counter, and the
// loop body advances every live droplet of the warp by exactly one step, so
// lanes stay converged however uneven the lifetimes are.
//
// A step is the body of the reference's trace loop
// (bake/globe/erosion/particle.py:421-769): bilinear value and gradient of
// the frozen surface, contravariant gradient through the inverse metric,
// gravity, inertia, stream-momentum push, unit-length step with on-device
// face crossing (cubesphere.transfer_velocity, cubesphere.py:204-220), the
// land (capacity law, cover / hardness blend, concurrency caps) or seafloor
// (deposit-only fan) mass transfer, evaporation and the stop rules, then the
// final deposits over the last SPREAD cells (particle.py:770-815).
//
// The reference applies each particle's change list serially against the
// live terrain (apply_changes, particle.py:821-1042).  Here each droplet
// applies its own entries in list order, one entry behind the trace (the
// erosion floor needs the next entry's cell), against the wave-start terrain
// plus its own earlier changes -- exactly the reference's result for a
// droplet that shares no cell with another of its wave.  The droplet's own
// per-cell changes live in a per-thread table in global scratch (one column
// per thread slot, so a warp's accesses coalesce) behind a 256-bit Bloom
// filter in registers; terrain change, tracks and stockpiles go out as
// int64 fixed-point atomics.
#pragma once
#include <cstdint>

#include "pge_crmath.cuh"
#include "pge_internal.cuh"

#if !defined(PGE_REAL) || !defined(PGE_VARIANT)
#error "define PGE_REAL (double or float) and PGE_VARIANT before including pge_droplets.cuh"
#endif

namespace pge {
namespace PGE_VARIANT {

typedef PGE_REAL R;

__constant__ double kBases[6][3][3] = {
    {{0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}, {1.0, 0.0, 0.0}},
    {{0.0, 0.0, 1.0}, {0.0, -1.0, 0.0}, {-1.0, 0.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, 1.0}, {0.0, 1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, 1.0}},
    {{-1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, -1.0}},
};

namespace {

constexpr double kPi = 3.14159265358979323846;
__device__ __forceinline__ R half_pi() { return R(kPi / 2.0); }
__device__ __forceinline__ R two_over_pi() { return R(2.0 / kPi); }

// tan / atan / sin / cos of the droplet precision.  CR (float64 only): correctly rounded double-double
// evaluations (pge_crmath.cuh), which give the C library's results the reference computes with
// wherever those are correctly rounded -- the exact (ordered) pass and the change-list hook use them;
// otherwise CUDA's own functions, for the order-free wave apply, whose results are not the
// reference's anyway.  They run inside the out-of-line face crossing and spawn direction below, so
// the droplet kernel itself holds one call site for each.
template <bool CR> __device__ __forceinline__ double m_tan(double x) { return CR ? cr::cr_tan(x) : tan(x); }
template <bool CR> __device__ __forceinline__ double m_atan(double x) { return CR ? cr::cr_atan(x) : atan(x); }
template <bool CR> __device__ __forceinline__ double m_sin(double x) { return CR ? cr::cr_sin(x) : sin(x); }
template <bool CR> __device__ __forceinline__ double m_cos(double x) { return CR ? cr::cr_cos(x) : cos(x); }
template <bool CR> __device__ __forceinline__ float m_tan(float x) { return tanf(x); }
template <bool CR> __device__ __forceinline__ float m_atan(float x) { return atanf(x); }
template <bool CR> __device__ __forceinline__ float m_sin(float x) { return sinf(x); }
template <bool CR> __device__ __forceinline__ float m_cos(float x) { return cosf(x); }

// ---------------------------------------------------------------------------
// cube-sphere mapping in droplet precision (cubesphere.py:70-220)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void face_axes(int f, R r[3], R u[3], R n[3])
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        r[k] = R(kBases[f][0][k]);
        u[k] = R(kBases[f][1][k]);
        n[k] = R(kBases[f][2][k]);
    }
}

template <bool CR = true>
__device__ void to_sphere(int face, R u, R v, R &x, R &y, R &z)
{
    R r[3], up[3], n[3];
    face_axes(face, r, up, n);
    R s = m_tan<CR>((u - R(0.5)) * half_pi());
    R t = m_tan<CR>((v - R(0.5)) * half_pi());
    R qx = n[0] + s * r[0] + t * up[0];
    R qy = n[1] + s * r[1] + t * up[1];
    R qz = n[2] + s * r[2] + t * up[2];
    R inv = R(1) / sqrt(qx * qx + qy * qy + qz * qz);
    x = qx * inv;
    y = qy * inv;
    z = qz * inv;
}

template <bool CR = true>
__device__ int from_sphere(R x, R y, R z, R &u, R &v)
{
    R ax = fabs(x), ay = fabs(y), az = fabs(z);
    int face;
    if (ax >= ay && ax >= az) face = x >= R(0) ? 0 : 1;
    else if (ay >= az) face = y >= R(0) ? 2 : 3;
    else face = z >= R(0) ? 4 : 5;
    R r[3], up[3], n[3];
    face_axes(face, r, up, n);
    R d = x * n[0] + y * n[1] + z * n[2];
    R s = (x * r[0] + y * r[1] + z * r[2]) / d;
    R t = (x * up[0] + y * up[1] + z * up[2]) / d;
    u = m_atan<CR>(s) * two_over_pi() + R(0.5);
    v = m_atan<CR>(t) * two_over_pi() + R(0.5);
    return face;
}

template <bool CR = true>
__device__ void jacobian(int face, R u, R v, R J[6])
{
    R r[3], up[3], n[3];
    face_axes(face, r, up, n);
    R s = m_tan<CR>((u - R(0.5)) * half_pi()), t = m_tan<CR>((v - R(0.5)) * half_pi());
    R dsdu = half_pi() * (R(1) + s * s);
    R dtdv = half_pi() * (R(1) + t * t);
    R qx = n[0] + s * r[0] + t * up[0];
    R qy = n[1] + s * r[1] + t * up[1];
    R qz = n[2] + s * r[2] + t * up[2];
    R ql = sqrt(qx * qx + qy * qy + qz * qz);
    R px = qx / ql, py = qy / ql, pz = qz / ql;
    R dux = r[0] * dsdu, duy = r[1] * dsdu, duz = r[2] * dsdu;
    R pd = px * dux + py * duy + pz * duz;
    J[0] = (dux - px * pd) / ql;
    J[1] = (duy - py * pd) / ql;
    J[2] = (duz - pz * pd) / ql;
    R dvx = up[0] * dtdv, dvy = up[1] * dtdv, dvz = up[2] * dtdv;
    pd = px * dvx + py * dvy + pz * dvz;
    J[3] = (dvx - px * pd) / ql;
    J[4] = (dvy - py * pd) / ql;
    J[5] = (dvz - pz * pd) / ql;
}

// particle face transition; returns the new face, (u, v, a, b) updated in place
template <bool CR = true>
__device__ int transfer_velocity(int face, R &u, R &v, R &a, R &b)
{
    if (u >= R(0) && u < R(1) && v >= R(0) && v < R(1)) return face;
    R x, y, z, u2, v2;
    to_sphere<CR>(face, u, v, x, y, z);
    int f2 = from_sphere<CR>(x, y, z, u2, v2);
    if (f2 == face) {
        R m = u2 < R(0) ? R(0) : u2;
        u = R(0.999999999) < m ? R(0.999999999) : m;
        m = v2 < R(0) ? R(0) : v2;
        v = R(0.999999999) < m ? R(0.999999999) : m;
        return face;
    }
    R J[6], K[6];
    jacobian<CR>(face, u, v, J);
    R wx = a * J[0] + b * J[3];
    R wy = a * J[1] + b * J[4];
    R wz = a * J[2] + b * J[5];
    jacobian<CR>(f2, u2, v2, K);
    R guu = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
    R guv = K[0] * K[3] + K[1] * K[4] + K[2] * K[5];
    R gvv = K[3] * K[3] + K[4] * K[4] + K[5] * K[5];
    R ru = K[0] * wx + K[1] * wy + K[2] * wz;
    R rv = K[3] * wx + K[4] * wy + K[5] * wz;
    R det = guu * gvv - guv * guv;
    a = (gvv * ru - guv * rv) / det;
    b = (guu * rv - guv * ru) / det;
    u = u2;
    v = v2;
    return f2;
}

// the crossing and the direction of a loaded spawn, out of line: the droplet kernel runs them rarely and
// their double-double arithmetic stays out of its register allocation
struct Crossed {
    R u, v, a, b;
    int face;
};
template <bool CR>
__device__ __noinline__ Crossed cross_out_of_line(int face, R u, R v, R a, R b)
{
    Crossed c{u, v, a, b, face};
    c.face = transfer_velocity<CR>(face, c.u, c.v, c.a, c.b);
    return c;
}
__device__ __forceinline__ int cross_face(bool cr, int face, R &u, R &v, R &a, R &b)
{
    const Crossed c = cr ? cross_out_of_line<true>(face, u, v, a, b) : cross_out_of_line<false>(face, u, v, a, b);
    u = c.u;
    v = c.v;
    a = c.a;
    b = c.b;
    return c.face;
}
struct Dir {
    R c, s;
};
template <bool CR>
__device__ __noinline__ Dir spawn_dir(R dir) { return Dir{m_cos<CR>(dir), m_sin<CR>(dir)}; }

// ---------------------------------------------------------------------------
// what a step reads about the cell a droplet stands in
// ---------------------------------------------------------------------------
struct View {
    long long cell;       // flat (f, ei, ej)
    int m;                // mask code
    float surf;           // the cell's own packed surface
    float evap, hard, sed, base;
    float g0, g1, g2, q0, q1, q2;
    double hs, accws;     // float64 terrain: height + sediment, wave-start net change
    float4 s00, s10, s01, s11;  // bilinear stencil around the droplet position
    R wi, wj;
};

__device__ __forceinline__ void load_view(const DropArgs &a, int f, R x, R y, int ei, int ej, View &v)
{
    const int NE = a.NE;
    R fi = x - R(0.5) + R(a.H), fj = y - R(0.5) + R(a.H);
    int i0 = (int)floor(fi), j0 = (int)floor(fj);
    if (i0 < 0) i0 = 0;
    if (i0 > NE - 2) i0 = NE - 2;
    if (j0 < 0) j0 = 0;
    if (j0 > NE - 2) j0 = NE - 2;
    R wi = fi - R(i0), wj = fj - R(j0);
    if (wi < R(0)) wi = R(0);
    if (wi > R(1)) wi = R(1);
    if (wj < R(0)) wj = R(0);
    if (wj > R(1)) wj = R(1);
    const long long fb = (long long)f * NE;
    const long long c00 = (fb + i0) * NE + j0;
    v.s00 = __ldg(a.A + c00);
    v.s01 = __ldg(a.A + c00 + 1);
    v.s10 = __ldg(a.A + c00 + NE);
    v.s11 = __ldg(a.A + c00 + NE + 1);
    v.wi = wi;
    v.wj = wj;
    const long long cc = (fb + ei) * NE + ej;
    v.cell = cc;
    const float4 b = __ldg(a.B + cc);
    v.evap = b.x;
    v.hard = b.y;
    v.sed = b.z;
    v.base = b.w;
    const long long mc = a.metric_shared ? (long long)ei * NE + ej : cc;
    const float4 g0 = __ldg(a.G + 2 * mc), g1 = __ldg(a.G + 2 * mc + 1);
    v.g0 = g0.x;
    v.g1 = g0.y;
    v.g2 = g0.z;
    v.q0 = g0.w;
    v.q1 = g1.x;
    v.q2 = g1.y;
    const double2 l = __ldg(a.L + cc);
    v.hs = l.x;
    v.accws = l.y;
    v.m = a.mask ? (int)__ldg(a.mask + cc) : PGE_MASK_ACTIVE;
    const int di = ei - i0, dj = ej - j0;
    if ((unsigned)di <= 1u && (unsigned)dj <= 1u)
        v.surf = di ? (dj ? v.s11.x : v.s10.x) : (dj ? v.s01.x : v.s00.x);
    else
        v.surf = __ldg(&a.A[cc].x);
}

// bilinear of one channel (c = 0..3) of the stencil
__device__ __forceinline__ R bilin(const View &v, int c)
{
    float h00, h10, h01, h11;
    if (c == 0) { h00 = v.s00.x; h10 = v.s10.x; h01 = v.s01.x; h11 = v.s11.x; }
    else if (c == 1) { h00 = v.s00.y; h10 = v.s10.y; h01 = v.s01.y; h11 = v.s11.y; }
    else if (c == 2) { h00 = v.s00.z; h10 = v.s10.z; h01 = v.s01.z; h11 = v.s11.z; }
    else { h00 = v.s00.w; h10 = v.s10.w; h01 = v.s01.w; h11 = v.s11.w; }
    const R wi = v.wi, wj = v.wj;
    return R(h00) * (R(1) - wi) * (R(1) - wj) + R(h10) * wi * (R(1) - wj) + R(h01) * (R(1) - wi) * wj + R(h11) * wi * wj;
}

// The routing surface's bilinear sample (and gradient) at (face, x, y), when
// any of the stencil's four cells carries the route flag (particle.py:228-233,
// 196-225); false: the route equals the terrain there and is not sampled.
__device__ __forceinline__ bool route_sample(const DropArgs &a, int f, R x, R y, bool grad, R &val, R &gi, R &gj)
{
    const int NE = a.NE;
    R fi = x - R(0.5) + R(a.H), fj = y - R(0.5) + R(a.H);
    int i0 = (int)floor(fi), j0 = (int)floor(fj);
    if (i0 < 0) i0 = 0;
    if (i0 > NE - 2) i0 = NE - 2;
    if (j0 < 0) j0 = 0;
    if (j0 > NE - 2) j0 = NE - 2;
    R wi = fi - R(i0), wj = fj - R(j0);
    if (wi < R(0)) wi = R(0);
    if (wi > R(1)) wi = R(1);
    if (wj < R(0)) wj = R(0);
    if (wj > R(1)) wj = R(1);
    const long long c00 = ((long long)f * NE + i0) * NE + j0;
    const float2 r00 = __ldg(a.R + c00), r01 = __ldg(a.R + c00 + 1), r10 = __ldg(a.R + c00 + NE), r11 = __ldg(a.R + c00 + NE + 1);
    float flag = r00.y + r10.y;
    flag = flag + r01.y;
    flag = flag + r11.y;
    if (flag == 0.0f) return false;
    val = R(r00.x) * (R(1) - wi) * (R(1) - wj) + R(r10.x) * wi * (R(1) - wj) + R(r01.x) * (R(1) - wi) * wj + R(r11.x) * wi * wj;
    if (grad) {
        const float d10 = r10.x - r00.x, d11 = r11.x - r01.x, d01 = r01.x - r00.x, d1110 = r11.x - r10.x;
        gi = R(d10) * (R(1) - wj) + R(d11) * wj;
        gj = R(d01) * (R(1) - wi) + R(d1110) * wi;
    }
    return true;
}

__device__ __forceinline__ R snorm(const View &v, R a, R b)
{
    R n2 = R(v.g0) * a * a + R(2) * R(v.g1) * a * b + R(v.g2) * b * b;
    if (n2 < R(0)) n2 = R(0);
    return sqrt(n2);
}

__device__ __forceinline__ R sdot(const View &v, R a, R b, R c, R d)
{
    return R(v.g0) * a * c + R(v.g1) * (a * d + b * c) + R(v.g2) * b * d;
}

__device__ __forceinline__ int cell_of(R x, int N)
{
    int i = (int)floor(x);
    if (i < 0) i = 0;
    if (i > N - 1) i = N - 1;
    return i;
}

// ---------------------------------------------------------------------------
// the droplet's own-change table: an open-addressing hash (linear probing)
// of `size` slots, private to the thread slot, in global scratch.  A key is
// (generation << 32 | cell); slots of any other generation are free, so a
// new droplet starts with an empty table without clearing it.  A 256-bit
// Bloom filter in registers answers "never changed" without a probe.
// ---------------------------------------------------------------------------
struct Table {
    unsigned long long *key;
    double *own;
    unsigned mask;  // size - 1
    unsigned long long gen;
    int cap, n;
    unsigned long long b0, b1, b2, b3;
    bool overflow;

    __device__ __forceinline__ void reset(unsigned long long g)
    {
        gen = g;
        n = 0;
        b0 = b1 = b2 = b3 = 0ull;
        overflow = false;
    }
    __device__ __forceinline__ static unsigned hash(long long c)
    {
        return (unsigned)(((unsigned long long)c * 0x9E3779B97F4A7C15ull) >> 32);
    }
    __device__ __forceinline__ bool maybe(long long c) const
    {
        const int b = (int)(hash(c) >> 24);
        const unsigned long long w = (b >> 6) == 0 ? b0 : (b >> 6) == 1 ? b1 : (b >> 6) == 2 ? b2 : b3;
        return (w >> (b & 63)) & 1ull;
    }
    // own change of cell c and its slot (-1: none)
    __device__ __forceinline__ double lookup(long long c, int &idx) const
    {
        idx = -1;
        if (!maybe(c)) return 0.0;
        const unsigned long long want = (gen << 32) | (unsigned)c;
        unsigned s = hash(c) & mask;
        for (unsigned i = 0; i <= mask; i++, s = (s + 1) & mask) {
            const unsigned long long k = key[s];
            if (k == want) {
                idx = (int)s;
                return own[s];
            }
            if ((k >> 32) != gen) break;  // a free slot ends the probe run
        }
        return 0.0;
    }
    __device__ __forceinline__ void store(long long c, int &idx, double value)
    {
        if (idx >= 0) {
            own[idx] = value;
            return;
        }
        if (n >= cap) {
            overflow = true;
            return;
        }
        unsigned s = hash(c) & mask;
        for (unsigned i = 0; i <= mask; i++, s = (s + 1) & mask)
            if ((key[s] >> 32) != gen) break;
        key[s] = (gen << 32) | (unsigned)c;
        own[s] = value;
        idx = (int)s;
        n++;
        const int b = (int)(hash(c) >> 24);
        const unsigned long long m = 1ull << (b & 63);
        switch (b >> 6) {
        case 0: b0 |= m; break;
        case 1: b1 |= m; break;
        case 2: b2 |= m; break;
        default: b3 |= m; break;
        }
    }
};

// one cell of the ledger: float64 terrain as the droplet sees it
struct LCell {
    long long cell;
    int m;
    float base;
    double hs, accws, own;
    int tidx;
    __device__ __forceinline__ double acc() const { return accws + own; }
    __device__ __forceinline__ double live() const { return hs + (accws + own); }
};

struct Entry {
    long long cell;
    double delta;
    float vol, ma, mb;
    int sidx;  // the step that made it (-1: a final deposit); the tape only
};

struct Ledger {
    double deficit, surplus;
    bool has_prev;
    double prev_live;
    long long death;
    long long prev_cell;  // cell of the last step entry (the tape's reference cell)
    int tap_n;            // entries taped
    int clamped;
    long long eroded_fx, deposited_fx;  // this thread's applied totals
};

__device__ __forceinline__ void load_lcell(const DropArgs &a, const Table &t, long long c, LCell &lc)
{
    lc.cell = c;
    const double2 l = __ldg(a.L + c);
    lc.hs = l.x;
    lc.accws = l.y;
    lc.base = __ldg(&a.B[c].w);
    lc.m = a.mask ? (int)__ldg(a.mask + c) : PGE_MASK_ACTIVE;
    lc.own = t.lookup(c, lc.tidx);
}

// Apply one change-list entry (particle.py:934-1018) at cell `c` against the
// droplet's view of the terrain.  `nx` is the next entry's cell (has_next).
// Updates c.own (and the table), emits the atomics and returns the applied
// change (0 when nothing moved).
template <bool TAPE>
__device__ __forceinline__ void tape_entry(const DropArgs &a, Ledger &L, long long row, const Entry &e, long long ref, int code)
{
    if (!TAPE) return;
    if (L.tap_n < a.tape.entries) {
        int4 *te = reinterpret_cast<int4 *>(a.tape.entry) + row * a.tape.entries + L.tap_n;
        *te = make_int4((int)e.cell, (int)ref, code, e.sidx);
    }
    L.tap_n++;
}

template <bool TAPE = false, bool ROUTE = false>
__device__ __forceinline__ void apply_entry(const DropArgs &a, Table &t, Ledger &L, const Entry &e, LCell &c, bool has_next,
                                            const LCell &nx, long long row = 0)
{
    const PgeParams &p = a.p;
    const double d = e.delta;
    const float v = e.vol;
    const bool is_step = v >= 0.0f;
    const int kind = (d < 0.0 ? 0 : PGE_TE_DEPOSIT) | (is_step ? PGE_TE_STEP : 0);
    if (c.m != PGE_MASK_ACTIVE) {
        tape_entry<TAPE>(a, L, row, e, -1, kind | PGE_TE_SKIP);
        return;
    }
    const double a0 = c.acc();
    const double s_c = c.hs + a0;
    const float b_c = c.base;
    double applied = 0.0;
    if (d < 0.0) {
        const double ew = -d;
        double e_act = ew;
        double room = p.iter_erode + a0;
        if (a.ecap) {
            const double r2 = __ldg(a.ecap + c.cell) + a0;
            if (r2 < room) room = r2;
        }
        int src = 0, fsrc = s_c >= (double)b_c ? 2 : 3;
        if (e_act > room) {
            e_act = room;
            src = 1;
        }
        double floor_ = s_c >= (double)b_c ? (double)b_c : s_c;
        if (ROUTE && a.lakes) {
            // a lake bed is never eroded below its water level (particle.py:952-956)
            const float2 rc = __ldg(a.R + c.cell);
            if (rc.y >= 1.5f && (double)rc.x > floor_) floor_ = (double)rc.x;
        }
        if (has_next) {
            const double ns = nx.live();
            if (ns > floor_) {
                floor_ = ns;
                fsrc = 4;
            }
        }
        if (e_act > s_c - floor_) {
            e_act = s_c - floor_;
            src = fsrc;
        }
        if (e_act < 0.0) {
            e_act = 0.0;
            src = 5;
        }
        if (e_act < ew) {
            L.clamped++;
            L.deficit += ew - e_act;
        }
        applied = -e_act;
        tape_entry<TAPE>(a, L, row, e, src == 4 ? nx.cell : -1, kind | (src << PGE_TE_SRC_SHIFT));
    } else {
        double want = d + L.surplus;
        L.surplus = 0.0;
        int take_code = 0;
        if (L.deficit > 0.0) {
            take_code = want < L.deficit ? 1 : 2;
            const double take = want < L.deficit ? want : L.deficit;
            want -= take;
            L.deficit -= take;
        }
        double d_act = want;
        int src = 0;
        const double room = p.iter_deposit - a0;
        if (d_act > room) {
            d_act = room;
            src = 1;
        }
        bool has_ref = false;
        double ref_live = 0.0;
        long long ref_cell = -1;
        if (is_step) {
            has_ref = L.has_prev;
            ref_live = L.prev_live;
            ref_cell = L.prev_cell;
        } else if (has_next) {
            has_ref = true;
            ref_live = nx.live();
            ref_cell = nx.cell;
        }
        if (has_ref) {
            double ceil_ = ref_live + p.dep_floor;
            if (s_c < (double)b_c && is_step) ceil_ -= p.dep_floor + p.fan_slope;
            const double lim = ceil_ - s_c;
            if (d_act > lim) {
                d_act = lim;
                src = 2;
            }
        }
        if (s_c < (double)b_c) {
            const double lim = (double)b_c - p.dep_floor - s_c;
            if (d_act > lim) {
                d_act = lim;
                src = 3;
            }
        }
        if (d_act < 0.0) {
            d_act = 0.0;
            src = 4;
        }
        if (d_act < want) L.clamped++;
        L.surplus = want - d_act;
        applied = d_act;
        tape_entry<TAPE>(a, L, row, e, src == 2 ? ref_cell : -1,
                         kind | (src << PGE_TE_SRC_SHIFT) | (take_code << PGE_TE_TAKE_SHIFT));
        if (!is_step && L.death < 0) L.death = c.cell;
    }
    if (applied != 0.0) {
        // the reference updates acc[c] in place: acc - e_act / acc + d_act
        c.own = c.own + applied;
        t.store(c.cell, c.tidx, c.own);
        const long long fx = fx_mass(applied);
        red_add(a.acc4 + 4 * c.cell, fx);
        if (fx < 0) L.eroded_fx -= fx;
        else L.deposited_fx += fx;
    }
    if (is_step) {
        if (v > 0.0f) {
            red_add(a.acc4 + 4 * c.cell + 1, fx_track((double)v));
            red_add(a.acc4 + 4 * c.cell + 2, fx_track((double)e.ma));
            red_add(a.acc4 + 4 * c.cell + 3, fx_track((double)e.mb));
        }
        L.has_prev = true;
        L.prev_live = c.live();
        L.prev_cell = c.cell;
    }
}

__device__ __forceinline__ int step_entries(int entries, int finals) { return entries - finals; }

__device__ __forceinline__ void sync_own(LCell &x, const LCell &changed)
{
    if (x.cell == changed.cell) {
        x.own = changed.own;
        x.tidx = changed.tidx;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
enum { ST_DROP, ST_STEPS, ST_ENTRIES, ST_CLAMPED, ST_OVER, ST_TOPEND, ST_DEFICIT, ST_LOSTOFF, ST_ERODED, ST_DEPOSITED,
       ST_DEATH0, ST_N = ST_DEATH0 + PGE_N_DEATHS };

// TAPE (with LEDGER): also record the adjoint's tape (a.tape, row = the droplet's index in the pass)
// ROUTE: steer on the routing surface a.R where it stands above the terrain
// LATERAL: cut the bank on the outside of the bend (erosion.lateral_rate > 0)
template <int MINB, bool LEDGER, bool TAPE = false, bool ROUTE = false, bool LATERAL = false>
__global__ void __launch_bounds__(256, MINB) droplet_kernel(const DropArgs a)
{
    const PgeParams &p = a.p;
    const int lane = threadIdx.x & 31;
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ unsigned long long sstat[ST_N];
    for (int k = threadIdx.x; k < ST_N; k += blockDim.x) sstat[k] = 0ull;
    __syncthreads();
    if (slot == 0 && a.counter_next) *a.counter_next = 0ull;
    const int N = a.N, H = a.H, NE = a.NE;
    const R Nf = R(N);
    const R volume0 = R(a.volume0);
    const R inv_sat = p.disc_saturation > 0.0 ? R(1.0 / p.disc_saturation) : R(0);
    const R k_dt = R(p.dt), k_friction = R(p.friction), k_density = R(p.density), k_kmom = R(p.k_mom),
            k_momscale = R(p.mom_scale), k_slope_gain = R(p.slope_gain), k_slope_sat = R(p.slope_sat),
            k_erod = R(p.erodibility), k_kdisc = R(p.k_disc), k_depr = R(p.deposition_rate), k_cover = R(p.cover_depth),
            k_maxe = R(p.max_erode), k_conc = R(p.conc_scale), k_ocean = R(p.ocean_rate), k_fanroom = R(p.fan_room),
            k_depfloor = R(p.dep_floor), k_evap = R(p.evap_rate), k_minvol = R(p.min_volume), k_dexp = R(p.disc_exponent);

    Table t;
    t.key = a.tkey + slot * (long long)(a.table_mask + 1);
    t.own = a.town + slot * (long long)(a.table_mask + 1);
    t.mask = a.table_mask;
    t.cap = a.table_cap;
    unsigned long long gen = a.gen_base;
    t.reset(gen);

    // droplet registers
    bool alive = false, done = lane >= a.lanes;  // lanes past a.lanes take no droplet
    long long d = 0;
    int f = 0, step = 0, uphill = 0, sea_steps = 0, nring = 0;
    R x = R(0), y = R(0), sa = R(0), sb = R(0), vol = R(0), sed = R(0);
    bool in_sea = false, has_hprev = false;
    bool in_lake = false;  // on an overflowing lake: crossing, no exchange with the bed (particle.py:417)
    float h_prev = 0.0f;
    int r0 = -1, r1 = -1, r2 = -1, r3 = -1, r4 = -1, r5 = -1, r6 = -1, r7 = -1;  // ring, newest first
    View cv;
    LCell cur, pend, nxt;
    Entry pe;
    bool has_pe = false;
    Ledger L;
    int rec_n = 0;
    int nbank = 0;  // bank entries (volume -2) and lake parks (volume -3) of this droplet: entries, not steps
    int parks = 0;  // loads this droplet has left in lakes (at most LAKE_PARKS, particle.py:418)

    while (true) {
        // ---- refill: lanes without a droplet take the next indices of the wave
        const unsigned need = __ballot_sync(0xffffffffu, !alive && !done);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(a.counter, (unsigned long long)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!alive && !done) {
                const long long di = a.d_begin + (long long)base + __popc(need & ((1u << lane) - 1u));
                if (di >= a.d_end) {
                    done = true;
                } else {
                    d = di;
                    alive = true;
                    f = a.sp_face[d];
                    x = R(a.sp_x[d]);
                    y = R(a.sp_y[d]);
                    sed = R(a.sp_sed[d]);
                    vol = volume0;
                    sa = R(0);
                    sb = R(0);
                    if (sed > R(0)) {
                        const R dir = R(a.sp_dir[d]);
                        const Dir dd = a.cr_trig ? spawn_dir<true>(dir) : spawn_dir<false>(dir);
                        sa = dd.c;
                        sb = dd.s;
                    }
                    step = uphill = sea_steps = nring = 0;
                    in_sea = has_hprev = in_lake = false;
                    r0 = r1 = r2 = r3 = r4 = r5 = r6 = r7 = -1;
                    has_pe = false;
                    L.deficit = L.surplus = 0.0;
                    L.has_prev = false;
                    L.prev_live = 0.0;
                    L.death = -1;
                    L.prev_cell = -1;
                    L.tap_n = 0;
                    L.clamped = 0;
                    L.eroded_fx = L.deposited_fx = 0;
                    t.reset(++gen);
                    rec_n = 0;
                    nbank = 0;
                    parks = 0;
                    const int ei = cell_of(x, N) + H, ej = cell_of(y, N) + H;
                    load_view(a, f, x, y, ei, ej, cv);
                    cur.cell = cv.cell;
                    cur.m = cv.m;
                    cur.base = cv.base;
                    cur.hs = cv.hs;
                    cur.accws = cv.accws;
                    cur.own = 0.0;
                    cur.tidx = -1;
                }
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        if (!alive) continue;

        // ---- one step of the trace (particle.py:421-769)
        int tb = 0;  // the tape's branch bits of this step
        const long long trow = d;  // the tape's row: the droplet's index in the pass
        if (TAPE) {
            double *ts = a.tape.state + (trow * (a.tape.steps + 1) + step) * 6;
            ts[0] = (double)x;
            ts[1] = (double)y;
            ts[2] = (double)sa;
            ts[3] = (double)sb;
            ts[4] = (double)sed;
            ts[5] = (double)vol;
            tb = f;
        }
        int cause = -1;
        bool exited = false;
        bool have_entry = false;
        bool have_bank = false;
        Entry bank_en;
        [[maybe_unused]] bool have_park = false;
        [[maybe_unused]] long long park_cell = 0;
        [[maybe_unused]] double park_delta = 0.0;
        bool moved = false;
        Entry en;
        do {
            if (step >= p.max_steps) { cause = PGE_DEATH_AGE; break; }
            const int m = cv.m;
            if (m == PGE_MASK_OUTSIDE) { exited = true; cause = PGE_DEATH_EXIT; break; }
            const float h_here = cv.surf, b_here = cv.base;
            if (step == 0 && h_here < b_here) in_sea = true;
            if (in_sea) {
                if (h_here >= b_here || sed * vol / volume0 < R(1e-4) || sea_steps >= p.ocean_steps) { cause = PGE_DEATH_OCEAN; break; }
                sea_steps++;
            }
            if (m == PGE_MASK_ACTIVE) {
                r7 = r6; r6 = r5; r5 = r4; r4 = r3; r3 = r2; r2 = r1; r1 = r0; r0 = (int)cv.cell;
                if (nring < SPREAD) nring++;
            }
            // forces
            R h0, gi, gj;
            {
                const R wi = cv.wi, wj = cv.wj;
                const float h00 = cv.s00.x, h10 = cv.s10.x, h01 = cv.s01.x, h11 = cv.s11.x;
                h0 = R(h00) * (R(1) - wi) * (R(1) - wj) + R(h10) * wi * (R(1) - wj) + R(h01) * (R(1) - wi) * wj + R(h11) * wi * wj;
                const float d10 = h10 - h00, d11 = h11 - h01, d01 = h01 - h00, d1110 = h11 - h10;
                gi = R(d10) * (R(1) - wj) + R(d11) * wj;
                gj = R(d01) * (R(1) - wi) + R(d1110) * wi;
            }
            R h0r = h0;
            if (ROUTE) {
                // a lake or pit: steer on the epsilon-filled routing surface where it is above the terrain;
                // erode on the terrain (particle.py:453-460)
                R r0, rgi, rgj;
                if (route_sample(a, f, x, y, true, r0, rgi, rgj) && r0 > h0) {
                    h0r = r0;
                    gi = rgi;
                    gj = rgj;
                }
            }
            const R di = R(cv.q0) * gi + R(cv.q1) * gj;
            const R dj = R(cv.q1) * gi + R(cv.q2) * gj;
            R s2 = gi * di + gj * dj;
            if (s2 < R(0)) {
                s2 = R(0);
                if (TAPE) tb |= PGE_TB_S2_ZERO;
            }
            const R nrm = k_slope_sat > R(0) ? k_slope_gain / sqrt(s2 + k_slope_sat * k_slope_sat) : k_slope_gain / sqrt(R(1) + s2);
            const R na = -di * nrm, nb = -dj * nrm;
            const R ma = bilin(cv, 2), mb = bilin(cv, 3);
            R q = bilin(cv, 1);
            if (q < R(0)) {
                q = R(0);
                if (TAPE) tb |= PGE_TB_Q_ZERO;
            }
            const R vol_rel = vol / volume0;
            [[maybe_unused]] const R psa = sa, psb = sb;  // the direction this step started with (the bend, particle.py:485-486)
            R fr = R(1) - k_dt * k_friction;
            if (fr < R(0)) {
                fr = R(0);
                if (TAPE) tb |= PGE_TB_FR_ZERO;
            }
            sa *= fr;
            sb *= fr;
            const R mlen = snorm(cv, ma, mb);
            R slen = snorm(cv, sa, sb);
            if (mlen > R(1e-12) && slen > R(1e-12)) {
                const R cosang = sdot(cv, ma, mb, sa, sb) / (mlen * slen);
                const R k = k_kmom * cosang * k_momscale / (vol + k_momscale * q);
                sa += k * ma;
                sb += k * mb;
                if (TAPE) tb |= PGE_TB_MOM;
            }
            const R accel = k_dt / (vol_rel * k_density);
            sa += accel * na;
            sb += accel * nb;
            slen = snorm(cv, sa, sb);
            if (slen < R(1e-12)) { cause = PGE_DEATH_STOP; break; }
            sa /= slen;
            sb /= slen;
            R nx = x + sa, ny = y + sb;
            int nf = f;
            if (a.spherical) {
                if (nx < R(0) || nx >= Nf || ny < R(0) || ny >= Nf) {
                    R u = nx / Nf, v = ny / Nf;
                    nf = cross_face(a.cr_trig != 0, f, u, v, sa, sb);
                    nx = u * Nf;
                    ny = v * Nf;
                    if (TAPE) {
                        // clamped coordinates: transfer_velocity's own clamp when the face stays, else the
                        // clamps below
                        tb |= PGE_TB_CROSS;
                        if (nf == f) {
                            tb |= PGE_TB_SAME_FACE;
                            if (u <= R(0) || u >= R(0.999999999)) tb |= PGE_TB_X_CLAMP;
                            if (v <= R(0) || v >= R(0.999999999)) tb |= PGE_TB_Y_CLAMP;
                        } else {
                            if (nx >= Nf || nx < R(0)) tb |= PGE_TB_X_CLAMP;
                            if (ny >= Nf || ny < R(0)) tb |= PGE_TB_Y_CLAMP;
                        }
                    }
                    if (nx >= Nf) nx = Nf * R(0.999999999);
                    if (ny >= Nf) ny = Nf * R(0.999999999);
                    if (nx < R(0)) nx = R(0);
                    if (ny < R(0)) ny = R(0);
                }
            } else if (nx < R(-H) || nx >= Nf + R(H) || ny < R(-H) || ny >= Nf + R(H)) {
                exited = true; cause = PGE_DEATH_EXIT; break;
            }
            const int nei = (int)floor(nx) + H, nej = (int)floor(ny) + H;
            if (nei < 0 || nei >= NE || nej < 0 || nej >= NE) { exited = true; cause = PGE_DEATH_EXIT; break; }
            View nv;
            load_view(a, nf, nx, ny, nei, nej, nv);
            // the droplet's own change of the new cell, probed while its loads are in flight
            nxt.cell = nv.cell;
            nxt.own = LEDGER ? t.lookup(nv.cell, nxt.tidx) : 0.0;
            if (nv.m == PGE_MASK_OUTSIDE) { exited = true; cause = PGE_DEATH_EXIT; break; }
            const R h1 = bilin(nv, 0);
            const R b1 = R(nv.base);
            const R dh = h0 - (h1 > b1 ? h1 : b1);
            R h1r = h1;
            if (ROUTE) {  // particle.py:556-559
                R r1, unused_i, unused_j;
                if (route_sample(a, nf, nx, ny, false, r1, unused_i, unused_j) && r1 > h1) h1r = r1;
            }
            const R dhr = h0r - h1r;
            // the next cell's lake flag (2 or 3 on an overflowing lake)
            const float nflag = ROUTE && a.lakes ? __ldg(&a.R[nv.cell].y) : 0.0f;
            if (TAPE && h1 > b1) tb |= PGE_TB_H1_ABOVE;
            // mass transfer at the cell we leave (particle.py:562-671)
            if (m == PGE_MASK_ACTIVE && in_sea) {
                R cdiff = -k_ocean * sed;
                R room = has_hprev ? R(h_prev) - R(h_here) : k_fanroom;
                if (TAPE) tb |= PGE_TB_SEA | (has_hprev ? 0 : PGE_TB_ROOM_FLOOR);
                if (room < k_fanroom) {
                    room = k_fanroom;
                    if (TAPE) tb |= PGE_TB_ROOM_FLOOR;
                }
                const R lim = R(b_here) - k_depfloor - R(h_here);
                int ssrc = 0;
                if (lim < room) {
                    room = lim;
                    ssrc = 1;
                }
                if (room < R(0)) {
                    room = R(0);
                    ssrc = 2;
                }
                if (-cdiff * vol_rel > room) {
                    cdiff = -room / vol_rel;
                    if (TAPE) tb |= PGE_TB_CLAMP;
                }
                if (TAPE) tb |= ssrc << PGE_TB_SEA_SHIFT;
                sed += cdiff;
                en.cell = cv.cell;
                en.delta = (double)(-cdiff * vol_rel);
                en.vol = 0.0f;
                en.ma = 0.0f;
                en.mb = 0.0f;
                en.sidx = step;
                have_entry = true;
            } else if (m == PGE_MASK_ACTIVE) {
                R qe;
                if (inv_sat <= R(0)) qe = R(0);
                else if (p.disc_exponent == 0.5) qe = sqrt(q * inv_sat);
                else if (p.disc_exponent > 0.0) qe = pow(q * inv_sat, k_dexp);
                else qe = erf(q * inv_sat);
                R ker = k_erod;
                if (LEDGER && a.erod) ker = k_erod * R(__ldg(a.erod + cv.cell));  // the wave apply's calibration field
                R c_eq = ker * dh * (R(1) + k_kdisc * qe);
                if (TAPE) tb |= PGE_TB_LAND;
                if (c_eq < R(0)) {
                    c_eq = R(0);
                    if (TAPE) tb |= PGE_TB_CEQ_ZERO;
                }
                R k_e;
                if (c_eq > sed) {
                    if (TAPE) tb |= PGE_TB_COVER;
                    const float sthick = cv.sed;
                    R w_cover;
                    if (k_cover > R(0)) {
                        w_cover = R(sthick) / k_cover;
                        if (w_cover > R(1)) w_cover = R(1);
                    } else {
                        w_cover = sthick > 0.0f ? R(1) : R(0);
                    }
                    k_e = k_depr * (w_cover + (R(1) - w_cover) * (R(1) - R(cv.hard)));
                } else {
                    k_e = k_depr;
                }
                if (a.roots) k_e *= R(1) - R(__ldg(a.roots + cv.cell));  // roots hold the ground (particle.py:615-618)
                R cdiff = k_e * (c_eq - sed);
                [[maybe_unused]] R trapped = R(0);
                if (ROUTE) {
                    if (in_lake) {
                        cdiff = R(0);  // crossing a lake: the bed sees nothing (particle.py:626-629)
                    } else if (sed > R(0) && nflag >= 1.5f) {
                        const R trap = -R(p.lake_trap) * sed;  // entering a lake: the load drops at the shore (630-634)
                        if (trap < cdiff) cdiff = trap;
                        if (nflag >= 2.5f) trapped = R(p.lake_trap) * sed;  // ...and this lake has room for the rest (636)
                    }
                }
                const R kexp = R(1) + q * k_conc;
                if (cdiff > R(0)) {
                    R ecap = dh / kexp;
                    int esrc = 0;
                    if (ecap > k_maxe) {
                        ecap = k_maxe;
                        esrc = 1;
                    }
                    if (ecap > R(h_here)) {
                        ecap = h_here > 0.0f ? R(h_here) : R(0);
                        esrc = h_here > 0.0f ? 2 : 3;
                    }
                    if (TAPE) tb |= PGE_TB_POS | (esrc << PGE_TB_ECAP_SHIFT);
                    if (cdiff * vol_rel > ecap) {
                        cdiff = ecap / vol_rel;
                        if (TAPE) tb |= PGE_TB_CLAMP;
                    }
                } else if (cdiff < R(0)) {
                    R room = has_hprev ? R(h_prev) - R(h_here) : k_depfloor;
                    if (TAPE) tb |= PGE_TB_NEG | (has_hprev ? 0 : PGE_TB_ROOM_FLOOR);
                    if (room < k_depfloor) {
                        room = k_depfloor;
                        if (TAPE) tb |= PGE_TB_ROOM_FLOOR;
                    }
                    const R dcap = room / kexp;
                    if (-cdiff * vol_rel > dcap) {
                        cdiff = -dcap / vol_rel;
                        if (TAPE) tb |= PGE_TB_CLAMP;
                    }
                }
                sed += cdiff;
                en.cell = cv.cell;
                en.delta = (double)(-cdiff * vol_rel);
                en.vol = (float)vol;
                en.ma = (float)(vol * sa);
                en.mb = (float)(vol * sb);
                en.sidx = step;
                have_entry = true;
                if (!LEDGER && ROUTE && a.parks && trapped > R(0) && parks < LAKE_PARKS) {
                    // a lake with room keeps what its shore did not take (particle.py:672-696): parked on the lake
                    // cell stepped onto, an entry of volume -3 after the step's own, for the apply to count
                    // against the lake's room
                    const R rest = trapped + cdiff;  // cdiff <= 0: what the shore took
                    if (rest > R(0)) {
                        parks++;
                        sed -= rest;
                        park_cell = nv.cell;
                        park_delta = (double)(rest * vol_rel);
                        have_park = true;
                    }
                }
                if (LATERAL && cdiff > R(0)) {
                    // the outside of the bend (particle.py:699-738): a droplet cutting and turning also cuts
                    // the bank one cell across the flow, down towards the bed it just eroded; the change
                    // list's room (two entries a step) always holds it
                    const R cross = psa * sb - psb * sa;
                    const R turn = cross > R(0) ? cross : -cross;
                    if (turn > R(1e-6)) {
                        const R sgn = cross > R(0) ? R(1) : R(-1);
                        const R bx = x + sgn * sb, by = y - sgn * sa;
                        const int bei = (int)floor(bx) + H, bej = (int)floor(by) + H;
                        if (bei >= 0 && bei < NE && bej >= 0 && bej < NE) {
                            const long long bc = ((long long)f * NE + bei) * NE + bej;
                            const int bm = a.mask ? (int)__ldg(a.mask + bc) : PGE_MASK_ACTIVE;
                            const float bank = bm == PGE_MASK_ACTIVE ? __ldg(&a.A[bc].x) - h_here : 0.0f;
                            if (bank > 0.0f) {
                                R lat = R(p.lateral_rate) * turn * cdiff;
                                R lcap = R(bank) / kexp;
                                if (lcap > k_maxe) lcap = k_maxe;
                                if (lat * vol_rel > lcap) lat = lcap / vol_rel;
                                if (lat > R(0)) {
                                    sed += lat;
                                    bank_en.cell = bc;
                                    bank_en.delta = (double)(-lat * vol_rel);
                                    bank_en.vol = -2.0f;
                                    bank_en.ma = 0.0f;
                                    bank_en.mb = 0.0f;
                                    bank_en.sidx = step;
                                    have_bank = true;
                                }
                            }
                        }
                    }
                }
            }
            // evaporation (mass conserving)
            R ev = R(1) - k_dt * k_evap * R(cv.evap);
            if (ev < R(0.01)) {
                ev = R(0.01);
                if (TAPE) tb |= PGE_TB_EV_CLAMP;
            }
            vol *= ev;
            sed /= ev;
            x = nx;
            y = ny;
            f = nf;
            h_prev = h_here;
            has_hprev = true;
            if (ROUTE) in_lake = nflag >= 1.5f;
            cv = nv;
            moved = true;
            if (TAPE) a.tape.bits[trow * (a.tape.steps + 1) + step] = tb;
            step++;
            // stop conditions
            if (nv.surf < nv.base && !in_sea) {
                in_sea = true;
                if (sed <= R(0)) { cause = PGE_DEATH_OCEAN; break; }
            }
            if (vol < k_minvol) { cause = in_sea ? PGE_DEATH_OCEAN : PGE_DEATH_EVAP; break; }
            if (dhr < R(0) && !in_lake) {
                uphill++;
                if (uphill > p.pit_steps) { cause = in_sea ? PGE_DEATH_OCEAN : PGE_DEATH_PIT; break; }
            } else {
                uphill = 0;
            }
        } while (false);

        // ---- the ledger, one entry behind the trace
        if (have_entry) {
            // `cur` still describes the cell the entry was made at
            if (has_pe && LEDGER) {
                apply_entry<TAPE, ROUTE>(a, t, L, pe, pend, true, cur, trow);
                sync_own(cur, pend);
                sync_own(nxt, pend);
            }
            pe = en;
            pend = cur;
            has_pe = true;
            if (a.rec_cell && rec_n < a.rec_cap) {
                const long long o = (d - a.rec_base) * a.rec_cap + rec_n;
                a.rec_cell[o] = (int32_t)en.cell;
                a.rec_delta[o] = en.delta;
                a.rec_vol[o] = en.vol;
                a.rec_mom[2 * o] = en.ma;
                a.rec_mom[2 * o + 1] = en.mb;
            }
            rec_n++;
        }
        if (!LEDGER && ROUTE && have_park) {
            if (a.rec_cell && rec_n < a.rec_cap) {
                const long long o = (d - a.rec_base) * a.rec_cap + rec_n;
                a.rec_cell[o] = (int32_t)park_cell;
                a.rec_delta[o] = park_delta;
                a.rec_vol[o] = -3.0f;
                a.rec_mom[2 * o] = 0.0f;
                a.rec_mom[2 * o + 1] = 0.0f;
            }
            if (a.park_k) a.park_k[(d - a.rec_base) * LAKE_PARKS + parks - 1] = rec_n;
            rec_n++;
            nbank++;
        }
        if (LATERAL && have_bank) {
            // the bank entry follows the step's own: the step entry is applied with the bank as its next
            // cell, the bank entry with the next step's cell (the reference's list order)
            LCell bk;
            bk.cell = bank_en.cell;
            if (LEDGER) {
                load_lcell(a, t, bank_en.cell, bk);
                apply_entry<TAPE, ROUTE>(a, t, L, pe, pend, true, bk, trow);
                sync_own(bk, pend);
                sync_own(cur, pend);
                sync_own(nxt, pend);
            }
            pe = bank_en;
            pend = bk;
            if (a.rec_cell && rec_n < a.rec_cap) {
                const long long o = (d - a.rec_base) * a.rec_cap + rec_n;
                a.rec_cell[o] = (int32_t)bank_en.cell;
                a.rec_delta[o] = bank_en.delta;
                a.rec_vol[o] = -2.0f;
                a.rec_mom[2 * o] = 0.0f;
                a.rec_mom[2 * o + 1] = 0.0f;
            }
            rec_n++;
            nbank++;
        }
        if (moved) {
            // the new cell becomes current (its own change was probed above)
            cur.cell = cv.cell;
            cur.m = cv.m;
            cur.base = cv.base;
            cur.hs = cv.hs;
            cur.accws = cv.accws;
            cur.own = nxt.own;
            cur.tidx = nxt.tidx;
        }
        if (cause < 0) continue;

        // ---- death: final deposits (particle.py:770-815) and the rest of the ledger
        if (in_sea && (cause == PGE_DEATH_AGE || cause == PGE_DEATH_STOP)) cause = PGE_DEATH_OCEAN;
        if (!exited) {
            const int ei = cell_of(x, N) + H, ej = cell_of(y, N) + H;
            const long long c = ((long long)f * NE + ei) * NE + ej;
            const int mc = a.mask ? (int)__ldg(a.mask + c) : PGE_MASK_ACTIVE;
            const float sc = __ldg(&a.A[c].x), bc = __ldg(&a.B[c].w);
            if (mc == PGE_MASK_ACTIVE && !(in_sea && sc >= bc)) {
                if (nring == 0 || r0 != (int)c) {
                    r7 = r6; r6 = r5; r5 = r4; r4 = r3; r3 = r2; r2 = r1; r1 = r0; r0 = (int)c;
                    if (nring < SPREAD) nring++;
                }
            }
        }
        int nout = 0;
        double load = 0.0;
        if (sed > R(0) && nring > 0 && (!exited || a.deposit_on_exit)) {
            load = (double)(sed * vol / volume0);
            nout = cause == PGE_DEATH_OCEAN ? 1 : nring;
        }
        const int ring[SPREAD] = {r0, r1, r2, r3, r4, r5, r6, r7};
        if (!LEDGER) {
            // record-only: the final deposits go to the change list, the ordered apply does the rest
            for (int r = 0; r < nout; r++) {
                if (a.rec_cell && rec_n < a.rec_cap) {
                    const long long o = (d - a.rec_base) * a.rec_cap + rec_n;
                    a.rec_cell[o] = ring[r];
                    a.rec_delta[o] = r == 0 ? load : 0.0;
                    a.rec_vol[o] = -1.0f;
                    a.rec_mom[2 * o] = 0.0f;
                    a.rec_mom[2 * o + 1] = 0.0f;
                }
                rec_n++;
            }
            atomicAdd(&sstat[ST_DROP], 1ull);
            atomicAdd(&sstat[ST_STEPS], (unsigned long long)step_entries(rec_n - nbank, nout));
            atomicAdd(&sstat[ST_ENTRIES], (unsigned long long)rec_n);
            atomicAdd(&sstat[ST_DEATH0 + cause], 1ull);
            if (a.rec_cell) {
                a.rec_count[d - a.rec_base] = rec_n;
                a.rec_death[d - a.rec_base] = (int8_t)cause;
            }
            if (a.park_n) a.park_n[d - a.rec_base] = parks;
            alive = false;
            continue;
        }
        if (nout > 0) load_lcell(a, t, ring[0], nxt);
        if (has_pe) {
            apply_entry<TAPE, ROUTE>(a, t, L, pe, pend, nout > 0, nxt, trow);
            if (nout > 0) sync_own(nxt, pend);
        }
        for (int r = 0; r < nout; r++) {
            LCell c = nxt;
            const bool more = r + 1 < nout;
            if (more) load_lcell(a, t, ring[r + 1], nxt);
            Entry fe;
            fe.cell = ring[r];
            fe.delta = r == 0 ? load : 0.0;
            fe.vol = -1.0f;
            fe.ma = fe.mb = 0.0f;
            fe.sidx = -1;
            apply_entry<TAPE, ROUTE>(a, t, L, fe, c, more, nxt, trow);
            if (more) sync_own(nxt, c);
            if (a.rec_cell && rec_n < a.rec_cap) {
                const long long o = (d - a.rec_base) * a.rec_cap + rec_n;
                a.rec_cell[o] = (int32_t)fe.cell;
                a.rec_delta[o] = fe.delta;
                a.rec_vol[o] = -1.0f;
                a.rec_mom[2 * o] = 0.0f;
                a.rec_mom[2 * o + 1] = 0.0f;
            }
            rec_n++;
        }
        // leftover load: the death cell's stockpile (particle.py:1019-1041)
        long long topend = 0, lostoff = 0;
        if (L.surplus > 0.0 && L.death >= 0) {
            LCell dc;
            load_lcell(a, t, L.death, dc);
            if (dc.live() < (double)dc.base) {
                double keep = L.surplus * (1.0 - p.offshore_writeoff);
                if (keep < 1e-4) keep = 0.0;
                topend = fx_mass(keep);
                lostoff = fx_mass(L.surplus) - topend;
            } else {
                topend = fx_mass(L.surplus);
            }
            if (topend) red_add(a.pend + L.death, topend);
        }
        if (TAPE) {
            const long long o = trow * (a.tape.steps + 1) + step;
            double *ts = a.tape.state + o * 6;
            ts[0] = (double)x;
            ts[1] = (double)y;
            ts[2] = (double)sa;
            ts[3] = (double)sb;
            ts[4] = (double)sed;
            ts[5] = (double)vol;
            a.tape.bits[o] = f;
            reinterpret_cast<int2 *>(a.tape.count)[trow] = make_int2(step + 1, L.tap_n);
        }
        atomicAdd(&sstat[ST_DROP], 1ull);
        atomicAdd(&sstat[ST_STEPS], (unsigned long long)step_entries(rec_n - nbank, nout));
        atomicAdd(&sstat[ST_ENTRIES], (unsigned long long)rec_n);
        if (L.clamped) atomicAdd(&sstat[ST_CLAMPED], (unsigned long long)L.clamped);
        if (t.overflow) atomicAdd(&sstat[ST_OVER], 1ull);
        if (topend) atomicAdd(&sstat[ST_TOPEND], (unsigned long long)topend);
        if (L.deficit > 0.0) atomicAdd(&sstat[ST_DEFICIT], (unsigned long long)fx_mass(L.deficit));
        if (lostoff) atomicAdd(&sstat[ST_LOSTOFF], (unsigned long long)lostoff);
        if (L.eroded_fx) atomicAdd(&sstat[ST_ERODED], (unsigned long long)L.eroded_fx);
        if (L.deposited_fx) atomicAdd(&sstat[ST_DEPOSITED], (unsigned long long)L.deposited_fx);
        atomicAdd(&sstat[ST_DEATH0 + cause], 1ull);
        if (a.rec_cell) {
            a.rec_count[d - a.rec_base] = rec_n;
            a.rec_death[d - a.rec_base] = (int8_t)cause;
        }
        alive = false;
    }

    // ---- flush the block's counters
    __syncthreads();
    if (threadIdx.x < ST_N) {
        int64_t *dst;
        const int k = threadIdx.x;
        PgeStats *st = a.stats;
        switch (k) {
        case ST_DROP: dst = &st->droplets; break;
        case ST_STEPS: dst = &st->droplet_steps; break;
        case ST_ENTRIES: dst = &st->entries; break;
        case ST_CLAMPED: dst = &st->clamped; break;
        case ST_OVER: dst = &st->overflow; break;
        case ST_TOPEND: dst = &st->to_pending_fx; break;
        case ST_DEFICIT: dst = &st->deficit_out_fx; break;
        case ST_LOSTOFF: dst = &st->lost_offshore_fx; break;
        case ST_ERODED: dst = &st->eroded_fx; break;
        case ST_DEPOSITED: dst = &st->deposited_fx; break;
        default: dst = &st->deaths[k - ST_DEATH0]; break;
        }
        if (sstat[k]) red_add(reinterpret_cast<long long *>(dst), (long long)sstat[k]);
    }
}

}  // namespace PGE_VARIANT
}  // namespace pge
