// pge_adjoint.cu -- the reverse of one taped wave-apply droplet pass.
//
// The forward (droplet_kernel<1, true, true>, one wave) recorded, per
// droplet, its state (x, y, a, b, sed, vol) at the start of every step and
// after the last, the face and the branches of every step (PGE_TB_*), and
// the branch code of every ledger entry (PGE_TE_*).  One thread reverses one
// droplet: the ledger's entries and the trace's steps are swept backwards
// together (the ledger's deficit / surplus adjoints only depend on later
// entries), each step's intermediates recomputed from its recorded start
// state.  What the pass reads of the terrain (bilinear stencils, the cell's
// own surface, the ledger's live heights) receives its adjoint by float64
// atomics into zbar_before, which starts as zbar_after (the fold adds the
// applied change to the surface, so the surface passes straight through).
//
// The model differentiated is the pass on its recorded path: the trace of
// particle.py:421-815 (bilinear sample and gradient, direction update with
// friction, momentum pull and gravity, metric normalisation, face transfer,
// capacity law, exchange rate, erosion cap and deposit room, evaporation,
// final load) and the ledger of particle.py:934-1018 (erosion floor,
// deposit ceiling, deficit and surplus carried down the path).  Branches are
// those the forward took; tracks, cover, hardness, evaporation field, base
// level and the droplet's own earlier changes inside its ledger bounds are
// constants.  With carry_path = 0 the position and direction adjoints are not
// handed from a step to the one before it (each step's incoming position and
// direction are constants; its own move is still differentiated).
#include <cmath>

#include "pge_internal.cuh"
#include "pge_maps.cuh"

namespace pge {
namespace adj {

// ---------------------------------------------------------------------------
// forward-mode duals for the face transfer's 4x4 Jacobian
// ---------------------------------------------------------------------------
struct D4 {
    double v, d[4];
};

__device__ __forceinline__ D4 mk(double v)
{
    D4 r;
    r.v = v;
    r.d[0] = r.d[1] = r.d[2] = r.d[3] = 0.0;
    return r;
}
__device__ __forceinline__ D4 operator+(const D4 &a, const D4 &b)
{
    D4 r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator-(const D4 &a, const D4 &b)
{
    D4 r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator*(const D4 &a, const D4 &b)
{
    D4 r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ D4 operator*(const D4 &a, double s)
{
    D4 r;
    r.v = a.v * s;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] * s;
    return r;
}
__device__ __forceinline__ D4 operator/(const D4 &a, const D4 &b)
{
    D4 r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
__device__ __forceinline__ D4 operator+(const D4 &a, double s)
{
    D4 r = a;
    r.v += s;
    return r;
}
__device__ __forceinline__ D4 dsqrt(const D4 &a)
{
    D4 r;
    r.v = sqrt(a.v);
    const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] * g;
    return r;
}
__device__ __forceinline__ D4 dtan(const D4 &a)
{
    D4 r;
    r.v = tan(a.v);  // as the taped wave-apply pass crosses faces (CUDA's own)
    const double g = 1.0 + r.v * r.v;
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] * g;
    return r;
}
__device__ __forceinline__ D4 datan(const D4 &a)
{
    D4 r;
    r.v = atan(a.v);
    const double g = 1.0 / (1.0 + a.v * a.v);
#pragma unroll
    for (int k = 0; k < 4; k++) r.d[k] = a.d[k] * g;
    return r;
}

// face frames (right, up, normal) of the cube-sphere faces (cubesphere.py's face bases)
__constant__ double kAxes[6][3][3] = {
    {{0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}, {1.0, 0.0, 0.0}},
    {{0.0, 0.0, 1.0}, {0.0, -1.0, 0.0}, {-1.0, 0.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, 1.0}, {0.0, 1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, 1.0}},
    {{-1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, -1.0}},
};
constexpr double kHalfPi = 1.57079632679489661923;
constexpr double kTwoOverPi = 0.63661977236758134308;

// tangent-plane basis of (face, u, v) on the unit sphere: d p / d u, d p / d v
__device__ __noinline__ void face_frame(int face, const D4 &u, const D4 &v, D4 J[6])
{
    const double(*ax)[3] = kAxes[face];
    const D4 s = dtan((u + (-0.5)) * kHalfPi), t = dtan((v + (-0.5)) * kHalfPi);
    const D4 dsdu = (s * s + 1.0) * kHalfPi, dtdv = (t * t + 1.0) * kHalfPi;
    D4 q[3], p[3];
    for (int k = 0; k < 3; k++) q[k] = s * ax[0][k] + t * ax[1][k] + ax[2][k];
    const D4 ql = dsqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    for (int k = 0; k < 3; k++) p[k] = q[k] / ql;
    D4 du[3], dv[3];
    for (int k = 0; k < 3; k++) {
        du[k] = dsdu * ax[0][k];
        dv[k] = dtdv * ax[1][k];
    }
    const D4 pu = p[0] * du[0] + p[1] * du[1] + p[2] * du[2];
    const D4 pv = p[0] * dv[0] + p[1] * dv[1] + p[2] * dv[2];
    for (int k = 0; k < 3; k++) {
        J[k] = (du[k] - p[k] * pu) / ql;
        J[3 + k] = (dv[k] - p[k] * pv) / ql;
    }
}

// the face transfer (cubesphere.transfer_velocity) on duals, for a move that
// lands on face f2 != face; (u, v, a, b) updated in place
__device__ __noinline__ void transfer_dual(int face, int f2, D4 &u, D4 &v, D4 &a, D4 &b)
{
    const double(*ax)[3] = kAxes[face];
    const D4 s = dtan((u + (-0.5)) * kHalfPi), t = dtan((v + (-0.5)) * kHalfPi);
    D4 q[3];
    for (int k = 0; k < 3; k++) q[k] = s * ax[0][k] + t * ax[1][k] + ax[2][k];
    const D4 ql = dsqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    D4 p[3];
    for (int k = 0; k < 3; k++) p[k] = q[k] / ql;
    const double(*bx)[3] = kAxes[f2];
    const D4 dn = p[0] * bx[2][0] + p[1] * bx[2][1] + p[2] * bx[2][2];
    const D4 s2 = (p[0] * bx[0][0] + p[1] * bx[0][1] + p[2] * bx[0][2]) / dn;
    const D4 t2 = (p[0] * bx[1][0] + p[1] * bx[1][1] + p[2] * bx[1][2]) / dn;
    const D4 u2 = datan(s2) * kTwoOverPi + 0.5, v2 = datan(t2) * kTwoOverPi + 0.5;
    D4 J[6], K[6];
    face_frame(face, u, v, J);
    D4 w[3];
    for (int k = 0; k < 3; k++) w[k] = a * J[k] + b * J[3 + k];
    face_frame(f2, u2, v2, K);
    const D4 guu = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
    const D4 guv = K[0] * K[3] + K[1] * K[4] + K[2] * K[5];
    const D4 gvv = K[3] * K[3] + K[4] * K[4] + K[5] * K[5];
    const D4 ru = K[0] * w[0] + K[1] * w[1] + K[2] * w[2];
    const D4 rv = K[3] * w[0] + K[4] * w[1] + K[5] * w[2];
    const D4 det = guu * gvv - guv * guv;
    a = (gvv * ru - guv * rv) / det;
    b = (guu * rv - guv * ru) / det;
    u = u2;
    v = v2;
}

// ---------------------------------------------------------------------------
// the reverse kernel
// ---------------------------------------------------------------------------
struct AdjArgs {
    int F, N, H, NE, metric_shared, carry_path;
    const float4 *__restrict__ A;
    const float4 *__restrict__ B;
    const float4 *__restrict__ G;
    const float *__restrict__ erod;
    PgeParams p;
    double volume0;
    PgeTape tape;
    long long d0, d1;  // the droplets (tape rows) of the wave reversed
    const double *__restrict__ zbar_after;
    double *zbar_before;
    double *ebar;
    double *pbar;
    int *error;
};

__device__ __forceinline__ void zadd(const AdjArgs &a, long long c, double v)
{
    if (v != 0.0) atomicAdd(a.zbar_before + c, v);
}

// a bilinear stencil of the packed samples at (face, x, y)
struct Stencil {
    long long c00;
    double wi, wj;
    bool ci, cj;  // weight clamped to [0, 1]
    float4 s00, s10, s01, s11;
};

__device__ __forceinline__ void stencil(const AdjArgs &a, int f, double x, double y, Stencil &s)
{
    const int NE = a.NE;
    const double fi = x - 0.5 + (double)a.H, fj = y - 0.5 + (double)a.H;
    int i0 = (int)floor(fi), j0 = (int)floor(fj);
    if (i0 < 0) i0 = 0;
    if (i0 > NE - 2) i0 = NE - 2;
    if (j0 < 0) j0 = 0;
    if (j0 > NE - 2) j0 = NE - 2;
    const double wi = fi - (double)i0, wj = fj - (double)j0;
    s.ci = wi < 0.0 || wi > 1.0;
    s.cj = wj < 0.0 || wj > 1.0;
    s.wi = wi < 0.0 ? 0.0 : (wi > 1.0 ? 1.0 : wi);
    s.wj = wj < 0.0 ? 0.0 : (wj > 1.0 ? 1.0 : wj);
    s.c00 = ((long long)f * NE + i0) * NE + j0;
    s.s00 = __ldg(a.A + s.c00);
    s.s01 = __ldg(a.A + s.c00 + 1);
    s.s10 = __ldg(a.A + s.c00 + NE);
    s.s11 = __ldg(a.A + s.c00 + NE + 1);
}

__device__ __forceinline__ int cell_idx(double x, int N)
{
    const int i = (int)floor(x);
    return i < 0 ? 0 : (i > N - 1 ? N - 1 : i);
}

__device__ __forceinline__ double bil(double v00, double v10, double v01, double v11, double wi, double wj)
{
    return v00 * (1.0 - wi) * (1.0 - wj) + v10 * wi * (1.0 - wj) + v01 * (1.0 - wi) * wj + v11 * wi * wj;
}

// the ledger's reverse for one entry: returns d(L)/d(proposed delta), updates
// the deficit / surplus adjoints and adds the bounds' terrain adjoints
__device__ __forceinline__ double ledger_rev(const AdjArgs &a, const int4 e, double &Db, double &Sb)
{
    const int code = e.z;
    if (code & PGE_TE_SKIP) return 0.0;
    const long long c = e.x;
    const double ab = __ldg(a.zbar_after + c);  // d L / d (applied change at c)
    const int src = (code >> PGE_TE_SRC_SHIFT) & 7;
    if (!(code & PGE_TE_DEPOSIT)) {
        // applied = -e_act; deficit += ew - e_act
        const double eb = -ab - Db;
        double ewb = Db;
        if (src == 0) ewb += eb;
        else if (src == 2) zadd(a, c, eb);  // e_act = s_c - base
        else if (src == 4) {                // e_act = s_c - (next cell's live height)
            zadd(a, c, eb);
            zadd(a, e.y, -eb);
        }
        return -ewb;  // ew = -delta
    }
    // applied = d_act; surplus = want - d_act
    const double dab = ab - Sb;
    double wantb = Sb;
    if (src == 0) wantb += dab;
    else if (src == 2) {  // d_act = (reference live height + consts) - s_c
        zadd(a, e.y, dab);
        zadd(a, c, -dab);
    } else if (src == 3) zadd(a, c, -dab);  // d_act = base - dep_floor - s_c
    const int take = (code >> PGE_TE_TAKE_SHIFT) & 3;
    double want0b;
    if (take == 1) {  // all of want went to the deficit: want = 0, deficit -= want0
        want0b = -Db;
    } else if (take == 2) {  // the whole deficit taken: want = want0 - deficit, deficit = 0
        want0b = wantb;
        Db = -wantb;
    } else {
        want0b = wantb;
    }
    Sb = want0b;  // want0 = delta + surplus (the surplus then cleared)
    return want0b;
}

__global__ void __launch_bounds__(128) adjoint_kernel(const AdjArgs a)
{
    const long long r = a.d0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double pb_ke = 0.0, pb_kr = 0.0, pb_kv = 0.0, pb_fr = 0.0;
    if (r < a.d1) {
        const PgeParams &p = a.p;
        const int N = a.N, NE = a.NE, H = a.H;
        const double V0 = a.volume0;
        const long long srow = r * (a.tape.steps + 1);
        const int2 cnt = reinterpret_cast<const int2 *>(a.tape.count)[r];
        const int ns = cnt.x < 1 ? 1 : (cnt.x > a.tape.steps + 1 ? a.tape.steps + 1 : cnt.x);
        int j = cnt.y < a.tape.entries ? cnt.y : a.tape.entries;
        if (cnt.y > a.tape.entries || cnt.x < 1 || cnt.x > a.tape.steps + 1) atomicOr(a.error, 1);
        const int4 *ent = reinterpret_cast<const int4 *>(a.tape.entry) + r * a.tape.entries;
        double Db = 0.0, Sb = 0.0;
        // final deposits: the first carries the load sed * vol / volume0
        double loadb = 0.0;
        j--;
        while (j >= 0) {
            const int4 e = ent[j];
            if (e.z & PGE_TE_STEP) break;
            loadb = ledger_rev(a, e, Db, Sb);
            j--;
        }
        const double *st = a.tape.state + srow * 6;
        double xn = st[(ns - 1) * 6 + 0], yn = st[(ns - 1) * 6 + 1];
        int fn = a.tape.bits[srow + ns - 1] & PGE_TB_FACE;
        const double sedf = st[(ns - 1) * 6 + 4], volf = st[(ns - 1) * 6 + 5];
        // adjoints of the state after the current step
        double xb = 0.0, yb = 0.0, sab = 0.0, sbb = 0.0, sedb = loadb * volf / V0, volb = loadb * sedf / V0;

        const double inv_sat = p.disc_saturation > 0.0 ? 1.0 / p.disc_saturation : 0.0;
        const double csat = p.slope_sat > 0.0 ? p.slope_sat * p.slope_sat : 1.0;
        for (int k = ns - 2; k >= 0; k--) {
            const int tb = a.tape.bits[srow + k];
            const int f = tb & PGE_TB_FACE;
            const double x = st[k * 6 + 0], y = st[k * 6 + 1], sa0 = st[k * 6 + 2], sb0 = st[k * 6 + 3], sed = st[k * 6 + 4],
                         vol = st[k * 6 + 5];
            double dbar = 0.0;
            if (tb & (PGE_TB_LAND | PGE_TB_SEA)) {
                if (j < 0 || !(ent[j].z & PGE_TE_STEP) || ent[j].w != k) {
                    atomicOr(a.error, 2);
                } else {
                    dbar = ledger_rev(a, ent[j], Db, Sb);
                    j--;
                }
            }
            // ---- recompute the step's forward values
            Stencil cs;
            stencil(a, f, x, y, cs);
            const int ei = cell_idx(x, N) + H, ej = cell_idx(y, N) + H;
            const long long cc = ((long long)f * NE + ei) * NE + ej;
            const float4 bc = __ldg(a.B + cc);
            const long long mc = a.metric_shared ? (long long)ei * NE + ej : cc;
            const float4 g0v = __ldg(a.G + 2 * mc), g1v = __ldg(a.G + 2 * mc + 1);
            const double G0 = g0v.x, G1 = g0v.y, G2 = g0v.z, Q0 = g0v.w, Q1 = g1v.x, Q2 = g1v.y;
            const double wi = cs.wi, wj = cs.wj;
            const double H00 = cs.s00.x, H10 = cs.s10.x, H01 = cs.s01.x, H11 = cs.s11.x;
            const double h0 = bil(H00, H10, H01, H11, wi, wj);
            const double gi = (H10 - H00) * (1.0 - wj) + (H11 - H01) * wj;
            const double gj = (H01 - H00) * (1.0 - wi) + (H11 - H10) * wi;
            const double di = Q0 * gi + Q1 * gj, dj = Q1 * gi + Q2 * gj;
            double s2 = gi * di + gj * dj;
            if (tb & PGE_TB_S2_ZERO) s2 = 0.0;
            const double nrm = p.slope_gain / sqrt(s2 + csat);
            const double na = -di * nrm, nb = -dj * nrm;
            const double ma = bil(cs.s00.z, cs.s10.z, cs.s01.z, cs.s11.z, wi, wj);
            const double mb = bil(cs.s00.w, cs.s10.w, cs.s01.w, cs.s11.w, wi, wj);
            double q = bil(cs.s00.y, cs.s10.y, cs.s01.y, cs.s11.y, wi, wj);
            if (tb & PGE_TB_Q_ZERO) q = 0.0;
            const double vr = vol / V0;
            const double fr = (tb & PGE_TB_FR_ZERO) ? 0.0 : 1.0 - p.dt * p.friction;
            const double sa1 = sa0 * fr, sb1 = sb0 * fr;
            const double mlen = sqrt(fmax(G0 * ma * ma + 2.0 * G1 * ma * mb + G2 * mb * mb, 0.0));
            const double slen1 = sqrt(fmax(G0 * sa1 * sa1 + 2.0 * G1 * sa1 * sb1 + G2 * sb1 * sb1, 0.0));
            double sa2 = sa1, sb2 = sb1, kk = 0.0, cosang = 0.0;
            const double den = vol + p.mom_scale * q;
            if (tb & PGE_TB_MOM) {
                cosang = (G0 * ma * sa1 + G1 * (ma * sb1 + mb * sa1) + G2 * mb * sb1) / (mlen * slen1);
                kk = p.k_mom * cosang * p.mom_scale / den;
                sa2 = sa1 + kk * ma;
                sb2 = sb1 + kk * mb;
            }
            const double accel = p.dt / (vr * p.density);
            const double sa3 = sa2 + accel * na, sb3 = sb2 + accel * nb;
            const double slen3 = sqrt(fmax(G0 * sa3 * sa3 + 2.0 * G1 * sa3 * sb3 + G2 * sb3 * sb3, 0.0));
            const double sa4 = sa3 / slen3, sb4 = sb3 / slen3;
            // the new cell
            Stencil ns_;
            stencil(a, fn, xn, yn, ns_);
            const int nei = cell_idx(xn, N) + H, nej = cell_idx(yn, N) + H;
            const long long nc = ((long long)fn * NE + nei) * NE + nej;
            const double b1 = __ldg(&a.B[nc].w);
            const double h1 = bil(ns_.s00.x, ns_.s10.x, ns_.s01.x, ns_.s11.x, ns_.wi, ns_.wj);
            const double dh = h0 - ((tb & PGE_TB_H1_ABOVE) ? h1 : b1);
            const double h_here = (double)__ldg(&a.A[cc].x);
            long long pc = -1;  // the previous step's own cell (h_prev)
            if (k > 0) {
                const int pf = a.tape.bits[srow + k - 1] & PGE_TB_FACE;
                pc = ((long long)pf * NE + cell_idx(st[(k - 1) * 6], N) + H) * NE + cell_idx(st[(k - 1) * 6 + 1], N) + H;
            }
            const double h_prev = pc >= 0 ? (double)__ldg(&a.A[pc].x) : 0.0;
            // mass transfer and evaporation
            const double ev = (tb & PGE_TB_EV_CLAMP) ? 0.01 : 1.0 - p.dt * p.evap_rate * (double)bc.x;
            double cdiff = 0.0, ceq = 0.0, ke = 0.0, kw = 1.0, kexp = 1.0, qe = 0.0, ker = p.erodibility, ecap = 0.0, room = 0.0,
                   dcap = 0.0;
            const double E = a.erod ? (double)__ldg(a.erod + cc) : 1.0;
            if (tb & PGE_TB_LAND) {
                if (inv_sat <= 0.0) qe = 0.0;
                else if (p.disc_exponent == 0.5) qe = sqrt(q * inv_sat);
                else if (p.disc_exponent > 0.0) qe = pow(q * inv_sat, p.disc_exponent);
                else qe = erf(q * inv_sat);
                ker = a.erod ? p.erodibility * E : p.erodibility;
                ceq = (tb & PGE_TB_CEQ_ZERO) ? 0.0 : ker * dh * (1.0 + p.k_disc * qe);
                if (tb & PGE_TB_COVER) {
                    const double sthick = bc.z;
                    double wc;
                    if (p.cover_depth > 0.0) wc = fmin(sthick / p.cover_depth, 1.0);
                    else wc = sthick > 0.0 ? 1.0 : 0.0;
                    kw = wc + (1.0 - wc) * (1.0 - (double)bc.y);
                }
                ke = p.deposition_rate * kw;
                cdiff = ke * (ceq - sed);
                kexp = 1.0 + q * p.conc_scale;
                if (tb & PGE_TB_CLAMP) {
                    if (tb & PGE_TB_POS) {
                        const int es = (tb >> PGE_TB_ECAP_SHIFT) & 3;
                        ecap = es == 0 ? dh / kexp : (es == 1 ? p.max_erode : (es == 2 ? h_here : 0.0));
                        cdiff = ecap / vr;
                    } else {
                        room = (tb & PGE_TB_ROOM_FLOOR) ? p.dep_floor : h_prev - h_here;
                        dcap = room / kexp;
                        cdiff = -dcap / vr;
                    }
                }
            } else if (tb & PGE_TB_SEA) {
                cdiff = -p.ocean_rate * sed;
                if (tb & PGE_TB_CLAMP) {
                    const int ss = (tb >> PGE_TB_SEA_SHIFT) & 3;
                    if (ss == 0) room = (tb & PGE_TB_ROOM_FLOOR) ? p.fan_room : h_prev - h_here;
                    else if (ss == 1) room = (double)bc.w - p.dep_floor - h_here;
                    else room = 0.0;
                    cdiff = -room / vr;
                }
            }
            const double sed1 = sed + cdiff;

            // ---- reverse
            double x_b = 0.0, y_b = 0.0, sa_b = 0.0, sb_b = 0.0, sed_b = 0.0, vol_b = 0.0, vr_b = 0.0, q_b = 0.0;
            double dh_b = 0.0;
            // evaporation: vol' = vol ev, sed' = sed1 / ev
            const double ev_b = volb * vol - sedb * sed1 / (ev * ev);
            vol_b += volb * ev;
            const double sed1_b = sedb / ev;
            if (!(tb & PGE_TB_EV_CLAMP)) pb_kv += -ev_b * p.dt * (double)bc.x;
            // entry delta = -cdiff vr; sed1 = sed + cdiff
            double cdiff_b = 0.0;
            sed_b += sed1_b;
            if (tb & (PGE_TB_LAND | PGE_TB_SEA)) {
                cdiff_b = -dbar * vr + sed1_b;
                vr_b += -dbar * cdiff;
            }
            if (tb & PGE_TB_LAND) {
                double kexp_b = 0.0;
                if (tb & PGE_TB_CLAMP) {
                    if (tb & PGE_TB_POS) {  // cdiff = ecap / vr
                        const double ecap_b = cdiff_b / vr;
                        vr_b -= cdiff_b * ecap / (vr * vr);
                        const int es = (tb >> PGE_TB_ECAP_SHIFT) & 3;
                        if (es == 0) {
                            dh_b += ecap_b / kexp;
                            kexp_b -= ecap_b * dh / (kexp * kexp);
                        } else if (es == 2) {
                            zadd(a, cc, ecap_b);
                        }
                    } else {  // cdiff = -(room / kexp) / vr
                        const double dcap_b = -cdiff_b / vr;
                        vr_b += cdiff_b * dcap / (vr * vr);
                        const double room_b = dcap_b / kexp;
                        kexp_b -= dcap_b * room / (kexp * kexp);
                        if (!(tb & PGE_TB_ROOM_FLOOR) && pc >= 0) {
                            zadd(a, pc, room_b);
                            zadd(a, cc, -room_b);
                        }
                    }
                } else {  // cdiff = ke (ceq - sed)
                    const double ke_b = cdiff_b * (ceq - sed);
                    const double ceq_b = cdiff_b * ke;
                    sed_b -= cdiff_b * ke;
                    pb_kr += ke_b * kw;
                    if (!(tb & PGE_TB_CEQ_ZERO)) {  // ceq = ker dh (1 + k_disc qe)
                        const double P1 = 1.0 + p.k_disc * qe;
                        const double ker_b = ceq_b * dh * P1;
                        dh_b += ceq_b * ker * P1;
                        const double qe_b = ceq_b * ker * dh * p.k_disc;
                        pb_ke += ker_b * E;
                        if (a.ebar) {
                            const double v = ker_b * p.erodibility;
                            if (v != 0.0) atomicAdd(a.ebar + cc, v);
                        }
                        if (inv_sat > 0.0 && !(tb & PGE_TB_Q_ZERO)) {
                            const double z = q * inv_sat;
                            double dq = 0.0;
                            if (p.disc_exponent == 0.5) dq = qe > 0.0 ? 0.5 * inv_sat / qe : 0.0;
                            else if (p.disc_exponent > 0.0) dq = z > 0.0 ? p.disc_exponent * pow(z, p.disc_exponent - 1.0) * inv_sat : 0.0;
                            else dq = 1.1283791670955126 * exp(-z * z) * inv_sat;  // d erf / dz = 2 / sqrt(pi) exp(-z^2)
                            q_b += qe_b * dq;
                        }
                    }
                }
                q_b += kexp_b * p.conc_scale;
            } else if (tb & PGE_TB_SEA) {
                if (tb & PGE_TB_CLAMP) {  // cdiff = -room / vr
                    const double room_b = -cdiff_b / vr;
                    vr_b += cdiff_b * room / (vr * vr);
                    const int ss = (tb >> PGE_TB_SEA_SHIFT) & 3;
                    if (ss == 0 && !(tb & PGE_TB_ROOM_FLOOR) && pc >= 0) {
                        zadd(a, pc, room_b);
                        zadd(a, cc, -room_b);
                    } else if (ss == 1) {
                        zadd(a, cc, -room_b);
                    }
                } else {
                    sed_b += -p.ocean_rate * cdiff_b;
                }
            }
            // dh = h0 - max(h1, base)
            const double h0_b = dh_b;
            const double h1_b = (tb & PGE_TB_H1_ABOVE) ? -dh_b : 0.0;
            // h1: bilinear at the new position
            double nxo_b = xb, nyo_b = yb;
            if (h1_b != 0.0) {
                zadd(a, ns_.c00, h1_b * (1.0 - ns_.wi) * (1.0 - ns_.wj));
                zadd(a, ns_.c00 + NE, h1_b * ns_.wi * (1.0 - ns_.wj));
                zadd(a, ns_.c00 + 1, h1_b * (1.0 - ns_.wi) * ns_.wj);
                zadd(a, ns_.c00 + NE + 1, h1_b * ns_.wi * ns_.wj);
                const double N00 = ns_.s00.x, N10 = ns_.s10.x, N01 = ns_.s01.x, N11 = ns_.s11.x;
                if (!ns_.ci) nxo_b += h1_b * ((N10 - N00) * (1.0 - ns_.wj) + (N11 - N01) * ns_.wj);
                if (!ns_.cj) nyo_b += h1_b * ((N01 - N00) * (1.0 - ns_.wi) + (N11 - N10) * ns_.wi);
            }
            // the move and the face transfer: (nx, ny, a, b)_out = T(x + a4, y + b4, a4, b4)
            if (tb & PGE_TB_X_CLAMP) nxo_b = 0.0;
            if (tb & PGE_TB_Y_CLAMP) nyo_b = 0.0;
            double nxi_b = nxo_b, nyi_b = nyo_b, sa4_b = sab, sb4_b = sbb;
            if ((tb & PGE_TB_CROSS) && !(tb & PGE_TB_SAME_FACE)) {
                const double Nf = (double)N;
                D4 u = mk((x + sa4) / Nf), v = mk((y + sb4) / Nf), da = mk(sa4), db = mk(sb4);
                u.d[0] = 1.0 / Nf;
                v.d[1] = 1.0 / Nf;
                da.d[2] = 1.0;
                db.d[3] = 1.0;
                transfer_dual(f, fn, u, v, da, db);
                // rows: nx_out = N u', ny_out = N v', a', b'
                nxi_b = nxo_b * Nf * u.d[0] + nyo_b * Nf * v.d[0] + sab * da.d[0] + sbb * db.d[0];
                nyi_b = nxo_b * Nf * u.d[1] + nyo_b * Nf * v.d[1] + sab * da.d[1] + sbb * db.d[1];
                sa4_b = nxo_b * Nf * u.d[2] + nyo_b * Nf * v.d[2] + sab * da.d[2] + sbb * db.d[2];
                sb4_b = nxo_b * Nf * u.d[3] + nyo_b * Nf * v.d[3] + sab * da.d[3] + sbb * db.d[3];
            }
            x_b += nxi_b;
            y_b += nyi_b;
            sa4_b += nxi_b;
            sb4_b += nyi_b;
            // normalisation in the metric: a4 = a3 / |a3|_G
            const double t = sa4_b * sa4 + sb4_b * sb4;
            const double sa3_b = (sa4_b - (G0 * sa4 + G1 * sb4) * t) / slen3;
            const double sb3_b = (sb4_b - (G1 * sa4 + G2 * sb4) * t) / slen3;
            // gravity: a3 = a2 + accel n
            const double accel_b = sa3_b * na + sb3_b * nb;
            const double na_b = sa3_b * accel, nb_b = sb3_b * accel;
            vr_b += -accel_b * accel / vr;
            // momentum pull: a2 = a1 + kk m
            double sa1_b = sa3_b, sb1_b = sb3_b, ma_b = 0.0, mb_b = 0.0;
            if (tb & PGE_TB_MOM) {
                const double kk_b = sa3_b * ma + sb3_b * mb;
                ma_b += sa3_b * kk;
                mb_b += sb3_b * kk;
                const double cos_b = kk_b * p.k_mom * p.mom_scale / den;
                const double den_b = -kk_b * kk / den;
                vol_b += den_b;
                q_b += den_b * p.mom_scale;
                const double dot_b = cos_b / (mlen * slen1);
                const double mlen_b = -cos_b * cosang / mlen, slen1_b = -cos_b * cosang / slen1;
                ma_b += dot_b * (G0 * sa1 + G1 * sb1) + mlen_b * (G0 * ma + G1 * mb) / mlen;
                mb_b += dot_b * (G1 * sa1 + G2 * sb1) + mlen_b * (G1 * ma + G2 * mb) / mlen;
                sa1_b += dot_b * (G0 * ma + G1 * mb) + slen1_b * (G0 * sa1 + G1 * sb1) / slen1;
                sb1_b += dot_b * (G1 * ma + G2 * mb) + slen1_b * (G1 * sa1 + G2 * sb1) / slen1;
            }
            // friction: a1 = a fr
            sa_b += sa1_b * fr;
            sb_b += sb1_b * fr;
            if (!(tb & PGE_TB_FR_ZERO)) pb_fr += -(sa1_b * sa0 + sb1_b * sb0) * p.dt;
            vol_b += vr_b / V0;
            // slope direction: n = -(Q g) nrm, nrm = gain / sqrt(s2 + c)
            double di_b = -na_b * nrm, dj_b = -nb_b * nrm;
            const double nrm_b = -(na_b * di + nb_b * dj);
            double gi_b = 0.0, gj_b = 0.0;
            if (!(tb & PGE_TB_S2_ZERO)) {
                const double s2_b = nrm_b * (-0.5) * nrm / (s2 + csat);
                gi_b += s2_b * di;
                di_b += s2_b * gi;
                gj_b += s2_b * dj;
                dj_b += s2_b * gj;
            }
            gi_b += di_b * Q0 + dj_b * Q1;
            gj_b += di_b * Q1 + dj_b * Q2;
            // the stencil: surface corners and the weights
            const double X = H00 - H01 - H10 + H11;
            zadd(a, cs.c00, h0_b * (1.0 - wi) * (1.0 - wj) - gi_b * (1.0 - wj) - gj_b * (1.0 - wi));
            zadd(a, cs.c00 + NE, h0_b * wi * (1.0 - wj) + gi_b * (1.0 - wj) - gj_b * wi);
            zadd(a, cs.c00 + 1, h0_b * (1.0 - wi) * wj - gi_b * wj + gj_b * (1.0 - wi));
            zadd(a, cs.c00 + NE + 1, h0_b * wi * wj + gi_b * wj + gj_b * wi);
            if (a.carry_path) {
                double wi_b = h0_b * gi + gj_b * X, wj_b = h0_b * gj + gi_b * X;
                wi_b += ma_b * (((double)cs.s10.z - cs.s00.z) * (1.0 - wj) + ((double)cs.s11.z - cs.s01.z) * wj) +
                        mb_b * (((double)cs.s10.w - cs.s00.w) * (1.0 - wj) + ((double)cs.s11.w - cs.s01.w) * wj);
                wj_b += ma_b * (((double)cs.s01.z - cs.s00.z) * (1.0 - wi) + ((double)cs.s11.z - cs.s10.z) * wi) +
                        mb_b * (((double)cs.s01.w - cs.s00.w) * (1.0 - wi) + ((double)cs.s11.w - cs.s10.w) * wi);
                if (!(tb & PGE_TB_Q_ZERO)) {
                    wi_b += q_b * (((double)cs.s10.y - cs.s00.y) * (1.0 - wj) + ((double)cs.s11.y - cs.s01.y) * wj);
                    wj_b += q_b * (((double)cs.s01.y - cs.s00.y) * (1.0 - wi) + ((double)cs.s11.y - cs.s10.y) * wi);
                }
                if (!cs.ci) x_b += wi_b;
                if (!cs.cj) y_b += wj_b;
                xb = x_b;
                yb = y_b;
                sab = sa_b;
                sbb = sb_b;
            }  // else: the incoming position and direction are held fixed
            sedb = sed_b;
            volb = vol_b;
            xn = x;
            yn = y;
            fn = f;
        }
        if (j >= 0) atomicOr(a.error, 4);  // entries left over: the tape and the steps disagree
    }
    // the rates' gradients: warp sums, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        pb_ke += __shfl_down_sync(0xffffffffu, pb_ke, o);
        pb_kr += __shfl_down_sync(0xffffffffu, pb_kr, o);
        pb_kv += __shfl_down_sync(0xffffffffu, pb_kv, o);
        pb_fr += __shfl_down_sync(0xffffffffu, pb_fr, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (pb_ke != 0.0) atomicAdd(a.pbar + 0, pb_ke);
        if (pb_kr != 0.0) atomicAdd(a.pbar + 1, pb_kr);
        if (pb_kv != 0.0) atomicAdd(a.pbar + 2, pb_kv);
        if (pb_fr != 0.0) atomicAdd(a.pbar + 3, pb_fr);
    }
}

__global__ void copy_kernel(long long n, const double *__restrict__ in, double *out)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        out[c] = in[c];
}

// mu += zeta; zeta = 0 (a wave's terrain adjoint joins the running one)
__global__ void gather_wave_kernel(long long n, double *mu, double *zeta)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const double z = zeta[c];
        if (z != 0.0) {
            mu[c] += z;
            zeta[c] = 0.0;
        }
    }
}

__global__ void halo_adjoint_kernel(long long K, const int32_t *dst, const int32_t *src, const double *w, double *zb)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < K; k += (long long)gridDim.x * blockDim.x) {
        const double g = zb[dst[k]];
        zb[dst[k]] = 0.0;
        if (g == 0.0) continue;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const double v = w[16 * k + q] * g;
            if (v != 0.0) atomicAdd(zb + src[16 * k + q], v);
        }
    }
}

__global__ void error_to_stats_kernel(const int *error, PgeStats *stats)
{
    if (*error) stats->errors = *error;
}

int blocks_for(long long n, int threads)
{
    const long long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 1048576 ? 1048576 : b));
}

}  // namespace adj

cudaError_t adjoint_pass(const PgeGrid &g, const PgeState &s, const PgeSpawns &sp, const PgeParams &p, const PgeTape &tape,
                         int carry_path, const double *zbar_after, double *zbar_before, double *ebar, double *pbar,
                         const Layout &lay, void *ws, cudaStream_t st)
{
    // the running adjoint mu (dL/d of the terrain after the waves not yet reversed) lives in zbar_before; each
    // wave's own terrain adjoint collects in zeta (the thermal scratch) and joins mu after the wave
    pack(g, s, lay, ws, st);
    adj::copy_kernel<<<adj::blocks_for(lay.ncell, 256), 256, 0, st>>>(lay.ncell, zbar_after, zbar_before);
    double *zeta = ws_ptr<double>(ws, lay.thermal);
    int *err = ws_ptr<int>(ws, lay.error);
    cudaError_t e = cudaMemsetAsync(err, 0, 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(zeta, 0, 8 * lay.ncell, st);
    if (e != cudaSuccess) return e;
    adj::AdjArgs a{};
    a.F = g.F;
    a.N = g.N;
    a.H = g.H;
    a.NE = g.N + 2 * g.H;
    a.metric_shared = g.metric_shared;
    a.carry_path = carry_path ? 1 : 0;
    a.A = ws_ptr<float4>(ws, lay.cellA);
    a.B = ws_ptr<float4>(ws, lay.cellB);
    a.G = ws_ptr<float4>(ws, lay.metric8);
    a.erod = s.erodibility;
    a.p = p;
    a.volume0 = sp.volume0;
    a.tape = tape;
    a.zbar_after = zbar_before;  // mu
    a.zbar_before = zeta;
    a.ebar = ebar;
    a.pbar = pbar;
    a.error = err;
    const long long P = sp.count, wave = p.wave;
    const long long nw = (P + wave - 1) / wave;
    long long *acc = ws_ptr<long long>(ws, lay.acc4);
    for (long long w = nw - 1; w >= 0; w--) {
        // the terrain wave w saw: its start accumulator, refreshed into the packed samples
        e = cudaMemcpy2DAsync(acc, 4 * sizeof(long long), tape.wave_acc + w * lay.ncell, sizeof(long long), sizeof(long long),
                              lay.ncell, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        refresh(s, lay, ws, st);
        a.d0 = w * wave;
        a.d1 = a.d0 + wave < P ? a.d0 + wave : P;
        adj::adjoint_kernel<<<adj::blocks_for(a.d1 - a.d0, 128), 128, 0, st>>>(a);
        adj::gather_wave_kernel<<<adj::blocks_for(lay.ncell, 256), 256, 0, st>>>(lay.ncell, zbar_before, zeta);
    }
    return cudaPeekAtLastError();
}

void adjoint_errors(const Layout &lay, void *ws, PgeStats *stats, cudaStream_t st)
{
    if (stats) adj::error_to_stats_kernel<<<1, 1, 0, st>>>(ws_ptr<int>(ws, lay.error), stats);
}

void halo_adjoint(const PgeHalo &h, double *zbar, cudaStream_t st)
{
    if (h.K > 0) adj::halo_adjoint_kernel<<<adj::blocks_for(h.K, 256), 256, 0, st>>>(h.K, h.dst, h.src, h.w, zbar);
}

}  // namespace pge
