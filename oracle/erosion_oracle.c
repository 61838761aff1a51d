/*
 * erosion_oracle.c -- CPU restatement of the bake's particle-erosion path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA library is
 * checked against: tests, the smoke check and the benchmark's CPU baseline
 * may load it; the product never does.
 *
 * It restates, in plain C with the same float64 arithmetic and evaluation
 * order, the reference's numba kernels (paths within the bake project):
 *
 *   cubesphere.to_sphere / from_sphere / jacobian / transfer_vector /
 *   transfer_velocity                    bake/globe/cubesphere.py:70-220
 *   particle.pack_samples                bake/globe/erosion/particle.py:164-191
 *   particle._clamp_ij/_sbilin/_sbilin_grad/_snorm/_sdot
 *                                        particle.py:108-252
 *   particle.trace_particles             particle.py:275-818
 *   particle.apply_changes               particle.py:821-1042
 *   particle.slope_erode_cap             particle.py:1045-1076
 *   particle.fold_changes                particle.py:1079-1101
 *   particle.thermal_pass_a/r/b          particle.py:1107-1227
 *   particle.ema_update                  particle.py:1230-1242
 *   particle.spawn_cells                 particle.py:1245-1260
 *
 * Scope: the plain path with or without the routing surface (particles steer
 * on it where it stands above the terrain) and with or without overflowing
 * lakes flagged by the caller (crossing without exchange, the load dropped at
 * the shore, the bed kept at the water level; no lake parks), with or
 * without roots (the exchange scaled by 1 - roots), with or without the
 * bank cut on the outside of bends (erosion.lateral_rate); masks 0/1/2, windows (spherical = 0) and
 * deposit-on-exit are supported.  Numba types the packed samples as float32 and so computes
 * the stencil differences of _sbilin_grad in float32; the change list keeps
 * volumes and momenta as float32.  Both are mirrored here.
 *
 * Build with -ffp-contract=off (no fused multiply-add), so every operation
 * rounds like the numba/LLVM code it restates.  The trace is parallel over
 * particles on a pthread pool with dynamic scheduling (like numba's prange
 * under parallel_chunksize); the apply is serial.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SPREAD 8
#define LAKE_PARKS 8

enum { MASK_OUTSIDE = 0, MASK_ACTIVE = 1, MASK_FROZEN = 2 };
enum { DEATH_AGE = 0, DEATH_OCEAN = 1, DEATH_EXIT = 2, DEATH_PIT = 3, DEATH_EVAP = 4, DEATH_STOP = 5 };
enum {
    S_SURF = 0, S_ROUTE = 1, S_DISCH = 2, S_MOMA = 3, S_MOMB = 4, S_EVAP = 5, S_HARD = 6, S_SED = 7,
    S_G = 8, S_GINV = 11, S_RFLAG = 14, S_BASE = 15, NS = 16
};

static const double BASES[6][3][3] = {
    {{0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}, {1.0, 0.0, 0.0}},
    {{0.0, 0.0, 1.0}, {0.0, -1.0, 0.0}, {-1.0, 0.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, 1.0}, {0.0, 1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, 0.0, -1.0}, {0.0, -1.0, 0.0}},
    {{1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, 1.0}},
    {{-1.0, 0.0, 0.0}, {0.0, -1.0, 0.0}, {0.0, 0.0, -1.0}},
};
static const double PI_ = 3.14159265358979323846;
#define HALF_PI (PI_ / 2.0)
#define TWO_OVER_PI (2.0 / PI_)

/* ------------------------------------------------------------------------ */
/* geometry (cubesphere.py:70-220)                                          */
/* ------------------------------------------------------------------------ */
void orc_to_sphere(int face, double u, double v, double *out)
{
    const double *r = BASES[face][0], *up = BASES[face][1], *n = BASES[face][2];
    double s = tan((u - 0.5) * HALF_PI);
    double t = tan((v - 0.5) * HALF_PI);
    double x = n[0] + s * r[0] + t * up[0];
    double y = n[1] + s * r[1] + t * up[1];
    double z = n[2] + s * r[2] + t * up[2];
    double inv = 1.0 / sqrt(x * x + y * y + z * z);
    out[0] = x * inv;
    out[1] = y * inv;
    out[2] = z * inv;
}

static int face_of(double x, double y, double z)
{
    double ax = fabs(x), ay = fabs(y), az = fabs(z);
    if (ax >= ay && ax >= az) return x >= 0.0 ? 0 : 1;
    if (ay >= az) return y >= 0.0 ? 2 : 3;
    return z >= 0.0 ? 4 : 5;
}

int orc_from_sphere(double x, double y, double z, double *u, double *v)
{
    int face = face_of(x, y, z);
    const double *r = BASES[face][0], *up = BASES[face][1], *n = BASES[face][2];
    double d = x * n[0] + y * n[1] + z * n[2];
    double s = (x * r[0] + y * r[1] + z * r[2]) / d;
    double t = (x * up[0] + y * up[1] + z * up[2]) / d;
    *u = atan(s) * TWO_OVER_PI + 0.5;
    *v = atan(t) * TWO_OVER_PI + 0.5;
    return face;
}

static void jacobian(int face, double u, double v, double *J)
{
    const double *r = BASES[face][0], *up = BASES[face][1], *n = BASES[face][2];
    double a = (u - 0.5) * HALF_PI, b = (v - 0.5) * HALF_PI;
    double s = tan(a), t = tan(b);
    double dsdu = HALF_PI * (1.0 + s * s);
    double dtdv = HALF_PI * (1.0 + t * t);
    double qx = n[0] + s * r[0] + t * up[0];
    double qy = n[1] + s * r[1] + t * up[1];
    double qz = n[2] + s * r[2] + t * up[2];
    double ql = sqrt(qx * qx + qy * qy + qz * qz);
    double px = qx / ql, py = qy / ql, pz = qz / ql;
    double dux = r[0] * dsdu, duy = r[1] * dsdu, duz = r[2] * dsdu;
    double pd = px * dux + py * duy + pz * duz;
    J[0] = (dux - px * pd) / ql;
    J[1] = (duy - py * pd) / ql;
    J[2] = (duz - pz * pd) / ql;
    double dvx = up[0] * dtdv, dvy = up[1] * dtdv, dvz = up[2] * dtdv;
    pd = px * dvx + py * dvy + pz * dvz;
    J[3] = (dvx - px * pd) / ql;
    J[4] = (dvy - py * pd) / ql;
    J[5] = (dvz - pz * pd) / ql;
}

static void transfer_vector(int fs, double us, double vs, double a, double b, int fd, double ud, double vd,
                            double *a2, double *b2)
{
    double J[6], K[6];
    jacobian(fs, us, vs, J);
    double wx = a * J[0] + b * J[3];
    double wy = a * J[1] + b * J[4];
    double wz = a * J[2] + b * J[5];
    jacobian(fd, ud, vd, K);
    double guu = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
    double guv = K[0] * K[3] + K[1] * K[4] + K[2] * K[5];
    double gvv = K[3] * K[3] + K[4] * K[4] + K[5] * K[5];
    double ru = K[0] * wx + K[1] * wy + K[2] * wz;
    double rv = K[3] * wx + K[4] * wy + K[5] * wz;
    double det = guu * gvv - guv * guv;
    *a2 = (gvv * ru - guv * rv) / det;
    *b2 = (guu * rv - guv * ru) / det;
}

int orc_transfer_velocity(int face, double u, double v, double a, double b, double *out)
{
    /* out = (u2, v2, a2, b2); returns the new face */
    if (u >= 0.0 && u < 1.0 && v >= 0.0 && v < 1.0) {
        out[0] = u; out[1] = v; out[2] = a; out[3] = b;
        return face;
    }
    double p[3], u2, v2;
    orc_to_sphere(face, u, v, p);
    int f2 = orc_from_sphere(p[0], p[1], p[2], &u2, &v2);
    if (f2 == face) {
        double m = u2 < 0.0 ? 0.0 : u2;
        u2 = 0.999999999 < m ? 0.999999999 : m;
        m = v2 < 0.0 ? 0.0 : v2;
        v2 = 0.999999999 < m ? 0.999999999 : m;
        out[0] = u2; out[1] = v2; out[2] = a; out[3] = b;
        return face;
    }
    transfer_vector(face, u, v, a, b, f2, u2, v2, &out[2], &out[3]);
    out[0] = u2; out[1] = v2;
    return f2;
}

/* batch wrappers for the golden-vector tests */
void orc_to_sphere_batch(int64_t n, const int32_t *face, const double *u, const double *v, double *xyz)
{
    for (int64_t k = 0; k < n; k++) orc_to_sphere(face[k], u[k], v[k], xyz + 3 * k);
}

void orc_from_sphere_batch(int64_t n, const double *xyz, int32_t *face, double *u, double *v)
{
    for (int64_t k = 0; k < n; k++) face[k] = orc_from_sphere(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], u + k, v + k);
}

void orc_transfer_velocity_batch(int64_t n, const int32_t *face, const double *uvab, int32_t *face2, double *out)
{
    for (int64_t k = 0; k < n; k++)
        face2[k] = orc_transfer_velocity(face[k], uvab[4 * k], uvab[4 * k + 1], uvab[4 * k + 2], uvab[4 * k + 3], out + 4 * k);
}

/* ------------------------------------------------------------------------ */
/* packed samples (particle.py:164-191), plain path: route = surface        */
/* ------------------------------------------------------------------------ */
void orc_pack(int64_t ncell, float *samp, const double *height, const double *sediment, const double *discharge,
              const double *momentum, const float *evap, const float *hardness, const float *metric,
              const float *metric_inv, const double *base, const double *route, const uint8_t *lake_flag)
{
    for (int64_t c = 0; c < ncell; c++) {
        float *s = samp + NS * c;
        double sd = sediment[c];
        double surf = height[c] + sd;
        s[S_SURF] = (float)surf;
        s[S_ROUTE] = (float)(route ? route[c] : surf);
        s[S_DISCH] = (float)discharge[c];
        s[S_MOMA] = (float)momentum[2 * c];
        s[S_MOMB] = (float)momentum[2 * c + 1];
        s[S_EVAP] = evap[c];
        s[S_HARD] = hardness[c];
        s[S_SED] = (float)sd;
        for (int k = 0; k < 3; k++) {
            s[S_G + k] = metric[3 * c + k];
            s[S_GINV + k] = metric_inv[3 * c + k];
        }
        /* 2 on an overflowing lake, 3 on one with room for its rivers' load, else 1 where the routing
           surface differs from the terrain (particle.py:186-190) */
        if (route && lake_flag && lake_flag[c] > 0)
            s[S_RFLAG] = lake_flag[c] > 1 ? 3.0f : 2.0f;
        else
            s[S_RFLAG] = (route && s[S_ROUTE] != s[S_SURF]) ? 1.0f : 0.0f;
        s[S_BASE] = (float)base[c];
    }
}

/* ------------------------------------------------------------------------ */
/* sampling helpers (particle.py:108-252)                                   */
/* ------------------------------------------------------------------------ */
typedef struct { const float *samp; int NE; } Samp;

static inline const float *cellp(const Samp *S, int f, int i, int j)
{
    return S->samp + ((int64_t)((int64_t)f * S->NE + i) * S->NE + j) * NS;
}

static inline void clamp_ij(double fi, double fj, int NE, int *i0, int *j0, double *wi, double *wj)
{
    int a = (int)floor(fi), b = (int)floor(fj);
    if (a < 0) a = 0;
    if (a > NE - 2) a = NE - 2;
    if (b < 0) b = 0;
    if (b > NE - 2) b = NE - 2;
    double x = fi - a, y = fj - b;
    if (x < 0.0) x = 0.0;
    if (x > 1.0) x = 1.0;
    if (y < 0.0) y = 0.0;
    if (y > 1.0) y = 1.0;
    *i0 = a; *j0 = b; *wi = x; *wj = y;
}

static inline double sbilin(const Samp *S, int f, double fi, double fj, int c)
{
    int i0, j0;
    double wi, wj;
    clamp_ij(fi, fj, S->NE, &i0, &j0, &wi, &wj);
    double h00 = cellp(S, f, i0, j0)[c], h10 = cellp(S, f, i0 + 1, j0)[c];
    double h01 = cellp(S, f, i0, j0 + 1)[c], h11 = cellp(S, f, i0 + 1, j0 + 1)[c];
    return h00 * (1.0 - wi) * (1.0 - wj) + h10 * wi * (1.0 - wj) + h01 * (1.0 - wi) * wj + h11 * wi * wj;
}

static inline void sbilin_grad(const Samp *S, int f, double fi, double fj, int c, double *val, double *gi, double *gj)
{
    int i0, j0;
    double wi, wj;
    clamp_ij(fi, fj, S->NE, &i0, &j0, &wi, &wj);
    float h00 = cellp(S, f, i0, j0)[c], h10 = cellp(S, f, i0 + 1, j0)[c];
    float h01 = cellp(S, f, i0, j0 + 1)[c], h11 = cellp(S, f, i0 + 1, j0 + 1)[c];
    *val = (double)h00 * (1.0 - wi) * (1.0 - wj) + (double)h10 * wi * (1.0 - wj) + (double)h01 * (1.0 - wi) * wj
         + (double)h11 * wi * wj;
    /* the stencil differences are float32 in the reference (float32 samples) */
    float d10 = h10 - h00, d11 = h11 - h01, d01 = h01 - h00, d1110 = h11 - h10;
    *gi = (double)d10 * (1.0 - wj) + (double)d11 * wj;
    *gj = (double)d01 * (1.0 - wi) + (double)d1110 * wi;
}

/* the routing surface differs from the terrain somewhere in the stencil (particle.py:228-233) */
static inline int rflag(const Samp *S, int f, double fi, double fj)
{
    int i0, j0;
    double wi, wj;
    clamp_ij(fi, fj, S->NE, &i0, &j0, &wi, &wj);
    float sum = cellp(S, f, i0, j0)[S_RFLAG] + cellp(S, f, i0 + 1, j0)[S_RFLAG];
    sum = sum + cellp(S, f, i0, j0 + 1)[S_RFLAG];
    sum = sum + cellp(S, f, i0 + 1, j0 + 1)[S_RFLAG];
    return sum != 0.0f;
}

static inline double snorm(const float *cp, double a, double b)
{
    double g0 = cp[S_G], g1 = cp[S_G + 1], g2 = cp[S_G + 2];
    double n2 = g0 * a * a + 2.0 * g1 * a * b + g2 * b * b;
    if (n2 < 0.0) n2 = 0.0;
    return sqrt(n2);
}

static inline double sdot(const float *cp, double a, double b, double c, double d)
{
    double g0 = cp[S_G], g1 = cp[S_G + 1], g2 = cp[S_G + 2];
    return g0 * a * c + g1 * (a * d + b * c) + g2 * b * d;
}

static inline int cell_of(double x, int N)
{
    int i = (int)floor(x);
    if (i < 0) i = 0;
    if (i > N - 1) i = N - 1;
    return i;
}

int orc_change_list_cap(int max_steps, int lateral)
{
    return (lateral ? 2 * max_steps : max_steps) + 2 * SPREAD + 1 + SPREAD + LAKE_PARKS;
}

/* ------------------------------------------------------------------------ */
/* trace (particle.py:275-818), plain path                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    double dt, density, friction, deposition_rate, evap_rate, k_mom, mom_scale, k_disc, disc_saturation,
        disc_exponent, slope_gain, slope_sat, erodibility, cover_depth, min_volume, max_erode, conc_scale,
        ocean_rate, fan_room, dep_floor, lake_trap, lateral_rate, lake_park;
    int32_t max_steps, pit_steps, ocean_steps, deposit_on_exit, N, H, spherical, F;
    int32_t use_route, pad;
    const float *roots; /* (F,NE,NE) the share of the exchange the plants hold back, or NULL */
} OrcTraceParams;

static void trace_one(const OrcTraceParams *P, const Samp *S, const uint8_t *mask, int f, double x, double y,
                      double sed, double dir, double volume0, int cap, int32_t *cl_cell, double *cl_delta,
                      float *cl_vol, float *cl_mom, int64_t *count, int64_t *lo_out, int64_t *hi_out,
                      int8_t *death)
{
    const int N = P->N, H = P->H, NE = N + 2 * H;
    const double Nf = (double)N;
    const double inv_sat = P->disc_saturation > 0.0 ? 1.0 / P->disc_saturation : 0.0;
    double vol = volume0, sa = 0.0, sb = 0.0;
    if (sed > 0.0) {
        sa = cos(dir);
        sb = sin(dir);
    }
    int n = 0, uphill = 0, nring = 0, rpos = 0, sea_steps = 0;
    int64_t lo = 2147483647, hi = -1;
    int32_t *ring = cl_cell + cap - SPREAD;
    double h_prev = -1e300;
    int exited = 0, in_sea = 0, cause = DEATH_AGE;
    int in_lake = 0; /* on an overflowing lake: crossing, no exchange with the bed (particle.py:417) */
    int parks = 0;   /* loads this droplet has left in lakes (at most LAKE_PARKS, particle.py:418) */
#define RECORD(CELL, DELTA, VOL, MA, MB)                                   \
    do {                                                                   \
        cl_cell[n] = (int32_t)(CELL);                                      \
        cl_delta[n] = (DELTA);                                             \
        cl_vol[n] = (float)(VOL);                                          \
        cl_mom[2 * n] = (float)(MA);                                       \
        cl_mom[2 * n + 1] = (float)(MB);                                   \
        n++;                                                               \
        if ((CELL) < lo) lo = (CELL);                                      \
        if ((CELL) > hi) hi = (CELL);                                      \
    } while (0)

    for (int step = 0; step < P->max_steps; step++) {
        int ei = cell_of(x, N) + H, ej = cell_of(y, N) + H;
        int64_t cidx = ((int64_t)f * NE + ei) * NE + ej;
        int m = mask[cidx];
        if (m == MASK_OUTSIDE) { exited = 1; cause = DEATH_EXIT; break; }
        const float *cp = S->samp + cidx * NS;
        float h_here = cp[S_SURF], b_here = cp[S_BASE];
        if (step == 0 && h_here < b_here) in_sea = 1;
        if (in_sea) {
            if (h_here >= b_here || sed * vol / volume0 < 1e-4 || sea_steps >= P->ocean_steps) { cause = DEATH_OCEAN; break; }
            sea_steps++;
        }
        if (m == MASK_ACTIVE) {
            ring[rpos] = (int32_t)cidx;
            rpos = (rpos + 1) % SPREAD;
            if (nring < SPREAD) nring++;
        }
        double fi = x - 0.5 + H, fj = y - 0.5 + H;
        double h0, gi, gj;
        sbilin_grad(S, f, fi, fj, S_SURF, &h0, &gi, &gj);
        double h0r = h0;
        if (P->use_route && rflag(S, f, fi, fj)) {
            /* steer on the routing surface where it is above the terrain (particle.py:453-460) */
            double r0, rgi, rgj;
            sbilin_grad(S, f, fi, fj, S_ROUTE, &r0, &rgi, &rgj);
            if (r0 > h0) {
                h0r = r0;
                gi = rgi;
                gj = rgj;
            }
        }
        double q0 = cp[S_GINV], q1 = cp[S_GINV + 1], q2 = cp[S_GINV + 2];
        double di = q0 * gi + q1 * gj;
        double dj = q1 * gi + q2 * gj;
        double s2 = gi * di + gj * dj;
        if (s2 < 0.0) s2 = 0.0;
        double nrm = P->slope_sat > 0.0 ? P->slope_gain / sqrt(s2 + P->slope_sat * P->slope_sat)
                                        : P->slope_gain / sqrt(1.0 + s2);
        double na = -di * nrm, nb = -dj * nrm;
        double ma = sbilin(S, f, fi, fj, S_MOMA);
        double mb = sbilin(S, f, fi, fj, S_MOMB);
        double q = sbilin(S, f, fi, fj, S_DISCH);
        if (q < 0.0) q = 0.0;
        double vol_rel = vol / volume0;
        const double psa = sa, psb = sb; /* the direction this step started with (the bend) */
        double fr = 1.0 - P->dt * P->friction;
        if (fr < 0.0) fr = 0.0;
        sa *= fr;
        sb *= fr;
        double mlen = snorm(cp, ma, mb);
        double slen = snorm(cp, sa, sb);
        if (mlen > 1e-12 && slen > 1e-12) {
            double cosang = sdot(cp, ma, mb, sa, sb) / (mlen * slen);
            double k = P->k_mom * cosang * P->mom_scale / (vol + P->mom_scale * q);
            sa += k * ma;
            sb += k * mb;
        }
        double acc = P->dt / (vol_rel * P->density);
        sa += acc * na;
        sb += acc * nb;
        slen = snorm(cp, sa, sb);
        if (slen < 1e-12) { cause = DEATH_STOP; break; }
        sa /= slen;
        sb /= slen;
        double nx = x + sa, ny = y + sb;
        int nf = f;
        if (P->spherical) {
            if (nx < 0.0 || nx >= Nf || ny < 0.0 || ny >= Nf) {
                double o[4];
                nf = orc_transfer_velocity(f, nx / Nf, ny / Nf, sa, sb, o);
                nx = o[0] * Nf;
                ny = o[1] * Nf;
                sa = o[2];
                sb = o[3];
                if (nx >= Nf) nx = Nf * 0.999999999;
                if (ny >= Nf) ny = Nf * 0.999999999;
                if (nx < 0.0) nx = 0.0;
                if (ny < 0.0) ny = 0.0;
            }
        } else if (nx < -H || nx >= Nf + H || ny < -H || ny >= Nf + H) {
            exited = 1; cause = DEATH_EXIT; break;
        }
        int nei = (int)floor(nx) + H, nej = (int)floor(ny) + H;
        if (nei < 0 || nei >= NE || nej < 0 || nej >= NE) { exited = 1; cause = DEATH_EXIT; break; }
        int64_t nidx = ((int64_t)nf * NE + nei) * NE + nej;
        if (mask[nidx] == MASK_OUTSIDE) { exited = 1; cause = DEATH_EXIT; break; }
        const float *np_ = S->samp + nidx * NS;
        double nfi = nx - 0.5 + H, nfj = ny - 0.5 + H;
        double h1 = sbilin(S, nf, nfi, nfj, S_SURF);
        double b1 = np_[S_BASE];
        double dh = h0 - (h1 > b1 ? h1 : b1);
        double h1r = h1;
        if (P->use_route && rflag(S, nf, nfi, nfj)) {
            double r1 = sbilin(S, nf, nfi, nfj, S_ROUTE);
            if (r1 > h1) h1r = r1;
        }
        double dhr = h0r - h1r;
        if (m == MASK_ACTIVE && in_sea) {
            double cdiff = -P->ocean_rate * sed;
            double room = h_prev > -1e300 ? h_prev - (double)h_here : P->fan_room;
            if (room < P->fan_room) room = P->fan_room;
            double lim = (double)b_here - P->dep_floor - (double)h_here;
            if (lim < room) room = lim;
            if (room < 0.0) room = 0.0;
            if (-cdiff * vol_rel > room) cdiff = -room / vol_rel;
            sed += cdiff;
            RECORD(cidx, -cdiff * vol_rel, 0.0, 0.0, 0.0);
        } else if (m == MASK_ACTIVE) {
            double qe;
            if (inv_sat <= 0.0) qe = 0.0;
            else if (P->disc_exponent == 0.5) qe = sqrt(q * inv_sat);
            else if (P->disc_exponent > 0.0) qe = pow(q * inv_sat, P->disc_exponent);
            else qe = erf(q * inv_sat);
            double c_eq = P->erodibility * dh * (1.0 + P->k_disc * qe);
            if (c_eq < 0.0) c_eq = 0.0;
            double k_e;
            if (c_eq > sed) {
                float sthick = cp[S_SED];
                double w_cover;
                if (P->cover_depth > 0.0) {
                    w_cover = (double)sthick / P->cover_depth;
                    if (w_cover > 1.0) w_cover = 1.0;
                } else {
                    w_cover = sthick > 0.0f ? 1.0 : 0.0;
                }
                k_e = P->deposition_rate * (w_cover + (1.0 - w_cover) * (1.0 - (double)cp[S_HARD]));
            } else {
                k_e = P->deposition_rate;
            }
            if (P->roots) k_e *= 1.0 - (double)P->roots[cidx]; /* roots hold the ground (particle.py:615-618) */
            double cdiff = k_e * (c_eq - sed);
            double trapped = 0.0;
            if (in_lake) {
                cdiff = 0.0; /* crossing a lake: the bed sees nothing (particle.py:626-629) */
            } else if (sed > 0.0 && np_[S_RFLAG] >= 1.5f) {
                double trap = -P->lake_trap * sed; /* entering a lake: the load drops at the shore (630-634) */
                if (trap < cdiff) cdiff = trap;
                if (np_[S_RFLAG] >= 2.5f) trapped = P->lake_trap * sed; /* ...and a lake with room keeps the rest */
            }
            double kexp = 1.0 + q * P->conc_scale;
            if (cdiff > 0.0) {
                double ecap = dh / kexp;
                if (ecap > P->max_erode) ecap = P->max_erode;
                if (ecap > h_here) ecap = h_here > 0.0f ? (double)h_here : 0.0;
                if (cdiff * vol_rel > ecap) cdiff = ecap / vol_rel;
            } else if (cdiff < 0.0) {
                double room = h_prev > -1e300 ? h_prev - (double)h_here : P->dep_floor;
                if (room < P->dep_floor) room = P->dep_floor;
                double dcap = room / kexp;
                if (-cdiff * vol_rel > dcap) cdiff = -dcap / vol_rel;
            }
            sed += cdiff;
            RECORD(cidx, -cdiff * vol_rel, vol, vol * sa, vol * sb);
            /* a lake keeps what its shore had no room for (particle.py:672-696): parked on the lake cell
               entered, an entry of volume -3 */
            if (P->lake_park > 0.0 && trapped > 0.0 && parks < LAKE_PARKS) {
                double rest = trapped + cdiff;
                if (rest > 0.0) {
                    parks++;
                    sed -= rest;
                    RECORD(nidx, rest * vol_rel, -3.0, 0.0, 0.0);
                }
            }
            /* the outside of the bend (particle.py:699-738): the bank one cell across the flow */
            if (P->lateral_rate > 0.0 && cdiff > 0.0 && n + 2 * SPREAD + 2 < cap) {
                double cross = psa * sb - psb * sa;
                double turn = cross > 0.0 ? cross : -cross;
                if (turn > 1e-6) {
                    double sgn = cross > 0.0 ? 1.0 : -1.0;
                    double bx = x + sgn * sb, by = y - sgn * sa;
                    int bei = (int)floor(bx) + H, bej = (int)floor(by) + H;
                    if (bei >= 0 && bei < NE && bej >= 0 && bej < NE) {
                        int64_t bcell = ((int64_t)f * NE + bei) * NE + bej;
                        if (mask[bcell] == MASK_ACTIVE) {
                            float bank = S->samp[bcell * NS + S_SURF] - h_here;
                            if (bank > 0.0f) {
                                double lat = P->lateral_rate * turn * cdiff;
                                double lcap = (double)bank / kexp;
                                if (lcap > P->max_erode) lcap = P->max_erode;
                                if (lat * vol_rel > lcap) lat = lcap / vol_rel;
                                if (lat > 0.0) {
                                    sed += lat;
                                    RECORD(bcell, -lat * vol_rel, -2.0, 0.0, 0.0);
                                }
                            }
                        }
                    }
                }
            }
        }
        double ev = 1.0 - P->dt * P->evap_rate * (double)cp[S_EVAP];
        if (ev < 0.01) ev = 0.01;
        vol *= ev;
        sed /= ev;
        x = nx;
        y = ny;
        f = nf;
        h_prev = h_here;
        in_lake = np_[S_RFLAG] >= 1.5f;
        if (np_[S_SURF] < np_[S_BASE] && !in_sea) {
            in_sea = 1;
            if (sed <= 0.0) { cause = DEATH_OCEAN; break; }
        }
        if (vol < P->min_volume) { cause = in_sea ? DEATH_OCEAN : DEATH_EVAP; break; }
        if (dhr < 0.0 && !in_lake) {
            uphill++;
            if (uphill > P->pit_steps) { cause = in_sea ? DEATH_OCEAN : DEATH_PIT; break; }
        } else {
            uphill = 0;
        }
    }
    if (in_sea && (cause == DEATH_AGE || cause == DEATH_STOP)) cause = DEATH_OCEAN;
    *death = (int8_t)cause;
    if (!exited) {
        int ei = cell_of(x, N) + H, ej = cell_of(y, N) + H;
        int64_t cidx = ((int64_t)f * NE + ei) * NE + ej;
        const float *cp = S->samp + cidx * NS;
        if (mask[cidx] == MASK_ACTIVE && !(in_sea && cp[S_SURF] >= cp[S_BASE])) {
            int newest = (rpos + SPREAD - 1) % SPREAD;
            if (nring == 0 || ring[newest] != (int32_t)cidx) {
                ring[rpos] = (int32_t)cidx;
                rpos = (rpos + 1) % SPREAD;
                if (nring < SPREAD) nring++;
            }
        }
    }
    if (sed > 0.0 && nring > 0 && (!exited || P->deposit_on_exit)) {
        double load = sed * vol / volume0;
        int nout = cause == DEATH_OCEAN ? 1 : nring;
        for (int r = 0; r < nout; r++) {
            int64_t c = ring[(rpos + SPREAD - 1 - r) % SPREAD];
            RECORD(c, r == 0 ? load : 0.0, -1.0, 0.0, 0.0);
        }
    }
#undef RECORD
    *count = n;
    *lo_out = lo;
    *hi_out = hi;
}

typedef struct {
    const OrcTraceParams *P;
    Samp S;
    const uint8_t *mask;
    const int64_t *sp_face;
    const double *sp_x, *sp_y, *sp_sed, *sp_dir;
    double volume0;
    int cap;
    int32_t *cl_cell;
    double *cl_delta;
    float *cl_vol, *cl_mom;
    int64_t *cl_count, *cl_lo, *cl_hi;
    int8_t *sp_death;
    int64_t np;
    int64_t next; /* shared work counter (chunks of 4 particles) */
} TraceJob;

static void *trace_worker(void *arg)
{
    TraceJob *J = (TraceJob *)arg;
    for (;;) {
        int64_t p0 = __atomic_fetch_add(&J->next, 4, __ATOMIC_RELAXED);
        if (p0 >= J->np) break;
        int64_t p1 = p0 + 4 < J->np ? p0 + 4 : J->np;
        for (int64_t p = p0; p < p1; p++) {
            int64_t b = p * J->cap;
            trace_one(J->P, &J->S, J->mask, (int)J->sp_face[p], J->sp_x[p], J->sp_y[p], J->sp_sed[p], J->sp_dir[p],
                      J->volume0, J->cap, J->cl_cell + b, J->cl_delta + b, J->cl_vol + b, J->cl_mom + 2 * b,
                      J->cl_count + p, J->cl_lo + p, J->cl_hi + p, J->sp_death + p);
        }
    }
    return NULL;
}

static int g_threads = 1;

/* number of host threads the trace uses (>= 1) */
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }
int orc_get_threads(void) { return g_threads; }

void orc_trace(const OrcTraceParams *P, const float *samp, const uint8_t *mask, int64_t np, const int64_t *sp_face,
               const double *sp_x, const double *sp_y, const double *sp_sed, const double *sp_dir, double volume0,
               int32_t *cl_cell, double *cl_delta, float *cl_vol, float *cl_mom, int64_t *cl_count, int64_t *cl_lo,
               int64_t *cl_hi, int8_t *sp_death)
{
    TraceJob J = {P, {samp, P->N + 2 * P->H}, mask, sp_face, sp_x, sp_y, sp_sed, sp_dir, volume0,
                  orc_change_list_cap(P->max_steps, P->lateral_rate > 0.0), cl_cell, cl_delta, cl_vol, cl_mom, cl_count, cl_lo, cl_hi,
                  sp_death, np, 0};
    int nt = g_threads;
    if (nt > 1 && np > 64) {
        pthread_t th[256];
        int started = 0;
        for (int t = 1; t < nt; t++)
            if (pthread_create(&th[started], NULL, trace_worker, &J) == 0) started++;
        trace_worker(&J);
        for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    } else {
        trace_worker(&J);
    }
}

/* ------------------------------------------------------------------------ */
/* serial apply (particle.py:821-1042), plain path                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    double iter_erode, iter_deposit, fan_slope, dep_floor, offshore_writeoff;
    int32_t use_erode_cap, use_route;
} OrcApplyParams;

void orc_apply(const OrcApplyParams *A, const int32_t *cl_cell, const double *cl_delta, const float *cl_vol,
               const float *cl_mom, int64_t np, const int64_t *cl_count, int cap, const double *height,
               const double *sediment, double *acc, double *pending, float *samp, double *disch_track,
               double *mom_track, const uint8_t *mask, const double *erode_cap, double *out4, double *lake_load,
               const int32_t *lake_id, double *lake_room)
{
    int64_t n_clamp = 0;
    double to_pending = 0.0, lost = 0.0, lost_offshore = 0.0;
    for (int64_t p = 0; p < np; p++) {
        int64_t base = p * cap;
        int64_t cnt = cl_count[p];
        double deficit = 0.0, surplus = 0.0, refused = 0.0;
        int64_t prev = -1, death = -1;
        for (int64_t k = 0; k < cnt; k++) {
            int64_t c = cl_cell[base + k];
            if (cl_vol[base + k] == -3.0f) {
                /* a load for a lake to keep (particle.py:912-933): the lake takes what it still has room for,
                   counted down in particle order; the rest goes where the particle ends */
                double take = cl_delta[base + k], rest = 0.0;
                int32_t lk = lake_id ? lake_id[c] : -1;
                if (lk < 0) {
                    rest = take;
                    take = 0.0;
                } else if (take > lake_room[lk]) {
                    rest = take - lake_room[lk];
                    take = lake_room[lk];
                }
                if (take > 0.0) {
                    lake_load[c] += take;
                    lake_room[lk] -= take;
                }
                refused += rest;
                continue;
            }
            if (mask[c] != MASK_ACTIVE) continue;
            double d = cl_delta[base + k];
            float v = cl_vol[base + k];
            int is_step = v >= 0.0f;
            double s_c = height[c] + sediment[c] + acc[c];
            float b_c = samp[c * NS + S_BASE];
            if (d < 0.0) {
                double e = -d, e_act = e;
                double room = A->iter_erode + acc[c];
                if (A->use_erode_cap) {
                    double r2 = erode_cap[c] + acc[c];
                    if (r2 < room) room = r2;
                }
                if (e_act > room) e_act = room;
                double floor_ = s_c >= b_c ? (double)b_c : s_c;
                if (A->use_route && samp[c * NS + S_RFLAG] >= 1.5f) {
                    double r_c = samp[c * NS + S_ROUTE]; /* a lake bed is never eroded below its water level */
                    if (r_c > floor_) floor_ = r_c;
                }
                if (k + 1 < cnt) {
                    int64_t nc = cl_cell[base + k + 1];
                    double ns = height[nc] + sediment[nc] + acc[nc];
                    if (ns > floor_) floor_ = ns;
                }
                if (e_act > s_c - floor_) e_act = s_c - floor_;
                if (e_act < 0.0) e_act = 0.0;
                if (e_act < e) {
                    n_clamp++;
                    deficit += e - e_act;
                }
                acc[c] -= e_act;
            } else {
                double want = d + surplus;
                surplus = 0.0;
                if (deficit > 0.0) {
                    double a = want < deficit ? want : deficit;
                    want -= a;
                    deficit -= a;
                }
                double d_act = want;
                double room = A->iter_deposit - acc[c];
                if (d_act > room) d_act = room;
                int64_t ref = -1;
                if (is_step) ref = prev;
                else if (k + 1 < cnt) ref = cl_cell[base + k + 1];
                if (ref >= 0) {
                    double ceil_ = height[ref] + sediment[ref] + acc[ref] + A->dep_floor;
                    if (s_c < b_c && is_step) ceil_ -= A->dep_floor + A->fan_slope;
                    double lim = ceil_ - s_c;
                    if (d_act > lim) d_act = lim;
                }
                if (s_c < b_c) {
                    double lim = (double)b_c - A->dep_floor - s_c;
                    if (d_act > lim) d_act = lim;
                }
                if (d_act < 0.0) d_act = 0.0;
                if (d_act < want) n_clamp++;
                surplus = want - d_act;
                acc[c] += d_act;
                if (!is_step && death < 0) death = c;
            }
            double a2 = acc[c];
            double s_new = height[c] + sediment[c] + a2;
            samp[c * NS + S_SURF] = (float)s_new;
            double sd = sediment[c] + a2;
            samp[c * NS + S_SED] = (float)(sd > 0.0 ? sd : 0.0);
            if (A->use_route && samp[c * NS + S_RFLAG] < 1.5f)  /* the route flag follows the live surface */
                samp[c * NS + S_RFLAG] = samp[c * NS + S_ROUTE] != samp[c * NS + S_SURF] ? 1.0f : 0.0f;
            if (is_step) {
                if (v > 0.0f) {
                    disch_track[c] += (double)v;
                    mom_track[2 * c] += (double)cl_mom[2 * (base + k)];
                    mom_track[2 * c + 1] += (double)cl_mom[2 * (base + k) + 1];
                }
                prev = c;
            }
        }
        surplus += refused;
        if (surplus > 0.0 && death >= 0) {
            if (height[death] + sediment[death] + acc[death] < samp[death * NS + S_BASE]) {
                double keep = surplus * (1.0 - A->offshore_writeoff);
                if (keep < 1e-4) keep = 0.0;
                pending[death] += keep;
                to_pending += keep;
                lost_offshore += surplus - keep;
            } else {
                pending[death] += surplus;
                to_pending += surplus;
            }
        }
        lost += deficit;
    }
    out4[0] = (double)n_clamp;
    out4[1] = to_pending;
    out4[2] = lost;
    out4[3] = lost_offshore;
}

/* ------------------------------------------------------------------------ */
/* per-iteration map passes                                                 */
/* ------------------------------------------------------------------------ */
void orc_slope_erode_cap(int F, int NE, const double *height, const double *sediment, const uint8_t *mask,
                         double coef, double exit_slope, double *out)
{
    double k = coef * sqrt(2.0);
    for (int f = 0; f < F; f++)
        for (int i = 0; i < NE; i++)
            for (int j = 0; j < NE; j++) {
                int64_t c = ((int64_t)f * NE + i) * NE + j;
                if (mask[c] != MASK_ACTIVE) { out[c] = 0.0; continue; }
                double h = height[c] + sediment[c];
                double gxn = i == 0 ? exit_slope : h - (height[c - NE] + sediment[c - NE]);
                double gxp = i == NE - 1 ? exit_slope : h - (height[c + NE] + sediment[c + NE]);
                double gyn = j == 0 ? exit_slope : h - (height[c - 1] + sediment[c - 1]);
                double gyp = j == NE - 1 ? exit_slope : h - (height[c + 1] + sediment[c + 1]);
                double gx = gxn > gxp ? gxn : gxp;
                double gy = gyn > gyp ? gyn : gyp;
                if (gx < 0.0) gx = 0.0;
                if (gy < 0.0) gy = 0.0;
                out[c] = k * sqrt(gx * gx + gy * gy);
            }
}

void orc_fold(int64_t ncell, double *height, double *sediment, double *acc, const uint8_t *mask)
{
    for (int64_t c = 0; c < ncell; c++) {
        double a = acc[c];
        acc[c] = 0.0;
        if (a == 0.0 || mask[c] != MASK_ACTIVE) continue;
        if (a > 0.0) {
            sediment[c] += a;
        } else {
            double take = -a, s = sediment[c];
            if (s >= take) {
                sediment[c] = s - take;
            } else {
                height[c] -= take - s;
                sediment[c] = 0.0;
            }
        }
    }
}

void orc_ema(int64_t ncell, double *discharge, double *momentum, double *disch_track, double *mom_track,
             const uint8_t *mask, double ema)
{
    for (int64_t c = 0; c < ncell; c++) {
        if (mask[c] == MASK_ACTIVE) {
            discharge[c] = (1.0 - ema) * discharge[c] + ema * disch_track[c];
            momentum[2 * c] = (1.0 - ema) * momentum[2 * c] + ema * mom_track[2 * c];
            momentum[2 * c + 1] = (1.0 - ema) * momentum[2 * c + 1] + ema * mom_track[2 * c + 1];
        }
        disch_track[c] = 0.0;
        mom_track[2 * c] = 0.0;
        mom_track[2 * c + 1] = 0.0;
    }
}

static const int D8[8][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 1}, {-1, 0}, {-1, -1}, {0, -1}, {1, -1}};

static inline double thermal_out(const double *h, const double *s, const float *metric, const double *talus,
                                 int64_t c, int NE, int k, double rate)
{
    int di = D8[k][0], dj = D8[k][1];
    int64_t nc = c + (int64_t)di * NE + dj;
    double d = (h[c] + s[c]) - (h[nc] + s[nc]);
    if (d <= 0.0) return 0.0;
    double g0 = metric[3 * c], g1 = metric[3 * c + 1], g2 = metric[3 * c + 2];
    double dist = sqrt(g0 * di * di + 2.0 * g1 * di * dj + g2 * dj * dj);
    double ex = d - talus[c] * dist;
    if (ex <= 0.0) return 0.0;
    return 0.5 * rate * ex;
}

/* one mass-wasting pass (maps.py:1074-1085 over particle.py:1127-1227);
 * out_total/scale/rscale are caller scratch (F*NE*NE doubles each) */
void orc_mass_wasting(int F, int NE, double *height, double *sediment, const float *metric, const double *talus,
                      const uint8_t *mask, double rate, double cap, double dep_floor, double *out_total,
                      double *scale, double *rscale, double *new_h, double *new_s)
{
    int64_t total = (int64_t)F * NE * NE;
    for (int64_t c = 0; c < total; c++) { out_total[c] = 0.0; scale[c] = 0.0; rscale[c] = 1.0; }
    for (int f = 0; f < F; f++)
        for (int i = 1; i < NE - 1; i++)
            for (int j = 1; j < NE - 1; j++) {
                int64_t c = ((int64_t)f * NE + i) * NE + j;
                out_total[c] = 0.0;
                scale[c] = 0.0;
                if (mask[c] != MASK_ACTIVE) continue;
                double S = 0.0, mx = 0.0;
                for (int k = 0; k < 8; k++) {
                    if (mask[c + (int64_t)D8[k][0] * NE + D8[k][1]] != MASK_ACTIVE) continue;
                    double o = thermal_out(height, sediment, metric, talus, c, NE, k, rate);
                    S += o;
                    if (o > mx) mx = o;
                }
                if (S <= 0.0) continue;
                double sc = 1.0;
                if (S > 2.0 * mx) sc = 2.0 * mx / S;
                if (cap > 0.0 && S * sc > cap) sc = cap / S;
                out_total[c] = S * sc;
                scale[c] = sc;
            }
    for (int f = 0; f < F; f++)
        for (int i = 1; i < NE - 1; i++)
            for (int j = 1; j < NE - 1; j++) {
                int64_t c = ((int64_t)f * NE + i) * NE + j;
                rscale[c] = 1.0;
                double surf = height[c] + sediment[c];
                if (surf >= 0.0 || mask[c] != MASK_ACTIVE) continue;
                double inflow = 0.0;
                for (int k = 0; k < 8; k++) {
                    int64_t nc = c + (int64_t)D8[k][0] * NE + D8[k][1];
                    double sc = scale[nc];
                    if (sc <= 0.0 || mask[nc] == MASK_OUTSIDE) continue;
                    inflow += sc * thermal_out(height, sediment, metric, talus, nc, NE, (k + 4) % 8, rate);
                }
                double room = -dep_floor - surf;
                if (room < 0.0) room = 0.0;
                if (inflow > room) rscale[c] = room / inflow;
            }
    memcpy(new_h, height, sizeof(double) * total);
    memcpy(new_s, sediment, sizeof(double) * total);
    for (int f = 0; f < F; f++)
        for (int i = 1; i < NE - 1; i++)
            for (int j = 1; j < NE - 1; j++) {
                int64_t c = ((int64_t)f * NE + i) * NE + j;
                double h = height[c], s = sediment[c];
                if (mask[c] != MASK_ACTIVE) { new_h[c] = h; new_s[c] = s; continue; }
                double inflow = 0.0, out = 0.0, sc_self = scale[c];
                for (int k = 0; k < 8; k++) {
                    int64_t nc = c + (int64_t)D8[k][0] * NE + D8[k][1];
                    if (mask[nc] == MASK_OUTSIDE) continue;
                    if (sc_self > 0.0 && mask[nc] == MASK_ACTIVE)
                        out += sc_self * rscale[nc] * thermal_out(height, sediment, metric, talus, c, NE, k, rate);
                    double sc = scale[nc];
                    if (sc <= 0.0) continue;
                    inflow += sc * thermal_out(height, sediment, metric, talus, nc, NE, (k + 4) % 8, rate);
                }
                inflow *= rscale[c];
                if (out > 0.0) {
                    if (s >= out) s -= out;
                    else { h -= out - s; s = 0.0; }
                }
                new_h[c] = h;
                new_s[c] = s + inflow;
            }
    memcpy(height, new_h, sizeof(double) * total);
    memcpy(sediment, new_s, sizeof(double) * total);
}

/* inverse-CDF spawn over sorted uniforms (particle.py:1245-1260) */
void orc_spawn_cells(int64_t M, const double *cdf, int64_t P, const double *u, int64_t *out)
{
    double total = cdf[M - 1];
    int64_t k = 0;
    for (int64_t p = 0; p < P; p++) {
        double target = u[p] * total;
        while (k < M - 1 && cdf[k] <= target) k++;
        out[p] = k;
    }
}

/* The C library's tan / atan / sin / cos (op 0..3) over an array: the values
 * the reference's numba code and this oracle's crossing compute, for checking
 * the library's own double-double versions against them. */
void orc_libm(int op, int64_t n, const double *x, double *y)
{
    for (int64_t i = 0; i < n; i++)
        y[i] = op == 0 ? tan(x[i]) : op == 1 ? atan(x[i]) : op == 2 ? sin(x[i]) : cos(x[i]);
}
