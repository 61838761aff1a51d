// pge_internal.cuh -- shared device-side definitions of libpgerosion.
//
// Packed per-iteration cell data (written by the pack kernel, frozen for the
// length of one wave, refreshed between waves):
//   cellA[c] = float4(surface, discharge, momentum_a, momentum_b)  -- read as
//              a 2x2 bilinear stencil every droplet step (one float4 per corner)
//   cellB[c] = float4(evap, hardness, sediment, base)              -- the cell's
//              own scalars
//   live[c]  = double2(height + sediment, net change at wave start) -- the
//              float64 terrain the ledger applies against
//   metric8  = two float4 per (face-shared) cell: (g_ii, g_ij, g_jj, ginv_ii),
//              (ginv_ij, ginv_jj, 0, 0)
//   route2[c] = float2(routing surface, flag: 1 where it differs from the
//              cell's packed surface) -- only when the state has a route
// These are the channels of the reference's packed float32 sample array
// (bake/globe/erosion/particle.py:146-191) split by access pattern.
//
// Accumulators (int64 fixed point, summed with integer atomics so a wave's
// result does not depend on thread order):
//   acc4[c] = (terrain change 2^-40, discharge track 2^-32, momentum a, b 2^-32)
//   pend[c] = stockpile 2^-40
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pgerosion.h"

namespace pge {

constexpr int SPREAD = 8;
constexpr int LAKE_PARKS = 8;
constexpr double FX_MASS = 1099511627776.0;  // 2^40
constexpr double FX_TRACK = 4294967296.0;    // 2^32
constexpr double INV_FX_MASS = 1.0 / FX_MASS;
constexpr double INV_FX_TRACK = 1.0 / FX_TRACK;

__host__ __device__ inline int change_list_cap(int max_steps) { return max_steps + 2 * SPREAD + 1 + SPREAD + LAKE_PARKS; }
// steps' worth of change-list room: two entries a step with the bank cut (particle.py:259-272)
__host__ __device__ inline int list_steps(const PgeParams &p) { return p.lateral_rate > 0.0 ? 2 * p.max_steps : p.max_steps; }
// distinct cells one droplet's ledger can change: one per step entry plus its final deposits
__host__ __device__ inline int ledger_table_cap(int max_steps) { return max_steps + SPREAD + 2; }
// hash slots per droplet thread: a power of two at least twice the table capacity
inline unsigned ledger_table_slots(int max_steps)
{
    unsigned s = 16;
    while (s < 2u * (unsigned)ledger_table_cap(max_steps)) s <<= 1;
    return s;
}

__device__ __forceinline__ long long fx_mass(double v) { return __double2ll_rn(v * FX_MASS); }
__device__ __forceinline__ long long fx_track(double v) { return __double2ll_rn(v * FX_TRACK); }
__device__ __forceinline__ void red_add(long long *p, long long v)
{
    atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// ---------------------------------------------------------------------------
// workspace layout
// ---------------------------------------------------------------------------
struct Layout {
    size_t cellA, cellB, live, metric8, route2, acc4, pend, tkey, town, counters, sortkeys, sortvals, cdf, cubtmp, cubtmp_bytes,
        partial, thermal, flags, pwv, pwnode, spread, total;
    // ordered apply (exact mode): one wave's change lists and ranks
    size_t w_cell, w_delta, w_vol, w_mom, w_count, w_death, w_desc, w_keys0, w_keys1, w_vals0, w_vals1, w_runstart,
        w_segpos, w_runscan, w_segscan, w_temp, w_temp_bytes, w_dth, w_keep, w_act, hand, terr, error;
    // the lake parks of one wave: per droplet its park count and entry indices, per park the refused rest
    size_t w_park_n, w_park_k, w_park_rest;
    size_t w_fin;  // the finish's gathered stockpile amounts, one double a slot
    size_t w_offsets;  // long lists: each droplet's first compacted entry, and the wave's total
    int64_t ncell, nmetric, nslots, table_cap, table_slots, max_droplets, max_wave, wave_slots, cap;
};

// records the calling thread's error message (read back with pge_last_error) and returns code
int pge_set_error(int code, const char *fmt, ...);
// the grid's own shape rules (faces, sizes, halo, int32 cell indices): PGE_OK or PGE_E_ARG with the message set
int check_shape(const PgeGrid *g);

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// number of per-thread ledger tables (one per resident droplet thread)
int64_t droplet_slots();
Layout layout(const PgeGrid &g);

template <typename T>
inline T *ws_ptr(void *ws, size_t off) { return reinterpret_cast<T *>(static_cast<char *>(ws) + off); }

struct DropArgs {
    int F, N, H, NE, spherical, deposit_on_exit, metric_shared;
    const float4 *__restrict__ A;
    const float4 *__restrict__ B;
    const double2 *__restrict__ L;
    const float4 *__restrict__ G;
    const uint8_t *__restrict__ mask;  // nullptr: all active
    const double *__restrict__ ecap;   // nullptr unless use_erode_cap
    const int32_t *sp_face;
    const double *sp_x, *sp_y, *sp_sed, *sp_dir;
    double volume0;
    long long d_begin, d_end;
    PgeParams p;
    long long *acc4;
    long long *pend;
    PgeStats *stats;
    unsigned long long *counter;       // this wave's droplet counter
    unsigned long long *counter_next;  // zeroed for the next wave
    unsigned long long *tkey;  // per-thread own-change hash tables (table_mask + 1 slots each)
    double *town;
    unsigned table_mask;
    int table_cap;
    unsigned long long gen_base;  // generation of this wave's first droplet (keys of older waves read as free)
    // change-list recording (parity hook); rec_cell == nullptr: off
    int32_t *rec_cell;
    double *rec_delta;
    float *rec_vol, *rec_mom;
    int64_t *rec_count;
    int8_t *rec_death;
    int rec_cap;
    long long rec_base;  // recorded droplet index = d - rec_base
    const float *erod;   // per-cell erodibility multiplier, or nullptr (1); read by the ledger variants
    const float2 *R;     // packed routing surface (route, flag) or nullptr: the ROUTE variants steer on it
    int lakes;           // the packed flags mark overflowing lakes (the ROUTE variants read the next cell's flag)
    const float *roots;  // per-cell share of the exchange the plants hold back, or nullptr (bare ground)
    PgeTape tape;        // the adjoint's record (the taped kernel variant only)
    int ledger;          // 1: apply each droplet's ledger inline; 0: record the change lists only
    int minb;  // kernel variant: registers for 1 or 2 resident blocks of 256 per SM
    int lanes; // droplets in flight per warp (1..32): fewer spread a latency-bound wave over more warps
    int cr_trig;  // 1: the face crossing's trig correctly rounded (the exact pass, the change-list hook); 0: CUDA's
    // lake parks (erosion.lake_fill, record-only variants): a droplet entering a lake with room parks the load its
    // shore did not take on the lake cell (an entry of volume -3); park_n[d - rec_base] counts them and
    // park_k[(d - rec_base) * LAKE_PARKS + j] is the j-th one's entry index (both may be nullptr with parks on:
    // the change-list hook)
    int parks;
    int32_t *park_n, *park_k;
};

// launchers of the two precisions (separate translation units: the float64
// one is compiled without FMA contraction so it rounds like the reference)
cudaError_t launch_droplets_f64(const DropArgs &a, int blocks, int threads, cudaStream_t st);
cudaError_t launch_droplets_f64_tape(const DropArgs &a, int blocks, int threads, cudaStream_t st);
cudaError_t launch_droplets_f64_route(const DropArgs &a, int blocks, int threads, cudaStream_t st);
cudaError_t launch_droplets_f64_lateral(const DropArgs &a, int blocks, int threads, cudaStream_t st);
int droplet_blocks_per_sm_f64_lateral(int threads, bool ledger, bool route);
int droplet_blocks_per_sm_f64_route(int threads, bool ledger);
int droplet_blocks_per_sm_f64_tape(int threads);
cudaError_t launch_droplets_f32(const DropArgs &a, int blocks, int threads, cudaStream_t st);
int droplet_blocks_per_sm_f64(int threads, int minb, bool ledger = true);
int droplet_blocks_per_sm_f32(int threads, int minb, bool ledger = true);
// parity hooks of the float64 trace's own code (pge_droplets_f64.cu): op 0..3 = tan, atan, sin, cos
// (4..7: CUDA's own, device only); the cube-sphere op 0 = to_sphere, 1 = from_sphere, 2 = transfer_velocity
cudaError_t launch_crmath(int op, long long n, const double *x, double *y, cudaStream_t st);
void crmath_host(int op, long long n, const double *x, double *y);
cudaError_t launch_cubesphere(int op, long long n, int32_t *face, double *uv, double *ab, double *xyz, cudaStream_t st);

}  // namespace pge
