/*
 * pgerosion.h -- C ABI of the B200 particle-erosion library (libpgerosion.so).
 *
 * The library replaces the per-iteration particle pass of the bake's erosion
 * stage and the plain map passes around it.  Paths below are within the
 * reference project (Gkrumbach07/procedural-generation, directory bake/):
 *
 *   pge_spawn_rain        maps.spawn_weights / spawn_particles /
 *                         particle.spawn_cells     globe/erosion/maps.py:793-833,
 *                                                  globe/erosion/particle.py:1245-1260
 *   pge_collect_pending   pending re-injection     globe/erosion/maps.py:886-903
 *   pge_trace_apply       pack_samples + the chunk loop of trace_particles /
 *                         apply_changes + fold_changes + ema_update
 *                                                  globe/erosion/maps.py:904-1047,
 *                                                  globe/erosion/particle.py:164-1101, 1230-1242
 *   pge_trace_changelist  trace_particles' change list, for parity checks
 *                                                  globe/erosion/particle.py:275-818
 *   pge_slope_erode_cap   slope_erode_cap (erosion.slope_limit_erode > 0)
 *                                                  globe/erosion/particle.py:1046-1076,
 *                                                  globe/erosion/maps.py:922-927
 *   pge_smooth_step       one step of apply_isostasy's flexural smoother
 *                         (FaceField.laplacian)    globe/erosion/maps.py:1331-1410,
 *                                                  globe/field.py:179-188, 372-404
 *   pge_thermal           thermal_erosion (talus pass + creep pass)
 *                                                  globe/erosion/maps.py:1050-1085,
 *                                                  globe/erosion/particle.py:1107-1227
 *   pge_uplift            apply_uplift             globe/erosion/maps.py:1088-1147
 *   pge_hold_datum        hold_datum               globe/erosion/maps.py:1446-1508
 *   pge_halo_gather       FaceField.exchange_halos globe/field.py:104-125
 *   pge_route_flood       ErosionState.refresh_route: the epsilon-filled routing
 *                         surface (priority_flood_eps)
 *                                                  globe/erosion/maps.py:351-358,
 *                                                  globe/erosion/route.py:31-125
 *   pge_sea_base          ErosionState.refresh_base: the base level of closed
 *                         below-sea basins (the sea mask)
 *                                                  globe/erosion/maps.py:360-420,
 *                                                  globe/hydro/run.py:64-83,
 *                                                  globe/hydro/lakes.py:19-46
 *   pge_window_lakes      ErosionState.refresh_lakes_window (lake_evap = 0): the
 *                         overflowing lakes of a window
 *                                                  globe/erosion/maps.py:629-673
 *   pge_lake_balance      ErosionState.refresh_lakes without erosion.lake_fill: the
 *                         planet's lakes by the hydro stage's flood, D8 routing and
 *                         evaporation balance (HOST code, host pointers)
 *                                                  globe/erosion/maps.py:422-479,
 *                                                  globe/hydro/priority_flood.py:127-191,
 *                                                  globe/hydro/routing.py:28-90,
 *                                                  globe/hydro/balance.py:63-284
 *   pge_lake_balance_fill pge_lake_balance with erosion.lake_fill: the loads the
 *                         lakes kept laid over their floors, the lakes numbered and
 *                         given their room (HOST code, host pointers)
 *                                                  globe/erosion/maps.py:422-479, 490-628
 *   pge_window_lake_balance  ErosionState._balance_window_lakes (window_lake_evap > 0):
 *                         a window's lakes settled against evaporation (HOST code)
 *                                                  globe/erosion/maps.py:675-736
 *   pge_basin_fill        fill_basins: sediment graded into the closed basins of a
 *                         fresh state (HOST code, host pointers)
 *                                                  globe/erosion/maps.py:1216-1229, 1278-1326
 *   pge_glacial           glacial.carve (the ice line of the evaporation field)
 *                                                  globe/erosion/glacial.py:100-257,
 *                                                  globe/erosion/maps.py:1580-1590
 *   pge_trace_apply_tape  pge_trace_apply (wave apply, one wave) recording each
 *                         droplet's steps and ledger branches for the adjoint
 *   pge_adjoint_pass      reverse of one taped droplet pass: gradients of the
 *                         surface after the pass with respect to the surface
 *                         before it, the per-cell erodibility field and the
 *                         erodibility, deposition, evaporation and friction rates
 *   pge_halo_adjoint      transpose of pge_halo_gather (scalar fields)
 *                         (the adjoint has no reference counterpart; it
 *                         differentiates the trace of particle.py:421-815 and the
 *                         ledger of particle.py:934-1018 along frozen paths)
 *
 * Conventions
 *   - Every pointer in the structs is a DEVICE pointer unless marked "host".
 *     Cell arrays are (F, NE, NE) row-major with NE = N + 2H; vector fields
 *     (momentum) are (F, NE, NE, 2).  Heights are in cell units.
 *   - The library never allocates device memory.  The caller passes one
 *     workspace of pge_workspace_bytes() bytes, 256-byte aligned.
 *   - Every call is asynchronous on the given CUDA stream (a cudaStream_t
 *     passed as void*; NULL = the legacy default stream) and returns 0 or a
 *     negative PGE_E* code; pge_last_error() describes the last failure of
 *     the calling thread.  Launch errors are checked with
 *     cudaPeekAtLastError; device-side overflow is counted in PgeStats.
 *   - Results do not depend on thread scheduling: the ordered apply does
 *     every float64 read and write of a cell in the serial order; the wave
 *     apply sums terrain changes, tracks and stockpiles as int64 fixed
 *     point; stat totals are int64 fixed point in both.
 *   - Calls on one state are not reentrant; order them on one stream.
 */
#ifndef PGEROSION_H
#define PGEROSION_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PGE_API __attribute__((visibility("default")))
#else
#define PGE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PGE_VERSION 1

enum {
    PGE_OK = 0,
    PGE_E_ARG = -1,       /* a null pointer, size or parameter out of range */
    PGE_E_WORKSPACE = -2, /* workspace too small */
    PGE_E_CUDA = -3,      /* a CUDA call failed */
    PGE_E_UNSUPPORTED = -4
};

/* droplet arithmetic precision of the trace (the ledger is always float64) */
enum { PGE_PREC_F64 = 0, PGE_PREC_F32 = 1 };

/* PGE_APPLY_ORDERED: the wave's change lists are applied in droplet order
 *   against the live terrain, float64 -- the reference's serial apply
 *   (particle.py:821-1042); with wave = the reference's chunk the whole pass
 *   is the reference's.
 * PGE_APPLY_WAVE: each droplet applies its own list against the wave-start
 *   terrain plus its own changes, merged with int64 fixed-point atomics:
 *   exact for droplets that share no cell, faster, but droplets that share
 *   cells each see the wave-start terrain. */
enum { PGE_APPLY_ORDERED = 0, PGE_APPLY_WAVE = 1 };

/* mask codes and death causes, as in globe/erosion/particle.py:54-76 */
enum { PGE_MASK_OUTSIDE = 0, PGE_MASK_ACTIVE = 1, PGE_MASK_FROZEN = 2 };
enum { PGE_DEATH_AGE = 0, PGE_DEATH_OCEAN, PGE_DEATH_EXIT, PGE_DEATH_PIT, PGE_DEATH_EVAP, PGE_DEATH_STOP, PGE_N_DEATHS };

/* fixed-point scales: value = integer * 2^-shift */
#define PGE_FX_MASS_SHIFT 40  /* terrain change, stockpiles, mass totals (cell units) */
#define PGE_FX_TRACK_SHIFT 32 /* discharge and momentum tracks (volume units) */

typedef struct PgeGrid {
    int32_t F;               /* faces: 6 on the sphere, 1 for a window */
    int32_t N;               /* interior cells per face edge */
    int32_t H;               /* halo width */
    int32_t spherical;       /* 1: droplets cross faces; 0: window, leaving it kills */
    int32_t deposit_on_exit; /* window mode: leaving droplets drop their load */
    int32_t metric_shared;   /* 1: metric tables are (NE, NE, 3), the same on every face */
    int32_t max_steps;       /* workspace capacity: the largest erosion.max_steps any call uses */
    int32_t wave_tables;     /* 1: the workspace holds the per-thread own-change tables that the wave
                                apply and pge_trace_changelist need (they grow with max_steps);
                                0: ordered apply and map passes only */
    int64_t max_droplets;    /* workspace capacity: the most spawns (rain + stockpiles) of one pass */
    int64_t max_wave;        /* workspace capacity: the largest wave of the exact (ordered) apply */
    int64_t max_threads;     /* the wave apply's resident droplet threads, each with its own-change table
                                (0: as many as the GPU holds, 1024 a multiprocessor); fewer keep the
                                tables small for a pass that shares the GPU with other worlds' passes */
} PgeGrid;

/* the ErosionState arrays (globe/erosion/maps.py:56-115) on the device */
typedef struct PgeState {
    double *height;          /* (F,NE,NE) bedrock height */
    double *sediment;        /* (F,NE,NE) */
    double *discharge;       /* (F,NE,NE) EMA of volume per iteration */
    double *momentum;        /* (F,NE,NE,2) EMA of volume * velocity */
    double *pending;         /* (F,NE,NE) stockpile re-injected next iteration */
    double *base;            /* (F,NE,NE) local base level (0 on the plain path) */
    const double *uplift;    /* (F,NE,NE) per-iteration uplift (cell units) */
    const float *hardness;   /* (F,NE,NE) */
    const float *precip;     /* (F,NE,NE) spawn weight */
    const float *evap;       /* (F,NE,NE) evaporation multiplier */
    const uint8_t *mask;     /* (F,NE,NE) or NULL: every cell active */
    const float *metric;     /* (NE,NE,3) or (F,NE,NE,3): g_ii, g_ij, g_jj */
    const float *metric_inv; /* same shape: inverse metric */
    const float *erodibility; /* (F,NE,NE) per-cell multiplier of erosion.erodibility, or NULL (1 everywhere; the
                                 reference's model): the calibrated field of the adjoint; wave apply only */
    const double *route;     /* (F,NE,NE) routing surface (pge_route_flood) or NULL: particles steer on it where it
                                stands above the terrain (particle.py:453-460, 556-559); float64 trace only */
    const uint8_t *lake_flag; /* (F,NE,NE) overflowing lakes (ErosionState.lake_flag, maps.py:87) or NULL; read only
                                 with `route`: 1 a lake, 2 a lake with room for its rivers' load (the same as 1
                                 unless lake_load is set).  A droplet entering a lake drops lake_trap of its load
                                 at the shore, crosses it without touching the bed and counts no pit steps on it;
                                 the bed is never eroded below the lake's routing surface (particle.py:186-190,
                                 626-636, 751-763, 952-956) */
    const float *roots;       /* (F,NE,NE) the share of a droplet's exchange with the bed the plants hold back
                                 (erosion.vegetation, maps.py:113; in [0, 1]) or NULL: bare ground.  The
                                 exchange rate on land is scaled by 1 - roots (particle.py:615-618); not with
                                 the adjoint's tape */
    double *lake_load;        /* (F,NE,NE) the lake parks (erosion.lake_fill, maps.py:105-107) or NULL: off.  With
                                 `route` and `lake_flag`, a droplet entering a lake flagged 2 that its shore had no
                                 room to take the trapped load for parks the rest on the lake cell it steps onto
                                 (a change-list entry of volume -3, at most 8 a droplet, particle.py:672-696);
                                 the ordered apply counts each lake's room down in droplet order, adds what it
                                 takes here and adds the rest to the droplet's leftover load (particle.py:
                                 912-933, 1019).  Ordered apply (and the change-list hook) only */
    const int32_t *lake_id;   /* (F,NE,NE) the lake of lake_room each cell belongs to, -1 none (read with lake_load) */
    double *lake_room;        /* (lakes) the room each lake has left (cell units), counted down in place */
    int64_t lakes;            /* entries of lake_room */
} PgeState;

/* droplet spawns of one iteration: rain first, then re-injected stockpiles */
typedef struct PgeSpawns {
    int32_t *face;
    double *x, *y;           /* fractional interior cell coordinates */
    double *sed;             /* initial load (0 for rain) */
    double *dir;             /* initial direction (radians) of a loaded droplet */
    int64_t count;
    double volume0;          /* spawn volume (host value) */
} PgeSpawns;

/* the plain-path scalar knobs, already in cell units (maps.py:958-1008) */
typedef struct PgeParams {
    double dt, density, friction, deposition_rate, evap_rate, k_mom, mom_scale, k_disc, disc_saturation,
        disc_exponent, slope_gain, slope_sat, erodibility, cover_depth, min_volume, max_erode, conc_scale,
        ocean_rate, fan_room, dep_floor, iter_erode, iter_deposit, fan_slope, offshore_writeoff, ema;
    double lake_trap;        /* share of the load dropped at the shore on entering a lake (erosion.lake_trap);
                                read only with s->lake_flag */
    double lateral_rate;     /* erosion.lateral_rate > 0: a droplet cutting its bed also cuts the bank one cell
                                across the flow on the outside of its bend (particle.py:699-738), an extra
                                change-list entry of volume -2; float64 trace only, not with the tape, and the
                                workspace's max_steps must hold 2 x max_steps (two entries a step) */
    int32_t max_steps, pit_steps, ocean_steps;
    int32_t wave;            /* droplets traced against one frozen terrain (the reference's chunk) */
    int32_t precision;       /* PGE_PREC_* */
    int32_t apply;           /* PGE_APPLY_*: how a wave's changes meet the terrain */
    int32_t use_erode_cap;   /* slope_limit_erode > 0: erode_cap passed to pge_trace_apply */
    int32_t threads_per_block; /* 0 = default */
    int32_t blocks_per_sm;     /* 0 = occupancy maximum */
    int32_t trace_lanes;       /* ordered apply: droplets per warp in each wave's trace; 0 = as few as keep
                                  every warp of the wave resident (fastest alone), up to 32 (smallest
                                  footprint, for passes of several worlds running at once) */
    int32_t apply_lanes;       /* ordered apply: droplets per warp in the apply, 0 = 1 .. 32; more hold
                                  fewer warps but lanes waiting on different hand-offs take turns
                                  (one per warp measured fastest, alone and with other passes) */
    int32_t brush_radius;      /* wave apply: 0 = each entry changes its own cell (the reference's one-cell write,
                                  particle.py:662-671); r = 1..PGE_BRUSH_MAX_RADIUS: each applied erosion or
                                  deposition is spread over the cells of its face within distance < r + 1
                                  with weights r + 1 - distance (integers of 1/PGE_BRUSH_SCALE), over the
                                  active cells only (the interior ones on the sphere), conserving: the
                                  integer shares are truncated and the rest stays on the entry's own cell.  No
                                  counterpart in the reference.  A droplet's own view of the terrain keeps
                                  its changes on their own cells; tracks and stockpiles are not spread */
} PgeParams;

#define PGE_BRUSH_MAX_RADIUS 4
#define PGE_BRUSH_SCALE 1024

/* counters of one droplet pass (device struct; the caller zeroes it) */
typedef struct PgeStats {
    int64_t droplets;
    int64_t droplet_steps;   /* change-list entries with volume >= 0 */
    int64_t entries;
    int64_t deaths[PGE_N_DEATHS];
    int64_t clamped;
    int64_t overflow;        /* droplets whose ledger table overflowed (never expected) */
    int64_t to_pending_fx;   /* mass totals, fixed point 2^-40 */
    int64_t deficit_out_fx;
    int64_t lost_offshore_fx;
    int64_t released_fx;
    int64_t eroded_fx;       /* terrain removed by the ledger (applied erosion) */
    int64_t deposited_fx;    /* terrain added by the ledger (applied deposition) */
    int64_t errors;          /* nonzero: an ordered-apply wait gave up (the pass is invalid) */
} PgeStats;

/* The tape of one wave-apply droplet pass, for the adjoint.  Row r of each
 * array is droplet r of the pass (rain, then re-injected stockpiles).  state[r, k] is
 * the droplet's (x, y, a, b, sed, vol) at the start of its k-th step; the row
 * after its last completed step is its final state.  bits[r, k] holds the
 * face (bits 0-2) and the branches that step took (PGE_TB_*).  entry[r, j]
 * is the ledger's j-th change: (cell, reference cell, branch code PGE_TE_*,
 * step index or -1 for a final deposit).  count[r] = (state rows, entries).
 * wave_acc[w] is the pass's int64 terrain accumulator (2^-40 cell units) as
 * wave w started: the terrain wave w's droplets saw. */
typedef struct PgeTape {
    double *state;    /* (droplets, steps + 1, 6) */
    int32_t *bits;    /* (droplets, steps + 1) */
    int32_t *entry;   /* (droplets, entries, 4) */
    int32_t *count;   /* (droplets, 2) */
    int64_t droplets; /* rows (>= the pass's spawn count) */
    int32_t steps;    /* >= max_steps */
    int32_t entries;  /* >= max_steps + 8 */
    int64_t *wave_acc; /* (waves, F*NE*NE) */
    int64_t waves;     /* >= the pass's waves, ceil(count / p->wave) */
} PgeTape;

/* tape bits of a step (the trace's branches, particle.py:421-769); whether a
 * bilinear weight was clamped to [0, 1] is not stored: it follows from the
 * recorded coordinates */
enum {
    PGE_TB_FACE = 0x7,            /* face the step starts on */
    PGE_TB_S2_ZERO = 1 << 5,      /* slope^2 clamped to 0 */
    PGE_TB_Q_ZERO = 1 << 6,       /* discharge sample clamped to 0 */
    PGE_TB_FR_ZERO = 1 << 7,      /* 1 - dt friction clamped to 0 */
    PGE_TB_MOM = 1 << 8,          /* the momentum pull was applied */
    PGE_TB_CROSS = 1 << 9,        /* the move left the face's square: transfer_velocity ran */
    PGE_TB_SAME_FACE = 1 << 10,   /* ... and came back to the same face (coordinates clamped) */
    PGE_TB_X_CLAMP = 1 << 11,     /* the new coordinate was clamped */
    PGE_TB_Y_CLAMP = 1 << 12,
    PGE_TB_H1_ABOVE = 1 << 15,    /* new height above the base: dh = h0 - h1 (else h0 - base) */
    PGE_TB_LAND = 1 << 16,        /* land mass transfer made an entry */
    PGE_TB_SEA = 1 << 17,         /* seafloor (fan) mass transfer made an entry */
    PGE_TB_CEQ_ZERO = 1 << 18,    /* capacity clamped to 0 */
    PGE_TB_COVER = 1 << 19,       /* capacity above the load: the cover / hardness blend */
    PGE_TB_POS = 1 << 20,         /* cdiff > 0 (erosion) */
    PGE_TB_NEG = 1 << 21,         /* cdiff < 0 (deposition) */
    PGE_TB_CLAMP = 1 << 22,       /* cdiff limited by the erosion cap / the deposit room */
    PGE_TB_ECAP_SHIFT = 23,       /* 2 bits: erosion cap = dh / kexp, max_erode, the cell's surface, 0 */
    PGE_TB_ROOM_FLOOR = 1 << 25,  /* deposit room = its floor (dep_floor / fan_room), not h_prev - h_here */
    PGE_TB_SEA_SHIFT = 26,        /* 2 bits: seafloor room as above, the base limit, or 0 */
    PGE_TB_EV_CLAMP = 1 << 28     /* evaporation factor clamped to 0.01 */
};

/* tape code of a ledger entry (particle.py:934-1018) */
enum {
    PGE_TE_DEPOSIT = 1 << 0,      /* delta >= 0 */
    PGE_TE_STEP = 1 << 1,         /* a step entry (else a final deposit) */
    PGE_TE_SKIP = 1 << 2,         /* inactive cell: nothing applied */
    PGE_TE_SRC_SHIFT = 4,         /* 3 bits, erosion: ew, room, floor = base, floor = surface, floor = next cell, 0;
                                     deposit: want, room, reference ceiling, base limit, 0 */
    PGE_TE_TAKE_SHIFT = 8         /* 2 bits, deposit: no deficit, all of want taken, all of the deficit taken */
};

/* halo gather tables (bake/globe/cubesphere.py:540-662) */
typedef struct PgeHalo {
    int64_t K;               /* halo rows */
    const int32_t *dst;      /* (K) flat halo cell */
    const int32_t *src;      /* (K,16) flat interior sources */
    const double *w;         /* (K,16) weights */
    const double *rot;       /* (K,16,2,2) vector rotations, or NULL */
} PgeHalo;

PGE_API int pge_version(void);
/* copies the calling thread's last error message (host buffer); returns its length */
PGE_API int pge_last_error(char *buf, size_t n);

/* Workspace bytes for a grid and its capacities (g->max_droplets,
 * g->max_steps).  Every call on that grid must be passed the same PgeGrid
 * and a workspace at least this large. */
PGE_API size_t pge_workspace_bytes(const PgeGrid *g);

/* Rain spawns (maps.spawn_particles): spawnable cells are interior, active,
 * surface >= base and precip > 0; u (count) host-drawn uniforms in [0,1)
 * (unsorted: the library sorts them), off (count,2) offsets.  Writes
 * spawns->face/x/y/sed/dir[0:count] and the spawn total weight to
 * *total_dev (device double; volume0 = total / count).  *nspawnable_dev
 * (device int64) receives the number of spawnable cells. */
PGE_API int pge_spawn_rain(const PgeGrid *g, const PgeState *s, const double *u, const double *off, int64_t count,
                   PgeSpawns *spawns, double *total_dev, int64_t *nspawnable_dev, void *ws, size_t ws_bytes,
                   void *stream);

/* Pending re-injection, stage 1: counts the cells with pending > 0 into
 * *count_dev (device int64). */
PGE_API int pge_count_pending(const PgeGrid *g, const PgeState *s, int64_t *count_dev, void *ws, size_t ws_bytes, void *stream);

/* Pending re-injection, stage 2: appends one loaded droplet per cell with
 * pending > 0, in flat-index order, at spawns[offset ...] (cell centre,
 * sed = the stockpile), adds the released mass to stats->released_fx and
 * zeroes pending.  dir must already hold the host-drawn directions. */
PGE_API int pge_collect_pending(const PgeGrid *g, PgeState *s, PgeSpawns *spawns, int64_t offset, PgeStats *stats,
                        void *ws, size_t ws_bytes, void *stream);

/* One droplet pass: pack the samples, trace every spawn in waves of
 * p->wave droplets (terrain frozen within a wave, refreshed between waves),
 * apply each droplet's erosion / deposition ledger against the wave-start
 * terrain plus its own changes, then fold the net change into
 * height / sediment, EMA-update discharge / momentum and write pending. */
PGE_API int pge_trace_apply(const PgeGrid *g, PgeState *s, const PgeSpawns *spawns, const PgeParams *p,
                    const double *erode_cap, PgeStats *stats, void *ws, size_t ws_bytes, void *stream);

/* Parity hook: trace and apply one wave exactly like pge_trace_apply and
 * also write every droplet's change list in the reference layout
 * (cap = max_steps + 2*8 + 1 + 8 + 8 entries per droplet): cell (int32),
 * requested delta (float64), volume and momentum (float32), count (int64)
 * and death cause (int8).  No fold / EMA; the net change stays in the
 * workspace accumulators (read them with pge_read_accumulators). */
PGE_API int pge_trace_changelist(const PgeGrid *g, PgeState *s, const PgeSpawns *spawns, const PgeParams *p,
                         int32_t *cl_cell, double *cl_delta, float *cl_vol, float *cl_mom, int64_t *cl_count,
                         int8_t *cl_death, PgeStats *stats, void *ws, size_t ws_bytes, void *stream);

/* Converts the workspace accumulators of the last pass to float64:
 * acc (F,NE,NE), disch_track (F,NE,NE), mom_track (F,NE,NE,2), pending (F,NE,NE). */
PGE_API int pge_read_accumulators(const PgeGrid *g, double *acc, double *disch_track, double *mom_track, double *pending,
                          void *ws, size_t ws_bytes, void *stream);

/* soillib's pit-free erosion cap: erode_cap (F,NE,NE) = coef * sqrt(2) * the Godunov downhill
 * slope of height + sediment (per axis the steeper one-sided downhill difference, exit_slope off
 * the array, 0 outside the active mask).  Computed once per iteration before the droplet pass and
 * passed to pge_trace_apply with p->use_erode_cap = 1 (coef = erosion.slope_limit_erode,
 * exit_slope = erosion.slope_limit_exit). */
PGE_API int pge_slope_erode_cap(const PgeGrid *g, const PgeState *s, double coef, double exit_slope, double *erode_cap,
                                void *stream);

/* One explicit step of the isostasy smoother on the sphere: the metric-aware Laplace-Beltrami
 * operator of in (F,NE,NE) in flux form at extended indices 1..NE-2 (0 on the outer ring; halos
 * exchanged first, with the linear tables), per m^2 and rounded to float32, then
 * out = (keep ? in : 0) + (kappa * lap) * cell_m^2.  metric_inv is the (NE,NE,3) inverse metric,
 * sqrt_det the (NE,NE) float32 sqrt(det g) of the metric, both shared by the faces.  in != out. */
PGE_API int pge_smooth_step(const PgeGrid *g, const float *metric_inv, const float *sqrt_det, const double *in, double *out,
                            double kappa, int32_t keep, double cell_m, void *stream);

/* Talus pass, then (creep_rate > 0) the creep pass with submerged cells frozen. */
PGE_API int pge_thermal(const PgeGrid *g, PgeState *s, double thermal_rate, double creep_rate, double thermal_max,
                double talus_soft, double talus_hard, double dep_floor, void *ws, size_t ws_bytes, void *stream);

/* height += min(uplift, cap) - mean over the active interior (cap < 0: none;
 * the mean is taken only when spherical). */
PGE_API int pge_uplift(const PgeGrid *g, PgeState *s, double cap, double scale, void *ws, size_t ws_bytes, void *stream);

/* Rigid shift so that round(land_fraction * M) interior cells have
 * height + sediment >= level; writes the shift (cell units) to *shift_dev. */
PGE_API int pge_hold_datum(const PgeGrid *g, PgeState *s, double land_fraction, double level, double *shift_dev, void *ws,
                   size_t ws_bytes, void *stream);

/* Fills the halo rows of one field from its interior: a scalar (F,NE,NE)
 * field, or with vector = 1 a (F,NE,NE,2) field rotated per source. */
PGE_API int pge_halo_gather(const PgeHalo *h, double *field, int32_t vector, void *stream);

/* The routing surface (route.py:31-125): the surface filled so that every
 * cell reached from a seed drains by at least eps per cell, as the reference's
 * priority flood computes it (value for value), with halo cells left at their
 * surface (refresh them with the linear halo exchange).  Seeds: interior cells
 * with surface < 0 and surface <= s->base, and (windows) cells next to an
 * outside or halo cell; s->mask (may be NULL) excludes outside cells; owner is
 * the (F,NE,NE) int32 owner table (cubesphere.py:664-674; the identity for a
 * window).  Surface = s->height + s->sediment.  Runs a relaxation to its fixed
 * point, synchronising the stream every 32 sweeps to test it; *sweeps (host,
 * may be NULL) gets the sweeps run; PGE_E_UNSUPPORTED if max_sweeps did not
 * reach the fixed point. */
PGE_API int pge_route_flood(const PgeGrid *g, const PgeState *s, const int32_t *owner, double eps, double *route, int64_t max_sweeps,
                            int64_t *sweeps, void *ws, size_t ws_bytes, void *stream);

/* The sea mask (maps.py:360-420): interior cells whose float32 surface
 * (s->height + s->sediment) is below 0 are joined into 8-connected
 * components through the owner table (int32, (F,NE,NE)); a component whose
 * area (area: (F,N,N) float32 interior cell areas, summed in float64)
 * reaches min_area is open ocean, and so is the largest; every other one is
 * a closed basin, whose cells get the basin's lowest surface as their base
 * level.  Writes base (F,NE,NE): that floor on closed-basin cells, 0 on the
 * rest of the interior and on the halos (copy each halo cell from its
 * nearest interior source afterwards, as the reference does); labels (may be
 * NULL) gets (F,N,N) int32 component ids (the lowest cell id of the
 * component, -1 above the waterline).  Components are joined along the
 * owner relation taken both ways (the reference walks it one way from each
 * component's lowest cell; they differ only where a cube corner's halo
 * mapping is one-sided).  Synchronises the stream every 16 sweeps; spherical
 * grids only. */
PGE_API int pge_sea_base(const PgeGrid *g, const PgeState *s, const int32_t *owner, const float *area, double min_area, double *base,
                         int32_t *labels, int64_t max_sweeps, int64_t *sweeps, void *ws, size_t ws_bytes, void *stream);

/* The lakes of a window (maps.py:629-673, erosion.window_lakes with
 * window_lake_evap = 0): lake_flag (F,NE,NE) = 1 on interior cells whose
 * mask is active (every cell when s->mask is NULL) and whose routing surface
 * s->route stands more than min_depth (cell units) above the surface
 * s->height + s->sediment (float64), 0 on the rest and on the halos.
 * lake_cells (device, may be NULL) gets their count.  Any grid; the planet's
 * lakes (maps.py:422-479) come from the hydro stage's balance instead. */
PGE_API int pge_window_lakes(const PgeGrid *g, const PgeState *s, double min_depth, uint8_t *lake_flag, int64_t *lake_cells,
                             void *stream);

/* counts of one lake refresh (maps.py:481-483 and the balance's, balance.py:270-279) */
typedef struct PgeLakeInfo {
    int64_t lake_cells;        /* cells deeper than min_depth under water, off the ocean */
    int64_t lake_cells_closed; /* of those, cells of lakes drawn below their rim */
    int64_t depressions, overflowing, closed, dry;
} PgeLakeInfo;

/* The planet's lakes (maps.py:422-479 with erosion.lake_fill off), on the
 * HOST: every pointer is a host pointer and no CUDA call is made.  The
 * reference's sequence is serial by construction -- every later step follows
 * the priority flood's pop order -- so it runs as one host pass between
 * iterations, as the reference's does.  Inputs, interior (6,N,N) arrays in
 * cell-id order (f*N + i)*N + j: surface (float32 height + sediment), ocean
 * (1 on the open sea: the flood's drains), precip (the spawn weight), pet (the
 * balance's potential evaporation: the state's evap, or lake_pet), cell_area
 * (float32 m^2); owner (6,NE,NE) int32 the extended flat index of the
 * interior cell owning each extended cell; metric (NE,NE,3) float32, shared
 * by the faces.  The flood fills every depression from the drains (a FIFO for
 * cells at or below the current level, a (level, push order) heap for the
 * rest; the lowest cell drains when there is no ocean), D8 descends the
 * filled surface by physical slope (flats to their flood parent), and one
 * upstream-first accumulation of the runoff (Budyko's curve with land_evap >
 * 0, else all of precip) solves each depression's level where its
 * evaporation (lake_evap x pet, or pet less the land's evaporation with
 * land_evap > 0) meets its inflow.  Outputs (6,N,N): lake_flag 1 on cells
 * of overflowing lakes deeper than min_depth (cell units); closed_level (may
 * be NULL) the water level (cell units) on cells of lakes drawn more than
 * 1e-4 below their rim (the caller's base level there), NaN elsewhere; water
 * (may be NULL) the water surface.  PGE_E_UNSUPPORTED if a land cell gets no
 * flow direction (the flood did not reach it).  The pass keeps its
 * full-size scratch (about 120 bytes a cell: 0.8 GB at N = 1024) on the
 * calling thread between calls, so that a refresh every few iterations
 * reuses its pages. */
PGE_API int pge_lake_balance(const PgeGrid *g, const int32_t *owner, const float *metric, const float *cell_area, double cell_size_m,
                             const float *surface, const uint8_t *ocean, const float *precip, const float *pet, double lake_evap,
                             double land_evap, double min_depth, uint8_t *lake_flag, float *water, float *closed_level,
                             PgeLakeInfo *info);

/* erosion.lake_fill's side of a lake refresh (maps.py:490-628), host arrays,
 * interior (6,N,N) in cell-id order unless noted */
typedef struct PgeLakeFill {
    double grade;          /* the lake plain's rise per cell from the outlet (cell units: basin_fill_grade x cell km) */
    double ice_evap;       /* a lake with a cell of evap <= ice_evap is frozen: it takes no load */
    double rise;           /* the plain stands at most this much above the water (cell units) */
    const float *evap;     /* evaporation field */
    const double *centres; /* (6,N,N,3) unit-sphere cell centres (the outlet distance) */
    const double *height;  /* bedrock and sediment (the surface after laying) */
    const double *sediment;
    double *lake_load;     /* in: the loads parked since the last refresh; out: zero */
    int32_t *lake_id;      /* in: the last refresh's lake of each cell (-1 none); out: this refresh's */
    double *lay;           /* out: sediment laid on each cell (the caller adds it to sediment; with the
                              isostasy, load_share x lay to its load) */
    double *pending;       /* out: loads that go on as stockpiles (their lake drained, or rounding), 0 elsewhere */
    double *lake_room;     /* out: the room each numbered lake has left, lake_room_cap entries at most */
    int64_t lake_room_cap;
    int64_t lakes;         /* out: lakes numbered (open, warm, with room left) */
    double parked, laid, stray, room; /* out: totals (cell units) */
} PgeLakeFill;

/* pge_lake_balance with erosion.lake_fill (maps.py:422-479 with `fill`, and
 * settle_lake_loads, maps.py:490-628), on the HOST.  After the balance, the
 * overflowing lakes (cells joined at one water level) receive the loads
 * parked on their cells since the last refresh (a load whose cell is no
 * longer under a lake goes to the lake of this refresh covering most of its
 * old lake, else on as a stockpile); each lake fills towards a plain graded
 * `grade` per flood step from its outlet and at most `rise` above its water,
 * the cells farthest from the outlet first; a lake with room left and no
 * frozen cell is numbered (lake_id, lake_room) and its cells flagged 2.
 * lake_flag then marks the lakes still deeper than min_depth over the
 * surface with the laid sediment.  Other arguments as pge_lake_balance. */
PGE_API int pge_lake_balance_fill(const PgeGrid *g, const int32_t *owner, const float *metric, const float *cell_area,
                                  double cell_size_m, const float *surface, const uint8_t *ocean, const float *precip,
                                  const float *pet, double lake_evap, double land_evap, double min_depth, uint8_t *lake_flag,
                                  float *water, float *closed_level, PgeLakeFill *fill, PgeLakeInfo *info);

/* The lakes of a window balanced against evaporation (maps.py:675-736,
 * erosion.window_lakes with window_lake_evap > 0), on the HOST (host
 * pointers, no CUDA call), over the whole (NE,NE) window array: the flat
 * priority flood draining to the cells not active and the array's border,
 * precip (the spawn weight) accumulated down the flood tree, every
 * depression (8-connected active cells the flood fills more than 1e-6 above
 * the float32 surface, numbered in raster order) settled where the inflow
 * reaching it meets lake_evap x max(evap, 0) summed over its cells under the
 * water (a dry one drops below its floor, one that cannot evaporate its
 * inflow spills).  lake (NE,NE) gets 1 on active cells more than min_depth
 * (cell units) under water; route (NE,NE, in/out) is lowered to the water on
 * them; counts (5 int64, may be NULL): depressions, overflowing, closed,
 * dry, lake cells.  The caller flags the interior. */
PGE_API int pge_window_lake_balance(const PgeGrid *g, const float *surface, const uint8_t *active, const float *precip,
                                    const float *evap, double lake_evap, double min_depth, double *route, uint8_t *lake,
                                    int64_t *counts);

/* The basin fill of a fresh state (maps.py:1278-1326, erosion.basin_fill_grade),
 * on the HOST (host pointers, no CUDA call): the same priority flood as
 * pge_lake_balance from the ocean drains (surface, ocean: interior (6,N,N)
 * float32 / uint8; owner as there), then every cell raised to at least
 * `step` (cell units per cell: basin_fill_grade x cell km / height unit)
 * above the cell that flooded it, in pop order; add (6,N,N) float64 gets
 * that plain less the surface (>= 0) on cells the flood left more than
 * min_depth (cell units, float32 test) under its fill and off the ocean, 0
 * elsewhere -- the sediment the caller adds.  basin (6,N,N) uint8 (may be
 * NULL) gets 1 on those cells, basin_cells (host, may be NULL) their count. */
PGE_API int pge_basin_fill(const PgeGrid *g, const int32_t *owner, const float *surface, const uint8_t *ocean, double step,
                           double min_depth, double *add, uint8_t *basin, int64_t *basin_cells);

/* The glacial pass (glacial.py:162-257), the ice line read from the
 * evaporation field: ice on active cells with evap <= ice_evap and surface
 * > 0 (or, with ice_prev non-NULL -- erosion.glacial_sticky -- ice there
 * before and still cold; ice_prev (F,NE,NE) uint8 is then updated); the bed
 * lowered by glacial_rate sqrt(max(discharge, 0) / disc_saturation)
 * (1 - 0.5 hardness) times the taper (glacial_ramp rings in from the
 * margin), capped at glacial_max and at the cell's base level (less 0.02);
 * the carved rock spread over the ice margin by discharge as sediment,
 * capped per cell at iter_deposit, the rest added to pending.  Lengths in
 * cell units.  Every rule runs on the extended arrays with neighbours
 * wrapping at each face array's edges (the reference's numpy rolls); refresh
 * the halos afterwards.  stats (host): ice cells, carved, moraine cells,
 * largest carve, outwash (parked).  Synchronises the stream. */
PGE_API int pge_glacial(const PgeGrid *g, PgeState *s, uint8_t *ice_prev, double glacial_rate, double glacial_max, int32_t glacial_ramp,
                        double ice_evap, double disc_saturation, double moraine_frac, double iter_deposit, double *stats, void *ws,
                        size_t ws_bytes, void *stream);

/* No counterpart in the reference: the adjoint of the particle pass.
 *
 * pge_trace_apply_tape: pge_trace_apply with p->apply = PGE_APPLY_WAVE,
 * float64, recording the tape (PgeTape).  The pass's result is
 * pge_trace_apply's, bit for bit.
 *
 * pge_adjoint_pass: the reverse of that pass.  s holds the pass's START
 * state (the one pge_trace_apply_tape read) and tape its record; zbar_after
 * is dL/d(surface after the pass) (F,NE,NE); writes dL/d(surface before the
 * pass) to zbar_before (a different buffer; waves are reversed last to
 * first, each against the terrain it saw) and ADDS dL/d(erodibility field)
 * to ebar (F,NE,NE; may be NULL) and dL/d(erodibility, deposition_rate,
 * evap_rate, friction) to pbar[0..3] (device doubles).  Each droplet's cell
 * path and every branch it took are held fixed; within them the load and
 * volume are differentiated along the whole path (capacity law, exchange
 * rate, erosion cap, deposit room, evaporation, final load, the ledger's
 * floors, ceilings, deficit and surplus) and the terrain through the
 * bilinear samples.  carry_path = 1: the droplet's position and direction
 * are differentiated along the whole path too (slope force, friction,
 * momentum pull, metric normalisation, face transfer): the exact derivative
 * of the pass on its path.  carry_path = 0: each step's incoming position
 * and direction are held fixed and only the step's own move is
 * differentiated (its new position's sample).  Held constant in both: the
 * discharge and momentum tracks, sediment cover, hardness, evaporation
 * field, base level, stockpiles and the droplet's own earlier changes inside
 * its ledger's bounds.  Float64 atomics: the sums' order (last bits) varies.
 * stats (may be NULL) gets errors != 0 if the tape and its steps disagree.
 *
 * pge_halo_adjoint: for each halo row, adds w * zbar[dst] to zbar[src] and
 * zeroes zbar[dst] (the transpose of the scalar pge_halo_gather). */
PGE_API int pge_trace_apply_tape(const PgeGrid *g, PgeState *s, const PgeSpawns *spawns, const PgeParams *p,
                                 const PgeTape *tape, PgeStats *stats, void *ws, size_t ws_bytes, void *stream);
PGE_API int pge_adjoint_pass(const PgeGrid *g, const PgeState *s, const PgeSpawns *spawns, const PgeParams *p,
                             const PgeTape *tape, int32_t carry_path, const double *zbar_after, double *zbar_before,
                             double *ebar, double *pbar, PgeStats *stats, void *ws, size_t ws_bytes, void *stream);
PGE_API int pge_halo_adjoint(const PgeHalo *h, double *zbar, void *stream);

/* Parity hooks of the float64 trace's own face-crossing code.
 *
 * pge_cubesphere_map runs, on the device, the functions the float64 droplet
 * kernel crosses cube faces with, over n records (device arrays):
 *   op 0: to_sphere(face[i], uv[2i], uv[2i+1]) -> xyz[3i..3i+2]
 *         (cubesphere.to_sphere, globe/cubesphere.py:71-88)
 *   op 1: from_sphere(xyz[3i..3i+2]) -> face[i], uv[2i..2i+1]
 *         (cubesphere.from_sphere, globe/cubesphere.py:97-111)
 *   op 2: transfer_velocity(face[i], uv[2i..], ab[2i..]) in place
 *         (cubesphere.transfer_velocity, globe/cubesphere.py:204-220)
 * pge_crmath (device arrays) and pge_crmath_host (host arrays) evaluate the
 * kernel's float64 tan, atan, sin, cos (op 0..3): double-double evaluations
 * rounded once, so that they give the C library's results that the
 * reference's math.tan / math.atan (cubesphere.py:73-74, 110-111) and
 * math.cos / math.sin (erosion/particle.py:400-401) return wherever those
 * are correctly rounded.  pge_crmath's op 4..7 evaluate CUDA's own tan,
 * atan, sin, cos instead, for comparison (the trace does not use them). */
PGE_API int pge_cubesphere_map(int32_t op, int64_t n, int32_t *face, double *uv, double *ab, double *xyz, void *stream);
PGE_API int pge_crmath(int32_t op, int64_t n, const double *x, double *y, void *stream);
PGE_API int pge_crmath_host(int32_t op, int64_t n, const double *x, double *y);

/* No counterpart in the reference.  pge_thermal for callers that cannot
 * allocate device memory -- a host that owns the whole device heap through
 * its own pool and forbids other allocations, or a loop that must not pay
 * cudaMalloc's latency and implicit synchronisation: no workspace, the
 * scratch is a static device array of PGE_NOALLOC_MAX_CELLS cells (10 MiB,
 * held by every GPU that loads the library until exit).  Grids with more
 * cells than that (F * NE * NE) are rejected with PGE_E_ARG, and so is any
 * grid pge_thermal rejects.  The first call on a device looks up the array's
 * device address (make it before any stream capture) and keeps it; the kept
 * address does not survive cudaDeviceReset, so do not call this entry point
 * again on a device the process has reset.  All calls share the array: calls
 * that overlap on the GPU race, so order them. */
#define PGE_NOALLOC_MAX_CELLS 262144
PGE_API int pge_thermal_noalloc(const PgeGrid *g, PgeState *s, double thermal_rate, double creep_rate, double thermal_max,
                                double talus_soft, double talus_hard, double dep_floor, void *stream);

#ifdef __cplusplus
}
#endif
#endif
