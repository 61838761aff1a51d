// pge_api.cu -- the extern "C" entry points of libpgerosion (include/pgerosion.h).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "pge_internal.cuh"
#include "pge_maps.cuh"
#include "pge_ordered.cuh"

namespace pge {

namespace {
thread_local char g_err[512] = "";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

}  // namespace

int pge_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

namespace {

int cuda_fail(cudaError_t e, const char *where)
{
    return fail(PGE_E_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

}  // namespace

// the geometry alone (calls that use no workspace); shared with pge_static.cu
int check_shape(const PgeGrid *g)
{
    if (!g) return fail(PGE_E_ARG, "grid is NULL");
    if (g->F < 1 || g->N < 2 || g->H < 1 || g->N < 2 * g->H) return fail(PGE_E_ARG, "bad grid F=%d N=%d H=%d", g->F, g->N, g->H);
    if (g->spherical && g->F != 6) return fail(PGE_E_ARG, "a spherical grid has 6 faces (F=%d)", g->F);
    const long long NE = g->N + 2LL * g->H;
    if ((long long)g->F * NE * NE >= (1LL << 31)) return fail(PGE_E_ARG, "grid too large for int32 cell indices");
    return PGE_OK;
}

namespace {

int check_grid(const PgeGrid *g)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (g->max_steps < 1 || g->max_droplets < 1 || g->max_wave < 1) return fail(PGE_E_ARG, "workspace capacities must be positive");
    if (g->max_wave > (1LL << 20)) return fail(PGE_E_ARG, "max_wave above 2^20");
    return PGE_OK;
}

int check_ws(const PgeGrid *g, void *ws, size_t bytes, Layout &lay)
{
    lay = layout(*g);
    if (!ws) return fail(PGE_E_ARG, "workspace is NULL");
    if (reinterpret_cast<uintptr_t>(ws) & 255) return fail(PGE_E_ARG, "workspace must be 256-byte aligned");
    if (bytes < lay.total) return fail(PGE_E_WORKSPACE, "workspace %zu bytes, need %zu", bytes, lay.total);
    return PGE_OK;
}

int check_state(const PgeState *s)
{
    if (!s || !s->height || !s->sediment || !s->discharge || !s->momentum || !s->pending || !s->base || !s->hardness ||
        !s->evap || !s->metric || !s->metric_inv)
        return fail(PGE_E_ARG, "state has a NULL array");
    return PGE_OK;
}

int check_params(const PgeGrid *g, const PgeParams *p)
{
    if (!p) return fail(PGE_E_ARG, "params is NULL");
    if (p->max_steps < 1 || p->max_steps > g->max_steps) return fail(PGE_E_ARG, "max_steps %d outside 1..%d", p->max_steps, g->max_steps);
    if (!(p->lateral_rate >= 0.0)) return fail(PGE_E_ARG, "lateral_rate must be >= 0");
    if (list_steps(*p) > g->max_steps)
        return fail(PGE_E_ARG, "the bank cut needs a workspace for 2 x max_steps = %d steps (grid max_steps %d)", list_steps(*p),
                    g->max_steps);
    if (p->wave < 1) return fail(PGE_E_ARG, "wave must be >= 1");
    if (p->apply != PGE_APPLY_ORDERED && p->apply != PGE_APPLY_WAVE) return fail(PGE_E_ARG, "unknown apply mode %d", p->apply);
    if (p->apply == PGE_APPLY_ORDERED && p->wave > g->max_wave)
        return fail(PGE_E_ARG, "wave %d above the workspace's max_wave %lld", p->wave, (long long)g->max_wave);
    if (p->precision != PGE_PREC_F64 && p->precision != PGE_PREC_F32) return fail(PGE_E_ARG, "unknown precision %d", p->precision);
    if (p->threads_per_block != 0 && (p->threads_per_block < 32 || p->threads_per_block > 256 || p->threads_per_block % 32))
        return fail(PGE_E_ARG, "threads_per_block must be a multiple of 32 in 32..256");
    if (p->trace_lanes < 0 || p->trace_lanes > 32) return fail(PGE_E_ARG, "trace_lanes %d outside 0..32", p->trace_lanes);
    if (p->apply_lanes < 0 || p->apply_lanes > 32) return fail(PGE_E_ARG, "apply_lanes %d outside 0..32", p->apply_lanes);
    if (p->brush_radius < 0 || p->brush_radius > PGE_BRUSH_MAX_RADIUS)
        return fail(PGE_E_ARG, "brush_radius %d outside 0..%d", p->brush_radius, PGE_BRUSH_MAX_RADIUS);
    if (p->brush_radius > 0 && p->apply != PGE_APPLY_WAVE)
        return fail(PGE_E_UNSUPPORTED, "the brush (brush_radius > 0) spreads changes with the wave apply's integer sums");
    return PGE_OK;
}

int sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return sms;
}

}  // namespace


// droplet threads resident at once (the kernel runs at most 1024 threads per SM)
__global__ void report_errors_kernel(const int *error, PgeStats *stats)
{
    if (*error) stats->errors = 1;
}

void report_errors(const int *error, PgeStats *stats, cudaStream_t st) { report_errors_kernel<<<1, 1, 0, st>>>(error, stats); }

__global__ void set_mode_kernel(unsigned long long *slot, unsigned long long v) { *slot = v; }

int64_t droplet_slots() { return (int64_t)sm_count() * 1024; }

Layout layout(const PgeGrid &g)
{
    Layout L{};
    const long long NE = g.N + 2LL * g.H;
    L.ncell = (long long)g.F * NE * NE;
    L.nmetric = g.metric_shared ? NE * NE : L.ncell;
    L.nslots = droplet_slots();
    if (g.max_threads > 0 && g.max_threads < L.nslots) L.nslots = g.max_threads < 256 ? 256 : g.max_threads / 256 * 256;
    L.table_cap = ledger_table_cap(g.max_steps);
    L.table_slots = ledger_table_slots(g.max_steps);
    L.max_droplets = g.max_droplets;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o = align256(o + bytes);
        return at;
    };
    L.cellA = take(16 * L.ncell);
    L.cellB = take(16 * L.ncell);
    L.live = take(16 * L.ncell);
    L.metric8 = take(32 * L.nmetric);
    L.route2 = take(8 * L.ncell);
    L.acc4 = take(32 * L.ncell);
    L.pend = take(8 * L.ncell);
    if (!g.wave_tables) L.table_slots = 0;  // no own-change tables: ordered apply and map passes only
    L.tkey = take(8 * L.nslots * L.table_slots);
    L.town = take(8 * L.nslots * L.table_slots);
    L.counters = take(256);
    L.sortkeys = take(8 * L.max_droplets);
    L.sortvals = L.sortkeys;
    L.cdf = take(16 * L.ncell);
    L.cubtmp_bytes = cub_temp_bytes(L.ncell, L.max_droplets);
    L.cubtmp = take(L.cubtmp_bytes);
    L.partial = take(64 * 1024);
    L.thermal = take(40 * L.ncell);
    L.flags = take(8 * L.ncell);
    L.pwv = take(8 * L.ncell);                  // compacted values of a pairwise sum / the spawn weights' integers
    L.pwnode = take(pairwise_scratch_bytes());  // the pairwise sum's tree
    L.spread = take(8 * L.ncell);               // the brush: each cell's net change as last spread
    // ordered apply
    L.cap = change_list_cap(g.max_steps);
    L.max_wave = g.max_wave;
    L.wave_slots = L.max_wave * L.cap;
    const long long ws = L.wave_slots;
    L.w_cell = take(4 * ws);
    L.w_delta = take(8 * ws);
    L.w_vol = take(4 * ws);
    L.w_mom = take(8 * ws);
    L.w_count = take(8 * L.max_wave);
    L.w_death = take(L.max_wave);
    L.w_desc = take(16 * ws);
    L.w_keys0 = take(8 * ws);
    L.w_keys1 = take(8 * ws);
    L.w_vals0 = take(4 * ws);
    L.w_vals1 = take(4 * ws);
    L.w_runstart = take(4 * ws);
    L.w_segpos = take(4 * ws);
    L.w_runscan = take(4 * ws);
    L.w_segscan = take(4 * ws);
    L.w_temp_bytes = ordered_temp_bytes(ws, L.max_wave);
    L.w_temp = take(L.w_temp_bytes);
    L.w_dth = take(4 * L.max_wave);
    L.w_keep = take(8 * L.max_wave);
    L.w_act = take(8 * ws);
    L.w_park_n = take(4 * L.max_wave);
    L.w_park_k = take(4 * LAKE_PARKS * L.max_wave);
    L.w_park_rest = take(8 * LAKE_PARKS * L.max_wave);
    L.w_fin = take(8 * ws);
    L.w_offsets = take(8 * (L.max_wave + 1));
    L.hand = take(16 * L.ncell);
    L.terr = take(16 * L.ncell);
    L.error = take(256);
    L.total = o;
    return L;
}

namespace {
int run_waves(const PgeGrid *g, PgeState *s, const PgeSpawns *sp, const PgeParams *p, const double *ecap, PgeStats *stats,
              void *ws, const Layout &lay, cudaStream_t st, int32_t *rec_cell, double *rec_delta, float *rec_vol,
              float *rec_mom, int64_t *rec_count, int8_t *rec_death, const PgeTape *tape = nullptr)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.acc4), 0, 32 * lay.ncell, st)) != cudaSuccess) return cuda_fail(e, "memset acc");
    if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.pend), 0, 8 * lay.ncell, st)) != cudaSuccess) return cuda_fail(e, "memset pending");
    if (p->brush_radius > 0 && (e = cudaMemsetAsync(ws_ptr<void>(ws, lay.spread), 0, 8 * lay.ncell, st)) != cudaSuccess)
        return cuda_fail(e, "memset spread");
    if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.counters), 0, 16, st)) != cudaSuccess) return cuda_fail(e, "memset counters");
    // own-change tables: generation 0 everywhere (free); waves then use generations (w + 1) << 24 onwards
    const bool ledger_pass = p->apply == PGE_APPLY_WAVE || rec_cell != nullptr;
    if (ledger_pass && !g->wave_tables)
        return fail(PGE_E_WORKSPACE, "the wave apply and the change-list hook need a workspace built with wave_tables = 1");
    if (lay.table_slots &&
        (e = cudaMemsetAsync(ws_ptr<void>(ws, lay.tkey), 0, 8 * lay.nslots * lay.table_slots, st)) != cudaSuccess)
        return cuda_fail(e, "memset tables");
    pack(*g, *s, lay, ws, st);
    const long long P = sp->count;
    if (P > 0) {
        const int threads = p->threads_per_block ? p->threads_per_block : 256;
        // blocks_per_sm >= 2 selects the kernel variant compiled for two resident blocks per SM
        const int minb = p->blocks_per_sm >= 2 ? 2 : 1;
        if (s->route && (p->precision != PGE_PREC_F64 || tape))
            return fail(PGE_E_UNSUPPORTED, "the routing surface needs the float64 trace and no tape");
        if (s->roots && tape) return fail(PGE_E_UNSUPPORTED, "the adjoint's tape does not differentiate the roots");
        const bool lateral = p->lateral_rate > 0.0;
        if (lateral && (p->precision != PGE_PREC_F64 || tape))
            return fail(PGE_E_UNSUPPORTED, "the bank cut (lateral_rate) needs the float64 trace and no tape");
        const bool parks = s->lake_load != nullptr;
        if (parks) {
            if (!s->route || !s->lake_flag || !s->lake_id || !s->lake_room || s->lakes < 1)
                return fail(PGE_E_ARG, "lake parks (lake_load) need route, lake_flag, lake_id and lake_room (lakes >= 1)");
            if (p->apply != PGE_APPLY_ORDERED && !rec_cell)
                return fail(PGE_E_UNSUPPORTED, "lake parks count each lake's room down in droplet order: ordered apply only");
        }
        int bps = tape ? droplet_blocks_per_sm_f64_tape(threads)
                  : lateral ? droplet_blocks_per_sm_f64_lateral(threads, true, s->route != nullptr)
                  : s->route ? droplet_blocks_per_sm_f64_route(threads, true)
                  : p->precision == PGE_PREC_F64 ? droplet_blocks_per_sm_f64(threads, minb) : droplet_blocks_per_sm_f32(threads, minb);
        if (p->blocks_per_sm > 0 && p->blocks_per_sm < bps) bps = p->blocks_per_sm;
        long long maxblocks = (long long)sm_count() * bps;
        if (maxblocks * threads > lay.nslots) maxblocks = lay.nslots / threads;
        DropArgs a{};
        a.F = g->F;
        a.N = g->N;
        a.H = g->H;
        a.NE = g->N + 2 * g->H;
        a.spherical = g->spherical;
        a.deposit_on_exit = g->deposit_on_exit;
        a.metric_shared = g->metric_shared;
        a.A = ws_ptr<float4>(ws, lay.cellA);
        a.B = ws_ptr<float4>(ws, lay.cellB);
        a.L = ws_ptr<double2>(ws, lay.live);
        a.G = ws_ptr<float4>(ws, lay.metric8);
        a.mask = s->mask;
        a.ecap = p->use_erode_cap ? ecap : nullptr;
        a.sp_face = sp->face;
        a.sp_x = sp->x;
        a.sp_y = sp->y;
        a.sp_sed = sp->sed;
        a.sp_dir = sp->dir;
        a.volume0 = sp->volume0;
        a.erod = s->erodibility;
        a.R = s->route ? ws_ptr<float2>(ws, lay.route2) : nullptr;
        a.lakes = s->route && s->lake_flag ? 1 : 0;
        a.roots = s->roots;
        if (tape) a.tape = *tape;
        a.p = *p;
        a.acc4 = ws_ptr<long long>(ws, lay.acc4);
        a.pend = ws_ptr<long long>(ws, lay.pend);
        a.stats = stats;
        a.tkey = ws_ptr<unsigned long long>(ws, lay.tkey);
        a.town = ws_ptr<double>(ws, lay.town);
        a.table_mask = lay.table_slots ? (unsigned)(lay.table_slots - 1) : 0u;
        a.table_cap = (int)lay.table_cap;
        a.rec_cell = rec_cell;
        a.rec_delta = rec_delta;
        a.rec_vol = rec_vol;
        a.rec_mom = rec_mom;
        a.rec_count = rec_count;
        a.rec_death = rec_death;
        a.rec_cap = change_list_cap(list_steps(*p));
        a.rec_base = 0;
        a.ledger = 1;
        a.minb = minb;
        a.lanes = 32;
        // the exact pass and the change-list hook follow the reference's arithmetic; the order-free wave apply
        // (and its tape, which the adjoint reverses with the same functions) takes CUDA's own trig
        a.cr_trig = (p->apply == PGE_APPLY_ORDERED || rec_cell != nullptr) ? 1 : 0;
        a.parks = parks ? 1 : 0;
        a.park_n = a.park_k = nullptr;
        // the change-list hook with lake parks records the lists only: the rooms are counted by the ordered apply
        if (parks && rec_cell) a.ledger = 0;
        unsigned long long *ctr = ws_ptr<unsigned long long>(ws, lay.counters);
        const long long wave = p->wave;
        const long long nw = (P + wave - 1) / wave;
        if (p->apply == PGE_APPLY_ORDERED && !rec_cell) {
            // exact mode: record each wave's change lists, then apply them in droplet order
            if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.hand), 0, 16 * lay.ncell, st)) != cudaSuccess) return cuda_fail(e, "memset hand");
            if ((e = ordered_terrain(lay.ncell, ws_ptr<double2>(ws, lay.live), ws_ptr<float4>(ws, lay.cellB), s->mask,
                                     ws_ptr<CellTerr>(ws, lay.terr), st)) != cudaSuccess)
                return cuda_fail(e, "ordered terrain");
            if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.error), 0, 4, st)) != cudaSuccess) return cuda_fail(e, "memset error");
            a.ledger = 0;
            a.rec_cell = ws_ptr<int32_t>(ws, lay.w_cell);
            a.rec_delta = ws_ptr<double>(ws, lay.w_delta);
            a.rec_vol = ws_ptr<float>(ws, lay.w_vol);
            a.rec_mom = ws_ptr<float>(ws, lay.w_mom);
            a.rec_count = ws_ptr<int64_t>(ws, lay.w_count);
            a.rec_death = ws_ptr<int8_t>(ws, lay.w_death);
            a.rec_cap = (int)lay.cap;
            OrderedWave ow{};
            OrderedArgs &oa = ow.a;
            oa.cell = a.rec_cell;
            oa.delta = a.rec_delta;
            oa.vol = a.rec_vol;
            oa.mom = a.rec_mom;
            oa.count = a.rec_count;
            oa.cap = (int)lay.cap;
            oa.desc = ws_ptr<EntryDesc>(ws, lay.w_desc);
            oa.terr = ws_ptr<CellTerr>(ws, lay.terr);
            oa.L = a.L;
            oa.sediment = s->sediment;
            oa.A = ws_ptr<float4>(ws, lay.cellA);
            oa.B = ws_ptr<float4>(ws, lay.cellB);
            oa.R = s->route ? ws_ptr<float2>(ws, lay.route2) : nullptr;
            oa.lakes = a.lakes;
            oa.mask = s->mask;
            oa.ecap = a.ecap;
            oa.acc4 = ws_ptr<double>(ws, lay.acc4);
            oa.pend = ws_ptr<double>(ws, lay.pend);
            oa.hand = ws_ptr<double2>(ws, lay.hand);
            oa.dth = ws_ptr<int32_t>(ws, lay.w_dth);
            oa.keep = ws_ptr<double>(ws, lay.w_keep);
            oa.act = ws_ptr<double>(ws, lay.w_act);
            oa.p = *p;
            oa.stats = stats;
            oa.error = ws_ptr<int>(ws, lay.error);
            ParkWave pw{};
            if (parks) {
                a.park_n = ws_ptr<int32_t>(ws, lay.w_park_n);
                a.park_k = ws_ptr<int32_t>(ws, lay.w_park_k);
                oa.park_n = a.park_n;
                oa.park_rest = ws_ptr<double>(ws, lay.w_park_rest);
                pw.cap = (int)lay.cap;
                pw.cell = a.rec_cell;
                pw.delta = a.rec_delta;
                pw.park_n = a.park_n;
                pw.park_k = a.park_k;
                pw.lake_id = s->lake_id;
                pw.lake_room = s->lake_room;
                pw.lakes = s->lakes;
                pw.lake_load = s->lake_load;
                pw.rest = ws_ptr<double>(ws, lay.w_park_rest);
                // the cell sort's scan buffers are free until the wave's own ranks
                pw.keys_in = ws_ptr<uint32_t>(ws, lay.w_runstart);
                pw.keys_out = ws_ptr<uint32_t>(ws, lay.w_segpos);
                pw.vals_in = ws_ptr<int32_t>(ws, lay.w_runscan);
                pw.vals_out = ws_ptr<int32_t>(ws, lay.w_segscan);
                pw.temp = ws_ptr<void>(ws, lay.w_temp);
                pw.temp_bytes = lay.w_temp_bytes;
            }
            ow.cap = (int)lay.cap;
            // sort keys: the cell, cbits wide; all ones marks a slot past its list's end
            int cbits = 0;
            while ((1LL << cbits) < lay.ncell + 1) cbits++;
            ow.end_bit = cbits;
            ow.invalid = (1ull << cbits) - 1ull;
            ow.keys_in = ws_ptr<unsigned long long>(ws, lay.w_keys0);
            ow.keys_out = ws_ptr<unsigned long long>(ws, lay.w_keys1);
            ow.vals_in = ws_ptr<int32_t>(ws, lay.w_vals0);
            ow.vals_out = ws_ptr<int32_t>(ws, lay.w_vals1);
            ow.runstart = ws_ptr<int32_t>(ws, lay.w_runstart);
            ow.segpos = ws_ptr<int32_t>(ws, lay.w_segpos);
            ow.runscan = ws_ptr<int32_t>(ws, lay.w_runscan);
            ow.segscan = ws_ptr<int32_t>(ws, lay.w_segscan);
            ow.temp = ws_ptr<void>(ws, lay.w_temp);
            ow.temp_bytes = lay.w_temp_bytes;
            ow.fin_kp = ws_ptr<double>(ws, lay.w_fin);
            ow.offsets = lay.cap >= COMPACT_CAP ? ws_ptr<long long>(ws, lay.w_offsets) : nullptr;
            oa.lanes = p->apply_lanes > 0 ? p->apply_lanes : 1;
            ow.max_blocks = (long long)sm_count() * ordered_blocks_per_sm(oa.lanes);
            const long long rec_warps =
                (long long)sm_count() * (lateral ? droplet_blocks_per_sm_f64_lateral(32, false, s->route != nullptr)
                                         : s->route ? droplet_blocks_per_sm_f64_route(32, false)
                                         : p->precision == PGE_PREC_F64 ? droplet_blocks_per_sm_f64(32, 1, false)
                                                                      : droplet_blocks_per_sm_f32(32, 1, false));
            // the plain float64 record-only trace also comes in a 128-register build: more warps resident,
            // so a wave that fits runs one droplet per warp (no lane waits on another droplet's branches)
            const bool plain64 = !lateral && !s->route && p->precision == PGE_PREC_F64;
            const long long rec_warps_lean = plain64 ? (long long)sm_count() * droplet_blocks_per_sm_f64(32, 2, false) : 0;
            int ebits = 1;
            while ((1LL << ebits) <= wave) ebits++;
            long long ebase = 0;
            for (long long w = 0; w < nw; w++) {
                a.d_begin = w * wave;
                a.d_end = a.d_begin + wave < P ? a.d_begin + wave : P;
                a.rec_base = a.d_begin;
                a.counter = ctr + (w & 1);
                a.counter_next = ctr + ((w + 1) & 1);
                // a small wave is latency-bound: spread it over every SM (one or two warps each)
                // a wave's trace is latency-bound (each droplet is a serial chain of steps): give each
                // warp as few droplets as keeps every warp resident, so lanes do not wait on each
                // other's branches
                const long long nd = a.d_end - a.d_begin;
                long long lanes = p->trace_lanes > 0 ? p->trace_lanes : (nd + rec_warps - 1) / rec_warps;
                a.minb = 1;
                if (p->trace_lanes == 0 && plain64 && nd <= rec_warps_lean) {
                    lanes = 1;
                    a.minb = 2;
                }
                a.lanes = (int)(lanes < 1 ? 1 : (lanes > 32 ? 32 : lanes));
                const int tpb = 32;
                long long blocks = (nd + a.lanes - 1) / a.lanes;
                if (blocks * tpb > droplet_slots()) blocks = droplet_slots() / tpb;  // no tables: the GPU's resident threads
                e = p->precision == PGE_PREC_F64 ? launch_droplets_f64(a, (int)blocks, tpb, st)
                                                 : launch_droplets_f32(a, (int)blocks, tpb, st);
                if (e != cudaSuccess) return cuda_fail(e, "droplet kernel");
                ow.nw = nd;
                oa.nw = ow.nw;
                if (parks) {
                    pw.nw = nd;
                    if ((e = park_wave(pw, st)) != cudaSuccess) return cuda_fail(e, "lake parks");
                }
                // epochs step by 2^ebits > wave, so a counter never reaches the next wave's values;
                // they are 32-bit, and start over (counters zeroed) before they would wrap
                if (((unsigned long long)(w - ebase + 2) << ebits) >= (1ull << 32)) {
                    if ((e = hand_reset(lay.ncell, oa.hand, st)) != cudaSuccess) return cuda_fail(e, "hand reset");
                    ebase = w;
                }
                oa.epoch = (uint32_t)((unsigned long long)(w - ebase + 1) << ebits);
                if ((e = ordered_wave(ow, st)) != cudaSuccess) return cuda_fail(e, "ordered apply");
            }
            report_errors(ws_ptr<int>(ws, lay.error), stats, st);
            if ((e = cudaPeekAtLastError()) != cudaSuccess) return cuda_fail(e, "droplet pass");
            return PGE_OK;
        }
        for (long long w = 0; w < nw; w++) {
            a.d_begin = w * wave;
            a.d_end = a.d_begin + wave < P ? a.d_begin + wave : P;
            a.counter = ctr + (w & 1);
            a.counter_next = ctr + ((w + 1) & 1);
            if (tape) {  // the terrain this wave sees: the accumulator's terrain column as the wave starts
                e = cudaMemcpy2DAsync(tape->wave_acc + w * lay.ncell, sizeof(long long), ws_ptr<long long>(ws, lay.acc4),
                                      4 * sizeof(long long), sizeof(long long), lay.ncell, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return cuda_fail(e, "tape wave start");
            }
            // 2^24 droplet generations per thread and wave; after 255 waves the tables are cleared again
            if (w > 0 && w % 255 == 0) {
                if ((e = cudaMemsetAsync(ws_ptr<void>(ws, lay.tkey), 0, 8 * lay.nslots * lay.table_slots, st)) != cudaSuccess)
                    return cuda_fail(e, "memset tables");
            }
            a.gen_base = (unsigned long long)(w % 255 + 1) << 24;
            long long blocks = (a.d_end - a.d_begin + threads - 1) / threads;
            if (blocks > maxblocks) blocks = maxblocks;
            e = tape ? launch_droplets_f64_tape(a, (int)blocks, threads, st)
                     : p->precision == PGE_PREC_F64 ? launch_droplets_f64(a, (int)blocks, threads, st)
                                                    : launch_droplets_f32(a, (int)blocks, threads, st);
            if (e != cudaSuccess) return cuda_fail(e, "droplet kernel");
            if (p->brush_radius > 0) brush_spread(*g, *s, lay, ws, p->brush_radius, st);
            if (w + 1 < nw) refresh(*s, lay, ws, st);
        }
    }
    if ((e = cudaPeekAtLastError()) != cudaSuccess) return cuda_fail(e, "droplet pass");
    return PGE_OK;
}
}  // namespace
}  // namespace pge

using namespace pge;

extern "C" {

PGE_API int pge_version(void) { return PGE_VERSION; }

PGE_API int pge_last_error(char *buf, size_t n)
{
    const int len = (int)strlen(g_err);
    if (buf && n) {
        strncpy(buf, g_err, n - 1);
        buf[n - 1] = 0;
    }
    return len;
}

PGE_API size_t pge_workspace_bytes(const PgeGrid *g)
{
    if (check_grid(g) != PGE_OK) return 0;
    return layout(*g).total;
}

PGE_API int pge_spawn_rain(const PgeGrid *g, const PgeState *s, const double *u, const double *off, int64_t count, PgeSpawns *sp,
                   double *total_dev, int64_t *nspawnable_dev, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    if (!s->precip || !u || !off || !sp || !sp->face || !sp->x || !sp->y || !sp->sed || !sp->dir || !total_dev)
        return fail(PGE_E_ARG, "spawn_rain: NULL pointer");
    if (count < 1 || count > g->max_droplets) return fail(PGE_E_ARG, "spawn count %lld outside 1..%lld", (long long)count, (long long)g->max_droplets);
    cudaError_t e = spawn_rain(*g, *s, lay, ws, u, off, count, *sp, total_dev, reinterpret_cast<long long *>(nspawnable_dev),
                               (cudaStream_t)stream);
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "spawn_rain");
}

PGE_API int pge_count_pending(const PgeGrid *g, const PgeState *s, int64_t *count_dev, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    cudaError_t e = count_pending(*g, *s, lay, ws, reinterpret_cast<long long *>(count_dev), (cudaStream_t)stream);
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "count_pending");
}

PGE_API int pge_collect_pending(const PgeGrid *g, PgeState *s, PgeSpawns *sp, int64_t offset, PgeStats *stats, void *ws,
                        size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    if (!sp || !sp->face || !sp->x || !sp->y || !sp->sed || !stats) return fail(PGE_E_ARG, "collect_pending: NULL pointer");
    if (offset < 0 || offset > g->max_droplets) return fail(PGE_E_ARG, "collect_pending: bad offset");
    cudaError_t e = collect_pending(*g, *s, lay, ws, *sp, offset, stats, (cudaStream_t)stream);
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "collect_pending");
}

PGE_API int pge_trace_apply(const PgeGrid *g, PgeState *s, const PgeSpawns *sp, const PgeParams *p, const double *erode_cap,
                    PgeStats *stats, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s)) || (r = check_params(g, p))) return r;
    if (!sp || !stats) return fail(PGE_E_ARG, "trace_apply: NULL spawns or stats");
    if (sp->count < 0 || sp->count > g->max_droplets) return fail(PGE_E_ARG, "spawn count %lld outside 0..%lld", (long long)sp->count, (long long)g->max_droplets);
    if (sp->count > 0 && (!sp->face || !sp->x || !sp->y || !sp->sed || !sp->dir || !(sp->volume0 > 0.0)))
        return fail(PGE_E_ARG, "trace_apply: incomplete spawns");
    if (p->use_erode_cap && !erode_cap) return fail(PGE_E_ARG, "use_erode_cap without erode_cap");
    if (s->erodibility && p->apply != PGE_APPLY_WAVE)
        return fail(PGE_E_UNSUPPORTED, "a per-cell erodibility field needs the wave apply");
    cudaStream_t st = (cudaStream_t)stream;
    if ((r = run_waves(g, s, sp, p, erode_cap, stats, ws, lay, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr))) return r;
    const int exact = p->apply == PGE_APPLY_ORDERED;
    set_mode_kernel<<<1, 1, 0, st>>>(ws_ptr<unsigned long long>(ws, lay.counters) + 4, exact);
    fold_ema(*s, lay, ws, p->ema, exact, st);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "fold_ema");
}

PGE_API int pge_trace_apply_tape(const PgeGrid *g, PgeState *s, const PgeSpawns *sp, const PgeParams *p, const PgeTape *tape,
                                 PgeStats *stats, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s)) || (r = check_params(g, p))) return r;
    if (!sp || !stats || !tape) return fail(PGE_E_ARG, "trace_apply_tape: NULL spawns, tape or stats");
    if (sp->count < 0 || sp->count > g->max_droplets)
        return fail(PGE_E_ARG, "spawn count %lld outside 0..%lld", (long long)sp->count, (long long)g->max_droplets);
    if (sp->count > 0 && (!sp->face || !sp->x || !sp->y || !sp->sed || !sp->dir || !(sp->volume0 > 0.0)))
        return fail(PGE_E_ARG, "trace_apply_tape: incomplete spawns");
    if (p->apply != PGE_APPLY_WAVE || p->precision != PGE_PREC_F64 || p->use_erode_cap)
        return fail(PGE_E_UNSUPPORTED, "the tape records a float64 wave-apply pass without the erode cap");
    if (!tape->state || !tape->bits || !tape->entry || !tape->count || !tape->wave_acc) return fail(PGE_E_ARG, "tape has a NULL array");
    if (p->brush_radius > 0) return fail(PGE_E_UNSUPPORTED, "the adjoint's tape does not differentiate the brush");
    const long long nw = (sp->count + p->wave - 1) / p->wave;
    if (tape->droplets < sp->count || tape->steps < p->max_steps || tape->entries < p->max_steps + SPREAD || tape->waves < nw)
        return fail(PGE_E_ARG, "tape too small: %lld rows x %d steps x %d entries x %lld waves for %lld droplets, max_steps %d, "
                    "%lld waves", (long long)tape->droplets, tape->steps, tape->entries, (long long)tape->waves,
                    (long long)sp->count, p->max_steps, nw);
    cudaStream_t st = (cudaStream_t)stream;
    if ((r = run_waves(g, s, sp, p, nullptr, stats, ws, lay, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, tape))) return r;
    set_mode_kernel<<<1, 1, 0, st>>>(ws_ptr<unsigned long long>(ws, lay.counters) + 4, 0ull);
    fold_ema(*s, lay, ws, p->ema, 0, st);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "trace_apply_tape");
}

PGE_API int pge_adjoint_pass(const PgeGrid *g, const PgeState *s, const PgeSpawns *sp, const PgeParams *p, const PgeTape *tape,
                             int32_t carry_path, const double *zbar_after, double *zbar_before, double *ebar, double *pbar,
                             PgeStats *stats, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s)) || (r = check_params(g, p))) return r;
    if (!sp || !tape || !zbar_after || !zbar_before || !pbar) return fail(PGE_E_ARG, "adjoint_pass: NULL pointer");
    if (zbar_after == zbar_before) return fail(PGE_E_ARG, "adjoint_pass: zbar_before must not alias zbar_after");
    if (!tape->state || !tape->bits || !tape->entry || !tape->count || !tape->wave_acc || tape->droplets < sp->count ||
        tape->steps < p->max_steps || tape->entries < 1 || tape->waves < (sp->count + p->wave - 1) / p->wave)
        return fail(PGE_E_ARG, "adjoint_pass: the tape does not cover the pass");
    if (sp->count > 0 && !(sp->volume0 > 0.0)) return fail(PGE_E_ARG, "adjoint_pass: volume0 must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = adjoint_pass(*g, *s, *sp, *p, *tape, carry_path, zbar_after, zbar_before, ebar, pbar, lay, ws, st);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint_pass");
    adjoint_errors(lay, ws, stats, st);
    e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "adjoint_pass");
}

PGE_API int pge_route_flood(const PgeGrid *g, const PgeState *s, const int32_t *owner, double eps, double *route, int64_t max_sweeps,
                            int64_t *sweeps, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay))) return r;
    if (!s || !s->height || !s->sediment || !s->base || !owner || !route) return fail(PGE_E_ARG, "route_flood: NULL pointer");
    if (!(eps >= 0.0) || max_sweeps < 1) return fail(PGE_E_ARG, "route_flood: eps must be >= 0 and max_sweeps >= 1");
    long long done = 0;
    cudaError_t e = route_flood(*g, *s, owner, eps, route, lay, ws, max_sweeps, &done, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "route_flood");
    if (sweeps) *sweeps = done;
    if (done < 0) return fail(PGE_E_UNSUPPORTED, "route_flood: not converged within %lld sweeps", (long long)max_sweeps);
    return PGE_OK;
}

PGE_API int pge_window_lakes(const PgeGrid *g, const PgeState *s, double min_depth, uint8_t *lake_flag, int64_t *lake_cells,
                             void *stream)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (!s || !s->height || !s->sediment || !s->route || !lake_flag) return fail(PGE_E_ARG, "window_lakes: NULL pointer");
    if (!(min_depth >= 0.0)) return fail(PGE_E_ARG, "window_lakes: min_depth must be >= 0");
    cudaError_t e = window_lakes(*g, *s, min_depth, lake_flag, lake_cells, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "window_lakes");
    return PGE_OK;
}

PGE_API int pge_lake_balance(const PgeGrid *g, const int32_t *owner, const float *metric, const float *cell_area, double cell_size_m,
                             const float *surface, const uint8_t *ocean, const float *precip, const float *pet, double lake_evap,
                             double land_evap, double min_depth, uint8_t *lake_flag, float *water, float *closed_level,
                             PgeLakeInfo *info)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (!g->spherical) return fail(PGE_E_UNSUPPORTED, "lake_balance: the planet's lakes (a window's come from pge_window_lakes)");
    if (!owner || !metric || !cell_area || !surface || !ocean || !precip || !pet || !lake_flag)
        return fail(PGE_E_ARG, "lake_balance: NULL pointer");
    if (!(cell_size_m > 0.0) || !(min_depth >= 0.0) || !(lake_evap >= 0.0) || !(land_evap >= 0.0))
        return fail(PGE_E_ARG, "lake_balance: cell_size_m must be > 0 and min_depth, lake_evap, land_evap >= 0");
    if (lake_balance_host(g->N, g->H, owner, metric, cell_area, cell_size_m, surface, ocean, precip, pet, lake_evap, land_evap,
                          min_depth, lake_flag, water, closed_level, nullptr, info) != 0)
        return fail(PGE_E_UNSUPPORTED, "lake_balance: a land cell has no flow direction (unreached by the flood)");
    return PGE_OK;
}

PGE_API int pge_lake_balance_fill(const PgeGrid *g, const int32_t *owner, const float *metric, const float *cell_area,
                                  double cell_size_m, const float *surface, const uint8_t *ocean, const float *precip,
                                  const float *pet, double lake_evap, double land_evap, double min_depth, uint8_t *lake_flag,
                                  float *water, float *closed_level, PgeLakeFill *fill, PgeLakeInfo *info)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (!g->spherical) return fail(PGE_E_UNSUPPORTED, "lake_balance_fill: the planet's lakes");
    if (!owner || !metric || !cell_area || !surface || !ocean || !precip || !pet || !lake_flag || !fill)
        return fail(PGE_E_ARG, "lake_balance_fill: NULL pointer");
    if (!fill->evap || !fill->centres || !fill->height || !fill->sediment || !fill->lake_load || !fill->lake_id || !fill->lay ||
        !fill->pending || !fill->lake_room || fill->lake_room_cap < 1)
        return fail(PGE_E_ARG, "lake_balance_fill: a NULL fill array or no lake_room entry");
    if (!(cell_size_m > 0.0) || !(min_depth >= 0.0) || !(lake_evap >= 0.0) || !(land_evap >= 0.0) || !(fill->grade >= 0.0) ||
        !(fill->rise >= 0.0))
        return fail(PGE_E_ARG, "lake_balance_fill: cell_size_m must be > 0 and min_depth, lake_evap, land_evap, grade, rise >= 0");
    const int rc = lake_balance_host(g->N, g->H, owner, metric, cell_area, cell_size_m, surface, ocean, precip, pet, lake_evap,
                                     land_evap, min_depth, lake_flag, water, closed_level, fill, info);
    if (rc == -1) return fail(PGE_E_UNSUPPORTED, "lake_balance_fill: a land cell has no flow direction (unreached by the flood)");
    if (rc == -2) return fail(PGE_E_ARG, "lake_balance_fill: more lakes take load than lake_room_cap (%lld)", (long long)fill->lake_room_cap);
    return PGE_OK;
}

PGE_API int pge_window_lake_balance(const PgeGrid *g, const float *surface, const uint8_t *active, const float *precip,
                                    const float *evap, double lake_evap, double min_depth, double *route, uint8_t *lake,
                                    int64_t *counts)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (g->spherical || g->F != 1) return fail(PGE_E_UNSUPPORTED, "window_lake_balance: a window (F = 1, not spherical)");
    if (!surface || !active || !precip || !evap || !route || !lake) return fail(PGE_E_ARG, "window_lake_balance: NULL pointer");
    if (!(lake_evap > 0.0) || !(min_depth >= 0.0)) return fail(PGE_E_ARG, "window_lake_balance: lake_evap must be > 0, min_depth >= 0");
    window_lake_balance_host(g->N + 2 * g->H, surface, active, precip, evap, lake_evap, min_depth, route, lake, counts);
    return PGE_OK;
}

PGE_API int pge_basin_fill(const PgeGrid *g, const int32_t *owner, const float *surface, const uint8_t *ocean, double step,
                           double min_depth, double *add, uint8_t *basin, int64_t *basin_cells)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (!g->spherical) return fail(PGE_E_UNSUPPORTED, "basin_fill: a global (spherical) pass");
    if (!owner || !surface || !ocean || !add) return fail(PGE_E_ARG, "basin_fill: NULL pointer");
    if (!(step >= 0.0) || !(min_depth >= 0.0)) return fail(PGE_E_ARG, "basin_fill: step and min_depth must be >= 0");
    basin_fill_host(g->N, g->H, owner, surface, ocean, step, min_depth, add, basin, basin_cells);
    return PGE_OK;
}

PGE_API int pge_sea_base(const PgeGrid *g, const PgeState *s, const int32_t *owner, const float *area, double min_area, double *base,
                         int32_t *labels, int64_t max_sweeps, int64_t *sweeps, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay))) return r;
    if (!g->spherical) return fail(PGE_E_UNSUPPORTED, "sea_base: the sea mask is a global (spherical) pass");
    if (!s || !s->height || !s->sediment || !owner || !area || !base) return fail(PGE_E_ARG, "sea_base: NULL pointer");
    if (max_sweeps < 1) return fail(PGE_E_ARG, "sea_base: max_sweeps must be >= 1");
    long long done = 0;
    cudaError_t e = sea_base(*g, *s, owner, area, min_area, base, labels, lay, ws, max_sweeps, &done, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "sea_base");
    if (sweeps) *sweeps = done;
    if (done < 0) return fail(PGE_E_UNSUPPORTED, "sea_base: labelling not converged within %lld sweeps", (long long)max_sweeps);
    return PGE_OK;
}

PGE_API int pge_glacial(const PgeGrid *g, PgeState *s, uint8_t *ice_prev, double glacial_rate, double glacial_max, int32_t glacial_ramp,
                        double ice_evap, double disc_saturation, double moraine_frac, double iter_deposit, double *stats, void *ws,
                        size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    if (!stats) return fail(PGE_E_ARG, "glacial: NULL stats");
    GlacialArgs ga;
    ga.rate = glacial_rate;
    ga.cap = glacial_max;
    ga.ramp = glacial_ramp;
    ga.ice_evap = (float)ice_evap;
    ga.sat = disc_saturation > 1e-9 ? disc_saturation : 1e-9;
    ga.dep_floor = 0.02;
    ga.moraine_frac = moraine_frac;
    ga.iter_deposit = iter_deposit;
    const int e = glacial(*g, *s, ice_prev, ga, stats, lay, ws, (cudaStream_t)stream);
    return e == 0 ? PGE_OK : cuda_fail((cudaError_t)(-e), "glacial");
}

PGE_API int pge_halo_adjoint(const PgeHalo *h, double *zbar, void *stream)
{
    if (!h || !zbar || (h->K > 0 && (!h->dst || !h->src || !h->w))) return fail(PGE_E_ARG, "halo_adjoint: NULL pointer");
    halo_adjoint(*h, zbar, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "halo_adjoint");
}

PGE_API int pge_trace_changelist(const PgeGrid *g, PgeState *s, const PgeSpawns *sp, const PgeParams *p, int32_t *cl_cell,
                         double *cl_delta, float *cl_vol, float *cl_mom, int64_t *cl_count, int8_t *cl_death,
                         PgeStats *stats, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s)) || (r = check_params(g, p))) return r;
    if (!sp || !stats || !cl_cell || !cl_delta || !cl_vol || !cl_mom || !cl_count || !cl_death)
        return fail(PGE_E_ARG, "trace_changelist: NULL pointer");
    if (sp->count < 1 || sp->count > g->max_droplets) return fail(PGE_E_ARG, "spawn count outside 1..max_droplets");
    r = run_waves(g, s, sp, p, nullptr, stats, ws, lay, (cudaStream_t)stream, cl_cell, cl_delta, cl_vol, cl_mom, cl_count, cl_death);
    if (r) return r;
    set_mode_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(ws_ptr<unsigned long long>(ws, lay.counters) + 4, 0ull);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "trace_changelist");
}

PGE_API int pge_read_accumulators(const PgeGrid *g, double *acc, double *disch_track, double *mom_track, double *pending, void *ws,
                          size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay))) return r;
    read_accumulators(lay, ws, acc, disch_track, mom_track, pending, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "read_accumulators");
}

PGE_API int pge_thermal(const PgeGrid *g, PgeState *s, double thermal_rate, double creep_rate, double thermal_max, double talus_soft,
                double talus_hard, double dep_floor, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    // talus = soft + (hard - soft) * hardness in float32 (numpy types the product by the float32 field)
    const float soft = (float)talus_soft, diff = (float)(talus_hard - talus_soft);
    thermal(*g, *s, lay, ws, thermal_rate, creep_rate, thermal_max, soft, diff, dep_floor, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "thermal");
}

PGE_API int pge_slope_erode_cap(const PgeGrid *g, const PgeState *s, double coef, double exit_slope, double *erode_cap,
                                void *stream)
{
    int r;
    if ((r = check_shape(g)) || (r = check_state(s))) return r;
    if (!erode_cap) return fail(PGE_E_ARG, "erode_cap is NULL");
    // the reference's k = coef * sqrt(2) (its cell diagonal), taken on the host in float64
    slope_erode_cap(*g, *s, coef * sqrt(2.0), exit_slope, erode_cap, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "slope erode cap");
}

PGE_API int pge_smooth_step(const PgeGrid *g, const float *metric_inv, const float *sqrt_det, const double *in, double *out,
                            double kappa, int32_t keep, double cell_m, void *stream)
{
    int r;
    if ((r = check_shape(g))) return r;
    if (!g->spherical) return fail(PGE_E_UNSUPPORTED, "the isostasy smoother runs on the sphere only");
    if (!metric_inv || !sqrt_det || !in || !out) return fail(PGE_E_ARG, "smooth_step: NULL array");
    if (in == out) return fail(PGE_E_ARG, "smooth_step: in and out must differ (every cell reads its neighbours' old values)");
    if (!(cell_m > 0.0)) return fail(PGE_E_ARG, "smooth_step: cell size must be positive");
    smooth_step(*g, in, metric_inv, sqrt_det, kappa, keep ? 1 : 0, cell_m, out, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "smooth step");
}

PGE_API int pge_uplift(const PgeGrid *g, PgeState *s, double cap, double scale, void *ws, size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    if (!s->uplift) return fail(PGE_E_ARG, "uplift field is NULL");
    uplift(*g, *s, lay, ws, cap, scale, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "uplift");
}

PGE_API int pge_hold_datum(const PgeGrid *g, PgeState *s, double land_fraction, double level, double *shift_dev, void *ws,
                   size_t ws_bytes, void *stream)
{
    int r;
    Layout lay;
    if ((r = check_grid(g)) || (r = check_ws(g, ws, ws_bytes, lay)) || (r = check_state(s))) return r;
    if (!shift_dev) return fail(PGE_E_ARG, "shift_dev is NULL");
    hold_datum(*g, *s, lay, ws, land_fraction, level, shift_dev, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "hold_datum");
}

PGE_API int pge_halo_gather(const PgeHalo *h, double *field, int32_t vector, void *stream)
{
    if (!h || !field || (h->K > 0 && (!h->dst || !h->src || !h->w || (vector && !h->rot))))
        return fail(PGE_E_ARG, "halo_gather: NULL pointer");
    halo_gather(*h, field, vector, (cudaStream_t)stream);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "halo_gather");
}

PGE_API int pge_crmath(int32_t op, int64_t n, const double *x, double *y, void *stream)
{
    if (op < 0 || op > 7 || n < 0 || (n > 0 && (!x || !y))) return fail(PGE_E_ARG, "crmath: bad op, size or pointer");
    cudaError_t e = launch_crmath(op, n, x, y, (cudaStream_t)stream);
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "crmath");
}

PGE_API int pge_crmath_host(int32_t op, int64_t n, const double *x, double *y)
{
    if (op < 0 || op > 3 || n < 0 || (n > 0 && (!x || !y))) return fail(PGE_E_ARG, "crmath_host: bad op, size or pointer");
    crmath_host(op, n, x, y);
    return PGE_OK;
}

PGE_API int pge_cubesphere_map(int32_t op, int64_t n, int32_t *face, double *uv, double *ab, double *xyz, void *stream)
{
    if (op < 0 || op > 2 || n < 0) return fail(PGE_E_ARG, "cubesphere_map: bad op or size");
    if (n > 0 && (!face || !uv || (op == 2 && !ab) || (op < 2 && !xyz))) return fail(PGE_E_ARG, "cubesphere_map: NULL pointer");
    cudaError_t e = launch_cubesphere(op, n, face, uv, ab, xyz, (cudaStream_t)stream);
    return e == cudaSuccess ? PGE_OK : cuda_fail(e, "cubesphere_map");
}

}  // extern "C"
