// pge_maps.cuh -- host-side launchers of the map passes (pge_maps.cu).
#pragma once
#include "pge_internal.cuh"

namespace pge {
void pack(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, cudaStream_t st);
void refresh(const PgeState &s, const Layout &lay, void *ws, cudaStream_t st);
void fold_ema(PgeState &s, const Layout &lay, void *ws, double ema, int exact, cudaStream_t st);
void read_accumulators(const Layout &lay, void *ws, double *acc, double *dtr, double *mtr, double *pending, cudaStream_t st);
void thermal(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double rate, double creep_rate, double cap, float soft,
             float diff, double dep_floor, cudaStream_t st);
void thermal_on_scratch(const PgeGrid &g, PgeState &s, double *tb, long long n, double rate, double creep_rate, double cap,
                        float soft, float diff, double dep_floor, cudaStream_t st);
void uplift(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double cap, double scale, cudaStream_t st);
void hold_datum(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, double land_fraction, double level,
                double *shift_dev, cudaStream_t st);
void halo_gather(const PgeHalo &h, double *field, int vector, cudaStream_t st);
void slope_erode_cap(const PgeGrid &g, const PgeState &s, double k, double exit_slope, double *out, cudaStream_t st);
void smooth_step(const PgeGrid &g, const double *in, const float *metric_inv, const float *sqrt_det, double kappa, int keep,
                 double cell_m, double *out, cudaStream_t st);
size_t cub_temp_bytes(int64_t ncell, int64_t max_droplets);
// the erode / deposit brush (PgeParams.brush_radius): the net change the wave apply accumulated since the last call,
// spread over each cell's footprint in integer shares, added to the accumulators' net-change column
void brush_spread(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, int r, cudaStream_t st);
// numpy's pairwise float64 sum (mean = 1: divided by the count) of a[0, *count), on the stream
size_t pairwise_scratch_bytes();
void pairwise_sum(const double *a, const long long *count, void *scratch, double *out, int mean, cudaStream_t st);
// the planet's lake balance on the host (pge_lakes.cpp), with erosion.lake_fill's settle when fill is set; 0,
// -1 when a land cell has no flow direction, -2 when more lakes take load than fill->lake_room_cap
int lake_balance_host(int N, int H, const int32_t *owner, const float *metric, const float *cell_area, double cell_size_m,
                      const float *surface, const uint8_t *ocean, const float *precip, const float *pet, double lake_evap,
                      double land_evap, double min_depth, uint8_t *lake_flag, float *water, float *closed_level,
                      PgeLakeFill *fill, PgeLakeInfo *info);
// the evaporation balance of a window's lakes on the host (pge_lakes.cpp)
void window_lake_balance_host(int W, const float *surface, const uint8_t *active, const float *precip, const float *evap,
                              double lake_evap, double min_depth, double *route, uint8_t *lake, int64_t *counts);
// the basin fill of a fresh state on the host (pge_lakes.cpp)
void basin_fill_host(int N, int H, const int32_t *owner, const float *surface, const uint8_t *ocean, double step, double min_depth,
                     double *add, uint8_t *basin, int64_t *basin_cells);
// the lakes of a window (route deeper than min_depth over the surface on active interior cells)
cudaError_t window_lakes(const PgeGrid &g, const PgeState &st, double min_depth, uint8_t *flag, int64_t *count, cudaStream_t stream);
// routing surface (epsilon-filled priority flood); *sweeps_out < 0: not converged within max_sweeps
cudaError_t route_flood(const PgeGrid &g, const PgeState &st, const int32_t *owner, double eps, double *route, const Layout &lay,
                        void *ws, long long max_sweeps, long long *sweeps_out, cudaStream_t s);
// sea mask: base level of closed below-sea basins; *sweeps_out < 0: the labelling did not converge
cudaError_t sea_base(const PgeGrid &g, const PgeState &st, const int32_t *owner, const float *area, double min_area, double *base,
                     int32_t *label_out, const Layout &lay, void *ws, long long max_sweeps, long long *sweeps_out, cudaStream_t s);
// glacial pass (erosion/glacial.py:162-257), lengths in cell units; returns 0 or -cudaError
struct GlacialArgs {
    double rate, cap, sat, dep_floor, moraine_frac, iter_deposit;
    float ice_evap;
    int ramp;
};
int glacial(const PgeGrid &g, PgeState &st, uint8_t *ice_prev, const GlacialArgs &ga, double stats[5], const Layout &lay, void *ws,
            cudaStream_t s);
// the adjoint (pge_adjoint.cu)
cudaError_t adjoint_pass(const PgeGrid &g, const PgeState &s, const PgeSpawns &sp, const PgeParams &p, const PgeTape &tape,
                         int carry_path, const double *zbar_after, double *zbar_before, double *ebar, double *pbar,
                         const Layout &lay, void *ws, cudaStream_t st);
void adjoint_errors(const Layout &lay, void *ws, PgeStats *stats, cudaStream_t st);
void halo_adjoint(const PgeHalo &h, double *zbar, cudaStream_t st);
cudaError_t spawn_rain(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, const double *u, const double *off,
                       long long P, PgeSpawns &sp, double *total_dev, long long *nspawn_dev, cudaStream_t st);
cudaError_t count_pending(const PgeGrid &g, const PgeState &s, const Layout &lay, void *ws, long long *count_dev, cudaStream_t st);
cudaError_t collect_pending(const PgeGrid &g, PgeState &s, const Layout &lay, void *ws, PgeSpawns &sp, long long offset,
                            PgeStats *stats, cudaStream_t st);
}  // namespace pge
