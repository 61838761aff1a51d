// pge_ordered.cuh -- the droplet-ordered apply of one wave (pge_ordered.cu).
#pragma once
#include "pge_internal.cuh"

namespace pge {

// one entry of a wave's change lists as the ordered apply reads it (built by the rank kernel)
struct alignas(16) EntryDesc {
    int32_t cell;
    uint32_t dflags;  // D (distinct earlier droplets of the wave at the cell) | ENTRY_* flags
    double delta;
};
constexpr uint32_t ENTRY_D_MASK = 0xffffffu;
constexpr uint32_t ENTRY_LAST = 1u << 24;   // its droplet's last visit to the cell
constexpr uint32_t ENTRY_FIRST = 1u << 25;  // its droplet's first visit to the cell
constexpr uint32_t ENTRY_STEP = 1u << 26;   // a step entry (vol >= 0), not a final deposit
constexpr uint32_t ENTRY_PARK = 1u << 27;   // a lake park (vol -3): its cell is visited and handed on unchanged

// a cell's read-only terrain for the ordered apply (built once per pass)
struct alignas(16) CellTerr {
    double hs;        // height + sediment at the start of the pass
    float base;
    uint32_t active;  // 1: the cell's mask is PGE_MASK_ACTIVE
};

struct OrderedArgs {
    // the wave's change lists, `cap` slots per droplet
    const int32_t *cell;
    const double *delta;
    const float *vol;
    const float *mom;
    const int64_t *count;
    int cap;
    long long nw;
    const EntryDesc *desc;
    const CellTerr *terr;
    // terrain
    const double2 *L;  // x: height + sediment
    const double *sediment;
    float4 *A;
    float4 *B;
    float2 *R;  // packed routing surface (route, flag) or nullptr: flags follow the live surface
    int lakes;  // R's flags mark overflowing lakes: a lake bed is not eroded below its routing surface
    const uint8_t *mask;
    const double *ecap;
    // per cell: the live net change and the hand-off counter, one 16-byte word
    double2 *hand;
    uint32_t epoch;  // this wave's: a cell with D earlier visitors is free once its counter reads epoch + D
    int lanes;  // droplets per warp in the apply
    // per droplet: the stockpile cell (-1: none) and the amount it adds there
    int32_t *dth;
    double *keep;
    // per slot: the amount the entry actually eroded or deposited (its statistics are summed later)
    double *act;
    // float64 accumulators in serial order: (net change, discharge, momentum a, b) and the stockpile
    double *acc4;
    double *pend;
    PgeParams p;
    PgeStats *stats;
    int *error;
    // lake parks (nullptr: off): per droplet its park count, per park (LAKE_PARKS a droplet) the rest its lake
    // had no room for, added to the droplet's leftover load in list order
    const int32_t *park_n;
    const double *park_rest;
};

// the lake parks of one wave (erosion.lake_fill): each lake's room counted down in droplet order
struct ParkWave {
    long long nw;  // droplets of the wave
    int cap;
    const int32_t *cell;
    const double *delta;
    const int32_t *park_n, *park_k;  // per droplet its parks and their entry indices
    const int32_t *lake_id;          // per cell
    double *lake_room;               // per lake, counted down in place
    long long lakes;
    double *lake_load;               // per cell, the loads the lakes took
    double *rest;                    // out: per park the rest refused
    uint32_t *keys_in, *keys_out;
    int32_t *vals_in, *vals_out;
    int end_bit;
    void *temp;
    size_t temp_bytes;
};

// what each sorted slot adds to its cell, gathered in sorted order for the finish
struct FinishRows {
    float *v, *m0, *m1;  // step volume and momentum (0 unless a step of volume > 0 on an active cell)
    double *amt;         // the amount applied, negative for an erosion entry
    double *kp;          // the droplet's stockpile where this is its last visit to its stockpile cell, else -1
};

struct OrderedWave {
    OrderedArgs a;
    long long nw;
    int cap, end_bit;
    unsigned long long invalid;
    unsigned long long *keys_in, *keys_out;
    int32_t *vals_in, *vals_out, *runstart, *segpos, *runscan, *segscan;
    void *temp;
    size_t temp_bytes;
    long long max_blocks;
    double *fin_kp;  // one double a slot: the gathered stockpile amounts
    // long lists: the recorded entries compacted before the ranks (nullptr: every slot goes through them);
    // max_wave + 1 int64: each droplet's first entry, then the wave's total
    long long *offsets;
};

// the list length above which a wave's entries are compacted before their ranks (a host read a wave)
#ifndef PGE_COMPACT_CAP
#define PGE_COMPACT_CAP 512
#endif
constexpr int COMPACT_CAP = PGE_COMPACT_CAP;

size_t ordered_temp_bytes(long long nslots, long long max_wave);
cudaError_t park_wave(const ParkWave &pw, cudaStream_t st);
int ordered_blocks_per_sm(int lanes);  // resident blocks of the apply kernel per SM
cudaError_t ordered_wave(const OrderedWave &w, cudaStream_t st);
cudaError_t hand_reset(long long ncell, double2 *hand, cudaStream_t st);
cudaError_t ordered_terrain(long long ncell, const double2 *L, const float4 *B, const uint8_t *mask, CellTerr *terr, cudaStream_t st);

}  // namespace pge
