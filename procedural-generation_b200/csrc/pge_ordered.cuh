// pge_ordered.cuh -- the droplet-ordered apply of one wave (pge_ordered.cu).
#pragma once
#include "pge_internal.cuh"

namespace pge {

struct OrderedArgs {
    // the wave's change lists, `cap` slots per droplet
    const int32_t *cell;
    const double *delta;
    const float *vol;
    const float *mom;
    const int64_t *count;
    int cap;
    long long nw;
    // per slot: distinct earlier droplets at the slot's cell, last visit of its droplet there
    const int32_t *D;
    const uint8_t *last;
    // terrain
    const double2 *L;  // x: height + sediment
    const double *sediment;
    float4 *A;
    float4 *B;
    const uint8_t *mask;
    const double *ecap;
    // per cell: the live net change and the hand-off counter, one 16-byte word
    double2 *hand;
    unsigned long long epoch;
    // per droplet: the stockpile cell (-1: none) and the amount it adds there
    int32_t *dth;
    double *keep;
    // float64 accumulators in serial order: (net change, discharge, momentum a, b) and the stockpile
    double *acc4;
    double *pend;
    PgeParams p;
    PgeStats *stats;
    int *error;
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
};

size_t ordered_temp_bytes(long long nslots);
int ordered_blocks_per_sm(int threads);
cudaError_t ordered_wave(const OrderedWave &w, cudaStream_t st);

}  // namespace pge
