// scoring.cuh -- arguments and launchers of the scoring kernels.
#pragma once
#include "common.cuh"

namespace wg {

struct DnaDev {
    const float *fy, *fz, *rbb0, *rbb1;
    double x0, rise, r_bb, spacing;
    uint32_t grid_N, n_bp_per, n_bp;
};

struct ScoreScratch {
    uint32_t* info;
    long long* last_brk;
    uint32_t *cnt0, *cnt1;
    long long* cs_in;
    unsigned long long* base;
    unsigned long long* u64;   // [0] ssb [1] ssb0 [2] ssb1 [3] cand [4] total draws
    uint32_t* fib;             // 3 per fibre
};

cudaError_t launch_score(const float4* rad, const uint32_t* alive, unsigned long long n, const DnaDev& d,
                         double r_d, double p, int dedupe, uint32_t s0, uint32_t* hits_words,
                         const ScoreScratch& sc, cudaStream_t s);
cudaError_t launch_cluster(const uint8_t* hits, const DnaDev& d, uint32_t n_fibers, uint32_t* out, cudaStream_t s);
uint32_t lcg_jump_host(uint32_t s, unsigned long long k);

}  // namespace wg
