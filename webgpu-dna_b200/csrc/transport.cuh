// transport.cuh -- arguments and launchers of the transport kernels.
#pragma once
#include "common.cuh"

namespace wg {

struct TArgs {
    uint32_t np;
    float box, ce;
    uint32_t ms;
    float be;
    uint32_t vc, max_sec;
    unsigned long long max_rad;
    float start_half;
    uint32_t dna_enable, dna_grid_n;
    float dna_rise, dna_spacing, dna_x0, dna_r_bb;
    uint32_t sec_steps, k0, k1, epoch, pid_base;
    uint32_t pub_epoch;            // epoch written when a queued record is published (= epoch)
    unsigned long long ready_ns;   // bound of a lane's wait for a queued record
    unsigned long long idle_ns;    // bound of a warp's wait without work
    // scheduling (results do not depend on it): primaries a warp may start per
    // iteration, secondaries a warp keeps after spilling its stash and the
    // stash level that spills (0: every secondary goes to the global queue),
    // and the queue poll period of a busy warp (iterations - 1, a power of two - 1)
    uint32_t prim_take, stash_keep, stash_spill, poll_mask;
    Tables tab;
    const float* E_prim;           // optional per-primary energy (NULL: be)
    float* results;
    uint32_t* dose;
    float4* rad;
    unsigned long long* key;
    SecRec* secq;
    DevState* st;
};

// resident CTAs of the transport kernel on `device`: per SM as many as fit,
// at most ctas_per_sm (0 = no limit)
int transport_blocks(int device, uint32_t ctas_per_sm);
constexpr uint32_t TRANSPORT_STASH = 48;   // stash capacity per warp (records)
cudaError_t launch_transport(const TArgs& a, int blocks, cudaStream_t s);
cudaError_t launch_canon(const unsigned long long* key, const float4* rad, unsigned long long n, uint32_t np,
                         uint32_t* cnt, unsigned long long* off, uint32_t* cur, uint32_t* perm, float4* out,
                         uint32_t* err, cudaStream_t s);
cudaError_t launch_reduce(const float* results, uint32_t np, const uint32_t* dose, uint32_t nvox,
                          unsigned long long* out, cudaStream_t s);

}  // namespace wg
