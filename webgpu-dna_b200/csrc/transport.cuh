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
    Tables tab;
    const float* E_prim;           // optional per-primary energy (NULL: be)
    float* results;
    uint32_t* dose;
    float4* rad;
    unsigned long long* key;
    SecRec* secq;
    DevState* st;
};

int transport_blocks(int device);
cudaError_t launch_transport(const TArgs& a, int blocks, cudaStream_t s);
cudaError_t launch_canon(const unsigned long long* key, const float4* rad, unsigned long long n, uint32_t np,
                         uint32_t* cnt, unsigned long long* off, uint32_t* cur, uint32_t* perm, float4* out,
                         uint32_t* err, cudaStream_t s);
cudaError_t launch_reduce(const float* results, uint32_t np, const uint32_t* dose, uint32_t nvox,
                          unsigned long long* out, cudaStream_t s);

}  // namespace wg
