// chemgrid.cuh -- the grid-hash diffusion-reaction chemistry backend.
#pragma once
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace wg {

struct CgStep { float dt; uint32_t step; };

struct CgArgs {
    const float4* rad;       // the first n rad_buf entries
    uint32_t n, k0, k1;
    float4* pos;             // n: x, y, z, kind
    uint32_t* alive;         // n
    int* head;               // 2^23 bucket heads
    int* next;               // n
    uint32_t* prod;          // 2: H2O2, H2 made
    uint32_t* counts;        // 8 x 5: t = 0 and the 7 checkpoints
    CgStep* st;
};

struct CgGraphKey {
    float4* pos; uint32_t* alive; int* head; int* next; uint32_t* prod; uint32_t* counts; CgStep* st;
    uint32_t n, k0, k1;
};

constexpr uint32_t CG_HASH_SIZE = 8388608u;
constexpr uint32_t CG_CHEM_N = 8000000u;   // CHEM_N, src/physics/constants.ts:57

cudaError_t cg_run(const CgArgs& a, cudaStream_t s, cudaGraphExec_t* cache, CgGraphKey* key);

}  // namespace wg
