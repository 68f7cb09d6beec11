// surrogate_api.cuh -- what the surrogate entry points need from a context.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

struct wgdna_ctx;

namespace wg {

struct SgState;

struct CtxView {
    int device;
    cudaStream_t stream;
    const float4* rad;                   // canonical rad_buf of the last transport
    const unsigned long long* seg_off;   // its per-track offsets
    uint32_t nseg;
    bool have_transport;
    const float* Eprim;                  // per-primary energies of that transport, or null
    float E0;                            // its energy otherwise
    SgState** sg;
    unsigned long long mma_ns;           // bound of a surrogate kernel's tensor-core wait
    bool mma_give_up_first;              // test switch: the first wait of a tile gives up at once
};

void sg_free(SgState* s);

}  // namespace wg

int ctx_view(wgdna_ctx* c, wg::CtxView* v);
