// irt.cuh -- arguments and launchers of the IRT kernels.
#pragma once
#include "common.cuh"

namespace wg {

struct IrtConst {
    double sigma[9], sigma_eff[9], rc[9], kdif[9], kobs[9], prob[9], a_pdc[9], coth_sig[9];
    double acc_s[9], acc_c[9], acc_add[9];   // acceptance-radius bound (irt.cu r_acc)
    double kact[9];
    int type[9], nprod[9], prod0[9], prod1[9];
    int map[36];
    double D[6];
    double sig_oh, sig_h, sig_eaq, r_cut2;
};

struct IArgs {
    const float4* rad;
    const unsigned long long* seg_off;   // nseg + 1
    uint32_t nseg, k0, k1, cap, ecap, nwarps;
    uint32_t pid_base;                   // global id of segment 0
    double *px, *py, *pz, *tb;           // [warp][cap]
    int8_t* sp;
    uint8_t* alive;
    uint16_t* lst;                       // [warp][6][cap]: alive particles of each species
    uint16_t* lpos;                      // [warp][cap]: position of a particle in its list
    double* ev_t;                        // [warp][2*ecap]: initial events, then heap overflow
    uint32_t* ev_ab;                     // packed (a << 16) | b
    uint32_t* track_next;
    double* acc_tl;                      // 35
    unsigned long long* acc;             // [0..8] rxn, 9 reacted, 10 pairs, 11 events, 12 tracks
    uint32_t* err;
};

cudaError_t irt_set_constants(const IrtConst& c);
int irt_blocks(int device);
cudaError_t launch_irt(const IArgs& a, int blocks, cudaStream_t s);
cudaError_t launch_group_keys(const float4* rad, unsigned long long n, unsigned long long* key, uint32_t* maxpid,
                              cudaStream_t s);
cudaError_t launch_seg_max(const unsigned long long* off, uint32_t nseg, unsigned long long* out, cudaStream_t s);

}  // namespace wg
