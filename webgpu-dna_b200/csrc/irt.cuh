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
    // f32 prefilter bounds of r_acc (irt.cu pair_maybe): (s + add)(1+1e-6) + 1e-6,
    // add(1+1e-6) + 1e-6 and s c (1+1e-6)^2
    float fa0[9], fkb0[9], fk[9];
    float fs[9], fsc[9], fadd[9];        // acc_s, acc_s * acc_c, acc_add rounded up to f32
    double t16[16];                      // per-track curve times 10^(-3 + 0.4 k) ns
};

// the Philox4x32-10 key schedule: rk[2r], rk[2r+1] = the keys of round r
inline void philox_round_keys(uint32_t k0, uint32_t k1, uint32_t* rk) {
    for (int r = 0; r < 10; ++r) { rk[2 * r] = k0 + (uint32_t)r * 0x9E3779B9u; rk[2 * r + 1] = k1 + (uint32_t)r * 0xBB67AE85u; }
}

struct IArgs {
    const float4* rad;
    const unsigned long long* seg_off;   // nseg + 1
    uint32_t nseg, k0, k1, pid_base;
    // the Philox key schedule (k0 + r W0, k1 + r W1 for rounds r = 0..9), so the
    // pairing kernel's Philox takes its round keys from the parameter bank
    uint32_t rk[20];
    // per-track storage (irt.cu tbase / ebase)
    double *px, *py, *pz, *tb;
    int8_t* sp;
    uint8_t* alive;
    uint16_t* lst;                       // 6 lists per track: alive particles of each species
    uint16_t* lpos;                      // position of a particle in its list
    float4* rec;                         // the lists' records: f32 shadow x, y, z and birth time
    float4* pf;                          // f32 shadow (x, y, z relative to the track origin; w: species bits)
    float* tdel;                         // per track: bound on the shadow's distance error (nm)
    double* ev_t;                        // initial events of each track
    uint32_t* ev_ab;                     // packed (a << 16) | b
    uint32_t *tn, *th2, *ttiles, *tev, *tlc;   // per track: particles, H2 markers, tiles, events, 6 list lengths
    unsigned long long* toff;            // nseg + 1: prefix of ttiles
    uint32_t* order;                     // nseg: tracks in the order the event kernel takes them
    // per-warp heap overflow of the event kernel
    double* hov_t;
    uint32_t* hov_ab;
    uint32_t hcap;
    uint32_t* counters;                  // [0] load, [1] init items, [2] loop tracks, [3] largest track
    double* acc_tl;                      // 35
    unsigned long long* acc;             // [0..8] rxn, 9 reacted, 10 pairs, 11 events, 12 tracks
    float* curves;                       // optional: per track 16 x 5 counts (OH, eaq, H, H2O2, H2)
    uint32_t* err;
};

cudaError_t irt_set_constants(const IrtConst& c);
// Resident blocks per SM of the pairing and event kernels: as many as fit, at
// most the given number (0 = no limit).  The heap overflow is sized per event
// warp, so irt_warps and launch_irt must see the same limits.
struct IrtShape { uint32_t init_per_sm, loop_per_sm; };
int irt_warps(int device, const IrtShape& shape);
// ev (optional, 3 events): recorded after the load, the initial pairing and the sort
cudaError_t launch_irt(const IArgs& a, int device, const IrtShape& shape, cudaStream_t s, cudaEvent_t* ev = nullptr);
// A captured IRT launch sequence and what it was captured for (irt.cu irt_graph_run).
struct IrtGraphKey { IArgs a; IrtShape shape; int device; cudaEvent_t* ev; };
struct IrtGraph {
    cudaGraphExec_t exec = nullptr;
    IrtGraphKey key;
    bool off = false;                    // capturing failed once: plain launches from then on
};
cudaError_t irt_graph_run(const IArgs& a, int device, const IrtShape& shape, cudaStream_t s, cudaEvent_t* ev,
                          IrtGraph* g);
cudaError_t launch_group_keys(const float4* rad, unsigned long long n, unsigned long long* key, uint32_t* maxpid,
                              cudaStream_t s);
cudaError_t launch_seg_max(const unsigned long long* off, uint32_t nseg, unsigned long long* out, cudaStream_t s);

}  // namespace wg
