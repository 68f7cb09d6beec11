// common.cuh -- shared definitions of the CUDA path (device structs, errors).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/wgdna.h"

namespace wg {

// Error bits raised on the device (read back after each stage).
enum : uint32_t {
    DERR_QUEUE_WAIT = 1u << 0,     // a bounded wait for a queued secondary gave up
    DERR_IDLE_WAIT = 1u << 1,      // a warp waited too long for work / termination
    DERR_KEY_RANGE = 1u << 2,      // secondary index or sequence overflowed the key
    DERR_TRACK_SIZE = 1u << 3,     // a track exceeded the per-block capacity
    DERR_HEAP = 1u << 4,           // IRT event storage overflow
    DERR_SEG_SORT = 1u << 5,       // a rad_buf segment exceeded the sort capacity
};

// Default bounds of the device-side waits (wgdna_set_wait_limits changes them
// per context): a lane waiting for a queued secondary, a transport warp without
// work, a surrogate kernel waiting for its tensor-core step.
constexpr unsigned long long WG_QUEUE_WAIT_NS = 2000000000ull;   // 2 s
constexpr unsigned long long WG_IDLE_WAIT_NS = 30000000000ull;   // 30 s
constexpr unsigned long long WG_MMA_WAIT_NS = 1000000000ull;     // 1 s

// Cross-section tables (public/cross_sections.wgsl:9-72) in device memory.
struct Tables {
    // small tables, copied to shared memory by the transport kernel, in this order
    const float* small;            // see the S_* offsets
    const float2* xcw;             // 5 x (N_WE*N_WR) (Born CDF, energy transfer) pairs
    float log_xe0, inv_log_xe_step, log_xae0, inv_log_xae_step;
    uint32_t xn, n_ae, n_ac, n_we, n_wr, n_vib;
};

// offsets inside Tables::small (floats)
constexpr int XN_ = 100, NAE_ = 25, NAC_ = 25, NWE_ = 58, NWR_ = 250, NVIB_ = 38;
constexpr int S_XE = 0;
constexpr int S_XI = S_XE + XN_;
constexpr int S_XC = S_XI + XN_;
constexpr int S_XL = S_XC + XN_;
constexpr int S_XSF = S_XL + XN_;          // 5 x 100
constexpr int S_XEF = S_XSF + 5 * XN_;     // 5 x 100
constexpr int S_XAE = S_XEF + 5 * XN_;
constexpr int S_XAC = S_XAE + NAE_;        // 625
constexpr int S_XWE = S_XAC + NAE_ * NAC_;
constexpr int S_XVE = S_XWE + NWE_;
constexpr int S_XVS = S_XVE + NVIB_;
constexpr int S_XVMF = S_XVS + NVIB_;      // 38 x 9
constexpr int S_VIB = S_XVMF + NVIB_ * 9;  // 9
constexpr int S_GUIDE = S_VIB + 9;         // 5 x 58 x 16: Born CDF at breakpoints 0, 16, ..., 240
constexpr int GUIDES = 16;
constexpr int S_TOTAL = S_GUIDE + 5 * NWE_ * GUIDES;
constexpr int S_TOTAL_PAD = (S_TOTAL + 3) & ~3;

// Global state of one transport run (device memory, zeroed before the run).
// The counters that many warps update or poll each sit on their own 128-byte
// line so that polling one does not stall atomics on another.
struct __align__(128) Line32 { uint32_t v; uint32_t pad[31]; };
struct __align__(128) Line64 { unsigned long long v; unsigned long long pad[15]; };
struct DevState {
    uint32_t counters[8];      // primary.wgsl:24-35 semantics
    uint32_t sec_stats[8];     // secondary.wgsl sec_stats
    uint32_t dbg[8];           // primary.wgsl dbg (dbg[2] = escaped count)
    unsigned long long rad_drop;   // rad_buf entries dropped at capacity
    unsigned long long steps;      // electron steps taken
    double dep_f64;                // every deposit, f64
    uint32_t sec_drop;             // secondaries dropped at capacity
    uint32_t err;
    Line64 rad_next;               // rad_buf slots reserved (may exceed capacity)
    Line32 sec_tail;               // secondaries emitted (counters[6])
    Line32 sec_qtail;              // secondaries placed in the global queue
    Line32 sec_head;               // queued secondaries taken
    Line32 prim_next;              // primaries taken
    Line32 busy;                   // warps holding work
};

// One queued secondary (the Particle struct of primary.wgsl:14, with the
// primary id and emission index instead of the RNG state).
struct __align__(16) SecRec {
    float4 pe;        // x, y, z, E
    float4 dir;       // dx, dy, dz, (unused)
    uint4 meta;       // pid, sub, epoch (ready flag), 0
};

// A secondary waiting in a warp's shared-memory stash.
struct StashRec { float x, y, z, E, dx, dy, dz; uint32_t pid, sub; };

// Set-up that must happen once on every device that runs a kernel (constant
// memory, function attributes): run(f) calls f with the current device when it
// has not yet succeeded on that device.  Thread-safe; a failed f is retried.
struct DeviceOnce {
    std::mutex mu;
    unsigned long long done[4] = {0, 0, 0, 0};   // device ordinals 0..255
    template <class F> cudaError_t run(F f) {
        int d = 0;
        cudaError_t e = cudaGetDevice(&d);
        if (e != cudaSuccess) return e;
        if (d < 0 || d >= 256) return f();
        std::lock_guard<std::mutex> lk(mu);
        if ((done[d >> 6] >> (d & 63)) & 1ull) return cudaSuccess;
        e = f();
        if (e == cudaSuccess) done[d >> 6] |= 1ull << (d & 63);
        return e;
    }
};

// Elapsed time between two recorded events, or 0 when the runtime cannot
// time them; a failed query leaves no error pending for a later launch check.
inline float elapsed_ms(cudaEvent_t a, cudaEvent_t b, bool* ok = nullptr) {
    float ms = 0.0f;
    const bool good = cudaEventElapsedTime(&ms, a, b) == cudaSuccess;
    if (!good) { cudaGetLastError(); ms = 0.0f; }
    if (ok) *ok = good;
    return ms;
}

}  // namespace wg

#define WG_CUDA_OK(expr)                                                     \
    do {                                                                     \
        cudaError_t e_ = (expr);                                             \
        if (e_ != cudaSuccess) {                                             \
            wg_set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,          \
                         cudaGetErrorString(e_));                            \
            return WGDNA_ERR_CUDA;                                           \
        }                                                                    \
    } while (0)

void wg_set_error(const char* fmt, ...);
