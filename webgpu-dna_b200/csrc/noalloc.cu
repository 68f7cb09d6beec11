// noalloc.cu -- direct SSB scoring that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host that runs under another
// framework's memory pool, or one held to a fixed device-memory budget.  For
// them this
// entry point runs the same scoring kernels as wgdna_score_direct on the
// caller's device buffers, with its scratch in a fixed array that every GPU
// loading this library holds until the process exits.  The first call on a
// device looks up the array's device address; make that call before any
// stream capture.
#include <cstring>
#include <mutex>

#include "scoring.cuh"

namespace wg {

// At most 4,194,304 rad_buf entries per call; 16.1 MB of scratch per device.
constexpr unsigned long long NOALLOC_MAX_ENTRIES = 1ull << 22;
constexpr unsigned long long NOALLOC_TILES = NOALLOC_MAX_ENTRIES / 1024;
constexpr size_t NA_INFO = 0;                                             // u32 per entry
constexpr size_t NA_LAST = NA_INFO + 4 * NOALLOC_MAX_ENTRIES;              // i64 per tile
constexpr size_t NA_CNT0 = NA_LAST + 8 * NOALLOC_TILES;                    // u32 per tile
constexpr size_t NA_CNT1 = NA_CNT0 + 4 * NOALLOC_TILES;                    // u32 per tile
constexpr size_t NA_CSIN = NA_CNT1 + 4 * NOALLOC_TILES;                    // i64 per tile
constexpr size_t NA_BASE = NA_CSIN + 8 * NOALLOC_TILES;                    // u64 per tile
constexpr size_t NA_U64 = NA_BASE + 8 * NOALLOC_TILES;                     // 8 x u64 results
constexpr size_t NOALLOC_BYTES = NA_U64 + 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_addr[256];   // device address of the array, per device ordinal

}  // namespace wg

using namespace wg;

extern "C" int wgdna_score_direct_noalloc(const float* d_rad, uint64_t rad_n, const float* d_fy, const float* d_fz,
                                          const float* d_rbb0, const float* d_rbb1, const wgdna_dna_info* dna,
                                          uint32_t lcg_state, uint8_t* d_hits, void* cuda_stream,
                                          wgdna_ssb_result* out) {
    if (!dna || !d_hits || !out || (!d_rad && rad_n) || !d_fy || !d_fz || !d_rbb0 || !d_rbb1) {
        wg_set_error("wgdna_score_direct_noalloc: NULL argument");
        return WGDNA_ERR_ARG;
    }
    if (rad_n > NOALLOC_MAX_ENTRIES) {
        wg_set_error("wgdna_score_direct_noalloc: rad_n %llu exceeds the %llu-entry limit of its fixed scratch; "
                     "split the list where consecutive entries differ and chain lcg_state / hits",
                     (unsigned long long)rad_n, NOALLOC_MAX_ENTRIES);
        return WGDNA_ERR_CAPACITY;
    }
    if (((uintptr_t)d_hits & 3u) != 0 || ((uintptr_t)d_rad & 15u) != 0) {
        wg_set_error("wgdna_score_direct_noalloc: hits must be 4-byte and rad 16-byte aligned");
        return WGDNA_ERR_ARG;
    }
    if ((unsigned long long)dna->n_bp * 2 >= (1ull << 29)) {
        wg_set_error("wgdna_score_direct_noalloc: DNA target too large");
        return WGDNA_ERR_CAPACITY;
    }
    int dev = 0;
    WG_CUDA_OK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) { wg_set_error("wgdna_score_direct_noalloc: device %d out of range", dev); return WGDNA_ERR_ARG; }
    unsigned char* base;
    {
        // one-time set-up per device, with that device current: the host-side
        // name of the array is not a device address, so ask the runtime for it
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                wg_set_error("wgdna_score_direct_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return WGDNA_ERR_CUDA;
            }
            g_noalloc_addr[dev] = (unsigned char*)p;
        }
        base = g_noalloc_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)cuda_stream;
    ScoreScratch sc;
    sc.info = (uint32_t*)(base + NA_INFO);
    sc.last_brk = (long long*)(base + NA_LAST);
    sc.cnt0 = (uint32_t*)(base + NA_CNT0);
    sc.cnt1 = (uint32_t*)(base + NA_CNT1);
    sc.cs_in = (long long*)(base + NA_CSIN);
    sc.base = (unsigned long long*)(base + NA_BASE);
    sc.u64 = (unsigned long long*)(base + NA_U64);
    sc.fib = nullptr;
    DnaDev d;
    d.fy = d_fy; d.fz = d_fz; d.rbb0 = d_rbb0; d.rbb1 = d_rbb1;
    d.x0 = dna->x0; d.rise = dna->rise; d.r_bb = dna->r_bb; d.spacing = dna->spacing_nm;
    d.grid_N = dna->grid_N; d.n_bp_per = dna->n_bp_per; d.n_bp = dna->n_bp;
    // launch_score clears the result counters (the only scratch that must start
    // at zero); the per-entry and per-tile scratch is fully rewritten
    WG_CUDA_OK(launch_score((const float4*)d_rad, nullptr, rad_n, d, 0.29, 0.15, 1, lcg_state, (uint32_t*)d_hits,
                            sc, s));
    unsigned long long u[8];
    WG_CUDA_OK(cudaMemcpyAsync(u, sc.u64, sizeof u, cudaMemcpyDeviceToHost, s));
    WG_CUDA_OK(cudaStreamSynchronize(s));
    memset(out, 0, sizeof *out);
    out->ssb = u[0]; out->ssb0 = u[1]; out->ssb1 = u[2]; out->candidates = u[3];
    unsigned long long draws = rad_n ? u[4] : 0;
    out->in_reach = draws;
    out->lcg_state = lcg_jump_host(lcg_state, draws);
    return WGDNA_OK;
}
