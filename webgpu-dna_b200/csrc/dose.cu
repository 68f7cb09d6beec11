// dose.cu -- dose-grid reductions (sumDoseEV and the projection sums of
// renderDoseProjection, src/scoring/dose.ts:13-85) and the dose-based
// scoring of src/scoring/ssb-dsb.ts: scoreDirectSSB (:227-283) and
// expectedDSBLocal (:285-334).  Per-site values are computed with the
// reference's f64 operations in its order (bit-identical lambda); the sums
// over sites are f64 reductions in another order than the reference's loop.
#include "dose.cuh"

namespace wg {

__global__ void k_dose_sum(const uint32_t* dose, uint64_t n, unsigned long long* out) {
    unsigned long long s = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        s += dose[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// axis 0: sum over z into [y][x]; axis 1: sum over x into [z][y]
__global__ void k_dose_proj(const uint32_t* dose, uint32_t vc, int axis, float* proj) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vc * vc) return;
    const uint32_t a = i / vc, b = i - a * vc;
    unsigned long long s = 0;
    for (uint32_t c = 0; c < vc; ++c)
        s += axis == 0 ? dose[((uint64_t)c * vc + a) * vc + b] : dose[((uint64_t)a * vc + b) * vc + c];
    proj[i] = (float)(double)s;
}

__global__ void k_voxel_ssb(DoseDna d, const uint32_t* dose, uint32_t vc, double box_nm, float* lambda,
                            double* direct) {
    const uint64_t nbp = (uint64_t)d.n_fibers * d.n_bp_per;
    const double vox_nm = (2 * box_nm) / vc;
    const double vox_vol = vox_nm * vox_nm * vox_nm;
    const double half = box_nm, inv_vox = 1 / vox_nm;
    const double r = 0.29;
    const double bb_vol_per_bp = (4.0 / 3) * 3.141592653589793 * r * r * r;
    const double K = ((bb_vol_per_bp / vox_vol) * 0.15) / 22;
    double acc = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nbp; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t fi = (uint32_t)(i / d.n_bp_per), b = (uint32_t)(i - (uint64_t)fi * d.n_bp_per);
        float l0 = 0.0f, l1 = 0.0f;
        const double bx = d.x0 + b * d.rise;
        const double vx = floor((bx + half) * inv_vox);
        if (!(vx < 0 || vx >= vc)) {
            const double fy = d.fy[fi], fz = d.fz[fi];
            const double y0 = fy + d.rbb0[2 * b], z0 = fz + d.rbb0[2 * b + 1];
            const double y1 = fy + d.rbb1[2 * b], z1 = fz + d.rbb1[2 * b + 1];
            const double vy0 = floor((y0 + half) * inv_vox), vz0 = floor((z0 + half) * inv_vox);
            const double vy1 = floor((y1 + half) * inv_vox), vz1 = floor((z1 + half) * inv_vox);
            if (vy0 >= 0 && vy0 < vc && vz0 >= 0 && vz0 < vc) {
                const double l = dose[(uint64_t)((vz0 * vc + vy0) * vc + vx)] / 100.0 * K;
                l0 = (float)l;
                acc += l;
            }
            if (vy1 >= 0 && vy1 < vc && vz1 >= 0 && vz1 < vc) {
                const double l = dose[(uint64_t)((vz1 * vc + vy1) * vc + vx)] / 10.0 * K;   // sic: /10 on strand 1
                l1 = (float)l;
                acc += l;
            }
        }
        lambda[i] = l0;
        lambda[nbp + i] = l1;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(direct, acc);
}

// one warp per fibre: densities s = (float)(lambda + hit), window of +-10 bp
__global__ void k_expected_dsb(DoseDna d, const float* lambda, const uint8_t* hits, double* out) {
    const int W = 10;
    const int lane = threadIdx.x & 31;
    const uint32_t fi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (fi >= d.n_fibers) return;
    const uint64_t nbp = (uint64_t)d.n_fibers * d.n_bp_per, base = (uint64_t)fi * d.n_bp_per;
    const int n_per = (int)d.n_bp_per;
    auto dens = [&](int strand, int b) -> float {
        const uint64_t k = strand * nbp + base + b;
        return (float)((double)lambda[k] + ((hits && hits[k] == 1) ? 1.0 : 0.0));
    };
    bool any0 = false, any1 = false;
    for (int b = lane; b < n_per; b += 32) { any0 |= dens(0, b) != 0.0f; any1 |= dens(1, b) != 0.0f; }
    if (!__any_sync(0xffffffffu, any0) || !__any_sync(0xffffffffu, any1)) return;
    double e = 0;
    for (int b = lane; b < n_per; b += 32) {
        const float s0 = dens(0, b);
        if (s0 == 0.0f) continue;
        double win = 0;
        const int lo = b - W < 0 ? 0 : b - W, hi = b + W > n_per - 1 ? n_per - 1 : b + W;
        for (int c = lo; c <= hi; ++c) win += dens(1, c);
        e += s0 * win;
    }
    for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if (lane == 0 && e != 0.0) atomicAdd(out, e);
}

cudaError_t launch_dose_sum(const uint32_t* dose, uint64_t n, unsigned long long* out, cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(out, 0, 8, s); if (me_ != cudaSuccess) return me_; }
    k_dose_sum<<<592, 256, 0, s>>>(dose, n, out);
    return cudaGetLastError();
}

cudaError_t launch_dose_projection(const uint32_t* dose, uint32_t vc, int axis, float* proj, cudaStream_t s) {
    k_dose_proj<<<(vc * vc + 255) / 256, 256, 0, s>>>(dose, vc, axis, proj);
    return cudaGetLastError();
}

cudaError_t launch_voxel_ssb(const DoseDna& d, const uint32_t* dose, uint32_t vc, double box_nm, float* lambda,
                             double* direct, cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(direct, 0, 8, s); if (me_ != cudaSuccess) return me_; }
    k_voxel_ssb<<<592, 256, 0, s>>>(d, dose, vc, box_nm, lambda, direct);
    return cudaGetLastError();
}

cudaError_t launch_expected_dsb(const DoseDna& d, const float* lambda, const uint8_t* hits, double* out,
                                cudaStream_t s) {
    { cudaError_t me_ = cudaMemsetAsync(out, 0, 8, s); if (me_ != cudaSuccess) return me_; }
    k_expected_dsb<<<(d.n_fibers * 32 + 127) / 128, 128, 0, s>>>(d, lambda, hits, out);
    return cudaGetLastError();
}

}  // namespace wg
