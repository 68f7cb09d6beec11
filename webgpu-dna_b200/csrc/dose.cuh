// dose.cuh -- reductions of the dose grid and the dose-based DNA scoring.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace wg {

struct DoseDna {
    const float *fy, *fz, *rbb0, *rbb1;
    uint32_t n_fibers, n_bp_per;
    double x0, rise;
};

cudaError_t launch_dose_sum(const uint32_t* dose, uint64_t n, unsigned long long* out, cudaStream_t s);
cudaError_t launch_dose_projection(const uint32_t* dose, uint32_t vc, int axis, float* proj, cudaStream_t s);
cudaError_t launch_voxel_ssb(const DoseDna& d, const uint32_t* dose, uint32_t vc, double box_nm, float* lambda,
                             double* direct, cudaStream_t s);
cudaError_t launch_expected_dsb(const DoseDna& d, const float* lambda, const uint8_t* hits, double* out,
                                cudaStream_t s);

}  // namespace wg
