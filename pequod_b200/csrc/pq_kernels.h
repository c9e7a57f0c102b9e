// pq_kernels.h -- host-side launch interface of the device kernels.
#pragma once

#include <cuda_runtime.h>

#include "pq_common.cuh"

namespace pq {

// Everything one grouped launch needs: the device member array and, per
// kernel family, the CTA prefix sums over members (device arrays).
struct LaunchSet {
    const Member* members;  // device
    int nmem;
    int maxL, maxN, maxJ, maxI, maxPitch;
    const int* prefix_rows_interior;  // jj - 2 CTAs per member
    int ctas_rows_interior;
    const int* prefix_rows_all;       // jj CTAs per member
    int ctas_rows_all;
    const int* prefix_tri;            // L * ceil(n / 8) CTAs per member
    int ctas_tri;
    const int* prefix_cab;            // cabaret_ctas(ii, jj, L) CTAs per member
    int ctas_cab;
    int dst_group;                    // modes per DST CTA pass (0: automatic)
    int sm_count;                     // SMs of the device (persistent grids)
};


// pq_helm.cu
cudaError_t launch_dst_forward(const LaunchSet& ls, int prologue, cudaStream_t st);
cudaError_t launch_dst_inverse(const LaunchSet& ls, int epilogue, cudaStream_t st);
cudaError_t launch_tridiag(const LaunchSet& ls, int do_mean, cudaStream_t st);

// pq_cabaret.cu
// predict_next: also apply the next step's predictor + beta (fixed dt only)
cudaError_t launch_cabaret_fused(const LaunchSet& ls, int predict_next, cudaStream_t st);
int cabaret_ctas(int ii, int jj, int L, int sh);  // CTAs of k_cabaret_fused per member (band height sh)
cudaError_t launch_rel(const LaunchSet& ls, cudaStream_t st);
cudaError_t launch_energy(const LaunchSet& ls, cudaStream_t st);

}  // namespace pq
