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
    const Member* one = nullptr;  // host copy of a context's single member (passed by value to the
                                  // step kernels), null for grouped launches
    int maxL, maxN, maxJ, maxI, maxPitch;
    const int* prefix_rows_interior;  // jj - 2 CTAs per member
    int ctas_rows_interior;
    const int* prefix_rows_all;       // jj CTAs per member
    int ctas_rows_all;
    const int* prefix_tri;            // L * ceil(n / 8) CTAs per member
    int ctas_tri;
    const int* prefix_cab;            // cabaret_ctas(ii, jj, L) CTAs per member
    int ctas_cab;
    const int* prefix_dst[2];         // DST CTAs per member, forward [0] and inverse [1]
    int ctas_dst[2];                  //   (ceil(rows / dst_rows_per_cta) per member)
    int dst_group;                    // row groups per DST CTA (0: automatic)
    int dst_lanes[2];                 // lanes P per DST unit (values per lane M / P), forward [0] / inverse [1]
    int cab_kernel;                   // CABARET formulation: 0 tiles, 1 warp sweeps, 2 two-column sweeps (FP32)
    int periodic;                     // channel periodic in j: every row is transformed
    int sm_count;                     // SMs of the device (persistent grids)
    int pdl;                          // launch the step kernels with programmatic dependent launch
    int gemm_bc = 0;                  // mixed form: the row DSTs leave the baroclinic modes to the
                                      // tensor-core DST (node rows in Member::gbuf)
};

// The by-value member argument of a launch and whether the kernel uses it.
inline const Member& member_arg(const LaunchSet& ls) {
    static const Member none{};
    return ls.one ? *ls.one : none;
}
inline int member_arg_used(const LaunchSet& ls) { return (ls.one != nullptr && ls.nmem == 1) ? 1 : 0; }

// Launch `kernel` on `st`, with programmatic stream serialisation when pdl
// is set: the kernel may be scheduled before its predecessor in the stream
// has finished, and waits for it in pdl_wait_then_release().
template <typename... KArgs, typename... Args>
inline cudaError_t launch_step_kernel(int pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                      cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}


// pq_helm.cu
// Lanes per DST unit for complex length M = N/2 and L modes by default
// (dir 0 forward, 1 inverse), and rows per DST CTA for P lanes per unit and
// row-group setting c.
int dst_lanes_default(int M, int L, int dir);
int dst_lanes_batched(int M);
int dst_max_threads_host(int V);
int dst_rows_per_cta_host(int P, int c);
// f32: the mixed form (FP32 layer fields and baroclinic spectral rows)
cudaError_t launch_dst_forward(const LaunchSet& ls, int prologue, int f32, cudaStream_t st);
cudaError_t launch_dst_inverse(const LaunchSet& ls, int epilogue, int f32, cudaStream_t st);
cudaError_t launch_tridiag(const LaunchSet& ls, int do_mean, int f32, cudaStream_t st);

// pq_cabaret.cu
// predict_next: also apply the next step's predictor + beta (fixed dt only)
cudaError_t launch_cabaret_fused(const LaunchSet& ls, int predict_next, int f32, cudaStream_t st);
// The channel (periodic j) CABARET step after the inversion: four
// node-parallel kernels; channel_ctas is the last kernel's CTA count.
cudaError_t launch_cabaret_channel(const LaunchSet& ls, int f32, cudaStream_t st);
int channel_ctas(int ii, int jj);
// The quad eddy covariances of the step (before its CABARET kernel).
cudaError_t launch_quad(const LaunchSet& ls, int f32, int lf, cudaStream_t st);
// CTAs of the (persistent) sweep kernel per member: band height sh, nc
// columns per lane, FP32 fields when f32; at most the CTAs resident at once.
int cabaret_ctas(int ii, int jj, int L, int sh, int nc, bool f32);
// An upper bound of cabaret_ctas over every tuning with bands of at least min_sh rows.
int cabaret_ctas_bound(int ii, int jj, int L, int min_sh);
int cabaret_tile_ctas(int ii, int jj, int L);     // CTAs of the tile kernel per member
cudaError_t launch_rel(const LaunchSet& ls, int f32, cudaStream_t st);
cudaError_t launch_init_finish(const LaunchSet& ls, int f32, cudaStream_t st);
// pq_leapfrog.cu
cudaError_t launch_lf_step(const LaunchSet& ls, double ra_nu, double ra_alpha, cudaStream_t st);
cudaError_t launch_lf_forward_euler(const LaunchSet& ls, cudaStream_t st);
cudaError_t launch_lf_rel_bc(const LaunchSet& ls, int copy_old, int advance_time, cudaStream_t st);
cudaError_t launch_lf_average(const LaunchSet& ls, cudaStream_t st);
// Elementwise FP64 <-> FP32 copy of `count` values (to_f32: double -> float).
cudaError_t launch_convert(void* dst, const void* src, size_t count, int to_f32, cudaStream_t st);
cudaError_t launch_energy(const LaunchSet& ls, cudaStream_t st);

}  // namespace pq
