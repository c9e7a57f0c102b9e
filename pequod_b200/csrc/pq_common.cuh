// pq_common.cuh -- shared device-side definitions for the pequod_b200 kernels.
//
// Device layout (one ensemble member): every field is node-shaped,
// [layer][j][i] with i fastest, i in [0, ii), j in [0, jj), a row pitch of
// `pitch` elements (a multiple of 32, so every row starts on a 256-byte
// boundary for doubles).  The reference's one-node halos are never read on a
// single rank (every stencil in qg3p_aux.F90 stays inside fa_*), so the
// device arrays hold the nodes only; host-side copies convert to and from the
// reference's (ii+2, jj+2, L) / FLUX_II / FLUX_JJ layouts.
//
// Face arrays use the same node shape:
//   ui, uimo, zeta_fi  at [l][j][a], a in [1, ii-1]: the face between nodes
//                      (a-1, j) and (a, j)  (reference FLUX_II index a+2)
//   uj, ujmo, zeta_fj  at [l][b][i], b in [1, jj-1]: the face between nodes
//                      (i, b-1) and (i, b)  (reference FLUX_JJ index b+2)
//
// The spectral scratch `spec` holds, for mode m and interior row j, the DST
// coefficient of wavenumber k (1..n, n = ii-2) at [m][j][k-1].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PQ_MAXL 8

namespace pq {

// Scalars that change during a run live on the device so that a captured
// CUDA graph can replay steps with an adaptive time step.
struct Scalars {
    double dt;         // current non-dimensional time step
    double tweight_a;  // CABARET time weights (qg3.F90:457-459)
    double tweight_u;
    double max_u;      // max |u| over the faces, from the last fused step
    double cfl;        // max_u * dt
    double psiC[PQ_MAXL];   // mass correction per mode; channel: coefficient of corr (wall i = 0)
    double psiC2[PQ_MAXL];  // channel: coefficient of corr2 (wall i = ii - 1)
    double ekin[PQ_MAXL];
    double epot;
    double model_time;  // advanced by dt at the end of every fused step
    // dt and time weights the last step ran with (dt above is already the
    // next step's when adaptive stepping is on); what the reference's state
    // holds after a step, since it adapts at the start of the next one.
    double dt_last, tweight_a_last, tweight_u_last;
    double diag_time;  // diagnostic_time: the summed dt of the steps in psi_av
};

// Device status bits (read by the host after a step).
enum StatusBits : int {
    ST_NAN_PSIC = 1,      // NaN psiC: the reference aborts (qg3p_aux.F90:504-510)
    ST_LARGE_PSIC = 2,    // |psiC| > 1e100: the reference warns (:511-517)
    ST_NAN_ENERGY = 4,    // NaN energy: the reference aborts (qg3p_diagnostics.F90:858-861)
    ST_SMALL_DT = 8,      // dt < 1e-6 after adaptation: the reference warns (qg3p_aux.F90:982-986)
    ST_MMA_TIMEOUT = 16,  // a bounded wait of the tensor-core DST ran out (its output is not valid)
};

// Per-member device descriptor.  Lives in device global memory (an array of
// these for a batch); kernels find their member from the CTA index.
struct Member {
    int ii, jj, L, pitch;
    int n;       // DST length, ii - 2
    int N;       // ii - 1, a power of two
    int M;       // N / 2, the complex FFT length
    int logM;
    long long lstride;  // elements per layer (pitch * jj)
    int bc_type;        // 1 partial slip, 2 no slip, 3 free slip
    int limiter;
    double alpha;       // partial-slip alpha (non-dimensional)
    double viscosity, visc_bot;
    double z2m[PQ_MAXL * PQ_MAXL];  // row-major [m][l]
    double m2z[PQ_MAXL * PQ_MAXL];  // row-major [l][m]
    double ss[PQ_MAXL], s1[PQ_MAXL], s2[PQ_MAXL], beta[PQ_MAXL];
    double h[PQ_MAXL];  // non-dimensional layer thicknesses
    double htot;
    double mean_scale;  // 1 / (g_ii_int * g_jj_int)
    // Helmholtz tables (shared between members of the same size)
    const double2* tw;      // [M]  exp(-2 pi i t / M)
    const double* was;      // [N/2] 2 sin(k pi / N), index k (0 unused)
    const double2* wsplit;  // [M]  exp(-2 pi i q / N)
    const double* wmean;    // [n]  2 * sum_i sin(i k pi / N), index k-1
    const float2* tw_f;     // FP32 copies of tw, wsplit, was (mixed path)
    const float2* wsplit_f;
    const float* was_f;
    int periodic;           // 1: channel periodic in j
    const double* pb;       // periodic_coefficients b, c of the channel,
    const double* pc;       //   [(m * jj + j) * n + k-1], j 0-based
    int mixed;              // 1: FP32 storage of the CABARET fields and the
                            // baroclinic spectral rows (see spec64)
    // Compressed tridiagonal pivots, per (mode, k): piv[off + p - 1] for
    // p < len, then the fixed point piv_fix.
    const int* piv_off;     // [L * n]
    const int* piv_len;     // [L * n]
    const double* piv;
    const double* piv_fix;  // [L * n]
    // Fields (FP64 path; the mixed path reinterprets the storage pointers).
    // Fields that the fused step reads at neighbour nodes or faces owned by
    // another CTA are ping-ponged: [cur] is read, [cur ^ 1] written.
    void* zeta_old[2];
    void* zeta;       // zeta after predictor and beta (input of the inversion)
    void* zeta_next;  // the same for the next step (written by the fused step)
    double* psi;
    void* res;             // corrector residual of the previous step (read by the predictor)
    void* res_out;         // this step's residual (written by the corrector); ping-ponged
                           // so that the previous step's stays readable
    void* res_beta;        // res_beta of this step
    void* res_beta_other;  // of the previous step (read by the predictor) or
                           // of the next step (written by the fused step)
    void* ui;         // written by the fused step, read by the next step's beta term
    void* uj;
    void* uimo[2];
    void* ujmo[2];
    void* zfi[2];
    void* zfj[2];
    void* rel;
    double* psi_other;  // leapfrog: the other time level's psi and rel
    void* rel_other;
    void* helm_io;    // in/out buffer of the stand-alone helm() entry point
    void* flux_i;
    void* flux_j;
    void* spec;
    double* spec64;   // barotropic-mode spectral rows of the mixed path (FP64)
    void* gbuf;       // mixed path with the tensor-core DST: baroclinic node rows (FP32),
                      // the DST's input (forward) and output (inverse)
    const double* corr;
    // Channel (momentum correction, correction_function_momentum): the second
    // correction function, the spectral weights of the two walls' mean PV
    // (per wavenumber), and per mode the inverse 2 x 2 wall matrix.
    const double* corr2;
    const double* wwall;       // [n]: wall i = 0; the other wall has (-1)^(k+1) times it
    const double* inv_corr_a;  // [L][4], column-major 2 x 2
    const double* wind;
    double* partials;     // [L * ntiles_tri]
    double* maxu_part;    // [ntiles_cab]
    unsigned int* counters;  // [4] last-block counters
    Scalars* sc;
    int* status;
    int ntiles_tri;       // tri_ctas(n, jj, L)
    int ntiles_cab;
    int cab_sh;           // output rows per warp of the fused CABARET sweep
    int cur;              // ping-pong parity for ui / zfi / zfj (host-managed)
    int adapt_dt;
    double target_cfl, max_dt, max_dt_increase;
    // Time average of psi (qg3.F90:672-680, 725): when psi_av is set, a step
    // whose model time after its first half increment exceeds av_threshold
    // (max_spin - start_time) adds dt * psi to psi_av (node-shaped like psi)
    // and dt to the scalars' diag_time.
    double* psi_av;
    double av_threshold;
    // The quad eddy covariances (qg3.F90:683-721) when on: 23 accumulator
    // fields node-shaped like psi, quad_stride doubles apart, in the
    // reference's output order.
    double* quad;
    long long quad_stride;
};

// Programmatic dependent launch: the step kernels are launched so that the
// next one may be scheduled while this one finishes.  pdl_wait() first waits
// until the predecessor has completed and its writes are visible (a no-op
// without the launch attribute); nothing is read or written before it.
// pdl_release() lets the successor be scheduled once every CTA of this grid
// has passed it: called after a CTA's main work, so that the successor's
// CTAs overlap only this grid's tail.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Whether the CABARET step now running accumulates the time average (model
// time after the step's first half increment, qg3.F90:656, 672).  Read by
// every CTA before the last one advances model_time.
__device__ __forceinline__ bool cab_average_gate(const Member& Mb) {
    return Mb.psi_av != nullptr && Mb.sc->model_time + 0.5 * Mb.sc->dt > Mb.av_threshold;
}

// Tridiagonal solve geometry: W warps of row chunks per wavenumber column,
// 8 / W columns per CTA of 256 threads (chosen so a lane's chunk stays
// short, and its column segments 32 bytes wide: measured on B200 against W
// one step up and down at 129..2049 rows; at 2049 rows W = 4 would read
// 16-byte segments, half a DRAM sector).
__host__ __device__ inline int tri_warps(int jj) {
    const int Mr = jj - 2;
    return Mr > 64 ? 2 : 1;
}
__host__ __device__ inline int tri_ctas(int n, int jj, int L) {
    const int KT = 8 / tri_warps(jj);
    return L * ((n + KT - 1) / KT);
}

// The descriptor of this CTA's member into shared memory dst (every thread
// takes part; the caller synchronises).  A context's own launches (use_one)
// carry their single member by value in the kernel's parameters, so the copy
// needs no global-memory round trip before the CTA's first real load (about
// 1-2 us per kernel at the step's sizes); grouped launches (batches, the
// server) read it from the device array through the CTA prefix sums.
__device__ __forceinline__ int find_member(const int* __restrict__ prefix, int nmem, int cta, int* local);
__device__ __forceinline__ void cta_member(Member& dst, const Member& one, int use_one,
                                           const Member* __restrict__ mems, const int* __restrict__ prefix,
                                           int nmem, int cta, int* local) {
    const Member* src;
    if (use_one) {
        *local = cta;
        src = &one;
    } else {
        src = mems + find_member(prefix, nmem, cta, local);
    }
    static_assert(sizeof(Member) % 8 == 0, "Member copies in 8-byte words");
    const int n = sizeof(Member) / 8;
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = s[t];
}

// Map a flat CTA index to (member, local CTA) given prefix sums.
__device__ __forceinline__ int find_member(const int* __restrict__ prefix, int nmem, int cta, int* local) {
    int lo = 0, hi = nmem - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= cta)
            lo = mid;
        else
            hi = mid - 1;
    }
    *local = cta - prefix[lo];
    return lo;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <typename T>
struct Cplx;
template <>
struct Cplx<double> {
    typedef double2 type;
    __device__ static double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Cplx<float> {
    typedef float2 type;
    __device__ static float2 make(float a, float b) { return make_float2(a, b); }
};

// Warp-level inclusive prefix sum.
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide reductions of n partial results that other CTAs wrote (the
// "last CTA finishes" pattern): every thread of the block takes part, the
// values are read through L2 (__ldcg: written by other SMs after their
// fence), and the result is valid in thread 0.  The sum has a fixed order
// (per-thread strided sums, warp butterflies, warps in order), so it does not
// depend on which CTA finished last.  red: shared scratch of blockDim/32.
__device__ __forceinline__ double block_max_l2(const double* p, int n, double* red) {
    double m = 0.0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) m = fmax(m, __ldcg(p + q));
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_sum_l2(const double* p, int n, long long stride, double* red) {
    double s = 0.0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) s += __ldcg(p + q * stride);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
    __syncthreads();
    return r;
}

// Relative vorticity at node (i, j) of layer l from zeta and psi
// (rel_from_zeta_and_psi) with the boundary condition of apply_rel_bc.
// ps(i, j, l) reads staged psi.  Corners take the j-boundary formula, which
// the reference applies last.
template <class PS>
__device__ __forceinline__ double rel_node(const Member& Mb, PS ps, double zeta, int i, int j, int l) {
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L;
    const bool bj = !Mb.periodic && (j == 0 || j == jj - 1), bi = (i == 0 || i == ii - 1);
    if (bj || bi) {
        if (Mb.bc_type == 3) return 0.0;
        int di = 0, dj = 0;
        if (bj)
            dj = (j == 0) ? 1 : -1;
        else
            di = (i == 0) ? 1 : -1;
        const double p0 = ps(i, j, l), p1 = ps(i + di, j + dj, l), p2 = ps(i + 2 * di, j + 2 * dj, l);
        if (Mb.bc_type == 1) {
            const double cff = Mb.alpha / (Mb.alpha + 3.0);
            return cff * (-3.5 * p0 + 4.0 * p1 - 0.5 * p2);
        }
        return 2.0 * (p1 - p0);
    }
    if (L == 1) return zeta;
    const double p = ps(i, j, l);
    if (l == 0) return zeta + Mb.s2[0] * (p - ps(i, j, 1));
    if (l == L - 1) return zeta + Mb.s1[l] * (p - ps(i, j, l - 1));
    return zeta + Mb.s1[l] * (p - ps(i, j, l - 1)) + Mb.s2[l] * (p - ps(i, j, l + 1));
}

// Boundary relative PV from rel and psi (update_zeta_bc).
template <class PS>
__device__ __forceinline__ double zeta_bc_node(const Member& Mb, PS ps, double rel, int i, int j, int l) {
    const int L = Mb.L;
    if (L == 1) return rel;
    const double p = ps(i, j, l);
    if (l == 0) return rel - Mb.s2[0] * (p - ps(i, j, 1));
    if (l == L - 1) return rel - Mb.s1[l] * (p - ps(i, j, l - 1));
    return rel - Mb.s1[l] * (p - ps(i, j, l - 1)) - Mb.s2[l] * (p - ps(i, j, l + 1));
}

}  // namespace pq
