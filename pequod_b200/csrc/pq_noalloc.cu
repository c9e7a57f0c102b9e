// pq_noalloc.cu -- energy diagnostics that allocate no device memory.
//
// pq_energy (pq_api.cu) reduces per-row partial sums through scratch memory
// that the context allocated.  Some callers have no context and may not
// allocate: a host driver whose device memory is reserved up front (by an
// HBM budget, or by a caching allocator that owns the whole device) and
// that hands this library only the arrays it already owns, so that a
// cudaMalloc would fail or break the budget; or a driver that keeps its
// streams pipelined and cannot afford the device-wide synchronisation a
// cudaMalloc / cudaFree may cause.  For them this file provides the same
// reduction with its scratch in a fixed, file-scope device array.
//
// The array (below) holds PQ_NOALLOC_MAX_JJ rows of PQ_MAX_LAYERS + 1 partial
// sums plus a completion counter, about 300 KB; every GPU that loads the
// library keeps it until the process exits.  All calls share it: calls whose
// device work overlaps (different streams, or different host threads on one
// device) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "pequod_b200.h"

namespace {

constexpr int kRows = PQ_NOALLOC_MAX_JJ;
constexpr int kCols = PQ_MAX_LAYERS + 1;

struct __align__(256) NoAllocScratch {
    double partials[kRows * kCols];
    unsigned int counter;
};

// The scratch.  In host code `g_scratch` only names the symbol; its device
// address comes from cudaGetSymbolAddress (see scratch_address).
static __device__ __align__(256) NoAllocScratch g_scratch;

struct EnergyArgs {
    const double* psi;
    double* out;
    int ii, jj, L, ld, periodic;
    double fac[PQ_MAX_LAYERS];   // 0.5 s2_k h_k / H, k = 1..L-1
    double hfrac[PQ_MAX_LAYERS]; // h_k / H
    double cff;                  // 1 / (g_ii_int g_jj_int): (ii-1)(jj-1), channel (ii-1) jj
};

// Same reduction as k_energy (pq_cabaret.cu): one CTA per row of nodes, the
// last CTA adds the row partials in row order.  A channel (periodic in j)
// has no j boundary: full row weights, and the kinetic-energy corners of
// row 0 reach back to row jj - 1.
__global__ void __launch_bounds__(256) k_energy_noalloc(EnergyArgs a, NoAllocScratch* s) {
    __shared__ double red[8][kCols];
    __shared__ int is_last;
    const int j = blockIdx.x, ii = a.ii, jj = a.jj, L = a.L;
    const long long ls = (long long)a.ld * jj;
    double acc[kCols];
    for (int q = 0; q <= L; ++q) acc[q] = 0.0;
    const double wj = (!a.periodic && (j == 0 || j == jj - 1)) ? 0.5 : 1.0;
    const long long back = (j == 0) ? (long long)(jj - 1) * a.ld : -(long long)a.ld;  // row j-1, wrapped
    for (int i = threadIdx.x; i < ii; i += blockDim.x) {
        const double w = wj * ((i == 0 || i == ii - 1) ? 0.5 : 1.0);
        const long long o = (long long)j * a.ld + i;
        for (int k = 0; k < L - 1; ++k) {
            const double d = a.psi[o + k * ls] - a.psi[o + (k + 1) * ls];
            acc[L] += w * a.fac[k] * (d * d);
        }
        if (i >= 1 && (j >= 1 || a.periodic)) {
            for (int k = 0; k < L; ++k) {
                const double* p = a.psi + k * ls;
                const double x = p[o - 1] + p[o] - p[o - 1 + back] - p[o + back];
                const double y = p[o + back] + p[o] - p[o - 1 + back] - p[o - 1];
                acc[k] += 0.25 * (x * x + y * y);
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q <= L; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q <= L; ++q) {
            double t = 0.0;
            for (int w = 0; w < 8; ++w) t += red[w][q];
            s->partials[(long long)j * kCols + q] = t;
        }
        __threadfence();
        is_last = (atomicAdd(&s->counter, 1u) == (unsigned)(jj - 1));
    }
    __syncthreads();
    if (!is_last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double* part = s->partials;
    double tot[kCols];
    for (int q = 0; q <= L; ++q) tot[q] = 0.0;
    for (int r = 0; r < jj; ++r)
        for (int q = 0; q <= L; ++q) tot[q] += part[(long long)r * kCols + q];
    for (int k = 0; k < L; ++k) a.out[k] = 0.5 * a.cff * a.hfrac[k] * tot[k];
    a.out[L] = a.cff * tot[L];
    s->counter = 0u;
}

// Device address of the scratch, looked up once per device (with that device
// current) and cached.
std::mutex g_mu;
NoAllocScratch* g_addr[64] = {nullptr};

cudaError_t scratch_address(int dev, NoAllocScratch** out) {
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" PQ_API int pq_energy_noalloc(const double* psi, int ii, int jj, int layers, int ld, int periodic_j,
                                        const double* h, const double* s2, double* out, void* stream) {
    if (!psi || !out || !h || (layers > 1 && !s2)) return PQ_ERR_ARG;
    if (ii < 2 || jj < 2 || ld < ii || layers < 1 || (periodic_j != 0 && periodic_j != 1)) return PQ_ERR_ARG;
    if (jj > PQ_NOALLOC_MAX_JJ || layers > PQ_MAX_LAYERS) return PQ_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PQ_ERR_CUDA;
    NoAllocScratch* s = nullptr;
    if (scratch_address(dev, &s) != cudaSuccess) return PQ_ERR_CUDA;
    EnergyArgs a;
    a.psi = psi;
    a.out = out;
    a.ii = ii;
    a.jj = jj;
    a.L = layers;
    a.ld = ld;
    a.periodic = periodic_j;
    double htot = 0.0;
    for (int k = 0; k < layers; ++k) htot += h[k];
    for (int k = 0; k < PQ_MAX_LAYERS; ++k) a.fac[k] = a.hfrac[k] = 0.0;
    for (int k = 0; k < layers; ++k) {
        a.hfrac[k] = h[k] / htot;
        if (k + 1 < layers) a.fac[k] = 0.5 * s2[k] * h[k] / htot;
    }
    a.cff = 1.0 / ((double)(ii - 1) * (double)(periodic_j ? jj : jj - 1));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The completion counter must start at zero on every call.
    if (cudaMemsetAsync(&s->counter, 0, sizeof(unsigned int), st) != cudaSuccess) return PQ_ERR_CUDA;
    k_energy_noalloc<<<jj, 256, 0, st>>>(a, s);
    if (cudaGetLastError() != cudaSuccess) return PQ_ERR_CUDA;
    return PQ_OK;
}
