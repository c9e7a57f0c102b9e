// pq_helm.cu -- the Helmholtz (PV-inversion) kernels.
//
// The reference solves, per vertical mode, (d_xx + d_yy - ss) psi = zeta by a
// DST-I along i (FFTPACK sint, qg3p_helmholtz.F90:1370-1591), a tridiagonal
// solve along j with precomputed reciprocal pivots (ge_local, :1028-1059),
// and the inverse DST (helm, :614-769).  Here that is three kernels:
//
//   k_dst_rows<FWD>  one CTA per interior row j: load (optionally apply the
//                    CABARET predictor + beta step and the z_to_modes
//                    projection), scale by 0.5/(ii-1), DST every mode row in
//                    shared memory, write the spectral rows.
//   k_tridiag        one CTA per (mode, 8 consecutive wavenumbers): the whole
//                    column strip is staged in shared memory; each warp owns
//                    one wavenumber, each lane a chunk of rows, and the
//                    forward / backward Thomas recurrences are solved as
//                    chunked first-order linear recurrences (local sweep,
//                    warp scan of the affine chunk maps, fix-up sweep).  The
//                    same CTA accumulates the domain mean of the solution in
//                    spectral space; the last CTA of a member finishes psiC.
//   k_dst_rows<INV>  one CTA per row j: inverse DST of every mode row, then
//                    the mass-corrected back-projection (modes_to_z_btcu,
//                    qg3p_diagnostics.F90:615-635) straight into psi.
//
// DST-I of length n = N - 1 (N = ii - 1 = 2^p), FFTPACK convention
// X_k = 2 sum_m x_m sin(m k pi / N): the sequence is pre-twiddled into a real
// sequence c of length N (as sint1 does), c is packed into N/2 complex points
// and transformed by a radix-4/2 Stockham FFT in shared memory, the real-FFT
// split gives C_q = R_q + i I_q, and X_2q = -I_q, X_2q+1 = R_0/2 + sum_{p<=q} R_p
// (the odd outputs are a prefix sum, done as a block scan).
#include <type_traits>

#include "pq_common.cuh"
#include "pq_kernels.h"

namespace pq {

enum { PRO_PLAIN = 0, PRO_MODAL = 1, PRO_STEP = 2 };
enum { EPI_SPEC = 0, EPI_HELM = 1, EPI_PV = 2 };

constexpr int TRI_THREADS = 256;

// ---------------------------------------------------------------------------
// Row DSTs: one group of P lanes per (row, mode) unit.
//
// The complex FFT of length M = N/2 is a Stockham FFT in which every lane of
// a group owns V = M / P values for the whole transform: the pre-twiddle
// computes a lane's first-pass inputs straight into registers, each radix-8
// (then 4 or 2) pass is a set of V/R in-register butterflies, and values cross
// lanes only through the unit's shared-memory row between passes (under
// __syncwarp, never a block barrier).  The real-FFT split and the prefix sum
// of the odd outputs run on V contiguous wavenumbers per lane with one
// segmented warp scan.  V = 8 up to M = 256 (P = M/8 lanes), then 16, 32.
//
// Unit buffer (U scalars per unit): plain real row x[k] (input), padded
// complex rows (Stockham passes, index t -> t + t/8), padded real output row
// (index k -> k + 2*(k/16), so that the pair stores of the split are
// bank-conflict free).

__device__ __forceinline__ int cpad(int t) { return t + (t >> 3); }
__device__ __forceinline__ int xpad(int k) { return k + ((k >> 4) << 1); }

template <typename T2> __device__ __forceinline__ T2 c_mi(T2 a) {  // a * (-i)
    T2 r;
    r.x = a.y;
    r.y = -a.x;
    return r;
}

// In-register forward DFT of R points (R = 2, 4, 8), natural order.
template <int R, typename T2> __device__ __forceinline__ void dft_reg(T2* v) {
    if constexpr (R == 2) {
        const T2 a = cadd(v[0], v[1]), b = csub(v[0], v[1]);
        v[0] = a;
        v[1] = b;
    } else if constexpr (R == 4) {
        const T2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]), t3 = c_mi(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[1] = cadd(t1, t3);
        v[2] = csub(t0, t2);
        v[3] = csub(t1, t3);
    } else {
        using T = decltype(v[0].x);
        const T c8 = (T)0.70710678118654752440;  // sqrt(2)/2
        const T2 e0 = cadd(v[0], v[4]), e1 = csub(v[0], v[4]), e2 = cadd(v[2], v[6]), e3 = c_mi(csub(v[2], v[6]));
        const T2 E0 = cadd(e0, e2), E1 = cadd(e1, e3), E2 = csub(e0, e2), E3 = csub(e1, e3);
        const T2 o0 = cadd(v[1], v[5]), o1 = csub(v[1], v[5]), o2 = cadd(v[3], v[7]), o3 = c_mi(csub(v[3], v[7]));
        T2 O0 = cadd(o0, o2), O1 = cadd(o1, o3), O2 = csub(o0, o2), O3 = csub(o1, o3);
        // W8^1 = (1 - i)/sqrt2, W8^2 = -i, W8^3 = (-1 - i)/sqrt2
        T2 t;
        t.x = c8 * (O1.x + O1.y);
        t.y = c8 * (O1.y - O1.x);
        O1 = t;
        O2 = c_mi(O2);
        t.x = c8 * (O3.y - O3.x);
        t.y = -c8 * (O3.x + O3.y);
        O3 = t;
        v[0] = cadd(E0, O0);
        v[1] = cadd(E1, O1);
        v[2] = cadd(E2, O2);
        v[3] = cadd(E3, O3);
        v[4] = csub(E0, O0);
        v[5] = csub(E1, O1);
        v[6] = csub(E2, O2);
        v[7] = csub(E3, O3);
    }
}

// Barrier of one unit's P lanes: the warp (P <= 32) or the unit's warps by a
// named barrier (P > 32; id 1 + uid, never 0, which __syncthreads uses).
__device__ __forceinline__ void unit_sync(int P, int uid) {
    if (P <= 32)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;\n" ::"r"(1 + uid), "r"(P) : "memory");
}

// One radix-R Stockham pass over the unit's M values (Ns = length of the
// sub-transforms already done).  Lane p owns butterflies j = p + P*b; its
// values v[b*R + r] are the butterfly inputs j + r*(M/R).  With `load` false
// the inputs are already in registers (first pass).  Output is stored to the
// unit's padded complex row.
template <int V, int R, typename T2>
__device__ __forceinline__ void fft_pass(T2 (&v)[V], T2* z, int p, int P, int uid, int M, int logM, int Ns,
                                         int logNs, const T2* __restrict__ tw, bool load) {
    constexpr int logR = (R == 8) ? 3 : (R == 4) ? 2 : 1;
    const int MR = M >> logR;
    if (load) {
#pragma unroll
        for (int b = 0; b < V / R; ++b)
#pragma unroll
            for (int r = 0; r < R; ++r) v[b * R + r] = z[cpad(p + P * b + r * MR)];
    }
    const int lst = logM - logR - logNs;  // log2(M / (Ns R))
#pragma unroll
    for (int b = 0; b < V / R; ++b) {
        const int j = p + P * b, k = j & (Ns - 1);
        if (k) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], __ldg(&tw[(r * k) << lst]));
        }
        dft_reg<R>(&v[b * R]);
    }
    unit_sync(P, uid);
#pragma unroll
    for (int b = 0; b < V / R; ++b) {
        const int j = p + P * b, k = j & (Ns - 1);
        const int o = ((j >> logNs) << (logNs + logR)) + k;
#pragma unroll
        for (int r = 0; r < R; ++r) z[cpad(o + r * Ns)] = v[b * R + r];
    }
    unit_sync(P, uid);
}

// DST-I (FFTPACK sint convention, qg3p_helmholtz.F90:1370-1426) of the real
// row held in the unit buffer (x_k at buf[k], k = 1..N-1), output X_k at
// buf[xpad(k)], k = 1..N-1.  Every lane of the unit must call this; uid
// names the unit's barrier, utot is P/32 scalars of scratch for units wider
// than a warp.
template <int V, typename T>
__device__ __forceinline__ void dst_unit(T* buf, int p, int P, int uid, T* utot, int N, int M, int logM,
                                         const typename Cplx<T>::type* __restrict__ tw,
                                         const typename Cplx<T>::type* __restrict__ wsp,
                                         const T* __restrict__ was) {
    using T2 = typename Cplx<T>::type;
    constexpr int R0 = V >= 8 ? 8 : V;
    T2 v[V];
    // Pre-twiddle (sint1, :1404-1413) into the first pass's inputs:
    // c_k = (x_k - x_{N-k}) + 2 sin(k pi / N) (x_k + x_{N-k}), c_0 = 0,
    // packed c_{2t} + i c_{2t+1}.
    {
        const int MR0 = M / R0;
#pragma unroll
        for (int b = 0; b < V / R0; ++b)
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const int t = p + P * b + r * MR0;
                const int k = 2 * t;
                const T2 xa = *reinterpret_cast<const T2*>(buf + k);  // x_k, x_{k+1}
                const T xb0 = buf[N - k], xb1 = buf[N - k - 1];
                const bool lo = 2 * k < N;  // then k + 1 <= N/2 too
                const T w0 = __ldg(&was[lo ? k : N - k]), w1 = __ldg(&was[lo ? k + 1 : N - k - 1]);
                const T c0 = (t == 0) ? (T)0 : (xa.x - xb0) + w0 * (xa.x + xb0);
                const T c1 = (xa.y - xb1) + w1 * (xa.y + xb1);
                v[b * R0 + r].x = c0;
                v[b * R0 + r].y = c1;
            }
    }
    T2* z = reinterpret_cast<T2*>(buf);
    {
        int Ns = 1, logNs = 0;
        bool first = true;
        while (Ns < M) {
            const int rem = M >> logNs;
            if constexpr (V >= 8) {
                if (rem >= 8) {
                    fft_pass<V, 8>(v, z, p, P, uid, M, logM, Ns, logNs, tw, !first);
                    Ns <<= 3;
                    logNs += 3;
                    first = false;
                    continue;
                }
            }
            if constexpr (V >= 4) {
                if (rem >= 4) {
                    fft_pass<V, 4>(v, z, p, P, uid, M, logM, Ns, logNs, tw, !first);
                    Ns <<= 2;
                    logNs += 2;
                    first = false;
                    continue;
                }
            }
            fft_pass<V, 2>(v, z, p, P, uid, M, logM, Ns, logNs, tw, !first);
            Ns <<= 1;
            logNs += 1;
            first = false;
        }
    }
    // Real-FFT split on V contiguous wavenumbers q = p*V + e:
    // C_q = E_q + W_q O_q, R_q = Re C_q (halved at q = 0), X_2q = -Im C_q,
    // X_{2q+1} = sum_{s <= q} R_s.
    T Xe[V], Xo[V];
    T run = (T)0;
#pragma unroll
    for (int e = 0; e < V; ++e) {
        const int q = p * V + e;
        const T2 zq = z[cpad(q)];
        const T2 zr = z[cpad((M - q) & (M - 1))];
        const T ex = (T)0.5 * (zq.x + zr.x), ey = (T)0.5 * (zq.y - zr.y);
        const T dx = zq.x - zr.x, dy = zq.y + zr.y;
        T2 O;
        O.x = (T)0.5 * dy;
        O.y = (T)-0.5 * dx;
        const T2 w = __ldg(&wsp[q]);
        const T cx = ex + (w.x * O.x - w.y * O.y);
        const T cy = ey + (w.x * O.y + w.y * O.x);
        Xe[e] = (q == 0) ? (T)0 : -cy;
        run += (q == 0) ? (T)0.5 * cx : cx;
        Xo[e] = run;
    }
    // Segmented (width P) exclusive scan of the lanes' totals: in the warp
    // (or P-lane segment), then across the unit's warps.
    T incl = run;
    const int PW = P < 32 ? P : 32;
    for (int d = 1; d < PW; d <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, incl, d, PW);
        if ((p & (PW - 1)) >= d) incl += y;
    }
    if (P > 32) {
        if ((p & 31) == 31) utot[p >> 5] = incl;
        unit_sync(P, uid);
        T add = (T)0;
        for (int w = 0; w < (p >> 5); ++w) add += utot[w];
        incl += add;
    }
    const T excl = incl - run;
    unit_sync(P, uid);
#pragma unroll
    for (int e = 0; e < V; ++e) {
        const int q = p * V + e;
        T2 pr;
        pr.x = Xe[e];
        pr.y = Xo[e] + excl;
        *reinterpret_cast<T2*>(buf + xpad(2 * q)) = pr;
    }
    unit_sync(P, uid);
}

// Launch geometry shared by host and device: lanes P and values V = M / P
// per unit, rows per CTA (whole warps: 32 / P rows per group for P < 32),
// scalars per unit buffer.  Default P (measured per grid size on B200): one
// warp per unit up to M = 256 (fewer values per lane, more warps in flight,
// shorter dependent chains), two warps (a named barrier between passes) from
// M = 512 in both directions (the inverse's 8-value units in a register-
// capped instance, whose back-projection otherwise held it to two CTAs per
// SM), when a row's L units fit the kernel's thread bound; dir is kept for
// callers that ask per direction.
// Threads a DST CTA may have: 320 for 16 values per lane (five layers of
// two-warp units at M = 1024), else 256, the bound the others' register
// use was tuned for.
__host__ __device__ constexpr int dst_max_threads(int V) { return V == 16 ? 320 : 256; }
__host__ __device__ inline int dst_lanes_default_hd(int M, int L, int dir) {
    (void)dir;
    if (M <= 256) return M / 2 < 32 ? (M / 2 < 1 ? 1 : M / 2) : 32;
    return L * 64 <= dst_max_threads(M / 64) ? 64 : 32;
}
__host__ __device__ inline int dst_rows_per_cta(int P, int c) {
    if (c <= 0) c = 1;  // one row group per CTA: the most CTAs, measured fastest
    return c * (P >= 32 ? 1 : 32 / P);
}
__host__ __device__ inline int dst_unit_len(int N) { return (N + N / 8 + 2 + 1) & ~1; }

__device__ __forceinline__ void cp16(void* dst, const void* src, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp8z(double* dst, const double* src, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void cp4z(void* dst, const void* src, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 4 : 0) : "memory");
}

// Row DST kernel.  A CTA holds R rows x L modes = L*R units of P lanes,
// ordered mode-major (unit (m, r) at index m*R + r), so that every warp's
// units share one mode.
//
// Forward (EPI_SPEC, interior rows 1..jj-2): the raw layer rows are copied
// asynchronously into shared memory (16-byte copies: node k of a row and
// entry k of the buffer have the same alignment), projected onto the modes
// (z_to_modes) and scaled by 0.5/(ii-1); PRO_STEP instead computes the
// CABARET predictor + beta update per node in registers.  Each unit then
// transforms its row and writes spec(m, j, k-1) = X_k.
//
// Inverse (EPI_HELM / EPI_PV, rows 0..jj-1): the solved spectral rows are
// copied in (spec offset k-1 -> buffer entry k), transformed, and written
// out; for EPI_PV the correction rows corr_m (m >= 1) are prefetched into
// shared memory before the transform and the mass-corrected back-projection
// writes psi.
//
// S is the storage type of the state and spectral fields.  S = float is the
// mixed form: the layer fields and the baroclinic spectral rows are FP32 and
// transformed in FP32, while the barotropic mode (m = 0) is kept in FP64
// end to end (spec64), as are the projection, the back-projection and psi.
// The row-DST kernel's body; k_dst and k_dst_capped below are its kernels.
template <typename S, int V, int PRO, int EPI>
__device__ __forceinline__ void dst_body(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem,
                                         int row_offset, int c, int corr_smem, int psic_here, const Member& one,
                                         int use_one, int gemm_bc) {
    constexpr bool MX = sizeof(S) == 4;
    __shared__ Member Mb;
    __shared__ double psic_s[PQ_MAXL];                   // closed basin: psiC of the inverse
    __shared__ double psic_red[dst_max_threads(V) / 32 * PQ_MAXL];
    extern __shared__ __align__(16) double sm[];
    pdl_wait();
    int local;
    cta_member(Mb, one, use_one, mems, prefix, nmem, blockIdx.x, &local);
    __syncthreads();
    const int L = Mb.L, N = Mb.N, M = Mb.M, logM = Mb.logM, n = Mb.n, ii = Mb.ii, jj = Mb.jj, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int P = M / V;
    const int R = dst_rows_per_cta(P, c);
    const int U = dst_unit_len(N);
    const int j0 = row_offset + local * R;                 // first row of this CTA
    // one past the last row; a channel periodic in j transforms every row
    const int jend = (EPI == EPI_SPEC && !Mb.periodic) ? jj - 1 : jj;
    const int nthr = blockDim.x;
    double* extra = sm + (size_t)L * R * U;                 // EPI_PV: corr rows [R][L-1][pitch];
                                                            // mixed forward: staged rows [R][L][N] (FP32)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = nthr >> 5;
    auto ubuf = [&](int m, int r) { return sm + (size_t)(m * R + r) * U; };
    // Unit (m, r) buffers hold FP64 values, except the baroclinic ones of the mixed form.
    auto fp64_mode = [&](int m) { return !MX || m == 0; };
    auto put = [&](int m, int r, int k, double v) {
        if (fp64_mode(m))
            ubuf(m, r)[k] = v;
        else
            reinterpret_cast<float*>(ubuf(m, r))[k] = (float)v;
    };
    auto get = [&](int m, int r, int k) -> double {
        return fp64_mode(m) ? ubuf(m, r)[k] : (double)reinterpret_cast<const float*>(ubuf(m, r))[k];
    };

    // ---------------- stage the rows --------------------------------------
    if (EPI == EPI_SPEC) {
        const double cff = 0.5 / (double)(ii - 1);
        if (PRO != PRO_STEP) {
            // The stand-alone helm input (helm_io) is FP64 in either form.
            using ST = std::conditional_t<PRO == PRO_PLAIN, double, S>;
            const ST* src = reinterpret_cast<const ST*>(PRO == PRO_PLAIN ? Mb.helm_io : Mb.zeta);
            // Layer l of row j0 + r: FP64 into unit (l, r) (projected in place
            // below), FP32 into the staging rows; one warp per row.
            constexpr int PER16 = 16 / sizeof(ST);
            for (int rl = warp; rl < R * L; rl += nwarp) {
                const int r = rl / L, l = rl - r * L;
                const int j = j0 + r;
                const bool ok = j < jend;
                const ST* g = src + l * ls + (long long)(ok ? j : 1) * pitch;
                ST* d = MX ? reinterpret_cast<ST*>(extra) + (size_t)rl * N : reinterpret_cast<ST*>(ubuf(l, r));
                for (int q = lane; q < N / PER16; q += 32) cp16(d + PER16 * q, g + PER16 * q, ok);
            }
            cp_commit_wait_all();
            __syncthreads();
            // Node k of the L layer rows -> node k of the L mode rows (in
            // place for FP64: a node's values are read before they are written).
            // z_to_modes with an exact layer count up to five: loops unrolled to
            // L, z2m in registers (as the back-projection below).
            auto exact = [&](auto lc) {
                constexpr int LC = decltype(lc)::value;
                double zm[LC][LC];
#pragma unroll
                for (int m = 0; m < LC; ++m)
#pragma unroll
                    for (int l = 0; l < LC; ++l) zm[m][l] = Mb.z2m[m * PQ_MAXL + l];
                for (int r = 0; r < R; ++r)
                    for (int k = threadIdx.x; k < N; k += nthr) {
                        double z[LC];
#pragma unroll
                        for (int l = 0; l < LC; ++l)
                            z[l] = MX ? (double)reinterpret_cast<const ST*>(extra)[(size_t)(r * LC + l) * N + k]
                                      : ubuf(l, r)[k];
#pragma unroll
                        for (int m = 0; m < LC; ++m) {
                            // z_to_modes, qg3p_diagnostics.F90:545-549
                            double sacc = 0.0;
#pragma unroll
                            for (int l = 0; l < LC; ++l) sacc += zm[m][l] * z[l];
                            put(m, r, k, cff * sacc);
                        }
                    }
            };
            bool done = false;
            if constexpr (PRO == PRO_MODAL) {
                done = true;
                switch (L) {
                    case 1: exact(std::integral_constant<int, 1>{}); break;
                    case 2: exact(std::integral_constant<int, 2>{}); break;
                    case 3: exact(std::integral_constant<int, 3>{}); break;
                    case 4: exact(std::integral_constant<int, 4>{}); break;
                    case 5: exact(std::integral_constant<int, 5>{}); break;
                    default: done = false;
                }
            }
            if (!done)
            for (int r = 0; r < R; ++r)
                for (int k = threadIdx.x; k < N; k += nthr) {
                    double z[PQ_MAXL];
#pragma unroll
                    for (int l = 0; l < PQ_MAXL; ++l)
                        if (l < L)
                            z[l] = MX ? (double)reinterpret_cast<const ST*>(extra)[(size_t)(r * L + l) * N + k]
                                      : ubuf(l, r)[k];
                    if constexpr (PRO == PRO_PLAIN) {
#pragma unroll
                        for (int m = 0; m < PQ_MAXL; ++m)
                            if (m < L) put(m, r, k, cff * z[m]);
                    } else {
#pragma unroll 1
                        for (int m = 0; m < L; ++m) {
                            // z_to_modes, qg3p_diagnostics.F90:545-549
                            double sacc = 0.0;
#pragma unroll
                            for (int l = 0; l < PQ_MAXL; ++l)
                                if (l < L) sacc += Mb.z2m[m * PQ_MAXL + l] * z[l];
                            put(m, r, k, cff * sacc);
                        }
                    }
                }
        } else {
            const double dt = Mb.sc->dt, ta = Mb.sc->tweight_a;
            const S* __restrict__ zo = reinterpret_cast<const S*>(Mb.zeta_old[Mb.cur]);
            const S* __restrict__ rs = reinterpret_cast<const S*>(Mb.res);
            const S* __restrict__ rbo = reinterpret_cast<const S*>(Mb.res_beta_other);
            S* __restrict__ rb = reinterpret_cast<S*>(Mb.res_beta);
            const S* __restrict__ ui = reinterpret_cast<const S*>(Mb.ui);
            S* __restrict__ zp = reinterpret_cast<S*>(Mb.zeta);
            // Exact layer counts up to five: loops unrolled to L, beta and
            // z2m in registers (as the modal prologue); the same arithmetic.
            auto exact = [&](auto lc) {
                constexpr int LC = decltype(lc)::value;
                double zm[LC][LC], bt[LC];
#pragma unroll
                for (int m = 0; m < LC; ++m) {
                    bt[m] = Mb.beta[m];
#pragma unroll
                    for (int l = 0; l < LC; ++l) zm[m][l] = Mb.z2m[m * PQ_MAXL + l];
                }
                for (int r = 0; r < R; ++r) {
                    const int j = j0 + r;
                    const bool ok = j < jend;
                    for (int k = 1 + threadIdx.x; k <= n; k += nthr) {
                        const long long o = (long long)j * pitch + k;
                        double a0[LC], a1[LC], a2[LC], a3[LC], a4[LC];
#pragma unroll
                        for (int l = 0; l < LC; ++l) {
                            if (ok) {
                                const long long ol = o + l * ls;
                                a0[l] = zo[ol];
                                a1[l] = rs[ol];
                                a2[l] = ui[ol];
                                a3[l] = ui[ol + 1];
                                a4[l] = rbo[ol];
                            }
                        }
                        double z[LC];
#pragma unroll
                        for (int l = 0; l < LC; ++l) {
                            double zz = 0.0;
                            if (ok) {
                                const long long ol = o + l * ls;
                                // cabaret_predictor, qg3p_aux.F90:1012-1018
                                zz = a0[l] + 0.5 * dt * a1[l];
                                // cabaret_beta, qg3p_aux.F90:1051-1059
                                const double rbn = dt * (0.5 * (a3[l] + a2[l]) * bt[l]);
                                zz = zz + (1.0 + ta) * rbn - ta * a4[l];
                                rb[ol] = (S)rbn;
                                zp[ol] = (S)zz;
                                if (MX) zz = (double)(S)zz;  // the stored (FP32) value
                            }
                            z[l] = zz;
                        }
#pragma unroll
                        for (int m = 0; m < LC; ++m) {
                            double sacc = 0.0;
#pragma unroll
                            for (int l = 0; l < LC; ++l) sacc += zm[m][l] * z[l];
                            put(m, r, k, cff * sacc);
                        }
                    }
                }
            };
            bool done = true;
            switch (L) {
                case 1: exact(std::integral_constant<int, 1>{}); break;
                case 2: exact(std::integral_constant<int, 2>{}); break;
                case 3: exact(std::integral_constant<int, 3>{}); break;
                case 4: exact(std::integral_constant<int, 4>{}); break;
                case 5: exact(std::integral_constant<int, 5>{}); break;
                default: done = false;
            }
            if (!done)
            for (int r = 0; r < R; ++r) {
                const int j = j0 + r;
                const bool ok = j < jend;
                for (int k = 1 + threadIdx.x; k <= n; k += nthr) {
                    const long long o = (long long)j * pitch + k;
                    double a0[PQ_MAXL], a1[PQ_MAXL], a2[PQ_MAXL], a3[PQ_MAXL], a4[PQ_MAXL];
                    // All loads of the node first, then the arithmetic and stores.
#pragma unroll
                    for (int l = 0; l < PQ_MAXL; ++l) {
                        if (l < L && ok) {
                            const long long ol = o + l * ls;
                            a0[l] = zo[ol];
                            a1[l] = rs[ol];
                            a2[l] = ui[ol];
                            a3[l] = ui[ol + 1];
                            a4[l] = rbo[ol];
                        }
                    }
                    double z[PQ_MAXL];
#pragma unroll
                    for (int l = 0; l < PQ_MAXL; ++l) {
                        if (l < L) {
                            double zz = 0.0;
                            if (ok) {
                                const long long ol = o + l * ls;
                                // cabaret_predictor, qg3p_aux.F90:1012-1018
                                zz = a0[l] + 0.5 * dt * a1[l];
                                // cabaret_beta, qg3p_aux.F90:1051-1059
                                const double rbn = dt * (0.5 * (a3[l] + a2[l]) * Mb.beta[l]);
                                zz = zz + (1.0 + ta) * rbn - ta * a4[l];
                                rb[ol] = (S)rbn;
                                zp[ol] = (S)zz;
                                if (MX) zz = (double)(S)zz;  // the stored (FP32) value
                            }
                            z[l] = zz;
                        }
                    }
#pragma unroll 1
                    for (int m = 0; m < L; ++m) {
                        double sacc = 0.0;
#pragma unroll
                        for (int l = 0; l < PQ_MAXL; ++l)
                            if (l < L) sacc += Mb.z2m[m * PQ_MAXL + l] * z[l];
                        put(m, r, k, cff * sacc);
                    }
                }
            }
        }
    } else {
        // unit (m, r) entries 1..n <- spec(m, j, 0..n-1); one warp per unit row
        for (int rm = warp; rm < R * L; rm += nwarp) {
            const int m = rm / R, r = rm - m * R;
            const int j = j0 + r;
            const bool ok = (Mb.periodic || (j >= 1 && j <= jj - 2)) && j < jend;
            if (fp64_mode(m)) {
                const double* g = (MX ? Mb.spec64 : reinterpret_cast<const double*>(Mb.spec)) + m * ls +
                                  (long long)(ok ? j : 1) * pitch - 1;
                double* d = ubuf(m, r);
                for (int k = 1 + lane; k <= n; k += 32) cp8z(d + k, g + k, ok);
            } else if (gemm_bc) {
                // Rows the tensor-core DST already took back to node values:
                // straight to the positions the back-projection reads.
                const float* g = reinterpret_cast<const float*>(Mb.gbuf) + m * ls + (long long)(ok ? j : 1) * pitch - 1;
                float* d = reinterpret_cast<float*>(ubuf(m, r));
                for (int k = 1 + lane; k <= n; k += 32) cp4z(d + xpad(k), g + k, ok);
            } else {
                const float* g = reinterpret_cast<const float*>(Mb.spec) + m * ls + (long long)(ok ? j : 1) * pitch - 1;
                float* d = reinterpret_cast<float*>(ubuf(m, r));
                for (int k = 1 + lane; k <= n; k += 32) cp4z(d + k, g + k, ok);
            }
        }
        if (EPI == EPI_PV && psic_here) {
            // psiC_m = (sum of the tridiagonal CTAs' partial means of mode m)
            // / (g_ii_int g_jj_int) (modes_to_z_correct_mass,
            // qg3p_aux.F90:482-521), summed in the same fixed order by every
            // CTA while its rows load (one pass for all modes); the member's
            // first CTA publishes it and flags a NaN (the reference aborts,
            // :504-510) or a value above 1e100 (it warns, :511-517).
            const int KT = 8 / tri_warps(jj), tpm = (n + KT - 1) / KT;
            double acc[PQ_MAXL];
#pragma unroll
            for (int mm = 0; mm < PQ_MAXL; ++mm) acc[mm] = 0.0;
            for (int q = threadIdx.x; q < tpm; q += nthr)
#pragma unroll
                for (int mm = 0; mm < PQ_MAXL; ++mm)
                    if (mm < L) acc[mm] += __ldcg(Mb.partials + (long long)mm * tpm + q);
#pragma unroll
            for (int mm = 0; mm < PQ_MAXL; ++mm) {
                if (mm < L) {
                    const double w = warp_sum(acc[mm]);
                    if (lane == 0) psic_red[warp * PQ_MAXL + mm] = w;
                }
            }
            __syncthreads();
            if (threadIdx.x < L) {
                const int mm = threadIdx.x;
                double t = 0.0;
                for (int w = 0; w < nwarp; ++w) t += psic_red[w * PQ_MAXL + mm];
                const double pc = t * Mb.mean_scale;
                psic_s[mm] = pc;
                if (local == 0) {
                    Mb.sc->psiC[mm] = pc;
                    if (pc != pc)
                        atomicOr(Mb.status, (int)ST_NAN_PSIC);
                    else if (fabs(pc) > 1.0e100)
                        atomicOr(Mb.status, (int)ST_LARGE_PSIC);
                }
            }
        }
        if (EPI == EPI_PV && corr_smem) {
            const double* corr = Mb.corr;
            const int cw = pitch >> 1;
            for (int rm = warp; rm < R * (L - 1); rm += nwarp) {
                const int r = rm / (L - 1), m = 1 + rm - r * (L - 1);
                const int j = j0 + r;
                const bool ok = j < jend;
                const double* g = corr + m * ls + (long long)(ok ? j : 0) * pitch;
                double* d = extra + (size_t)rm * pitch;
                for (int q = lane; q < cw; q += 32) cp16(d + 2 * q, g + 2 * q, ok);
            }
        }
        cp_commit_wait_all();
    }
    __syncthreads();

    // ---------------- per-unit transform ----------------------------------
    const int u = threadIdx.x / P, p = threadIdx.x & (P - 1);
    const int um = u / R, ur = u - um * R;
    const int ju = j0 + ur;
    double* buf = ubuf(um, ur);
    const bool interior = (Mb.periodic || (ju >= 1 && ju <= jj - 2)) && ju < jend;
    __shared__ double utot[8][2];  // cross-warp scan totals of units wider than a warp
    // With gemm_bc the baroclinic rows (a whole warp's or unit's mode) are
    // transformed by the tensor-core DST instead (pq_dst_mma.cu).
    if (fp64_mode(um))
        dst_unit<V, double>(buf, p, P, u, utot[u & 7], N, M, logM, Mb.tw, Mb.wsplit, Mb.was);
    else if (!gemm_bc)
        dst_unit<V, float>(reinterpret_cast<float*>(buf), p, P, u, reinterpret_cast<float*>(utot[u & 7]), N, M, logM,
                           Mb.tw_f, Mb.wsplit_f, Mb.was_f);
    pdl_release();

    if (EPI == EPI_SPEC) {
        if (ju < jend) {
            if (fp64_mode(um)) {
                double* spec = (MX ? Mb.spec64 : reinterpret_cast<double*>(Mb.spec)) + um * ls +
                               (long long)ju * pitch - 1;
                for (int k = 1 + p; k <= n; k += P) spec[k] = buf[xpad(k)];
            } else if (gemm_bc) {
                // node values of the projected row, for the tensor-core DST
                float* g = reinterpret_cast<float*>(Mb.gbuf) + um * ls + (long long)ju * pitch - 1;
                const float* fb = reinterpret_cast<const float*>(buf);
                for (int k = 1 + p; k <= n; k += P) g[k] = fb[k];
            } else {
                float* spec = reinterpret_cast<float*>(Mb.spec) + um * ls + (long long)ju * pitch - 1;
                const float* fb = reinterpret_cast<const float*>(buf);
                for (int k = 1 + p; k <= n; k += P) spec[k] = fb[xpad(k)];
            }
        }
    } else if (EPI == EPI_HELM) {
        // helm's in-place output: interior entries of interior rows, row
        // i = ii zeroed (:758-761); ge_local zeroes psi(2:ii-1, 1)
        // (:1055-1057).  helm_io is FP64 in either form (the mixed form's
        // FP32 units are widened).
        double* io = reinterpret_cast<double*>(Mb.helm_io) + um * ls + (long long)ju * pitch;
        if (interior) {
            if (fp64_mode(um))
                for (int k = 1 + p; k <= n; k += P) io[k] = buf[xpad(k)];
            else
                for (int k = 1 + p; k <= n; k += P) io[k] = (double)reinterpret_cast<const float*>(buf)[xpad(k)];
            if (p == 0) io[ii - 1] = 0.0;
        } else if (ju == 0 && !Mb.periodic) {
            for (int k = 1 + p; k <= n; k += P) io[k] = 0.0;
        }
    } else {
        // psi_l = phi_1 - psiC_1 + sum_{m>=2} m2z(l,m) (phi_m - psiC_m corr_m)
        // (modes_to_z_btcu, qg3p_diagnostics.F90:615-635) on every node of the
        // row; phi is zero on the boundary (apply_dirichlet_bc(0),
        // qg3p_aux.F90:470).
        __syncthreads();
        // A channel (modes_to_z_correct_momentum + modes_to_z, qg3p_aux.F90:
        // 524-575) subtracts psiC_m corr_m + psiC2_m corr2_m from the
        // baroclinic modes; its psiC_0 is zero.
        const double* psiC = Mb.sc->psiC;
        const double* psiC2 = Mb.sc->psiC2;
        double pc[PQ_MAXL], pc2[PQ_MAXL];
#pragma unroll
        for (int m = 0; m < PQ_MAXL; ++m) {
            pc[m] = (m < L) ? (psic_here ? psic_s[m] : psiC[m]) : 0.0;
            pc2[m] = (m < L && Mb.periodic) ? psiC2[m] : 0.0;
        }
        double* psi = Mb.psi;
        // Exact layer counts up to five (every configuration here) run with
        // the loops unrolled to L and m2z in registers: the loops below,
        // unrolled to PQ_MAXL under predicates, issue several times the
        // instructions and shared-memory loads (measured 0.6-0.8 us per node
        // row pass at 513 x 513 x 3 against ~0.1 us for L = 3).
        auto exact = [&](auto lc) {
            constexpr int LC = decltype(lc)::value;
            double mz[LC][LC];
#pragma unroll
            for (int l = 0; l < LC; ++l)
#pragma unroll
                for (int m = 1; m < LC; ++m) mz[l][m] = Mb.m2z[l * PQ_MAXL + m];
            const double* c2b = Mb.corr2;
            for (int r = 0; r < R; ++r) {
                const int j = j0 + r;
                if (j >= jend) break;
                const double* crs = extra + ((long long)r * (LC - 1) - 1) * pitch;  // staged corr rows
                const double* crg = Mb.corr + (long long)j * pitch;
                for (int i = threadIdx.x; i < ii; i += nthr) {
                    const bool inner = (Mb.periodic || (j >= 1 && j <= jj - 2)) && i >= 1 && i <= n;
                    double ph[LC];
#pragma unroll
                    for (int m = 0; m < LC; ++m) ph[m] = inner ? get(m, r, xpad(i)) : 0.0;
#pragma unroll
                    for (int m = 1; m < LC; ++m)
                        ph[m] -= pc[m] * (corr_smem ? crs[m * (long long)pitch + i] : crg[m * ls + i]);
                    if (Mb.periodic) {
                        const double* c2 = c2b + (long long)j * pitch + i;
#pragma unroll
                        for (int m = 1; m < LC; ++m) ph[m] -= pc2[m] * c2[m * ls];
                    }
                    const double b0 = ph[0] - pc[0];
                    const long long o = (long long)j * pitch + i;
#pragma unroll
                    for (int l = 0; l < LC; ++l) {
                        double dot = 0.0;
#pragma unroll
                        for (int m = 1; m < LC; ++m) dot += mz[l][m] * ph[m];
                        psi[o + l * ls] = b0 + dot;
                    }
                }
            }
        };
        switch (L) {
            case 1: exact(std::integral_constant<int, 1>{}); return;
            case 2: exact(std::integral_constant<int, 2>{}); return;
            case 3: exact(std::integral_constant<int, 3>{}); return;
            case 4: exact(std::integral_constant<int, 4>{}); return;
            case 5: exact(std::integral_constant<int, 5>{}); return;
            default: break;
        }
        for (int r = 0; r < R; ++r)
            for (int i = threadIdx.x; i < ii; i += nthr) {
                const int j = j0 + r;
                if (j >= jend) break;
                const bool inner = (Mb.periodic || (j >= 1 && j <= jj - 2)) && i >= 1 && i <= n;
                // corr_m at cr[m * cst] (staged rows, or the field itself)
                const double* cr = corr_smem ? extra + ((long long)r * (L - 1) - 1) * pitch + i
                                             : Mb.corr + (long long)j * pitch + i;
                const long long cst = corr_smem ? (long long)pitch : ls;
                double ph[PQ_MAXL];
#pragma unroll
                for (int m = 0; m < PQ_MAXL; ++m)
                    if (m < L) ph[m] = inner ? get(m, r, xpad(i)) : 0.0;
#pragma unroll
                for (int m = 1; m < PQ_MAXL; ++m)
                    if (m < L) ph[m] -= pc[m] * cr[m * cst];
                if (Mb.periodic) {
                    const double* c2 = Mb.corr2 + (long long)j * pitch + i;
#pragma unroll
                    for (int m = 1; m < PQ_MAXL; ++m)
                        if (m < L) ph[m] -= pc2[m] * c2[m * ls];
                }
                const double b0 = ph[0] - pc[0];
                const long long o = (long long)j * pitch + i;
#pragma unroll
                for (int l = 0; l < PQ_MAXL; ++l) {
                    if (l < L) {
                        double dot = 0.0;
#pragma unroll
                        for (int m = 1; m < PQ_MAXL; ++m)
                            if (m < L) dot += Mb.m2z[l * PQ_MAXL + m] * ph[m];
                        psi[o + l * ls] = b0 + dot;
                    }
                }
            }
    }
}

template <typename S, int V, int PRO, int EPI>
__global__ void __launch_bounds__(dst_max_threads(V)) k_dst(const Member* __restrict__ mems, const int* __restrict__ prefix,
                                                             int nmem, int row_offset, int c, int corr_smem,
                                                             int psic_here, const __grid_constant__ Member one,
                                                             int use_one, int gemm_bc) {
    dst_body<S, V, PRO, EPI>(mems, prefix, nmem, row_offset, c, corr_smem, psic_here, one, use_one, gemm_bc);
}
// The inverse with 64-lane units of 8 values: registers capped so that three
// 256-thread CTAs fit (80), hence four of its 192-thread CTAs, where its
// back-projection would otherwise take 166 registers and allow two; the
// epilogue spills a little.  (An explicit bound on the other instances would
// raise their register counts, so they keep the plain one.)
template <typename S, int V, int PRO, int EPI>
__global__ void __launch_bounds__(dst_max_threads(V), 3)
    k_dst_capped(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem, int row_offset, int c,
                 int corr_smem, int psic_here, const __grid_constant__ Member one, int use_one, int gemm_bc) {
    dst_body<S, V, PRO, EPI>(mems, prefix, nmem, row_offset, c, corr_smem, psic_here, one, use_one, gemm_bc);
}

// ---------------------------------------------------------------------------
// Tridiagonal solves along j for 8 wavenumbers of one mode.
//
// The strip (Mr = jj - 2 rows x 8 wavenumbers) is staged in shared memory by
// wavenumber, and within a wavenumber by chunk: row p (0-based) of chunk
// q = p / R, t = p % R lives at c*CS + q*RS + t with RS = R | 1 odd and CS
// from tri_cs, so the 32 lanes of a warp (one chunk each) and the half-warps
// of the staging and write-back phases hit distinct banks.  Lane q of warp c
// runs the forward and backward Thomas recurrences of its chunk of
// wavenumber c, on registers for chunks of 4, 8 or 16 rows (RR).
// Column stride of the strip in doubles: NQ*RS plus a pad that makes the 16
// threads of a half-warp of the staging and write-back phases -- KT columns
// x 16/KT chunks each -- hit 16 distinct 8-byte bank pairs: NQ*RS is a
// multiple of 16, so c*CS + q*RS = RS*(c*16/KT + q) (mod 16) with RS odd.
// In the solve phase a warp's lanes (one column, 32 chunks) are RS apart.
__host__ __device__ inline int tri_cs(int NQ, int RS, int KT) { return NQ * RS + (RS * (16 / KT)) % 16; }

struct PivotRow {
    const double* piv;  // explicit reciprocal pivots, piv[p - 1] for p <= len
    int len;
    double fix;         // the fixed point for p > len
    __device__ __forceinline__ double operator()(int p) const { return p <= len ? __ldg(&piv[p - 1]) : fix; }
};

// S = float: the mixed form, whose baroclinic spectral rows are FP32 (staged
// and solved in FP64); the barotropic mode (m = 0) comes from spec64.
// Tridiagonal solves along j.  A CTA of 256 threads solves KT = 8 / W
// wavenumber columns of one mode, W warps per column: the column's rows are
// split into 32 W chunks of R rows, one per lane, staged in shared memory
// (chunk q of column c at c*CS + q*RS, RS = R | 1 odd, so a warp's 32 chunk
// accesses hit 32 banks).  Each lane runs the forward and backward Thomas
// recurrences of its chunk as first-order affine recurrences (local sweep,
// scan of the affine chunk maps -- in the warp, then across the column's
// warps through shared memory -- and a fix-up sweep).  GS = true: the
// reciprocal pivots of the strip are staged beside it (same layout), so the
// recurrences never wait on a global load; used whenever both strips fit.
// The CTA also accumulates the domain mean of the solution in spectral space;
// the last CTA of a member finishes psiC.
template <typename S, bool GS, int RR>
__global__ void __launch_bounds__(TRI_THREADS) k_tridiag(const Member* __restrict__ mems,
                                                          const int* __restrict__ prefix, int nmem, int do_mean,
                                                          const __grid_constant__ Member one, int use_one) {
    __shared__ Member Mb;
    __shared__ double wpart[TRI_THREADS / 32];
    __shared__ double wpart2[TRI_THREADS / 32];  // channel: the second wall
    __shared__ double tot[2][TRI_THREADS / 32][2];  // per-warp affine totals (forward, backward)
    __shared__ int is_last;
    extern __shared__ __align__(16) double strip[];
    pdl_wait();
    int local;
    cta_member(Mb, one, use_one, mems, prefix, nmem, blockIdx.x, &local);
    __syncthreads();
    const int n = Mb.n, jj = Mb.jj, pitch = Mb.pitch;
    const int W = tri_warps(jj), KT = 8 / W, NQ = 32 * W;
    const int tiles_per_mode = (n + KT - 1) / KT;
    const int m = local / tiles_per_mode;
    const int tile = local - m * tiles_per_mode;
    const int k0 = tile * KT;  // 0-based column (wavenumber k0+1)
    const int Mr = jj - 2;
    const int R = (Mr + NQ - 1) / NQ;
    const int RS = R | 1;
    const int CS = tri_cs(NQ, RS, KT);
    const bool f32 = sizeof(S) == 4 && m > 0;  // this mode's rows are FP32
    double* spec = ((sizeof(S) == 4) ? Mb.spec64 : reinterpret_cast<double*>(Mb.spec)) + (long long)m * Mb.lstride;
    float* specf = reinterpret_cast<float*>(Mb.spec) + (long long)m * Mb.lstride;
    double* gstrip = strip + KT * CS;  // pivots (GS)

    // Stage: thread -> (column c = tid % KT, chunk q = tid / KT); loop over t.
    // Asynchronous 8-byte copies (cp.async), so the loads of a thread do not
    // wait for one another; columns past n are zero-filled (source size 0).
    // FP32 rows are loaded and widened in registers.
    {
        const int c = threadIdx.x % KT, q = threadIdx.x / KT;
        const bool colok = (k0 + c < n);
        const long long go = (long long)(q * R + 1) * pitch + (colok ? k0 + c : 0);
        double* sdst = strip + c * CS + q * RS;
        const int Rq = min(R, Mr - q * R);
        if (GS) {
            // g(p) for the rows p = q*R + 1 .. of this chunk: the stored
            // reciprocal pivots up to len, then the fixed point.
            double* gdst = gstrip + c * CS + q * RS;
            if (colok) {
                const int mk = m * n + k0 + c;
                const int off = __ldg(&Mb.piv_off[mk]), len = __ldg(&Mb.piv_len[mk]);
                const double fix = __ldg(&Mb.piv_fix[mk]);
                const unsigned gbase = (unsigned)__cvta_generic_to_shared(gdst);
                for (int t = 0; t < Rq; ++t) {
                    const int pp = q * R + 1 + t;
                    if (pp <= len)
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(gbase + 8u * t),
                                     "l"(Mb.piv + off + pp - 1)
                                     : "memory");
                    else
                        gdst[t] = fix;
                }
            } else {
                for (int t = 0; t < Rq; ++t) gdst[t] = 0.0;
            }
        }
        if (!f32) {
            const double* g = spec + go;
            const unsigned sbase = (unsigned)__cvta_generic_to_shared(sdst);
            const int nbytes = colok ? 8 : 0;
            for (int t = 0; t < Rq; ++t)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sbase + 8u * t),
                             "l"(g + (long long)t * pitch), "r"(nbytes)
                             : "memory");
        } else {
            // FP32 rows: asynchronous 4-byte copies into the upper half of
            // the chunk's slots (float t at float offset RS + t), widened in
            // place below (double t covers floats 2t, 2t + 1 < RS + t for
            // t < RS, so each float is read before it is overwritten).
            const float* g = specf + go;
            const unsigned fbase = (unsigned)__cvta_generic_to_shared(reinterpret_cast<float*>(sdst) + RS);
            const int nbytes = colok ? 4 : 0;
            for (int t = 0; t < Rq; ++t)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(fbase + 4u * t),
                             "l"(g + (long long)t * pitch), "r"(nbytes)
                             : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        if (f32) {
            const float* fsrc = reinterpret_cast<const float*>(sdst) + RS;
            for (int t = 0; t < Rq; ++t) sdst[t] = (double)fsrc[t];
        }
        // Register sweeps: the rows past the column's end are zeros (after
        // the widening above, whose staging area they overlap).
        if (RR > 0 && R == RR)
            for (int t = max(Rq, 0); t < R; ++t) sdst[t] = 0.0;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = warp % KT, h = warp / KT;  // column, and which W-th of it
    const int q = h * 32 + lane;             // chunk
    const int kk = k0 + c;                   // 0-based wavenumber index
    const bool active = kk < n;
    const int a = q * R + 1;                 // first row position (1-based) of the chunk
    const int cnt = max(0, min(R, Mr - q * R));
    const int b = a + cnt - 1;
    double* s = strip + c * CS + q * RS;     // s[t] is position a + t
    const double* gs = gstrip + c * CS + q * RS;  // GS: gs[t] = g(a + t)
    PivotRow g{nullptr, 0, 0.0};
    if (!GS && active) {
        const int mk = m * n + kk;
        g = PivotRow{Mb.piv + __ldg(&Mb.piv_off[mk]), __ldg(&Mb.piv_len[mk]), __ldg(&Mb.piv_fix[mk])};
    }
    // g(p) for p in [a - 1, b]: g(a - 1) is the previous chunk's last pivot.
    auto G = [&](int p) -> double {
        if constexpr (GS) {
            const int t = p - a;
            return t >= 0 ? gs[t] : gstrip[c * CS + (q - 1) * RS + (R - 1)];
        } else {
            return g(p);
        }
    };
    // Register sweeps (RR > 0 and R == RR: every chunk exactly RR rows, the
    // column's end padded with rows whose value and pivot are 0) take the
    // chunk into v[] and its pivots into gv[] (gv[u] = g(a + u - 1)) once,
    // without the lambda, so that both arrays stay in registers: the loops
    // below have constant trip counts and no guards (a guard on a chunk's row
    // count turns a loop bound into a runtime one and the arrays into local
    // memory).  A padded row's x is 0 (pivot 0), so it changes no real row,
    // no chunk map that a real row uses, and no column sum.  Four sweeps on
    // registers: two shared-memory accesses per row instead of eight.
    const bool regs = RR > 0 && R == RR;
    constexpr int RV = RR > 0 ? RR : 1;
    double v[RV] = {}, gv[RV + 1] = {};
    if constexpr (RR > 0) {
        if (regs) {
#pragma unroll
            for (int u = 0; u <= RR; ++u) {
                const int p = a + u - 1;
                double gg;
                if constexpr (GS)
                    gg = u >= 1 ? gs[u - 1] : gstrip[c * CS + max(q - 1, 0) * RS + (R - 1)];
                else
                    gg = g(max(p, 1));
                gv[u] = (active && p >= 1 && p <= Mr) ? gg : 0.0;
            }
#pragma unroll
            for (int t = 0; t < RR; ++t) v[t] = s[t];
        }
    }

    // Forward elimination, local: y~_a = f_a, y~_p = f_p - g_{p-1} y~_{p-1};
    // y_p = y~_p + A_p y_{a-1}, A_a = -g_{a-1}, A_p = -g_{p-1} A_{p-1}.
    double A = 1.0, cend = 0.0;
    if (active && cnt > 0) {
        if (regs) {
            A = (a > 1) ? -gv[0] : 0.0;
            double y = v[0];
#pragma unroll
            for (int t = 1; t < RV; ++t) {
                const double gp = gv[t];
                y = v[t] - gp * y;
                v[t] = y;
                A = -gp * A;
            }
            cend = y;
        } else {
            A = (a > 1) ? -G(a - 1) : 0.0;
            double y = s[0];
            for (int t = 1; t < cnt; ++t) {
                const double gp = G(a + t - 1);
                y = s[t] - gp * y;
                s[t] = y;
                A = -gp * A;
            }
            cend = y;
        }
    }
    // Inclusive scan of the affine chunk maps y_out = c + A y_in in the warp,
    // then the column's earlier warps' totals composed in order.
    double sA = A, sc = cend;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double pA = __shfl_up_sync(0xffffffffu, sA, o);
        const double pc = __shfl_up_sync(0xffffffffu, sc, o);
        if (lane >= o) {
            sc = sc + sA * pc;
            sA = sA * pA;
        }
    }
    if (lane == 31) {
        tot[0][warp][0] = sA;
        tot[0][warp][1] = sc;
    }
    __syncthreads();
    double y0 = 0.0;  // y entering this warp's first chunk
    for (int hh = 0; hh < h; ++hh) y0 = tot[0][hh * KT + c][1] + tot[0][hh * KT + c][0] * y0;
    const double eA = __shfl_up_sync(0xffffffffu, sA, 1), ec = __shfl_up_sync(0xffffffffu, sc, 1);
    const double yin = (lane == 0) ? y0 : ec + eA * y0;
    // Fix-up of y, then the local back substitution from the chunk end:
    // x~_b = y_b g_b, x~_p = (y_p - x~_{p+1}) g_p; x_p = x~_p + B_p x_{b+1},
    // B_b = -g_b, B_p = -g_p B_{p+1}.
    double B = 1.0, cstart = 0.0;
    if (active && cnt > 0) {
        if (regs) {
            double Ap = (a > 1) ? -gv[0] : 0.0;
            v[0] = v[0] + Ap * yin;
#pragma unroll
            for (int t = 1; t < RV; ++t) {
                Ap = -gv[t] * Ap;
                v[t] = v[t] + Ap * yin;
            }
            const double gb = gv[RV];  // g(b)
            double x = v[RV - 1] * gb;
            v[RV - 1] = x;
            B = -gb;
#pragma unroll
            for (int t = RV - 2; t >= 0; --t) {
                const double gp = gv[t + 1];
                x = (v[t] - x) * gp;
                v[t] = x;
                B = -gp * B;
            }
            cstart = x;
        } else {
            double Ap = (a > 1) ? -G(a - 1) : 0.0;
            const double gb = G(b);
            s[0] = s[0] + Ap * yin;
            for (int t = 1; t < cnt; ++t) {
                Ap = -G(a + t - 1) * Ap;
                s[t] = s[t] + Ap * yin;
            }
            double x = s[cnt - 1] * gb;
            s[cnt - 1] = x;
            B = -gb;
            for (int t = cnt - 2; t >= 0; --t) {
                const double gp = G(a + t);
                x = (s[t] - x) * gp;
                s[t] = x;
                B = -gp * B;
            }
            cstart = x;
        }
    }
    // Reverse inclusive scan of x_start = c + B x_next, then the column's
    // later warps' totals composed in order.
    double rB = B, rc = cstart;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double nB = __shfl_down_sync(0xffffffffu, rB, o);
        const double nc = __shfl_down_sync(0xffffffffu, rc, o);
        if (lane + o < 32) {
            rc = rc + rB * nc;
            rB = rB * nB;
        }
    }
    if (lane == 0) {
        tot[1][warp][0] = rB;
        tot[1][warp][1] = rc;
    }
    __syncthreads();
    double x0 = 0.0;  // x entering this warp's last chunk from above
    for (int hh = W - 1; hh > h; --hh) x0 = tot[1][hh * KT + c][1] + tot[1][hh * KT + c][0] * x0;
    const double nB = __shfl_down_sync(0xffffffffu, rB, 1), nc = __shfl_down_sync(0xffffffffu, rc, 1);
    const double xin = (lane == 31) ? x0 : nc + nB * x0;
    double lsum = 0.0;
    if (active && cnt > 0) {
        if (regs) {
            double Bp = -gv[RV];
#pragma unroll
            for (int t = RV - 1; t >= 0; --t) {
                if (t < RV - 1) Bp = -gv[t + 1] * Bp;
                const double u = v[t] + Bp * xin;
                lsum += u;
                s[t] = u;
            }
        } else {
            double Bp = -G(b);
            double u = s[cnt - 1] + Bp * xin;
            s[cnt - 1] = u;
            lsum += u;
            for (int t = cnt - 2; t >= 0; --t) {
                Bp = -G(a + t) * Bp;
                u = s[t] + Bp * xin;
                s[t] = u;
                lsum += u;
            }
        }
    }
    if (Mb.periodic) {
        // periodic_ge (qg3p_helmholtz.F90:565-610): the cyclic closure
        // through the rows 1 and jj, which the Thomas solve above leaves
        // out, as two rank-one corrections with the precomputed b, c.
        __syncthreads();
        double z1 = 0.0, zj = 0.0;
        if (active) {
            const double* pb = Mb.pb + (long long)m * jj * n + kk;
            const double* pc = Mb.pc + (long long)m * jj * n + kk;
            if (lane == 0) {
                const int ql = (Mr - 1) / R, tl = (Mr - 1) - ql * R;
                const double z2 = strip[c * CS];                 // row 2 (1-based) after the solve
                const double zl = strip[c * CS + ql * RS + tl];  // row jj-1
                // rows 1 and jj (0 and jj-1) of this mode's spectral field
                const double z1i = f32 ? (double)specf[kk] : spec[kk];
                const double zji = f32 ? (double)specf[(long long)(jj - 1) * pitch + kk]
                                       : spec[(long long)(jj - 1) * pitch + kk];
                z1 = (z1i - z2) / __ldg(&pb[0]);
                zj = ((zji - zl) - z1 * __ldg(&pb[(long long)(jj - 1) * n])) / __ldg(&pc[(long long)(jj - 1) * n]);
            }
            z1 = __shfl_sync(0xffffffffu, z1, 0);
            zj = __shfl_sync(0xffffffffu, zj, 0);
        }
        __syncthreads();  // every warp has read rows 1 and jj before they are written
        if (active && h == 0 && lane == 0) {
            const double r0 = z1 - zj * __ldg(&Mb.pc[(long long)m * jj * n + kk]);
            if (f32) {
                specf[kk] = (float)r0;
                specf[(long long)(jj - 1) * pitch + kk] = (float)zj;
            } else {
                spec[kk] = r0;
                spec[(long long)(jj - 1) * pitch + kk] = zj;
            }
        }
        if (active)
            for (int t = 0; t < cnt; ++t) {
                const long long row = a + t;  // 0-based grid row
                s[t] = (s[t] - z1 * __ldg(&Mb.pb[((long long)m * jj + row) * n + kk])) -
                       zj * __ldg(&Mb.pc[((long long)m * jj + row) * n + kk]);
            }
        if (do_mean) {
            // The column sum over every row of the closed solution.
            lsum = 0.0;
            for (int t = 0; t < cnt; ++t) lsum += s[t];
            if (active && h == 0 && lane == 0) lsum += (z1 - zj * __ldg(&Mb.pc[(long long)m * jj * n + kk])) + zj;
        }
    }
    // Closed basin: the domain mean of the mode (wmean weights).  Channel:
    // the mean PV of the two walls (zeta_boundary of the solved mode,
    // qg3p_aux.F90:289-379), linear in the column sums: sum_j phi(i, j) =
    // 2 sum_k sin(i k pi / N) C_k, so wall i = 0 gets wwall[k] C_k and wall
    // ii - 1 gets (-1)^(k+1) wwall[k] C_k.
    double colsum = 0.0, colsum2 = 0.0;
    if (active && do_mean) {
        const double cs = warp_sum(lsum);
        if (Mb.periodic) {
            const double w = __ldg(&Mb.wwall[kk]);
            colsum = cs * w;
            colsum2 = (kk & 1) ? -colsum : colsum;
        } else {
            colsum = cs * __ldg(&Mb.wmean[kk]);
        }
    }
    if (lane == 0) {
        wpart[warp] = colsum;
        wpart2[warp] = colsum2;
    }
    pdl_release();
    __syncthreads();
    {
        const int cc = threadIdx.x % KT, qq = threadIdx.x / KT;
        if (k0 + cc < n) {
            const long long go = (long long)(qq * R + 1) * pitch + k0 + cc;
            const double* ssrc = strip + cc * CS + qq * RS;
            const int Rq = min(R, Mr - qq * R);
            if (!f32) {
                double* gdst = spec + go;
                for (int t = 0; t < Rq; ++t) gdst[(long long)t * pitch] = ssrc[t];
            } else {
                float* gdst = specf + go;
                for (int t = 0; t < Rq; ++t) gdst[(long long)t * pitch] = (float)ssrc[t];
            }
        }
    }
    if (!do_mean) return;
    if (threadIdx.x == 0) {
        double t = 0.0, t2 = 0.0;
        for (int w = 0; w < TRI_THREADS / 32; ++w) {
            t += wpart[w];
            t2 += wpart2[w];
        }
        Mb.partials[local] = t;
        if (Mb.periodic) Mb.partials[Mb.ntiles_tri + local] = t2;
    }
    // do_mean 2 (closed basin, an inverse DST of one wave): its CTAs sum the
    // partials themselves (psiC_m, while their rows load), so no CTA here
    // waits on a counter.
    if (!Mb.periodic && do_mean == 2) return;
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[0], 1u);
        is_last = (prev == (unsigned)(Mb.ntiles_tri - 1));
    }
    __syncthreads();
    if (!is_last) return;
    // Last CTA of this member, every sum in a fixed order so that the result
    // is independent of CTA timing.  Closed basin: psiC_m = (sum of partials)
    // / (g_ii_int g_jj_int).  Channel (modes_to_z_correct_momentum,
    // qg3p_aux.F90:524-575): the baroclinic modes' coefficients of the two
    // correction functions, inv_corr_a times the wall PV means; the
    // barotropic mode is not corrected.
    __threadfence();
    for (int mm = 0; mm < Mb.L; ++mm) {
        const double t = block_sum_l2(Mb.partials + (long long)mm * tiles_per_mode, tiles_per_mode, 1, wpart);
        double t2 = 0.0;
        if (Mb.periodic)
            t2 = block_sum_l2(Mb.partials + Mb.ntiles_tri + (long long)mm * tiles_per_mode, tiles_per_mode, 1,
                              wpart2);
        if (threadIdx.x == 0) {
            double pc, pc2 = 0.0;
            if (Mb.periodic) {
                const double* A = Mb.inv_corr_a + 4 * mm;
                pc = mm == 0 ? 0.0 : A[0] * t + A[2] * t2;
                pc2 = mm == 0 ? 0.0 : A[1] * t + A[3] * t2;
                Mb.sc->psiC2[mm] = pc2;
            } else {
                pc = t * Mb.mean_scale;
            }
            Mb.sc->psiC[mm] = pc;
            if (pc != pc || pc2 != pc2) atomicOr(Mb.status, (int)ST_NAN_PSIC);
            else if (fabs(pc) > 1.0e100 || fabs(pc2) > 1.0e100) atomicOr(Mb.status, (int)ST_LARGE_PSIC);
        }
    }
    if (threadIdx.x == 0) Mb.counters[0] = 0u;
}

__host__ __device__ inline size_t tri_smem_bytes(int jj) {
    const int W = tri_warps(jj), KT = 8 / W, NQ = 32 * W;
    const int Mr = jj - 2, R = (Mr + NQ - 1) / NQ, RS = R | 1;
    return (size_t)KT * (NQ * RS + 16) * sizeof(double);  // tri_cs pads by at most 15
}

// ---------------------------------------------------------------------------
// Host launchers.
int dst_lanes_default(int M, int L, int dir) { return dst_lanes_default_hd(M, L, dir); }
// Batched solves fill the GPU with many members' rows: throughput, not one
// row's latency, bounds them, so units keep 8 values per lane (fewer passes
// and shared-memory round trips per value) up to M = 256, then one warp.
int dst_lanes_batched(int M) {
    const int V = M <= 2 ? 2 : M == 4 ? 4 : M <= 256 ? 8 : M / 32;
    return M / V;
}
int dst_max_threads_host(int V) { return dst_max_threads(V); }
int dst_rows_per_cta_host(int P, int c) { return dst_rows_per_cta(P, c); }

// Whether the inverse DST sums the closed basin's psiC itself: when its grid
// is one wave (at most four CTAs per SM; measured: +1 % per step at 513^2 x 3,
// +2.4 % at 129^2, but -1.2 % at 1025^2, whose inverse runs in several waves),
// so that the tridiagonal kernel's CTAs skip the last-CTA counter.  The
// tridiagonal launch and the inverse launch decide from the same LaunchSet.
static int psic_in_inverse(const LaunchSet& ls) {
    return (!ls.periodic && ls.ctas_dst[1] <= 4 * ls.sm_count) ? 1 : 0;
}

template <typename S, int V, int PRO, int EPI>
static cudaError_t launch_dst_v(const LaunchSet& ls, cudaStream_t st) {
    const int M = ls.maxN / 2, L = ls.maxL;
    const int R = dst_rows_per_cta(M / V, ls.dst_group);
    const int threads = L * R * (M / V);
    size_t bytes = (size_t)L * R * dst_unit_len(ls.maxN) * sizeof(double);
    const size_t cbytes = (size_t)R * (L - 1) * ls.maxPitch * sizeof(double);
    const int corr_smem = (EPI == EPI_PV && !ls.periodic && bytes + cbytes <= 200 * 1024) ? 1 : 0;
    if (corr_smem) bytes += cbytes;
    if (sizeof(S) == 4 && EPI == EPI_SPEC && PRO != PRO_STEP)
        bytes += (size_t)R * L * ls.maxN * (PRO == PRO_PLAIN ? sizeof(double) : sizeof(float));
    // The inverse with 64-lane units of 8 values takes the register-capped
    // instance (1025^2 x 3: 41.1 -> 37.3 us mixed, 44.5 -> 41.7 us FP64).
    void (*kern)(const Member*, const int*, int, int, int, int, int, Member, int, int) = k_dst<S, V, PRO, EPI>;
    if constexpr (EPI == EPI_PV && V == 8) {
        if (M / V == 64) kern = k_dst_capped<S, V, PRO, EPI>;
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    const int dir = (EPI == EPI_SPEC) ? 0 : 1;
    return launch_step_kernel(ls.pdl, kern, dim3(ls.ctas_dst[dir]), dim3(threads), bytes, st,
                              ls.members, ls.prefix_dst[dir], ls.nmem, (EPI == EPI_SPEC && !ls.periodic) ? 1 : 0,
                              ls.dst_group, corr_smem, (EPI == EPI_PV) ? psic_in_inverse(ls) : 0, member_arg(ls),
                              member_arg_used(ls), sizeof(S) == 4 ? ls.gemm_bc : 0);
}

template <typename S, int PRO, int EPI>
static cudaError_t launch_dst(const LaunchSet& ls, cudaStream_t st) {
    switch (ls.maxN / 2 / ls.dst_lanes[EPI == EPI_SPEC ? 0 : 1]) {
        case 2: return launch_dst_v<S, 2, PRO, EPI>(ls, st);
        case 4: return launch_dst_v<S, 4, PRO, EPI>(ls, st);
        case 8: return launch_dst_v<S, 8, PRO, EPI>(ls, st);
        case 16: return launch_dst_v<S, 16, PRO, EPI>(ls, st);
        case 32: return launch_dst_v<S, 32, PRO, EPI>(ls, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_dst_forward(const LaunchSet& ls, int prologue, int f32, cudaStream_t st) {
    switch (prologue) {
        case PRO_PLAIN:
            return f32 ? launch_dst<float, PRO_PLAIN, EPI_SPEC>(ls, st) : launch_dst<double, PRO_PLAIN, EPI_SPEC>(ls, st);
        case PRO_MODAL:
            return f32 ? launch_dst<float, PRO_MODAL, EPI_SPEC>(ls, st) : launch_dst<double, PRO_MODAL, EPI_SPEC>(ls, st);
        default:
            return f32 ? launch_dst<float, PRO_STEP, EPI_SPEC>(ls, st) : launch_dst<double, PRO_STEP, EPI_SPEC>(ls, st);
    }
}

cudaError_t launch_dst_inverse(const LaunchSet& ls, int epilogue, int f32, cudaStream_t st) {
    if (epilogue == EPI_HELM)
        return f32 ? launch_dst<float, PRO_PLAIN, EPI_HELM>(ls, st) : launch_dst<double, PRO_PLAIN, EPI_HELM>(ls, st);
    return f32 ? launch_dst<float, PRO_PLAIN, EPI_PV>(ls, st) : launch_dst<double, PRO_PLAIN, EPI_PV>(ls, st);
}

template <typename S, bool GS, int RR>
static cudaError_t launch_tri(const LaunchSet& ls, int do_mean, size_t bytes, cudaStream_t st) {
    cudaError_t e =
        cudaFuncSetAttribute(k_tridiag<S, GS, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    cudaError_t le = launch_step_kernel(ls.pdl, k_tridiag<S, GS, RR>, dim3(ls.ctas_tri), dim3(TRI_THREADS), bytes, st,
                                        ls.members, ls.prefix_tri, ls.nmem, do_mean, member_arg(ls),
                                        member_arg_used(ls));
    if (le != cudaSuccess) return le;
    return cudaGetLastError();
}

// Resident CTAs per SM of k_tridiag<S, GS, RR> with `bytes` of shared memory
// (cached per host thread for the last size asked: contexts may be driven
// from several threads).
template <typename S, bool GS, int RR>
static int tri_resident(size_t bytes) {
    thread_local size_t cached_bytes = 0;
    thread_local int cached = 0;
    if (cached_bytes != bytes) {
        int n = 0;
        if (cudaFuncSetAttribute(k_tridiag<S, GS, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tridiag<S, GS, RR>, TRI_THREADS, bytes) !=
                cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        cached_bytes = bytes;
        cached = n;
    }
    return cached;
}

// Register sweeps read each pivot once per row, from the pivot table: staging
// the pivots beside the strip measured slower for them (1025^2 x 3: 33.4 us
// without, 36.5 with, mixed; 31.8 / 35.2 FP64), so only the shared-memory
// sweeps stage them.
template <typename S, int RR>
static cudaError_t launch_tri_gs(const LaunchSet& ls, int do_mean, size_t bytes, size_t gs_limit, cudaStream_t st) {
    if constexpr (RR > 0) {
        return launch_tri<S, false, RR>(ls, do_mean, bytes, st);
    } else {
        const bool gs =
            2 * bytes <= gs_limit && tri_resident<S, true, RR>(2 * bytes) >= tri_resident<S, false, RR>(bytes);
        return gs ? launch_tri<S, true, RR>(ls, do_mean, 2 * bytes, st)
                  : launch_tri<S, false, RR>(ls, do_mean, bytes, st);
    }
}

cudaError_t launch_tridiag(const LaunchSet& ls, int do_mean_in, int f32, cudaStream_t st) {
    const size_t bytes = tri_smem_bytes(ls.maxJ);
    const int do_mean = (do_mean_in && psic_in_inverse(ls)) ? 2 : do_mean_in;
    // Pivots staged beside the strip when both fit (the FP32 form, whose
    // strip is loaded synchronously, only while two CTAs still fit an SM) and
    // the staging costs no resident CTA per SM: measured on B200, staging that
    // lowers occupancy is slower (1025 x 1025 x 3: -2 % FP64, -4 % mixed per
    // step; 2049 x 2049 x 5 FP64: -4 %).
    // Chunks of 4, 8 or 16 rows are solved in registers (the instance for
    // the largest member's chunk length; a member whose chunks differ takes
    // the shared-memory sweeps inside it).
    const int W = tri_warps(ls.maxJ), R = (ls.maxJ - 2 + 32 * W - 1) / (32 * W);
    if (f32) {
        if (R == 4) return launch_tri_gs<float, 4>(ls, do_mean, bytes, 100 * 1024, st);
        if (R == 8) return launch_tri_gs<float, 8>(ls, do_mean, bytes, 100 * 1024, st);
        if (R == 16) return launch_tri_gs<float, 16>(ls, do_mean, bytes, 100 * 1024, st);
        return launch_tri_gs<float, 0>(ls, do_mean, bytes, 100 * 1024, st);
    }
    if (R == 4) return launch_tri_gs<double, 4>(ls, do_mean, bytes, 160 * 1024, st);
    if (R == 8) return launch_tri_gs<double, 8>(ls, do_mean, bytes, 160 * 1024, st);
    if (R == 16) return launch_tri_gs<double, 16>(ls, do_mean, bytes, 160 * 1024, st);
    return launch_tri_gs<double, 0>(ls, do_mean, bytes, 160 * 1024, st);
}

}  // namespace pq
