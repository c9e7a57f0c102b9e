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
#include "pq_common.cuh"
#include "pq_kernels.h"

namespace pq {

enum { PRO_PLAIN = 0, PRO_MODAL = 1, PRO_STEP = 2 };
enum { EPI_SPEC = 0, EPI_HELM = 1, EPI_PV = 2 };

constexpr int DST_THREADS = 256;
constexpr int TRI_THREADS = 256;
constexpr int TRI_KT = 8;   // wavenumbers per tridiagonal CTA (one per warp)

__device__ __forceinline__ void load_member(Member& dst, const Member* src) {
    const int n = sizeof(Member) / 4;
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = s[t];
}

// Complex scratch rows are padded by one entry per 8 (index t -> t + t/8) so
// that the strided writes of the early Stockham stages hit distinct banks.
__device__ __forceinline__ int cpad(int t) { return t + (t >> 3); }
__host__ __device__ inline int crow(int M) { return M + (M >> 3); }  // padded row length

__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }  // a * (-i)

// Stockham FFT (radix 8, then 4, then 2) of G complex rows of length
// M = 2^logM in shared memory, forward sign; row g at a + g*crow(M), padded
// indexing.  Returns the buffer that holds the result (a or b).
__device__ double2* fft_stockham(double2* a, double2* b, int G, int M, int logM, const double2* tw) {
    const int MP = crow(M);
    int Ns = 1, logNs = 0;
    const double c8 = 0.70710678118654752440;  // sqrt(2)/2
    while (Ns * 8 <= M) {
        const int M8 = M >> 3, logM8 = logM - 3;
        const int lst = logM8 - logNs;  // log2(M / (8 Ns))
        for (int w = threadIdx.x; w < G * M8; w += blockDim.x) {
            const int g = w >> logM8, jj = w & (M8 - 1);
            const double2* ag = a + g * MP;
            double2* bg = b + g * MP;
            double2 v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = ag[cpad(jj + r * M8)];
            const int k = jj & (Ns - 1);
            if (k) {
#pragma unroll
                for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], tw[(r * k) << lst]);
            }
            // 8-point DFT: two 4-point DFTs of the even and odd inputs.
            const double2 e0 = cadd(v[0], v[4]), e1 = csub(v[0], v[4]), e2 = cadd(v[2], v[6]),
                          e3 = mul_mi(csub(v[2], v[6]));
            const double2 E0 = cadd(e0, e2), E1 = cadd(e1, e3), E2 = csub(e0, e2), E3 = csub(e1, e3);
            const double2 o0 = cadd(v[1], v[5]), o1 = csub(v[1], v[5]), o2 = cadd(v[3], v[7]),
                          o3 = mul_mi(csub(v[3], v[7]));
            double2 O0 = cadd(o0, o2), O1 = cadd(o1, o3), O2 = csub(o0, o2), O3 = csub(o1, o3);
            // W8^1 = (1 - i)/sqrt2, W8^2 = -i, W8^3 = (-1 - i)/sqrt2
            O1 = make_double2(c8 * (O1.x + O1.y), c8 * (O1.y - O1.x));
            O2 = mul_mi(O2);
            O3 = make_double2(c8 * (O3.y - O3.x), -c8 * (O3.x + O3.y));
            const int idx = ((jj >> logNs) << (logNs + 3)) + k;
            bg[cpad(idx)] = cadd(E0, O0);
            bg[cpad(idx + Ns)] = cadd(E1, O1);
            bg[cpad(idx + 2 * Ns)] = cadd(E2, O2);
            bg[cpad(idx + 3 * Ns)] = cadd(E3, O3);
            bg[cpad(idx + 4 * Ns)] = csub(E0, O0);
            bg[cpad(idx + 5 * Ns)] = csub(E1, O1);
            bg[cpad(idx + 6 * Ns)] = csub(E2, O2);
            bg[cpad(idx + 7 * Ns)] = csub(E3, O3);
        }
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
        Ns <<= 3;
        logNs += 3;
    }
    if (Ns * 4 <= M) {
        const int M4 = M >> 2, logM4 = logM - 2;
        const int lst = logM4 - logNs;
        for (int w = threadIdx.x; w < G * M4; w += blockDim.x) {
            const int g = w >> logM4, jj = w & (M4 - 1);
            const double2* ag = a + g * MP;
            double2* bg = b + g * MP;
            double2 v0 = ag[cpad(jj)], v1 = ag[cpad(jj + M4)], v2 = ag[cpad(jj + 2 * M4)], v3 = ag[cpad(jj + 3 * M4)];
            const int k = jj & (Ns - 1);
            if (k) {
                v1 = cmul(v1, tw[k << lst]);
                v2 = cmul(v2, tw[(2 * k) << lst]);
                v3 = cmul(v3, tw[(3 * k) << lst]);
            }
            const double2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = mul_mi(csub(v1, v3));
            const int idx = ((jj >> logNs) << (logNs + 2)) + k;
            bg[cpad(idx)] = cadd(t0, t2);
            bg[cpad(idx + Ns)] = cadd(t1, t3);
            bg[cpad(idx + 2 * Ns)] = csub(t0, t2);
            bg[cpad(idx + 3 * Ns)] = csub(t1, t3);
        }
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
        Ns <<= 2;
        logNs += 2;
    }
    if (Ns < M) {
        const int M2 = M >> 1, logM2 = logM - 1;
        const int lst = logM2 - logNs;
        for (int w = threadIdx.x; w < G * M2; w += blockDim.x) {
            const int g = w >> logM2, jj = w & (M2 - 1);
            const double2* ag = a + g * MP;
            double2* bg = b + g * MP;
            double2 v0 = ag[cpad(jj)], v1 = ag[cpad(jj + M2)];
            const int k = jj & (Ns - 1);
            if (k) v1 = cmul(v1, tw[k << lst]);
            const int idx = ((jj >> logNs) << (logNs + 1)) + k;
            bg[cpad(idx)] = cadd(v0, v1);
            bg[cpad(idx + Ns)] = csub(v0, v1);
        }
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
    }
    return a;
}

// In-place DST-I (FFTPACK sint convention) of G real rows held in shared
// memory at xr + g*xs, entries 1..n (entries 0 and N are scratch).
// za, zb: shared complex scratch of G*crow(M) each.  tw, wsp, was: the
// twiddle tables staged in shared memory.
__device__ void dst_rows(double* xr, int xs, int G, double2* za, double2* zb, const Member& Mb, const double2* tw,
                         const double2* wsp, const double* was) {
    const int N = Mb.N, M = Mb.M, N2 = N >> 1, logM = Mb.logM, MP = crow(M);
    // Pre-twiddle (sint1, qg3p_helmholtz.F90:1404-1413) and pack.
    for (int w = threadIdx.x; w < G * M; w += blockDim.x) {
        const int g = w >> logM, t = w & (M - 1);
        const double* x = xr + g * xs;
        double c[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int k = 2 * t + e;
            double v;
            if (k == 0) {
                v = 0.0;
            } else if (k == N2) {
                v = 4.0 * x[N2];
            } else if (k < N2) {
                const double xa = x[k], xb = x[N - k];
                v = (xa - xb) + was[k] * (xa + xb);
            } else {
                const int kk = N - k;
                const double xa = x[kk], xb = x[k];
                v = was[kk] * (xa + xb) - (xa - xb);
            }
            c[e] = v;
        }
        za[g * MP + cpad(t)] = make_double2(c[0], c[1]);
    }
    __syncthreads();
    double2* Z = fft_stockham(za, zb, G, M, logM, tw);
    double2* other = (Z == za) ? zb : za;
    // Real-FFT split; even outputs directly, R_q to scratch for the scan.
    for (int w = threadIdx.x; w < G * M; w += blockDim.x) {
        const int g = w >> logM, q = w & (M - 1);
        const double2* Zg = Z + g * MP;
        const double2 zq = Zg[cpad(q)];
        const double2 zr = Zg[cpad((M - q) & (M - 1))];
        const double2 zc = make_double2(zr.x, -zr.y);
        const double2 E = make_double2(0.5 * (zq.x + zc.x), 0.5 * (zq.y + zc.y));
        const double2 d = csub(zq, zc);
        const double2 O = make_double2(0.5 * d.y, -0.5 * d.x);
        const double2 C = cadd(E, cmul(wsp[q], O));
        reinterpret_cast<double*>(other + g * MP)[q] = (q == 0) ? 0.5 * C.x : C.x;
        if (q >= 1) xr[g * xs + 2 * q] = -C.y;
    }
    __syncthreads();
    // X_{2q+1} = inclusive prefix sum of R over q: one warp per row, each lane
    // a contiguous run of M/32 values (or one value when M < 32).
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int per = M >= 32 ? (M >> 5) : 1;
    for (int g = warp; g < G; g += nw) {
        const double* Rg = reinterpret_cast<const double*>(other + g * MP);
        const int q0 = lane * per;
        double loc = 0.0;
        for (int e = 0; e < per; ++e)
            if (q0 + e < M) loc += Rg[q0 + e];
        const double incl = warp_inclusive_scan(loc);
        double run = incl - loc;
        double* x = xr + g * xs;
        for (int e = 0; e < per; ++e) {
            const int q = q0 + e;
            if (q < M) {
                run += Rg[q];
                x[2 * q + 1] = run;
            }
        }
    }
    __syncthreads();
}

// Persistent, software-pipelined row transforms.
//
// Each CTA walks the rows (tasks) blockIdx.x, blockIdx.x + gridDim.x, ...
// With two staging buffers it issues the asynchronous copies (cp.async) of the
// next row's inputs before transforming the current row, so the global-load
// latency of a row overlaps the previous row's FFT.  A staging buffer holds
// the L real rows (stride N + 2, entries 1..n) and, for the psi epilogue, the
// L - 1 correction rows of the baroclinic modes (stride cs).

__device__ __forceinline__ void cp8(double* dst, const double* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

struct DstPlan {
    int G, nbuf;
    size_t buf_doubles;  // per staging buffer
    size_t bytes;        // dynamic shared memory
};

// Shared-memory tables of the DST for transform length N: tw[M], wsplit[M]
// (complex), was[N/2 + 1]; rounded up to an even count so that the complex
// scratch behind it stays 16-byte aligned.
__host__ __device__ inline size_t dst_tab_doubles(int N) { return ((size_t)2 * N + (N / 2 + 3)) & ~(size_t)1; }

__host__ inline DstPlan dst_plan(int L, int N, int ii, int want_G, bool with_corr) {
    DstPlan p;
    const int M = N / 2;
    (void)ii;
    (void)with_corr;
    p.buf_doubles = (size_t)L * (N + 2);
    int G = want_G > 0 ? (want_G < L ? want_G : L) : L;
    auto total = [&](int g, int nb) {
        return nb * p.buf_doubles * sizeof(double) + dst_tab_doubles(N) * sizeof(double) +
               2 * (size_t)g * crow(M) * sizeof(double2);
    };
    if (want_G <= 0)
        while (G > 1 && total(G, 2) > 110 * 1024) --G;
    p.G = G;
    p.nbuf = total(G, 2) <= 200 * 1024 ? 2 : 1;
    p.bytes = total(G, p.nbuf);
    return p;
}

template <int PRO, int EPI>
__global__ void __launch_bounds__(DST_THREADS) k_dst_rows(const Member* __restrict__ mems,
                                                            const int* __restrict__ prefix, int nmem, int G,
                                                            int nbuf, int row_offset, int total, size_t bufd) {
    __shared__ Member Mb;
    extern __shared__ __align__(16) double sm[];
    double* bufs[2] = {sm, sm + bufd};
    double* tab = sm + nbuf * bufd;  // twiddle tables of the current member
    double2* s_tw = reinterpret_cast<double2*>(tab);
    double2* za = nullptr;  // set once the member's N is known

    // Asynchronous copies of a task's inputs into a staging buffer.
    auto issue = [&](int task, double* buf) {
        int loc;
        const int mi = find_member(prefix, nmem, task, &loc);
        const Member* M = mems + mi;
        const int j = loc + row_offset;
        const int L = M->L, n = M->n, N = M->N, jj = M->jj, pitch = M->pitch;
        const long long ls = M->lstride;
        const int xs = N + 2;
        if (EPI == EPI_SPEC) {
            if (PRO == PRO_STEP) return;  // loaded synchronously (needs four fields)
            const double* src = reinterpret_cast<const double*>(PRO == PRO_PLAIN ? M->helm_io : M->zeta);
            for (int l = 0; l < L; ++l) {
                const double* g = src + l * ls + (long long)j * pitch;
                for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) cp8(buf + l * xs + k, g + k);
            }
        } else {
            if (j >= 1 && j <= jj - 2) {
                const double* spec = reinterpret_cast<const double*>(M->spec);
                for (int m = 0; m < L; ++m) {
                    const double* g = spec + m * ls + (long long)j * pitch - 1;
                    for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) cp8(buf + m * xs + k, g + k);
                }
            }
        }
    };

    int cur_mi = -1, it = 0;
    int task = blockIdx.x;
    if (task < total) issue(task, bufs[0]);
    cp_commit();
    for (; task < total; task += gridDim.x, ++it) {
        double* xr = bufs[nbuf == 2 ? (it & 1) : 0];
        const int nt = task + gridDim.x;
        if (nbuf == 2) {
            if (nt < total) issue(nt, bufs[(it + 1) & 1]);
            cp_commit();
            cp_wait1();
        } else {
            cp_wait0();
        }
        __syncthreads();
        int local;
        const int mi = find_member(prefix, nmem, task, &local);
        if (mi != cur_mi) {
            load_member(Mb, mems + mi);
            __syncthreads();
            // Stage this member's twiddle tables in shared memory.
            const int Mm = Mb.M, Nn = Mb.N;
            for (int t = threadIdx.x; t < Mm; t += blockDim.x) {
                s_tw[t] = Mb.tw[t];
                s_tw[Mm + t] = Mb.wsplit[t];
            }
            for (int t = threadIdx.x; t <= Nn / 2; t += blockDim.x) tab[4 * Mm + t] = Mb.was[t];
            za = reinterpret_cast<double2*>(tab + dst_tab_doubles(Nn));
            __syncthreads();
            cur_mi = mi;
        }
        const double2* t_tw = s_tw;
        const double2* t_ws = s_tw + Mb.M;
        const double* t_was = tab + 4 * Mb.M;
        const int j = local + row_offset;
        const int L = Mb.L, N = Mb.N, n = Mb.n, ii = Mb.ii, jj = Mb.jj, pitch = Mb.pitch;
        const long long ls = Mb.lstride;
        const int xs = N + 2;
        double2* zb = za + (size_t)G * crow(Mb.M);
        const bool interior_row = (j >= 1 && j <= jj - 2);

        if (EPI == EPI_SPEC) {
            // ---------------- forward: prologue ----------------------------------
            const double cff = 0.5 / (double)(ii - 1);
            for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) {
                const long long o = (long long)j * pitch + k;
                double v[PQ_MAXL];
                double z[PQ_MAXL];
                if (PRO == PRO_STEP) {
                    const double dt = Mb.sc->dt, ta = Mb.sc->tweight_a;
                    const double* zo = reinterpret_cast<const double*>(Mb.zeta_old[Mb.cur]);
                    const double* rs = reinterpret_cast<const double*>(Mb.res);
                    double* rb = reinterpret_cast<double*>(Mb.res_beta);
                    const double* ui = reinterpret_cast<const double*>(Mb.ui);
                    double* zp = reinterpret_cast<double*>(Mb.zeta);
                    for (int l = 0; l < L; ++l) {
                        const long long ol = o + l * ls;
                        // cabaret_predictor, qg3p_aux.F90:1012-1018
                        double zz = zo[ol] + 0.5 * dt * rs[ol];
                        // cabaret_beta, qg3p_aux.F90:1051-1059
                        const double rbn = dt * (0.5 * (ui[ol + 1] + ui[ol]) * Mb.beta[l]);
                        zz = zz + (1.0 + ta) * rbn - ta * rb[ol];
                        rb[ol] = rbn;
                        zp[ol] = zz;
                        z[l] = zz;
                    }
                } else {
                    for (int l = 0; l < L; ++l) z[l] = xr[l * xs + k];
                }
                if (PRO == PRO_PLAIN) {
                    for (int m = 0; m < L; ++m) v[m] = z[m];
                } else {
                    // z_to_modes, qg3p_diagnostics.F90:545-549
                    for (int m = 0; m < L; ++m) {
                        double s = 0.0;
                        for (int l = 0; l < L; ++l) s += Mb.z2m[m * PQ_MAXL + l] * z[l];
                        v[m] = s;
                    }
                }
                for (int m = 0; m < L; ++m) xr[m * xs + k] = cff * v[m];
            }
            __syncthreads();
            for (int m0 = 0; m0 < L; m0 += G)
                dst_rows(xr + m0 * xs, xs, min(G, L - m0), za, zb, Mb, t_tw, t_ws, t_was);
            double* spec = reinterpret_cast<double*>(Mb.spec);
            for (int m = 0; m < L; ++m) {
                double* g = spec + m * ls + (long long)j * pitch - 1;
                for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) g[k] = xr[m * xs + k];
            }
        } else {
            // ---------------- inverse: DST of the solved spectral rows ----------
            if (interior_row)
                for (int m0 = 0; m0 < L; m0 += G)
                    dst_rows(xr + m0 * xs, xs, min(G, L - m0), za, zb, Mb, t_tw, t_ws, t_was);
            if (EPI == EPI_HELM) {
                // helm's in-place output: interior entries of interior rows, row
                // i = ii zeroed (:758-761); ge_local zeroes psi(2:ii-1, 1) (:1055-1057).
                double* io = reinterpret_cast<double*>(Mb.helm_io);
                if (interior_row) {
                    for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x)
                        for (int m = 0; m < L; ++m) io[(long long)j * pitch + k + m * ls] = xr[m * xs + k];
                    if (threadIdx.x == 0)
                        for (int m = 0; m < L; ++m) io[(long long)j * pitch + (ii - 1) + m * ls] = 0.0;
                } else if (j == 0) {
                    for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x)
                        for (int m = 0; m < L; ++m) io[k + m * ls] = 0.0;
                }
            } else {
                // psi_l = phi_1 - psiC_1 + sum_{m>=2} m2z(l,m) (phi_m - psiC_m corr_m)
                // (modes_to_z_btcu) on every node of row j; phi is zero on the
                // boundary (apply_dirichlet_bc(0), qg3p_aux.F90:470).
                const double* psiC = Mb.sc->psiC;
                const double* corr = Mb.corr;
                double* psi = Mb.psi;
                for (int i = threadIdx.x; i < ii; i += blockDim.x) {
                    const bool inner = interior_row && i >= 1 && i <= n;
                    const long long o = (long long)j * pitch + i;
                    double ph[PQ_MAXL];
                    for (int m = 0; m < L; ++m) ph[m] = inner ? xr[m * xs + i] : 0.0;
                    for (int l = 0; l < L; ++l) {
                        double dot = 0.0;
                        for (int m = 1; m < L; ++m)
                            dot += Mb.m2z[l * PQ_MAXL + m] * (ph[m] - psiC[m] * corr[o + m * ls]);
                        psi[o + l * ls] = (ph[0] - psiC[0]) + dot;
                    }
                }
            }
        }
        __syncthreads();
        if (nbuf == 1) {
            if (nt < total) issue(nt, bufs[0]);
            cp_commit();
        }
    }
    cp_wait0();
}

// ---------------------------------------------------------------------------
// Tridiagonal solves along j for 8 wavenumbers of one mode.
//
// The strip (Mr = jj - 2 rows x 8 wavenumbers) is staged in shared memory by
// wavenumber, and within a wavenumber by chunk: row p (0-based) of chunk
// q = p / R, t = p % R lives at c*CS + q*RS + t with RS = R | 1 and
// CS = 32*RS + 1 both odd, so the 32 lanes of a warp (one chunk each) hit 32
// distinct banks and the staging writes of 8 wavenumbers do too.  Lane q of
// warp c runs the forward and backward Thomas recurrences of its chunk of
// wavenumber c.
struct PivotRow {
    const double* piv;  // explicit reciprocal pivots, piv[p - 1] for p <= len
    int len;
    double fix;         // the fixed point for p > len
    __device__ __forceinline__ double operator()(int p) const { return p <= len ? __ldg(&piv[p - 1]) : fix; }
};

__global__ void __launch_bounds__(TRI_THREADS) k_tridiag(const Member* __restrict__ mems,
                                                          const int* __restrict__ prefix, int nmem, int do_mean) {
    __shared__ Member Mb;
    __shared__ double wpart[TRI_KT];
    __shared__ int is_last;
    extern __shared__ __align__(16) double strip[];
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    load_member(Mb, mems + mi);
    __syncthreads();
    const int n = Mb.n, jj = Mb.jj, pitch = Mb.pitch;
    const int tiles_per_mode = (n + TRI_KT - 1) / TRI_KT;
    const int m = local / tiles_per_mode;
    const int tile = local - m * tiles_per_mode;
    const int k0 = tile * TRI_KT;  // 0-based column (wavenumber k0+1)
    const int Mr = jj - 2;
    const int R = (Mr + 31) >> 5;
    const int RS = R | 1;
    const int CS = 32 * RS + 1;
    double* spec = reinterpret_cast<double*>(Mb.spec) + (long long)m * Mb.lstride;

    // Stage: thread -> (column c = tid & 7, chunk q = tid >> 3); loop over t.
    // Asynchronous 8-byte copies (cp.async), so the loads of a thread do not
    // wait for one another; columns past n are zero-filled (source size 0).
    {
        const int c = threadIdx.x & 7, q = threadIdx.x >> 3;
        const bool colok = (k0 + c < n);
        const double* g = spec + (long long)(q * R + 1) * pitch + (colok ? k0 + c : 0);
        double* sdst = strip + c * CS + q * RS;
        const int Rq = min(R, Mr - q * R);
        const unsigned sbase = (unsigned)__cvta_generic_to_shared(sdst);
        const int nbytes = colok ? 8 : 0;
        for (int t = 0; t < Rq; ++t)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sbase + 8u * t),
                         "l"(g + (long long)t * pitch), "r"(nbytes)
                         : "memory");
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = warp;
    const int kk = k0 + c;  // 0-based wavenumber index
    double colsum = 0.0;
    if (kk < n) {
        const int mk = m * n + kk;
        PivotRow g{Mb.piv + __ldg(&Mb.piv_off[mk]), __ldg(&Mb.piv_len[mk]), __ldg(&Mb.piv_fix[mk])};
        const int a = lane * R + 1;                 // first row position (1-based) of the chunk
        const int cnt = max(0, min(R, Mr - lane * R));
        const int b = a + cnt - 1;
        double* s = strip + c * CS + lane * RS;     // s[t] is position a + t
        // Forward elimination, local: y~_a = f_a, y~_p = f_p - g_{p-1} y~_{p-1};
        // y_p = y~_p + A_p y_{a-1}, A_a = -g_{a-1}, A_p = -g_{p-1} A_{p-1}.
        double A = 1.0, cend = 0.0;
        if (cnt > 0) {
            double y = s[0];
            A = (a > 1) ? -g(a - 1) : 0.0;
            for (int t = 1; t < cnt; ++t) {
                const double gp = g(a + t - 1);
                y = s[t] - gp * y;
                s[t] = y;
                A = -gp * A;
            }
            cend = y;
        }
        // Inclusive scan of the affine chunk maps y_out = c + A y_in.
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
        double yin = __shfl_up_sync(0xffffffffu, sc, 1);
        if (lane == 0) yin = 0.0;
        // Fix-up of y, then the local back substitution from the chunk end:
        // x~_b = y_b g_b, x~_p = (y_p - x~_{p+1}) g_p; x_p = x~_p + B_p x_{b+1},
        // B_b = -g_b, B_p = -g_p B_{p+1}.
        double B = 1.0, cstart = 0.0;
        if (cnt > 0) {
            double Ap = (a > 1) ? -g(a - 1) : 0.0;
            s[0] = s[0] + Ap * yin;
            for (int t = 1; t < cnt; ++t) {
                Ap = -g(a + t - 1) * Ap;
                s[t] = s[t] + Ap * yin;
            }
            const double gb = g(b);
            double x = s[cnt - 1] * gb;
            s[cnt - 1] = x;
            B = -gb;
            for (int t = cnt - 2; t >= 0; --t) {
                const double gp = g(a + t);
                x = (s[t] - x) * gp;
                s[t] = x;
                B = -gp * B;
            }
            cstart = x;
        }
        // Reverse inclusive scan of x_start = c + B x_next.
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
        double xin = __shfl_down_sync(0xffffffffu, rc, 1);
        if (lane == 31) xin = 0.0;
        double lsum = 0.0;
        if (cnt > 0) {
            double Bp = -g(b);
            double v = s[cnt - 1] + Bp * xin;
            s[cnt - 1] = v;
            lsum += v;
            for (int t = cnt - 2; t >= 0; --t) {
                Bp = -g(a + t) * Bp;
                v = s[t] + Bp * xin;
                s[t] = v;
                lsum += v;
            }
        }
        if (do_mean) colsum = warp_sum(lsum) * __ldg(&Mb.wmean[kk]);
    }
    if (lane == 0) wpart[warp] = colsum;
    __syncthreads();
    {
        const int cc = threadIdx.x & 7, q = threadIdx.x >> 3;
        if (k0 + cc < n) {
            double* gdst = spec + (long long)(q * R + 1) * pitch + k0 + cc;
            const double* ssrc = strip + cc * CS + q * RS;
            const int Rq = min(R, Mr - q * R);
            for (int t = 0; t < Rq; ++t) gdst[(long long)t * pitch] = ssrc[t];
        }
    }
    if (!do_mean) return;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < TRI_KT; ++w) t += wpart[w];
        Mb.partials[local] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[0], 1u);
        is_last = (prev == (unsigned)(Mb.ntiles_tri - 1));
    }
    __syncthreads();
    if (!is_last) return;
    // Last CTA of this member: psiC_m = (sum of partials) / (g_ii_int g_jj_int),
    // summed in a fixed order so that the result is independent of CTA timing.
    if (threadIdx.x < Mb.L) {
        __threadfence();
        const int mm = threadIdx.x;
        const volatile double* part = Mb.partials;
        double t = 0.0;
        for (int q = 0; q < tiles_per_mode; ++q) t += part[mm * tiles_per_mode + q];
        const double pc = t * Mb.mean_scale;
        Mb.sc->psiC[mm] = pc;
        if (pc != pc) atomicOr(Mb.status, (int)ST_NAN_PSIC);
        else if (fabs(pc) > 1.0e100) atomicOr(Mb.status, (int)ST_LARGE_PSIC);
    }
    if (threadIdx.x == 0) Mb.counters[0] = 0u;
}

__host__ __device__ inline size_t tri_smem_bytes(int jj) {
    const int Mr = jj - 2, R = (Mr + 31) >> 5, RS = R | 1;
    return (size_t)TRI_KT * (32 * RS + 1) * sizeof(double);
}

// ---------------------------------------------------------------------------
// Host launchers.
template <int PRO, int EPI>
static cudaError_t launch_dst(const LaunchSet& ls, cudaStream_t st) {
    const DstPlan p = dst_plan(ls.maxL, ls.maxN, ls.maxI, ls.dst_group, EPI == EPI_PV);
    cudaError_t e = cudaFuncSetAttribute(k_dst_rows<PRO, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.bytes);
    if (e != cudaSuccess) return e;
    const int* prefix = (EPI == EPI_SPEC) ? ls.prefix_rows_interior : ls.prefix_rows_all;
    const int total = (EPI == EPI_SPEC) ? ls.ctas_rows_interior : ls.ctas_rows_all;
    // Persistent grid: as many CTAs as fit on the device at once.
    int per_sm = (int)((227 * 1024) / (p.bytes + 2048));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    int grid = ls.sm_count * per_sm;
    if (grid > total) grid = total;
    k_dst_rows<PRO, EPI><<<grid, DST_THREADS, p.bytes, st>>>(ls.members, prefix, ls.nmem, p.G, p.nbuf,
                                                            EPI == EPI_SPEC ? 1 : 0, total, p.buf_doubles);
    return cudaGetLastError();
}

cudaError_t launch_dst_forward(const LaunchSet& ls, int prologue, cudaStream_t st) {
    switch (prologue) {
        case PRO_PLAIN: return launch_dst<PRO_PLAIN, EPI_SPEC>(ls, st);
        case PRO_MODAL: return launch_dst<PRO_MODAL, EPI_SPEC>(ls, st);
        default: return launch_dst<PRO_STEP, EPI_SPEC>(ls, st);
    }
}

cudaError_t launch_dst_inverse(const LaunchSet& ls, int epilogue, cudaStream_t st) {
    if (epilogue == EPI_HELM) return launch_dst<PRO_PLAIN, EPI_HELM>(ls, st);
    return launch_dst<PRO_PLAIN, EPI_PV>(ls, st);
}

cudaError_t launch_tridiag(const LaunchSet& ls, int do_mean, cudaStream_t st) {
    const size_t bytes = tri_smem_bytes(ls.maxJ);
    cudaError_t e = cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    k_tridiag<<<ls.ctas_tri, TRI_THREADS, bytes, st>>>(ls.members, ls.prefix_tri, ls.nmem, do_mean);
    return cudaGetLastError();
}

}  // namespace pq
