// pq_dst_mma.cu -- the sine transforms of the mixed form's baroclinic modes
// as dense DST-matrix contractions on the tensor cores (tcgen05, sm_100a).
//
// The transform is FFTPACK's unnormalised DST-I of the rows (sint,
// qg3p_helmholtz.F90:1370-1426, applied along i at :676-681 and :758-761):
//     X_k = 2 sum_{m=1}^{n} x_m sin(m k pi / N),   k = 1..n,  N = n + 1 = 2^p.
// It is its own inverse up to the factor 2N that the forward pre-scale
// 0.5 / (ii - 1) removes, so the forward and inverse passes are the same
// contraction.  The symmetry sin((N - m) k pi / N) = (-1)^(k+1) sin(m k pi / N)
// folds each row first:
//     odd  k = 2q + 1:  X_k = sum_{m=1}^{N/2} u_m C(m, k),  u_m = x_m + x_{N-m}  (u_{N/2} = x_{N/2})
//     even k = 2q:      X_k = sum_{m=1}^{N/2} v_m C(m, k),  v_m = x_m - x_{N-m}  (v_{N/2} = 0)
// with C(m, k) = 2 sin(m k pi / N): two products of (rows x N/2) by
// (N/2 x N/2), half the flops of the unfolded matrix.
//
// Precision: the rows are FP32 and the accumulation FP32 (in tensor
// memory); each operand is split into three BF16 terms, a = a1 + a2 + a3
// (a1 = bf16(a), a2 = bf16(a - a1), a3 = bf16(a - a1 - a2), 24 significant
// bits together), and the six products a_i c_j with i + j <= 4 are summed:
// the dropped terms are below 2^-24 relative, so the result has FP32
// accuracy (compensated three-term BF16 split).  The barotropic mode never
// comes here; it keeps its FP64 transform.
//
// Kernel.  A CTA computes a 128-row by NT-column tile of one parity's
// product: rows are (mode, j) pairs of the baroclinic spectral rows, columns
// are output wavenumbers.  Per 64-wide K block:
//   warps 0-7   load the FP32 rows (x_m and its mirror x_{N-m}; eight rows
//               per warp in flight at once), fold, split, and write the
//               three A terms into shared memory in the 128-byte-swizzled
//               K-major layout the MMA reads;
//   warp 8      one thread loads the three B-term tiles (the split DST
//               matrix, a constant table) with TMA (cp.async.bulk.tensor);
//   warp 9      one thread issues 4 K-steps x 6 tcgen05.mma (M 128, N NT,
//               K 16, BF16 x BF16 -> FP32 in tensor memory) and commits to
//               the stage's "empty" barrier.
// Two stages of shared memory alternate.  After the last K block the eight
// loader warps read the accumulator out of tensor memory (tcgen05.ld, each
// warp its lane quarter and half the columns), stage it through shared
// memory and write the output rows.
//
// Every wait is bounded: a wait that runs out sets ST_MMA_TIMEOUT in the
// member's status word, the CTA stops issuing work, waits (bounded) for the
// copies and products it already issued, frees its tensor memory and exits.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "pq_ctx.h"
#include "pq_dst_mma.h"

namespace pq {

namespace {

constexpr int BM = 128;        // rows per CTA (the MMA's M)
constexpr int BK = 64;         // K elements per stage (one 128-byte swizzle row of BF16)
constexpr int STAGES = 2;
constexpr int LOADERS = 8;      // loader / epilogue warps
constexpr int NTHREADS = 32 * (LOADERS + 2);  // + a TMA warp and an MMA warp
constexpr int RB = 8;          // rows a loader warp has in flight at once
constexpr unsigned kSpinLimit = 1u << 22;

__host__ __device__ constexpr int a_tile_bytes() { return BM * BK * 2; }           // 16 KB per term
__host__ __device__ constexpr int b_tile_bytes(int nt) { return nt * BK * 2; }     // nt x 64 BF16
__host__ __device__ constexpr int stage_bytes(int nt) { return 3 * a_tile_bytes() + 3 * b_tile_bytes(nt); }
__host__ __device__ constexpr int smem_bytes(int nt) { return STAGES * stage_bytes(nt) + 1024 /*align*/ + 256; }

// ---- PTX wrappers -------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of the given parity; false if it ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, const volatile int* abort_flag) {
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if (abort_flag && *abort_flag) return false;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// K-major operand tile in the 128-byte swizzle: rows of 128 bytes, groups of
// eight rows 1024 bytes apart (stride byte offset), version 1, layout 2.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
    unsigned long long d = 0;
    d |= (unsigned long long)((addr & 0x3FFFFu) >> 4);
    d |= (unsigned long long)1 << 16;             // leading byte offset (unused by this layout)
    d |= (unsigned long long)(1024 >> 4) << 32;   // stride byte offset
    d |= (unsigned long long)1 << 46;             // descriptor version
    d |= (unsigned long long)2 << 61;             // 128-byte swizzle
    return d;
}

// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major,
// N = nt, M = 128.
__host__ __device__ constexpr unsigned instr_desc(int nt) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(nt >> 3) << 17) | ((unsigned)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(unsigned tmem_d, unsigned long long a, unsigned long long b, unsigned idesc,
                                         unsigned accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float* v) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// Three-term BF16 split of an FP32 value (round to nearest even at each term).
__device__ __forceinline__ void split3(float a, __nv_bfloat16& a1, __nv_bfloat16& a2, __nv_bfloat16& a3) {
    a1 = __float2bfloat16_rn(a);
    const float r1 = a - __bfloat162float(a1);
    a2 = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(a2);
    a3 = __float2bfloat16_rn(r2);
}

// Byte offset of (row r, column c) (c even) in a 128-byte-swizzled K-major tile.
__device__ __forceinline__ unsigned sw128(int r, int c) {
    return (unsigned)(r * 128 + ((((c >> 3) ^ (r & 7)) & 7) << 4) + (c & 7) * 2);
}

}  // namespace

template <int NT>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_dst_mma(const DstMmaArgs a, const __grid_constant__ CUtensorMap tmB) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) unsigned long long bars[3 * STAGES + 1];  // full_a, full_b, empty, done
    __shared__ unsigned tmem_base_s;
    __shared__ volatile int abort_s;
    unsigned char* smem = reinterpret_cast<unsigned char*>(((size_t)smem_raw + 1023) & ~(size_t)1023);
    const unsigned sbase = smem_u32(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x;
    const int par = blockIdx.y & 1;           // 0: odd outputs, 1: even outputs
    const int n0 = (blockIdx.y >> 1) * NT;    // first output index q of this tile
    const int N = a.N, H = N / 2, Kp = a.Kp, nkb = Kp / BK;
    auto full_a = [&](int s) { return smem_u32(&bars[s]); };
    auto full_b = [&](int s) { return smem_u32(&bars[STAGES + s]); };
    auto empty = [&](int s) { return smem_u32(&bars[2 * STAGES + s]); };
    const unsigned done_bar = smem_u32(&bars[3 * STAGES]);

    __shared__ long long rowoff[BM];  // element offset of each tile row in x / y (-1: past the last row)
    if (threadIdx.x == 0) {
        abort_s = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full_a(s), 32 * LOADERS);
            mbar_init(full_b(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(done_bar, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < BM) {
        const int row = mt * BM + threadIdx.x;
        rowoff[threadIdx.x] =
            row < a.rows ? (long long)(1 + row / a.nj) * a.ls + (long long)(a.jlo + row % a.nj) * a.pitch : -1;
    }
    if (warp == 0) {
        // Tensor memory: NT (>= 32, a power of two) FP32 columns x 128 lanes.
        const unsigned dst = smem_u32(&tmem_base_s);
        const unsigned ncols = NT < 32 ? 32 : NT;
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst), "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_base_s;
    bool ok = true;

    if (warp < LOADERS) {
        // ---- loaders: fold, split, swizzled stores of the three A terms ----
        // Warp w owns tile rows 16w .. 16w + 15, RB at a time with every load
        // of the batch in flight together; lane l owns K-block columns l and
        // l + 32 (coalesced reads of x_m and of the mirrored x_{N-m}).
        constexpr int ROWS = BM / LOADERS;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % STAGES;
            if (kb >= STAGES) ok = mbar_wait(empty(s), ((kb / STAGES) - 1) & 1, &abort_s);
            if (!ok) break;
            unsigned char* at = smem + s * stage_bytes(NT);
            for (int rb = 0; rb < ROWS; rb += RB) {
                float xa[RB][2], xb[RB][2];
#pragma unroll
                for (int u = 0; u < RB; ++u) {
                    const long long o = rowoff[warp * ROWS + rb + u];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int m = kb * BK + lane + 32 * e + 1;  // 1-based input index
                        xa[u][e] = (o >= 0 && m <= H) ? __ldg(a.x + o + m - 1) : 0.f;
                        xb[u][e] = (o >= 0 && m < H) ? __ldg(a.x + o + N - m - 1) : 0.f;
                    }
                }
#pragma unroll
                for (int u = 0; u < RB; ++u) {
                    const int r = warp * ROWS + rb + u;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        // u_m = x_m + x_{N-m} (u_{N/2} = x_{N/2}); v_m = x_m - x_{N-m} (v_{N/2} = 0)
                        const int m = kb * BK + lane + 32 * e + 1;
                        const float v = par == 0 ? xa[u][e] + xb[u][e] : (m < H ? xa[u][e] - xb[u][e] : 0.f);
                        __nv_bfloat16 t1, t2, t3;
                        split3(v, t1, t2, t3);
                        const int c = lane + 32 * e;
                        const unsigned off = (unsigned)(r * 128 + ((((c >> 3) ^ (r & 7)) & 7) << 4) + (c & 7) * 2);
                        *reinterpret_cast<__nv_bfloat16*>(at + 0 * a_tile_bytes() + off) = t1;
                        *reinterpret_cast<__nv_bfloat16*>(at + 1 * a_tile_bytes() + off) = t2;
                        *reinterpret_cast<__nv_bfloat16*>(at + 2 * a_tile_bytes() + off) = t3;
                    }
                }
            }
            fence_async_smem();
            mbar_arrive(full_a(s));
        }
        if (!ok) abort_s = 1;
    } else if (warp == LOADERS) {
        // ---- TMA producer of the B terms ----------------------------------
        if (lane == 0) {
            const int yb = par * 3 * H + n0;
            int issued = 0;
            for (int kb = 0; kb < nkb && ok; ++kb) {
                const int s = kb % STAGES;
                if (kb >= STAGES) ok = mbar_wait(empty(s), ((kb / STAGES) - 1) & 1, &abort_s);
                if (!ok) break;
                const unsigned bt = sbase + s * stage_bytes(NT) + 3 * a_tile_bytes();
                mbar_expect_tx(full_b(s), 3 * b_tile_bytes(NT));
#pragma unroll
                for (int q = 0; q < 3; ++q) tma_load_2d(bt + q * b_tile_bytes(NT), &tmB, kb * BK, yb + q * H, full_b(s));
                issued = kb + 1;
            }
            if (!ok) abort_s = 1;
            // The copies this thread issued have all landed before the CTA's
            // shared memory is reused or released (immediate when the products
            // consumed them; bounded otherwise).
            for (int kb = issued - STAGES < 0 ? 0 : issued - STAGES; kb < issued; ++kb)
                mbar_wait(full_b(kb % STAGES), (kb / STAGES) & 1, nullptr);
        }
    } else {
        // ---- MMA issuer ------------------------------------------------------
        if (lane == 0) {
            const unsigned idesc = instr_desc(NT);
            for (int kb = 0; kb < nkb && ok; ++kb) {
                const int s = kb % STAGES;
                ok = mbar_wait(full_a(s), (kb / STAGES) & 1, &abort_s) &&
                     mbar_wait(full_b(s), (kb / STAGES) & 1, &abort_s);
                if (!ok) break;
                tc_fence_after();
                const unsigned as = sbase + s * stage_bytes(NT);
                const unsigned bs = as + 3 * a_tile_bytes();
#pragma unroll
                for (int kk = 0; kk < BK / 16; ++kk) {
                    // the six products a_i c_j, i + j <= 4 (terms 1-based)
                    const unsigned long long a1 = smem_desc(as + 0 * a_tile_bytes() + kk * 32);
                    const unsigned long long a2 = smem_desc(as + 1 * a_tile_bytes() + kk * 32);
                    const unsigned long long a3 = smem_desc(as + 2 * a_tile_bytes() + kk * 32);
                    const unsigned long long b1 = smem_desc(bs + 0 * b_tile_bytes(NT) + kk * 32);
                    const unsigned long long b2 = smem_desc(bs + 1 * b_tile_bytes(NT) + kk * 32);
                    const unsigned long long b3 = smem_desc(bs + 2 * b_tile_bytes(NT) + kk * 32);
                    const unsigned first = (kb == 0 && kk == 0) ? 0u : 1u;
                    mma_bf16(tmem, a3, b1, idesc, first);  // smallest terms first
                    mma_bf16(tmem, a2, b2, idesc, 1u);
                    mma_bf16(tmem, a1, b3, idesc, 1u);
                    mma_bf16(tmem, a2, b1, idesc, 1u);
                    mma_bf16(tmem, a1, b2, idesc, 1u);
                    mma_bf16(tmem, a1, b1, idesc, 1u);
                }
                mma_commit(empty(s));  // the stage's shared memory is free once these products finish
            }
            mma_commit(done_bar);  // every product issued so far
            if (!ok) abort_s = 1;
        }
    }

    // ---- epilogue: accumulator -> shared memory -> output rows -------------
    bool done_ok = true;
    if (warp < LOADERS) {
        done_ok = mbar_wait(done_bar, 0, nullptr);
        tc_fence_after();
    }
    __syncthreads();  // every role has finished issuing; shared memory is reusable
    const bool good = done_ok && !abort_s;
    if (warp < LOADERS && good) {
        // Warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (its lane
        // quarter), columns [0, NT/2) for w < 4 and [NT/2, NT) above.
        float* stage = reinterpret_cast<float*>(smem);  // [128][NT + 1]
        const int r = (warp & 3) * 32 + lane;
        constexpr int HALF = NT / 2 < 32 ? 32 : NT / 2;
        const int c_begin = (warp < 4 || NT < 64) ? 0 : HALF;
        const int c_end = NT < 64 ? (warp < 4 ? NT : 0) : c_begin + HALF;
#pragma unroll 1
        for (int c = c_begin; c < c_end; c += 32) {
            float v[32];
            tmem_ld32(tmem + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)c, v);
#pragma unroll
            for (int q = 0; q < 32; ++q) stage[r * (NT + 1) + c + q] = v[q];
        }
        tc_fence_before();
        asm volatile("bar.sync 1, %0;\n" ::"r"(32 * LOADERS) : "memory");
        // Output wavenumber k = 2q + 1 (odd) or 2q (even, q >= 1), stored at k - 1.
        for (int rr = warp; rr < BM; rr += LOADERS) {
            const long long o = rowoff[rr];
            if (o < 0) break;
            float* y = a.y + o;
            for (int c = lane; c < NT; c += 32) {
                const int q = n0 + c;
                const int k = par == 0 ? 2 * q + 1 : 2 * q;
                if (k >= 1 && k <= N - 1) y[k - 1] = stage[rr * (NT + 1) + c];
            }
        }
    }
    if (!good && threadIdx.x == 0) atomicOr(a.status, (int)ST_MMA_TIMEOUT);
    if (warp == LOADERS + 1 && lane == 0) {
        // the products this thread issued have finished before the tensor
        // memory is freed (immediate unless a wait ran out)
        mbar_wait(done_bar, 0, nullptr);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        const unsigned ncols = NT < 32 ? 32 : NT;
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// ---------------------------------------------------------------------------
// Host side.

namespace {

// Round-to-nearest-even FP32 -> BF16 bits (host).
unsigned short bf16_bits(float f) {
    unsigned u;
    std::memcpy(&u, &f, 4);
    const unsigned lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    return (unsigned short)(u >> 16);
}
float bf16_value(unsigned short b) {
    const unsigned u = (unsigned)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

int dst_mma_tile_n(int N) {
    const int H = N / 2;
    return H >= 128 ? 128 : H;
}

bool dst_mma_supported(int N) { return N >= 64 && (N & (N - 1)) == 0; }

size_t dst_mma_table_bytes(int N) {
    const int H = N / 2, Kp = H < BK ? BK : H;
    return (size_t)6 * H * Kp * sizeof(unsigned short);
}

// The split DST matrices: [parity][term][q][m], q output index (row), m
// input index (column, K-major), BF16.  Parity 0: C(m+1, 2q+1); parity 1:
// C(m+1, 2q) (row q = 0 zero); columns m+1 > N/2 are zero padding.
void dst_mma_table(int N, std::vector<unsigned short>& out) {
    const int H = N / 2, Kp = H < BK ? BK : H;
    out.assign((size_t)6 * H * Kp, 0);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int par = 0; par < 2; ++par)
        for (int q = 0; q < H; ++q) {
            const int k = par == 0 ? 2 * q + 1 : 2 * q;
            for (int m = 1; m <= H; ++m) {
                const long double c = 2.0L * sinl(pi * (long double)m * (long double)k / (long double)N);
                const float f = (float)c;
                const unsigned short t1 = bf16_bits(f);
                const float r1 = (float)(c - (long double)bf16_value(t1));
                const unsigned short t2 = bf16_bits(r1);
                const float r2 = (float)(c - (long double)bf16_value(t1) - (long double)bf16_value(t2));
                const unsigned short t3 = bf16_bits(r2);
                const unsigned short t[3] = {t1, t2, t3};
                for (int term = 0; term < 3; ++term)
                    out[((size_t)(par * 3 + term) * H + q) * Kp + (m - 1)] = t[term];
            }
        }
}

int dst_mma_tensor_map(CUtensorMap* map, void* table, int N) {
    static EncodeTiledFn encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return -1;
        encode = reinterpret_cast<EncodeTiledFn>(fn);
    }
    const int H = N / 2, Kp = H < BK ? BK : H, NT = dst_mma_tile_n(N);
    const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)6 * H};
    const cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)NT};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, table, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

template <int NT>
static cudaError_t launch_nt(const DstMmaArgs& a, const CUtensorMap& map, cudaStream_t st) {
    const int H = a.N / 2;
    const size_t smem = smem_bytes(NT);
    // per device and cheap: set on every launch, as the row-DST launches do
    cudaError_t e = cudaFuncSetAttribute(k_dst_mma<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((a.rows + BM - 1) / BM), (unsigned)(2 * (H / NT)));
    k_dst_mma<NT><<<grid, NTHREADS, smem, st>>>(a, map);
    return cudaGetLastError();
}

cudaError_t launch_dst_mma(const DstMmaArgs& a, const CUtensorMap& map, cudaStream_t st) {
    if (a.rows <= 0) return cudaSuccess;
    switch (dst_mma_tile_n(a.N)) {
        case 128: return launch_nt<128>(a, map, st);
        case 64: return launch_nt<64>(a, map, st);
        case 32: return launch_nt<32>(a, map, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pq
