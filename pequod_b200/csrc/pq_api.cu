// pq_api.cu -- the C ABI: contexts, device state, tables and the time loop.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pequod_b200.h"
#include "pq_common.cuh"
#include "pq_kernels.h"
#include "pq_ctx.h"
#include "pq_dst_mma.h"

using namespace pq;

namespace pq {

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

}  // namespace pq

namespace pq {

int fail(pq_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(pq_ctx* c, cudaError_t e, const char* where) {
    return fail(c, PQ_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Pivots of the tridiagonal j-solves, exactly as allocate_h1d_c computes
// ge_fact (qg3p_helmholtz.F90:794-809), compressed: for each (mode, k) the
// reciprocal pivots g_p, p = 1..jj-2, are stored until the pivot recurrence
// reaches a bitwise fixed point; the fixed point is stored once.
struct PivotTables {
    std::vector<int> off, len;
    std::vector<double> piv, fix;
};

PivotTables build_pivots(int ii, int jj, int L, const double* ss) {
    PivotTables t;
    const int n = ii - 2, Mr = jj - 2;
    t.off.resize((size_t)L * n);
    t.len.resize((size_t)L * n);
    t.fix.resize((size_t)L * n);
    const double norm_fact = 3.14159265358979323846 / (2.0 * (double)(ii - 1));
    std::vector<double> raw(Mr + 1);
    for (int m = 0; m < L; ++m)
        for (int k = 1; k <= n; ++k) {
            const double s = std::sin((double)k * norm_fact);
            const double diag = -2.0 - ss[m] - 4.0 * (s * s);
            raw[1] = diag;
            int conv = 0;  // first p with raw[p] == raw[p-1]
            for (int p = 2; p <= Mr; ++p) {
                raw[p] = diag - 1.0 / raw[p - 1];
                if (raw[p] == raw[p - 1]) {
                    conv = p;
                    break;
                }
            }
            const size_t mk = (size_t)m * n + (k - 1);
            t.off[mk] = (int)t.piv.size();
            if (conv) {
                for (int p = 1; p <= conv - 2; ++p) t.piv.push_back(1.0 / raw[p]);
                t.len[mk] = conv - 2;
                t.fix[mk] = 1.0 / raw[conv - 1];
            } else {
                for (int p = 1; p <= Mr; ++p) t.piv.push_back(1.0 / raw[p]);
                t.len[mk] = Mr;
                t.fix[mk] = 1.0 / raw[Mr];
            }
        }
    if (t.piv.empty()) t.piv.push_back(0.0);
    return t;
}

// Copy between a dense (ii, jj, L) host/device array and a pitched field.
int copy_in(pq_ctx* c, void* dst, const double* src, int kind) {
    const size_t w = (size_t)c->ii * sizeof(double);
    CK(cudaMemcpy2DAsync(dst, (size_t)c->pitch * sizeof(double), src, w, w, (size_t)c->jj * c->L,
                         kind == PQ_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
    return PQ_OK;
}

int copy_out(pq_ctx* c, double* dst, const void* src, int kind) {
    const size_t w = (size_t)c->ii * sizeof(double);
    CK(cudaMemcpy2DAsync(dst, w, src, (size_t)c->pitch * sizeof(double), w, (size_t)c->jj * c->L,
                         kind == PQ_PTR_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
    return PQ_OK;
}

// State fields (the CABARET fields, zeta and rel) are FP32 in the mixed
// form: copies go through the FP64 helm_io field and a conversion kernel.
int copy_in_state(pq_ctx* c, void* dst, const double* src, int kind) {
    if (!c->mixed) return copy_in(c, dst, src, kind);
    int rc = copy_in(c, c->hm[0].helm_io, src, kind);
    if (rc) return rc;
    CK(launch_convert(dst, c->hm[0].helm_io, (size_t)c->pitch * c->jj * c->L, 1, c->stream));
    return PQ_OK;
}

int copy_out_state(pq_ctx* c, double* dst, const void* src, int kind) {
    if (!c->mixed) return copy_out(c, dst, src, kind);
    CK(launch_convert(c->hm[0].helm_io, src, (size_t)c->pitch * c->jj * c->L, 0, c->stream));
    return copy_out(c, dst, c->hm[0].helm_io, kind);
}

int join_exchange(pq_ctx* c) {
    if (c->x.last >= 0) CK(cudaStreamWaitEvent(c->stream, c->x.done[c->x.last], 0));
    c->x.last = -1;
    c->x.sequence = false;
    return PQ_OK;
}

int check_status(pq_ctx* c) {
    int rc = join_exchange(c);
    if (rc) return rc;
    int st = 0;
    CK(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (st & (ST_NAN_PSIC)) return fail(c, PQ_ERR_NAN, "NaN psiC encountered");
    if (st & (ST_NAN_ENERGY)) return fail(c, PQ_ERR_NAN, "NaN value encountered in energy");
    return PQ_OK;
}

int upload_members(pq_ctx* c) {
    CK(cudaMemcpyAsync(c->d_members, c->hm, 2 * sizeof(Member), cudaMemcpyHostToDevice, c->stream));
    return PQ_OK;
}

// The three Helmholtz kernels.
namespace {

// Arguments of the tensor-core DST over the baroclinic rows: forward (dir 0)
// from the node rows in gbuf to the spectral rows, inverse (dir 1) back.
DstMmaArgs mma_args(const pq_ctx* c, int dir) {
    const Member& m = c->hm[0];
    DstMmaArgs a;
    a.x = static_cast<const float*>(dir == 0 ? m.gbuf : m.spec);
    a.y = static_cast<float*>(dir == 0 ? m.spec : m.gbuf);
    a.ls = m.lstride;
    a.pitch = m.pitch;
    a.N = m.N;
    a.Kp = std::max(64, m.N / 2);
    a.nj = c->periodic ? c->jj : c->jj - 2;
    a.jlo = c->periodic ? 0 : 1;
    a.rows = (c->L - 1) * a.nj;
    a.status = c->d_status;
    return a;
}

}  // namespace

int set_dst_algo(pq_ctx* c, int algo) {
    if (algo != PQ_DST_BUTTERFLY && algo != PQ_DST_TENSOR) return fail(c, PQ_ERR_ARG, "dst_algo is 1 or 2");
    if (algo == PQ_DST_TENSOR) {
        if (!c->mixed || c->leapfrog)
            return fail(c, PQ_ERR_UNSUPPORTED, "the tensor-core DST serves the mixed-precision form");
        if (!dst_mma_supported(c->hm[0].N)) return fail(c, PQ_ERR_UNSUPPORTED, "the tensor-core DST needs ii >= 65");
        if (!c->mma_mem) {
            const size_t gbytes = align256((size_t)c->L * c->hm[0].lstride * sizeof(float));
            const size_t tbytes = dst_mma_table_bytes(c->hm[0].N);
            void* mem = nullptr;
            if (cudaMalloc(&mem, gbytes + tbytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(c, PQ_ERR_NOMEM, "allocation of the tensor-core DST buffers failed");
            }
            c->mma_mem = mem;
            c->mma_bytes = gbytes + tbytes;
            std::vector<unsigned short> table;
            dst_mma_table(c->hm[0].N, table);
            void* tab = static_cast<char*>(mem) + gbytes;
            CK(cudaMemsetAsync(mem, 0, gbytes, c->stream));
            CK(cudaMemcpyAsync(tab, table.data(), tbytes, cudaMemcpyHostToDevice, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            if (dst_mma_tensor_map(&c->mma_map, tab, c->hm[0].N) != 0)
                return fail(c, PQ_ERR_CUDA, "cuTensorMapEncodeTiled failed for the DST table");
            for (int p = 0; p < 2; ++p) c->hm[p].gbuf = mem;
            int rc = upload_members(c);
            if (rc) return rc;
        }
    }
    if (algo != c->dst_algo) {
        c->dst_algo = algo;
        // captured step graphs hold the old kernel sequence
        for (auto& g : c->graph1)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
        if (c->graph2) {
            cudaGraphExecDestroy(c->graph2);
            c->graph2 = nullptr;
        }
    }
    return PQ_OK;
}

int run_inversion(pq_ctx* c, int par, int prologue, cudaEvent_t* ev) {
    const int f32 = c->mixed ? 1 : 0;
    const bool tc = f32 && c->dst_algo == PQ_DST_TENSOR && c->mma_mem;
    LaunchSet ls = c->ls[par];
    ls.gemm_bc = tc ? 1 : 0;
    CK(launch_dst_forward(ls, prologue, f32, c->stream));
    if (tc) CK(launch_dst_mma(mma_args(c, 0), c->mma_map, c->stream));
    if (ev) CK(cudaEventRecord(ev[1], c->stream));
    CK(launch_tridiag(ls, 1, f32, c->stream));
    if (ev) CK(cudaEventRecord(ev[2], c->stream));
    if (tc) CK(launch_dst_mma(mma_args(c, 1), c->mma_map, c->stream));
    CK(launch_dst_inverse(ls, EPI_PV, f32, c->stream));
    if (ev) CK(cudaEventRecord(ev[3], c->stream));
    return PQ_OK;
}

int run_helm(pq_ctx* c, int par, int prologue, int epilogue, int mean) {
    if (epilogue == EPI_PV && mean && c->mixed) return run_inversion(c, par, prologue, nullptr);
    // The stand-alone helm entry (PRO_PLAIN / EPI_HELM) is always FP64, and
    // runs the row DSTs with the batched solver's geometry, so that a batch
    // member and the same problem through pq_helm agree bit for bit.
    const int f32 = (c->mixed && epilogue == EPI_PV) ? 1 : 0;
    LaunchSet ls = c->ls[par];
    if (prologue == PRO_PLAIN) {
        ls.dst_group = 0;
        for (int dir = 0; dir < 2; ++dir) {
            ls.dst_lanes[dir] = dst_lanes_batched(c->hm[par].M);
            const int R = dst_rows_per_cta_host(ls.dst_lanes[dir], 0);
            const int rows = dir == 1 ? c->jj : (c->periodic ? c->jj : c->jj - 2);
            ls.ctas_dst[dir] = (rows + R - 1) / R;
        }
    }
    CK(launch_dst_forward(ls, prologue, f32, c->stream));
    CK(launch_tridiag(ls, mean, f32, c->stream));
    CK(launch_dst_inverse(ls, epilogue, f32, c->stream));
    return PQ_OK;
}

int run_step(pq_ctx* c, int par) {
    cudaEvent_t* ev = nullptr;
    if (c->timing) {
        c->events.emplace_back();
        ev = c->events.back().e;
        for (int k = 0; k < 5; ++k) CK(cudaEventCreate(&ev[k]));
        CK(cudaEventRecord(ev[0], c->stream));
    }
    if (c->leapfrog) {
        // One DOLEAPFROG sub-step on level par (qg3.F90:615-651): centred
        // step + RAW filter, inversion, rel and boundary zeta, model_time.
        CK(launch_lf_step(c->ls[par], c->desc.ra_nu, c->desc.ra_alpha, c->stream));
        CK(launch_dst_forward(c->ls[par], PRO_MODAL, 0, c->stream));
        if (ev) CK(cudaEventRecord(ev[1], c->stream));
        CK(launch_tridiag(c->ls[par], 1, 0, c->stream));
        if (ev) CK(cudaEventRecord(ev[2], c->stream));
        CK(launch_dst_inverse(c->ls[par], EPI_PV, 0, c->stream));
        if (ev) CK(cudaEventRecord(ev[3], c->stream));
        CK(launch_lf_rel_bc(c->ls[par], 0, 1, c->stream));
        if (ev) CK(cudaEventRecord(ev[4], c->stream));
        if (c->quad) CK(launch_quad(c->ls[par], 0, 1, c->stream));
        if (c->psi_av) CK(launch_lf_average(c->ls[par], c->stream));
        c->zpar = par;
        return PQ_OK;
    }
    const int f32 = c->mixed ? 1 : 0;
    if (c->periodic) {
        // Channel: predictor + beta in the forward DST, the momentum-corrected
        // inversion, then the four channel CABARET kernels.
        int rc = run_inversion(c, par, PRO_STEP, ev);
        if (rc) return rc;
        if (c->quad) CK(launch_quad(c->ls[par], f32, 0, c->stream));
        CK(launch_cabaret_channel(c->ls[par], f32, c->stream));
        if (ev) CK(cudaEventRecord(ev[4], c->stream));
        c->pred_ready = false;
        c->zpar = par;
        return PQ_OK;
    }
    // The predictor + beta update runs in the forward DST unless the previous
    // fused step already produced this step's inversion input.
    int rc = run_inversion(c, par, (c->fuse && c->pred_ready) ? PRO_MODAL : PRO_STEP, ev);
    if (rc) return rc;
    if (c->quad) CK(launch_quad(c->ls[par], f32, 0, c->stream));
    CK(launch_cabaret_fused(c->ls[par], c->fuse ? 1 : 0, f32, c->stream));
    if (ev) CK(cudaEventRecord(ev[4], c->stream));
    c->pred_ready = c->fuse;
    c->zpar = par;
    return PQ_OK;
}

}  // namespace pq

extern "C" {

const char* pq_last_error(const pq_ctx* c) { return c ? c->err.c_str() : "null context"; }

size_t pq_device_bytes(const pq_ctx* c) { return c ? c->arena_bytes + c->mma_bytes : 0; }

void* pq_stream(pq_ctx* c) { return c ? (void*)c->stream : nullptr; }

long pq_last_launch_count(const pq_ctx* c) { return c ? c->last_launches : 0; }

void pq_destroy(pq_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph2) cudaGraphExecDestroy(c->graph2);
    for (auto& g : c->graph1)
        if (g) cudaGraphExecDestroy(g);
    if (c->arena) cudaFree(c->arena);
    if (c->mma_mem) cudaFree(c->mma_mem);
    if (c->psi_av) cudaFree(c->psi_av);
    if (c->quad) cudaFree(c->quad);
    if (c->x.in) {
        cudaStreamSynchronize(c->x.in);
        cudaStreamSynchronize(c->x.out);
        for (int s = 0; s < 2; ++s) {
            cudaFree(c->x.stage_in[s]);
            cudaFree(c->x.stage_out[s]);
            cudaEventDestroy(c->x.ready[s]);
            cudaEventDestroy(c->x.consumed[s]);
            cudaEventDestroy(c->x.produced[s]);
            cudaEventDestroy(c->x.done[s]);
        }
        cudaEventDestroy(c->x.entry);
        cudaStreamDestroy(c->x.in);
        cudaStreamDestroy(c->x.out);
    }
    if (c->d_members) cudaFree(c->d_members);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

int pq_create(pq_ctx** out, const pq_model_desc* d, int device) {
    return create_ctx(out, d, device, false, nullptr);
}

}  // extern "C"

int pq::create_ctx(pq_ctx** out, const pq_model_desc* d, int device, bool helm_only, cudaStream_t stream) {
    if (!out || !d) return PQ_ERR_ARG;
    *out = nullptr;
    const int ii = d->ii, jj = d->jj, L = d->layers;
    if (ii < 5 || jj < 5 || !is_pow2(ii - 1) || L < 1 || L > PQ_MAX_LAYERS) return PQ_ERR_ARG;
    if (d->precision != PQ_PREC_FP64 && d->precision != PQ_PREC_MIXED) return PQ_ERR_UNSUPPORTED;
    if (d->scheme != PQ_SCHEME_CABARET && d->scheme != PQ_SCHEME_LEAPFROG) return PQ_ERR_UNSUPPORTED;
    // The leapfrog scheme runs in FP64 with a fixed dt (the reference's
    // adaptive step is a CABARET routine).
    if (d->scheme == PQ_SCHEME_LEAPFROG && (d->precision != PQ_PREC_FP64 || d->adapt_dt)) return PQ_ERR_UNSUPPORTED;
    pq_ctx* c = new pq_ctx;
    c->device = device;
    c->desc = *d;
    c->ii = ii;
    c->jj = jj;
    c->L = L;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        int rc = cuda_fail(c, e, "cudaSetDevice");
        *out = c;
        return rc;
    }
    *out = c;
    c->helm_only = helm_only;
    if (stream) {
        c->stream = stream;
        c->own_stream = false;
    } else {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    }
    int sm_count = 0;
    CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
    if (d->force_wind) c->wind.assign(d->force_wind, d->force_wind + (size_t)ii * jj);
    c->desc.force_wind = nullptr;

    const int n = ii - 2, N = ii - 1, M = N / 2;
    int logM = 0;
    while ((1 << logM) < M) ++logM;
    c->pitch = (ii + 31) & ~31;
    const size_t lstride = (size_t)c->pitch * jj;
    c->field_bytes = lstride * L * sizeof(double);
    const int ntiles_tri = tri_ctas(n, jj, L);
    // CABARET formulation and band height by grid size (measured on B200,
    // pq_tuning overrides): tiles up to 700 rows; above, persistent warp
    // sweeps, two columns per lane in the mixed form beyond 1500 rows.  Bands
    // (swept 8..48): short ones keep the end of the sweep queue short, tall
    // ones cut halo rows -- 1025 x 1025 x 3: 24 (FP64), 16 (mixed);
    // 2049 x 2049 x 5: 40 (FP64), 24 (mixed, two columns).
    const bool mixed = d->precision == PQ_PREC_MIXED;
    const int cab_kernel = jj <= 700 ? 0 : (mixed && jj > 1500) ? 2 : 1;
    const int cab_sh = jj <= 300 ? 8 : jj <= 700 ? 32 : jj <= 1500 ? (mixed ? 16 : 24) : (mixed ? 24 : 40);
    const int ntiles_cab = d->periodic_j ? channel_ctas(ii, jj)
                           : cab_kernel == 0 ? cabaret_tile_ctas(ii, jj, L)
                                             : cabaret_ctas(ii, jj, L, cab_sh, cab_kernel, mixed);
    const int ntiles_cab_max =
        std::max({cabaret_ctas_bound(ii, jj, L, kMinBand), cabaret_tile_ctas(ii, jj, L), channel_ctas(ii, jj)});

    // Tables.
    std::vector<double2> tw(M), wsplit(M);
    for (int t = 0; t < M; ++t) {
        const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)M;
        tw[t] = make_double2((double)cosl(a), (double)-sinl(a));
        const long double b = 2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)N;
        wsplit[t] = make_double2((double)cosl(b), (double)-sinl(b));
    }
    std::vector<double> was(N / 2 + 1, 0.0), wmean(n, 0.0);
    for (int k = 1; k <= N / 2; ++k)
        was[k] = (double)(2.0L * sinl(3.141592653589793238462643383279502884L * (long double)k / (long double)N));
    for (int k = 1; k <= n; ++k)
        if (k & 1)
            wmean[k - 1] = (double)(2.0L / tanl(3.141592653589793238462643383279502884L * (long double)k /
                                                (2.0L * (long double)N)));
    PivotTables pv = build_pivots(ii, jj, L, d->ss);

    // Arena layout.
    const int nfields = helm_only ? 2 /*helm_io, spec*/ + (d->precision == PQ_PREC_MIXED ? 1 /*spec64*/ : 0)
                                  : 2 /*zeta_old*/ + 2 /*zeta*/ + 1 /*psi*/ + 2 /*res*/ + 2 /*res_beta*/ +
                                        1 /*ui*/ + 1 /*uj*/ + 2 /*uimo*/ + 2 /*ujmo*/ + 2 /*zfi*/ + 2 /*zfj*/ +
                                        1 /*rel*/ + 1 /*helm_io*/ + 1 /*spec*/ + 1 /*corr*/ + 1 /*spec64*/ +
                                        2 /*leapfrog psi(2), rel(2)*/ + (d->periodic_j ? 1 /*corr2*/ : 0);
    const size_t fb = align256(c->field_bytes);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align256(bytes);
        return o;
    };
    const size_t o_fields = take(fb * nfields);
    const size_t o_wind = take(lstride * sizeof(double));
    const size_t o_tw = take(M * sizeof(double2));
    const size_t o_ws = take(M * sizeof(double2));
    const size_t o_was = take(was.size() * sizeof(double));
    std::vector<float2> tw_f(M), wsplit_f(M);
    std::vector<float> was_f(was.size());
    for (int t = 0; t < M; ++t) {
        tw_f[t] = make_float2((float)tw[t].x, (float)tw[t].y);
        wsplit_f[t] = make_float2((float)wsplit[t].x, (float)wsplit[t].y);
    }
    for (size_t k = 0; k < was.size(); ++k) was_f[k] = (float)was[k];
    const size_t o_twf = take(M * sizeof(float2));
    const size_t o_wsf = take(M * sizeof(float2));
    const size_t o_wasf = take(was_f.size() * sizeof(float));
    const size_t o_wm = take(wmean.size() * sizeof(double));
    const size_t o_poff = take(pv.off.size() * sizeof(int));
    const size_t o_plen = take(pv.len.size() * sizeof(int));
    const size_t o_piv = take(pv.piv.size() * sizeof(double));
    const size_t o_pfix = take(pv.fix.size() * sizeof(double));
    // periodic_coefficients (qg3p_helmholtz.F90:473-559) of a channel: for
    // each (mode, k) the vectors b, c over j = 1..jj, computed exactly as the
    // reference does from the pivots e of poinit_j (:429-469).
    std::vector<double> pbv, pcv;
    if (d->periodic_j) {
        pbv.assign((size_t)L * jj * n, 0.0);
        pcv.assign((size_t)L * jj * n, 0.0);
        const double cff = 3.14159265358979323846 / (2.0 * (double)(ii - 1));
        std::vector<double> e(jj + 1), b(jj + 1), cc(jj + 1);
        for (int mm = 0; mm < L; ++mm)
            for (int k = 1; k <= n; ++k) {
                const double sn = std::sin((double)k * cff);
                const double v = -2.0 - d->ss[mm] - 4.0 * (sn * sn);
                for (int j = 1; j <= jj; ++j) e[j] = v;
                for (int j = 3; j <= jj - 1; ++j) e[j] = e[j] - 1.0 / e[j - 1];
                for (int j = 2; j <= jj - 1; ++j) e[j] = 1.0 / e[j];
                b[1] = v;
                b[2] = 1.0;
                for (int j = 3; j <= jj - 1; ++j) b[j] = 0.0;
                b[jj] = 1.0;
                cc[1] = 1.0;
                for (int j = 2; j <= jj - 2; ++j) cc[j] = 0.0;
                cc[jj - 1] = 1.0;
                cc[jj] = v;
                for (int j = 3; j <= jj - 1; ++j) {
                    b[j] = b[j] - b[j - 1] * e[j - 1];
                    cc[j] = cc[j] - cc[j - 1] * e[j - 1];
                }
                b[jj - 1] = b[jj - 1] * e[jj - 1];
                cc[jj - 1] = cc[jj - 1] * e[jj - 1];
                for (int j = jj - 2; j >= 2; --j) {
                    b[j] = (b[j] - b[j + 1]) * e[j];
                    cc[j] = (cc[j] - cc[j + 1]) * e[j];
                }
                b[1] = b[1] - b[2];
                cc[1] = cc[1] - cc[2];
                b[jj] = b[jj] - b[jj - 1];
                cc[jj] = cc[jj] - cc[jj - 1];
                cc[1] = cc[1] / b[1];
                for (int j = 2; j <= jj; ++j) cc[j] = cc[j] - cc[1] * b[j];
                for (int j = 1; j <= jj; ++j) {
                    pbv[((size_t)mm * jj + (j - 1)) * n + (k - 1)] = b[j];
                    pcv[((size_t)mm * jj + (j - 1)) * n + (k - 1)] = cc[j];
                }
            }
    }
    const size_t o_pb = take(pbv.size() * sizeof(double));
    const size_t o_pc = take(pcv.size() * sizeof(double));
    // Channel wall weights (zeta_boundary of a solved mode in spectral space,
    // qg3p_aux.F90:289-379): sum_j phi(i, j) = 2 sum_k sin(i k pi / N) C_k
    // for node i, and phi is 0 on the walls, so the mean PV of wall i = 0 is
    // sum_k wwall[k] C_k (the other wall takes (-1)^(k+1) wwall[k]).
    std::vector<double> wwall(n, 0.0);
    if (d->periodic_j) {
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int k = 1; k <= n; ++k) {
            const long double s1 = sinl(pi * k / N), s2 = sinl(2.0L * pi * k / N);
            long double w = 0.0L;
            if (d->bc_type == PQ_BC_PARTIAL_SLIP)
                w = ((long double)d->alpha / ((long double)d->alpha + 3.0L)) * 2.0L * (4.0L * s1 - 0.5L * s2);
            else if (d->bc_type == PQ_BC_NO_SLIP)
                w = 2.0L * 2.0L * s1;
            wwall[k - 1] = (double)(w / (long double)jj);
        }
    }
    const size_t o_ww = take(wwall.size() * sizeof(double));
    const size_t o_ica = take((size_t)4 * PQ_MAXL * sizeof(double));
    const size_t npart = std::max((size_t)2 * ntiles_tri, (size_t)jj * (PQ_MAXL + 1));
    const size_t o_part = take(npart * sizeof(double));
    const size_t o_maxu = take(ntiles_cab_max * sizeof(double));
    const size_t o_cnt = take(4 * sizeof(unsigned));
    const size_t o_sc = take(sizeof(Scalars));
    const size_t o_st = take(sizeof(int));
    c->arena_bytes = off;
    e = cudaMalloc(&c->arena, off);
    if (e != cudaSuccess) return fail(c, PQ_ERR_NOMEM, "device allocation failed");
    CK(cudaMemsetAsync(c->arena, 0, off, c->stream));
    char* A = c->arena;
    CK(cudaMemcpyAsync(A + o_tw, tw.data(), M * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_ws, wsplit.data(), M * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_was, was.data(), was.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_twf, tw_f.data(), M * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_wsf, wsplit_f.data(), M * sizeof(float2), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_wasf, was_f.data(), was_f.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_wm, wmean.data(), wmean.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_ww, wwall.data(), wwall.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_poff, pv.off.data(), pv.off.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_plen, pv.len.data(), pv.len.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_piv, pv.piv.data(), pv.piv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(A + o_pfix, pv.fix.data(), pv.fix.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (!pbv.empty()) {
        CK(cudaMemcpyAsync(A + o_pb, pbv.data(), pbv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(A + o_pc, pcv.data(), pcv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    if (!c->wind.empty())
        CK(cudaMemcpy2DAsync(A + o_wind, (size_t)c->pitch * sizeof(double), c->wind.data(), (size_t)ii * sizeof(double),
                             (size_t)ii * sizeof(double), jj, cudaMemcpyHostToDevice, c->stream));

    Member m;
    std::memset(&m, 0, sizeof(m));
    m.ii = ii;
    m.jj = jj;
    m.L = L;
    m.pitch = c->pitch;
    m.n = n;
    m.N = N;
    m.M = M;
    m.logM = logM;
    m.lstride = (long long)lstride;
    m.bc_type = d->bc_type;
    m.limiter = d->limiter;
    m.alpha = d->alpha;
    m.viscosity = d->viscosity;
    m.visc_bot = d->visc_bot;
    for (int a = 0; a < L; ++a) {
        for (int b = 0; b < L; ++b) {
            m.z2m[a * PQ_MAXL + b] = d->z2m[a + L * b];  // z2m(m=a, l=b)
            m.m2z[a * PQ_MAXL + b] = d->m2z[a + L * b];  // m2z(l=a, m=b)
        }
        m.ss[a] = d->ss[a];
        m.s1[a] = d->s1[a];
        m.s2[a] = d->s2[a];
        m.beta[a] = d->beta[a];
        m.h[a] = d->h[a];
        m.htot += d->h[a];
    }
    // 1 / (g_ii_int g_jj_int); a channel has jj distinct rows.
    m.mean_scale = 1.0 / ((double)(ii - 1) * (double)(d->periodic_j ? jj : jj - 1));
    m.wwall = reinterpret_cast<const double*>(A + o_ww);
    m.inv_corr_a = reinterpret_cast<const double*>(A + o_ica);
    m.tw = reinterpret_cast<const double2*>(A + o_tw);
    m.wsplit = reinterpret_cast<const double2*>(A + o_ws);
    m.was = reinterpret_cast<const double*>(A + o_was);
    m.tw_f = reinterpret_cast<const float2*>(A + o_twf);
    m.wsplit_f = reinterpret_cast<const float2*>(A + o_wsf);
    m.was_f = reinterpret_cast<const float*>(A + o_wasf);
    m.mixed = d->precision == PQ_PREC_MIXED ? 1 : 0;
    c->mixed = m.mixed != 0;
    m.wmean = reinterpret_cast<const double*>(A + o_wm);
    m.piv_off = reinterpret_cast<const int*>(A + o_poff);
    m.piv_len = reinterpret_cast<const int*>(A + o_plen);
    m.piv = reinterpret_cast<const double*>(A + o_piv);
    m.piv_fix = reinterpret_cast<const double*>(A + o_pfix);
    m.periodic = d->periodic_j ? 1 : 0;
    m.pb = pbv.empty() ? nullptr : reinterpret_cast<const double*>(A + o_pb);
    m.pc = pcv.empty() ? nullptr : reinterpret_cast<const double*>(A + o_pc);
    c->periodic = d->periodic_j != 0;
    char* F = A + o_fields;
    int fi = 0;
    auto fld = [&]() { return (void*)(F + fb * (fi++)); };
    void *zpb0 = nullptr, *zpb1 = nullptr, *rb0 = nullptr, *rb1 = nullptr, *rel2 = nullptr, *rs1 = nullptr;
    double* psi2 = nullptr;
    if (helm_only) {
        m.helm_io = fld();
        m.spec = fld();
        if (d->precision == PQ_PREC_MIXED) m.spec64 = (double*)fld();
    } else {
        m.zeta_old[0] = fld();
        m.zeta_old[1] = fld();
        zpb0 = fld();
        m.psi = (double*)fld();
        m.res = fld();
        rb0 = fld();
        m.ui = fld();
        m.uj = fld();
        m.uimo[0] = fld();
        m.uimo[1] = fld();
        m.ujmo[0] = fld();
        m.ujmo[1] = fld();
        m.zfi[0] = fld();
        m.zfi[1] = fld();
        m.zfj[0] = fld();
        m.zfj[1] = fld();
        zpb1 = fld();
        rb1 = fld();
        rs1 = fld();
        m.rel = fld();
        m.helm_io = fld();
        m.spec = fld();
        m.corr = (const double*)fld();
        m.spec64 = (double*)fld();
        psi2 = (double*)fld();
        rel2 = fld();
        if (d->periodic_j) m.corr2 = (const double*)fld();
    }
    m.wind = c->wind.empty() ? nullptr : reinterpret_cast<const double*>(A + o_wind);
    m.partials = reinterpret_cast<double*>(A + o_part);
    m.maxu_part = reinterpret_cast<double*>(A + o_maxu);
    m.counters = reinterpret_cast<unsigned*>(A + o_cnt);
    m.sc = reinterpret_cast<Scalars*>(A + o_sc);
    m.status = reinterpret_cast<int*>(A + o_st);
    m.ntiles_tri = ntiles_tri;
    m.ntiles_cab = ntiles_cab;
    m.cab_sh = cab_sh;
    m.adapt_dt = d->adapt_dt;
    m.target_cfl = d->target_cfl;
    m.max_dt = d->max_dt;
    m.max_dt_increase = d->max_dt_increase;
    c->d_sc = m.sc;
    c->d_status = m.status;
    c->hm[0] = m;
    c->hm[1] = m;
    c->hm[0].cur = 0;
    c->hm[1].cur = 1;
    // zeta (after predictor and beta) and res_beta are ping-ponged so that
    // the fused step can write the next step's values.
    c->hm[0].zeta = c->hm[1].zeta_next = zpb0;
    c->hm[1].zeta = c->hm[0].zeta_next = zpb1;
    c->hm[0].res_beta = c->hm[1].res_beta_other = rb0;
    c->hm[1].res_beta = c->hm[0].res_beta_other = rb1;
    // The corrector writes the other parity's res: a step of parity p reads
    // res[p] (the previous step's) and writes res[p ^ 1].
    c->hm[0].res = c->hm[1].res_out = m.res;
    c->hm[1].res = c->hm[0].res_out = rs1;
    // The fused next-step predictor needs a fixed dt and the closed basin's
    // fused CABARET kernels; the channel steps through its own kernels.
    c->fuse = !d->adapt_dt && !d->periodic_j;
    c->leapfrog = d->scheme == PQ_SCHEME_LEAPFROG;
    if (c->leapfrog) {
        // Level descriptors: hm[p] advances level p with the other level q.
        c->fuse = false;
        void* zl[2] = {zpb0, zpb1};
        double* pl[2] = {m.psi, psi2};
        void* rl[2] = {m.rel, rel2};
        for (int p = 0; p < 2; ++p) {
            const int q = p ^ 1;
            Member& h = c->hm[p];
            h.zeta = zl[p];
            h.zeta_next = zl[q];
            h.zeta_old[0] = m.zeta_old[p];
            h.zeta_old[1] = m.zeta_old[q];
            h.psi = pl[p];
            h.psi_other = pl[q];
            h.rel = rl[p];
            h.rel_other = rl[q];
        }
    }

    e = cudaMalloc(&c->d_members, 2 * sizeof(Member) + 256);
    if (e != cudaSuccess) return fail(c, PQ_ERR_NOMEM, "device allocation failed");
    c->d_prefix = reinterpret_cast<int*>(reinterpret_cast<char*>(c->d_members) + 2 * sizeof(Member));
    CK(cudaMemsetAsync(c->d_prefix, 0, 256, c->stream));
    int rc = upload_members(c);
    if (rc) return rc;
    for (int p = 0; p < 2; ++p) {
        LaunchSet& s = c->ls[p];
        s.members = c->d_members + p;
        s.one = &c->hm[p];  // the same descriptor, passed by value to the step kernels
        s.nmem = 1;
        s.maxL = L;
        s.maxN = N;
        s.maxPitch = c->pitch;
        s.maxJ = jj;
        s.maxI = ii;
        s.prefix_rows_interior = s.prefix_rows_all = s.prefix_tri = s.prefix_cab = c->d_prefix;
        s.ctas_rows_interior = jj - 2;
        s.ctas_rows_all = jj;
        s.ctas_tri = ntiles_tri;
        s.ctas_cab = ntiles_cab;
        s.dst_group = 0;
        s.pdl = 0;
        s.dst_lanes[0] = dst_lanes_default(N / 2, L, 0);
        s.dst_lanes[1] = dst_lanes_default(N / 2, L, 1);
        s.cab_kernel = cab_kernel;
        s.sm_count = sm_count;
        s.prefix_dst[0] = s.prefix_dst[1] = c->d_prefix;
        s.periodic = c->periodic ? 1 : 0;
        const int R0 = dst_rows_per_cta_host(s.dst_lanes[0], 0), R1 = dst_rows_per_cta_host(s.dst_lanes[1], 0);
        s.ctas_dst[0] = ((c->periodic ? jj : jj - 2) + R0 - 1) / R0;
        s.ctas_dst[1] = (jj + R1 - 1) / R1;
    }
    // Scalars: dt and the initial time weights.
    Scalars sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.dt = sc.dt_last = d->dt;
    sc.tweight_a = sc.tweight_a_last = 0.5;
    sc.tweight_u = sc.tweight_u_last = 0.5;
    CK(cudaMemcpyAsync(c->d_sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream));

    // Correction function for mass conservation, correction_function_mass
    // (qg3p_aux.F90:196-230): solve with a unit right-hand side, Dirichlet 0,
    // then corr = (1 + ss psi) / (1 + ss mean(psi)) with the plain interior
    // mean the reference uses there.
    if (!helm_only && !c->periodic) {
        std::vector<double> ones((size_t)ii * jj * L, 1.0);
        rc = copy_in(c, m.helm_io, ones.data(), PQ_PTR_HOST);
        if (rc) return rc;
        rc = run_helm(c, 0, PRO_PLAIN, EPI_HELM, 0);
        if (rc) return rc;
        std::vector<double> h((size_t)ii * jj * L);
        rc = copy_out(c, h.data(), m.helm_io, PQ_PTR_HOST);
        if (rc) return rc;
        CK(cudaStreamSynchronize(c->stream));
        for (int l = 0; l < L; ++l) {
            double* p = h.data() + (size_t)ii * jj * l;
            for (int i = 0; i < ii; ++i) p[i] = p[i + (size_t)ii * (jj - 1)] = 0.0;
            for (int j = 0; j < jj; ++j) p[(size_t)ii * j] = p[(size_t)ii * j + ii - 1] = 0.0;
            double s = 0.0;
            for (int j = 1; j < jj - 1; ++j)
                for (int i = 1; i < ii - 1; ++i) s += p[i + (size_t)ii * j];
            const double mean = s / ((double)(ii - 1) * (double)(jj - 1));
            const double den = 1.0 + d->ss[l] * mean;
            for (size_t k = 0; k < (size_t)ii * jj; ++k) p[k] = (1.0 + d->ss[l] * p[k]) / den;
        }
        rc = copy_in(c, (void*)m.corr, h.data(), PQ_PTR_HOST);
        if (rc) return rc;
    }
    if (!helm_only && c->periodic) {
        // correction_function_momentum (qg3p_aux.F90:233-285): Helmholtz
        // solutions with zero right-hand side and psi = 1 on wall i = 0 and 0
        // on wall i = ii - 1 (corr), and the other way round (corr2), through
        // the laplace_bc lifting (qg3p_laplace_bc.F90:128-150, 227-251); then
        // per baroclinic mode the inverse of the 2 x 2 matrix of their wall PV
        // means (zeta_boundary, :289-379).
        const size_t nn = (size_t)ii * jj;
        std::vector<double> cf[2];
        double zb[2][2][PQ_MAXL];  // [function][wall][mode]
        for (int w = 0; w < 2; ++w) {
            const double bb = w == 0 ? 1.0 : 0.0, bd = w == 0 ? 0.0 : 1.0;
            std::vector<double> h(nn * L, 0.0);
            for (int l = 0; l < L; ++l)
                for (int j = 0; j < jj; ++j) {
                    h[(size_t)l * nn + (size_t)ii * j + 1] -= bb;
                    h[(size_t)l * nn + (size_t)ii * j + ii - 2] -= bd;
                }
            rc = copy_in(c, m.helm_io, h.data(), PQ_PTR_HOST);
            if (rc) return rc;
            rc = run_helm(c, 0, PRO_PLAIN, EPI_HELM, 0);
            if (rc) return rc;
            rc = copy_out(c, h.data(), m.helm_io, PQ_PTR_HOST);
            if (rc) return rc;
            CK(cudaStreamSynchronize(c->stream));
            for (int l = 0; l < L; ++l)
                for (int j = 0; j < jj; ++j) {
                    h[(size_t)l * nn + (size_t)ii * j] = bb;
                    h[(size_t)l * nn + (size_t)ii * j + ii - 1] = bd;
                }
            for (int l = 0; l < L; ++l) {
                const double* p = h.data() + (size_t)l * nn;
                double sb = 0.0, sd = 0.0;
                if (d->bc_type == PQ_BC_PARTIAL_SLIP) {
                    const double cff = d->alpha / (d->alpha + 3.0);
                    for (int j = 0; j < jj; ++j) {
                        const double* r = p + (size_t)ii * j;
                        sb = sb + cff * (-3.5 * r[0] + 4.0 * r[1] - 0.5 * r[2]);
                    }
                    for (int j = 0; j < jj; ++j) {
                        const double* r = p + (size_t)ii * j;
                        sd = sd + cff * (-3.5 * r[ii - 1] + 4.0 * r[ii - 2] - 0.5 * r[ii - 3]);
                    }
                } else if (d->bc_type == PQ_BC_NO_SLIP) {
                    for (int j = 0; j < jj; ++j) sb = sb + 2.0 * (p[(size_t)ii * j + 1] - p[(size_t)ii * j]);
                    for (int j = 0; j < jj; ++j)
                        sd = sd + 2.0 * (p[(size_t)ii * j + ii - 2] - p[(size_t)ii * j + ii - 1]);
                }
                for (int j = 0; j < jj; ++j) sb = sb - d->ss[l] * p[(size_t)ii * j];
                for (int j = 0; j < jj; ++j) sd = sd - d->ss[l] * p[(size_t)ii * j + ii - 1];
                zb[w][0][l] = sb / (double)jj;
                zb[w][1][l] = sd / (double)jj;
            }
            cf[w] = std::move(h);
        }
        rc = copy_in(c, (void*)m.corr, cf[0].data(), PQ_PTR_HOST);
        if (rc) return rc;
        rc = copy_in(c, (void*)m.corr2, cf[1].data(), PQ_PTR_HOST);
        if (rc) return rc;
        // inverse(z_b(mode, :, :)): rows = walls, columns = functions;
        // column-major [a11, a21, a12, a22].
        std::vector<double> ica((size_t)4 * PQ_MAXL, 0.0);
        for (int l = 1; l < L; ++l) {
            const double a11 = zb[0][0][l], a21 = zb[0][1][l], a12 = zb[1][0][l], a22 = zb[1][1][l];
            const double det = a11 * a22 - a12 * a21;
            if (!(std::fabs(det) > 0.0) || det != det) {
                // No momentum correction exists (e.g. a baroclinic mode with
                // ss = 0 and free slip): the context still solves Helmholtz
                // problems, but refuses the time step.
                c->channel_singular = true;
                continue;
            }
            ica[4 * l + 0] = a22 / det;
            ica[4 * l + 1] = -a21 / det;
            ica[4 * l + 2] = -a12 / det;
            ica[4 * l + 3] = a11 / det;
        }
        CK(cudaMemcpyAsync((void*)m.inv_corr_a, ica.data(), ica.size() * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return PQ_OK;
}

extern "C" {

int pq_helm(pq_ctx* c, double* zeta, int ptr_kind) {
    if (!c || !zeta) return PQ_ERR_ARG;
    CK(cudaSetDevice(c->device));
    int rc = copy_in(c, c->hm[0].helm_io, zeta, ptr_kind);
    if (rc) return rc;
    rc = run_helm(c, c->cur, PRO_PLAIN, EPI_HELM, 0);
    if (rc) return rc;
    rc = copy_out(c, zeta, c->hm[0].helm_io, ptr_kind);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->last_launches = 3;
    return PQ_OK;
}

int pq_pv_inversion(pq_ctx* c, const double* zeta, double* psi, int ptr_kind) {
    if (!c || !zeta || !psi) return PQ_ERR_ARG;
    if (c->channel_singular) return fail(c, PQ_ERR_UNSUPPORTED, "singular channel correction matrix");
    CK(cudaSetDevice(c->device));
    int rc = copy_in_state(c, c->hm[c->cur].zeta, zeta, ptr_kind);
    if (rc) return rc;
    c->pred_ready = false;
    c->zpar = c->cur;
    rc = run_helm(c, c->cur, PRO_MODAL, EPI_PV, 1);
    if (rc) return rc;
    rc = copy_out(c, psi, c->hm[0].psi, ptr_kind);
    if (rc) return rc;
    c->last_launches = 3;
    return check_status(c);
}

int pq_init_perturb(pq_ctx* c, const double* zeta_ic, int ptr_kind) {
    if (!c || !zeta_ic) return PQ_ERR_ARG;
    if (c->channel_singular) return fail(c, PQ_ERR_UNSUPPORTED, "singular channel correction matrix");
    CK(cudaSetDevice(c->device));
    const int ii = c->ii, jj = c->jj, L = c->L;
    const int nlev = c->leapfrog ? 2 : 1;  // init_rand fills both leapfrog levels
    std::vector<double> z((size_t)ii * jj * L * nlev);
    if (ptr_kind == PQ_PTR_DEVICE)
        CK(cudaMemcpy(z.data(), zeta_ic, z.size() * sizeof(double), cudaMemcpyDeviceToHost));
    else
        std::memcpy(z.data(), zeta_ic, z.size() * sizeof(double));
    // apply_dirichlet_bc(0, zeta), qg3.F90:383 (a channel has walls at
    // i = 0 and ii - 1 only, qg3p_laplace_bc.F90:227-251).
    for (int l = 0; l < L * nlev; ++l) {
        double* p = z.data() + (size_t)ii * jj * l;
        if (!c->periodic)
            for (int i = 0; i < ii; ++i) p[i] = p[i + (size_t)ii * (jj - 1)] = 0.0;
        for (int j = 0; j < jj; ++j) p[(size_t)ii * j] = p[(size_t)ii * j + ii - 1] = 0.0;
    }
    const Member& m = c->hm[0];
    // Zero all CABARET fields and both parities (qg3.F90:393-404).
    const size_t fb = align256(c->field_bytes);
    // Fields 0..18 of the arena: zeta_old[2], zeta[0], psi, res[0], res_beta[0],
    // ui, uj, uimo[2], ujmo[2], zeta_fi[2], zeta_fj[2], zeta[1], res_beta[1],
    // res[1] (corr is kept).
    CK(cudaMemsetAsync(m.zeta_old[0], 0, fb * 19, c->stream));
    int rc = copy_in_state(c, m.zeta, z.data(), PQ_PTR_HOST);
    if (rc) return rc;
    Scalars sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.dt = c->desc.dt;
    sc.tweight_a = 0.5;
    sc.tweight_u = 0.5;
    sc.model_time = c->desc.dt / 2.0;
    sc.dt_last = sc.dt;
    sc.tweight_a_last = sc.tweight_a;
    sc.tweight_u_last = sc.tweight_u;
    CK(cudaMemcpyAsync(c->d_sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    // diagnostic_time = 0, psi_av = 0, the quad sums 0 (qg3.F90:502-503, 540-558)
    if (c->psi_av) CK(cudaMemsetAsync(c->psi_av, 0, c->field_bytes, c->stream));
    if (c->quad) CK(cudaMemsetAsync(c->quad, 0, 23 * c->field_bytes, c->stream));
    // zeta was cleared together with the other fields; upload it again.
    rc = copy_in_state(c, m.zeta, z.data(), PQ_PTR_HOST);
    if (rc) return rc;
    c->cur = 0;
    c->zpar = 0;
    c->pred_ready = false;
    if (c->leapfrog) {
        // Both levels start from the initial condition (qg3.F90:382-404),
        // then FORWARD_EULER_START (:463-497) makes level 2 one dt ahead.
        sc.model_time = 0.0;
        CK(cudaMemcpyAsync(c->d_sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream));
        rc = copy_in_state(c, c->hm[1].zeta, z.data() + (size_t)ii * jj * L, PQ_PTR_HOST);
        if (rc) return rc;
        for (int p = 0; p < 2; ++p) {
            rc = run_helm(c, p, PRO_MODAL, EPI_PV, 1);
            if (rc) return rc;
            CK(launch_lf_rel_bc(c->ls[p], 1, 0, c->stream));
        }
        CK(launch_lf_forward_euler(c->ls[0], c->stream));
        rc = run_helm(c, 1, PRO_MODAL, EPI_PV, 1);
        if (rc) return rc;
        CK(launch_lf_rel_bc(c->ls[1], 1, 1, c->stream));
        c->initialized = true;
        return check_status(c);
    }
    rc = run_helm(c, 0, PRO_MODAL, EPI_PV, 1);
    if (rc) return rc;
    CK(launch_init_finish(c->ls[0], c->mixed ? 1 : 0, c->stream));
    c->initialized = true;
    return check_status(c);
}

int pq_step(pq_ctx* c, int nsteps) {
    int rc = pq_step_async(c, nsteps);
    if (rc) return rc;
    return check_status(c);
}

int pq_cabaret_step(pq_ctx* c, double dt, double tweight_a, double tweight_u) {
    if (!c) return PQ_ERR_ARG;
    if (!c->initialized) return fail(c, PQ_ERR_STATE, "pq_cabaret_step before pq_init_perturb");
    if (c->leapfrog) return fail(c, PQ_ERR_UNSUPPORTED, "pq_cabaret_step is the CABARET scheme's step");
    // cabaret_adapt_dt's own checks, qg3p_aux.F90:982-988
    if (!(dt > 0.0) || !(tweight_a >= 0.0) || !(tweight_u >= 0.0 && tweight_u <= 1.0))
        return fail(c, PQ_ERR_ARG, "dt > 0, tweight_a >= 0 and 0 <= tweight_u <= 1 required");
    CK(cudaSetDevice(c->device));
    static_assert(offsetof(Scalars, tweight_a) == offsetof(Scalars, dt) + sizeof(double) &&
                      offsetof(Scalars, tweight_u) == offsetof(Scalars, dt) + 2 * sizeof(double),
                  "dt and the time weights are adjacent");
    const double v[3] = {dt, tweight_a, tweight_u};
    CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->d_sc) + offsetof(Scalars, dt), v, sizeof(v),
                       cudaMemcpyHostToDevice, c->stream));
    // The predictor fused into the previous step used that step's dt.
    c->pred_ready = false;
    return pq_step(c, 1);
}

int pq_check(pq_ctx* c) {
    if (!c) return PQ_ERR_ARG;
    return check_status(c);
}

int pq_step_exchange(pq_ctx* c, const double* zeta_in, double* psi_out, int ptr_kind) {
    if (!c) return PQ_ERR_ARG;
    if (!c->initialized) return fail(c, PQ_ERR_STATE, "pq_step_exchange before pq_init_perturb");
    CK(cudaSetDevice(c->device));
    if (ptr_kind == PQ_PTR_HOST && zeta_in && psi_out) {
        // Pipelined: H2D into staging slot s on the input stream, D2D into
        // the state and the step on the context's stream, D2D of psi into
        // the output slot, D2H on the output stream.  A slot is reused two
        // calls later, after the events that guard it.
        auto& x = c->x;
        const size_t bytes = (size_t)c->ii * c->jj * c->L * sizeof(double);
        if (!x.in) {
            CK(cudaStreamCreateWithFlags(&x.in, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&x.out, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&x.entry, cudaEventDisableTiming));
            for (int s = 0; s < 2; ++s) {
                if (cudaMalloc(&x.stage_in[s], bytes) != cudaSuccess || cudaMalloc(&x.stage_out[s], bytes) != cudaSuccess) {
                    cudaGetLastError();
                    return fail(c, PQ_ERR_NOMEM, "cudaMalloc of the exchange staging buffers failed");
                }
                CK(cudaEventCreateWithFlags(&x.ready[s], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&x.consumed[s], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&x.produced[s], cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&x.done[s], cudaEventDisableTiming));
            }
        }
        const int s = x.slot;
        x.slot ^= 1;
        if (!x.sequence) {
            // The first copy of a sequence follows everything already on the
            // context's stream.
            CK(cudaEventRecord(x.entry, c->stream));
            CK(cudaStreamWaitEvent(x.in, x.entry, 0));
            x.sequence = true;
        }
        CK(cudaStreamWaitEvent(x.in, x.consumed[s], 0));
        CK(cudaMemcpyAsync(x.stage_in[s], zeta_in, bytes, cudaMemcpyHostToDevice, x.in));
        CK(cudaEventRecord(x.ready[s], x.in));
        CK(cudaStreamWaitEvent(c->stream, x.ready[s], 0));
        int rc = copy_in_state(c, c->hm[c->cur].zeta_old[c->cur], x.stage_in[s], PQ_PTR_DEVICE);
        if (rc) return rc;
        CK(cudaEventRecord(x.consumed[s], c->stream));
        c->pred_ready = false;
        rc = pq_step_async(c, 1);
        if (rc) return rc;
        CK(cudaStreamWaitEvent(c->stream, x.done[s], 0));
        rc = copy_out(c, x.stage_out[s], c->hm[0].psi, PQ_PTR_DEVICE);
        if (rc) return rc;
        CK(cudaEventRecord(x.produced[s], c->stream));
        CK(cudaStreamWaitEvent(x.out, x.produced[s], 0));
        CK(cudaMemcpyAsync(psi_out, x.stage_out[s], bytes, cudaMemcpyDeviceToHost, x.out));
        CK(cudaEventRecord(x.done[s], x.out));
        x.last = s;
        return PQ_OK;
    }
    if (zeta_in) {
        int rc = copy_in_state(c, c->hm[c->cur].zeta_old[c->cur], zeta_in, ptr_kind);
        if (rc) return rc;
        c->pred_ready = false;
    }
    int rc = pq_step_async(c, 1);
    if (rc) return rc;
    if (psi_out) {
        rc = copy_out(c, psi_out, c->hm[0].psi, ptr_kind);
        if (rc) return rc;
    }
    return PQ_OK;
}

int pq_step_async(pq_ctx* c, int nsteps) {
    if (!c || nsteps < 0) return PQ_ERR_ARG;
    if (!c->initialized) return fail(c, PQ_ERR_STATE, "pq_step before pq_init_perturb");
    CK(cudaSetDevice(c->device));
    int done = 0;
    long launches = 0;
    // One step at parity par: a captured one-step graph once the step's
    // variant is settled (fused predictor ready, or not fusing), else eager
    // (also when per-kernel timing is on).
    auto one = [&](int par) -> int {
        if (c->timing || (c->fuse && !c->pred_ready)) return run_step(c, par);
        if (!c->graph1[par]) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
            const int rc = run_step(c, par);
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&c->graph1[par], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
        } else {
            CK(cudaGraphLaunch(c->graph1[par], c->stream));
            c->pred_ready = c->fuse;
            c->zpar = par;
            return PQ_OK;
        }
        CK(cudaGraphLaunch(c->graph1[par], c->stream));
        return PQ_OK;
    };
    // Single steps until the two-step graph's entry state: parity 0 and, with
    // the fused predictor, the next step's inversion input already computed.
    while (done < nsteps && (c->cur == 1 || (c->fuse && !c->pred_ready))) {
        int rc = one(c->cur);
        if (rc) return rc;
        c->cur ^= 1;
        ++done;
        launches += step_launches(c);
    }
    if (nsteps - done >= 2) {
        if (!c->graph2) {
            cudaGraph_t g;
            const bool timing = c->timing;
            c->timing = false;  // no per-kernel events inside the graph
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
            int rc = run_step(c, 0);
            if (rc == PQ_OK) rc = run_step(c, 1);
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            c->timing = timing;
            if (rc) return rc;
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&c->graph2, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
        }
        while (nsteps - done >= 2) {
            CK(cudaGraphLaunch(c->graph2, c->stream));
            done += 2;
            launches += 2 * step_launches(c);
        }
    }
    if (done < nsteps) {
        int rc = one(0);
        if (rc) return rc;
        c->cur = 1;
        ++done;
        launches += step_launches(c);
    }
    c->last_launches = launches;
    return PQ_OK;
}

int pq_set_tuning(pq_ctx* c, const pq_tuning* t) {
    if (!c || !t) return PQ_ERR_ARG;
    if (t->cab_band < kMinBand || t->cab_band > kMaxBand) return fail(c, PQ_ERR_ARG, "cab_band out of range");
    CK(cudaSetDevice(c->device));  // the CTA counts below query this device's occupancy
    CK(cudaStreamSynchronize(c->stream));
    if (t->dst_group < 0 || c->L * t->dst_group > 8) return fail(c, PQ_ERR_ARG, "dst_group out of range");
    if (t->cab_kernel < 0 || t->cab_kernel > 2) return fail(c, PQ_ERR_ARG, "cab_kernel out of range");
    if (t->cab_kernel == 2 && !c->mixed)
        return fail(c, PQ_ERR_ARG, "cab_kernel 2 (two columns per lane) needs the mixed form's FP32 fields");
    if (t->pdl < 0 || t->pdl > 1) return fail(c, PQ_ERR_ARG, "pdl is 0 or 1");
    if (t->dst_algo < 0 || t->dst_algo > PQ_DST_TENSOR) return fail(c, PQ_ERR_ARG, "dst_algo is 0, 1 or 2");
    if (t->dst_algo) {
        const int rc = set_dst_algo(c, t->dst_algo);
        if (rc) return rc;
    }
    const int M = c->hm[0].M;
    int P[2];
    for (int dir = 0; dir < 2; ++dir) {
        const int want = dir == 0 ? t->dst_lanes : t->dst_lanes_inv;
        P[dir] = want > 0 ? want : dst_lanes_default(M, c->L, dir);
        const int V = M / P[dir];
        const int R = dst_rows_per_cta_host(P[dir], t->dst_group);
        if (!is_pow2(P[dir]) || P[dir] > 64 || V * P[dir] != M || V < 2 || V > 32 ||
            c->L * R * P[dir] > dst_max_threads_host(V))
            return fail(c, PQ_ERR_ARG, "dst_lanes out of range for this grid and dst_group");
    }
    for (int p = 0; p < 2; ++p) {
        c->hm[p].cab_sh = t->cab_band;
        c->hm[p].ntiles_cab = c->periodic   ? channel_ctas(c->ii, c->jj)
                              : t->cab_kernel ? cabaret_ctas(c->ii, c->jj, c->L, t->cab_band, t->cab_kernel, c->mixed)
                                              : cabaret_tile_ctas(c->ii, c->jj, c->L);
        c->ls[p].cab_kernel = t->cab_kernel;
        c->ls[p].ctas_cab = c->hm[p].ntiles_cab;
        c->ls[p].dst_group = t->dst_group;
        c->ls[p].pdl = t->pdl;
        c->ls[p].dst_lanes[0] = P[0];
        c->ls[p].dst_lanes[1] = P[1];
        const int R0 = dst_rows_per_cta_host(P[0], t->dst_group), R1 = dst_rows_per_cta_host(P[1], t->dst_group);
        c->ls[p].ctas_dst[0] = ((c->periodic ? c->jj : c->jj - 2) + R0 - 1) / R0;
        c->ls[p].ctas_dst[1] = (c->jj + R1 - 1) / R1;
    }
    int rc = upload_members(c);
    if (rc) return rc;
    for (auto& g : c->graph1)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    if (c->graph2) {
        cudaGraphExecDestroy(c->graph2);
        c->graph2 = nullptr;
    }
    CK(cudaStreamSynchronize(c->stream));
    return PQ_OK;
}

int pq_autotune(pq_ctx* c, int* choice) {
    if (!c) return PQ_ERR_ARG;
    CK(cudaSetDevice(c->device));
    // The decision per shape, for the process.
    static std::mutex mu;
    static std::map<std::vector<int>, int> cache;
    const std::vector<int> key = {c->ii, c->jj, c->L, c->periodic ? 1 : 0, c->mixed ? 1 : 0};
    int best = PQ_DST_BUTTERFLY;
    const bool candidates = c->mixed && !c->leapfrog && !c->helm_only && c->L > 1 && dst_mma_supported(c->hm[0].N);
    if (candidates) {
        bool known = false;
        {
            std::lock_guard<std::mutex> lk(mu);
            auto it = cache.find(key);
            if (it != cache.end()) {
                best = it->second;
                known = true;
            }
        }
        if (!known) {
            // Time the inversion (forward DST, tridiagonal, inverse DST) of
            // the current zeta with each algorithm; psi and the scalars it
            // overwrites are saved and restored, nothing else changes.
            const int prev = c->dst_algo;
            int rc = set_dst_algo(c, PQ_DST_TENSOR);
            if (rc) return rc;
            void* save = nullptr;
            if (cudaMalloc(&save, c->field_bytes + sizeof(Scalars)) != cudaSuccess) {
                cudaGetLastError();
                return fail(c, PQ_ERR_NOMEM, "autotune: scratch allocation failed");
            }
            char* sv = static_cast<char*>(save);
            CK(cudaMemcpyAsync(sv, c->hm[0].psi, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaMemcpyAsync(sv + c->field_bytes, c->d_sc, sizeof(Scalars), cudaMemcpyDeviceToDevice, c->stream));
            cudaEvent_t e0, e1;
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            float ms[3] = {0.f, 0.f, 0.f};
            const int algos[2] = {PQ_DST_BUTTERFLY, PQ_DST_TENSOR};
            for (int round = 0; round < 2 && !rc; ++round)  // two rounds: the second is kept
                for (int a = 0; a < 2 && !rc; ++a) {
                    rc = set_dst_algo(c, algos[a]);
                    for (int w = 0; w < 3 && !rc; ++w) rc = run_inversion(c, c->zpar, PRO_MODAL, nullptr);
                    if (rc) break;
                    CK(cudaEventRecord(e0, c->stream));
                    for (int k = 0; k < 10 && !rc; ++k) rc = run_inversion(c, c->zpar, PRO_MODAL, nullptr);
                    CK(cudaEventRecord(e1, c->stream));
                    CK(cudaEventSynchronize(e1));
                    CK(cudaEventElapsedTime(&ms[algos[a]], e0, e1));
                }
            CK(cudaMemcpyAsync(c->hm[0].psi, sv, c->field_bytes, cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaMemcpyAsync(c->d_sc, sv + c->field_bytes, sizeof(Scalars), cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaFree(save);
            if (rc) {
                set_dst_algo(c, prev);
                return rc;
            }
            rc = check_status(c);
            if (rc) return rc;
            best = ms[PQ_DST_TENSOR] < ms[PQ_DST_BUTTERFLY] ? PQ_DST_TENSOR : PQ_DST_BUTTERFLY;
            std::lock_guard<std::mutex> lk(mu);
            cache[key] = best;
        }
    }
    const int rc = set_dst_algo(c, best);
    if (rc) return rc;
    if (choice) *choice = best;
    return PQ_OK;
}

int pq_get_tuning(pq_ctx* c, pq_tuning* t) {
    if (!c || !t) return PQ_ERR_ARG;
    std::memset(t, 0, sizeof(*t));
    t->cab_band = c->hm[0].cab_sh;
    t->cab_kernel = c->ls[0].cab_kernel;
    t->dst_group = c->ls[0].dst_group;
    t->dst_lanes = c->ls[0].dst_lanes[0];
    t->dst_lanes_inv = c->ls[0].dst_lanes[1];
    t->pdl = c->ls[0].pdl;
    t->dst_algo = c->dst_algo;
    return PQ_OK;
}

int pq_sync(pq_ctx* c) {
    if (!c) return PQ_ERR_ARG;
    int rc = join_exchange(c);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return PQ_OK;
}

int pq_join(pq_ctx* c) {
    if (!c) return PQ_ERR_ARG;
    CK(cudaSetDevice(c->device));
    return join_exchange(c);
}

int pq_kernel_timing(pq_ctx* c, int enable) {
    if (!c) return PQ_ERR_ARG;
    c->timing = enable != 0;
    return PQ_OK;
}

int pq_kernel_times(pq_ctx* c, double* ms, long* launches) {
    if (!c || !ms || !launches) return PQ_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 4; ++k) {
        ms[k] = 0.0;
        launches[k] = 0;
    }
    for (auto& s : c->events) {
        for (int k = 0; k < 4; ++k) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, s.e[k], s.e[k + 1]));
            ms[k] += t;
            launches[k] += 1;
        }
        for (int k = 0; k < 5; ++k) cudaEventDestroy(s.e[k]);
    }
    c->events.clear();
    return PQ_OK;
}

int pq_energy(pq_ctx* c, double* ekin, double* epot) {
    if (!c || !ekin || !epot) return PQ_ERR_ARG;
    CK(cudaSetDevice(c->device));
    // energy(strat, psi BNLEAPFROG, ...) (qg3.F90:744): the second time level
    // for the leapfrog scheme.
    CK(launch_energy(c->ls[c->leapfrog ? 1 : 0], c->stream));
    Scalars sc;
    CK(cudaMemcpyAsync(&sc, c->d_sc, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    int rc = check_status(c);
    for (int k = 0; k < c->L; ++k) ekin[k] = sc.ekin[k];
    *epot = sc.epot;
    return rc;
}

int pq_cfl(pq_ctx* c, double* cfl) {
    if (!c || !cfl) return PQ_ERR_ARG;
    Scalars sc;
    CK(cudaMemcpyAsync(&sc, c->d_sc, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *cfl = sc.cfl;  // max |u| times the dt of the step that produced u
    return PQ_OK;
}

}  // extern "C"

namespace pq {

// Clears the CABARET fields of both parities (as pq_init_perturb does),
// installs `sc` and the status word, and resets the step parity; the caller
// then writes the prognostic fields with pq_set_field.  Used by the
// checkpoint pickup.
int reset_prognostic(pq_ctx* c, const Scalars& sc) {
    CK(cudaSetDevice(c->device));
    if (!c->leapfrog) CK(cudaMemsetAsync(c->hm[0].zeta_old[0], 0, align256(c->field_bytes) * 19, c->stream));
    CK(cudaMemcpyAsync(c->d_sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    if (c->psi_av) CK(cudaMemsetAsync(c->psi_av, 0, c->field_bytes, c->stream));
    if (c->quad) CK(cudaMemsetAsync(c->quad, 0, 23 * c->field_bytes, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->cur = 0;
    c->zpar = 0;
    c->pred_ready = false;
    return PQ_OK;
}

int step_launches(const pq_ctx* c) {
    const int tc = (c->mixed && c->dst_algo == PQ_DST_TENSOR && c->mma_mem && c->L > 1) ? 2 : 0;
    return (c->leapfrog ? (c->psi_av ? 6 : 5) : c->periodic ? 7 : 4) + (c->quad ? 1 : 0) + tc;
}

int read_scalars(pq_ctx* c, Scalars* sc) {
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(sc, c->d_sc, sizeof(*sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PQ_OK;
}

}  // namespace pq

extern "C" {

int pq_get_scalars(pq_ctx* c, double* out4) {
    if (!c || !out4) return PQ_ERR_ARG;
    Scalars sc;
    CK(cudaMemcpyAsync(&sc, c->d_sc, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out4[0] = sc.dt_last;
    out4[1] = sc.tweight_a_last;
    out4[2] = sc.tweight_u_last;
    out4[3] = sc.model_time;
    return PQ_OK;
}

}  // extern "C"

namespace {

// Reference-layout geometry of a field: leading dims and the offset of the
// device node (0, 0) inside it.
struct RefShape {
    int n1, n2;  // leading dims
    int oi, oj;  // reference (0-based) index of device node/face (0, 0)
};

bool ref_shape(int field, int ii, int jj, RefShape* s) {
    switch (field) {
        case PQ_F_PSI:
        case PQ_F_ZETA:
        case PQ_F_REL:
        case PQ_F_ZETA_OLD: *s = {ii + 2, jj + 2, 1, 1}; return true;
        case PQ_F_UI:
        case PQ_F_UIMO:
        case PQ_F_ZETA_FI: *s = {ii + 3, jj + 2, 1, 1}; return true;
        case PQ_F_UJ:
        case PQ_F_UJMO:
        case PQ_F_ZETA_FJ: *s = {ii + 2, jj + 3, 1, 1}; return true;
        case PQ_F_RES:
        case PQ_F_RES_BETA:
        case PQ_F_CORR: *s = {ii, jj, 0, 0}; return true;
        case PQ_F_PSI2:
        case PQ_F_ZETA2:
        case PQ_F_REL2:
        case PQ_F_ZETA_OLD2: *s = {ii + 2, jj + 2, 1, 1}; return true;
    }
    return false;
}

void* field_ptr(pq_ctx* c, int field) {
    const Member& m = c->hm[c->cur];
    const int cur = c->cur;
    if (c->leapfrog) {
        // Time levels 1 and 2 live in the level descriptors hm[0], hm[1].
        const Member& a = c->hm[0];
        const Member& b = c->hm[1];
        switch (field) {
            case PQ_F_PSI: return a.psi;
            case PQ_F_ZETA: return a.zeta;
            case PQ_F_REL: return a.rel;
            case PQ_F_ZETA_OLD: return a.zeta_old[0];
            case PQ_F_PSI2: return b.psi;
            case PQ_F_ZETA2: return b.zeta;
            case PQ_F_REL2: return b.rel;
            case PQ_F_ZETA_OLD2: return b.zeta_old[0];
        }
    }
    switch (field) {
        case PQ_F_PSI: return m.psi;
        case PQ_F_ZETA:
        case PQ_F_ZETA_OLD: return m.zeta_old[cur];
        case PQ_F_REL: return m.rel;
        case PQ_F_UI: return m.ui;
        case PQ_F_UJ: return m.uj;
        case PQ_F_UIMO: return m.uimo[cur];
        case PQ_F_UJMO: return m.ujmo[cur];
        case PQ_F_ZETA_FI: return m.zfi[cur];
        case PQ_F_ZETA_FJ: return m.zfj[cur];
        case PQ_F_RES: return m.res;
        case PQ_F_RES_BETA: return m.res_beta_other;  // res_beta of the last step
        case PQ_F_CORR: return (void*)m.corr;
    }
    return nullptr;
}

}  // namespace

extern "C" {

int pq_get_field(pq_ctx* c, int field, double* out) {
    if (!c || !out) return PQ_ERR_ARG;
    RefShape s;
    if (!ref_shape(field, c->ii, c->jj, &s)) return fail(c, PQ_ERR_ARG, "unknown field");
    CK(cudaSetDevice(c->device));
    // The closed-basin step keeps rel in registers: rebuild it.  The channel
    // and leapfrog steps store it.
    if (field == PQ_F_REL && !c->leapfrog && !c->periodic)
        CK(launch_rel(c->ls[c->zpar], c->mixed ? 1 : 0, c->stream));
    if (!field_ptr(c, field)) return fail(c, PQ_ERR_ARG, "field not held by this scheme");
    std::vector<double> dense((size_t)c->ii * c->jj * c->L);
    int rc = (field == PQ_F_PSI || field == PQ_F_PSI2 || field == PQ_F_CORR)
                 ? copy_out(c, dense.data(), field_ptr(c, field), PQ_PTR_HOST)
                                                      : copy_out_state(c, dense.data(), field_ptr(c, field), PQ_PTR_HOST);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)s.n1 * s.n2 * c->L;
    std::memset(out, 0, n * sizeof(double));
    for (int l = 0; l < c->L; ++l)
        for (int j = 0; j < c->jj; ++j)
            for (int i = 0; i < c->ii; ++i)
                out[(size_t)(i + s.oi) + (size_t)s.n1 * ((j + s.oj) + (size_t)s.n2 * l)] =
                    dense[(size_t)i + (size_t)c->ii * (j + (size_t)c->jj * l)];
    return PQ_OK;
}

int pq_set_field(pq_ctx* c, int field, const double* in) {
    if (!c || !in) return PQ_ERR_ARG;
    RefShape s;
    if (!ref_shape(field, c->ii, c->jj, &s) || field == PQ_F_CORR) return fail(c, PQ_ERR_ARG, "unknown field");
    if (!field_ptr(c, field)) return fail(c, PQ_ERR_ARG, "field not held by this scheme");
    CK(cudaSetDevice(c->device));
    std::vector<double> dense((size_t)c->ii * c->jj * c->L);
    for (int l = 0; l < c->L; ++l)
        for (int j = 0; j < c->jj; ++j)
            for (int i = 0; i < c->ii; ++i)
                dense[(size_t)i + (size_t)c->ii * (j + (size_t)c->jj * l)] =
                    in[(size_t)(i + s.oi) + (size_t)s.n1 * ((j + s.oj) + (size_t)s.n2 * l)];
    int rc = (field == PQ_F_PSI || field == PQ_F_PSI2) ? copy_in(c, field_ptr(c, field), dense.data(), PQ_PTR_HOST)
                                 : copy_in_state(c, field_ptr(c, field), dense.data(), PQ_PTR_HOST);
    if (rc) return rc;
    if (field == PQ_F_ZETA && !c->leapfrog) {
        rc = copy_in_state(c, c->hm[c->cur].zeta, dense.data(), PQ_PTR_HOST);
        c->zpar = c->cur;
    }
    if (rc) return rc;
    c->pred_ready = false;
    CK(cudaStreamSynchronize(c->stream));
    c->initialized = true;
    return PQ_OK;
}

}  // extern "C"
