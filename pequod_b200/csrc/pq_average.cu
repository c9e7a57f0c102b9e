// pq_average.cu -- the time-averaged streamfunction (host side).
//
// The reference accumulates psi_av = sum of dt * psi%sdata over the steps
// whose model time exceeds max_spin, with diagnostic_time the summed dt
// (qg3.F90:93, 502-503, 672-680, 725), and writes psi_av / diagnostic_time
// to qg<L>_<ii>_s_av.d (:886-899).  Here the sum is a node-shaped FP64 field
// (the layout of psi) added to inside the fused CABARET kernel (the channel:
// inside its rel kernel; the leapfrog scheme: one small kernel per sub-step),
// so a step costs one extra read and write of the sum and no launch; the
// host only starts, reads and writes it.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pequod_b200.h"
#include "pq_common.cuh"
#include "pq_ctx.h"

using namespace pq;

namespace {

void drop_graphs(pq_ctx* c) {
    if (c->graph2) cudaGraphExecDestroy(c->graph2);
    c->graph2 = nullptr;
    for (auto& g : c->graph1) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

bool put_record(FILE* f, const double* p, size_t n) {
    const int32_t nb = (int32_t)(n * sizeof(double));
    return std::fwrite(&nb, 4, 1, f) == 1 && std::fwrite(p, sizeof(double), n, f) == n &&
           std::fwrite(&nb, 4, 1, f) == 1;
}

}  // namespace

extern "C" {

int pq_average(pq_ctx* c, int enable, double threshold) {
    if (!c || enable < 0 || enable > 2) return PQ_ERR_ARG;
    if (c->helm_only) return fail(c, PQ_ERR_UNSUPPORTED, "no time loop on this context");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (enable == 2 && !c->quad) {
        void* p = nullptr;
        if (cudaMalloc(&p, 23 * c->field_bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, PQ_ERR_NOMEM, "cudaMalloc of the quad accumulators failed");
        }
        c->quad = static_cast<double*>(p);
    } else if (enable != 2 && c->quad) {
        CK(cudaFree(c->quad));
        c->quad = nullptr;
    }
    if (c->quad) CK(cudaMemsetAsync(c->quad, 0, 23 * c->field_bytes, c->stream));
    if (enable && !c->psi_av) {
        void* p = nullptr;
        if (cudaMalloc(&p, c->field_bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, PQ_ERR_NOMEM, "cudaMalloc of the time-average field failed");
        }
        c->psi_av = static_cast<double*>(p);
    } else if (!enable && c->psi_av) {
        CK(cudaFree(c->psi_av));
        c->psi_av = nullptr;
    }
    if (c->psi_av) CK(cudaMemsetAsync(c->psi_av, 0, c->field_bytes, c->stream));
    for (int p = 0; p < 2; ++p) {
        c->hm[p].psi_av = c->psi_av;
        c->hm[p].av_threshold = threshold;
        c->hm[p].quad = c->quad;
        c->hm[p].quad_stride = (long long)(c->field_bytes / sizeof(double));
    }
    int rc = upload_members(c);
    if (rc) return rc;
    Scalars sc;
    if ((rc = read_scalars(c, &sc))) return rc;
    sc.diag_time = 0.0;
    CK(cudaMemcpyAsync(c->d_sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // The leapfrog step (average) or the CABARET step (quad) gains or loses
    // a kernel: capture the graphs again.
    drop_graphs(c);
    return PQ_OK;
}

int pq_get_average(pq_ctx* c, double* psi_av, double* diagnostic_time) {
    if (!c) return PQ_ERR_ARG;
    if (!c->psi_av) return fail(c, PQ_ERR_STATE, "the time average is not on (pq_average)");
    Scalars sc;
    int rc = read_scalars(c, &sc);
    if (rc) return rc;
    if (diagnostic_time) *diagnostic_time = sc.diag_time;
    if (!psi_av) return PQ_OK;
    if (!(sc.diag_time > 0.0)) return fail(c, PQ_ERR_STATE, "no step has entered the time average yet");
    if ((rc = copy_out(c, psi_av, c->psi_av, PQ_PTR_HOST))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    const double cff = 1.0 / sc.diag_time;  // qg3.F90:891
    const size_t n = (size_t)c->ii * c->jj * c->L;
    for (size_t k = 0; k < n; ++k) psi_av[k] = psi_av[k] * cff;
    return PQ_OK;
}

// Layers of quad accumulator q: the interface ones (uu_i, vv_i, sc_ub,
// sc_vb, sc_bb_i) have L - 1.
static int quad_layers(const pq_ctx* c, int q) {
    return (q == 2 || q == 3 || q == 19 || q == 20 || q == 22) ? c->L - 1 : c->L;
}

int pq_get_quad(pq_ctx* c, int q, double* out) {
    if (!c || q < 0 || q >= 23 || !out) return PQ_ERR_ARG;
    if (!c->quad) return fail(c, PQ_ERR_STATE, "the quad covariances are not on (pq_average mode 2)");
    Scalars sc;
    int rc = read_scalars(c, &sc);
    if (rc) return rc;
    if (!(sc.diag_time > 0.0)) return fail(c, PQ_ERR_STATE, "no step has entered the time average yet");
    const int nl = quad_layers(c, q);
    if (nl <= 0) return PQ_OK;
    const size_t w = (size_t)c->ii * sizeof(double);
    CK(cudaMemcpy2DAsync(out, w, c->quad + (size_t)q * (c->field_bytes / sizeof(double)),
                         (size_t)c->pitch * sizeof(double), w, (size_t)c->jj * nl, cudaMemcpyDeviceToHost,
                         c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double cff = 1.0 / sc.diag_time;  // qg3.F90:891
    const size_t n = (size_t)c->ii * c->jj * nl;
    for (size_t k = 0; k < n; ++k) out[k] = out[k] * cff;
    return PQ_OK;
}

int pq_write_quad(pq_ctx* c, const char* path, double t_scale, double start_time_day) {
    if (!c || !path) return PQ_ERR_ARG;
    if (!c->quad) return fail(c, PQ_ERR_STATE, "the quad covariances are not on (pq_average mode 2)");
    double sc4[4];
    int rc = pq_get_scalars(c, sc4);
    if (rc) return rc;
    const double model_time_day = (c->leapfrog ? sc4[3] : sc4[3] - 0.5 * sc4[0]) * t_scale / 86400.0;
    const double total_time_day = start_time_day + model_time_day;
    std::vector<std::vector<double>> f(23);
    for (int q = 0; q < 23; ++q) {
        f[q].assign((size_t)c->ii * c->jj * std::max(quad_layers(c, q), 0), 0.0);
        if ((rc = pq_get_quad(c, q, f[q].data()))) return rc;
    }
    // qg3.F90:903-929: the two times, then each accumulator's whole data
    // array times 1 / diagnostic_time as one record.
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(c, PQ_ERR_ARG, std::string("Failed to open output file ") + path);
    bool ok = put_record(fp, &model_time_day, 1) && put_record(fp, &total_time_day, 1);
    for (int q = 0; q < 23 && ok; ++q) ok = put_record(fp, f[q].data(), f[q].size());
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(c, PQ_ERR_ARG, std::string("write failed: ") + path);
    return PQ_OK;
}

int pq_write_average(pq_ctx* c, const char* path, double t_scale, double start_time_day) {
    if (!c || !path) return PQ_ERR_ARG;
    double dtime = 0.0;
    std::vector<double> av((size_t)c->ii * c->jj * c->L);
    int rc = pq_get_average(c, av.data(), &dtime);
    if (rc) return rc;
    double sc4[4];
    if ((rc = pq_get_scalars(c, sc4))) return rc;
    // The reference writes at its data output, which for CABARET lies half
    // a step before the end of the step (qg3.F90:656-661, 886-899).
    const double model_time_day = (c->leapfrog ? sc4[3] : sc4[3] - 0.5 * sc4[0]) * t_scale / 86400.0;
    const double total_time_day = start_time_day + model_time_day;
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(c, PQ_ERR_ARG, std::string("Failed to open output file ") + path);
    bool ok = put_record(f, &model_time_day, 1) && put_record(f, &total_time_day, 1);
    const size_t n = (size_t)c->ii * c->jj;
    for (int l = 0; l < c->L && ok; ++l) ok = put_record(f, av.data() + n * l, n);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(c, PQ_ERR_ARG, std::string("write failed: ") + path);
    return PQ_OK;
}

}  // extern "C"
