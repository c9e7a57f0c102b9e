// pq_ensemble.cu -- an ensemble of runs of one configuration stepped
// together (the batched form of the time step).
//
// n members share a shape (ii, jj, L, precision) and a stream.  After each
// member's START_PERTURB initialisation and first step (which runs on its
// own: the fused next-step predictor does not exist yet), every step is one
// launch per kernel over all members -- the forward row DSTs, the
// tridiagonal solves, the inverse row DSTs with the back-projection and the
// fused CABARET kernel -- each CTA finding its member through prefix sums
// over the member descriptors, plus, when the tensor-core DST serves the
// mixed form, one tensor-core launch per member and direction.  The step
// sequence is captured once as CUDA graphs (two steps, and one step of each
// parity) and replayed.  A member's results equal the same run alone: every
// kernel computes each member independently.
#include <cstring>
#include <string>
#include <vector>

#include "pq_ctx.h"
#include "pq_dst_mma.h"

using namespace pq;

struct pq_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<pq_ctx*> m;
    std::vector<char> ready;  // initialised
    bool stepping = false;    // every member past its first step, in lockstep
    int cur = 0;              // parity of the next merged step
    Member* d_desc = nullptr; // [2][n]: the members at parity 0, then parity 1
    int* d_pref = nullptr;    // prefix sums: fwd DST, inv DST, tridiagonal, CABARET
    LaunchSet ls[2];
    cudaGraphExec_t g2 = nullptr, g1[2] = {nullptr, nullptr};
    std::string err;
};

namespace {

int efail(pq_ensemble* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    return code;
}

#define EK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return efail(e, PQ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void drop_graphs(pq_ensemble* e) {
    if (e->g2) cudaGraphExecDestroy(e->g2);
    for (auto& g : e->g1)
        if (g) cudaGraphExecDestroy(g);
    e->g2 = e->g1[0] = e->g1[1] = nullptr;
}

// Device descriptors of every member at both parities and the grouped
// launch sets (the members' own descriptors as they are now).
int build_launch_sets(pq_ensemble* e) {
    const int n = (int)e->m.size();
    std::vector<Member> hd(2 * n);
    for (int p = 0; p < 2; ++p)
        for (int k = 0; k < n; ++k) hd[p * n + k] = e->m[k]->hm[p];
    const LaunchSet& l0 = e->m[0]->ls[0];
    std::vector<int> hp(4 * n);
    for (int k = 0; k < n; ++k) {
        hp[k] = k * l0.ctas_dst[0];
        hp[n + k] = k * l0.ctas_dst[1];
        hp[2 * n + k] = k * l0.ctas_tri;
        hp[3 * n + k] = k * l0.ctas_cab;
    }
    EK(cudaMemcpyAsync(e->d_desc, hd.data(), hd.size() * sizeof(Member), cudaMemcpyHostToDevice, e->stream));
    EK(cudaMemcpyAsync(e->d_pref, hp.data(), hp.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    for (int p = 0; p < 2; ++p) {
        LaunchSet s = e->m[0]->ls[p];
        s.members = e->d_desc + p * n;
        s.one = nullptr;
        s.nmem = n;
        s.prefix_dst[0] = e->d_pref;
        s.prefix_dst[1] = e->d_pref + n;
        s.prefix_tri = e->d_pref + 2 * n;
        s.prefix_cab = e->d_pref + 3 * n;
        s.ctas_dst[0] = n * l0.ctas_dst[0];
        s.ctas_dst[1] = n * l0.ctas_dst[1];
        s.ctas_tri = n * l0.ctas_tri;
        s.ctas_cab = n * l0.ctas_cab;
        const pq_ctx* c0 = e->m[0];
        s.gemm_bc = (c0->mixed && c0->dst_algo == PQ_DST_TENSOR && c0->mma_mem) ? 1 : 0;
        e->ls[p] = s;
    }
    return PQ_OK;
}

// One merged step of parity p (fixed dt: the predictor is fused).
int merged_step(pq_ensemble* e, int p) {
    const LaunchSet& ls = e->ls[p];
    const int f32 = e->m[0]->mixed ? 1 : 0;
    EK(launch_dst_forward(ls, PRO_MODAL, f32, e->stream));
    if (ls.gemm_bc)
        for (pq_ctx* c : e->m) {
            DstMmaArgs a{};
            const Member& h = c->hm[0];
            a.x = static_cast<const float*>(h.gbuf);
            a.y = static_cast<float*>(h.spec);
            a.ls = h.lstride;
            a.pitch = h.pitch;
            a.N = h.N;
            a.Kp = h.N / 2 > 64 ? h.N / 2 : 64;
            a.nj = c->jj - 2;
            a.jlo = 1;
            a.rows = (c->L - 1) * a.nj;
            a.status = c->d_status;
            EK(launch_dst_mma(a, c->mma_map, e->stream));
        }
    EK(launch_tridiag(ls, 1, f32, e->stream));
    if (ls.gemm_bc)
        for (pq_ctx* c : e->m) {
            DstMmaArgs a{};
            const Member& h = c->hm[0];
            a.x = static_cast<const float*>(h.spec);
            a.y = static_cast<float*>(h.gbuf);
            a.ls = h.lstride;
            a.pitch = h.pitch;
            a.N = h.N;
            a.Kp = h.N / 2 > 64 ? h.N / 2 : 64;
            a.nj = c->jj - 2;
            a.jlo = 1;
            a.rows = (c->L - 1) * a.nj;
            a.status = c->d_status;
            EK(launch_dst_mma(a, c->mma_map, e->stream));
        }
    EK(launch_dst_inverse(ls, EPI_PV, f32, e->stream));
    EK(launch_cabaret_fused(ls, 1, f32, e->stream));
    return PQ_OK;
}

int capture(pq_ensemble* e, cudaGraphExec_t* out, int p0, int steps) {
    cudaGraph_t g;
    EK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    int rc = PQ_OK;
    for (int s = 0; s < steps && !rc; ++s) rc = merged_step(e, p0 ^ (s & 1));
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) return rc;
    EK(ce);
    ce = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    EK(ce);
    return PQ_OK;
}

}  // namespace

extern "C" {

int pq_ensemble_create(pq_ensemble** out, int n, const pq_model_desc* d, int device) {
    if (!out || n < 1 || !d) return PQ_ERR_ARG;
    pq_ensemble* e = new pq_ensemble;
    *out = e;
    e->device = device;
    if (d->scheme != PQ_SCHEME_CABARET || d->adapt_dt || d->periodic_j)
        return efail(e, PQ_ERR_UNSUPPORTED, "an ensemble steps closed-basin CABARET runs with a fixed dt");
    EK(cudaSetDevice(device));
    EK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    for (int k = 0; k < n; ++k) {
        pq_ctx* c = nullptr;
        const int rc = create_ctx(&c, d, device, false, e->stream);
        if (rc) {
            const std::string msg = c ? c->err : std::string("context creation failed");
            if (c) pq_destroy(c);
            return efail(e, rc, "member " + std::to_string(k) + ": " + msg);
        }
        e->m.push_back(c);
    }
    e->ready.assign(n, 0);
    if (cudaMalloc(&e->d_desc, 2 * n * sizeof(Member)) != cudaSuccess ||
        cudaMalloc(&e->d_pref, 4 * n * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return efail(e, PQ_ERR_NOMEM, "ensemble descriptor allocation failed");
    }
    return PQ_OK;
}

void pq_ensemble_destroy(pq_ensemble* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    drop_graphs(e);
    for (pq_ctx* c : e->m) pq_destroy(c);
    if (e->d_desc) cudaFree(e->d_desc);
    if (e->d_pref) cudaFree(e->d_pref);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* pq_ensemble_last_error(const pq_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }
void* pq_ensemble_stream(pq_ensemble* e) { return e ? (void*)e->stream : nullptr; }
int pq_ensemble_size(const pq_ensemble* e) { return e ? (int)e->m.size() : 0; }

pq_ctx* pq_ensemble_member(pq_ensemble* e, int k) {
    if (!e || k < 0 || k >= (int)e->m.size()) return nullptr;
    return e->m[k];
}

int pq_ensemble_autotune(pq_ensemble* e, int* choice) {
    if (!e) return PQ_ERR_ARG;
    if (e->stepping) return efail(e, PQ_ERR_STATE, "autotune before the first step");
    int best = PQ_DST_BUTTERFLY;
    int rc = pq_autotune(e->m[0], &best);
    if (rc) return efail(e, rc, e->m[0]->err);
    for (size_t k = 1; k < e->m.size(); ++k) {
        rc = set_dst_algo(e->m[k], best);
        if (rc) return efail(e, rc, e->m[k]->err);
    }
    if (choice) *choice = best;
    return PQ_OK;
}

int pq_ensemble_set_dst_algo(pq_ensemble* e, int algo) {
    if (!e) return PQ_ERR_ARG;
    if (e->stepping) return efail(e, PQ_ERR_STATE, "choose the DST algorithm before the first step");
    for (pq_ctx* c : e->m) {
        const int rc = set_dst_algo(c, algo);
        if (rc) return efail(e, rc, c->err);
    }
    return PQ_OK;
}

int pq_ensemble_init(pq_ensemble* e, int k, const double* zeta_ic, int ptr_kind) {
    if (!e || k < 0 || k >= (int)e->m.size()) return PQ_ERR_ARG;
    if (e->stepping) return efail(e, PQ_ERR_STATE, "initialise every member before the first step");
    const int rc = pq_init_perturb(e->m[k], zeta_ic, ptr_kind);
    if (rc) return efail(e, rc, "member " + std::to_string(k) + ": " + e->m[k]->err);
    e->ready[k] = 1;
    return PQ_OK;
}

int pq_ensemble_step_async(pq_ensemble* e, int nsteps) {
    if (!e || nsteps < 0) return PQ_ERR_ARG;
    for (char r : e->ready)
        if (!r) return efail(e, PQ_ERR_STATE, "every member must be initialised before stepping");
    EK(cudaSetDevice(e->device));
    if (nsteps == 0) return PQ_OK;
    if (!e->stepping) {
        // Each member's first step alone (it computes the predictor the
        // merged steps then fuse), then the grouped descriptors.
        for (pq_ctx* c : e->m) {
            const int rc = run_step(c, c->cur);
            if (rc) return efail(e, rc, c->err);
            c->cur ^= 1;
        }
        e->cur = e->m[0]->cur;
        const int rc = build_launch_sets(e);
        if (rc) return rc;
        e->stepping = true;
        if (--nsteps == 0) return PQ_OK;
    }
    while (nsteps > 0) {
        if (nsteps >= 2 && e->cur == 0) {
            if (!e->g2) {
                const int rc = capture(e, &e->g2, 0, 2);
                if (rc) return rc;
            }
            EK(cudaGraphLaunch(e->g2, e->stream));
            nsteps -= 2;
            continue;
        }
        if (!e->g1[e->cur]) {
            const int rc = capture(e, &e->g1[e->cur], e->cur, 1);
            if (rc) return rc;
        }
        EK(cudaGraphLaunch(e->g1[e->cur], e->stream));
        e->cur ^= 1;
        --nsteps;
    }
    // The members' own bookkeeping follows the merged steps (parity, the
    // fused predictor), so that their fields and diagnostics read right.
    for (pq_ctx* c : e->m) {
        c->cur = e->cur;
        c->zpar = e->cur ^ 1;
        c->pred_ready = true;
    }
    return PQ_OK;
}

// Wait for the stream; PQ_ERR_NAN names the first member whose status
// reports a NaN (the reference aborts there).
int pq_ensemble_sync(pq_ensemble* e) {
    if (!e) return PQ_ERR_ARG;
    EK(cudaSetDevice(e->device));
    EK(cudaStreamSynchronize(e->stream));
    for (size_t k = 0; k < e->m.size(); ++k) {
        pq_ctx* c = e->m[k];
        const int rc = check_status(c);
        if (rc) return efail(e, rc, "member " + std::to_string(k) + ": " + c->err);
    }
    return PQ_OK;
}

int pq_ensemble_step(pq_ensemble* e, int nsteps) {
    const int rc = pq_ensemble_step_async(e, nsteps);
    if (rc) return rc;
    return pq_ensemble_sync(e);
}

}  // extern "C"
