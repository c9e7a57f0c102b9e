// pq_ctx.h -- the context behind the C ABI handle and the host helpers
// shared by the single-model API, the batched solver and the server.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pequod_b200.h"
#include "pq_common.cuh"
#include "pq_kernels.h"

struct pq_ctx {
    using Member = pq::Member;
    using LaunchSet = pq::LaunchSet;
    using Scalars = pq::Scalars;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;   // false: the stream belongs to a batch / server
    bool helm_only = false;   // only helm_io and spec are allocated
    pq_model_desc desc{};
    std::vector<double> wind;
    Member hm[2];               // host copies of the two parity descriptors
    Member* d_members = nullptr;  // device: [2]
    int* d_prefix = nullptr;      // device: {0}
    LaunchSet ls[2];
    char* arena = nullptr;
    size_t arena_bytes = 0;
    Scalars* d_sc = nullptr;
    int* d_status = nullptr;
    int cur = 0;          // parity of the next step
    bool initialized = false;
    bool fuse = false;        // fixed dt: the CABARET kernel applies the next predictor
    bool mixed = false;       // PQ_PREC_MIXED
    bool periodic = false;    // channel periodic in j
    bool channel_singular = false;  // channel without a momentum correction (singular wall matrix): pq_helm only
    bool leapfrog = false;    // PQ_SCHEME_LEAPFROG: cur is the level advanced next (lf - 1)
    bool pred_ready = false;  // zeta[cur] / res_beta[cur] already hold the next step's predictor
    int zpar = 0;             // parity whose zeta entered the last inversion
    cudaGraphExec_t graph2 = nullptr;     // two steps (parity 0, 1)
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};  // one step of each parity
    std::string err;
    long last_launches = 0;
    // Per-kernel CUDA-event timing of eagerly launched steps.
    struct StepEvents {
        cudaEvent_t e[5];
    };
    bool timing = false;
    std::vector<StepEvents> events;
    // host copies of layout facts
    int ii = 0, jj = 0, L = 0, pitch = 0;
    size_t field_bytes = 0;  // bytes of one L-layer field
    // Row-DST algorithm of the mixed form's baroclinic modes (pq_tuning.dst_algo):
    // PQ_DST_BUTTERFLY, or PQ_DST_TENSOR with its node-row buffer (gbuf) and
    // the split DST matrices in mma_mem and their TMA descriptor.
    int dst_algo = PQ_DST_BUTTERFLY;
    void* mma_mem = nullptr;
    size_t mma_bytes = 0;
    CUtensorMap mma_map;
    double* psi_av = nullptr;  // time average of psi (pq_average), FP64, node-shaped like psi
    double* quad = nullptr;    // the 23 quad eddy-covariance accumulators (pq_average mode 2)
    // Pipelined host exchange (pq_step_exchange with host buffers): the
    // copies run on their own streams through two dense device staging slots
    // each way, so that a step's input and output transfers overlap the
    // neighbouring steps' kernels.
    struct Exchange {
        cudaStream_t in = nullptr, out = nullptr;
        double* stage_in[2] = {nullptr, nullptr};
        double* stage_out[2] = {nullptr, nullptr};
        cudaEvent_t entry = nullptr, ready[2] = {}, consumed[2] = {}, produced[2] = {}, done[2] = {};
        int slot = 0;
        int last = -1;          // slot of the newest output copy, -1: none pending
        bool sequence = false;  // copies issued since the last join
    } x;
};

namespace pq {

enum { PRO_PLAIN = 0, PRO_MODAL = 1, PRO_STEP = 2 };
enum { EPI_SPEC = 0, EPI_HELM = 1, EPI_PV = 2 };

constexpr int kMinBand = 4;  // smallest CABARET band height a tuning may select
constexpr int kMaxBand = 128;

size_t align256(size_t x);
bool is_pow2(int x);
int fail(pq_ctx* c, int code, const std::string& msg);
int cuda_fail(pq_ctx* c, cudaError_t e, const char* where);

#define CK(call)                                                \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return pq::cuda_fail(c, e_, #call); \
    } while (0)

// Dense (ii, jj, L) <-> pitched field copies on the context's stream;
// *_state convert to / from FP32 for the mixed form's state fields.
int copy_in(pq_ctx* c, void* dst, const double* src, int kind);
int copy_out(pq_ctx* c, double* dst, const void* src, int kind);
int copy_in_state(pq_ctx* c, void* dst, const double* src, int kind);
int copy_out_state(pq_ctx* c, double* dst, const void* src, int kind);
int check_status(pq_ctx* c);
int upload_members(pq_ctx* c);
int run_helm(pq_ctx* c, int par, int prologue, int epilogue, int mean);
// The inversion of a step (forward DST with `prologue`, tridiagonal,
// inverse DST with the back-projection), through the tensor-core DST when
// the context selected it; ev (or null): events after each of the three.
int run_inversion(pq_ctx* c, int par, int prologue, cudaEvent_t* ev);
// Select the row-DST algorithm (allocating the tensor-core DST's buffers).
int set_dst_algo(pq_ctx* c, int algo);
int run_step(pq_ctx* c, int par);
// Checkpoint pickup support: clear the prognostic fields and install the
// scalars (reset_prognostic); copy the device scalars to the host.
int reset_prognostic(pq_ctx* c, const Scalars& sc);
int read_scalars(pq_ctx* c, Scalars* sc);
// Kernel launches of one step (the leapfrog time average adds one).
int step_launches(const pq_ctx* c);
// Order the context's stream after the pipelined exchange copies issued so
// far (no host wait).
int join_exchange(pq_ctx* c);
// pq_create's body.  helm_only: allocate only the Helmholtz fields (helm_io,
// spec) -- the batched solver's members; stream: use this stream instead of
// creating one (not owned).
int create_ctx(pq_ctx** out, const pq_model_desc* d, int device, bool helm_only, cudaStream_t stream);

}  // namespace pq
