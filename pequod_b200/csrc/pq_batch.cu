// pq_batch.cu -- batched Helmholtz solves: many independent helm problems
// (qg3p_helmholtz.F90:614-769, one helm_cache per problem) of mixed sizes and
// mode counts solved by grouped launches.
//
// Members are grouped into classes that share a launch geometry: the row
// DSTs by (ii, L) (the lane-group shape depends on ii, the CTA on L), the
// tridiagonal solves by jj (its shared-memory strip).  Each class is one
// launch over all its members (a per-member CTA prefix maps CTAs to
// members).  A solve is three phases -- forward DSTs, tridiagonal solves,
// inverse DSTs -- whose classes are independent; the whole solve is captured
// once as a CUDA graph with the classes of a phase on parallel branches.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "pq_ctx.h"

using namespace pq;

struct pq_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<pq_ctx*> mem;
    std::string err;
    struct Class {
        LaunchSet ls;
        std::vector<int> idx;
    };
    std::vector<Class> dst_cls, tri_cls;
    Member* d_dst = nullptr;  // member descriptors in DST-class order
    Member* d_tri = nullptr;  // in tridiagonal-class order
    int* d_pref = nullptr;    // every class's CTA prefix arrays
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;
    cudaGraphExec_t graph = nullptr;
    size_t bytes = 0;
};

namespace {

int bfail(pq_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

#define BK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return bfail(b, PQ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// The three phases, each class of a phase on side stream (class index mod S),
// joined back into b->stream.
int enqueue_solve(pq_batch* b) {
    const int S = (int)b->side.size();
    auto phase = [&](std::vector<pq_batch::Class>& cls, int what) -> int {
        BK(cudaEventRecord(b->ev[0], b->stream));
        for (int s = 0; s < S; ++s) BK(cudaStreamWaitEvent(b->side[s], b->ev[0], 0));
        for (size_t k = 0; k < cls.size(); ++k) {
            cudaStream_t st = b->side[k % S];
            cudaError_t e;
            if (what == 0)
                e = launch_dst_forward(cls[k].ls, PRO_PLAIN, 0, st);
            else if (what == 1)
                e = launch_tridiag(cls[k].ls, 0, 0, st);
            else
                e = launch_dst_inverse(cls[k].ls, EPI_HELM, 0, st);
            if (e != cudaSuccess) return bfail(b, PQ_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
        }
        for (int s = 0; s < S; ++s) {
            BK(cudaEventRecord(b->ev[1 + s], b->side[s]));
            BK(cudaStreamWaitEvent(b->stream, b->ev[1 + s], 0));
        }
        return PQ_OK;
    };
    int rc = phase(b->dst_cls, 0);
    if (!rc) rc = phase(b->tri_cls, 1);
    if (!rc) rc = phase(b->dst_cls, 2);
    return rc;
}

}  // namespace

extern "C" {

const char* pq_batch_last_error(const pq_batch* b) { return b ? b->err.c_str() : "null batch"; }
size_t pq_batch_device_bytes(const pq_batch* b) { return b ? b->bytes : 0; }
void* pq_batch_stream(pq_batch* b) { return b ? (void*)b->stream : nullptr; }

void pq_batch_destroy(pq_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (pq_ctx* c : b->mem) pq_destroy(c);
    if (b->d_dst) cudaFree(b->d_dst);
    for (cudaStream_t s : b->side) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int pq_batch_create(pq_batch** out, int n, const int* ii, const int* jj, const int* layers, const double* ss,
                    int device) {
    if (!out || n <= 0 || !ii || !jj || !layers || !ss) return PQ_ERR_ARG;
    *out = nullptr;
    pq_batch* b = new pq_batch;
    *out = b;
    b->device = device;
    BK(cudaSetDevice(device));
    BK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    int sm_count = 0;
    BK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device));
    // One helm-only context per member: tables, pivots and the helm_io /
    // spectral fields, all on the batch's stream.
    size_t so = 0;
    for (int k = 0; k < n; ++k) {
        pq_model_desc d;
        std::memset(&d, 0, sizeof(d));
        d.ii = ii[k];
        d.jj = jj[k];
        d.layers = layers[k];
        d.limiter = 1;
        d.bc_type = PQ_BC_FREE_SLIP;
        d.dt = 1.0;
        const int L = layers[k];
        if (L < 1 || L > PQ_MAX_LAYERS) return bfail(b, PQ_ERR_ARG, "layers out of range");
        for (int a = 0; a < L; ++a) {
            d.ss[a] = ss[so + a];
            d.h[a] = 1.0;
            d.m2z[a + L * a] = 1.0;
            d.z2m[a + L * a] = 1.0;
        }
        so += L;
        pq_ctx* c = nullptr;
        const int rc = create_ctx(&c, &d, device, true, b->stream);
        if (rc) {
            const std::string msg = c ? c->err : std::string("member rejected");
            if (c) pq_destroy(c);
            return bfail(b, rc, "member " + std::to_string(k) + ": " + msg);
        }
        b->mem.push_back(c);
        b->bytes += c->arena_bytes;
    }
    // Classes.
    std::map<std::pair<int, int>, std::vector<int>> dk;
    std::map<int, std::vector<int>> tk;
    for (int k = 0; k < n; ++k) {
        dk[{ii[k], layers[k]}].push_back(k);
        tk[jj[k]].push_back(k);
    }
    std::vector<Member> hd, ht;
    std::vector<int> pref;
    struct Pending {
        size_t mem_off, pref_off[3];
    };
    std::vector<Pending> pd, pt;
    for (auto& kv : dk) {
        pq_batch::Class cl{};
        cl.idx = kv.second;
        Pending p;
        p.mem_off = hd.size();
        const int I = kv.first.first, L = kv.first.second, N = I - 1;
        int maxJ = 0, maxPitch = 0;
        for (int dir = 0; dir < 2; ++dir) {
            cl.ls.dst_lanes[dir] = dst_lanes_batched(N / 2);
            const int R = dst_rows_per_cta_host(cl.ls.dst_lanes[dir], 0);
            p.pref_off[dir] = pref.size();
            int acc = 0;
            for (int k : cl.idx) {
                pref.push_back(acc);
                const int rows = dir == 0 ? jj[k] - 2 : jj[k];
                acc += (rows + R - 1) / R;
            }
            cl.ls.ctas_dst[dir] = acc;
        }
        for (int k : cl.idx) {
            hd.push_back(b->mem[k]->hm[0]);
            maxJ = std::max(maxJ, jj[k]);
            maxPitch = std::max(maxPitch, b->mem[k]->pitch);
        }
        LaunchSet& s = cl.ls;
        s.nmem = (int)cl.idx.size();
        s.maxL = L;
        s.maxN = N;
        s.maxI = I;
        s.maxJ = maxJ;
        s.maxPitch = maxPitch;
        s.dst_group = 0;
        s.sm_count = sm_count;
        b->dst_cls.push_back(cl);
        pd.push_back(p);
    }
    for (auto& kv : tk) {
        pq_batch::Class cl{};
        cl.idx = kv.second;
        Pending p;
        p.mem_off = ht.size();
        p.pref_off[2] = pref.size();
        int acc = 0, maxL = 0, maxN = 0, maxI = 0, maxPitch = 0;
        for (int k : cl.idx) {
            pref.push_back(acc);
            const Member& m = b->mem[k]->hm[0];
            acc += m.ntiles_tri;
            ht.push_back(m);
            maxL = std::max(maxL, m.L);
            maxN = std::max(maxN, m.N);
            maxI = std::max(maxI, m.ii);
            maxPitch = std::max(maxPitch, m.pitch);
        }
        LaunchSet& s = cl.ls;
        s.nmem = (int)cl.idx.size();
        s.ctas_tri = acc;
        s.maxL = maxL;
        s.maxN = maxN;
        s.maxI = maxI;
        s.maxJ = kv.first;
        s.maxPitch = maxPitch;
        s.sm_count = sm_count;
        b->tri_cls.push_back(cl);
        pt.push_back(p);
    }
    // Device copies: descriptors in both orders, then the prefix arrays.
    const size_t mbytes = align256(sizeof(Member) * (size_t)n);
    void* dev = nullptr;
    BK(cudaMalloc(&dev, 2 * mbytes + align256(sizeof(int) * pref.size())));
    b->d_dst = static_cast<Member*>(dev);
    b->d_tri = reinterpret_cast<Member*>(static_cast<char*>(dev) + mbytes);
    b->d_pref = reinterpret_cast<int*>(static_cast<char*>(dev) + 2 * mbytes);
    b->bytes += 2 * mbytes + align256(sizeof(int) * pref.size());
    BK(cudaMemcpyAsync(b->d_dst, hd.data(), sizeof(Member) * n, cudaMemcpyHostToDevice, b->stream));
    BK(cudaMemcpyAsync(b->d_tri, ht.data(), sizeof(Member) * n, cudaMemcpyHostToDevice, b->stream));
    BK(cudaMemcpyAsync(b->d_pref, pref.data(), sizeof(int) * pref.size(), cudaMemcpyHostToDevice, b->stream));
    for (size_t q = 0; q < b->dst_cls.size(); ++q) {
        LaunchSet& s = b->dst_cls[q].ls;
        s.members = b->d_dst + pd[q].mem_off;
        s.prefix_dst[0] = b->d_pref + pd[q].pref_off[0];
        s.prefix_dst[1] = b->d_pref + pd[q].pref_off[1];
    }
    for (size_t q = 0; q < b->tri_cls.size(); ++q) {
        LaunchSet& s = b->tri_cls[q].ls;
        s.members = b->d_tri + pt[q].mem_off;
        s.prefix_tri = b->d_pref + pt[q].pref_off[2];
    }
    const int S = (int)std::min<size_t>(8, std::max(b->dst_cls.size(), b->tri_cls.size()));
    b->side.resize(S);
    for (auto& st : b->side) BK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->ev.resize(1 + S);
    for (auto& e : b->ev) BK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    BK(cudaStreamSynchronize(b->stream));
    return PQ_OK;
}

int pq_batch_set_rhs(pq_batch* b, int k, const double* rhs, int ptr_kind) {
    if (!b || !rhs || k < 0 || k >= (int)b->mem.size()) return PQ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    pq_ctx* c = b->mem[k];
    const int rc = copy_in(c, c->hm[0].helm_io, rhs, ptr_kind);
    return rc ? bfail(b, rc, c->err) : PQ_OK;
}

int pq_batch_get(pq_batch* b, int k, double* out, int ptr_kind) {
    if (!b || !out || k < 0 || k >= (int)b->mem.size()) return PQ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    pq_ctx* c = b->mem[k];
    const int rc = copy_out(c, out, c->hm[0].helm_io, ptr_kind);
    return rc ? bfail(b, rc, c->err) : PQ_OK;
}

int pq_batch_solve_async(pq_batch* b) {
    if (!b) return PQ_ERR_ARG;
    BK(cudaSetDevice(b->device));
    if (!b->graph) {
        cudaGraph_t g;
        BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
        const int rc = enqueue_solve(b);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return bfail(b, PQ_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return bfail(b, PQ_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    }
    BK(cudaGraphLaunch(b->graph, b->stream));
    return PQ_OK;
}

int pq_batch_sync(pq_batch* b) {
    if (!b) return PQ_ERR_ARG;
    BK(cudaStreamSynchronize(b->stream));
    return PQ_OK;
}

int pq_batch_helm(pq_batch* b, double* const* zeta, int ptr_kind) {
    if (!b || !zeta) return PQ_ERR_ARG;
    for (size_t k = 0; k < b->mem.size(); ++k) {
        const int rc = pq_batch_set_rhs(b, (int)k, zeta[k], ptr_kind);
        if (rc) return rc;
    }
    int rc = pq_batch_solve_async(b);
    if (rc) return rc;
    for (size_t k = 0; k < b->mem.size(); ++k) {
        rc = pq_batch_get(b, (int)k, zeta[k], ptr_kind);
        if (rc) return rc;
    }
    return pq_batch_sync(b);
}

int pq_batch_launch_count(const pq_batch* b) {
    return b ? (int)(2 * b->dst_cls.size() + b->tri_cls.size()) : 0;
}

}  // extern "C"
