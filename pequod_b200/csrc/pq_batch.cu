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
//
// Precision (pq_batch_create_ex): FP64 throughout, or the mixed form --
// the first layer of every member (the barotropic, ss = 0 problem of a
// stratified model) keeps the FP64 transforms and the other layers are
// transformed in FP32 -- by the FP32 butterfly or by the tensor-core DST
// (three-term BF16 split, FP32 accumulation; one launch per member and
// direction between the class launches), chosen per DST class (ii, L):
// fixed, or measured at creation by timing the class's forward and inverse
// launches both ways (the autotuner).  The tridiagonal solves are FP64.
#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "pq_ctx.h"
#include "pq_dst_mma.h"

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
    int f32 = 0;                     // mixed form
    std::vector<int> tensor;         // per DST class: 1 when the tensor-core DST transforms its FP32 layers
    void* mma_mem = nullptr;         // the tensor-core DST's node rows (per member) and tables (per N)
    std::vector<size_t> gbuf_off;    // per member, into mma_mem (0: none)
    std::map<int, CUtensorMap> maps;  // per N
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
// The tensor-core DST of member k's FP32 layers: forward (dir 0) from its
// node rows to its spectral rows, inverse (dir 1) back.
cudaError_t member_mma(pq_batch* b, int k, int dir, cudaStream_t st) {
    const pq_ctx* c = b->mem[k];
    const Member& h = c->hm[0];
    DstMmaArgs a{};
    a.x = static_cast<const float*>(dir == 0 ? h.gbuf : h.spec);
    a.y = static_cast<float*>(dir == 0 ? h.spec : h.gbuf);
    a.ls = h.lstride;
    a.pitch = h.pitch;
    a.N = h.N;
    a.Kp = h.N / 2 > 64 ? h.N / 2 : 64;
    a.nj = c->jj - 2;
    a.jlo = 1;
    a.rows = (c->L - 1) * a.nj;
    a.status = c->d_status;
    return launch_dst_mma(a, b->maps.at(h.N), st);
}

// One DST class's launches in direction `dir` (0 forward, 1 inverse) on st.
cudaError_t class_dst(pq_batch* b, size_t q, int dir, cudaStream_t st) {
    pq_batch::Class& cl = b->dst_cls[q];
    cudaError_t e = cudaSuccess;
    if (dir == 0) {
        e = launch_dst_forward(cl.ls, PRO_PLAIN, b->f32, st);
        if (cl.ls.gemm_bc)
            for (int k : cl.idx)
                if (e == cudaSuccess) e = member_mma(b, k, 0, st);
    } else {
        if (cl.ls.gemm_bc)
            for (int k : cl.idx)
                if (e == cudaSuccess) e = member_mma(b, k, 1, st);
        if (e == cudaSuccess) e = launch_dst_inverse(cl.ls, EPI_HELM, b->f32, st);
    }
    return e;
}

int enqueue_solve(pq_batch* b) {
    const int S = (int)b->side.size();
    auto phase = [&](std::vector<pq_batch::Class>& cls, int what) -> int {
        BK(cudaEventRecord(b->ev[0], b->stream));
        for (int s = 0; s < S; ++s) BK(cudaStreamWaitEvent(b->side[s], b->ev[0], 0));
        for (size_t k = 0; k < cls.size(); ++k) {
            cudaStream_t st = b->side[k % S];
            cudaError_t e;
            if (what == 0)
                e = class_dst(b, k, 0, st);
            else if (what == 1)
                e = launch_tridiag(cls[k].ls, 0, b->f32, st);
            else
                e = class_dst(b, k, 1, st);
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
    if (b->mma_mem) cudaFree(b->mma_mem);
    for (cudaStream_t s : b->side) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int pq_batch_create(pq_batch** out, int n, const int* ii, const int* jj, const int* layers, const double* ss,
                    int device) {
    return pq_batch_create_ex(out, n, ii, jj, layers, ss, PQ_PREC_FP64, PQ_DST_BUTTERFLY, device);
}

int pq_batch_create_ex(pq_batch** out, int n, const int* ii, const int* jj, const int* layers, const double* ss,
                       int precision, int dst_algo, int device) {
    if (!out || n <= 0 || !ii || !jj || !layers || !ss) return PQ_ERR_ARG;
    *out = nullptr;
    pq_batch* b = new pq_batch;
    *out = b;
    b->device = device;
    if (precision != PQ_PREC_FP64 && precision != PQ_PREC_MIXED) return bfail(b, PQ_ERR_ARG, "bad precision");
    if (dst_algo < 0 || dst_algo > PQ_DST_TENSOR) return bfail(b, PQ_ERR_ARG, "dst_algo is 0, 1 or 2");
    if (precision == PQ_PREC_FP64 && dst_algo == PQ_DST_TENSOR)
        return bfail(b, PQ_ERR_UNSUPPORTED, "the tensor-core DST serves the mixed form");
    b->f32 = precision == PQ_PREC_MIXED ? 1 : 0;
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
        d.precision = precision;
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
    // The tensor-core DST's buffers: node rows per eligible member, one
    // split table (and TMA descriptor) per transform length.
    const bool tensor_possible = b->f32 && dst_algo != PQ_DST_BUTTERFLY;
    if (tensor_possible) {
        std::map<int, size_t> table_off;
        size_t off = 0;
        b->gbuf_off.assign(n, 0);
        for (int k = 0; k < n; ++k) {
            const pq_ctx* c = b->mem[k];
            if (c->L < 2 || !dst_mma_supported(c->hm[0].N)) continue;
            off = align256(off);
            if (off == 0) off = 256;  // 0 marks "none"
            b->gbuf_off[k] = off;
            off += (size_t)c->L * c->hm[0].lstride * sizeof(float);
            if (!table_off.count(c->hm[0].N)) table_off[c->hm[0].N] = 0;
        }
        for (auto& kv : table_off) {
            off = align256(off);
            kv.second = off;
            off += dst_mma_table_bytes(kv.first);
        }
        if (off) {
            if (cudaMalloc(&b->mma_mem, off) != cudaSuccess) {
                cudaGetLastError();
                return bfail(b, PQ_ERR_NOMEM, "allocation of the tensor-core DST buffers failed");
            }
            b->bytes += off;
            char* base = static_cast<char*>(b->mma_mem);
            BK(cudaMemsetAsync(base, 0, off, b->stream));
            for (auto& kv : table_off) {
                std::vector<unsigned short> t;
                dst_mma_table(kv.first, t);
                BK(cudaMemcpyAsync(base + kv.second, t.data(), t.size() * sizeof(unsigned short),
                                   cudaMemcpyHostToDevice, b->stream));
                CUtensorMap m;
                if (dst_mma_tensor_map(&m, base + kv.second, kv.first) != 0)
                    return bfail(b, PQ_ERR_CUDA, "cuTensorMapEncodeTiled failed");
                b->maps[kv.first] = m;
            }
            for (int k = 0; k < n; ++k)
                if (b->gbuf_off[k])
                    for (int p = 0; p < 2; ++p) b->mem[k]->hm[p].gbuf = base + b->gbuf_off[k];
        }
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
    // Row-DST algorithm per DST class: the tensor-core DST where it applies
    // (mixed form, two or more layers, ii >= 65), fixed or timed.
    b->tensor.assign(b->dst_cls.size(), 0);
    for (size_t q = 0; q < b->dst_cls.size(); ++q) {
        pq_batch::Class& cl = b->dst_cls[q];
        const int k0 = cl.idx[0];
        const bool eligible = tensor_possible && !b->gbuf_off.empty() && b->gbuf_off[k0] != 0;
        if (!eligible) continue;
        if (dst_algo == PQ_DST_TENSOR) {
            cl.ls.gemm_bc = 1;
            continue;
        }
        // the autotuner: forward + inverse launches of this class, both ways
        // (on the zeroed fields: nothing has been set yet)
        cudaEvent_t e0, e1;
        BK(cudaEventCreate(&e0));
        BK(cudaEventCreate(&e1));
        float ms[2] = {0.f, 0.f};
        for (int round = 0; round < 2; ++round)
            for (int v = 0; v < 2; ++v) {
                cl.ls.gemm_bc = v;
                for (int w = 0; w < 2; ++w) {
                    BK(class_dst(b, q, 0, b->stream));
                    BK(class_dst(b, q, 1, b->stream));
                }
                BK(cudaEventRecord(e0, b->stream));
                for (int r = 0; r < 5; ++r) {
                    BK(class_dst(b, q, 0, b->stream));
                    BK(class_dst(b, q, 1, b->stream));
                }
                BK(cudaEventRecord(e1, b->stream));
                BK(cudaEventSynchronize(e1));
                BK(cudaEventElapsedTime(&ms[v], e0, e1));
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cl.ls.gemm_bc = ms[1] < ms[0] ? 1 : 0;
    }
    for (size_t q = 0; q < b->dst_cls.size(); ++q) b->tensor[q] = b->dst_cls[q].ls.gemm_bc;
    // Fields back to zero after the timing (the members start from nothing).
    for (pq_ctx* c : b->mem) {
        BK(cudaMemsetAsync(c->hm[0].helm_io, 0, c->field_bytes, b->stream));
    }
    BK(cudaStreamSynchronize(b->stream));
    for (pq_ctx* c : b->mem) {
        const int rc = check_status(c);
        if (rc) return bfail(b, rc, c->err);
    }
    return PQ_OK;
}

int pq_batch_member_dst_algo(const pq_batch* b, int k) {
    if (!b || k < 0 || k >= (int)b->mem.size()) return -1;
    for (size_t q = 0; q < b->dst_cls.size(); ++q)
        for (int m : b->dst_cls[q].idx)
            if (m == k) return b->tensor.empty() || !b->tensor[q] ? PQ_DST_BUTTERFLY : PQ_DST_TENSOR;
    return -1;
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
    if (!b) return 0;
    int n = (int)(2 * b->dst_cls.size() + b->tri_cls.size());
    for (size_t q = 0; q < b->dst_cls.size(); ++q)
        if (!b->tensor.empty() && b->tensor[q]) n += 2 * (int)b->dst_cls[q].idx.size();
    return n;
}

}  // extern "C"
