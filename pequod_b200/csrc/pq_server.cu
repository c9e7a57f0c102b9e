// pq_server.cu -- serving many model runs on one GPU, continuously batched.
//
// A run is a CABARET time integration (fixed dt) from an initial PV field
// for a number of steps.  Runs are queued on submission and admitted while
// the HBM budget allows; admission initialises the run (pq_init_perturb) and
// takes its first step on its own (the predictor of the first step is not
// yet fused).  From then on every scheduling round advances all active runs
// by the same number of steps with merged launches: the runs are grouped by
// shape (ii, jj, L, precision), and each group's four kernels of a step are
// single launches over all its members, each member with the descriptor of
// its own step parity, on the group's own stream.  Runs leave the batch when
// they finish and new ones join at the next round -- continuous batching.
// Finished runs' contexts stay in a pool keyed by their configuration and
// are reused by later runs of the same configuration (no device allocation
// in steady state); idle pooled contexts are freed when the budget needs
// the room.  A run's result does not depend on what it was batched with:
// the kernels compute every member independently.
//
// Faults stay with the run that raised them.  The reference aborts the
// whole program on a NaN psiC or energy (qg3p_aux.F90:504-510,
// qg3p_diagnostics.F90:858-861); here the device status word of every
// active run is read back after each round, and a run whose word reports a
// NaN -- or whose admission fails (an invalid description, a failed
// allocation, a NaN already in its initial inversion) -- is marked failed
// with that error and evicted: its context is destroyed (not pooled) and
// the other runs carry on untouched.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "pq_ctx.h"

using namespace pq;

struct pq_server {
    int device = 0;
    size_t budget = 0;
    size_t held = 0;  // device bytes of live contexts (active + pooled)
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;
    cudaEvent_t round_done = nullptr;
    bool round_pending = false;
    std::chrono::steady_clock::time_point t0;
    struct Run {
        long id = 0;
        pq_model_desc desc{};
        std::vector<double> wind, ic, psi;
        int nsteps = 0, done = 0;
        int state = 0;  // 0 queued, 1 running, 2 finished, 3 failed
        int error = 0;  // PQ_ERR_* of a failed run
        std::string msg;
        pq_ctx* c = nullptr;
        size_t bytes = 0;
        double t_submit = 0, t_start = 0, t_done = 0;
        std::string key;
    };
    std::map<long, Run> runs;
    std::deque<long> queue;
    std::vector<long> active;
    long next_id = 1;
    std::multimap<std::string, pq_ctx*> pool;
    std::map<std::string, size_t> known_bytes;  // measured context size per configuration
    Member* d_desc = nullptr;
    size_t desc_cap = 0;
    int* d_pref = nullptr;
    size_t pref_cap = 0;
    int sm_count = 0;
    long launches = 0;
    std::string err;
    // Status words of the active runs, copied after each round (pinned).
    int* h_status = nullptr;
    size_t status_cap = 0;
    std::vector<long> status_ids;
};

namespace {

int sfail(pq_server* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    return code;
}

#define SK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return sfail(s, PQ_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

double now(const pq_server* s) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

// Configuration key: the description bytes (without the wind pointer) and a
// hash of the wind field.
std::string config_key(const pq_model_desc& d, const std::vector<double>& wind) {
    pq_model_desc k = d;
    k.force_wind = nullptr;
    std::string key(reinterpret_cast<const char*>(&k), sizeof(k));
    unsigned long long h = 1469598103934665603ull;
    const unsigned char* p = reinterpret_cast<const unsigned char*>(wind.data());
    for (size_t i = 0; i < wind.size() * sizeof(double); ++i) h = (h ^ p[i]) * 1099511628211ull;
    key.append(reinterpret_cast<const char*>(&h), sizeof(h));
    return key;
}

// Device bytes a context of this description takes before one exists: its
// 28 fields, the uncompressed pivot tables as a bound, and 1 MB for the rest.
size_t estimate_bytes(const pq_model_desc& d) {
    const size_t pitch = (size_t)((d.ii + 31) & ~31);
    const size_t field = align256(pitch * d.jj * d.layers * sizeof(double));
    return 28 * field + (size_t)d.layers * (d.ii - 2) * d.jj * sizeof(double) + ((size_t)1 << 20);
}

void release_ctx(pq_server* s, pq_server::Run& r) {
    s->pool.emplace(r.key, r.c);
    r.c = nullptr;
}

// Free idle pooled contexts until `need` more bytes fit the budget.
void evict(pq_server* s, size_t need) {
    for (auto it = s->pool.begin(); it != s->pool.end() && s->held + need > s->budget;) {
        s->held -= it->second->arena_bytes;
        pq_destroy(it->second);
        it = s->pool.erase(it);
    }
}

// Mark a run failed with `code` and drop its context (destroyed, not
// pooled: its state is not trusted).  The caller removes it from the active
// list or the queue.
void fail_run(pq_server* s, pq_server::Run& r, int code, const std::string& msg) {
    r.state = 3;
    r.error = code;
    r.msg = "run " + std::to_string(r.id) + ": " + msg;
    r.t_done = now(s);
    r.ic.clear();
    r.ic.shrink_to_fit();
    if (r.c) {
        s->held -= std::min(s->held, r.c->arena_bytes);
        pq_destroy(r.c);
        r.c = nullptr;
    }
}

// Evict the active runs whose device status reported a NaN in the round
// just completed (the status words were copied at its end).
void evict_faulted(pq_server* s) {
    std::vector<long> bad;
    for (size_t k = 0; k < s->status_ids.size(); ++k)
        if (s->h_status[k] & (ST_NAN_PSIC | ST_NAN_ENERGY)) bad.push_back(s->status_ids[k]);
    s->status_ids.clear();
    if (bad.empty()) return;
    std::vector<long> keep;
    for (long id : s->active)
        if (std::find(bad.begin(), bad.end(), id) == bad.end()) keep.push_back(id);
    for (long id : bad) {
        pq_server::Run& r = s->runs[id];
        fail_run(s, r, PQ_ERR_NAN, "NaN psiC or energy after " + std::to_string(r.done) +
                                       " steps (the reference aborts here)");
    }
    s->active.swap(keep);
}

int retire(pq_server* s) {
    std::vector<long> keep;
    for (long id : s->active) {
        pq_server::Run& r = s->runs[id];
        if (r.done < r.nsteps) {
            keep.push_back(id);
            continue;
        }
        r.psi.resize((size_t)r.desc.ii * r.desc.jj * r.desc.layers);
        pq_ctx* c = r.c;
        int rc = copy_out(c, r.psi.data(), c->hm[0].psi, PQ_PTR_HOST);
        if (!rc) rc = check_status(c);  // synchronises the stream, reports NaNs
        if (rc == PQ_ERR_CUDA) return sfail(s, rc, "run " + std::to_string(id) + ": " + c->err);
        if (rc) {
            r.psi.clear();
            fail_run(s, r, rc, c->err);
            continue;
        }
        r.t_done = now(s);
        r.state = 2;
        release_ctx(s, r);
    }
    s->active.swap(keep);
    return PQ_OK;
}

int admit(pq_server* s) {
    while (!s->queue.empty()) {
        pq_server::Run& r = s->runs[s->queue.front()];
        pq_ctx* c = nullptr;
        auto it = s->pool.find(r.key);
        if (it != s->pool.end()) {
            c = it->second;
            s->pool.erase(it);
        } else {
            auto kb = s->known_bytes.find(r.key);
            const size_t need = kb != s->known_bytes.end() ? kb->second : r.bytes;
            if (s->held + need > s->budget) evict(s, need);
            if (s->held + need > s->budget) break;  // wait for running work to finish
            pq_model_desc d = r.desc;
            d.force_wind = r.wind.empty() ? nullptr : r.wind.data();
            const int rc = create_ctx(&c, &d, s->device, false, s->stream);
            if (rc) {
                // This run alone fails (an invalid description or a failed
                // allocation); the queue moves on.
                const std::string msg = c ? c->err : std::string("context creation failed");
                if (c) pq_destroy(c);
                cudaGetLastError();
                fail_run(s, r, rc, "admission: " + msg);
                s->queue.pop_front();
                continue;
            }
            s->held += c->arena_bytes;
            s->known_bytes[r.key] = c->arena_bytes;
        }
        r.c = c;
        int rc = pq_init_perturb(c, r.ic.data(), PQ_PTR_HOST);
        if (!rc && r.nsteps > 0) {
            // The first step on its own: the following ones reuse the
            // predictor the fused CABARET kernel computes.
            rc = run_step(c, c->cur);
            c->cur ^= 1;
            r.done = 1;
            s->launches += 4;
        }
        if (rc == PQ_ERR_CUDA) return sfail(s, rc, "initialising run " + std::to_string(r.id) + ": " + c->err);
        if (rc) {
            fail_run(s, r, rc, "initialisation: " + c->err);
            s->queue.pop_front();
            continue;
        }
        r.state = 1;
        r.t_start = now(s);
        r.ic.clear();
        r.ic.shrink_to_fit();
        s->active.push_back(r.id);
        s->queue.pop_front();
    }
    return PQ_OK;
}

// One scheduling round, one launch per kernel per shape group and step.
// The group with the most work per step (cell-layers over its members, with
// a floor for the latency-bound small grids) advances up to max_steps steps;
// cheaper groups advance proportionally more (up to 64 max_steps), so that
// every group's share of the round takes about the same time on its own
// stream and a small run does not wait for the big grids' pace -- each group
// stops at its nearest member's end.
int round_steps(pq_server* s, int max_steps) {
    if (s->active.empty()) return PQ_OK;
    std::map<std::vector<int>, std::vector<long>> groups;
    for (long id : s->active) {
        const pq_model_desc& d = s->runs[id].desc;
        groups[{d.ii, d.jj, d.layers, d.precision}].push_back(id);
    }
    std::vector<int> Kg;
    {
        std::vector<double> work;
        double wmax = 0.0;
        for (auto& kv : groups) {
            const pq_model_desc& d = s->runs[kv.second[0]].desc;
            const double w = std::max((double)d.ii * d.jj * d.layers * kv.second.size(), 5.0e5);
            work.push_back(w);
            wmax = std::max(wmax, w);
        }
        size_t q = 0;
        for (auto& kv : groups) {
            int rem = max_steps * 64;
            for (long id : kv.second) rem = std::min(rem, s->runs[id].nsteps - s->runs[id].done);
            const double k = (double)max_steps * wmax / work[q++];
            Kg.push_back(std::max(0, std::min(rem, (int)std::min(k, (double)max_steps * 64))));
        }
    }
    // Host staging: for each group two descriptor arrays (the members at
    // their current parity and at the next), then its prefix arrays.
    std::vector<Member> hd;
    std::vector<int> hp;
    struct G {
        size_t d0, d1, pfwd, pinv, ptri, pcab;
        LaunchSet ls;
        int f32;
    };
    std::vector<G> gs;
    for (auto& kv : groups) {
        G g;
        const std::vector<long>& ids = kv.second;
        const pq_ctx* c0 = s->runs[ids[0]].c;
        g.d0 = hd.size();
        for (long id : ids) hd.push_back(s->runs[id].c->hm[s->runs[id].c->cur]);
        g.d1 = hd.size();
        for (long id : ids) hd.push_back(s->runs[id].c->hm[s->runs[id].c->cur ^ 1]);
        const LaunchSet& l0 = c0->ls[0];
        auto prefix = [&](int per) {
            const size_t off = hp.size();
            for (size_t k = 0; k < ids.size(); ++k) hp.push_back((int)k * per);
            return off;
        };
        g.pfwd = prefix(l0.ctas_dst[0]);
        g.pinv = prefix(l0.ctas_dst[1]);
        g.ptri = prefix(l0.ctas_tri);
        g.pcab = prefix(l0.ctas_cab);
        g.ls = l0;
        g.ls.one = nullptr;  // the group's descriptors come from the device array
        const int n = (int)ids.size();
        g.ls.nmem = n;
        g.ls.ctas_dst[0] = n * l0.ctas_dst[0];
        g.ls.ctas_dst[1] = n * l0.ctas_dst[1];
        g.ls.ctas_tri = n * l0.ctas_tri;
        g.ls.ctas_cab = n * l0.ctas_cab;
        g.f32 = c0->mixed ? 1 : 0;
        gs.push_back(g);
    }
    if (hd.size() > s->desc_cap) {
        if (s->d_desc) cudaFree(s->d_desc);
        s->desc_cap = hd.size() * 2;
        SK(cudaMalloc(&s->d_desc, s->desc_cap * sizeof(Member)));
    }
    if (hp.size() > s->pref_cap) {
        if (s->d_pref) cudaFree(s->d_pref);
        s->pref_cap = hp.size() * 2;
        SK(cudaMalloc(&s->d_pref, s->pref_cap * sizeof(int)));
    }
    SK(cudaMemcpyAsync(s->d_desc, hd.data(), hd.size() * sizeof(Member), cudaMemcpyHostToDevice, s->stream));
    SK(cudaMemcpyAsync(s->d_pref, hp.data(), hp.size() * sizeof(int), cudaMemcpyHostToDevice, s->stream));
    // Fork: every group stream waits for the admissions and the uploads.
    const int S = (int)s->side.size();
    SK(cudaEventRecord(s->ev[0], s->stream));
    for (int q = 0; q < S; ++q) SK(cudaStreamWaitEvent(s->side[q], s->ev[0], 0));
    for (size_t q = 0; q < gs.size(); ++q) {
        G& g = gs[q];
        const int K = Kg[q];
        cudaStream_t st = s->side[q % S];
        g.ls.prefix_dst[0] = s->d_pref + g.pfwd;
        g.ls.prefix_dst[1] = s->d_pref + g.pinv;
        g.ls.prefix_tri = s->d_pref + g.ptri;
        g.ls.prefix_cab = s->d_pref + g.pcab;
        for (int t = 0; t < K; ++t) {
            g.ls.members = s->d_desc + ((t & 1) ? g.d1 : g.d0);
            cudaError_t e = launch_dst_forward(g.ls, PRO_MODAL, g.f32, st);
            if (e == cudaSuccess) e = launch_tridiag(g.ls, 1, g.f32, st);
            if (e == cudaSuccess) e = launch_dst_inverse(g.ls, EPI_PV, g.f32, st);
            if (e == cudaSuccess) e = launch_cabaret_fused(g.ls, 1, g.f32, st);
            if (e != cudaSuccess) return sfail(s, PQ_ERR_CUDA, std::string("group step: ") + cudaGetErrorString(e));
        }
        s->launches += 4L * K;
    }
    for (int q = 0; q < S; ++q) {
        SK(cudaEventRecord(s->ev[1 + q], s->side[q]));
        SK(cudaStreamWaitEvent(s->stream, s->ev[1 + q], 0));
    }
    // Every active run's status word, read at the next poll.
    if (s->active.size() > s->status_cap) {
        if (s->h_status) cudaFreeHost(s->h_status);
        s->h_status = nullptr;
        s->status_cap = s->active.size() * 2;
        SK(cudaMallocHost(&s->h_status, s->status_cap * sizeof(int)));
    }
    s->status_ids = s->active;
    for (size_t k = 0; k < s->active.size(); ++k)
        SK(cudaMemcpyAsync(s->h_status + k, s->runs[s->active[k]].c->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                           s->stream));
    SK(cudaEventRecord(s->round_done, s->stream));
    s->round_pending = true;
    size_t q = 0;
    for (auto& kv : groups) {
        const int K = Kg[q++];
        if (K <= 0) continue;
        for (long id : kv.second) {
            pq_server::Run& r = s->runs[id];
            pq_ctx* c = r.c;
            c->zpar = c->cur ^ ((K - 1) & 1);
            c->cur ^= (K & 1);
            c->pred_ready = true;
            r.done += K;
        }
    }
    return PQ_OK;
}

}  // namespace

extern "C" {

int pq_server_create(pq_server** out, size_t hbm_budget_bytes, int device) {
    if (!out) return PQ_ERR_ARG;
    pq_server* s = new pq_server;
    *out = s;
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->t0 = std::chrono::steady_clock::now();
    SK(cudaSetDevice(device));
    SK(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device));
    SK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->side.resize(8);
    for (auto& st : s->side) SK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    s->ev.resize(1 + s->side.size());
    for (auto& e : s->ev) SK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SK(cudaEventCreateWithFlags(&s->round_done, cudaEventDisableTiming));
    return PQ_OK;
}

void pq_server_destroy(pq_server* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& kv : s->runs)
        if (kv.second.c) pq_destroy(kv.second.c);
    for (auto& kv : s->pool) pq_destroy(kv.second);
    if (s->d_desc) cudaFree(s->d_desc);
    if (s->d_pref) cudaFree(s->d_pref);
    if (s->h_status) cudaFreeHost(s->h_status);
    for (auto& st : s->side) cudaStreamDestroy(st);
    for (auto& e : s->ev) cudaEventDestroy(e);
    if (s->round_done) cudaEventDestroy(s->round_done);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

const char* pq_server_last_error(const pq_server* s) { return s ? s->err.c_str() : "null server"; }
size_t pq_server_device_bytes(const pq_server* s) { return s ? s->held : 0; }
double pq_server_clock(const pq_server* s) { return s ? now(s) : 0.0; }
long pq_server_launches(const pq_server* s) { return s ? s->launches : 0; }

int pq_server_submit(pq_server* s, const pq_model_desc* d, const double* zeta_ic, int nsteps, long* id) {
    if (!s || !d || !zeta_ic || nsteps < 0 || !id) return PQ_ERR_ARG;
    if (d->scheme != PQ_SCHEME_CABARET || d->adapt_dt || d->periodic_j)
        return sfail(s, PQ_ERR_UNSUPPORTED, "the server runs closed-basin CABARET runs with a fixed dt");
    pq_server::Run r;
    r.id = s->next_id++;
    r.desc = *d;
    r.nsteps = nsteps;
    r.bytes = estimate_bytes(*d);
    if (r.bytes > s->budget) return sfail(s, PQ_ERR_BUDGET, "run larger than the HBM budget");
    if (d->force_wind) r.wind.assign(d->force_wind, d->force_wind + (size_t)d->ii * d->jj);
    r.desc.force_wind = nullptr;
    r.ic.assign(zeta_ic, zeta_ic + (size_t)d->ii * d->jj * d->layers);
    r.key = config_key(r.desc, r.wind);
    r.t_submit = now(s);
    *id = r.id;
    s->queue.push_back(r.id);
    s->runs.emplace(r.id, std::move(r));
    return PQ_OK;
}

int pq_server_poll(pq_server* s, int max_steps, int* active, int* queued) {
    if (!s || max_steps < 1) return PQ_ERR_ARG;
    SK(cudaSetDevice(s->device));
    if (s->round_pending) {
        SK(cudaEventSynchronize(s->round_done));
        s->round_pending = false;
        evict_faulted(s);
    }
    int rc = retire(s);
    if (!rc) rc = admit(s);
    if (!rc) rc = round_steps(s, max_steps);
    if (active) *active = (int)s->active.size();
    if (queued) *queued = (int)s->queue.size();
    return rc;
}

int pq_server_status(pq_server* s, long id) {
    if (!s) return -1;
    auto it = s->runs.find(id);
    return it == s->runs.end() ? -1 : it->second.state;
}

int pq_server_collect(pq_server* s, long id, double* psi, double* t3) {
    if (!s) return PQ_ERR_ARG;
    auto it = s->runs.find(id);
    if (it == s->runs.end()) return sfail(s, PQ_ERR_NOTFOUND, "unknown run id");
    if (it->second.state != 2 && it->second.state != 3) return sfail(s, PQ_ERR_STATE, "run not finished");
    if (t3) {
        t3[0] = it->second.t_submit;
        t3[1] = it->second.t_start;
        t3[2] = it->second.t_done;
    }
    if (it->second.state == 3) {
        // A failed run: its error code and message, no psi.
        const int code = it->second.error;
        s->err = it->second.msg;
        s->runs.erase(it);
        return code;
    }
    if (psi) std::memcpy(psi, it->second.psi.data(), it->second.psi.size() * sizeof(double));
    s->runs.erase(it);
    return PQ_OK;
}

}  // extern "C"
