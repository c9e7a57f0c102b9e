// pq_checkpoint.cu -- checkpoint dump and pickup in the reference's file
// format (host code; one-time set-up around the time loop, not on its path).
//
// Files are Fortran unformatted stream records (qg3p_io.F90:574-651 read,
// :653-760 write): a 4-byte byte count, the REAL(8) data column-major, the
// byte count again.
//   _s.d       model_time_day, total_time_day, L x psi%sdata(:, :, l),
//              L x zeta%sdata(:, :, l); the leapfrog scheme writes both time
//              levels in one record per layer (qg3.F90:836-856).
//   _s_supp.d  (CABARET, qg3.F90:858-881) model_time_day, total_time_day, dt,
//              L x ui%data(fa_i_min+1:fa_i_max, fa_j_min+1:fa_j_max-1, l),
//              L x uj%data(fa_i_min+1:fa_i_max-1, fa_j_min+1:fa_j_max, l),
//              L x zeta_fi, L x zeta_fj (the same ranges),
//              L x res(:ii, :jj, l), L x res_beta(:ii, :jj, l).
// The reference writes its checkpoint inside a step, after the flux and
// before the corrector (qg3.F90:807-934 precede the exit point and the
// corrector :940-956): psi, ui, uj, zeta_fi, zeta_fj and res_beta of the
// step, zeta before the corrector, res of the step before, and model_time
// half a step short.  The device stops after whole steps, so the dump
// rebuilds that state: zeta - dt/2 res on the interior nodes, the previous
// step's res (kept by the step's res ping-pong), model_time - dt/2.  A pickup
// then finishes the step with the corrector and carries on exactly as the
// uninterrupted run.
// The state moves through pq_get_field / pq_set_field in the reference's
// array layouts, so the device layout (pitched, FP32 state in the mixed form)
// never shows here.  Reference-layout arrays are indexed below with the
// reference's own 1-based indices: a full data array (ii+2, jj+2) has its
// boundary nodes at 2 and ii+1, a FLUX_II array (ii+3, jj+2) its boundary
// faces at 2 and ii+2.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pequod_b200.h"
#include "pq_common.cuh"
#include "pq_ctx.h"

using namespace pq;

namespace {

constexpr double kDayS = 86400.0;  // day_s, qg3p_params.F90:104

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

bool put_record(FILE* f, const double* p, size_t n) {
    const int32_t nb = (int32_t)(n * sizeof(double));
    return std::fwrite(&nb, 4, 1, f) == 1 && std::fwrite(p, sizeof(double), n, f) == n &&
           std::fwrite(&nb, 4, 1, f) == 1;
}

// read_unformatted: the record's byte count must equal n REAL(8) values.
bool get_record(FILE* f, double* p, size_t n) {
    int32_t a = 0, b = 0;
    if (std::fread(&a, 4, 1, f) != 1 || (size_t)a != n * sizeof(double)) return false;
    if (std::fread(p, sizeof(double), n, f) != n) return false;
    return std::fread(&b, 4, 1, f) == 1 && b == a;
}

// fne (test_tools): |a - b| above 10 * max(spacing(a), epsilon).
bool fne(double a, double b) {
    const double eps = 2.220446049250313e-16;
    const double sp = std::nextafter(std::fabs(a), INFINITY) - std::fabs(a);
    return std::fabs(a - b) > 10.0 * std::fmax(sp, eps);
}

// A reference-layout array (n1, n2, L) with the reference's 1-based indices.
struct Ref {
    std::vector<double> v;
    int n1 = 0, n2 = 0;
    Ref(int a, int b, int L) : v((size_t)a * b * L, 0.0), n1(a), n2(b) {}
    double& operator()(int i, int j, int l) {
        return v[(size_t)(i - 1) + (size_t)n1 * ((size_t)(j - 1) + (size_t)n2 * (size_t)(l - 1))];
    }
};

struct Range {
    int i0, i1, j0, j1;
    size_t count() const { return (size_t)(i1 - i0 + 1) * (j1 - j0 + 1); }
};

// The owned interior rows f_j_min..f_j_max of one process
// (qg3p_base.F90:893-912): a closed basin has no j neighbour, rows 3..jj;
// a channel is its own j neighbour, rows 2..jj+1 (every row, the halo rows
// 1 and jj+2 copies of rows jj+1 and 2).  fa_j_min = lo - 1, fa_j_max =
// hi + 1; in i there is never a neighbour (f_i 3..ii, fa_i 2..ii+1).
struct Rows {
    int lo, hi;
};
Rows rows_of(const pq_ctx* c) { return c->periodic ? Rows{2, c->jj + 1} : Rows{3, c->jj}; }

// The saved face ranges: FLUX_II faces i in [fa_i_min+1, fa_i_max], rows
// [fa_j_min+1, fa_j_max-1]; FLUX_JJ columns [fa_i_min+1, fa_i_max-1], faces
// [fa_j_min+1, fa_j_max] (qg3.F90:864-875).
Range fi_range(int ii, Rows r) { return {3, ii + 1, r.lo, r.hi}; }
Range fj_range(int ii, Rows r) { return {3, ii, r.lo, r.hi + 1}; }

void pack(Ref& a, const Range& r, int l, std::vector<double>& out) {
    out.clear();
    for (int j = r.j0; j <= r.j1; ++j)
        for (int i = r.i0; i <= r.i1; ++i) out.push_back(a(i, j, l));
}

void unpack(Ref& a, const Range& r, int l, const std::vector<double>& in) {
    size_t k = 0;
    for (int j = r.j0; j <= r.j1; ++j)
        for (int i = r.i0; i <= r.i1; ++i) a(i, j, l) = in[k++];
}

bool supported(pq_ctx* c) {
    if (c->helm_only) return !fail(c, PQ_ERR_UNSUPPORTED, "checkpoint of a Helmholtz-only context");
    return true;
}

// rel_from_psi (qg3p_aux.F90:579-603) with apply_rel_bc (:779-915) for one
// process: the five-point Laplacian on the interior nodes f_i x f_j, then the
// i boundaries and the j boundaries (which own the corners).  A channel is
// its own j neighbour: psi's halo rows are filled first (update(psi),
// qg3.F90:355), every row is interior and there are no j boundaries.
void rel_from_psi(const pq_model_desc& d, Ref& psi, Ref& rel) {
    const int ii = d.ii, jj = d.jj, L = d.layers;
    const bool per = d.periodic_j != 0;
    if (per)
        for (int l = 1; l <= L; ++l)
            for (int i = 2; i <= ii + 1; ++i) {
                psi(i, 1, l) = psi(i, jj + 1, l);
                psi(i, jj + 2, l) = psi(i, 2, l);
            }
    for (int l = 1; l <= L; ++l)
        for (int j = per ? 2 : 3; j <= (per ? jj + 1 : jj); ++j)
            for (int i = 3; i <= ii; ++i)
                rel(i, j, l) = -4.0 * psi(i, j, l) + psi(i - 1, j, l) + psi(i, j + 1, l) + psi(i + 1, j, l) +
                               psi(i, j - 1, l);
    // Boundary node (i, j) with its first and second inward neighbours.
    auto bc = [&](int i, int j, int di, int dj, int l) {
        const double p0 = psi(i, j, l), p1 = psi(i + di, j + dj, l), p2 = psi(i + 2 * di, j + 2 * dj, l);
        if (d.bc_type == PQ_BC_PARTIAL_SLIP) {
            const double cff = d.alpha / (d.alpha + 3.0);
            return cff * (-3.5 * p0 + 4.0 * p1 - 0.5 * p2);
        }
        if (d.bc_type == PQ_BC_NO_SLIP) return 2.0 * (p1 - p0);
        return 0.0;
    };
    for (int l = 1; l <= L; ++l) {
        for (int j = 2; j <= jj + 1; ++j) {
            rel(2, j, l) = bc(2, j, 1, 0, l);
            rel(ii + 1, j, l) = bc(ii + 1, j, -1, 0, l);
        }
        if (!per)
            for (int i = 2; i <= ii + 1; ++i) {
                rel(i, 2, l) = bc(i, 2, 0, 1, l);
                rel(i, jj + 1, l) = bc(i, jj + 1, 0, -1, l);
            }
    }
}

int get_ref(pq_ctx* c, int field, Ref& a) { return pq_get_field(c, field, a.v.data()); }
int set_ref(pq_ctx* c, int field, Ref& a) { return pq_set_field(c, field, a.v.data()); }

}  // namespace

extern "C" {

int pq_write_checkpoint(pq_ctx* c, const char* s_path, const char* supp_path, double t_scale,
                        double start_time_day) {
    if (!c || !s_path) return PQ_ERR_ARG;
    if (!supported(c)) return PQ_ERR_UNSUPPORTED;
    if (!c->initialized) return fail(c, PQ_ERR_STATE, "pq_write_checkpoint before the state is initialised");
    const int ii = c->ii, jj = c->jj, L = c->L;
    const bool lf = c->leapfrog;
    if (lf && c->cur != 0)
        return fail(c, PQ_ERR_STATE, "the leapfrog state is dumped after the second sub-step of a pair (qg3.F90:823)");
    double sc4[4];
    int rc = pq_get_scalars(c, sc4);
    if (rc) return rc;
    const double dt = sc4[0];  // the dt the last step ran with
    // qg3.F90:661; CABARET dumps half a step before the step's end.
    const double model_time_day = (lf ? sc4[3] : sc4[3] - 0.5 * dt) * t_scale / kDayS;
    const double total_time_day = start_time_day + model_time_day;
    Ref psi(ii + 2, jj + 2, L), zeta(ii + 2, jj + 2, L), psi2(ii + 2, jj + 2, L), zeta2(ii + 2, jj + 2, L);
    if ((rc = get_ref(c, PQ_F_PSI, psi)) || (rc = get_ref(c, PQ_F_ZETA, zeta))) return rc;
    if (lf && ((rc = get_ref(c, PQ_F_PSI2, psi2)) || (rc = get_ref(c, PQ_F_ZETA2, zeta2)))) return rc;
    Ref res(ii, jj, L), res_prev(ii, jj, L);
    if (!lf) {
        // zeta before the corrector (cabaret_corrector, qg3p_aux.F90:1630-1638,
        // touches interior nodes only) and the res the reference still holds.
        if ((rc = get_ref(c, PQ_F_RES, res))) return rc;
        if ((rc = copy_out_state(c, res_prev.v.data(), c->hm[c->cur].res_out, PQ_PTR_HOST))) return rc;
        CK(cudaStreamSynchronize(c->stream));
        const Rows rw = rows_of(c);
        for (int l = 1; l <= L; ++l)
            for (int j = rw.lo; j <= rw.hi; ++j)
                for (int i = 3; i <= ii; ++i) zeta(i, j, l) = zeta(i, j, l) - 0.5 * dt * res(i - 1, j - 1, l);
    }
    {
        File out;
        out.f = std::fopen(s_path, "wb");
        if (!out.f) return fail(c, PQ_ERR_ARG, std::string("Failed to open output file ") + s_path);
        bool ok = put_record(out.f, &model_time_day, 1) && put_record(out.f, &total_time_day, 1);
        const Range sd{2, ii + 1, 2, jj + 1};  // sdata
        std::vector<double> rec, rec2;
        for (Ref* f : {&psi, &zeta})
            for (int l = 1; l <= L && ok; ++l) {
                pack(*f, sd, l, rec);
                if (lf) {
                    pack(f == &psi ? psi2 : zeta2, sd, l, rec2);
                    rec.insert(rec.end(), rec2.begin(), rec2.end());
                }
                ok = put_record(out.f, rec.data(), rec.size());
            }
        if (!ok || std::fflush(out.f) != 0) return fail(c, PQ_ERR_ARG, std::string("write failed: ") + s_path);
    }
    if (lf || !supp_path) return PQ_OK;
    Ref ui(ii + 3, jj + 2, L), uj(ii + 2, jj + 3, L), zfi(ii + 3, jj + 2, L), zfj(ii + 2, jj + 3, L);
    Ref rb(ii, jj, L);
    if ((rc = get_ref(c, PQ_F_UI, ui)) || (rc = get_ref(c, PQ_F_UJ, uj)) || (rc = get_ref(c, PQ_F_ZETA_FI, zfi)) ||
        (rc = get_ref(c, PQ_F_ZETA_FJ, zfj)) || (rc = get_ref(c, PQ_F_RES_BETA, rb)))
        return rc;
    if (c->periodic) {
        // The device keeps j faces 2..jj+1; face jj+2 is face 2 of the next
        // period (update(uj, level_1), qg3.F90:795-803).
        for (int l = 1; l <= L; ++l)
            for (int i = 2; i <= ii + 1; ++i) {
                uj(i, jj + 2, l) = uj(i, 2, l);
                zfj(i, jj + 2, l) = zfj(i, 2, l);
            }
    }
    File out;
    out.f = std::fopen(supp_path, "wb");
    if (!out.f) return fail(c, PQ_ERR_ARG, std::string("Failed to open output file ") + supp_path);
    bool ok = put_record(out.f, &model_time_day, 1) && put_record(out.f, &total_time_day, 1) &&
              put_record(out.f, &dt, 1);
    const Range ri = fi_range(ii, rows_of(c)), rj = fj_range(ii, rows_of(c)), rs{1, ii, 1, jj};
    std::vector<double> rec;
    const std::pair<Ref*, Range> order[] = {{&ui, ri},  {&uj, rj},       {&zfi, ri},
                                            {&zfj, rj}, {&res_prev, rs}, {&rb, rs}};
    for (const auto& fr : order)
        for (int l = 1; l <= L && ok; ++l) {
            pack(*fr.first, fr.second, l, rec);
            ok = put_record(out.f, rec.data(), rec.size());
        }
    if (!ok || std::fflush(out.f) != 0) return fail(c, PQ_ERR_ARG, std::string("write failed: ") + supp_path);
    return PQ_OK;
}

int pq_read_checkpoint(pq_ctx* c, const char* s_path, const char* supp_path, double* total_time_day) {
    if (!c || !s_path) return PQ_ERR_ARG;
    if (!supported(c)) return PQ_ERR_UNSUPPORTED;
    const bool lf = c->leapfrog;
    if (!lf && !supp_path) return fail(c, PQ_ERR_ARG, "the CABARET pickup needs the _s_supp file");
    const int ii = c->ii, jj = c->jj, L = c->L;
    const pq_model_desc& d = c->desc;
    Ref psi(ii + 2, jj + 2, L), zeta(ii + 2, jj + 2, L), psi2(ii + 2, jj + 2, L), zeta2(ii + 2, jj + 2, L);
    double mtd = 0.0, ttd = 0.0;
    const Range sd{2, ii + 1, 2, jj + 1};
    {
        File in;
        in.f = std::fopen(s_path, "rb");
        if (!in.f) return fail(c, PQ_ERR_ARG, std::string("Failed to open input file ") + s_path);
        bool ok = get_record(in.f, &mtd, 1) && get_record(in.f, &ttd, 1);
        const size_t n = (size_t)ii * jj;
        std::vector<double> rec(n * (lf ? 2 : 1));
        for (Ref* f : {&psi, &zeta})
            for (int l = 1; l <= L && ok; ++l) {
                ok = get_record(in.f, rec.data(), rec.size());
                if (!ok) break;
                unpack(*f, sd, l, std::vector<double>(rec.begin(), rec.begin() + n));
                if (lf) unpack(f == &psi ? psi2 : zeta2, sd, l, std::vector<double>(rec.begin() + n, rec.end()));
            }
        if (!ok) return fail(c, PQ_ERR_ARG, std::string("unexpected record in ") + s_path);
    }
    if (lf) {
        // Leapfrog pickup (qg3.F90:341-363): rel from psi on both levels,
        // zeta_old = zeta, model_time = 0, no forward-Euler start (:461-497).
        Ref rel(ii + 2, jj + 2, L), rel2(ii + 2, jj + 2, L);
        rel_from_psi(d, psi, rel);
        rel_from_psi(d, psi2, rel2);
        Scalars sc;
        std::memset(&sc, 0, sizeof(sc));
        sc.dt = sc.dt_last = d.dt;
        sc.tweight_a = sc.tweight_u = sc.tweight_a_last = sc.tweight_u_last = 0.5;
        int rc = reset_prognostic(c, sc);
        if (rc) return rc;
        const std::pair<int, Ref*> sets[] = {{PQ_F_PSI, &psi},   {PQ_F_ZETA, &zeta},      {PQ_F_REL, &rel},
                                             {PQ_F_ZETA_OLD, &zeta}, {PQ_F_PSI2, &psi2},  {PQ_F_ZETA2, &zeta2},
                                             {PQ_F_REL2, &rel2},  {PQ_F_ZETA_OLD2, &zeta2}};
        for (const auto& s : sets)
            if ((rc = set_ref(c, s.first, *s.second))) return rc;
        if (total_time_day) *total_time_day = ttd;
        return PQ_OK;
    }
    Ref ui(ii + 3, jj + 2, L), uj(ii + 2, jj + 3, L), zfi(ii + 3, jj + 2, L), zfj(ii + 2, jj + 3, L);
    Ref res(ii, jj, L), rb(ii, jj, L);
    double dt = 0.0;
    {
        File in;
        in.f = std::fopen(supp_path, "rb");
        if (!in.f) return fail(c, PQ_ERR_ARG, std::string("Failed to open input file ") + supp_path);
        double mts = 0.0, tts = 0.0;
        bool ok = get_record(in.f, &mts, 1) && get_record(in.f, &tts, 1);
        if (ok && (fne(mts, mtd) || fne(tts, ttd)))
            return fail(c, PQ_ERR_ARG, "Input times do not match in CABARET checkpoint data");
        ok = ok && get_record(in.f, &dt, 1);
        const Range ri = fi_range(ii, rows_of(c)), rj = fj_range(ii, rows_of(c)), rs{1, ii, 1, jj};
        const std::pair<Ref*, Range> order[] = {{&ui, ri}, {&uj, rj}, {&zfi, ri}, {&zfj, rj}, {&res, rs}, {&rb, rs}};
        std::vector<double> rec;
        for (const auto& fr : order)
            for (int l = 1; l <= L && ok; ++l) {
                rec.resize(fr.second.count());
                ok = get_record(in.f, rec.data(), rec.size());
                if (ok) unpack(*fr.first, fr.second, l, rec);
            }
        if (!ok) return fail(c, PQ_ERR_ARG, std::string("unexpected record in ") + supp_path);
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, PQ_ERR_ARG, "checkpoint dt is not a positive number");
    // CABARET pickup (qg3.F90:316-340): face velocities of psi into
    // uimo / ujmo (cabaret_cell_boundaries_velocity, qg3p_aux.F90:1168-1231),
    // flux = u * zeta_f (cabaret_flux, :1547-1594), corrector half step
    // (cabaret_corrector, :1597-1642).
    // A channel first fills psi's halo rows (update(psi), qg3.F90:324).
    const Rows rw = rows_of(c);
    Ref pe(ii + 2, jj + 2, L), uimo(ii + 3, jj + 2, L), ujmo(ii + 2, jj + 3, L);
    Ref fli(ii + 3, jj + 2, L), flj(ii + 2, jj + 3, L);
    for (int l = 1; l <= L; ++l) {
        if (c->periodic)
            for (int i = 2; i <= ii + 1; ++i) {
                psi(i, 1, l) = psi(i, jj + 1, l);
                psi(i, jj + 2, l) = psi(i, 2, l);
            }
        for (int j = rw.lo; j <= rw.hi + 1; ++j)
            for (int i = 3; i <= ii + 1; ++i)
                pe(i, j, l) = 0.25 * (psi(i, j, l) + psi(i, j - 1, l) + psi(i - 1, j, l) + psi(i - 1, j - 1, l));
        for (int j = rw.lo; j <= rw.hi; ++j)
            for (int i = 3; i <= ii + 1; ++i) uimo(i, j, l) = -pe(i, j + 1, l) + pe(i, j, l);
        for (int j = rw.lo; j <= rw.hi + 1; ++j)
            for (int i = 3; i <= ii; ++i) ujmo(i, j, l) = pe(i + 1, j, l) - pe(i, j, l);
        for (int j = rw.lo; j <= rw.hi; ++j)
            for (int i = 2; i <= ii + 2; ++i) fli(i, j, l) = ui(i, j, l) * zfi(i, j, l);
        for (int j = rw.lo; j <= rw.hi + 1; ++j)
            for (int i = 3; i <= ii; ++i) flj(i, j, l) = uj(i, j, l) * zfj(i, j, l);
        for (int j = rw.lo; j <= rw.hi; ++j)
            for (int i = 3; i <= ii; ++i) {
                const double r = -(fli(i + 1, j, l) - fli(i, j, l) + flj(i, j + 1, l) - flj(i, j, l));
                res(i - 1, j - 1, l) = r;
                zeta(i, j, l) = zeta(i, j, l) + 0.5 * dt * r;
            }
    }
    // cabaret_cfl of the checkpoint's face velocities: the first step adapts
    // dt from it (cabaret_adapt_dt, qg3p_aux.F90:946-990), which the device
    // applies at the end of the step before; apply it here instead.
    double mu = 0.0;
    for (int l = 1; l <= L; ++l) {
        for (int j = rw.lo; j <= rw.hi; ++j)
            for (int i = 3; i <= ii + 1; ++i) mu = std::fmax(mu, std::fabs(ui(i, j, l)));
        for (int j = rw.lo; j <= rw.hi + 1; ++j)
            for (int i = 3; i <= ii; ++i) mu = std::fmax(mu, std::fabs(uj(i, j, l)));
    }
    Scalars sc;
    std::memset(&sc, 0, sizeof(sc));
    sc.dt = sc.dt_last = dt;
    sc.tweight_a = sc.tweight_u = sc.tweight_a_last = sc.tweight_u_last = 0.5;
    sc.model_time = dt / 2.0;  // qg3.F90:455
    sc.max_u = mu;
    sc.cfl = mu * dt;
    if (d.adapt_dt) {
        const double eps = 2.220446049250313e-16;
        const double sp = std::nextafter(std::fabs(mu), INFINITY) - std::fabs(mu);
        double ndt = dt;
        if (std::fabs(mu) > 10.0 * std::fmax(sp, eps)) ndt = std::fmin(std::fmin(d.target_cfl / mu, dt * d.max_dt_increase), d.max_dt);
        sc.dt = ndt;
        sc.tweight_a = 0.5 * ndt / dt;
        sc.tweight_u = ndt / (dt + ndt);
    }
    int rc = reset_prognostic(c, sc);
    if (rc) return rc;
    const std::pair<int, Ref*> sets[] = {{PQ_F_PSI, &psi},       {PQ_F_ZETA, &zeta},    {PQ_F_UI, &ui},
                                         {PQ_F_UJ, &uj},         {PQ_F_UIMO, &uimo},    {PQ_F_UJMO, &ujmo},
                                         {PQ_F_ZETA_FI, &zfi},   {PQ_F_ZETA_FJ, &zfj},  {PQ_F_RES, &res},
                                         {PQ_F_RES_BETA, &rb}};
    for (const auto& s : sets)
        if ((rc = set_ref(c, s.first, *s.second))) return rc;
    if (total_time_day) *total_time_day = ttd;
    return PQ_OK;
}

}  // extern "C"
