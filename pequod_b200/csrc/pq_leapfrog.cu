// pq_leapfrog.cu -- the leapfrog scheme (config.h without CABARET).
//
// One DOLEAPFROG sub-step (qg3.F90:615-651) advances level lf with the
// other level m:
//   zeta_centred           zeta_lf += 2 dt * F(psi_m, rel_m, rel_lf)   qg3p_aux.F90:2027-2202
//   robert_asselin_filter  RAW filter of zeta_lf, zeta_m, zeta_old_m   :1719-1786, weights :48-64
//   invert_level           psi_lf, rel_lf, update_zeta_bc(zeta_lf)
// F is the centred flux-form Jacobian of psi and the PV
// q = beta_y + rel + stratification coupling, plus wind forcing, lateral
// viscosity on rel and bottom friction (zeta_tendency, :1790-1939).  Here
// the centred step and the filter are one pointwise kernel (they read only
// psi_m, rel_m and rel_lf at neighbours, none of which they write), the
// inversion is the shared Helmholtz path, and rel + the boundary zeta update
// is one kernel per level.  A level's descriptor (Member) carries
//   zeta = zeta_lf, zeta_next = zeta_m, zeta_old[0] = zeta_old_lf,
//   zeta_old[1] = zeta_old_m, psi = psi_lf, psi_other = psi_m,
//   rel = rel_lf, rel_other = rel_m.
#include "pq_common.cuh"
#include "pq_kernels.h"

namespace pq {

// The centred increment at interior node (i, j) of layer l (without the
// factor T): the reference's centred_increment / zeta_tendency body.
__device__ __forceinline__ double lf_increment(const Member& Mb, const double* __restrict__ psi,
                                               const double* __restrict__ rel, const double* __restrict__ relp,
                                               int i, int j, int l) {
    const int L = Mb.L, pitch = Mb.pitch, ii = Mb.ii, jj = Mb.jj;
    const long long ls = Mb.lstride;
    const long long o = (long long)j * pitch + i + l * ls;
    // Row neighbours.  Only a channel (periodic in j) steps rows 0 and jj-1,
    // whose neighbours wrap (the reference's halo rows hold those rows).
    const int jm = (j == 0) ? jj - 1 : j - 1, jp = (j == jj - 1) ? 0 : j + 1;
    auto at = [&](int di, int dj) {
        return (long long)(dj == 0 ? j : (dj > 0 ? jp : jm)) * pitch + i + di + l * ls;
    };
    // beta * y with y measured from the basin centre (p_beta_y, qg3.F90:303-307)
    const double by = Mb.beta[l];
    auto q = [&](int di, int dj) {
        const long long p = at(di, dj);
        double v = by * (0.5 * (double)(ii - 3) - (double)(i + di)) + rel[p];
        if (L > 1) {
            if (l == 0)
                v += Mb.s2[0] * psi[p + ls];
            else if (l == L - 1)
                v += Mb.s1[l] * psi[p - ls];
            else
                v += Mb.s1[l] * psi[p - ls] + Mb.s2[l] * psi[p + ls];
        }
        return v;
    };
    auto ps = [&](int di, int dj) { return psi[at(di, dj)]; };
    const double jac = 0.25 * ((q(0, 1) * (ps(-1, 1) - ps(1, 1))) - (q(0, -1) * (ps(-1, -1) - ps(1, -1))) -
                               (q(-1, 0) * (ps(-1, 1) - ps(-1, -1))) + (q(1, 0) * (ps(1, 1) - ps(1, -1))));
    const double lap = -4.0 * relp[o] + relp[o - 1] + relp[o + 1] + relp[at(0, -1)] + relp[at(0, 1)];
    const double nu = Mb.viscosity, vb = Mb.visc_bot;
    const double w = (l == 0 && Mb.wind) ? Mb.wind[(long long)j * pitch + i] : 0.0;
    if (L == 1) return jac + w + nu * (lap - vb * relp[o]);  // friction inside the bracket for one layer
    if (l == 0) return jac + w + nu * lap;
    if (l == L - 1) return jac + nu * lap - vb * relp[o];
    return jac + nu * lap;
}

// zeta_centred + robert_asselin_filter for level lf; one thread per node.
__global__ void k_lf_step(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem, double ra_nu,
                          double ra_alpha) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = local;
    if (i >= ii) return;
    double* zl = reinterpret_cast<double*>(Mb.zeta);
    double* zm = reinterpret_cast<double*>(Mb.zeta_next);
    const double* ol = reinterpret_cast<const double*>(Mb.zeta_old[0]);
    double* om = reinterpret_cast<double*>(Mb.zeta_old[1]);
    const double* psim = Mb.psi_other;
    const double* relm = reinterpret_cast<const double*>(Mb.rel_other);
    const double* rell = reinterpret_cast<const double*>(Mb.rel);
    const double T = 2.0 * Mb.sc->dt;
    // RA_DOUBLE_FILTER weights, qg3p_aux.F90:48-64
    const double w21 = 0.5 * ra_nu * ra_alpha, w22 = 1.0 - 2.0 * w21;
    const double w11 = -0.5 * ra_nu * (1.0 - ra_alpha), w12 = -2.0 * w11, w13 = 1.0 + w11;
    const bool interior = i > 0 && i < ii - 1 && (Mb.periodic || (j > 0 && j < jj - 1));
    for (int l = 0; l < L; ++l) {
        const long long o = (long long)j * pitch + i + l * ls;
        double lphi = zl[o];
        if (interior) lphi = lphi + T * lf_increment(Mb, psim, relm, rell, i, j, l);
        const double zmv = zm[o], olv = ol[o];
        zl[o] = w11 * olv + w12 * zmv + w13 * lphi;
        const double nm = w21 * (olv + lphi) + w22 * zmv;
        zm[o] = nm;
        om[o] = nm;
    }
}

// FORWARD_EULER_START (qg3.F90:463-497): zeta_2 = zeta_1 + dt F(psi_1, rel_1,
// rel_1) on the interior; run with the level-1 descriptor (zeta = zeta_1,
// zeta_next = zeta_2).
__global__ void k_lf_forward_euler(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = local;
    if (i < 1 || i >= ii - 1 || (!Mb.periodic && (j < 1 || j >= jj - 1))) return;
    const double* z1 = reinterpret_cast<const double*>(Mb.zeta);
    double* z2 = reinterpret_cast<double*>(Mb.zeta_next);
    const double* rel = reinterpret_cast<const double*>(Mb.rel);
    const double dt = Mb.sc->dt;
    for (int l = 0; l < L; ++l) {
        const long long o = (long long)j * pitch + i + l * ls;
        z2[o] = z1[o] + dt * lf_increment(Mb, Mb.psi, rel, rel, i, j, l);
    }
}

// invert_level's rel_from_zeta_and_psi + apply_rel_bc + update_zeta_bc for
// the level of the descriptor; optionally zeta_old = zeta afterwards, and
// model_time += dt.  One thread per node.
__global__ void k_lf_rel_bc(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem,
                            int copy_old, int advance_time) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = local;
    if (advance_time && i == 0 && j == 0) Mb.sc->model_time += Mb.sc->dt;
    if (i >= ii) return;
    double* z = reinterpret_cast<double*>(Mb.zeta);
    double* rel = reinterpret_cast<double*>(Mb.rel);
    double* zo = reinterpret_cast<double*>(Mb.zeta_old[0]);
    const double* psi = Mb.psi;
    auto ps = [&](int a, int b, int l) { return psi[(long long)b * pitch + a + l * ls]; };
    const bool interior = i > 0 && i < ii - 1 && (Mb.periodic || (j > 0 && j < jj - 1));
    for (int l = 0; l < L; ++l) {
        const long long o = (long long)j * pitch + i + l * ls;
        const double r = rel_node(Mb, ps, z[o], i, j, l);
        rel[o] = r;
        const double zn = interior ? z[o] : zeta_bc_node(Mb, ps, r, i, j, l);
        z[o] = zn;
        if (copy_old) zo[o] = zn;
    }
}

// psi_av += dt * psi of the level just advanced and diagnostic_time += dt
// (qg3.F90:672-680, 725) once model_time, already advanced by this
// sub-step, exceeds the threshold.  Launched after k_lf_rel_bc only while
// the time average is on; no thread of this kernel writes model_time.
__global__ void k_lf_average(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    if (Mb.psi_av == nullptr || !(Mb.sc->model_time > Mb.av_threshold)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = local;
    const double dt = Mb.sc->dt;
    if (i == 0 && j == 0) Mb.sc->diag_time += dt;
    if (i >= Mb.ii) return;
    for (int l = 0; l < Mb.L; ++l) {
        const long long o = (long long)j * Mb.pitch + i + l * Mb.lstride;
        Mb.psi_av[o] += dt * Mb.psi[o];
    }
}

static dim3 node_grid(const LaunchSet& ls) { return dim3((ls.maxI + 127) / 128, ls.maxJ * ls.nmem); }

cudaError_t launch_lf_step(const LaunchSet& ls, double ra_nu, double ra_alpha, cudaStream_t st) {
    k_lf_step<<<node_grid(ls), 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem, ra_nu, ra_alpha);
    return cudaGetLastError();
}

cudaError_t launch_lf_forward_euler(const LaunchSet& ls, cudaStream_t st) {
    k_lf_forward_euler<<<node_grid(ls), 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

cudaError_t launch_lf_average(const LaunchSet& ls, cudaStream_t st) {
    k_lf_average<<<node_grid(ls), 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

cudaError_t launch_lf_rel_bc(const LaunchSet& ls, int copy_old, int advance_time, cudaStream_t st) {
    k_lf_rel_bc<<<node_grid(ls), 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem, copy_old, advance_time);
    return cudaGetLastError();
}

}  // namespace pq
