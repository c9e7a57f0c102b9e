// pq_cabaret.cu -- the CABARET advection step after the PV inversion, fused.
//
// One CTA owns a 32 x 8 tile of nodes (all layers).  It stages psi (all
// layers, halo 2) and, layer by layer, the inputs with the halo each stage
// needs, then computes in shared memory, in the reference's order
// (qg3.F90:641-957):
//   rel_from_zeta_and_psi + apply_rel_bc     qg3p_aux.F90:738-915
//   update_zeta_bc                           :643-734
//   cabaret_forcing                          :1065-1164
//   cabaret_cell_boundaries_time_integrated  :1235-1313
//   cabaret_extrapolator (+ limiter)         :1317-1544
//   cabaret_flux                             :1547-1594
//   cabaret_corrector + set(zeta_old, zeta)  :1597-1642, qg3.F90:957
// and writes back only the fields the next step needs.  Halo values are
// recomputed, never exchanged.  The face fields that are read at neighbour
// faces (ui, zeta_fi, zeta_fj) are ping-ponged; the others are updated in
// place (each face is read and written by its owner CTA only).
#include "pq_common.cuh"
#include "pq_kernels.h"

namespace pq {

constexpr int CAB_THREADS = CAB_TX * CAB_TY;
constexpr int HW = CAB_TX + 4;  // staged width (halo 2)
constexpr int HH = CAB_TY + 4;  // staged height (halo 2)
constexpr int HA = HW * HH;

__device__ __forceinline__ void load_member_c(Member& dst, const Member* src) {
    const int n = sizeof(Member) / 4;
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int t = threadIdx.x; t < n; t += blockDim.x) d[t] = s[t];
}

// Relative vorticity at node (i, j) of layer l from zeta and psi
// (rel_from_zeta_and_psi) with the boundary condition of apply_rel_bc.
// ps(i, j, l) reads staged psi.  Corners take the j-boundary formula, which
// the reference applies last.
template <class PS>
__device__ __forceinline__ double rel_node(const Member& Mb, PS ps, double zeta, int i, int j, int l) {
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L;
    const bool bj = (j == 0 || j == jj - 1), bi = (i == 0 || i == ii - 1);
    if (bj || bi) {
        if (Mb.bc_type == 3) return 0.0;
        int di = 0, dj = 0;
        if (bj)
            dj = (j == 0) ? 1 : -1;
        else
            di = (i == 0) ? 1 : -1;
        const double p0 = ps(i, j, l), p1 = ps(i + di, j + dj, l), p2 = ps(i + 2 * di, j + 2 * dj, l);
        if (Mb.bc_type == 1) {
            const double cff = Mb.alpha / (Mb.alpha + 3.0);
            return cff * (-3.5 * p0 + 4.0 * p1 - 0.5 * p2);
        }
        return 2.0 * (p1 - p0);
    }
    if (L == 1) return zeta;
    const double p = ps(i, j, l);
    if (l == 0) return zeta + Mb.s2[0] * (p - ps(i, j, 1));
    if (l == L - 1) return zeta + Mb.s1[l] * (p - ps(i, j, l - 1));
    return zeta + Mb.s1[l] * (p - ps(i, j, l - 1)) + Mb.s2[l] * (p - ps(i, j, l + 1));
}

// Boundary relative PV from rel and psi (update_zeta_bc).
template <class PS>
__device__ __forceinline__ double zeta_bc_node(const Member& Mb, PS ps, double rel, int i, int j, int l) {
    const int L = Mb.L;
    if (L == 1) return rel;
    const double p = ps(i, j, l);
    if (l == 0) return rel - Mb.s2[0] * (p - ps(i, j, 1));
    if (l == L - 1) return rel - Mb.s1[l] * (p - ps(i, j, l - 1));
    return rel - Mb.s1[l] * (p - ps(i, j, l - 1)) - Mb.s2[l] * (p - ps(i, j, l + 1));
}

__global__ void __launch_bounds__(CAB_THREADS) k_cabaret_fused(const Member* __restrict__ mems,
                                                                 const int* __restrict__ prefix, int nmem) {
    __shared__ Member Mb;
    __shared__ double sRel[HA], sZf[HA], sZo[HA], sZp[HA];
    __shared__ double sUi[HA], sUj[HA], sFi[HA], sFj[HA];
    __shared__ double sFlxI[HA], sFlxJ[HA];
    __shared__ double red[CAB_THREADS / 32];
    __shared__ int is_last;
    extern __shared__ __align__(16) double sPsi[];  // [L][HA]
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    load_member_c(Mb, mems + mi);
    __syncthreads();
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int ntx = (ii + CAB_TX - 1) / CAB_TX;
    const int ty = local / ntx, tx = local - ty * ntx;
    const int i0 = tx * CAB_TX, j0 = ty * CAB_TY;
    const int ib = i0 - 2, jb = j0 - 2;  // staged origin
    const double dt = Mb.sc->dt, tu = Mb.sc->tweight_u;
    const int cur = Mb.cur, nxt = cur ^ 1;

    auto sidx = [&](int i, int j) { return (j - jb) * HW + (i - ib); };
    auto inside = [&](int i, int j) { return i >= 0 && i < ii && j >= 0 && j < jj; };
    auto ps = [&](int i, int j, int l) { return sPsi[l * HA + sidx(i, j)]; };

    // P0: psi, all layers, halo 2.
    for (int t = threadIdx.x; t < L * HA; t += blockDim.x) {
        const int l = t / HA, r = t - l * HA;
        const int j = jb + r / HW, i = ib + r % HW;
        sPsi[t] = inside(i, j) ? Mb.psi[(long long)j * pitch + i + l * ls] : 0.0;
    }

    const double* zeta_pb = reinterpret_cast<const double*>(Mb.zeta);
    const double* zeta_old = reinterpret_cast<const double*>(Mb.zeta_old[cur]);
    double* zeta_new = reinterpret_cast<double*>(Mb.zeta_old[nxt]);
    double* res = reinterpret_cast<double*>(Mb.res);
    double* ui_new = reinterpret_cast<double*>(Mb.ui);
    double* uj = reinterpret_cast<double*>(Mb.uj);
    const double* uimo = reinterpret_cast<const double*>(Mb.uimo[cur]);
    double* uimo_new = reinterpret_cast<double*>(Mb.uimo[nxt]);
    const double* ujmo = reinterpret_cast<const double*>(Mb.ujmo[cur]);
    double* ujmo_new = reinterpret_cast<double*>(Mb.ujmo[nxt]);
    const double* zfi_old = reinterpret_cast<const double*>(Mb.zfi[cur]);
    double* zfi_new = reinterpret_cast<double*>(Mb.zfi[nxt]);
    const double* zfj_old = reinterpret_cast<const double*>(Mb.zfj[cur]);
    double* zfj_new = reinterpret_cast<double*>(Mb.zfj[nxt]);
    double umax = 0.0;

    for (int l = 0; l < L; ++l) {
        const long long lo = l * ls;
        // P1: staged zeta (after predictor + beta) and zeta_old, halo 2.
        for (int r = threadIdx.x; r < HA; r += blockDim.x) {
            const int j = jb + r / HW, i = ib + r % HW;
            const bool in = inside(i, j);
            const long long o = (long long)j * pitch + i + lo;
            const bool interior = in && i > 0 && i < ii - 1 && j > 0 && j < jj - 1;
            sZp[r] = interior ? zeta_pb[o] : 0.0;
            sZo[r] = in ? zeta_old[o] : 0.0;
            // Face fields read at neighbour faces: zeta_fi (i-faces) and
            // zeta_fj (j-faces), plus the old velocities for extrapolation.
            sFi[r] = in ? zfi_old[o] : 0.0;
            sFj[r] = in ? zfj_old[o] : 0.0;
        }
        __syncthreads();
        // P2: relative vorticity on the staged region.
        for (int r = threadIdx.x; r < HA; r += blockDim.x) {
            const int j = jb + r / HW, i = ib + r % HW;
            sRel[r] = inside(i, j) ? rel_node(Mb, ps, sZp[r], i, j, l) : 0.0;
        }
        __syncthreads();
        // P3: zeta after update_zeta_bc and cabaret_forcing, halo 1.
        for (int r = threadIdx.x; r < HA; r += blockDim.x) {
            const int j = jb + r / HW, i = ib + r % HW;
            double v = 0.0;
            if (inside(i, j) && i >= ib + 1 && i < ib + HW - 1 && j >= jb + 1 && j < jb + HH - 1) {
                const bool boundary = (i == 0 || i == ii - 1 || j == 0 || j == jj - 1);
                if (boundary) {
                    v = zeta_bc_node(Mb, ps, sRel[r], i, j, l);
                } else {
                    const double rc = sRel[r];
                    const double lap = -4.0 * rc + sRel[r - 1] + sRel[r + 1] + sRel[r - HW] + sRel[r + HW];
                    double rv;
                    const double nu = Mb.viscosity, vb = Mb.visc_bot;
                    if (L == 1) {
                        const double fw = Mb.wind ? Mb.wind[(long long)j * pitch + i] : 0.0;
                        rv = dt * (fw - vb * rc + nu * lap);
                    } else if (l == 0) {
                        const double fw = Mb.wind ? Mb.wind[(long long)j * pitch + i] : 0.0;
                        rv = dt * (fw + nu * lap);
                    } else if (l == L - 1) {
                        rv = dt * (-vb * rc + nu * lap);
                    } else {
                        rv = dt * nu * lap;
                    }
                    v = sZp[r] + rv;
                }
            }
            sZf[r] = v;
        }
        // P4: face velocities (time-extrapolated), i-faces a in [i0-1, i0+33]
        // on interior rows, j-faces b in [j0-1, j0+9] on interior columns.
        // psi_edge(a, b) is the corner value between nodes a-1, a and b-1, b.
        auto pe = [&](int a, int b) {
            return 0.25 * (ps(a, b, l) + ps(a, b - 1, l) + ps(a - 1, b, l) + ps(a - 1, b - 1, l));
        };
        for (int r = threadIdx.x; r < HA; r += blockDim.x) {
            const int j = jb + r / HW, i = ib + r % HW;
            double u = 0.0;
            // i-face a = i on row j
            if (i >= 1 && i <= ii - 1 && j >= 1 && j <= jj - 2 && i >= i0 - 1 && i <= i0 + CAB_TX + 1 &&
                j >= j0 && j < j0 + CAB_TY) {
                const double uim = -pe(i, j + 1) + pe(i, j);
                const long long o = (long long)j * pitch + i + lo;
                u = (1.0 + tu) * uim - tu * uimo[o];
                if (i >= i0 && i < i0 + CAB_TX) {
                    // owner: record the new extrapolation base
                    sFlxI[r] = uim;
                }
            }
            sUi[r] = u;
            double w = 0.0;
            if (i >= 1 && i <= ii - 2 && j >= 1 && j <= jj - 1 && j >= j0 - 1 && j <= j0 + CAB_TY + 1 &&
                i >= i0 && i < i0 + CAB_TX) {
                const double ujm = pe(i + 1, j) - pe(i, j);
                const long long o = (long long)j * pitch + i + lo;
                w = (1.0 + tu) * ujm - tu * ujmo[o];
                if (j >= j0 && j < j0 + CAB_TY) sFlxJ[r] = ujm;
            }
            sUj[r] = w;
        }
        __syncthreads();
        // Write the owned face velocities and extrapolation bases; track max |u|.
        for (int r = threadIdx.x; r < CAB_TX * CAB_TY; r += blockDim.x) {
            const int i = i0 + (r % CAB_TX), j = j0 + (r / CAB_TX);
            const int s = sidx(i, j);
            const long long o = (long long)j * pitch + i + lo;
            if (i >= 1 && i <= ii - 1 && j >= 1 && j <= jj - 2) {
                ui_new[o] = sUi[s];
                uimo_new[o] = sFlxI[s];
                umax = fmax(umax, fabs(sUi[s]));
            }
            if (i >= 1 && i <= ii - 2 && j >= 1 && j <= jj - 1) {
                uj[o] = sUj[s];
                ujmo_new[o] = sFlxJ[s];
                umax = fmax(umax, fabs(sUj[s]));
            }
        }
        __syncthreads();
        // P5: extrapolator + limiter, then fluxes, on faces a in [i0, i0+32]
        // (rows of the tile) and b in [j0, j0+8] (columns of the tile).
        const bool lim = Mb.limiter != 0;
        for (int r = threadIdx.x; r < HA; r += blockDim.x) {
            const int j = jb + r / HW, i = ib + r % HW;
            double fxi = 0.0;
            if (i >= 1 && i <= ii - 1 && j >= 1 && j <= jj - 2 && i >= i0 && i <= i0 + CAB_TX && j >= j0 &&
                j < j0 + CAB_TY) {
                const double u1 = sUi[r], fi1 = sFi[r];
                double fi2, psi_n, psi_o, d_f;
                if (u1 >= 0.0) {
                    const int up = r - 1;  // node a-1
                    if (i > 1) {
                        const double u2 = sUi[r - 1];
                        fi2 = sFi[r - 1];
                        const double v0 = (u1 + u2) / 2.0;
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi1 - fi2);
                    } else {
                        fi2 = sZf[up];
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o);
                    }
                } else {
                    const int up = r;  // node a
                    if (i < ii - 1) {
                        const double u2 = sUi[r + 1];
                        fi2 = sFi[r + 1];
                        const double v0 = (u1 + u2) / 2.0;
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi2 - fi1);
                    } else {
                        fi2 = sZf[up];
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o);
                    }
                }
                double v = 2.0 * psi_n - fi2;
                if (lim) {
                    const double fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
                    const double fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
                    if (v > fmx) v = fmx;
                    if (v < fmn) v = fmn;
                }
                if (i < i0 + CAB_TX) zfi_new[(long long)j * pitch + i + lo] = v;
                fxi = u1 * v;
            }
            double fxj = 0.0;
            if (i >= 1 && i <= ii - 2 && j >= 1 && j <= jj - 1 && j >= j0 && j <= j0 + CAB_TY && i >= i0 &&
                i < i0 + CAB_TX) {
                const double u1 = sUj[r], fi1 = sFj[r];
                double fi2, psi_n, psi_o, d_f;
                if (u1 >= 0.0) {
                    const int up = r - HW;
                    if (j > 1) {
                        const double u2 = sUj[r - HW];
                        fi2 = sFj[r - HW];
                        const double v0 = (u1 + u2) / 2.0;
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi1 - fi2);
                    } else {
                        fi2 = sZf[up];
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o);
                    }
                } else {
                    const int up = r;
                    if (j < jj - 1) {
                        const double u2 = sUj[r + HW];
                        fi2 = sFj[r + HW];
                        const double v0 = (u1 + u2) / 2.0;
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi2 - fi1);
                    } else {
                        fi2 = sZf[up];
                        psi_n = sZf[up];
                        psi_o = sZo[up];
                        d_f = -(psi_n - psi_o);
                    }
                }
                double v = 2.0 * psi_n - fi2;
                if (lim) {
                    const double fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
                    const double fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
                    if (v > fmx) v = fmx;
                    if (v < fmn) v = fmn;
                }
                if (j < j0 + CAB_TY) zfj_new[(long long)j * pitch + i + lo] = v;
                fxj = u1 * v;
            }
            sFlxI[r] = fxi;
            sFlxJ[r] = fxj;
        }
        __syncthreads();
        // P6: corrector on the tile's nodes; zeta_old <- zeta.
        {
            const int i = i0 + (threadIdx.x % CAB_TX), j = j0 + (threadIdx.x / CAB_TX);
            if (i < ii && j < jj) {
                const int s = sidx(i, j);
                const long long o = (long long)j * pitch + i + lo;
                const bool boundary = (i == 0 || i == ii - 1 || j == 0 || j == jj - 1);
                double z = sZf[s];
                if (!boundary) {
                    const double rr = -(sFlxI[s + 1] - sFlxI[s] + sFlxJ[s + HW] - sFlxJ[s]);
                    res[o] = rr;
                    z = z + 0.5 * dt * rr;
                }
                zeta_new[o] = z;
            }
        }
        __syncthreads();
    }

    // Max |u| of the new face velocities (cabaret_cfl / cabaret_adapt_dt);
    // the last CTA of the member finishes the reduction and, when adaptive
    // time stepping is on, sets dt and the time weights for the next step
    // (cabaret_adapt_dt, qg3p_aux.F90:946-990).
    umax = warp_max(umax);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = umax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < CAB_THREADS / 32; ++w) t = fmax(t, red[w]);
        Mb.maxu_part[local] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[1], 1u);
        is_last = (prev == (unsigned)(Mb.ntiles_cab - 1));
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        const volatile double* part = Mb.maxu_part;
        double mu = 0.0;
        for (int q = 0; q < Mb.ntiles_cab; ++q) mu = fmax(mu, part[q]);
        Scalars* sc = Mb.sc;
        sc->max_u = mu;
        sc->cfl = mu * sc->dt;
        sc->model_time += sc->dt;
        if (Mb.adapt_dt) {
            const double old_dt = sc->dt;
            double ndt = old_dt;
            const double tol = 10.0 * fmax(fabs(mu) * 2.220446049250313e-16, 2.220446049250313e-16);
            if (fabs(mu) > tol) {
                ndt = Mb.target_cfl / mu;
                ndt = fmin(fmin(ndt, old_dt * Mb.max_dt_increase), Mb.max_dt);
            }
            sc->dt = ndt;
            sc->tweight_a = 0.5 * ndt / old_dt;
            sc->tweight_u = ndt / (old_dt + ndt);
            if (ndt < 1.0e-6) atomicOr(Mb.status, (int)ST_SMALL_DT);
        }
        Mb.counters[1] = 0u;
    }
}

cudaError_t launch_cabaret_fused(const LaunchSet& ls, cudaStream_t st) {
    const size_t bytes = (size_t)ls.maxL * HA * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_cabaret_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    k_cabaret_fused<<<ls.ctas_cab, CAB_THREADS, bytes, st>>>(ls.members, ls.prefix_cab, ls.nmem);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// rel on demand (rel_from_zeta_and_psi + apply_rel_bc) from the zeta that
// entered the inversion and the current psi.  One thread per node.
__global__ void k_rel(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int j = local;
    const double* zp = reinterpret_cast<const double*>(Mb.zeta);
    double* rel = reinterpret_cast<double*>(Mb.rel);
    auto ps = [&](int i, int jn, int l) { return Mb.psi[(long long)jn * pitch + i + l * ls]; };
    for (int i = threadIdx.x; i < ii; i += blockDim.x)
        for (int l = 0; l < L; ++l) {
            const long long o = (long long)j * pitch + i + l * ls;
            const bool interior = i > 0 && i < ii - 1 && j > 0 && j < jj - 1;
            rel[o] = rel_node(Mb, ps, interior ? zp[o] : 0.0, i, j, l);
        }
}

cudaError_t launch_rel(const LaunchSet& ls, cudaStream_t st) {
    k_rel<<<ls.ctas_rows_all, 256, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

// End of the START_PERTURB initialisation (qg3.F90:389-391, 450-452): rel
// from zeta and the new psi, boundary zeta from update_zeta_bc, and
// zeta_old = zeta.  One thread per node, one CTA per row.
__global__ void k_init_finish(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int j = local;
    const double* zp = reinterpret_cast<const double*>(Mb.zeta);
    double* rel = reinterpret_cast<double*>(Mb.rel);
    double* zo = reinterpret_cast<double*>(Mb.zeta_old[Mb.cur]);
    auto ps = [&](int i, int jn, int l) { return Mb.psi[(long long)jn * pitch + i + l * ls]; };
    for (int i = threadIdx.x; i < ii; i += blockDim.x)
        for (int l = 0; l < L; ++l) {
            const long long o = (long long)j * pitch + i + l * ls;
            const bool interior = i > 0 && i < ii - 1 && j > 0 && j < jj - 1;
            const double r = rel_node(Mb, ps, zp[o], i, j, l);
            rel[o] = r;
            zo[o] = interior ? zp[o] : zeta_bc_node(Mb, ps, r, i, j, l);
        }
}

cudaError_t launch_init_finish(const LaunchSet& ls, cudaStream_t st) {
    k_init_finish<<<ls.ctas_rows_all, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// energy, qg3p_diagnostics.F90:778-863: one CTA per row j computes the row's
// trapezoid-weighted potential-energy sum and the kinetic-energy sums of the
// cells whose upper-right node is on the row; the last CTA adds the row
// partials in row order and scales them.
__global__ void __launch_bounds__(256) k_energy(const Member* __restrict__ mems, const int* __restrict__ prefix,
                                                 int nmem) {
    __shared__ double red[8][PQ_MAXL + 1];
    __shared__ int is_last;
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int j = local;
    const double* psi = Mb.psi;
    double acc[PQ_MAXL + 1];
    for (int q = 0; q <= L; ++q) acc[q] = 0.0;
    const double wj = (j == 0 || j == jj - 1) ? 0.5 : 1.0;
    for (int i = threadIdx.x; i < ii; i += blockDim.x) {
        const double w = wj * ((i == 0 || i == ii - 1) ? 0.5 : 1.0);
        const long long o = (long long)j * pitch + i;
        for (int k = 0; k < L - 1; ++k) {
            const double fac = 0.5 * Mb.s2[k] * Mb.h[k] / Mb.htot;
            const double d = psi[o + k * ls] - psi[o + (k + 1) * ls];
            acc[L] += w * fac * (d * d);
        }
        if (i >= 1 && j >= 1) {
            for (int k = 0; k < L; ++k) {
                const long long lo = k * ls;
                const double a = psi[o - 1 + lo] + psi[o + lo] - psi[o - 1 - pitch + lo] - psi[o - pitch + lo];
                const double b = psi[o - pitch + lo] + psi[o + lo] - psi[o - 1 - pitch + lo] - psi[o - 1 + lo];
                acc[k] += 0.25 * (a * a + b * b);
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q <= L; ++q) {
        const double v = warp_sum(acc[q]);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q <= L; ++q) {
            double t = 0.0;
            for (int w = 0; w < 8; ++w) t += red[w][q];
            Mb.partials[(long long)local * (PQ_MAXL + 1) + q] = t;
        }
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[2], 1u);
        is_last = (prev == (unsigned)(jj - 1));
    }
    __syncthreads();
    if (!is_last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double* part = Mb.partials;
    double tot[PQ_MAXL + 1];
    for (int q = 0; q <= L; ++q) tot[q] = 0.0;
    for (int r = 0; r < jj; ++r)
        for (int q = 0; q <= L; ++q) tot[q] += part[(long long)r * (PQ_MAXL + 1) + q];
    Scalars* sc = Mb.sc;
    const double cff = Mb.mean_scale;
    const double epot = cff * tot[L];
    sc->epot = epot;
    bool bad = (epot != epot);
    for (int k = 0; k < L; ++k) {
        const double ek = 0.5 * cff * (Mb.h[k] / Mb.htot) * tot[k];
        sc->ekin[k] = ek;
        bad = bad || (ek != ek);
    }
    if (bad) atomicOr(Mb.status, (int)ST_NAN_ENERGY);
    Mb.counters[2] = 0u;
}

cudaError_t launch_energy(const LaunchSet& ls, cudaStream_t st) {
    k_energy<<<ls.ctas_rows_all, 256, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

}  // namespace pq
