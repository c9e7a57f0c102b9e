// pq_cabaret.cu -- the CABARET advection step after the PV inversion, fused.
//
// Everything between the PV inversion and the next step's predictor, in the
// reference's order (qg3.F90:641-957), in one pass over the fields:
//   rel_from_zeta_and_psi + apply_rel_bc     qg3p_aux.F90:738-915
//   update_zeta_bc                           :643-734
//   cabaret_forcing                          :1065-1164
//   cabaret_cell_boundaries_time_integrated  :1235-1313
//   cabaret_extrapolator (+ limiter)         :1317-1544
//   cabaret_flux                             :1547-1594
//   cabaret_corrector + set(zeta_old, zeta)  :1597-1642, qg3.F90:957
// writing back only the fields the next step needs.  Halo values are
// recomputed, never exchanged.  Fields read at nodes or faces owned by another
// warp (zeta_old, uimo, ujmo, zeta_fi, zeta_fj) are ping-ponged.
#include <algorithm>

#include "pq_common.cuh"
#include "pq_kernels.h"

namespace pq {

// Sweep decomposition: a warp owns one layer of a strip of 32 NC columns --
// NC consecutive columns per lane, cab_sw(NC) = 32 NC - 4 output columns plus
// 2 halo columns on each side -- and marches down a band of Mb.cab_sh output
// rows (a tuning parameter).  Every per-lane quantity lives in registers as
// a rolling window over rows; the i-neighbours come from the lane's own
// columns or, across a lane boundary, from warp shuffles.  At iteration r
// (s = r - 2) the warp loads psi row s+2 and the inputs of rows s, s-1, and
// produces
//   rel(s), zeta after BC/forcing at row s-1, uj on face row s, ui on row s-1,
//   zeta_fj on face row s-1, zeta_fi on row s-1, and res / zeta_old at row s-2,
// so output row o is final at iteration o + 4.
// NC = 2 (FP32 fields only, pq_tuning.cab_kernel = 2): each row access of a
// field is one 8-byte vector per lane (16 bytes for psi) and one shuffle
// serves two columns, 26 % fewer instructions per node than NC = 1; it needs
// more registers (two CTAs per SM instead of three), so it pays on large
// grids (2049^2 x 5) and not at 1025^2.
constexpr int CAB_WARPS = 4;
constexpr int CAB_D = 4;  // depth of the per-warp cp.async row pipeline
// Streamed inputs of one iteration (rows relative to s = r - 2).
enum { F_PSI2 = 0, F_ZPB, F_PSIM, F_PSIP, F_ZO, F_UIMO, F_UJMO, F_FIO, F_FJ, F_WIND, F_RB, CAB_NF };
__host__ __device__ constexpr int cab_sw(int nc) { return 32 * nc - 4; }  // output columns per warp
// Ring stage layout: each field a slot of the warp's 32 NC values at their
// own width (FP64 for psi and the wind, T for the rest), in enum order.
__host__ __device__ constexpr bool cab_f64_field(int f) {
    return f == F_PSI2 || f == F_PSIM || f == F_PSIP || f == F_WIND;
}
template <typename T, int NC>
__host__ __device__ constexpr int cab_slot(int f) {  // offset of field f in a stage, in doubles
    int o = 0;
    for (int k = 0; k < f; ++k) o += cab_f64_field(k) ? 32 * NC : 32 * NC * (int)sizeof(T) / 8;
    return o;
}
template <typename T, int NC>
__host__ __device__ constexpr int cab_ring() {  // doubles per warp
    return CAB_D * cab_slot<T, NC>(CAB_NF);
}

__device__ __forceinline__ double shup(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ double shdn(double v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
__device__ __forceinline__ float shup(float v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ float shdn(float v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// Neighbours of a lane's NC columns: o[c] = v at column (c - 1), (c + 1),
// (c - 2), (c + 2) of the lane's frame.  Every lane must call them (shuffles).
template <int NC, typename V>
__device__ __forceinline__ void col_up(const V (&v)[NC], V (&o)[NC]) {
    const V t = shup(v[NC - 1], 1);
#pragma unroll
    for (int c = NC - 1; c > 0; --c) o[c] = v[c - 1];
    o[0] = t;
}
template <int NC, typename V>
__device__ __forceinline__ void col_dn(const V (&v)[NC], V (&o)[NC]) {
    const V t = shdn(v[0], 1);
#pragma unroll
    for (int c = 0; c < NC - 1; ++c) o[c] = v[c + 1];
    o[NC - 1] = t;
}
template <int NC, typename V>
__device__ __forceinline__ void col_up2(const V (&v)[NC], V (&o)[NC]) {
    if constexpr (NC == 1) {
        o[0] = shup(v[0], 2);
    } else {
        const V t0 = shup(v[NC - 2], 1), t1 = shup(v[NC - 1], 1);
#pragma unroll
        for (int c = NC - 1; c > 1; --c) o[c] = v[c - 2];
        o[0] = t0;
        o[1] = t1;
    }
}
template <int NC, typename V>
__device__ __forceinline__ void col_dn2(const V (&v)[NC], V (&o)[NC]) {
    if constexpr (NC == 1) {
        o[0] = shdn(v[0], 2);
    } else {
        const V t0 = shdn(v[0], 1), t1 = shdn(v[1], 1);
#pragma unroll
        for (int c = 0; c < NC - 2; ++c) o[c] = v[c + 2];
        o[NC - 2] = t0;
        o[NC - 1] = t1;
    }
}
// NC consecutive values: one vector access (shared or global memory).
template <int NC, typename V>
__device__ __forceinline__ void vld(const V* p, V (&v)[NC]) {
    if constexpr (NC == 1) {
        v[0] = p[0];
    } else if constexpr (sizeof(V) == 8) {
        const double2 t = *reinterpret_cast<const double2*>(p);
        v[0] = t.x;
        v[1] = t.y;
    } else {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x;
        v[1] = t.y;
    }
}
template <int NC, typename V>
__device__ __forceinline__ void vst(V* p, const V (&v)[NC]) {
    if constexpr (NC == 1) {
        p[0] = v[0];
    } else if constexpr (sizeof(V) == 8) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    } else {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    }
}
template <int BYTES>
__device__ __forceinline__ void cp_async_ca(unsigned dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(src), "n"(BYTES), "r"(src_bytes)
                 : "memory");
}

// One warp's sweep over layer l of the strip starting at column i0 and the
// band starting at row j0.  EDGE = false is the specialisation for warps
// whose whole footprint (columns i0-2 .. i0+32NC-3, rows j0-4 .. j0+sh+3)
// lies at least two nodes inside the domain: no bounds checks, no boundary
// branches, vector loads and stores.  PRED = true also applies the next
// step's cabaret_predictor and cabaret_beta (fixed dt) to every interior
// node it finishes, writing the next step's inversion input zeta_next and
// res_beta_other.  T is the type of the CABARET fields (double, or float in
// the mixed form); psi is FP64 and everything computed from psi differences
// (the rel coupling, the boundary rel, the corner streamfunction and the face
// velocities before the time weighting) is evaluated in FP64.  Returns the
// largest |u| of the faces it wrote.
template <bool EDGE, bool PRED, typename T, int NC>
__device__ __forceinline__ double cab_sweep(const Member& Mb, int l, int i0, int j0, int lane, double* ring) {
    static_assert(NC == 1 || NC == 2, "one or two columns per lane");
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int ib = i0 - 2 + NC * lane;  // the lane's first column
    int ic[NC];
    bool in_i[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        ic[c] = ib + c;
        in_i[c] = !EDGE || (ic[c] >= 0 && ic[c] < ii);
    }
    constexpr int HL = 2 / NC;  // halo lanes on each side
    // Owner lanes of their columns' nodes, i-faces (a = i) and j-faces.
    const bool out_lane = lane >= HL && lane < 32 - HL;
    const int cur = Mb.cur, nxt = cur ^ 1;
    const double dt64 = Mb.sc->dt;
    const T dt = (T)dt64, tu = (T)Mb.sc->tweight_u;
    const bool avg = cab_average_gate(Mb);
    double* const psi_av = Mb.psi_av;
    const T hdt = (T)0.5 * dt;
    const int SH = Mb.cab_sh;
    // All fields of a member live in one allocation: address them by 32-bit
    // element offsets from one base (fewer live registers than 16 pointers);
    // FP64 fields (psi, wind) from B, T fields from BT.  Every field starts
    // on a 256-byte boundary and rows are a multiple of 32 values apart, so
    // the lane's NC values (from an even column when NC = 2) are aligned for
    // one vector access.
    const double* B = Mb.psi;
    const T* BT = reinterpret_cast<const T*>(B);
    auto ofs = [&](const void* f) { return (int)(reinterpret_cast<const double*>(f) - B); };
    auto ofst = [&](const void* f) { return (int)(reinterpret_cast<const T*>(f) - BT); };
    const int lo = (int)(l * ls) + ib;  // layer and column part of every offset
    const int o_psil = lo;
    const int o_psim = (l > 0) ? lo - (int)ls : lo;
    const int o_psip = (l < L - 1) ? lo + (int)ls : lo;
    const int o_zpb = ofst(Mb.zeta) + lo;
    const int o_zo = ofst(Mb.zeta_old[cur]) + lo;
    const int o_zn = ofst(Mb.zeta_old[nxt]) + lo;
    const int o_res = ofst(Mb.res_out) + lo;
    const int o_ui = ofst(Mb.ui) + lo;
    const int o_uj = ofst(Mb.uj) + lo;
    const int o_uimo = ofst(Mb.uimo[cur]) + lo;
    const int o_uimon = ofst(Mb.uimo[nxt]) + lo;
    const int o_ujmo = ofst(Mb.ujmo[cur]) + lo;
    const int o_ujmon = ofst(Mb.ujmo[nxt]) + lo;
    const int o_fio = ofst(Mb.zfi[cur]) + lo;
    const int o_fin = ofst(Mb.zfi[nxt]) + lo;
    const int o_fjo = ofst(Mb.zfj[cur]) + lo;
    const int o_fjn = ofst(Mb.zfj[nxt]) + lo;
    const int o_rb = PRED ? ofst(Mb.res_beta) + lo : 0;
    const int o_rbn = PRED ? ofst(Mb.res_beta_other) + lo : 0;
    const int o_zpn = PRED ? ofst(Mb.zeta_next) + lo : 0;
    const T ta = (T)Mb.sc->tweight_a, beta_l = (T)Mb.beta[l];
    const bool has_wind = (l == 0 && Mb.wind);
    const int o_wind = has_wind ? ofs(Mb.wind) + ib : 0;
    T* W = const_cast<T*>(BT);
    const T nu = (T)Mb.viscosity, vb = (T)Mb.visc_bot;
    const double s1 = Mb.s1[l], s2 = Mb.s2[l];
    const int bc = Mb.bc_type;
    const double cffbc = Mb.alpha / (Mb.alpha + 3.0);
    const bool lim = Mb.limiter != 0;
    const bool top = (l == 0), bottom = (l == L - 1);
    T umax = 0;  // |u| is exact in T: widened once at the end

    auto ld = [&](int off, int row, int c) -> double {
        if (EDGE) return (in_i[c] && row >= 0 && row < jj) ? B[off + c + row * pitch] : 0.0;
        return B[off + c + row * pitch];
    };
    // rel_from_zeta_and_psi coupling for an interior node.
    auto rel_int = [&](T z, double p, double pm, double pp) -> T {
        if (L == 1) return z;
        if (top) return (T)((double)z + s2 * (p - pp));
        if (bottom) return (T)((double)z + s1 * (p - pm));
        return (T)((double)z + s1 * (p - pm) + s2 * (p - pp));
    };
    // Limited upwind extrapolation (cabaret_extrapolator, interior branch).
    // The upwind side only selects the inputs and the sign of the gradient
    // term, so both directions evaluate one instance (no divergent branch).
    auto extrap = [&](T u1, T u2, T fi1, T fi2, T psi_n, T psi_o, bool pos) -> T {
        const T v0 = (u1 + u2) / (T)2;
        const T dfi = pos ? fi1 - fi2 : fi2 - fi1;
        const T d_f = -(psi_n - psi_o) * (T)2 - dt * v0 * dfi;
        T v = (T)2 * psi_n - fi2;
        if (lim) {
            const T fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
            const T fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
            if (v > fmx) v = fmx;
            if (v < fmn) v = fmn;
        }
        return v;
    };
    // The wall branch of the extrapolator: upwind node on the boundary.
    auto extrap_wall = [&](T fi1, T psi_n, T psi_o) -> T {
        const T fi2 = psi_n;
        const T d_f = -(psi_n - psi_o);
        T v = (T)2 * psi_n - fi2;
        if (lim) {
            const T fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
            const T fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
            if (v > fmx) v = fmx;
            if (v < fmn) v = fmn;
        }
        return v;
    };

    // Row copies of iteration r into ring stage r % CAB_D: per field one
    // cp.async of the lane's NC values (interior warps), or one per value
    // (edge warps: values outside the domain, and zeta at non-interior nodes,
    // are zero-filled by a source size of 0, the source then the field base).
    // Slots: cab_slot (each field at its own width).
    constexpr int STAGE = cab_slot<T, NC>(CAB_NF);
    constexpr int S_PSI2 = cab_slot<T, NC>(F_PSI2), S_ZPB = cab_slot<T, NC>(F_ZPB), S_PSIM = cab_slot<T, NC>(F_PSIM),
                  S_PSIP = cab_slot<T, NC>(F_PSIP), S_ZO = cab_slot<T, NC>(F_ZO), S_UIMO = cab_slot<T, NC>(F_UIMO),
                  S_UJMO = cab_slot<T, NC>(F_UJMO), S_FIO = cab_slot<T, NC>(F_FIO), S_FJ = cab_slot<T, NC>(F_FJ),
                  S_WIND = cab_slot<T, NC>(F_WIND), S_RB = cab_slot<T, NC>(F_RB);
    auto cp64 = [&](double* slot, int off, int row) {
        const unsigned sa = (unsigned)__cvta_generic_to_shared(slot + NC * lane);
        if (!EDGE) {
            cp_async_ca<8 * NC>(sa, B + (off + row * pitch), 8 * NC);
        } else {
            const bool rok = row >= 0 && row < jj;
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const bool ok = rok && in_i[c];
                cp_async_ca<8>(sa + 8u * c, ok ? B + (off + c + row * pitch) : B, ok ? 8 : 0);
            }
        }
    };
    auto cpt = [&](double* slot, int off, int row, bool node_int) {
        const unsigned sa = (unsigned)__cvta_generic_to_shared(reinterpret_cast<T*>(slot) + NC * lane);
        if (!EDGE) {
            cp_async_ca<(int)sizeof(T) * NC>(sa, BT + (off + row * pitch), (int)sizeof(T) * NC);
        } else {
            const bool rok = node_int ? (row > 0 && row < jj - 1) : (row >= 0 && row < jj);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const bool ok = rok && (node_int ? (ic[c] > 0 && ic[c] < ii - 1) : in_i[c]);
                cp_async_ca<(int)sizeof(T)>(sa + (unsigned)sizeof(T) * c, ok ? BT + (off + c + row * pitch) : BT,
                                            ok ? (int)sizeof(T) : 0);
            }
        }
    };
    auto issue = [&](int rr) {
        const int ss = rr - 2;
        double* d = ring + (rr % CAB_D) * STAGE;
        cp64(d + S_PSI2, o_psil, ss + 2);
        cpt(d + S_ZPB, o_zpb, ss, true);
        if (L > 1) {
            cp64(d + S_PSIM, o_psim, ss);
            cp64(d + S_PSIP, o_psip, ss);
        }
        cpt(d + S_ZO, o_zo, ss - 1, false);
        cpt(d + S_UIMO, o_uimo, ss - 1, false);
        cpt(d + S_UJMO, o_ujmo, ss, false);
        cpt(d + S_FIO, o_fio, ss - 1, false);
        cpt(d + S_FJ, o_fjo, ss, false);
        if (has_wind) cp64(d + S_WIND, o_wind, ss - 1);
        if (PRED) cpt(d + S_RB, o_rb, ss - 2, false);
    };
    for (int rr = j0; rr < j0 + CAB_D - 1; ++rr) {
        issue(rr);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // Rolling windows.
    double P0[NC], P1[NC], P2[NC], P3[NC], P4[NC];
    T Rm2[NC], Rm1[NC];    // rel rows s-2, s-1
    T ZFm2[NC];            // zeta after forcing, row s-2
    T ZOm2[NC];            // zeta_old row s-2
    T UJm2[NC], UJm1[NC];  // uj faces s-2, s-1
    T FJm2[NC], FJm1[NC];  // zeta_fj (old) faces s-2, s-1
    T FLJm2[NC];           // flux_j face s-2
    T FLI[NC];             // flux_i row s-2 (face a = i)
    T UIm2[NC];            // ui row s-2 (face a = i)
    T zpb_prev[NC];
    double pm_prev[NC], pp_prev[NC], pe_prev[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        P0[c] = 0;
        P1[c] = ld(o_psil, j0 - 4, c);
        P2[c] = ld(o_psil, j0 - 3, c);
        P3[c] = ld(o_psil, j0 - 2, c);
        P4[c] = ld(o_psil, j0 - 1, c);
        Rm2[c] = Rm1[c] = ZFm2[c] = ZOm2[c] = UJm2[c] = UJm1[c] = FJm2[c] = FJm1[c] = FLJm2[c] = FLI[c] = UIm2[c] =
            zpb_prev[c] = 0;
        pm_prev[c] = pp_prev[c] = pe_prev[c] = 0;
    }
    // The left neighbour of P1 (psi row s-1) is, for the lane's first column,
    // the previous row's left neighbour of P2 (carried over, so the corner
    // needs no second shuffle), for the others the lane's own column.
    double up1_prev0 = shup(P2[NC - 1], 1);

    const int rend = j0 + SH + 4;
#pragma unroll 1
    for (int r = j0; r < rend; ++r) {
        const int s = r - 2;
        // ---- loads -----------------------------------------------------------
        // Keep CAB_D - 1 iterations of row copies in flight.
        if (r + CAB_D - 1 < rend) issue(r + CAB_D - 1);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(CAB_D - 1) : "memory");
        const double* st = ring + (r % CAB_D) * STAGE;
        auto get64 = [&](int so, double(&v)[NC]) { vld<NC>(st + so + NC * lane, v); };
        auto gett = [&](int so, T(&v)[NC]) { vld<NC>(reinterpret_cast<const T*>(st + so) + NC * lane, v); };
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            P0[c] = P1[c];
            P1[c] = P2[c];
            P2[c] = P3[c];
            P3[c] = P4[c];
        }
        get64(S_PSI2, P4);
        T zpb_s[NC], zo_1[NC], uimo_1[NC], ujmo_s[NC], fio_1[NC], fj_s[NC], w_1[NC], rb_2[NC];
        double pm_s[NC], pp_s[NC];
        gett(S_ZPB, zpb_s);
        if (L > 1) {
            get64(S_PSIM, pm_s);
            get64(S_PSIP, pp_s);
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) pm_s[c] = pp_s[c] = 0.0;
        }
        gett(S_ZO, zo_1);
        gett(S_UIMO, uimo_1);
        gett(S_UJMO, ujmo_s);
        gett(S_FIO, fio_1);
        gett(S_FJ, fj_s);
        if (has_wind) {
            double w[NC];
            get64(S_WIND, w);
#pragma unroll
            for (int c = 0; c < NC; ++c) w_1[c] = (T)w[c];
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) w_1[c] = (T)0;
        }
        if (PRED) {
            gett(S_RB, rb_2);
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) rb_2[c] = (T)0;
        }

        // ---- rel(s): rel_from_zeta_and_psi + apply_rel_bc -------------------
        double up1[NC], up2[NC], dn1[NC], dn2[NC];
        col_up(P2, up1);
        if (EDGE) {
            col_up2(P2, up2);
            col_dn(P2, dn1);
            col_dn2(P2, dn2);
        }
        T rel_s[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            rel_s[c] = 0;
            if (!EDGE) {
                rel_s[c] = rel_int(zpb_s[c], P2[c], pm_s[c], pp_s[c]);
            } else if (in_i[c] && s >= 0 && s < jj) {
                const int i = ic[c];
                const bool bj = (s == 0 || s == jj - 1), bi = (i == 0 || i == ii - 1);
                if (bj || bi) {
                    if (bc != 3) {
                        double q1, q2;
                        if (bj) {
                            q1 = (s == 0) ? P3[c] : P1[c];
                            q2 = (s == 0) ? P4[c] : P0[c];
                        } else {
                            q1 = (i == 0) ? dn1[c] : up1[c];
                            q2 = (i == 0) ? dn2[c] : up2[c];
                        }
                        rel_s[c] = (T)((bc == 1) ? cffbc * (-3.5 * P2[c] + 4.0 * q1 - 0.5 * q2) : 2.0 * (q1 - P2[c]));
                    }
                } else {
                    rel_s[c] = rel_int(zpb_s[c], P2[c], pm_s[c], pp_s[c]);
                }
            }
        }

        // ---- zeta at row s-1 after update_zeta_bc and cabaret_forcing -------
        const int s1r = s - 1;
        T rl_up[NC], rl_dn[NC];
        col_up(Rm1, rl_up);
        col_dn(Rm1, rl_dn);
        T zf_1[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            zf_1[c] = 0;
            const int i = ic[c];
            if (!EDGE || (in_i[c] && s1r >= 0 && s1r < jj)) {
                const bool bnd = EDGE && (s1r == 0 || s1r == jj - 1 || i == 0 || i == ii - 1);
                if (bnd) {
                    if (L == 1)
                        zf_1[c] = Rm1[c];
                    else if (top)
                        zf_1[c] = (T)((double)Rm1[c] - s2 * (P1[c] - pp_prev[c]));
                    else if (bottom)
                        zf_1[c] = (T)((double)Rm1[c] - s1 * (P1[c] - pm_prev[c]));
                    else
                        zf_1[c] = (T)((double)Rm1[c] - s1 * (P1[c] - pm_prev[c]) - s2 * (P1[c] - pp_prev[c]));
                } else {
                    const T lap = (T)-4 * Rm1[c] + rl_up[c] + rl_dn[c] + Rm2[c] + rel_s[c];
                    T rv;
                    if (L == 1)
                        rv = dt * (w_1[c] - vb * Rm1[c] + nu * lap);
                    else if (top)
                        rv = dt * (w_1[c] + nu * lap);
                    else if (bottom)
                        rv = dt * (-vb * Rm1[c] + nu * lap);
                    else
                        rv = dt * nu * lap;
                    zf_1[c] = zpb_prev[c] + rv;
                }
            }
        }

        // ---- corner psi and face velocities ------------------------------------
        // pe_here: corner between nodes (i-1, i) x (s-1, s).
        double left1[NC], pe_here[NC], pe_dn[NC];  // left1: psi row s-1, column i-1
        left1[0] = up1_prev0;
#pragma unroll
        for (int c = 1; c < NC; ++c) left1[c] = P1[c - 1];
#pragma unroll
        for (int c = 0; c < NC; ++c) pe_here[c] = 0.25 * (P2[c] + P1[c] + up1[c] + left1[c]);
        col_dn(pe_here, pe_dn);
        T uj_s[NC], ujm_s[NC], ui_1[NC], uim_1[NC];
        bool fj_ok[NC], fi_ok[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            const int i = ic[c];
            uj_s[c] = ujm_s[c] = 0;  // face b = s, column i
            fj_ok[c] = !EDGE || (s >= 1 && s <= jj - 1 && i >= 1 && i <= ii - 2);
            if (fj_ok[c]) {
                ujm_s[c] = (T)(pe_dn[c] - pe_here[c]);
                uj_s[c] = ((T)1 + tu) * ujm_s[c] - tu * ujmo_s[c];
            }
            ui_1[c] = uim_1[c] = 0;  // row s-1, face a = i
            fi_ok[c] = !EDGE || (i >= 1 && i <= ii - 1 && s1r >= 1 && s1r <= jj - 2);
            if (fi_ok[c]) {
                uim_1[c] = (T)(-pe_here[c] + pe_prev[c]);
                ui_1[c] = ((T)1 + tu) * uim_1[c] - tu * uimo_1[c];
            }
        }

        // ---- extrapolator, j-faces: face b = s-1 -------------------------------
        T fjn[NC];
        bool bfj_ok[NC];
        const int bf = s - 1;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            fjn[c] = 0;
            bfj_ok[c] = !EDGE || (bf >= 1 && bf <= jj - 1 && ic[c] >= 1 && ic[c] <= ii - 2);
            if (bfj_ok[c]) {
                const T u1 = UJm1[c];
                const bool pos = u1 >= (T)0;
                if (!EDGE)
                    fjn[c] = extrap(u1, pos ? UJm2[c] : uj_s[c], FJm1[c], pos ? FJm2[c] : fj_s[c],
                                    pos ? ZFm2[c] : zf_1[c], pos ? ZOm2[c] : zo_1[c], pos);
                else if (pos)
                    fjn[c] = bf > 1 ? extrap(u1, UJm2[c], FJm1[c], FJm2[c], ZFm2[c], ZOm2[c], true)
                                    : extrap_wall(FJm1[c], ZFm2[c], ZOm2[c]);
                else
                    fjn[c] = bf < jj - 1 ? extrap(u1, uj_s[c], FJm1[c], fj_s[c], zf_1[c], zo_1[c], false)
                                         : extrap_wall(FJm1[c], zf_1[c], zo_1[c]);
            }
        }

        // ---- extrapolator, i-faces on row s-1: face a = i ------------------------
        T ui_up[NC], ui_dn[NC], fi_up[NC], fi_dn[NC], zf_up[NC], zo_up[NC];
        col_up(ui_1, ui_up);
        col_dn(ui_1, ui_dn);
        col_up(fio_1, fi_up);
        col_dn(fio_1, fi_dn);
        col_up(zf_1, zf_up);
        col_up(zo_1, zo_up);
        T fin[NC], flj_1[NC], fli_1[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            fin[c] = 0;
            if (fi_ok[c]) {
                const int i = ic[c];
                const T u1 = ui_1[c];
                const bool pos = u1 >= (T)0;
                if (!EDGE)
                    fin[c] = extrap(u1, pos ? ui_up[c] : ui_dn[c], fio_1[c], pos ? fi_up[c] : fi_dn[c],
                                    pos ? zf_up[c] : zf_1[c], pos ? zo_up[c] : zo_1[c], pos);
                else if (pos)
                    fin[c] = i > 1 ? extrap(u1, ui_up[c], fio_1[c], fi_up[c], zf_up[c], zo_up[c], true)
                                   : extrap_wall(fio_1[c], zf_up[c], zo_up[c]);
                else
                    fin[c] = i < ii - 1 ? extrap(u1, ui_dn[c], fio_1[c], fi_dn[c], zf_1[c], zo_1[c], false)
                                        : extrap_wall(fio_1[c], zf_1[c], zo_1[c]);
            }
            flj_1[c] = UJm1[c] * fjn[c];  // flux_j on face s-1
            fli_1[c] = ui_1[c] * fin[c];  // flux_i on row s-1, face i
        }

        // ---- corrector at row o = s-2 -----------------------------------------
        const int o = s - 2;
        T fli_dn[NC], ui_e[NC];  // flux_i and (PRED) ui on face a = i + 1, row o
        col_dn(FLI, fli_dn);
        if (PRED) {
            col_dn(UIm2, ui_e);
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) ui_e[c] = (T)0;
        }
        if ((o >= j0 && o < j0 + SH) && (!EDGE || (o >= 0 && o < jj))) {
            T z[NC], rr[NC], zz[NC], rbn[NC];
            bool bnd[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int i = ic[c];
                bnd[c] = EDGE && (o == 0 || o == jj - 1 || i == 0 || i == ii - 1);
                rr[c] = -(fli_dn[c] - FLI[c] + flj_1[c] - FLJm2[c]);
                z[c] = ZFm2[c];
                if (!bnd[c]) z[c] = z[c] + hdt * rr[c];
                zz[c] = rbn[c] = 0;
                if (PRED) {
                    // Next step: cabaret_predictor (qg3p_aux.F90:1012-1018) and
                    // cabaret_beta (:1051-1059) with this step's ui.
                    zz[c] = z[c] + hdt * rr[c];
                    rbn[c] = dt * ((T)0.5 * (ui_e[c] + UIm2[c]) * beta_l);
                    zz[c] = zz[c] + ((T)1 + ta) * rbn[c] - ta * rb_2[c];
                }
            }
            const int ro = o * pitch;
            if (!EDGE) {
                if (out_lane) {
                    vst<NC>(W + (o_res + ro), rr);
                    if (PRED) {
                        vst<NC>(W + (o_rbn + ro), rbn);
                        vst<NC>(W + (o_zpn + ro), zz);
                    }
                    vst<NC>(W + (o_zn + ro), z);
                }
            } else {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (out_lane && in_i[c]) {
                        if (!bnd[c]) {
                            W[o_res + c + ro] = rr[c];
                            if (PRED) {
                                W[o_rbn + c + ro] = rbn[c];
                                W[o_zpn + c + ro] = zz[c];
                            }
                        }
                        W[o_zn + c + ro] = z[c];
                    }
                }
            }
            if (avg && out_lane) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    if (in_i[c]) psi_av[o_psil + c + ro] += dt64 * B[o_psil + c + ro];
            }
        }
        // ---- owned face writes ---------------------------------------------------
        const bool row_i = s1r >= j0 && s1r < j0 + SH, row_j = s >= j0 && s < j0 + SH, row_b = bf >= j0 && bf < j0 + SH;
        if (!EDGE) {
            if (out_lane) {
                if (row_i) {
                    vst<NC>(W + (o_ui + s1r * pitch), ui_1);
                    vst<NC>(W + (o_uimon + s1r * pitch), uim_1);
                    vst<NC>(W + (o_fin + s1r * pitch), fin);
#pragma unroll
                    for (int c = 0; c < NC; ++c) umax = fmax(umax, fabs(ui_1[c]));
                }
                if (row_j) {
                    vst<NC>(W + (o_uj + s * pitch), uj_s);
                    vst<NC>(W + (o_ujmon + s * pitch), ujm_s);
#pragma unroll
                    for (int c = 0; c < NC; ++c) umax = fmax(umax, fabs(uj_s[c]));
                }
                if (row_b) vst<NC>(W + (o_fjn + bf * pitch), fjn);
            }
        } else {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (out_lane && in_i[c]) {
                    if (fi_ok[c] && row_i) {
                        W[o_ui + c + s1r * pitch] = ui_1[c];
                        W[o_uimon + c + s1r * pitch] = uim_1[c];
                        W[o_fin + c + s1r * pitch] = fin[c];
                        umax = fmax(umax, fabs(ui_1[c]));
                    }
                    if (fj_ok[c] && row_j) {
                        W[o_uj + c + s * pitch] = uj_s[c];
                        W[o_ujmon + c + s * pitch] = ujm_s[c];
                        umax = fmax(umax, fabs(uj_s[c]));
                    }
                    if (bfj_ok[c] && row_b) W[o_fjn + c + bf * pitch] = fjn[c];
                }
            }
        }
        // ---- shift the windows ---------------------------------------------------
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            Rm2[c] = Rm1[c];
            Rm1[c] = rel_s[c];
            ZFm2[c] = zf_1[c];
            ZOm2[c] = zo_1[c];
            UJm2[c] = UJm1[c];
            UJm1[c] = uj_s[c];
            FJm2[c] = FJm1[c];
            FJm1[c] = fj_s[c];
            FLJm2[c] = flj_1[c];
            FLI[c] = fli_1[c];
            UIm2[c] = ui_1[c];
            zpb_prev[c] = zpb_s[c];
            pm_prev[c] = pm_s[c];
            pp_prev[c] = pp_s[c];
            pe_prev[c] = pe_here[c];
        }
        up1_prev0 = up1[0];
    }
    return (double)umax;
}

// Last CTA of a member: max |u| over the CTAs' partial maxima, the CFL
// number, model time, and when adaptive stepping is on dt and the time
// weights for the next step (cabaret_cfl / cabaret_adapt_dt,
// qg3p_aux.F90:920-990).
// Called by every thread of the last CTA; red: shared scratch of blockDim/32.
__device__ void finish_step(const Member& Mb, double* red) {
    __threadfence();
    const double mu = block_max_l2(Mb.maxu_part, Mb.ntiles_cab, red);
    if (threadIdx.x != 0) return;
    Scalars* sc = Mb.sc;
    if (cab_average_gate(Mb)) sc->diag_time += sc->dt;
    sc->max_u = mu;
    sc->cfl = mu * sc->dt;
    sc->dt_last = sc->dt;
    sc->tweight_a_last = sc->tweight_a;
    sc->tweight_u_last = sc->tweight_u;
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
    Mb.counters[3] = 0u;  // the sweep queue of k_cabaret_fused
}

// Three CTAs per SM (at most 168 registers) with one column per lane:
// measured 16 % faster than the unconstrained allocation (two CTAs) at
// 1025 x 1025 x 3 FP64, 15 % at 2049 x 2049 x 5; four CTAs spill heavily
// and are slower.  Two columns per lane: two CTAs per SM, no spills.
//
// Persistent: a member's CTAs (at most the resident ones, cabaret_ctas) share
// its (layer, strip, band) sweeps through a counter (counters[3]); each warp
// claims the next sweep when it finishes one, so warps run until the queue is
// empty instead of idling in partly filled CTAs and waves.  The boundary
// bands (bounds checks and boundary branches: slower) are claimed first, so
// the last sweeps claimed are interior ones.  The last CTA resets the counter.
template <bool PRED, typename T, int NC>
__global__ void __launch_bounds__(CAB_WARPS * 32, NC == 2 ? 2 : 3)
    k_cabaret_fused(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem,
                    const __grid_constant__ Member one, int use_one) {
    __shared__ Member Mb;
    __shared__ double red[CAB_WARPS];
    __shared__ int is_last;
    extern __shared__ __align__(16) double cab_smem[];  // [CAB_WARPS][cab_ring<T, NC>()]
    pdl_wait();
    int local;
    cta_member(Mb, one, use_one, mems, prefix, nmem, blockIdx.x, &local);
    __syncthreads();
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L;
    const int SH = Mb.cab_sh;
    constexpr int SW = cab_sw(NC);
    const int nstrips = (ii + SW - 1) / SW, nbands = (jj + SH - 1) / SH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntasks = nstrips * nbands * L;
    double* ring = cab_smem + warp * cab_ring<T, NC>();
    double umax = 0.0;
    for (;;) {
        int task = 0;
        if (lane == 0) task = (int)atomicAdd(&Mb.counters[3], 1u);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= ntasks) break;
        const int l = task % L;
        const int sb = task / L;
        const int strip = sb % nstrips, bq = sb / nstrips;
        const int band = nbands < 3 ? bq : bq == 0 ? 0 : bq == 1 ? nbands - 1 : bq - 1;
        const int i0 = strip * SW, j0 = band * SH;
        // Footprint: columns i0-2 .. i0+32NC-3, rows j0-4 .. j0+SH+3.
        const bool interior =
            (i0 - 2 >= 2) && (i0 + 32 * NC - 3 <= ii - 3) && (j0 - 4 >= 2) && (j0 + SH + 3 <= jj - 3);
        const double u = interior ? cab_sweep<false, PRED, T, NC>(Mb, l, i0, j0, lane, ring)
                                  : cab_sweep<true, PRED, T, NC>(Mb, l, i0, j0, lane, ring);
        umax = fmax(umax, u);
        __syncwarp();  // the ring's last reads before the next sweep's copies
    }
    pdl_release();

    // Max |u| of the new face velocities (cabaret_cfl / cabaret_adapt_dt);
    // the last CTA of the member finishes the reduction and, when adaptive
    // time stepping is on, sets dt and the time weights for the next step
    // (cabaret_adapt_dt, qg3p_aux.F90:946-990).
    umax = warp_max(umax);
    if (lane == 0) red[warp] = umax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < CAB_WARPS; ++w) t = fmax(t, red[w]);
        Mb.maxu_part[local] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[1], 1u);
        is_last = (prev == (unsigned)(Mb.ntiles_cab - 1));
    }
    __syncthreads();
    if (is_last) finish_step(Mb, red);
}

// ---------------------------------------------------------------------------
// Tile formulation of the same fused step: one CTA (8 warps) per (layer,
// CT_X x CT_Y tile of output nodes).  Every stage is computed once per node
// or face of the tile's footprint into shared memory, stages separated by
// block barriers; lane = column, warps stride over rows.  All footprint
// arrays share one 32-column frame whose column 0 is node i0-2 and row 0 is
// node j0-2 (a face a sits in the column of node a, a corner between columns
// c-1 and c in column c).  For outputs i in [i0, i0+CT_X), j in [j0, j0+CT_Y):
//   psi (3 layers), zeta, rel   nodes [i0-2, i0+CT_X+1] x [j0-2, j0+CT_Y+1]
//   corner psi                  columns [i0-1, i0+CT_X+1], rows [j0-1, j0+CT_Y+1]
//   zeta after forcing, zeta_old   nodes [i0-1, i0+CT_X] x [j0-1, j0+CT_Y]
//   ui, zeta_fi (old)           faces a in [i0-1, i0+CT_X+1], rows [j0, j0+CT_Y)
//   uj, zeta_fj (old)           faces b in [j0-1, j0+CT_Y+1], columns [i0, i0+CT_X)
//   flux_i / flux_j             faces a in [i0, i0+CT_X] / b in [j0, j0+CT_Y]
// Each output node owns face a = i (ui, uimo, zeta_fi) and face b = j (uj,
// ujmo, zeta_fj), as in the sweep.  EDGE = false: the whole footprint is at
// least one node inside the domain, so no bounds checks or boundary branches.
constexpr int CT_X = 28, CT_Y = 16, CT_THREADS = 256, CT_W = 32, CT_H = CT_Y + 4;
constexpr int CT_N = CT_W * CT_H;  // entries of one frame array

template <typename T>
struct TileSmem {
    // doubles: psi, psi above, psi below, corner psi; T: zeta, rel, zf, zo,
    // ui, fio, uj, fj.  The fluxes reuse the psi-above / psi-below space.
    static constexpr size_t bytes() { return 4 * CT_N * sizeof(double) + 8 * CT_N * sizeof(T); }
};

// rows handled by a warp in a frame row range of length h: ceil(h / 8)
__host__ __device__ constexpr int ct_rows(int h) { return (h + 7) / 8; }

template <bool PRED, bool EDGE, typename T>
// FP64: the CTA's CFL partial and its count towards the last-CTA step finish
// are issued right after the face velocities (stage 3), so that the
// counter's round trip overlaps the extrapolation and the corrector (+1 % per
// step at 513^2 x 3, +2.6 % at 257^2); every scalar the later stages need is
// read before (the last CTA may advance them once every CTA has counted).
// FP32 (64-80 registers, where the extra live values cost more: -5 % at 513^2)
// counts at the end.  *is_last is set by thread 0 at the end.
__device__ __forceinline__ void cab_tile(const Member& Mb, int l, int i0, int j0, char* smem, double* red,
                                         int* is_last, int local) {
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int cur = Mb.cur, nxt = cur ^ 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T dt = (T)Mb.sc->dt, tu = (T)Mb.sc->tweight_u, ta = (T)Mb.sc->tweight_a;
    constexpr bool EARLY = sizeof(T) == 8;
    const bool avg_early = EARLY && cab_average_gate(Mb);
    const double dt64_early = EARLY ? Mb.sc->dt : 0.0;
    const T hdt = (T)0.5 * dt;
    const double s1 = Mb.s1[l], s2 = Mb.s2[l];
    const int bc = Mb.bc_type;
    const double cffbc = Mb.alpha / (Mb.alpha + 3.0);
    const bool lim = Mb.limiter != 0;
    const bool top = (l == 0), bottom = (l == L - 1);
    const T nu = (T)Mb.viscosity, vb = (T)Mb.visc_bot, beta_l = (T)Mb.beta[l];
    const long long lo = l * ls;
    // This lane's column: node i0 - 2 + lane; the row of frame row r is j0 - 2 + r.
    const int ic = i0 - 2 + lane;
    const long long gcol = lo + ic;
    auto grow = [&](int r) { return (long long)(j0 - 2 + r) * pitch; };
    const bool col_in = !EDGE || (ic >= 0 && ic < ii);
    const bool col_int = !EDGE || (ic > 0 && ic < ii - 1);
    auto row_in = [&](int r) { return !EDGE || (j0 - 2 + r >= 0 && j0 - 2 + r < jj); };
    auto row_int = [&](int r) { return !EDGE || (j0 - 2 + r > 0 && j0 - 2 + r < jj - 1); };
    const bool ui_col = !EDGE || (ic >= 1 && ic <= ii - 1);   // face a = ic can exist
    const bool uj_col = !EDGE || (ic >= 1 && ic <= ii - 2);   // column ic can carry j-faces
    auto ui_row = [&](int r) { return !EDGE || (j0 - 2 + r >= 1 && j0 - 2 + r <= jj - 2); };
    auto uj_row = [&](int r) { return !EDGE || (j0 - 2 + r >= 1 && j0 - 2 + r <= jj - 1); };

    double* sPsi = reinterpret_cast<double*>(smem);
    double* sPm = sPsi + CT_N;
    double* sPp = sPm + CT_N;
    double* sPe = sPp + CT_N;
    T* sZpb = reinterpret_cast<T*>(sPe + CT_N);
    T* sRel = sZpb + CT_N;
    T* sZf = sRel + CT_N;
    T* sZo = sZf + CT_N;
    T* sUi = sZo + CT_N;
    T* sFio = sUi + CT_N;
    T* sUj = sFio + CT_N;
    T* sFj = sUj + CT_N;
    T* sFli = reinterpret_cast<T*>(sPm);  // after the face velocities
    T* sFlj = sFli + CT_N;
    auto X = [&](int r, int c) { return r * CT_W + c; };  // frame index

    // Limited upwind extrapolation (cabaret_extrapolator, interior branch).
    auto extrap = [&](T u1, T u2, T fi1, T fi2, T psi_n, T psi_o, bool pos) -> T {
        const T v0 = (u1 + u2) / (T)2;
        const T d_f = pos ? -(psi_n - psi_o) * (T)2 - dt * v0 * (fi1 - fi2)
                          : -(psi_n - psi_o) * (T)2 - dt * v0 * (fi2 - fi1);
        T v = (T)2 * psi_n - fi2;
        if (lim) {
            const T fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
            const T fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
            if (v > fmx) v = fmx;
            if (v < fmn) v = fmn;
        }
        return v;
    };
    // The wall branch: upwind node on the boundary.
    auto extrap_wall = [&](T fi1, T psi_n, T psi_o) -> T {
        const T fi2 = psi_n;
        const T d_f = -(psi_n - psi_o);
        T v = (T)2 * psi_n - fi2;
        if (lim) {
            const T fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
            const T fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
            if (v > fmx) v = fmx;
            if (v < fmn) v = fmn;
        }
        return v;
    };

    const T* zpb = reinterpret_cast<const T*>(Mb.zeta);
    const double* wind = (top && Mb.wind) ? Mb.wind : nullptr;
    // ---- loads used by later stages, issued first (held in registers) -----
    // frame rows: zf 1..CT_Y+2, ui rows 2..CT_Y+1, uj rows 1..CT_Y+3, outputs 2..CT_Y+1
    constexpr int NZ = ct_rows(CT_Y + 2), NU = ct_rows(CT_Y), NV = ct_rows(CT_Y + 3);
    T rWind[NZ], rUimo[NU], rUjmo[NV], rRb[NU];
    {
        const T* uimo = reinterpret_cast<const T*>(Mb.uimo[cur]);
        const T* ujmo = reinterpret_cast<const T*>(Mb.ujmo[cur]);
        const T* rb = reinterpret_cast<const T*>(Mb.res_beta);
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
            const int r = 1 + warp + 8 * k;
            rWind[k] = (wind && r < CT_Y + 3 && lane >= 1 && lane <= CT_X + 2 && col_int && row_int(r))
                           ? (T)wind[grow(r) + ic]
                           : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NU; ++k) {
            const int r = 2 + warp + 8 * k;
            const bool ok = r < CT_Y + 2;
            rUimo[k] = (ok && lane >= 1 && lane <= CT_X + 3 && ui_col && ui_row(r)) ? uimo[grow(r) + gcol] : (T)0;
            rRb[k] = (PRED && ok && lane >= 2 && lane < CT_X + 2 && col_int && row_int(r)) ? rb[grow(r) + gcol] : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const int r = 1 + warp + 8 * k;
            rUjmo[k] = (r < CT_Y + 4 && lane >= 2 && lane < CT_X + 2 && uj_col && uj_row(r)) ? ujmo[grow(r) + gcol]
                                                                                             : (T)0;
        }
    }

    // ---- stage 1: psi (three layers), zeta, zeta_old, old face values ------
    {
        constexpr int NP = ct_rows(CT_H);
        const double* psi = Mb.psi;
        const long long om = (l > 0) ? -ls : 0, op = (l < L - 1) ? ls : 0;
        const T* zold = reinterpret_cast<const T*>(Mb.zeta_old[cur]);
        const T* fio = reinterpret_cast<const T*>(Mb.zfi[cur]);
        const T* fjo = reinterpret_cast<const T*>(Mb.zfj[cur]);
        double vP[NP], vM[NP], vQ[NP];
        T vZ[NP], vO[NZ], vF[NU], vG[NV];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int r = warp + 8 * k;
            const bool ok = r < CT_H && col_in && row_in(r);
            const long long o = grow(r) + gcol;
            vP[k] = ok ? psi[o] : 0.0;
            vM[k] = (ok && L > 1) ? psi[o + om] : 0.0;
            vQ[k] = (ok && L > 1) ? psi[o + op] : 0.0;
            vZ[k] = (ok && col_int && row_int(r)) ? zpb[o] : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
            const int r = 1 + warp + 8 * k;
            vO[k] = (r < CT_Y + 3 && lane >= 1 && lane <= CT_X + 2 && col_in && row_in(r)) ? zold[grow(r) + gcol]
                                                                                           : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NU; ++k) {
            const int r = 2 + warp + 8 * k;
            vF[k] = (r < CT_Y + 2 && lane >= 1 && lane <= CT_X + 3 && ui_col && ui_row(r)) ? fio[grow(r) + gcol]
                                                                                          : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const int r = 1 + warp + 8 * k;
            vG[k] = (r < CT_Y + 4 && lane >= 2 && lane < CT_X + 2 && uj_col && uj_row(r)) ? fjo[grow(r) + gcol]
                                                                                          : (T)0;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int r = warp + 8 * k;
            if (r < CT_H) {
                sPsi[X(r, lane)] = vP[k];
                sPm[X(r, lane)] = vM[k];
                sPp[X(r, lane)] = vQ[k];
                sZpb[X(r, lane)] = vZ[k];
            }
        }
#pragma unroll
        for (int k = 0; k < NZ; ++k) {
            const int r = 1 + warp + 8 * k;
            if (r < CT_Y + 3) sZo[X(r, lane)] = vO[k];
        }
#pragma unroll
        for (int k = 0; k < NU; ++k) {
            const int r = 2 + warp + 8 * k;
            if (r < CT_Y + 2) sFio[X(r, lane)] = vF[k];
        }
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const int r = 1 + warp + 8 * k;
            if (r < CT_Y + 4) sFj[X(r, lane)] = vG[k];
        }
    }
    __syncthreads();

    // ---- stage 2: rel (rel_from_zeta_and_psi + apply_rel_bc), corner psi ---
#pragma unroll
    for (int k = 0; k < ct_rows(CT_H); ++k) {
        const int r = warp + 8 * k;
        if (r >= CT_H) break;
        const int q = X(r, lane);
        T rel = (T)0;
        if (col_in && row_in(r)) {
            const int j = j0 - 2 + r;
            const double p = sPsi[q];
            const bool bj = EDGE && (j == 0 || j == jj - 1), bi = EDGE && (ic == 0 || ic == ii - 1);
            if (bj || bi) {
                // Corners take the j-boundary formula, which the reference applies last.
                if (bc != 3) {
                    double q1, q2;
                    if (bj) {
                        const int d = (j == 0) ? CT_W : -CT_W;
                        q1 = sPsi[q + d];
                        q2 = sPsi[q + 2 * d];
                    } else {
                        const int d = (ic == 0) ? 1 : -1;
                        q1 = sPsi[q + d];
                        q2 = sPsi[q + 2 * d];
                    }
                    rel = (T)((bc == 1) ? cffbc * (-3.5 * p + 4.0 * q1 - 0.5 * q2) : 2.0 * (q1 - p));
                }
            } else {
                const T z = sZpb[q];
                if (L == 1)
                    rel = z;
                else if (top)
                    rel = (T)((double)z + s2 * (p - sPp[q]));
                else if (bottom)
                    rel = (T)((double)z + s1 * (p - sPm[q]));
                else
                    rel = (T)((double)z + s1 * (p - sPm[q]) + s2 * (p - sPp[q]));
            }
        }
        sRel[q] = rel;
    }
#pragma unroll
    for (int k = 0; k < ct_rows(CT_Y + 3); ++k) {
        const int r = 1 + warp + 8 * k;  // corner between rows r-1 and r
        if (r >= CT_H) break;
        if (lane >= 1) {
            const int q = X(r, lane);     // corner between columns lane-1 and lane
            sPe[q] = 0.25 * (sPsi[q] + sPsi[q - CT_W] + sPsi[q - 1] + sPsi[q - CT_W - 1]);
        }
    }
    __syncthreads();

    // ---- stage 3: zeta after update_zeta_bc + forcing; face velocities -----
    double umax = 0.0;
#pragma unroll
    for (int k = 0; k < NZ; ++k) {
        const int r = 1 + warp + 8 * k;
        if (r >= CT_Y + 3) break;
        if (lane < 1 || lane > CT_X + 2) continue;
        const int q = X(r, lane);
        T zf = (T)0;
        if (col_in && row_in(r)) {
            const T R = sRel[q];
            if (EDGE && !(col_int && row_int(r))) {
                const double p = sPsi[q];
                if (L == 1)
                    zf = R;
                else if (top)
                    zf = (T)((double)R - s2 * (p - sPp[q]));
                else if (bottom)
                    zf = (T)((double)R - s1 * (p - sPm[q]));
                else
                    zf = (T)((double)R - s1 * (p - sPm[q]) - s2 * (p - sPp[q]));
            } else {
                const T lap = (T)-4 * R + sRel[q - 1] + sRel[q + 1] + sRel[q - CT_W] + sRel[q + CT_W];
                const T w = rWind[k];
                T rv;
                if (L == 1)
                    rv = dt * (w - vb * R + nu * lap);
                else if (top)
                    rv = dt * (w + nu * lap);
                else if (bottom)
                    rv = dt * (-vb * R + nu * lap);
                else
                    rv = dt * nu * lap;
                zf = sZpb[q] + rv;
            }
        }
        sZf[q] = zf;
    }
    T* ui_g = reinterpret_cast<T*>(Mb.ui);
    T* uimo_n = reinterpret_cast<T*>(Mb.uimo[nxt]);
    T* uj_g = reinterpret_cast<T*>(Mb.uj);
    T* ujmo_n = reinterpret_cast<T*>(Mb.ujmo[nxt]);
    const bool own_col = lane >= 2 && lane < CT_X + 2;  // columns of the tile's outputs
#pragma unroll
    for (int k = 0; k < NU; ++k) {
        const int r = 2 + warp + 8 * k;  // face a = ic on row r
        if (r >= CT_Y + 2) break;
        if (lane < 1 || lane > CT_X + 3) continue;
        const int q = X(r, lane);
        T u = (T)0;
        if (ui_col && ui_row(r)) {
            // corners (a, rows r-1|r) and (a, rows r|r+1)
            const T um = (T)(sPe[q] - sPe[q + CT_W]);
            u = ((T)1 + tu) * um - tu * rUimo[k];
            if (own_col) {
                const long long o = grow(r) + gcol;
                ui_g[o] = u;
                uimo_n[o] = um;
                umax = fmax(umax, (double)fabs(u));
            }
        }
        sUi[q] = u;
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const int r = 1 + warp + 8 * k;  // face b = row r, column ic
        if (r >= CT_Y + 4) break;
        if (!own_col) continue;
        const int q = X(r, lane);
        T u = (T)0;
        if (uj_col && uj_row(r)) {
            // corners (columns ic|ic+1, rows r-1|r) and (ic-1|ic, r-1|r)
            const T um = (T)(sPe[q + 1] - sPe[q]);
            u = ((T)1 + tu) * um - tu * rUjmo[k];
            if (r >= 2 && r < CT_Y + 2) {
                const long long o = grow(r) + gcol;
                uj_g[o] = u;
                ujmo_n[o] = um;
                umax = fmax(umax, (double)fabs(u));
            }
        }
        sUj[q] = u;
    }
    unsigned prev = 0u;
    auto count = [&]() {
        umax = warp_max(umax);
        if (lane == 0) red[warp] = umax;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = 0.0;
            for (int w = 0; w < CT_THREADS / 32; ++w) m = fmax(m, red[w]);
            Mb.maxu_part[local] = m;
            __threadfence();
            prev = atomicAdd(&Mb.counters[1], 1u);
        }
    };
    if constexpr (EARLY)
        count();
    else
        __syncthreads();

    // ---- stage 4: extrapolated face values (cabaret_extrapolator) and fluxes
    T* fin_g = reinterpret_cast<T*>(Mb.zfi[nxt]);
    T* fjn_g = reinterpret_cast<T*>(Mb.zfj[nxt]);
#pragma unroll
    for (int k = 0; k < NU; ++k) {
        const int r = 2 + warp + 8 * k;  // face a = ic on row r, a in [i0, i0+CT_X]
        if (r >= CT_Y + 2) break;
        if (lane < 2 || lane > CT_X + 2) continue;
        const int q = X(r, lane);
        T flux = (T)0;
        if (ui_col && ui_row(r)) {
            const T u1 = sUi[q];
            T f;
            if (u1 >= (T)0)
                f = (!EDGE || ic > 1) ? extrap(u1, sUi[q - 1], sFio[q], sFio[q - 1], sZf[q - 1], sZo[q - 1], true)
                                      : extrap_wall(sFio[q], sZf[q - 1], sZo[q - 1]);
            else
                f = (!EDGE || ic < ii - 1) ? extrap(u1, sUi[q + 1], sFio[q], sFio[q + 1], sZf[q], sZo[q], false)
                                           : extrap_wall(sFio[q], sZf[q], sZo[q]);
            if (own_col) fin_g[grow(r) + gcol] = f;
            flux = u1 * f;
        }
        sFli[q] = flux;
    }
#pragma unroll
    for (int k = 0; k < ct_rows(CT_Y + 1); ++k) {
        const int r = 2 + warp + 8 * k;  // face b = row r in [j0, j0+CT_Y], column ic
        if (r >= CT_Y + 3) break;
        if (!own_col) continue;
        const int q = X(r, lane);
        const int b = j0 - 2 + r;
        T flux = (T)0;
        if (uj_col && uj_row(r)) {
            const T u1 = sUj[q];
            T f;
            if (u1 >= (T)0)
                f = (!EDGE || b > 1)
                        ? extrap(u1, sUj[q - CT_W], sFj[q], sFj[q - CT_W], sZf[q - CT_W], sZo[q - CT_W], true)
                        : extrap_wall(sFj[q], sZf[q - CT_W], sZo[q - CT_W]);
            else
                f = (!EDGE || b < jj - 1) ? extrap(u1, sUj[q + CT_W], sFj[q], sFj[q + CT_W], sZf[q], sZo[q], false)
                                          : extrap_wall(sFj[q], sZf[q], sZo[q]);
            if (r < CT_Y + 2) fjn_g[grow(r) + gcol] = f;
            flux = u1 * f;
        }
        sFlj[q] = flux;
    }
    __syncthreads();

    // ---- stage 5: cabaret_corrector (+ the next step's predictor and beta) --
    T* res_g = reinterpret_cast<T*>(Mb.res_out);
    T* zn_g = reinterpret_cast<T*>(Mb.zeta_old[nxt]);
    T* rbn_g = reinterpret_cast<T*>(Mb.res_beta_other);
    T* zpn_g = reinterpret_cast<T*>(Mb.zeta_next);
    const bool avg = EARLY ? avg_early : cab_average_gate(Mb);
    const double dt64 = EARLY ? dt64_early : Mb.sc->dt;
#pragma unroll
    for (int k = 0; k < NU; ++k) {
        const int r = 2 + warp + 8 * k;
        if (r >= CT_Y + 2) break;
        if (!own_col || !(col_in && row_in(r))) continue;
        const int q = X(r, lane);
        const long long o = grow(r) + gcol;
        if (avg) Mb.psi_av[o] += dt64 * sPsi[q];
        T z = sZf[q];
        if (col_int && row_int(r)) {
            const T rr = -(sFli[q + 1] - sFli[q] + sFlj[q + CT_W] - sFlj[q]);
            res_g[o] = rr;
            z = z + hdt * rr;
            if (PRED) {
                // cabaret_predictor (qg3p_aux.F90:1012-1018) and cabaret_beta
                // (:1051-1059) of the next step with this step's ui.
                T zz = z + hdt * rr;
                const T rbn = dt * ((T)0.5 * (sUi[q + 1] + sUi[q]) * beta_l);
                zz = zz + ((T)1 + ta) * rbn - ta * rRb[k];
                rbn_g[o] = rbn;
                zpn_g[o] = zz;
            }
        }
        zn_g[o] = z;
    }
    if constexpr (!EARLY) count();
    if (threadIdx.x == 0) *is_last = (prev == (unsigned)(Mb.ntiles_cab - 1));
}

// MINB: CTAs per SM the register allocation must allow.  Three (80
// registers): the FP32 form always, FP64 on grids of many waves, where the
// extra resident CTA hides more latency than the tighter allocation costs
// (measured -8 % at 513 x 513 x 3); one for short FP64 grids.
template <bool PRED, typename T, int MINB>
__global__ void __launch_bounds__(CT_THREADS, MINB) k_cabaret_tile(const Member* __restrict__ mems,
                                                              const int* __restrict__ prefix, int nmem,
                                                              const __grid_constant__ Member one, int use_one) {
    __shared__ Member Mb;
    __shared__ double red[CT_THREADS / 32];
    __shared__ int is_last;
    extern __shared__ __align__(16) char tsm[];
    pdl_wait();
    int local;
    cta_member(Mb, one, use_one, mems, prefix, nmem, blockIdx.x, &local);
    __syncthreads();
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L;
    const int tx = (ii + CT_X - 1) / CT_X;
    const int l = local % L;
    const int tile = local / L;
    const int i0 = (tile % tx) * CT_X, j0 = (tile / tx) * CT_Y;
    // Interior tiles: footprint [i0-2, i0+CT_X+1] x [j0-2, j0+CT_Y+1] inside
    // the interior nodes.
    const bool inner = i0 - 2 >= 1 && i0 + CT_X + 1 <= ii - 2 && j0 - 2 >= 1 && j0 + CT_Y + 1 <= jj - 2;
    if (inner)
        cab_tile<PRED, false, T>(Mb, l, i0, j0, tsm, red, &is_last, local);
    else
        cab_tile<PRED, true, T>(Mb, l, i0, j0, tsm, red, &is_last, local);
    pdl_release();
    __syncthreads();
    if (is_last) finish_step(Mb, red);
}

// CTAs of k_cabaret_fused resident on the current device at once (at least 1).
template <typename T, int NC>
static int cabaret_resident_t() {
    const size_t bytes = (size_t)CAB_WARPS * cab_ring<T, NC>() * sizeof(double);
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(k_cabaret_fused<true, T, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cabaret_fused<true, T, NC>, CAB_WARPS * 32, bytes) !=
            cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return std::max(1, per * sms);
}

int cabaret_ctas_bound(int ii, int jj, int L, int min_sh) {
    const int sw = cab_sw(1), nstrips = (ii + sw - 1) / sw, nbands = (jj + min_sh - 1) / min_sh;
    return (nstrips * nbands * L + CAB_WARPS - 1) / CAB_WARPS;
}

int cabaret_ctas(int ii, int jj, int L, int sh, int nc, bool f32) {
    const int sw = cab_sw(nc);
    const int nstrips = (ii + sw - 1) / sw, nbands = (jj + sh - 1) / sh;
    const int need = (nstrips * nbands * L + CAB_WARPS - 1) / CAB_WARPS;
    const int resident = !f32 ? cabaret_resident_t<double, 1>()
                         : nc == 2 ? cabaret_resident_t<float, 2>()
                                   : cabaret_resident_t<float, 1>();
    return std::min(need, resident);
}

int cabaret_tile_ctas(int ii, int jj, int L) {
    return ((ii + CT_X - 1) / CT_X) * ((jj + CT_Y - 1) / CT_Y) * L;
}

template <bool PRED, typename T, int NC>
static cudaError_t launch_sweeps(const LaunchSet& ls, cudaStream_t st) {
    const size_t bytes = (size_t)CAB_WARPS * cab_ring<T, NC>() * sizeof(double);
    cudaError_t e =
        cudaFuncSetAttribute(k_cabaret_fused<PRED, T, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    cudaError_t le = launch_step_kernel(ls.pdl, k_cabaret_fused<PRED, T, NC>, dim3(ls.ctas_cab),
                                        dim3(CAB_WARPS * 32), bytes, st, ls.members, ls.prefix_cab, ls.nmem,
                                        member_arg(ls), member_arg_used(ls));
    if (le != cudaSuccess) return le;
    return cudaGetLastError();
}

template <bool PRED, typename T>
static cudaError_t launch_cab(const LaunchSet& ls, cudaStream_t st) {
    if (ls.cab_kernel == 0) {
        const size_t tb = TileSmem<T>::bytes();
        // CTAs per SM the registers must allow (measured on B200): FP64 three
        // on grids of many waves, else one; FP32 four on grids of more than two
        // CTAs per SM (40 KB of shared memory each: +2.9 % per step at
        // 513^2 x 3, +5.1 % at 257^2; -4.8 % on 129^2's 135 CTAs), else three.
        void (*kern)(const Member*, const int*, int, Member, int);
        if constexpr (sizeof(T) == 4)
            kern = ls.ctas_cab > 2 * ls.sm_count ? k_cabaret_tile<PRED, T, 4> : k_cabaret_tile<PRED, T, 3>;
        else
            kern = ls.ctas_cab > 4 * ls.sm_count ? k_cabaret_tile<PRED, T, 3> : k_cabaret_tile<PRED, T, 1>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb);
        if (e != cudaSuccess) return e;
        return launch_step_kernel(ls.pdl, kern, dim3(ls.ctas_cab), dim3(CT_THREADS), tb, st, ls.members,
                                  ls.prefix_cab, ls.nmem, member_arg(ls), member_arg_used(ls));
    }
    if constexpr (sizeof(T) == 4) {
        if (ls.cab_kernel == 2) return launch_sweeps<PRED, T, 2>(ls, st);
    }
    return launch_sweeps<PRED, T, 1>(ls, st);
}


// ---------------------------------------------------------------------------
// The channel (periodic in j) CABARET step: the same sub-steps as the fused
// closed-basin kernels (qg3.F90:640-807, 940-956), as four node-parallel
// kernels.  Every row is interior in j; rows, j-faces and corners wrap
// modulo jj (the reference's halo rows and seam faces, qg3p_base.F90:
// 1887-1956, 2964-3003, hold exactly the wrapped values); the walls are the
// columns i = 0 and ii - 1.  One thread per (column, row) with all layers;
// face a (i-faces) and face b (j-faces) belong to node (a, b).  Arithmetic
// in FP64, fields stored as T.
namespace {

struct ChannelIdx {
    int ii, jj, pitch;
    long long ls;
    __device__ __forceinline__ long long at(int i, int j, int l) const {
        j = j < 0 ? j + jj : (j >= jj ? j - jj : j);
        return (long long)j * pitch + i + l * ls;
    }
};

// rel_from_zeta_and_psi + apply_rel_bc, then update_zeta_bc on the walls.
// rel is also kept in FP64 (in helm_io, free during a step) for the forcing's
// Laplacian, whose differences would lose the mixed form's FP32 digits.
template <typename T>
__global__ void k_ch_rel(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = local;
    if (i >= Mb.ii) return;
    const long long o = (long long)j * Mb.pitch + i;
    T* z = reinterpret_cast<T*>(Mb.zeta);
    T* rel = reinterpret_cast<T*>(Mb.rel);
    double* rel64 = reinterpret_cast<double*>(Mb.helm_io);
    auto ps = [&](int a, int b, int l) { return Mb.psi[(long long)b * Mb.pitch + a + l * Mb.lstride]; };
    const bool wall = (i == 0 || i == Mb.ii - 1);
    // psi_av += dt * psi once model time passes the threshold (qg3.F90:672-680).
    double* av = cab_average_gate(Mb) ? Mb.psi_av : nullptr;
    const double dt = Mb.sc->dt;
    for (int l = 0; l < Mb.L; ++l) {
        const long long ol = o + l * Mb.lstride;
        const double r = rel_node(Mb, ps, (double)z[ol], i, j, l);
        rel[ol] = (T)r;
        rel64[ol] = r;
        if (wall) z[ol] = (T)zeta_bc_node(Mb, ps, r, i, j, l);
        if (av) av[ol] = av[ol] + dt * Mb.psi[ol];
    }
}

// cabaret_forcing (qg3p_aux.F90:1065-1164) on the interior columns, and the
// time-integrated cell-boundary velocities (cabaret_cell_boundaries_
// time_integrated, :1235-1313) of the faces a = i (i-faces) and b = j
// (j-faces) of this node.
template <typename T>
__global__ void k_ch_force_cell(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, L = Mb.L, i = blockIdx.x * blockDim.x + threadIdx.x, j = local;
    if (i >= ii) return;
    const ChannelIdx X{ii, Mb.jj, Mb.pitch, Mb.lstride};
    const int cur = Mb.cur, nxt = cur ^ 1;
    const double dt = Mb.sc->dt, tu = Mb.sc->tweight_u;
    T* z = reinterpret_cast<T*>(Mb.zeta);
    const double* rel = reinterpret_cast<const double*>(Mb.helm_io);  // FP64 rel of k_ch_rel
    const double* psi = Mb.psi;
    const double nu = Mb.viscosity, vb = Mb.visc_bot;
    if (i >= 1 && i <= ii - 2) {
        for (int l = 0; l < L; ++l) {
            auto rp = [&](int a, int b) { return rel[X.at(a, b, l)]; };
            const double lap = -4.0 * rp(i, j) + rp(i - 1, j) + rp(i + 1, j) + rp(i, j - 1) + rp(i, j + 1);
            const double wnd = (l == 0 && Mb.wind) ? Mb.wind[X.at(i, j, 0)] : 0.0;
            double rv;
            if (L == 1)
                rv = dt * (wnd - vb * rp(i, j) + nu * lap);
            else if (l == 0)
                rv = dt * (wnd + nu * lap);
            else if (l < L - 1)
                rv = dt * nu * lap;
            else
                rv = dt * (-vb * rp(i, j) + nu * lap);
            const long long o = X.at(i, j, l);
            z[o] = (T)((double)z[o] + rv);
        }
    }
    // psi_edge(a, b): the corner between nodes a-1, a and rows b-1, b.
    auto pe = [&](int a, int b, int l) {
        return 0.25 * (psi[X.at(a, b, l)] + psi[X.at(a, b - 1, l)] + psi[X.at(a - 1, b, l)] + psi[X.at(a - 1, b - 1, l)]);
    };
    T* ui = reinterpret_cast<T*>(Mb.ui);
    T* uj = reinterpret_cast<T*>(Mb.uj);
    const T* uimo = reinterpret_cast<const T*>(Mb.uimo[cur]);
    const T* ujmo = reinterpret_cast<const T*>(Mb.ujmo[cur]);
    T* uimn = reinterpret_cast<T*>(Mb.uimo[nxt]);
    T* ujmn = reinterpret_cast<T*>(Mb.ujmo[nxt]);
    for (int l = 0; l < L; ++l) {
        const long long o = X.at(i, j, l);
        if (i >= 1) {  // i-face a = i, row j
            const double uim = -pe(i, j + 1, l) + pe(i, j, l);
            ui[o] = (T)((1.0 + tu) * uim - tu * (double)uimo[o]);
            uimn[o] = (T)uim;
        }
        if (i >= 1 && i <= ii - 2) {  // j-face b = j of column i
            const double ujm = pe(i + 1, j, l) - pe(i, j, l);
            uj[o] = (T)((1.0 + tu) * ujm - tu * (double)ujmo[o]);
            ujmn[o] = (T)ujm;
        }
    }
}

// cabaret_extrapolator (qg3p_aux.F90:1317-1544) for the faces of this node;
// the j-faces of a channel always take the interior branch.
template <typename T>
__global__ void k_ch_extrap(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, L = Mb.L, i = blockIdx.x * blockDim.x + threadIdx.x, j = local;
    if (i < 1 || i >= ii) return;
    const ChannelIdx X{ii, Mb.jj, Mb.pitch, Mb.lstride};
    const int cur = Mb.cur, nxt = cur ^ 1;
    const double dt = Mb.sc->dt;
    const bool lim = Mb.limiter != 0;
    const T* z = reinterpret_cast<const T*>(Mb.zeta);
    const T* zo = reinterpret_cast<const T*>(Mb.zeta_old[cur]);
    const T* ui = reinterpret_cast<const T*>(Mb.ui);
    const T* uj = reinterpret_cast<const T*>(Mb.uj);
    const T* fio = reinterpret_cast<const T*>(Mb.zfi[cur]);
    const T* fjo = reinterpret_cast<const T*>(Mb.zfj[cur]);
    T* fin = reinterpret_cast<T*>(Mb.zfi[nxt]);
    T* fjn = reinterpret_cast<T*>(Mb.zfj[nxt]);
    auto limit = [&](double v, double fi1, double fi2, double psi_n, double d_f) {
        if (lim) {
            const double fmx = fmax(fmax(fi1, fi2), psi_n) - d_f;
            const double fmn = fmin(fmin(fi1, fi2), psi_n) - d_f;
            if (v > fmx) v = fmx;
            if (v < fmn) v = fmn;
        }
        return v;
    };
    for (int l = 0; l < L; ++l) {
        const long long o = X.at(i, j, l);
        {  // i-face a = i between nodes i-1 and i
            const double u1 = ui[o], fi1 = fio[o];
            double fi2, psi_n, psi_o, d_f;
            if (u1 >= 0.0) {
                psi_n = z[o - 1];
                psi_o = zo[o - 1];
                if (i > 1) {
                    const double u2 = ui[o - 1];
                    fi2 = fio[o - 1];
                    const double v0 = (u1 + u2) / 2.0;
                    d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi1 - fi2);
                } else {
                    fi2 = psi_n;
                    d_f = -(psi_n - psi_o);
                }
            } else {
                psi_n = z[o];
                psi_o = zo[o];
                if (i < ii - 1) {
                    const double u2 = ui[o + 1];
                    fi2 = fio[o + 1];
                    const double v0 = (u1 + u2) / 2.0;
                    d_f = -(psi_n - psi_o) * 2.0 - dt * v0 * (fi2 - fi1);
                } else {
                    fi2 = psi_n;
                    d_f = -(psi_n - psi_o);
                }
            }
            fin[o] = (T)limit(2.0 * psi_n - fi2, fi1, fi2, psi_n, d_f);
        }
        if (i <= ii - 2) {  // j-face b = j between rows j-1 and j of column i
            const double u1 = uj[o], fi1 = fjo[o];
            double u2, fi2, psi_n, psi_o, d_f;
            if (u1 >= 0.0) {
                const long long om = X.at(i, j - 1, l);
                u2 = uj[om];
                fi2 = fjo[om];
                psi_n = z[om];
                psi_o = zo[om];
                d_f = -(psi_n - psi_o) * 2.0 - dt * ((u1 + u2) / 2.0) * (fi1 - fi2);
            } else {
                const long long op = X.at(i, j + 1, l);
                u2 = uj[op];
                fi2 = fjo[op];
                psi_n = z[o];
                psi_o = zo[o];
                d_f = -(psi_n - psi_o) * 2.0 - dt * ((u1 + u2) / 2.0) * (fi2 - fi1);
            }
            fjn[o] = (T)limit(2.0 * psi_n - fi2, fi1, fi2, psi_n, d_f);
        }
    }
}

// cabaret_flux + cabaret_corrector (qg3p_aux.F90:1547-1642), zeta_old =
// zeta; the largest |u| of this node's faces, and the last CTA's
// cabaret_cfl / cabaret_adapt_dt / model time (finish_step).
template <typename T>
__global__ void __launch_bounds__(128) k_ch_corrector(const Member* __restrict__ mems, const int* __restrict__ prefix,
                                                       int nmem) {
    __shared__ double red[4];
    __shared__ int is_last;
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, L = Mb.L, i = blockIdx.x * blockDim.x + threadIdx.x, j = local;
    const ChannelIdx X{ii, Mb.jj, Mb.pitch, Mb.lstride};
    const int nxt = Mb.cur ^ 1;
    double umax = 0.0;
    if (i < ii) {
        const double hdt = 0.5 * Mb.sc->dt;
        const T* z = reinterpret_cast<const T*>(Mb.zeta);
        const T* ui = reinterpret_cast<const T*>(Mb.ui);
        const T* uj = reinterpret_cast<const T*>(Mb.uj);
        const T* fin = reinterpret_cast<const T*>(Mb.zfi[nxt]);
        const T* fjn = reinterpret_cast<const T*>(Mb.zfj[nxt]);
        T* res = reinterpret_cast<T*>(Mb.res_out);
        T* zn = reinterpret_cast<T*>(Mb.zeta_old[nxt]);
        for (int l = 0; l < L; ++l) {
            const long long o = X.at(i, j, l);
            if (i >= 1) umax = fmax(umax, fabs((double)ui[o]));
            if (i >= 1 && i <= ii - 2) umax = fmax(umax, fabs((double)uj[o]));
            double zz = z[o];
            if (i >= 1 && i <= ii - 2) {
                const long long op = X.at(i, j + 1, l);
                const double fl0 = (double)ui[o] * (double)fin[o], fl1 = (double)ui[o + 1] * (double)fin[o + 1];
                const double fj0 = (double)uj[o] * (double)fjn[o], fj1 = (double)uj[op] * (double)fjn[op];
                const double r = -(fl1 - fl0 + fj1 - fj0);
                res[o] = (T)r;
                zz = zz + hdt * r;
            }
            zn[o] = (T)zz;
        }
    }
    umax = warp_max(umax);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = umax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 4; ++w) t = fmax(t, red[w]);
        const int cta = blockIdx.x + gridDim.x * local;
        Mb.maxu_part[cta] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&Mb.counters[1], 1u);
        is_last = (prev == (unsigned)(Mb.ntiles_cab - 1));
    }
    __syncthreads();
    if (is_last) finish_step(Mb, red);
}

}  // namespace

cudaError_t launch_cabaret_channel(const LaunchSet& ls, int f32, cudaStream_t st) {
    const dim3 g((ls.maxI + 127) / 128, ls.maxJ * ls.nmem);
    if (f32) {
        k_ch_rel<float><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_force_cell<float><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_extrap<float><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_corrector<float><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    } else {
        k_ch_rel<double><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_force_cell<double><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_extrap<double><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
        k_ch_corrector<double><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    }
    return cudaGetLastError();
}

int channel_ctas(int ii, int jj) { return ((ii + 127) / 128) * jj; }


// ---------------------------------------------------------------------------
// The quad eddy covariances of a step (qg3.F90:683-721), at the point of the
// reference's diagnostics: psi of the inversion, rel (rel_from_zeta_and_psi
// with its boundary condition) and zeta with its boundary PV.  The zonal and
// meridional velocities (qg3p_diagnostics.F90:941-1107) are 0 on the nodes
// the reference never writes, rel / alpha, 0 or NaN on the walls by the
// velocity boundary condition; interface velocities (:1163-1194), thickness
// (:1197-1227), the dt-weighted products (:1360-1427) and the scaled
// buoyancy correlations (:1430-1537).  One thread per node, all layers.
// Launched before the step's CABARET kernel, so the model-time gate is the
// one the fused kernel uses for psi_av.  lf: a leapfrog sub-step, launched
// after its rel kernel on the level just inverted (psi, rel, zeta
// BLEAPFROG); its gate is the model time already advanced by the sub-step,
// as k_lf_average's.
template <typename T>
__global__ void k_quad(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem, int lf) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.y, &local);
    const Member& Mb = mems[mi];
    if (Mb.quad == nullptr) return;
    if (lf ? !(Mb.psi_av != nullptr && Mb.sc->model_time > Mb.av_threshold) : !cab_average_gate(Mb)) return;
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride, qs = Mb.quad_stride;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = local;
    if (i >= ii) return;
    const double dt = Mb.sc->dt;
    const T* zp = reinterpret_cast<const T*>(Mb.zeta);
    auto ps = [&](int a, int b, int l) { return Mb.psi[(long long)b * pitch + a + l * ls]; };
    const long long o = (long long)j * pitch + i;
    // A channel (periodic j) has no j walls: every row is interior and its
    // j neighbours wrap.
    const bool per = Mb.periodic != 0;
    const bool in_i = i > 0 && i < ii - 1, in_j = per || (j > 0 && j < jj - 1);
    const int jm = (per && j == 0) ? jj - 1 : j - 1, jp = (per && j == jj - 1) ? 0 : j + 1;
    const int bc = Mb.bc_type;  // u, v on a wall from rel: rel / alpha, 0, or NaN
    double P[PQ_MAXL], R[PQ_MAXL], Z[PQ_MAXL], U[PQ_MAXL], V[PQ_MAXL], Tn[PQ_MAXL];
#pragma unroll
    for (int l = 0; l < PQ_MAXL; ++l) {
        if (l >= L) break;
        P[l] = ps(i, j, l);
        const double r = rel_node(Mb, ps, (in_i && in_j) ? (double)zp[o + l * ls] : 0.0, i, j, l);
        R[l] = r;
        Z[l] = (in_i && in_j) ? (double)zp[o + l * ls] : zeta_bc_node(Mb, ps, r, i, j, l);
        auto wall = [&]() { return bc == 1 ? r / Mb.alpha : bc == 2 ? 0.0 : __longlong_as_double(0x7ff8000000000000LL); };
        U[l] = (in_i && in_j) ? 0.5 * (ps(i + 1, j, l) - ps(i - 1, j, l)) : (in_j ? wall() : 0.0);
        V[l] = (in_i && in_j) ? 0.5 * (ps(i, jp, l) - ps(i, jm, l)) : (in_i ? wall() : 0.0);
    }
#pragma unroll
    for (int l = 0; l < PQ_MAXL; ++l) {
        if (l >= L) break;
        if (L == 1)
            Tn[l] = 0.0;
        else if (l == 0)
            Tn[l] = -Mb.s2[0] * (P[0] - P[1]);
        else if (l == L - 1)
            Tn[l] = -Mb.s1[l] * (P[l] - P[l - 1]);
        else
            Tn[l] = -Mb.s1[l] * (P[l] - P[l - 1]) - Mb.s2[l] * (P[l] - P[l + 1]);
    }
    double* q = Mb.quad + o;
    auto add = [&](int f, int l, double v) { q[f * qs + l * ls] += v; };
#pragma unroll
    for (int l = 0; l < PQ_MAXL; ++l) {
        if (l >= L) break;
        add(0, l, dt * U[l] * U[l]);
        add(1, l, dt * V[l] * V[l]);
        add(4, l, dt * U[l] * V[l]);
        add(5, l, dt * U[l] * R[l]);
        add(6, l, dt * V[l] * R[l]);
        add(7, l, dt * R[l] * R[l]);
        add(8, l, dt * P[l] * R[l]);
        add(9, l, dt * U[l] * Z[l]);
        add(10, l, dt * V[l] * Z[l]);
        add(11, l, dt * Z[l] * Z[l]);
        add(12, l, dt * Z[l] * R[l]);
        add(13, l, dt * P[l] * P[l]);
        add(14, l, dt * P[l] * Z[l]);
        add(15, l, dt * U[l] * Tn[l]);
        add(16, l, dt * V[l] * Tn[l]);
        add(17, l, dt * Tn[l] * R[l]);
        add(18, l, dt * Tn[l] * Tn[l]);
        if (l < L - 1) {
            const double ui = 0.5 * (U[l] + U[l + 1]), vi = 0.5 * (V[l] + V[l + 1]);
            add(2, l, dt * ui * ui);
            add(3, l, dt * vi * vi);
            const double dp = P[l] - P[l + 1];
            const double scb = Mb.s2[l] * Mb.h[l] * dp;
            add(19, l, dt * (0.5 * (U[l + 1] + U[l]) * scb));
            add(20, l, dt * (0.5 * (V[l + 1] + V[l]) * scb));
            add(22, l, dt * (Mb.s2[l] * Mb.h[l] * (dp * dp) / (Mb.h[l] + Mb.h[l + 1])));
        }
        if (L > 1) {
            double sbb;
            if (l == 0) {
                const double a = P[1] - P[0];
                sbb = 0.25 * (Mb.s2[0] * (a * a));
            } else if (l == L - 1) {
                const double a = P[l - 1] - P[l];
                sbb = 0.25 * (Mb.s1[l] * (a * a));
            } else {
                const double a = P[l - 1] - P[l], b = P[l + 1] - P[l];
                sbb = 0.25 * (Mb.s1[l] * (a * a) + Mb.s2[l] * (b * b));
            }
            add(21, l, dt * sbb);
        }
    }
}

cudaError_t launch_quad(const LaunchSet& ls, int f32, int lf, cudaStream_t st) {
    const dim3 g((ls.maxI + 127) / 128, ls.maxJ * ls.nmem);
    if (f32)
        k_quad<float><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem, lf);
    else
        k_quad<double><<<g, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem, lf);
    return cudaGetLastError();
}

cudaError_t launch_cabaret_fused(const LaunchSet& ls, int predict_next, int f32, cudaStream_t st) {
    if (f32) return predict_next ? launch_cab<true, float>(ls, st) : launch_cab<false, float>(ls, st);
    return predict_next ? launch_cab<true, double>(ls, st) : launch_cab<false, double>(ls, st);
}

// ---------------------------------------------------------------------------
// rel on demand (rel_from_zeta_and_psi + apply_rel_bc) from the zeta that
// entered the inversion and the current psi.  One thread per node.
template <typename T>
__global__ void k_rel(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int j = local;
    const T* zp = reinterpret_cast<const T*>(Mb.zeta);
    T* rel = reinterpret_cast<T*>(Mb.rel);
    auto ps = [&](int i, int jn, int l) { return Mb.psi[(long long)jn * pitch + i + l * ls]; };
    for (int i = threadIdx.x; i < ii; i += blockDim.x)
        for (int l = 0; l < L; ++l) {
            const long long o = (long long)j * pitch + i + l * ls;
            const bool interior = i > 0 && i < ii - 1 && (Mb.periodic || (j > 0 && j < jj - 1));
            rel[o] = (T)rel_node(Mb, ps, interior ? (double)zp[o] : 0.0, i, j, l);
        }
}

cudaError_t launch_rel(const LaunchSet& ls, int f32, cudaStream_t st) {
    if (f32)
        k_rel<float><<<ls.ctas_rows_all, 256, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    else
        k_rel<double><<<ls.ctas_rows_all, 256, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    return cudaGetLastError();
}

// End of the START_PERTURB initialisation (qg3.F90:389-391, 450-452): rel
// from zeta and the new psi, boundary zeta from update_zeta_bc, and
// zeta_old = zeta.  One thread per node, one CTA per row.
template <typename T>
__global__ void k_init_finish(const Member* __restrict__ mems, const int* __restrict__ prefix, int nmem) {
    int local;
    const int mi = find_member(prefix, nmem, blockIdx.x, &local);
    const Member& Mb = mems[mi];
    const int ii = Mb.ii, jj = Mb.jj, L = Mb.L, pitch = Mb.pitch;
    const long long ls = Mb.lstride;
    const int j = local;
    const T* zp = reinterpret_cast<const T*>(Mb.zeta);
    T* rel = reinterpret_cast<T*>(Mb.rel);
    T* zo = reinterpret_cast<T*>(Mb.zeta_old[Mb.cur]);
    auto ps = [&](int i, int jn, int l) { return Mb.psi[(long long)jn * pitch + i + l * ls]; };
    for (int i = threadIdx.x; i < ii; i += blockDim.x)
        for (int l = 0; l < L; ++l) {
            const long long o = (long long)j * pitch + i + l * ls;
            const bool interior = i > 0 && i < ii - 1 && (Mb.periodic || (j > 0 && j < jj - 1));
            const double r = rel_node(Mb, ps, (double)zp[o], i, j, l);
            rel[o] = (T)r;
            zo[o] = interior ? zp[o] : (T)zeta_bc_node(Mb, ps, r, i, j, l);
        }
}

cudaError_t launch_init_finish(const LaunchSet& ls, int f32, cudaStream_t st) {
    if (f32)
        k_init_finish<float><<<ls.ctas_rows_all, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
    else
        k_init_finish<double><<<ls.ctas_rows_all, 128, 0, st>>>(ls.members, ls.prefix_rows_all, ls.nmem);
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
    // A channel has no j boundary: full weights, and the kinetic-energy
    // corners of row 0 reach back to row jj - 1.
    const double wj = (!Mb.periodic && (j == 0 || j == jj - 1)) ? 0.5 : 1.0;
    const long long back = (j == 0) ? (long long)(jj - 1) * pitch : -(long long)pitch;  // row j-1, wrapped
    for (int i = threadIdx.x; i < ii; i += blockDim.x) {
        const double w = wj * ((i == 0 || i == ii - 1) ? 0.5 : 1.0);
        const long long o = (long long)j * pitch + i;
        for (int k = 0; k < L - 1; ++k) {
            const double fac = 0.5 * Mb.s2[k] * Mb.h[k] / Mb.htot;
            const double d = psi[o + k * ls] - psi[o + (k + 1) * ls];
            acc[L] += w * fac * (d * d);
        }
        if (i >= 1 && (j >= 1 || Mb.periodic)) {
            for (int k = 0; k < L; ++k) {
                const long long lo = k * ls;
                const double a = psi[o - 1 + lo] + psi[o + lo] - psi[o - 1 + back + lo] - psi[o + back + lo];
                const double b = psi[o + back + lo] + psi[o + lo] - psi[o - 1 + back + lo] - psi[o - 1 + lo];
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
    if (!is_last) return;
    __threadfence();
    double tot[PQ_MAXL + 1];
    for (int q = 0; q <= L; ++q) tot[q] = block_sum_l2(Mb.partials + q, jj, PQ_MAXL + 1, &red[0][0]);
    if (threadIdx.x != 0) return;
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

namespace pq {

// FP64 <-> FP32 copies of pitched fields (the mixed form's state I/O).
__global__ void k_convert(void* __restrict__ dst, const void* __restrict__ src, size_t count, int to_f32) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride) {
        if (to_f32)
            static_cast<float*>(dst)[t] = (float)static_cast<const double*>(src)[t];
        else
            static_cast<double*>(dst)[t] = (double)static_cast<const float*>(src)[t];
    }
}

cudaError_t launch_convert(void* dst, const void* src, size_t count, int to_f32, cudaStream_t st) {
    size_t blocks = (count + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_convert<<<(unsigned)blocks, 256, 0, st>>>(dst, src, count, to_f32);
    return cudaGetLastError();
}

}  // namespace pq
