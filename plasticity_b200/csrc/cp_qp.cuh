// cp_qp.cuh -- the per-quadrature-point constitutive update and tangent,
// one thread per qp, FP64 (the plain drop-in form of calculatePlasticity).
//
// Follows src/materialModels/crystalPlasticity/calculatePlasticity.cc:13-1022
// and inactiveSlipRemoval.cc:4-124 with these restatements (same math,
// different operation order):
//   * Schmid tensors are never stored for all systems: resolved shears are
//     m . (R^T X R) . n with the lattice's crystal-frame m, n; the
//     potentially active systems keep S = (R m)(R n)^T as its two vectors and
//     S : X is formed as (R m) . X (R n).  The sorted kernel (cp_qp2.cuh)
//     forms every product in the same order, so the two kernels give the
//     same bits.
//   * Only the A[PA,PA] block of the consistency matrix is built (the only
//     block inactive_slip_removal reads, inactiveSlipRemoval.cc:16-24), with
//     the j-dependent factor hoisted out of the i loop (:273-306).
//   * The pseudo-inverse solve A_PA^+ b (LAPACK SVD, :26,:99) is an LU solve
//     with partial pivoting: identical for the nonsingular A_PA the update
//     produces; a zero pivot sets CP_QP_SINGULAR.
//   * dels_delF (:131,:548-579) is identically zero (it starts at zero and is
//     only ever multiplied by its previous value), so it is not carried.
//   * The Gateaux series sum_l dFp^l S dFp^(k-l) (:645-676, :748-779) uses the
//     recurrence D_k = dFp D_{k-1} + S dFp^k, shared by the A2 and S_PA
//     series; matrixExponential(-del_FP) of :682 is evaluated once.
//   * The 3^7 / 3^8 loops of the final tangent (:857-939) are evaluated as
//     3x3 products per column (k,l); the "rotation back" with L = I is a copy.
#pragma once

#include <stdint.h>

#include "cp_math.cuh"

#ifndef CP_MAX_SYSTEMS
#define CP_MAX_SYSTEMS 64
#endif

namespace cp {

constexpr int NM = CP_MAX_SYSTEMS;
constexpr int EXP_TERM_CAP = 64;     // matrixExponential series terms
constexpr int GATEAUX_TERM_CAP = 64;  // count3 terms

// status bits (include/cp_gpu.h)
constexpr int QP_NONFINITE = 1, QP_SINGULAR = 2, QP_ACTIVE_OVERFLOW = 4, QP_SERIES_CAP = 8,
              QP_SLIP_SEARCH_CAP = 16, QP_ILL_CONDITIONED = 32;

// Per-lattice constants, one copy in global memory per lattice.
struct LatDev {
    int n, ns, nw, twinning;
    double C[36];
    double m[NM * 3], nn[NM * 3];
    double q[NM * NM];
    double s0[NM], h0[NM], ss[NM], a[NM], C1[NM], C2[NM];
    double twin_thr, twin_sat, twin_shear;
};

struct Opts {
    double tol;
    int max_search, max_solver, multiphase;
};

// Structure-of-arrays history of one lattice group: component c of qp i is at
// field[c * count + i].
struct GroupDev {
    int64_t count;
    const int64_t* qp;  // caller-order index of internal qp i
    double *Fp_c, *Fe_c, *s_c, *W_c, *rot_c, *rotnew_c, *tw_c, *sl_c;
    int* twin_c;
    double *Fp_i, *Fe_i, *s_i, *W_i, *rot_i, *rotnew_i, *tw_i, *sl_i;
    int* twin_i;
    const int* where;  // internal index of the qp bound j-th in the group (null: j itself)
};

struct QpOut {
    double* P;     // 9, row-major (may be null)
    double* T;     // 9 (may be null)
    double* dPdF;  // 81, dPdF[27m+9n+3o+p] (may be null)
    double scale;  // multiplies P and dPdF (JxW in the fused assembly, else 1)
};

__host__ __device__ __forceinline__ double ldg(const double* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

__host__ __device__ __forceinline__ M3 load_soa3(const double* __restrict__ f, int64_t cnt, int64_t i) {
    M3 m;
#pragma unroll
    for (int c = 0; c < 9; ++c) m.a[c] = f[c * cnt + i];
    return m;
}
__host__ __device__ __forceinline__ void store_soa3(double* __restrict__ f, int64_t cnt, int64_t i, const M3& m) {
#pragma unroll
    for (int c = 0; c < 9; ++c) f[c * cnt + i] = m.a[c];
}

// resolved shear m . (R^T X R) . n in the crystal frame
__host__ __device__ __forceinline__ double resolved(const LatDev& L, int s, const M3& Xc) {
    const double m0 = ldg(&L.m[3 * s]), m1 = ldg(&L.m[3 * s + 1]), m2 = ldg(&L.m[3 * s + 2]);
    const double n0 = ldg(&L.nn[3 * s]), n1 = ldg(&L.nn[3 * s + 1]), n2 = ldg(&L.nn[3 * s + 2]);
    const double y0 = dot3(Xc(0, 0), n0, Xc(0, 1), n1, Xc(0, 2), n2);
    const double y1 = dot3(Xc(1, 0), n0, Xc(1, 1), n1, Xc(1, 2), n2);
    const double y2 = dot3(Xc(2, 0), n0, Xc(2, 1), n1, Xc(2, 2), n2);
    return dot3(m0, y0, m1, y1, m2, y2);
}

// S : X = (R m)^T X (R n) for a Schmid tensor stored as its two vectors
// v = (R m, R n); the one product form both update kernels use, so that the
// plain and the sorted kernel round alike
__host__ __device__ __forceinline__ double schmid_dot(const double* v, const M3& X) {
    const double y0 = dot3(X(0, 0), v[3], X(0, 1), v[4], X(0, 2), v[5]);
    const double y1 = dot3(X(1, 0), v[3], X(1, 1), v[4], X(1, 2), v[5]);
    const double y2 = dot3(X(2, 0), v[3], X(2, 1), v[4], X(2, 2), v[5]);
    return dot3(v[0], y0, v[1], y1, v[2], y2);
}
__host__ __device__ __forceinline__ M3 schmid_of(const double* v) {
    M3 S;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S(i, j) = v[i] * v[3 + j];
    return S;
}
__host__ __device__ __forceinline__ void schmid_vectors(const LatDev& L, int s, const M3& R, double* v) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        v[i] = dot3(R(i, 0), ldg(&L.m[3 * s]), R(i, 1), ldg(&L.m[3 * s + 1]), R(i, 2), ldg(&L.m[3 * s + 2]));
        v[3 + i] = dot3(R(i, 0), ldg(&L.nn[3 * s]), R(i, 1), ldg(&L.nn[3 * s + 1]), R(i, 2), ldg(&L.nn[3 * s + 2]));
    }
}

// New Rodrigues vector of a twin reorientation (rod2quat, quatproduct,
// quat2rod; updateAfterIncrement.cc:781-821, called at
// calculatePlasticity.cc:985-1012): the qp's rotation (r0, r1, r2) composed
// with the 180-degree rotation about twin system sys's normal.
__host__ __device__ __forceinline__ void twin_rotation(const LatDev& L, int sys, double r0, double r1, double r2,
                                                       double out[3]) {
    const double dot = dot3(r0, r0, r1, r1, r2, r2);
    const double c = cos(atan(sqrt(dot)));
    const double q2[4] = {c, c * r0, c * r1, c * r2};
    const double q1[4] = {0.0, ldg(&L.nn[3 * sys]), ldg(&L.nn[3 * sys + 1]), ldg(&L.nn[3 * sys + 2])};
    const double a = q2[0], b = q1[0];
    const double d1 = dot3(q1[1], q2[1], q1[2], q2[2], q1[3], q2[3]);
    double qp0 = fmad(a, b, -d1);
    double qp1 = fmad(-q1[2], q2[3], fmad(q2[2], q1[3], fmad(b, q2[1], a * q1[1])));
    double qp2 = fmad(q1[1], q2[3], fmad(-q2[1], q1[3], fmad(b, q2[2], a * q1[2])));
    double qp3 = fmad(-q1[1], q2[2], fmad(q2[1], q1[2], fmad(b, q2[3], a * q1[3])));
    if (qp0 < 0) {
        qp0 = -qp0;
        qp1 = -qp1;
        qp2 = -qp2;
        qp3 = -qp3;
    }
    if (fabs(qp0) < 1e-4) qp0 = 1e-4;
    const double iq = 1 / qp0;
    out[0] = qp1 * iq;
    out[1] = qp2 * iq;
    out[2] = qp3 * iq;
}

// matrixExponential (matrixOperations.cc:165-186)
__host__ __device__ __forceinline__ M3 matexp(const M3& A, int* terms, int* status) {
    M3 E = eye3(), t = eye3();
    double count = 1.0;
    int k = 0;
    while (frob(t) > 1.0e-10) {
        if (k >= EXP_TERM_CAP) {
            *status |= QP_SERIES_CAP;
            break;
        }
        t = mul(t, A);
        t = scale(1.0 / count, t);
        axpy(E, 1.0, t);
        count += 1.0;
        ++k;
    }
    if (terms) *terms = k;
    return E;
}

// In-place LU with partial pivoting of a row-major m x m block (leading
// dimension ld) and solve for nrhs right-hand sides stored row-major (m x
// nrhs, leading dimension ldb).  Returns nonzero on a zero pivot.  *cond
// (optional) receives max|u_jj| / min|u_jj|, a cheap estimate of the
// condition number used to flag numerically singular active-set blocks.
__host__ __device__ __forceinline__ int lu_solve(double* A, int m, int ld, double* B, int nrhs, int ldb,
                                                 double* cond = nullptr) {
    int sing = 0;
    double pmin = 1e308, pmax = 0.0;
    for (int j = 0; j < m; ++j) {
        int r = j;
        double mx = fabs(A[j * ld + j]);
        for (int i = j + 1; i < m; ++i) {
            const double v = fabs(A[i * ld + j]);
            if (v > mx) {
                mx = v;
                r = i;
            }
        }
        pmin = fmin(pmin, mx);
        pmax = fmax(pmax, mx);
        if (mx == 0.0) {
            sing = 1;
            continue;
        }
        if (r != j) {
            for (int c = 0; c < m; ++c) {
                const double t = A[j * ld + c];
                A[j * ld + c] = A[r * ld + c];
                A[r * ld + c] = t;
            }
            for (int c = 0; c < nrhs; ++c) {
                const double t = B[j * ldb + c];
                B[j * ldb + c] = B[r * ldb + c];
                B[r * ldb + c] = t;
            }
        }
        const double piv = 1.0 / A[j * ld + j];
        for (int i = j + 1; i < m; ++i) {
            const double f = A[i * ld + j] * piv;
            if (f == 0.0) continue;
            for (int c = j + 1; c < m; ++c) A[i * ld + c] -= f * A[j * ld + c];
            for (int c = 0; c < nrhs; ++c) B[i * ldb + c] -= f * B[j * ldb + c];
        }
    }
    for (int j = m - 1; j >= 0; --j) {
        const double d = A[j * ld + j];
        for (int c = 0; c < nrhs; ++c) {
            double s = B[j * ldb + c];
            for (int k = j + 1; k < m; ++k) s -= A[j * ld + k] * B[k * ldb + c];
            B[j * ldb + c] = s / d;
        }
    }
    if (cond) *cond = m == 0 ? 1.0 : (pmin > 0.0 ? pmax / pmin : 1e308);
    return sing;
}

// D_k recurrence for the Gateaux series; returns S + sum_k cm(k) D_k and
// S + sum_k cp(k) D_k with cm(k) = (-1)^k/(k+1)!, cp(k) = 1/(k+1)!.
__host__ __device__ __forceinline__ void gateaux_pair(const M3& S, const M3& P, int count3, M3& dminus, M3& dplus) {
    dminus = S;
    dplus = S;
    M3 D = S, Pk = eye3();
    double fact = 1.0;
    for (int k = 1; k <= count3; ++k) {
        Pk = mul(Pk, P);
        M3 D2 = mul(P, D);
        axpy(D2, 1.0, mul(S, Pk));
        D = D2;
        fact *= (double)(k + 1);
        const double cpk = 1.0 / fact;
        const double cmk = ((k & 1) ? -1.0 : 1.0) / fact;
        axpy(dminus, cmk, D);
        axpy(dplus, cpk, D);
    }
}

// Per-thread scratch sized by the lattice class (NT systems, PMAX rows of A).
template <int NT, int PMAX>
struct QpScratch {
    double s[NT], W[NT], tau_tr[NT], b[NT], x_old[NT], x[NT], h[NT], tn[NT];
    double A[PMAX * PMAX];
    double Apa[PMAX * PMAX];
    double rhs[PMAX * 9];
    double Sv[PMAX * 6];  // Schmid tensor of PA system k as its vectors R m, R n
    unsigned char pa[NT], pa0[NT], cur[NT];
};

// The whole calculatePlasticity for internal qp i of group g.
template <int NT, int PMAX>
__host__ __device__ int qp_update(const LatDev& L, const Opts& o, const GroupDev& g, int64_t i, const M3& F, int flag,
                         double F_e, double F_r, const QpOut& out, int32_t* stats_out, int lattice_id) {
    QpScratch<NT, PMAX> w;
    const int n = L.n, ns = L.ns, nw = L.nw;
    const int64_t cnt = g.count;
    int status = 0;
    const double tol1 = o.tol;

    // ---- load history (calculatePlasticity.cc:28-35)
    const M3 FP_t = load_soa3(g.Fp_c, cnt, i);
    for (int a = 0; a < n; ++a) {
        w.s[a] = g.s_c[(int64_t)a * cnt + i];
        w.W[a] = g.W_c[(int64_t)a * cnt + i];
    }
    const double r0 = g.rot_c[i], r1 = g.rot_c[cnt + i], r2 = g.rot_c[2 * cnt + i];

    // ---- rotation and rotated stiffness (:39-77)
    const M3 R = odfpoint(r0, r1, r2);
    const Sym6 D2 = elasticmoduli(R, L.C);

    // W_kh_t (the increment-start backstress) is needed for the tangent signs
    // (:596,:697,:704,:788); keep the trial signs relative to it.
    unsigned long long neg_t_bits = 0ull;  // bit a: (tau_trial_a - W_kh_t_a) < 0, for a < 64

    M3 FP_tau = FP_t;
    M3 Fpn_inv = inv(FP_t);
    M3 FE_tau = mul(F, Fpn_inv);
    M3 FP_t2 = FP_tau, CE_tr = zero3(), Tst = zero3(), Tst_tr = zero3(), Ce_tau = zero3(), del_FP = zero3();
    M3 T_tau, P_tau;
    double dFp[81];
    bool dFp_nonzero = false;
    int nPA = 0, p0 = -1, rounds_total = 0, e_terms = 0, c_terms = 0;
    double maxcond = 1.0;
    int iter1 = 1;

    while (true) {
        if (iter1 > o.max_search) {
            status |= QP_SLIP_SEARCH_CAP;
            break;
        }
        // ---- trial kinematics and stress (:160-196)
        FP_t2 = FP_tau;
        Fpn_inv = inv(FP_t2);
        const M3 FE_tr = mul(F, Fpn_inv);
        CE_tr = mulTN(FE_tr, FE_tr);
        M3 Ee = CE_tr;
        Ee(0, 0) -= 1.0;
        Ee(1, 1) -= 1.0;
        Ee(2, 2) -= 1.0;
        Ee = scale(0.5, Ee);
        Tst_tr = voigt_apply(D2, Ee);
        Tst = Tst_tr;
        {
            const double dFe = det(FE_tau);
            const M3 t = scale(1.0 / dFe, mul(FE_tau, Tst_tr));
            T_tau = mulNT(t, FE_tau);
            P_tau = scale(dFe, mulNT(T_tau, inv(F)));
        }
        // ---- resolved shears and the potentially active set (:199-244)
        const M3 X = mul(CE_tr, Tst_tr);
        const M3 Xc = mulTN(R, mul(X, R));
        nPA = 0;
        for (int a = 0; a < n; ++a) {
            double t = resolved(L, a, Xc);
            if (a > ns - 1 && (t - w.W[a]) < 0) t = w.W[a];
            w.tau_tr[a] = t;
            w.b[a] = fabs(t - w.W[a]) - w.s[a];
            if (w.b[a] >= tol1) {
                if (nPA < PMAX) {
                    w.pa[nPA] = (unsigned char)a;
                } else {
                    status |= QP_ACTIVE_OVERFLOW;
                }
                ++nPA;
            }
        }
        if (nPA > PMAX) nPA = PMAX;
        if (p0 < 0) p0 = nPA;
        if (nPA == 0) break;
        // signs relative to the increment-start backstress W_kh_t, as the
        // tangent uses them (:596,:697,:704,:788), for this pass's trial shears
        neg_t_bits = 0ull;
        for (int k = 0; k < nPA; ++k) {
            const int a = w.pa[k];
            if ((w.tau_tr[a] - g.W_c[(int64_t)a * cnt + i]) < 0) neg_t_bits |= (1ull << a);
        }
        const int p_init = nPA;
        for (int k = 0; k < p_init; ++k) w.pa0[k] = w.pa[k];

        // ---- hardening moduli h_beta of the PA systems (:252-262), A[PA,PA] (:265-306)
        for (int k = 0; k < p_init; ++k) {
            const int a = w.pa[k];
            w.h[k] = ldg(&L.h0[a]) * pow((1 - w.s[a] / ldg(&L.ss[a])), ldg(&L.a[a]));
            schmid_vectors(L, a, R, w.Sv + 6 * k);
        }
        for (int kj = 0; kj < p_init; ++kj) {
            const int bsys = w.pa[kj];
            const M3 Sj = schmid_of(w.Sv + 6 * kj);
            const M3 Y = sym(mul(CE_tr, Sj));
            M3 Mj = mul(CE_tr, voigt_apply(D2, Y));
            axpy(Mj, 2.0, mul(Y, Tst_tr));
            const double dj = w.tau_tr[bsys] - w.W[bsys];
            // column kj of A; rows use S_i : Mj
            for (int ki = 0; ki < p_init; ++ki) {
                const int asys = w.pa[ki];
                const double di = w.tau_tr[asys] - w.W[asys];
                const double sm = schmid_dot(w.Sv + 6 * ki, Mj);
                double v = ldg(&L.q[asys * NM + bsys]) * w.h[kj];
                v += (di * dj < 0.0) ? -sm : sm;
                const double kin = ldg(&L.C1[asys]) - ldg(&L.C2[asys]) * w.W[asys];
                v += (di < 0.0) ? -kin : kin;
                w.A[ki * PMAX + kj] = v;
            }
        }

        // ---- consistency iterations (:311-448)
        for (int k = 0; k < p_init; ++k) w.x_old[k] = 0.0;  // x_old indexed by position in pa0
        int count1 = 0;
        // cur[k]: 1 if pa0[k] is still in PA
        for (int k = 0; k < p_init; ++k) w.cur[k] = 1;
        auto bpa_norm = [&]() {
            double mx = 0.0;
            for (int k = 0; k < p_init; ++k)
                if (w.cur[k]) mx = fmax(mx, fabs(w.b[w.pa0[k]]));
            return mx;
        };
        while (bpa_norm() > tol1) {
            count1 += 1;
            if (count1 > o.max_solver) break;
            // inactive_slip_removal (inactiveSlipRemoval.cc:4-124)
            for (int k = 0; k < p_init; ++k) w.x[k] = 0.0;
            for (;;) {
                // gather the current PA block and right-hand side
                int m = 0;
                for (int k = 0; k < p_init; ++k)
                    if (w.cur[k]) w.pa[m++] = (unsigned char)k;  // pa holds positions into pa0 here
                for (int r = 0; r < m; ++r) {
                    const int kr = w.pa[r];
                    w.rhs[r] = w.b[w.pa0[kr]];
                    for (int c = 0; c < m; ++c) w.Apa[r * PMAX + c] = w.A[kr * PMAX + w.pa[c]];
                }
                double cnd = 1.0;
                if (lu_solve(w.Apa, m, PMAX, w.rhs, 1, 1, &cnd)) status |= QP_SINGULAR;
                maxcond = fmax(maxcond, cnd);
                ++rounds_total;
                for (int k = 0; k < p_init; ++k) w.x[k] = 0.0;
                for (int r = 0; r < m; ++r) w.x[w.pa[r]] = w.rhs[r];
                bool removed = false;
                for (int k = 0; k < p_init; ++k)
                    if (w.cur[k] && (w.x_old[k] + w.x[k]) < 0) {
                        w.cur[k] = 0;
                        removed = true;
                    }
                // systems outside PA have x = 0 and x_old >= 0 (accumulated from
                // non-negative totals), so they never trigger a removal
                if (!removed) break;
            }
            for (int k = 0; k < p_init; ++k) w.x_old[k] += w.x[k];
            nPA = 0;
            for (int k = 0; k < p_init; ++k) nPA += w.cur[k];

            // del_FP = sum +-x_old S (:337-357)
            del_FP = zero3();
            for (int k = 0; k < p_init; ++k) {
                if (w.x_old[k] == 0.0) continue;
                const int a = w.pa0[k];
                const double sgn = ((w.tau_tr[a] - w.W[a]) > 0) ? w.x_old[k] : -w.x_old[k];
                axpy(del_FP, sgn, schmid_of(w.Sv + 6 * k));
            }
            FP_tau = mul(matexp(del_FP, &e_terms, &status), FP_t2);
            // (:361-396)
            FE_tau = mul(F, inv(FP_tau));
            Ce_tau = mulTN(FE_tau, FE_tau);
            M3 E2 = Ce_tau;
            E2(0, 0) -= 1.0;
            E2(1, 1) -= 1.0;
            E2(2, 2) -= 1.0;
            E2 = scale(0.5, E2);
            Tst = voigt_apply(D2, E2);
            const M3 Xn = mul(Ce_tau, Tst);
            const M3 Xnc = mulTN(R, mul(Xn, R));
            // resolved shears of the PA systems, twin clamp against the
            // backstress before this iteration's update (:380-396)
            for (int k = 0; k < p_init; ++k) {
                if (!w.cur[k]) continue;
                const int a = w.pa0[k];
                double t = resolved(L, a, Xnc);
                if (a > ns - 1 && (w.tau_tr[a] - w.W[a]) < 0) t = w.W[a];
                w.tn[k] = t;
            }
            // hardening (:399-429): s_a += sum_j q_aj h_j x_j over the PA systems
            for (int a = 0; a < n; ++a) {
                double h1 = 0.0;
                for (int k = 0; k < p_init; ++k)
                    if (w.x[k] != 0.0) h1 += ldg(&L.q[a * NM + w.pa0[k]]) * w.h[k] * w.x[k];
                double sv = w.s[a] + h1;
                const double sat = ldg(&L.ss[a]);
                if (sv > sat) sv = sat;
                w.s[a] = sv;
            }
            // backstress (:431-436), then b on the PA systems (:438-446)
            for (int k = 0; k < p_init; ++k) {
                const int a = w.pa0[k];
                if ((w.tau_tr[a] - w.W[a]) > 0)
                    w.W[a] = w.W[a] + (ldg(&L.C1[a]) - ldg(&L.C2[a]) * w.W[a]) * w.x[k];
                else
                    w.W[a] = w.W[a] + (-ldg(&L.C1[a]) - ldg(&L.C2[a]) * w.W[a]) * w.x[k];
            }
            for (int k = 0; k < p_init; ++k) {
                if (!w.cur[k]) continue;
                const int a = w.pa0[k];
                w.b[a] = fabs(w.tn[k] - w.W[a]) - w.s[a];
            }
        }

        // ---- fractions (:450-456), written only on this branch
        for (int t = 0; t < nw; ++t) {
            double xo = 0.0;
            for (int k = 0; k < p_init; ++k)
                if (w.pa0[k] == ns + t) xo = w.x_old[k];
            g.tw_i[(int64_t)t * cnt + i] = g.tw_c[(int64_t)t * cnt + i] + xo / L.twin_shear;
        }
        for (int t = 0; t < ns; ++t) {
            double xo = 0.0;
            for (int k = 0; k < p_init; ++k)
                if (w.pa0[k] == t) xo = w.x_old[k];
            g.sl_i[(int64_t)t * cnt + i] = g.sl_c[(int64_t)t * cnt + i] + xo;
        }

        // ---- stresses at the updated state (:458-468)
        Fpn_inv = inv(FP_tau);
        FE_tau = mul(F, Fpn_inv);
        {
            const double dFe = det(FE_tau);
            const M3 t = scale(1.0 / dFe, mul(FE_tau, Tst));
            T_tau = mulNT(t, FE_tau);
            P_tau = scale(det(F), mulNT(T_tau, inv(F)));
        }

        if (flag == 1) {
            // ---- tangent inside the slip-search loop (:473-828)
            // final active set, in pa0 order
            int act[PMAX];
            int p = 0;
            for (int k = 0; k < p_init; ++k)
                if (w.cur[k]) act[p++] = k;
            // delb_delF (p x 9) into rhs: column kl of d tau / dF contracted with S
            for (int kl = 0; kl < 9; ++kl) {
                const int kk = kl / 3, l = kl % 3;
                M3 dFe;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int j = 0; j < 3; ++j) dFe(a, j) = (a == kk) ? Fpn_inv(l, j) : 0.0;
                if (dFp_nonzero) {
                    M3 X1;
#pragma unroll
                    for (int c = 0; c < 9; ++c) X1.a[c] = dFp[c * 9 + kl];
                    const M3 t = mul(mul(FE_tau, X1), Fpn_inv);
#pragma unroll
                    for (int c = 0; c < 9; ++c) dFe.a[c] -= t.a[c];
                }
                const M3 G = mulTN(dFe, FE_tau);  // G(i,j) = sum_a dFe(a,i) Fe(a,j)
                M3 dE;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) dE(a, b) = 0.5 * (G(a, b) + G(b, a));
                const M3 dT = voigt_apply(D2, dE);
                M3 dtau = mul(Ce_tau, dT);
                axpy(dtau, 2.0, mul(dE, Tst));
                for (int r = 0; r < p; ++r) {
                    const int k = act[r];
                    double v = schmid_dot(w.Sv + 6 * k, dtau);
                    if (neg_t_bits >> w.pa0[k] & 1ull) v = -v;
                    w.rhs[r * 9 + kl] = v;
                }
            }
            // count3 (:607-619)
            {
                double tol2 = 1.0;
                int count3 = 0;
                M3 t2 = eye3();
                const double lim = fmax(tol1 / 1e4, 1e-12);
                while (tol2 > lim) {
                    if (count3 >= GATEAUX_TERM_CAP) {
                        status |= QP_SERIES_CAP;
                        break;
                    }
                    count3 += 1;
                    M3 t1 = scale(1.0 / count3, mul(del_FP, t2));
                    tol2 = frob(t1);
                    t2 = t1;
                }
                c_terms = count3;
            }
            // A2 (:622-709) into Apa, S_PA columns (:734-796) into A's spare rows
            const M3 X6 = mul(CE_tr, matexp(scale(-1.0, del_FP), nullptr, &status));
            double SPA[9 * PMAX];
            for (int cj = 0; cj < p; ++cj) {
                const int kj = act[cj];
                const int bsys = w.pa0[kj];
                const M3 Sj = schmid_of(w.Sv + 6 * kj);
                M3 dm, dp;
                gateaux_pair(Sj, del_FP, c_terms, dm, dp);
                const M3 Y = sym(mulTN(dm, X6));
                M3 Mj = mul(Ce_tau, voigt_apply(D2, Y));
                axpy(Mj, 2.0, mul(Y, Tst));
                const bool nj = (neg_t_bits >> bsys) & 1ull;
                for (int ci = 0; ci < p; ++ci) {
                    const int ki = act[ci];
                    const int asys = w.pa0[ki];
                    const bool ni = (neg_t_bits >> asys) & 1ull;
                    const double sm = schmid_dot(w.Sv + 6 * ki, Mj);
                    double v = ldg(&L.q[asys * NM + bsys]) * w.h[kj];
                    v += (ni ^ nj) ? -sm : sm;
                    const double kin = ldg(&L.C1[asys]) - ldg(&L.C2[asys]) * w.W[asys];
                    v += ni ? -kin : kin;
                    w.Apa[ci * PMAX + cj] = v;
                }
                const M3 spa = mul(dp, FP_t2);
#pragma unroll
                for (int c = 0; c < 9; ++c) SPA[c * PMAX + cj] = nj ? -spa.a[c] : spa.a[c];
            }
            // delgamma_delF = A2^{-1} delb_delF (:712-729)
            if (lu_solve(w.Apa, p, PMAX, w.rhs, 9, 9)) status |= QP_SINGULAR;
            // delFp_delF = exp(del_FP) delFp_delF_prev + S_PA delgamma (:799-821)
            double nd[81];
            if (dFp_nonzero) {
                const M3 ex = matexp(del_FP, nullptr, &status);
                for (int a = 0; a < 3; ++a)
                    for (int j = 0; j < 3; ++j)
                        for (int kl = 0; kl < 9; ++kl)
                            nd[(3 * a + j) * 9 + kl] = ex(a, 0) * dFp[(0 + j) * 9 + kl] + ex(a, 1) * dFp[(3 + j) * 9 + kl] +
                                                       ex(a, 2) * dFp[(6 + j) * 9 + kl];
            } else {
                for (int c = 0; c < 81; ++c) nd[c] = 0.0;
            }
            for (int r = 0; r < 9; ++r)
                for (int kl = 0; kl < 9; ++kl) {
                    double s = 0.0;
                    for (int c = 0; c < p; ++c) s += SPA[r * PMAX + c] * w.rhs[c * 9 + kl];
                    nd[r * 9 + kl] += s;
                }
            for (int c = 0; c < 81; ++c) dFp[c] = nd[c];
            dFp_nonzero = true;
        }
        ++iter1;
    }

    // ---- final tangent (:835-940)
    if (flag == 1 && out.dPdF) {
        const M3 Finv = inv(F);
        const M3 t1 = mulNT(Tst, mul(Finv, FE_tau));  // T* (F^-1 Fe)^T
        const M3 t2 = mul(Finv, FE_tau);
        const M3 t3 = mul(FE_tau, Tst);
        const M3 t5 = mulNT(t3, F);
        const M3 Z = mulNT(t5, Finv);  // Z(i,l) = sum_a t5(i,a) Finv(l,a)
        for (int kl = 0; kl < 9; ++kl) {
            const int kk = kl / 3, l = kl % 3;
            M3 dFe;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int j = 0; j < 3; ++j) dFe(a, j) = (a == kk) ? Fpn_inv(l, j) : 0.0;
            if (dFp_nonzero) {
                M3 X1;
#pragma unroll
                for (int c = 0; c < 9; ++c) X1.a[c] = dFp[c * 9 + kl];
                const M3 t = mul(mul(FE_tau, X1), Fpn_inv);
#pragma unroll
                for (int c = 0; c < 9; ++c) dFe.a[c] -= t.a[c];
            }
            // dT*(ij) = sum_ab TM(ij,ab) (dFe^T Fe)(a,b)
            const M3 Y = mulTN(dFe, FE_tau);
            M3 Ys;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) Ys(a, b) = 0.5 * (Y(a, b) + Y(b, a));
            const M3 dTs = voigt_apply(D2, Ys);
            M3 PK = mul(dFe, t1);
            axpy(PK, 1.0, mulNT(mul(FE_tau, dTs), t2));
            axpy(PK, -1.0, mulNT(mul(t3, dFe), Finv));
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int j = 0; j < 3; ++j) PK(a, j) -= Finv(j, kk) * Z(a, l);
#pragma unroll
            for (int c = 0; c < 9; ++c) out.dPdF[c * 9 + kl] = out.scale * PK.a[c];
        }
    }

    // ---- outputs and history (:942-959)
    if (out.P)
#pragma unroll
        for (int c = 0; c < 9; ++c) out.P[c] = out.scale * P_tau.a[c];
    if (out.T)
#pragma unroll
        for (int c = 0; c < 9; ++c) out.T[c] = T_tau.a[c];
    store_soa3(g.Fe_i, cnt, i, FE_tau);
    store_soa3(g.Fp_i, cnt, i, FP_tau);
    for (int a = 0; a < n; ++a) {
        g.s_i[(int64_t)a * cnt + i] = w.s[a];
        g.W_i[(int64_t)a * cnt + i] = w.W[a];
    }

    // ---- twin reorientation (:962-1019)
    if (L.twinning) {
        double F_T;
        if (!o.multiphase)
            F_T = (F_r > 0) ? L.twin_thr + (L.twin_sat * F_e / F_r) : L.twin_thr;
        else
            F_T = L.twin_thr;
        if (F_T > 1.0) F_T = 1.0;
        int pos = 0;
        double tmax = g.tw_i[i];
        for (int t = 1; t < nw; ++t) {
            const double v = g.tw_i[(int64_t)t * cnt + i];
            if (v > tmax) {
                tmax = v;
                pos = t;
            }
        }
        if (g.twin_c[i] != 1 && F_r > 0 && tmax > F_T) {
            double rr[3];
            twin_rotation(L, ns + pos, r0, r1, r2, rr);
            for (int t = 0; t < 3; ++t) {
                g.rot_i[(int64_t)t * cnt + i] = rr[t];
                g.rotnew_i[(int64_t)t * cnt + i] = rr[t];
            }
            g.twin_i[i] = 1;
            for (int t = 0; t < nw; ++t) g.s_i[(int64_t)(ns + t) * cnt + i] = 100000;
        }
    }

    bool finite = true;
#pragma unroll
    for (int c = 0; c < 9; ++c) finite = finite && isfinite(P_tau.a[c]);
    if (!finite) status |= QP_NONFINITE;
    if (maxcond > 1e12) status |= QP_ILL_CONDITIONED;
    if (stats_out) {
        stats_out[0] = p0 < 0 ? 0 : p0;
        stats_out[1] = nPA;
        stats_out[2] = rounds_total;
        stats_out[3] = e_terms;
        stats_out[4] = c_terms;
        stats_out[5] = iter1;
        stats_out[6] = lattice_id;
        stats_out[7] = maxcond >= 1e99 ? 99 : (int)ceil(log10(maxcond));
    }
    return status;
}

}  // namespace cp
