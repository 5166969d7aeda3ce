// cp_qp2.cuh -- the per-qp constitutive update with compact per-thread state
// (the optimised form of cp_qp.cuh's qp_update; same math, same order of the
// reference's steps, see cp_qp.cuh's header for the restatements).
//
// Differences from the plain form, all about where intermediate values live:
//   * no per-thread arrays over all n systems: the per-system loops read the
//     history straight from the structure-of-arrays group (coalesced across a
//     warp), and the _iter arrays of CRSS and backstress are the working
//     storage of the current values (initialised from _conv on entry);
//   * per-thread arrays are compact over the potentially active set of the
//     current pass (capacity PMAX), so the touched scratch grows with p0^2, not
//     PMAX^2.  The matrices that are solved (removal rounds, tangent) use the
//     row stride PMAX, not their size: local memory is interleaved across the
//     lanes of a warp and coalesces only when every lane addresses the same
//     relative offset, which a fixed stride keeps true while the lanes' active
//     sets shrink to different sizes;
//   * qps arrive sorted by potentially-active-set size (classify_kernel +
//     counting sort), so the threads of a warp run solves of similar size.
#pragma once

#include "cp_qp.cuh"

namespace cp {

// Per-thread scratch of qp_update2: each array is its own local variable and
// this struct only points at them.  Arrays that are fields of one local
// struct, indexed at run time, may alias as far as the compiler can tell, so
// every scratch store would order the loads after it; distinct variables
// cannot alias, which leaves it free to batch loads.
struct Scratch2 {
    unsigned char *pa0, *cur, *pos;
    double *tau_tr, *b, *h, *x_old, *x, *tn, *kin;
    double* A;    // S_PA of the tangent, 9 rows of leading dimension PMAX
    double* Apa;  // the matrix being solved, leading dimension PMAX
    double* rhs;  // right-hand sides, 9 per row
};

// a_i[c] -= f a_j[c] for c in [c0, m) on two distinct rows of one matrix.
// Four columns per step, all loads before the stores: with rows of one array
// the compiler must otherwise assume a store may feed the next load and runs
// the loop one memory round trip per column.  Same operation per element.
__host__ __device__ __forceinline__ void row_axpy(double* ai, const double* aj, double f, int c0, int m) {
    int c = c0;
    for (; c + 4 <= m; c += 4) {
        const double x0 = aj[c], x1 = aj[c + 1], x2 = aj[c + 2], x3 = aj[c + 3];
        const double y0 = ai[c], y1 = ai[c + 1], y2 = ai[c + 2], y3 = ai[c + 3];
        ai[c] = y0 - f * x0;
        ai[c + 1] = y1 - f * x1;
        ai[c + 2] = y2 - f * x2;
        ai[c + 3] = y3 - f * x3;
    }
    for (; c < m; ++c) ai[c] -= f * aj[c];
}
// The same on four rows i0..i0+3 at once (row stride ld): the pivot row's
// columns are loaded once per step and all 16 row entries before any store.
__host__ __device__ __forceinline__ void rows4_axpy(double* a, int ld, const double* aj, const double f[4], int c0,
                                                   int m) {
    double* a0 = a;
    double* a1 = a + ld;
    double* a2 = a + 2 * ld;
    double* a3 = a + 3 * ld;
    int c = c0;
    for (; c + 4 <= m; c += 4) {
        double x[4], y0[4], y1[4], y2[4], y3[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x[u] = aj[c + u];
            y0[u] = a0[c + u];
            y1[u] = a1[c + u];
            y2[u] = a2[c + u];
            y3[u] = a3[c + u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0[c + u] = y0[u] - f[0] * x[u];
            a1[c + u] = y1[u] - f[1] * x[u];
            a2[c + u] = y2[u] - f[2] * x[u];
            a3[c + u] = y3[u] - f[3] * x[u];
        }
    }
    for (; c < m; ++c) {
        const double x = aj[c];
        const double y0 = a0[c], y1 = a1[c], y2 = a2[c], y3 = a3[c];
        a0[c] = y0 - f[0] * x;
        a1[c] = y1 - f[1] * x;
        a2[c] = y2 - f[2] * x;
        a3[c] = y3 - f[3] * x;
    }
}

__host__ __device__ __forceinline__ void row_swap(double* a, double* b, int m) {
    int c = 0;
    for (; c + 4 <= m; c += 4) {
        const double x0 = a[c], x1 = a[c + 1], x2 = a[c + 2], x3 = a[c + 3];
        const double y0 = b[c], y1 = b[c + 1], y2 = b[c + 2], y3 = b[c + 3];
        a[c] = y0, a[c + 1] = y1, a[c + 2] = y2, a[c + 3] = y3;
        b[c] = x0, b[c + 1] = x1, b[c + 2] = x2, b[c + 3] = x3;
    }
    for (; c < m; ++c) {
        const double t = a[c];
        a[c] = b[c];
        b[c] = t;
    }
}

// Two elimination steps j, j+1 on rows i0..i0+3 (row stride ld), columns
// [c0, m): a_i[c] = (a_i[c] - f_i p[c]) - g_i q[c], with p, q the pivot rows
// of steps j and j+1.  Each element sees the two subtractions of the
// one-step-at-a-time elimination in the same order, but is loaded and stored
// once for both.
__host__ __device__ __forceinline__ void rows4_axpy2(double* a, int ld, const double* p, const double* q,
                                                    const double f[4], const double g[4], int c0, int m) {
    double* a0 = a;
    double* a1 = a + ld;
    double* a2 = a + 2 * ld;
    double* a3 = a + 3 * ld;
    int c = c0;
    for (; c + 2 <= m; c += 2) {
        double x[2], z[2], y0[2], y1[2], y2[2], y3[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            x[u] = p[c + u];
            z[u] = q[c + u];
            y0[u] = a0[c + u];
            y1[u] = a1[c + u];
            y2[u] = a2[c + u];
            y3[u] = a3[c + u];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            a0[c + u] = (y0[u] - f[0] * x[u]) - g[0] * z[u];
            a1[c + u] = (y1[u] - f[1] * x[u]) - g[1] * z[u];
            a2[c + u] = (y2[u] - f[2] * x[u]) - g[2] * z[u];
            a3[c + u] = (y3[u] - f[3] * x[u]) - g[3] * z[u];
        }
    }
    for (; c < m; ++c) {
        const double x = p[c], z = q[c];
        const double y0 = a0[c], y1 = a1[c], y2 = a2[c], y3 = a3[c];
        a0[c] = (y0 - f[0] * x) - g[0] * z;
        a1[c] = (y1 - f[1] * x) - g[1] * z;
        a2[c] = (y2 - f[2] * x) - g[2] * z;
        a3[c] = (y3 - f[3] * x) - g[3] * z;
    }
}

// lu_solve (cp_qp.cuh) with the batched row operations above and NRHS known
// at compile time: Gaussian elimination with partial pivoting on the rows,
// same pivots and same arithmetic per element, so the same results.
//
// With PAIR, steps are taken two at a time where both pivots are non-zero
// (worth it for the larger solves only): column j+1 and row j+1 receive step
// j's update first so that pivot j+1 is chosen on the same values, and the
// rest of the trailing matrix then takes both updates in one pass.  Step j's
// multiplier of row i is recomputed as a_i[j] times the pivot's reciprocal
// wherever it is used (the same product each time).  A row swap of step j+1 before step j's update
// of the columns right of j+1 changes nothing: that update of a row uses only
// the row itself (its column j included, swapped with it) and pivot row j.
template <int NRHS, bool PAIR>
__host__ __device__ __forceinline__ int lu_solve_b(double* A, int m, int ld, double* B, double* cond = nullptr) {
    int sing = 0;
    double pmin = 1e308, pmax = 0.0;
    // pivot search of step j and its row swap; false for a zero column
    auto pivot = [&](int j) -> bool {
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
            return false;
        }
        if (r != j) {
            row_swap(A + j * ld, A + r * ld, m);
#pragma unroll
            for (int c = 0; c < NRHS; ++c) {
                const double t = B[j * NRHS + c];
                B[j * NRHS + c] = B[r * NRHS + c];
                B[r * NRHS + c] = t;
            }
        }
        return true;
    };
    // step j alone on rows [i, m), columns [c0, m), pivot reciprocal piv (a
    // zero multiplier leaves its row's finite entries unchanged, as skipping
    // it would)
    auto step1 = [&](int j, double piv, int i, int c0, const double* bj) {
        for (; i + 4 <= m; i += 4) {
            double f[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) f[r] = A[(i + r) * ld + j] * piv;
            rows4_axpy(A + i * ld, ld, A + j * ld, f, c0, m);
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < NRHS; ++c) B[(i + r) * NRHS + c] -= f[r] * bj[c];
        }
        for (; i < m; ++i) {
            const double f = A[i * ld + j] * piv;
            if (f == 0.0) continue;
            row_axpy(A + i * ld, A + j * ld, f, c0, m);
#pragma unroll
            for (int c = 0; c < NRHS; ++c) B[i * NRHS + c] -= f * bj[c];
        }
    };
    int j = 0;
    while (j < m) {
        if (!pivot(j)) {
            ++j;
            continue;
        }
        const double piv = 1.0 / A[j * ld + j];
        double bj[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) bj[c] = B[j * NRHS + c];
        if (!PAIR || j + 1 == m) {
            step1(j, piv, j + 1, j + 1, bj);
            ++j;
            continue;
        }
        // step j on column j+1, then the pivot of step j+1 on those values
        {
            const double u = A[j * ld + j + 1];
            for (int i = j + 1; i < m; ++i) A[i * ld + j + 1] = A[i * ld + j + 1] - (A[i * ld + j] * piv) * u;
        }
        if (!pivot(j + 1)) {
            step1(j, piv, j + 1, j + 2, bj);
            j += 2;
            continue;
        }
        // row j+1 takes the rest of step j; then both steps on the rows below
        const double f1 = A[(j + 1) * ld + j] * piv;
        if (f1 != 0.0) {
            row_axpy(A + (j + 1) * ld, A + j * ld, f1, j + 2, m);
#pragma unroll
            for (int c = 0; c < NRHS; ++c) B[(j + 1) * NRHS + c] -= f1 * bj[c];
        }
        const double piv1 = 1.0 / A[(j + 1) * ld + j + 1];
        double bj1[NRHS];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) bj1[c] = B[(j + 1) * NRHS + c];
        int i = j + 2;
        for (; i + 4 <= m; i += 4) {
            double f[4], g[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                f[r] = A[(i + r) * ld + j] * piv;
                g[r] = A[(i + r) * ld + j + 1] * piv1;
            }
            rows4_axpy2(A + i * ld, ld, A + j * ld, A + (j + 1) * ld, f, g, j + 2, m);
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < NRHS; ++c)
                    B[(i + r) * NRHS + c] = (B[(i + r) * NRHS + c] - f[r] * bj[c]) - g[r] * bj1[c];
        }
        for (; i < m; ++i) {
            const double f = A[i * ld + j] * piv;
            const double g = A[i * ld + j + 1] * piv1;
            double* ai = A + i * ld;
            const double* p = A + j * ld;
            const double* q = A + (j + 1) * ld;
            for (int c = j + 2; c < m; ++c) ai[c] = (ai[c] - f * p[c]) - g * q[c];
#pragma unroll
            for (int c = 0; c < NRHS; ++c) B[i * NRHS + c] = (B[i * NRHS + c] - f * bj[c]) - g * bj1[c];
        }
        j += 2;
    }
    for (int j = m - 1; j >= 0; --j) {
        const double d = A[j * ld + j];
#pragma unroll
        for (int c = 0; c < NRHS; ++c) {
            double s = B[j * NRHS + c];
            for (int k = j + 1; k < m; ++k) s -= A[j * ld + k] * B[k * NRHS + c];
            B[j * NRHS + c] = s / d;
        }
    }
    if (cond) *cond = m == 0 ? 1.0 : (pmin > 0.0 ? pmax / pmin : 1e308);
    return sing;
}

// Final tangent (:835-940) from the converged kinematics: for each kl,
// dFe = d(Fe)/dF_kl = E_kl Fp^-1 - Fe dFp_kl Fp^-1 (x1(kl, X) gives the
// column dFp_kl and returns false when dFp is zero), the stress derivative and
// the reference's PK_Stiff5 terms as written; dPdF[c * 9 + kl] = scale * PK.
template <class SymD, class X1Src>
__host__ __device__ __forceinline__ void final_tangent(const M3& F, const M3& FE_tau, const M3& Fpn_inv, const M3& Tst,
                                                       const SymD& D2, const X1Src& x1, double scale, double* dPdF) {
    const M3 Finv = inv(F);
    const M3 t1 = mulNT(Tst, mul(Finv, FE_tau));
    const M3 t2 = mul(Finv, FE_tau);
    const M3 t3 = mul(FE_tau, Tst);
    const M3 Z = mulNT(mulNT(t3, F), Finv);
    for (int kl = 0; kl < 9; ++kl) {
        const int kk = kl / 3, l = kl % 3;
        M3 dFe;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int j = 0; j < 3; ++j) dFe(a, j) = (a == kk) ? Fpn_inv(l, j) : 0.0;
        M3 X1;
        if (x1(kl, X1)) {
            const M3 t = mul(mul(FE_tau, X1), Fpn_inv);
#pragma unroll
            for (int c = 0; c < 9; ++c) dFe.a[c] -= t.a[c];
        }
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
        for (int c = 0; c < 9; ++c) dPdF[c * 9 + kl] = scale * PK.a[c];
    }
}

// Trial state of one slip-search pass (:160-196) and the potentially active
// set count; shared by classify_kernel and qp_update2.
struct Trial {
    M3 Fpn_inv, CE, Tst, Xc;
};

template <class SymD>
__host__ __device__ __forceinline__ Trial trial_state(const M3& F, const M3& FP, const SymD& D2, const M3& R) {
    Trial t;
    t.Fpn_inv = inv(FP);
    const M3 FE = mul(F, t.Fpn_inv);
    t.CE = mulTN(FE, FE);
    M3 Ee = t.CE;
    Ee(0, 0) -= 1.0;
    Ee(1, 1) -= 1.0;
    Ee(2, 2) -= 1.0;
    Ee = scale(0.5, Ee);
    t.Tst = voigt_apply(D2, Ee);
    t.Xc = mulTN(R, mul(mul(t.CE, t.Tst), R));
    return t;
}

// Potentially active systems at the increment start (first pass), the sort
// key of the update.
__host__ __device__ __forceinline__ int count_potentially_active(const LatDev& L, const Opts& o, const GroupDev& g,
                                                                  int64_t i, const M3& F) {
    const int64_t cnt = g.count;
    const int n = L.n, ns = L.ns;
    const M3 R = odfpoint(g.rot_c[i], g.rot_c[cnt + i], g.rot_c[2 * cnt + i]);
    const Sym6 D2 = elasticmoduli(R, L.C);
    const Trial t = trial_state(F, load_soa3(g.Fp_c, cnt, i), D2, R);
    int p0 = 0;
    for (int a = 0; a < n; ++a) {
        const double W = g.W_c[(int64_t)a * cnt + i];
        double tau = resolved(L, a, t.Xc);
        if (a > ns - 1 && (tau - W) < 0) tau = W;
        p0 += (fabs(tau - W) - g.s_c[(int64_t)a * cnt + i]) >= o.tol;
    }
    return p0;
}

template <int PMAX>
__host__ __device__ int qp_update2(const LatDev& L, const Opts& o, const GroupDev& g, int64_t i, const M3& F, int flag,
                                   double F_e, double F_r, const QpOut& out, int32_t* stats_out, int lattice_id,
                                   double* d2_slot, int d2_stride) {
    constexpr bool kPairLU = PMAX > 32;  // paired elimination steps for the BCC-sized solves
    unsigned char pa0_[PMAX], cur_[PMAX], pos_[PMAX];
    double tau_tr_[PMAX], b_[PMAX], h_[PMAX], x_old_[PMAX], x_[PMAX], tn_[PMAX], kin_[PMAX];
    double A_[9 * PMAX], Apa_[PMAX * PMAX], rhs_[PMAX * 9];
    const Scratch2 w{pa0_, cur_, pos_, tau_tr_, b_, h_, x_old_, x_, tn_, kin_, A_, Apa_, rhs_};
    const int n = L.n, ns = L.ns, nw = L.nw;
    const int64_t cnt = g.count;
    int status = 0;
    const double tol1 = o.tol;
    double* __restrict__ s_cur = g.s_i;  // current CRSS of every system, [a * cnt + i]
    double* __restrict__ W_cur = g.W_i;  // current backstress

    // ---- history (:28-35): the _iter CRSS/backstress start as the _conv
    // values; the first pass's potentially-active-set loop copies them as it
    // reads them (here only when there is no pass at all)
    if (o.max_search < 1)
        for (int a = 0; a < n; ++a) {
            s_cur[(int64_t)a * cnt + i] = g.s_c[(int64_t)a * cnt + i];
            W_cur[(int64_t)a * cnt + i] = g.W_c[(int64_t)a * cnt + i];
        }
    const double r0 = g.rot_c[i], r1 = g.rot_c[cnt + i], r2 = g.rot_c[2 * cnt + i];
    const M3 R = odfpoint(r0, r1, r2);
    // the rotated stiffness lives in the caller's slot (shared memory in the
    // kernel: 21 doubles that would otherwise hold registers all along)
    {
        const Sym6 D2v = elasticmoduli(R, L.C);
#pragma unroll
        for (int e = 0; e < 21; ++e) d2_slot[e * d2_stride] = D2v.c[e];
    }
    const Sym6Ref D2{d2_slot, d2_stride};

    unsigned long long neg_t_bits = 0ull;
    M3 FP_tau = load_soa3(g.Fp_c, cnt, i);
    M3 Fpn_inv = inv(FP_tau);
    M3 FE_tau = mul(F, Fpn_inv);
    M3 FP_t2 = FP_tau, CE_tr = zero3(), Tst = zero3(), Ce_tau = zero3(), del_FP = zero3();
    M3 T_tau, P_tau;
    double dFp[81];
    bool dFp_nonzero = false;
    // With one slip-search pass (the shipped setting) the final tangent reads
    // dFp = S_PA delgamma column by column from S_PA (kept in w.A) and
    // delgamma (kept in w.rhs) instead of materialising the 9x9 dFp.
    int lazy_p = -1;
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
        const Trial tr = trial_state(F, FP_t2, D2, R);
        Fpn_inv = tr.Fpn_inv;
        CE_tr = tr.CE;
        const M3 Tst_tr = tr.Tst;
        Tst = Tst_tr;
        {
            const double dFe = det(FE_tau);
            const M3 t = scale(1.0 / dFe, mul(FE_tau, Tst_tr));
            T_tau = mulNT(t, FE_tau);
            P_tau = scale(dFe, mulNT(T_tau, inv(F)));
        }
        // ---- resolved shears, potentially active set (:199-244), compact
        // (four systems' history loads in flight at a time: a load after a
        // store to the same arrays would otherwise wait for it)
        // The row constants of the consistency matrix (:252-306) are formed as
        // each PA member is found, from the CRSS and backstress in registers:
        // h_beta in w.h[k]; bit k of neg_d is the sign of tau_tr - W of PA
        // entry k, w.kin[k] the signed kinematic term of its row (the
        // reference's sign test di * dj < 0 equals neg_d_i != neg_d_j here,
        // since |tau_tr - W| >= s + tol > 0 for every PA member).  Bit a of
        // neg_t_bits is the sign of tau_tr - W at the increment start (the
        // same W in the first pass).
        nPA = 0;
        neg_t_bits = 0ull;
        unsigned long long neg_d = 0ull;
        for (int a0 = 0; a0 < n; a0 += 4) {
            double Wq[4], sq[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int a = a0 + u;
                if (a < n) {
                    if (iter1 == 1) {
                        Wq[u] = g.W_c[(int64_t)a * cnt + i];
                        sq[u] = g.s_c[(int64_t)a * cnt + i];
                    } else {
                        Wq[u] = W_cur[(int64_t)a * cnt + i];
                        sq[u] = s_cur[(int64_t)a * cnt + i];
                    }
                }
            }
            if (iter1 == 1)
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int a = a0 + u;
                    if (a < n) {
                        W_cur[(int64_t)a * cnt + i] = Wq[u];
                        s_cur[(int64_t)a * cnt + i] = sq[u];
                    }
                }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int a = a0 + u;
                if (a >= n) continue;
                const double W = Wq[u], sa = sq[u];
                double t = resolved(L, a, tr.Xc);
                if (a > ns - 1 && (t - W) < 0) t = W;
                const double bb = fabs(t - W) - sa;
                if (bb >= tol1) {
                    if (nPA < PMAX) {
                        const int k = nPA;
                        w.pa0[k] = (unsigned char)a;
                        w.tau_tr[k] = t;
                        w.b[k] = bb;
                        w.h[k] = ldg(&L.h0[a]) * pow((1 - sa / ldg(&L.ss[a])), ldg(&L.a[a]));
                        const double kin = ldg(&L.C1[a]) - ldg(&L.C2[a]) * W;
                        const bool ng = (t - W) < 0.0;
                        if (ng) neg_d |= (1ull << k);
                        if (ng && iter1 == 1) neg_t_bits |= (1ull << a);
                        w.kin[k] = ng ? -kin : kin;
                    } else {
                        status |= QP_ACTIVE_OVERFLOW;
                    }
                    ++nPA;
                }
            }
        }
        if (nPA > PMAX) nPA = PMAX;
        if (p0 < 0) p0 = nPA;
        if (nPA == 0) break;
        const int p_init = nPA;
        if (iter1 > 1)
            for (int k = 0; k < p_init; ++k) {
                const int a = w.pa0[k];
                if ((w.tau_tr[k] - g.W_c[(int64_t)a * cnt + i]) < 0) neg_t_bits |= (1ull << a);
            }

        // ---- A[PA,PA] (:265-306), packed p_init x p_init
        // A[PA,PA] is not stored: each removal round builds the rows and
        // columns of its current set straight into the matrix it solves
        // (same expression per entry, so the same values as a stored A).
        // Column j needs M_j = Ce [D2 : sym(Ce S_j)] + 2 sym(Ce S_j) T*; two
        // columns per pass, so each row's Schmid vectors are formed once per
        // pair.  The Schmid vectors R m, R n of a PA system are recomputed from
        // the lattice's constants (read-only, cached on chip) wherever they are
        // needed rather than kept per thread: the same values each time, and
        // 6 doubles per PA system less local memory.
        auto column_M = [&](int kj) {
            double svj[6];
            schmid_vectors(L, w.pa0[kj], R, svj);
            const M3 Sj = schmid_of(svj);
            const M3 Y = sym(mul(CE_tr, Sj));
            M3 Mj = mul(CE_tr, voigt_apply(D2, Y));
            axpy(Mj, 2.0, mul(Y, Tst_tr));
            return Mj;
        };
        auto build_active = [&](int m) {
            int c = 0;
            for (; c + 2 <= m; c += 2) {
                const int kj0 = w.pos[c], kj1 = w.pos[c + 1];
                const M3 M0 = column_M(kj0), M1 = column_M(kj1);
                const int b0 = w.pa0[kj0], b1 = w.pa0[kj1];
                const unsigned long long n0 = (neg_d >> kj0) & 1ull, n1 = (neg_d >> kj1) & 1ull;
                const double h0 = w.h[kj0], h1 = w.h[kj1];
                for (int r = 0; r < m; ++r) {
                    const int ki = w.pos[r];
                    const int asys = w.pa0[ki];
                    double sv[6];
                    schmid_vectors(L, asys, R, sv);
                    const unsigned long long ni = (neg_d >> ki) & 1ull;
                    const double kin = w.kin[ki];
                    const double sm0 = schmid_dot(sv, M0), sm1 = schmid_dot(sv, M1);
                    double v0 = ldg(&L.q[asys * NM + b0]) * h0;
                    double v1 = ldg(&L.q[asys * NM + b1]) * h1;
                    v0 += (ni ^ n0) ? -sm0 : sm0;
                    v1 += (ni ^ n1) ? -sm1 : sm1;
                    v0 += kin;
                    v1 += kin;
                    w.Apa[r * PMAX + c] = v0;
                    w.Apa[r * PMAX + c + 1] = v1;
                }
            }
            for (; c < m; ++c) {
                const int kj = w.pos[c];
                const int bsys = w.pa0[kj];
                const M3 Mj = column_M(kj);
                const unsigned long long nj = (neg_d >> kj) & 1ull;
                const double hj = w.h[kj];
                for (int r = 0; r < m; ++r) {
                    const int ki = w.pos[r];
                    const int asys = w.pa0[ki];
                    double svi[6];
                    schmid_vectors(L, asys, R, svi);
                    const double sm = schmid_dot(svi, Mj);
                    double v = ldg(&L.q[asys * NM + bsys]) * hj;
                    v += (((neg_d >> ki) & 1ull) ^ nj) ? -sm : sm;
                    v += w.kin[ki];
                    w.Apa[r * PMAX + c] = v;
                }
            }
        };

        // ---- consistency iterations (:311-448)
        for (int k = 0; k < p_init; ++k) {
            w.x_old[k] = 0.0;
            w.cur[k] = 1;
        }
        int count1 = 0;
        while (true) {
            double bmax = 0.0;
            for (int k = 0; k < p_init; ++k)
                if (w.cur[k]) bmax = fmax(bmax, fabs(w.b[k]));
            if (!(bmax > tol1)) break;
            count1 += 1;
            if (count1 > o.max_solver) break;
            // inactive_slip_removal (inactiveSlipRemoval.cc:4-124)
            for (;;) {
                int m = 0;
                for (int k = 0; k < p_init; ++k)
                    if (w.cur[k]) w.pos[m++] = (unsigned char)k;
                for (int r = 0; r < m; ++r) w.rhs[r] = w.b[w.pos[r]];
                build_active(m);
                double cnd = 1.0;
                if (lu_solve_b<1, kPairLU>(w.Apa, m, PMAX, w.rhs, &cnd)) status |= QP_SINGULAR;
                maxcond = fmax(maxcond, cnd);
                ++rounds_total;
                for (int k = 0; k < p_init; ++k) w.x[k] = 0.0;
                for (int r = 0; r < m; ++r) w.x[w.pos[r]] = w.rhs[r];
                bool removed = false;
                for (int k = 0; k < p_init; ++k)
                    if (w.cur[k] && (w.x_old[k] + w.x[k]) < 0) {
                        w.cur[k] = 0;
                        removed = true;
                    }
                if (!removed) break;
            }
            for (int k = 0; k < p_init; ++k) w.x_old[k] += w.x[k];
            nPA = 0;
            for (int k = 0; k < p_init; ++k) nPA += w.cur[k];

            // del_FP (:337-357)
            del_FP = zero3();
            for (int k = 0; k < p_init; ++k) {
                if (w.x_old[k] == 0.0) continue;
                const int a = w.pa0[k];
                const double sgn =
                    ((w.tau_tr[k] - W_cur[(int64_t)a * cnt + i]) > 0) ? w.x_old[k] : -w.x_old[k];
                double svk[6];
                schmid_vectors(L, a, R, svk);
                axpy(del_FP, sgn, schmid_of(svk));
            }
            FP_tau = mul(matexp(del_FP, &e_terms, &status), FP_t2);
            FE_tau = mul(F, inv(FP_tau));
            Ce_tau = mulTN(FE_tau, FE_tau);
            M3 E2 = Ce_tau;
            E2(0, 0) -= 1.0;
            E2(1, 1) -= 1.0;
            E2(2, 2) -= 1.0;
            E2 = scale(0.5, E2);
            Tst = voigt_apply(D2, E2);
            const M3 Xnc = mulTN(R, mul(mul(Ce_tau, Tst), R));
            for (int k = 0; k < p_init; ++k) {
                if (!w.cur[k]) continue;
                const int a = w.pa0[k];
                const double Wa = W_cur[(int64_t)a * cnt + i];
                double t = resolved(L, a, Xnc);
                if (a > ns - 1 && (w.tau_tr[k] - Wa) < 0) t = Wa;
                w.tn[k] = t;
            }
            // hardening of every system (:399-429).  Only systems with a
            // non-zero increment contribute; up to four of them (the usual
            // case) are gathered into registers once, in PA order, so the sum
            // over them is the same sequence of operations as the full loop.
            int nzc = 0, za0 = 0, za1 = 0, za2 = 0, za3 = 0;
            double zh0 = 0.0, zh1 = 0.0, zh2 = 0.0, zh3 = 0.0, zx0 = 0.0, zx1 = 0.0, zx2 = 0.0, zx3 = 0.0;
            for (int k = 0; k < p_init; ++k) {
                const double xk = w.x[k];
                if (xk == 0.0) continue;
                const int ak = w.pa0[k];
                const double hk = w.h[k];
                if (nzc == 0) {
                    za0 = ak; zh0 = hk; zx0 = xk;
                } else if (nzc == 1) {
                    za1 = ak; zh1 = hk; zx1 = xk;
                } else if (nzc == 2) {
                    za2 = ak; zh2 = hk; zx2 = xk;
                } else if (nzc == 3) {
                    za3 = ak; zh3 = hk; zx3 = xk;
                }
                ++nzc;
            }
            for (int a0 = 0; a0 < n; a0 += 4) {  // four systems' CRSS loads in flight at a time
                double sq[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (a0 + u < n) sq[u] = s_cur[(int64_t)(a0 + u) * cnt + i];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int a = a0 + u;
                    if (a >= n) continue;
                    double h1 = 0.0;
                    if (nzc <= 4) {
                        const double* qa = L.q + a * NM;
                        if (nzc > 0) h1 += ldg(&qa[za0]) * zh0 * zx0;
                        if (nzc > 1) h1 += ldg(&qa[za1]) * zh1 * zx1;
                        if (nzc > 2) h1 += ldg(&qa[za2]) * zh2 * zx2;
                        if (nzc > 3) h1 += ldg(&qa[za3]) * zh3 * zx3;
                    } else {
                        for (int k = 0; k < p_init; ++k)
                            if (w.x[k] != 0.0) h1 += ldg(&L.q[a * NM + w.pa0[k]]) * w.h[k] * w.x[k];
                    }
                    double sv = sq[u] + h1;
                    const double sat = ldg(&L.ss[a]);
                    if (sv > sat) sv = sat;
                    s_cur[(int64_t)a * cnt + i] = sv;
                }
            }
            // backstress (:431-436) and b (:438-446) of the PA systems
            // (one pass: each PA system's backstress is read once and its b
            // formed from the value just computed, the one stored)
            for (int k = 0; k < p_init; ++k) {
                const int a = w.pa0[k];
                const double W0 = W_cur[(int64_t)a * cnt + i];
                double Wa;
                if ((w.tau_tr[k] - W0) > 0)
                    Wa = W0 + (ldg(&L.C1[a]) - ldg(&L.C2[a]) * W0) * w.x[k];
                else
                    Wa = W0 + (-ldg(&L.C1[a]) - ldg(&L.C2[a]) * W0) * w.x[k];
                W_cur[(int64_t)a * cnt + i] = Wa;
                if (w.cur[k]) w.b[k] = fabs(w.tn[k] - Wa) - s_cur[(int64_t)a * cnt + i];
            }
        }

        // ---- fractions (:450-456)
        // Systems outside PA get _conv + 0, PA systems _conv + their total
        // increment (PA members are distinct systems).
        for (int t0 = 0; t0 < nw; t0 += 4) {  // four loads in flight at a time
            double c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t0 + u < nw) c[u] = g.tw_c[(int64_t)(t0 + u) * cnt + i];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t0 + u < nw) g.tw_i[(int64_t)(t0 + u) * cnt + i] = c[u] + 0.0;
        }
        for (int t0 = 0; t0 < ns; t0 += 4) {
            double c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t0 + u < ns) c[u] = g.sl_c[(int64_t)(t0 + u) * cnt + i];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (t0 + u < ns) g.sl_i[(int64_t)(t0 + u) * cnt + i] = c[u] + 0.0;
        }
        for (int k = 0; k < p_init; ++k) {
            const int a = w.pa0[k];
            if (a < ns)
                g.sl_i[(int64_t)a * cnt + i] = g.sl_c[(int64_t)a * cnt + i] + w.x_old[k];
            else
                g.tw_i[(int64_t)(a - ns) * cnt + i] = g.tw_c[(int64_t)(a - ns) * cnt + i] + w.x_old[k] / L.twin_shear;
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
            int p = 0;
            for (int k = 0; k < p_init; ++k)
                if (w.cur[k]) w.pos[p++] = (unsigned char)k;
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
                const M3 G = mulTN(dFe, FE_tau);
                M3 dE;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) dE(a, b) = 0.5 * (G(a, b) + G(b, a));
                const M3 dT = voigt_apply(D2, dE);
                M3 dtau = mul(Ce_tau, dT);
                axpy(dtau, 2.0, mul(dE, Tst));
                for (int r = 0; r < p; ++r) {
                    const int k = w.pos[r];
                    double svk[6];
                    schmid_vectors(L, w.pa0[k], R, svk);
                    double v = schmid_dot(svk, dtau);
                    if (neg_t_bits >> w.pa0[k] & 1ull) v = -v;
                    w.rhs[r * 9 + kl] = v;
                }
            }
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
            const M3 X6 = mul(CE_tr, matexp(scale(-1.0, del_FP), nullptr, &status));
            // S_PA (9 x p, :734-796): 9 rows of stride PMAX
            double* SPA = w.A;
            for (int cj = 0; cj < p; ++cj) {
                const int kj = w.pos[cj];
                const int bsys = w.pa0[kj];
                double svj[6];
                schmid_vectors(L, bsys, R, svj);
                const M3 Sj = schmid_of(svj);
                M3 dm, dp;
                gateaux_pair(Sj, del_FP, c_terms, dm, dp);
                const M3 Y = sym(mulTN(dm, X6));
                M3 Mj = mul(Ce_tau, voigt_apply(D2, Y));
                axpy(Mj, 2.0, mul(Y, Tst));
                const bool nj = (neg_t_bits >> bsys) & 1ull;
                for (int ci = 0; ci < p; ++ci) {
                    const int ki = w.pos[ci];
                    const int asys = w.pa0[ki];
                    const bool ni = (neg_t_bits >> asys) & 1ull;
                    double svi[6];
                    schmid_vectors(L, asys, R, svi);
                    const double sm = schmid_dot(svi, Mj);
                    double v = ldg(&L.q[asys * NM + bsys]) * w.h[kj];
                    v += (ni ^ nj) ? -sm : sm;
                    const double Wa = W_cur[(int64_t)asys * cnt + i];
                    const double kin = ldg(&L.C1[asys]) - ldg(&L.C2[asys]) * Wa;
                    v += ni ? -kin : kin;
                    w.Apa[ci * PMAX + cj] = v;
                }
                const M3 spa = mul(dp, FP_t2);
#pragma unroll
                for (int c = 0; c < 9; ++c) SPA[c * PMAX + cj] = nj ? -spa.a[c] : spa.a[c];
            }
            if (lu_solve_b<9, kPairLU>(w.Apa, p, PMAX, w.rhs)) status |= QP_SINGULAR;
            if (o.max_search == 1) {  // this is the last pass: keep S_PA and delgamma
                lazy_p = p;
                ++iter1;
                continue;
            }
            double nd[81];
            if (dFp_nonzero) {
                const M3 ex = matexp(del_FP, nullptr, &status);
                for (int a = 0; a < 3; ++a)
                    for (int j = 0; j < 3; ++j)
                        for (int kl = 0; kl < 9; ++kl)
                            nd[(3 * a + j) * 9 + kl] = ex(a, 0) * dFp[(0 + j) * 9 + kl] +
                                                       ex(a, 1) * dFp[(3 + j) * 9 + kl] +
                                                       ex(a, 2) * dFp[(6 + j) * 9 + kl];
            } else {
#pragma unroll
                for (int c = 0; c < 81; ++c) nd[c] = 0.0;
            }
            for (int r = 0; r < 9; ++r)
                for (int kl = 0; kl < 9; ++kl) {
                    double sacc = 0.0;
                    for (int c = 0; c < p; ++c) sacc += SPA[r * PMAX + c] * w.rhs[c * 9 + kl];
                    nd[r * 9 + kl] += sacc;
                }
#pragma unroll
            for (int c = 0; c < 81; ++c) dFp[c] = nd[c];
            dFp_nonzero = true;
        }
        ++iter1;
    }

    // ---- outputs and history (:942-959), written before the final tangent
    // so that P, T and Fp are not held through it; CRSS/backstress are
    // already in _iter
    if (out.P)
#pragma unroll
        for (int c = 0; c < 9; ++c) out.P[c] = out.scale * P_tau.a[c];
    if (out.T)
#pragma unroll
        for (int c = 0; c < 9; ++c) out.T[c] = T_tau.a[c];
    store_soa3(g.Fe_i, cnt, i, FE_tau);
    store_soa3(g.Fp_i, cnt, i, FP_tau);
    {
        bool finite = true;
#pragma unroll
        for (int c = 0; c < 9; ++c) finite = finite && isfinite(P_tau.a[c]);
        if (!finite) status |= QP_NONFINITE;
    }

    // ---- final tangent (:835-940)
    if (flag == 1 && out.dPdF) {
        const bool plastic = dFp_nonzero || lazy_p > 0;
        auto x1 = [&](int kl, M3& X1) -> bool {
            if (!plastic) return false;
            if (lazy_p > 0) {
#pragma unroll
                for (int c = 0; c < 9; ++c) {
                    double acc = 0.0;
                    for (int r = 0; r < lazy_p; ++r) acc += w.A[c * PMAX + r] * w.rhs[r * 9 + kl];
                    X1.a[c] = acc;
                }
            } else {
#pragma unroll
                for (int c = 0; c < 9; ++c) X1.a[c] = dFp[c * 9 + kl];
            }
            return true;
        };
        final_tangent(F, FE_tau, Fpn_inv, Tst, D2, x1, out.scale, out.dPdF);
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
            for (int t = 0; t < nw; ++t) s_cur[(int64_t)(ns + t) * cnt + i] = 100000;
        }
    }

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
