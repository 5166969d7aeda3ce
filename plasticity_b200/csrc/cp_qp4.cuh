// cp_qp4.cuh -- the per-qp constitutive update on four lanes per qp, with its
// scratch in shared memory (the quad form of cp_qp2.cuh's qp_update2; same
// math, same operation order per value, so the same bits).
//
// Why: the thread-per-qp update keeps its active-set matrix, right-hand sides
// and per-system vectors in per-thread local memory; at the 8-16 warps per SM
// its 3x3 state allows, that scratch spills out of L1 and L2 and every access
// waits on an L2 or DRAM round trip.  Here a quad of lanes shares one qp: the
// 3x3 kinematics run redundantly in the four lanes (same values in each), the
// work over systems, matrix rows and columns and tangent columns is split
// over the lanes, and the p0-sized scratch lives in a per-qp area of shared
// memory sized by the qp's potentially active set, so it is never evicted.
//
// Order of operations: every stored value is formed by the same expression
// as in qp_update2 (entries of the consistency and tangent matrices, the LU's
// element updates, hardening sums in PA order, the back substitution's dot
// products in index order).  Only the owner of each piece changes, which
// does not change a bit.  Sums whose order matters and that cannot be split
// (del_FP over the PA systems, the hardening gather) run in every lane.
//
// Scope: one slip-search pass (cp_options_t.max_slip_search_iterations = 1,
// the reference's default), where the tangent is the lazy S_PA / delgamma
// form.  Other settings take the thread-per-qp kernel.
#pragma once

#include "cp_qp2.cuh"

namespace cp {

// The four lanes of one qp: lane index within the quad, the quad's lane mask
// and the position of its lowest lane in the warp.
struct Quad {
    int l;
    unsigned mask;
    int base;
};

__device__ __forceinline__ void qsync(const Quad& q) { __syncwarp(q.mask); }

// Row stride of the solved matrices: odd, so that the lanes of a quad,
// working on different rows of one column, fall on different banks.
__host__ __device__ __forceinline__ int quad_ld(int P) { return P | 1; }

// Doubles of one qp's shared-memory area for capacity P (potentially active
// systems stored) and n systems, odd so that the areas of the eight quads of
// a warp start on different banks.  Layout: rotated stiffness (21), Schmid
// vectors (6P), hardening moduli h (P), backstress of the PA systems (P),
// CRSS and increment-start backstress of every system (2n), then a region used first by the removal rounds
// (matrix P*ld, right-hand side, tau_tr, b, x_old, x, tau_new, kin: P each)
// and then by the tangent (matrix, 9 right-hand sides and S_PA: 9P each),
// then the byte arrays pa0, cur, pos (P each) and the system -> PA slot map
// (n).
__host__ __device__ __forceinline__ int quad_area_doubles(int P, int n) {
    const int ld = quad_ld(P);
    const int a = 21 + 8 * P + 2 * n + P * ld + 18 * P + (3 * P + n + 7) / 8;
    return a | 1;
}

struct Area4 {
    double *D2, *Sv, *h, *WP, *sS, *WS;
    double *Apa, *rhs, *tau_tr, *b, *x_old, *x, *tn, *kin;  // removal rounds
    double *rhs9, *SPA;                                    // tangent (overlays the vectors)
    unsigned char *pa0, *cur, *pos, *kof;
    int ld;
};

__device__ __forceinline__ Area4 quad_carve(double* base, int P, int n) {
    Area4 w;
    w.ld = quad_ld(P);
    double* p = base;
    w.D2 = p;
    p += 21;
    w.Sv = p;
    p += 6 * P;
    w.h = p;
    p += P;
    w.WP = p;
    p += P;
    w.sS = p;
    p += n;
    w.WS = p;
    p += n;
    w.Apa = p;
    p += P * w.ld;
    double* v = p;
    w.rhs = v;
    w.tau_tr = v + P;
    w.b = v + 2 * P;
    w.x_old = v + 3 * P;
    w.x = v + 4 * P;
    w.tn = v + 5 * P;
    w.kin = v + 6 * P;
    w.rhs9 = v;
    w.SPA = v + 9 * P;
    p += 18 * P;
    unsigned char* c = reinterpret_cast<unsigned char*>(p);
    w.pa0 = c;
    w.cur = c + P;
    w.pos = c + 2 * P;
    w.kof = c + 3 * P;
    return w;
}

// Positions k < p with on[k] set, in ascending k, into pos; returns their count.
__device__ __forceinline__ int quad_compact(const unsigned char* on, int p, unsigned char* pos, const Quad& q) {
    int m = 0;
    for (int k0 = 0; k0 < p; k0 += 4) {
        const int k = k0 + q.l;
        const bool set = k < p && on[k];
        const unsigned bits = (__ballot_sync(q.mask, set) >> q.base) & 0xFu;
        if (set) pos[m + __popc(bits & ((1u << q.l) - 1u))] = (unsigned char)k;
        m += __popc(bits);
    }
    qsync(q);
    return m;
}

// lu_solve_b on the quad: Gaussian elimination with partial pivoting of the
// m x m block A (row stride ld) in shared memory, NRHS right-hand sides in B
// (row-major, m x NRHS).  Each step: the pivot search over column j split
// over the lanes and combined to the first row holding the largest |a_ij|
// (the sequential search's choice), the row swap and the row updates split
// over the lanes, every element updated as a_ic - f_i a_jc with f_i = a_ij *
// (1 / a_jj), as in the thread-per-qp solve.  Back substitution: one column of
// B per lane, dot products in index order.  Returns nonzero on a zero pivot;
// *cond as lu_solve_b.
template <int NRHS>
__device__ __forceinline__ int lu4(double* A, int m, int ld, double* B, double* cond, const Quad& q) {
    int sing = 0;
    double pmin = 1e308, pmax = 0.0;
    const int l = q.l;
    for (int j = 0; j < m; ++j) {
        double mx = -1.0;
        int r = 0x7fffffff;
        for (int i = j + l; i < m; i += 4) {
            const double v = fabs(A[i * ld + j]);
            if (v > mx) {
                mx = v;
                r = i;
            }
        }
#pragma unroll
        for (int s = 1; s <= 2; s <<= 1) {
            const double om = __shfl_xor_sync(q.mask, mx, s);
            const int orr = __shfl_xor_sync(q.mask, r, s);
            if (om > mx || (om == mx && orr < r)) {
                mx = om;
                r = orr;
            }
        }
        {
            const double dj = fabs(A[j * ld + j]);
            if (dj != dj) {  // a NaN diagonal: the sequential search keeps row j
                mx = dj;
                r = j;
            }
        }
        pmin = fmin(pmin, mx);
        pmax = fmax(pmax, mx);
        if (mx == 0.0) {
            sing = 1;
            continue;
        }
        if (r != j) {
            for (int c = j + l; c < m; c += 4) {
                const double t = A[j * ld + c];
                A[j * ld + c] = A[r * ld + c];
                A[r * ld + c] = t;
            }
            for (int c = l; c < NRHS; c += 4) {
                const double t = B[j * NRHS + c];
                B[j * NRHS + c] = B[r * NRHS + c];
                B[r * NRHS + c] = t;
            }
            qsync(q);
        }
        const double piv = 1.0 / A[j * ld + j];
        for (int i = j + 1 + l; i < m; i += 4) {
            const double f = A[i * ld + j] * piv;
            if (f == 0.0) continue;
            double* ai = A + i * ld;
            const double* aj = A + j * ld;
            int c = j + 1;
            for (; c + 2 <= m; c += 2) {
                const double x0 = aj[c], x1 = aj[c + 1];
                const double y0 = ai[c], y1 = ai[c + 1];
                ai[c] = y0 - f * x0;
                ai[c + 1] = y1 - f * x1;
            }
            if (c < m) ai[c] = ai[c] - f * aj[c];
#pragma unroll
            for (int cc = 0; cc < NRHS; ++cc) B[i * NRHS + cc] -= f * B[j * NRHS + cc];
        }
        qsync(q);
    }
    for (int c = l; c < NRHS; c += 4)
        for (int j = m - 1; j >= 0; --j) {
            const double d = A[j * ld + j];
            double s = B[j * NRHS + c];
            for (int k = j + 1; k < m; ++k) s -= A[j * ld + k] * B[k * NRHS + c];
            B[j * NRHS + c] = s / d;
        }
    qsync(q);
    if (cond) *cond = m == 0 ? 1.0 : (pmin > 0.0 ? pmax / pmin : 1e308);
    return sing;
}

// final_tangent (cp_qp2.cuh) split into its kl-independent products and
// one column kl of dP/dF, with the same expressions, for one column per lane.
struct TangentPrep {
    M3 Finv, t1, t2, t3, Z;
};
__device__ __forceinline__ TangentPrep final_tangent_prep(const M3& F, const M3& FE_tau, const M3& Tst) {
    TangentPrep p;
    p.Finv = inv(F);
    p.t1 = mulNT(Tst, mul(p.Finv, FE_tau));
    p.t2 = mul(p.Finv, FE_tau);
    p.t3 = mul(FE_tau, Tst);
    p.Z = mulNT(mulNT(p.t3, F), p.Finv);
    return p;
}
template <class SymD, class X1Src>
__device__ __forceinline__ void final_tangent_col(const TangentPrep& p, const M3& FE_tau, const M3& Fpn_inv,
                                                  const SymD& D2, const X1Src& x1, int kl, double scale,
                                                  double* dPdF) {
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
    M3 PK = mul(dFe, p.t1);
    axpy(PK, 1.0, mulNT(mul(FE_tau, dTs), p.t2));
    axpy(PK, -1.0, mulNT(mul(p.t3, dFe), p.Finv));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int j = 0; j < 3; ++j) PK(a, j) -= p.Finv(j, kk) * p.Z(a, l);
#pragma unroll
    for (int c = 0; c < 9; ++c) dPdF[c * 9 + kl] = scale * PK.a[c];
}

// Outputs of one qp on the quad (caller order; any may be null).
struct QuadOut {
    double* P;     // 9, times scale
    double* dPdF;  // 81, times scale
    double scale;
    double* T;      // 9
    double* keepT;  // 9 (post-pass: T kept for the averages)
    double* keepF;  // 9
};

// calculatePlasticity for internal qp i of group g on the quad q, scratch in
// the shared-memory area 'area' of capacity P (P >= the qp's potentially
// active systems, capped at PMAX).  Requires o.max_search == 1.  Every lane
// returns the same status.
template <int PMAX>
__device__ int qp_update4(const LatDev& L, const Opts& o, const GroupDev& g, int64_t i, const M3& F, int flag,
                          double F_e, double F_r, const QuadOut& out, int32_t* stats_out, int lattice_id,
                          double* area, int P, const Quad q) {
    const int n = L.n, ns = L.ns, nw = L.nw;
    const int64_t cnt = g.count;
    const int l = q.l;
    int status = 0;
    const double tol1 = o.tol;
    const Area4 w = quad_carve(area, P, n);

    const double r0 = g.rot_c[i], r1 = g.rot_c[cnt + i], r2 = g.rot_c[2 * cnt + i];
    const M3 R = odfpoint(r0, r1, r2);
    {
        const Sym6 D2v = elasticmoduli(R, L.C);
#pragma unroll
        for (int e = 0; e < 21; ++e)
            if ((e & 3) == l) w.D2[e] = D2v.c[e];
    }
    qsync(q);
    const Sym6Ref D2{w.D2, 1};

    // history of every system (:28-35): each lane's CRSS and backstress, all
    // loads in flight at once, into the area
    for (int a0 = l; a0 < n; a0 += 16) {
        double sv[4], wv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int a = a0 + 4 * u;
            if (a < n) {
                sv[u] = g.s_c[(int64_t)a * cnt + i];
                wv[u] = g.W_c[(int64_t)a * cnt + i];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int a = a0 + 4 * u;
            if (a < n) {
                w.sS[a] = sv[u];
                w.WS[a] = wv[u];
            }
        }
    }
    qsync(q);

    unsigned long long neg_t_bits = 0ull;
    M3 FP_tau = load_soa3(g.Fp_c, cnt, i);
    M3 Fpn_inv = inv(FP_tau);
    M3 FE_tau = mul(F, Fpn_inv);
    const M3 FP_t2 = FP_tau;
    M3 CE_tr, Tst, Ce_tau = zero3(), del_FP = zero3();
    M3 T_tau, P_tau;
    int nPA = 0, p0 = 0, rounds_total = 0, e_terms = 0, c_terms = 0, lazy_p = -1;
    double maxcond = 1.0;
    int iter1 = 1;

    // ---- trial kinematics and stress (:160-196)
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
    // ---- resolved shears, potentially active set (:199-244): system a on
    // lane a % 4; the PA members keep their row constants (h, Schmid vectors,
    // signed kinematic term) and the increment-start CRSS / backstress
    unsigned long long neg_d = 0ull;
    for (int a0 = 0; a0 < n; a0 += 4) {
        const int a = a0 + l;
        bool pa = false;
        double t = 0.0, W = 0.0, sa = 0.0, bb = 0.0;
        if (a < n) {
            W = w.WS[a];
            sa = w.sS[a];
            t = resolved(L, a, tr.Xc);
            if (a > ns - 1 && (t - W) < 0) t = W;
            bb = fabs(t - W) - sa;
            pa = bb >= tol1;
        }
        const unsigned bits = (__ballot_sync(q.mask, pa) >> q.base) & 0xFu;
        if (a < n) w.kof[a] = 0xFF;
        if (pa) {
            const int k = nPA + __popc(bits & ((1u << l) - 1u));
            if (k < P) {
                w.kof[a] = (unsigned char)k;
                w.pa0[k] = (unsigned char)a;
                w.tau_tr[k] = t;
                w.b[k] = bb;
                w.WP[k] = W;
                w.h[k] = ldg(&L.h0[a]) * pow((1 - sa / ldg(&L.ss[a])), ldg(&L.a[a]));
                schmid_vectors(L, a, R, w.Sv + 6 * k);
                const double kin = ldg(&L.C1[a]) - ldg(&L.C2[a]) * W;
                const bool ng = (t - W) < 0.0;
                if (ng) {
                    neg_d |= (1ull << k);
                    neg_t_bits |= (1ull << a);
                }
                w.kin[k] = ng ? -kin : kin;
            }
        }
        nPA += __popc(bits);
    }
    neg_d |= __shfl_xor_sync(q.mask, neg_d, 1);
    neg_d |= __shfl_xor_sync(q.mask, neg_d, 2);
    neg_t_bits |= __shfl_xor_sync(q.mask, neg_t_bits, 1);
    neg_t_bits |= __shfl_xor_sync(q.mask, neg_t_bits, 2);
    if (nPA > PMAX) status |= QP_ACTIVE_OVERFLOW;
    if (nPA > P) {
        if (P < PMAX) status |= QP_ACTIVE_OVERFLOW;  // the area is smaller than the set (never for a sorted launch)
        nPA = P;
    }
    p0 = nPA;
    qsync(q);

    if (nPA > 0) {
        const int p_init = nPA;
        const int ld = w.ld;
        // column j of the consistency matrix needs M_j = Ce [D2 : sym(Ce S_j)] + 2 sym(Ce S_j) T*
        auto build_active = [&](int m) {
            for (int c = l; c < m; c += 4) {
                const int kj = w.pos[c];
                const int bsys = w.pa0[kj];
                const M3 Sj = schmid_of(w.Sv + 6 * kj);
                const M3 Y = sym(mul(CE_tr, Sj));
                M3 Mj = mul(CE_tr, voigt_apply(D2, Y));
                axpy(Mj, 2.0, mul(Y, Tst_tr));
                const unsigned long long nj = (neg_d >> kj) & 1ull;
                const double hj = w.h[kj];
                for (int r = 0; r < m; ++r) {
                    const int ki = w.pos[r];
                    const int asys = w.pa0[ki];
                    const double sm = schmid_dot(w.Sv + 6 * ki, Mj);
                    double v = ldg(&L.q[asys * NM + bsys]) * hj;
                    v += (((neg_d >> ki) & 1ull) ^ nj) ? -sm : sm;
                    v += w.kin[ki];
                    w.Apa[r * ld + c] = v;
                }
            }
            qsync(q);
        };

        // ---- consistency iterations (:311-448)
        for (int k = l; k < p_init; k += 4) {
            w.x_old[k] = 0.0;
            w.cur[k] = 1;
        }
        qsync(q);
        int count1 = 0;
        while (true) {
            double bmax = 0.0;
            for (int k = l; k < p_init; k += 4)
                if (w.cur[k]) bmax = fmax(bmax, fabs(w.b[k]));
            bmax = fmax(bmax, __shfl_xor_sync(q.mask, bmax, 1));
            bmax = fmax(bmax, __shfl_xor_sync(q.mask, bmax, 2));
            if (!(bmax > tol1)) break;
            count1 += 1;
            if (count1 > o.max_solver) break;
            // inactive_slip_removal (inactiveSlipRemoval.cc:4-124)
            for (;;) {
                const int m = quad_compact(w.cur, p_init, w.pos, q);
                for (int r = l; r < m; r += 4) w.rhs[r] = w.b[w.pos[r]];
                build_active(m);
                double cnd = 1.0;
                if (lu4<1>(w.Apa, m, ld, w.rhs, &cnd, q)) status |= QP_SINGULAR;
                maxcond = fmax(maxcond, cnd);
                ++rounds_total;
                for (int k = l; k < p_init; k += 4) w.x[k] = 0.0;
                qsync(q);
                for (int r = l; r < m; r += 4) w.x[w.pos[r]] = w.rhs[r];
                qsync(q);
                bool removed = false;
                for (int k = l; k < p_init; k += 4)
                    if (w.cur[k] && (w.x_old[k] + w.x[k]) < 0) {
                        w.cur[k] = 0;
                        removed = true;
                    }
                removed = __any_sync(q.mask, removed);
                qsync(q);
                if (!removed) break;
            }
            int act = 0;
            for (int k = l; k < p_init; k += 4) {
                w.x_old[k] += w.x[k];
                act += w.cur[k];
            }
            act += __shfl_xor_sync(q.mask, act, 1);
            act += __shfl_xor_sync(q.mask, act, 2);
            nPA = act;
            qsync(q);

            // del_FP (:337-357), in PA order in every lane
            del_FP = zero3();
            for (int k = 0; k < p_init; ++k) {
                if (w.x_old[k] == 0.0) continue;
                const double sgn = ((w.tau_tr[k] - w.WP[k]) > 0) ? w.x_old[k] : -w.x_old[k];
                axpy(del_FP, sgn, schmid_of(w.Sv + 6 * k));
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
            for (int k = l; k < p_init; k += 4) {
                if (!w.cur[k]) continue;
                const int a = w.pa0[k];
                const double Wa = w.WP[k];
                double t = resolved(L, a, Xnc);
                if (a > ns - 1 && (w.tau_tr[k] - Wa) < 0) t = Wa;
                w.tn[k] = t;
            }
            // hardening of every system (:399-429): the non-zero increments
            // gathered in PA order (every lane), the systems split over lanes
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
            for (int a = l; a < n; a += 4) {
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
                double sv = w.sS[a] + h1;
                const double sat = ldg(&L.ss[a]);
                if (sv > sat) sv = sat;
                w.sS[a] = sv;
            }
            qsync(q);
            // backstress (:431-436) and b (:438-446) of the PA systems
            for (int k = l; k < p_init; k += 4) {
                const int a = w.pa0[k];
                double Wa = w.WP[k];
                if ((w.tau_tr[k] - Wa) > 0)
                    Wa = Wa + (ldg(&L.C1[a]) - ldg(&L.C2[a]) * Wa) * w.x[k];
                else
                    Wa = Wa + (-ldg(&L.C1[a]) - ldg(&L.C2[a]) * Wa) * w.x[k];
                w.WP[k] = Wa;
                if (w.cur[k]) w.b[k] = fabs(w.tn[k] - Wa) - w.sS[a];
            }
            qsync(q);
        }

        // ---- fractions (:450-456): PA systems _conv + their total increment,
        // the others _conv + 0 (each lane's loads in flight at once)
        for (int t0 = l; t0 < ns; t0 += 16) {  // four loads per lane in flight
            double cv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int t = t0 + 4 * u;
                if (t < ns) cv[u] = g.sl_c[(int64_t)t * cnt + i];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int t = t0 + 4 * u;
                if (t < ns) {
                    const int k = w.kof[t];
                    g.sl_i[(int64_t)t * cnt + i] = (k < p_init) ? cv[u] + w.x_old[k] : cv[u] + 0.0;
                }
            }
        }
        for (int t = l; t < nw; t += 4) {
            const int k = w.kof[ns + t];
            const double c = g.tw_c[(int64_t)t * cnt + i];
            g.tw_i[(int64_t)t * cnt + i] = (k < p_init) ? c + w.x_old[k] / L.twin_shear : c + 0.0;
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
            // ---- tangent inside the slip-search loop (:473-828), lazy form
            qsync(q);  // the removal rounds' vectors become the tangent's arrays
            const int p = quad_compact(w.cur, p_init, w.pos, q);
            for (int kl = l; kl < 9; kl += 4) {
                const int kk = kl / 3, ll = kl % 3;
                M3 dFe;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int j = 0; j < 3; ++j) dFe(a, j) = (a == kk) ? Fpn_inv(ll, j) : 0.0;
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
                    double v = schmid_dot(w.Sv + 6 * k, dtau);
                    if (neg_t_bits >> w.pa0[k] & 1ull) v = -v;
                    w.rhs9[r * 9 + kl] = v;
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
            // S_PA (9 x p, row stride P) and the tangent's matrix, one column per lane
            for (int cj = l; cj < p; cj += 4) {
                const int kj = w.pos[cj];
                const int bsys = w.pa0[kj];
                const M3 Sj = schmid_of(w.Sv + 6 * kj);
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
                    const double sm = schmid_dot(w.Sv + 6 * ki, Mj);
                    double v = ldg(&L.q[asys * NM + bsys]) * w.h[kj];
                    v += (ni ^ nj) ? -sm : sm;
                    const double Wa = w.WP[ki];
                    const double kin = ldg(&L.C1[asys]) - ldg(&L.C2[asys]) * Wa;
                    v += ni ? -kin : kin;
                    w.Apa[ci * ld + cj] = v;
                }
                const M3 spa = mul(dp, FP_t2);
#pragma unroll
                for (int c = 0; c < 9; ++c) w.SPA[c * P + cj] = nj ? -spa.a[c] : spa.a[c];
            }
            qsync(q);
            if (lu4<9>(w.Apa, p, ld, w.rhs9, nullptr, q)) status |= QP_SINGULAR;
            lazy_p = p;
        }
        iter1 = 2;  // the pass counter passes max_search == 1
        status |= QP_SLIP_SEARCH_CAP;
    }

    // ---- outputs and history (:942-959)
    for (int c = l; c < 9; c += 4) {
        if (out.P) out.P[c] = out.scale * P_tau.a[c];
        if (out.T) out.T[c] = T_tau.a[c];
        if (out.keepT) {
            out.keepT[c] = T_tau.a[c];
            out.keepF[c] = F.a[c];
        }
        g.Fe_i[c * cnt + i] = FE_tau.a[c];
        g.Fp_i[c * cnt + i] = FP_tau.a[c];
    }
    {
        bool finite = true;
#pragma unroll
        for (int c = 0; c < 9; ++c) finite = finite && isfinite(P_tau.a[c]);
        if (!finite) status |= QP_NONFINITE;
    }

    // ---- final tangent (:835-940), one column kl per lane
    if (flag == 1 && out.dPdF) {
        const bool plastic = lazy_p > 0;
        const TangentPrep tp = final_tangent_prep(F, FE_tau, Tst);
        auto x1 = [&](int kl, M3& X1) -> bool {
            if (!plastic) return false;
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                double acc = 0.0;
                for (int r = 0; r < lazy_p; ++r) acc += w.SPA[c * P + r] * w.rhs9[r * 9 + kl];
                X1.a[c] = acc;
            }
            return true;
        };
        for (int kl = l; kl < 9; kl += 4) final_tangent_col(tp, FE_tau, Fpn_inv, D2, x1, kl, out.scale, out.dPdF);
    }

    // ---- backstress into the history: the PA systems' updated values, the
    // others' increment-start values
    for (int a = l; a < n; a += 4) {
        const int k = w.kof[a];
        g.W_i[(int64_t)a * cnt + i] = k < p0 ? w.WP[k] : w.WS[a];
    }

    // ---- twin reorientation (:962-1019)
    qsync(q);  // tw_i of every lane
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
            if (l < 3) {
                const double v = l == 0 ? rr[0] : (l == 1 ? rr[1] : rr[2]);
                g.rot_i[(int64_t)l * cnt + i] = v;
                g.rotnew_i[(int64_t)l * cnt + i] = v;
            } else {
                g.twin_i[i] = 1;
            }
            for (int t = l; t < nw; t += 4) w.sS[ns + t] = 100000;
        }
    }
    qsync(q);
    // ---- CRSS of every system into the history
    for (int a = l; a < n; a += 4) g.s_i[(int64_t)a * cnt + i] = w.sS[a];

    if (maxcond > 1e12) status |= QP_ILL_CONDITIONED;
    if (stats_out && l == 0) {
        stats_out[0] = p0;
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
