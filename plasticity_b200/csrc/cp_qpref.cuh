// cp_qpref.cuh -- calculatePlasticity in the reference's own operation order
// (cp_options_t.reference_order = 1).
//
// The optimised updates (cp_qp.cuh, cp_qp2.cuh) restructure the reference's
// arithmetic: Schmid tensors as vector pairs, only the potentially active
// block of the consistency matrix, LU instead of the SVD pseudo-inverse, FMA
// contraction.  Their results agree with the reference's to rounding, which
// is enough wherever the active-set solves are well conditioned; where a solve
// has condition > 1e12 its result is set by rounding and the active set that
// follows can differ.  This form evaluates every value the way
// src/materialModels/crystalPlasticity/calculatePlasticity.cc writes it:
//   * deal.II FullMatrix semantics for every 3x3 and 9x9 product (sums
//     accumulated from zero in index order), the reference's temporaries;
//   * the consistency matrix over all systems (:265-306), the active-set
//     solves by the pseudo-inverse of LAPACKFullMatrix::compute_inverse_svd(0)
//     (inactiveSlipRemoval.cc:26,99), restated as a one-sided Jacobi SVD;
//   * FullMatrix::invert for the tangent's matrices (:573, :714): closed form
//     up to 3x3, Gauss-Jordan with partial pivoting above;
//   * no contraction of multiply-add pairs: the translation unit that
//     instantiates it is compiled with -fmad=false;
//   * pow, the Gateaux-series factorials and the twin rotation's cos(atan(.))
//     by the functions below, which use only correctly rounded operations, so
//     that a host build computes the same bits.
// It is slow (per-qp scratch of ~6 n^2 doubles in global memory, n the
// lattice's systems) and meant for reproducing a CPU run bit for bit, not for
// throughput.
#pragma once

#include "cp_qp.cuh"

#ifdef __CUDACC__
#define CP_REF __host__ __device__
#else
#define CP_REF inline
#endif

namespace cp {
namespace ref {

// ---- elementary functions from correctly rounded operations --------------
// ln 2 = LN2_HI + LN2_LO with LN2_HI's low 21 significand bits zero, so
// k * LN2_HI is exact for |k| < 2^21.
constexpr double LN2_HI = 0.693147180369123816490;
constexpr double LN2_LO = 1.90821492927058770002e-10;
constexpr double INV_LN2 = 1.44269504088896338700;
constexpr double SQRT_HALF = 0.70710678118654752440;

// natural log of a finite x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m - 1)/(m + 1), by its series in s^2 (|s| < 0.172,
// 12 terms reach 2^-60)
CP_REF double ref_log(double x) {
    int e = 0;
    double m = frexp(x, &e);
    if (m < SQRT_HALF) {
        m = m * 2.0;
        e = e - 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double p = 1.0 / 25.0;
    for (int j = 11; j >= 0; --j) p = p * z + 1.0 / (double)(2 * j + 1);
    const double lnm = (2.0 * s) * p;
    const double de = (double)e;
    return (de * LN2_HI + lnm) + de * LN2_LO;
}

// exp of t: t = k ln2 + r with |r| <= ln2/2 (Cody-Waite reduction), e^r by
// its Taylor series in nested form (18 terms), scaled by 2^k
CP_REF double ref_exp(double t) {
    if (t != t) return t;
    if (t > 709.782712893384) return (double)INFINITY;
    if (t < -745.2) return 0.0;
    const double kd = floor(t * INV_LN2 + 0.5);
    const double r = (t - kd * LN2_HI) - kd * LN2_LO;
    double p = 1.0;
    for (int j = 18; j >= 1; --j) p = 1.0 + (r / (double)j) * p;
    return ldexp(p, (int)kd);
}

// x^y as exp(y ln x), with the IEEE special cases that the hardening laws can
// meet (a zero base, a zero exponent, a negative base with an integral
// exponent)
CP_REF double ref_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    if (x == 0.0) return y > 0.0 ? 0.0 : (double)INFINITY;
    double ax = x;
    double sign = 1.0;
    if (x < 0.0) {
        if (floor(y) != y) return (x - x) / (x - x);
        ax = -x;
        if (fmod(y, 2.0) != 0.0) sign = -1.0;
    }
    if (ax == (double)INFINITY) return sign * (y > 0.0 ? (double)INFINITY : 0.0);
    return sign * ref_exp(y * ref_log(ax));
}

// ---- 3x3 with deal.II FullMatrix call semantics ---------------------------
struct R3 {
    double a[3][3];
};
CP_REF R3 r_zero() {
    R3 m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m.a[i][j] = 0.0;
    return m;
}
CP_REF R3 r_eye() {
    R3 m = r_zero();
    m.a[0][0] = m.a[1][1] = m.a[2][2] = 1.0;
    return m;
}
// A.mmult(C, B): C = A B
CP_REF R3 r_mmult(const R3& A, const R3& B) {
    R3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[i][k] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
// A.Tmmult(C, B): C = A^T B
CP_REF R3 r_Tmmult(const R3& A, const R3& B) {
    R3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[k][i] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
// A.mTmult(C, B): C = A B^T
CP_REF R3 r_mTmult(const R3& A, const R3& B) {
    R3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[i][k] * B.a[j][k];
            C.a[i][j] = s;
        }
    return C;
}
CP_REF R3 r_scale(double c, const R3& A) {
    R3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = c * A.a[i][j];
    return C;
}
// A.add(c, B): A += c B
CP_REF void r_add(R3& A, double c, const R3& B) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A.a[i][j] += c * B.a[i][j];
}
CP_REF void r_symmetrize(R3& A) {
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j) {
            const double t = (A.a[i][j] + A.a[j][i]) / 2;
            A.a[i][j] = A.a[j][i] = t;
        }
}
CP_REF double r_frob(const R3& A) {
    double s = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s += A.a[i][j] * A.a[i][j];
    return sqrt(s);
}
// FullMatrix::determinant: cofactor expansion along the first row
CP_REF double r_det(const R3& A) {
    return A.a[0][0] * (A.a[1][1] * A.a[2][2] - A.a[1][2] * A.a[2][1]) -
           A.a[0][1] * (A.a[1][0] * A.a[2][2] - A.a[1][2] * A.a[2][0]) +
           A.a[0][2] * (A.a[1][0] * A.a[2][1] - A.a[1][1] * A.a[2][0]);
}
// FullMatrix::invert for 3x3: adjugate times 1/det
CP_REF R3 r_inv(const R3& A) {
    const double c00 = A.a[1][1] * A.a[2][2] - A.a[1][2] * A.a[2][1];
    const double c01 = A.a[1][2] * A.a[2][0] - A.a[1][0] * A.a[2][2];
    const double c02 = A.a[1][0] * A.a[2][1] - A.a[1][1] * A.a[2][0];
    const double det = A.a[0][0] * c00 + A.a[0][1] * c01 + A.a[0][2] * c02;
    const double r = 1.0 / det;
    R3 B;
    B.a[0][0] = c00 * r;
    B.a[1][0] = c01 * r;
    B.a[2][0] = c02 * r;
    B.a[0][1] = (A.a[0][2] * A.a[2][1] - A.a[0][1] * A.a[2][2]) * r;
    B.a[1][1] = (A.a[0][0] * A.a[2][2] - A.a[0][2] * A.a[2][0]) * r;
    B.a[2][1] = (A.a[0][1] * A.a[2][0] - A.a[0][0] * A.a[2][1]) * r;
    B.a[0][2] = (A.a[0][1] * A.a[1][2] - A.a[0][2] * A.a[1][1]) * r;
    B.a[1][2] = (A.a[0][2] * A.a[1][0] - A.a[0][0] * A.a[1][2]) * r;
    B.a[2][2] = (A.a[0][0] * A.a[1][1] - A.a[0][1] * A.a[1][0]) * r;
    return B;
}
CP_REF R3 r_load(const double* p) {
    R3 m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m.a[i][j] = p[3 * i + j];
    return m;
}
CP_REF void r_store(const R3& m, double* p) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p[3 * i + j] = m.a[i][j];
}

// Dmat.vmult(vecform(A)) then matform (matrixOperations.cc:133-163), D a
// row-major 6x6
CP_REF R3 r_voigt(const double* D, const R3& A) {
    const double v[6] = {A.a[0][0], A.a[1][1], A.a[2][2], A.a[1][2], A.a[0][2], A.a[0][1]};
    double w[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0.0;
        for (int j = 0; j < 6; ++j) s += D[6 * i + j] * v[j];
        w[i] = s;
    }
    R3 B;
    B.a[0][0] = w[0];
    B.a[1][1] = w[1];
    B.a[2][2] = w[2];
    B.a[1][2] = w[3];
    B.a[0][2] = w[4];
    B.a[0][1] = w[5];
    B.a[2][1] = w[3];
    B.a[2][0] = w[4];
    B.a[1][0] = w[5];
    return B;
}

// matrixExponential (matrixOperations.cc:165-186): Taylor terms until the
// last one's Frobenius norm is <= 1e-10
CP_REF R3 r_matexp(const R3& A, int* terms, int* status) {
    R3 E = r_eye(), t = r_eye();
    double count = 1;
    int k = 0;
    while (r_frob(t) > 1.0e-10) {
        if (k >= EXP_TERM_CAP) {
            *status |= QP_SERIES_CAP;
            break;
        }
        R3 t2 = r_mmult(t, A);
        t2 = r_scale(1 / count, t2);
        t = t2;
        r_add(E, 1.0, t);
        count = count + 1.0;
        ++k;
    }
    if (terms) *terms = k;
    return E;
}

// odfpoint (rotationOperations.cc:4-51)
CP_REF R3 r_odfpoint(const double r[3]) {
    double rdotr = 0.0;
    for (int i = 0; i < 3; ++i) rdotr = rdotr + r[i] * r[i];
    const double term1 = 1.0 - rdotr;
    const double term2 = 1.0 + rdotr;
    R3 R = r_eye();
    for (int i = 0; i < 3; ++i) R.a[i][i] = R.a[i][i] * term1;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R.a[i][j] = R.a[i][j] + 2.0 * (r[i] * r[j]);
    R.a[0][1] = R.a[0][1] - 2.0 * r[2];
    R.a[0][2] = R.a[0][2] + 2.0 * r[1];
    R.a[1][2] = R.a[1][2] - 2.0 * r[0];
    R.a[1][0] = R.a[1][0] + 2.0 * r[2];
    R.a[2][0] = R.a[2][0] - 2.0 * r[1];
    R.a[2][1] = R.a[2][1] + 2.0 * r[0];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R.a[i][j] = R.a[i][j] * 1.0 / term2;
    return R;
}

// elasticmoduli (matrixOperations.cc:189-234): Ar = N(R) C N(R)^T, row-major
CP_REF void r_elasticmoduli(const R3& Rm, const double* C, double* Ar) {
    double N[6][6];
    for (int i = 0; i < 3; ++i) {
        N[i][0] = Rm.a[i][0] * Rm.a[i][0];
        N[i][1] = Rm.a[i][1] * Rm.a[i][1];
        N[i][2] = Rm.a[i][2] * Rm.a[i][2];
        N[i][3] = 2.0 * Rm.a[i][1] * Rm.a[i][2];
        N[i][4] = 2.0 * Rm.a[i][2] * Rm.a[i][0];
        N[i][5] = 2.0 * Rm.a[i][0] * Rm.a[i][1];
    }
    const int pr[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    for (int r = 0; r < 3; ++r) {
        const int p = pr[r][0], q = pr[r][1];
        N[3 + r][0] = Rm.a[p][0] * Rm.a[q][0];
        N[3 + r][1] = Rm.a[p][1] * Rm.a[q][1];
        N[3 + r][2] = Rm.a[p][2] * Rm.a[q][2];
    }
    N[3][3] = Rm.a[1][1] * Rm.a[2][2] + Rm.a[1][2] * Rm.a[2][1];
    N[3][4] = Rm.a[1][2] * Rm.a[2][0] + Rm.a[1][0] * Rm.a[2][2];
    N[3][5] = Rm.a[1][0] * Rm.a[2][1] + Rm.a[1][1] * Rm.a[2][0];
    N[4][3] = Rm.a[0][1] * Rm.a[2][2] + Rm.a[0][2] * Rm.a[2][1];
    N[4][4] = Rm.a[0][2] * Rm.a[2][0] + Rm.a[0][0] * Rm.a[2][2];
    N[4][5] = Rm.a[0][0] * Rm.a[2][1] + Rm.a[0][1] * Rm.a[2][0];
    N[5][3] = Rm.a[0][1] * Rm.a[1][2] + Rm.a[0][2] * Rm.a[1][1];
    N[5][4] = Rm.a[0][2] * Rm.a[1][0] + Rm.a[0][0] * Rm.a[1][2];
    N[5][5] = Rm.a[0][0] * Rm.a[1][1] + Rm.a[0][1] * Rm.a[1][0];
    double T[6][6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += N[i][k] * C[6 * k + j];
            T[i][j] = s;
        }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += T[i][k] * N[j][k];
            Ar[6 * i + j] = s;
        }
}

// FullMatrix::invert: closed form up to 3x3, in-place Gauss-Jordan with
// partial (row) pivoting above; M (n^2) and perm (n) are workspace.  Returns
// 1 on a zero pivot (or a non-finite small-case inverse).
CP_REF int r_invert(const double* A, int n, double* B, double* M, int* perm) {
    if (n == 0) return 0;
    if (n == 1) {
        B[0] = 1.0 / A[0];
        return A[0] == 0.0;
    }
    if (n == 2) {
        const double t = 1.0 / (A[0] * A[3] - A[1] * A[2]);
        B[0] = A[3] * t;
        B[1] = -A[1] * t;
        B[2] = -A[2] * t;
        B[3] = A[0] * t;
        return !isfinite(t);
    }
    if (n == 3) {
        r_store(r_inv(r_load(A)), B);
        return !isfinite(B[0]);
    }
    for (int i = 0; i < n * n; ++i) M[i] = A[i];
    for (int i = 0; i < n; ++i) perm[i] = i;
    int sing = 0;
    for (int j = 0; j < n; ++j) {
        int r = j;
        double mx = fabs(M[j * n + j]);
        for (int i = j + 1; i < n; ++i)
            if (fabs(M[i * n + j]) > mx) {
                mx = fabs(M[i * n + j]);
                r = i;
            }
        if (mx == 0.0) sing = 1;
        if (r != j) {
            for (int k = 0; k < n; ++k) {
                const double t = M[j * n + k];
                M[j * n + k] = M[r * n + k];
                M[r * n + k] = t;
            }
            const int t = perm[j];
            perm[j] = perm[r];
            perm[r] = t;
        }
        const double piv = 1.0 / M[j * n + j];
        for (int i = 0; i < n; ++i) M[i * n + j] *= piv;
        M[j * n + j] = piv;
        for (int k = 0; k < n; ++k) {
            if (k == j) continue;
            for (int i = 0; i < n; ++i) {
                if (i == j) continue;
                M[i * n + k] -= M[i * n + j] * M[j * n + k];
            }
        }
        for (int k = 0; k < n; ++k) M[j * n + k] *= -piv;
        M[j * n + j] = piv;
    }
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) B[i * n + perm[k]] = M[i * n + k];
    return sing;
}

// Pseudo-inverse of LAPACKFullMatrix::compute_inverse_svd(0.0)
// (inactiveSlipRemoval.cc:26,99) by one-sided (Hestenes) Jacobi SVD:
// cyclic sweeps over column pairs (i < j) of U = A V until no pair is
// rotated (|gamma| <= 1e-15 sqrt(alpha beta)) or 60 sweeps, singular values
// the column norms, A^+ = V diag(1/s^2) U^T with singular values not above
// 0 treated as zero.  U, V (n^2) and s (n) are workspace; *cond receives
// s_max / s_min.
CP_REF int r_pinv_svd(const double* A, int n, double* Ainv, double* U, double* V, double* s, double* cond) {
    *cond = 1.0;
    if (n == 0) return 0;
    for (int i = 0; i < n * n; ++i) {
        U[i] = A[i];
        V[i] = 0.0;
    }
    for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
    const double eps = 1e-15;
    for (int sweep = 0; sweep < 60; ++sweep) {
        int rotated = 0;
        for (int i = 0; i < n - 1; ++i)
            for (int j = i + 1; j < n; ++j) {
                double alpha = 0.0, beta = 0.0, gamma = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double ui = U[k * n + i], uj = U[k * n + j];
                    alpha += ui * ui;
                    beta += uj * uj;
                    gamma += ui * uj;
                }
                if (gamma == 0.0 || fabs(gamma) <= eps * sqrt(alpha * beta)) continue;
                rotated = 1;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t);
                const double sn = c * t;
                for (int k = 0; k < n; ++k) {
                    const double ui = U[k * n + i], uj = U[k * n + j];
                    U[k * n + i] = c * ui - sn * uj;
                    U[k * n + j] = sn * ui + c * uj;
                    const double vi = V[k * n + i], vj = V[k * n + j];
                    V[k * n + i] = c * vi - sn * vj;
                    V[k * n + j] = sn * vi + c * vj;
                }
            }
        if (!rotated) break;
    }
    double smax = 0.0;
    for (int i = 0; i < n; ++i) {
        double ss = 0.0;
        for (int k = 0; k < n; ++k) ss += U[k * n + i] * U[k * n + i];
        s[i] = sqrt(ss);
        smax = fmax(smax, s[i]);
    }
    {
        double smin = smax;
        for (int i = 0; i < n; ++i) smin = fmin(smin, s[i]);
        *cond = smin > 0.0 ? smax / smin : (double)INFINITY;
    }
    int sing = 0;
    for (int i = 0; i < n; ++i) {
        if (s[i] > 0.0 * smax && s[i] > 0.0) {
            s[i] = 1.0 / s[i];
        } else {
            s[i] = 0.0;
            sing = 1;
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += V[i * n + k] * (s[k] * s[k]) * U[j * n + k];
            Ainv[i * n + j] = acc;
        }
    return sing;
}

// the Gateaux-series terms (calculatePlasticity.cc:645-676, 748-779):
// D = S + sum_{k=1..count3} coef(k) sum_{l=0..k} dFp^l S dFp^(k-l),
// coef(k) = (+-1)^k / (k+1)!, the factorial as the product 2 * 3 * ... * (k+1)
CP_REF R3 r_gateaux(const R3& S, const R3& dFp, int count3, bool alternating) {
    R3 diff = S;
    double fact = 1.0;
    for (int k = 1; k <= count3; ++k) {
        R3 t4 = r_zero();
        for (int l = 0; l <= k; ++l) {
            R3 t1 = r_eye(), t2 = r_eye();
            for (int m = 0; m < l; ++m) t1 = r_mmult(t1, dFp);
            for (int m = 0; m < k - l; ++m) t2 = r_mmult(t2, dFp);
            const R3 t5 = r_mmult(t1, S);
            const R3 t6 = r_mmult(t5, t2);
            r_add(t4, 1.0, t6);
        }
        fact = fact * (double)(k + 1);
        const double coef = (alternating ? ((k & 1) ? -1.0 : 1.0) : 1.0) / fact;
        t4 = r_scale(coef, t4);
        r_add(diff, 1.0, t4);
    }
    return diff;
}

// doubles of per-qp scratch for a lattice of n systems
CP_REF int64_t scratch_doubles(int n) { return 6ll * n * n + 80ll * n + 1024; }

// Component c (row-major 3x3) of a structure-of-arrays field, qp i
CP_REF R3 soa_load(const double* f, int64_t cnt, int64_t i) {
    R3 m;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m.a[r][c] = f[(3 * r + c) * cnt + i];
    return m;
}
CP_REF void soa_store(double* f, int64_t cnt, int64_t i, const R3& m) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) f[(3 * r + c) * cnt + i] = m.a[r][c];
}

// calculatePlasticity (calculatePlasticity.cc:13-1022) for internal qp i of a
// lattice group: F (9, row-major) in; P, T, dPdF (dPdF[9 a + b] = dP_a/dF_b,
// times out.scale), the _iter history and the stats out.  w: this qp's
// scratch_doubles(L.n) doubles.
CP_REF int qp_update_ref(const LatDev& L, const Opts& o, const GroupDev& g, int64_t i, const double* Fin, int flag,
                         double F_e, double F_r, const QpOut& out, int32_t* stats_out, int lattice_id, double* w) {
    const int n = L.n, ns = L.ns, nw = L.nw;
    const int64_t cnt = g.count;
    int status = 0;
    const double tol1 = o.tol;
    // ---- scratch
    double* p = w;
    auto take = [&](int64_t k) {
        double* r = p;
        p += k;
        return r;
    };
    double* Sf = take(9 * (int64_t)n);  // Schmid tensors, 9 per system
    double* s_alpha_t = take(n);
    double* W_kh_t = take(n);
    double* s_alpha_tau = take(n);
    double* W_kh_tau = take(n);
    double* tau_trial = take(n);
    double* b = take(n);
    double* tau = take(n);
    double* x_beta_old = take(n);
    double* x_beta = take(n);
    double* h_beta = take(n);
    double* delh = take(n);
    double* x1 = take(n);
    double* bpa = take(n);
    double* sv = take(n);
    int* PA = reinterpret_cast<int*>(take(n));
    int* PAn = reinterpret_cast<int*>(take(n));
    int* pos0 = reinterpret_cast<int*>(take(n));  // system -> index in the pass's first PA, or -1
    int* iperm = reinterpret_cast<int*>(take(n));
    double* dels_delF = take(9 * (int64_t)n);
    double* dels_delF_prev = take(9 * (int64_t)n);
    double* delb = take(9 * (int64_t)n);
    double* dg = take(9 * (int64_t)n);
    double* S_PA = take(9 * (int64_t)n);
    double* Dmat2 = take(36);
    double* Dmat = take(36);
    double* TM = take(81);
    double* delFp_delF = take(81);
    double* delFp_delF_prev = take(81);
    double* delFe_delF = take(81);
    double* delEtrial_delF = take(81);
    double* delT_delF = take(81);
    double* deltau_delF = take(81);
    double* Ac = take((int64_t)n * n);  // A[PA0, PA0] of the pass (:265-306)
    double* Wk = take(5ll * n * n);     // per-phase workspace
    if (p - w > scratch_doubles(n)) return QP_ACTIVE_OVERFLOW;  // (the layout above fits by construction)
    auto S = [&](int a) -> R3 { return r_load(Sf + 9 * a); };
    auto h_ab = [&](int a, int c) { return ldg(&L.q[a * NM + c]) * h_beta[c]; };

    R3 F_tau;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) F_tau.a[r][c] = Fin[3 * r + c];
    const R3 FP_t = soa_load(g.Fp_c, cnt, i);
    for (int a = 0; a < n; ++a) {
        s_alpha_t[a] = g.s_c[(int64_t)a * cnt + i];
        W_kh_t[a] = g.W_c[(int64_t)a * cnt + i];
    }
    const double rot1[3] = {g.rot_c[i], g.rot_c[cnt + i], g.rot_c[2 * cnt + i]};

    // ---- :39-77 rotation, rotated stiffness, engineering-shear Dmat, 9x9 TM
    const R3 rotmat = r_odfpoint(rot1);
    r_elasticmoduli(rotmat, L.C, Dmat2);
    for (int e = 0; e < 36; ++e) Dmat[e] = Dmat2[e];
    for (int r = 0; r < 6; ++r)
        for (int c = 3; c < 6; ++c) Dmat[6 * r + c] = 2 * Dmat[6 * r + c];
    {
        const int vec2[9] = {0, 5, 4, 5, 1, 3, 4, 3, 2};
        for (int r = 0; r < 9; ++r)
            for (int c = 0; c < 9; ++c) TM[9 * r + c] = Dmat2[6 * vec2[r] + vec2[c]];
    }
    // ---- :79-112 Schmid tensors in sample coordinates (the B tensor of
    // :96-106 is built from a zero CE_tau_trial and never read)
    for (int a = 0; a < n; ++a) {
        R3 t;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) t.a[r][c] = ldg(&L.m[3 * a + r]) * ldg(&L.nn[3 * a + c]);
        const R3 t2 = r_mmult(rotmat, t);
        r_store(r_mTmult(t2, rotmat), Sf + 9 * a);
    }

    // ---- :114-151
    R3 FP_tau = FP_t;
    R3 Fpn_inv = r_inv(FP_t);
    R3 FE_tau = r_mmult(F_tau, Fpn_inv);
    for (int a = 0; a < n; ++a) {
        s_alpha_tau[a] = s_alpha_t[a];
        W_kh_tau[a] = W_kh_t[a];
        x_beta_old[a] = 0.0;
        x_beta[a] = 0.0;
        tau[a] = 0.0;
        tau_trial[a] = 0.0;
    }
    for (int e = 0; e < 81; ++e) delFp_delF[e] = 0.0;
    // dels_delF starts at zero (:148) and is only re-assigned as
    // inv(I - term_ds) dels_delF_prev with dels_delF_prev = dels_delF
    for (int e = 0; e < 9 * n; ++e) {
        dels_delF[e] = 0.0;
        dels_delF_prev[e] = 0.0;
    }

    R3 FP_t2 = FP_tau, CE_tau_trial = r_zero(), T_star_tau = r_zero(), T_star_tau_trial = r_zero();
    R3 Ce_tau = r_zero(), del_FP = r_zero(), T_tau = r_zero(), P_tau = r_zero();
    double det_FE_tau, det_F_tau;
    int nPA = 0, p0 = -1, rounds_total = 0, e_terms = 0, c_terms = 0;
    double maxcond = 1.0;
    unsigned iter1 = 1;

    while (iter1) {
        if (iter1 > (unsigned)o.max_search) {
            status |= QP_SLIP_SEARCH_CAP;
            break;
        }
        // ---- :160-176 trial kinematics
        FP_t2 = FP_tau;
        Fpn_inv = r_inv(FP_t2);
        const R3 FE_tau_trial = r_mmult(F_tau, Fpn_inv);
        CE_tau_trial = r_Tmmult(FE_tau_trial, FE_tau_trial);
        R3 Ee = CE_tau_trial;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Ee.a[r][c] = 0.5 * (Ee.a[r][c] - (r == c ? 1.0 : 0.0));
        // ---- :180-196 trial stress
        T_star_tau_trial = r_voigt(Dmat, Ee);
        T_star_tau = T_star_tau_trial;
        det_FE_tau = r_det(FE_tau);
        R3 t = r_mmult(FE_tau, T_star_tau_trial);
        t = r_scale(1.0 / det_FE_tau, t);
        T_tau = r_mTmult(t, FE_tau);
        det_F_tau = r_det(F_tau);
        R3 Finv = r_inv(F_tau);
        {
            const R3 t2 = r_mTmult(T_tau, Finv);
            P_tau = r_scale(det_FE_tau, t2);
        }
        // ---- :199-244 resolved shear and the potentially active set
        t = r_mmult(CE_tau_trial, T_star_tau_trial);
        nPA = 0;
        for (int a = 0; a < n; ++a) {
            const R3 Sa = S(a);
            double r = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk) r += t.a[j][kk] * Sa.a[j][kk];
            tau_trial[a] = r;
            if (a > ns - 1) {
                if ((tau_trial[a] - W_kh_tau[a]) < 0) tau_trial[a] = W_kh_tau[a];
            }
            b[a] = fabs(tau_trial[a] - W_kh_tau[a]) - s_alpha_tau[a];
            pos0[a] = -1;
            if (b[a] >= tol1) {
                pos0[a] = nPA;
                PA[nPA++] = a;
            }
        }
        if (p0 < 0) p0 = nPA;
        for (int a = 0; a < n; ++a) tau[a] = tau_trial[a];
        if (nPA == 0) break;
        const int nPA0 = nPA;

        // ---- :250-306 hardening moduli and the consistency matrix A over the
        // potentially active systems (the only entries inactive_slip_removal reads)
        for (int a = 0; a < ns; ++a) h_beta[a] = ldg(&L.h0[a]) * ref_pow((1 - s_alpha_tau[a] / ldg(&L.ss[a])), ldg(&L.a[a]));
        for (int a = 0; a < nw; ++a)
            h_beta[ns + a] = ldg(&L.h0[ns + a]) * ref_pow((1 - s_alpha_tau[ns + a] / ldg(&L.ss[ns + a])), ldg(&L.a[ns + a]));
        for (int jj = 0; jj < nPA0; ++jj) {
            const int bj = PA[jj];
            const R3 Sj = S(bj);
            R3 temp2 = r_mmult(CE_tau_trial, Sj);
            r_symmetrize(temp2);
            R3 temp3 = r_voigt(Dmat, temp2);
            R3 temp1 = r_mmult(CE_tau_trial, temp3);
            temp3 = r_mmult(temp2, T_star_tau_trial);
            r_add(temp1, 2.0, temp3);
            for (int ii = 0; ii < nPA0; ++ii) {
                const int ai = PA[ii];
                const R3 Si = S(ai);
                double Aij = h_ab(ai, bj);
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        if (((tau_trial[ai] - W_kh_tau[ai]) * (tau_trial[bj] - W_kh_tau[bj])) < 0.0)
                            Aij -= Si.a[kk][l] * temp1.a[kk][l];
                        else
                            Aij += Si.a[kk][l] * temp1.a[kk][l];
                    }
                if ((tau_trial[ai] - W_kh_tau[ai]) < 0.0)
                    Aij -= ldg(&L.C1[ai]) - ldg(&L.C2[ai]) * W_kh_tau[ai];
                else
                    Aij += ldg(&L.C1[ai]) - ldg(&L.C2[ai]) * W_kh_tau[ai];
                Ac[ii * nPA0 + jj] = Aij;
            }
        }

        // ---- :311-448 consistency iterations
        for (int a = 0; a < n; ++a) x_beta_old[a] = 0.0;
        unsigned count1 = 0;
        while (true) {
            double mx = 0.0;
            for (int q = 0; q < nPA; ++q) mx = fmax(mx, fabs(b[PA[q]]));
            if (!(mx > tol1)) break;
            count1 = count1 + 1;
            if (count1 > (unsigned)o.max_solver) break;
            for (int a = 0; a < n; ++a) x_beta[a] = 0.0;
            // inactive_slip_removal (inactiveSlipRemoval.cc:4-124)
            {
                double* Apa = Wk;
                double* Ainv = Wk + (int64_t)n * n;
                double* U = Wk + 2ll * n * n;
                double* V = Wk + 3ll * n * n;
                int m = nPA;
                int rounds = 0;
                for (int a = 0; a < n; ++a) x1[a] = 0.0;
                for (;;) {
                    for (int r = 0; r < m; ++r) {
                        bpa[r] = b[PA[r]];
                        for (int c = 0; c < m; ++c) Apa[r * m + c] = Ac[pos0[PA[r]] * nPA0 + pos0[PA[c]]];
                    }
                    double cnd = 1.0;
                    if (r_pinv_svd(Apa, m, Ainv, U, V, sv, &cnd)) status |= QP_SINGULAR;
                    maxcond = fmax(maxcond, cnd);
                    ++rounds;
                    for (int a = 0; a < n; ++a) x1[a] = 0.0;
                    for (int r = 0; r < m; ++r) {
                        double s = 0.0;
                        for (int c = 0; c < m; ++c) s += Ainv[r * m + c] * bpa[c];
                        x1[PA[r]] = s;
                    }
                    // systems whose total increment would turn negative leave the set
                    int mn = 0;
                    for (int r = 0; r < m; ++r)
                        if (!((x_beta_old[PA[r]] + x1[PA[r]]) < 0)) PAn[mn++] = PA[r];
                    if (mn == m) break;
                    for (int r = 0; r < mn; ++r) PA[r] = PAn[r];
                    m = mn;
                }
                nPA = m;
                rounds_total += rounds;
                for (int a = 0; a < n; ++a) x_beta[a] = x1[a];
                for (int a = 0; a < n; ++a) x_beta_old[a] += x_beta[a];
            }
            del_FP = r_zero();
            for (int a = 0; a < n; ++a) {
                const R3 Sa = S(a);
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk) {
                        if ((tau_trial[a] - W_kh_tau[a]) > 0)
                            del_FP.a[j][kk] = del_FP.a[j][kk] + x_beta_old[a] * Sa.a[j][kk];
                        else
                            del_FP.a[j][kk] = del_FP.a[j][kk] - x_beta_old[a] * Sa.a[j][kk];
                    }
            }
            FP_tau = r_mmult(r_matexp(del_FP, &e_terms, &status), FP_t2);
            // ---- :361-396
            const R3 tinv = r_inv(FP_tau);
            FE_tau = r_mmult(F_tau, tinv);
            Ce_tau = r_Tmmult(FE_tau, FE_tau);
            R3 E2 = Ce_tau;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) E2.a[r][c] = 0.5 * (E2.a[r][c] - (r == c ? 1.0 : 0.0));
            T_star_tau = r_voigt(Dmat, E2);
            const R3 ct = r_mmult(Ce_tau, T_star_tau);
            for (int a = 0; a < n; ++a) {
                const R3 Sa = S(a);
                double r = 0.0;
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk) r += ct.a[j][kk] * Sa.a[j][kk];
                tau[a] = r;
                if (a > ns - 1) {
                    if ((tau_trial[a] - W_kh_tau[a]) < 0) tau[a] = W_kh_tau[a];
                }
            }
            // ---- :399-436 hardening, saturation caps, backstress
            for (int a = 0; a < n; ++a) {
                double h1 = 0;
                for (int c = 0; c < n; ++c) h1 = h1 + h_ab(a, c) * x_beta[c];
                s_alpha_tau[a] = s_alpha_tau[a] + h1;
            }
            for (int a = 0; a < ns; ++a)
                if (s_alpha_tau[a] > ldg(&L.ss[a])) s_alpha_tau[a] = ldg(&L.ss[a]);
            for (int a = 0; a < nw; ++a)
                if (s_alpha_tau[ns + a] > ldg(&L.ss[ns + a])) s_alpha_tau[ns + a] = ldg(&L.ss[ns + a]);
            for (int a = 0; a < n; ++a) {
                if ((tau_trial[a] - W_kh_tau[a]) > 0)
                    W_kh_tau[a] = W_kh_tau[a] + (ldg(&L.C1[a]) - ldg(&L.C2[a]) * W_kh_tau[a]) * (x_beta[a]);
                else
                    W_kh_tau[a] = W_kh_tau[a] + (-ldg(&L.C1[a]) - ldg(&L.C2[a]) * W_kh_tau[a]) * (x_beta[a]);
            }
            for (int a = 0; a < n; ++a) b[a] = fabs(tau[a] - W_kh_tau[a]) - s_alpha_tau[a];
        }

        // ---- :450-456 twin and slip fractions
        for (int a = 0; a < nw; ++a)
            g.tw_i[(int64_t)a * cnt + i] = g.tw_c[(int64_t)a * cnt + i] + x_beta_old[a + ns] / L.twin_shear;
        for (int a = 0; a < ns; ++a) g.sl_i[(int64_t)a * cnt + i] = g.sl_c[(int64_t)a * cnt + i] + x_beta_old[a];

        // ---- :458-468 stresses at the updated state
        Fpn_inv = r_inv(FP_tau);
        FE_tau = r_mmult(F_tau, Fpn_inv);
        det_FE_tau = r_det(FE_tau);
        t = r_mmult(FE_tau, T_star_tau);
        t = r_scale(1.0 / det_FE_tau, t);
        T_tau = r_mTmult(t, FE_tau);
        det_F_tau = r_det(F_tau);
        Finv = r_inv(F_tau);
        P_tau = r_mTmult(T_tau, Finv);
        P_tau = r_scale(det_F_tau, P_tau);

        if (flag == 1) {
            // ---- :473-499
            for (int e = 0; e < 81; ++e) delFp_delF_prev[e] = delFp_delF[e];
            for (int e = 0; e < 9 * n; ++e) dels_delF_prev[e] = dels_delF[e];
            {
                const R3 temp1 = r_mmult(F_tau, Fpn_inv);
                for (int r = 0; r < 3; ++r)
                    for (int j = 0; j < 3; ++j)
                        for (int kk = 0; kk < 3; ++kk)
                            for (int l = 0; l < 3; ++l) {
                                double v = 0.0;
                                for (int a = 0; a < 3; ++a)
                                    for (int bb = 0; bb < 3; ++bb)
                                        v = v - temp1.a[r][a] * delFp_delF[(3 * a + bb) * 9 + 3 * kk + l] *
                                                    Fpn_inv.a[bb][j];
                                if (r == kk) v = v + Fpn_inv.a[l][j];
                                delFe_delF[(3 * r + j) * 9 + 3 * kk + l] = v;
                            }
            }
            // ---- :501-514
            for (int r = 0; r < 3; ++r)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                v = v + 0.5 * (delFe_delF[(3 * a + r) * 9 + 3 * kk + l] * FE_tau.a[a][j] +
                                               delFe_delF[(3 * a + j) * 9 + 3 * kk + l] * FE_tau.a[a][r]);
                            delEtrial_delF[(3 * r + j) * 9 + 3 * kk + l] = v;
                        }
            // (:518-530 compute two exponentials that are overwritten before use)
            for (int r = 0; r < 9; ++r)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < 9; ++kk) s += TM[9 * r + kk] * delEtrial_delF[kk * 9 + j];
                    delT_delF[r * 9 + j] = s;
                }
            // ---- :533-545
            for (int r = 0; r < 3; ++r)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                v = v + 2 * delEtrial_delF[(3 * r + a) * 9 + 3 * kk + l] * T_star_tau.a[a][j] +
                                    Ce_tau.a[r][a] * delT_delF[(3 * a + j) * 9 + 3 * kk + l];
                            deltau_delF[(3 * r + j) * 9 + 3 * kk + l] = v;
                        }
            // ---- :548-579 hardening sensitivity: dels_delF = inv(I - term_ds) dels_delF_prev
            for (int a = 0; a < ns; ++a)
                delh[a] = ldg(&L.h0[a]) * ref_pow((1 - s_alpha_tau[a] / ldg(&L.ss[a])), (ldg(&L.a[a]) - 1)) *
                          (-1.0 / ldg(&L.ss[a]));
            for (int a = 0; a < nw; ++a)
                delh[ns + a] = ldg(&L.h0[ns + a]) *
                               ref_pow((1 - s_alpha_tau[ns + a] / ldg(&L.ss[ns + a])), (ldg(&L.a[ns + a]) - 1)) *
                               (-1.0 / ldg(&L.ss[ns + a]));
            {
                double* Im = Wk;
                double* Iinv = Wk + (int64_t)n * n;
                double* Mt = Wk + 2ll * n * n;
                for (int kk = 0; kk < n; ++kk)
                    for (int l = 0; l < n; ++l)
                        Im[kk * n + l] = (kk == l ? 1.0 : 0.0) - x_beta_old[l] * ldg(&L.q[kk * NM + l]) * delh[l];
                r_invert(Im, n, Iinv, Mt, iperm);
                for (int a = 0; a < n; ++a)
                    for (int j = 0; j < 9; ++j) {
                        double s = 0.0;
                        for (int kk = 0; kk < n; ++kk) s += Iinv[a * n + kk] * dels_delF_prev[kk * 9 + j];
                        dels_delF[a * 9 + j] = s;
                    }
            }
            // ---- :581-604 delb_delF = +-(deltau_delF^T vec(S_PA(k)))
            for (int kk = 0; kk < nPA; ++kk) {
                const double* v1 = Sf + 9 * PA[kk];
                for (int l = 0; l < 9; ++l) {
                    double s = 0.0;
                    for (int m = 0; m < 9; ++m) s += deltau_delF[m * 9 + l] * v1[m];
                    if ((tau_trial[PA[kk]] - W_kh_t[PA[kk]]) < 0) s = -1.0 * s;
                    delb[kk * 9 + l] = s;
                }
            }
            // ---- :607-619 number of Gateaux-series terms
            double tol2 = 1.0;
            unsigned count3 = 0;
            {
                R3 t1 = r_zero(), t2b = r_eye();
                while (tol2 > fmax(tol1 / 1e4, 1e-12)) {
                    count3 = count3 + 1;
                    t1 = r_mmult(del_FP, t2b);
                    t1 = r_scale((1.0 / count3), t1);
                    tol2 = r_frob(t1);
                    t2b = t1;
                    if (count3 > 200) {
                        status |= QP_SERIES_CAP;
                        break;
                    }
                }
            }
            c_terms = (int)count3;
            // ---- :622-709 A2 (matrixExponential(-del_FP) at :682 is the same
            // for every entry and is evaluated once)
            double* A2 = Wk;
            double* A2inv = Wk + (int64_t)n * n;
            double* Mt = Wk + 2ll * n * n;
            for (int r = 0; r < nPA; ++r)
                for (int c = 0; c < nPA; ++c) A2[r * nPA + c] = h_ab(PA[r], PA[c]);
            int mst = 0;
            const R3 expm = r_matexp(r_scale(-1.0, del_FP), nullptr, &mst);
            const R3 temp6 = r_mmult(CE_tau_trial, expm);
            for (int c = 0; c < nPA; ++c) {
                const R3 diff = r_gateaux(S(PA[c]), del_FP, (int)count3, true);
                R3 temp2 = r_Tmmult(diff, temp6);
                r_symmetrize(temp2);
                R3 temp3 = r_voigt(Dmat, temp2);
                R3 tmp = r_mmult(Ce_tau, temp3);
                temp3 = r_mmult(temp2, T_star_tau);
                r_add(tmp, 2.0, temp3);
                const bool nj = (tau_trial[PA[c]] - W_kh_t[PA[c]]) < 0.0;
                for (int r = 0; r < nPA; ++r) {
                    const int ar = PA[r];
                    const R3 Sr = S(ar);
                    double a2 = A2[r * nPA + c];
                    const bool ni = (tau_trial[ar] - W_kh_t[ar]) < 0.0;
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            if (ni ^ nj)
                                a2 -= Sr.a[kk][l] * tmp.a[kk][l];
                            else
                                a2 += Sr.a[kk][l] * tmp.a[kk][l];
                        }
                    if (ni)
                        a2 -= ldg(&L.C1[ar]) - ldg(&L.C2[ar]) * W_kh_tau[ar];
                    else
                        a2 += ldg(&L.C1[ar]) - ldg(&L.C2[ar]) * W_kh_tau[ar];
                    A2[r * nPA + c] = a2;
                }
            }
            // ---- :712-729 delgamma_delF = inv(A2) (delb_delF - dels_delF[PA])
            if (r_invert(A2, nPA, A2inv, Mt, iperm)) status |= QP_SINGULAR;
            for (int r = 0; r < nPA; ++r)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < nPA; ++kk)
                        s += A2inv[r * nPA + kk] * (delb[kk * 9 + j] - dels_delF[PA[kk] * 9 + j]);
                    dg[r * 9 + j] = s;
                }
            // ---- :734-796 S_PA (9 x nPA)
            for (int c = 0; c < nPA; ++c) {
                const R3 diff = r_gateaux(S(PA[c]), del_FP, (int)count3, false);
                const R3 t1 = r_mmult(diff, FP_t2);
                const bool nj = (tau_trial[PA[c]] - W_kh_t[PA[c]]) < 0;
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) S_PA[(3 * kk + l) * nPA + c] = nj ? -t1.a[kk][l] : t1.a[kk][l];
            }
            // ---- :799-821 delFp_delF = exp(del_FP) delFp_delF_prev + S_PA delgamma
            const R3 expp = r_matexp(del_FP, nullptr, &mst);
            for (int r = 0; r < 3; ++r)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                v = v + expp.a[r][a] * delFp_delF_prev[(3 * a + j) * 9 + 3 * kk + l];
                            delFp_delF[(3 * r + j) * 9 + 3 * kk + l] = v;
                        }
            for (int r = 0; r < 9; ++r)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < nPA; ++kk) s += S_PA[r * nPA + kk] * dg[kk * 9 + j];
                    delFp_delF[r * 9 + j] += 1.0 * s;
                }
        }
        iter1 = iter1 + 1;
    }

    // ---- :835-940 final tangent
    if (flag == 1 && out.dPdF) {
        double* dFe = delFe_delF;
        double* dTs = delEtrial_delF;  // delTstar
        const R3 temp1 = r_mmult(F_tau, Fpn_inv);
        for (int r = 0; r < 3; ++r)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                v = v - temp1.a[r][a] * delFp_delF[(3 * a + bb) * 9 + 3 * kk + l] * Fpn_inv.a[bb][j];
                        if (r == kk) v = v + Fpn_inv.a[l][j];
                        dFe[(3 * r + j) * 9 + 3 * kk + l] = v;
                    }
        for (int r = 0; r < 3; ++r)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                for (int c = 0; c < 3; ++c)
                                    v = v + TM[(3 * r + j) * 9 + 3 * a + bb] * dFe[(3 * c + a) * 9 + 3 * kk + l] *
                                                FE_tau.a[c][bb];
                        dTs[(3 * r + j) * 9 + 3 * kk + l] = v;
                    }
        const R3 temp4 = r_inv(F_tau);
        const R3 tmp = r_mmult(temp4, FE_tau);
        const R3 t1 = r_mTmult(T_star_tau, tmp);
        const R3 t2 = r_mmult(temp4, FE_tau);
        const R3 t3 = r_mmult(FE_tau, T_star_tau);
        const R3 t5 = r_mTmult(t3, F_tau);
        for (int r = 0; r < 3; ++r)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            for (int bb = 0; bb < 3; ++bb)
                                v = v + (r == a ? 1.0 : 0.0) * dFe[(3 * a + bb) * 9 + 3 * kk + l] * t1.a[bb][j] +
                                    FE_tau.a[r][a] * dTs[(3 * a + bb) * 9 + 3 * kk + l] * t2.a[j][bb] -
                                    t3.a[r][a] * dFe[(3 * a + bb) * 9 + 3 * kk + l] * temp4.a[j][bb];
                            v = v - t5.a[r][a] * temp4.a[j][kk] * temp4.a[l][a];
                        }
                        // :916-939 rotate back with L = I (a copy)
                        out.dPdF[(3 * r + j) * 9 + 3 * kk + l] = out.scale * v;
                    }
    }

    // ---- :942-959 outputs and history
    if (out.P)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) out.P[3 * r + c] = out.scale * P_tau.a[r][c];
    if (out.T) r_store(T_tau, out.T);
    soa_store(g.Fe_i, cnt, i, FE_tau);
    soa_store(g.Fp_i, cnt, i, FP_tau);
    for (int a = 0; a < n; ++a) {
        g.s_i[(int64_t)a * cnt + i] = s_alpha_tau[a];
        g.W_i[(int64_t)a * cnt + i] = W_kh_tau[a];
    }

    // ---- :962-1019 twin reorientation (rod2quat's cos(atan(|r|)) as
    // 1/sqrt(1 + r.r), updateAfterIncrement.cc:781-821)
    if (L.twinning) {
        double F_T;
        if (!o.multiphase) {
            if (F_r > 0)
                F_T = L.twin_thr + (L.twin_sat * F_e / F_r);
            else
                F_T = L.twin_thr;
        } else {
            F_T = L.twin_thr;
        }
        if (F_T > 1.0) F_T = 1.0;
        int twin_pos = 0;
        double twin_max = g.tw_i[i];
        for (int a = 1; a < nw; ++a)
            if (g.tw_i[(int64_t)a * cnt + i] > twin_max) {
                twin_max = g.tw_i[(int64_t)a * cnt + i];
                twin_pos = a;
            }
        if (g.twin_c[i] != 1 && F_r > 0 && twin_max > F_T) {
            double rod[3] = {rot1[0], rot1[1], rot1[2]};
            const double dotrod = rod[0] * rod[0] + rod[1] * rod[1] + rod[2] * rod[2];
            const double cphiby2 = 1.0 / sqrt(1.0 + dotrod);
            const double quat2[4] = {cphiby2, cphiby2 * rod[0], cphiby2 * rod[1], cphiby2 * rod[2]};
            const double quat1[4] = {0, ldg(&L.nn[3 * (ns + twin_pos)]), ldg(&L.nn[3 * (ns + twin_pos) + 1]),
                                     ldg(&L.nn[3 * (ns + twin_pos) + 2])};
            double qp[4];
            const double a0 = quat2[0], b0 = quat1[0];
            const double dot1 = quat1[1] * quat2[1] + quat1[2] * quat2[2] + quat1[3] * quat2[3];
            qp[0] = (a0 * b0) - dot1;
            qp[1] = a0 * quat1[1] + b0 * quat2[1] + quat2[2] * quat1[3] - quat1[2] * quat2[3];
            qp[2] = a0 * quat1[2] + b0 * quat2[2] - quat2[1] * quat1[3] + quat1[1] * quat2[3];
            qp[3] = a0 * quat1[3] + b0 * quat2[3] + quat2[1] * quat1[2] - quat1[1] * quat2[2];
            if (qp[0] < 0)
                for (int c = 0; c < 4; ++c) qp[c] = -qp[c];
            if (fabs(qp[0]) < 1e-4) qp[0] = 1e-4;
            const double inv = 1 / qp[0];
            for (int c = 0; c <= 2; ++c) rod[c] = qp[c + 1] * inv;
            for (int c = 0; c < 3; ++c) {
                g.rot_i[(int64_t)c * cnt + i] = rod[c];
                g.rotnew_i[(int64_t)c * cnt + i] = rod[c];
            }
            g.twin_i[i] = 1;
            for (int a = 0; a < nw; ++a) g.s_i[(int64_t)(ns + a) * cnt + i] = 100000;
        }
    }

    bool finite = true;
    if (out.P)
        for (int c = 0; c < 9; ++c) finite = finite && isfinite(out.P[c]);
    if (flag == 1 && out.dPdF)
        for (int c = 0; c < 81; ++c) finite = finite && isfinite(out.dPdF[c]);
    if (!finite) status |= QP_NONFINITE;
    if (maxcond > 1e12) status |= QP_ILL_CONDITIONED;
    if (stats_out) {
        stats_out[0] = p0 < 0 ? 0 : p0;
        stats_out[1] = nPA;
        stats_out[2] = rounds_total;
        stats_out[3] = e_terms;
        stats_out[4] = c_terms;
        stats_out[5] = (int)iter1;
        stats_out[6] = lattice_id;
        stats_out[7] = isfinite(maxcond) ? (int)fmin(99.0, ceil(log10(maxcond))) : 99;
    }
    return status;
}

}  // namespace ref
}  // namespace cp
