/*
 * cp_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE ONLY; see cp_oracle.h).
 *
 * A line-by-line FP64 restatement of PRISMS-Plasticity's rate-independent
 * crystal-plasticity update.  Every block cites the reference file:line it
 * follows (paths relative to src/materialModels/crystalPlasticity/ unless
 * stated).  Computations the reference performs but whose results are never
 * read are skipped and say so; everything that can change a result is kept in
 * the reference's order.  Compile with -ffp-contract=off so every operation
 * rounds as written.
 */
#include "cp_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int NM = CP_MAX_SYSTEMS;

/* ---- the parity build (-DCP_ORACLE_PARITY, libcp_oracle_parity.so) -------
 * std::pow, std::tgamma and std::cos(std::atan(.)) are glibc's; a GPU has its
 * own.  The parity build replaces them with functions made only of correctly
 * rounded operations, so that a device evaluation of the same operations
 * (cp_options_t.reference_order) reproduces this build bit for bit:
 *   pow(x, y) = exp(y log x): log by 2 atanh((m-1)/(m+1)) on the mantissa
 *   m in [sqrt(1/2), sqrt(2)) (12 series terms in s^2), exp by Cody-Waite
 *   reduction with ln 2 split in two and 18 nested Taylor terms;
 *   tgamma(k + 2) = (k+1)! as the product 2 * 3 * ... * (k+1);
 *   cos(atan(r)) = 1 / sqrt(1 + r^2). */
const double P_LN2_HI = 0.693147180369123816490;
const double P_LN2_LO = 1.90821492927058770002e-10;
const double P_INV_LN2 = 1.44269504088896338700;
const double P_SQRT_HALF = 0.70710678118654752440;

double parity_log(double x) {
    int e = 0;
    double m = std::frexp(x, &e);
    if (m < P_SQRT_HALF) {
        m = m * 2.0;
        e = e - 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double p = 1.0 / 25.0;
    for (int j = 11; j >= 0; --j) p = p * z + 1.0 / (double)(2 * j + 1);
    const double lnm = (2.0 * s) * p;
    const double de = (double)e;
    return (de * P_LN2_HI + lnm) + de * P_LN2_LO;
}
double parity_exp(double t) {
    if (t != t) return t;
    if (t > 709.782712893384) return INFINITY;
    if (t < -745.2) return 0.0;
    const double kd = std::floor(t * P_INV_LN2 + 0.5);
    const double r = (t - kd * P_LN2_HI) - kd * P_LN2_LO;
    double p = 1.0;
    for (int j = 18; j >= 1; --j) p = 1.0 + (r / (double)j) * p;
    return std::ldexp(p, (int)kd);
}
double parity_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    if (x == 0.0) return y > 0.0 ? 0.0 : INFINITY;
    double ax = x, sign = 1.0;
    if (x < 0.0) {
        if (std::floor(y) != y) return (x - x) / (x - x);
        ax = -x;
        if (std::fmod(y, 2.0) != 0.0) sign = -1.0;
    }
    if (ax == INFINITY) return sign * (y > 0.0 ? INFINITY : 0.0);
    return sign * parity_exp(y * parity_log(ax));
}
#ifdef CP_ORACLE_PARITY
inline double o_pow(double x, double y) { return parity_pow(x, y); }
inline double o_fact(int k) {  /* (k+1)! = tgamma(k + 2) */
    double f = 1.0;
    for (int j = 1; j <= k; ++j) f = f * (double)(j + 1);
    return f;
}
inline double o_cos_atan(double r2) { return 1.0 / std::sqrt(1.0 + r2); }
#else
inline double o_pow(double x, double y) { return std::pow(x, y); }
inline double o_fact(int k) { return std::tgamma(k + 2); }
inline double o_cos_atan(double r2) { return std::cos(std::atan(std::sqrt(r2))); }
#endif

/* ---- 3x3 helpers with deal.II FullMatrix call semantics ------------------ */
struct M3 {
    double a[3][3];
};

inline M3 zero3() {
    M3 m;
    std::memset(m.a, 0, sizeof m.a);
    return m;
}
inline M3 eye3() {
    M3 m = zero3();
    m.a[0][0] = m.a[1][1] = m.a[2][2] = 1.0;
    return m;
}
inline M3 load3(const double* p) {
    M3 m;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m.a[i][j] = p[3 * i + j];
    return m;
}
inline void store3(const M3& m, double* p) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) p[3 * i + j] = m.a[i][j];
}
/* A.mmult(C,B): C = A B */
inline M3 mmult(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[i][k] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
/* A.Tmmult(C,B): C = A^T B */
inline M3 Tmmult(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[k][i] * B.a[k][j];
            C.a[i][j] = s;
        }
    return C;
}
/* A.mTmult(C,B): C = A B^T */
inline M3 mTmult(const M3& A, const M3& B) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A.a[i][k] * B.a[j][k];
            C.a[i][j] = s;
        }
    return C;
}
inline M3 scale3(double c, const M3& A) {
    M3 C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = c * A.a[i][j];
    return C;
}
/* A.add(c,B): A += c B */
inline void add3(M3& A, double c, const M3& B) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A.a[i][j] += c * B.a[i][j];
}
inline void symmetrize3(M3& A) {
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j) {
            const double t = (A.a[i][j] + A.a[j][i]) / 2;
            A.a[i][j] = A.a[j][i] = t;
        }
}
inline double frob3(const M3& A) {
    double s = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s += A.a[i][j] * A.a[i][j];
    return std::sqrt(s);
}
/* determinant by cofactor expansion along the first row */
inline double det3(const M3& A) {
    const double (*a)[3] = A.a;
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
           a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
/* inverse by the adjugate: inv = adj(A) * (1/det) */
inline M3 inv3(const M3& A) {
    const double (*a)[3] = A.a;
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    const double r = 1.0 / det;
    M3 B;
    B.a[0][0] = c00 * r;
    B.a[1][0] = c01 * r;
    B.a[2][0] = c02 * r;
    B.a[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * r;
    B.a[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * r;
    B.a[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * r;
    B.a[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * r;
    B.a[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * r;
    B.a[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * r;
    return B;
}

/* vecform / matform, matrixOperations.cc:133-163 (Voigt 11,22,33,23,13,12) */
inline void vecform(const M3& A, double v[6]) {
    v[0] = A.a[0][0];
    v[1] = A.a[1][1];
    v[2] = A.a[2][2];
    v[3] = A.a[1][2];
    v[4] = A.a[0][2];
    v[5] = A.a[0][1];
}
inline M3 matform(const double v[6]) {
    M3 A;
    A.a[0][0] = v[0];
    A.a[1][1] = v[1];
    A.a[2][2] = v[2];
    A.a[1][2] = v[3];
    A.a[0][2] = v[4];
    A.a[0][1] = v[5];
    A.a[2][1] = v[3];
    A.a[2][0] = v[4];
    A.a[1][0] = v[5];
    return A;
}
/* Dmat.vmult(out, vecform(A)) then matform */
inline M3 voigt_apply(const double D[6][6], const M3& A) {
    double v[6], w[6];
    vecform(A, v);
    for (int i = 0; i < 6; ++i) {
        double s = 0.0;
        for (int j = 0; j < 6; ++j) s += D[i][j] * v[j];
        w[i] = s;
    }
    return matform(w);
}

/* matrixExponential, matrixOperations.cc:165-186: Taylor series until the
 * Frobenius norm of the last term is <= 1e-10. */
inline M3 matexp(const M3& A, int* terms) {
    M3 E = eye3(), t = eye3();
    double count = 1;
    int k = 0;
    while (frob3(t) > 1.0e-10) {
        M3 t2 = mmult(t, A);
        t2 = scale3(1 / count, t2);
        t = t2;
        add3(E, 1.0, t);
        count = count + 1.0;
        ++k;
    }
    if (terms) *terms = k;
    return E;
}

/* odfpoint, rotationOperations.cc:4-51: Rodrigues vector -> rotation. */
inline M3 odfpoint(const double r[3]) {
    double rdotr = 0.0;
    for (int i = 0; i < 3; ++i) rdotr = rdotr + r[i] * r[i];
    const double term1 = 1.0 - rdotr;
    const double term2 = 1.0 + rdotr;
    M3 R = eye3();
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

/* elasticmoduli, matrixOperations.cc:189-234: Ar = N(R) C N(R)^T with the
 * 6x6 Bond-type rotation N built from R. */
inline void elasticmoduli(const M3& Rm, const double C[6][6], double Ar[6][6]) {
    const double (*R)[3] = Rm.a;
    double N[6][6];
    for (int i = 0; i < 3; ++i) {
        N[i][0] = R[i][0] * R[i][0];
        N[i][1] = R[i][1] * R[i][1];
        N[i][2] = R[i][2] * R[i][2];
        N[i][3] = 2.0 * R[i][1] * R[i][2];
        N[i][4] = 2.0 * R[i][2] * R[i][0];
        N[i][5] = 2.0 * R[i][0] * R[i][1];
    }
    /* rows 3,4,5 pair (1,2), (2,0), (0,1) */
    const int pr[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    for (int r = 0; r < 3; ++r) {
        const int p = pr[r][0], q = pr[r][1];
        N[3 + r][0] = R[p][0] * R[q][0];
        N[3 + r][1] = R[p][1] * R[q][1];
        N[3 + r][2] = R[p][2] * R[q][2];
    }
    N[3][3] = R[1][1] * R[2][2] + R[1][2] * R[2][1];
    N[3][4] = R[1][2] * R[2][0] + R[1][0] * R[2][2];
    N[3][5] = R[1][0] * R[2][1] + R[1][1] * R[2][0];
    N[4][3] = R[0][1] * R[2][2] + R[0][2] * R[2][1];
    N[4][4] = R[0][2] * R[2][0] + R[0][0] * R[2][2];
    N[4][5] = R[0][0] * R[2][1] + R[0][1] * R[2][0];
    N[5][3] = R[0][1] * R[1][2] + R[0][2] * R[1][1];
    N[5][4] = R[0][2] * R[1][0] + R[0][0] * R[1][2];
    N[5][5] = R[0][0] * R[1][1] + R[0][1] * R[1][0];
    double T[6][6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += N[i][k] * C[k][j];
            T[i][j] = s;
        }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += T[i][k] * N[j][k];
            Ar[i][j] = s;
        }
}

/* ---- dense n x n helpers -------------------------------------------------- */

/* FullMatrix::invert: closed form up to 3x3, Gauss-Jordan with partial
 * (row) pivoting above.  Returns 0, or 1 if a pivot is exactly zero. */
int invert_n(const double* A, int n, double* B) {
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
        return !std::isfinite(t);
    }
    if (n == 3) {
        M3 m = load3(A);
        store3(inv3(m), B);
        return !std::isfinite(B[0]);
    }
    std::vector<double> M(A, A + (size_t)n * n);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    int sing = 0;
    /* in-place Gauss-Jordan: M <- M^{-1} (columns permuted by the pivot rows) */
    for (int j = 0; j < n; ++j) {
        int r = j;
        double mx = std::fabs(M[(size_t)j * n + j]);
        for (int i = j + 1; i < n; ++i)
            if (std::fabs(M[(size_t)i * n + j]) > mx) {
                mx = std::fabs(M[(size_t)i * n + j]);
                r = i;
            }
        if (mx == 0.0) sing = 1;
        if (r != j) {
            for (int k = 0; k < n; ++k) std::swap(M[(size_t)j * n + k], M[(size_t)r * n + k]);
            std::swap(perm[j], perm[r]);
        }
        const double piv = 1.0 / M[(size_t)j * n + j];
        for (int i = 0; i < n; ++i) M[(size_t)i * n + j] *= piv;
        M[(size_t)j * n + j] = piv;
        for (int k = 0; k < n; ++k) {
            if (k == j) continue;
            for (int i = 0; i < n; ++i) {
                if (i == j) continue;
                M[(size_t)i * n + k] -= M[(size_t)i * n + j] * M[(size_t)j * n + k];
            }
        }
        for (int k = 0; k < n; ++k) M[(size_t)j * n + k] *= -piv;
        M[(size_t)j * n + j] = piv;
    }
    /* undo the row exchanges as column exchanges of the inverse */
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) B[(size_t)i * n + perm[k]] = M[(size_t)i * n + k];
    return sing;
}

/* Pseudo-inverse by one-sided (Hestenes) Jacobi SVD, standing in for
 * LAPACKFullMatrix::compute_inverse_svd(0.0) (inactiveSlipRemoval.cc:26,99):
 * A = U S V^T, A^+ = V S^+ U^T, where singular values not above
 * threshold*max are treated as zero (threshold 0: only exact zeros). */
int pinv_svd(const double* A, int n, double* Ainv, double* cond = nullptr) {
    if (cond) *cond = 1.0;
    if (n == 0) return 0;
    std::vector<double> U(A, A + (size_t)n * n), V((size_t)n * n, 0.0), s(n);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    const double eps = 1e-15;
    for (int sweep = 0; sweep < 60; ++sweep) {
        int rotated = 0;
        for (int i = 0; i < n - 1; ++i)
            for (int j = i + 1; j < n; ++j) {
                double alpha = 0.0, beta = 0.0, gamma = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double ui = U[(size_t)k * n + i], uj = U[(size_t)k * n + j];
                    alpha += ui * ui;
                    beta += uj * uj;
                    gamma += ui * uj;
                }
                if (gamma == 0.0 || std::fabs(gamma) <= eps * std::sqrt(alpha * beta)) continue;
                rotated = 1;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t);
                const double sn = c * t;
                for (int k = 0; k < n; ++k) {
                    const double ui = U[(size_t)k * n + i], uj = U[(size_t)k * n + j];
                    U[(size_t)k * n + i] = c * ui - sn * uj;
                    U[(size_t)k * n + j] = sn * ui + c * uj;
                    const double vi = V[(size_t)k * n + i], vj = V[(size_t)k * n + j];
                    V[(size_t)k * n + i] = c * vi - sn * vj;
                    V[(size_t)k * n + j] = sn * vi + c * vj;
                }
            }
        if (!rotated) break;
    }
    double smax = 0.0;
    for (int i = 0; i < n; ++i) {
        double ss = 0.0;
        for (int k = 0; k < n; ++k) ss += U[(size_t)k * n + i] * U[(size_t)k * n + i];
        s[i] = std::sqrt(ss);
        smax = std::max(smax, s[i]);
    }
    const double threshold = 0.0;
    if (cond) {
        double smin = smax;
        for (int i = 0; i < n; ++i) smin = std::min(smin, s[i]);
        *cond = smin > 0.0 ? smax / smin : INFINITY;
    }
    int sing = 0;
    std::vector<double> sinv(n);
    for (int i = 0; i < n; ++i) {
        if (s[i] > threshold * smax && s[i] > 0.0) {
            sinv[i] = 1.0 / s[i];
        } else {
            sinv[i] = 0.0;
            sing = 1;
        }
    }
    /* A^+ = V diag(1/s^2) (A V)^T, with (A V) = U_unnormalised = U_n diag(s) */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k)
                acc += V[(size_t)i * n + k] * (sinv[k] * sinv[k]) * U[(size_t)j * n + k];
            Ainv[(size_t)i * n + j] = acc;
        }
    return sing;
}

/* Cyclic Jacobi eigen-decomposition of a symmetric 3x3, standing in for
 * LAPACK syevx (reorient.cc:35,48).  evecs columns are eigenvectors. */
void eig_sym3(const M3& C, double ev[3], M3& V) {
    M3 A = C;
    V = eye3();
    for (int sweep = 0; sweep < 50; ++sweep) {
        const double off = A.a[0][1] * A.a[0][1] + A.a[0][2] * A.a[0][2] + A.a[1][2] * A.a[1][2];
        const double dia = A.a[0][0] * A.a[0][0] + A.a[1][1] * A.a[1][1] + A.a[2][2] * A.a[2][2];
        if (off <= 1e-32 * dia || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = A.a[p][q];
                if (apq == 0.0) continue;
                const double theta = (A.a[q][q] - A.a[p][p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = A.a[k][p], akq = A.a[k][q];
                    A.a[k][p] = c * akp - s * akq;
                    A.a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A.a[p][k], aqk = A.a[q][k];
                    A.a[p][k] = c * apk - s * aqk;
                    A.a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V.a[k][p], vkq = V.a[k][q];
                    V.a[k][p] = c * vkp - s * vkq;
                    V.a[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) ev[i] = A.a[i][i];
}

/* ---- per-lattice constants (multiphaseInit.cc:4-67, init.cc:29-196) ----- */
struct Lattice {
    int ns, nw, n;
    double C[6][6];
    double m[NM][3], nn[NM][3];
    const double* q; /* row stride NM */
    const double *h0, *ss, *a, *C1, *C2;
    double twin_thr, twin_sat, twin_shear;
    int twinning;
};

Lattice make_lattice(const cp_material_t* mat) {
    Lattice L;
    L.ns = mat->n_slip;
    L.nw = mat->n_twin;
    L.n = L.ns + L.nw;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) L.C[i][j] = mat->elastic_stiffness[6 * i + j];
    for (int i = 0; i < L.n; ++i)
        for (int j = 0; j < 3; ++j) {
            L.m[i][j] = mat->slip_direction[3 * i + j];
            L.nn[i][j] = mat->slip_normal[3 * i + j];
        }
    L.q = mat->latent_hardening;
    L.h0 = mat->initial_hardening_modulus;
    L.ss = mat->saturation_stress;
    L.a = mat->power_law_exponent;
    L.C1 = mat->kinematic_c1;
    L.C2 = mat->kinematic_c2;
    L.twin_thr = mat->twin_threshold_fraction;
    L.twin_sat = mat->twin_saturation_factor;
    L.twin_shear = mat->twin_shear;
    L.twinning = mat->twinning_enabled;
    return L;
}

/* inactive_slip_removal, inactiveSlipRemoval.cc:4-124.  b and A are taken
 * by value in the reference; PA/n_PA are updated in place; x_old += x. */
int inactive_slip_removal(int n, std::vector<int>& PA, const double* b,
                          const std::vector<double>& A, double* x_old, double* x,
                          int* rounds, double* maxcond) {
    double cnd = 1.0;
    int sing = 0;
    int nPA = (int)PA.size();
    std::vector<double> Apa((size_t)nPA * nPA), Ainv((size_t)nPA * nPA), bpa(nPA), x1(n, 0.0);
    for (int i = 0; i < nPA; ++i) {
        bpa[i] = b[PA[i]];
        for (int j = 0; j < nPA; ++j) Apa[(size_t)i * nPA + j] = A[(size_t)PA[i] * NM + PA[j]];
    }
    sing |= pinv_svd(Apa.data(), nPA, Ainv.data(), &cnd);
    *maxcond = std::max(*maxcond, cnd);
    *rounds = 1;
    for (int i = 0; i < nPA; ++i) {
        double s = 0.0;
        for (int j = 0; j < nPA; ++j) s += Ainv[(size_t)i * nPA + j] * bpa[j];
        x1[PA[i]] = s;
    }
    for (;;) {
        std::vector<int> row;
        for (int i = 0; i < n; ++i)
            if ((x_old[i] + x1[i]) < 0) row.push_back(i);
        if (row.empty()) break;
        std::vector<int> PAn;
        for (int i = 0; i < nPA; ++i) {
            int keep = 1;
            for (int r : row)
                if (PA[i] == r) keep = 0;
            if (keep) PAn.push_back(PA[i]);
        }
        PA = PAn;
        const int m = (int)PA.size();
        Apa.assign((size_t)m * m, 0.0);
        Ainv.assign((size_t)m * m, 0.0);
        bpa.assign(m, 0.0);
        for (int i = 0; i < m; ++i) {
            bpa[i] = b[PA[i]];
            for (int j = 0; j < m; ++j) Apa[(size_t)i * m + j] = A[(size_t)PA[i] * NM + PA[j]];
        }
        sing |= pinv_svd(Apa.data(), m, Ainv.data(), &cnd);
        *maxcond = std::max(*maxcond, cnd);
        ++*rounds;
        std::fill(x1.begin(), x1.end(), 0.0);
        nPA = m;
        for (int i = 0; i < nPA; ++i) {
            double s = 0.0;
            for (int j = 0; j < nPA; ++j) s += Ainv[(size_t)i * nPA + j] * bpa[j];
            x1[PA[i]] = s;
        }
    }
    for (int i = 0; i < n; ++i) x[i] = x1[i];
    for (int i = 0; i < n; ++i) x_old[i] += x[i];
    return sing;
}

/* rod2quat / quatproduct / quat2rod, updateAfterIncrement.cc:781-821 */
void rod2quat(double quat[4], const double rod[3]) {
    const double dotrod = rod[0] * rod[0] + rod[1] * rod[1] + rod[2] * rod[2];
    const double cphiby2 = o_cos_atan(dotrod);
    quat[0] = cphiby2;
    quat[1] = cphiby2 * rod[0];
    quat[2] = cphiby2 * rod[1];
    quat[3] = cphiby2 * rod[2];
}
void quatproduct(double qp[4], const double q2[4], const double q1[4]) {
    const double a = q2[0], b = q1[0];
    const double dot1 = q1[1] * q2[1] + q1[2] * q2[2] + q1[3] * q2[3];
    qp[0] = (a * b) - dot1;
    qp[1] = a * q1[1] + b * q2[1] + q2[2] * q1[3] - q1[2] * q2[3];
    qp[2] = a * q1[2] + b * q2[2] - q2[1] * q1[3] + q1[1] * q2[3];
    qp[3] = a * q1[3] + b * q2[3] + q2[1] * q1[2] - q1[1] * q2[2];
    if (qp[0] < 0)
        for (int i = 0; i < 4; ++i) qp[i] = -qp[i];
}
void quat2rod(double quat[4], double rod[3]) {
    if (std::fabs(quat[0]) < 1e-4) quat[0] = 1e-4;
    const double inv = 1 / quat[0];
    for (int i = 0; i <= 2; ++i) rod[i] = quat[i + 1] * inv;
}

/* the Gateaux-series terms of calculatePlasticity.cc:645-676 / 748-779:
 * D = S + sum_{k=1..count3} coef(k) sum_{l=0..k} dFp^l S dFp^(k-l) */
M3 gateaux_series(const M3& S, const M3& dFp, int count3, bool alternating) {
    M3 diff = S;
    for (int k = 1; k <= count3; ++k) {
        M3 t4 = zero3();
        for (int l = 0; l <= k; ++l) {
            M3 t1 = eye3(), t2 = eye3();
            for (int m = 0; m < l; ++m) t1 = mmult(t1, dFp);
            for (int m = 0; m < k - l; ++m) t2 = mmult(t2, dFp);
            M3 t5 = mmult(t1, S);
            M3 t6 = mmult(t5, t2);
            add3(t4, 1.0, t6);
        }
        const double coef = (alternating ? ((k & 1) ? -1.0 : 1.0) : 1.0) / o_fact(k);
        t4 = scale3(coef, t4);
        add3(diff, 1.0, t4);
    }
    return diff;
}

struct QpIO {
    const double* F;
    double *P, *T, *dPdF;
    int32_t* stats;
    int32_t* status;
};

/* calculatePlasticity, calculatePlasticity.cc:13-1022, for qp k. */
int calculate_plasticity(const Lattice& L, const cp_options_t& opt, const or_state& st,
                         int64_t k, const QpIO& io, int flag, double F_e, double F_r) {
    const int n = L.n, ns = L.ns, nw = L.nw;
    int status = 0;
    const double tol1 = opt.stress_tolerance;
    const M3 F_tau = load3(io.F);
    const M3 FP_t = load3(st.Fp_conv + 9 * k);
    double s_alpha_t[NM], W_kh_t[NM];
    for (int i = 0; i < n; ++i) {
        s_alpha_t[i] = st.s_conv[k * n + i];
        W_kh_t[i] = st.W_conv[k * n + i];
    }
    double rot1[3] = {st.rot_conv[3 * k], st.rot_conv[3 * k + 1], st.rot_conv[3 * k + 2]};

    /* :39-77 rotation, rotated stiffness, engineering-shear Dmat, 9x9 TM */
    const M3 rotmat = odfpoint(rot1);
    double Dmat2[6][6], Dmat[6][6], TM[9][9];
    elasticmoduli(rotmat, L.C, Dmat2);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Dmat[i][j] = Dmat2[i][j];
    for (int i = 0; i < 6; ++i)
        for (int j = 3; j < 6; ++j) Dmat[i][j] = 2 * Dmat[i][j];
    const int vec2[9] = {0, 5, 4, 5, 1, 3, 4, 3, 2};
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) TM[i][j] = Dmat2[vec2[i]][vec2[j]];

    /* :79-112 Schmid tensors in sample coordinates.  B (=2 sym(CE_tau_trial S))
     * is skipped: CE_tau_trial is still the zero matrix there (declared :47,
     * first assigned :168) and B is never read. */
    std::vector<M3> S(n);
    for (int i = 0; i < n; ++i) {
        M3 t = zero3();
        for (int j = 0; j < 3; ++j)
            for (int kk = 0; kk < 3; ++kk) t.a[j][kk] = L.m[i][j] * L.nn[i][kk];
        M3 t2 = mmult(rotmat, t);
        S[i] = mTmult(t2, rotmat);
    }

    /* :114-151 */
    double s_alpha_tau[NM], W_kh_tau[NM];
    double tau_trial[NM], b[NM], tau[NM], x_beta_old[NM], x_beta[NM];
    double h_beta[NM];
    std::vector<double> h_ab((size_t)NM * NM, 0.0), A((size_t)NM * NM, 0.0);
    std::vector<int> PA;
    M3 FP_tau = FP_t;
    M3 Fpn_inv = inv3(FP_t);
    M3 FE_tau = mmult(F_tau, Fpn_inv);
    for (int i = 0; i < n; ++i) {
        s_alpha_tau[i] = s_alpha_t[i];
        W_kh_tau[i] = W_kh_t[i];
        x_beta_old[i] = 0.0;
        x_beta[i] = 0.0;
        tau[i] = 0.0;
        tau_trial[i] = 0.0;
    }
    double delFp_delF[9][9], delFp_delF_prev[9][9];
    std::memset(delFp_delF, 0, sizeof delFp_delF);
    /* dels_delF (:131) starts at zero (:148) and is only ever re-assigned as
     * inv(I - term_ds) * dels_delF_prev with dels_delF_prev = dels_delF (:477,
     * :579), so it stays exactly zero; its A_ds update (:823-827) is
     * overwritten at :477 before use.  It is carried here anyway. */
    std::vector<double> dels_delF((size_t)n * 9, 0.0), dels_delF_prev((size_t)n * 9, 0.0);

    M3 FP_t2 = FP_tau, CE_tau_trial = zero3(), T_star_tau = zero3(), T_star_tau_trial = zero3();
    M3 Ce_tau = zero3(), del_FP = zero3(), T_tau = zero3(), P_tau = zero3();
    double det_FE_tau, det_F_tau;
    int nPA = 0, p0 = -1, rounds_total = 0, e_terms = 0, c_terms = 0;
    double maxcond = 1.0;
    unsigned iter1 = 1;

    while (iter1) {
        if (iter1 > (unsigned)opt.max_slip_search_iterations) {
            status |= CP_QP_SLIP_SEARCH_CAP;
            break;
        }
        /* :160-176 trial kinematics */
        FP_t2 = FP_tau;
        Fpn_inv = inv3(FP_t2);
        M3 FE_tau_trial = mmult(F_tau, Fpn_inv);
        CE_tau_trial = Tmmult(FE_tau_trial, FE_tau_trial);
        M3 Ee = CE_tau_trial;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Ee.a[i][j] = 0.5 * (Ee.a[i][j] - (i == j ? 1.0 : 0.0));
        /* :180-196 trial stress */
        T_star_tau_trial = voigt_apply(Dmat, Ee);
        T_star_tau = T_star_tau_trial;
        det_FE_tau = det3(FE_tau);
        M3 t = mmult(FE_tau, T_star_tau_trial);
        t = scale3(1.0 / det_FE_tau, t);
        T_tau = mTmult(t, FE_tau);
        det_F_tau = det3(F_tau);
        M3 Finv = inv3(F_tau);
        M3 t2 = mTmult(T_tau, Finv);
        P_tau = scale3(det_FE_tau, t2);
        /* :199-244 resolved shear and potentially active set */
        t = mmult(CE_tau_trial, T_star_tau_trial);
        PA.clear();
        for (int i = 0; i < n; ++i) {
            double r = 0.0;
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk) r += t.a[j][kk] * S[i].a[j][kk];
            tau_trial[i] = r;
            if (i > ns - 1) {
                if ((tau_trial[i] - W_kh_tau[i]) < 0) tau_trial[i] = W_kh_tau[i];
            }
            b[i] = std::fabs(tau_trial[i] - W_kh_tau[i]) - s_alpha_tau[i];
            if (b[i] >= tol1) PA.push_back(i);
        }
        nPA = (int)PA.size();
        if (p0 < 0) p0 = nPA;
        for (int i = 0; i < n; ++i) tau[i] = tau_trial[i];
        if (nPA == 0) break;

        /* :250-306 hardening moduli and the consistency matrix A */
        for (int i = 0; i < ns; ++i)
            h_beta[i] = L.h0[i] * o_pow((1 - s_alpha_tau[i] / L.ss[i]), L.a[i]);
        for (int i = 0; i < nw; ++i)
            h_beta[ns + i] = L.h0[ns + i] * o_pow((1 - s_alpha_tau[ns + i] / L.ss[ns + i]), L.a[ns + i]);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                h_ab[(size_t)i * NM + j] = L.q[(size_t)i * NM + j] * h_beta[j];
                A[(size_t)i * NM + j] = h_ab[(size_t)i * NM + j];
            }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                M3 temp2 = mmult(CE_tau_trial, S[j]);
                symmetrize3(temp2);
                M3 temp3 = voigt_apply(Dmat, temp2);
                M3 temp1 = mmult(CE_tau_trial, temp3);
                temp3 = mmult(temp2, T_star_tau_trial);
                add3(temp1, 2.0, temp3);
                double& Aij = A[(size_t)i * NM + j];
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        if (((tau_trial[i] - W_kh_tau[i]) * (tau_trial[j] - W_kh_tau[j])) < 0.0)
                            Aij -= S[i].a[kk][l] * temp1.a[kk][l];
                        else
                            Aij += S[i].a[kk][l] * temp1.a[kk][l];
                    }
                if ((tau_trial[i] - W_kh_tau[i]) < 0.0)
                    Aij -= L.C1[i] - L.C2[i] * W_kh_tau[i];
                else
                    Aij += L.C1[i] - L.C2[i] * W_kh_tau[i];
            }

        /* :311-448 consistency iterations */
        for (int i = 0; i < n; ++i) x_beta_old[i] = 0.0;
        unsigned count1 = 0;
        auto bpa_norm = [&]() {
            double mx = 0.0;
            for (int i : PA) mx = std::max(mx, std::fabs(b[i]));
            return mx;
        };
        while (bpa_norm() > tol1) {
            count1 = count1 + 1;
            if (count1 > (unsigned)opt.max_solver_iterations) break;
            for (int i = 0; i < n; ++i) x_beta[i] = 0.0;
            int rounds = 0;
            if (inactive_slip_removal(n, PA, b, A, x_beta_old, x_beta, &rounds, &maxcond)) status |= CP_QP_SINGULAR;
            rounds_total += rounds;
            nPA = (int)PA.size();
            del_FP = zero3();
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk) {
                        if ((tau_trial[i] - W_kh_tau[i]) > 0)
                            del_FP.a[j][kk] = del_FP.a[j][kk] + x_beta_old[i] * S[i].a[j][kk];
                        else
                            del_FP.a[j][kk] = del_FP.a[j][kk] - x_beta_old[i] * S[i].a[j][kk];
                    }
            FP_tau = mmult(matexp(del_FP, &e_terms), FP_t2);
            /* :361-396 */
            M3 tinv = inv3(FP_tau);
            FE_tau = mmult(F_tau, tinv);
            Ce_tau = Tmmult(FE_tau, FE_tau);
            M3 E2 = Ce_tau;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) E2.a[i][j] = 0.5 * (E2.a[i][j] - (i == j ? 1.0 : 0.0));
            T_star_tau = voigt_apply(Dmat, E2);
            M3 ct = mmult(Ce_tau, T_star_tau);
            for (int i = 0; i < n; ++i) {
                double r = 0.0;
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk) r += ct.a[j][kk] * S[i].a[j][kk];
                tau[i] = r;
                if (i > ns - 1) {
                    if ((tau_trial[i] - W_kh_tau[i]) < 0) tau[i] = W_kh_tau[i];
                }
            }
            /* :399-436 hardening, saturation caps, backstress */
            for (int i = 0; i < n; ++i) {
                double h1 = 0;
                for (int j = 0; j < n; ++j) h1 = h1 + h_ab[(size_t)i * NM + j] * x_beta[j];
                s_alpha_tau[i] = s_alpha_tau[i] + h1;
            }
            for (int i = 0; i < ns; ++i)
                if (s_alpha_tau[i] > L.ss[i]) s_alpha_tau[i] = L.ss[i];
            for (int i = 0; i < nw; ++i)
                if (s_alpha_tau[ns + i] > L.ss[ns + i]) s_alpha_tau[ns + i] = L.ss[ns + i];
            for (int i = 0; i < n; ++i) {
                if ((tau_trial[i] - W_kh_tau[i]) > 0)
                    W_kh_tau[i] = W_kh_tau[i] + (L.C1[i] - L.C2[i] * W_kh_tau[i]) * (x_beta[i]);
                else
                    W_kh_tau[i] = W_kh_tau[i] + (-L.C1[i] - L.C2[i] * W_kh_tau[i]) * (x_beta[i]);
            }
            for (int i = 0; i < n; ++i) b[i] = std::fabs(tau[i] - W_kh_tau[i]) - s_alpha_tau[i];
        }

        /* :450-456 twin and slip fractions (written only on this branch) */
        for (int i = 0; i < nw; ++i)
            st.twinfrac_iter[k * nw + i] = st.twinfrac_conv[k * nw + i] + x_beta_old[i + ns] / L.twin_shear;
        for (int i = 0; i < ns; ++i)
            st.slipfrac_iter[k * ns + i] = st.slipfrac_conv[k * ns + i] + x_beta_old[i];

        /* :458-468 stresses at the updated state */
        Fpn_inv = inv3(FP_tau);
        FE_tau = mmult(F_tau, Fpn_inv);
        det_FE_tau = det3(FE_tau);
        t = mmult(FE_tau, T_star_tau);
        t = scale3(1.0 / det_FE_tau, t);
        T_tau = mTmult(t, FE_tau);
        det_F_tau = det3(F_tau);
        Finv = inv3(F_tau);
        P_tau = mTmult(T_tau, Finv);
        P_tau = scale3(det_F_tau, P_tau);

        if (flag == 1) {
            /* :473-499 */
            std::memcpy(delFp_delF_prev, delFp_delF, sizeof delFp_delF);
            dels_delF_prev = dels_delF;
            double delFe_delF[9][9], delEtrial_delF[9][9], delT_delF[9][9], deltau_delF[9][9];
            const M3 temp1 = mmult(F_tau, Fpn_inv);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                for (int bb = 0; bb < 3; ++bb)
                                    v = v - temp1.a[i][a] * delFp_delF[3 * a + bb][3 * kk + l] * Fpn_inv.a[bb][j];
                            if (i == kk) v = v + Fpn_inv.a[l][j];
                            delFe_delF[3 * i + j][3 * kk + l] = v;
                        }
            /* :501-514 */
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                v = v + 0.5 * (delFe_delF[3 * a + i][3 * kk + l] * FE_tau.a[a][j] +
                                               delFe_delF[3 * a + j][3 * kk + l] * FE_tau.a[a][i]);
                            delEtrial_delF[3 * i + j][3 * kk + l] = v;
                        }
            /* :518-530 compute two matrix exponentials whose results are
             * overwritten before use (temp1 at :526, temp2 at :612): skipped. */
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < 9; ++kk) s += TM[i][kk] * delEtrial_delF[kk][j];
                    delT_delF[i][j] = s;
                }
            /* :533-545 */
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a)
                                v = v + 2 * delEtrial_delF[3 * i + a][3 * kk + l] * T_star_tau.a[a][j] +
                                    Ce_tau.a[i][a] * delT_delF[3 * a + j][3 * kk + l];
                            deltau_delF[3 * i + j][3 * kk + l] = v;
                        }
            /* :548-579 hardening sensitivity; dels_delF = inv(I - term_ds) dels_delF_prev */
            double delh[NM];
            for (int i = 0; i < ns; ++i)
                delh[i] = L.h0[i] * o_pow((1 - s_alpha_tau[i] / L.ss[i]), (L.a[i] - 1)) * (-1.0 / L.ss[i]);
            for (int i = 0; i < nw; ++i)
                delh[ns + i] = L.h0[ns + i] * o_pow((1 - s_alpha_tau[ns + i] / L.ss[ns + i]), (L.a[ns + i] - 1)) *
                               (-1.0 / L.ss[ns + i]);
            {
                std::vector<double> Im((size_t)n * n), Iinv((size_t)n * n);
                for (int kk = 0; kk < n; ++kk)
                    for (int l = 0; l < n; ++l)
                        Im[(size_t)kk * n + l] = (kk == l ? 1.0 : 0.0) - x_beta_old[l] * L.q[(size_t)kk * NM + l] * delh[l];
                invert_n(Im.data(), n, Iinv.data());
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < 9; ++j) {
                        double s = 0.0;
                        for (int kk = 0; kk < n; ++kk) s += Iinv[(size_t)i * n + kk] * dels_delF_prev[(size_t)kk * 9 + j];
                        dels_delF[(size_t)i * 9 + j] = s;
                    }
            }
            /* :581-604 delb_delF = +-(deltau_delF^T vec(S_PA(k))) */
            std::vector<double> delb((size_t)nPA * 9);
            for (int kk = 0; kk < nPA; ++kk) {
                double v1[9];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) v1[3 * i + j] = S[PA[kk]].a[i][j];
                for (int l = 0; l < 9; ++l) {
                    double s = 0.0;
                    for (int m = 0; m < 9; ++m) s += deltau_delF[m][l] * v1[m];
                    if ((tau_trial[PA[kk]] - W_kh_t[PA[kk]]) < 0) s = -1.0 * s;
                    delb[(size_t)kk * 9 + l] = s;
                }
            }
            /* :607-619 number of Gateaux-series terms */
            double tol2 = 1.0;
            unsigned count3 = 0;
            {
                M3 t1 = zero3(), t2b = eye3();
                while (tol2 > std::max(tol1 / 1e4, 1e-12)) {
                    count3 = count3 + 1;
                    t1 = mmult(del_FP, t2b);
                    t1 = scale3((1.0 / count3), t1);
                    tol2 = frob3(t1);
                    t2b = t1;
                    if (count3 > 200) {
                        status |= CP_QP_SERIES_CAP;
                        break;
                    }
                }
            }
            c_terms = (int)count3;
            /* :622-709 A2.  matrixExponential(-del_FP) at :682 is the same
             * value for every (i,j); it is evaluated once. */
            std::vector<double> A2((size_t)nPA * nPA);
            for (int i = 0; i < nPA; ++i)
                for (int j = 0; j < nPA; ++j) A2[(size_t)i * nPA + j] = h_ab[(size_t)PA[i] * NM + PA[j]];
            const M3 expm = matexp(scale3(-1.0, del_FP), nullptr);
            const M3 temp6 = mmult(CE_tau_trial, expm);
            for (int j = 0; j < nPA; ++j) {
                const M3 diff = gateaux_series(S[PA[j]], del_FP, (int)count3, true);
                for (int i = 0; i < nPA; ++i) {
                    M3 temp2 = Tmmult(diff, temp6);
                    symmetrize3(temp2);
                    M3 temp3 = voigt_apply(Dmat, temp2);
                    M3 tmp = mmult(Ce_tau, temp3);
                    temp3 = mmult(temp2, T_star_tau);
                    add3(tmp, 2.0, temp3);
                    double& a2 = A2[(size_t)i * nPA + j];
                    const bool ni = (tau_trial[PA[i]] - W_kh_t[PA[i]]) < 0.0;
                    const bool nj = (tau_trial[PA[j]] - W_kh_t[PA[j]]) < 0.0;
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            if (ni ^ nj)
                                a2 -= S[PA[i]].a[kk][l] * tmp.a[kk][l];
                            else
                                a2 += S[PA[i]].a[kk][l] * tmp.a[kk][l];
                        }
                    if (ni)
                        a2 -= L.C1[PA[i]] - L.C2[PA[i]] * W_kh_tau[PA[i]];
                    else
                        a2 += L.C1[PA[i]] - L.C2[PA[i]] * W_kh_tau[PA[i]];
                }
            }
            /* :712-729 delgamma_delF = inv(A2) (delb_delF - dels_delF[PA]) */
            std::vector<double> A2inv((size_t)nPA * nPA), dg((size_t)nPA * 9);
            if (invert_n(A2.data(), nPA, A2inv.data())) status |= CP_QP_SINGULAR;
            for (int i = 0; i < nPA; ++i)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < nPA; ++kk)
                        s += A2inv[(size_t)i * nPA + kk] * (delb[(size_t)kk * 9 + j] - dels_delF[(size_t)PA[kk] * 9 + j]);
                    dg[(size_t)i * 9 + j] = s;
                }
            /* :734-796 S_PA (9 x nPA) */
            std::vector<double> S_PA((size_t)9 * nPA);
            for (int j = 0; j < nPA; ++j) {
                const M3 diff = gateaux_series(S[PA[j]], del_FP, (int)count3, false);
                const M3 t1 = mmult(diff, FP_t2);
                const bool nj = (tau_trial[PA[j]] - W_kh_t[PA[j]]) < 0;
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) S_PA[(size_t)(3 * kk + l) * nPA + j] = nj ? -t1.a[kk][l] : t1.a[kk][l];
            }
            /* :799-821 delFp_delF = exp(del_FP) delFp_delF_prev + S_PA delgamma */
            const M3 expp = matexp(del_FP, nullptr);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l) {
                            double v = 0.0;
                            for (int a = 0; a < 3; ++a) v = v + expp.a[i][a] * delFp_delF_prev[3 * a + j][3 * kk + l];
                            delFp_delF[3 * i + j][3 * kk + l] = v;
                        }
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j) {
                    double s = 0.0;
                    for (int kk = 0; kk < nPA; ++kk) s += S_PA[(size_t)i * nPA + kk] * dg[(size_t)kk * 9 + j];
                    delFp_delF[i][j] += 1.0 * s;
                }
            /* :823-827 (dead: dels_delF_prev is reassigned at :477 before use) */
        }
        iter1 = iter1 + 1;
    }

    /* :835-940 final tangent */
    if (flag == 1) {
        double delFe_delF[9][9], delTstar[9][9], PK[9][9];
        const M3 temp1 = mmult(F_tau, Fpn_inv);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                v = v - temp1.a[i][a] * delFp_delF[3 * a + bb][3 * kk + l] * Fpn_inv.a[bb][j];
                        if (i == kk) v = v + Fpn_inv.a[l][j];
                        delFe_delF[3 * i + j][3 * kk + l] = v;
                    }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                for (int c = 0; c < 3; ++c)
                                    v = v + TM[3 * i + j][3 * a + bb] * delFe_delF[3 * c + a][3 * kk + l] * FE_tau.a[c][bb];
                        delTstar[3 * i + j][3 * kk + l] = v;
                    }
        const M3 temp4 = inv3(F_tau);
        const M3 tmp = mmult(temp4, FE_tau);
        const M3 t1 = mTmult(T_star_tau, tmp);
        const M3 t2 = mmult(temp4, FE_tau);
        const M3 t3 = mmult(FE_tau, T_star_tau);
        const M3 t5 = mTmult(t3, F_tau);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int kk = 0; kk < 3; ++kk)
                    for (int l = 0; l < 3; ++l) {
                        double v = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            for (int bb = 0; bb < 3; ++bb)
                                v = v + (i == a ? 1.0 : 0.0) * delFe_delF[3 * a + bb][3 * kk + l] * t1.a[bb][j] +
                                    FE_tau.a[i][a] * delTstar[3 * a + bb][3 * kk + l] * t2.a[j][bb] -
                                    t3.a[i][a] * delFe_delF[3 * a + bb][3 * kk + l] * temp4.a[j][bb];
                            v = v - t5.a[i][a] * temp4.a[j][kk] * temp4.a[l][a];
                        }
                        PK[3 * i + j][3 * kk + l] = v;
                    }
        /* :916-939 the "rotation back" uses L = I, i.e. a copy */
        if (io.dPdF)
            for (int i = 0; i < 9; ++i)
                for (int j = 0; j < 9; ++j) io.dPdF[9 * i + j] = PK[i][j];
    }

    /* :942-959 outputs and history */
    if (io.P) store3(P_tau, io.P);
    if (io.T) store3(T_tau, io.T);
    store3(FE_tau, st.Fe_iter + 9 * k);
    store3(FP_tau, st.Fp_iter + 9 * k);
    for (int i = 0; i < n; ++i) {
        st.s_iter[k * n + i] = s_alpha_tau[i];
        st.W_iter[k * n + i] = W_kh_tau[i];
    }

    /* :962-1019 twin reorientation */
    if (L.twinning) {
        double F_T;
        if (!opt.enable_multiphase) {
            if (F_r > 0)
                F_T = L.twin_thr + (L.twin_sat * F_e / F_r);
            else
                F_T = L.twin_thr;
        } else {
            F_T = L.twin_thr;
        }
        if (F_T > 1.0) F_T = 1.0;
        int twin_pos = 0;
        double twin_max = st.twinfrac_iter[k * nw];
        for (int i = 1; i < nw; ++i)
            if (st.twinfrac_iter[k * nw + i] > twin_max) {
                twin_max = st.twinfrac_iter[k * nw + i];
                twin_pos = i;
            }
        if (st.twin_conv[k] != 1) {
            if (F_r > 0) {
                if (twin_max > F_T) {
                    double rod[3] = {st.rot_conv[3 * k], st.rot_conv[3 * k + 1], st.rot_conv[3 * k + 2]};
                    double quat2[4], quat1[4], quatprod[4];
                    rod2quat(quat2, rod);
                    quat1[0] = 0;
                    quat1[1] = L.nn[ns + twin_pos][0];
                    quat1[2] = L.nn[ns + twin_pos][1];
                    quat1[3] = L.nn[ns + twin_pos][2];
                    quatproduct(quatprod, quat2, quat1);
                    quat2rod(quatprod, rod);
                    for (int i = 0; i < 3; ++i) {
                        st.rot_iter[3 * k + i] = rod[i];
                        st.rotnew_iter[3 * k + i] = rod[i];
                    }
                    st.twin_iter[k] = 1;
                    for (int i = 0; i < nw; ++i) st.s_iter[k * n + ns + i] = 100000;
                }
            }
        }
    }

    bool finite = true;
    if (io.P)
        for (int i = 0; i < 9; ++i) finite &= std::isfinite(io.P[i]);
    if (flag == 1 && io.dPdF)
        for (int i = 0; i < 81; ++i) finite &= std::isfinite(io.dPdF[i]);
    if (!finite) status |= CP_QP_NONFINITE;
    if (maxcond > 1e12) status |= CP_QP_ILL_CONDITIONED;
    if (io.stats) {
        io.stats[0] = p0 < 0 ? 0 : p0;
        io.stats[1] = nPA;
        io.stats[2] = rounds_total;
        io.stats[3] = e_terms;
        io.stats[4] = c_terms;
        io.stats[5] = (int)iter1;
        io.stats[6] = 0;
        io.stats[7] = std::isfinite(maxcond) ? std::min(99, (int)std::ceil(std::log10(maxcond))) : 99;
    }
    if (io.status) *io.status = status;
    return status;
}

int set_threads(int32_t nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    return omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

} /* namespace */

extern "C" {

int oracle_update(const cp_material_t* mat, const cp_options_t* opt, const or_state* st,
                  const double* F, int32_t flag, double F_e, double F_r, double* P, double* T,
                  double* dPdF, int32_t* stats, int32_t* status, int32_t nthreads) {
    if (!mat || !opt || !st || !F) return CP_E_ARG;
    const Lattice L = make_lattice(mat);
    if (L.n <= 0 || L.n > NM) return CP_E_ARG;
    set_threads(nthreads);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (int64_t k = 0; k < st->n_qp; ++k) {
        QpIO io;
        io.F = F + 9 * k;
        io.P = P ? P + 9 * k : nullptr;
        io.T = T ? T + 9 * k : nullptr;
        io.dPdF = (dPdF && flag == 1) ? dPdF + 81 * k : nullptr;
        io.stats = stats ? stats + 8 * k : nullptr;
        io.status = status ? status + k : nullptr;
        bad |= calculate_plasticity(L, *opt, *st, k, io, flag, F_e, F_r);
    }
    return bad & (CP_QP_NONFINITE | CP_QP_SINGULAR) ? 1 : 0;
}

int oracle_assemble(const cp_material_t* mat, const cp_options_t* opt, const or_state* st,
                    int64_t n_cells, const double* U, const double* gradN, const double* JxW,
                    int32_t uniform, double F_e, double F_r, double* Ke, double* Re, int32_t* stats,
                    int32_t* status, int32_t nthreads) {
    if (!mat || !opt || !st || !U || !gradN || !JxW || !Ke || !Re) return CP_E_ARG;
    if (st->n_qp != 8 * n_cells) return CP_E_ARG;
    const Lattice L = make_lattice(mat);
    set_threads(nthreads);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(| : bad)
    for (int64_t c = 0; c < n_cells; ++c) {
        const double* g = uniform ? gradN : gradN + (size_t)c * 8 * 8 * 3;
        const double* w = uniform ? JxW : JxW + (size_t)c * 8;
        const double* Ul = U + 24 * c;
        double* K = Ke + 576 * c;
        double* R = Re + 24 * c;
        for (int i = 0; i < 576; ++i) K[i] = 0.0;
        for (int i = 0; i < 24; ++i) R[i] = 0.0;
        /* getElementalValues.cc:127-163 */
        for (int q = 0; q < 8; ++q) {
            double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, P[9], dPdF[81];
            for (int d = 0; d < 24; ++d) {
                const int i = d % 3;
                const double* gd = g + (q * 8 + d / 3) * 3;
                for (int j = 0; j < 3; ++j) F[3 * i + j] += Ul[d] * gd[j];
            }
            for (int i = 0; i < 3; ++i) F[4 * i] += 1;
            const int64_t k = 8 * c + q;
            QpIO io{F, P, nullptr, dPdF, stats ? stats + 8 * k : nullptr, status ? status + k : nullptr};
            bad |= calculate_plasticity(L, *opt, *st, k, io, 1, F_e, F_r);
            for (int d = 0; d < 24; ++d) {
                const int i = d % 3;
                const double* gd = g + (q * 8 + d / 3) * 3;
                for (int j = 0; j < 3; ++j) R[d] -= gd[j] * P[3 * i + j] * w[q];
            }
            for (int d1 = 0; d1 < 24; ++d1) {
                const int i = d1 % 3;
                const double* g1 = g + (q * 8 + d1 / 3) * 3;
                for (int d2 = 0; d2 < 24; ++d2) {
                    const int j = d2 % 3;
                    const double* g2 = g + (q * 8 + d2 / 3) * 3;
                    for (int kk = 0; kk < 3; ++kk)
                        for (int l = 0; l < 3; ++l)
                            K[24 * d1 + d2] += g1[kk] * dPdF[27 * i + 9 * kk + 3 * j + l] * g2[l] * w[q];
                }
            }
        }
    }
    return bad & (CP_QP_NONFINITE | CP_QP_SINGULAR) ? 1 : 0;
}

int oracle_reorient(const or_state* st, int32_t nthreads) {
    if (!st) return CP_E_ARG;
    set_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < st->n_qp; ++k) {
        /* updateAfterIncrement.cc:287 rotnew_conv = rotnew_iter */
        for (int i = 0; i < 3; ++i) st->rotnew_conv[3 * k + i] = st->rotnew_iter[3 * k + i];
        /* reorient.cc:24-93 */
        M3 Fe_old = load3(st->Fe_conv + 9 * k), Fe_new = load3(st->Fe_iter + 9 * k);
        if (st->twin_conv[k] != st->twin_iter[k]) Fe_old = Fe_new;
        M3 R_pair[2];
        for (int w = 0; w < 2; ++w) {
            const M3& Fe = w == 0 ? Fe_old : Fe_new;
            const M3 C = Tmmult(Fe, Fe);
            double ev[3];
            M3 V;
            eig_sym3(C, ev, V);
            M3 Lam = eye3();
            for (int i = 0; i < 3; ++i) Lam.a[i][i] = std::sqrt(ev[i]);
            M3 U = mmult(V, Lam);
            U = mTmult(U, V);
            const M3 Rinv = inv3(U);
            R_pair[w] = mmult(Fe, Rinv);
        }
        M3 Om = R_pair[1];
        add3(Om, -1.0, R_pair[0]);
        Om = mTmult(Om, R_pair[1]);
        const double* rold = st->rotnew_conv + 3 * k;
        double ov[3];
        ov[0] = -0.5 * (Om.a[1][2] - Om.a[2][1]);
        ov[1] = 0.5 * (Om.a[0][2] - Om.a[2][0]);
        ov[2] = -0.5 * (Om.a[0][1] - Om.a[1][0]);
        const double dot = ov[0] * rold[0] + ov[1] * rold[1] + ov[2] * rold[2];
        double dt[3], cr[3], dr[3], rn[3];
        for (int i = 0; i < 3; ++i) dt[i] = dot * rold[i];
        cr[0] = ov[1] * rold[2] - ov[2] * rold[1];
        cr[1] = ov[2] * rold[0] - ov[0] * rold[2];
        cr[2] = ov[0] * rold[1] - ov[1] * rold[0];
        for (int i = 0; i < 3; ++i) {
            dr[i] = 0.0;
            dr[i] += ov[i];
            dr[i] += dt[i];
            dr[i] += cr[i];
            dr[i] = 0.5 * dr[i];
            rn[i] = 0.0;
            rn[i] += rold[i];
            rn[i] += dr[i];
        }
        const double mx = 10000;
        const double nrm = std::sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
        if (nrm > mx)
            for (int i = 0; i < 3; ++i) rn[i] = rn[i] * mx / nrm;
        for (int i = 0; i < 3; ++i) st->rotnew_conv[3 * k + i] = rn[i];
        /* updateAfterIncrement.cc:295 rotnew_iter = rotnew_conv */
        for (int i = 0; i < 3; ++i) st->rotnew_iter[3 * k + i] = rn[i];
    }
    return 0;
}

void oracle_odfpoint(const double r[3], double R[9]) { store3(odfpoint(r), R); }

void oracle_elasticmoduli(const double R[9], const double C[36], double out[36]) {
    double Cm[6][6], Ar[6][6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Cm[i][j] = C[6 * i + j];
    elasticmoduli(load3(R), Cm, Ar);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) out[6 * i + j] = Ar[i][j];
}

int oracle_matrix_exponential(const double A[9], double out[9]) {
    int terms = 0;
    store3(matexp(load3(A), &terms), out);
    return terms;
}

int oracle_pinv_svd(const double* A, int n, double* Ainv) { return pinv_svd(A, n, Ainv, nullptr); }

int oracle_invert(const double* A, int n, double* Ainv) { return invert_n(A, n, Ainv); }

double oracle_parity_pow(double x, double y) { return parity_pow(x, y); }

void oracle_eig_sym3(const double C[9], double evals[3], double evecs[9]) {
    M3 V;
    eig_sym3(load3(C), evals, V);
    store3(V, evecs);
}

} /* extern "C" */
