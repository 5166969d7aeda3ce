// cp_math.cuh -- FP64 3x3 / Voigt helpers for the qp kernels (device + host).
//
// Semantics follow the reference's deal.II FullMatrix calls:
//   A.mmult(C,B)  C = A B        A.Tmmult(C,B)  C = A^T B
//   A.mTmult(C,B) C = A B^T      symmetrize     (A + A^T)/2
// and vecform/matform of matrixOperations.cc:133-163 (Voigt 11,22,33,23,13,12).
#pragma once

#ifdef __CUDACC__
#include <cuda_runtime.h>
#define CP_HD __host__ __device__ __forceinline__
#else
// host-only compilation of the kernel sources (tests build them with g++ to
// check the device code path against the oracle without a GPU)
#include <cmath>
#define __host__
#define __device__
#define __forceinline__ inline
#define __restrict__
#define CP_HD inline
using std::fabs;
using std::fmax;
using std::fmin;
using std::ceil;
using std::log10;
using std::isfinite;
using std::pow;
using std::sqrt;
using std::cos;
using std::atan;
#endif

namespace cp {

// Every multiply-add of the helpers below is an explicit fused multiply-add
// in a fixed order: left to the compiler, a product shared by two
// expressions (det and inv of one matrix, say) is fused in one kernel and not
// in another, so the same source would round differently in the plain, sorted
// and quad forms of the update.  Written out, each helper gives the same bits
// wherever it is inlined.
CP_HD double fmad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
// a0 b0 + a1 b1 + a2 b2 as fma(a2, b2, fma(a1, b1, a0 b0))
CP_HD double dot3(double a0, double b0, double a1, double b1, double a2, double b2) {
    return fmad(a2, b2, fmad(a1, b1, a0 * b0));
}

struct M3 {
    double a[9];
    CP_HD double& operator()(int i, int j) { return a[3 * i + j]; }
    CP_HD double operator()(int i, int j) const { return a[3 * i + j]; }
};

CP_HD M3 zero3() {
    M3 m;
#pragma unroll
    for (int i = 0; i < 9; ++i) m.a[i] = 0.0;
    return m;
}
CP_HD M3 eye3() {
    M3 m = zero3();
    m.a[0] = m.a[4] = m.a[8] = 1.0;
    return m;
}
CP_HD M3 mul(const M3& A, const M3& B) {
    M3 C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = dot3(A(i, 0), B(0, j), A(i, 1), B(1, j), A(i, 2), B(2, j));
    return C;
}
CP_HD M3 mulTN(const M3& A, const M3& B) {  // A^T B
    M3 C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = dot3(A(0, i), B(0, j), A(1, i), B(1, j), A(2, i), B(2, j));
    return C;
}
CP_HD M3 mulNT(const M3& A, const M3& B) {  // A B^T
    M3 C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = dot3(A(i, 0), B(j, 0), A(i, 1), B(j, 1), A(i, 2), B(j, 2));
    return C;
}
CP_HD M3 scale(double c, const M3& A) {
    M3 C;
#pragma unroll
    for (int i = 0; i < 9; ++i) C.a[i] = c * A.a[i];
    return C;
}
CP_HD void axpy(M3& Y, double c, const M3& X) {
#pragma unroll
    for (int i = 0; i < 9; ++i) Y.a[i] = fmad(c, X.a[i], Y.a[i]);
}
CP_HD M3 sym(const M3& A) {
    M3 S = A;
    S(0, 1) = S(1, 0) = (A(0, 1) + A(1, 0)) / 2;
    S(0, 2) = S(2, 0) = (A(0, 2) + A(2, 0)) / 2;
    S(1, 2) = S(2, 1) = (A(1, 2) + A(2, 1)) / 2;
    return S;
}
CP_HD double frob(const M3& A) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) s = fmad(A.a[i], A.a[i], s);
    return sqrt(s);
}
CP_HD double dot9(const M3& A, const M3& B) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) s = fmad(A.a[i], B.a[i], s);
    return s;
}
// a b - c d as fma(a, b, -(c d))
CP_HD double diff2(double a, double b, double c, double d) { return fmad(a, b, -(c * d)); }
CP_HD double det(const M3& A) {
    const double m0 = diff2(A(1, 1), A(2, 2), A(1, 2), A(2, 1));
    const double m1 = diff2(A(1, 0), A(2, 2), A(1, 2), A(2, 0));
    const double m2 = diff2(A(1, 0), A(2, 1), A(1, 1), A(2, 0));
    return fmad(A(0, 2), m2, fmad(-A(0, 1), m1, A(0, 0) * m0));
}
// inverse by the adjugate, inv = adj(A) * (1/det)
CP_HD M3 inv(const M3& A) {
    const double c00 = diff2(A(1, 1), A(2, 2), A(1, 2), A(2, 1));
    const double c01 = diff2(A(1, 2), A(2, 0), A(1, 0), A(2, 2));
    const double c02 = diff2(A(1, 0), A(2, 1), A(1, 1), A(2, 0));
    const double d = dot3(A(0, 0), c00, A(0, 1), c01, A(0, 2), c02);
    const double r = 1.0 / d;
    M3 B;
    B(0, 0) = c00 * r;
    B(1, 0) = c01 * r;
    B(2, 0) = c02 * r;
    B(0, 1) = diff2(A(0, 2), A(2, 1), A(0, 1), A(2, 2)) * r;
    B(1, 1) = diff2(A(0, 0), A(2, 2), A(0, 2), A(2, 0)) * r;
    B(2, 1) = diff2(A(0, 1), A(2, 0), A(0, 0), A(2, 1)) * r;
    B(0, 2) = diff2(A(0, 1), A(1, 2), A(0, 2), A(1, 1)) * r;
    B(1, 2) = diff2(A(0, 2), A(1, 0), A(0, 0), A(1, 2)) * r;
    B(2, 2) = diff2(A(0, 0), A(1, 1), A(0, 1), A(1, 0)) * r;
    return B;
}

// Symmetric 6x6 stiffness stored as its 21-entry upper triangle, row by row.
struct Sym6 {
    double c[21];
    CP_HD double operator()(int i, int j) const {
        if (i > j) {
            const int t = i;
            i = j;
            j = t;
        }
        return c[i * 6 - i * (i - 1) / 2 + (j - i)];
    }
};

// The same 21 entries held elsewhere (e.g. a per-thread slot in shared
// memory, entry e at p[e * stride]).
struct Sym6Ref {
    const double* p;
    int stride;
    CP_HD double operator()(int i, int j) const {
        if (i > j) {
            const int t = i;
            i = j;
            j = t;
        }
        return p[(i * 6 - i * (i - 1) / 2 + (j - i)) * stride];
    }
};

// matform(D * vecform_eng(X)): stress from a symmetric strain-like tensor,
// with the engineering-shear doubling of the reference's Dmat
// (calculatePlasticity.cc:64-68) applied to the shear inputs.
template <class SymD>
CP_HD M3 voigt_apply(const SymD& D, const M3& X) {
    const double v0 = X(0, 0), v1 = X(1, 1), v2 = X(2, 2);
    const double v3 = 2.0 * X(1, 2), v4 = 2.0 * X(0, 2), v5 = 2.0 * X(0, 1);
    double w[6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
        w[i] = fmad(D(i, 5), v5, fmad(D(i, 4), v4, fmad(D(i, 3), v3, fmad(D(i, 2), v2, fmad(D(i, 1), v1, D(i, 0) * v0)))));
    M3 A;
    A(0, 0) = w[0];
    A(1, 1) = w[1];
    A(2, 2) = w[2];
    A(1, 2) = A(2, 1) = w[3];
    A(0, 2) = A(2, 0) = w[4];
    A(0, 1) = A(1, 0) = w[5];
    return A;
}

// odfpoint (rotationOperations.cc:4-51)
CP_HD M3 odfpoint(double r0, double r1, double r2) {
    const double rr = dot3(r0, r0, r1, r1, r2, r2);
    const double t1 = 1.0 - rr, inv2 = 1.0 / (1.0 + rr);
    const double r[3] = {r0, r1, r2};
    M3 R;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) R(i, j) = fmad(2.0, r[i] * r[j], i == j ? t1 : 0.0);
    R(0, 1) = fmad(-2.0, r2, R(0, 1));
    R(0, 2) = fmad(2.0, r1, R(0, 2));
    R(1, 2) = fmad(-2.0, r0, R(1, 2));
    R(1, 0) = fmad(2.0, r2, R(1, 0));
    R(2, 0) = fmad(-2.0, r1, R(2, 0));
    R(2, 1) = fmad(2.0, r0, R(2, 1));
#pragma unroll
    for (int i = 0; i < 9; ++i) R.a[i] = R.a[i] * inv2;
    return R;
}

// elasticmoduli (matrixOperations.cc:189-234): N(R) C N(R)^T, C symmetric.
CP_HD Sym6 elasticmoduli(const M3& R, const double* __restrict__ C) {
    double N[6][6];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        N[i][0] = R(i, 0) * R(i, 0);
        N[i][1] = R(i, 1) * R(i, 1);
        N[i][2] = R(i, 2) * R(i, 2);
        N[i][3] = 2.0 * R(i, 1) * R(i, 2);
        N[i][4] = 2.0 * R(i, 2) * R(i, 0);
        N[i][5] = 2.0 * R(i, 0) * R(i, 1);
    }
    const int P[3] = {1, 2, 0}, Q[3] = {2, 0, 1};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int p = P[r], q = Q[r];
        N[3 + r][0] = R(p, 0) * R(q, 0);
        N[3 + r][1] = R(p, 1) * R(q, 1);
        N[3 + r][2] = R(p, 2) * R(q, 2);
        N[3 + r][3] = fmad(R(p, 2), R(q, 1), R(p, 1) * R(q, 2));
        N[3 + r][4] = fmad(R(p, 0), R(q, 2), R(p, 2) * R(q, 0));
        N[3 + r][5] = fmad(R(p, 1), R(q, 0), R(p, 0) * R(q, 1));
    }
    double T[6][6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) s = fmad(N[i][k], C[6 * k + j], s);
            T[i][j] = s;
        }
    Sym6 out;
    int idx = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 6; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) s = fmad(T[i][k], N[j][k], s);
            out.c[idx++] = s;
        }
    return out;
}

}  // namespace cp
