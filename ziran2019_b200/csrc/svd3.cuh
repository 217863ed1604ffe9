// Batched 3x3 SVD in registers: implicit-shift QR on the bidiagonal form with a
// Wilkinson shift (Gast, Fu, Jiang, Teran 2016, "Implicit-shifted Symmetric QR
// Singular Value Decomposition of 3x3 Matrices"), the algorithm of
// Lib/Ziran/Math/Linear/ImplicitQRSVD.h:219-532 and Givens.h:33-270.
//
// Output convention of the reference: F = U diag(sigma) V^T with U, V proper
// rotations, |sigma0| >= |sigma1| >= |sigma2|, only sigma2 may be negative.
// All Givens rows are compile-time constants so every matrix stays in
// registers.  The QR sweep is capped (the reference loop is not); the cap is
// never reached for finite input in the tests.
#pragma once
#include "mat3.cuh"

namespace zmpm {

// 1 / sqrt(x) for x > 0, the normalisation of every rotation.  The reference
// divides by sqrt(x); the reciprocal square root is one instruction sequence
// instead of two.  FP32: rsqrtf (up to 2 ulp) refined by one Newton-Raphson
// step y <- y (1 + (1 - x y^2) / 2), which keeps the rotations orthogonal to
// FP32 round-off; FP64: rsqrt (1 ulp).
ZMPM_HD float rsq(float x)
{
#ifdef __CUDA_ARCH__
    const float y = rsqrtf(x);
    const float e = fmaf(-x * y, y, 1.0f);
    return fmaf(0.5f * y, e, y);
#else
    return 1.0f / std::sqrt(x);
#endif
}
ZMPM_HD double rsq(double x)
{
#ifdef __CUDA_ARCH__
    return rsqrt(x);
#else
    return 1.0 / std::sqrt(x);
#endif
}

template <class T>
ZMPM_HD void giv(T a, T b, T& c, T& s) // ( c -s ; s c ) (a b)^T = (* 0)^T
{
    T d = a * a + b * b;
    c = T(1);
    s = T(0);
    if (d != T(0)) {
        T t = rsq(d);
        c = a * t;
        s = -b * t;
    }
}
template <class T>
ZMPM_HD void giv_unconv(T a, T b, T& c, T& s) // ( c -s ; s c ) (a b)^T = (0 *)^T
{
    T d = a * a + b * b;
    c = T(0);
    s = T(1);
    if (d != T(0)) {
        T t = rsq(d);
        s = a * t;
        c = b * t;
    }
}
template <int I, int K, class T>
ZMPM_HD void rot_rows(M3<T>& A, T c, T s)
{
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        T t1 = A(I, j), t2 = A(K, j);
        A(I, j) = c * t1 - s * t2;
        A(K, j) = s * t1 + c * t2;
    }
}
template <int I, int K, class T>
ZMPM_HD void rot_cols(M3<T>& A, T c, T s)
{
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        T t1 = A(j, I), t2 = A(j, K);
        A(j, I) = c * t1 - s * t2;
        A(j, K) = s * t1 + c * t2;
    }
}

template <class T>
ZMPM_HD void svd_zero_chase(M3<T>& H, M3<T>& U, M3<T>& V)
{
    T c1, s1, c2, s2, c3, s3;
    giv(H(0, 0), H(1, 0), c1, s1);
    if (H(1, 0) != T(0))
        giv(H(0, 0) * H(0, 1) + H(1, 0) * H(1, 1), H(0, 0) * H(0, 2) + H(1, 0) * H(1, 2), c2, s2);
    else
        giv(H(0, 1), H(0, 2), c2, s2);
    rot_rows<0, 1>(H, c1, s1);
    rot_cols<1, 2>(H, c2, s2);
    rot_cols<1, 2>(V, c2, s2);
    giv(H(1, 1), H(2, 1), c3, s3);
    rot_rows<1, 2>(H, c3, s3);
    rot_cols<0, 1>(U, c1, s1);
    rot_cols<1, 2>(U, c3, s3);
}

// 2x2 SVD of [[a00 a01][a10 a11]] as Givens pairs (ImplicitQRSVD.h:95-160)
template <class T>
ZMPM_HD void svd2_givens(T a00, T a01, T a10, T a11, T& uc, T& us, T& s0, T& s1, T& vc, T& vs)
{
    T x0 = a00 + a11, x1 = a10 - a01;
    T den2 = x0 * x0 + x1 * x1;
    uc = T(1);
    us = T(0);
    if (den2 != T(0)) {
        T t = rsq(den2);
        uc = x0 * t;
        us = -x1 * t;
    }
    T x = uc * a00 - us * a10, y = uc * a01 - us * a11, z = us * a01 + uc * a11;
    T cosine, sine;
    T y2 = y * y;
    if (y2 == T(0)) {
        cosine = T(1);
        sine = T(0);
        s0 = x;
        s1 = z;
    }
    else {
        T tau = T(0.5) * (x - z);
        T w = sqrt(tau * tau + y2);
        T t = (tau > T(0)) ? y / (tau + w) : y / (tau - w);
        cosine = rsq(t * t + T(1));
        sine = -t * cosine;
        T c2 = cosine * cosine, csy = T(2) * cosine * sine * y, s2 = sine * sine;
        s0 = c2 * x - csy + s2 * z;
        s1 = s2 * x + csy + c2 * z;
    }
    if (s0 < s1) {
        T tmp = s0;
        s0 = s1;
        s1 = tmp;
        vc = -sine;
        vs = cosine;
    }
    else {
        vc = cosine;
        vs = sine;
    }
    T nc = uc * vc - us * vs;
    T ns = us * vc + uc * vs;
    uc = nc;
    us = ns;
}

template <int TT, class T>
ZMPM_HD void svd_process(M3<T>& B, M3<T>& U, T sig[3], M3<T>& V)
{
    constexpr int other = (TT == 1) ? 0 : 2;
    sig[other] = B(other, other);
    T uc, us, vc, vs, s0, s1;
    svd2_givens(B(TT, TT), B(TT, TT + 1), B(TT + 1, TT), B(TT + 1, TT + 1), uc, us, s0, s1, vc, vs);
    sig[TT] = s0;
    sig[TT + 1] = s1;
    rot_cols<TT, TT + 1>(U, uc, us);
    rot_cols<TT, TT + 1>(V, vc, vs);
}

template <int I, class T>
ZMPM_HD void neg_col(M3<T>& A)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) A(r, I) = -A(r, I);
}
template <int I, int J, class T>
ZMPM_HD void swap_col(M3<T>& A)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        T t = A(r, I);
        A(r, I) = A(r, J);
        A(r, J) = t;
    }
}
template <class T>
ZMPM_HD void swap_s(T& a, T& b)
{
    T t = a;
    a = b;
    b = t;
}

template <class T>
ZMPM_HD void svd_sort0(M3<T>& U, T sig[3], M3<T>& V)
{
    if (fabs(sig[1]) >= fabs(sig[2])) {
        if (sig[1] < T(0)) {
            sig[1] = -sig[1];
            neg_col<1>(U);
            sig[2] = -sig[2];
            neg_col<2>(U);
        }
        return;
    }
    if (sig[2] < T(0)) {
        sig[1] = -sig[1];
        neg_col<1>(U);
        sig[2] = -sig[2];
        neg_col<2>(U);
    }
    swap_s(sig[1], sig[2]);
    swap_col<1, 2>(U);
    swap_col<1, 2>(V);
    if (sig[1] > sig[0]) {
        swap_s(sig[0], sig[1]);
        swap_col<0, 1>(U);
        swap_col<0, 1>(V);
    }
    else {
        neg_col<2>(U);
        neg_col<2>(V);
    }
}

template <class T>
ZMPM_HD void svd_sort1(M3<T>& U, T sig[3], M3<T>& V)
{
    if (fabs(sig[0]) >= sig[1]) {
        if (sig[0] < T(0)) {
            sig[0] = -sig[0];
            neg_col<0>(U);
            sig[2] = -sig[2];
            neg_col<2>(U);
        }
        return;
    }
    swap_s(sig[0], sig[1]);
    swap_col<0, 1>(U);
    swap_col<0, 1>(V);
    if (fabs(sig[1]) < fabs(sig[2])) {
        swap_s(sig[1], sig[2]);
        swap_col<1, 2>(U);
        swap_col<1, 2>(V);
    }
    else {
        neg_col<1>(U);
        neg_col<1>(V);
    }
    if (sig[1] < T(0)) {
        sig[1] = -sig[1];
        neg_col<1>(U);
        sig[2] = -sig[2];
        neg_col<2>(U);
    }
}

template <class T>
struct SvdTol;
template <>
struct SvdTol<double> {
    static constexpr double value = 1024 * 2.220446049250313080847e-16;
};
template <>
struct SvdTol<float> {
    static constexpr float value = 128 * 1.1920928955078125e-07f;
};

template <class T>
ZMPM_HD int svd3(const M3<T>& A, M3<T>& U, T sig[3], M3<T>& V)
{
    M3<T> B = A;
    U = m3_identity<T>();
    V = m3_identity<T>();
    {
        T c, s;
        giv(B(1, 0), B(2, 0), c, s);
        rot_rows<1, 2>(B, c, s);
        rot_cols<1, 2>(U, c, s);
        svd_zero_chase(B, U, V);
    }
    T a1 = B(0, 0), b1 = B(0, 1), a2 = B(1, 1), a3 = B(2, 2), b2 = B(1, 2);
    T g1 = a1 * b1, g2 = a2 * b2;
    T tol = SvdTol<T>::value;
    T scale = T(0.5) * sqrt(a1 * a1 + a2 * a2 + a3 * a3 + b1 * b1 + b2 * b2);
    tol *= (scale > T(1) ? scale : T(1));
    int count = 0;
    while (fabs(b2) > tol && fabs(b1) > tol && fabs(a1) > tol && fabs(a2) > tol && fabs(a3) > tol && count < 100) {
        // Wilkinson shift of the trailing 2x2 of B^T B
        T ta1 = a2 * a2 + b1 * b1, tb1 = g2, ta2 = a3 * a3 + b2 * b2;
        T d = T(0.5) * (ta1 - ta2);
        T bs = tb1 * tb1;
        T mu = ta2 - copysign(bs / (fabs(d) + sqrt(d * d + bs)), d);
        T c, s;
        giv(a1 * a1 - mu, g1, c, s);
        rot_cols<0, 1>(B, c, s);
        rot_cols<0, 1>(V, c, s);
        svd_zero_chase(B, U, V);
        a1 = B(0, 0);
        b1 = B(0, 1);
        a2 = B(1, 1);
        a3 = B(2, 2);
        b2 = B(1, 2);
        g1 = a1 * b1;
        g2 = a2 * b2;
        ++count;
    }
    if (fabs(b2) <= tol) {
        svd_process<0>(B, U, sig, V);
        svd_sort0(U, sig, V);
    }
    else if (fabs(b1) <= tol) {
        svd_process<1>(B, U, sig, V);
        svd_sort1(U, sig, V);
    }
    else if (fabs(a2) <= tol) {
        T c, s;
        giv_unconv(B(1, 2), B(2, 2), c, s);
        rot_rows<1, 2>(B, c, s);
        rot_cols<1, 2>(U, c, s);
        svd_process<0>(B, U, sig, V);
        svd_sort0(U, sig, V);
    }
    else if (fabs(a3) <= tol) {
        T c, s;
        giv(B(1, 1), B(1, 2), c, s);
        rot_cols<1, 2>(B, c, s);
        rot_cols<1, 2>(V, c, s);
        giv(B(0, 0), B(0, 2), c, s);
        rot_cols<0, 2>(B, c, s);
        rot_cols<0, 2>(V, c, s);
        svd_process<0>(B, U, sig, V);
        svd_sort0(U, sig, V);
    }
    else {
        T c, s;
        giv_unconv(B(0, 1), B(1, 1), c, s);
        rot_rows<0, 1>(B, c, s);
        rot_cols<0, 1>(U, c, s);
        giv_unconv(B(0, 2), B(2, 2), c, s);
        rot_rows<0, 2>(B, c, s);
        rot_cols<0, 2>(U, c, s);
        svd_process<1>(B, U, sig, V);
        svd_sort1(U, sig, V);
    }
    return count;
}

} // namespace zmpm
