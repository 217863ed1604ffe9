// TEST INFRASTRUCTURE -- NOT PART OF THE PRODUCT.
//
// CPU oracle for the implicit (backward-Euler) APIC MPM substep of ziran2019
// (Lib/MPM over Lib/SPGrid).  It restates the reference algorithm in plain
// C++17 + OpenMP because the reference itself cannot be built here (it needs
// Eigen3, TBB, OpenVDB and partio, none of which are present).  Only the test
// suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and
// only to check results and as the timed CPU baseline; the CUDA library never
// calls it.
//
// Parity pinning:
//   * SPGrid addressing (Linear_Offset, Packed_Add, page map) is pinned against
//     the reference's own SPGrid sources compiled into oracle/_ref (see
//     oracle/ref_spgrid_driver.cpp and tests/golden/).
//   * Everything Eigen-based (constitutive models, SVD, Krylov, transfers) is
//     "parity unpinned" by reference outputs: the reference ships no tests or
//     golden vectors, so it is pinned by analytic known-answer tests only
//     (partition of unity, conservation, SVD reconstruction, FD checks of
//     P/dP/HVP, return-map idempotence).
//
// The grid mirrors SPGrid: a MAP_NORESERVE virtual array of GridState structs
// over the full 4096^3 domain, addressed by the SPGrid byte offset
// (SPGrid_Utilities.cpp:103-109).  P2G runs the reference's 8-colour schedule,
// so per-node summation order is the reference's (colour -> block -> sorted
// particle).  Reductions use fixed 256-node chunks summed in order.

#include "../include/zmpm.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <map>
#include <vector>

#include <parallel/algorithm>
#include <immintrin.h>
#include <sys/mman.h>
#include <omp.h>

namespace zo {

using u64 = uint64_t;

// ------------------------------------------------------------------ SPGrid --
// SPGrid_Mask<log2_struct, log2_field=log2_struct, 3, log2_page=12>,
// Lib/SPGrid/Core/SPGrid_Mask.h:22-52 (masks), :150-157 (Linear_Offset),
// :237-245 (Packed_Add); Bit_Spread/Bit_Pack are pdep/pext
// (SPGrid_Utilities.h:80-359, SPGrid_Utilities.cpp:43-62).
struct Mask {
    int log2_struct = 0, block_bits = 0, xbits = 0, ybits = 0, zbits = 0;
    u64 xmask = 0, ymask = 0, zmask = 0;

    explicit Mask(int l2s)
    {
        log2_struct = l2s;
        block_bits = 12 - l2s;
        zbits = block_bits / 3 + (block_bits % 3 > 0);
        ybits = block_bits / 3 + (block_bits % 3 > 1);
        xbits = block_bits / 3;
        const int sh = 3 - block_bits % 3;
        const u64 hi = ~0ull << 12;
        const u64 pz = (0x9249249249249249ull << sh) & hi;
        const u64 py = (0x2492492492492492ull << sh) & hi;
        const u64 px = (0x4924924924924924ull << sh) & hi;
        const u64 ez = ((1ull << zbits) - 1) << l2s;
        const u64 ey = ((1ull << ybits) - 1) << (l2s + zbits);
        const u64 ex = ((1ull << xbits) - 1) << (l2s + zbits + ybits);
        xmask = px | ex;
        ymask = py | ey;
        zmask = pz | ez;
        init_stencil();
    }
    // BMI2 pdep/pext, the reference's HASWELL path (SPGrid_Utilities.cpp:23-41)
    static u64 deposit(u64 data, u64 mask) { return _pdep_u64(data, mask); }
    static u64 extract(u64 data, u64 mask) { return _pext_u64(data, mask); }
    u64 stencil[27]; // Linear_Offset(i,j,k), i,j,k in {0,1,2}
    void init_stencil()
    {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) stencil[9 * i + 3 * j + k] = linear_offset(i, j, k);
    }
    u64 linear_offset(int i, int j, int k) const
    {
        return deposit((u64)(int64_t)i, xmask) | deposit((u64)(int64_t)j, ymask) | deposit((u64)(int64_t)k, zmask);
    }
    void coord(u64 off, int c[3]) const
    {
        c[0] = (int32_t)extract(off, xmask);
        c[1] = (int32_t)extract(off, ymask);
        c[2] = (int32_t)extract(off, zmask);
    }
    u64 packed_add(u64 a, u64 b) const
    {
        const u64 w = xmask | ymask | zmask;
        const u64 rx = ((a | ~xmask) + (b & xmask)) & xmask;
        const u64 ry = ((a | ~ymask) + (b & ymask)) & ymask;
        const u64 rz = ((a | ~zmask) + (b & zmask)) & zmask;
        const u64 rw = ((a | w) + (b & ~w)) & ~w;
        return rx | ry | rz | rw;
    }
    int bx() const { return 1 << xbits; }
    int by() const { return 1 << ybits; }
    int bz() const { return 1 << zbits; }
    int elements() const { return 1 << block_bits; }
};

// GridState<T,3>, Lib/MPM/MpmGrid.h:14-43 (field order must not change).
template <class T>
struct GridState {
    T v[3];
    T m;
    T new_v[3];
    typename std::conditional<std::is_same<T, float>::value, int32_t, int64_t>::type idx;
    T padding[6];
    T phase_field;
    T phase_field_multiplier;
};
static_assert(sizeof(GridState<double>) == 128, "GridState<double,3> must be 128 B");
static_assert(sizeof(GridState<float>) == 64, "GridState<float,3> must be 64 B");

struct VMem {
    void* p = nullptr;
    size_t n = 0;
    bool map(size_t bytes)
    {
        n = bytes;
        p = mmap(nullptr, n, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        if (p == MAP_FAILED) {
            p = nullptr;
            return false;
        }
        return true;
    }
    void unmap()
    {
        if (p) munmap(p, n);
        p = nullptr;
    }
};

// ------------------------------------------------------------ 3x3 algebra --
template <class T>
struct M3 {
    T a[3][3];
    static M3 zero()
    {
        M3 m;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) m.a[i][j] = 0;
        return m;
    }
    static M3 identity()
    {
        M3 m = zero();
        m.a[0][0] = m.a[1][1] = m.a[2][2] = 1;
        return m;
    }
    T& operator()(int i, int j) { return a[i][j]; }
    const T& operator()(int i, int j) const { return a[i][j]; }
};
template <class T>
static M3<T> mul(const M3<T>& A, const M3<T>& B)
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][0] * B.a[0][j] + A.a[i][1] * B.a[1][j] + A.a[i][2] * B.a[2][j];
    return C;
}
template <class T>
static M3<T> mulT(const M3<T>& A, const M3<T>& B) // A * B^T
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][0] * B.a[j][0] + A.a[i][1] * B.a[j][1] + A.a[i][2] * B.a[j][2];
    return C;
}
template <class T>
static M3<T> Tmul(const M3<T>& A, const M3<T>& B) // A^T * B
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[0][i] * B.a[0][j] + A.a[1][i] * B.a[1][j] + A.a[2][i] * B.a[2][j];
    return C;
}
template <class T>
static M3<T> transpose(const M3<T>& A)
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[j][i];
    return C;
}
template <class T>
static M3<T> scaled(const M3<T>& A, T s)
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][j] * s;
    return C;
}
template <class T>
static M3<T> add(const M3<T>& A, const M3<T>& B)
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][j] + B.a[i][j];
    return C;
}
template <class T>
static T contract(const M3<T>& A, const M3<T>& B)
{
    T s = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s += A.a[i][j] * B.a[i][j];
    return s;
}
template <class T>
static T det(const M3<T>& m)
{
    return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[2][1] * m.a[1][2])
        - m.a[1][0] * (m.a[0][1] * m.a[2][2] - m.a[2][1] * m.a[0][2])
        + m.a[2][0] * (m.a[0][1] * m.a[1][2] - m.a[1][1] * m.a[0][2]);
}
// J F^{-T}, Lib/Ziran/Math/Linear/DenseExt.h:240-252
template <class T>
static M3<T> cofactor(const M3<T>& F)
{
    M3<T> A;
    A.a[0][0] = F.a[1][1] * F.a[2][2] - F.a[1][2] * F.a[2][1];
    A.a[0][1] = F.a[1][2] * F.a[2][0] - F.a[1][0] * F.a[2][2];
    A.a[0][2] = F.a[1][0] * F.a[2][1] - F.a[1][1] * F.a[2][0];
    A.a[1][0] = F.a[0][2] * F.a[2][1] - F.a[0][1] * F.a[2][2];
    A.a[1][1] = F.a[0][0] * F.a[2][2] - F.a[0][2] * F.a[2][0];
    A.a[1][2] = F.a[0][1] * F.a[2][0] - F.a[0][0] * F.a[2][1];
    A.a[2][0] = F.a[0][1] * F.a[1][2] - F.a[0][2] * F.a[1][1];
    A.a[2][1] = F.a[0][2] * F.a[1][0] - F.a[0][0] * F.a[1][2];
    A.a[2][2] = F.a[0][0] * F.a[1][1] - F.a[0][1] * F.a[1][0];
    return A;
}
template <class T>
static M3<T> udiagvt(const M3<T>& U, const T d[3], const M3<T>& V) // U diag(d) V^T
{
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C.a[i][j] = U.a[i][0] * d[0] * V.a[j][0] + U.a[i][1] * d[1] * V.a[j][1] + U.a[i][2] * d[2] * V.a[j][2];
    return C;
}

// ------------------------------------------------------------------ SVD ----
// Implicit-shift QR SVD of 3x3 matrices (Gast et al.), as in
// Lib/Ziran/Math/Linear/ImplicitQRSVD.h:219-532 and Givens.h:33-270.
template <class T>
struct Givens {
    int i, k;
    T c, s;
    Givens(int i_, int k_) : i(i_), k(k_), c(1), s(0) {}
    void compute(T a, T b)
    {
        T d = a * a + b * b;
        c = 1;
        s = 0;
        T sd = std::sqrt(d);
        if (sd) {
            T t = 1 / sd;
            c = a * t;
            s = -b * t;
        }
    }
    void computeUnconventional(T a, T b)
    {
        T d = a * a + b * b;
        c = 0;
        s = 1;
        T sd = std::sqrt(d);
        if (sd) {
            T t = 1 / sd;
            s = a * t;
            c = b * t;
        }
    }
    void rowRotation(M3<T>& A) const
    {
        for (int j = 0; j < 3; ++j) {
            T t1 = A.a[i][j], t2 = A.a[k][j];
            A.a[i][j] = c * t1 - s * t2;
            A.a[k][j] = s * t1 + c * t2;
        }
    }
    void columnRotation(M3<T>& A) const
    {
        for (int j = 0; j < 3; ++j) {
            T t1 = A.a[j][i], t2 = A.a[j][k];
            A.a[j][i] = c * t1 - s * t2;
            A.a[j][k] = s * t1 + c * t2;
        }
    }
};

template <class T>
static void zeroChase(M3<T>& H, M3<T>& U, M3<T>& V)
{
    Givens<T> r1(0, 1);
    r1.compute(H.a[0][0], H.a[1][0]);
    Givens<T> r2(1, 2);
    if (H.a[1][0] != 0)
        r2.compute(H.a[0][0] * H.a[0][1] + H.a[1][0] * H.a[1][1], H.a[0][0] * H.a[0][2] + H.a[1][0] * H.a[1][2]);
    else
        r2.compute(H.a[0][1], H.a[0][2]);
    r1.rowRotation(H);
    r2.columnRotation(H);
    r2.columnRotation(V);
    Givens<T> r3(1, 2);
    r3.compute(H.a[1][1], H.a[2][1]);
    r3.rowRotation(H);
    r1.columnRotation(U);
    r3.columnRotation(U);
}

template <class T>
static void makeUpperBidiag(M3<T>& H, M3<T>& U, M3<T>& V)
{
    U = M3<T>::identity();
    V = M3<T>::identity();
    Givens<T> r(1, 2);
    r.compute(H.a[1][0], H.a[2][0]);
    r.rowRotation(H);
    r.columnRotation(U);
    zeroChase(H, U, V);
}

// 2x2 SVD of the block [[a00,a01],[a10,a11]] in Givens form (ImplicitQRSVD.h:95-160)
template <class T>
static void svd2(T a00, T a01, T a10, T a11, T& uc, T& us, T& s0, T& s1, T& vc, T& vs)
{
    // polar: R from x = (a00 + a11, a10 - a01)
    T x0 = a00 + a11, x1 = a10 - a01;
    T den = std::sqrt(x0 * x0 + x1 * x1);
    uc = 1;
    us = 0;
    if (den != 0) {
        uc = x0 / den;
        us = -x1 / den;
    }
    // S = G A with G = [[c,-s],[s,c]] (rowRotation)
    T S00 = uc * a00 - us * a10, S01 = uc * a01 - us * a11;
    T S11 = us * a01 + uc * a11;
    T cosine, sine;
    T x = S00, y = S01, z = S11;
    T y2 = y * y;
    if (y2 == 0) {
        cosine = 1;
        sine = 0;
        s0 = x;
        s1 = z;
    }
    else {
        T tau = T(0.5) * (x - z);
        T w = std::sqrt(tau * tau + y2);
        T t = (tau > 0) ? y / (tau + w) : y / (tau - w);
        cosine = T(1) / std::sqrt(t * t + T(1));
        sine = -t * cosine;
        T c2 = cosine * cosine;
        T csy = 2 * cosine * sine * y;
        T s2 = sine * sine;
        s0 = c2 * x - csy + s2 * z;
        s1 = s2 * x + csy + c2 * z;
    }
    if (s0 < s1) {
        std::swap(s0, s1);
        vc = -sine;
        vs = cosine;
    }
    else {
        vc = cosine;
        vs = sine;
    }
    // U *= V
    T nc = uc * vc - us * vs;
    T ns = us * vc + uc * vs;
    uc = nc;
    us = ns;
}

template <class T>
static void process2(int t, M3<T>& B, M3<T>& U, T sigma[3], M3<T>& V)
{
    int other = (t == 1) ? 0 : 2;
    sigma[other] = B.a[other][other];
    Givens<T> u(t, t + 1), v(t, t + 1);
    svd2(B.a[t][t], B.a[t][t + 1], B.a[t + 1][t], B.a[t + 1][t + 1], u.c, u.s, sigma[t], sigma[t + 1], v.c, v.s);
    u.columnRotation(U);
    v.columnRotation(V);
}

template <class T>
static void flipSign(int i, M3<T>& U, T sigma[3])
{
    sigma[i] = -sigma[i];
    for (int r = 0; r < 3; ++r) U.a[r][i] = -U.a[r][i];
}
template <class T>
static void swapCol(M3<T>& A, int i, int j)
{
    for (int r = 0; r < 3; ++r) std::swap(A.a[r][i], A.a[r][j]);
}
template <class T>
static void negCol(M3<T>& A, int i)
{
    for (int r = 0; r < 3; ++r) A.a[r][i] = -A.a[r][i];
}

template <class T>
static void sort0(M3<T>& U, T sigma[3], M3<T>& V)
{
    if (std::fabs(sigma[1]) >= std::fabs(sigma[2])) {
        if (sigma[1] < 0) {
            flipSign(1, U, sigma);
            flipSign(2, U, sigma);
        }
        return;
    }
    if (sigma[2] < 0) {
        flipSign(1, U, sigma);
        flipSign(2, U, sigma);
    }
    std::swap(sigma[1], sigma[2]);
    swapCol(U, 1, 2);
    swapCol(V, 1, 2);
    if (sigma[1] > sigma[0]) {
        std::swap(sigma[0], sigma[1]);
        swapCol(U, 0, 1);
        swapCol(V, 0, 1);
    }
    else {
        negCol(U, 2);
        negCol(V, 2);
    }
}

template <class T>
static void sort1(M3<T>& U, T sigma[3], M3<T>& V)
{
    if (std::fabs(sigma[0]) >= sigma[1]) {
        if (sigma[0] < 0) {
            flipSign(0, U, sigma);
            flipSign(2, U, sigma);
        }
        return;
    }
    std::swap(sigma[0], sigma[1]);
    swapCol(U, 0, 1);
    swapCol(V, 0, 1);
    if (std::fabs(sigma[1]) < std::fabs(sigma[2])) {
        std::swap(sigma[1], sigma[2]);
        swapCol(U, 1, 2);
        swapCol(V, 1, 2);
    }
    else {
        negCol(U, 1);
        negCol(V, 1);
    }
    if (sigma[1] < 0) {
        flipSign(1, U, sigma);
        flipSign(2, U, sigma);
    }
}

template <class T>
static T wilkinsonShift(T a1, T b1, T a2)
{
    T d = T(0.5) * (a1 - a2);
    T bs = b1 * b1;
    return a2 - std::copysign(bs / (std::fabs(d) + std::sqrt(d * d + bs)), d);
}

template <class T>
static T svd_tol();
template <>
double svd_tol<double>() { return 1024 * std::numeric_limits<double>::epsilon(); }
template <>
float svd_tol<float>() { return 128 * std::numeric_limits<float>::epsilon(); }

template <class T>
static int svd3(const M3<T>& A, M3<T>& U, T sigma[3], M3<T>& V)
{
    M3<T> B = A;
    makeUpperBidiag(B, U, V);
    int count = 0;
    T tol = svd_tol<T>();
    Givens<T> r(0, 1);
    T alpha_1 = B.a[0][0], beta_1 = B.a[0][1], alpha_2 = B.a[1][1], alpha_3 = B.a[2][2], beta_2 = B.a[1][2];
    T gamma_1 = alpha_1 * beta_1, gamma_2 = alpha_2 * beta_2;
    tol *= std::max(T(0.5) * std::sqrt(alpha_1 * alpha_1 + alpha_2 * alpha_2 + alpha_3 * alpha_3 + beta_1 * beta_1 + beta_2 * beta_2), T(1));
    // the reference loop has no cap; a cap keeps a pathological input from hanging a test
    while (std::fabs(beta_2) > tol && std::fabs(beta_1) > tol && std::fabs(alpha_1) > tol && std::fabs(alpha_2) > tol
        && std::fabs(alpha_3) > tol && count < 1000) {
        T mu = wilkinsonShift(alpha_2 * alpha_2 + beta_1 * beta_1, gamma_2, alpha_3 * alpha_3 + beta_2 * beta_2);
        r.compute(alpha_1 * alpha_1 - mu, gamma_1);
        r.columnRotation(B);
        r.columnRotation(V);
        zeroChase(B, U, V);
        alpha_1 = B.a[0][0];
        beta_1 = B.a[0][1];
        alpha_2 = B.a[1][1];
        alpha_3 = B.a[2][2];
        beta_2 = B.a[1][2];
        gamma_1 = alpha_1 * beta_1;
        gamma_2 = alpha_2 * beta_2;
        count++;
    }
    if (std::fabs(beta_2) <= tol) {
        process2(0, B, U, sigma, V);
        sort0(U, sigma, V);
    }
    else if (std::fabs(beta_1) <= tol) {
        process2(1, B, U, sigma, V);
        sort1(U, sigma, V);
    }
    else if (std::fabs(alpha_2) <= tol) {
        Givens<T> r1(1, 2);
        r1.computeUnconventional(B.a[1][2], B.a[2][2]);
        r1.rowRotation(B);
        r1.columnRotation(U);
        process2(0, B, U, sigma, V);
        sort0(U, sigma, V);
    }
    else if (std::fabs(alpha_3) <= tol) {
        Givens<T> r1(1, 2);
        r1.compute(B.a[1][1], B.a[1][2]);
        r1.columnRotation(B);
        r1.columnRotation(V);
        Givens<T> r2(0, 2);
        r2.compute(B.a[0][0], B.a[0][2]);
        r2.columnRotation(B);
        r2.columnRotation(V);
        process2(0, B, U, sigma, V);
        sort0(U, sigma, V);
    }
    else if (std::fabs(alpha_1) <= tol) {
        Givens<T> r1(0, 1);
        r1.computeUnconventional(B.a[0][1], B.a[1][1]);
        r1.rowRotation(B);
        r1.columnRotation(U);
        Givens<T> r2(0, 2);
        r2.computeUnconventional(B.a[0][2], B.a[2][2]);
        r2.rowRotation(B);
        r2.columnRotation(U);
        process2(1, B, U, sigma, V);
        sort1(U, sigma, V);
    }
    return count;
}

// ------------------------------------------------------------ math tools ---
// Lib/Ziran/Math/MathTools.h:163-262
template <class T>
static T clamp_small_magnitude(T x, T eps)
{
    if (x < -eps) return x;
    if (x < 0) return -eps;
    if (x < eps) return eps;
    return x;
}
template <class T>
static T log_1px_over_x(T x, T eps) { return std::fabs(x) < eps ? T(1) : std::log1p(x) / x; }
template <class T>
static T diff_log_over_diff(T x, T y, T eps) { return log_1px_over_x(x / y - 1, eps) / y; }
template <class T>
static T diff_interlock_log_over_diff(T x, T y, T logy, T eps) { return logy - y * diff_log_over_diff(x, y, eps); }

// ---------------------------------------------------- constitutive models --
template <class T>
struct Model {
    int32_t kind = ZMPM_MODEL_NONE;
    T mu = 0, lambda = 0, kappa = 0, g = 1;
};

// Scratch of one particle.  SvdBasedIsotropicHelper<T,3> coefficients
// (SvdBasedIsotropicHelper.h:97-162) for the SVD-based models.
template <class T>
struct Scratch {
    M3<T> F, FinvT, U, V;
    T J = 1, logJ = 0;
    T sigma[3] = { 1, 1, 1 }, logS[3] = { 0, 0, 0 };
    T psi[3], psi_d[3], psi_o[3]; // psi0..2, psi00/11/22, psi01/02/12
    T m[3], p[3];                 // m01,m02,m12, p01,p02,p12
};

template <class T>
static void isotropicContract(const Scratch<T>& s, const M3<T>& A, M3<T>& B)
{
    // B = dPdF(Sigma) : A, SvdBasedIsotropicHelper.h:151-162
    B.a[0][0] = s.psi_d[0] * A.a[0][0] + s.psi_o[0] * A.a[1][1] + s.psi_o[1] * A.a[2][2];
    B.a[1][1] = s.psi_o[0] * A.a[0][0] + s.psi_d[1] * A.a[1][1] + s.psi_o[2] * A.a[2][2];
    B.a[2][2] = s.psi_o[1] * A.a[0][0] + s.psi_o[2] * A.a[1][1] + s.psi_d[2] * A.a[2][2];
    B.a[0][1] = ((s.m[0] + s.p[0]) * A.a[0][1] + (s.m[0] - s.p[0]) * A.a[1][0]) / 2;
    B.a[1][0] = ((s.m[0] - s.p[0]) * A.a[0][1] + (s.m[0] + s.p[0]) * A.a[1][0]) / 2;
    B.a[0][2] = ((s.m[1] + s.p[1]) * A.a[0][2] + (s.m[1] - s.p[1]) * A.a[2][0]) / 2;
    B.a[2][0] = ((s.m[1] - s.p[1]) * A.a[0][2] + (s.m[1] + s.p[1]) * A.a[2][0]) / 2;
    B.a[1][2] = ((s.m[2] + s.p[2]) * A.a[1][2] + (s.m[2] - s.p[2]) * A.a[2][1]) / 2;
    B.a[2][1] = ((s.m[2] - s.p[2]) * A.a[1][2] + (s.m[2] + s.p[2]) * A.a[2][1]) / 2;
}

template <class T>
static void updateScratch(const Model<T>& c, const M3<T>& F, Scratch<T>& s)
{
    s.F = F;
    if (c.kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        // NeoHookeanBorden::updateScratch, NeoHookeanBorden.cpp:24-35
        s.J = det(F);
        M3<T> JFinvT = cofactor(F);
        s.FinvT = scaled(JFinvT, T(1) / s.J);
        s.logJ = std::log(s.J);
        return;
    }
    if (c.kind != ZMPM_MODEL_STVK_HENCKY_ISOTROPIC && c.kind != ZMPM_MODEL_FIXED_COROTATED) return;
    svd3(F, s.U, s.sigma, s.V);
    const T eps = T(1e-6);
    const T mu = c.mu, lambda = c.lambda;
    const T* sg = s.sigma;
    if (c.kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
        // StvkWithHenckyIsotropic::updateScratch (3D), StvkWithHenckyIsotropic.h:114-143
        for (int d = 0; d < 3; ++d) s.logS[d] = std::log(std::fabs(sg[d]));
        const T* L = s.logS;
        T g = 2 * mu + lambda;
        T sum_log = L[0] + L[1] + L[2];
        T prod01 = sg[0] * sg[1], prod02 = sg[0] * sg[2], prod12 = sg[1] * sg[2];
        s.psi[0] = (2 * mu * L[0] + lambda * sum_log) / sg[0];
        s.psi[1] = (2 * mu * L[1] + lambda * sum_log) / sg[1];
        s.psi[2] = (2 * mu * L[2] + lambda * sum_log) / sg[2];
        s.psi_d[0] = (g * (1 - L[0]) - lambda * (L[1] + L[2])) / (sg[0] * sg[0]);
        s.psi_d[1] = (g * (1 - L[1]) - lambda * (L[0] + L[2])) / (sg[1] * sg[1]);
        s.psi_d[2] = (g * (1 - L[2]) - lambda * (L[0] + L[1])) / (sg[2] * sg[2]);
        s.psi_o[0] = lambda / (sg[0] * sg[1]);
        s.psi_o[1] = lambda / (sg[0] * sg[2]);
        s.psi_o[2] = lambda / (sg[1] * sg[2]);
        s.m[0] = -(lambda * sum_log + 2 * mu * diff_interlock_log_over_diff(sg[0], sg[1], L[1], eps)) / prod01;
        s.m[1] = -(lambda * sum_log + 2 * mu * diff_interlock_log_over_diff(sg[0], sg[2], L[2], eps)) / prod02;
        s.m[2] = -(lambda * sum_log + 2 * mu * diff_interlock_log_over_diff(sg[1], sg[2], L[2], eps)) / prod12;
    }
    else {
        // Fixed corotated, psi = mu sum (s_i-1)^2 + lambda/2 (J-1)^2 written in
        // the same SVD-isotropic form (derivatives of psi-hat in sigma).
        T J = sg[0] * sg[1] * sg[2];
        T c0 = sg[1] * sg[2], c1 = sg[0] * sg[2], c2 = sg[0] * sg[1];
        s.J = J;
        s.psi[0] = 2 * mu * (sg[0] - 1) + lambda * (J - 1) * c0;
        s.psi[1] = 2 * mu * (sg[1] - 1) + lambda * (J - 1) * c1;
        s.psi[2] = 2 * mu * (sg[2] - 1) + lambda * (J - 1) * c2;
        s.psi_d[0] = 2 * mu + lambda * c0 * c0;
        s.psi_d[1] = 2 * mu + lambda * c1 * c1;
        s.psi_d[2] = 2 * mu + lambda * c2 * c2;
        s.psi_o[0] = lambda * sg[2] * (2 * J - 1);
        s.psi_o[1] = lambda * sg[1] * (2 * J - 1);
        s.psi_o[2] = lambda * sg[0] * (2 * J - 1);
        s.m[0] = 2 * mu - lambda * (J - 1) * sg[2];
        s.m[1] = 2 * mu - lambda * (J - 1) * sg[1];
        s.m[2] = 2 * mu - lambda * (J - 1) * sg[0];
    }
    s.p[0] = (s.psi[0] + s.psi[1]) / clamp_small_magnitude(sg[0] + sg[1], eps);
    s.p[1] = (s.psi[0] + s.psi[2]) / clamp_small_magnitude(sg[0] + sg[2], eps);
    s.p[2] = (s.psi[1] + s.psi[2]) / clamp_small_magnitude(sg[1] + sg[2], eps);
}

template <class T>
static T psi(const Model<T>& c, const Scratch<T>& s)
{
    if (c.kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        // NeoHookeanBorden::psi, NeoHookeanBorden.cpp:37-52
        M3<T> JaF = scaled(s.F, std::pow(s.J, -T(1) / T(3)));
        T psi_dev = c.mu / 2 * (contract(JaF, JaF) - 3);
        T psi_vol = c.kappa / 2 * ((s.J * s.J - 1) / 2 - std::log(s.J));
        T psi_pos = (s.J >= 1) ? (psi_vol + psi_dev) : psi_dev;
        T psi_neg = (s.J >= 1) ? T(0) : psi_vol;
        return c.g * psi_pos + psi_neg;
    }
    if (c.kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
        T tr = s.logS[0] + s.logS[1] + s.logS[2];
        return c.mu * (s.logS[0] * s.logS[0] + s.logS[1] * s.logS[1] + s.logS[2] * s.logS[2]) + T(0.5) * c.lambda * tr * tr;
    }
    if (c.kind == ZMPM_MODEL_FIXED_COROTATED) {
        T a = s.sigma[0] - 1, b = s.sigma[1] - 1, d = s.sigma[2] - 1, J = s.sigma[0] * s.sigma[1] * s.sigma[2];
        return c.mu * (a * a + b * b + d * d) + T(0.5) * c.lambda * (J - 1) * (J - 1);
    }
    return 0;
}

template <class T>
static M3<T> firstPiola(const Model<T>& c, const Scratch<T>& s)
{
    if (c.kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        // kirchhoff (NeoHookeanBorden.cpp:67-83), then P = tau F^{-T}
        // (HyperelasticConstitutiveModel.h:85-90)
        M3<T> B = mulT(s.F, s.F);
        T tr = B.a[0][0] + B.a[1][1] + B.a[2][2];
        M3<T> devB = B;
        for (int d = 0; d < 3; ++d) devB.a[d][d] = B.a[d][d] - T(1) / 3 * tr;
        M3<T> tau_dev = scaled(devB, c.mu * std::pow(s.J, -T(2) / T(3)));
        T prime = c.kappa / 2 * (s.J - 1 / s.J);
        T vol = s.J * prime;
        M3<T> tau;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                T tv = (i == j) ? vol : T(0);
                tau.a[i][j] = (s.J >= 1) ? c.g * (tau_dev.a[i][j] + tv) : c.g * tau_dev.a[i][j] + tv;
            }
        return mul(tau, s.FinvT);
    }
    if (c.kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC || c.kind == ZMPM_MODEL_FIXED_COROTATED)
        return udiagvt(s.U, s.psi, s.V);
    return M3<T>::zero();
}

template <class T>
static M3<T> firstPiolaDifferential(const Model<T>& c, const Scratch<T>& s, const M3<T>& dF)
{
    if (c.kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        // NeoHookeanBorden::firstPiolaDifferential, NeoHookeanBorden.cpp:85-111
        T FinvT_dF = contract(s.FinvT, dF);
        T deltaJ = s.J * FinvT_dF;
        T FcontractF = contract(s.F, s.F);
        M3<T> deltaFinvT = scaled(mul(mul(s.FinvT, transpose(dF)), s.FinvT), T(-1));
        T a = -T(1) / 3;
        T muJ2a = c.mu * std::pow(s.J, T(2) * a);
        T prime = c.kappa / 2 * (s.J - T(1) / s.J);
        T prime2 = c.kappa / 2 * (T(1) + T(1) / (s.J * s.J));
        T F_dF = contract(s.F, dF);
        M3<T> dP;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                T dev = 2 * a * muJ2a * FinvT_dF * (a * FcontractF * s.FinvT.a[i][j] + s.F.a[i][j]);
                dev += muJ2a * (2 * a * F_dF * s.FinvT.a[i][j] + a * FcontractF * deltaFinvT.a[i][j] + dF.a[i][j]);
                T vol = deltaJ * prime * s.FinvT.a[i][j] + s.J * deltaJ * prime2 * s.FinvT.a[i][j] + s.J * prime * deltaFinvT.a[i][j];
                dP.a[i][j] = (s.J >= 1) ? c.g * (dev + vol) : c.g * dev + vol;
            }
        return dP;
    }
    if (c.kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC || c.kind == ZMPM_MODEL_FIXED_COROTATED) {
        // StvkWithHenckyIsotropic::firstPiolaDifferential, StvkWithHenckyIsotropic.h:164-170
        M3<T> D = mul(Tmul(s.U, dF), s.V);
        M3<T> K;
        isotropicContract(s, D, K);
        return mulT(mul(s.U, K), s.V);
    }
    return M3<T>::zero();
}

// ------------------------------------------------------------ plasticity --
template <class T>
struct Plastic {
    int32_t kind = ZMPM_PLASTIC_NONE;
    T yield_stress = 0, xi = 0, fail_stress = 0;
    int32_t broken = 0;
    T crack_normal[3] = { 0, 0, 0 };
    // Drucker-Prager (alpha, beta, cohesion, volume_correction) and Cam-Clay
    // (M, beta, xi, hardeningOn) members, log Jp of both
    T a = 0, beta = 0, cx = 0, logJp = 0;
    int32_t flag = 0;
};

// sin of an angle in degrees with the reference's constant for pi
// (PlasticityApplier.cpp:17, :255)
template <class T>
static T sinDegrees(T angle)
{
    return std::sin(angle / T(180) * T(3.141592653));
}

// DruckerPragerStvkHencky::projectStrain, PlasticityApplier.cpp:272-317
template <class T>
static void druckerPragerProject(const Model<T>& c, Plastic<T>& p, M3<T>& F)
{
    M3<T> U, V;
    T sigma[3];
    svd3(F, U, sigma, V);
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(std::abs(sigma[d]), T(1e-4))) - p.cx;
    const T esum = eps[0] + eps[1] + eps[2];
    const T tr = esum + p.logJp;
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    const T hat2 = hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2];
    if (tr >= T(0)) { // case II: the tip
        const T ec = std::exp(p.cx);
        M3<T> Us = scaled(U, ec);
        F = mulT(Us, V);
        if (p.flag) p.logJp = p.beta * esum + p.logJp;
        return;
    }
    else if (c.mu == 0)
        return;
    p.logJp = 0;
    const T hn = std::sqrt(hat2);
    const T dg = hn + (T(3) * c.lambda + T(2) * c.mu) / (T(2) * c.mu) * tr * p.a;
    T H[3], eH[3];
    for (int d = 0; d < 3; ++d) H[d] = (dg <= 0) ? eps[d] + p.cx : eps[d] - (dg / hn) * hat[d] + p.cx;
    for (int d = 0; d < 3; ++d) eH[d] = std::exp(H[d]);
    F = udiagvt(U, eH, V);
}

// NonAssociativeCamClay::projectStrain, PlasticityApplier.cpp:112-136, through
// Compare_With_Physbam (:35-110), the branch the reference runs
template <class T>
static void camClayProject(const Model<T>& c, Plastic<T>& p, M3<T>& F)
{
    M3<T> U, V;
    T Se[3];
    svd3(F, U, Se, V);
    const T p0 = c.kappa * (T(0.00001) + std::sinh(p.cx * std::max(-p.logJp, T(0))));
    const T a = (T(1) + T(2) * p.beta) * (T(6) - T(3)) / T(2);
    const T b = p.beta * p0, cc = p0, M2 = p.a * p.a;
    T Je = 1;
    for (int i = 0; i < 3; ++i) Je *= Se[i];
    T Se2[3];
    for (int i = 0; i < 3; ++i) Se2[i] = Se[i] * Se[i];
    T mean = 0;
    for (int i = 0; i < 3; ++i) mean += Se2[i];
    mean /= T(3);
    const T sc = c.mu * std::pow(Je, -T(2) / T(3));
    T s[3];
    for (int i = 0; i < 3; ++i) s[i] = sc * (Se2[i] - mean);
    const T Uprime = c.kappa / T(2) * (Je - 1 / Je);
    const T p_trial = -Uprime * Je;
    if (p_trial > cc || p_trial < -b) { // the tips
        const T Je_new = (p_trial > cc) ? std::sqrt(-2 * cc / c.kappa + 1) : std::sqrt(2 * b / c.kappa + 1);
        const T r = std::pow(Je_new, T(1) / T(3));
        for (int i = 0; i < 3; ++i) Se[i] = r;
        p.logJp += std::log(Je / Je_new);
        F = udiagvt(U, Se, V);
        return;
    }
    const T k = std::sqrt(-M2 * (p_trial + b) * (p_trial - cc) / a);
    const T sn = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    const T y = a * (sn * sn) + M2 * (p_trial + b) * (p_trial - cc);
    if (y < T(1e-4)) { // inside: the strain is rebuilt from its SVD
        F = udiagvt(U, Se, V);
        return;
    }
    const T pc = (T(1) - p.beta) * p0 / 2;
    if (p0 > T(1e-4) && p_trial < p0 - T(1e-4) && p_trial > -p.beta * p0 + T(1e-4)) {
        const T aa = M2 * ((p_trial - pc) * (p_trial - pc)) / (a * (sn * sn));
        const T dd = 1 + aa;
        const T ff = aa * p.beta * p0 - aa * p0 - 2 * pc;
        const T gg = pc * pc - aa * p.beta * (p0 * p0);
        const T zz = std::sqrt(std::abs(ff * ff - 4 * dd * gg));
        const T p1 = (-ff + zz) / (2 * dd);
        const T p2 = (-ff - zz) / (2 * dd);
        const T p_fake = (p_trial - pc) * (p1 - pc) > 0 ? p1 : p2;
        const T Je_new_fake = std::sqrt(std::abs(-2 * p_fake / c.kappa + 1));
        if (Je_new_fake > T(1e-4)) p.logJp += std::log(Je / Je_new_fake);
    }
    const T g = k / c.mu * std::pow(Je, T(2) / T(3));
    const T tr = T(1) / T(3) * (Se2[0] + Se2[1] + Se2[2]);
    for (int i = 0; i < 3; ++i) Se[i] = std::sqrt(g * s[i] / sn + tr * T(1));
    F = udiagvt(U, Se, V);
}

// VonMisesStvkHencky::projectStrain, PlasticityApplier.cpp:462-502
template <class T>
static void vonMisesProject(const Model<T>& c, Plastic<T>& p, M3<T>& F)
{
    M3<T> U, V;
    T sigma[3];
    svd3(F, U, sigma, V);
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(sigma[d], T(1e-4)));
    T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    T hat2 = hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2];
    T hat_norm = std::sqrt(hat2);
    T delta_gamma = hat_norm - p.yield_stress / (2 * c.mu);
    if (delta_gamma <= 0) return;
    p.yield_stress -= p.xi * delta_gamma;
    T H[3], expH[3];
    for (int d = 0; d < 3; ++d) H[d] = eps[d] - (delta_gamma / hat_norm) * hat[d];
    T tau_0 = 2 * c.mu * H[0] + c.lambda * (H[0] + H[1] + H[2]);
    for (int d = 0; d < 3; ++d) expH[d] = std::exp(H[d]);
    F = udiagvt(U, expH, V);
    if (tau_0 >= p.fail_stress) {
        p.broken = 1;
        for (int d = 0; d < 3; ++d) p.crack_normal[d] = V.a[d][0];
    }
}

// Reverse mode of vonMisesProject with a constant yield stress (xi = 0): F =
// Pi(Fp) = U diag(f(sigma)) V^T with f_i = exp(tr(eps)/3 + r n_i), r =
// yield / (2 mu), n the unit deviatoric Hencky strain, an isotropic map of Fp.
// Given Gb = dL/dF returns dL/dFp and adds dL/dE (r ~ 1/E at fixed nu) to gE.
// The derivative of an isotropic matrix function: with A = U^T dFp V the
// output's U^T dF V has diagonal J diag(A) (J = df/dsigma) and off-diagonal
// entries (f_i - f_j)/(s_i - s_j) sym(A)_ij + (f_i + f_j)/(s_i + s_j) skew(A)_ij;
// its transpose swaps J for J^T and keeps the off-diagonal part.
template <class T>
static M3<T> vonMisesAdjoint(const Model<T>& c, const Plastic<T>& p, const M3<T>& Fp, const M3<T>& Gb, T& gE)
{
    M3<T> U, V;
    T s[3];
    svd3(Fp, U, s, V);
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(s[d], T(1e-4)));
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - tr / T(3);
    const T hn = std::sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T r = p.yield_stress / (2 * c.mu);
    if (!(hn - r > 0)) return Gb;
    T n[3], f[3], J[3][3];
    for (int d = 0; d < 3; ++d) {
        n[d] = hat[d] / hn;
        f[d] = std::exp(tr / 3 + r * n[d]);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            // d eps_j / d s_j = 1/s_j; d n_i / d eps_j = (delta_ij - 1/3 - n_i n_j) / |hat|
            T dn = (T(i == j) - T(1) / 3 - n[i] * n[j]) / hn;
            J[i][j] = s[j] > T(1e-4) ? f[i] * (T(1) / 3 + r * dn) / s[j] : T(0);
        }
    M3<T> A = mul(Tmul(U, Gb), V), Ab;
    for (int j = 0; j < 3; ++j) Ab.a[j][j] = J[0][j] * A.a[0][0] + J[1][j] * A.a[1][1] + J[2][j] * A.a[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            if (i == j) continue;
            T a = std::fabs(s[i] - s[j]) > T(1e-12) * std::fabs(s[0]) ? (f[i] - f[j]) / (s[i] - s[j]) : J[i][i] - J[i][j];
            T b = (f[i] + f[j]) / (s[i] + s[j]);
            Ab.a[i][j] = a * (A.a[i][j] + A.a[j][i]) / 2 + b * (A.a[i][j] - A.a[j][i]) / 2;
        }
    const T E = c.mu * (3 * c.lambda + 2 * c.mu) / (c.lambda + c.mu);
    gE += -(r / E) * (A.a[0][0] * f[0] * n[0] + A.a[1][1] * f[1] * n[1] + A.a[2][2] * f[2] * n[2]);
    return mulT(mul(U, Ab), V);
}

// ---------------------------------------------------------------- damage --
template <class T>
struct Damage {
    int32_t kind = ZMPM_DAMAGE_NONE;
    T c = 1, k = T(0.001), sigma_f = 0;
    // PhaseField members (PhaseField.h:13-22) of ZMPM_DAMAGE_PHASE_FIELD
    T H = 0, l0 = 0, one_over_sigma_c = 0, pf_Fp = 1, H_max = std::numeric_limits<T>::max(), vol = 0;
    bool allow_damage = true;
};

// NeoHookeanBorden::get_psi_pos (NeoHookeanBorden.cpp:53-66): the part of the
// energy that the phase field degrades.
template <class T>
static T neoHookeanBordenPsiPos(const Model<T>& c, const M3<T>& F)
{
    const T J = det(F);
    const T a = std::pow(J, -T(1) / T(3));
    T tr = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tr += (a * F.a[i][j]) * (a * F.a[i][j]);
    const T psi_dev = c.mu / 2 * (tr - 3);
    const T psi_vol = c.kappa / 2 * ((J * J - 1) / 2 - std::log(J));
    return (J >= 1) ? (psi_vol + psi_dev) : psi_dev;
}

// PhaseField::Get_Sigma_C_Based_On_Max_Deformation (PhaseField.h:58-68):
// 1 / psi((1 + percentage) I) of the model (NeoHookeanBorden::psi, .cpp:38-51).
template <class T>
static T phaseFieldOneOverSigmaC(const Model<T>& c, T percentage)
{
    M3<T> F = M3<T>::identity();
    for (int i = 0; i < 3; ++i) F.a[i][i] = 1 + percentage;
    const T J = det(F);
    const T psi_pos = neoHookeanBordenPsiPos(c, F);
    const T psi_vol = c.kappa / 2 * ((J * J - 1) / 2 - std::log(J));
    const T psi_neg = (J >= 1) ? T(0) : psi_vol;
    return T(1) / (c.g * psi_pos + psi_neg);
}

// Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Golub & Van Loan, Matrix Computations, 8.5.2).
template <class T>
static T sym3_max_eig_jacobi(M3<T> A)
{
    for (int sweep = 0; sweep < 50; ++sweep) {
        T off = A.a[0][1] * A.a[0][1] + A.a[0][2] * A.a[0][2] + A.a[1][2] * A.a[1][2];
        if (off == 0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A.a[p][q] == 0) continue;
                T theta = (A.a[q][q] - A.a[p][p]) / (2 * A.a[p][q]);
                T t = (theta >= 0 ? T(1) : T(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                T c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 3; ++k) { // A <- J^T A J
                    T akp = A.a[k][p], akq = A.a[k][q];
                    A.a[k][p] = c * akp - s * akq;
                    A.a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    T apk = A.a[p][k], aqk = A.a[q][k];
                    A.a[p][k] = c * apk - s * aqk;
                    A.a[q][k] = s * apk + c * aqk;
                }
            }
    }
    return std::max(A.a[0][0], std::max(A.a[1][1], A.a[2][2]));
}

// ---- the first eigenvalue of Eigen's general (real, non-symmetric) eigensolver
// FractureSimulation.h:539-543 takes sigma_max = cauchy.eigenvalues()[0].real()
// from Eigen::EigenSolver, i.e. the first diagonal entry (or 2x2 block) of the
// real Schur form that its RealSchur produces.  Eigen is not part of the
// reference tree (find_package(Eigen3), version unpinned; 3.3 on the
// reference's platform), so this restates its published method for a 3x3
// matrix: scaling by the largest |a_ij|, Householder reduction to upper
// Hessenberg form, and the Francis double-shift QR iteration of EISPACK hqr /
// JAMA hqr2 (Golub & Van Loan, Matrix Computations, 7.5) with deflation when a
// subdiagonal entry falls below eps (|t_kk| + |t_k-1,k-1|), exceptional shifts
// at iterations 10 and 30 of one eigenvalue, and a 2x2 block with real
// eigenvalues split by the rotation that keeps each diagonal entry with its
// nearer eigenvalue.  Returns the real part of the first eigenvalue in that
// order.  Parity unpinned (no Eigen here); checked by known answers.

// Householder vector of (x0, x1[, x2]) in the form I - tau (1, e)(1, e)^T with
// (I - tau ...) x = (beta, 0, 0).
static void householder(const double* x, int n, double& tau, double& beta, double* ess)
{
    double tail = 0;
    for (int i = 1; i < n; ++i) tail += x[i] * x[i];
    const double c0 = x[0];
    if (tail <= std::numeric_limits<double>::min()) {
        tau = 0;
        beta = c0;
        for (int i = 1; i < n; ++i) ess[i - 1] = 0;
        return;
    }
    beta = std::sqrt(c0 * c0 + tail);
    if (c0 >= 0) beta = -beta;
    for (int i = 1; i < n; ++i) ess[i - 1] = x[i] / (c0 - beta);
    tau = (beta - c0) / beta;
}
// T[r0..r0+n)[c0..c1) <- H T with H = I - tau v v^T, v = (1, ess)
static void reflect_left(double T[3][3], int r0, int n, int c0, int c1, double tau, const double* ess)
{
    for (int c = c0; c < c1; ++c) {
        double d = T[r0][c];
        for (int i = 1; i < n; ++i) d += ess[i - 1] * T[r0 + i][c];
        T[r0][c] -= tau * d;
        for (int i = 1; i < n; ++i) T[r0 + i][c] -= tau * ess[i - 1] * d;
    }
}
// T[r0..r1)[c0..c0+n) <- T H
static void reflect_right(double T[3][3], int r0, int r1, int c0, int n, double tau, const double* ess)
{
    for (int r = r0; r < r1; ++r) {
        double d = T[r][c0];
        for (int i = 1; i < n; ++i) d += ess[i - 1] * T[r][c0 + i];
        T[r][c0] -= tau * d;
        for (int i = 1; i < n; ++i) T[r][c0 + i] -= tau * ess[i - 1] * d;
    }
}

static double eigen_first_eigenvalue(const double A[3][3])
{
    const int n = 3;
    const double eps = std::numeric_limits<double>::epsilon();
    double scale = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) scale = std::max(scale, std::fabs(A[i][j]));
    if (scale < std::numeric_limits<double>::min()) return 0;
    double T[3][3];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) T[i][j] = A[i][j] / scale;
    { // Hessenberg: one reflection of column 0 below the subdiagonal
        double x[2] = { T[1][0], T[2][0] }, tau, beta, ess[1];
        householder(x, 2, tau, beta, ess);
        T[1][0] = beta;
        T[2][0] = 0;
        reflect_left(T, 1, 2, 1, 3, tau, ess);
        reflect_right(T, 0, 3, 1, 2, tau, ess);
    }
    double norm = 0; // of the upper Hessenberg part
    for (int j = 0; j < n; ++j)
        for (int i = 0; i <= std::min(j + 1, n - 1); ++i) norm += std::fabs(T[i][j]);
    if (norm == 0) return 0;
    int iu = n - 1, iter = 0, total = 0;
    double exshift = 0;
    while (iu >= 0) {
        int il = iu; // the lowest row of the active block (small subdiagonal above it)
        while (il > 0) {
            double s = std::fabs(T[il - 1][il - 1]) + std::fabs(T[il][il]);
            if (s == 0) s = norm;
            if (std::fabs(T[il][il - 1]) < eps * s) break;
            --il;
        }
        if (il == iu) { // one eigenvalue
            T[iu][iu] += exshift;
            if (iu > 0) T[iu][iu - 1] = 0;
            --iu;
            iter = 0;
        }
        else if (il == iu - 1) { // a 2x2 block
            const double p = 0.5 * (T[iu - 1][iu - 1] - T[iu][iu]);
            const double q = p * p + T[iu][iu - 1] * T[iu - 1][iu];
            T[iu][iu] += exshift;
            T[iu - 1][iu - 1] += exshift;
            if (q >= 0) { // two real eigenvalues: rotate the block upper triangular
                const double z = std::sqrt(std::fabs(q));
                const double a = p >= 0 ? p + z : p - z, b = T[iu][iu - 1];
                const double r = std::hypot(a, b);
                const double c = r == 0 ? 1.0 : a / r, sn = r == 0 ? 0.0 : b / r;
                for (int k = iu - 1; k < n; ++k) { // left: rows iu-1, iu
                    const double t0 = T[iu - 1][k], t1 = T[iu][k];
                    T[iu - 1][k] = c * t0 + sn * t1;
                    T[iu][k] = -sn * t0 + c * t1;
                }
                for (int k = 0; k <= iu; ++k) { // right: columns iu-1, iu
                    const double t0 = T[k][iu - 1], t1 = T[k][iu];
                    T[k][iu - 1] = c * t0 + sn * t1;
                    T[k][iu] = -sn * t0 + c * t1;
                }
                T[iu][iu - 1] = 0;
            }
            if (iu > 1) T[iu - 1][iu - 2] = 0;
            iu -= 2;
            iter = 0;
        }
        else { // Francis double-shift step on rows il..iu
            double x = T[iu][iu], y = T[iu - 1][iu - 1], w = T[iu][iu - 1] * T[iu - 1][iu];
            if (iter == 10) { // exceptional shift
                exshift += x;
                for (int i = 0; i <= iu; ++i) T[i][i] -= x;
                const double s = std::fabs(T[iu][iu - 1]) + std::fabs(T[iu - 1][iu - 2]);
                x = y = 0.75 * s;
                w = -0.4375 * s * s;
            }
            if (iter == 30) {
                double s = 0.5 * (y - x);
                s = s * s + w;
                if (s > 0) {
                    s = std::sqrt(s);
                    if (y < x) s = -s;
                    s = x - w / (0.5 * (y - x) + s);
                    for (int i = 0; i <= iu; ++i) T[i][i] -= s;
                    exshift += s;
                    x = y = w = 0.964;
                }
            }
            ++iter;
            if (++total > 40 * n) break;
            int im = iu - 2;
            double v[3];
            for (;; --im) {
                const double tmm = T[im][im], r = x - tmm, s = y - tmm;
                v[0] = (r * s - w) / T[im + 1][im] + T[im][im + 1];
                v[1] = T[im + 1][im + 1] - tmm - r - s;
                v[2] = T[im + 2][im + 1];
                if (im == il) break;
                const double lhs = T[im][im - 1] * (std::fabs(v[1]) + std::fabs(v[2]));
                const double rhs = v[0] * (std::fabs(T[im - 1][im - 1]) + std::fabs(tmm) + std::fabs(T[im + 1][im + 1]));
                if (std::fabs(lhs) < eps * rhs) break;
            }
            for (int k = im; k <= iu - 2; ++k) {
                const bool first = k == im;
                if (!first) {
                    v[0] = T[k][k - 1];
                    v[1] = T[k + 1][k - 1];
                    v[2] = T[k + 2][k - 1];
                }
                double tau, beta, ess[2];
                householder(v, 3, tau, beta, ess);
                if (beta != 0) {
                    if (first && k > il)
                        T[k][k - 1] = -T[k][k - 1];
                    else if (!first)
                        T[k][k - 1] = beta;
                    reflect_left(T, k, 3, k, n, tau, ess);
                    reflect_right(T, 0, std::min(iu, k + 3) + 1, k, 3, tau, ess);
                }
            }
            {
                double v2[2] = { T[iu - 1][iu - 2], T[iu][iu - 2] }, tau, beta, ess[1];
                householder(v2, 2, tau, beta, ess);
                if (beta != 0) {
                    T[iu - 1][iu - 2] = beta;
                    reflect_left(T, iu - 1, 2, iu - 1, n, tau, ess);
                    reflect_right(T, 0, iu + 1, iu - 1, 2, tau, ess);
                }
            }
            for (int i = im + 2; i <= iu; ++i) {
                T[i][i - 2] = 0;
                if (i > im + 2) T[i][i - 3] = 0;
            }
        }
    }
    // EigenSolver: a real eigenvalue where the subdiagonal is zero, else a
    // complex pair whose real part is the block's mean
    if (T[1][0] == 0) return T[0][0] * scale;
    return 0.5 * (T[0][0] + T[1][1]) * scale;
}

template <class T>
static T rankine_first_eigenvalue(const M3<T>& A)
{
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = (double)A.a[i][j];
    return (T)eigen_first_eigenvalue(a);
}

// FractureSimulation::solvePhaseFieldSystemNaive, FractureSimulation.h:509-554
// (principal Cauchy stress of the undegraded NeoHookeanBorden stress): the
// largest eigenvalue (ZMPM_DAMAGE_RANKINE) or, as the reference computes it,
// the first eigenvalue of Eigen's general eigensolver (ZMPM_DAMAGE_RANKINE_REFERENCE).
template <class T>
static void rankineUpdate(Model<T>& c, Damage<T>& d, const M3<T>& F)
{
    T J = det(F);
    M3<T> B = mulT(F, F);
    T tr = B.a[0][0] + B.a[1][1] + B.a[2][2];
    T sdev = c.mu * std::pow(J, -T(2) / T(3));
    T vol = J * (c.kappa / 2 * (J - 1 / J));
    M3<T> cauchy;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T dv = (i == j) ? B.a[i][j] - T(1) / 3 * tr : B.a[i][j];
            cauchy.a[i][j] = ((i == j) ? sdev * dv + vol : sdev * dv) / J;
        }
    T smax = d.kind == ZMPM_DAMAGE_RANKINE_REFERENCE ? rankine_first_eigenvalue(cauchy) : sym3_max_eig_jacobi(cauchy);
    T newC = d.c;
    if (smax > d.sigma_f) newC = std::min(d.c, d.sigma_f / smax);
    d.c = newC;
    c.g = newC * newC * (1 - d.k) + d.k;
}

// ------------------------------------------------------- viscoelastic --
// Second elastic strain Fe ("Fe_Nonequilibrated") with the reference's only
// instantiated model StvkWithHencky (MpmParticlesHandle3d.cpp:9).
template <class T>
struct Visco {
    int32_t on = 0;
    T mu = 0, lambda = 0, vd = 1, vv = 1; // StvkWithHencky(E, nu), viscosity_d, viscosity_v
};

// FElasticNonequilibratedBasedMpmForceHelper::evolveStrain,
// FElasticNonequilibratedBasedMpmForceHelper.h:62-87: backward-Euler relaxation
// of the Hencky strain of Fe (deviatoric rate alpha, volumetric rate alpha + 3 beta).
template <class T>
static void viscousCoefficients(const Visco<T>& v, T dt, T& a, T& b)
{
    T alpha = T(2.0) * v.mu / v.vd;
    T beta = T(2.0) * (T(2.0) * v.mu + v.lambda * 3) / (T(9.0) * v.vv) - T(2.0) * v.mu / (v.vd * 3);
    a = T(1.0) / (T(1.0) + dt * alpha);
    b = dt * beta / (T(1.0) + dt * (alpha + 3 * beta));
}

template <class T>
static void viscousReturn(const Visco<T>& v, T dt, M3<T>& Fe)
{
    M3<T> U, V;
    T sigma[3];
    svd3(Fe, U, sigma, V);
    T a, b;
    viscousCoefficients(v, dt, a, b);
    T et[3];
    for (int d = 0; d < 3; ++d) et[d] = std::log(std::fabs(sigma[d]));
    // `epsilon_trial.trace()` of a 3-vector: Eigen's trace of a 3x1 matrix is
    // its single diagonal coefficient, epsilon_trial(0)
    T tr = et[0];
    T ex[3];
    for (int d = 0; d < 3; ++d) ex[d] = std::exp(a * (et[d] - b * tr));
    Fe = udiagvt(U, ex, V);
}

// ------------------------------------------------------------------ ADMM --
// Diagonal (singular-value space) derivatives of psi = mu |log S|^2 +
// lambda/2 tr(log S)^2, StvkWithHenckyIsotropic.h:218-269 (identical in
// StvkWithHencky.cpp:154-183).
template <class T>
static void henckyDiagonal(T mu, T lambda, const T s[3], T dE[3], T ddE[3][3])
{
    T L[3];
    for (int d = 0; d < 3; ++d) L[d] = std::log(std::fabs(s[d]));
    T sum_log = L[0] + L[1] + L[2];
    T g = 2 * mu + lambda;
    for (int d = 0; d < 3; ++d) dE[d] = (2 * mu * L[d] + lambda * sum_log) / s[d];
    ddE[0][0] = (g * (1 - L[0]) - lambda * (L[1] + L[2])) / (s[0] * s[0]);
    ddE[1][1] = (g * (1 - L[1]) - lambda * (L[0] + L[2])) / (s[1] * s[1]);
    ddE[2][2] = (g * (1 - L[2]) - lambda * (L[0] + L[1])) / (s[2] * s[2]);
    ddE[0][1] = ddE[1][0] = lambda / (s[0] * s[1]);
    ddE[0][2] = ddE[2][0] = lambda / (s[0] * s[2]);
    ddE[1][2] = ddE[2][1] = lambda / (s[1] * s[2]);
}

// Eigenvalues of a symmetric 3x3 matrix by cyclic Jacobi rotations.
template <class T>
static void sym3EigJacobi(M3<T> A, T ev[3])
{
    for (int sweep = 0; sweep < 50; ++sweep) {
        T off = A.a[0][1] * A.a[0][1] + A.a[0][2] * A.a[0][2] + A.a[1][2] * A.a[1][2];
        if (off == 0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A.a[p][q] == 0) continue;
                T theta = (A.a[q][q] - A.a[p][p]) / (2 * A.a[p][q]);
                T t = (theta >= 0 ? T(1) : T(-1)) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                T c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    T akp = A.a[k][p], akq = A.a[k][q];
                    A.a[k][p] = c * akp - s * akq;
                    A.a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    T apk = A.a[p][k], aqk = A.a[q][k];
                    A.a[p][k] = c * apk - s * aqk;
                    A.a[q][k] = s * apk + c * aqk;
                }
            }
    }
    for (int d = 0; d < 3; ++d) ev[d] = A.a[d][d];
}

// Squared Frobenius norms of makePD / makePD2D (AdmmFormula.h:12-35): the
// eigenvalues clamped at zero.
template <class T>
static T makePDNorm2(const M3<T>& A)
{
    T ev[3];
    sym3EigJacobi(A, ev);
    T s = 0;
    for (int d = 0; d < 3; ++d) s += ev[d] > 0 ? ev[d] * ev[d] : T(0);
    return s;
}
template <class T>
static T makePD2DNorm2(T a, T b, T d)
{
    T m = (a + d) / 2, r = std::sqrt((a - d) * (a - d) / 4 + b * b);
    T l0 = m - r, l1 = m + r;
    return (l0 > 0 ? l0 * l0 : T(0)) + (l1 > 0 ? l1 * l1 : T(0));
}

// StvkWithHenckyIsotropic::Bij (3D), StvkWithHenckyIsotropic.h:180-216:
// [[P+M, M-P], [M-P, P+M]] with P = B_Pij, M = B_Mij.
template <class T>
static void henckyBij(T mu, T lambda, const T s[3], int i, int j, T clamp, T& P, T& M)
{
    auto clampMag = [&](T x) {
        T mag = x > 0 ? x : -x;
        T sign = x > 0 ? T(1) : T(-1);
        return (mag > clamp ? mag : clamp) * sign;
    };
    T dE[3], ddE[3][3];
    henckyDiagonal(mu, lambda, s, dE, ddE);
    P = T(0.5) * (dE[i] + dE[j]) / clampMag(s[i] + s[j]);
    T L[3];
    for (int d = 0; d < 3; ++d) L[d] = std::log(std::fabs(s[d]));
    T sum_log = L[0] + L[1] + L[2];
    M = T(-0.5) * (lambda * sum_log + 2 * mu * diff_interlock_log_over_diff(s[i], s[j], L[j], T(1e-8))) / (s[i] * s[j]);
}

// VonMisesStvkHencky::projectSigma / projectSigmaAndDerivative,
// PlasticityApplier.cpp:526-602.
template <class T>
static bool vmProjectSigma(T mu, T ys, const T s[3], T out[3], T D[3][3])
{
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(s[d], T(1e-4)));
    T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    T hat_norm = std::sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    T delta_gamma = hat_norm - ys / (2 * mu);
    if (delta_gamma <= 0) {
        for (int r = 0; r < 3; ++r) {
            out[r] = s[r];
            for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
        }
        return false;
    }
    T w[3];
    for (int d = 0; d < 3; ++d) w[d] = 1 / s[d];
    T sv[3];
    for (int d = 0; d < 3; ++d) sv[d] = eps[d] - tr / 3 * T(1);
    T snorm = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    T sh[3];
    for (int d = 0; d < 3; ++d) sh[d] = sv[d] / snorm;
    for (int d = 0; d < 3; ++d) out[d] = std::exp(eps[d] - (delta_gamma / hat_norm) * hat[d]);
    T k1 = T(1) - ys / (2 * mu * snorm), k2 = ys / (2 * mu * snorm);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            T Iw = r == c ? w[c] : T(0);
            D[r][c] = out[r] * (Iw - k1 * (Iw - w[c] / T(3)) - k2 * sh[r] * sh[c] * w[c]);
        }
    return true;
}

// DruckerPragerStvkHencky::projectSigma, PlasticityApplier.cpp:319-347 (no
// log Jp: the ADMM local step's view of the return map).
template <class T>
static void dpProjectSigma(T mu, T lambda, T alpha, T cohesion, const T s[3], T out[3])
{
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(std::abs(s[d]), T(1e-4))) - cohesion;
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    if (tr >= 0) {
        for (int d = 0; d < 3; ++d) out[d] = std::exp(cohesion) * T(1);
        return;
    }
    const T hn = std::sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T dg = hn + (T(3) * lambda + T(2) * mu) / (T(2) * mu) * tr * alpha;
    for (int d = 0; d < 3; ++d) out[d] = std::exp((dg <= 0) ? eps[d] + cohesion : eps[d] - (dg / hn) * hat[d] + cohesion);
}

// DruckerPragerStvkHencky::projectSigmaAndDerivative, PlasticityApplier.cpp:387-423.
template <class T>
static void dpProjectSigmaDerivative(T mu, T lambda, T alpha, T cohesion, const T s[3], T out[3], T D[3][3])
{
    T eps[3];
    for (int d = 0; d < 3; ++d) eps[d] = std::log(std::max(std::abs(s[d]), T(1e-4))) - cohesion;
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    const T hn = std::sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T dg = hn + (T(3) * lambda + T(2) * mu) / (T(2) * mu) * tr * alpha;
    if (dg <= 0) { // inside the yield surface
        for (int r = 0; r < 3; ++r) {
            out[r] = std::exp(eps[r] + cohesion);
            for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
        }
        return;
    }
    if (tr > 0 || hn == 0) { // the tip
        for (int r = 0; r < 3; ++r) {
            out[r] = std::exp(cohesion) * T(1);
            for (int c = 0; c < 3; ++c) D[r][c] = T(0);
        }
        return;
    }
    T w[3], sv[3], sh[3];
    for (int d = 0; d < 3; ++d) {
        w[d] = T(1) / s[d];
        sv[d] = eps[d] - tr / T(3) * T(1);
    }
    const T sn = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    for (int d = 0; d < 3; ++d) sh[d] = sv[d] / sn;
    const T pp = alpha * tr * (T(3) * lambda + T(2) * mu) / (T(2) * mu * sn);
    for (int d = 0; d < 3; ++d) out[d] = std::exp(eps[d] - (dg / hn) * hat[d] + cohesion);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const T m1 = ((T(1) + T(2) * pp) / T(3) * T(1) - pp / tr * eps[r]) * w[c];
            const T m2 = pp * ((r == c ? T(1) : T(0)) - sh[r] * sh[c]) * w[c];
            D[r][c] = out[r] * (m1 - m2);
        }
}

// The viscous map in singular-value space and its derivative,
// AdmmSimulationFoam.h:583-595.
template <class T>
static void viscousSigma(const Visco<T>& v, T dt, const T zi[3], T zp[3], T D[3][3])
{
    T a, b;
    viscousCoefficients(v, dt, a, b);
    T et[3];
    for (int d = 0; d < 3; ++d) et[d] = std::log(std::fabs(zi[d]));
    T tr = et[0]; // epsilon_trial.trace() of a 3-vector, as in viscousReturn
    for (int d = 0; d < 3; ++d) zp[d] = std::exp(a * (et[d] - b * tr));
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) D[r][c] = zp[r] * a * ((r == c ? 1 / zi[c] : T(0)) - b * (1 / zi[c]));
}

template <class T>
static M3<T> inverse3(const M3<T>& A)
{
    M3<T> C = cofactor(A);
    T det = A.a[0][0] * C.a[0][0] + A.a[0][1] * C.a[0][1] + A.a[0][2] * C.a[0][2];
    M3<T> inv;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) inv.a[r][c] = C.a[c][r] / det;
    return inv;
}

// One strain of AdmmSimulation::FStepSolve (AdmmSimulationFoam.h:507-615):
// SVD of the target FDb, then a Newton solve in singular values for
// argmin vol psi(P(z)) + coeff/2 |z - sigma|^2 starting from the current F.
// mode 0: elastic, 1: von Mises projection, 2: viscous map, 3: Drucker-Prager
// projection (alpha = ys, cohesion).
template <class T>
static M3<T> admmLocalSolve(const M3<T>& FDb, const M3<T>& Fcur, T vol, T coeff, T mu, T lambda, int mode, T ys, const Visco<T>& vis,
    T dt, int iters, T tol, T cohesion = T(0))
{
    M3<T> U, V;
    T sigma[3];
    svd3(FDb, U, sigma, V);
    M3<T> W = Tmul(U, mul(Fcur, V));
    T zi[3] = { W.a[0][0], W.a[1][1], W.a[2][2] };
    for (int j = 0; j < iters; ++j) {
        T zp[3], D[3][3];
        if (mode == 1)
            vmProjectSigma(mu, ys, zi, zp, D);
        else if (mode == 3)
            dpProjectSigmaDerivative(mu, lambda, ys, cohesion, zi, zp, D);
        else if (mode == 2)
            viscousSigma(vis, dt, zi, zp, D);
        else
            for (int r = 0; r < 3; ++r) {
                zp[r] = zi[r];
                for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
            }
        T dE[3], ddE[3][3];
        henckyDiagonal(mu, lambda, zp, dE, ddE);
        T g[3];
        for (int d = 0; d < 3; ++d) g[d] = vol * dE[d] + coeff * (zi[d] - sigma[d]);
        M3<T> Pm;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                T acc = ddE[r][0] * D[0][c] + ddE[r][1] * D[1][c] + ddE[r][2] * D[2][c];
                Pm.a[r][c] = vol * acc + (r == c ? coeff : T(0));
            }
        M3<T> inv = inverse3(Pm);
        T step[3];
        for (int r = 0; r < 3; ++r) step[r] = inv.a[r][0] * (-g[0]) + inv.a[r][1] * (-g[1]) + inv.a[r][2] * (-g[2]);
        for (int d = 0; d < 3; ++d) zi[d] += step[d];
        if (std::sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]) < tol) break;
    }
    return udiagvt(U, zi, V);
}

// initOmega for one strain, AdmmSimulationFoam.h:236-270:
// omega = sqrt(vol sqrt(|makePD(d2E)|^2 + sum_ij |makePD2D(B_ij)|^2)).
template <class T>
static T admmOmega(const M3<T>& Fa, T vol, T mu, T lambda, bool vm, T ys, bool dp = false, T alpha = T(0), T cohesion = T(0))
{
    M3<T> U, V;
    T sigma[3];
    svd3(Fa, U, sigma, V);
    T dE[3], ddE[3][3];
    henckyDiagonal(mu, lambda, sigma, dE, ddE);
    M3<T> A;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) A.a[r][c] = ddE[r][c];
    T total = makePDNorm2(A);
    if (vm) {
        T sp[3], D[3][3];
        vmProjectSigma(mu, ys, sigma, sp, D);
        for (int d = 0; d < 3; ++d) sigma[d] = sp[d];
    }
    else if (dp) {
        T sp[3];
        dpProjectSigma(mu, lambda, alpha, cohesion, sigma, sp);
        for (int d = 0; d < 3; ++d) sigma[d] = sp[d];
    }
    const int pairs[3][2] = { { 0, 1 }, { 0, 2 }, { 1, 2 } };
    for (auto& pr : pairs) {
        T P, M;
        henckyBij(mu, lambda, sigma, pr[0], pr[1], T(1e-6), P, M);
        total += makePD2DNorm2(P + M, M - P, P + M);
    }
    return std::sqrt(vol * std::sqrt(total));
}

// ------------------------------------------------------------- colliders --
template <class T>
struct Collider {
    zmpm_collider d;
    // state at the current time (updateState)
    T R[3][3];
    T omega[3];
    T b[3], dbdt[3];
    T s = 1, dsdt = 0;

    void setRotation()
    {
        T w = (T)d.rotation[0], x = (T)d.rotation[1], y = (T)d.rotation[2], z = (T)d.rotation[3];
        T n = std::sqrt(w * w + x * x + y * y + z * z);
        if (n == 0) {
            w = 1;
            x = y = z = 0;
            n = 1;
        }
        w /= n;
        x /= n;
        y /= n;
        z /= n;
        R[0][0] = 1 - 2 * (y * y + z * z);
        R[0][1] = 2 * (x * y - w * z);
        R[0][2] = 2 * (x * z + w * y);
        R[1][0] = 2 * (x * y + w * z);
        R[1][1] = 1 - 2 * (x * x + z * z);
        R[1][2] = 2 * (y * z - w * x);
        R[2][0] = 2 * (x * z - w * y);
        R[2][1] = 2 * (y * z + w * x);
        R[2][2] = 1 - 2 * (x * x + y * y);
    }
    void update(double time)
    {
        setRotation();
        for (int i = 0; i < 3; ++i) {
            omega[i] = (T)d.angular_velocity[i];
            b[i] = (T)(d.translation[i] + time * d.translation_velocity[i]);
            dbdt[i] = (T)d.translation_velocity[i];
        }
        s = (T)(d.scale + time * d.scale_velocity);
        dsdt = (T)d.scale_velocity;
    }
    // AnalyticLevelSet::queryInside for the three shapes (AnalyticLevelSet.cpp:111-119, 272-287, 435-451, 504-539)
    bool queryInside(const T X[3], T N[3], T* phi_out = nullptr) const
    {
        if (d.shape == ZMPM_HALF_SPACE) {
            T n[3] = { (T)d.b[0], (T)d.b[1], (T)d.b[2] };
            T nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for (int i = 0; i < 3; ++i) n[i] /= nn;
            T phi = n[0] * (X[0] - (T)d.a[0]) + n[1] * (X[1] - (T)d.a[1]) + n[2] * (X[2] - (T)d.a[2]);
            if (phi <= 0) {
                if (phi_out) *phi_out = phi;
                for (int i = 0; i < 3; ++i) N[i] = n[i];
                return true;
            }
            return false;
        }
        if (d.shape == ZMPM_SPHERE) {
            T tc[3] = { X[0] - (T)d.a[0], X[1] - (T)d.a[1], X[2] - (T)d.a[2] };
            T d2 = tc[0] * tc[0] + tc[1] * tc[1] + tc[2] * tc[2];
            T r = (T)d.radius;
            if (d2 < r * r) {
                T dist = std::sqrt(d2);
                if (phi_out) *phi_out = dist - r;
                if (dist < T(1e-7)) {
                    N[0] = 1;
                    N[1] = N[2] = 0;
                }
                else
                    for (int i = 0; i < 3; ++i) N[i] = (1 / dist) * tc[i];
                return true;
            }
            return false;
        }
        // axis-aligned box: half edges h, centre c, signed distance
        // min(max_i d_i, 0) + |max(d, 0)| with d_i = |X_i - c_i| - h_i
        T h[3], ctr[3], xp[3], dd[3];
        for (int i = 0; i < 3; ++i) {
            h[i] = ((T)d.b[i] - (T)d.a[i]) / T(2);
            ctr[i] = ((T)d.a[i] + (T)d.b[i]) / T(2);
            xp[i] = X[i] - ctr[i];
            dd[i] = std::fabs(xp[i]) - h[i];
        }
        int imax = 0;
        for (int i = 1; i < 3; ++i)
            if (dd[i] > dd[imax]) imax = i;
        T q2 = 0;
        for (int i = 0; i < 3; ++i) {
            T q = dd[i] > 0 ? dd[i] : T(0);
            q2 += q * q;
        }
        T phi = std::min(dd[imax], T(0)) + std::sqrt(q2);
        if (phi > 0) return false;
        if (phi_out) *phi_out = phi;
        for (int i = 0; i < 3; ++i) N[i] = 0;
        N[imax] = xp[imax] >= 0 ? T(1) : T(-1);
        return true;
    }
    // AnalyticCollisionObject::queryInside (world space), CollisionObject.cpp:232-246
    bool queryInsideWorld(const T x[3], T& phi, T n[3]) const
    {
        T xb[3] = { x[0] - b[0], x[1] - b[1], x[2] - b[2] };
        T one_over_s = 1 / s;
        T X[3];
        for (int i = 0; i < 3; ++i) X[i] = (R[0][i] * xb[0] + R[1][i] * xb[1] + R[2][i] * xb[2]) * one_over_s;
        T N[3];
        if (!queryInside(X, N, &phi)) return false;
        for (int i = 0; i < 3; ++i) n[i] = R[i][0] * N[0] + R[i][1] * N[1] + R[i][2] * N[2];
        phi *= s;
        return true;
    }

    // AnalyticCollisionObject::getBoundaryVelocityAndNormal, CollisionObject.cpp:313-338
    bool boundaryVelocityAndNormal(const T x[3], T vb[3], T n[3]) const
    {
        if (d.type == ZMPM_GHOST) return false;
        T xb[3] = { x[0] - b[0], x[1] - b[1], x[2] - b[2] };
        T one_over_s = 1 / s;
        T X[3];
        for (int i = 0; i < 3; ++i) X[i] = (R[0][i] * xb[0] + R[1][i] * xb[1] + R[2][i] * xb[2]) * one_over_s;
        T N[3];
        if (!queryInside(X, N)) return false;
        vb[0] = omega[1] * xb[2] - omega[2] * xb[1];
        vb[1] = omega[2] * xb[0] - omega[0] * xb[2];
        vb[2] = omega[0] * xb[1] - omega[1] * xb[0];
        for (int i = 0; i < 3; ++i) vb[i] += (dsdt * one_over_s) * xb[i] + dbdt[i];
        for (int i = 0; i < 3; ++i) n[i] = R[i][0] * N[0] + R[i][1] * N[1] + R[i][2] * N[2];
        return true;
    }

    // AnalyticCollisionObject::detectAndResolveCollision, CollisionObject.cpp:340-400
    bool detectAndResolve(const T x[3], T v[3], T n[3]) const
    {
        if (d.type == ZMPM_GHOST) return false;
        T xb[3] = { x[0] - b[0], x[1] - b[1], x[2] - b[2] };
        T one_over_s = 1 / s;
        T X[3];
        for (int i = 0; i < 3; ++i) X[i] = (R[0][i] * xb[0] + R[1][i] * xb[1] + R[2][i] * xb[2]) * one_over_s;
        T N[3];
        if (!queryInside(X, N)) return false;
        T vo[3];
        vo[0] = omega[1] * xb[2] - omega[2] * xb[1];
        vo[1] = omega[2] * xb[0] - omega[0] * xb[2];
        vo[2] = omega[0] * xb[1] - omega[1] * xb[0];
        for (int i = 0; i < 3; ++i) vo[i] += (dsdt * one_over_s) * xb[i] + dbdt[i];
        for (int i = 0; i < 3; ++i) v[i] -= vo[i];
        if (d.type == ZMPM_STICKY) {
            v[0] = v[1] = v[2] = 0;
        }
        else {
            for (int i = 0; i < 3; ++i) n[i] = R[i][0] * N[0] + R[i][1] * N[1] + R[i][2] * N[2];
            T dot = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
            if (d.type == ZMPM_SLIP || dot < 0) {
                for (int i = 0; i < 3; ++i) v[i] -= n[i] * dot;
                T fr = (T)d.friction;
                if (fr != 0 && dot < 0) {
                    T vn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    if (-dot * fr < vn)
                        for (int i = 0; i < 3; ++i) v[i] += v[i] / vn * dot * fr;
                    else
                        v[0] = v[1] = v[2] = 0;
                }
            }
        }
        for (int i = 0; i < 3; ++i) v[i] += vo[i];
        return true;
    }
};

// AnalyticCollisionObject::multiObjectCollision, CollisionObject.cpp:66-105
template <class T>
static bool multiObjectCollision(const std::vector<Collider<T>>& objs, const T x[3], T v[3], M3<T>& K)
{
    bool any = false;
    int slip = 0;
    K = M3<T>::zero();
    for (const auto& o : objs) {
        if (o.d.type == ZMPM_GHOST) continue;
        T n[3] = { 0, 0, 0 };
        bool col = o.detectAndResolve(x, v, n);
        any = col || any;
        if (!col) continue;
        if (o.d.type == ZMPM_STICKY) {
            K = M3<T>::identity();
            break;
        }
        for (int c = 0; c < slip; ++c) {
            T dot = K.a[0][c] * n[0] + K.a[1][c] * n[1] + K.a[2][c] * n[2];
            for (int i = 0; i < 3; ++i) n[i] -= dot * K.a[i][c];
        }
        T len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (len) {
            for (int i = 0; i < 3; ++i) K.a[i][slip] = n[i] / len;
            if (++slip == 3) break;
        }
    }
    return any;
}

// ---------------------------------------------------------------- B-spline --
// Quadratic B-spline, BSplines.h:16-29,55-81, MathTools.h:15-25; the stencil
// loop order and products of MpmGrid::iterateKernel (MpmGrid.h:220-271).
static inline int int_floor(double x)
{
    int i = (int)x;
    return i - (i > x);
}
static inline int int_floor(float x)
{
    int i = (int)x;
    return i - (i > x);
}
template <class T>
struct Spline {
    T w[3][3], dw[3][3];
    int base[3];
    T one_over_dx;
    Spline(const T X[3], T dx)
    {
        one_over_dx = 1 / dx;
        for (int d = 0; d < 3; ++d) {
            T x = one_over_dx * X[d];
            base[d] = int_floor(x - T(0.5));
            T d0 = x - base[d];
            T z = T(1.5) - d0;
            w[d][0] = T(0.5) * z * z;
            T d1 = d0 - 1;
            w[d][1] = T(0.75) - d1 * d1;
            T d2 = 1 - d1;
            T zz = T(1.5) - d2;
            w[d][2] = T(0.5) * zz * zz;
            dw[d][0] = -z;
            dw[d][1] = -T(2) * d1;
            dw[d][2] = zz;
        }
    }
};

// ----------------------------------------------------------------- sim ----
template <class T>
struct Sim {
    using G = GridState<T>;
    Mask mask;
    double dx_d;
    T dx, gravity[3], apic_rpic_ratio, cfl;
    double time = 0;

    // particles, in the order they were added
    int64_t P = 0;
    std::vector<T> X, V, Cm, F, Fn, mass, vol;
    std::vector<Model<T>> model;
    std::vector<Plastic<T>> plastic;
    std::vector<Damage<T>> damage;
    std::vector<Visco<T>> visco;
    std::vector<T> Fe;                                   // Fe_Nonequilibrated [P][9]
    std::vector<T> admm_y, admm_omega, admm_last_dv;     // ADMM state carried across substeps: [P][18], [P][2], [P][3]
    std::vector<Scratch<T>> scratch;
    std::vector<M3<T>> gradV, stress;
    struct Checkpoint {
        std::vector<T> X, V, Cm, F, Fe, y, omega, lastdv;
        std::vector<Model<T>> model;
        std::vector<Plastic<T>> plastic;
        std::vector<Damage<T>> damage;
        double time = 0;
    };
    std::map<int, Checkpoint> checkpoints;
    std::vector<Collider<T>> colliders;

    // binning
    std::vector<u64> sorter, base_offset;
    std::vector<int32_t> order;
    std::vector<std::pair<int, int>> group;
    std::vector<u64> block_offset;
    std::vector<u64> blocks;
    VMem grid, pagemap;
    size_t pagemap_bytes = 0;
    int64_t N = 0;

    // Newton objective
    T dt = 0;
    std::vector<T> mvec, dv, vn; // [N], [N*3], [N*3]
    std::vector<uint8_t> collided;
    std::vector<M3<T>> proj;
    bool implicit_ready = false;
    std::string err;

    explicit Sim(int l2s) : mask(l2s) {}
    ~Sim()
    {
        grid.unmap();
        pagemap.unmap();
    }

    bool init(const zmpm_config& c)
    {
        dx_d = c.dx;
        dx = (T)c.dx;
        for (int d = 0; d < 3; ++d) gravity[d] = (T)c.gravity[d];
        apic_rpic_ratio = (T)c.apic_rpic_ratio;
        cfl = (T)c.cfl;
        // SPGrid allocator over 4096^3 nodes (MpmGrid.h:83-111)
        size_t elems = (size_t)1 << 36;
        if (!grid.map(elems * sizeof(G))) return false;
        pagemap_bytes = ((elems >> mask.block_bits) + 63) / 64 * 8;
        return pagemap.map(pagemap_bytes);
    }

    G& at(u64 offset) const { return *reinterpret_cast<G*>(reinterpret_cast<char*>(grid.p) + offset); }

    template <class F_>
    void iterateKernel(const Spline<T>& sp, u64 base, F_&& f) const
    {
        for (int i = 0; i < 3; ++i) {
            T wi = sp.w[0][i];
            T dwidxi = sp.one_over_dx * sp.dw[0][i];
            for (int j = 0; j < 3; ++j) {
                T wj = sp.w[1][j];
                T wij = wi * wj;
                T dwijdxi = dwidxi * wj;
                T dwijdxj = wi * sp.one_over_dx * sp.dw[1][j];
                for (int k = 0; k < 3; ++k) {
                    T wk = sp.w[2][k];
                    T wijk = wij * wk;
                    T dw[3] = { dwijdxi * wk, dwijdxj * wk, wij * sp.one_over_dx * sp.dw[2][k] };
                    int node[3] = { sp.base[0] + i, sp.base[1] + j, sp.base[2] + k };
                    G& g = at(mask.packed_add(base, mask.stencil[9 * i + 3 * j + k]));
                    f(node, wijk, dw, g);
                }
            }
        }
    }

    // iterateGrid / iterateTouchedGrid, MpmGrid.h:139-218
    template <class F_>
    void iterateBlocks(bool active_only, F_&& f)
    {
        const int bxn = mask.bx(), byn = mask.by(), bzn = mask.bz();
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < (int64_t)blocks.size(); ++b) {
            u64 base = blocks[b];
            int bc[3];
            mask.coord(base, bc);
            for (int i = 0; i < bxn; ++i)
                for (int j = 0; j < byn; ++j)
                    for (int k = 0; k < bzn; ++k) {
                        G& g = at(mask.packed_add(base, mask.linear_offset(i, j, k)));
                        if (active_only && g.idx < 0) continue;
                        int node[3] = { bc[0] + i, bc[1] + j, bc[2] + k };
                        f(node, g);
                    }
        }
    }

    // --------------------------------------------------------- binning --
    // MpmSimulationBase::sortParticlesAndPolluteGrid, MpmSimulationBase.cpp:1032-1103
    int sortParticlesAndPolluteGrid()
    {
        const int index_bits = 32 - mask.block_bits;
        if (P >= ((int64_t)1 << index_bits)) {
            err = "too many particles for the key encoding";
            return ZMPM_BAD_ARG;
        }
        sorter.resize(P);
        base_offset.resize(P);
        order.resize(P);
        T one_over_dx = T(1) / dx;
        int bad = 0;
#pragma omp parallel for reduction(| : bad)
        for (int64_t i = 0; i < P; ++i) {
            int b[3];
            for (int d = 0; d < 3; ++d) b[d] = int_floor(X[3 * i + d] * one_over_dx - T(0.5));
            for (int d = 0; d < 3; ++d) bad |= (b[d] < 0 || b[d] > 4096 - 16);
            u64 off = mask.linear_offset(b[0], b[1], b[2]);
            sorter[i] = ((off >> mask.log2_struct) << index_bits) + (u64)i;
        }
        if (bad) {
            err = "particle outside the SPGrid domain";
            return ZMPM_OUT_OF_GRID;
        }
        __gnu_parallel::sort(sorter.begin(), sorter.end());
        group.clear();
        block_offset.clear();
        int last = 0;
        for (int64_t i = 0; i < P; ++i)
            if (i == P - 1 || (sorter[i] >> 32) != (sorter[i + 1] >> 32)) {
                group.emplace_back(last, (int)i);
                block_offset.push_back(sorter[i] >> 32);
                last = (int)i + 1;
            }
        // page map: Clear re-maps the bitmap (SPGrid_Page_Map.h:38-43)
        pagemap.unmap();
        if (!pagemap.map(pagemap_bytes)) return ZMPM_NO_MEMORY;
        blocks.clear();
        u64* pm = static_cast<u64*>(pagemap.p);
        auto set_page = [&](u64 off) { // Set_Page, SPGrid_Page_Map.h:61-70
            u64 m = 1ull << ((off >> 12) & 0x3f);
            u64& e = pm[off >> 18];
            if (m & ~e) {
                e |= m;
                blocks.push_back((off >> 12) << 12);
            }
        };
        const int bxn = mask.bx(), byn = mask.by(), bzn = mask.bz();
        for (int64_t i = 0; i < P; ++i) {
            order[i] = (int32_t)(sorter[i] & ((1ull << index_bits) - 1));
            u64 off = (sorter[i] >> index_bits) << mask.log2_struct;
            base_offset[order[i]] = off;
            if (i == P - 1 || (sorter[i] >> 32) != (sorter[i + 1] >> 32)) {
                set_page(off);
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        for (int c = 0; c < 2; ++c) set_page(mask.packed_add(off, mask.linear_offset(bxn * a, byn * b, bzn * c)));
            }
        }
        const int epb = mask.elements();
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < (int64_t)blocks.size(); ++b) {
            G* g = &at(blocks[b]);
            std::memset(g, 0, 4096);
            for (int e = 0; e < epb; ++e) g[e].idx = -1;
        }
        return ZMPM_OK;
    }

    // MpmGrid::getNumNodes, MpmGrid.h:123-136
    int64_t getNumNodes()
    {
        int64_t n = 0;
        const int epb = mask.elements();
        for (size_t b = 0; b < blocks.size(); ++b) {
            G* g = &at(blocks[b]);
            for (int e = 0; e < epb; ++e)
                if (g[e].m != 0) g[e].idx = n++;
        }
        return n;
    }

    template <class F_>
    void coloredGroups(F_&& f)
    {
        for (u64 color = 0; color < 8; ++color) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t gi = 0; gi < (int64_t)group.size(); ++gi) {
                if ((block_offset[gi] & 7) != color) continue;
                for (int idx = group[gi].first; idx <= group[gi].second; ++idx) f(order[idx]);
            }
        }
    }

    // ------------------------------------------------------------- P2G --
    // particlesToGridHelper<APIC,deg2>, MpmSimulationBase.cpp:563-608, and the
    // normalisation of particlesToGrid, :474-485
    void particlesToGrid()
    {
        coloredGroups([&](int i) {
            const T* Xp = &X[3 * i];
            T m = mass[i];
            T mom[3] = { m * V[3 * i], m * V[3 * i + 1], m * V[3 * i + 2] };
            T C[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) C[r][c] = m * Cm[9 * i + 3 * r + c];
            Spline<T> sp(Xp, dx);
            iterateKernel(sp, base_offset[i], [&](const int node[3], T w, const T*, G& g) {
                T xi[3];
                for (int d = 0; d < 3; ++d) xi[d] = node[d] * dx - Xp[d];
                for (int r = 0; r < 3; ++r) g.v[r] += (C[r][0] * xi[0] + C[r][1] * xi[1] + C[r][2] * xi[2] + mom[r]) * w;
                g.m += m * w;
            });
        });
        N = getNumNodes();
        iterateBlocks(true, [&](const int*, G& g) {
            for (int d = 0; d < 3; ++d) g.v[d] /= g.m;
        });
    }

    // ----------------------------------------------------- Newton setup --
    // startBackwardEuler + buildMassMatrix + buildInitialDvAndVnForNewton,
    // MpmSimulationBase.cpp:610-633, 793-802, 1105-1136
    void startBackwardEuler()
    {
        mvec.assign(N, 0);
        dv.assign(3 * N, 0);
        vn.assign(3 * N, 0);
        collided.assign(N, 0);
        proj.assign(N, M3<T>::identity());
        for (auto& c : colliders) c.update(time);
        iterateBlocks(true, [&](const int node[3], G& g) {
            int64_t id = g.idx;
            mvec[id] = g.m;
            T vi[3] = { g.v[0], g.v[1], g.v[2] };
            T xi[3] = { node[0] * dx, node[1] * dx, node[2] * dx };
            M3<T> K;
            bool any = multiObjectCollision(colliders, xi, vi, K);
            if (any) {
                collided[id] = 1;
                M3<T> P = M3<T>::identity();
                M3<T> KK = mulT(K, K);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) P.a[r][c] -= KK.a[r][c];
                proj[id] = P;
                for (int d = 0; d < 3; ++d) dv[3 * id + d] = vi[d] - g.v[d];
            }
            else
                for (int d = 0; d < 3; ++d) dv[3 * id + d] = gravity[d] * dt;
            for (int d = 0; d < 3; ++d) vn[3 * id + d] = g.v[d];
        });
        Fn = F; // backupStrain
        implicit_ready = true;
    }

    void project(std::vector<T>& v) const
    {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            if (!collided[i]) continue;
            const M3<T>& Pm = proj[i];
            T a = v[3 * i], b = v[3 * i + 1], c = v[3 * i + 2];
            for (int r = 0; r < 3; ++r) v[3 * i + r] = Pm.a[r][0] * a + Pm.a[r][1] * b + Pm.a[r][2] * c;
        }
    }

    // evalInterpolantAndGradient, MpmForceBase.cpp:213-244 (gradient only;
    // the interpolated value is not used on the implicit path)
    void evalGradient(const std::vector<T>& field, bool add_vn, std::vector<M3<T>>& grad)
    {
        iterateBlocks(false, [&](const int*, G& g) {
            g.new_v[0] = g.new_v[1] = g.new_v[2] = 0;
        });
        iterateBlocks(true, [&](const int*, G& g) {
            int64_t id = g.idx;
            for (int d = 0; d < 3; ++d) g.new_v[d] = (add_vn ? vn[3 * id + d] : T(0)) + field[3 * id + d];
        });
        grad.resize(P);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            M3<T> gr = M3<T>::zero();
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T, const T* dw, G& g) {
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) gr.a[r][c] += g.new_v[r] * dw[c];
            });
            grad[i] = gr;
        }
    }

    // rasterizeForceToTVStack<false>, MpmForceBase.cpp:102-152
    void rasterize(T scale, const std::vector<M3<T>>& S, std::vector<T>& out)
    {
        iterateBlocks(true, [&](const int*, G& g) {
            g.new_v[0] = g.new_v[1] = g.new_v[2] = 0;
        });
        coloredGroups([&](int i) {
            const M3<T>& s = S[i];
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T, const T* dw, G& g) {
                for (int r = 0; r < 3; ++r) {
                    T delta = s.a[r][0] * dw[0] + s.a[r][1] * dw[1] + s.a[r][2] * dw[2];
                    g.new_v[r] -= scale * delta;
                }
            });
        });
        iterateBlocks(true, [&](const int*, G& g) {
            for (int d = 0; d < 3; ++d) out[3 * g.idx + d] += g.new_v[d];
        });
    }

    // updateState -> MpmForceBase::updatePositionBasedState, MpmForceBase.cpp:306-344
    // (G2P of vn+dv, F=(I+dt gradV)Fn, scratch, stress V0 P Fn^T)
    void updateState(const std::vector<T>& dvin)
    {
        evalGradient(dvin, true, gradV);
        stress.resize(P);
        scratch.resize(P);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            M3<T> Fnp = load9(Fn, i);
            M3<T> A = M3<T>::identity();
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A.a[r][c] += dt * gradV[i].a[r][c];
            M3<T> Fp = mul(A, Fnp);
            store9(F, i, Fp);
            if (model[i].kind == ZMPM_MODEL_NONE) {
                stress[i] = M3<T>::zero();
                continue;
            }
            updateScratch(model[i], Fp, scratch[i]);
            M3<T> Pp = firstPiola(model[i], scratch[i]);
            stress[i] = mulT(scaled(Pp, vol[i]), Fnp);
        }
    }

    // computeResidual + computeNorm, BackwardEuler.h:101-140
    T computeResidual(std::vector<T>& r)
    {
        r.assign(3 * N, 0);
        for (int64_t i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) r[3 * i + d] = dt * gravity[d] * mvec[i];
        rasterize(dt, stress, r);
        for (int64_t i = 0; i < N; ++i) // MassLumpedInertia::addScaledForces, Inertia.cpp:32-41
            for (int d = 0; d < 3; ++d) r[3 * i + d] -= (dt / dt) * mvec[i] * dv[3 * i + d];
        project(r);
        return computeNorm(r);
    }

    T reduce(const std::function<T(int64_t)>& term) const
    {
        const int64_t chunk = 256;
        int64_t nch = (N + chunk - 1) / chunk;
        std::vector<T> part(nch, 0);
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nch; ++c) {
            T s = 0;
            for (int64_t i = c * chunk; i < std::min(N, (c + 1) * chunk); ++i) s += term(i);
            part[c] = s;
        }
        T s = 0;
        for (T v : part) s += v;
        return s;
    }
    T computeNorm(const std::vector<T>& r) const
    {
        return std::sqrt(reduce([&](int64_t i) {
            return (r[3 * i] * r[3 * i] + r[3 * i + 1] * r[3 * i + 1] + r[3 * i + 2] * r[3 * i + 2]) / mvec[i];
        }));
    }
    T dot(const std::vector<T>& a, const std::vector<T>& b) const
    {
        return reduce([&](int64_t i) { return a[3 * i] * b[3 * i] + a[3 * i + 1] * b[3 * i + 1] + a[3 * i + 2] * b[3 * i + 2]; });
    }

    // multiply, BackwardEuler.h:322-351: b = M x + dt^2 sum dS grad w
    int64_t hvp_count = 0;
    bool admm_mode = false;
    void multiply(const std::vector<T>& x, std::vector<T>& b)
    {
        if (admm_mode) {
            admmMultiply(x, b);
            return;
        }
        hvp_count++;
        b.assign(3 * N, 0);
        T scale = -(dt * dt);
        T iscale = scale / (dt * dt);
        for (int64_t i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) b[3 * i + d] -= iscale * mvec[i] * x[3 * i + d];
        std::vector<M3<T>> gdv;
        evalGradient(x, false, gdv);
        std::vector<M3<T>> dS(P);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            if (model[i].kind == ZMPM_MODEL_NONE) {
                dS[i] = M3<T>::zero();
                continue;
            }
            M3<T> Fnp = load9(Fn, i);
            M3<T> dP = firstPiolaDifferential(model[i], scratch[i], mul(gdv[i], Fnp));
            dS[i] = mulT(scaled(dP, vol[i]), Fnp);
        }
        rasterize(scale, dS, b);
    }
    void precondition(const std::vector<T>& in, std::vector<T>& out) const
    {
        const std::vector<T>& pre = admm_mode ? admm_pre : mvec;
        out.resize(3 * N);
        for (int64_t i = 0; i < N; ++i)
            for (int d = 0; d < 3; ++d) out[3 * i + d] = in[3 * i + d] / pre[i];
    }

    // Minres::solve, Minres.h:69-149.  Newton's solves start from x = 0, so
    // A x = 0 is not evaluated; `warm` starts from the given x (ADMM's dvStep).
    int minres(std::vector<T>& x, const std::vector<T>& b, T rel_tol, T abs_tol, int max_it, bool warm = false)
    {
        std::vector<T> mk(3 * N, 0), mkm1(3 * N, 0), mkm2(3 * N, 0), z(3 * N, 0), qkm1(3 * N, 0), qk(3 * N, 0), qkp1;
        T g_c[3] = { 1, 1, 1 }, g_s[3] = { 0, 0, 0 }; // Gk, Gkm1, Gkm2
        T gamma = 0, delta = 0, epsilon = 0, beta_kp1 = 0, alpha_k = 0, beta_k = 0, tk = 0;
        if (warm) {
            multiply(x, qkp1);
            for (int64_t i = 0; i < 3 * N; ++i) qkp1[i] = b[i] - qkp1[i];
        }
        else
            qkp1 = b;
        project(qkp1);
        precondition(qkp1, z);
        T rnorm = std::sqrt(dot(z, qkp1));
        beta_kp1 = rnorm;
        T local_tol = std::min(rel_tol * rnorm, abs_tol);
        if (rnorm < local_tol) return 0;
        if (rnorm > 0)
            for (int64_t i = 0; i < 3 * N; ++i) {
                qkp1[i] /= beta_kp1;
                z[i] /= beta_kp1;
            }
        T rhs0 = rnorm, rhs1 = 0;
        for (int k = 0; k < max_it; ++k) {
            if (rnorm < local_tol) return k;
            mkm2.swap(mkm1);
            mkm1.swap(mk);
            mk = z;
            beta_k = beta_kp1;
            qkm1.swap(qkp1);
            qkm1.swap(qk);
            multiply(mk, qkp1);
            project(qkp1);
            alpha_k = dot(mk, qkp1);
            for (int64_t i = 0; i < 3 * N; ++i) qkp1[i] -= alpha_k * qk[i];
            for (int64_t i = 0; i < 3 * N; ++i) qkp1[i] -= beta_k * qkm1[i];
            precondition(qkp1, z);
            beta_kp1 = std::sqrt(std::max(T(0), dot(z, qkp1)));
            if (beta_kp1 > 0)
                for (int64_t i = 0; i < 3 * N; ++i) {
                    qkp1[i] /= beta_kp1;
                    z[i] /= beta_kp1;
                }
            // applyAllPreviousGivensRotationsAndDetermineNewGivens, Minres.h:151-175
            g_c[2] = g_c[1];
            g_s[2] = g_s[1];
            g_c[1] = g_c[0];
            g_s[1] = g_s[0];
            T e0 = 0, e1 = beta_k; // Gkm2 row rotation of (0, beta_k)
            {
                T t1 = e0, t2 = e1;
                e0 = g_c[2] * t1 - g_s[2] * t2;
                e1 = g_s[2] * t1 + g_c[2] * t2;
            }
            epsilon = e0;
            T d0 = e1, d1 = alpha_k;
            {
                T t1 = d0, t2 = d1;
                d0 = g_c[1] * t1 - g_s[1] * t2;
                d1 = g_s[1] * t1 + g_c[1] * t2;
            }
            delta = d0;
            T t0 = d1, tt1 = beta_kp1;
            {
                Givens<T> G(0, 1);
                G.compute(t0, tt1);
                g_c[0] = G.c;
                g_s[0] = G.s;
            }
            {
                T a1 = t0, a2 = tt1;
                t0 = g_c[0] * a1 - g_s[0] * a2;
            }
            gamma = t0;
            {
                T a1 = rhs0, a2 = rhs1;
                rhs0 = g_c[0] * a1 - g_s[0] * a2;
                rhs1 = g_s[0] * a1 + g_c[0] * a2;
            }
            tk = rhs0;
            T residual = rhs1;
            rhs0 = residual;
            rhs1 = 0;
            rnorm = residual < 0 ? -residual : residual;
            for (int64_t i = 0; i < 3 * N; ++i) mk[i] = (mk[i] - delta * mkm1[i] - epsilon * mkm2[i]) / gamma;
            for (int64_t i = 0; i < 3 * N; ++i) x[i] += tk * mk[i];
        }
        return max_it;
    }

    // ConjugateGradient::solve, ConjugateGradient.h:99-147 (x starts at zero)
    int cg(std::vector<T>& x, const std::vector<T>& b, T rel_tol, T abs_tol, int max_it)
    {
        std::vector<T> r = b, q, p, temp;
        project(r);
        precondition(r, q);
        p = q;
        T zTrk = dot(r, q);
        T rnorm = std::sqrt(zTrk);
        T local_tol = std::min(rel_tol * rnorm, abs_tol);
        for (int cnt = 0; cnt < max_it; ++cnt) {
            if (rnorm < local_tol) return cnt;
            multiply(p, temp);
            project(temp);
            T alpha = zTrk / dot(temp, p);
            for (int64_t i = 0; i < 3 * N; ++i) {
                x[i] += p[i] * alpha;
                r[i] -= temp[i] * alpha;
            }
            precondition(r, q);
            T zTrk_last = zTrk;
            zTrk = dot(q, r);
            T beta = zTrk / zTrk_last;
            for (int64_t i = 0; i < 3 * N; ++i) p[i] = q[i] + beta * p[i];
            rnorm = std::sqrt(zTrk);
        }
        return max_it;
    }

    // NewtonsMethod::solve, NewtonsMethod.h:42-66
    bool newton(const zmpm_solver& s, zmpm_stats& st)
    {
        std::vector<T> r, step;
        bool first = true;
        for (int it = 0; it < s.newton_max_iterations; ++it) {
            updateState(dv);
            T rn = computeResidual(r);
            if (first) st.newton_residual_initial = (double)rn;
            first = false;
            st.newton_residual_final = (double)rn;
            if (!(rn == rn)) st.status_flags |= 1;
            if (rn < (T)s.newton_tolerance) return true;
            T rel = std::min(T(0.5), (T)s.linear_solve_tolerance_scale * std::sqrt(std::max(rn, (T)s.newton_tolerance)));
            step.assign(3 * N, 0);
            int k = (s.linear_solver == ZMPM_CG)
                ? cg(step, r, rel, (T)s.krylov_tolerance, s.krylov_max_iterations)
                : minres(step, r, rel, (T)s.krylov_tolerance, s.krylov_max_iterations);
            st.krylov_iterations += k;
            st.newton_iterations += 1;
            for (int64_t i = 0; i < 3 * N; ++i) dv[i] += step[i];
        }
        return false;
    }

    // --------------------------------------------------------- adjoint --
    // Reverse mode of one implicit substep (no reference counterpart).  With
    // v* = vn + dv the converged Newton solution of
    //   G(v*) = M v* - q - dt M g + dt sum_p V0 P(F_p) Fn_p^T grad w_ip = 0 (free nodes),
    //   F_p = (I + dt sum_j v*_j grad w_jp^T) Fn_p,  q_i = sum_p w_ip m_p (v_p + C_p (x_i - x_p)),
    // the implicit function theorem gives dL/dtheta = -lambda^T dG/dtheta with
    // (M + dt^2 K) lambda = P dL/dv* (the Newton Hessian, projected).  Binning
    // (base nodes) is held fixed.

    // Weights, gradients and Hessians of the quadratic B-spline stencil.
    template <class F_>
    void iterateKernel2(const Spline<T>& sp, u64 base, F_&& f) const
    {
        const T idx = sp.one_over_dx, idx2 = sp.one_over_dx * sp.one_over_dx;
        const T dd[3] = { T(1), T(-2), T(1) };
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    T Nx = sp.w[0][i], Ny = sp.w[1][j], Nz = sp.w[2][k];
                    T Dx = sp.dw[0][i], Dy = sp.dw[1][j], Dz = sp.dw[2][k];
                    T w = Nx * Ny * Nz;
                    T dw[3] = { Dx * Ny * Nz * idx, Nx * Dy * Nz * idx, Nx * Ny * Dz * idx };
                    T H[3][3];
                    H[0][0] = dd[i] * Ny * Nz * idx2;
                    H[1][1] = Nx * dd[j] * Nz * idx2;
                    H[2][2] = Nx * Ny * dd[k] * idx2;
                    H[0][1] = H[1][0] = Dx * Dy * Nz * idx2;
                    H[0][2] = H[2][0] = Dx * Ny * Dz * idx2;
                    H[1][2] = H[2][1] = Nx * Dy * Dz * idx2;
                    int node[3] = { sp.base[0] + i, sp.base[1] + j, sp.base[2] + k };
                    G& g = at(mask.packed_add(base, mask.stencil[9 * i + 3 * j + k]));
                    f(node, w, dw, H, g);
                }
    }

    static T youngsModulus(const Model<T>& c)
    {
        if (c.kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
            T lam = c.kappa - T(0.666666) * c.mu;
            return c.mu * (3 * lam + 2 * c.mu) / (lam + c.mu);
        }
        return c.mu * (3 * c.lambda + 2 * c.mu) / (c.lambda + c.mu);
    }

    int adjointSubstep(double dt_in, const zmpm_solver& s, double tol, double* gx, double* gv, double* gC, double* gF, double* gE,
        zmpm_stats& st)
    {
        for (int64_t i = 0; i < P; ++i) {
            const bool vm = plastic[i].kind == ZMPM_PLASTIC_VON_MISES && plastic[i].xi == 0 && model[i].kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC;
            if ((plastic[i].kind != ZMPM_PLASTIC_NONE && !vm) || damage[i].kind != ZMPM_DAMAGE_NONE || visco[i].on) {
                err = "the adjoint supports elastic particles and von Mises (StvkWithHenckyIsotropic, xi = 0) only";
                return ZMPM_UNSUPPORTED;
            }
        }
        if (s.integrator != ZMPM_NEWTON) {
            err = "the adjoint differentiates the Newton substep";
            return ZMPM_UNSUPPORTED;
        }
        const std::vector<T> X0 = X, V0v = V, C0 = Cm, F0 = F;
        int rc = substep(dt_in, s, st);
        if (rc != ZMPM_OK && rc != ZMPM_CFL_VIOLATION) return rc;
        // the operators below evaluate at the pre-substep positions; keep s_{n+1}
        const std::vector<T> X1 = X, F1 = F;
        X = X0;
        // the Hessian and stresses at the converged solution
        updateState(dv);
        const T dtt = dt;
        std::vector<T> vstar(3 * N);
        for (int64_t n = 0; n < N; ++n)
            for (int d = 0; d < 3; ++d) vstar[3 * n + d] = vn[3 * n + d] + dv[3 * n + d];
        auto in3 = [&](const double* a, int64_t i, int d) { return a ? (T)a[3 * i + d] : T(0); };
        auto in9 = [&](const double* a, int64_t i) {
            M3<T> m = M3<T>::zero();
            if (a)
                for (int q = 0; q < 9; ++q) m.a[q / 3][q % 3] = (T)a[9 * i + q];
            return m;
        };
        const T D_inv = 4 / (dx * dx);
        std::vector<T> xbar(3 * P), vbar(3 * P, 0), Cbar(9 * P, 0), Fbar(9 * P, 0);
        // (1) G2P: v_p' = sum w v*, C_p' = D^-1 sum w v* (x_i - x_p)^T,
        //     F_p' = (I + dt grad v*) Fn, x_p' = x_p + dt v_p'
        std::vector<T> vsbar(3 * N, 0);
        coloredGroups([&](int i) {
            const T* xp = &X0[3 * i];
            T vt[3], xb[3];
            for (int d = 0; d < 3; ++d) {
                vt[d] = in3(gv, i, d) + dtt * in3(gx, i, d);
                xb[d] = in3(gx, i, d);
            }
            M3<T> Cb = in9(gC, i), Fb = in9(gF, i), Fn_ = load9(F0, i);
            Spline<T> sp(xp, dx);
            if (plastic[i].kind == ZMPM_PLASTIC_VON_MISES) {
                // the projection's input Fp = (I + dt grad v*) Fn
                M3<T> Ap = M3<T>::identity();
                iterateKernel2(sp, base_offset[i], [&](const int*, T, const T* dw, const T (*)[3], G& g) {
                    if (g.idx < 0) return;
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) Ap.a[r][c] += dtt * vstar[3 * g.idx + r] * dw[c];
                });
                T gEp = 0;
                Fb = vonMisesAdjoint(model[i], plastic[i], mul(Ap, Fn_), Fb, gEp);
                if (gE) gE[i] += (double)gEp;
            }
            M3<T> FnFbT = mulT(Fn_, Fb); // Fn gF^T
            M3<T> gvs = M3<T>::zero();
            iterateKernel2(sp, base_offset[i], [&](const int node[3], T w, const T* dw, const T H[3][3], G& g) {
                const int64_t id = g.idx;
                if (id < 0) return;
                const T* v = &vstar[3 * id];
                T xi[3];
                for (int d = 0; d < 3; ++d) xi[d] = node[d] * dx - xp[d];
                // Fb Fn^T grad w
                T fd[3], cx[3];
                for (int r = 0; r < 3; ++r) {
                    fd[r] = 0;
                    cx[r] = 0;
                    for (int c = 0; c < 3; ++c) {
                        T FbFnT = Fb.a[r][0] * Fn_.a[c][0] + Fb.a[r][1] * Fn_.a[c][1] + Fb.a[r][2] * Fn_.a[c][2];
                        fd[r] += FbFnT * dw[c];
                        cx[r] += Cb.a[r][c] * xi[c];
                    }
                }
                for (int d = 0; d < 3; ++d) vsbar[3 * id + d] += w * vt[d] + D_inv * w * cx[d] + dtt * fd[d];
                T vdot = v[0] * vt[0] + v[1] * vt[1] + v[2] * vt[2];
                T vCx = v[0] * cx[0] + v[1] * cx[1] + v[2] * cx[2];
                T CTv[3], q[3];
                for (int c = 0; c < 3; ++c) CTv[c] = Cb.a[0][c] * v[0] + Cb.a[1][c] * v[1] + Cb.a[2][c] * v[2];
                for (int r = 0; r < 3; ++r) q[r] = FnFbT.a[r][0] * v[0] + FnFbT.a[r][1] * v[1] + FnFbT.a[r][2] * v[2];
                for (int d = 0; d < 3; ++d) {
                    xb[d] += vdot * dw[d] + D_inv * (vCx * dw[d] - w * CTv[d]);
                    xb[d] += dtt * (H[d][0] * q[0] + H[d][1] * q[1] + H[d][2] * q[2]);
                }
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) gvs.a[r][c] += v[r] * dw[c];
            });
            M3<T> A = M3<T>::identity();
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A.a[r][c] += dtt * gvs.a[r][c];
            store9(Fbar, i, Tmul(A, Fb));
            for (int d = 0; d < 3; ++d) xbar[3 * i + d] = xb[d];
        });
        // (2) adjoint solve (M + dt^2 K) lambda = P vsbar, CG with the Newton operator
        project(vsbar);
        std::vector<T> lam(3 * N, 0);
        int kit = cg(lam, vsbar, (T)tol, T(1e300), 100000);
        st.krylov_iterations += kit;
        // (3) grid adjoints: qbar = lambda, mbar = -lambda . (v* - dt g)
        std::vector<T> mbar(N);
        for (int64_t n = 0; n < N; ++n) {
            T a = 0;
            for (int d = 0; d < 3; ++d) a += lam[3 * n + d] * (vstar[3 * n + d] - dtt * gravity[d]);
            mbar[n] = -a;
        }
        // (4) particle adjoints of the force term, of P2G and of E
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            const T* xp = &X0[3 * i];
            Spline<T> sp(xp, dx);
            M3<T> Lam = M3<T>::zero(), Vs = M3<T>::zero();
            iterateKernel2(sp, base_offset[i], [&](const int*, T, const T* dw, const T (*)[3], G& g) {
                if (g.idx < 0) return;
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) {
                        Lam.a[r][c] += lam[3 * g.idx + r] * dw[c];
                        Vs.a[r][c] += vstar[3 * g.idx + r] * dw[c];
                    }
            });
            M3<T> Fn_ = load9(F0, i);
            M3<T> Fb = load9(Fbar, i);
            T xb[3] = { xbar[3 * i], xbar[3 * i + 1], xbar[3 * i + 2] };
            T vb[3] = { 0, 0, 0 };
            M3<T> Cb = M3<T>::zero();
            if (model[i].kind != ZMPM_MODEL_NONE) {
                M3<T> A = M3<T>::identity();
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) A.a[r][c] += dtt * Vs.a[r][c];
                M3<T> Fp = mul(A, Fn_);
                Scratch<T> sc;
                updateScratch(model[i], Fp, sc);
                M3<T> Pp = firstPiola(model[i], sc);
                M3<T> LF = mul(Lam, Fn_);
                M3<T> dPL = firstPiolaDifferential(model[i], sc, LF);
                T c0 = dtt * vol[i];
                M3<T> t1 = Tmul(A, dPL), t2 = Tmul(Lam, Pp);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) Fb.a[r][c] -= c0 * (t1.a[r][c] + t2.a[r][c]);
                if (gE) gE[i] -= (double)(c0 * contract(Pp, LF) / youngsModulus(model[i]));
                M3<T> Q1 = mulT(dPL, Fn_), Q2 = mulT(Pp, Fn_);
                iterateKernel2(sp, base_offset[i], [&](const int*, T, const T*, const T H[3][3], G& g) {
                    if (g.idx < 0) return;
                    const T* v = &vstar[3 * g.idx];
                    const T* l = &lam[3 * g.idx];
                    T a[3], b[3];
                    for (int c = 0; c < 3; ++c) {
                        a[c] = Q1.a[0][c] * v[0] + Q1.a[1][c] * v[1] + Q1.a[2][c] * v[2];
                        b[c] = Q2.a[0][c] * l[0] + Q2.a[1][c] * l[1] + Q2.a[2][c] * l[2];
                    }
                    for (int d = 0; d < 3; ++d)
                        xb[d] -= c0 * (dtt * (H[d][0] * a[0] + H[d][1] * a[1] + H[d][2] * a[2]) + (H[d][0] * b[0] + H[d][1] * b[1] + H[d][2] * b[2]));
                });
            }
            // P2G: q_i = sum w m (v + C (x_i - x_p)), m_i = sum w m
            const T mp = mass[i];
            M3<T> Cp = load9(C0, i);
            const T* vp = &V0v[3 * i];
            iterateKernel2(sp, base_offset[i], [&](const int node[3], T w, const T* dw, const T (*)[3], G& g) {
                if (g.idx < 0) return;
                const T* l = &lam[3 * g.idx];
                T xi[3];
                for (int d = 0; d < 3; ++d) xi[d] = node[d] * dx - xp[d];
                T u[3];
                for (int r = 0; r < 3; ++r) u[r] = vp[r] + Cp.a[r][0] * xi[0] + Cp.a[r][1] * xi[1] + Cp.a[r][2] * xi[2];
                T lu = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
                for (int d = 0; d < 3; ++d) {
                    vb[d] += w * mp * l[d];
                    T CTl = Cp.a[0][d] * l[0] + Cp.a[1][d] * l[1] + Cp.a[2][d] * l[2];
                    xb[d] += mp * lu * dw[d] - w * mp * CTl + mbar[g.idx] * mp * dw[d];
                }
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) Cb.a[r][c] += w * mp * l[r] * xi[c];
            });
            for (int d = 0; d < 3; ++d) {
                if (gx) gx[3 * i + d] = (double)xb[d];
                if (gv) gv[3 * i + d] = (double)vb[d];
            }
            for (int q = 0; q < 9; ++q) {
                if (gC) gC[9 * i + q] = (double)Cb.a[q / 3][q % 3];
                if (gF) gF[9 * i + q] = (double)Fb.a[q / 3][q % 3];
            }
        }
        X = X1;
        F = F1;
        return rc;
    }

    // ------------------------------------------------------------ ADMM --
    // AdmmSimulation (Projects/admm/AdmmSimulationFoam.h).  Strain slot 0 is F
    // with the particle's Hencky model (and von Mises projection if it has
    // one), slot 1 is Fe with its StvkWithHencky model (viscoelastic particles).
    std::vector<T> admm_pre;              // preconditioner per node
    std::vector<T> admm_val;              // assembled 125-entry stencil [N][125]
    std::vector<int32_t> admm_idx;        // its column node ids
    std::vector<M3<T>> admm_F[2];         // local variables F (AdmmSimulation::F)
    std::vector<M3<T>> admm_gvn;          // grad vn at particles (for bFu)

    bool isHencky(int64_t i) const { return model[i].kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC; }
    M3<T> strainN(int k, int64_t i) const { return k == 0 ? load9(Fn, i) : load9(Fe, i); }
    T& omegaOf(int k, int64_t i) { return admm_omega[2 * i + k]; }
    M3<T> yOf(int k, int64_t i) const
    {
        M3<T> m;
        for (int q = 0; q < 9; ++q) m.a[q / 3][q % 3] = admm_y[18 * i + 9 * k + q];
        return m;
    }
    void setY(int k, int64_t i, const M3<T>& m)
    {
        for (int q = 0; q < 9; ++q) admm_y[18 * i + 9 * k + q] = m.a[q / 3][q % 3];
    }

    // AnalyticCollisionObject::multiObjectCollisionWithFakeSeparate,
    // CollisionObject.cpp:108-156: a SEPARATE object whose boundary the node
    // already leaves does not collide.
    static bool multiObjectCollisionFakeSeparate(const std::vector<Collider<T>>& objs, const T x[3], T v[3], M3<T>& K)
    {
        bool any = false;
        int slip = 0;
        K = M3<T>::zero();
        for (const auto& o : objs) {
            if (o.d.type == ZMPM_GHOST) continue;
            T n[3] = { 0, 0, 0 };
            T old[3] = { v[0], v[1], v[2] };
            bool col = o.detectAndResolve(x, v, n);
            if (col && o.d.type == ZMPM_SEPARATE) {
                T vb[3] = { 0, 0, 0 }, nb[3] = { 0, 0, 0 };
                o.boundaryVelocityAndNormal(x, vb, nb);
                T dot = (old[0] - vb[0]) * nb[0] + (old[1] - vb[1]) * nb[1] + (old[2] - vb[2]) * nb[2];
                if (dot > 0) {
                    for (int d = 0; d < 3; ++d) v[d] = old[d];
                    col = false;
                }
            }
            any = col || any;
            if (!col) continue;
            if (o.d.type == ZMPM_STICKY) {
                K = M3<T>::identity();
                break;
            }
            for (int c = 0; c < slip; ++c) {
                T dot = K.a[0][c] * n[0] + K.a[1][c] * n[1] + K.a[2][c] * n[2];
                for (int i = 0; i < 3; ++i) n[i] -= dot * K.a[i][c];
            }
            T len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (len) {
                for (int i = 0; i < 3; ++i) K.a[i][slip] = n[i] / len;
                if (++slip == 3) break;
            }
        }
        return any;
    }

    // updateCollisionNodes, AdmmSimulationFoam.h:276-293
    void admmUpdateCollisionNodes()
    {
        collided.assign(N, 0);
        proj.assign(N, M3<T>::identity());
        iterateBlocks(true, [&](const int node[3], G& g) {
            int64_t id = g.idx;
            T vi[3], xi[3];
            for (int d = 0; d < 3; ++d) {
                vi[d] = dv[3 * id + d] + vn[3 * id + d];
                xi[d] = node[d] * dx;
            }
            M3<T> K;
            if (multiObjectCollisionFakeSeparate(colliders, xi, vi, K)) {
                collided[id] = 1;
                M3<T> Pm = M3<T>::identity();
                M3<T> KK = mulT(K, K);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) Pm.a[r][c] -= KK.a[r][c];
                proj[id] = Pm;
                for (int d = 0; d < 3; ++d) dv[3 * id + d] = vi[d] - vn[3 * id + d];
            }
        });
    }

    // initStep (AdmmSimulationFoam.h:297-403) and initMultiplierAndPreconditioner (:407-505)
    void admmInit(T rho)
    {
        for (auto& c : colliders) c.update(time);
        mvec.assign(N, 0);
        vn.assign(3 * N, 0);
        dv.assign(3 * N, 0);
        iterateBlocks(true, [&](const int*, G& g) {
            int64_t id = g.idx;
            mvec[id] = g.m;
            for (int d = 0; d < 3; ++d) vn[3 * id + d] = g.v[d];
        });
        Fn = F; // backupStrain
        // dv from the previous substep's particle dv (:304-320)
        std::vector<T> dvw(N, 0);
        coloredGroups([&](int i) {
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T w, const T*, G& g) {
                if (g.idx < 0) return;
                for (int d = 0; d < 3; ++d) dv[3 * g.idx + d] += admm_last_dv[3 * i + d] * w;
                dvw[g.idx] += w;
            });
        });
        for (int64_t id = 0; id < N; ++id)
            for (int d = 0; d < 3; ++d) dv[3 * id + d] = dv[3 * id + d] * dt / dvw[id];
        admmUpdateCollisionNodes();
        // initial local variables F = (I + dt grad(vn + dv)) Fn (:329-339)
        std::vector<M3<T>> grad;
        evalGradient(dv, true, grad);
        evalGradient(std::vector<T>(3 * N, 0), true, admm_gvn);
        for (int k = 0; k < 2; ++k) admm_F[k].assign(P, M3<T>::identity());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !visco[i].on) continue;
                M3<T> Sn = strainN(k, i);
                M3<T> Fa = Sn;
                M3<T> t = mul(grad[i], Sn);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) Fa.a[r][c] += dt * t.a[r][c];
                admm_F[k][i] = Fa;
            }
            // initOmega (:222-274) and the rescaled dual variables (:355-371)
            if (!isHencky(i)) continue;
            T om0 = admm_omega[2 * i], om1 = admm_omega[2 * i + 1];
            bool vm = plastic[i].kind == ZMPM_PLASTIC_VON_MISES, dp = plastic[i].kind == ZMPM_PLASTIC_DRUCKER_PRAGER;
            admm_omega[2 * i] = admmOmega(admm_F[0][i], vol[i], model[i].mu, model[i].lambda, vm, plastic[i].yield_stress, dp, plastic[i].a,
                plastic[i].cx);
            if (visco[i].on) admm_omega[2 * i + 1] = admmOmega(admm_F[1][i], vol[i], visco[i].mu, visco[i].lambda, false, T(0));
            for (int q = 0; q < 9; ++q) {
                admm_y[18 * i + q] = admm_y[18 * i + q] * om0 / admm_omega[2 * i];
                admm_y[18 * i + 9 + q] = admm_y[18 * i + 9 + q] * om1 / admm_omega[2 * i + 1];
            }
        }
        // assembled global matrix M + sum_p rho omega^2 dt^2 (Fn^T grad w)(Fn^T grad w)^T
        // per node pair, and its diagonal as preconditioner
        admm_val.assign((size_t)N * 125, 0);
        admm_idx.assign((size_t)N * 125, 0);
        admm_pre = mvec;
        coloredGroups([&](int i) {
            Spline<T> sp(&X[3 * i], dx);
            int nodes[27][3], ids[27], cnt = 0;
            T ftdw[2][27][3];
            iterateKernel(sp, base_offset[i], [&](const int node[3], T, const T* dw, G& g) {
                if (g.idx < 0) return;
                for (int d = 0; d < 3; ++d) nodes[cnt][d] = node[d];
                ids[cnt] = (int)g.idx;
                for (int k = 0; k < 2; ++k) {
                    if (k == 1 && !visco[i].on) continue;
                    M3<T> Sn = strainN(k, i);
                    for (int c = 0; c < 3; ++c) ftdw[k][cnt][c] = Sn.a[0][c] * dw[0] + Sn.a[1][c] * dw[1] + Sn.a[2][c] * dw[2];
                }
                ++cnt;
            });
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !visco[i].on) continue;
                T om = admm_omega[2 * i + k];
                T coeff = rho * om * om * dt * dt;
                for (int p = 0; p < cnt; ++p) {
                    for (int q = 0; q < cnt; ++q) {
                        int off = 25 * (nodes[q][0] - nodes[p][0] + 2) + 5 * (nodes[q][1] - nodes[p][1] + 2) + nodes[q][2] - nodes[p][2] + 2;
                        size_t e = (size_t)ids[p] * 125 + off;
                        admm_idx[e] = ids[q];
                        admm_val[e] += coeff * (ftdw[k][p][0] * ftdw[k][q][0] + ftdw[k][p][1] * ftdw[k][q][1] + ftdw[k][p][2] * ftdw[k][q][2]);
                    }
                    admm_pre[ids[p]] += coeff * (ftdw[k][p][0] * ftdw[k][p][0] + ftdw[k][p][1] * ftdw[k][p][1] + ftdw[k][p][2] * ftdw[k][p][2]);
                }
            }
        });
    }

    // GlobalSystem multiplier, AdmmSimulationFoam.h:127-143
    void admmMultiply(const std::vector<T>& x, std::vector<T>& b)
    {
        hvp_count++;
        b.assign(3 * N, 0);
#pragma omp parallel for schedule(static)
        for (int64_t n = 0; n < N; ++n) {
            T r[3] = { mvec[n] * x[3 * n], mvec[n] * x[3 * n + 1], mvec[n] * x[3 * n + 2] };
            const T* val = &admm_val[(size_t)n * 125];
            const int32_t* idx = &admm_idx[(size_t)n * 125];
            for (int k = 0; k < 125; ++k)
                for (int d = 0; d < 3; ++d) r[d] += x[3 * idx[k] + d] * val[k];
            for (int d = 0; d < 3; ++d) b[3 * n + d] = r[d];
        }
    }

    // FStep + FStepSolve, AdmmSimulationFoam.h:507-636
    void admmFStep(T rho, T local_tol)
    {
        std::vector<M3<T>> grad;
        evalGradient(dv, true, grad);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            if (!isHencky(i)) continue;
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !visco[i].on) continue;
                M3<T> Sn = strainN(k, i);
                T om = admm_omega[2 * i + k];
                M3<T> y = yOf(k, i);
                M3<T> FDb = Sn;
                M3<T> t = mul(grad[i], Sn);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) FDb.a[r][c] = (Sn.a[r][c] + (-y.a[r][c] / (om * rho))) + dt * t.a[r][c];
                T coeff = rho * om * om;
                if (k == 0) {
                    const bool dp = plastic[i].kind == ZMPM_PLASTIC_DRUCKER_PRAGER;
                    int mode = plastic[i].kind == ZMPM_PLASTIC_VON_MISES ? 1 : (dp ? 3 : 0);
                    admm_F[0][i] = admmLocalSolve(FDb, admm_F[0][i], vol[i], coeff, model[i].mu, model[i].lambda, mode,
                        dp ? plastic[i].a : plastic[i].yield_stress, visco[i], dt, 5, local_tol, dp ? plastic[i].cx : T(0));
                }
                else
                    admm_F[1][i] = admmLocalSolve(FDb, admm_F[1][i], vol[i], coeff, visco[i].mu, visco[i].lambda, 2, T(0), visco[i], dt, 20,
                        local_tol);
            }
        }
    }

    // dvStep, AdmmSimulationFoam.h:163-220: rhs = dt M g + sum_p dt rho omega^2
    // bFu Fn^T grad w with bFu = F - Fn + y/(omega rho) - dt grad(vn) Fn; MINRES
    // from the current dv.
    int admmDvStep(T rho, T tol, T rel_tol, int max_it)
    {
        std::vector<T> rhs(3 * N);
        for (int64_t n = 0; n < N; ++n)
            for (int d = 0; d < 3; ++d) rhs[3 * n + d] = dt * mvec[n] * gravity[d];
        std::vector<M3<T>> R(P);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            M3<T> acc = M3<T>::zero();
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !visco[i].on) continue;
                M3<T> Sn = strainN(k, i);
                T om = admm_omega[2 * i + k];
                M3<T> y = yOf(k, i);
                M3<T> t = mul(admm_gvn[i], Sn);
                M3<T> bFu;
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c)
                        bFu.a[r][c] = admm_F[k][i].a[r][c] - Sn.a[r][c] + y.a[r][c] / (om * rho) - dt * t.a[r][c];
                M3<T> Rk = mulT(scaled(bFu, dt * rho * om * om), Sn);
                acc = add(acc, Rk);
            }
            R[i] = acc;
        }
        rasterize(T(-1), R, rhs);
        admm_mode = true;
        int k = minres(dv, rhs, rel_tol, tol, max_it, true);
        admm_mode = false;
        return k;
    }

    // uStep, AdmmSimulationFoam.h:638-671: y += rho omega (F - (I + dt grad(vn + dv)) Fn)
    void admmUStep(T rho)
    {
        std::vector<M3<T>> grad;
        evalGradient(dv, true, grad);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            for (int k = 0; k < 2; ++k) {
                if (k == 1 && !visco[i].on) continue;
                M3<T> Sn = strainN(k, i);
                T om = admm_omega[2 * i + k];
                M3<T> y = yOf(k, i);
                M3<T> t = mul(grad[i], Sn);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) {
                        T tmp = admm_F[k][i].a[r][c] - Sn.a[r][c] - dt * t.a[r][c];
                        y.a[r][c] += rho * om * tmp;
                    }
                setY(k, i, y);
            }
        }
    }

    // admmStep, AdmmSimulationFoam.h:766-801
    int admmStep(const zmpm_solver& s, zmpm_stats& st)
    {
        const T rho = (T)s.admm_rho_scale;
        admmInit(rho);
        // residual_current is 1 (its computation is commented out, :779-780), so
        // the MINRES relative tolerance is min(0.5, sqrt(max(1, 1e-6))) = 0.5
        const T rel = std::min(T(0.5), T(1) * std::sqrt(std::max(T(1), T(1e-6))));
        for (int it = 0; it < s.admm_iterations; ++it) {
            admmUpdateCollisionNodes();
            admmFStep(rho, (T)s.admm_local_tolerance);
            st.krylov_iterations += admmDvStep(rho, (T)s.admm_global_tolerance, rel, s.admm_global_max_iterations);
            admmUStep(rho);
            st.newton_iterations += 1;
        }
        // last_dv = sum_i dv_i w_ip / (dt sum_i w_ip) (:788-800)
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            T acc[3] = { 0, 0, 0 }, wsum = 0;
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T w, const T*, G& g) {
                if (g.idx < 0) return;
                for (int d = 0; d < 3; ++d) acc[d] += dv[3 * g.idx + d] * w;
                wsum += w;
            });
            for (int d = 0; d < 3; ++d) admm_last_dv[3 * i + d] = acc[d] / (wsum * dt);
        }
        return ZMPM_OK;
    }

    // -------------------------------------------------------- explicit --
    // The symplectic branch of advanceOneTimeStep, MpmSimulationBase.cpp:264-281.
    const std::vector<T>* g2p_v = nullptr; // grid velocities for G2P (explicit substep)
    bool mls = false;                      // mls_mpm: G2P velocity gradient = C

    // ---------------------------------------------- phase-field fracture --
    // FractureSimulation members (FractureSimulation.h:48-63)
    T pf_M = 0, pf_delete = 0, pf_cg_tol = T(1e-6);
    bool pf_lumping = true;
    int pf_cg_max = 100;
    int pf_iters = 0;
    T pf_res = 0;

    bool anyPhaseField() const
    {
        for (const auto& d : damage)
            if (d.kind == ZMPM_DAMAGE_PHASE_FIELD) return true;
        return false;
    }

    // MpmSimulationBase::evalMaxParticleSpeed (MpmSimulationBase.cpp:1143-1166)
    void maxParticleSpeed(T& speed, T lo[3], T hi[3]) const
    {
        T m[7];
        m[0] = 0;
        for (int k = 1; k < 7; ++k) m[k] = std::numeric_limits<float>::lowest();
        for (int64_t i = 0; i < P; ++i) {
            T v2 = 0;
            for (int d = 0; d < 3; ++d) {
                v2 += V[3 * i + d] * V[3 * i + d];
                m[1 + d] = std::max(m[1 + d], X[3 * i + d]);
                m[4 + d] = std::max(m[4 + d], -X[3 * i + d]);
            }
            m[0] = std::max(m[0], std::sqrt(v2));
        }
        speed = m[0];
        for (int d = 0; d < 3; ++d) {
            hi[d] = m[1 + d];
            lo[d] = -m[4 + d];
        }
    }

    // AnalyticCollisionObject::evalMaxSpeed (CollisionObject.cpp:159-196) with
    // AnalyticLevelSet::getBounds of spheres and boxes; returns false for a
    // rotating or scaling half space, whose bounds the reference does not have.
    static bool colliderMaxSpeed(const zmpm_collider& c, double time, const T pmin[3], const T pmax[3], T& speed)
    {
        const T om[3] = { (T)c.angular_velocity[0], (T)c.angular_velocity[1], (T)c.angular_velocity[2] };
        const T dbdt[3] = { (T)c.translation_velocity[0], (T)c.translation_velocity[1], (T)c.translation_velocity[2] };
        const T dsdt = (T)c.scale_velocity;
        if (!(dsdt != 0 || std::sqrt(om[0] * om[0] + om[1] * om[1] + om[2] * om[2]) != 0)) {
            speed = std::sqrt(dbdt[0] * dbdt[0] + dbdt[1] * dbdt[1] + dbdt[2] * dbdt[2]);
            return true;
        }
        T lo[3], hi[3];
        if (c.shape == ZMPM_SPHERE)
            for (int d = 0; d < 3; ++d) {
                lo[d] = (T)(c.a[d] - c.radius);
                hi[d] = (T)(c.a[d] + c.radius);
            }
        else if (c.shape == ZMPM_BOX)
            for (int d = 0; d < 3; ++d) {
                lo[d] = (T)c.a[d];
                hi[d] = (T)c.b[d];
            }
        else
            return false;
        Collider<T> co;
        co.d = c;
        co.setRotation();
        const T s_ = (T)(c.scale + time * c.scale_velocity), ios = 1 / s_;
        T b[3];
        for (int d = 0; d < 3; ++d) b[d] = (T)(c.translation[d] + time * c.translation_velocity[d]);
        std::vector<std::array<T, 3>> pts;
        for (int i = 0; i < 8; ++i) {
            T x[3], Xm[3];
            for (int d = 0; d < 3; ++d) x[d] = (i & (1 << d)) ? pmin[d] : pmax[d];
            for (int r = 0; r < 3; ++r) Xm[r] = (co.R[0][r] * (x[0] - b[0]) + co.R[1][r] * (x[1] - b[1]) + co.R[2][r] * (x[2] - b[2])) * ios;
            bool any_a = false, any_b = false;
            for (int d = 0; d < 3; ++d) {
                any_a = any_a || lo[d] < Xm[d];
                any_b = any_b || Xm[d] < hi[d];
            }
            if (any_a && any_b) pts.push_back({ x[0], x[1], x[2] });
        }
        for (int i = 0; i < 8; ++i) {
            T Xm[3], x[3];
            for (int d = 0; d < 3; ++d) Xm[d] = (i & (1 << d)) ? lo[d] : hi[d];
            for (int r = 0; r < 3; ++r) x[r] = (co.R[r][0] * Xm[0] + co.R[r][1] * Xm[1] + co.R[r][2] * Xm[2]) * s_ + b[r];
            bool any_a = false, any_b = false;
            for (int d = 0; d < 3; ++d) {
                any_a = any_a || pmin[d] < x[d];
                any_b = any_b || x[d] < pmax[d];
            }
            if (any_a && any_b) pts.push_back({ x[0], x[1], x[2] });
        }
        speed = 0;
        for (const auto& x : pts) {
            const T xb[3] = { x[0] - b[0], x[1] - b[1], x[2] - b[2] };
            const T v[3] = { om[1] * xb[2] - om[2] * xb[1] + (dsdt * ios) * xb[0] + dbdt[0], om[2] * xb[0] - om[0] * xb[2] + (dsdt * ios) * xb[1] + dbdt[1],
                om[0] * xb[1] - om[1] * xb[0] + (dsdt * ios) * xb[2] + dbdt[2] };
            speed = std::max(speed, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        }
        return true;
    }

    // MpmSimulationBase::calculateDt (MpmSimulationBase.cpp:766-790)
    int calculateDt(double max_dt, double& dt_out)
    {
        T v, lo[3], hi[3];
        maxParticleSpeed(v, lo, hi);
        for (int d = 0; d < 3; ++d) {
            lo[d] -= (2 + 2) * dx;
            hi[d] += (2 + 2) * dx;
        }
        for (const auto& c : colliders) {
            T sc;
            if (!colliderMaxSpeed(c.d, time, lo, hi, sc)) {
                err = "a rotating or scaling half space has no bounds (AnalyticLevelSet::getBounds)";
                return ZMPM_BAD_ARG;
            }
            v = std::max(v, sc);
        }
        dt_out = v ? (double)(cfl * dx / v) : max_dt;
        return ZMPM_OK;
    }

    // FractureSimulation::deleteParticles (FractureSimulation.h:172-207)
    void deletePhaseFieldParticles()
    {
        for (int64_t i = 0; i < P; ++i)
            if (damage[i].kind == ZMPM_DAMAGE_PHASE_FIELD && damage[i].c < pf_delete) {
                for (int d = 0; d < 3; ++d) {
                    X[3 * i + d] = 4;
                    V[3 * i + d] = 0;
                }
                store9(F, i, M3<T>::identity());
                damage[i].allow_damage = false;
            }
    }

    // FractureSimulation::solvePhaseFieldSystem (FractureSimulation.h:257-456)
    // with phaseP2G (:208-255) and phaseG2P (:458-507), after P2G.  Node vectors
    // are indexed by GridState::idx; nodes outside the index set are skipped as
    // in the reference (`if (node_id < 0) return`).
    void solvePhaseField()
    {
        const T M = pf_M, one_over_dt = T(1) / dt;
        std::vector<T> phase(N, 0), mult(N, 0);
        if (M > 0) {
            coloredGroups([&](int i) {
                Spline<T> sp(&X[3 * i], dx);
                iterateKernel(sp, base_offset[i], [&](const int*, T w, const T*, G& g) {
                    if (g.idx < 0) return;
                    mult[g.idx] += w;
                    phase[g.idx] += damage[i].c * w;
                });
            });
            for (int64_t n = 0; n < N; ++n) phase[n] /= mult[n];
        }
        for (int64_t i = 0; i < P; ++i) damage[i].vol = vol[i] * det(load9(F, i));
        // right-hand side (:318-342) and the Jacobi diagonal of the
        // preconditioner (:409-441)
        std::vector<T> rhs(N, 0), diag(N, 0);
        coloredGroups([&](int i) {
            const Damage<T>& ph = damage[i];
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T w, const T*, G& g) {
                if (g.idx < 0) return;
                const int64_t n = g.idx;
                if (M > 0) {
                    rhs[n] += (M + phase[n] / dt) * ph.vol * w;
                    diag[n] += ph.vol * (M * ph.pf_Fp + one_over_dt) * w;
                }
                else {
                    rhs[n] += ph.vol * w;
                    diag[n] += ph.vol * ph.pf_Fp * w;
                }
            });
        });
        // the matrix-free operator (:344-407)
        std::vector<T> cs(P), gc(3 * P);
        auto multiply = [&](const std::vector<T>& x, std::vector<T>& b) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < P; ++i) {
                T c0 = 0, g0[3] = { 0, 0, 0 };
                Spline<T> sp(&X[3 * i], dx);
                iterateKernel(sp, base_offset[i], [&](const int*, T w, const T* dw, G& g) {
                    if (g.idx < 0) return;
                    if (!pf_lumping) c0 += x[g.idx] * w;
                    for (int d = 0; d < 3; ++d) g0[d] += x[g.idx] * dw[d];
                });
                const Damage<T>& ph = damage[i];
                if (!pf_lumping) c0 *= ph.vol * ph.pf_Fp;
                cs[i] = c0;
                for (int d = 0; d < 3; ++d) gc[3 * i + d] = g0[d] * (ph.vol * T(4) * ph.l0 * ph.l0);
            }
            b.assign(N, 0);
            coloredGroups([&](int i) {
                const Damage<T>& ph = damage[i];
                Spline<T> sp(&X[3 * i], dx);
                iterateKernel(sp, base_offset[i], [&](const int*, T w, const T* dw, G& g) {
                    if (g.idx < 0) return;
                    const int64_t n = g.idx;
                    if (!pf_lumping)
                        b[n] += cs[i] * w;
                    else if (M > 0)
                        b[n] += ph.vol * (ph.pf_Fp * M + one_over_dt) * w * x[n];
                    else
                        b[n] += ph.vol * ph.pf_Fp * w * x[n];
                    const T gd = gc[3 * i] * dw[0] + gc[3 * i + 1] * dw[1] + gc[3 * i + 2] * dw[2];
                    b[n] += (M > 0) ? gd * M : gd;
                });
            });
        };
        // Projects/fracture/ConjugateGradient.h:53-104 from x = 0 (so r = b)
        std::vector<T> x(N, 0), r = rhs, mr(N), sdir(N, 0), q(N);
        auto dot = [&](const std::vector<T>& a, const std::vector<T>& b) {
            T acc = 0;
            for (int64_t n = 0; n < N; ++n) acc += a[n] * b[n];
            return acc;
        };
        T norm = std::sqrt(dot(r, r));
        const T rel_tol = norm * (sizeof(T) == 4 ? T(1e-6) : T(1e-12));
        T rho_old = std::numeric_limits<T>::max();
        int it;
        for (it = 0;; ++it) {
            for (int64_t n = 0; n < N; ++n) mr[n] = r[n] / diag[n];
            const T rho = dot(mr, r);
            if (it == 0)
                sdir = mr;
            else
                for (int64_t n = 0; n < N; ++n) sdir[n] = rho / rho_old * sdir[n] + mr[n];
            multiply(sdir, q);
            const T sq = dot(sdir, q);
            const T alpha = sq ? rho / sq : std::numeric_limits<T>::max();
            for (int64_t n = 0; n < N; ++n) {
                x[n] = alpha * sdir[n] + x[n];
                r[n] = -alpha * q[n] + r[n];
            }
            rho_old = rho;
            norm = std::sqrt(dot(r, r));
            if (norm < pf_cg_tol || norm < rel_tol || it == pf_cg_max) break;
        }
        pf_iters = it;
        pf_res = norm;
        for (int64_t n = 0; n < N; ++n) phase[n] = (M > 0) ? x[n] - phase[n] : x[n];
        // phaseG2P
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            Damage<T>& ph = damage[i];
            if (!ph.allow_damage) continue;
            T pf = 0;
            Spline<T> sp(&X[3 * i], dx);
            iterateKernel(sp, base_offset[i], [&](const int*, T w, const T*, G& g) {
                if (g.idx >= 0) pf += w * phase[g.idx];
            });
            const T new_c = (M > 0) ? ph.c + pf : pf;
            ph.c = std::max(std::min(ph.c, new_c), T(0));
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            Damage<T>& ph = damage[i];
            if (model[i].kind != ZMPM_MODEL_NEOHOOKEAN_BORDEN) continue;
            // PhaseField::Update_Phase_Field_Fp (PhaseField.h:70-76)
            const T psi_pos = neoHookeanBordenPsiPos(model[i], load9(F, i));
            if (psi_pos > ph.H) {
                ph.H = std::min(psi_pos, ph.H_max);
                ph.pf_Fp = 4 * ph.l0 * (1 - ph.k) * ph.H * ph.one_over_sigma_c + 1;
            }
            model[i].g = ph.c * ph.c * (1 - ph.k) + ph.k;
        }
    }

    // MLS force of particlesToGridWithForceHelper<APIC, quadratic, MLS>
    // (MpmSimulationBase.cpp:527-541): f_i -= (S_p (x_i - x_p)) w_ip D^-1
    void rasterizeMls(const std::vector<M3<T>>& S, std::vector<T>& out)
    {
        const T D_inverse = 4 / (dx * dx);
        iterateBlocks(true, [&](const int*, G& g) {
            g.new_v[0] = g.new_v[1] = g.new_v[2] = 0;
        });
        coloredGroups([&](int i) {
            const M3<T>& st = S[i];
            const T* Xp = &X[3 * i];
            Spline<T> sp(Xp, dx);
            iterateKernel(sp, base_offset[i], [&](const int node[3], T w, const T*, G& g) {
                T xm[3];
                for (int d = 0; d < 3; ++d) xm[d] = node[d] * dx - Xp[d];
                for (int r = 0; r < 3; ++r) g.new_v[r] -= (st.a[r][0] * xm[0] + st.a[r][1] * xm[1] + st.a[r][2] * xm[2]) * (w * D_inverse);
            });
        });
        iterateBlocks(true, [&](const int*, G& g) {
            for (int d = 0; d < 3; ++d) out[3 * g.idx + d] += g.new_v[d];
        });
    }

    int substepExplicit(double dt_in, const zmpm_solver& s, zmpm_stats& st)
    {
        dt = (T)dt_in;
        implicit_ready = false;
        // forcesUpdateParticleState + FBasedMpmForceHelper::updateState
        // (MpmSimulationBase.cpp:682-700, FBasedMpmForceHelper.cpp:44-64): V0 tau(F)
        stress.resize(P);
        scratch.resize(P);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            if (model[i].kind == ZMPM_MODEL_NONE) {
                stress[i] = M3<T>::zero();
                continue;
            }
            M3<T> Fp = load9(F, i);
            updateScratch(model[i], Fp, scratch[i]);
            stress[i] = mulT(scaled(firstPiola(model[i], scratch[i]), vol[i]), Fp);
            if (visco[i].on) {
                // FElasticNonequilibratedBasedMpmForceHelper::updateState (h:39-60): + V0 tau(Fe)
                Model<T> mv;
                mv.kind = ZMPM_MODEL_STVK_HENCKY_ISOTROPIC;
                mv.mu = visco[i].mu;
                mv.lambda = visco[i].lambda;
                Scratch<T> sv;
                M3<T> Fe_ = load9(Fe, i);
                updateScratch(mv, Fe_, sv);
                stress[i] = add(stress[i], mulT(scaled(firstPiola(mv, sv), vol[i]), Fe_));
            }
        }
        int rc = sortParticlesAndPolluteGrid();
        if (rc != ZMPM_OK) return rc;
        // particlesToGridWithForceHelper<APIC, quadratic, !MLS> (:500-560): mass,
        // momentum, and f_i -= sum_p V0 tau_p grad w_ip, then the normalisation
        particlesToGrid();
        std::vector<T> f(3 * N, 0);
        if (s.mls_mpm)
            rasterizeMls(stress, f);
        else
            rasterize(T(1), stress, f);
        // FractureSimulation::particlesToGrid runs the damage update after P2G
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i)
            if ((damage[i].kind == ZMPM_DAMAGE_RANKINE || damage[i].kind == ZMPM_DAMAGE_RANKINE_REFERENCE) &&
                model[i].kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN)
                rankineUpdate(model[i], damage[i], load9(F, i));
        if (anyPhaseField()) solvePhaseField();
        // gridVelocityExplicitUpdate (:818-865)
        for (auto& c : colliders) c.update(time);
        mvec.assign(N, 0);
        vn.assign(3 * N, 0);
        std::vector<T> vnew(3 * N, 0);
        std::vector<uint8_t> collided_e(N, 0);
        iterateBlocks(true, [&](const int node[3], G& g) {
            const int64_t id = g.idx;
            mvec[id] = g.m;
            const T dt_over_mi = dt / g.m;
            T xi[3], vi[3];
            for (int d = 0; d < 3; ++d) {
                vn[3 * id + d] = g.v[d];
                xi[d] = node[d] * dx;
                vi[d] = g.v[d] + gravity[d] * dt + f[3 * id + d] * dt_over_mi;
            }
            M3<T> K;
            collided_e[id] = multiObjectCollision(colliders, xi, vi, K) ? 1 : 0;
            for (int d = 0; d < 3; ++d) vnew[3 * id + d] = vi[d];
        });
        // the colliders move to t + dt before trialCollision (:273-279)
        for (auto& c : colliders) c.update(time + dt_in);
        if (s.trial_collision) {
            // MpmSimulationBase::trialCollision (:298-311) and
            // AnalyticCollisionObject::trialCollision (CollisionObject.cpp:48-64)
            iterateBlocks(true, [&](const int node[3], G& g) {
                const int64_t id = g.idx;
                if (collided_e[id]) return;
                T* vi = &vnew[3 * id];
                const T xi[3] = { node[0] * dx, node[1] * dx, node[2] * dx };
                for (const auto& o : colliders) {
                    if (o.d.type == ZMPM_GHOST) continue;
                    const T xt[3] = { xi[0] + dt * vi[0], xi[1] + dt * vi[1], xi[2] + dt * vi[2] };
                    T phi, n[3];
                    if (o.queryInsideWorld(xt, phi, n))
                        for (int d = 0; d < 3; ++d) vi[d] -= (phi / dt) * n[d];
                }
            });
        }
        dv.assign(3 * N, 0);
        for (int64_t i = 0; i < 3 * N; ++i) dv[i] = vnew[i] - vn[i];
        g2p_v = &vnew;
        mls = s.mls_mpm != 0;
        int too_fast = gridToParticles();
        g2p_v = nullptr;
        mls = false;
        time += dt_in;
        st.newton_converged = 1;
        st.cfl_violation = too_fast;
        st.phase_field_iterations = pf_iters;
        st.phase_field_residual = (double)pf_res;
        st.num_particles = P;
        st.num_groups = (int64_t)group.size();
        st.num_blocks = (int64_t)blocks.size();
        st.num_nodes = N;
        int64_t nc = 0;
        for (auto c : collided_e) nc += c;
        st.num_collision_nodes = nc;
        return too_fast ? ZMPM_CFL_VIOLATION : ZMPM_OK;
    }

    // ------------------------------------------------------------- G2P --
    // constructNewVelocityFromNewtonResult + gridToParticlesHelper<APIC,deg2,!MLS>
    // + evolveStrain + applyPlasticity, MpmSimulationBase.cpp:867-877, 906-1030
    int gridToParticles()
    {
        iterateBlocks(false, [&](const int*, G& g) {
            g.new_v[0] = g.new_v[1] = g.new_v[2] = 0;
        });
        iterateBlocks(true, [&](const int*, G& g) {
            for (int d = 0; d < 3; ++d) g.new_v[d] = g2p_v ? (*g2p_v)[3 * g.idx + d] : g.v[d] + dv[3 * g.idx + d];
        });
        T D_inverse = 4 / (dx * dx);
        int too_fast = 0;
        gradV.resize(P);
#pragma omp parallel for schedule(static) reduction(| : too_fast)
        for (int64_t i = 0; i < P; ++i) {
            T* Xp = &X[3 * i];
            T picV[3] = { 0, 0, 0 };
            M3<T> Bp = M3<T>::zero(), gr = M3<T>::zero();
            Spline<T> sp(Xp, dx);
            iterateKernel(sp, base_offset[i], [&](const int node[3], T w, const T* dw, G& g) {
                T xi[3];
                for (int d = 0; d < 3; ++d) xi[d] = node[d] * dx - Xp[d];
                for (int r = 0; r < 3; ++r) {
                    picV[r] += w * g.new_v[r];
                    for (int c = 0; c < 3; ++c) {
                        Bp.a[r][c] += w * g.new_v[r] * xi[c];
                        gr.a[r][c] += g.new_v[r] * dw[c];
                    }
                }
            });
            for (int d = 0; d < 3; ++d) V[3 * i + d] = picV[d];
            T a = (apic_rpic_ratio + 1) * T(0.5), bcoef = (apic_rpic_ratio - 1) * T(0.5);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) Cm[9 * i + 3 * r + c] = a * (Bp.a[r][c] * D_inverse) + bcoef * (Bp.a[c][r] * D_inverse);
            // MLS: gradVp = C_p (MpmSimulationBase.cpp:958-961)
            gradV[i] = mls ? load9(Cm, i) : gr;
            T inc2 = 0;
            for (int d = 0; d < 3; ++d) {
                T inc = (T)dt * picV[d];
                Xp[d] += inc;
                inc2 += inc * inc;
            }
            too_fast |= (inc2 > dx * dx);
        }
        // evolveStrain with the G2P velocity gradient, FBasedMpmForceHelper.cpp:95-109
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i) {
            if (model[i].kind == ZMPM_MODEL_NONE) continue;
            M3<T> A = M3<T>::identity();
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) A.a[r][c] += (T)dt * gradV[i].a[r][c];
            M3<T> Fp = mul(A, load9(F, i));
            if (plastic[i].kind == ZMPM_PLASTIC_VON_MISES)
                vonMisesProject(model[i], plastic[i], Fp);
            else if (plastic[i].kind == ZMPM_PLASTIC_DRUCKER_PRAGER)
                druckerPragerProject(model[i], plastic[i], Fp);
            else if (plastic[i].kind == ZMPM_PLASTIC_CAM_CLAY)
                camClayProject(model[i], plastic[i], Fp);
            store9(F, i, Fp);
            if (visco[i].on) {
                M3<T> Fep = mul(A, load9(Fe, i));
                viscousReturn(visco[i], (T)dt, Fep);
                store9(Fe, i, Fep);
            }
        }
        return too_fast;
    }

    static M3<T> load9(const std::vector<T>& a, int64_t i)
    {
        M3<T> m;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) m.a[r][c] = a[9 * i + 3 * r + c];
        return m;
    }
    static void store9(std::vector<T>& a, int64_t i, const M3<T>& m)
    {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) a[9 * i + 3 * r + c] = m.a[r][c];
    }

    int beginImplicit(double dt_in)
    {
        dt = (T)dt_in;
        implicit_ready = false;
        int st = sortParticlesAndPolluteGrid();
        if (st != ZMPM_OK) return st;
        particlesToGrid();
        // FractureSimulation::particlesToGrid runs the damage update after P2G
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < P; ++i)
            if ((damage[i].kind == ZMPM_DAMAGE_RANKINE || damage[i].kind == ZMPM_DAMAGE_RANKINE_REFERENCE) &&
                model[i].kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN)
                rankineUpdate(model[i], damage[i], load9(F, i));
        if (anyPhaseField()) solvePhaseField();
        startBackwardEuler();
        return ZMPM_OK;
    }

    // MpmSimulationBase::advanceOneTimeStep (implicit), MpmSimulationBase.cpp:256-296
    int substep(double dt_in, const zmpm_solver& s, zmpm_stats& st)
    {
        std::memset(&st, 0, sizeof(st));
        hvp_count = 0;
        bool any_visco = false, all_models = true;
        for (int64_t i = 0; i < P; ++i) {
            any_visco = any_visco || visco[i].on;
            all_models = all_models && model[i].kind != ZMPM_MODEL_NONE;
        }
        bool conv = true;
        if (s.mls_mpm && s.integrator != ZMPM_EXPLICIT) {
            err = "mls_mpm requires the explicit integrator (MpmSimulationBase.cpp:102-106)";
            return ZMPM_BAD_ARG;
        }
        pf_iters = 0;
        pf_res = 0;
        if (s.integrator == ZMPM_ADMM)
            for (int64_t i = 0; i < P; ++i)
                if (plastic[i].kind == ZMPM_PLASTIC_CAM_CLAY) {
                    err = "the ADMM F-step has no Cam-Clay projection (AdmmSimulationFoam.h:617-633 lists none)";
                    return ZMPM_UNSUPPORTED;
                }
        if (anyPhaseField()) {
            if (s.integrator == ZMPM_ADMM) {
                err = "the phase-field solve belongs to FractureSimulation; AdmmSimulation does not run it";
                return ZMPM_BAD_ARG;
            }
            deletePhaseFieldParticles(); // FractureSimulation::reinitialize
        }
        if (s.integrator == ZMPM_EXPLICIT) return substepExplicit(dt_in, s, st);
        if (s.integrator == ZMPM_ADMM) {
            // AdmmSimulation::advanceOneTimeStep, AdmmSimulationFoam.h:816-837
            if (!all_models) {
                err = "ADMM needs an F-based model on every particle";
                return ZMPM_BAD_ARG;
            }
            dt = (T)dt_in;
            implicit_ready = false;
            int rc = sortParticlesAndPolluteGrid();
            if (rc != ZMPM_OK) return rc;
            particlesToGrid();
            admmStep(s, st);
        }
        else {
            if (any_visco) {
                err = "viscoelastic particles need the ADMM integrator (StvkWithHencky has no stress differential)";
                return ZMPM_BAD_ARG;
            }
            int rc = beginImplicit(dt_in);
            if (rc != ZMPM_OK) return rc;
            conv = newton(s, st);
            F = Fn; // restoreStrain
        }
        int too_fast = gridToParticles();
        time += dt_in;
        implicit_ready = false;
        st.newton_converged = conv ? 1 : 0;
        st.cfl_violation = too_fast;
        st.hvp_count = (int32_t)hvp_count;
        st.phase_field_iterations = pf_iters;
        st.phase_field_residual = (double)pf_res;
        st.num_particles = P;
        st.num_groups = (int64_t)group.size();
        st.num_blocks = (int64_t)blocks.size();
        st.num_nodes = N;
        int64_t nc = 0;
        for (auto c : collided) nc += c;
        st.num_collision_nodes = nc;
        if (st.status_flags & 1) return ZMPM_NAN_DETECTED;
        return too_fast ? ZMPM_CFL_VIOLATION : ZMPM_OK;
    }
};

// Type-erased handle over the float / double instantiations.
struct Ctx {
    zmpm_config cfg;
    bool is_double = true;
    std::unique_ptr<Sim<double>> d;
    std::unique_ptr<Sim<float>> f;
    std::string err;
};

} // namespace zo

using zo::Ctx;

#define DISPATCH(ctx, ...)               \
    do {                                 \
        if ((ctx)->is_double) {          \
            auto& S = *(ctx)->d;         \
            __VA_ARGS__;                 \
        }                                \
        else {                           \
            auto& S = *(ctx)->f;         \
            __VA_ARGS__;                 \
        }                                \
    } while (0)

template <class SimT>
static void add_particles_impl(SimT& S, int64_t n, const double* x, const double* v, const double* m, const double* vol)
{
    using T = typename std::remove_reference<decltype(S.dx)>::type;
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) {
            S.X.push_back((T)x[3 * i + d]);
            S.V.push_back(v ? (T)v[3 * i + d] : T(0));
        }
        for (int k = 0; k < 9; ++k) {
            S.Cm.push_back(T(0));
            S.F.push_back((k % 4 == 0) ? T(1) : T(0));
        }
        S.mass.push_back((T)m[i]);
        S.vol.push_back((T)vol[i]);
        S.model.emplace_back();
        S.plastic.emplace_back();
        S.damage.emplace_back();
        S.visco.emplace_back();
        for (int k = 0; k < 9; ++k) S.Fe.push_back((k % 4 == 0) ? T(1) : T(0));
        for (int k = 0; k < 18; ++k) S.admm_y.push_back(T(0));
        S.admm_omega.push_back(T(1));
        S.admm_omega.push_back(T(1));
        for (int k = 0; k < 3; ++k) S.admm_last_dv.push_back(T(0));
    }
    S.P += n;
    S.Fn = S.F;
}

extern "C" {

// The oracle exports the same interface as include/zmpm.h with the prefix
// zoracle_.  The config's precision picks the instantiation: ZMPM_FP64 ->
// double with GridState<double> (2x4x4 pages); anything else -> float with
// GridState<float> (4x4x4 pages), the reference's T=float build.
int zoracle_create(const zmpm_config* cfg, Ctx** out)
{
    if (!cfg || !out || !(cfg->dx > 0)) return ZMPM_BAD_ARG;
    auto* c = new (std::nothrow) Ctx();
    if (!c) return ZMPM_NO_MEMORY;
    c->cfg = *cfg;
    c->is_double = (cfg->precision == ZMPM_FP64);
    bool ok;
    if (c->is_double) {
        c->d.reset(new zo::Sim<double>(7));
        ok = c->d->init(*cfg);
    }
    else {
        c->f.reset(new zo::Sim<float>(6));
        ok = c->f->init(*cfg);
    }
    if (!ok) {
        delete c;
        return ZMPM_NO_MEMORY;
    }
    *out = c;
    return ZMPM_OK;
}

int zoracle_destroy(Ctx* c)
{
    delete c;
    return ZMPM_OK;
}

const char* zoracle_last_error(const Ctx* c)
{
    if (!c) return "null context";
    if (c->is_double) return c->d->err.c_str();
    return c->f->err.c_str();
}

int zoracle_add_particles(Ctx* c, int64_t n, const double* x, const double* v, const double* m, const double* vol, int64_t* lower)
{
    if (!c || n < 0 || (n && (!x || !m || !vol))) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        if (lower) *lower = S.P;
        add_particles_impl(S, n, x, v, m, vol);
    });
    return ZMPM_OK;
}

int zoracle_add_fbased_force(Ctx* c, int64_t lo, int64_t hi, int32_t kind, double E, double nu)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        T Et = (T)E, nut = (T)nu;
        T lambda = Et * nut / ((T(1) + nut) * (T(1) - T(2) * nut));
        T mu = Et / (T(2) * (T(1) + nut));
        for (int64_t i = lo; i < hi; ++i) {
            S.model[i].kind = kind;
            S.model[i].mu = mu;
            S.model[i].lambda = lambda;
            S.model[i].kappa = (T)0.666666 * mu + lambda;
            S.model[i].g = 1;
        }
    });
    return ZMPM_OK;
}

int zoracle_set_lame(Ctx* c, int64_t lo, int64_t hi, const double* mu, const double* lambda)
{
    if (!c || !mu || !lambda) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i) {
            S.model[i].mu = (T)mu[i - lo];
            S.model[i].lambda = (T)lambda[i - lo];
            S.model[i].kappa = (T)0.666666 * S.model[i].mu + S.model[i].lambda;
        }
    });
    return ZMPM_OK;
}

int zoracle_add_plasticity(Ctx* c, int64_t lo, int64_t hi, int32_t kind, double ys, double xi, double fs)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        if (kind != ZMPM_PLASTIC_NONE && kind != ZMPM_PLASTIC_VON_MISES) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i) {
            S.plastic[i].kind = kind;
            S.plastic[i].yield_stress = (T)ys;
            S.plastic[i].xi = (T)xi;
            S.plastic[i].fail_stress = (T)fs;
        }
    });
    return ZMPM_OK;
}

int zoracle_add_drucker_prager(Ctx* c, int64_t lo, int64_t hi, double friction_angle, double beta, double cohesion, int32_t vc)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i)
            if (S.model[i].kind != ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
                S.err = "Drucker-Prager needs StvkWithHenckyIsotropic particles";
                return ZMPM_BAD_ARG;
            }
        // DruckerPragerStvkHencky::DruckerPragerStvkHencky, PlasticityApplier.cpp:247-255
        const T sin_phi = zo::sinDegrees((T)friction_angle);
        const T alpha = std::sqrt(T(2) / T(3)) * T(2) * sin_phi / (T(3) - sin_phi);
        for (int64_t i = lo; i < hi; ++i) {
            zo::Plastic<T>& p = S.plastic[i];
            p = zo::Plastic<T>();
            p.kind = ZMPM_PLASTIC_DRUCKER_PRAGER;
            p.a = alpha;
            p.beta = (T)beta;
            p.cx = (T)cohesion;
            p.flag = vc ? 1 : 0;
            p.logJp = 0;
            // reported by get_plastic_state in the library's per-kind layout
            p.yield_stress = p.a;
            p.xi = p.beta;
            p.fail_stress = p.cx;
            p.broken = p.flag;
        }
    });
    return ZMPM_OK;
}

int zoracle_add_cam_clay(Ctx* c, int64_t lo, int64_t hi, double logJp, double friction_angle, double beta, double xi, int32_t hardening)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i)
            if (S.model[i].kind != ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
                S.err = "Cam-Clay needs NeoHookeanBorden particles";
                return ZMPM_BAD_ARG;
            }
        // NonAssociativeCamClay::NonAssociativeCamClay with dim = 3, PlasticityApplier.cpp:10-20
        const T sin_phi = zo::sinDegrees((T)friction_angle);
        const T mc = std::sqrt(T(2) / T(3)) * T(2) * sin_phi / (T(3) - sin_phi);
        const T M = mc * T(3) / std::sqrt(T(2) / (T(6) - T(3)));
        for (int64_t i = lo; i < hi; ++i) {
            zo::Plastic<T>& p = S.plastic[i];
            p = zo::Plastic<T>();
            p.kind = ZMPM_PLASTIC_CAM_CLAY;
            p.a = M;
            p.beta = (T)beta;
            p.cx = (T)xi;
            p.flag = hardening ? 1 : 0;
            p.logJp = (T)logJp;
            p.yield_stress = p.a;
            p.xi = p.beta;
            p.fail_stress = p.cx;
            p.broken = p.flag;
        }
    });
    return ZMPM_OK;
}

int zoracle_get_log_jp(Ctx* c, double* out)
{
    if (!c || !out) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < S.P; ++i) out[i] = S.plastic[i].logJp;
    });
    return ZMPM_OK;
}

// One Drucker-Prager (kind 2) or Cam-Clay (kind 3) projection of a row-major F
// in place, for known-answer tests: params = (alpha or M, beta, cohesion or xi),
// model (mu, lambda, kappa).
int zoracle_plastic_project(int32_t kind, double mu, double lambda, double kappa, const double* params, int32_t flag, double* logJp,
    double* F)
{
    zo::Model<double> c;
    c.mu = mu;
    c.lambda = lambda;
    c.kappa = kappa;
    zo::Plastic<double> p;
    p.kind = kind;
    p.a = params[0];
    p.beta = params[1];
    p.cx = params[2];
    p.flag = flag;
    p.logJp = *logJp;
    zo::M3<double> Fm;
    for (int i = 0; i < 9; ++i) Fm.a[i / 3][i % 3] = F[i];
    if (kind == ZMPM_PLASTIC_DRUCKER_PRAGER)
        zo::druckerPragerProject(c, p, Fm);
    else if (kind == ZMPM_PLASTIC_CAM_CLAY)
        zo::camClayProject(c, p, Fm);
    else
        return ZMPM_BAD_ARG;
    for (int i = 0; i < 9; ++i) F[i] = Fm.a[i / 3][i % 3];
    *logJp = p.logJp;
    return ZMPM_OK;
}

// Drucker-Prager in singular values for known-answer tests: projectSigma
// (D = NULL) or projectSigmaAndDerivative.
int zoracle_dp_project_sigma(double mu, double lambda, double alpha, double cohesion, const double* s, double* out, double* D)
{
    if (!s || !out) return ZMPM_BAD_ARG;
    if (!D) {
        zo::dpProjectSigma(mu, lambda, alpha, cohesion, s, out);
        return ZMPM_OK;
    }
    double Dm[3][3];
    zo::dpProjectSigmaDerivative(mu, lambda, alpha, cohesion, s, out, Dm);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) D[3 * r + c] = Dm[r][c];
    return ZMPM_OK;
}

int zoracle_add_damage(Ctx* c, int64_t lo, int64_t hi, int32_t kind, double sigma_f, double residual_phase)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i) {
            S.damage[i].kind = kind;
            S.damage[i].sigma_f = (T)sigma_f;
            S.damage[i].k = (T)residual_phase;
            S.damage[i].c = 1;
        }
    });
    return ZMPM_OK;
}

int zoracle_get_damage(Ctx* c, double* out)
{
    if (!c || !out) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < S.P; ++i) out[i] = S.damage[i].c;
    });
    return ZMPM_OK;
}

int zoracle_add_phase_field(Ctx* c, int64_t lo, int64_t hi, double percentage, double l0, int32_t allow_damage, double residual_phase)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i)
            if (S.model[i].kind != ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
                S.err = "the phase field needs NeoHookeanBorden particles";
                return ZMPM_BAD_ARG;
            }
        for (int64_t i = lo; i < hi; ++i) {
            zo::Damage<T>& d = S.damage[i];
            d = zo::Damage<T>();
            d.kind = ZMPM_DAMAGE_PHASE_FIELD;
            d.k = (T)residual_phase;
            d.c = 1;
            d.H = 0;
            d.l0 = (T)l0;
            d.one_over_sigma_c = phaseFieldOneOverSigmaC(S.model[i], (T)percentage);
            d.pf_Fp = 1;
            d.vol = S.vol[i];
            d.allow_damage = allow_damage != 0;
        }
    });
    return ZMPM_OK;
}

int zoracle_set_phase_field_solver(Ctx* c, double M, int32_t lumping, double del, int32_t cg_max, double cg_tol)
{
    if (!c || !(M >= 0) || cg_max < 0 || !(cg_tol >= 0)) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        S.pf_M = (T)M;
        S.pf_lumping = lumping != 0;
        S.pf_delete = (T)del;
        S.pf_cg_max = cg_max;
        S.pf_cg_tol = (T)cg_tol;
    });
    return ZMPM_OK;
}

int zoracle_get_phase_field(Ctx* c, double* cc, double* H, double* fp, double* vol)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < S.P; ++i) {
            if (cc) cc[i] = S.damage[i].c;
            if (H) H[i] = S.damage[i].H;
            if (fp) fp[i] = S.damage[i].pf_Fp;
            if (vol) vol[i] = S.damage[i].vol;
        }
    });
    return ZMPM_OK;
}

int zoracle_max_particle_speed(Ctx* c, double* speed, double* lo, double* hi)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        T v, l[3], h[3];
        S.maxParticleSpeed(v, l, h);
        if (speed) *speed = (double)v;
        for (int d = 0; d < 3; ++d) {
            if (lo) lo[d] = (double)l[d];
            if (hi) hi[d] = (double)h[d];
        }
    });
    return ZMPM_OK;
}

int zoracle_calculate_dt(Ctx* c, double max_dt, double* dt)
{
    if (!c || !dt || !(max_dt > 0)) return ZMPM_BAD_ARG;
    DISPATCH(c, { return S.calculateDt(max_dt, *dt); });
    return ZMPM_OK;
}

int zoracle_set_phase_field_sigma_c(Ctx* c, const double* isc)
{
    if (!c || !isc) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        for (int64_t i = 0; i < S.P; ++i) S.damage[i].one_over_sigma_c = (T)isc[i];
    });
    return ZMPM_OK;
}

int zoracle_add_viscoelastic(Ctx* c, int64_t lo, int64_t hi, double E, double nu, double vd, double vv)
{
    if (!c || !(vd > 0) || !(vv > 0)) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (lo < 0 || hi > S.P || lo > hi) return ZMPM_BAD_ARG;
        for (int64_t i = lo; i < hi; ++i)
            if (S.model[i].kind != ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) return ZMPM_BAD_ARG;
        T Et = (T)E, nut = (T)nu;
        for (int64_t i = lo; i < hi; ++i) {
            auto& v = S.visco[i];
            v.on = 1;
            v.lambda = Et * nut / ((T(1) + nut) * (T(1) - T(2) * nut)); // StvkWithHencky.cpp:16-20
            v.mu = Et / (T(2) * (T(1) + nut));
            v.vd = (T)vd;
            v.vv = (T)vv;
            for (int q = 0; q < 9; ++q) S.Fe[9 * i + q] = (q % 4 == 0) ? T(1) : T(0);
        }
    });
    return ZMPM_OK;
}

int zoracle_get_viscoelastic_strain(Ctx* c, double* Fe)
{
    if (!c || !Fe) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < 9 * S.P; ++i) Fe[i] = S.Fe[i];
    });
    return ZMPM_OK;
}

int zoracle_set_viscoelastic_strain(Ctx* c, const double* Fe)
{
    if (!c || !Fe) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        for (int64_t i = 0; i < 9 * S.P; ++i) S.Fe[i] = (T)Fe[i];
    });
    return ZMPM_OK;
}

// The viscous return map alone on one strain (test hook).
int zoracle_viscous_return(double E, double nu, double vd, double vv, double dt, double* F)
{
    zo::Visco<double> v;
    v.lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
    v.mu = E / (2 * (1 + nu));
    v.vd = vd;
    v.vv = vv;
    zo::M3<double> m;
    for (int q = 0; q < 9; ++q) m.a[q / 3][q % 3] = F[q];
    zo::viscousReturn(v, dt, m);
    for (int q = 0; q < 9; ++q) F[q] = m.a[q / 3][q % 3];
    return ZMPM_OK;
}

int zoracle_adjoint_substep(Ctx* c, double dt, const zmpm_solver* s, double tol, double* gx, double* gv, double* gC, double* gF,
    double* gE, zmpm_stats* st)
{
    if (!c || !s || !(dt > 0)) return ZMPM_BAD_ARG;
    zmpm_stats local;
    if (!st) st = &local;
    int rc;
    DISPATCH(c, { rc = S.adjointSubstep(dt, *s, tol, gx, gv, gC, gF, gE, *st); });
    return rc;
}

int zoracle_checkpoint_save(Ctx* c, int32_t slot)
{
    if (!c || slot < 0) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        auto& k = S.checkpoints[slot];
        k.X = S.X;
        k.V = S.V;
        k.Cm = S.Cm;
        k.F = S.F;
        k.Fe = S.Fe;
        k.y = S.admm_y;
        k.omega = S.admm_omega;
        k.lastdv = S.admm_last_dv;
        k.model = S.model;
        k.plastic = S.plastic;
        k.damage = S.damage;
        k.time = S.time;
    });
    return ZMPM_OK;
}

int zoracle_checkpoint_load(Ctx* c, int32_t slot)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        auto it = S.checkpoints.find(slot);
        if (it == S.checkpoints.end() || it->second.X.size() != S.X.size()) return ZMPM_BAD_ARG;
        auto& k = it->second;
        S.X = k.X;
        S.V = k.V;
        S.Cm = k.Cm;
        S.F = k.F;
        S.Fe = k.Fe;
        S.admm_y = k.y;
        S.admm_omega = k.omega;
        S.admm_last_dv = k.lastdv;
        S.model = k.model;
        S.plastic = k.plastic;
        S.damage = k.damage;
        S.time = k.time;
    });
    return ZMPM_OK;
}

int zoracle_add_collision_object(Ctx* c, const zmpm_collider* o, int32_t* id)
{
    if (!c || !o) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        zo::Collider<T> col;
        col.d = *o;
        col.update(S.time);
        if (id) *id = (int32_t)S.colliders.size();
        S.colliders.push_back(col);
    });
    return ZMPM_OK;
}

int zoracle_set_collision_object(Ctx* c, int32_t id, const zmpm_collider* o)
{
    if (!c || !o) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        if (id < 0 || id >= (int32_t)S.colliders.size()) return ZMPM_BAD_ARG;
        S.colliders[id].d = *o;
    });
    return ZMPM_OK;
}

int zoracle_get_particles(Ctx* c, double* x, double* v, double* C, double* F)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < 3 * S.P; ++i) {
            if (x) x[i] = S.X[i];
            if (v) v[i] = S.V[i];
        }
        for (int64_t i = 0; i < 9 * S.P; ++i) {
            if (C) C[i] = S.Cm[i];
            if (F) F[i] = S.F[i];
        }
    });
    return ZMPM_OK;
}

int zoracle_set_particles(Ctx* c, const double* x, const double* v, const double* C, const double* F)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        for (int64_t i = 0; i < 3 * S.P; ++i) {
            if (x) S.X[i] = (T)x[i];
            if (v) S.V[i] = (T)v[i];
        }
        for (int64_t i = 0; i < 9 * S.P; ++i) {
            if (C) S.Cm[i] = (T)C[i];
            if (F) S.F[i] = (T)F[i];
        }
    });
    return ZMPM_OK;
}

int zoracle_get_plastic_state(Ctx* c, double* ys, int32_t* broken)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < S.P; ++i) {
            if (ys) ys[i] = S.plastic[i].yield_stress;
            if (broken) broken[i] = S.plastic[i].broken;
        }
    });
    return ZMPM_OK;
}

int64_t zoracle_num_particles(const Ctx* c)
{
    if (!c) return -1;
    return c->is_double ? c->d->P : c->f->P;
}

double zoracle_time(const Ctx* c)
{
    if (!c) return 0;
    return c->is_double ? c->d->time : c->f->time;
}

int zoracle_substep(Ctx* c, double dt, const zmpm_solver* s, zmpm_stats* st)
{
    if (!c || !s || !(dt > 0)) return ZMPM_BAD_ARG;
    zmpm_stats local;
    if (!st) st = &local;
    int rc;
    double t0 = omp_get_wtime();
    DISPATCH(c, { rc = S.substep(dt, *s, *st); });
    st->ms_total = (omp_get_wtime() - t0) * 1e3;
    return rc;
}

int zoracle_bin(Ctx* c, int64_t* counts)
{
    if (!c) return ZMPM_BAD_ARG;
    int rc;
    DISPATCH(c, {
        rc = S.sortParticlesAndPolluteGrid();
        if (counts) {
            counts[0] = S.P;
            counts[1] = (int64_t)S.group.size();
            counts[2] = (int64_t)S.blocks.size();
        }
    });
    return rc;
}

int zoracle_bin_fetch(Ctx* c, zmpm_bin_result* out)
{
    if (!c || !out) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        for (int64_t i = 0; i < S.P; ++i) {
            if (out->particle_sorter) out->particle_sorter[i] = S.sorter[i];
            if (out->particle_order) out->particle_order[i] = S.order[i];
            if (out->particle_base_offset) out->particle_base_offset[i] = S.base_offset[i];
        }
        for (size_t g = 0; g < S.group.size(); ++g) {
            if (out->particle_group) {
                out->particle_group[2 * g] = S.group[g].first;
                out->particle_group[2 * g + 1] = S.group[g].second;
            }
            if (out->block_offset) out->block_offset[g] = S.block_offset[g];
        }
        for (size_t b = 0; b < S.blocks.size(); ++b)
            if (out->page_offsets) out->page_offsets[b] = S.blocks[b];
    });
    return ZMPM_OK;
}

int zoracle_begin_implicit(Ctx* c, double dt, int64_t* n)
{
    if (!c || !(dt > 0)) return ZMPM_BAD_ARG;
    int rc;
    DISPATCH(c, {
        rc = S.beginImplicit(dt);
        if (n) *n = S.N;
    });
    return rc;
}

int zoracle_get_grid(Ctx* c, double* m, double* v, int32_t* coord)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        if (!S.implicit_ready) return ZMPM_NOT_READY;
        S.iterateBlocks(true, [&](const int node[3], decltype(S.at(0))& g) {
            int64_t id = g.idx;
            if (m) m[id] = g.m;
            for (int d = 0; d < 3; ++d) {
                if (v) v[3 * id + d] = g.v[d];
                if (coord) coord[3 * id + d] = node[d];
            }
        });
    });
    return ZMPM_OK;
}

int zoracle_get_initial_dv(Ctx* c, double* dv, int32_t* col)
{
    if (!c) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        if (!S.implicit_ready) return ZMPM_NOT_READY;
        for (int64_t i = 0; i < S.N; ++i) {
            for (int d = 0; d < 3; ++d)
                if (dv) dv[3 * i + d] = S.dv[3 * i + d];
            if (col) col[i] = S.collided[i];
        }
    });
    return ZMPM_OK;
}

int zoracle_residual(Ctx* c, const double* dvin, double* r, double* norm)
{
    if (!c || !dvin) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (!S.implicit_ready) return ZMPM_NOT_READY;
        for (int64_t i = 0; i < 3 * S.N; ++i) S.dv[i] = (T)dvin[i];
        S.updateState(S.dv);
        std::vector<T> res;
        T nr = S.computeResidual(res);
        if (r)
            for (int64_t i = 0; i < 3 * S.N; ++i) r[i] = res[i];
        if (norm) *norm = nr;
    });
    return ZMPM_OK;
}

int zoracle_multiply(Ctx* c, const double* x, double* b, int32_t fp32)
{
    (void)fp32;
    if (!c || !x || !b) return ZMPM_BAD_ARG;
    DISPATCH(c, {
        using T = typename std::remove_reference<decltype(S.dx)>::type;
        if (!S.implicit_ready || S.scratch.size() != (size_t)S.P) return ZMPM_NOT_READY;
        std::vector<T> xi(3 * S.N), bo;
        for (int64_t i = 0; i < 3 * S.N; ++i) xi[i] = (T)x[i];
        S.multiply(xi, bo);
        for (int64_t i = 0; i < 3 * S.N; ++i) b[i] = bo[i];
    });
    return ZMPM_OK;
}

// Single-particle model evaluation for known-answer and FD tests:
// given F (row-major), returns psi, P and dP:dF.
int zoracle_model_eval(int32_t kind, double E, double nu, const double* F, const double* dF, double* psi_out, double* P_out, double* dP_out)
{
    zo::Model<double> c;
    c.kind = kind;
    c.lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
    c.mu = E / (2 * (1 + nu));
    c.kappa = 0.666666 * c.mu + c.lambda;
    zo::M3<double> Fm, dFm;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            Fm.a[r][k] = F[3 * r + k];
            dFm.a[r][k] = dF ? dF[3 * r + k] : 0;
        }
    zo::Scratch<double> s;
    zo::updateScratch(c, Fm, s);
    if (psi_out) *psi_out = zo::psi(c, s);
    zo::M3<double> P = zo::firstPiola(c, s), dP = zo::firstPiolaDifferential(c, s, dFm);
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            if (P_out) P_out[3 * r + k] = P.a[r][k];
            if (dP_out) dP_out[3 * r + k] = dP.a[r][k];
        }
    return ZMPM_OK;
}

// 3x3 SVD of the oracle (F = U diag(sigma) V^T), double or float.
int zoracle_svd3(const double* F, double* U, double* sigma, double* V, int32_t fp32)
{
    if (fp32) {
        zo::M3<float> A, Uf, Vf;
        float s[3];
        for (int i = 0; i < 9; ++i) A.a[i / 3][i % 3] = (float)F[i];
        int it = zo::svd3(A, Uf, s, Vf);
        for (int i = 0; i < 9; ++i) {
            U[i] = Uf.a[i / 3][i % 3];
            V[i] = Vf.a[i / 3][i % 3];
        }
        for (int d = 0; d < 3; ++d) sigma[d] = s[d];
        return it;
    }
    zo::M3<double> A, Ud, Vd;
    double s[3];
    for (int i = 0; i < 9; ++i) A.a[i / 3][i % 3] = F[i];
    int it = zo::svd3(A, Ud, s, Vd);
    for (int i = 0; i < 9; ++i) {
        U[i] = Ud.a[i / 3][i % 3];
        V[i] = Vd.a[i / 3][i % 3];
    }
    for (int d = 0; d < 3; ++d) sigma[d] = s[d];
    return it;
}

// Von Mises return map on one F (row-major, in place); returns the new yield stress.
// The first eigenvalue of Eigen's general eigensolver for a 3x3 matrix (row-major).
double zoracle_eigen_first_eigenvalue(const double* A)
{
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = A[3 * i + j];
    return zo::eigen_first_eigenvalue(a);
}

int zoracle_von_mises(int32_t kind, double E, double nu, double yield_stress, double xi, double* F, double* ys_out)
{
    zo::Model<double> c;
    c.kind = kind;
    c.lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
    c.mu = E / (2 * (1 + nu));
    zo::Plastic<double> p;
    p.kind = ZMPM_PLASTIC_VON_MISES;
    p.yield_stress = yield_stress;
    p.xi = xi;
    p.fail_stress = 1e300;
    zo::M3<double> Fm;
    for (int i = 0; i < 9; ++i) Fm.a[i / 3][i % 3] = F[i];
    zo::vonMisesProject(c, p, Fm);
    for (int i = 0; i < 9; ++i) F[i] = Fm.a[i / 3][i % 3];
    if (ys_out) *ys_out = p.yield_stress;
    return ZMPM_OK;
}

// SPGrid helpers for the golden-vector tests.
uint64_t zoracle_linear_offset(int32_t log2_struct, int32_t i, int32_t j, int32_t k)
{
    return zo::Mask(log2_struct).linear_offset(i, j, k);
}
uint64_t zoracle_packed_add(int32_t log2_struct, uint64_t a, uint64_t b)
{
    return zo::Mask(log2_struct).packed_add(a, b);
}
void zoracle_masks(int32_t log2_struct, uint64_t* xyz)
{
    zo::Mask m(log2_struct);
    xyz[0] = m.xmask;
    xyz[1] = m.ymask;
    xyz[2] = m.zmask;
}

} // extern "C"
