// 3x3 matrices held in registers (row-major a[3*r+c]).
#pragma once
#include "common.cuh"

namespace zmpm {

template <class T>
struct M3 {
    T a[9];
    ZMPM_HD T& operator()(int r, int c) { return a[3 * r + c]; }
    ZMPM_HD const T& operator()(int r, int c) const { return a[3 * r + c]; }
};

template <class T>
ZMPM_HD M3<T> m3_zero()
{
    M3<T> m;
#pragma unroll
    for (int i = 0; i < 9; ++i) m.a[i] = T(0);
    return m;
}
template <class T>
ZMPM_HD M3<T> m3_identity()
{
    M3<T> m = m3_zero<T>();
    m.a[0] = m.a[4] = m.a[8] = T(1);
    return m;
}
template <class T>
ZMPM_HD M3<T> m3_mul(const M3<T>& A, const M3<T>& B)
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = A(i, 0) * B(0, j) + A(i, 1) * B(1, j) + A(i, 2) * B(2, j);
    return C;
}
template <class T>
ZMPM_HD M3<T> m3_mulT(const M3<T>& A, const M3<T>& B) // A B^T
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = A(i, 0) * B(j, 0) + A(i, 1) * B(j, 1) + A(i, 2) * B(j, 2);
    return C;
}
template <class T>
ZMPM_HD M3<T> m3_Tmul(const M3<T>& A, const M3<T>& B) // A^T B
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = A(0, i) * B(0, j) + A(1, i) * B(1, j) + A(2, i) * B(2, j);
    return C;
}
template <class T>
ZMPM_HD M3<T> m3_transpose(const M3<T>& A)
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = A(j, i);
    return C;
}
template <class T>
ZMPM_HD T m3_contract(const M3<T>& A, const M3<T>& B)
{
    T s = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) s += A.a[i] * B.a[i];
    return s;
}
template <class T>
ZMPM_HD T m3_det(const M3<T>& m)
{
    return m(0, 0) * (m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) - m(1, 0) * (m(0, 1) * m(2, 2) - m(2, 1) * m(0, 2))
        + m(2, 0) * (m(0, 1) * m(1, 2) - m(1, 1) * m(0, 2));
}
// cofactor matrix J F^{-T}
template <class T>
ZMPM_HD M3<T> m3_cofactor(const M3<T>& F)
{
    M3<T> A;
    A(0, 0) = F(1, 1) * F(2, 2) - F(1, 2) * F(2, 1);
    A(0, 1) = F(1, 2) * F(2, 0) - F(1, 0) * F(2, 2);
    A(0, 2) = F(1, 0) * F(2, 1) - F(1, 1) * F(2, 0);
    A(1, 0) = F(0, 2) * F(2, 1) - F(0, 1) * F(2, 2);
    A(1, 1) = F(0, 0) * F(2, 2) - F(0, 2) * F(2, 0);
    A(1, 2) = F(0, 1) * F(2, 0) - F(0, 0) * F(2, 1);
    A(2, 0) = F(0, 1) * F(1, 2) - F(0, 2) * F(1, 1);
    A(2, 1) = F(0, 2) * F(1, 0) - F(0, 0) * F(1, 2);
    A(2, 2) = F(0, 0) * F(1, 1) - F(0, 1) * F(1, 0);
    return A;
}
// U diag(d) V^T
template <class T>
ZMPM_HD M3<T> m3_udvt(const M3<T>& U, const T d[3], const M3<T>& V)
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C(i, j) = U(i, 0) * d[0] * V(j, 0) + U(i, 1) * d[1] * V(j, 1) + U(i, 2) * d[2] * V(j, 2);
    return C;
}
template <class T, class S>
ZMPM_HD M3<T> m3_cast(const M3<S>& A)
{
    M3<T> C;
#pragma unroll
    for (int i = 0; i < 9; ++i) C.a[i] = T(A.a[i]);
    return C;
}

} // namespace zmpm
