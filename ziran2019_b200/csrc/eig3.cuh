// The first eigenvalue of a real 3x3 matrix in the order of Eigen's general
// eigensolver, as FractureSimulation::solvePhaseFieldSystemNaive takes it
// (sigma_max = cauchy.eigenvalues()[0].real(), Projects/fracture/
// FractureSimulation.h:539-543).  Eigen (not in the reference tree; 3.3 on the
// reference's platform) returns the eigenvalues in the order of the real Schur
// form its RealSchur computes; this is that published method for n = 3:
//   1. scale by the largest |a_ij|;
//   2. Householder reduction to upper Hessenberg form (one reflection of
//      column 0);
//   3. Francis double-shift QR (Golub & Van Loan, Matrix Computations, 7.5;
//      EISPACK hqr): deflate where a subdiagonal entry falls below
//      eps (|t_k-1,k-1| + |t_kk|) (the Hessenberg norm when that sum is zero),
//      exceptional shifts at the 10th and 30th iteration of an eigenvalue, and
//      a 2x2 block with real eigenvalues rotated upper triangular so that each
//      diagonal entry keeps its nearer eigenvalue;
//   4. the first eigenvalue: t_00, or the real part of the first 2x2 block's
//      complex pair.
// FP64, per particle in local memory (the loop bounds depend on the data).
#pragma once
#include <cfloat>

namespace zmpm {

struct Eig3 {
    double t[3][3];

    // (beta, tau, essential part e) of the reflection I - tau (1, e)(1, e)^T
    // that maps x (length n) to (beta, 0, ...)
    __device__ static void reflector(const double* x, int n, double& tau, double& beta, double* e)
    {
        double tail = 0;
        for (int i = 1; i < n; ++i) tail += x[i] * x[i];
        const double c0 = x[0];
        if (tail <= DBL_MIN) {
            tau = 0;
            beta = c0;
            for (int i = 1; i < n; ++i) e[i - 1] = 0;
            return;
        }
        beta = sqrt(c0 * c0 + tail);
        if (c0 >= 0) beta = -beta;
        for (int i = 1; i < n; ++i) e[i - 1] = x[i] / (c0 - beta);
        tau = (beta - c0) / beta;
    }
    __device__ void left(int r0, int n, int c0, int c1, double tau, const double* e)
    {
        for (int c = c0; c < c1; ++c) {
            double d = t[r0][c];
            for (int i = 1; i < n; ++i) d += e[i - 1] * t[r0 + i][c];
            t[r0][c] -= tau * d;
            for (int i = 1; i < n; ++i) t[r0 + i][c] -= tau * e[i - 1] * d;
        }
    }
    __device__ void right(int r0, int r1, int c0, int n, double tau, const double* e)
    {
        for (int r = r0; r < r1; ++r) {
            double d = t[r][c0];
            for (int i = 1; i < n; ++i) d += e[i - 1] * t[r][c0 + i];
            t[r][c0] -= tau * d;
            for (int i = 1; i < n; ++i) t[r][c0 + i] -= tau * e[i - 1] * d;
        }
    }

    __device__ double first_eigenvalue(const double A[9])
    {
        double scale = 0;
        for (int i = 0; i < 9; ++i) scale = fmax(scale, fabs(A[i]));
        if (scale < DBL_MIN) return 0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) t[i][j] = A[3 * i + j] / scale;
        {
            const double x[2] = { t[1][0], t[2][0] };
            double tau, beta, e[1];
            reflector(x, 2, tau, beta, e);
            t[1][0] = beta;
            t[2][0] = 0;
            left(1, 2, 1, 3, tau, e);
            right(0, 3, 1, 2, tau, e);
        }
        double norm = 0;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i <= (j + 1 < 2 ? j + 1 : 2); ++i) norm += fabs(t[i][j]);
        if (norm == 0) return 0;
        int iu = 2, iter = 0, total = 0;
        double exshift = 0;
        while (iu >= 0) {
            int il = iu;
            while (il > 0) {
                double s = fabs(t[il - 1][il - 1]) + fabs(t[il][il]);
                if (s == 0) s = norm;
                if (fabs(t[il][il - 1]) < DBL_EPSILON * s) break;
                --il;
            }
            if (il == iu) {
                t[iu][iu] += exshift;
                if (iu > 0) t[iu][iu - 1] = 0;
                --iu;
                iter = 0;
            }
            else if (il == iu - 1) {
                const double p = 0.5 * (t[iu - 1][iu - 1] - t[iu][iu]);
                const double q = p * p + t[iu][iu - 1] * t[iu - 1][iu];
                t[iu][iu] += exshift;
                t[iu - 1][iu - 1] += exshift;
                if (q >= 0) {
                    const double z = sqrt(fabs(q));
                    const double a = p >= 0 ? p + z : p - z, b = t[iu][iu - 1];
                    const double r = hypot(a, b);
                    const double c = r == 0 ? 1.0 : a / r, sn = r == 0 ? 0.0 : b / r;
                    for (int k = iu - 1; k < 3; ++k) {
                        const double t0 = t[iu - 1][k], t1 = t[iu][k];
                        t[iu - 1][k] = c * t0 + sn * t1;
                        t[iu][k] = -sn * t0 + c * t1;
                    }
                    for (int k = 0; k <= iu; ++k) {
                        const double t0 = t[k][iu - 1], t1 = t[k][iu];
                        t[k][iu - 1] = c * t0 + sn * t1;
                        t[k][iu] = -sn * t0 + c * t1;
                    }
                    t[iu][iu - 1] = 0;
                }
                if (iu > 1) t[iu - 1][iu - 2] = 0;
                iu -= 2;
                iter = 0;
            }
            else {
                double x = t[iu][iu], y = t[iu - 1][iu - 1], w = t[iu][iu - 1] * t[iu - 1][iu];
                if (iter == 10) {
                    exshift += x;
                    for (int i = 0; i <= iu; ++i) t[i][i] -= x;
                    const double s = fabs(t[iu][iu - 1]) + fabs(t[iu - 1][iu - 2]);
                    x = y = 0.75 * s;
                    w = -0.4375 * s * s;
                }
                if (iter == 30) {
                    double s = 0.5 * (y - x);
                    s = s * s + w;
                    if (s > 0) {
                        s = sqrt(s);
                        if (y < x) s = -s;
                        s = x - w / (0.5 * (y - x) + s);
                        for (int i = 0; i <= iu; ++i) t[i][i] -= s;
                        exshift += s;
                        x = y = w = 0.964;
                    }
                }
                ++iter;
                if (++total > 120) break; // the iteration cap of RealSchur (40 per row)
                int im = iu - 2;
                double v[3];
                for (;; --im) {
                    const double tmm = t[im][im], r = x - tmm, s = y - tmm;
                    v[0] = (r * s - w) / t[im + 1][im] + t[im][im + 1];
                    v[1] = t[im + 1][im + 1] - tmm - r - s;
                    v[2] = t[im + 2][im + 1];
                    if (im == il) break;
                    const double lhs = t[im][im - 1] * (fabs(v[1]) + fabs(v[2]));
                    const double rhs = v[0] * (fabs(t[im - 1][im - 1]) + fabs(tmm) + fabs(t[im + 1][im + 1]));
                    if (fabs(lhs) < DBL_EPSILON * rhs) break;
                }
                for (int k = im; k <= iu - 2; ++k) {
                    const bool first = k == im;
                    if (!first) {
                        v[0] = t[k][k - 1];
                        v[1] = t[k + 1][k - 1];
                        v[2] = t[k + 2][k - 1];
                    }
                    double tau, beta, e[2];
                    reflector(v, 3, tau, beta, e);
                    if (beta != 0) {
                        if (first && k > il)
                            t[k][k - 1] = -t[k][k - 1];
                        else if (!first)
                            t[k][k - 1] = beta;
                        left(k, 3, k, 3, tau, e);
                        right(0, (iu < k + 3 ? iu : k + 3) + 1, k, 3, tau, e);
                    }
                }
                {
                    const double v2[2] = { t[iu - 1][iu - 2], t[iu][iu - 2] };
                    double tau, beta, e[1];
                    reflector(v2, 2, tau, beta, e);
                    if (beta != 0) {
                        t[iu - 1][iu - 2] = beta;
                        left(iu - 1, 2, iu - 1, 3, tau, e);
                        right(0, iu + 1, iu - 1, 2, tau, e);
                    }
                }
                for (int i = im + 2; i <= iu; ++i) {
                    t[i][i - 2] = 0;
                    if (i > im + 2) t[i][i - 3] = 0;
                }
            }
        }
        if (t[1][0] == 0) return t[0][0] * scale;
        return 0.5 * (t[0][0] + t[1][1]) * scale;
    }
};

} // namespace zmpm
