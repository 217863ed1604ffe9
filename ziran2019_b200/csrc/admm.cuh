// Per-particle arithmetic of the ADMM integrator and of the viscoelastic strain
// (Projects/admm/AdmmSimulationFoam.h, AdmmFormula.h,
// Lib/MPM/Force/FElasticNonequilibratedBasedMpmForceHelper.h).  Everything
// runs in registers in the template precision T; SVDs use svd3.cuh.
#pragma once
#include "mat3.cuh"
#include "models.cuh"
#include "svd3.cuh"

namespace zmpm {

// alpha = 2 mu / nu_d, beta = 2 (2 mu + 3 lambda) / (9 nu_v) - 2 mu / (3 nu_d)
// (FElasticNonequilibratedBasedMpmForceHelper.h:74-75); returns
// a = 1 / (1 + dt alpha) and b = dt beta / (1 + dt (alpha + 3 beta)).
template <class T>
ZMPM_HD void viscous_coefficients(T mu, T lambda, T vd, T vv, T dt, T& a, T& b)
{
    const T alpha = T(2.0) * mu / vd;
    const T beta = T(2.0) * (T(2.0) * mu + lambda * T(3)) / (T(9.0) * vv) - T(2.0) * mu / (vd * T(3));
    a = T(1.0) / (T(1.0) + dt * alpha);
    b = dt * beta / (T(1.0) + dt * (alpha + T(3) * beta));
}

// The viscous return map of evolveStrain (h:77-85) on Fe = U diag(s) V^T:
// eps = a (log|s| - b t), Fe <- U exp(eps) V^T.  t is the reference's
// `epsilon_trial.trace()` of a 3-vector, which Eigen evaluates as the single
// diagonal coefficient of a 3x1 matrix: log|s_0|.
template <class T>
ZMPM_D void viscous_return(T mu, T lambda, T vd, T vv, T dt, M3<T>& Fe)
{
    M3<T> U, V;
    T s[3];
    svd3(Fe, U, s, V);
    T a, b;
    viscous_coefficients(mu, lambda, vd, vv, dt, a, b);
    T et[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) et[d] = log(fabs(s[d]));
    const T t = et[0];
    T ex[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) ex[d] = exp(a * (et[d] - b * t));
    Fe = m3_udvt(U, ex, V);
}

// d psi / d sigma and d^2 psi / d sigma^2 of psi = mu |log s|^2 + lambda/2
// (tr log s)^2: StvkWithHenckyIsotropic::firstPiolaDiagonal /
// firstPiolaDerivativeDiagonal (StvkWithHenckyIsotropic.h:218-269).
template <class T>
ZMPM_HD void hencky_diag(T mu, T lambda, const T s[3], T dE[3], T ddE[3][3])
{
    T L[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) L[d] = log(fabs(s[d]));
    const T sum_log = L[0] + L[1] + L[2];
    const T g = T(2) * mu + lambda;
#pragma unroll
    for (int d = 0; d < 3; ++d) dE[d] = (T(2) * mu * L[d] + lambda * sum_log) / s[d];
    ddE[0][0] = (g * (T(1) - L[0]) - lambda * (L[1] + L[2])) / (s[0] * s[0]);
    ddE[1][1] = (g * (T(1) - L[1]) - lambda * (L[0] + L[2])) / (s[1] * s[1]);
    ddE[2][2] = (g * (T(1) - L[2]) - lambda * (L[0] + L[1])) / (s[2] * s[2]);
    ddE[0][1] = ddE[1][0] = lambda / (s[0] * s[1]);
    ddE[0][2] = ddE[2][0] = lambda / (s[0] * s[2]);
    ddE[1][2] = ddE[2][1] = lambda / (s[1] * s[2]);
}

// Eigenvalues of a symmetric 3x3 matrix by cyclic Jacobi rotations (Golub &
// Van Loan, Matrix Computations, 8.5.2); at most 50 sweeps.
template <class T>
ZMPM_HD void sym3_eig(T A[3][3], T ev[3])
{
    for (int sweep = 0; sweep < 50; ++sweep) {
        const T off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        if (off == T(0)) break;
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int q = p + 1; q < 3; ++q) {
                if (A[p][q] == T(0)) continue;
                const T theta = (A[q][q] - A[p][p]) / (T(2) * A[p][q]);
                const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
                const T c = T(1) / sqrt(t * t + T(1)), sn = t * c;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const T akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - sn * akq;
                    A[k][q] = sn * akp + c * akq;
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const T apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - sn * aqk;
                    A[q][k] = sn * apk + c * aqk;
                }
            }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) ev[d] = A[d][d];
}

// |makePD(A)|_F^2 and |makePD2D([[a, b], [b, d]])|_F^2 (AdmmFormula.h:12-35):
// sums of the squared eigenvalues clamped at zero.
template <class T>
ZMPM_HD T make_pd_norm2(const T A[3][3])
{
    T B[3][3], ev[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) B[r][c] = A[r][c];
    sym3_eig(B, ev);
    T s = T(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) s += ev[d] > T(0) ? ev[d] * ev[d] : T(0);
    return s;
}
template <class T>
ZMPM_HD T make_pd2_norm2(T a, T b, T d)
{
    const T m = (a + d) / T(2), r = sqrt((a - d) * (a - d) / T(4) + b * b);
    const T l0 = m - r, l1 = m + r;
    return (l0 > T(0) ? l0 * l0 : T(0)) + (l1 > T(0) ? l1 * l1 : T(0));
}

// StvkWithHenckyIsotropic::Bij (3D), StvkWithHenckyIsotropic.h:180-216: the
// 2x2 block [[P+M, M-P], [M-P, P+M]]; returns P and M.
template <class T>
ZMPM_HD void hencky_bij(T mu, T lambda, const T s[3], int i, int j, T clamp, T& P, T& M)
{
    T dE[3], ddE[3][3];
    hencky_diag(mu, lambda, s, dE, ddE);
    const T x = s[i] + s[j];
    const T mag = x > T(0) ? x : -x;
    const T cl = (mag > clamp ? mag : clamp) * (x > T(0) ? T(1) : T(-1));
    P = T(0.5) * (dE[i] + dE[j]) / cl;
    const T Lj = log(fabs(s[j]));
    const T sum_log = log(fabs(s[0])) + log(fabs(s[1])) + log(fabs(s[2]));
    M = T(-0.5) * (lambda * sum_log + T(2) * mu * diff_interlock_log_over_diff(s[i], s[j], Lj, T(1e-8))) / (s[i] * s[j]);
}

// VonMisesStvkHencky::projectSigmaAndDerivative, PlasticityApplier.cpp:580-602.
template <class T>
ZMPM_HD void vm_project_sigma(T mu, T ys, const T s[3], T out[3], T D[3][3])
{
    T eps[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) eps[d] = log(s[d] > T(1e-4) ? s[d] : T(1e-4));
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    const T hat_norm = sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T delta_gamma = hat_norm - ys / (T(2) * mu);
    if (delta_gamma <= T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            out[r] = s[r];
#pragma unroll
            for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
        }
        return;
    }
    T w[3], sv[3], sh[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        w[d] = T(1) / s[d];
        sv[d] = eps[d] - tr / T(3) * T(1);
    }
    const T snorm = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sh[d] = sv[d] / snorm;
        out[d] = exp(eps[d] - (delta_gamma / hat_norm) * hat[d]);
    }
    const T k1 = T(1) - ys / (T(2) * mu * snorm), k2 = ys / (T(2) * mu * snorm);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T Iw = r == c ? w[c] : T(0);
            D[r][c] = out[r] * (Iw - k1 * (Iw - w[c] / T(3)) - k2 * sh[r] * sh[c] * w[c]);
        }
}

// DruckerPragerStvkHencky::projectSigma (PlasticityApplier.cpp:319-347): the
// return map in singular values without log Jp, as initOmega uses it.
template <class T>
ZMPM_HD void dp_project_sigma(T mu, T lambda, T alpha, T cohesion, const T s[3], T out[3])
{
    T eps[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T a = fabs(s[d]);
        eps[d] = log(a > T(1e-4) ? a : T(1e-4)) - cohesion;
    }
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    if (tr >= T(0)) {
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] = exp(cohesion) * T(1);
        return;
    }
    const T hn = sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T dg = hn + (T(3) * lambda + T(2) * mu) / (T(2) * mu) * tr * alpha;
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = exp((dg <= T(0)) ? eps[d] + cohesion : eps[d] - (dg / hn) * hat[d] + cohesion);
}

// DruckerPragerStvkHencky::projectSigmaAndDerivative (PlasticityApplier.cpp:
// 387-423), the F-step's projection: inside (identity), tip (zero derivative)
// or cone, D = diag(out) (((1 + 2p)/3 - p eps / k) w^T - p (I - s s^T) diag(w)).
template <class T>
ZMPM_HD void dp_project_sigma_derivative(T mu, T lambda, T alpha, T cohesion, const T s[3], T out[3], T D[3][3])
{
    T eps[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T a = fabs(s[d]);
        eps[d] = log(a > T(1e-4) ? a : T(1e-4)) - cohesion;
    }
    const T tr = eps[0] + eps[1] + eps[2];
    T hat[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) hat[d] = eps[d] - (tr / T(3)) * T(1);
    const T hn = sqrt(hat[0] * hat[0] + hat[1] * hat[1] + hat[2] * hat[2]);
    const T dg = hn + (T(3) * lambda + T(2) * mu) / (T(2) * mu) * tr * alpha;
    if (dg <= T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            out[r] = exp(eps[r] + cohesion);
#pragma unroll
            for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
        }
        return;
    }
    if (tr > T(0) || hn == T(0)) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            out[r] = exp(cohesion) * T(1);
#pragma unroll
            for (int c = 0; c < 3; ++c) D[r][c] = T(0);
        }
        return;
    }
    T w[3], sv[3], sh[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        w[d] = T(1) / s[d];
        sv[d] = eps[d] - tr / T(3) * T(1);
    }
    const T sn = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sh[d] = sv[d] / sn;
        out[d] = exp(eps[d] - (dg / hn) * hat[d] + cohesion);
    }
    const T pp = alpha * tr * (T(3) * lambda + T(2) * mu) / (T(2) * mu * sn);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T m1 = ((T(1) + T(2) * pp) / T(3) * T(1) - pp / tr * eps[r]) * w[c];
            const T m2 = pp * ((r == c ? T(1) : T(0)) - sh[r] * sh[c]) * w[c];
            D[r][c] = out[r] * (m1 - m2);
        }
}

// The viscous map in singular values and its derivative, AdmmSimulationFoam.h:583-595.
template <class T>
ZMPM_HD void viscous_sigma(T mu, T lambda, T vd, T vv, T dt, const T zi[3], T zp[3], T D[3][3])
{
    T a, b;
    viscous_coefficients(mu, lambda, vd, vv, dt, a, b);
    T et[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) et[d] = log(fabs(zi[d]));
    const T t = et[0]; // `epsilon_trial.trace()` of a 3-vector, as in viscous_return
#pragma unroll
    for (int d = 0; d < 3; ++d) zp[d] = exp(a * (et[d] - b * t));
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) D[r][c] = zp[r] * a * ((r == c ? T(1) / zi[c] : T(0)) - b * (T(1) / zi[c]));
}

enum AdmmLocalMode { ADMM_ELASTIC = 0, ADMM_VON_MISES = 1, ADMM_VISCOUS = 2, ADMM_DRUCKER_PRAGER = 3 };

struct AdmmStrainParams {
    double mu, lambda, ys, vd, vv;
    double alpha, cohesion; // Drucker-Prager
};

// One strain of AdmmSimulation::FStepSolve (AdmmSimulationFoam.h:507-615): SVD of
// the target FDb, then Newton in singular values on
// vol psi(P(z)) + coeff/2 |z - sigma|^2 from z = diag(U^T F V).
template <class T>
ZMPM_D M3<T> admm_local_solve(const M3<T>& FDb, const M3<T>& Fcur, T vol, T coeff, const AdmmStrainParams& p, int mode, T dt, int iters,
    T tol)
{
    M3<T> U, V;
    T sigma[3];
    svd3(FDb, U, sigma, V);
    const M3<T> W = m3_Tmul(U, m3_mul(Fcur, V));
    T zi[3] = { W(0, 0), W(1, 1), W(2, 2) };
    const T mu = (T)p.mu, lambda = (T)p.lambda;
    for (int j = 0; j < iters; ++j) {
        T zp[3], D[3][3];
        if (mode == ADMM_VON_MISES)
            vm_project_sigma(mu, (T)p.ys, zi, zp, D);
        else if (mode == ADMM_DRUCKER_PRAGER)
            dp_project_sigma_derivative(mu, lambda, (T)p.alpha, (T)p.cohesion, zi, zp, D);
        else if (mode == ADMM_VISCOUS)
            viscous_sigma(mu, lambda, (T)p.vd, (T)p.vv, dt, zi, zp, D);
        else {
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                zp[r] = zi[r];
#pragma unroll
                for (int c = 0; c < 3; ++c) D[r][c] = r == c ? T(1) : T(0);
            }
        }
        T dE[3], ddE[3][3];
        hencky_diag(mu, lambda, zp, dE, ddE);
        T g[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d] = vol * dE[d] + coeff * (zi[d] - sigma[d]);
        M3<T> Pm;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) Pm(r, c) = vol * (ddE[r][0] * D[0][c] + ddE[r][1] * D[1][c] + ddE[r][2] * D[2][c]) + (r == c ? coeff : T(0));
        // step = P^-1 (-g) with P^-1 = adj(P) / det(P)
        const M3<T> C = m3_cofactor(Pm);
        const T det = Pm(0, 0) * C(0, 0) + Pm(0, 1) * C(0, 1) + Pm(0, 2) * C(0, 2);
        T step[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) step[r] = (C(0, r) / det) * (-g[0]) + (C(1, r) / det) * (-g[1]) + (C(2, r) / det) * (-g[2]);
#pragma unroll
        for (int d = 0; d < 3; ++d) zi[d] += step[d];
        if (sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]) < tol) break;
    }
    return m3_udvt(U, zi, V);
}

// initOmega for one strain (AdmmSimulationFoam.h:236-270):
// omega = sqrt(vol sqrt(|makePD(d2E)|^2 + sum_ij |makePD2D(B_ij)|^2)), with
// sigma projected onto the yield surface for the B_ij terms under von Mises
// and Drucker-Prager (pkind).
template <class T>
ZMPM_D T admm_omega(const M3<T>& Fa, T vol, T mu, T lambda, int pkind, T ys, T alpha = T(0), T cohesion = T(0))
{
    M3<T> U, V;
    T s[3];
    svd3(Fa, U, s, V);
    T dE[3], ddE[3][3];
    hencky_diag(mu, lambda, s, dE, ddE);
    T total = make_pd_norm2(ddE);
    if (pkind == ZMPM_PLASTIC_VON_MISES) {
        T sp[3], D[3][3];
        vm_project_sigma(mu, ys, s, sp, D);
#pragma unroll
        for (int d = 0; d < 3; ++d) s[d] = sp[d];
    }
    else if (pkind == ZMPM_PLASTIC_DRUCKER_PRAGER) {
        T sp[3];
        dp_project_sigma(mu, lambda, alpha, cohesion, s, sp);
#pragma unroll
        for (int d = 0; d < 3; ++d) s[d] = sp[d];
    }
    const int pi_[3] = { 0, 0, 1 }, pj_[3] = { 1, 2, 2 };
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        T P, M;
        hencky_bij(mu, lambda, s, pi_[k], pj_[k], T(1e-6), P, M);
        total += make_pd2_norm2(P + M, M - P, P + M);
    }
    return sqrt(vol * sqrt(total));
}

} // namespace zmpm
