// Constitutive models, their Hessian-vector scratch, and return maps, per
// particle in registers.
//
// update(): F -> stress S = V0 P(F) Fn^T (FBasedMpmForceHelper::updateImplicitState,
//           Lib/MPM/Force/FBasedMpmForceHelper.cpp:68-92) and the scratch the
//           Hessian-vector product needs.
// hvp():    grad(dv) -> dS = V0 dP(grad(dv) Fn) Fn^T
//           (FBasedMpmForceHelper::computeStressDifferential, :132-154).
//
// Scratch slots (NS = 34, stored [slot][particle] in the HVP precision):
//   SVD-isotropic models (StvkWithHenckyIsotropic, fixed corotated):
//     0-8 U, 9-17 W = Fn V, 18-29 the SvdBasedIsotropicHelper coefficients
//     (psi00,psi11,psi22, psi01,psi02,psi12, m01,m02,m12, p01,p02,p12)
//     pre-multiplied by V0, so dS = U K(U^T grad(dv) W) W^T.
//   NeoHookeanBorden: 0-8 F, 9-17 F^{-T}, 18-26 Fn, 27 J, 28 mu J^{-2/3},
//     29 kappa/2 (J - 1/J), 30 kappa/2 (1 + 1/J^2), 31 g, 32 V0, 33 F:F.
#pragma once
#include "svd3.cuh"
#include "../../include/zmpm.h"

namespace zmpm {

constexpr int NS = 34;

template <class T>
ZMPM_HD T clamp_small_magnitude(T x, T eps)
{
    if (x < -eps) return x;
    if (x < T(0)) return -eps;
    if (x < eps) return eps;
    return x;
}
// (x log y - y log x)/(x - y) evaluated as MathTools.h:247-252 does
template <class T>
ZMPM_HD T diff_interlock_log_over_diff(T x, T y, T logy, T eps)
{
    T p = x / y - T(1);
    T l1p = (fabs(p) < eps) ? T(1) : log1p(p) / p;
    return logy - y * (l1p / y);
}

// SvdBasedIsotropicHelper::dPdFOfSigmaContract (SvdBasedIsotropicHelper.h:151-162)
// with coefficients c = (psi00,psi11,psi22, psi01,psi02,psi12, m01,m02,m12, p01,p02,p12)
template <class T>
ZMPM_HD M3<T> iso_contract(const T c[12], const M3<T>& A)
{
    M3<T> B;
    B(0, 0) = c[0] * A(0, 0) + c[3] * A(1, 1) + c[4] * A(2, 2);
    B(1, 1) = c[3] * A(0, 0) + c[1] * A(1, 1) + c[5] * A(2, 2);
    B(2, 2) = c[4] * A(0, 0) + c[5] * A(1, 1) + c[2] * A(2, 2);
    B(0, 1) = ((c[6] + c[9]) * A(0, 1) + (c[6] - c[9]) * A(1, 0)) / T(2);
    B(1, 0) = ((c[6] - c[9]) * A(0, 1) + (c[6] + c[9]) * A(1, 0)) / T(2);
    B(0, 2) = ((c[7] + c[10]) * A(0, 2) + (c[7] - c[10]) * A(2, 0)) / T(2);
    B(2, 0) = ((c[7] - c[10]) * A(0, 2) + (c[7] + c[10]) * A(2, 0)) / T(2);
    B(1, 2) = ((c[8] + c[11]) * A(1, 2) + (c[8] - c[11]) * A(2, 1)) / T(2);
    B(2, 1) = ((c[8] - c[11]) * A(1, 2) + (c[8] + c[11]) * A(2, 1)) / T(2);
    return B;
}

// Derivatives of psi-hat(sigma) for the SVD-isotropic models.
// psi[3] = d psi / d sigma_i; c[12] = second-order coefficients.
template <class T>
ZMPM_HD void iso_coefficients(int kind, T mu, T lambda, const T sg[3], T psi[3], T c[12])
{
    const T eps = T(1e-6);
    if (kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
        // StvkWithHenckyIsotropic::updateScratch (3D), StvkWithHenckyIsotropic.h:114-143
        T L0 = log(fabs(sg[0])), L1 = log(fabs(sg[1])), L2 = log(fabs(sg[2]));
        T g = T(2) * mu + lambda;
        T sum_log = L0 + L1 + L2;
        psi[0] = (T(2) * mu * L0 + lambda * sum_log) / sg[0];
        psi[1] = (T(2) * mu * L1 + lambda * sum_log) / sg[1];
        psi[2] = (T(2) * mu * L2 + lambda * sum_log) / sg[2];
        c[0] = (g * (T(1) - L0) - lambda * (L1 + L2)) / (sg[0] * sg[0]);
        c[1] = (g * (T(1) - L1) - lambda * (L0 + L2)) / (sg[1] * sg[1]);
        c[2] = (g * (T(1) - L2) - lambda * (L0 + L1)) / (sg[2] * sg[2]);
        c[3] = lambda / (sg[0] * sg[1]);
        c[4] = lambda / (sg[0] * sg[2]);
        c[5] = lambda / (sg[1] * sg[2]);
        c[6] = -(lambda * sum_log + T(2) * mu * diff_interlock_log_over_diff(sg[0], sg[1], L1, eps)) / (sg[0] * sg[1]);
        c[7] = -(lambda * sum_log + T(2) * mu * diff_interlock_log_over_diff(sg[0], sg[2], L2, eps)) / (sg[0] * sg[2]);
        c[8] = -(lambda * sum_log + T(2) * mu * diff_interlock_log_over_diff(sg[1], sg[2], L2, eps)) / (sg[1] * sg[2]);
    }
    else {
        // fixed corotated: psi-hat = mu sum (s_i - 1)^2 + lambda/2 (J - 1)^2
        T J = sg[0] * sg[1] * sg[2];
        T c0 = sg[1] * sg[2], c1 = sg[0] * sg[2], c2 = sg[0] * sg[1];
        psi[0] = T(2) * mu * (sg[0] - T(1)) + lambda * (J - T(1)) * c0;
        psi[1] = T(2) * mu * (sg[1] - T(1)) + lambda * (J - T(1)) * c1;
        psi[2] = T(2) * mu * (sg[2] - T(1)) + lambda * (J - T(1)) * c2;
        c[0] = T(2) * mu + lambda * c0 * c0;
        c[1] = T(2) * mu + lambda * c1 * c1;
        c[2] = T(2) * mu + lambda * c2 * c2;
        c[3] = lambda * sg[2] * (T(2) * J - T(1));
        c[4] = lambda * sg[1] * (T(2) * J - T(1));
        c[5] = lambda * sg[0] * (T(2) * J - T(1));
        c[6] = T(2) * mu - lambda * (J - T(1)) * sg[2];
        c[7] = T(2) * mu - lambda * (J - T(1)) * sg[1];
        c[8] = T(2) * mu - lambda * (J - T(1)) * sg[0];
    }
    c[9] = (psi[0] + psi[1]) / clamp_small_magnitude(sg[0] + sg[1], eps);
    c[10] = (psi[0] + psi[2]) / clamp_small_magnitude(sg[0] + sg[2], eps);
    c[11] = (psi[1] + psi[2]) / clamp_small_magnitude(sg[1] + sg[2], eps);
}

// Kirchhoff stress of NeoHookeanBorden (NeoHookeanBorden.cpp:67-83) and
// P = tau F^{-T} (HyperelasticConstitutiveModel.h:85-90).
template <class T>
ZMPM_HD M3<T> nh_first_piola(T mu, T kappa, T g, T J, const M3<T>& F, const M3<T>& FinvT)
{
    M3<T> B = m3_mulT(F, F);
    T tr = B(0, 0) + B(1, 1) + B(2, 2);
    T sdev = mu * pow(J, -T(2) / T(3));
    T vol = J * (kappa / T(2) * (J - T(1) / J));
    M3<T> tau;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T dv = (i == j) ? B(i, j) - T(1) / T(3) * tr : B(i, j);
            T td = sdev * dv;
            T tv = (i == j) ? vol : T(0);
            tau(i, j) = (J >= T(1)) ? g * (td + tv) : g * td + tv;
        }
    return m3_mul(tau, FinvT);
}

// Computes S = V0 P(F) Fn^T and writes the Hessian scratch of particle p.
// With `degenerate` set (FP32 evaluation), SVD-based models stop after the
// SVD and report whether the singular values are too close to inversion
// (|sigma2| <= 0.2) or too stretched (sigma0 >= 5) for FP32; the caller then
// re-evaluates the particle in FP64.
template <class T, class TH>
ZMPM_D M3<T> model_update(int kind, const ModelParams& mp, T V0, const M3<T>& F, const M3<T>& Fn, TH* __restrict__ scr,
    int64_t stride, int64_t p, bool* degenerate = nullptr)
{
    if (kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        T J = m3_det(F);
        M3<T> FinvT = m3_cofactor(F);
#pragma unroll
        for (int i = 0; i < 9; ++i) FinvT.a[i] *= T(1) / J;
        T mu = (T)mp.mu, kappa = (T)mp.kappa, g = (T)mp.g;
        M3<T> P = nh_first_piola(mu, kappa, g, J, F, FinvT);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            scr[i * stride + p] = (TH)F.a[i];
            scr[(9 + i) * stride + p] = (TH)FinvT.a[i];
            scr[(18 + i) * stride + p] = (TH)Fn.a[i];
        }
        scr[27 * stride + p] = (TH)J;
        scr[28 * stride + p] = (TH)(mu * pow(J, T(2) * (-T(1) / T(3))));
        scr[29 * stride + p] = (TH)(kappa / T(2) * (J - T(1) / J));
        scr[30 * stride + p] = (TH)(kappa / T(2) * (T(1) + T(1) / (J * J)));
        scr[31 * stride + p] = (TH)g;
        scr[32 * stride + p] = (TH)V0;
        scr[33 * stride + p] = (TH)m3_contract(F, F);
        M3<T> VP = P;
#pragma unroll
        for (int i = 0; i < 9; ++i) VP.a[i] *= V0;
        return m3_mulT(VP, Fn);
    }
    if (kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC || kind == ZMPM_MODEL_FIXED_COROTATED) {
        M3<T> U, V;
        T sg[3];
        svd3(F, U, sg, V);
        if (degenerate) {
            const bool bad = !(fabs(sg[2]) > T(0.2) && sg[0] < T(5));
            *degenerate = bad;
            if (bad) return m3_zero<T>();
        }
        T psi[3], c[12];
        iso_coefficients(kind, (T)mp.mu, (T)mp.lambda, sg, psi, c);
        M3<T> P = m3_udvt(U, psi, V);
        M3<T> W = m3_mul(Fn, V);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            scr[i * stride + p] = (TH)U.a[i];
            scr[(9 + i) * stride + p] = (TH)W.a[i];
        }
#pragma unroll
        for (int i = 0; i < 12; ++i) scr[(18 + i) * stride + p] = (TH)(c[i] * V0);
        M3<T> VP = P;
#pragma unroll
        for (int i = 0; i < 9; ++i) VP.a[i] *= V0;
        return m3_mulT(VP, Fn);
    }
    return m3_zero<T>();
}

// dS = V0 dP(G Fn) Fn^T from the stored scratch; G = grad(dv) at the particle.
template <class TH>
ZMPM_D M3<TH> model_hvp(int kind, const TH* __restrict__ scr, int64_t stride, int64_t p, const M3<TH>& G)
{
    if (kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
        M3<TH> F, FinvT, Fn;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            F.a[i] = scr[i * stride + p];
            FinvT.a[i] = scr[(9 + i) * stride + p];
            Fn.a[i] = scr[(18 + i) * stride + p];
        }
        TH J = scr[27 * stride + p], muJ2a = scr[28 * stride + p], prime = scr[29 * stride + p];
        TH prime2 = scr[30 * stride + p], g = scr[31 * stride + p], V0 = scr[32 * stride + p];
        TH FcF = scr[33 * stride + p];
        M3<TH> dF = m3_mul(G, Fn);
        // NeoHookeanBorden::firstPiolaDifferential, NeoHookeanBorden.cpp:85-111
        TH FinvT_dF = m3_contract(FinvT, dF);
        TH deltaJ = J * FinvT_dF;
        M3<TH> dFinvT = m3_mul(m3_mulT(FinvT, dF), FinvT); // F^{-T} dF^T F^{-T}
        TH a = -TH(1) / TH(3);
        TH F_dF = m3_contract(F, dF);
        M3<TH> dP;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            TH dfi = -dFinvT.a[i];
            TH dev = TH(2) * a * muJ2a * FinvT_dF * (a * FcF * FinvT.a[i] + F.a[i]);
            dev += muJ2a * (TH(2) * a * F_dF * FinvT.a[i] + a * FcF * dfi + dF.a[i]);
            TH vol = deltaJ * prime * FinvT.a[i] + J * deltaJ * prime2 * FinvT.a[i] + J * prime * dfi;
            dP.a[i] = ((J >= TH(1)) ? g * (dev + vol) : g * dev + vol) * V0;
        }
        return m3_mulT(dP, Fn);
    }
    if (kind == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC || kind == ZMPM_MODEL_FIXED_COROTATED) {
        M3<TH> U, W;
        TH c[12];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            U.a[i] = scr[i * stride + p];
            W.a[i] = scr[(9 + i) * stride + p];
        }
#pragma unroll
        for (int i = 0; i < 12; ++i) c[i] = scr[(18 + i) * stride + p];
        M3<TH> D = m3_mul(m3_Tmul(U, G), W);
        M3<TH> K = iso_contract(c, D);
        return m3_mulT(m3_mul(U, K), W);
    }
    return m3_zero<TH>();
}

// VonMisesStvkHencky::projectStrain, Lib/Ziran/Physics/PlasticityApplier.cpp:462-502,
// on F = U diag(sg) V^T; updates F, the yield stress and the broken flag.
template <class T>
ZMPM_D void von_mises_from_svd(T mu, T lambda, T& yield_stress, T xi, T fail_stress, int& broken, T crack[3], M3<T>& F, const M3<T>& U,
    const T sg[3], const M3<T>& V)
{
    T e[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) e[d] = log(sg[d] > T(1e-4) ? sg[d] : T(1e-4));
    T tr = e[0] + e[1] + e[2];
    T h[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) h[d] = e[d] - (tr / T(3));
    T hn = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    T dg = hn - yield_stress / (T(2) * mu);
    if (dg <= T(0)) return;
    yield_stress -= xi * dg;
    T H[3], eH[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) H[d] = e[d] - (dg / hn) * h[d];
    T tau0 = T(2) * mu * H[0] + lambda * (H[0] + H[1] + H[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) eH[d] = exp(H[d]);
    F = m3_udvt(U, eH, V);
    if (tau0 >= fail_stress) {
        broken = 1;
#pragma unroll
        for (int d = 0; d < 3; ++d) crack[d] = V(d, 0);
    }
}

template <class T>
ZMPM_D void von_mises_project(T mu, T lambda, T& yield_stress, T xi, T fail_stress, int& broken, T crack[3], M3<T>& F)
{
    M3<T> U, V;
    T sg[3];
    svd3(F, U, sg, V);
    von_mises_from_svd(mu, lambda, yield_stress, xi, fail_stress, broken, crack, F, U, sg, V);
}

// Adjoint of von_mises_project (perfect plasticity, xi = 0) at the trial
// strain Fp: given Gb = dL/dF of the projected F, returns dL/dFp, and adds
// dL/dE to *gE (the yield radius r = yield_stress / (2 mu) scales as 1/E at
// fixed Poisson ratio).  Inside the yield surface the map is the identity.
// Outside, the projected singular values are f_i = exp(tr(eps)/3 + r n_i)
// with eps_i = log max(sigma_i, 1e-4) and n the unit deviatoric direction, an
// isotropic function of Fp: with A = U^T Gb V the adjoint is
// U Abar V^T, Abar_jj = sum_i (df_i/dsigma_j) A_ii and, off the diagonal,
// (f_i - f_j)/(sigma_i - sigma_j) on the symmetric part and (f_i + f_j) /
// (sigma_i + sigma_j) on the antisymmetric part of A (both self-adjoint; the
// first taken at its limit for equal singular values).  The map is not
// differentiable on the yield surface itself (dgamma = 0).
template <class T>
ZMPM_D M3<T> von_mises_adjoint(T mu, T yield_stress, T E, const M3<T>& Fp, const M3<T>& Gb, T* gE)
{
    M3<T> U, V;
    T sg[3];
    svd3(Fp, U, sg, V);
    T e[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) e[d] = log(sg[d] > T(1e-4) ? sg[d] : T(1e-4));
    const T tr = e[0] + e[1] + e[2];
    T h[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) h[d] = e[d] - tr / T(3);
    const T hn = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    const T r = yield_stress / (T(2) * mu);
    if (!(hn - r > T(0))) return Gb;
    T n[3], f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        n[d] = h[d] / hn;
        f[d] = exp(tr / T(3) + r * n[d]);
    }
    T J[3][3]; // df_i / dsigma_j
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const T dn = ((i == j ? T(1) : T(0)) - T(1) / T(3) - n[i] * n[j]) / hn;
            J[i][j] = sg[j] > T(1e-4) ? f[i] * (T(1) / T(3) + r * dn) / sg[j] : T(0);
        }
    const M3<T> A = m3_mul(m3_Tmul(U, Gb), V);
    M3<T> Ab;
#pragma unroll
    for (int j = 0; j < 3; ++j) Ab(j, j) = J[0][j] * A(0, 0) + J[1][j] * A(1, 1) + J[2][j] * A(2, 2);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (i == j) continue;
            const T ds = sg[i] - sg[j];
            const T a = fabs(ds) > T(1e-12) * fabs(sg[0]) ? (f[i] - f[j]) / ds : J[i][i] - J[i][j];
            const T b = (f[i] + f[j]) / (sg[i] + sg[j]);
            Ab(i, j) = a * (A(i, j) + A(j, i)) / T(2) + b * (A(i, j) - A(j, i)) / T(2);
        }
    // dL/dr = sum_i A_ii f_i n_i, dr/dE = -r / E
    *gE += -(r / E) * (A(0, 0) * f[0] * n[0] + A(1, 1) * f[1] * n[1] + A(2, 2) * f[2] * n[2]);
    return m3_mulT(m3_mul(U, Ab), V);
}

// DruckerPragerStvkHencky::projectStrain (PlasticityApplier.cpp:272-317):
// Hencky strain of the SVD less the cohesion; the trace with log Jp >= 0 sends
// F to the cone tip exp(cohesion) U V^T (and, with the volume correction, the
// excess volume into log Jp), else log Jp = 0 and the strain is projected onto
// the cone of friction coefficient alpha.
template <class T>
ZMPM_D void drucker_prager_project(T mu, T lambda, T alpha, T beta, T cohesion, int volume_correction, T& logJp, M3<T>& F)
{
    M3<T> U, V;
    T sg[3];
    svd3(F, U, sg, V);
    T e[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T a = fabs(sg[d]);
        e[d] = log(a > T(1e-4) ? a : T(1e-4)) - cohesion;
    }
    const T esum = e[0] + e[1] + e[2];
    const T tr = esum + logJp;
    T h[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) h[d] = e[d] - (tr / T(3));
    const T h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
    if (tr >= T(0)) {
        const T ec = exp(cohesion);
        const T one[3] = { ec, ec, ec };
        F = m3_udvt(U, one, V);
        if (volume_correction) logJp = beta * esum + logJp;
        return;
    }
    if (mu == T(0)) return;
    logJp = T(0);
    const T hn = sqrt(h2);
    const T dg = hn + (T(3) * lambda + T(2) * mu) / (T(2) * mu) * tr * alpha;
    T eH[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) eH[d] = exp((dg <= T(0)) ? e[d] + cohesion : e[d] - (dg / hn) * h[d] + cohesion);
    F = m3_udvt(U, eH, V);
}

// NonAssociativeCamClay::projectStrain (PlasticityApplier.cpp:112-136) through
// Compare_With_Physbam (:35-110), the branch the reference runs: pressure
// p = -kappa/2 (J - 1/J) J and deviatoric s of the SVD; tips beyond p0 and
// -beta p0; outside the ellipse a (s:s) + M^2 (p + beta p0)(p - p0) <= 1e-4 the
// deviatoric part is scaled onto it, and log Jp takes the "fake hardening"
// step towards the ellipse centre.  Inside, F is rebuilt from its SVD.
template <class T>
ZMPM_D void cam_clay_project(T mu, T kappa, T M, T beta, T xi, T& logJp, M3<T>& F)
{
    M3<T> U, V;
    T Se[3];
    svd3(F, U, Se, V);
    const T nl = -logJp;
    const T p0 = kappa * (T(0.00001) + sinh(xi * (nl > T(0) ? nl : T(0))));
    const T a = (T(1) + T(2) * beta) * (T(6) - T(3)) / T(2);
    const T b = beta * p0, c = p0, M2 = M * M;
    T Je = T(1);
#pragma unroll
    for (int i = 0; i < 3; ++i) Je *= Se[i];
    T Se2[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) Se2[i] = Se[i] * Se[i];
    T mean = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) mean += Se2[i];
    mean /= T(3);
    const T sc = mu * pow(Je, -T(2) / T(3));
    T s[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = sc * (Se2[i] - mean);
    const T p_trial = -(kappa / T(2) * (Je - T(1) / Je)) * Je;
    if (p_trial > c || p_trial < -b) {
        const T Je_new = (p_trial > c) ? sqrt(-T(2) * c / kappa + T(1)) : sqrt(T(2) * b / kappa + T(1));
        const T r = pow(Je_new, T(1) / T(3));
        const T rr[3] = { r, r, r };
        logJp += log(Je / Je_new);
        F = m3_udvt(U, rr, V);
        return;
    }
    const T k = sqrt(-M2 * (p_trial + b) * (p_trial - c) / a);
    const T sn = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    const T y = a * (sn * sn) + M2 * (p_trial + b) * (p_trial - c);
    if (y < T(1e-4)) {
        F = m3_udvt(U, Se, V);
        return;
    }
    const T pc = (T(1) - beta) * p0 / T(2);
    if (p0 > T(1e-4) && p_trial < p0 - T(1e-4) && p_trial > -beta * p0 + T(1e-4)) {
        const T aa = M2 * ((p_trial - pc) * (p_trial - pc)) / (a * (sn * sn));
        const T dd = T(1) + aa;
        const T ff = aa * beta * p0 - aa * p0 - T(2) * pc;
        const T gg = pc * pc - aa * beta * (p0 * p0);
        const T zz = sqrt(fabs(ff * ff - T(4) * dd * gg));
        const T p1 = (-ff + zz) / (T(2) * dd);
        const T p2 = (-ff - zz) / (T(2) * dd);
        const T p_fake = (p_trial - pc) * (p1 - pc) > T(0) ? p1 : p2;
        const T Je_new_fake = sqrt(fabs(-T(2) * p_fake / kappa + T(1)));
        if (Je_new_fake > T(1e-4)) logJp += log(Je / Je_new_fake);
    }
    const T g = k / mu * pow(Je, T(2) / T(3));
    const T tr = T(1) / T(3) * (Se2[0] + Se2[1] + Se2[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) Se[i] = sqrt(g * s[i] / sn + tr);
    F = m3_udvt(U, Se, V);
}

} // namespace zmpm
