// Particle <-> grid transfers of the implicit substep (helpers in xfer.cuh).
//
// Kernels
//  k_p2g_reg particlesToGridHelper<APIC> (MpmSimulationBase.cpp:563-608)
//  k_stress  MpmForceBase::updatePositionBasedState (MpmForceBase.cpp:306-344):
//            G2P of grad(vn+dv), F = (I + dt grad v) Fn, stress and Hessian scratch
//            (the FP64 evaluation of a MIXED solve whose FP32 residual stalled)
//  k_force   rasterizeForceToTVStack (MpmForceBase.cpp:102-152); also the
//            explicit substep's and ADMM's force scatter
//  k_update_fused  updatePositionBasedState + rasterizeForceToTVStack in one
//            pass (gather of grad v, F, stress and Hessian scratch, force scatter)
//  k_hvp_fused  MpmForceBase::addScaledForceDifferential (MpmForceBase.cpp:259-302):
//            G2P of grad(dv), dS = V0 dP Fn^T, P2G of dS grad w in one pass
//  k_op_fused  ADMM's global operator in the same one-pass form
//  k_g2p     gridToParticlesHelper<APIC> (MpmSimulationBase.cpp:906-1016) +
//            evolveStrain + applyPlasticity (:1018-1030)
#include "admm.cuh"
#include "eig3.cuh"
#include "fused.cuh"
#include "hvp.cuh"
#include "xfer.cuh"

namespace zmpm {

// ------------------------------------------------------------------ P2G ----
// Also writes each particle's fractional cell offsets (frac) for the FP32 HVP.
// P2G with per-cell register accumulation: thread -> one cell of the page and
// every (blockDim/NPB)-th particle of it; NCP of the four grid components
// (mass, momentum x, y, z) are summed for the cell's 27 stencil nodes in
// registers per pass and added to the shared window once per pass, so the
// window sees one atomic per (thread, node, component) instead of one per
// (particle, node, component).  APIC P2G: m_i += w m_p, (mv)_i += w m_p (v_p +
// C_p (x_i - x_p)), in FP64 or, in MIXED contexts, FP32 (the grid sums are
// FP64 in global memory either way).
template <class L, class TH, int NCP>
__global__ void __launch_bounds__(XF_THREADS, 3) k_p2g_reg(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, double* __restrict__ gm, double* __restrict__ gmv,
    TH* __restrict__ frac)
{
    using TA = TH; // arithmetic: FP64, or FP32 in MIXED contexts (the stored fractions' type)
    constexpr int NPB = L::NPB;
    __shared__ __align__(16) TA acc[8 * 4 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<4, NPB>(acc);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    const int ce = threadIdx.x % NPB;
    const int lx = ce >> (L::YB + L::ZB), ly = (ce >> L::ZB) & (L::BY - 1), lz = ce & (L::BZ - 1);
    const int cnt = cl.cnt[ce], first = s0 + cl.start[ce];
    const TA tdx = TA(dx);
#pragma unroll 1
    for (int c0 = 0; c0 < 4; c0 += NCP) {
        TA a[27][NCP];
#pragma unroll
        for (int n = 0; n < 27; ++n)
#pragma unroll
            for (int c = 0; c < NCP; ++c) a[n][c] = TA(0);
        for (int r = threadIdx.x / NPB; r < cnt; r += blockDim.x / NPB) {
            const int s = first + r;
            const short4 b = base[s];
            double xp[3];
            TA fr[3], w[3][3], dwr[3][3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                xp[d] = pd[(PD_X + d) * cap + s];
                const double d0 = inv_dx * xp[d] - (double)((&b.x)[d]);
                if (c0 == 0) frac[d * cap + s] = (TH)d0;
                fr[d] = (TA)d0;
                bspline(fr[d], w[d], dwr[d]);
            }
            const double mass = pd[PD_M * cap + s];
            TA mom[NCP], Cm[NCP][3];
#pragma unroll
            for (int c = 0; c < NCP; ++c) {
                const int comp = c0 + c; // 0: mass, 1..3: momentum row comp-1
                if (comp == 0) {
                    mom[c] = (TA)mass;
                    Cm[c][0] = Cm[c][1] = Cm[c][2] = TA(0);
                }
                else {
                    const int rr = comp - 1;
                    mom[c] = (TA)(mass * pd[(PD_V + rr) * cap + s]);
#pragma unroll
                    for (int q = 0; q < 3; ++q) Cm[c][q] = (TA)(mass * pd[(PD_C + 3 * rr + q) * cap + s]);
                }
            }
            for_stencil<L>(lx, ly, lz, w, dwr, TA(inv_dx), [&](int, int, int i, int j, int k, TA wijk, const TA*) {
                // x_i - x_p: FP64 from the positions, FP32 from the cell fractions
                TA xi[3];
                if constexpr (sizeof(TA) == 8) {
                    xi[0] = (b.x + i) * dx - xp[0];
                    xi[1] = (b.y + j) * dx - xp[1];
                    xi[2] = (b.z + k) * dx - xp[2];
                }
                else {
                    xi[0] = (TA(i) - fr[0]) * tdx;
                    xi[1] = (TA(j) - fr[1]) * tdx;
                    xi[2] = (TA(k) - fr[2]) * tdx;
                }
                const int n = 9 * i + 3 * j + k;
#pragma unroll
                for (int c = 0; c < NCP; ++c) a[n][c] += (Cm[c][0] * xi[0] + Cm[c][1] * xi[1] + Cm[c][2] * xi[2] + mom[c]) * wijk;
            });
        }
        if (threadIdx.x / NPB < cnt) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        int e;
                        const int t = win_slot<L>(lx + i, ly + j, lz + k, e);
                        TA* dst = acc + t * 4 * NPB + e;
#pragma unroll
                        for (int c = 0; c < NCP; ++c) atomicAdd(dst + (c0 + c) * NPB, a[9 * i + 3 * j + k][c]);
                    }
        }
    }
    __syncthreads();
    flush_window<4, 1, NPB>(acc, nbr, gm, gmv);
}

// APIC P2G as a fused per-page kernel (fused.cuh): phase 1 writes each
// particle's cell fractions (also to `frac`, for the Newton kernels), its mass
// and the affine form of its momentum; phase 2 (scatter_p2g) sums them into the
// window by (component, occupied cell) items.  T: arithmetic (FP32 in MIXED
// contexts); the window is flushed into the FP64 grid sums.
template <class L, class T, int CH>
__global__ void __launch_bounds__(FUSED_THREADS) k_p2g_fused(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, double* __restrict__ gm, double* __restrict__ gmv,
    T* __restrict__ frac)
{
    constexpr int NPB = L::NPB;
    using SM = ScatterSmem<L, T, CH, 16, 4>;
    __shared__ SM sm;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) sm.nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<4, NPB>(sm.acc);
    const int s0 = group_start[g], n = group_start[g + 1] - s0;
    build_cell_layout<L>(sm.cl, base, s0, s0 + n);
    list_occupied(sm);
    const double inv_dx = 1.0 / dx;
    const T tdx = T(dx);
    for (int c0 = 0; c0 < n; c0 += CH) {
        const int c1 = c0 + CH < n ? c0 + CH : n;
        __syncthreads();
        for (int p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
            const int64_t s = s0 + p;
            T* rc = sm.rec + (p - c0);
            const short4 b = base[s];
            T fr[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double d0 = inv_dx * pd[(PD_X + d) * cap + s] - (double)((&b.x)[d]);
                fr[d] = (T)d0;
                frac[d * cap + s] = fr[d];
                rc[d * SM::FS] = fr[d];
            }
            const double mass = pd[PD_M * cap + s];
            rc[3 * SM::FS] = (T)mass;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                T mC[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) mC[q] = (T)(mass * pd[(PD_C + 3 * r + q) * cap + s]);
                const T mv = (T)(mass * pd[(PD_V + r) * cap + s]);
                rc[(4 + 4 * r) * SM::FS] = mv - tdx * (mC[0] * fr[0] + mC[1] * fr[1] + mC[2] * fr[2]);
#pragma unroll
                for (int q = 0; q < 3; ++q) rc[(5 + 4 * r + q) * SM::FS] = tdx * mC[q];
            }
        }
        __syncthreads();
        scatter_p2g(sm, c0, c1);
    }
    __syncthreads();
    flush_window<4, 1, NPB>(sm.acc, sm.nbr, gm, gmv);
}

// -------------------------------------------------------------- damage -----
// Largest eigenvalue of a symmetric 3x3 matrix by the trigonometric solution
// of the characteristic cubic (O. K. Smith, "Eigenvalues of a symmetric 3x3
// matrix", CACM 4(4), 1961).
__device__ __forceinline__ double sym3_max_eig(const M3<double>& A)
{
    const double p1 = A(0, 1) * A(0, 1) + A(0, 2) * A(0, 2) + A(1, 2) * A(1, 2);
    const double q = (A(0, 0) + A(1, 1) + A(2, 2)) / 3.0;
    const double a = A(0, 0) - q, b = A(1, 1) - q, c = A(2, 2) - q;
    const double p2 = a * a + b * b + c * c + 2.0 * p1;
    if (p2 == 0.0) return q;
    const double p = sqrt(p2 / 6.0);
    M3<double> B = A;
    B(0, 0) = a;
    B(1, 1) = b;
    B(2, 2) = c;
#pragma unroll
    for (int i = 0; i < 9; ++i) B.a[i] /= p;
    double r = m3_det(B) / 2.0;
    r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
    const double phi = acos(r) / 3.0;
    return q + 2.0 * p * cos(phi);
}

// FractureSimulation::solvePhaseFieldSystemNaive (FractureSimulation.h:509-554)
// for particles with Rankine damage and NeoHookeanBorden: Cauchy stress of the
// undegraded (g = 1) Kirchhoff stress, c <- min(c, sigma_F / sigma_max) when
// sigma_max > sigma_F, g = c^2 (1 - k) + k.  sigma_max: the largest eigenvalue
// (ZMPM_DAMAGE_RANKINE) or the reference's first eigenvalue of Eigen's general
// eigensolver (ZMPM_DAMAGE_RANKINE_REFERENCE, eig3.cuh); first_not_max counts
// the particles of the latter whose first eigenvalue is not the largest.
__global__ void k_rankine(double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, int64_t P,
    unsigned long long* __restrict__ first_not_max)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P) return;
    const int dkind = pi[PI_DAMAGE * cap + s];
    if ((dkind != ZMPM_DAMAGE_RANKINE && dkind != ZMPM_DAMAGE_RANKINE_REFERENCE) || pi[PI_KIND * cap + s] != ZMPM_MODEL_NEOHOOKEAN_BORDEN) return;
    M3<double> F;
#pragma unroll
    for (int q = 0; q < 9; ++q) F.a[q] = pd[(PD_F + q) * cap + s];
    const double J = m3_det(F);
    const double mu = pd[PD_MU * cap + s], kappa = pd[PD_KAPPA * cap + s];
    // NeoHookeanBorden::kirchhoff with g = 1 (NeoHookeanBorden.cpp:67-83)
    M3<double> B = m3_mulT(F, F);
    const double tr = B(0, 0) + B(1, 1) + B(2, 2);
    const double sdev = mu * pow(J, -2.0 / 3.0);
    const double vol = J * (kappa / 2 * (J - 1 / J));
    M3<double> cauchy;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const double dv = (i == j) ? B(i, j) - 1.0 / 3.0 * tr : B(i, j);
            cauchy(i, j) = ((i == j) ? sdev * dv + vol : sdev * dv) / J;
        }
    double sigma_max = sym3_max_eig(cauchy);
    if (dkind == ZMPM_DAMAGE_RANKINE_REFERENCE) {
        Eig3 eig;
        const double first = eig.first_eigenvalue(cauchy.a);
        if (!(fabs(first - sigma_max) <= 1e-9 * fabs(sigma_max))) atomicAdd(first_not_max, 1ull);
        sigma_max = first;
    }
    const double sigma_f = pd[PD_SIGMA_F * cap + s];
    double c = pd[PD_PF_C * cap + s];
    const double k = pd[PD_PF_K * cap + s];
    if (sigma_max > sigma_f) c = fmin(c, sigma_f / sigma_max);
    pd[PD_PF_C * cap + s] = c;
    pd[PD_G * cap + s] = c * c * (1 - k) + k;
}

int launch_damage(Ctx* ctx)
{
    if (!ctx->has_damage || ctx->P == 0) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    k_rankine<<<(unsigned)((ctx->P + 255) / 256), 256, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->P,
        reinterpret_cast<unsigned long long*>(&dc->first_not_max));
    ++g_kernel_launches;
    return ZMPM_OK;
}

// --------------------------------------------------------------- update ----
// Two kernels per Newton iteration (MpmForceBase::updatePositionBasedState then
// rasterizeForceToTVStack, MpmForceBase.cpp:306-344, 102-152):
//  k_stress: grad v at the particle from vstar = vn + dv, F = (I + dt grad v) Fn,
//            S = V0 P(F) Fn^T (to `stress`) and the Hessian scratch; particles in
//            slot order so every particle array is read coalesced.
//  k_force : facc -= sum_p S_p grad w_ip, layered conflict-free scatter.
// gate (MIXED contexts, which launch an FP32 and an FP64 pair of k_stress /
// k_force per Newton iteration): 0 always runs, 1 runs while the solve's
// residual is FP32, 2 once it is FP64.  frac_x: B-spline weights from the FP64
// positions instead of the stored fractions (the FP64 residual of MIXED).
__device__ __forceinline__ bool gated_off(const SolverScalars* sc, int gate)
{
    return sc && (sc->newton_done || (gate != 0 && (gate == 1) == (sc->fp64_res != 0)));
}

template <class L, class TS, class TH>
__global__ void __launch_bounds__(XF_THREADS) k_stress(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, double dt,
    const TH* __restrict__ frac, const double* __restrict__ vstar, TS* __restrict__ stress, TH* __restrict__ scr,
    const SolverScalars* __restrict__ sc, int32_t* __restrict__ flags, int gate, int frac_x)
{
    if (gated_off(sc, gate)) return;
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(win, vstar, nbr, &bar, flags);
    const TS inv_dx = TS(1.0 / dx);
    const TS tdt = TS(dt);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const int kind = pi[PI_KIND * cap + s];
        if (kind == ZMPM_MODEL_NONE) {
#pragma unroll
            for (int q = 0; q < 9; ++q) stress[q * cap + s] = TS(0);
            continue;
        }
        const short4 b = base[s];
        TS w[3][3], dwr[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            bspline(frac_x ? (TS)((1.0 / dx) * pd[(PD_X + d) * cap + s] - (double)((&b.x)[d])) : (TS)frac[d * cap + s], w[d], dwr[d]);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        M3<TS> gv = m3_zero<TS>();
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, TS, const TS* dw) {
            const double* vv = win + t * 3 * NPB + e;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                TS vr = (TS)vv[r * NPB];
#pragma unroll
                for (int c = 0; c < 3; ++c) gv(r, c) += vr * dw[c];
            }
        });
        M3<TS> Fn, A = m3_identity<TS>();
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            Fn.a[q] = (TS)pd[(PD_F + q) * cap + s];
            A.a[q] += tdt * gv.a[q];
        }
        M3<TS> F = m3_mul(A, Fn);
        ModelParams mp{ pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_KAPPA * cap + s], pd[PD_G * cap + s] };
        const double V0 = pd[PD_VOL * cap + s];
        bool degenerate = false;
        M3<TS> S = model_update<TS, TH>(kind, mp, (TS)V0, F, Fn, scr, cap, s, sizeof(TS) == 4 ? &degenerate : nullptr);
        if constexpr (sizeof(TS) == 4) {
            if (degenerate) { // FP64 re-evaluation of near-degenerate particles
                M3<double> Fnd, Ad = m3_identity<double>();
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    Fnd.a[q] = pd[(PD_F + q) * cap + s];
                    Ad.a[q] += dt * (double)gv.a[q];
                }
                S = m3_cast<TS>(model_update<double, TH>(kind, mp, V0, m3_mul(Ad, Fnd), Fnd, scr, cap, s, nullptr));
            }
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) stress[q * cap + s] = S.a[q];
    }
}

// Explicit substep: FBasedMpmForceHelper::updateState (FBasedMpmForceHelper.cpp:
// 44-64) stores V0 tau(F) = V0 P(F) F^T per particle (slot order), plus V0
// tau(Fe) for viscoelastic particles (FElasticNonequilibratedBasedMpmForceHelper.h:
// 39-60).  TS precision with the FP64 re-evaluation of near-degenerate SVDs.
template <class TS, class TH>
__global__ void __launch_bounds__(XF_THREADS) k_explicit_stress(const double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap,
    int64_t P, TS* __restrict__ stress, TH* __restrict__ scr)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P) return;
    const int kind = pi[PI_KIND * cap + s];
    M3<TS> S = m3_zero<TS>();
    if (kind != ZMPM_MODEL_NONE) {
        M3<TS> F;
#pragma unroll
        for (int q = 0; q < 9; ++q) F.a[q] = (TS)pd[(PD_F + q) * cap + s];
        const ModelParams mp{ pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_KAPPA * cap + s], pd[PD_G * cap + s] };
        const double V0 = pd[PD_VOL * cap + s];
        bool degenerate = false;
        S = model_update<TS, TH>(kind, mp, (TS)V0, F, F, scr, cap, s, sizeof(TS) == 4 ? &degenerate : nullptr);
        if constexpr (sizeof(TS) == 4) {
            if (degenerate) {
                M3<double> Fd;
#pragma unroll
                for (int q = 0; q < 9; ++q) Fd.a[q] = pd[(PD_F + q) * cap + s];
                S = m3_cast<TS>(model_update<double, TH>(kind, mp, V0, Fd, Fd, scr, cap, s, nullptr));
            }
        }
        if (pi[PI_VISCO * cap + s]) {
            M3<double> Fe;
#pragma unroll
            for (int q = 0; q < 9; ++q) Fe.a[q] = pd[(PD_FE + q) * cap + s];
            const ModelParams mv{ pd[PD_VMU * cap + s], pd[PD_VLAM * cap + s], 0.0, 1.0 };
            const M3<double> Se = model_update<double, TH>(ZMPM_MODEL_STVK_HENCKY_ISOTROPIC, mv, V0, Fe, Fe, scr, cap, s, nullptr);
#pragma unroll
            for (int q = 0; q < 9; ++q) S.a[q] += (TS)Se.a[q];
        }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) stress[q * cap + s] = S.a[q];
}

int launch_explicit_stress(Ctx* ctx)
{
    const int64_t P = ctx->P;
    if (P == 0) return ZMPM_OK;
    const unsigned nb = (unsigned)((P + XF_THREADS - 1) / XF_THREADS);
    if (ctx->mixed)
        k_explicit_stress<float, float><<<nb, XF_THREADS, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, P,
            ctx->stress.as<float>(), ctx->scratch.as<float>());
    else
        k_explicit_stress<double, double><<<nb, XF_THREADS, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, P,
            ctx->stress.as<double>(), ctx->scratch.as<double>());
    ++g_kernel_launches;
    return ZMPM_OK;
}

// MLS = true: the MLS-MPM weight of particlesToGridWithForceHelper
// (MpmSimulationBase.cpp:527-541), facc -= (S_p (x_i - x_p)) w_ip D^-1 with
// D^-1 = 4 / dx^2, in place of S_p grad w_ip.
template <class L, class TS, class TH, bool MLS = false>
__global__ void __launch_bounds__(XF_THREADS) k_force(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    int64_t cap, const short4* __restrict__ base, double dx, const TH* __restrict__ frac, const TS* __restrict__ stress,
    double* __restrict__ facc, const SolverScalars* __restrict__ sc, int gate = 0, const double* __restrict__ xpos = nullptr)
{
    if (gated_off(sc, gate)) return;
    constexpr int NPB = L::NPB;
    __shared__ __align__(16) TS acc[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<3, NPB>(acc);
    const TS inv_dx = TS(1.0 / dx);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    // Thread -> one cell of the page and every (blockDim/NPB)-th particle of
    // it; the cell's particles share one 27-node stencil, so their terms are
    // summed in registers and added to the shared window once per thread (FP32
    // keeps all 81 sums in registers, FP64 one force component per pass).
    const int ce = threadIdx.x % NPB;
    const int lx = ce >> (L::YB + L::ZB), ly = (ce >> L::ZB) & (L::BY - 1), lz = ce & (L::BZ - 1);
    const int cnt = cl.cnt[ce], first = s0 + cl.start[ce];
    constexpr int NCP = sizeof(TS) == 4 ? 3 : 1;
#pragma unroll 1
    for (int c0 = 0; c0 < 3; c0 += NCP) {
        TS a[27][NCP];
#pragma unroll
        for (int n = 0; n < 27; ++n)
#pragma unroll
            for (int c = 0; c < NCP; ++c) a[n][c] = TS(0);
        for (int r = threadIdx.x / NPB; r < cnt; r += blockDim.x / NPB) {
            const int s = first + r;
            TS w[3][3], dwr[3][3], fr[3];
            if (xpos) {
                const short4 b = base[s];
#pragma unroll
                for (int d = 0; d < 3; ++d) fr[d] = (TS)((1.0 / dx) * xpos[d * cap + s] - (double)((&b.x)[d]));
            }
            else
#pragma unroll
                for (int d = 0; d < 3; ++d) fr[d] = (TS)frac[d * cap + s];
#pragma unroll
            for (int d = 0; d < 3; ++d) bspline(fr[d], w[d], dwr[d]);
            TS row[NCP][3];
#pragma unroll
            for (int c = 0; c < NCP; ++c)
#pragma unroll
                for (int q2 = 0; q2 < 3; ++q2) row[c][q2] = stress[(3 * (c0 + c) + q2) * cap + s];
            if constexpr (MLS) {
                const TS tdx = (TS)dx, dinv = TS(4.0 / (dx * dx));
                for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int, int, int i, int j, int k, TS wijk, const TS*) {
                    const int n = 9 * i + 3 * j + k;
                    const TS xm[3] = { ((TS)i - fr[0]) * tdx, ((TS)j - fr[1]) * tdx, ((TS)k - fr[2]) * tdx };
                    const TS q = wijk * dinv;
#pragma unroll
                    for (int c = 0; c < NCP; ++c) a[n][c] -= (row[c][0] * xm[0] + row[c][1] * xm[1] + row[c][2] * xm[2]) * q;
                });
            }
            else
                for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int, int, int i, int j, int k, TS, const TS* dw) {
                    const int n = 9 * i + 3 * j + k;
#pragma unroll
                    for (int c = 0; c < NCP; ++c) a[n][c] -= row[c][0] * dw[0] + row[c][1] * dw[1] + row[c][2] * dw[2];
                });
        }
        if (threadIdx.x / NPB < cnt) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        int e;
                        const int t = win_slot<L>(lx + i, ly + j, lz + k, e);
#pragma unroll
                        for (int c = 0; c < NCP; ++c) atomicAdd(acc + t * 3 * NPB + (c0 + c) * NPB + e, a[9 * i + 3 * j + k][c]);
                    }
        }
    }
    __syncthreads();
    flush_window<3, 3, NPB>(acc, nbr, facc, nullptr);
}

// ------------------------------------------------------- fused products ----
// The Hessian-vector product (hvp.cuh) as one CTA per particle group (the
// zmpm_multiply hook; the solves run it inside their persistent kernels).
template <class L, class T, class TX, int CH>
__global__ void __launch_bounds__(FUSED_THREADS) k_hvp_fused(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, const T* __restrict__ frac,
    const T* __restrict__ scr, const TX* __restrict__ x, double* __restrict__ out, int32_t* __restrict__ flags)
{
    __shared__ HvpSmem<L, T, TX, CH> hs;
    const int g = blockIdx.x;
    hvp_group<L, T, TX, CH>(hs, g, group_start[g], group_start[g + 1], group_nbr, HvpModel<T>{ pi, scr, cap }, cap, base, dx, frac, x, out,
        flags);
}

// ADMM's global operator (the matrix-free product of dvStep's MINRES,
// AdmmSimulationFoam.h:167-170 with the B of initMultiplierAndPreconditioner):
// out += sum_p (grad(x)_p B_p) grad w_ip, one CTA per particle group.
template <class L, class T, int CH>
__global__ void __launch_bounds__(FUSED_THREADS) k_op_fused(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    int64_t cap, const short4* __restrict__ base, double dx, const T* __restrict__ frac, const T* __restrict__ B, const double* __restrict__ x,
    double* __restrict__ out, int32_t* __restrict__ flags)
{
    __shared__ HvpSmem<L, T, double, CH> hs;
    const int g = blockIdx.x;
    hvp_group<L, T, double, CH>(hs, g, group_start[g], group_start[g + 1], group_nbr, AdmmOpModel<T>{ B, cap }, cap, base, dx, frac, x, out,
        flags);
}

// MpmForceBase::updatePositionBasedState + rasterizeForceToTVStack
// (MpmForceBase.cpp:306-344, 102-152) in one kernel: phase 1 gathers grad(v)
// of vstar = vn + dv at each particle, F = (I + dt grad v) Fn (evolveStrain on
// the restored Fn, FBasedMpmForceHelper.cpp:95-109), S = V0 P(F) Fn^T and the
// Hessian scratch (updateImplicitState, :68-92); FP32 evaluations of
// near-degenerate SVDs are redone in FP64.  Phase 2 adds -S_p grad w_ip to
// facc.  gate as k_stress / k_force.
template <class L, class T, class TX, int CH>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_update_fused(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, double dt,
    const T* __restrict__ frac, const TX* __restrict__ vstar, T* __restrict__ scr, double* __restrict__ facc,
    const SolverScalars* __restrict__ sc, int32_t* __restrict__ flags, int gate, unsigned long long* __restrict__ svd64)
{
    if (gated_off(sc, gate)) return;
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) TX win[VecWindow<NPB, TX>::ELEMS];
    __shared__ ScatterSmem<L, T, CH> sm;
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) sm.nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<3, NPB>(sm.acc);
    __syncthreads();
    stage_vec_window<NPB, TX>(win, vstar, sm.nbr, &bar, flags);
    const int s0 = group_start[g], n = group_start[g + 1] - s0;
    build_cell_layout<L>(sm.cl, base, s0, s0 + n);
    list_occupied(sm);
    const T inv_dx = T(1.0 / dx);
    const T tdt = T(dt);
    for (int c0 = 0; c0 < n; c0 += CH) {
        const int c1 = c0 + CH < n ? c0 + CH : n;
        __syncthreads();
        for (int p = c0 + threadIdx.x; p < c1; p += blockDim.x) {
            const int64_t s = s0 + p;
            T* rc = sm.rec + (p - c0);
            T fr[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                fr[d] = frac[d * cap + s];
                rc[d * sm.FS] = fr[d];
            }
            const int kind = pi[PI_KIND * cap + s];
            M3<T> S = m3_zero<T>();
            if (kind != ZMPM_MODEL_NONE) {
                const short4 b = base[s];
                T w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all(fr[d], w[d], dw[d]);
                const StencilOffsets<L> so(b.x & (L::BX - 1), b.y & (L::BY - 1), b.z & (L::BZ - 1));
                M3<T> gv;
                if constexpr (sizeof(T) == 4 && sizeof(TX) == 4)
                    gather_gradient_f32<L>(win, so, w, dw, gv.a);
                else
                    gather_gradient<L, T, TX>(win, so, w, dw, gv.a);
                M3<T> Fn, A = m3_identity<T>();
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    Fn.a[q] = (T)pd[(PD_F + q) * cap + s];
                    A.a[q] += tdt * (gv.a[q] * inv_dx);
                }
                const ModelParams mp{ pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_KAPPA * cap + s], pd[PD_G * cap + s] };
                const double V0 = pd[PD_VOL * cap + s];
                bool degenerate = false;
                S = model_update<T, T>(kind, mp, (T)V0, m3_mul(A, Fn), Fn, scr, cap, s, sizeof(T) == 4 ? &degenerate : nullptr);
                if constexpr (sizeof(T) == 4) {
                    if (degenerate) { // FP64 re-evaluation of near-degenerate particles
                        atomicAdd(svd64, 1ull);
                        M3<double> Fnd, Ad = m3_identity<double>();
#pragma unroll
                        for (int q = 0; q < 9; ++q) {
                            Fnd.a[q] = pd[(PD_F + q) * cap + s];
                            Ad.a[q] += dt * ((double)gv.a[q] * (1.0 / dx));
                        }
                        S = m3_cast<T>(model_update<double, T>(kind, mp, V0, m3_mul(Ad, Fnd), Fnd, scr, cap, s, nullptr));
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) rc[(3 + 3 * r + c) * sm.FS] = -S(r, c) * inv_dx;
        }
        __syncthreads();
        scatter_rows(sm, c0, c1);
    }
    __syncthreads();
    flush_window<3, 3, NPB>(sm.acc, sm.nbr, facc, nullptr);
}

// chunk sizes: the particle records of a chunk fill 24 KB (FP32) / 18 KB (FP64), which keeps
// the static shared memory of a CTA below 48 KB
template <class T>
constexpr int fused_chunk() { return sizeof(T) == 4 ? 512 : 192; }

// ------------------------------------------------------------------ G2P ----
// MpmSimulationBase::applyPlasticity (MpmSimulationBase.cpp:1018-1030) on one
// particle (slot s): the return map of its plasticity kind applied to F, with
// the kind's state (log Jp; yield stress, broken flag and crack normal) updated
// in the pools.
__device__ __forceinline__ void apply_return_map(double* __restrict__ pd, int32_t* __restrict__ pi, int64_t cap, int64_t s, M3<double>& F)
{
    const int pkind = pi[PI_PKIND * cap + s];
    if (pkind == ZMPM_PLASTIC_DRUCKER_PRAGER || pkind == ZMPM_PLASTIC_CAM_CLAY) {
        double logJp = pd[PD_LOGJP * cap + s];
        if (pkind == ZMPM_PLASTIC_DRUCKER_PRAGER)
            drucker_prager_project<double>(pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_YS * cap + s], pd[PD_XI * cap + s],
                pd[PD_FS * cap + s], pi[PI_BROKEN * cap + s], logJp, F);
        else
            cam_clay_project<double>(pd[PD_MU * cap + s], pd[PD_KAPPA * cap + s], pd[PD_YS * cap + s], pd[PD_XI * cap + s],
                pd[PD_FS * cap + s], logJp, F);
        pd[PD_LOGJP * cap + s] = logJp;
    }
    if (pkind == ZMPM_PLASTIC_VON_MISES) {
        double ys = pd[PD_YS * cap + s];
        int broken = pi[PI_BROKEN * cap + s];
        double crack[3] = { pd[(PD_CRACK + 0) * cap + s], pd[(PD_CRACK + 1) * cap + s], pd[(PD_CRACK + 2) * cap + s] };
        von_mises_project<double>(pd[PD_MU * cap + s], pd[PD_LAM * cap + s], ys, pd[PD_XI * cap + s], pd[PD_FS * cap + s], broken, crack, F);
        pd[PD_YS * cap + s] = ys;
        pi[PI_BROKEN * cap + s] = broken;
#pragma unroll
        for (int d = 0; d < 3; ++d) pd[(PD_CRACK + d) * cap + s] = crack[d];
    }
}

// applyPlasticity as its own pass (slot order), for callers that run
// gridToParticles without it.
__global__ void k_plasticity(double* __restrict__ pd, int32_t* __restrict__ pi, int64_t cap, int64_t P)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P || pi[PI_KIND * cap + s] == ZMPM_MODEL_NONE || pi[PI_PKIND * cap + s] == ZMPM_PLASTIC_NONE) return;
    M3<double> F;
#pragma unroll
    for (int q = 0; q < 9; ++q) F.a[q] = pd[(PD_F + q) * cap + s];
    apply_return_map(pd, pi, cap, s, F);
#pragma unroll
    for (int q = 0; q < 9; ++q) pd[(PD_F + q) * cap + s] = F.a[q];
}

int launch_plasticity(Ctx* ctx)
{
    if (ctx->P == 0) return ZMPM_OK;
    k_plasticity<<<(unsigned)((ctx->P + 127) / 128), 128, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->P);
    ++g_kernel_launches;
    return ZMPM_OK;
}

// MIXED: applyPlasticity on an FP32 F.  Von Mises runs in FP32 on its FP32
// SVD unless the singular values are near inversion (|sigma2| <= 0.2) or
// strongly stretched (sigma0 >= 5), where it runs in FP64; the other return
// maps run in FP64.
__device__ __forceinline__ void apply_return_map_f32(double* __restrict__ pd, int32_t* __restrict__ pi, int64_t cap, int64_t s, M3<float>& F)
{
    const int pkind = pi[PI_PKIND * cap + s];
    if (pkind == ZMPM_PLASTIC_NONE) return;
    if (pkind == ZMPM_PLASTIC_VON_MISES) {
        M3<float> U, V;
        float sg[3];
        svd3(F, U, sg, V);
        if (fabsf(sg[2]) > 0.2f && sg[0] < 5.f) {
            float ys = (float)pd[PD_YS * cap + s];
            int broken = pi[PI_BROKEN * cap + s];
            float crack[3] = { (float)pd[(PD_CRACK + 0) * cap + s], (float)pd[(PD_CRACK + 1) * cap + s], (float)pd[(PD_CRACK + 2) * cap + s] };
            const float ys0 = ys;
            const int broken0 = broken;
            von_mises_from_svd<float>((float)pd[PD_MU * cap + s], (float)pd[PD_LAM * cap + s], ys, (float)pd[PD_XI * cap + s],
                (float)pd[PD_FS * cap + s], broken, crack, F, U, sg, V);
            if (ys != ys0) pd[PD_YS * cap + s] = ys;
            if (broken != broken0) {
                pi[PI_BROKEN * cap + s] = broken;
#pragma unroll
                for (int d = 0; d < 3; ++d) pd[(PD_CRACK + d) * cap + s] = crack[d];
            }
            return;
        }
    }
    M3<double> Fd = m3_cast<double>(F);
    apply_return_map(pd, pi, cap, s, Fd);
    F = m3_cast<float>(Fd);
}

// gridToParticlesHelper<APIC> (MpmSimulationBase.cpp:906-1016): v_p = sum w v_i,
// B = sum w v_i (x_i - x_p)^T, C = ((1 + r) B D^-1 + (r - 1) (B D^-1)^T) / 2 with
// D^-1 = 4 / dx^2, grad v_p = sum v_i grad w^T, x_p += dt v_p and the CFL flag;
// then evolveStrain F = (I + dt grad v) Fn (FBasedMpmForceHelper.cpp:95-109, and
// the viscoelastic Fe's relaxation) and, with `plastic`, applyPlasticity.
// T: the arithmetic (FP32 in MIXED contexts: weights from the stored cell
// fractions, positions advanced in FP64).  FP64: three CTAs per SM (at most
// 168 registers; the form is latency bound on FP64 chains).  FP32: four (128
// registers, a few spilled words).
template <class L, class T, class TX>
__global__ void __launch_bounds__(XF_THREADS, sizeof(T) == 4 ? 4 : 3) k_g2p(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, const T* __restrict__ frac, double dx,
    double dt, double apic_rpic_ratio, const TX* __restrict__ vnew, int32_t* __restrict__ flags, int mls, int plastic)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) TX win[VecWindow<NPB, TX>::ELEMS];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_vec_window<NPB, TX>(win, vnew, nbr, &bar, flags);
    const T inv_dx = T(1.0 / dx), tdx = T(dx);
    const T D_inverse = T(4.0 / (dx * dx));
    const T ca = T((apic_rpic_ratio + 1) * 0.5), cb = T((apic_rpic_ratio - 1) * 0.5);
    const T tdt = T(dt);
    int too_fast = 0;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        T fr[3], w[3][3], dwr[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            fr[d] = frac[d * cap + s];
            bspline(fr[d], w[d], dwr[d]);
        }
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        const StencilOffsets<L> so(lx, ly, lz);
        T pv[3] = { 0, 0, 0 };
        M3<T> Bp = m3_zero<T>(), gv = m3_zero<T>();
        double xp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) xp[d] = pd[(PD_X + d) * cap + s];
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int, int, int i, int j, int k, T wijk, const T* dw) {
            TX vv[3];
            VecWindow<NPB, TX>::node(win, so.X[i] + so.Y[j] + so.Z[k], vv);
            // x_i - x_p: FP64 from the node and particle positions, FP32 from the cell fractions
            T xi[3];
            if constexpr (sizeof(T) == 8) {
                xi[0] = (b.x + i) * dx - xp[0];
                xi[1] = (b.y + j) * dx - xp[1];
                xi[2] = (b.z + k) * dx - xp[2];
            }
            else {
                xi[0] = (T(i) - fr[0]) * tdx;
                xi[1] = (T(j) - fr[1]) * tdx;
                xi[2] = (T(k) - fr[2]) * tdx;
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const T vr = (T)vv[r];
                pv[r] += wijk * vr;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    Bp(r, c) += wijk * vr * xi[c];
                    gv(r, c) += vr * dw[c];
                }
            }
        });
        double inc2 = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            pd[(PD_V + d) * cap + s] = pv[d];
            const double inc = dt * (double)pv[d];
            pd[(PD_X + d) * cap + s] = xp[d] + inc;
            inc2 += inc * inc;
        }
        too_fast |= (inc2 > dx * dx);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T cn = ca * (Bp(r, c) * D_inverse) + cb * (Bp(c, r) * D_inverse);
                pd[(PD_C + 3 * r + c) * cap + s] = cn;
                if (mls) gv(r, c) = cn; // MLS: gradVp = C_p (MpmSimulationBase.cpp:958-961)
            }
        const int kind = pi[PI_KIND * cap + s];
        if (kind == ZMPM_MODEL_NONE) continue;
        // evolveStrain (FBasedMpmForceHelper.cpp:95-109) on the restored F = Fn
        M3<T> F0, A = m3_identity<T>();
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            F0.a[q] = (T)pd[(PD_F + q) * cap + s];
            A.a[q] += tdt * gv.a[q];
        }
        M3<T> F = m3_mul(A, F0);
        if (plastic) {
            if constexpr (sizeof(T) == 8)
                apply_return_map(pd, pi, cap, s, F);
            else
                apply_return_map_f32(pd, pi, cap, s, F);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) pd[(PD_F + q) * cap + s] = F.a[q];
        if (pi[PI_VISCO * cap + s]) {
            // FElasticNonequilibratedBasedMpmForceHelper::evolveStrain (h:62-87), FP64
            M3<double> Fe;
#pragma unroll
            for (int q = 0; q < 9; ++q) Fe.a[q] = pd[(PD_FE + q) * cap + s];
            Fe = m3_mul(m3_cast<double>(A), Fe);
            viscous_return<double>(pd[PD_VMU * cap + s], pd[PD_VLAM * cap + s], pd[PD_VD * cap + s], pd[PD_VV * cap + s], dt, Fe);
#pragma unroll
            for (int q = 0; q < 9; ++q) pd[(PD_FE + q) * cap + s] = Fe.a[q];
        }
    }
    if (__syncthreads_or(too_fast) && threadIdx.x == 0) atomicOr(flags, (int32_t)FLAG_CFL);
}

// ------------------------------------------------------------- launchers --
template <class L>
static int p2g_impl(Ctx* ctx)
{
    const int64_t G = ctx->G;
    if (G == 0) return ZMPM_OK;
    if (ctx->mixed)
        k_p2g_fused<L, float, 384><<<(unsigned)G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->frac.as<float>());
    else
        k_p2g_reg<L, double, 2><<<(unsigned)G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->frac.as<double>());
    ++g_kernel_launches;
    return ZMPM_OK;
}
int launch_p2g(Ctx* ctx) { return ctx->layout == 1 ? p2g_impl<Layout244>(ctx) : p2g_impl<Layout444>(ctx); }

template <class L>
static int update_impl(Ctx* ctx, bool gated)
{
    const int64_t G = ctx->G;
    if (G == 0) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    const SolverScalars* sc = gated ? ctx->scal.as<SolverScalars>() : nullptr;
    if (ctx->mixed) {
        // FP32 stress and force; inside a solve also the FP64 pair, which runs
        // instead once the FP32 residual stalled (FP32 Hessian scratch either
        // way).  The FP32 pass gathers from the FP32 copy of vstar, which the
        // Newton solve keeps current; the hooks and the adjoint set vstar directly.
        const int gate = sc ? 1 : 0;
        if (!sc || !ctx->vstarf_valid) {
            int rc = refresh_vstar_f32(ctx);
            if (rc) return rc;
            ctx->vstarf_valid = true;
        }
        k_update_fused<L, float, float, fused_chunk<float>()><<<(unsigned)G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt,
            ctx->frac.as<float>(), ctx->vstarf.as<float>(), ctx->scratch.as<float>(), ctx->facc.as<double>(), sc, &dc->flags, gate,
            reinterpret_cast<unsigned long long*>(&dc->svd_fp64));
        ++g_kernel_launches;
        if (sc) {
            k_stress<L, double, float><<<(unsigned)G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
                ctx->group_nbr.as<int32_t>(), ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx,
                ctx->dt, ctx->frac.as<float>(), ctx->vstar.as<double>(), ctx->stress.as<double>(), ctx->scratch.as<float>(), sc, &dc->flags, 2,
                1);
            ++g_kernel_launches;
            k_force<L, double, float><<<(unsigned)G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
                ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<float>(), ctx->stress.as<double>(), ctx->facc.as<double>(), sc, 2,
                ctx->pd.as<double>() + PD_X * ctx->Pcap);
            ++g_kernel_launches;
        }
    }
    else {
        k_update_fused<L, double, double, fused_chunk<double>()><<<(unsigned)G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt,
            ctx->frac.as<double>(), ctx->vstar.as<double>(), ctx->scratch.as<double>(), ctx->facc.as<double>(), sc, &dc->flags, 0,
            reinterpret_cast<unsigned long long*>(&dc->svd_fp64));
        ++g_kernel_launches;
    }
    return ZMPM_OK;
}
int launch_update(Ctx* ctx, bool gated) { return ctx->layout == 1 ? update_impl<Layout244>(ctx, gated) : update_impl<Layout444>(ctx, gated); }

// out += dt^-2 (Hessian part of A) x: the fused product, T the context's HVP
// precision, on an FP64 input vector
template <class L>
static int hvp_impl(Ctx* ctx, const double* x, double* out)
{
    const int64_t G = ctx->G;
    if (G == 0) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    if (ctx->mixed)
        k_hvp_fused<L, float, double, fused_chunk<float>()><<<(unsigned)G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<float>(),
            ctx->scratch.as<float>(), x, out, &dc->flags);
    else
        k_hvp_fused<L, double, double, fused_chunk<double>()><<<(unsigned)G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<double>(),
            ctx->scratch.as<double>(), x, out, &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

int launch_hvp(Ctx* ctx, const double* x, double* out, bool fp32)
{
    if (fp32 != ctx->mixed) return ZMPM_UNSUPPORTED;
    return ctx->layout == 1 ? hvp_impl<Layout244>(ctx, x, out) : hvp_impl<Layout444>(ctx, x, out);
}

template <class L, class TH>
static int force_scatter_impl(Ctx* ctx, double* out, bool mls)
{
    if (mls)
        k_force<L, TH, TH, true><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<TH>(), ctx->stress.as<TH>(), out, nullptr);
    else
        k_force<L, TH, TH><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(), ctx->Pcap,
            ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<TH>(), ctx->stress.as<TH>(), out, nullptr);
    ++g_kernel_launches;
    return ZMPM_OK;
}
// out -= sum_p stress_p grad w_ip with `stress` in the HVP precision (the MLS
// weight when mls).
int launch_force_scatter(Ctx* ctx, double* out, bool mls)
{
    if (!ctx->G) return ZMPM_OK;
    if (ctx->mixed)
        return ctx->layout == 1 ? force_scatter_impl<Layout244, float>(ctx, out, mls) : force_scatter_impl<Layout444, float>(ctx, out, mls);
    return ctx->layout == 1 ? force_scatter_impl<Layout244, double>(ctx, out, mls) : force_scatter_impl<Layout444, double>(ctx, out, mls);
}

// out += sum_p (grad(x)_p B_p) grad w_ip (ADMM's global operator).
template <class L>
static int admm_op_impl(Ctx* ctx, const double* x, double* out)
{
    DevCounters* dc = ctx->counters.as<DevCounters>();
    if (ctx->mixed)
        k_op_fused<L, float, fused_chunk<float>()><<<(unsigned)ctx->G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<float>(), ctx->adm_B.as<float>(), x, out,
            &dc->flags);
    else
        k_op_fused<L, double, fused_chunk<double>()><<<(unsigned)ctx->G, FUSED_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(),
            ctx->group_nbr.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<double>(), ctx->adm_B.as<double>(), x,
            out, &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}
int launch_admm_op(Ctx* ctx, const double* x, double* out)
{
    if (!ctx->G) return ZMPM_OK;
    return ctx->layout == 1 ? admm_op_impl<Layout244>(ctx, x, out) : admm_op_impl<Layout444>(ctx, x, out);
}

template <class L>
static int g2p_impl(Ctx* ctx, bool plastic)
{
    const int64_t G = ctx->G;
    if (G == 0) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    if (ctx->mixed)
        k_g2p<L, float, float><<<(unsigned)G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->frac.as<float>(), ctx->cfg.dx, ctx->dt,
            ctx->cfg.apic_rpic_ratio, ctx->vstarf.as<float>(), &dc->flags, ctx->mls ? 1 : 0, plastic ? 1 : 0);
    else
        k_g2p<L, double, double><<<(unsigned)G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->frac.as<double>(), ctx->cfg.dx, ctx->dt,
            ctx->cfg.apic_rpic_ratio, ctx->vstar.as<double>(), &dc->flags, ctx->mls ? 1 : 0, plastic ? 1 : 0);
    ++g_kernel_launches;
    return ZMPM_OK;
}
int launch_g2p(Ctx* ctx, bool plastic) { return ctx->layout == 1 ? g2p_impl<Layout244>(ctx, plastic) : g2p_impl<Layout444>(ctx, plastic); }

} // namespace zmpm
