// Particle kernels of the ADMM substep (AdmmSimulation, Projects/admm/
// AdmmSimulationFoam.h).  One CTA per particle group, as in transfer.cu.
//
// The reference assembles the global matrix M + sum_p rho omega^2 dt^2
// (Fn^T grad w_ip)(Fn^T grad w_jp)^T as a 125-entry stencil per node
// (initMultiplierAndPreconditioner, :407-505) and multiplies it in MINRES.
// Here the product is matrix-free: with B_p = rho dt^2 (omega_0^2 Fn Fn^T +
// omega_1^2 Fe Fe^T) (6 numbers per particle),
//     (A x)_i = m_i x_i + sum_p (grad x_p B_p) grad w_ip,  grad x_p = sum_j x_j grad w_jp^T,
// the same gather -> 3x3 -> scatter shape as the Newton Hessian product, so it
// runs through the same per-group product (hvp.cuh, AdmmOpModel): k_op_fused
// for the right-hand side's product, the persistent MINRES for the solve.
// Per product that is 6 numbers per particle instead of 125 values + 125
// indices per node.
//
// Kernels
//  k_admm_dvinit   dv_i = sum_p last_dv_p w_ip, w_i = sum_p w_ip (initStep :304-320)
//  k_admm_init     F = (I + dt grad(vn+dv)) Fn (and Fe), grad vn, omega
//                  (initOmega :222-274), y <- y omega_old / omega, B
//  k_admm_pre      preconditioner m_i + sum_p grad w^T B grad w (:477-503)
//  k_admm_local    FStepSolve (:507-615) for F and Fe, then the dvStep
//                  right-hand side stress dt rho omega^2 bFu Fn^T (:163-205)
//  k_admm_dual     uStep (:638-671)
//  k_admm_lastdv   last_dv = sum dv w / (dt sum w) (:788-800)
#include "admm.cuh"
#include "xfer.cuh"

namespace zmpm {

namespace {

// Grad of a staged window vector at one particle, weights from X in FP64.
template <class L>
__device__ __forceinline__ void particle_weights(const double* __restrict__ pd, int64_t cap, int s, short4 b, double inv_dx, double w[3][3],
    double dwr[3][3])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) bspline(inv_dx * pd[(PD_X + d) * cap + s] - (double)((&b.x)[d]), w[d], dwr[d]);
}

template <class L>
__device__ __forceinline__ M3<double> window_grad(const double* win, int lx, int ly, int lz, const double w[3][3], const double dwr[3][3],
    double inv_dx)
{
    constexpr int NPB = L::NPB;
    M3<double> G = m3_zero<double>();
    for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double, const double* dw) {
        const double* vv = win + t * 3 * NPB + e;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double vr = vv[r * NPB];
#pragma unroll
            for (int c = 0; c < 3; ++c) G(r, c) += vr * dw[c];
        }
    });
    return G;
}

__device__ __forceinline__ M3<double> load9(const double* __restrict__ pd, int64_t cap, int f, int s)
{
    M3<double> m;
#pragma unroll
    for (int q = 0; q < 9; ++q) m.a[q] = pd[(int64_t)(f + q) * cap + s];
    return m;
}
__device__ __forceinline__ void store9(double* __restrict__ pd, int64_t cap, int f, int s, const M3<double>& m)
{
#pragma unroll
    for (int q = 0; q < 9; ++q) pd[(int64_t)(f + q) * cap + s] = m.a[q];
}

// (I + dt G) S computed as S + dt (G S)
__device__ __forceinline__ M3<double> advect(const M3<double>& S, const M3<double>& G, double dt)
{
    const M3<double> t = m3_mul(G, S);
    M3<double> r;
#pragma unroll
    for (int q = 0; q < 9; ++q) r.a[q] = S.a[q] + dt * t.a[q];
    return r;
}

} // namespace

// ------------------------------------------------------------- dv init ----
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_admm_dvinit(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, double* __restrict__ wsum, double* __restrict__ dv)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(16) double acc[8 * 4 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<4, NPB>(acc);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    for (int q = threadIdx.x; q < cl.layers * NPB; q += blockDim.x) {
        const int r = q / NPB, ce = q % NPB;
        if (r >= cl.cnt[ce]) continue;
        const int s = s0 + cl.start[ce] + r;
        const short4 b = base[s];
        double w[3][3], dwr[3][3];
        particle_weights<L>(pd, cap, s, b, inv_dx, w, dwr);
        const double ld[3] = { pd[(PD_LASTDV + 0) * cap + s], pd[(PD_LASTDV + 1) * cap + s], pd[(PD_LASTDV + 2) * cap + s] };
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double wijk, const double*) {
            double* a = acc + t * 4 * NPB + e;
            atomicAdd(a, wijk);
#pragma unroll
            for (int d = 0; d < 3; ++d) atomicAdd(a + (1 + d) * NPB, ld[d] * wijk);
        });
    }
    __syncthreads();
    flush_window<4, 1, NPB>(acc, nbr, wsum, dv);
}

// ---------------------------------------------------------------- init ----
template <class L, class TH>
__global__ void __launch_bounds__(XF_THREADS) k_admm_init(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, double dt, double rho,
    const double* __restrict__ vstar, const double* __restrict__ vn, double* __restrict__ aF, double* __restrict__ gvn, TH* __restrict__ B,
    int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ __align__(128) double win2[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar[2];
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(win, vstar, nbr, &bar[0], flags);
    stage_window<NPB>(win2, vn, nbr, &bar[1], flags);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        double w[3][3], dwr[3][3];
        particle_weights<L>(pd, cap, s, b, inv_dx, w, dwr);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        const M3<double> gv = window_grad<L>(win, lx, ly, lz, w, dwr, inv_dx);
        const M3<double> gn = window_grad<L>(win2, lx, ly, lz, w, dwr, inv_dx);
        store9(gvn, cap, 0, s, gn);
        const M3<double> Fn = load9(pd, cap, PD_F, s);
        const M3<double> Fa0 = advect(Fn, gv, dt);
        store9(aF, cap, 0, s, Fa0);
        const bool visco = pi[PI_VISCO * cap + s] != 0;
        M3<double> Fe = m3_identity<double>();
        if (visco) {
            Fe = load9(pd, cap, PD_FE, s);
            store9(aF, cap, 9, s, advect(Fe, gv, dt));
        }
        double om0 = pd[(PD_OMEGA + 0) * cap + s], om1 = pd[(PD_OMEGA + 1) * cap + s];
        if (pi[PI_KIND * cap + s] == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
            const double vol = pd[PD_VOL * cap + s];
            const int pkind = pi[PI_PKIND * cap + s];
            // Drucker-Prager: PD_YS = alpha, PD_FS = cohesion
            const double n0 = admm_omega<double>(Fa0, vol, pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pkind, pd[PD_YS * cap + s],
                pd[PD_YS * cap + s], pd[PD_FS * cap + s]);
            double n1 = om1;
            if (visco) n1 = admm_omega<double>(load9(aF, cap, 9, s), vol, pd[PD_VMU * cap + s], pd[PD_VLAM * cap + s], ZMPM_PLASTIC_NONE, 0.0);
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                pd[(PD_Y + q) * cap + s] = pd[(PD_Y + q) * cap + s] * om0 / n0;
                pd[(PD_Y + 9 + q) * cap + s] = pd[(PD_Y + 9 + q) * cap + s] * om1 / n1;
            }
            om0 = n0;
            om1 = n1;
            pd[(PD_OMEGA + 0) * cap + s] = om0;
            pd[(PD_OMEGA + 1) * cap + s] = om1;
        }
        // B = rho dt^2 (omega_0^2 Fn Fn^T + omega_1^2 Fe Fe^T)
        const double c0 = rho * om0 * om0 * dt * dt, c1 = visco ? rho * om1 * om1 * dt * dt : 0.0;
        const M3<double> A0 = m3_mulT(Fn, Fn), A1 = m3_mulT(Fe, Fe);
        const int ri[6] = { 0, 0, 0, 1, 1, 2 }, ci[6] = { 0, 1, 2, 1, 2, 2 };
#pragma unroll
        for (int k = 0; k < 6; ++k) B[(int64_t)k * cap + s] = (TH)(c0 * A0(ri[k], ci[k]) + c1 * A1(ri[k], ci[k]));
    }
}

// ------------------------------------------------------ preconditioner ----
template <class L, class TH>
__global__ void __launch_bounds__(XF_THREADS) k_admm_pre(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    int64_t cap, const short4* __restrict__ base, double dx, const TH* __restrict__ frac, const TH* __restrict__ B, double* __restrict__ pre)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(16) TH acc[8 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<1, NPB>(acc);
    const TH inv_dx = TH(1.0 / dx);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    for (int q = threadIdx.x; q < cl.layers * NPB; q += blockDim.x) {
        const int r = q / NPB, ce = q % NPB;
        if (r >= cl.cnt[ce]) continue;
        const int s = s0 + cl.start[ce] + r;
        const short4 b = base[s];
        TH w[3][3], dwr[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) bspline(frac[d * cap + s], w[d], dwr[d]);
        TH Bs[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) Bs[k] = B[(int64_t)k * cap + s];
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, TH, const TH* dw) {
            const TH v = Bs[0] * dw[0] * dw[0] + Bs[3] * dw[1] * dw[1] + Bs[5] * dw[2] * dw[2]
                + TH(2) * (Bs[1] * dw[0] * dw[1] + Bs[2] * dw[0] * dw[2] + Bs[4] * dw[1] * dw[2]);
            atomicAdd(acc + t * NPB + e, v);
        });
    }
    __syncthreads();
    flush_window<1, 1, NPB>(acc, nbr, pre, nullptr);
}

// ------------------------------------------------------------ F step ------
template <class L, class TH>
__global__ void __launch_bounds__(XF_THREADS) k_admm_local(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, double dt,
    double rho, double local_tol, const double* __restrict__ vstar, double* __restrict__ aF, const double* __restrict__ gvn,
    TH* __restrict__ stress, int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(win, vstar, nbr, &bar, flags);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        double w[3][3], dwr[3][3];
        particle_weights<L>(pd, cap, s, b, inv_dx, w, dwr);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        const M3<double> gv = window_grad<L>(win, lx, ly, lz, w, dwr, inv_dx);
        const M3<double> gn = load9(gvn, cap, 0, s);
        const bool hencky = pi[PI_KIND * cap + s] == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC;
        const int nk = pi[PI_VISCO * cap + s] ? 2 : 1;
        const double vol = pd[PD_VOL * cap + s];
        M3<double> R = m3_zero<double>();
        for (int k = 0; k < nk; ++k) {
            const M3<double> Sn = load9(pd, cap, k == 0 ? PD_F : PD_FE, s);
            const M3<double> y = load9(pd, cap, PD_Y + 9 * k, s);
            const double om = pd[(PD_OMEGA + k) * cap + s];
            M3<double> Fa = load9(aF, cap, 9 * k, s);
            if (hencky) {
                // FDb = Fn - y / (omega rho) + dt grad(vn + dv) Fn
                const M3<double> t = m3_mul(gv, Sn);
                M3<double> FDb;
#pragma unroll
                for (int q = 0; q < 9; ++q) FDb.a[q] = (Sn.a[q] + (-y.a[q] / (om * rho))) + dt * t.a[q];
                AdmmStrainParams p;
                int mode, iters;
                if (k == 0) {
                    p = { pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_YS * cap + s], 1.0, 1.0, pd[PD_YS * cap + s], pd[PD_FS * cap + s] };
                    const int pk = pi[PI_PKIND * cap + s];
                    mode = pk == ZMPM_PLASTIC_VON_MISES ? ADMM_VON_MISES : (pk == ZMPM_PLASTIC_DRUCKER_PRAGER ? ADMM_DRUCKER_PRAGER : ADMM_ELASTIC);
                    iters = 5;
                }
                else {
                    p = { pd[PD_VMU * cap + s], pd[PD_VLAM * cap + s], 0.0, pd[PD_VD * cap + s], pd[PD_VV * cap + s], 0.0, 0.0 };
                    mode = ADMM_VISCOUS;
                    iters = 20;
                }
                Fa = admm_local_solve<double>(FDb, Fa, vol, rho * om * om, p, mode, dt, iters, local_tol);
                store9(aF, cap, 9 * k, s, Fa);
            }
            // bFu = F - Fn + y / (omega rho) - dt grad(vn) Fn; R += dt rho omega^2 bFu Fn^T
            const M3<double> tn = m3_mul(gn, Sn);
            M3<double> bFu;
#pragma unroll
            for (int q = 0; q < 9; ++q) bFu.a[q] = Fa.a[q] - Sn.a[q] + y.a[q] / (om * rho) - dt * tn.a[q];
            const double c = dt * rho * om * om;
#pragma unroll
            for (int q = 0; q < 9; ++q) bFu.a[q] *= c;
            const M3<double> Rk = m3_mulT(bFu, Sn);
#pragma unroll
            for (int q = 0; q < 9; ++q) R.a[q] += Rk.a[q];
        }
        // the force scatter subtracts stress . grad w, so store -R
#pragma unroll
        for (int q = 0; q < 9; ++q) stress[(int64_t)q * cap + s] = (TH)(-R.a[q]);
    }
}

// ------------------------------------------------------------ dual step ---
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_admm_dual(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, double dt, double rho,
    const double* __restrict__ vstar, const double* __restrict__ aF, int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(win, vstar, nbr, &bar, flags);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        double w[3][3], dwr[3][3];
        particle_weights<L>(pd, cap, s, b, inv_dx, w, dwr);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        const M3<double> gv = window_grad<L>(win, lx, ly, lz, w, dwr, inv_dx);
        const int nk = pi[PI_VISCO * cap + s] ? 2 : 1;
        for (int k = 0; k < nk; ++k) {
            const M3<double> Sn = load9(pd, cap, k == 0 ? PD_F : PD_FE, s);
            const M3<double> Fa = load9(aF, cap, 9 * k, s);
            const double om = pd[(PD_OMEGA + k) * cap + s];
            const M3<double> t = m3_mul(gv, Sn);
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                const double tmp = Fa.a[q] - Sn.a[q] - dt * t.a[q];
                pd[(int64_t)(PD_Y + 9 * k + q) * cap + s] += rho * om * tmp;
            }
        }
    }
}

// ------------------------------------------------------------- last dv ----
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_admm_lastdv(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, double dt, const double* __restrict__ dv,
    int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(win, dv, nbr, &bar, flags);
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        double w[3][3], dwr[3][3];
        particle_weights<L>(pd, cap, s, b, inv_dx, w, dwr);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        double acc[3] = { 0, 0, 0 }, wsum = 0;
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double wijk, const double*) {
            const double* vv = win + t * 3 * NPB + e;
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] += vv[d * NPB] * wijk;
            wsum += wijk;
        });
#pragma unroll
        for (int d = 0; d < 3; ++d) pd[(PD_LASTDV + d) * cap + s] = acc[d] / (wsum * dt);
    }
}

// ------------------------------------------------------------ launchers ---
namespace {

template <class L>
int dvinit_impl(Ctx* ctx)
{
    k_admm_dvinit<L><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
        ctx->pd.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->adm_w.as<double>(), ctx->dv.as<double>());
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <class L, class TH>
int init_impl(Ctx* ctx, double rho)
{
    DevCounters* dc = ctx->counters.as<DevCounters>();
    k_admm_init<L, TH><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
        ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, rho, ctx->vstar.as<double>(),
        ctx->vn.as<double>(), ctx->adm_F.as<double>(), ctx->adm_gvn.as<double>(), ctx->adm_B.as<TH>(), &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <class L, class TH>
int pre_impl(Ctx* ctx)
{
    k_admm_pre<L, TH><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(), ctx->Pcap,
        ctx->base.as<short4>(), ctx->cfg.dx, ctx->frac.as<TH>(), ctx->adm_B.as<TH>(), ctx->adm_pre.as<double>());
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <class L, class TH>
int local_impl(Ctx* ctx, double rho, double local_tol)
{
    DevCounters* dc = ctx->counters.as<DevCounters>();
    k_admm_local<L, TH><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
        ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, rho, local_tol,
        ctx->vstar.as<double>(), ctx->adm_F.as<double>(), ctx->adm_gvn.as<double>(), ctx->stress.as<TH>(), &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <class L>
int dual_impl(Ctx* ctx, double rho)
{
    DevCounters* dc = ctx->counters.as<DevCounters>();
    k_admm_dual<L><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
        ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, rho, ctx->vstar.as<double>(),
        ctx->adm_F.as<double>(), &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <class L>
int lastdv_impl(Ctx* ctx)
{
    DevCounters* dc = ctx->counters.as<DevCounters>();
    k_admm_lastdv<L><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
        ctx->pd.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, ctx->dv.as<double>(), &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

} // namespace

#define ZMPM_BY_LAYOUT(fn, ...) (ctx->layout == 1 ? fn<Layout244>(__VA_ARGS__) : fn<Layout444>(__VA_ARGS__))
#define ZMPM_BY_LAYOUT_TH(fn, ...)                                                                                     \
    (ctx->mixed ? (ctx->layout == 1 ? fn<Layout244, float>(__VA_ARGS__) : fn<Layout444, float>(__VA_ARGS__))         \
                : (ctx->layout == 1 ? fn<Layout244, double>(__VA_ARGS__) : fn<Layout444, double>(__VA_ARGS__)))

int launch_admm_dvinit(Ctx* ctx) { return ctx->G ? ZMPM_BY_LAYOUT(dvinit_impl, ctx) : ZMPM_OK; }
int launch_admm_init(Ctx* ctx, double rho) { return ctx->G ? ZMPM_BY_LAYOUT_TH(init_impl, ctx, rho) : ZMPM_OK; }
int launch_admm_pre(Ctx* ctx) { return ctx->G ? ZMPM_BY_LAYOUT_TH(pre_impl, ctx) : ZMPM_OK; }
int launch_admm_local(Ctx* ctx, double rho, double local_tol) { return ctx->G ? ZMPM_BY_LAYOUT_TH(local_impl, ctx, rho, local_tol) : ZMPM_OK; }
int launch_admm_dual(Ctx* ctx, double rho) { return ctx->G ? ZMPM_BY_LAYOUT(dual_impl, ctx, rho) : ZMPM_OK; }
int launch_admm_lastdv(Ctx* ctx) { return ctx->G ? ZMPM_BY_LAYOUT(lastdv_impl, ctx) : ZMPM_OK; }

} // namespace zmpm
