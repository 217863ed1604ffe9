// Reverse mode of one implicit substep (zmpm_adjoint_substep; the reference has
// no differentiation).  With v* = vn + dv the converged Newton solution of
//   G(v*) = M v* - q - dt M g + dt sum_p V0 P(F_p) Fn_p^T grad w_ip = 0 (free nodes),
//   F_p = (I + dt sum_j v*_j grad w_jp^T) Fn_p,  q_i = sum_p w_ip m_p (v_p + C_p (x_i - x_p)),
// and G2P v_p' = sum w v*, C_p' = D^-1 sum w v* (x_i - x_p)^T, F_p' = (I + dt grad v*) Fn,
// x_p' = x_p + dt v_p', the implicit function theorem gives
// dL/dtheta = -lambda^T dG/dtheta with (M + dt^2 K) lambda = P dL/dv*: the
// Newton Hessian, applied by the same HVP kernels.  Binning is held fixed.
//
// Kernels (one CTA per particle group, as the forward transfers)
//  k_adj_g2p       G2P reverse: scatters dL/dv* to the grid, writes dL/dx and
//                  dL/dFn of the G2P terms (B-spline Hessians for the x terms)
//  k_adj_particle  force, P2G and E reverse: gathers lambda and v*, adds the
//                  -lambda^T dG/d(x, v, C, Fn, E) terms
#include "xfer.cuh"
#include "models.cuh"

namespace zmpm {

namespace {

// Iterates the 27 stencil nodes with weight, gradient and Hessian of w_ip
// with respect to x_p (per axis the quadratic B-spline's second derivative in
// cells is 1, -2, 1).
template <class L, class Fn>
__device__ __forceinline__ void for_stencil_h(int lx, int ly, int lz, const double w[3][3], const double dwr[3][3], double inv_dx, Fn&& f)
{
    const double idx2 = inv_dx * inv_dx;
    const double dd[3] = { 1.0, -2.0, 1.0 };
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double Nx = w[0][i], Ny = w[1][j], Nz = w[2][k];
                const double Dx = dwr[0][i], Dy = dwr[1][j], Dz = dwr[2][k];
                const double wt = Nx * Ny * Nz;
                const double dw[3] = { Dx * Ny * Nz * inv_dx, Nx * Dy * Nz * inv_dx, Nx * Ny * Dz * inv_dx };
                double H[3][3];
                H[0][0] = dd[i] * Ny * Nz * idx2;
                H[1][1] = Nx * dd[j] * Nz * idx2;
                H[2][2] = Nx * Ny * dd[k] * idx2;
                H[0][1] = H[1][0] = Dx * Dy * Nz * idx2;
                H[0][2] = H[2][0] = Dx * Ny * Dz * idx2;
                H[1][2] = H[2][1] = Nx * Dy * Dz * idx2;
                int e;
                const int t = win_slot<L>(lx + i, ly + j, lz + k, e);
                f(t, e, i, j, k, wt, dw, H);
            }
}

__device__ __forceinline__ M3<double> ld9(const double* __restrict__ a, int64_t cap, int f, int s)
{
    M3<double> m;
#pragma unroll
    for (int q = 0; q < 9; ++q) m.a[q] = a[(int64_t)(f + q) * cap + s];
    return m;
}

} // namespace

// ---------------------------------------------------------------- G2P -----
// With von Mises plasticity the G2P output is F' = Pi((I + dt grad v*) Fn), so
// dL/dF of the projection's input replaces dL/dF' first (von_mises_adjoint),
// and the yield radius' dependence on E starts dL/dE (AJ_OE; k_adj_particle
// adds the force term's).
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_adj_g2p(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, const int32_t* __restrict__ pi, double* __restrict__ aj, int64_t cap, const short4* __restrict__ base,
    double dx, double dt, const double* __restrict__ vstar, double* __restrict__ vsbar, int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double win[8 * 3 * NPB];
    __shared__ __align__(16) double acc[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar;
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<3, NPB>(acc);
    __syncthreads();
    stage_window<NPB>(win, vstar, nbr, &bar, flags);
    const double inv_dx = 1.0 / dx, D_inv = 4.0 / (dx * dx);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    for (int q = threadIdx.x; q < cl.layers * NPB; q += blockDim.x) {
        const int r = q / NPB, ce = q % NPB;
        if (r >= cl.cnt[ce]) continue;
        const int s = s0 + cl.start[ce] + r;
        const short4 b = base[s];
        double xp[3], w[3][3], dwr[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xp[d] = aj[(AJ_X0 + d) * cap + s];
            bspline(inv_dx * xp[d] - (double)((&b.x)[d]), w[d], dwr[d]);
        }
        double vt[3], xb[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xb[d] = aj[(AJ_GX + d) * cap + s];
            vt[d] = aj[(AJ_GV + d) * cap + s] + dt * xb[d];
        }
        const M3<double> Cb = ld9(aj, cap, AJ_GC, s), Fn = ld9(aj, cap, AJ_F0, s);
        M3<double> Fb = ld9(aj, cap, AJ_GF, s);
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        double gE = 0;
        if (pi[PI_PKIND * cap + s] == ZMPM_PLASTIC_VON_MISES && pi[PI_KIND * cap + s] != ZMPM_MODEL_NONE) {
            // the projection's input F' = (I + dt grad v*) Fn
            M3<double> A = m3_identity<double>();
            for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double, const double* dw) {
                const double* vv = win + t * 3 * NPB + e;
#pragma unroll
                for (int rr = 0; rr < 3; ++rr)
#pragma unroll
                    for (int c = 0; c < 3; ++c) A(rr, c) += dt * vv[rr * NPB] * dw[c];
            });
            const double mu = pd[PD_MU * cap + s], lm = pd[PD_LAM * cap + s];
            const double E = mu * (3 * lm + 2 * mu) / (lm + mu);
            Fb = von_mises_adjoint<double>(mu, pd[PD_YS * cap + s], E, m3_mul(A, Fn), Fb, &gE);
        }
        aj[AJ_OE * cap + s] = gE;
        const M3<double> FbFnT = m3_mulT(Fb, Fn), FnFbT = m3_mulT(Fn, Fb);
        M3<double> gvs = m3_zero<double>();
        for_stencil_h<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int i, int j, int k, double wt, const double* dw, const double (*H)[3]) {
            const double* vv = win + t * 3 * NPB + e;
            const double v[3] = { vv[0], vv[NPB], vv[2 * NPB] };
            const double xi[3] = { (b.x + i) * dx - xp[0], (b.y + j) * dx - xp[1], (b.z + k) * dx - xp[2] };
            double fd[3], cx[3], CTv[3], qv[3];
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) {
                fd[rr] = FbFnT(rr, 0) * dw[0] + FbFnT(rr, 1) * dw[1] + FbFnT(rr, 2) * dw[2];
                cx[rr] = Cb(rr, 0) * xi[0] + Cb(rr, 1) * xi[1] + Cb(rr, 2) * xi[2];
                CTv[rr] = Cb(0, rr) * v[0] + Cb(1, rr) * v[1] + Cb(2, rr) * v[2];
                qv[rr] = FnFbT(rr, 0) * v[0] + FnFbT(rr, 1) * v[1] + FnFbT(rr, 2) * v[2];
            }
            double* a = acc + t * 3 * NPB + e;
#pragma unroll
            for (int d = 0; d < 3; ++d) atomicAdd(a + d * NPB, wt * vt[d] + D_inv * wt * cx[d] + dt * fd[d]);
            const double vdot = v[0] * vt[0] + v[1] * vt[1] + v[2] * vt[2];
            const double vCx = v[0] * cx[0] + v[1] * cx[1] + v[2] * cx[2];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                xb[d] += vdot * dw[d] + D_inv * (vCx * dw[d] - wt * CTv[d]);
                xb[d] += dt * (H[d][0] * qv[0] + H[d][1] * qv[1] + H[d][2] * qv[2]);
            }
#pragma unroll
            for (int rr = 0; rr < 3; ++rr)
#pragma unroll
                for (int c = 0; c < 3; ++c) gvs(rr, c) += v[rr] * dw[c];
        });
        M3<double> A = m3_identity<double>();
#pragma unroll
        for (int k2 = 0; k2 < 9; ++k2) A.a[k2] += dt * gvs.a[k2];
        const M3<double> FbN = m3_Tmul(A, Fb);
#pragma unroll
        for (int k2 = 0; k2 < 9; ++k2) aj[(int64_t)(AJ_OF + k2) * cap + s] = FbN.a[k2];
#pragma unroll
        for (int d = 0; d < 3; ++d) aj[(AJ_OX + d) * cap + s] = xb[d];
    }
    __syncthreads();
    flush_window<3, 3, NPB>(acc, nbr, vsbar, nullptr);
}

// -------------------------------------------------- force, P2G and E -------
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_adj_particle(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, const int32_t* __restrict__ pi, double* __restrict__ aj, int64_t cap, const short4* __restrict__ base,
    double dx, double dt, double gx, double gy, double gz, const double* __restrict__ lam, const double* __restrict__ vstar,
    int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    __shared__ __align__(128) double wl[8 * 3 * NPB];
    __shared__ __align__(128) double wv[8 * 3 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ __align__(8) uint64_t bar[2];
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    stage_window<NPB>(wl, lam, nbr, &bar[0], flags);
    stage_window<NPB>(wv, vstar, nbr, &bar[1], flags);
    const double inv_dx = 1.0 / dx;
    const double grav[3] = { gx, gy, gz };
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        double xp[3], w[3][3], dwr[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xp[d] = aj[(AJ_X0 + d) * cap + s];
            bspline(inv_dx * xp[d] - (double)((&b.x)[d]), w[d], dwr[d]);
        }
        const int lx = b.x & (L::BX - 1), ly = b.y & (L::BY - 1), lz = b.z & (L::BZ - 1);
        M3<double> Lam = m3_zero<double>(), Vs = m3_zero<double>();
        for_stencil_h<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double, const double* dw, const double (*)[3]) {
            const double* l = wl + t * 3 * NPB + e;
            const double* v = wv + t * 3 * NPB + e;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    Lam(r, c) += l[r * NPB] * dw[c];
                    Vs(r, c) += v[r * NPB] * dw[c];
                }
        });
        const M3<double> Fn = ld9(aj, cap, AJ_F0, s);
        M3<double> Fb = ld9(aj, cap, AJ_OF, s);
        double xb[3] = { aj[(AJ_OX + 0) * cap + s], aj[(AJ_OX + 1) * cap + s], aj[(AJ_OX + 2) * cap + s] };
        double gE = 0;
        const int kind = pi[PI_KIND * cap + s];
        if (kind != ZMPM_MODEL_NONE) {
            M3<double> A = m3_identity<double>();
#pragma unroll
            for (int k2 = 0; k2 < 9; ++k2) A.a[k2] += dt * Vs.a[k2];
            const M3<double> F = m3_mul(A, Fn);
            const ModelParams mp{ pd[PD_MU * cap + s], pd[PD_LAM * cap + s], pd[PD_KAPPA * cap + s], pd[PD_G * cap + s] };
            // P and dP(Lambda Fn) through the model plugin with V0 = 1, Fn = I
            double scr[NS];
            const M3<double> P = model_update<double, double>(kind, mp, 1.0, F, m3_identity<double>(), scr, 1, 0);
            const M3<double> LF = m3_mul(Lam, Fn);
            const M3<double> dPL = model_hvp<double>(kind, scr, 1, 0, LF);
            const double c0 = dt * pd[PD_VOL * cap + s];
            const M3<double> t1 = m3_Tmul(A, dPL), t2 = m3_Tmul(Lam, P);
#pragma unroll
            for (int k2 = 0; k2 < 9; ++k2) Fb.a[k2] -= c0 * (t1.a[k2] + t2.a[k2]);
            // dP/dE = P/E at fixed Poisson ratio
            double mu = mp.mu, lm = kind == ZMPM_MODEL_NEOHOOKEAN_BORDEN ? mp.kappa - 0.666666 * mp.mu : mp.lambda;
            const double E = mu * (3 * lm + 2 * mu) / (lm + mu);
            gE = -c0 * m3_contract(P, LF) / E;
            const M3<double> Q1 = m3_mulT(dPL, Fn), Q2 = m3_mulT(P, Fn);
            for_stencil_h<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double, const double*, const double (*H)[3]) {
                const double* l = wl + t * 3 * NPB + e;
                const double* v = wv + t * 3 * NPB + e;
                double a[3], bb[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    a[c] = Q1(0, c) * v[0] + Q1(1, c) * v[NPB] + Q1(2, c) * v[2 * NPB];
                    bb[c] = Q2(0, c) * l[0] + Q2(1, c) * l[NPB] + Q2(2, c) * l[2 * NPB];
                }
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    xb[d] -= c0 * (dt * (H[d][0] * a[0] + H[d][1] * a[1] + H[d][2] * a[2]) + (H[d][0] * bb[0] + H[d][1] * bb[1] + H[d][2] * bb[2]));
            });
        }
        // P2G: q_i = sum w m (v + C (x_i - x_p)) with qbar = lambda; m_i = sum w m with
        // mbar = -lambda . (v* - dt g)
        const double mp_ = pd[PD_M * cap + s];
        const M3<double> Cp = ld9(aj, cap, AJ_C0, s);
        const double vp[3] = { aj[(AJ_V0 + 0) * cap + s], aj[(AJ_V0 + 1) * cap + s], aj[(AJ_V0 + 2) * cap + s] };
        double vb[3] = { 0, 0, 0 };
        M3<double> Cb = m3_zero<double>();
        for_stencil_h<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int i, int j, int k, double wt, const double* dw, const double (*)[3]) {
            const double* lp = wl + t * 3 * NPB + e;
            const double* vsp = wv + t * 3 * NPB + e;
            const double l[3] = { lp[0], lp[NPB], lp[2 * NPB] };
            const double xi[3] = { (b.x + i) * dx - xp[0], (b.y + j) * dx - xp[1], (b.z + k) * dx - xp[2] };
            double u[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) u[r] = vp[r] + Cp(r, 0) * xi[0] + Cp(r, 1) * xi[1] + Cp(r, 2) * xi[2];
            const double lu = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
            const double mbar = -(l[0] * (vsp[0] - dt * grav[0]) + l[1] * (vsp[NPB] - dt * grav[1]) + l[2] * (vsp[2 * NPB] - dt * grav[2]));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                vb[d] += wt * mp_ * l[d];
                const double CTl = Cp(0, d) * l[0] + Cp(1, d) * l[1] + Cp(2, d) * l[2];
                xb[d] += mp_ * lu * dw[d] - wt * mp_ * CTl + mbar * mp_ * dw[d];
            }
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) Cb(r, c) += wt * mp_ * l[r] * xi[c];
        });
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            aj[(AJ_OX + d) * cap + s] = xb[d];
            aj[(AJ_OV + d) * cap + s] = vb[d];
        }
#pragma unroll
        for (int k2 = 0; k2 < 9; ++k2) {
            aj[(int64_t)(AJ_OC + k2) * cap + s] = Cb.a[k2];
            aj[(int64_t)(AJ_OF + k2) * cap + s] = Fb.a[k2];
        }
        aj[AJ_OE * cap + s] += gE;
    }
}

// ------------------------------------------------------------ launchers ---
int launch_adj_g2p(Ctx* ctx, double* vsbar)
{
    if (!ctx->G) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    if (ctx->layout == 1)
        k_adj_g2p<Layout244><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->adj.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt,
            ctx->vstar.as<double>(), vsbar, &dc->flags);
    else
        k_adj_g2p<Layout444><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->adj.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt,
            ctx->vstar.as<double>(), vsbar, &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

int launch_adj_particle(Ctx* ctx, const double* lam)
{
    if (!ctx->G) return ZMPM_OK;
    DevCounters* dc = ctx->counters.as<DevCounters>();
    const double* g = ctx->cfg.gravity;
    if (ctx->layout == 1)
        k_adj_particle<Layout244><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->adj.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, g[0], g[1],
            g[2], lam, ctx->vstar.as<double>(), &dc->flags);
    else
        k_adj_particle<Layout444><<<(unsigned)ctx->G, XF_THREADS, 0, ctx->stream>>>(ctx->group_start.as<int32_t>(), ctx->group_nbr.as<int32_t>(),
            ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->adj.as<double>(), ctx->Pcap, ctx->base.as<short4>(), ctx->cfg.dx, ctx->dt, g[0], g[1],
            g[2], lam, ctx->vstar.as<double>(), &dc->flags);
    ++g_kernel_launches;
    return ZMPM_OK;
}

} // namespace zmpm
