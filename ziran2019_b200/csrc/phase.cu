// CD-MPM phase-field solve after P2G: FractureSimulation::solvePhaseFieldSystem
// (Projects/fracture/FractureSimulation.h:257-456) with phaseP2G (:208-255) and
// phaseG2P (:458-507), and FractureSimulation::deleteParticles (:172-207).
//
// The grid unknown is one scalar per node, kept with the solve's other node
// scalars in one block-dense array [B][PN_FIELDS][NPB] (FP64).  Particle
// passes run one CTA per particle group like P2G/G2P: they stage the 8 pages
// around the group's page in shared memory, accumulate in a shared window and
// flush it with global atomics.  The CG (Projects/fracture/ConjugateGradient.h:
// 53-104, Jacobi preconditioner with the lumped diagonal) keeps its scalars on
// the device; its reductions are per-CTA partials summed in a fixed order by a
// one-CTA kernel, so the iteration is deterministic.  The host enqueues
// iterations in batches (1, 4, then 16) and reads the "active" flag between
// batches; kernels of iterations past convergence return at once.
#include <algorithm>
#include <cfloat>

#include "internal.cuh"
#include "mat3.cuh"
#include "node.cuh"
#include "xfer.cuh"

namespace zmpm {

enum PfNode { PN_MULT = 0, PN_PHASE = 1, PN_VS = 2, PN_DIAG = 3, PN_X = 4, PN_R = 5, PN_S = 6, PN_Q = 7, PN_FIELDS = 8 };

struct PfScalars {
    int32_t active;  // 1 while the CG iterates
    int32_t it;      // current iteration index (`iterations` of the reference loop)
    int32_t iters;   // iterations reported when the loop stopped
    int32_t pad;
    double rho, rho_old, alpha, norm, rel_tol;
};

struct PfParams {
    double M;        // parabolic_M (0: elliptic)
    double dt, one_over_dt;
    double tol;      // absolute CG tolerance
    int lumping;
    int max_it;
};

template <int NPB>
__device__ __forceinline__ double* pf_node(double* pfn, int64_t n, int f)
{
    const int64_t b = n / NPB;
    const int e = (int)(n - b * NPB);
    return pfn + (b * PN_FIELDS + f) * NPB + e;
}

// ------------------------------------------------------------- particles --
// deleteParticles: c < threshold parks the particle at (4, 4, 4) with V = 0,
// F = I and no further damage.
__global__ void k_pf_delete(double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, int64_t P, double threshold)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P) return;
    if (pi[PI_DAMAGE * cap + s] != ZMPM_DAMAGE_PHASE_FIELD || !(pd[PD_PF_C * cap + s] < threshold)) return;
    for (int d = 0; d < 3; ++d) {
        pd[(PD_X + d) * cap + s] = 4.0;
        pd[(PD_V + d) * cap + s] = 0.0;
    }
    for (int q = 0; q < 9; ++q) pd[(PD_F + q) * cap + s] = (q % 4 == 0) ? 1.0 : 0.0;
    pd[PD_PF_ALLOW * cap + s] = 0.0;
}

// Quadratic B-spline weights of particle slot s from its position and base node.
template <class L>
__device__ __forceinline__ void pf_weights(const double* __restrict__ pd, int64_t cap, int64_t s, short4 b, double inv_dx, double w[3][3],
    double dwr[3][3], int& lx, int& ly, int& lz)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) bspline(inv_dx * pd[(PD_X + d) * cap + s] - (double)((&b.x)[d]), w[d], dwr[d]);
    lx = b.x & (L::BX - 1);
    ly = b.y & (L::BY - 1);
    lz = b.z & (L::BZ - 1);
}

// Loads field f of the 8 pages around a group into win[8][NPB].
template <int NPB>
__device__ __forceinline__ void pf_stage(double* win, const double* __restrict__ pfn, const int32_t* nbr, int f)
{
    for (int i = threadIdx.x; i < 8 * NPB; i += blockDim.x) {
        const int t = i / NPB, e = i - t * NPB;
        win[i] = pfn[((int64_t)nbr[t] * PN_FIELDS + f) * NPB + e];
    }
}

// Adds window acc[8][NC][NPB] into fields f0 .. f0 + NC - 1.
template <int NC, int NPB>
__device__ __forceinline__ void pf_flush(const double* acc, const int32_t* nbr, double* __restrict__ pfn, int f0)
{
    for (int i = threadIdx.x; i < 8 * NC * NPB; i += blockDim.x) {
        const double v = acc[i];
        if (v == 0.0) continue;
        const int t = i / (NC * NPB);
        const int r = i - t * NC * NPB;
        const int c = r / NPB, e = r - c * NPB;
        atomicAdd(&pfn[((int64_t)nbr[t] * PN_FIELDS + f0 + c) * NPB + e], v);
    }
}

// phaseP2G + the right-hand side and preconditioner sums: per particle
// vol = V0 det F, then sum_p w, sum_p c w (normalised phase field of the
// parabolic form), sum_p vol w and the lumped diagonal sum_p vol pf_Fp w (or
// vol (M pf_Fp + 1/dt) w).  Layered scatter (as P2G): a thread takes one cell
// and every layers-th particle of it, sums the cell's 27 node contributions in
// FP64 registers (two fields per pass) and adds them to the window once.
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_pf_p2g(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, PfParams p, double* __restrict__ pfn)
{
    constexpr int NPB = L::NPB;
    __shared__ double acc[8 * 4 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<4, NPB>(acc);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    const double inv_dx = 1.0 / dx;
    const int ce = threadIdx.x % NPB, layer = threadIdx.x / NPB, layers = blockDim.x / NPB;
    const int cnt = cl.cnt[ce], first = s0 + cl.start[ce];
    // pass 0: sum vol w and the diagonal (fields PN_VS, PN_DIAG); pass 1 (parabolic
    // only): sum w and sum c w (fields PN_MULT, PN_PHASE)
#pragma unroll 1
    for (int pass = 0; pass < ((p.M > 0) ? 2 : 1); ++pass) {
        double a[27][2];
#pragma unroll
        for (int m = 0; m < 27; ++m) a[m][0] = a[m][1] = 0.0;
        int lx = 0, ly = 0, lz = 0;
        for (int r = layer; r < cnt; r += layers) {
            const int s = first + r;
            double w[3][3], dwr[3][3];
            pf_weights<L>(pd, cap, s, base[s], inv_dx, w, dwr, lx, ly, lz);
            double v0, v1;
            if (pass == 0) {
                M3<double> F;
#pragma unroll
                for (int q = 0; q < 9; ++q) F.a[q] = pd[(PD_F + q) * cap + s];
                const double vol = pd[PD_VOL * cap + s] * m3_det(F);
                pd[PD_PF_VOL * cap + s] = vol;
                const double fp = pd[PD_PF_FP * cap + s];
                v0 = vol;
                v1 = (p.M > 0) ? vol * (p.M * fp + p.one_over_dt) : vol * fp;
            }
            else {
                v0 = 1.0;
                v1 = pd[PD_PF_C * cap + s];
            }
            for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int, int, int i, int j, int k, double wijk, const double*) {
                const int m = 9 * i + 3 * j + k;
                a[m][0] += v0 * wijk;
                a[m][1] += v1 * wijk;
            });
        }
        if (layer < cnt) {
            const int cx = ce >> (L::YB + L::ZB), cy = (ce >> L::ZB) & (L::BY - 1), cz = ce & (L::BZ - 1);
            const int f0 = (pass == 0) ? PN_VS : PN_MULT;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        int e;
                        const int t = win_slot<L>(cx + i, cy + j, cz + k, e);
                        double* dst = acc + t * 4 * NPB + f0 * NPB + e;
                        atomicAdd(dst, a[9 * i + 3 * j + k][0]);
                        atomicAdd(dst + NPB, a[9 * i + 3 * j + k][1]);
                    }
        }
    }
    __syncthreads();
    pf_flush<4, NPB>(acc, nbr, pfn, PN_MULT);
}

// The operator of the CG without its lumped mass (that is diag * x, added by
// k_pf_sq): q_i = sum_p [c_p w_ip] + M' (4 l0^2 vol_p grad c_p) . grad w_ip,
// grad c_p = sum_j s_j grad w_jp, c_p = vol pf_Fp sum_j s_j w_jp (consistent
// mass, lumping off only), M' = parabolic_M or 1.  Gather from the staged
// window, layered scatter as in k_pf_p2g.
template <class L, bool LUMP>
__global__ void __launch_bounds__(XF_THREADS) k_pf_apply(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    const double* __restrict__ pd, int64_t cap, const short4* __restrict__ base, double dx, PfParams p, double* __restrict__ pfn,
    const PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    constexpr int NPB = L::NPB;
    __shared__ double win[8 * NPB];
    __shared__ double acc[8 * NPB];
    __shared__ int32_t nbr[8];
    __shared__ CellLayout<L> cl;
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<1, NPB>(acc);
    const int s0 = group_start[g], s1 = group_start[g + 1];
    build_cell_layout<L>(cl, base, s0, s1);
    pf_stage<NPB>(win, pfn, nbr, PN_S);
    __syncthreads();
    const double inv_dx = 1.0 / dx;
    const double mg = (p.M > 0) ? p.M : 1.0;
    const int ce = threadIdx.x % NPB, layer = threadIdx.x / NPB, layers = blockDim.x / NPB;
    const int cnt = cl.cnt[ce], first = s0 + cl.start[ce];
    double a[27];
#pragma unroll
    for (int m = 0; m < 27; ++m) a[m] = 0.0;
    int lx = 0, ly = 0, lz = 0;
    for (int r = layer; r < cnt; r += layers) {
        const int s = first + r;
        double w[3][3], dwr[3][3];
        pf_weights<L>(pd, cap, s, base[s], inv_dx, w, dwr, lx, ly, lz);
        double c0 = 0, g0[3] = { 0, 0, 0 };
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double wijk, const double* dw) {
            const double xv = win[t * NPB + e];
            if (!LUMP) c0 += xv * wijk;
#pragma unroll
            for (int d = 0; d < 3; ++d) g0[d] += xv * dw[d];
        });
        const double vol = pd[PD_PF_VOL * cap + s], l0 = pd[PD_PF_L0 * cap + s];
        if (!LUMP) c0 *= vol * pd[PD_PF_FP * cap + s];
        const double gs = vol * 4.0 * l0 * l0;
#pragma unroll
        for (int d = 0; d < 3; ++d) g0[d] *= gs;
        for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int, int, int i, int j, int k, double wijk, const double* dw) {
            double v = (g0[0] * dw[0] + g0[1] * dw[1] + g0[2] * dw[2]) * mg;
            if (!LUMP) v += c0 * wijk;
            a[9 * i + 3 * j + k] += v;
        });
    }
    if (layer < cnt) {
        const int cx = ce >> (L::YB + L::ZB), cy = (ce >> L::ZB) & (L::BY - 1), cz = ce & (L::BZ - 1);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    int e;
                    const int t = win_slot<L>(cx + i, cy + j, cz + k, e);
                    atomicAdd(acc + t * NPB + e, a[9 * i + 3 * j + k]);
                }
    }
    __syncthreads();
    pf_flush<1, NPB>(acc, nbr, pfn, PN_Q);
}

// NeoHookeanBorden::get_psi_pos (NeoHookeanBorden.cpp:53-66).
__device__ __forceinline__ double nhb_psi_pos(double mu, double kappa, const M3<double>& F)
{
    const double J = m3_det(F);
    const double a = pow(J, -1.0 / 3.0);
    double tr = 0;
#pragma unroll
    for (int q = 0; q < 9; ++q) tr += (a * F.a[q]) * (a * F.a[q]);
    const double psi_dev = mu / 2 * (tr - 3);
    const double psi_vol = kappa / 2 * ((J * J - 1) / 2 - log(J));
    return (J >= 1) ? psi_vol + psi_dev : psi_dev;
}

// phaseG2P: c <- max(min(c, c_new), 0) with c_new = sum_i w_ip phi_i (elliptic)
// or c + sum_i w_ip phi_i (parabolic) for particles that may be damaged; then
// Update_Phase_Field_Fp (PhaseField.h:70-76) and g = c^2 (1 - k) + k for every
// NeoHookeanBorden particle.
template <class L>
__global__ void __launch_bounds__(XF_THREADS) k_pf_g2p(const int32_t* __restrict__ group_start, const int32_t* __restrict__ group_nbr,
    double* __restrict__ pd, const int32_t* __restrict__ pi, int64_t cap, const short4* __restrict__ base, double dx, PfParams p,
    const double* __restrict__ pfn)
{
    constexpr int NPB = L::NPB;
    __shared__ double win[8 * NPB];
    __shared__ int32_t nbr[8];
    const int g = blockIdx.x;
    if (threadIdx.x < 8) nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    __syncthreads();
    pf_stage<NPB>(win, pfn, nbr, PN_PHASE);
    __syncthreads();
    const double inv_dx = 1.0 / dx;
    const int s0 = group_start[g], s1 = group_start[g + 1];
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        double c = pd[PD_PF_C * cap + s];
        if (pd[PD_PF_ALLOW * cap + s] != 0.0) {
            double w[3][3], dwr[3][3];
            int lx, ly, lz;
            pf_weights<L>(pd, cap, s, base[s], inv_dx, w, dwr, lx, ly, lz);
            double pf = 0;
            for_stencil<L>(lx, ly, lz, w, dwr, inv_dx, [&](int t, int e, int, int, int, double wijk, const double*) { pf += wijk * win[t * NPB + e]; });
            const double new_c = (p.M > 0) ? c + pf : pf;
            const double lo = (new_c < c) ? new_c : c; // std::min(c, new_c)
            c = (lo < 0.0) ? 0.0 : lo;                 // std::max(., 0)
            pd[PD_PF_C * cap + s] = c;
        }
        if (pi[PI_KIND * cap + s] != ZMPM_MODEL_NEOHOOKEAN_BORDEN) continue;
        M3<double> F;
#pragma unroll
        for (int q = 0; q < 9; ++q) F.a[q] = pd[(PD_F + q) * cap + s];
        const double psi_pos = nhb_psi_pos(pd[PD_MU * cap + s], pd[PD_KAPPA * cap + s], F);
        double H = pd[PD_PF_H * cap + s];
        const double k = pd[PD_PF_K * cap + s];
        if (psi_pos > H) {
            const double hmax = pd[PD_PF_HMAX * cap + s];
            H = (hmax < psi_pos) ? hmax : psi_pos;
            pd[PD_PF_H * cap + s] = H;
            pd[PD_PF_FP * cap + s] = 4 * pd[PD_PF_L0 * cap + s] * (1 - k) * H * pd[PD_PF_ISC * cap + s] + 1;
        }
        pd[PD_G * cap + s] = c * c * (1 - k) + k;
    }
}

// ------------------------------------------------------------------ nodes --
// Start of the CG from x = 0: phi = sum c w / sum w (parabolic), b = (M + phi/dt)
// sum vol w (or sum vol w), r = b; partials of r.r and (r / diag).r.  Nodes with
// m == 0 (outside the reference's index set) hold zero.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_pf_init(int64_t nn, const double* __restrict__ gm, double* __restrict__ pfn, PfParams p,
    double* __restrict__ part_rr, double* __restrict__ part_rho)
{
    double rr = 0, rho = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < nn; n += (int64_t)gridDim.x * ND_THREADS) {
        double* nd = pf_node<NPB>(pfn, n, 0);
        double ph = 0, r = 0;
        if (gm[n] != 0) {
            if (p.M > 0) ph = nd[PN_PHASE * NPB] / nd[PN_MULT * NPB];
            const double vs = nd[PN_VS * NPB];
            r = (p.M > 0) ? (p.M + ph / p.dt) * vs : vs;
            rr += r * r;
            rho += (r / nd[PN_DIAG * NPB]) * r;
        }
        nd[PN_PHASE * NPB] = ph;
        nd[PN_X * NPB] = 0;
        nd[PN_R * NPB] = r;
        nd[PN_S * NPB] = 0;
        nd[PN_Q * NPB] = 0;
    }
    rr = block_sum(rr);
    rho = block_sum(rho);
    if (threadIdx.x == 0) {
        part_rr[blockIdx.x] = rr;
        part_rho[blockIdx.x] = rho;
    }
}

__global__ void __launch_bounds__(ND_THREADS) k_pf_start(const double* __restrict__ part_rr, const double* __restrict__ part_rho, int nparts,
    PfScalars* __restrict__ sc)
{
    const double rr = reduce_partials(part_rr, nparts);
    const double rho = reduce_partials(part_rho, nparts);
    if (threadIdx.x == 0) {
        const double norm = sqrt(rr);
        sc->norm = norm;
        sc->rel_tol = norm * 1e-12; // ConjugateGradient.h:66 (double)
        sc->rho = rho;
        sc->rho_old = DBL_MAX;
        sc->alpha = 0;
        sc->it = 0;
        sc->iters = 0;
        sc->active = 1;
    }
}

// s = r / diag (first iteration) or (rho / rho_old) s + r / diag; q = 0.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_pf_dir(int64_t nn, const double* __restrict__ gm, double* __restrict__ pfn,
    const PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    const bool first = sc->it == 0;
    const double beta = sc->rho / sc->rho_old;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < nn; n += (int64_t)gridDim.x * ND_THREADS) {
        if (gm[n] == 0) continue;
        double* nd = pf_node<NPB>(pfn, n, 0);
        const double mr = nd[PN_R * NPB] / nd[PN_DIAG * NPB];
        nd[PN_S * NPB] = first ? mr : beta * nd[PN_S * NPB] + mr;
        nd[PN_Q * NPB] = 0;
    }
}

// q += diag * s (the lumped mass); partial s.q.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_pf_sq(int64_t nn, const double* __restrict__ gm, double* __restrict__ pfn, int lumping,
    double* __restrict__ part, const PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < nn; n += (int64_t)gridDim.x * ND_THREADS) {
        if (gm[n] == 0) continue;
        double* nd = pf_node<NPB>(pfn, n, 0);
        const double s = nd[PN_S * NPB];
        double q = nd[PN_Q * NPB];
        if (lumping) q += nd[PN_DIAG * NPB] * s;
        nd[PN_Q * NPB] = q;
        acc += s * q;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(ND_THREADS) k_pf_alpha(const double* __restrict__ part, int nparts, PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    const double sq = reduce_partials(part, nparts);
    if (threadIdx.x == 0) sc->alpha = (sq != 0) ? sc->rho / sq : DBL_MAX;
}

// x = alpha s + x, r = -alpha q + r; partials of r.r and (r / diag).r.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_pf_update(int64_t nn, const double* __restrict__ gm, double* __restrict__ pfn,
    double* __restrict__ part_rr, double* __restrict__ part_rho, const PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    const double alpha = sc->alpha;
    double rr = 0, rho = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < nn; n += (int64_t)gridDim.x * ND_THREADS) {
        if (gm[n] == 0) continue;
        double* nd = pf_node<NPB>(pfn, n, 0);
        nd[PN_X * NPB] = alpha * nd[PN_S * NPB] + nd[PN_X * NPB];
        const double r = -alpha * nd[PN_Q * NPB] + nd[PN_R * NPB];
        nd[PN_R * NPB] = r;
        rr += r * r;
        rho += (r / nd[PN_DIAG * NPB]) * r;
    }
    rr = block_sum(rr);
    rho = block_sum(rho);
    if (threadIdx.x == 0) {
        part_rr[blockIdx.x] = rr;
        part_rho[blockIdx.x] = rho;
    }
}

// End of an iteration: |r|, the stopping test of ConjugateGradient.h:96-99.
__global__ void __launch_bounds__(ND_THREADS) k_pf_end(const double* __restrict__ part_rr, const double* __restrict__ part_rho, int nparts,
    PfParams p, PfScalars* __restrict__ sc)
{
    if (!sc->active) return;
    const double rr = reduce_partials(part_rr, nparts);
    const double rho = reduce_partials(part_rho, nparts);
    if (threadIdx.x == 0) {
        const double norm = sqrt(rr);
        sc->norm = norm;
        sc->rho_old = sc->rho;
        sc->rho = rho;
        const int it = sc->it;
        if (norm < p.tol || norm < sc->rel_tol || it == p.max_it) {
            sc->active = 0;
            sc->iters = it;
        }
        else
            sc->it = it + 1;
    }
}

// phi = x - phi (parabolic) or x.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_pf_final(int64_t nn, const double* __restrict__ gm, double* __restrict__ pfn, PfParams p)
{
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < nn; n += (int64_t)gridDim.x * ND_THREADS) {
        if (gm[n] == 0) continue;
        double* nd = pf_node<NPB>(pfn, n, 0);
        nd[PN_PHASE * NPB] = (p.M > 0) ? nd[PN_X * NPB] - nd[PN_PHASE * NPB] : nd[PN_X * NPB];
    }
}

// ------------------------------------------------------------- host side --
int launch_phase_field_delete(Ctx* ctx)
{
    if (ctx->P == 0) return ZMPM_OK;
    k_pf_delete<<<(unsigned)((ctx->P + 255) / 256), 256, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->pi.as<int32_t>(), ctx->Pcap, ctx->P,
        ctx->pf_delete);
    ++g_kernel_launches;
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

template <class L>
static int phase_field_impl(Ctx* ctx, int32_t* iterations, double* residual)
{
    constexpr int NPB = L::NPB;
    cudaStream_t st = ctx->stream;
    const int64_t nn = ctx->B * NPB, G = ctx->G;
    *iterations = 0;
    *residual = 0;
    if (nn == 0 || G == 0) return ZMPM_OK;
    ZMPM_CUDA(ctx->pfn.ensure((size_t)PN_FIELDS * nn * sizeof(double)));
    ZMPM_CUDA(ctx->pfsc.ensure(sizeof(PfScalars)));
    ZMPM_CUDA(cudaMemsetAsync(ctx->pfn.p, 0, (size_t)PN_FIELDS * nn * sizeof(double), st));
    PfParams p;
    p.M = ctx->pf_M;
    p.dt = ctx->dt;
    p.one_over_dt = 1.0 / ctx->dt;
    p.tol = ctx->pf_cg_tol;
    p.lumping = ctx->pf_lumping ? 1 : 0;
    p.max_it = ctx->pf_cg_max;
    int64_t c = (nn + ND_THREADS - 1) / ND_THREADS;
    const int nb = (int)(c < 1 ? 1 : (c > RED_MAX_CTAS ? RED_MAX_CTAS : c));
    double* red = ctx->red.as<double>();
    double* pA = red + RED_A * RED_MAX_CTAS;
    double* pB = red + RED_B * RED_MAX_CTAS;
    PfScalars* sc = ctx->pfsc.as<PfScalars>();
    double* pfn = ctx->pfn.as<double>();
    const double* gm = ctx->gm.as<double>();
    const int32_t* gs = ctx->group_start.as<int32_t>();
    const int32_t* gn = ctx->group_nbr.as<int32_t>();
    const short4* base = ctx->base.as<short4>();
    double* pd = ctx->pd.as<double>();
    const double dx = ctx->cfg.dx;

    k_pf_p2g<L><<<(unsigned)G, XF_THREADS, 0, st>>>(gs, gn, pd, ctx->Pcap, base, dx, p, pfn);
    k_pf_init<NPB><<<nb, ND_THREADS, 0, st>>>(nn, gm, pfn, p, pA, pB);
    k_pf_start<<<1, ND_THREADS, 0, st>>>(pA, pB, nb, sc);
    g_kernel_launches += 3;
    ZMPM_CUDA(cudaGetLastError());
    // iterations are enqueued in batches; the flag read between batches ends the loop
    PfScalars hs{};
    const int total = p.max_it + 1;
    for (int k = 0; k < total;) {
        // the reference's default tolerance usually stops the CG after its first
        // iteration: check after 1, then after 4 more, then every 16
        const int batch = std::min(k == 0 ? 1 : (k == 1 ? 4 : 16), total - k);
        for (int j = 0; j < batch; ++j) {
            k_pf_dir<NPB><<<nb, ND_THREADS, 0, st>>>(nn, gm, pfn, sc);
            if (p.lumping)
                k_pf_apply<L, true><<<(unsigned)G, XF_THREADS, 0, st>>>(gs, gn, pd, ctx->Pcap, base, dx, p, pfn, sc);
            else
                k_pf_apply<L, false><<<(unsigned)G, XF_THREADS, 0, st>>>(gs, gn, pd, ctx->Pcap, base, dx, p, pfn, sc);
            k_pf_sq<NPB><<<nb, ND_THREADS, 0, st>>>(nn, gm, pfn, p.lumping, pA, sc);
            k_pf_alpha<<<1, ND_THREADS, 0, st>>>(pA, nb, sc);
            k_pf_update<NPB><<<nb, ND_THREADS, 0, st>>>(nn, gm, pfn, pA, pB, sc);
            k_pf_end<<<1, ND_THREADS, 0, st>>>(pA, pB, nb, p, sc);
        }
        ZMPM_CUDA(cudaGetLastError());
        k += batch;
        ZMPM_CUDA(cudaMemcpyAsync(&hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, st));
        ZMPM_CUDA(cudaStreamSynchronize(st));
        // kernels that did work: the iterations that ran, 6 each
        if (!hs.active) break;
    }
    g_kernel_launches += 6 * (int64_t)(hs.active ? hs.it : hs.iters + 1);
    k_pf_final<NPB><<<nb, ND_THREADS, 0, st>>>(nn, gm, pfn, p);
    k_pf_g2p<L><<<(unsigned)G, XF_THREADS, 0, st>>>(gs, gn, pd, ctx->pi.as<int32_t>(), ctx->Pcap, base, dx, p, pfn);
    g_kernel_launches += 2;
    ZMPM_CUDA(cudaGetLastError());
    *iterations = hs.active ? hs.it : hs.iters;
    *residual = hs.norm;
    return ZMPM_OK;
}

int run_phase_field(Ctx* ctx, int32_t* iterations, double* residual)
{
    return ctx->layout == 1 ? phase_field_impl<Layout244>(ctx, iterations, residual) : phase_field_impl<Layout444>(ctx, iterations, residual);
}

} // namespace zmpm
