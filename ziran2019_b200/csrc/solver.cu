// Grid-node kernels and the backward-Euler Newton solve.
//
// Node vectors are block-dense: [B][3][NPB] doubles, B pages in page-map
// order.  Nodes with m == 0 hold zero in every vector, so they drop out of
// every product (the reference never stores them: getNumNodes,
// MpmGrid.h:123-136).
//
// Reductions are deterministic: each node kernel writes one FP64 partial per
// CTA (fixed grid size for a given B) and the next kernel's CTAs all reduce
// the partials in the same fixed order in their prologue, so every CTA sees
// bit-identical scalars (alpha, beta, norms) without a host round trip.
// Scalars that one kernel both reads and updates are double-buffered by
// iteration parity.
//
// Newton (NewtonsMethod.h:42-66):
//   update -> residual -> check/init -> [Krylov iteration] x K -> dv += step
// MINRES follows Minres.h:69-175, CG follows ConjugateGradient.h:99-147
// (the working `solve`), both with the 1/m preconditioner
// (MpmSimulationBase.cpp:617-623) and the collision projection.
#include "internal.cuh"
#include "mat3.cuh"

namespace zmpm {

constexpr int ND_THREADS = 256;

int launch_p2g(Ctx* ctx);
int launch_g2p(Ctx* ctx);
int launch_hvp_gated(Ctx* ctx, const double* x, double* out, bool gated, int it);

// ------------------------------------------------------------ reductions --
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// Block sum; result valid in every thread.
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double ws[ND_THREADS / 32];
    __shared__ double total;
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = (lane < ND_THREADS / 32) ? ws[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) total = t;
    }
    __syncthreads();
    return total;
}
// Sum of n partials in a fixed order (identical in every CTA).
__device__ __forceinline__ double reduce_partials(const double* __restrict__ part, int n)
{
    double s = 0;
    for (int i = threadIdx.x; i < n; i += ND_THREADS) s += part[i];
    return block_sum(s);
}

struct NodeGeom {
    int64_t nn;        // B * NPB
    int parts;         // CTAs of node kernels
};

template <int NPB>
__device__ __forceinline__ int64_t vidx(int64_t n, int d) // component d of node n in [B][3][NPB]
{
    int64_t b = n / NPB;
    int e = (int)(n - b * NPB);
    return (b * 3 + d) * NPB + e;
}

__device__ __forceinline__ void project3(const int8_t* col, const double* P6, int64_t nn, int64_t n, double v[3])
{
    if (!col[n]) return;
    double p00 = P6[n], p01 = P6[nn + n], p02 = P6[2 * nn + n], p11 = P6[3 * nn + n], p12 = P6[4 * nn + n], p22 = P6[5 * nn + n];
    double a = v[0], b = v[1], c = v[2];
    v[0] = p00 * a + p01 * b + p02 * c;
    v[1] = p01 * a + p11 * b + p12 * c;
    v[2] = p02 * a + p12 * b + p22 * c;
}

// ------------------------------------------------------- collision query --
// AnalyticLevelSet::queryInside for half space, sphere and axis-aligned box.
__device__ bool collider_inside(const DevCollider& c, const double X[3], double N[3])
{
    if (c.shape == ZMPM_HALF_SPACE) {
        double nn = sqrt(c.b[0] * c.b[0] + c.b[1] * c.b[1] + c.b[2] * c.b[2]);
        double n[3] = { c.b[0] / nn, c.b[1] / nn, c.b[2] / nn };
        double phi = n[0] * (X[0] - c.a[0]) + n[1] * (X[1] - c.a[1]) + n[2] * (X[2] - c.a[2]);
        if (phi <= 0) {
            N[0] = n[0];
            N[1] = n[1];
            N[2] = n[2];
            return true;
        }
        return false;
    }
    if (c.shape == ZMPM_SPHERE) {
        double t[3] = { X[0] - c.a[0], X[1] - c.a[1], X[2] - c.a[2] };
        double d2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (d2 < c.radius * c.radius) {
            double d = sqrt(d2);
            if (d < 1e-7) {
                N[0] = 1;
                N[1] = N[2] = 0;
            }
            else {
                N[0] = (1 / d) * t[0];
                N[1] = (1 / d) * t[1];
                N[2] = (1 / d) * t[2];
            }
            return true;
        }
        return false;
    }
    double h[3], xp[3], dd[3];
    for (int i = 0; i < 3; ++i) {
        h[i] = (c.b[i] - c.a[i]) / 2;
        xp[i] = X[i] - (c.a[i] + c.b[i]) / 2;
        dd[i] = fabs(xp[i]) - h[i];
    }
    int im = 0;
    for (int i = 1; i < 3; ++i)
        if (dd[i] > dd[im]) im = i;
    double q2 = 0;
    for (int i = 0; i < 3; ++i) {
        double q = dd[i] > 0 ? dd[i] : 0.0;
        q2 += q * q;
    }
    double phi = fmin(dd[im], 0.0) + sqrt(q2);
    if (phi > 0) return false;
    N[0] = N[1] = N[2] = 0;
    N[im] = xp[im] >= 0 ? 1.0 : -1.0;
    return true;
}

// AnalyticCollisionObject::detectAndResolveCollision (CollisionObject.cpp:340-400)
__device__ bool collider_resolve(const DevCollider& c, const double x[3], double v[3], double n[3])
{
    if (c.type == ZMPM_GHOST) return false;
    double xb[3] = { x[0] - c.t[0], x[1] - c.t[1], x[2] - c.t[2] };
    double ios = 1 / c.s;
    double X[3];
    for (int i = 0; i < 3; ++i) X[i] = (c.R[i] * xb[0] + c.R[3 + i] * xb[1] + c.R[6 + i] * xb[2]) * ios;
    double N[3];
    if (!collider_inside(c, X, N)) return false;
    double vo[3] = { c.omega[1] * xb[2] - c.omega[2] * xb[1], c.omega[2] * xb[0] - c.omega[0] * xb[2], c.omega[0] * xb[1] - c.omega[1] * xb[0] };
    for (int i = 0; i < 3; ++i) vo[i] += (c.dsdt * ios) * xb[i] + c.dtdt[i];
    for (int i = 0; i < 3; ++i) v[i] -= vo[i];
    if (c.type == ZMPM_STICKY) {
        v[0] = v[1] = v[2] = 0;
    }
    else {
        for (int i = 0; i < 3; ++i) n[i] = c.R[3 * i] * N[0] + c.R[3 * i + 1] * N[1] + c.R[3 * i + 2] * N[2];
        double dot = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
        if (c.type == ZMPM_SLIP || dot < 0) {
            for (int i = 0; i < 3; ++i) v[i] -= n[i] * dot;
            if (c.friction != 0 && dot < 0) {
                double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                if (-dot * c.friction < vn)
                    for (int i = 0; i < 3; ++i) v[i] += v[i] / vn * dot * c.friction;
                else
                    v[0] = v[1] = v[2] = 0;
            }
        }
    }
    for (int i = 0; i < 3; ++i) v[i] += vo[i];
    return true;
}

// ------------------------------------------------------------- grid init --
// particlesToGrid normalisation (MpmSimulationBase.cpp:474-485) +
// buildInitialDvAndVnForNewton (:1105-1136): vn, dv, vstar = vn + dv,
// collision projection P = I - K K^T, active-node count.
template <class L>
__global__ void __launch_bounds__(ND_THREADS) k_grid_init(NodeGeom ng, const double* __restrict__ gm, const double* __restrict__ gmv,
    const int4* __restrict__ block_page, double dx, double gx, double gy, double gz, double dt, const DevCollider* __restrict__ cols, int ncols,
    double* __restrict__ vn, double* __restrict__ dv, double* __restrict__ vstar, int8_t* __restrict__ col, double* __restrict__ P6,
    unsigned long long* __restrict__ nactive, int32_t* __restrict__ flags)
{
    constexpr int NPB = L::NPB;
    int local = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const int64_t b = n / NPB;
        const int e = (int)(n - b * NPB);
        const double m = gm[n];
        double v[3] = { 0, 0, 0 }, d[3] = { 0, 0, 0 };
        int8_t c = 0;
        double P[6] = { 1, 0, 0, 1, 0, 1 };
        if (m != 0) {
            ++local;
            for (int k = 0; k < 3; ++k) v[k] = gmv[vidx<NPB>(n, k)] / m;
            const int4 bp = block_page[b];
            const int lx = e >> (L::YB + L::ZB), ly = (e >> L::ZB) & (L::BY - 1), lz = e & (L::BZ - 1);
            double xi[3] = { (bp.x * L::BX + lx) * dx, (bp.y * L::BY + ly) * dx, (bp.z * L::BZ + lz) * dx };
            double vi[3] = { v[0], v[1], v[2] };
            // AnalyticCollisionObject::multiObjectCollision (CollisionObject.cpp:66-105)
            bool any = false;
            int slip = 0;
            double K[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
            for (int o = 0; o < ncols; ++o) {
                if (cols[o].type == ZMPM_GHOST) continue;
                double nrm[3] = { 0, 0, 0 };
                bool hit = collider_resolve(cols[o], xi, vi, nrm);
                any = hit || any;
                if (!hit) continue;
                if (cols[o].type == ZMPM_STICKY) {
                    for (int r = 0; r < 3; ++r)
                        for (int q = 0; q < 3; ++q) K[r][q] = (r == q) ? 1.0 : 0.0;
                    break;
                }
                for (int q = 0; q < slip; ++q) {
                    double dd = K[0][q] * nrm[0] + K[1][q] * nrm[1] + K[2][q] * nrm[2];
                    for (int r = 0; r < 3; ++r) nrm[r] -= dd * K[r][q];
                }
                double len = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
                if (len != 0) {
                    for (int r = 0; r < 3; ++r) K[r][slip] = nrm[r] / len;
                    if (++slip == 3) break;
                }
            }
            if (any) {
                c = 1;
                double KK[3][3];
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) KK[r][q] = K[r][0] * K[q][0] + K[r][1] * K[q][1] + K[r][2] * K[q][2];
                P[0] = 1 - KK[0][0];
                P[1] = -KK[0][1];
                P[2] = -KK[0][2];
                P[3] = 1 - KK[1][1];
                P[4] = -KK[1][2];
                P[5] = 1 - KK[2][2];
                for (int k = 0; k < 3; ++k) d[k] = vi[k] - v[k];
            }
            else {
                d[0] = gx * dt;
                d[1] = gy * dt;
                d[2] = gz * dt;
            }
        }
        for (int k = 0; k < 3; ++k) {
            int64_t vi = vidx<NPB>(n, k);
            vn[vi] = v[k];
            dv[vi] = d[k];
            vstar[vi] = (m != 0) ? v[k] + d[k] : 0.0;
        }
        col[n] = c;
        for (int k = 0; k < 6; ++k) P6[k * ng.nn + n] = P[k];
    }
    __shared__ int tot;
    if (threadIdx.x == 0) tot = 0;
    __syncthreads();
    atomicAdd(&tot, local);
    __syncthreads();
    if (threadIdx.x == 0 && tot) atomicAdd(nactive, (unsigned long long)tot);
}

// ------------------------------------------------------- Newton residual --
// r = project(dt m g + dt f - m dv) with f = facc (BackwardEuler.h:101-124,
// Inertia.cpp:32-41); zeroes facc; partial sum of |r|^2/m (computeNorm).
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_residual(NodeGeom ng, const double* __restrict__ gm, double* __restrict__ facc,
    const double* __restrict__ dv, const int8_t* __restrict__ col, const double* __restrict__ P6, double gx, double gy, double gz, double dt,
    double* __restrict__ res, double* __restrict__ part, const SolverScalars* __restrict__ sc)
{
    if (sc && sc->newton_done) return;
    double acc = 0;
    const double g[3] = { gx, gy, gz };
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        double r[3] = { 0, 0, 0 };
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            if (m != 0) r[k] = dt * g[k] * m + dt * facc[i] - (dt / dt) * m * dv[i];
            facc[i] = 0;
        }
        if (m != 0) {
            project3(col, P6, ng.nn, n, r);
            acc += (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) / m;
        }
        for (int k = 0; k < 3; ++k) res[vidx<NPB>(n, k)] = r[k];
    }
    double s = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Solver buffers of one linear solve.
struct KrylovBufs {
    double *x, *r, *p, *q, *tmp;      // CG
    double *Q[3], *M[3], *Z[2];       // MINRES
    double* hacc;                     // Hessian accumulator
};

struct NewtonParams {
    int32_t minres;
    double tol, abs_tol, tol_scale, dt;
};

// Newton check (NewtonsMethod.h:48-61) + start of the linear solve: x = 0,
// CG: r = res, q = r/m, p = q, partial r.q;  MINRES: Q0 = res, Z0 = res/m,
// Q1 = Q2 = M* = 0, partial z.q.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_newton_check(NodeGeom ng, const double* __restrict__ gm, const double* __restrict__ res,
    KrylovBufs kb, NewtonParams np, double* __restrict__ part_in, double* __restrict__ part_out, SolverScalars* __restrict__ sc, int first)
{
    if (sc->newton_done) return;
    const double norm = sqrt(reduce_partials(part_in, ng.parts));
    const bool done = (norm < np.tol) || !(norm == norm);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (first) sc->res_initial = norm;
        sc->res_final = norm;
        if (done) {
            sc->newton_done = 1;
            sc->converged = (norm == norm) ? 1 : 0;
            sc->stop_at = 0;
        }
        else {
            double mx = norm > np.tol ? norm : np.tol;
            double rel = np.tol_scale * sqrt(mx);
            sc->rel_tol = rel < 0.5 ? rel : 0.5;
        }
    }
    if (done) return;
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            double rv = res[i];
            double z = (m != 0) ? rv / m : 0.0;
            kb.x[i] = 0;
            if (np.minres) {
                kb.Q[0][i] = rv;
                kb.Q[1][i] = 0;
                kb.Q[2][i] = 0;
                kb.M[0][i] = 0;
                kb.M[1][i] = 0;
                kb.M[2][i] = 0;
                kb.Z[0][i] = z;
            }
            else {
                kb.r[i] = rv;
                kb.q[i] = z;
                kb.p[i] = z;
            }
            acc += z * rv;
        }
    }
    double s = block_sum(acc);
    if (threadIdx.x == 0) part_out[blockIdx.x] = s;
}

// Initial preconditioned norm and local tolerance; MINRES normalises Q0, Z0.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_krylov_start(NodeGeom ng, KrylovBufs kb, NewtonParams np, const double* __restrict__ part_in,
    SolverScalars* __restrict__ sc)
{
    if (sc->newton_done) return;
    const double dotv = reduce_partials(part_in, ng.parts);
    const double rnorm = sqrt(dotv);
    const double rel = sc->rel_tol;
    const double lt = fmin(rel * rnorm, np.abs_tol);
    const bool active = !(rnorm < lt);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->rnorm = rnorm;
        sc->local_tol = lt;
        sc->stop_at = active ? 0x7fffffff : 0;
        if (np.minres) {
            double* mr = sc->mr[0];
            mr[MR_GC0] = mr[MR_GC1] = mr[MR_GC2] = 1;
            mr[MR_GS0] = mr[MR_GS1] = mr[MR_GS2] = 0;
            mr[MR_RHS0] = rnorm;
            mr[MR_RHS1] = 0;
            mr[MR_BETA_KP1] = rnorm;
        }
        else {
            sc->zTrk = dotv;
            sc->mr[0][0] = dotv; // CG keeps zTrk double-buffered in mr[parity][0]
        }
    }
    if (!np.minres || !active || !(rnorm > 0)) return;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS)
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            kb.Q[0][i] /= rnorm;
            kb.Z[0][i] /= rnorm;
        }
}

// out = project(m x + dt^2 hacc), zero hacc, partial dot(out, w).
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_apply_A(NodeGeom ng, const double* __restrict__ gm, const int8_t* __restrict__ col,
    const double* __restrict__ P6, double dt2, const double* __restrict__ xin, double* __restrict__ hacc, double* __restrict__ out,
    double* __restrict__ part, const SolverScalars* __restrict__ sc, int gated, int project, int it)
{
    if (gated && (sc->newton_done || it >= sc->stop_at)) return;
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        double o[3], xv[3];
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            xv[k] = xin[i];
            o[k] = (m != 0) ? m * xv[k] + dt2 * hacc[i] : 0.0;
            hacc[i] = 0;
        }
        if (m != 0 && project) project3(col, P6, ng.nn, n, o);
        for (int k = 0; k < 3; ++k) {
            out[vidx<NPB>(n, k)] = o[k];
            acc += o[k] * xv[k];
        }
    }
    if (part) {
        double s = block_sum(acc);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

// ---------------------------------------------------------------- CG ------
// x += alpha p; r -= alpha tmp; q = r/m; partial q.r
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_cg_b(NodeGeom ng, const double* __restrict__ gm, KrylovBufs kb, const double* __restrict__ part_in,
    double* __restrict__ part_out, const SolverScalars* __restrict__ sc, int it)
{
    if (sc->newton_done || it >= sc->stop_at) return;
    const double alpha = sc->mr[it & 1][0] / reduce_partials(part_in, ng.parts);
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            kb.x[i] += kb.p[i] * alpha;
            double r = kb.r[i] - kb.tmp[i] * alpha;
            kb.r[i] = r;
            double q = (m != 0) ? r / m : 0.0;
            kb.q[i] = q;
            acc += q * r;
        }
    }
    double s = block_sum(acc);
    if (threadIdx.x == 0) part_out[blockIdx.x] = s;
}

// beta, p = q + beta p, convergence
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_cg_c(NodeGeom ng, KrylovBufs kb, const double* __restrict__ part_in, SolverScalars* __restrict__ sc, int it,
    int nit)
{
    if (sc->newton_done || it >= sc->stop_at) return;
    const double zTrk = reduce_partials(part_in, ng.parts);
    const double beta = zTrk / sc->mr[it & 1][0];
    const double rnorm = sqrt(zTrk);
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->mr[(it + 1) & 1][0] = zTrk;
        sc->rnorm = rnorm;
        sc->krylov_iters += 1;
        sc->hvp_count += 1;
        if (nit < 64) sc->kcount[nit] += 1;
        if (rnorm < sc->local_tol) sc->stop_at = it + 1; // the reference tests at the next loop top
    }
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS)
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            kb.p[i] = kb.q[i] + beta * kb.p[i];
        }
}

// ------------------------------------------------------------- MINRES -----
// qkp1 -= alpha qk + beta_k qkm1; z = qkp1/m; partial z.qkp1
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_mr_b(NodeGeom ng, const double* __restrict__ gm, double* __restrict__ qkp1,
    const double* __restrict__ qk, const double* __restrict__ qkm1, double* __restrict__ zout, const double* __restrict__ part_in,
    double* __restrict__ part_out, const SolverScalars* __restrict__ sc, int it)
{
    if (sc->newton_done || it >= sc->stop_at) return;
    const double alpha = reduce_partials(part_in, ng.parts);
    const double beta_k = sc->mr[it & 1][MR_BETA_KP1];
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            double q = qkp1[i];
            q -= alpha * qk[i];
            q -= beta_k * qkm1[i];
            qkp1[i] = q;
            double z = (m != 0) ? q / m : 0.0;
            zout[i] = z;
            acc += z * q;
        }
    }
    double s = block_sum(acc);
    if (threadIdx.x == 0) part_out[blockIdx.x] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // alpha of this iteration is needed by the Givens update in k_mr_c
        const_cast<SolverScalars*>(sc)->mr[(it + 1) & 1][MR_TK] = alpha;
    }
}

// Givens update (Minres.h:151-175), normalisation, search direction and x.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_mr_c(NodeGeom ng, double* __restrict__ qkp1, double* __restrict__ zout,
    const double* __restrict__ zin, const double* __restrict__ mkm1, const double* __restrict__ mkm2, double* __restrict__ mk_out,
    double* __restrict__ x, const double* __restrict__ part_in, SolverScalars* __restrict__ sc, int it, int nit)
{
    if (sc->newton_done || it >= sc->stop_at) return;
    const double dz = reduce_partials(part_in, ng.parts);
    const double* cur = sc->mr[it & 1];
    const double alpha_k = sc->mr[(it + 1) & 1][MR_TK];
    const double beta_k = cur[MR_BETA_KP1];
    const double beta_kp1 = sqrt(dz > 0 ? dz : 0.0);
    // Gkm2 = Gkm1, Gkm1 = Gk
    double c2 = cur[MR_GC1], s2 = cur[MR_GS1], c1 = cur[MR_GC0], s1 = cur[MR_GS0];
    double e0 = c2 * 0 - s2 * beta_k, e1 = s2 * 0 + c2 * beta_k;
    const double epsilon = e0;
    double d0 = c1 * e1 - s1 * alpha_k, d1 = s1 * e1 + c1 * alpha_k;
    const double delta = d0;
    double t0 = d1, t1 = beta_kp1;
    double c0 = 1, s0 = 0;
    {
        double dd = t0 * t0 + t1 * t1;
        double sd = sqrt(dd);
        if (sd != 0) {
            double tt = 1 / sd;
            c0 = t0 * tt;
            s0 = -t1 * tt;
        }
    }
    const double gamma = c0 * t0 - s0 * t1;
    const double r0 = cur[MR_RHS0], r1 = cur[MR_RHS1];
    const double tk = c0 * r0 - s0 * r1;
    const double residual = s0 * r0 + c0 * r1;
    const double rnorm = residual < 0 ? -residual : residual;
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* nx = sc->mr[(it + 1) & 1];
        nx[MR_GC0] = c0;
        nx[MR_GS0] = s0;
        nx[MR_GC1] = c1;
        nx[MR_GS1] = s1;
        nx[MR_GC2] = c2;
        nx[MR_GS2] = s2;
        nx[MR_RHS0] = residual;
        nx[MR_RHS1] = 0;
        nx[MR_BETA_KP1] = beta_kp1;
        sc->rnorm = rnorm;
        sc->krylov_iters += 1;
        sc->hvp_count += 1;
        if (nit < 64) sc->kcount[nit] += 1;
        if (rnorm < sc->local_tol) sc->stop_at = it + 1; // the reference tests at the next loop top
    }
    const bool norm = beta_kp1 > 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS)
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            if (norm) {
                qkp1[i] /= beta_kp1;
                zout[i] /= beta_kp1;
            }
            double mk = (zin[i] - delta * mkm1[i] - epsilon * mkm2[i]) / gamma;
            mk_out[i] = mk;
            x[i] += tk * mk;
        }
}


// dv += step; vstar = vn + dv on active nodes.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_newton_step(NodeGeom ng, const double* __restrict__ gm, const double* __restrict__ step,
    const double* __restrict__ vn, double* __restrict__ dv, double* __restrict__ vstar, SolverScalars* __restrict__ sc)
{
    if (sc->newton_done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->newton_iters += 1;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const bool act = gm[n] != 0;
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            double d = dv[i] + step[i];
            dv[i] = d;
            vstar[i] = act ? vn[i] + d : 0.0;
        }
    }
}

// ------------------------------------------------------------ host side --
static NodeGeom node_geom(const Ctx* ctx)
{
    NodeGeom ng;
    ng.nn = ctx->B * ctx->npb();
    int64_t c = (ng.nn + ND_THREADS - 1) / ND_THREADS;
    ng.parts = (int)(c < 1 ? 1 : (c > RED_MAX_CTAS ? RED_MAX_CTAS : c));
    return ng;
}

int ensure_node_buffers(Ctx* ctx)
{
    const int64_t nn = ctx->B * ctx->npb();
    const size_t vec = (size_t)(3 * nn) * sizeof(double);
    ZMPM_CUDA(ctx->gm.ensure(nn * sizeof(double)));
    ZMPM_CUDA(ctx->gmv.ensure(vec));
    ZMPM_CUDA(ctx->vn.ensure(vec));
    ZMPM_CUDA(ctx->dv.ensure(vec));
    ZMPM_CUDA(ctx->vstar.ensure(vec));
    ZMPM_CUDA(ctx->facc.ensure(vec));
    ZMPM_CUDA(ctx->res.ensure(vec));
    ZMPM_CUDA(ctx->proj.ensure(6 * nn * sizeof(double)));
    ZMPM_CUDA(ctx->collided.ensure(nn));
    for (int i = 0; i < 10; ++i) ZMPM_CUDA(ctx->kv[i].ensure(vec));
    return ZMPM_OK;
}

int run_p2g(Ctx* ctx)
{
    cudaStream_t st = ctx->stream;
    const int64_t nn = ctx->B * ctx->npb();
    int rc = ensure_node_buffers(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaMemsetAsync(ctx->gm.p, 0, nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->gmv.p, 0, 3 * nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->facc.p, 0, 3 * nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->kv[9].p, 0, 3 * nn * sizeof(double), st)); // Hessian accumulator
    rc = launch_p2g(ctx);
    if (rc) return rc;
    rc = upload_colliders(ctx, ctx->time);
    if (rc) return rc;
    NodeGeom ng = node_geom(ctx);
    DevCounters* dc = ctx->counters.as<DevCounters>();
    const double* g = ctx->cfg.gravity;
    if (nn > 0) {
        if (ctx->layout == 1)
            k_grid_init<Layout244><<<ng.parts, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->block_page.as<int4>(),
                ctx->cfg.dx, g[0], g[1], g[2], ctx->dt, ctx->dcolliders.as<DevCollider>(), (int)ctx->colliders.size(), ctx->vn.as<double>(),
                ctx->dv.as<double>(), ctx->vstar.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
                reinterpret_cast<unsigned long long*>(&dc->N), &dc->flags);
        else
            k_grid_init<Layout444><<<ng.parts, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->block_page.as<int4>(),
                ctx->cfg.dx, g[0], g[1], g[2], ctx->dt, ctx->dcolliders.as<DevCollider>(), (int)ctx->colliders.size(), ctx->vn.as<double>(),
                ctx->dv.as<double>(), ctx->vstar.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
                reinterpret_cast<unsigned long long*>(&dc->N), &dc->flags);
        ++g_kernel_launches;
    }
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

int launch_residual(Ctx* ctx)
{
    NodeGeom ng = node_geom(ctx);
    if (ng.nn == 0) return ZMPM_OK;
    const double* g = ctx->cfg.gravity;
    double* part = ctx->red.as<double>() + RED_A * RED_MAX_CTAS;
    if (ctx->layout == 1)
        k_residual<32><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->gm.as<double>(), ctx->facc.as<double>(), ctx->dv.as<double>(),
            ctx->collided.as<int8_t>(), ctx->proj.as<double>(), g[0], g[1], g[2], ctx->dt, ctx->res.as<double>(), part, ctx->scal.as<SolverScalars>());
    else
        k_residual<64><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->gm.as<double>(), ctx->facc.as<double>(), ctx->dv.as<double>(),
            ctx->collided.as<int8_t>(), ctx->proj.as<double>(), g[0], g[1], g[2], ctx->dt, ctx->res.as<double>(), part, ctx->scal.as<SolverScalars>());
    ++g_kernel_launches;
    return ZMPM_OK;
}

// b = m x + dt^2 q (no projection, the reference's multiply).
int finalize_multiply(Ctx* ctx, const double* x, double* q)
{
    NodeGeom ng = node_geom(ctx);
    if (ng.nn == 0) return ZMPM_OK;
    const double dt2 = ctx->dt * ctx->dt;
    if (ctx->layout == 1)
        k_apply_A<32><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(), dt2, x,
            ctx->kv[9].as<double>(), q, nullptr, nullptr, 0, 0, 0);
    else
        k_apply_A<64><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(), dt2, x,
            ctx->kv[9].as<double>(), q, nullptr, nullptr, 0, 0, 0);
    ++g_kernel_launches;
    return ZMPM_OK;
}

template <int NPB>
static int newton_impl(Ctx* ctx, const zmpm_solver& s)
{
    cudaStream_t st = ctx->stream;
    NodeGeom ng = node_geom(ctx);
    SolverScalars* sc = ctx->scal.as<SolverScalars>();
    double* part = ctx->red.as<double>();
    double *pA = part + RED_A * RED_MAX_CTAS, *pB = part + RED_B * RED_MAX_CTAS, *pC = part + RED_C * RED_MAX_CTAS;
    KrylovBufs kb;
    double** v = reinterpret_cast<double**>(ctx->kv);
    (void)v;
    kb.x = ctx->kv[0].as<double>();
    kb.r = ctx->kv[1].as<double>();
    kb.p = ctx->kv[2].as<double>();
    kb.q = ctx->kv[3].as<double>();
    kb.tmp = ctx->kv[4].as<double>();
    kb.Q[0] = ctx->kv[1].as<double>();
    kb.Q[1] = ctx->kv[2].as<double>();
    kb.Q[2] = ctx->kv[3].as<double>();
    kb.M[0] = ctx->kv[4].as<double>();
    kb.M[1] = ctx->kv[5].as<double>();
    kb.M[2] = ctx->kv[6].as<double>();
    kb.Z[0] = ctx->kv[7].as<double>();
    kb.Z[1] = ctx->kv[8].as<double>();
    kb.hacc = ctx->kv[9].as<double>();
    NewtonParams np{ s.linear_solver == ZMPM_MINRES ? 1 : 0, s.newton_tolerance, s.krylov_tolerance, s.linear_solve_tolerance_scale, ctx->dt };
    const double dt2 = ctx->dt * ctx->dt;
    ZMPM_CUDA(cudaMemsetAsync(sc, 0, sizeof(SolverScalars), st));
    if (ng.nn == 0) return ZMPM_OK;
    const int nb = ng.parts;
    const bool prof = ctx->profiling && s.newton_max_iterations <= 64;
    ctx->prof_newton = prof ? s.newton_max_iterations : 0;
    ctx->prof_krylov = s.krylov_max_iterations;
    if (prof) {
        size_t need = 2 * (size_t)s.newton_max_iterations * s.krylov_max_iterations;
        while (ctx->hvp_ev.size() < need) {
            cudaEvent_t e;
            ZMPM_CUDA(cudaEventCreate(&e));
            ctx->hvp_ev.push_back(e);
        }
    }
    for (int it = 0; it < s.newton_max_iterations; ++it) {
        int rc = launch_update(ctx);
        if (rc) return rc;
        rc = launch_residual(ctx);
        if (rc) return rc;
        k_newton_check<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->res.as<double>(), kb, np, pA, pB, sc, it == 0 ? 1 : 0);
        ++g_kernel_launches;
        k_krylov_start<NPB><<<nb, ND_THREADS, 0, st>>>(ng, kb, np, pB, sc);
        ++g_kernel_launches;
        for (int k = 0; k < s.krylov_max_iterations; ++k) {
            if (np.minres) {
                double* zin = kb.Z[k & 1];
                double* zout = kb.Z[(k + 1) & 1];
                double* qk = kb.Q[k % 3];
                double* qkm1 = kb.Q[(k + 2) % 3];
                double* qkp1 = kb.Q[(k + 1) % 3];
                double* mk = kb.M[k % 3];
                double* mkm1 = kb.M[(k + 2) % 3];
                double* mkm2 = kb.M[(k + 1) % 3];
                if (prof) ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * (it * s.krylov_max_iterations + k)], st));
                launch_hvp_gated(ctx, zin, kb.hacc, true, k);
                if (prof) ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * (it * s.krylov_max_iterations + k) + 1], st));
                k_apply_A<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(), dt2, zin,
                    kb.hacc, qkp1, pA, sc, 1, 1, k);
                ++g_kernel_launches;
                k_mr_b<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), qkp1, qk, qkm1, zout, pA, pC, sc, k);
                ++g_kernel_launches;
                k_mr_c<NPB><<<nb, ND_THREADS, 0, st>>>(ng, qkp1, zout, zin, mkm1, mkm2, mk, kb.x, pC, sc, k, it);
                ++g_kernel_launches;
            }
            else {
                if (prof) ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * (it * s.krylov_max_iterations + k)], st));
                launch_hvp_gated(ctx, kb.p, kb.hacc, true, k);
                if (prof) ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * (it * s.krylov_max_iterations + k) + 1], st));
                k_apply_A<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(), dt2, kb.p,
                    kb.hacc, kb.tmp, pA, sc, 1, 1, k);
                ++g_kernel_launches;
                k_cg_b<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), kb, pA, pC, sc, k);
                ++g_kernel_launches;
                k_cg_c<NPB><<<nb, ND_THREADS, 0, st>>>(ng, kb, pC, sc, k, it);
                ++g_kernel_launches;
            }
        }
        k_newton_step<NPB><<<nb, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), kb.x, ctx->vn.as<double>(), ctx->dv.as<double>(),
            ctx->vstar.as<double>(), sc);
        ++g_kernel_launches;
        ZMPM_CUDA(cudaGetLastError());
    }
    // the reference evaluates the residual once more only at the top of the
    // next Newton iteration; vstar already holds vn + dv of the last step.
    return ZMPM_OK;
}

int run_newton(Ctx* ctx, const zmpm_solver& s)
{
    return ctx->layout == 1 ? newton_impl<32>(ctx, s) : newton_impl<64>(ctx, s);
}

int run_g2p(Ctx* ctx)
{
    int rc = launch_g2p(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

} // namespace zmpm
