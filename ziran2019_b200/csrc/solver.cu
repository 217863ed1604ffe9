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
#include <algorithm>

#include "hvp.cuh"
#include "internal.cuh"
#include "mat3.cuh"
#include "node.cuh"

namespace zmpm {

int launch_p2g(Ctx* ctx);
int launch_g2p(Ctx* ctx, bool plastic);

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
__device__ bool collider_inside(const DevCollider& c, const double X[3], double N[3], double* phi_out = nullptr)
{
    if (c.shape == ZMPM_HALF_SPACE) {
        double nn = sqrt(c.b[0] * c.b[0] + c.b[1] * c.b[1] + c.b[2] * c.b[2]);
        double n[3] = { c.b[0] / nn, c.b[1] / nn, c.b[2] / nn };
        double phi = n[0] * (X[0] - c.a[0]) + n[1] * (X[1] - c.a[1]) + n[2] * (X[2] - c.a[2]);
        if (phi <= 0) {
            if (phi_out) *phi_out = phi;
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
            if (phi_out) *phi_out = d - c.radius;
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
    if (phi_out) *phi_out = phi;
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

// AnalyticCollisionObject::queryInside in world space (CollisionObject.cpp:232-246):
// signed distance scaled by s, world normal.
__device__ bool collider_query_world(const DevCollider& c, const double x[3], double& phi, double n[3])
{
    double xb[3] = { x[0] - c.t[0], x[1] - c.t[1], x[2] - c.t[2] };
    double ios = 1 / c.s;
    double X[3];
    for (int i = 0; i < 3; ++i) X[i] = (c.R[i] * xb[0] + c.R[3 + i] * xb[1] + c.R[6 + i] * xb[2]) * ios;
    double N[3];
    if (!collider_inside(c, X, N, &phi)) return false;
    for (int i = 0; i < 3; ++i) n[i] = c.R[3 * i] * N[0] + c.R[3 * i + 1] * N[1] + c.R[3 * i + 2] * N[2];
    phi *= c.s;
    return true;
}

// AnalyticCollisionObject::getBoundaryVelocityAndNormal (CollisionObject.cpp:313-338)
__device__ bool collider_boundary(const DevCollider& c, const double x[3], double vb[3], double n[3])
{
    if (c.type == ZMPM_GHOST) return false;
    double xb[3] = { x[0] - c.t[0], x[1] - c.t[1], x[2] - c.t[2] };
    double ios = 1 / c.s;
    double X[3];
    for (int i = 0; i < 3; ++i) X[i] = (c.R[i] * xb[0] + c.R[3 + i] * xb[1] + c.R[6 + i] * xb[2]) * ios;
    double N[3];
    if (!collider_inside(c, X, N)) return false;
    vb[0] = c.omega[1] * xb[2] - c.omega[2] * xb[1];
    vb[1] = c.omega[2] * xb[0] - c.omega[0] * xb[2];
    vb[2] = c.omega[0] * xb[1] - c.omega[1] * xb[0];
    for (int i = 0; i < 3; ++i) vb[i] += (c.dsdt * ios) * xb[i] + c.dtdt[i];
    for (int i = 0; i < 3; ++i) n[i] = c.R[3 * i] * N[0] + c.R[3 * i + 1] * N[1] + c.R[3 * i + 2] * N[2];
    return true;
}

// AnalyticCollisionObject::multiObjectCollision (CollisionObject.cpp:66-105), or
// with fake_separate multiObjectCollisionWithFakeSeparate (:108-156), where a
// SEPARATE object the node already leaves does not collide.  Returns whether
// any object collided; vi is resolved and P6 = I - K K^T (xx, xy, xz, yy, yz, zz).
__device__ bool multi_collide(const DevCollider* __restrict__ cols, int ncols, const double xi[3], double vi[3], double P6[6], bool fake_separate)
{
    bool any = false;
    int slip = 0;
    double K[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
    for (int o = 0; o < ncols; ++o) {
        if (cols[o].type == ZMPM_GHOST) continue;
        double nrm[3] = { 0, 0, 0 };
        const double old[3] = { vi[0], vi[1], vi[2] };
        bool hit = collider_resolve(cols[o], xi, vi, nrm);
        if (hit && fake_separate && cols[o].type == ZMPM_SEPARATE) {
            double vb[3] = { 0, 0, 0 }, nb[3] = { 0, 0, 0 };
            collider_boundary(cols[o], xi, vb, nb);
            if ((old[0] - vb[0]) * nb[0] + (old[1] - vb[1]) * nb[1] + (old[2] - vb[2]) * nb[2] > 0) {
                vi[0] = old[0];
                vi[1] = old[1];
                vi[2] = old[2];
                hit = false;
            }
        }
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
    double KK[3][3];
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) KK[r][q] = K[r][0] * K[q][0] + K[r][1] * K[q][1] + K[r][2] * K[q][2];
    if (any) {
        P6[0] = 1 - KK[0][0];
        P6[1] = -KK[0][1];
        P6[2] = -KK[0][2];
        P6[3] = 1 - KK[1][1];
        P6[4] = -KK[1][2];
        P6[5] = 1 - KK[2][2];
    }
    return any;
}

// ------------------------------------------------------------- grid init --
// particlesToGrid normalisation (MpmSimulationBase.cpp:474-485) +
// buildInitialDvAndVnForNewton (:1105-1136): vn, dv, vstar = vn + dv,
// collision projection P = I - K K^T, active-node count.
template <class L>
__global__ void __launch_bounds__(ND_THREADS) k_grid_init(NodeGeom ng, const double* __restrict__ gm, const double* __restrict__ gmv,
    const int4* __restrict__ block_page, double dx, double gx, double gy, double gz, double dt, const DevCollider* __restrict__ cols, int ncols,
    double* __restrict__ vn, double* __restrict__ dv, double* __restrict__ vstar, int8_t* __restrict__ col, double* __restrict__ P6,
    unsigned long long* __restrict__ nactive, int32_t* __restrict__ flags, float4* __restrict__ vstar_f)
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
            if (multi_collide(cols, ncols, xi, vi, P, false)) {
                c = 1;
                for (int k = 0; k < 3; ++k) d[k] = vi[k] - v[k];
            }
            else {
                d[0] = gx * dt;
                d[1] = gy * dt;
                d[2] = gz * dt;
            }
        }
        double vs[3];
        for (int k = 0; k < 3; ++k) {
            int64_t vi = vidx<NPB>(n, k);
            vn[vi] = v[k];
            dv[vi] = d[k];
            vs[k] = (m != 0) ? v[k] + d[k] : 0.0;
            vstar[vi] = vs[k];
        }
        if (vstar_f) vstar_f[n] = make_float4((float)vs[0], (float)vs[1], (float)vs[2], 0.f);
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

// ------------------------------------------------------ explicit update --
// particlesToGrid normalisation + gridVelocityExplicitUpdate
// (MpmSimulationBase.cpp:474-485, 818-865): vn = (mv)/m, v = vn + dt g +
// f dt/m with the colliders at t (cols), then for nodes that did not collide
// trialCollision with the colliders moved to t + dt (cols1;
// MpmSimulationBase.cpp:298-311, CollisionObject.cpp:48-64):
// v -= (phi(x_i + dt v) / dt) n.  vstar = v, dv = v - vn, facc zeroed.
template <class L>
__global__ void __launch_bounds__(ND_THREADS) k_grid_explicit(NodeGeom ng, const double* __restrict__ gm, const double* __restrict__ gmv,
    double* __restrict__ facc, const int4* __restrict__ block_page, double dx, double gx, double gy, double gz, double dt,
    const DevCollider* __restrict__ cols, const DevCollider* __restrict__ cols1, int ncols, int trial, double* __restrict__ vn,
    double* __restrict__ dv, double* __restrict__ vstar, int8_t* __restrict__ col, unsigned long long* __restrict__ nactive)
{
    constexpr int NPB = L::NPB;
    const double g[3] = { gx, gy, gz };
    int local = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const int64_t b = n / NPB;
        const int e = (int)(n - b * NPB);
        const double m = gm[n];
        double v[3] = { 0, 0, 0 }, vi[3] = { 0, 0, 0 };
        int8_t c = 0;
        if (m != 0) {
            ++local;
            const double dt_over_mi = dt / m;
            for (int k = 0; k < 3; ++k) {
                v[k] = gmv[vidx<NPB>(n, k)] / m;
                vi[k] = v[k] + g[k] * dt + facc[vidx<NPB>(n, k)] * dt_over_mi;
            }
            const int4 bp = block_page[b];
            const int lx = e >> (L::YB + L::ZB), ly = (e >> L::ZB) & (L::BY - 1), lz = e & (L::BZ - 1);
            const double xi[3] = { (bp.x * L::BX + lx) * dx, (bp.y * L::BY + ly) * dx, (bp.z * L::BZ + lz) * dx };
            double P[6];
            c = multi_collide(cols, ncols, xi, vi, P, false) ? 1 : 0;
            if (!c && trial)
                for (int o = 0; o < ncols; ++o) {
                    if (cols1[o].type == ZMPM_GHOST) continue;
                    const double xt[3] = { xi[0] + dt * vi[0], xi[1] + dt * vi[1], xi[2] + dt * vi[2] };
                    double phi, nrm[3];
                    if (collider_query_world(cols1[o], xt, phi, nrm))
                        for (int k = 0; k < 3; ++k) vi[k] -= (phi / dt) * nrm[k];
                }
        }
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            vn[i] = v[k];
            dv[i] = vi[k] - v[k];
            vstar[i] = vi[k];
            facc[i] = 0;
        }
        col[n] = c;
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

// Solver buffers of one linear solve.  MINRES rotates its three Lanczos
// vectors Q, three search directions M and two preconditioned vectors Z by the
// iteration index k read from device memory, so the same kernels (and the same
// graph body) serve every iteration.
struct KrylovBufs {
    double *x, *r, *p, *q, *tmp;      // CG
    double *Q[3], *M[3], *Z[2];       // MINRES
    float* Zf[2];                     // FP32 node-major copies of Z ([B][NPB][4]) for the FP32 product (MIXED MINRES), or null
    float* pf;                        // FP32 node-major copy of p for the FP32 product (MIXED CG), or null
    double* hacc;                     // Hessian accumulator
    const double* pre;                // diagonal preconditioner per node (the mass for Newton)
};

struct NewtonParams {
    int32_t minres, kmax, nmax;
    int32_t escalate;                 // MIXED: FP64 residual once the FP32 one stalls
    double tol, abs_tol, tol_scale, dt;
};

__device__ __forceinline__ bool krylov_off(const SolverScalars* sc) { return sc->newton_done || !sc->kactive; }

// Role selection by iteration index without indexing the parameter arrays at
// run time (which would copy the kernel parameters to local memory).
__device__ __forceinline__ double* sel3(double* const (&a)[3], int i) { return i == 0 ? a[0] : (i == 1 ? a[1] : a[2]); }
template <class T>
__device__ __forceinline__ T* sel2(T* const (&a)[2], int i) { return i == 0 ? a[0] : a[1]; }

// The Newton residual of k_residual fused with the operands of the linear
// solve's start, in one node pass: r = project(dt m g + dt f - m dv), facc
// zeroed, x = 0, and from r the Krylov start vectors (CG: r, q = p = r/pre;
// MINRES: Q0 = r, Z0 = r/pre and its FP32 copy, Q1 = Q2 = M* = Z1 = 0);
// partials of |r|^2/m (computeNorm, BackwardEuler.h:101-140) and of z.r.
// When k_newton_start then finds the norm converged these vectors go unused.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS, 4) k_residual_start(NodeGeom ng, const double* __restrict__ gm, double* __restrict__ facc,
    const double* __restrict__ dv, const int8_t* __restrict__ col, const double* __restrict__ P6, double gx, double gy, double gz, double dt,
    KrylovBufs kb, int minres, double* __restrict__ part_norm, double* __restrict__ part_zr, const SolverScalars* __restrict__ sc)
{
    if (sc->newton_done) return;
    double acc = 0, zr = 0;
    const double g[3] = { gx, gy, gz };
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        double r[3] = { 0, 0, 0 };
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            if (m != 0) r[k] = dt * g[k] * m + dt * facc[i] - (dt / dt) * m * dv[i];
            facc[i] = 0;
        }
        if (m != 0) {
            project3(col, P6, ng.nn, n, r);
            acc += (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) / m;
        }
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            const double rv = r[k];
            const double z = (m != 0) ? rv / kb.pre[n] : 0.0;
            kb.x[i] = 0;
            if (minres) {
                kb.Q[0][i] = rv;
                kb.Q[1][i] = 0;
                kb.Q[2][i] = 0;
                kb.M[0][i] = 0;
                kb.M[1][i] = 0;
                kb.M[2][i] = 0;
                kb.Z[0][i] = z;
                kb.Z[1][i] = 0;
                if (kb.Zf[0]) {
                    kb.Zf[0][4 * n + k] = (float)z;
                    kb.Zf[1][4 * n + k] = 0;
                }
            }
            else {
                kb.r[i] = rv;
                kb.q[i] = z;
                kb.p[i] = z;
                if (kb.pf) kb.pf[4 * n + k] = (float)z;
            }
            zr += z * rv;
        }
    }
    const double s0 = block_sum(acc);
    const double s1 = block_sum(zr);
    if (threadIdx.x == 0) {
        part_norm[blockIdx.x] = s0;
        part_zr[blockIdx.x] = s1;
    }
}

// Newton check (NewtonsMethod.h:48-61) and, unless converged, the start of
// the linear solve (k_krylov_start's scalars).  One CTA.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_newton_start(NodeGeom ng, NewtonParams np, const double* __restrict__ part_norm,
    const double* __restrict__ part_zr, SolverScalars* __restrict__ sc)
{
    if (sc->newton_done) return;
    const double norm = sqrt(reduce_partials(part_norm, ng.parts));
    const bool done = (norm < np.tol) || !(norm == norm);
    const double dotv = reduce_partials(part_zr, ng.parts);
    if (threadIdx.x != 0) return;
    if (sc->nit == 0) sc->res_initial = norm;
    // MIXED: a norm that did not halve means FP32 stress round-off now
    // dominates the residual; the rest of the solve evaluates it in FP64, and
    // this iteration takes no step (the residual is re-evaluated first)
    const bool stall = np.escalate && !done && !sc->fp64_res && sc->nit > 0 && !(norm <= 0.5 * sc->res_final);
    if (stall) sc->fp64_res = 1;
    sc->skip_step = stall ? 1 : 0;
    sc->res_final = norm;
    if (done) {
        sc->newton_done = 1;
        sc->converged = (norm == norm) ? 1 : 0;
        sc->kactive = 0;
        return;
    }
    const double mx = norm > np.tol ? norm : np.tol;
    const double rel0 = np.tol_scale * sqrt(mx);
    const double rel = rel0 < 0.5 ? rel0 : 0.5;
    sc->rel_tol = rel;
    // Minres.h:73-98, ConjugateGradient.h:108-117
    const double rnorm = sqrt(dotv);
    const double lt = fmin(rel * rnorm, np.abs_tol);
    const bool active = !(rnorm < lt) && np.kmax > 0 && !stall;
    sc->rnorm = rnorm;
    sc->local_tol = lt;
    sc->kit = 0;
    sc->kactive = active ? 1 : 0;
    if (np.minres) {
        double* mr = sc->mr[0];
        mr[MR_GC0] = mr[MR_GC1] = mr[MR_GC2] = 1;
        mr[MR_GS0] = mr[MR_GS1] = mr[MR_GS2] = 0;
        mr[MR_RHS0] = rnorm;
        mr[MR_RHS1] = 0;
        mr[MR_BETA_KP1] = rnorm;
    }
    else
        sc->mr[0][0] = dotv; // CG keeps zTrk double-buffered in mr[parity][0]
}

// Initial preconditioned norm and local tolerance (Minres.h:73-98,
// ConjugateGradient.h:108-117); MINRES keeps Q0, Z0 unnormalised (beta_0 =
// the norm divides them where they are read).  One CTA.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_krylov_start(NodeGeom ng, KrylovBufs kb, NewtonParams np, const double* __restrict__ part_in,
    SolverScalars* __restrict__ sc)
{
    if (sc->newton_done) return;
    const double dotv = reduce_partials(part_in, ng.parts);
    const double rnorm = sqrt(dotv);
    const double rel = sc->rel_tol;
    const double lt = fmin(rel * rnorm, np.abs_tol);
    const bool active = !(rnorm < lt) && np.kmax > 0 && !sc->skip_step;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->rnorm = rnorm;
        sc->local_tol = lt;
        sc->kit = 0;
        sc->kactive = active ? 1 : 0;
        if (np.minres) {
            double* mr = sc->mr[0];
            mr[MR_GC0] = mr[MR_GC1] = mr[MR_GC2] = 1;
            mr[MR_GS0] = mr[MR_GS1] = mr[MR_GS2] = 0;
            mr[MR_RHS0] = rnorm;
            mr[MR_RHS1] = 0;
            mr[MR_BETA_KP1] = rnorm;
        }
        else
            sc->mr[0][0] = dotv; // CG keeps zTrk double-buffered in mr[parity][0]
    }
}

// out = project(m x + dt^2 hacc) (BackwardEuler.h:322-351 then Minres.h:116);
// zeroes hacc; partial dot(out, x) when part != null.
// SKIP: massless slots (zero in every Krylov vector) are not touched.
template <int NPB, bool SKIP>
__device__ __forceinline__ void apply_A_body(NodeGeom ng, const double* __restrict__ gm, const int8_t* __restrict__ col,
    const double* __restrict__ P6, double dt2, const double* __restrict__ xin, double* __restrict__ hacc, double* __restrict__ out,
    double* __restrict__ part, int project)
{
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        if (SKIP && m == 0) continue;
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

// The reference's multiply without projection (test hooks).
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_apply_A(NodeGeom ng, const double* __restrict__ gm, const int8_t* __restrict__ col,
    const double* __restrict__ P6, double dt2, const double* __restrict__ xin, double* __restrict__ hacc, double* __restrict__ out)
{
    apply_A_body<NPB, false>(ng, gm, col, P6, dt2, xin, hacc, out, nullptr, 0);
}

// MINRES keeps its Lanczos vectors Q_j and preconditioned vectors Z_j
// unnormalised (Minres.h:170-173 divides them by beta_j at the end of
// iteration j - 1); every reader divides by beta_j, the same rounding as the
// stored normalised vector.  beta_j = 0 leaves them as they are, as there.
__device__ __forceinline__ double mr_norm(double v, double beta) { return beta > 0 ? v / beta : v; }

// The search direction of iteration j = k - 1 (Minres.h:167-170):
// M_j = (Z_j - delta M_{j-1} - epsilon M_{j-2}) / gamma, then x += t M_j.
// The Lanczos step computes its scalars; the vector update runs in the next
// iteration's operator pass or, after the last iteration, where the solve's x
// is used (k_newton_step, k_admm_dv_update).
struct MrPending {
    const double *z, *m1, *m2;
    double* out;
    double delta, eps, gamma, t, beta;
    bool on;
};
__device__ __forceinline__ MrPending mr_pending(const KrylovBufs& kb, const double* pend, int k)
{
    MrPending p;
    p.on = k > 0;
    p.z = sel2(kb.Z, (k + 1) & 1);   // Z_{k-1}, unnormalised
    p.m1 = sel3(kb.M, (k + 1) % 3);  // M_{k-2}
    p.m2 = sel3(kb.M, k % 3);        // M_{k-3}
    p.out = sel3(kb.M, (k + 2) % 3); // M_{k-1}
    p.delta = pend[0];
    p.eps = pend[1];
    p.gamma = pend[2];
    p.t = pend[3];
    p.beta = pend[4];                // beta_{k-1}
    return p;
}
__device__ __forceinline__ double mr_direction(const MrPending& p, int64_t i)
{
    return (mr_norm(p.z[i], p.beta) - p.delta * p.m1[i] - p.eps * p.m2[i]) / p.gamma;
}

// The Givens update of MINRES iteration k (Minres.h:151-175): from the state
// cur of iteration k (Minres.h:16-24), alpha = Z_k . W, beta_k and dz =
// Z~_{k+1} . Q~_{k+1}, the state of iteration k + 1 into nx and the deferred
// search direction's delta, epsilon, gamma, t and beta into pend; returns the
// preconditioned residual norm.
__device__ __forceinline__ double mr_givens(const double* cur, double alpha, double beta_k, double dz, double* nx, double* pend)
{
    const double beta_kp1 = sqrt(dz > 0 ? dz : 0.0);
    // Gkm2 = Gkm1, Gkm1 = Gk
    double c2 = cur[MR_GC1], s2 = cur[MR_GS1], c1 = cur[MR_GC0], s1 = cur[MR_GS0];
    double e0 = c2 * 0 - s2 * beta_k, e1 = s2 * 0 + c2 * beta_k;
    const double epsilon = e0;
    double d0 = c1 * e1 - s1 * alpha, d1 = s1 * e1 + c1 * alpha;
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
    nx[MR_GC0] = c0;
    nx[MR_GS0] = s0;
    nx[MR_GC1] = c1;
    nx[MR_GS1] = s1;
    nx[MR_GC2] = c2;
    nx[MR_GS2] = s2;
    nx[MR_RHS0] = residual;
    nx[MR_RHS1] = 0;
    nx[MR_BETA_KP1] = beta_kp1;
    pend[0] = delta;
    pend[1] = epsilon;
    pend[2] = gamma;
    pend[3] = tk;
    pend[4] = beta_k;
    return residual < 0 ? -residual : residual;
}

// ------------------------------------------------ persistent Krylov -----
// One cooperative launch runs a whole linear solve of the Newton iteration
// (ConjugateGradient::solve, ConjugateGradient.h:99-147, on the Newton
// operator): per iteration the Hessian-vector product of p (hvp_share over
// each CTA's even share of the particle groups), A p with its
// partial dot, the x / r / q update with its partial dot and p = q + beta p,
// separated by grid-wide barriers.  Every CTA reduces the per-CTA partials in
// the same fixed order, so all hold bit-identical scalars and take the same
// loop decision.  The barrier waits are bounded: a CTA that gives up raises
// FLAG_TIMEOUT and the abort flag, and every CTA returns at its next barrier.

// Block sum for FUSED_THREADS threads; the result in every thread.
__device__ __forceinline__ double block_sum_fused(double v)
{
    __shared__ double ws[FUSED_THREADS / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) ws[w] = v;
    __syncthreads();
    double t = 0;
#pragma unroll
    for (int i = 0; i < FUSED_THREADS / 32; ++i) t += ws[i];
    return t;
}
// Sum of n partials written by other CTAs of this kernel (read through L2), in
// a fixed order identical in every CTA.
__device__ __forceinline__ double reduce_partials_fused(const double* part, int n)
{
    double s = 0;
    for (int i = threadIdx.x; i < n; i += FUSED_THREADS) s += __ldcg(part + i);
    return block_sum_fused(s);
}

// Bounded grid-wide barrier (sense by generation count).  Returns false in
// every thread of the CTA when this CTA gave up after `limit` polls or another
// CTA did; the caller then returns.
__device__ __forceinline__ bool grid_sync(GridSync* gs, long long limit, int32_t* flags)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &gs->gen;
        volatile unsigned* vabort = &gs->abort;
        int good = 1;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&gs->count, 1u) == gridDim.x - 1) {
            gs->count = 0;
            __threadfence();
            atomicAdd(&gs->gen, 1u);
        }
        else {
            long long it = 0;
            while (*vgen == g) {
                if (*vabort) {
                    good = 0;
                    break;
                }
                if (++it > limit) {
                    atomicOr(flags, (int32_t)FLAG_TIMEOUT);
                    atomicExch(&gs->abort, 1u);
                    good = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (*vabort) good = 0;
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

struct HvpArgs {
    const int32_t *group_start, *group_nbr, *pi;
    const short4* base;
    const void *frac, *scr; // in the product's precision
    int64_t cap;
    double dx;
    int G;
};

// The product of x into out over this CTA's share of the particle groups.  A
// group's cost is about K particles' worth of fixed work (staging the window,
// the cell layout, the flush) plus its particles, so group g spans the
// weights [W(g), W(g + 1)), W(g) = group_start[g] + K g; the total weight is
// split evenly over the grid and a group whose weight range a share boundary
// cuts is split into two pieces at the matching particle (pieces of one group
// add to the same nodes).  K measured on B200 at 1M particles: about 192
// FP32 particles, 128 FP64 ones (the per-particle work costs more in FP64).
template <class L, class T, class TX, int CH, class Model>
__device__ __forceinline__ void hvp_share(HvpSmem<L, T, TX, CH>& hs, const HvpArgs& ha, const Model& model, const TX* x, double* out,
    int32_t* flags, int& phase)
{
    constexpr int PIECE_COST = sizeof(T) == 4 ? 192 : 128;
    if (ha.G <= 0) return;
    const int32_t* __restrict__ gs = ha.group_start;
    const int64_t total = (int64_t)gs[ha.G] + (int64_t)PIECE_COST * ha.G;
    const int64_t w0 = total * blockIdx.x / gridDim.x, w1 = total * (blockIdx.x + 1) / gridDim.x;
    if (w0 >= w1) return;
    int a = 0, b = ha.G - 1; // the last group whose weight range starts at or before w0
    while (a < b) {
        const int m = (a + b + 1) >> 1;
        if ((int64_t)gs[m] + (int64_t)PIECE_COST * m <= w0)
            a = m;
        else
            b = m - 1;
    }
    for (int g = a; g < ha.G; ++g) {
        const int g0 = gs[g], n = gs[g + 1] - g0;
        const int64_t wp = (int64_t)g0 + (int64_t)PIECE_COST * g + PIECE_COST; // weight of the group's first particle
        if (wp - PIECE_COST >= w1) break;
        const int64_t lo = w0 - wp, hi = w1 - wp;
        const int s0 = g0 + (int)(lo < 0 ? 0 : (lo > n ? n : lo)), s1 = g0 + (int)(hi < 0 ? 0 : (hi > n ? n : hi));
        if (s0 < s1)
            hvp_group<L, T, TX, CH>(hs, g, s0, s1, ha.group_nbr, model, ha.cap, ha.base, ha.dx, static_cast<const T*>(ha.frac), x, out, flags,
                phase++);
    }
}

template <class L, class T, class TX>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_cg_persistent(NodeGeom ng, HvpArgs ha, const double* __restrict__ gm,
    const int8_t* __restrict__ col, const double* __restrict__ P6, double dt2, KrylovBufs kb, double* __restrict__ part_a,
    double* __restrict__ part_b, SolverScalars* __restrict__ sc, int kmax, GridSync* __restrict__ gs, long long limit, int32_t* __restrict__ flags)
{
    if (sc->newton_done || !sc->kactive) return;
    constexpr int NPB = L::NPB;
    constexpr int CH = sizeof(T) == 4 ? 512 : 192;
    __shared__ HvpSmem<L, T, TX, CH> hs;
    if (threadIdx.x == 0) mbar_init(&hs.bar, 1);
    __syncthreads();
    int phase = 0;
    const int nit = sc->nit;
    int k = sc->kit;
    double zTr = sc->mr[k & 1][0];
    // the product's input: p, or its FP32 node-major copy when TX is float
    const TX* pin;
    if constexpr (sizeof(TX) == 4)
        pin = reinterpret_cast<const TX*>(kb.pf);
    else
        pin = reinterpret_cast<const TX*>(kb.p);
    const double local_tol = sc->local_tol;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
    for (;;) {
        // the Hessian-vector product of p into hacc
        hvp_share<L, T, TX, CH>(hs, ha, HvpModel<T>{ ha.pi, static_cast<const T*>(ha.scr), ha.cap }, pin, kb.hacc, flags, phase);
        if (!grid_sync(gs, limit, flags)) return;
        // tmp = project(m p + dt^2 hacc), hacc = 0; partial p . tmp (BackwardEuler.h:322-351)
        // (two nodes per step, every load issued before the arithmetic, as in
        // k_mr_persistent; massless nodes hold zeros and are not written)
        double acc = 0;
        for (int64_t n = t0; n < ng.nn; n += 2 * nt) {
            const bool in1 = n + nt < ng.nn;
            const int64_t nu[2] = { n, in1 ? n + nt : n };
            const double mm[2] = { gm[nu[0]], in1 ? gm[nu[1]] : 0.0 };
            double pv[2][3], hv[2][3];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t i = vidx<NPB>(nu[u], c);
                    pv[u][c] = kb.p[i];
                    hv[u][c] = kb.hacc[i];
                }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const double m = mm[u];
                if (m == 0) continue;
                double o[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    o[c] = m * pv[u][c] + dt2 * hv[u][c];
                    kb.hacc[vidx<NPB>(nu[u], c)] = 0;
                }
                project3(col, P6, ng.nn, nu[u], o);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    kb.tmp[vidx<NPB>(nu[u], c)] = o[c];
                    acc += o[c] * pv[u][c];
                }
            }
        }
        acc = block_sum_fused(acc);
        if (threadIdx.x == 0) part_a[blockIdx.x] = acc;
        if (!grid_sync(gs, limit, flags)) return;
        // x += alpha p; r -= alpha tmp; q = r / m; partial q . r
        const double alpha = zTr / reduce_partials_fused(part_a, gridDim.x);
        acc = 0;
        for (int64_t n = t0; n < ng.nn; n += 2 * nt) {
            const bool in1 = n + nt < ng.nn;
            const int64_t nu[2] = { n, in1 ? n + nt : n };
            const double mm[2] = { gm[nu[0]], in1 ? gm[nu[1]] : 0.0 };
            double xv[2][3], pv[2][3], rv[2][3], tv[2][3], pre[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                pre[u] = kb.pre[nu[u]];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t i = vidx<NPB>(nu[u], c);
                    xv[u][c] = kb.x[i];
                    pv[u][c] = kb.p[i];
                    rv[u][c] = kb.r[i];
                    tv[u][c] = kb.tmp[i];
                }
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (mm[u] == 0) continue;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t i = vidx<NPB>(nu[u], c);
                    kb.x[i] = xv[u][c] + pv[u][c] * alpha;
                    const double r = rv[u][c] - tv[u][c] * alpha;
                    kb.r[i] = r;
                    const double q = r / pre[u];
                    kb.q[i] = q;
                    acc += q * r;
                }
            }
        }
        acc = block_sum_fused(acc);
        if (threadIdx.x == 0) part_b[blockIdx.x] = acc;
        if (!grid_sync(gs, limit, flags)) return;
        // beta, p = q + beta p; the loop test of the next iteration
        const double zTr1 = reduce_partials_fused(part_b, gridDim.x);
        const double beta = zTr1 / zTr, rnorm = sqrt(zTr1);
        for (int64_t n = t0; n < ng.nn; n += 2 * nt) {
            const bool in1 = n + nt < ng.nn;
            const int64_t nu[2] = { n, in1 ? n + nt : n };
            const double mm[2] = { gm[nu[0]], in1 ? gm[nu[1]] : 0.0 };
            double qv[2][3], pv[2][3];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t i = vidx<NPB>(nu[u], c);
                    qv[u][c] = kb.q[i];
                    pv[u][c] = kb.p[i];
                }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                if (mm[u] == 0) continue;
                double pn[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    pn[c] = qv[u][c] + beta * pv[u][c];
                    kb.p[vidx<NPB>(nu[u], c)] = pn[c];
                }
                if (kb.pf) reinterpret_cast<float4*>(kb.pf)[nu[u]] = make_float4((float)pn[0], (float)pn[1], (float)pn[2], 0.f);
            }
        }
        ++k;
        zTr = zTr1;
        const bool go = !(rnorm < local_tol || k >= kmax);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc->mr[k & 1][0] = zTr1;
            sc->rnorm = rnorm;
            sc->krylov_iters += 1;
            sc->hvp_count += 1;
            sc->krylov_bodies += 1;
            if (nit < 64) sc->kcount[nit] += 1;
            sc->kit = k;
            if (!go) sc->kactive = 0;
        }
        if (!go) return;
        if (!grid_sync(gs, limit, flags)) return; // p complete before the next product
    }
}

// ------------------------------------------------ persistent MINRES -----
// One cooperative launch runs a whole MINRES solve (Minres.h:69-175) on the
// Newton operator (HvpModel; dt2 = dt^2, pre = m) or on ADMM's global operator
// (AdmmOpModel; dt2 = 1, pre = its preconditioner).  Per iteration k: the
// product of Z~_k (its FP32 node-major copy when TX is float) over each CTA's
// even share of the particle groups (hvp_share); the operator pass (the
// deferred direction of iteration k - 1, W = project(m Z_k + dt2 H Z_k),
// Minres.h:116, 167-170); the Lanczos step (Q~_{k+1} = W - alpha Q_k -
// beta_k Q_{k-1}, Z~_{k+1} = Q~_{k+1} / pre); the Givens update
// (Minres.h:151-175), which thread 0 of every CTA runs
// on the same fixed-order reductions, so every CTA holds the same MINRES state
// (in shared memory) and takes the same loop decision.  CTA 0 stores the state
// after each iteration (the Newton step applies the last deferred direction
// from it).  Three bounded grid barriers per iteration: the product is
// complete before the operator pass reads hacc, W before the Lanczos step, and
// Z~_{k+1} before the next product and the reduction of its norm.
// Nodes per thread and step in the node passes of k_mr_persistent (their
// loads all issue before the arithmetic: the passes are latency-bound).
constexpr int MR_UNROLL = 2;
template <class L, class T, class TX, class Model>
__global__ void __launch_bounds__(FUSED_THREADS, 4) k_mr_persistent(NodeGeom ng, HvpArgs ha, Model model, const double* __restrict__ gm,
    const int8_t* __restrict__ col, const double* __restrict__ P6, double dt2, KrylovBufs kb, double* __restrict__ part_a,
    double* __restrict__ part_b, SolverScalars* __restrict__ sc, int kmax, GridSync* __restrict__ gs, long long limit, int32_t* __restrict__ flags)
{
    if (sc->newton_done || !sc->kactive) return;
    constexpr int NPB = L::NPB;
    constexpr int CH = sizeof(T) == 4 ? 512 : 192;
    __shared__ HvpSmem<L, T, TX, CH> hs;
    // the MINRES state of iteration k (Minres.h:16-24), then the deferred
    // direction's scalars, beta_{k-1} and the residual norm
    __shared__ double mst[12 + 5 + 2];
    double* const pend = mst + 12;
    int k = sc->kit;
    if (threadIdx.x == 0) {
        mbar_init(&hs.bar, 1);
        for (int i = 0; i < 12; ++i) mst[i] = sc->mr[k & 1][i];
        for (int i = 0; i < 5; ++i) pend[i] = sc->pend[i];
        mst[17] = sc->mr[(k + 1) & 1][MR_BETA_KP1];
    }
    __syncthreads();
    int phase = 0;
    const int nit = sc->nit;
    const double local_tol = sc->local_tol;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
    for (;;) {
        // the product of Z~_k into hacc
        const TX* zin;
        if constexpr (sizeof(TX) == 4)
            zin = reinterpret_cast<const TX*>(sel2(kb.Zf, k & 1));
        else
            zin = reinterpret_cast<const TX*>(sel2(kb.Z, k & 1));
        hvp_share<L, T, TX, CH>(hs, ha, model, zin, kb.hacc, flags, phase);
        if (!grid_sync(gs, limit, flags)) return;
        // operator pass: the deferred direction of iteration k - 1;
        // W = project(m Z_k + dt2 H Z_k) into Q's slot k + 1; partial Z_k . W
        {
            const double* __restrict__ zk = sel2(kb.Z, k & 1);
            double* __restrict__ w = sel3(kb.Q, (k + 1) % 3);
            const MrPending pd = mr_pending(kb, pend, k);
            const double beta = mst[MR_BETA_KP1];
            double acc = 0;
            // MR_UNROLL nodes per step, every load issued before the arithmetic
            // (massless nodes hold zeros in every vector and are not written)
            for (int64_t n = t0; n < ng.nn; n += MR_UNROLL * nt) {
                int64_t nn2[MR_UNROLL];
                double mm[MR_UNROLL];
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u) {
                    const bool in = n + u * nt < ng.nn;
                    nn2[u] = in ? n + u * nt : n;
                    mm[u] = in ? gm[nn2[u]] : 0.0;
                }
                double zv[MR_UNROLL][3], hv[MR_UNROLL][3], mv[MR_UNROLL][3], xv[MR_UNROLL][3];
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int64_t i = vidx<NPB>(nn2[u], c);
                        zv[u][c] = zk[i];
                        hv[u][c] = kb.hacc[i];
                        mv[u][c] = pd.on ? mr_direction(pd, i) : 0.0;
                        xv[u][c] = pd.on ? kb.x[i] : 0.0;
                    }
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u) {
                    const double m = mm[u];
                    if (m == 0) continue;
                    double o[3], z[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int64_t i = vidx<NPB>(nn2[u], c);
                        if (pd.on) {
                            pd.out[i] = mv[u][c];
                            kb.x[i] = xv[u][c] + pd.t * mv[u][c];
                        }
                        z[c] = mr_norm(zv[u][c], beta);
                        o[c] = m * z[c] + dt2 * mr_norm(hv[u][c], beta);
                        kb.hacc[i] = 0;
                    }
                    project3(col, P6, ng.nn, nn2[u], o);
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        w[vidx<NPB>(nn2[u], c)] = o[c];
                        acc += o[c] * z[c];
                    }
                }
            }
            acc = block_sum_fused(acc);
            if (threadIdx.x == 0) part_a[blockIdx.x] = acc;
        }
        if (!grid_sync(gs, limit, flags)) return;
        // Lanczos step: Q~_{k+1} = W - alpha Q_k - beta_k Q_{k-1},
        // Z~_{k+1} = Q~_{k+1} / pre (and its FP32 copy); partial Z~_{k+1} . Q~_{k+1}
        const double alpha = reduce_partials_fused(part_a, gridDim.x);
        const double beta_k = mst[MR_BETA_KP1], beta_km1 = mst[17];
        {
            double* __restrict__ qkp1 = sel3(kb.Q, (k + 1) % 3);
            const double* __restrict__ qk = sel3(kb.Q, k % 3);
            const double* __restrict__ qkm1 = sel3(kb.Q, (k + 2) % 3);
            double* __restrict__ zout = sel2(kb.Z, (k + 1) & 1);
            float* __restrict__ zfout = sel2(kb.Zf, (k + 1) & 1);
            double acc = 0;
            for (int64_t n = t0; n < ng.nn; n += MR_UNROLL * nt) {
                int64_t nn2[MR_UNROLL];
                double mm[MR_UNROLL];
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u) {
                    const bool in = n + u * nt < ng.nn;
                    nn2[u] = in ? n + u * nt : n;
                    mm[u] = in ? gm[nn2[u]] : 0.0;
                }
                double pre[MR_UNROLL], qa[MR_UNROLL][3], qb[MR_UNROLL][3], qc[MR_UNROLL][3];
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u) {
                    pre[u] = kb.pre[nn2[u]];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int64_t i = vidx<NPB>(nn2[u], c);
                        qa[u][c] = qkp1[i];
                        qb[u][c] = qk[i];
                        qc[u][c] = qkm1[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < MR_UNROLL; ++u) {
                    if (mm[u] == 0) continue;
                    float zf[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int64_t i = vidx<NPB>(nn2[u], c);
                        double q = qa[u][c];
                        q -= alpha * mr_norm(qb[u][c], beta_k);
                        q -= beta_k * mr_norm(qc[u][c], beta_km1);
                        qkp1[i] = q;
                        const double z = q / pre[u];
                        zout[i] = z;
                        zf[c] = (float)z;
                        acc += z * q;
                    }
                    if (zfout) reinterpret_cast<float4*>(zfout)[nn2[u]] = make_float4(zf[0], zf[1], zf[2], 0.f);
                }
            }
            acc = block_sum_fused(acc);
            if (threadIdx.x == 0) part_b[blockIdx.x] = acc;
        }
        if (!grid_sync(gs, limit, flags)) return;
        const double dz = reduce_partials_fused(part_b, gridDim.x);
        if (threadIdx.x == 0) {
            double nx[12] = {};
            mst[18] = mr_givens(mst, alpha, beta_k, dz, nx, pend);
            for (int i = 0; i < 12; ++i) mst[i] = nx[i];
            mst[17] = beta_k;
        }
        __syncthreads();
        const double rnorm = mst[18];
        ++k;
        const bool go = !(rnorm < local_tol || k >= kmax);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            for (int i = 0; i < 12; ++i) sc->mr[k & 1][i] = mst[i];
            for (int i = 0; i < 5; ++i) sc->pend[i] = pend[i];
            sc->rnorm = rnorm;
            sc->krylov_iters += 1;
            sc->hvp_count += 1;
            sc->krylov_bodies += 1;
            if (nit < 64) sc->kcount[nit] += 1;
            sc->kit = k;
            if (!go) sc->kactive = 0;
        }
        if (!go) return;
    }
}

// dv += x (the linear solve's step, with MINRES's deferred last update);
// vstar = vn + dv on active nodes.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_newton_step(NodeGeom ng, const double* __restrict__ gm, KrylovBufs kb, int minres,
    const double* __restrict__ vn, double* __restrict__ dv, double* __restrict__ vstar, const SolverScalars* __restrict__ sc,
    float4* __restrict__ vstar_f)
{
    if (sc->newton_done) return;
    MrPending pd = mr_pending(kb, sc->pend, sc->kit);
    pd.on = pd.on && minres;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const bool act = gm[n] != 0;
        double vs[3];
        for (int k = 0; k < 3; ++k) {
            int64_t i = vidx<NPB>(n, k);
            double step = kb.x[i];
            if (pd.on) step += pd.t * mr_direction(pd, i);
            double d = dv[i] + step;
            dv[i] = d;
            vs[k] = act ? vn[i] + d : 0.0;
            vstar[i] = vs[k];
        }
        if (vstar_f) vstar_f[n] = make_float4((float)vs[0], (float)vs[1], (float)vs[2], 0.f);
    }
}

// The FP32 node-major copy of vstar ([B][NPB][4]) that the MIXED particle
// kernels gather from, for the substeps whose grid update writes only vstar.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_vstar_f32(NodeGeom ng, const double* __restrict__ vstar, float4* __restrict__ vstar_f)
{
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS)
        vstar_f[n] = make_float4((float)vstar[vidx<NPB>(n, 0)], (float)vstar[vidx<NPB>(n, 1)], (float)vstar[vidx<NPB>(n, 2)], 0.f);
}

// Ends a Newton iteration (NewtonsMethod.h:46 loop); as a graph, sets the
// Newton loop condition.
__global__ void k_newton_advance(SolverScalars* __restrict__ sc, int nmax, cudaGraphConditionalHandle hN, int use_graph, GridSync* __restrict__ gs)
{
    if (gs) *gs = GridSync{}; // the next persistent solve starts from a clean barrier
    if (!sc->newton_done) sc->newton_iters += 1;
    const int n = sc->nit + 1;
    sc->nit = n;
    if (use_graph) cudaGraphSetConditional(hN, (!sc->newton_done && n < nmax) ? 1u : 0u);
}

// ------------------------------------------------------------------ ADMM --
// updateCollisionNodes (AdmmSimulationFoam.h:276-293) on vi = dv + vn with the
// fake-separate rule, vstar = vn + dv and the right-hand side's dt m g (dvStep,
// :167-170).  With wsum (initStep, :304-320) dv is first replaced by
// dv dt / sum_p w_ip.
template <class L>
__global__ void __launch_bounds__(ND_THREADS) k_admm_collide(NodeGeom ng, const double* __restrict__ gm, const int4* __restrict__ block_page,
    double dx, double gx, double gy, double gz, double dt, const DevCollider* __restrict__ cols, int ncols, const double* __restrict__ vn,
    double* __restrict__ dv, double* __restrict__ vstar, int8_t* __restrict__ col, double* __restrict__ P6, double* __restrict__ rhs,
    const double* __restrict__ wsum)
{
    constexpr int NPB = L::NPB;
    const double g[3] = { gx, gy, gz };
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const int64_t b = n / NPB;
        const int e = (int)(n - b * NPB);
        const double m = gm[n];
        double v[3], d[3];
        for (int k = 0; k < 3; ++k) {
            v[k] = vn[vidx<NPB>(n, k)];
            d[k] = dv[vidx<NPB>(n, k)];
        }
        int8_t c = 0;
        double P[6] = { 1, 0, 0, 1, 0, 1 };
        if (m != 0) {
            if (wsum)
                for (int k = 0; k < 3; ++k) d[k] = d[k] * dt / wsum[n];
            const int4 bp = block_page[b];
            const int lx = e >> (L::YB + L::ZB), ly = (e >> L::ZB) & (L::BY - 1), lz = e & (L::BZ - 1);
            const double xi[3] = { (bp.x * L::BX + lx) * dx, (bp.y * L::BY + ly) * dx, (bp.z * L::BZ + lz) * dx };
            double vi[3] = { d[0] + v[0], d[1] + v[1], d[2] + v[2] };
            if (multi_collide(cols, ncols, xi, vi, P, true)) {
                c = 1;
                for (int k = 0; k < 3; ++k) d[k] = vi[k] - v[k];
            }
        }
        else
            d[0] = d[1] = d[2] = 0;
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            dv[i] = d[k];
            vstar[i] = (m != 0) ? v[k] + d[k] : 0.0;
            rhs[i] = (m != 0) ? dt * m * g[k] : 0.0;
        }
        col[n] = c;
        for (int k = 0; k < 6; ++k) P6[k * ng.nn + n] = P[k];
    }
}

// Start of dvStep's MINRES from the current dv (Minres.h:73-98): r =
// project(rhs - (m dv + hacc)), zeroes hacc; Q0 = r, Z0 = r / pre, the other
// Lanczos vectors and search directions 0, the correction x = 0; partial z.r.
// The relative tolerance is min(0.5, sqrt(max(residual, 1e-6))) with the
// reference's constant residual 1 (AdmmSimulationFoam.h:779-782): 0.5.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_admm_start(NodeGeom ng, const double* __restrict__ gm, const int8_t* __restrict__ col,
    const double* __restrict__ P6, const double* __restrict__ rhs, const double* __restrict__ dv, KrylovBufs kb, double* __restrict__ part,
    SolverScalars* __restrict__ sc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->rel_tol = 0.5;
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        double r[3];
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            r[k] = (m != 0) ? rhs[i] - (m * dv[i] + kb.hacc[i]) : 0.0;
            kb.hacc[i] = 0;
        }
        if (m != 0) project3(col, P6, ng.nn, n, r);
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            const double z = (m != 0) ? r[k] / kb.pre[n] : 0.0;
            kb.x[i] = 0;
            kb.Q[0][i] = r[k];
            kb.Q[1][i] = 0;
            kb.Q[2][i] = 0;
            kb.M[0][i] = 0;
            kb.M[1][i] = 0;
            kb.M[2][i] = 0;
            kb.Z[0][i] = z;
            kb.Z[1][i] = 0;
            acc += z * r[k];
        }
    }
    double t = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// dv += x (the MINRES correction, with its deferred last update); vstar =
// vn + dv on active nodes.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_admm_dv_update(NodeGeom ng, const double* __restrict__ gm, KrylovBufs kb,
    const double* __restrict__ vn, double* __restrict__ dv, double* __restrict__ vstar, const SolverScalars* __restrict__ sc)
{
    const MrPending pd = mr_pending(kb, sc->pend, sc->kit);
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const bool act = gm[n] != 0;
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            double x = kb.x[i];
            if (pd.on) x += pd.t * mr_direction(pd, i);
            const double d = dv[i] + x;
            dv[i] = d;
            vstar[i] = act ? vn[i] + d : 0.0;
        }
    }
}

// Ends an ADMM iteration (admmStep loop, AdmmSimulationFoam.h:776-784).
__global__ void k_admm_advance(SolverScalars* __restrict__ sc, int nmax, cudaGraphConditionalHandle hN, int use_graph, GridSync* __restrict__ gs)
{
    *gs = GridSync{}; // the next persistent solve starts from a clean barrier
    sc->newton_iters += 1;
    const int n = sc->nit + 1;
    sc->nit = n;
    if (n >= nmax) sc->converged = 1;
    if (use_graph) cudaGraphSetConditional(hN, n < nmax ? 1u : 0u);
}

// ---------------------------------------------------------------- adjoint --
// Start of the adjoint CG solve (ConjugateGradient.h:99-117 with x = 0):
// r = project(g), q = r / m, p = q, partial r.q; relative tolerance `tol`.
template <int NPB>
__global__ void __launch_bounds__(ND_THREADS) k_adj_cg_init(NodeGeom ng, const double* __restrict__ gm, const int8_t* __restrict__ col,
    const double* __restrict__ P6, const double* __restrict__ g, KrylovBufs kb, double tol, double* __restrict__ part,
    SolverScalars* __restrict__ sc)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->rel_tol = tol;
    double acc = 0;
    for (int64_t n = (int64_t)blockIdx.x * ND_THREADS + threadIdx.x; n < ng.nn; n += (int64_t)gridDim.x * ND_THREADS) {
        const double m = gm[n];
        double r[3];
        for (int k = 0; k < 3; ++k) r[k] = (m != 0) ? g[vidx<NPB>(n, k)] : 0.0;
        if (m != 0) project3(col, P6, ng.nn, n, r);
        for (int k = 0; k < 3; ++k) {
            const int64_t i = vidx<NPB>(n, k);
            const double q = (m != 0) ? r[k] / kb.pre[n] : 0.0;
            kb.x[i] = 0;
            kb.r[i] = r[k];
            kb.q[i] = q;
            kb.p[i] = q;
            if (kb.pf) kb.pf[4 * n + k] = (float)q;
            kb.hacc[i] = 0;
            acc += r[k] * q;
        }
    }
    double t = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
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
    ZMPM_CUDA(ctx->kvf.ensure((size_t)(8 * nn) * sizeof(float)));
    ZMPM_CUDA(ctx->vstarf.ensure((size_t)(4 * nn) * sizeof(float)));
    return ZMPM_OK;
}

int run_p2g(Ctx* ctx, bool damage)
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
    if (damage) {
        rc = launch_damage(ctx); // the fracture hook runs after particlesToGrid
        if (rc) return rc;
        if (ctx->has_pf) {
            rc = run_phase_field(ctx, &ctx->pf_iters, &ctx->pf_res);
            if (rc) return rc;
        }
    }
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
                reinterpret_cast<unsigned long long*>(&dc->N), &dc->flags, ctx->mixed ? ctx->vstarf.as<float4>() : nullptr);
        else
            k_grid_init<Layout444><<<ng.parts, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->block_page.as<int4>(),
                ctx->cfg.dx, g[0], g[1], g[2], ctx->dt, ctx->dcolliders.as<DevCollider>(), (int)ctx->colliders.size(), ctx->vn.as<double>(),
                ctx->dv.as<double>(), ctx->vstar.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
                reinterpret_cast<unsigned long long*>(&dc->N), &dc->flags, ctx->mixed ? ctx->vstarf.as<float4>() : nullptr);
        ++g_kernel_launches;
    }
    ctx->vstarf_valid = ctx->mixed; // k_grid_init wrote the FP32 copy
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

// The symplectic substep after binning, up to G2P (MpmSimulationBase.cpp:
// 264-281): particle stress, P2G of mass, momentum and force, the fracture
// hook, the explicit grid update with collisions and trial collision.
int run_explicit(Ctx* ctx, const zmpm_solver& s)
{
    ctx->vstarf_valid = false; // k_grid_explicit writes vstar only
    cudaStream_t st = ctx->stream;
    const int64_t nn = ctx->B * ctx->npb();
    int rc = ensure_node_buffers(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaMemsetAsync(ctx->scal.p, 0, sizeof(SolverScalars), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->gm.p, 0, nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->gmv.p, 0, 3 * nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->facc.p, 0, 3 * nn * sizeof(double), st));
    rc = launch_explicit_stress(ctx);
    if (rc) return rc;
    rc = launch_p2g(ctx);
    if (rc) return rc;
    rc = launch_force_scatter(ctx, ctx->facc.as<double>(), s.mls_mpm != 0);
    if (rc) return rc;
    rc = launch_damage(ctx);
    if (rc) return rc;
    if (ctx->has_pf) {
        rc = run_phase_field(ctx, &ctx->pf_iters, &ctx->pf_res);
        if (rc) return rc;
    }
    rc = upload_colliders(ctx, ctx->time, 0);
    if (rc) return rc;
    rc = upload_colliders(ctx, ctx->time + ctx->dt, 1);
    if (rc) return rc;
    if (nn > 0) {
        NodeGeom ng = node_geom(ctx);
        DevCounters* dc = ctx->counters.as<DevCounters>();
        const double* g = ctx->cfg.gravity;
        const DevCollider* c0 = ctx->dcolliders.as<DevCollider>();
        const DevCollider* c1 = c0 + MAX_COLLIDERS;
        const int nc = (int)ctx->colliders.size(), trial = s.trial_collision ? 1 : 0;
        if (ctx->layout == 1)
            k_grid_explicit<Layout244><<<ng.parts, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->facc.as<double>(),
                ctx->block_page.as<int4>(), ctx->cfg.dx, g[0], g[1], g[2], ctx->dt, c0, c1, nc, trial, ctx->vn.as<double>(), ctx->dv.as<double>(),
                ctx->vstar.as<double>(), ctx->collided.as<int8_t>(), reinterpret_cast<unsigned long long*>(&dc->N));
        else
            k_grid_explicit<Layout444><<<ng.parts, ND_THREADS, 0, st>>>(ng, ctx->gm.as<double>(), ctx->gmv.as<double>(), ctx->facc.as<double>(),
                ctx->block_page.as<int4>(), ctx->cfg.dx, g[0], g[1], g[2], ctx->dt, c0, c1, nc, trial, ctx->vn.as<double>(), ctx->dv.as<double>(),
                ctx->vstar.as<double>(), ctx->collided.as<int8_t>(), reinterpret_cast<unsigned long long*>(&dc->N));
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
            ctx->kv[9].as<double>(), q);
    else
        k_apply_A<64><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(), dt2, x,
            ctx->kv[9].as<double>(), q);
    ++g_kernel_launches;
    return ZMPM_OK;
}

namespace {

struct NewtonLaunch {
    Ctx* ctx;
    NodeGeom ng;
    KrylovBufs kb;
    NewtonParams np;
    SolverScalars* sc;
    double *pA, *pB, *pC;
    double dt2;
    int nb;
};

// First part of a Newton iteration: update, residual with the Krylov start
// vectors, check and Krylov start.
template <int NPB>
int launch_newton_head(const NewtonLaunch& L, cudaStream_t st)
{
    Ctx* ctx = L.ctx;
    int rc = launch_update(ctx);
    if (rc) return rc;
    const double* g = ctx->cfg.gravity;
    k_residual_start<NPB><<<L.nb, ND_THREADS, 0, st>>>(L.ng, ctx->gm.as<double>(), ctx->facc.as<double>(), ctx->dv.as<double>(),
        ctx->collided.as<int8_t>(), ctx->proj.as<double>(), g[0], g[1], g[2], ctx->dt, L.kb, L.np.minres, L.pA, L.pB, L.sc);
    k_newton_start<NPB><<<1, ND_THREADS, 0, st>>>(L.ng, L.np, L.pA, L.pB, L.sc);
    g_kernel_launches += 2;
    return ZMPM_OK;
}

template <int NPB>
int launch_newton_tail(const NewtonLaunch& L, cudaStream_t st, cudaGraphConditionalHandle hN, int use_graph)
{
    Ctx* ctx = L.ctx;
    k_newton_step<NPB><<<L.nb, ND_THREADS, 0, st>>>(L.ng, ctx->gm.as<double>(), L.kb, L.np.minres, ctx->vn.as<double>(), ctx->dv.as<double>(),
        ctx->vstar.as<double>(), L.sc, ctx->mixed ? ctx->vstarf.as<float4>() : nullptr);
    k_newton_advance<<<1, 1, 0, st>>>(L.sc, L.np.nmax, hN, use_graph, L.ctx->gsync.as<GridSync>());
    g_kernel_launches += 2;
    return ZMPM_OK;
}

// A persistent Krylov kernel as one cooperative launch of as many CTAs as fit
// on the device at once (all co-resident, which the grid barrier needs; the
// launch fails rather than oversubscribes), the grid size found once per
// kernel.  GridSync must be zero.
template <class... P, class... A>
int launch_coop(Ctx* ctx, cudaStream_t st, void (*kern)(P...), A&&... args)
{
    int& blocks = ctx->coop_blocks[reinterpret_cast<const void*>(kern)];
    if (blocks <= 0) {
        int per_sm = 0, sms = 0;
        ZMPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FUSED_THREADS, 0));
        ZMPM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        blocks = std::min(per_sm * sms, RED_MAX_CTAS);
        if (blocks <= 0) {
            ctx->err = "the persistent Krylov kernel does not fit on this device";
            return ZMPM_CUDA_ERROR;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(FUSED_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ZMPM_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...));
    ++g_kernel_launches;
    return ZMPM_OK;
}

static HvpArgs hvp_args(const Ctx* ctx)
{
    HvpArgs ha;
    ha.group_start = ctx->group_start.as<int32_t>();
    ha.group_nbr = ctx->group_nbr.as<int32_t>();
    ha.pi = ctx->pi.as<int32_t>();
    ha.base = ctx->base.as<short4>();
    ha.frac = ctx->frac.p;
    ha.scr = ctx->scratch.p;
    ha.cap = ctx->Pcap;
    ha.dx = ctx->cfg.dx;
    ha.G = (int)ctx->G;
    return ha;
}

// The persistent CG solve (k_cg_persistent) on the Newton operator.
template <int NPB>
int launch_cg_persistent(const NewtonLaunch& L, cudaStream_t st)
{
    Ctx* ctx = L.ctx;
    using Lay = typename std::conditional<NPB == 32, Layout244, Layout444>::type;
    const HvpArgs ha = hvp_args(ctx);
    int32_t* flags = &ctx->counters.as<DevCounters>()->flags;
    const double* gm = ctx->gm.as<double>();
    const int8_t* col = ctx->collided.as<int8_t>();
    const double* P6 = ctx->proj.as<double>();
    GridSync* gs = ctx->gsync.as<GridSync>();
    if (ctx->mixed) {
        if (!L.kb.pf) {
            ctx->err = "MIXED CG needs the FP32 copy of p";
            return ZMPM_BAD_ARG;
        }
        return launch_coop(ctx, st, k_cg_persistent<Lay, float, float>, L.ng, ha, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs,
            ctx->spin_limit, flags);
    }
    return launch_coop(ctx, st, k_cg_persistent<Lay, double, double>, L.ng, ha, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs,
        ctx->spin_limit, flags);
}

// The persistent MINRES solve (k_mr_persistent) on the Newton operator
// (MIXED: FP32 products on the FP32 copies of Z) or, admm = true, on ADMM's
// global operator.
template <int NPB>
int launch_mr_persistent(const NewtonLaunch& L, cudaStream_t st, bool admm)
{
    Ctx* ctx = L.ctx;
    using Lay = typename std::conditional<NPB == 32, Layout244, Layout444>::type;
    const HvpArgs ha = hvp_args(ctx);
    int32_t* flags = &ctx->counters.as<DevCounters>()->flags;
    const double* gm = ctx->gm.as<double>();
    const int8_t* col = ctx->collided.as<int8_t>();
    const double* P6 = ctx->proj.as<double>();
    GridSync* gs = ctx->gsync.as<GridSync>();
    const long long lim = ctx->spin_limit;
    if (admm) {
        if (ctx->mixed)
            return launch_coop(ctx, st, k_mr_persistent<Lay, float, double, AdmmOpModel<float>>, L.ng, ha,
                AdmmOpModel<float>{ ctx->adm_B.as<float>(), ctx->Pcap }, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs, lim, flags);
        return launch_coop(ctx, st, k_mr_persistent<Lay, double, double, AdmmOpModel<double>>, L.ng, ha,
            AdmmOpModel<double>{ ctx->adm_B.as<double>(), ctx->Pcap }, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs, lim, flags);
    }
    if (ctx->mixed) {
        if (!L.kb.Zf[0]) {
            ctx->err = "MIXED MINRES needs the FP32 copies of Z";
            return ZMPM_BAD_ARG;
        }
        return launch_coop(ctx, st, k_mr_persistent<Lay, float, float, HvpModel<float>>, L.ng, ha,
            HvpModel<float>{ ha.pi, ctx->scratch.as<float>(), ctx->Pcap }, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs, lim,
            flags);
    }
    return launch_coop(ctx, st, k_mr_persistent<Lay, double, double, HvpModel<double>>, L.ng, ha,
        HvpModel<double>{ ha.pi, ctx->scratch.as<double>(), ctx->Pcap }, gm, col, P6, L.dt2, L.kb, L.pA, L.pC, L.sc, L.np.kmax, gs, lim, flags);
}

#define ZMPM_CAP(expr)                                                                                                 \
    do {                                                                                                               \
        cudaError_t _e = (expr);                                                                                       \
        if (_e != cudaSuccess) {                                                                                       \
            ctx->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                                             \
            cudaStreamCaptureStatus _cs;                                                                               \
            if (cudaStreamIsCapturing(st, &_cs) == cudaSuccess && _cs != cudaStreamCaptureStatusNone) {               \
                cudaGraph_t _g;                                                                                        \
                cudaStreamEndCapture(st, &_g);                                                                         \
            }                                                                                                          \
            if (g) cudaGraphDestroy(g);                                                                                \
            return ZMPM_CUDA_ERROR;                                                                                    \
        }                                                                                                              \
    } while (0)

// A solver loop as one CUDA graph: WHILE(outer){ body(st, hN) }, its
// condition set on the device.
template <class Body>
int while_graph(Ctx* ctx, Body&& body, cudaGraphExec_t* exec_out)
{
    cudaStream_t st = ctx->stream;
    cudaGraph_t g = nullptr;
    ZMPM_CAP(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hN;
    ZMPM_CAP(cudaGraphConditionalHandleCreate(&hN, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams pN = {};
    pN.type = cudaGraphNodeTypeConditional;
    pN.conditional.handle = hN;
    pN.conditional.type = cudaGraphCondTypeWhile;
    pN.conditional.size = 1;
    cudaGraphNode_t nN;
    ZMPM_CAP(cudaGraphAddNode(&nN, g, nullptr, 0, &pN));
    ZMPM_CAP(cudaStreamBeginCaptureToGraph(st, pN.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = body(st, hN);
    cudaGraph_t tmp = nullptr;
    ZMPM_CAP(cudaStreamEndCapture(st, &tmp));
    if (rc) {
        cudaGraphDestroy(g);
        return rc;
    }
    ZMPM_CAP(cudaGraphInstantiate(exec_out, g, 0));
    cudaGraphDestroy(g);
    return ZMPM_OK;
}

// One Newton iteration with its linear solve as one persistent kernel
// (k_mr_persistent or k_cg_persistent): update, residual and Krylov start,
// Newton check, the solve, step and advance.
template <int NPB>
int launch_newton_iteration(const NewtonLaunch& L, cudaStream_t st, cudaGraphConditionalHandle hN, int use_graph)
{
    int rc = launch_newton_head<NPB>(L, st);
    if (rc) return rc;
    rc = L.np.minres ? launch_mr_persistent<NPB>(L, st, false) : launch_cg_persistent<NPB>(L, st);
    if (rc) return rc;
    return launch_newton_tail<NPB>(L, st, hN, use_graph);
}

// The Newton solve as one graph: WHILE(Newton){ iteration }.
template <int NPB>
int newton_graph(const NewtonLaunch& L, cudaGraphExec_t* exec_out)
{
    return while_graph(L.ctx, [&](cudaStream_t st, cudaGraphConditionalHandle hN) { return launch_newton_iteration<NPB>(L, st, hN, 1); },
        exec_out);
}

} // namespace

template <int NPB>
static int newton_impl(Ctx* ctx, const zmpm_solver& s)
{
    cudaStream_t st = ctx->stream;
    NewtonLaunch L;
    L.ctx = ctx;
    L.ng = node_geom(ctx);
    L.sc = ctx->scal.as<SolverScalars>();
    double* part = ctx->red.as<double>();
    L.pA = part + RED_A * RED_MAX_CTAS;
    L.pB = part + RED_B * RED_MAX_CTAS;
    L.pC = part + RED_C * RED_MAX_CTAS;
    L.kb.x = ctx->kv[0].as<double>();
    L.kb.r = ctx->kv[1].as<double>();
    L.kb.p = ctx->kv[2].as<double>();
    L.kb.q = ctx->kv[3].as<double>();
    L.kb.tmp = ctx->kv[4].as<double>();
    L.kb.Q[0] = ctx->kv[1].as<double>();
    L.kb.Q[1] = ctx->kv[2].as<double>();
    L.kb.Q[2] = ctx->kv[3].as<double>();
    L.kb.M[0] = ctx->kv[4].as<double>();
    L.kb.M[1] = ctx->kv[5].as<double>();
    L.kb.M[2] = ctx->kv[6].as<double>();
    L.kb.Z[0] = ctx->kv[7].as<double>();
    L.kb.Z[1] = ctx->kv[8].as<double>();
    L.kb.hacc = ctx->kv[9].as<double>();
    L.kb.pre = ctx->gm.as<double>();
    L.np.minres = s.linear_solver == ZMPM_MINRES ? 1 : 0;
    L.np.escalate = ctx->mixed ? 1 : 0;
    // MIXED MINRES runs its split FP32 product on FP32 copies of Z
    const bool zf = ctx->mixed && L.np.minres;
    L.kb.Zf[0] = zf ? ctx->kvf.as<float>() : nullptr;
    L.kb.Zf[1] = zf ? ctx->kvf.as<float>() + 4 * L.ng.nn : nullptr;
    // MIXED CG runs its FP32 product on an FP32 copy of p
    L.kb.pf = (ctx->mixed && !L.np.minres) ? ctx->kvf.as<float>() : nullptr;
    L.np.kmax = s.krylov_max_iterations;
    L.np.nmax = s.newton_max_iterations;
    L.np.tol = s.newton_tolerance;
    L.np.abs_tol = s.krylov_tolerance;
    L.np.tol_scale = s.linear_solve_tolerance_scale;
    L.np.dt = ctx->dt;
    L.dt2 = ctx->dt * ctx->dt;
    L.nb = L.ng.parts;
    ZMPM_CUDA(cudaMemsetAsync(L.sc, 0, sizeof(SolverScalars), st));
    // MIXED: start with the FP64 residual when the last solves needed it (any
    // nonzero byte sets the flag)
    if (ctx->mixed && ctx->fp64_res_run > 0 && ctx->fp64_res_run % 16 != 0)
        ZMPM_CUDA(cudaMemsetAsync(&L.sc->fp64_res, 1, 1, st));
    ctx->prof_newton = 0;
    ctx->graph_used = false;
    if (L.ng.nn == 0 || s.newton_max_iterations == 0) return ZMPM_OK;
    ZMPM_CUDA(cudaMemsetAsync(ctx->gsync.p, 0, sizeof(GridSync), st));
    const bool prof = ctx->profiling && s.newton_max_iterations <= 64;
    if (!prof) {
        // whole solve as one graph with device-side loop conditions
        cudaGraphExec_t exec = nullptr;
        const int64_t launches0 = g_kernel_launches;
        int rc = newton_graph<NPB>(L, &exec);
        if (rc) return rc;
        cudaError_t e = cudaGraphLaunch(exec, st);
        // kernels inside the graph are counted per executed loop body after the
        // substep (see zmpm_substep), not once at capture
        g_kernel_launches = launches0;
        ctx->graph_used = true;
        if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = exec; // released when the next solve launches its graph, or by zmpm_destroy
        ZMPM_CUDA(e);
        return ZMPM_OK;
    }
    // profiling: a host-driven Newton loop (every kernel a plain launch), each
    // linear solve's persistent kernel bracketed by events
    ctx->prof_newton = s.newton_max_iterations;
    while (ctx->hvp_ev.size() < 2 * (size_t)s.newton_max_iterations) {
        cudaEvent_t e;
        ZMPM_CUDA(cudaEventCreate(&e));
        ctx->hvp_ev.push_back(e);
    }
    for (int it = 0; it < s.newton_max_iterations; ++it) {
        int rc = launch_newton_head<NPB>(L, st);
        if (rc) return rc;
        ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * it], st));
        rc = L.np.minres ? launch_mr_persistent<NPB>(L, st, false) : launch_cg_persistent<NPB>(L, st);
        if (rc) return rc;
        ZMPM_CUDA(cudaEventRecord(ctx->hvp_ev[2 * it + 1], st));
        rc = launch_newton_tail<NPB>(L, st, 0, 0);
        if (rc) return rc;
        ZMPM_CUDA(cudaGetLastError());
    }
    return ZMPM_OK;
}

int run_newton(Ctx* ctx, const zmpm_solver& s)
{
    return ctx->layout == 1 ? newton_impl<32>(ctx, s) : newton_impl<64>(ctx, s);
}

// AdmmSimulation::admmStep (AdmmSimulationFoam.h:766-801) after P2G: initStep,
// the global operator's preconditioner, then per iteration the collision
// update, F step (+ dvStep right-hand side), dvStep's MINRES and the dual
// update; finally last_dv.  The iteration loop runs as one conditional graph
// like the Newton solve (host-driven when profiling or without graphs).
template <class L>
static int admm_impl(Ctx* ctx, const zmpm_solver& s)
{
    constexpr int NPB = L::NPB;
    cudaStream_t st = ctx->stream;
    const int64_t nn = ctx->B * NPB, cap = ctx->Pcap;
    const size_t TH = ctx->mixed ? sizeof(float) : sizeof(double);
    ZMPM_CUDA(ctx->adm_F.ensure(18 * cap * sizeof(double)));
    ZMPM_CUDA(ctx->adm_gvn.ensure(9 * cap * sizeof(double)));
    ZMPM_CUDA(ctx->adm_B.ensure(6 * cap * TH));
    ZMPM_CUDA(ctx->adm_pre.ensure(std::max<int64_t>(nn, 1) * sizeof(double)));
    ZMPM_CUDA(ctx->adm_rhs.ensure(std::max<int64_t>(3 * nn, 1) * sizeof(double)));
    ZMPM_CUDA(ctx->adm_w.ensure(std::max<int64_t>(nn, 1) * sizeof(double)));
    NewtonLaunch Lc;
    Lc.ctx = ctx;
    Lc.ng = node_geom(ctx);
    Lc.sc = ctx->scal.as<SolverScalars>();
    double* part = ctx->red.as<double>();
    Lc.pA = part + RED_A * RED_MAX_CTAS;
    Lc.pB = part + RED_B * RED_MAX_CTAS;
    Lc.pC = part + RED_C * RED_MAX_CTAS;
    KrylovBufs& kb = Lc.kb;
    kb.x = ctx->kv[0].as<double>();
    kb.r = kb.p = kb.q = kb.tmp = nullptr;
    kb.Q[0] = ctx->kv[1].as<double>();
    kb.Q[1] = ctx->kv[2].as<double>();
    kb.Q[2] = ctx->kv[3].as<double>();
    kb.M[0] = ctx->kv[4].as<double>();
    kb.M[1] = ctx->kv[5].as<double>();
    kb.M[2] = ctx->kv[6].as<double>();
    kb.Z[0] = ctx->kv[7].as<double>();
    kb.Z[1] = ctx->kv[8].as<double>();
    kb.Zf[0] = kb.Zf[1] = nullptr;
    kb.pf = nullptr;
    kb.hacc = ctx->kv[9].as<double>();
    kb.pre = ctx->adm_pre.as<double>();
    Lc.np.minres = 1;
    Lc.np.escalate = 0;
    Lc.np.kmax = s.admm_global_max_iterations;
    Lc.np.nmax = s.admm_iterations;
    Lc.np.tol = 0;
    Lc.np.abs_tol = s.admm_global_tolerance;
    Lc.np.tol_scale = 1;
    Lc.np.dt = ctx->dt;
    Lc.dt2 = 1.0;
    Lc.nb = Lc.ng.parts;
    const double rho = s.admm_rho_scale, local_tol = s.admm_local_tolerance;
    ZMPM_CUDA(cudaMemsetAsync(Lc.sc, 0, sizeof(SolverScalars), st));
    ctx->prof_newton = 0;
    ctx->graph_used = false;
    ctx->admm_iters = 0;
    if (nn == 0) return ZMPM_OK;
    const double* g = ctx->cfg.gravity;
    const int ncols = (int)ctx->colliders.size();
    const DevCollider* cols = ctx->dcolliders.as<DevCollider>();
    auto collide = [&](cudaStream_t sm, const double* wsum) {
        k_admm_collide<L><<<Lc.nb, ND_THREADS, 0, sm>>>(Lc.ng, ctx->gm.as<double>(), ctx->block_page.as<int4>(), ctx->cfg.dx, g[0], g[1], g[2],
            ctx->dt, cols, ncols, ctx->vn.as<double>(), ctx->dv.as<double>(), ctx->vstar.as<double>(), ctx->collided.as<int8_t>(),
            ctx->proj.as<double>(), ctx->adm_rhs.as<double>(), wsum);
        ++g_kernel_launches;
    };

    // initStep + initMultiplierAndPreconditioner
    ZMPM_CUDA(cudaMemsetAsync(ctx->dv.p, 0, 3 * nn * sizeof(double), st));
    ZMPM_CUDA(cudaMemsetAsync(ctx->adm_w.p, 0, nn * sizeof(double), st));
    int rc = launch_admm_dvinit(ctx);
    if (rc) return rc;
    collide(st, ctx->adm_w.as<double>());
    rc = launch_admm_init(ctx, rho);
    if (rc) return rc;
    ZMPM_CUDA(cudaMemcpyAsync(ctx->adm_pre.p, ctx->gm.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
    rc = launch_admm_pre(ctx);
    if (rc) return rc;

    // one ADMM iteration: collision update, local step and the right-hand
    // side, the MINRES solve as one persistent kernel, dv / vstar and the dual
    // update
    auto iteration = [&](cudaStream_t sm, cudaGraphConditionalHandle hN, int ug) {
        collide(sm, nullptr);
        int r = launch_admm_local(ctx, rho, local_tol);
        if (r) return r;
        r = launch_force_scatter(ctx, ctx->adm_rhs.as<double>());
        if (r) return r;
        r = launch_admm_op(ctx, ctx->dv.as<double>(), kb.hacc);
        if (r) return r;
        k_admm_start<NPB><<<Lc.nb, ND_THREADS, 0, sm>>>(Lc.ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
            ctx->adm_rhs.as<double>(), ctx->dv.as<double>(), kb, Lc.pB, Lc.sc);
        k_krylov_start<NPB><<<1, ND_THREADS, 0, sm>>>(Lc.ng, kb, Lc.np, Lc.pB, Lc.sc);
        g_kernel_launches += 2;
        r = launch_mr_persistent<NPB>(Lc, sm, true);
        if (r) return r;
        k_admm_dv_update<NPB><<<Lc.nb, ND_THREADS, 0, sm>>>(Lc.ng, ctx->gm.as<double>(), kb, ctx->vn.as<double>(), ctx->dv.as<double>(),
            ctx->vstar.as<double>(), Lc.sc);
        ++g_kernel_launches;
        r = launch_admm_dual(ctx, rho);
        if (r) return r;
        k_admm_advance<<<1, 1, 0, sm>>>(Lc.sc, Lc.np.nmax, hN, ug, ctx->gsync.as<GridSync>());
        ++g_kernel_launches;
        return (int)ZMPM_OK;
    };

    if (s.admm_iterations > 0) {
        ZMPM_CUDA(cudaMemsetAsync(ctx->gsync.p, 0, sizeof(GridSync), st));
        if (!ctx->profiling) {
            cudaGraphExec_t exec = nullptr;
            const int64_t launches0 = g_kernel_launches;
            rc = while_graph(ctx, [&](cudaStream_t sm, cudaGraphConditionalHandle hN) { return iteration(sm, hN, 1); }, &exec);
            if (rc) return rc;
            cudaError_t e = cudaGraphLaunch(exec, st);
            g_kernel_launches = launches0; // counted per executed iteration after the substep
            ctx->graph_used = true;
            if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = exec;
            ZMPM_CUDA(e);
        }
        else {
            for (int it = 0; it < s.admm_iterations; ++it) {
                rc = iteration(st, 0, 0);
                if (rc) return rc;
                ZMPM_CUDA(cudaGetLastError());
            }
        }
    }
    ctx->admm_iters = s.admm_iterations;
    rc = launch_admm_lastdv(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

// (M + dt^2 K) lambda = P g with CG on the Newton operator (the Hessian
// scratch must hold the converged state); g is ctx->res on entry, lambda is
// kv[0] on exit.  Returns the CG iteration count through stats.
int run_adjoint_solve(Ctx* ctx, double tol, int max_iterations)
{
    NewtonLaunch Lc;
    Lc.ctx = ctx;
    Lc.ng = node_geom(ctx);
    Lc.sc = ctx->scal.as<SolverScalars>();
    double* part = ctx->red.as<double>();
    Lc.pA = part + RED_A * RED_MAX_CTAS;
    Lc.pB = part + RED_B * RED_MAX_CTAS;
    Lc.pC = part + RED_C * RED_MAX_CTAS;
    KrylovBufs& kb = Lc.kb;
    kb.x = ctx->kv[0].as<double>();
    kb.r = ctx->kv[1].as<double>();
    kb.p = ctx->kv[2].as<double>();
    kb.q = ctx->kv[3].as<double>();
    kb.tmp = ctx->kv[4].as<double>();
    for (int k = 0; k < 3; ++k) kb.Q[k] = kb.M[k] = nullptr;
    kb.Z[0] = kb.Z[1] = nullptr;
    kb.Zf[0] = kb.Zf[1] = nullptr;
    kb.pf = ctx->mixed ? ctx->kvf.as<float>() : nullptr; // the FP32 product of a MIXED context runs on an FP32 copy of p
    kb.hacc = ctx->kv[9].as<double>();
    kb.pre = ctx->gm.as<double>();
    Lc.np.minres = 0;
    Lc.np.escalate = 0;
    Lc.np.kmax = max_iterations;
    Lc.np.nmax = 1;
    Lc.np.tol = 0;
    Lc.np.abs_tol = 1e300;
    Lc.np.tol_scale = 1;
    Lc.np.dt = ctx->dt;
    Lc.dt2 = ctx->dt * ctx->dt;
    Lc.nb = Lc.ng.parts;
    cudaStream_t st = ctx->stream;
    ZMPM_CUDA(cudaMemsetAsync(Lc.sc, 0, sizeof(SolverScalars), st));
    if (Lc.ng.nn == 0) return ZMPM_OK;
    if (ctx->layout == 1) {
        k_adj_cg_init<32><<<Lc.nb, ND_THREADS, 0, st>>>(Lc.ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
            ctx->res.as<double>(), kb, tol, Lc.pB, Lc.sc);
        k_krylov_start<32><<<1, ND_THREADS, 0, st>>>(Lc.ng, kb, Lc.np, Lc.pB, Lc.sc);
    }
    else {
        k_adj_cg_init<64><<<Lc.nb, ND_THREADS, 0, st>>>(Lc.ng, ctx->gm.as<double>(), ctx->collided.as<int8_t>(), ctx->proj.as<double>(),
            ctx->res.as<double>(), kb, tol, Lc.pB, Lc.sc);
        k_krylov_start<64><<<1, ND_THREADS, 0, st>>>(Lc.ng, kb, Lc.np, Lc.pB, Lc.sc);
    }
    g_kernel_launches += 2;
    ZMPM_CUDA(cudaMemsetAsync(ctx->gsync.p, 0, sizeof(GridSync), st));
    int rc = ctx->layout == 1 ? launch_cg_persistent<32>(Lc, st) : launch_cg_persistent<64>(Lc, st);
    if (rc) return rc;
    ZMPM_CUDA(cudaStreamSynchronize(st));
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

int run_admm(Ctx* ctx, const zmpm_solver& s)
{
    ctx->vstarf_valid = false; // the ADMM kernels write vstar only
    return ctx->layout == 1 ? admm_impl<Layout244>(ctx, s) : admm_impl<Layout444>(ctx, s);
}

// MIXED: vstar_f from vstar (the ADMM and explicit grid updates write vstar only).
int refresh_vstar_f32(Ctx* ctx)
{
    NodeGeom ng = node_geom(ctx);
    if (ng.nn == 0) return ZMPM_OK;
    if (ctx->layout == 1)
        k_vstar_f32<32><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->vstar.as<double>(), ctx->vstarf.as<float4>());
    else
        k_vstar_f32<64><<<ng.parts, ND_THREADS, 0, ctx->stream>>>(ng, ctx->vstar.as<double>(), ctx->vstarf.as<float4>());
    ++g_kernel_launches;
    return ZMPM_OK;
}

int run_g2p(Ctx* ctx, bool plastic)
{
    if (ctx->mixed && !ctx->vstarf_valid) {
        int rc = refresh_vstar_f32(ctx);
        if (rc) return rc;
    }
    int rc = launch_g2p(ctx, plastic);
    if (rc) return rc;
    ZMPM_CUDA(cudaGetLastError());
    return ZMPM_OK;
}

} // namespace zmpm
