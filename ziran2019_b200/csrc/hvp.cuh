// The Hessian-vector product of one particle group, shared by the per-group
// kernels (k_hvp_fused, k_op_fused) and the persistent Krylov kernels.
//
// MpmForceBase::addScaledForceDifferential (MpmForceBase.cpp:259-302) in one
// pass (fused.cuh): phase 1 gathers grad(x) at each particle from the staged
// window of the input vector and evaluates dS = V0 dP(grad(x) Fn) Fn^T from the
// Hessian scratch (computeStressDifferential, FBasedMpmForceHelper.cpp:132-
// 154); phase 2 adds dS grad w_ip to the nodes (rasterizeForceToTVStack with
// the differential, :102-152): out += sum_p dS_p grad w_ip.  T: arithmetic
// precision; TX: the input vector (FP32 node-major copy or FP64 vector).
// The per-particle map grad(x) -> dS is a model object: HvpModel (the
// constitutive model's differential from the Hessian scratch) or AdmmOpModel
// (the ADMM global operator's grad(x) B, AdmmSimulationFoam.h dvStep).
#pragma once
#include "fused.cuh"
#include "models.cuh"

namespace zmpm {

template <class L, class T, class TX, int CH>
struct HvpSmem {
    __align__(128) TX win[VecWindow<L::NPB, TX>::ELEMS];
    ScatterSmem<L, T, CH> sm;
    __align__(8) uint64_t bar;
};

// dS = V0 dP(G Fn) Fn^T from the Hessian scratch; particles without a model
// contribute nothing.
template <class T>
struct HvpModel {
    const int32_t* pi;
    const T* scr;
    int64_t cap;
    __device__ __forceinline__ bool active(int64_t s) const { return pi[PI_KIND * cap + s] != ZMPM_MODEL_NONE; }
    __device__ __forceinline__ M3<T> operator()(int64_t s, const M3<T>& G) const { return model_hvp<T>(pi[PI_KIND * cap + s], scr, cap, s, G); }
};

// ADMM's global operator: dS = G B with the particle's symmetric B (six
// entries, k_admm_init), every particle.
template <class T>
struct AdmmOpModel {
    const T* B;
    int64_t cap;
    __device__ __forceinline__ bool active(int64_t) const { return true; }
    __device__ __forceinline__ M3<T> operator()(int64_t s, const M3<T>& G) const
    {
        const T b00 = B[0 * cap + s], b01 = B[1 * cap + s], b02 = B[2 * cap + s], b11 = B[3 * cap + s], b12 = B[4 * cap + s],
                b22 = B[5 * cap + s];
        M3<T> d;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            d(r, 0) = G(r, 0) * b00 + G(r, 1) * b01 + G(r, 2) * b02;
            d(r, 1) = G(r, 0) * b01 + G(r, 1) * b11 + G(r, 2) * b12;
            d(r, 2) = G(r, 0) * b02 + G(r, 1) * b12 + G(r, 2) * b22;
        }
        return d;
    }
};

// All threads of the CTA call it for the slots [s0, s1) of group g (the whole
// group, or a piece of it when a persistent kernel splits the particles
// evenly over its CTAs: pieces of one group add to the same nodes); the CTA's
// shared state is reused piece after piece.  phase: -1 for a CTA's only group (the staging mbarrier is initialised
// here), else the count of windows this CTA staged before (the caller
// initialised the mbarrier once).
template <class L, class T, class TX, int CH, class Model>
__device__ __forceinline__ void hvp_group(HvpSmem<L, T, TX, CH>& hs, int g, int s0, int s1, const int32_t* __restrict__ group_nbr,
    const Model& model, int64_t cap, const short4* __restrict__ base, double dx,
    const T* __restrict__ frac, const TX* __restrict__ x, double* __restrict__ out, int32_t* __restrict__ flags, int phase = -1)
{
    constexpr int NPB = L::NPB;
    ScatterSmem<L, T, CH>& sm = hs.sm;
    __syncthreads(); // the previous group's flush is done with the shared state
    if (threadIdx.x < 8) sm.nbr[threadIdx.x] = group_nbr[8 * g + threadIdx.x];
    zero_window<3, NPB>(sm.acc);
    __syncthreads();
    stage_vec_window<NPB, TX>(hs.win, x, sm.nbr, &hs.bar, flags, phase);
    const TX* win = hs.win;
    const int n = s1 - s0;
    build_cell_layout<L>(sm.cl, base, s0, s1);
    list_occupied(sm);
    const T inv_dx = T(1.0 / dx);
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
            M3<T> dS = m3_zero<T>();
            if (model.active(s)) {
                const short4 b = base[s];
                T w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all(fr[d], w[d], dw[d]);
                const StencilOffsets<L> so(b.x & (L::BX - 1), b.y & (L::BY - 1), b.z & (L::BZ - 1));
                M3<T> G;
                if constexpr (sizeof(T) == 4 && sizeof(TX) == 4)
                    gather_gradient_f32<L>(win, so, w, dw, G.a);
                else
                    gather_gradient<L, T, TX>(win, so, w, dw, G.a);
#pragma unroll
                for (int q = 0; q < 9; ++q) G.a[q] *= inv_dx;
                dS = model(s, G);
            }
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) rc[(3 + 3 * r + c) * sm.FS] = dS(r, c) * inv_dx;
        }
        __syncthreads();
        scatter_rows(sm, c0, c1);
    }
    __syncthreads();
    flush_window<3, 3, NPB>(sm.acc, sm.nbr, out, nullptr);
}

} // namespace zmpm
