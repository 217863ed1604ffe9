// Helpers shared by the particle <-> grid kernels (transfer.cu, admm.cu).
//
// Work unit: one CTA per particle group (the particles whose base node lies in
// one SPGrid page, MpmSimulationBase.cpp:1055-1063).  Every stencil node of
// those particles lies in the 2x2x2 pages starting at the group's page, whose
// block indices binning stored in group_nbr[8g..8g+7].
//
//  gather  : the 8 page slabs of a grid vector ([3][NPB] contiguous per page)
//            are staged into shared memory with cp.async.bulk (bulk copy)
//            completing on an mbarrier; particles read their 27 nodes there.
//  scatter : particles accumulate into a shared [8][C][NPB] window with shared
//            atomics; the window is flushed with coalesced global atomics.
#pragma once
#include "internal.cuh"

namespace zmpm {

constexpr int XF_THREADS = 128;
constexpr long long STAGE_WAIT_LIMIT = 1ll << 22;

// ------------------------------------------------------------ TMA staging --
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)), "l"(src),
        "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after STAGE_WAIT_LIMIT polls and raises FLAG_TIMEOUT.
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* flags)
{
    long long it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++it > STAGE_WAIT_LIMIT) {
            atomicOr(flags, (int32_t)FLAG_TIMEOUT);
            return;
        }
    }
}

// Stages the 8 page slabs ([3][NPB] values each) of vector `vec` into win.
// Must be called by all threads of the CTA; nbr is in shared memory.  A slab
// is 3 NPB doubles or floats: a multiple of 16 bytes at a 16-byte aligned
// offset for NPB = 32 or 64.
template <int NPB, class T>
__device__ __forceinline__ void stage_window(T* win, const T* __restrict__ vec, const int32_t* nbr, uint64_t* bar, int32_t* flags)
{
    constexpr uint32_t SLAB = 3 * NPB * sizeof(T);
    static_assert(SLAB % 16 == 0, "bulk copies move multiples of 16 bytes");
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, 8 * SLAB);
#pragma unroll
        for (int t = 0; t < 8; ++t) bulk_g2s(win + t * 3 * NPB, vec + (int64_t)nbr[t] * 3 * NPB, SLAB, bar);
    }
    __syncthreads();
    mbar_wait_bounded(bar, 0, flags);
}

// ------------------------------------------------------------ B-spline ----
// Quadratic B-spline weights of one axis from d0 = x/dx - base (BSplines.h:55-81).
template <class T>
__device__ __forceinline__ void bspline(T d0, T w[3], T dw[3])
{
    T z = T(1.5) - d0;
    w[0] = T(0.5) * z * z;
    T d1 = d0 - T(1);
    w[1] = T(0.75) - d1 * d1;
    T d2 = T(1) - d1;
    T zz = T(1.5) - d2;
    w[2] = T(0.5) * zz * zz;
    dw[0] = -z;
    dw[1] = -T(2) * d1;
    dw[2] = zz;
}

// Window slot of stencil node (lx+i, ly+j, lz+k): page t in the 2x2x2
// neighbourhood, element e inside it.
template <class L>
__device__ __forceinline__ int win_slot(int wx, int wy, int wz, int& e)
{
    int t = ((wx >= L::BX) << 2) | ((wy >= L::BY) << 1) | (wz >= L::BZ);
    e = L::elem(wx & (L::BX - 1), wy & (L::BY - 1), wz & (L::BZ - 1));
    return t;
}

// Iterates the 27 stencil nodes in the order and with the products of
// MpmGrid::iterateKernel (MpmGrid.h:247-269).  f(t, e, node_offset_ijk, w, dw[3]).
template <class L, class T, class Fn>
__device__ __forceinline__ void for_stencil(int lx, int ly, int lz, const T w[3][3], const T dwr[3][3], T inv_dx, Fn&& f)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        T wi = w[0][i];
        T dwidxi = inv_dx * dwr[0][i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T wj = w[1][j];
            T wij = wi * wj;
            T dwijdxi = dwidxi * wj;
            T dwijdxj = wi * inv_dx * dwr[1][j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                T wk = w[2][k];
                T wijk = wij * wk;
                T dw[3] = { dwijdxi * wk, dwijdxj * wk, wij * inv_dx * dwr[2][k] };
                int e;
                int t = win_slot<L>(lx + i, ly + j, lz + k, e);
                f(t, e, i, j, k, wijk, dw);
            }
        }
    }
}

template <int NC, int NPB, class TA>
__device__ __forceinline__ void zero_window(TA* acc)
{
    for (int i = threadIdx.x; i < 8 * NC * NPB; i += blockDim.x) acc[i] = TA(0);
}
// Adds window [8][NC][NPB] into global block-dense arrays.  Component c < NC0
// goes to `a` ([B][NC0][NPB]), the rest to `b` ([B][NC-NC0][NPB]).
template <int NC, int NC0, int NPB, class TA>
__device__ __forceinline__ void flush_window(const TA* acc, const int32_t* nbr, double* __restrict__ a, double* __restrict__ b)
{
    for (int i = threadIdx.x; i < 8 * NC * NPB; i += blockDim.x) {
        TA v = acc[i];
        if (v == TA(0)) continue;
        int t = i / (NC * NPB);
        int r = i - t * NC * NPB;
        int c = r / NPB;
        int e = r - c * NPB;
        int64_t blk = nbr[t];
        if (c < NC0)
            atomicAdd(&a[(blk * NC0 + c) * NPB + e], (double)v);
        else
            atomicAdd(&b[(blk * (NC - NC0) + (c - NC0)) * NPB + e], (double)v);
    }
}


// ------------------------------------------------------ scatter ordering --
// Particles of a group are sorted by cell (element) then index.  Shared-memory
// scatters are issued in "layers": thread q handles the r-th particle (r = q /
// NPB) of cell e = q % NPB, so the 32 lanes of a warp hold particles of 32
// different cells and a warp-wide atomic at a fixed stencil offset never hits
// the same node twice.  A page holds NPB cells; cnt/start are per-cell counts
// and first slots inside the group.
template <class L>
struct CellLayout {
    int cnt[L::NPB];
    int start[L::NPB];
    int layers;
};

template <class L>
__device__ __forceinline__ void build_cell_layout(CellLayout<L>& cl, const short4* __restrict__ base, int s0, int s1)
{
    for (int e = threadIdx.x; e < L::NPB; e += blockDim.x) cl.cnt[e] = 0;
    __syncthreads();
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        const short4 b = base[s];
        atomicAdd(&cl.cnt[L::elem(b.x & (L::BX - 1), b.y & (L::BY - 1), b.z & (L::BZ - 1))], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        constexpr int PER = L::NPB / 32;
        const int lane = threadIdx.x;
        int c[PER], local = 0, mx = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            c[k] = cl.cnt[lane * PER + k];
            local += c[k];
            mx = c[k] > mx ? c[k] : mx;
        }
        int incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int n = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += n;
        }
        int run = incl - local;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            cl.start[lane * PER + k] = run;
            run += c[k];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            int n = __shfl_xor_sync(0xffffffffu, mx, o);
            mx = n > mx ? n : mx;
        }
        if (lane == 0) cl.layers = mx;
    }
    __syncthreads();
}

} // namespace zmpm
