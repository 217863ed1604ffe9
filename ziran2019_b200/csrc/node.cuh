// Node-kernel helpers shared by the Newton solver and the phase-field solve:
// launch width, deterministic block and partial-sum reductions, node-vector
// indexing of the block-dense [B][NC][NPB] layout.
#pragma once

#include <cstdint>

namespace zmpm {

constexpr int ND_THREADS = 256;


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

// The same sum read through L2 (ld.cg), for partials that other CTAs of the
// running kernel wrote.
__device__ __forceinline__ double reduce_partials_l2(const double* part, int n)
{
    double s = 0;
    for (int i = threadIdx.x; i < n; i += ND_THREADS) s += __ldcg(part + i);
    return block_sum(s);
}

// True in every thread of the CTA that finishes last among the kernel's CTAs;
// every CTA's earlier global writes (its partial sum) are then visible to it,
// so that CTA can run the scalar step that needs all partials inside the same
// kernel.  It puts the ticket back to 0 for the next kernel.  No CTA waits.
__device__ __forceinline__ bool last_cta(uint32_t* ticket)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
        if (last) {
            *ticket = 0;
            __threadfence();
        }
    }
    __syncthreads();
    return last;
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

} // namespace zmpm
