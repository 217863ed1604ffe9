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
