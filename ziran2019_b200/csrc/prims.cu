// Device primitives for the binning pass: exclusive prefix sums and a stable
// LSD radix sort of 64-bit keys (8-bit digits).
//
// Radix pass = histogram (one 256-bin count per 4096-key tile) -> exclusive
// scan of the digit-major count table -> stable scatter.  The scatter ranks
// keys inside a tile with __match_any_sync: warp w owns a contiguous run of the
// tile and walks it 32 keys at a time, so rank = (same-digit keys in earlier
// warps) + (same-digit keys earlier in this warp).  Equal digits keep their
// input order, which makes each pass stable.
#include "internal.cuh"

namespace zmpm {

thread_local int64_t g_kernel_launches = 0;

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// exclusive scan of one tile per CTA; tile totals to sums[blockIdx.x]
template <class T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const T* __restrict__ in, T* __restrict__ out, int64_t n, T* __restrict__ sums)
{
    __shared__ T warp_tot[SCAN_THREADS / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T run = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + i;
        T x = (idx < n) ? in[idx] : T(0);
        v[i] = run;
        run += x;
    }
    T incl = warp_incl_scan(run);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T t = (lane < SCAN_THREADS / 32) ? warp_tot[lane] : T(0);
        T ti = warp_incl_scan(t);
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = ti - t;
        if (lane == SCAN_THREADS / 32 - 1) sums[blockIdx.x] = ti;
    }
    __syncthreads();
    T off = warp_tot[warp] + (incl - run);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t idx = base + i;
        if (idx < n) out[idx] = v[i] + off;
    }
}

template <class T>
__global__ void k_scan_add(T* __restrict__ out, int64_t n, const T* __restrict__ offs)
{
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    const T o = offs[blockIdx.x];
    for (int i = threadIdx.x; i < SCAN_TILE; i += blockDim.x) {
        int64_t idx = base + i;
        if (idx < n) out[idx] += o;
    }
}

template <class T>
__global__ void k_scan_total(const T* __restrict__ in, const T* __restrict__ out, int64_t n, T* __restrict__ total)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *total = (n > 0) ? out[n - 1] + in[n - 1] : T(0);
}

template <class T>
static void scan_rec(const T* in, T* out, int64_t n, T* scratch, cudaStream_t st)
{
    if (n <= 0) return;
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    T* sums = scratch;
    T* sums_out = scratch + nb;
    k_scan_tile<T><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, out, n, sums);
    ++g_kernel_launches;
    if (nb > 1) {
        scan_rec<T>(sums, sums_out, nb, scratch + 2 * nb, st);
        k_scan_add<T><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(out, n, sums_out);
        ++g_kernel_launches;
    }
}

int64_t scan_scratch_elems(int64_t n)
{
    int64_t total = 0;
    while (n > 1) {
        int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
        total += 2 * nb;
        n = nb;
    }
    return total + 2;
}

template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, T* total, T* scratch, cudaStream_t st)
{
    scan_rec<T>(in, out, n, scratch, st);
    k_scan_total<T><<<1, 32, 0, st>>>(in, out, n, total);
    ++g_kernel_launches;
}
template void exclusive_scan<int32_t>(const int32_t*, int32_t*, int64_t, int32_t*, int32_t*, cudaStream_t);
template void exclusive_scan<int64_t>(const int64_t*, int64_t*, int64_t, int64_t*, int64_t*, cudaStream_t);

// ------------------------------------------------------------ radix sort --
constexpr int RADIX_THREADS = 256;
constexpr int RADIX_WARPS = RADIX_THREADS / 32;
constexpr int RADIX_IPT = 16; // keys per thread
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_IPT;

__global__ void __launch_bounds__(RADIX_THREADS) k_radix_hist(const uint64_t* __restrict__ keys, int64_t n, int shift, int32_t* __restrict__ hist, int ntiles)
{
    __shared__ int32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RADIX_TILE;
    for (int i = threadIdx.x; i < RADIX_TILE; i += RADIX_THREADS) {
        int64_t idx = base + i;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RADIX_THREADS) k_radix_scatter(const uint64_t* __restrict__ keys, uint64_t* __restrict__ out, int64_t n, int shift,
    const int32_t* __restrict__ offs, int ntiles)
{
    __shared__ int32_t cnt[RADIX_WARPS][256];
    for (int i = threadIdx.x; i < RADIX_WARPS * 256; i += RADIX_THREADS) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t wbase = (int64_t)blockIdx.x * RADIX_TILE + (int64_t)warp * (32 * RADIX_IPT);
    const unsigned lt = (1u << lane) - 1u;
    uint64_t k[RADIX_IPT];
    int32_t rank[RADIX_IPT];
    uint32_t dig[RADIX_IPT];
#pragma unroll
    for (int r = 0; r < RADIX_IPT; ++r) {
        int64_t idx = wbase + r * 32 + lane;
        bool valid = idx < n;
        k[r] = valid ? keys[idx] : 0ull;
        uint32_t d = valid ? (uint32_t)((k[r] >> shift) & 255u) : 256u;
        dig[r] = d;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int before = __popc(peers & lt);
        int leader = __ffs(peers) - 1;
        int c = (d < 256u) ? cnt[warp][d] : 0;
        rank[r] = c + before;
        __syncwarp();
        if (lane == leader && d < 256u) cnt[warp][d] = c + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps, per digit
    {
        int d = threadIdx.x;
        int run = 0;
#pragma unroll
        for (int w = 0; w < RADIX_WARPS; ++w) {
            int t = cnt[w][d];
            cnt[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RADIX_IPT; ++r) {
        uint32_t d = dig[r];
        if (d < 256u) {
            int64_t pos = (int64_t)offs[(int64_t)d * ntiles + blockIdx.x] + cnt[warp][d] + rank[r];
            out[pos] = k[r];
        }
    }
}

int64_t radix_scratch_elems(int64_t n)
{
    int64_t ntiles = (n + RADIX_TILE - 1) / RADIX_TILE;
    int64_t h = 256 * ntiles;
    return 2 * h + scan_scratch_elems(h) + 2;
}

// Sorts keys[0..n) on bits [lo_bit, lo_bit + nbits); `alt` is a second buffer
// of n keys.  Returns the buffer that holds the result.
uint64_t* radix_sort(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int nbits, int32_t* scratch, cudaStream_t st)
{
    if (n <= 1 || nbits <= 0) return keys;
    int ntiles = (int)((n + RADIX_TILE - 1) / RADIX_TILE);
    int64_t h = 256 * (int64_t)ntiles;
    int32_t* hist = scratch;
    int32_t* offs = scratch + h;
    int32_t* tot = scratch + 2 * h;
    int32_t* sscr = scratch + 2 * h + 2;
    uint64_t* src = keys;
    uint64_t* dst = alt;
    for (int b = 0; b < nbits; b += 8) {
        int shift = lo_bit + b;
        k_radix_hist<<<ntiles, RADIX_THREADS, 0, st>>>(src, n, shift, hist, ntiles);
        ++g_kernel_launches;
        exclusive_scan<int32_t>(hist, offs, h, tot, sscr, st);
        k_radix_scatter<<<ntiles, RADIX_THREADS, 0, st>>>(src, dst, n, shift, offs, ntiles);
        ++g_kernel_launches;
        uint64_t* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

} // namespace zmpm
