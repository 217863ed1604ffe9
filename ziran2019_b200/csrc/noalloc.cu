// Allocation-free particle key sort (zmpm_sort_keys_noalloc in include/zmpm.h).
//
// Some callers cannot call cudaMalloc: a host whose memory is pre-reserved by
// another allocator and forbids new device allocations, a real-time loop that
// cannot afford cudaMalloc's implicit device synchronisation, or code that only
// owns the buffers it was handed.  This entry point computes and sorts the
// SPGrid particle keys (the first part of sortParticlesAndPolluteGrid) using
// only the caller's input and output buffers plus the fixed scratch array
// below.
//
// The scratch is a file-scope static __device__ array, so every GPU that loads
// this library holds it (about 2.2 MB) until the process exits.  In host code
// the array's name is only a host-side stand-in, never a device address: the
// device address is looked up once per device with cudaGetSymbolAddress (with
// that device current) and passed to the kernels.  The first call on a device
// performs that lookup and caches the address for the life of the process; a
// caller that resets the device (cudaDeviceReset) invalidates that cached
// address, so this entry point must not be used after such a reset.  Each call
// synchronises its stream and copies a status word to host memory, so no call
// can be made inside a stream capture.
// Every call reuses the same array and it keeps the previous call's contents:
// the out-of-grid flag is cleared at the start of each call, and everything
// else is fully written before it is read.  Calls whose work overlaps on the
// GPU (concurrent streams, several host threads) race on the array.
#include <mutex>

#include "internal.cuh"

namespace zmpm {

namespace {

constexpr int64_t NOALLOC_MAX = ZMPM_NOALLOC_MAX_PARTICLES;
// radix_sort scratch for NOALLOC_MAX keys (int32 elements): 2 x 256 x tiles + scan levels
constexpr int64_t NOALLOC_RADIX_ELEMS = 2 * 256 * (NOALLOC_MAX / 4096 + 1) + 1024;
constexpr size_t OFF_KEYS = 0;
constexpr size_t OFF_RADIX = OFF_KEYS + NOALLOC_MAX * sizeof(uint64_t);
constexpr size_t OFF_FLAGS = OFF_RADIX + NOALLOC_RADIX_ELEMS * sizeof(int32_t);
constexpr size_t NOALLOC_BYTES = OFF_FLAGS + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[MAX_DEVICES] = {};

// Device address of the scratch array on `dev` (which must be current).
cudaError_t scratch_address(int dev, void** out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

__device__ __forceinline__ int floor_d(double u)
{
    int i = (int)u;
    return i - (i > u);
}
__device__ __forceinline__ int floor_f(float u)
{
    int i = (int)u;
    return i - (i > u);
}

// Keys of particles [0, n) from row-major positions x[n][3]; the particle index
// is the array index.  Same arithmetic as the binning pass of a context.
template <class L, class KT>
__global__ void k_noalloc_keys(const double* __restrict__ x, int64_t n, double inv_dx_d, float inv_dx_f, int px, int py, int pz,
    uint64_t* __restrict__ keys, int32_t* __restrict__ flags)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b[3];
    bool finite = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double xd = x[3 * i + d];
        finite = finite && isfinite(xd);
        if constexpr (sizeof(KT) == 8)
            b[d] = floor_d(__dsub_rn(__dmul_rn(xd, inv_dx_d), 0.5));
        else
            b[d] = floor_f(__fsub_rn(__fmul_rn((float)xd, inv_dx_f), 0.5f));
    }
    int p0 = b[0] >> L::XB, p1 = b[1] >> L::YB, p2 = b[2] >> L::ZB;
    // a non-finite coordinate converts to an arbitrary integer: it is out of the grid
    if (!finite || b[0] < 0 || b[1] < 0 || b[2] < 0 || p0 + 1 >= px || p1 + 1 >= py || p2 + 1 >= pz) {
        atomicOr(flags, 1);
        b[0] = b[1] = b[2] = 0;
        p0 = p1 = p2 = 0;
    }
    const int e = L::elem(b[0] & (L::BX - 1), b[1] & (L::BY - 1), b[2] & (L::BZ - 1));
    keys[i] = (L::page_index(p0, p1, p2) << 32) | ((uint64_t)e << L::INDEX_BITS) | (uint64_t)i;
}

int64_t bits_of(uint64_t v)
{
    int64_t n = 0;
    while (v) {
        ++n;
        v >>= 1;
    }
    return n;
}

template <class L, class KT>
int sort_keys(const double* x, int64_t n, double dx, int grid_log2, uint64_t* keys, cudaStream_t st, unsigned char* scratch)
{
    const int nn = 1 << grid_log2;
    const int px = nn / L::BX, py = nn / L::BY, pz = nn / L::BZ;
    const int key_bits = (int)bits_of((L::page_index(px - 1, py - 1, pz - 1) << L::BLOCK_BITS) | (uint64_t)(L::NPB - 1));
    uint64_t* alt = reinterpret_cast<uint64_t*>(scratch + OFF_KEYS);
    int32_t* radix = reinterpret_cast<int32_t*>(scratch + OFF_RADIX);
    int32_t* flags = reinterpret_cast<int32_t*>(scratch + OFF_FLAGS);
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t), st) != cudaSuccess) return ZMPM_CUDA_ERROR;
    k_noalloc_keys<L, KT><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, 1.0 / dx, 1.0f / (float)dx, px, py, pz, keys, flags);
    ++g_kernel_launches;
    // a launch failure of this call (peeked, so an error the caller left pending is not cleared)
    if (cudaPeekAtLastError() != cudaSuccess) return ZMPM_CUDA_ERROR;
    uint64_t* out = radix_sort(keys, alt, n, L::INDEX_BITS, key_bits, radix, st);
    if (out != keys && cudaMemcpyAsync(keys, out, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return ZMPM_CUDA_ERROR;
    int32_t hflag = 0;
    if (cudaMemcpyAsync(&hflag, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess) return ZMPM_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return ZMPM_CUDA_ERROR;
    return hflag ? ZMPM_OUT_OF_GRID : ZMPM_OK;
}

} // namespace
} // namespace zmpm

extern "C" int zmpm_sort_keys_noalloc(const double* x, int64_t n, double dx, int32_t precision, int32_t layout, int32_t grid_log2,
    uint64_t* keys, void* stream)
{
    using namespace zmpm;
    if (n < 0 || n > NOALLOC_MAX || (n > 0 && (!x || !keys)) || !(dx > 0) || grid_log2 < 4 || grid_log2 > 12) return ZMPM_BAD_ARG;
    if (precision != ZMPM_FP64 && precision != ZMPM_MIXED) return ZMPM_BAD_ARG;
    const int lay = layout == ZMPM_LAYOUT_AUTO ? (precision == ZMPM_MIXED ? ZMPM_LAYOUT_444 : ZMPM_LAYOUT_244) : layout;
    if (lay != ZMPM_LAYOUT_244 && lay != ZMPM_LAYOUT_444) return ZMPM_BAD_ARG;
    if (radix_scratch_elems(n) > NOALLOC_RADIX_ELEMS) return ZMPM_BAD_ARG;
    if (n == 0) return ZMPM_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return ZMPM_CUDA_ERROR;
    void* scratch = nullptr;
    if (scratch_address(dev, &scratch) != cudaSuccess) return ZMPM_CUDA_ERROR;
    unsigned char* sp = static_cast<unsigned char*>(scratch);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool f32 = precision == ZMPM_MIXED;
    if (lay == ZMPM_LAYOUT_244)
        return f32 ? sort_keys<Layout244, float>(x, n, dx, grid_log2, keys, st, sp) : sort_keys<Layout244, double>(x, n, dx, grid_log2, keys, st, sp);
    return f32 ? sort_keys<Layout444, float>(x, n, dx, grid_log2, keys, st, sp) : sort_keys<Layout444, double>(x, n, dx, grid_log2, keys, st, sp);
}
