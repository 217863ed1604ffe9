// Particle binning onto SPGrid pages, bit-exact with
// MpmSimulationBase::sortParticlesAndPolluteGrid (Lib/MPM/MpmSimulationBase.cpp:1032-1103).
//
//  1. key   = ((Linear_Offset(baseNode(x/dx)) >> data_bits) << (32 - block_bits)) + index
//             = page_index << 32 | element << index_bits | index        (k_keys)
//  2. sort  : the keys are unique, so any correct sort gives the reference's
//             order.  LSD: pass 0 places each key at its particle index
//             (k_keys), then 8-bit radix passes over the page/element bits.
//  3. groups: runs of equal page index (key >> 32), in sorted order.
//  4. pages : the reference calls Set_Page on each group's page and its 7
//             upper neighbours, in group order, and appends a page the first
//             time it is seen (SPGrid_Page_Map.h:61-70).  Emission e = 8g + t;
//             a page's block index is its rank among first emissions, found by
//             atomicMin(first[page], e) then a stable compaction of the
//             emissions that won.  This reproduces the first-touch order.
//  5. permutation of all particle state into sorted slots (coalesced passes).
#include "internal.cuh"

namespace zmpm {

constexpr int BIN_THREADS = 256;

static inline unsigned nblk(int64_t n, int t = BIN_THREADS) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ int int_floor_d(double u)
{
    int i = (int)u;
    return i - (i > u);
}
__device__ __forceinline__ int int_floor_f(float u)
{
    int i = (int)u;
    return i - (i > u);
}

struct PageDims {
    int px, py, pz;
    __device__ __forceinline__ int64_t index(int x, int y, int z) const { return ((int64_t)x * py + y) * pz + z; }
};

// KT: precision of the key arithmetic (double for FP64 runs, float for the
// mixed runs whose grid mirrors the reference's T=float build).
template <class L, class KT>
__global__ void k_keys(const double* __restrict__ x, int64_t cap, int64_t P, double inv_dx_d, float inv_dx_f, const int32_t* __restrict__ orig_id,
    uint64_t* __restrict__ keys_by_id, short4* __restrict__ base_by_id, PageDims pd, int32_t* __restrict__ flags)
{
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= P) return;
    int b[3];
    bool finite = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        finite = finite && isfinite(x[d * cap + s]);
        if constexpr (sizeof(KT) == 8) {
            double t = __dmul_rn(x[d * cap + s], inv_dx_d);
            b[d] = int_floor_d(__dsub_rn(t, 0.5));
        }
        else {
            float t = __fmul_rn((float)x[d * cap + s], inv_dx_f);
            b[d] = int_floor_f(__fsub_rn(t, 0.5f));
        }
    }
    int p0 = b[0] >> L::XB, p1 = b[1] >> L::YB, p2 = b[2] >> L::ZB;
    // a non-finite position converts to an arbitrary integer: it is out of the grid
    bool bad = !finite || b[0] < 0 || b[1] < 0 || b[2] < 0 || p0 + 1 >= pd.px || p1 + 1 >= pd.py || p2 + 1 >= pd.pz;
    if (bad) {
        atomicOr(flags, (int32_t)FLAG_OUT_OF_GRID);
        b[0] = b[1] = b[2] = 0;
        p0 = p1 = p2 = 0;
    }
    const int e = L::elem(b[0] & (L::BX - 1), b[1] & (L::BY - 1), b[2] & (L::BZ - 1));
    const uint64_t page = L::page_index(p0, p1, p2);
    const int32_t id = orig_id[s];
    keys_by_id[id] = (page << 32) | ((uint64_t)e << L::INDEX_BITS) | (uint64_t)id;
    base_by_id[id] = make_short4((short)b[0], (short)b[1], (short)b[2], 0);
}

__global__ void k_group_heads(const uint64_t* __restrict__ keys, int64_t P, int32_t* __restrict__ flag)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    flag[i] = (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32)) ? 1 : 0;
}

// New slot i receives particle keys[i] & idmask: gather every field from its
// old slot.  Also writes group starts and each group's page coordinates.
template <class L>
__global__ void k_permute(const uint64_t* __restrict__ keys, int64_t P, int64_t cap, int npd, const double* __restrict__ pd_src,
    double* __restrict__ pd_dst, const int32_t* __restrict__ pi_src, int32_t* __restrict__ pi_dst, int32_t* __restrict__ slot_of_id,
    const short4* __restrict__ base_by_id, short4* __restrict__ base, const int32_t* __restrict__ head, const int32_t* __restrict__ gidx,
    int32_t* __restrict__ group_start, int4* __restrict__ group_page)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const uint64_t k = keys[i];
    const int32_t id = (int32_t)(k & ((1ull << L::INDEX_BITS) - 1));
    const int32_t old = slot_of_id[id];
#pragma unroll 4
    for (int f = 0; f < npd; ++f) pd_dst[f * cap + i] = pd_src[f * cap + old];
#pragma unroll
    for (int f = 0; f < PI_FIELDS; ++f) pi_dst[f * cap + i] = pi_src[f * cap + old];
    pi_dst[PI_ID * cap + i] = id;
    slot_of_id[id] = (int32_t)i;
    short4 b = base_by_id[id];
    base[i] = b;
    if (head[i]) {
        int g = gidx[i];
        group_start[g] = (int32_t)i;
        group_page[g] = make_int4(b.x >> L::XB, b.y >> L::YB, b.z >> L::ZB, 0);
    }
}

__global__ void k_set_last(int32_t* __restrict__ group_start, const int32_t* __restrict__ G, int64_t P)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) group_start[*G] = (int32_t)P;
}

// Emission e = 8 g + t visits page (group page + (t>>2, (t>>1)&1, t&1)),
// the loop order of MpmSimulationBase.cpp:1081-1088.
__global__ void k_emit(const int4* __restrict__ group_page, int64_t G, PageDims pd, int32_t* __restrict__ first)
{
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 8 * G) return;
    int4 gp = group_page[e >> 3];
    int t = (int)(e & 7);
    int64_t idx = pd.index(gp.x + (t >> 2), gp.y + ((t >> 1) & 1), gp.z + (t & 1));
    atomicMin(&first[idx], (int32_t)e);
}

__global__ void k_mark_first(const int4* __restrict__ group_page, int64_t G, PageDims pd, const int32_t* __restrict__ first, int32_t* __restrict__ flag)
{
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 8 * G) return;
    int4 gp = group_page[e >> 3];
    int t = (int)(e & 7);
    int64_t idx = pd.index(gp.x + (t >> 2), gp.y + ((t >> 1) & 1), gp.z + (t & 1));
    flag[e] = (first[idx] == (int32_t)e) ? 1 : 0;
}

template <class L>
__global__ void k_blocks(const int4* __restrict__ group_page, int64_t G, PageDims pd, const int32_t* __restrict__ flag,
    const int32_t* __restrict__ pos, int32_t* __restrict__ page_block, int4* __restrict__ block_page, uint64_t* __restrict__ block_index)
{
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 8 * G || !flag[e]) return;
    int4 gp = group_page[e >> 3];
    int t = (int)(e & 7);
    int x = gp.x + (t >> 2), y = gp.y + ((t >> 1) & 1), z = gp.z + (t & 1);
    int b = pos[e];
    page_block[pd.index(x, y, z)] = b;
    block_page[b] = make_int4(x, y, z, 0);
    block_index[b] = L::page_index(x, y, z);
}

__global__ void k_group_nbr(const int4* __restrict__ group_page, int64_t G, PageDims pd, const int32_t* __restrict__ page_block,
    int32_t* __restrict__ first, int32_t* __restrict__ nbr)
{
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 8 * G) return;
    int4 gp = group_page[e >> 3];
    int t = (int)(e & 7);
    int64_t idx = pd.index(gp.x + (t >> 2), gp.y + ((t >> 1) & 1), gp.z + (t & 1));
    nbr[e] = page_block[idx];
    first[idx] = 0x7fffffff; // leave the first-touch table clean for the next pass
}

template <class L, class KT>
static int binning_impl(Ctx* ctx)
{
    cudaStream_t st = ctx->stream;
    const int64_t P = ctx->P, cap = ctx->Pcap;
    PageDims pdims{ ctx->pages[0], ctx->pages[1], ctx->pages[2] };
    DevCounters* dc = ctx->counters.as<DevCounters>();
    ZMPM_CUDA(cudaMemsetAsync(dc, 0, sizeof(DevCounters), st));
    if (P == 0) {
        ctx->G = ctx->B = 0;
        ctx->binned = true;
        return ZMPM_OK;
    }
    ZMPM_CUDA(ctx->keys.ensure(P * sizeof(uint64_t)));
    ZMPM_CUDA(ctx->keys_alt.ensure(P * sizeof(uint64_t)));
    ZMPM_CUDA(ctx->flags_i32.ensure(P * sizeof(int32_t)));
    ZMPM_CUDA(ctx->scan_i32.ensure((P + 1) * sizeof(int32_t)));
    ZMPM_CUDA(ctx->scan_scr.ensure((scan_scratch_elems(8 * P + 8) + 8) * sizeof(int32_t)));
    ZMPM_CUDA(ctx->radix_scr.ensure((radix_scratch_elems(P) + 8) * sizeof(int32_t)));
    ZMPM_CUDA(ctx->group_start.ensure((P + 1) * sizeof(int32_t)));
    ZMPM_CUDA(ctx->group_page.ensure(P * sizeof(int4)));

    k_keys<L, KT><<<nblk(P), BIN_THREADS, 0, st>>>(ctx->pdf(PD_X), cap, P, 1.0 / ctx->cfg.dx, 1.0f / (float)ctx->cfg.dx, ctx->pif(PI_ID), ctx->keys.as<uint64_t>(),
        ctx->base_by_id.as<short4>(), pdims, &dc->flags);
    ++g_kernel_launches;
    uint64_t* sorted = radix_sort(ctx->keys.as<uint64_t>(), ctx->keys_alt.as<uint64_t>(), P, L::INDEX_BITS, ctx->key_bits,
        ctx->radix_scr.as<int32_t>(), st);
    if (sorted != ctx->keys.as<uint64_t>()) std::swap(ctx->keys, ctx->keys_alt);
    const uint64_t* keys = ctx->keys.as<uint64_t>();

    int32_t* head = ctx->flags_i32.as<int32_t>();
    int32_t* gidx = ctx->scan_i32.as<int32_t>();
    int32_t* tot = ctx->scan_scr.as<int32_t>();
    int32_t* sscr = tot + 8;
    k_group_heads<<<nblk(P), BIN_THREADS, 0, st>>>(keys, P, head);
    ++g_kernel_launches;
    exclusive_scan<int32_t>(head, gidx, P, tot, sscr, st);
    k_permute<L><<<nblk(P), BIN_THREADS, 0, st>>>(keys, P, cap, ctx->pd_active, ctx->pd.as<double>(), ctx->pd_alt.as<double>(), ctx->pi.as<int32_t>(),
        ctx->pi_alt.as<int32_t>(), ctx->slot_of_id.as<int32_t>(), ctx->base_by_id.as<short4>(), ctx->base.as<short4>(), head, gidx,
        ctx->group_start.as<int32_t>(), ctx->group_page.as<int4>());
    ++g_kernel_launches;
    std::swap(ctx->pd, ctx->pd_alt);
    std::swap(ctx->pi, ctx->pi_alt);
    k_set_last<<<1, 32, 0, st>>>(ctx->group_start.as<int32_t>(), tot, P);
    ++g_kernel_launches;

    int32_t hG = 0;
    ZMPM_CUDA(cudaMemcpyAsync(&hG, tot, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    ZMPM_CUDA(cudaMemcpyAsync(&ctx->hcounters, dc, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
    ZMPM_CUDA(cudaStreamSynchronize(st));
    if (ctx->hcounters.flags & FLAG_OUT_OF_GRID) {
        ctx->err = "a particle's stencil leaves the grid (raise grid_log2 or move the scene)";
        return ZMPM_OUT_OF_GRID;
    }
    const int64_t G = hG;
    ctx->G = G;

    ZMPM_CUDA(ctx->group_nbr.ensure(8 * G * sizeof(int32_t)));
    ZMPM_CUDA(ctx->emit_flag.ensure(8 * G * sizeof(int32_t)));
    ZMPM_CUDA(ctx->emit_scan.ensure(8 * G * sizeof(int32_t)));
    const int4* gpage = ctx->group_page.as<int4>();
    int32_t* first = ctx->page_first.as<int32_t>();
    k_emit<<<nblk(8 * G), BIN_THREADS, 0, st>>>(gpage, G, pdims, first);
    ++g_kernel_launches;
    k_mark_first<<<nblk(8 * G), BIN_THREADS, 0, st>>>(gpage, G, pdims, first, ctx->emit_flag.as<int32_t>());
    ++g_kernel_launches;
    exclusive_scan<int32_t>(ctx->emit_flag.as<int32_t>(), ctx->emit_scan.as<int32_t>(), 8 * G, tot, sscr, st);
    int32_t hB = 0;
    ZMPM_CUDA(cudaMemcpyAsync(&hB, tot, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    ZMPM_CUDA(cudaStreamSynchronize(st));
    const int64_t B = hB;
    ctx->B = B;
    ZMPM_CUDA(ctx->block_page.ensure(B * sizeof(int4)));
    ZMPM_CUDA(ctx->block_index.ensure(B * sizeof(uint64_t)));
    k_blocks<L><<<nblk(8 * G), BIN_THREADS, 0, st>>>(gpage, G, pdims, ctx->emit_flag.as<int32_t>(), ctx->emit_scan.as<int32_t>(),
        ctx->page_block.as<int32_t>(), ctx->block_page.as<int4>(), ctx->block_index.as<uint64_t>());
    ++g_kernel_launches;
    k_group_nbr<<<nblk(8 * G), BIN_THREADS, 0, st>>>(gpage, G, pdims, ctx->page_block.as<int32_t>(), first, ctx->group_nbr.as<int32_t>());
    ++g_kernel_launches;
    ZMPM_CUDA(cudaGetLastError());
    ctx->binned = true;
    return ZMPM_OK;
}

int run_binning(Ctx* ctx)
{
    if (ctx->layout == 1) return ctx->mixed ? binning_impl<Layout244, float>(ctx) : binning_impl<Layout244, double>(ctx);
    return ctx->mixed ? binning_impl<Layout444, float>(ctx) : binning_impl<Layout444, double>(ctx);
}

} // namespace zmpm
