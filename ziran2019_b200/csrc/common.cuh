// Shared device/host definitions of the B200 implicit APIC MPM library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define ZMPM_HD __host__ __device__ __forceinline__
#define ZMPM_D __device__ __forceinline__

namespace zmpm {

// ----------------------------------------------------------- SPGrid layout --
// One SPGrid page (4 KiB) holds 2^block_bits GridState structs.  Within a page
// the element index packs z in the low bits, then y, then x
// (SPGrid_Mask.h:63-67), so element e = (lx << (YB+ZB)) | (ly << ZB) | lz.
// Page indices interleave the page coordinates with the masks of
// SPGrid_Mask.h:35-41 (evaluated below as constexpr).
template <int LOG2S>
struct Layout {
    static constexpr int LOG2_STRUCT = LOG2S;
    static constexpr int BLOCK_BITS = 12 - LOG2S;
    static constexpr int ZB = BLOCK_BITS / 3 + (BLOCK_BITS % 3 > 0);
    static constexpr int YB = BLOCK_BITS / 3 + (BLOCK_BITS % 3 > 1);
    static constexpr int XB = BLOCK_BITS / 3;
    static constexpr int BX = 1 << XB, BY = 1 << YB, BZ = 1 << ZB;
    static constexpr int NPB = 1 << BLOCK_BITS; // nodes per page
    static constexpr int WX = 2 * BX, WY = 2 * BY, WZ = 2 * BZ;
    static constexpr int INDEX_BITS = 32 - BLOCK_BITS; // particle index bits of the key
    static constexpr int SH = 3 - BLOCK_BITS % 3;
    static constexpr uint64_t HI = ~0ull << 12;
    static constexpr uint64_t PAGE_Z = (0x9249249249249249ull << SH) & HI;
    static constexpr uint64_t PAGE_Y = (0x2492492492492492ull << SH) & HI;
    static constexpr uint64_t PAGE_X = (0x4924924924924924ull << SH) & HI;
    static constexpr uint64_t ELEM_Z = ((1ull << ZB) - 1) << LOG2S;
    static constexpr uint64_t ELEM_Y = ((1ull << YB) - 1) << (LOG2S + ZB);
    static constexpr uint64_t ELEM_X = ((1ull << XB) - 1) << (LOG2S + ZB + YB);
    static constexpr uint64_t XMASK = PAGE_X | ELEM_X;
    static constexpr uint64_t YMASK = PAGE_Y | ELEM_Y;
    static constexpr uint64_t ZMASK = PAGE_Z | ELEM_Z;

    ZMPM_HD static int elem(int lx, int ly, int lz) { return (lx << (YB + ZB)) | (ly << ZB) | lz; }
    // deposit the bits of c (c >= 0) into the set bits of mask, lowest first
    ZMPM_HD static uint64_t deposit(uint32_t c, uint64_t mask)
    {
        uint64_t r = 0;
        while (c) {
            uint64_t low = mask & (~mask + 1); // lowest set bit of mask
            if (c & 1u) r |= low;
            mask ^= low;
            c >>= 1;
        }
        return r;
    }
    ZMPM_HD static uint32_t extract(uint64_t v, uint64_t mask)
    {
        uint32_t r = 0;
        int k = 0;
        while (mask) {
            uint64_t low = mask & (~mask + 1);
            if (v & low) r |= 1u << k;
            mask ^= low;
            ++k;
        }
        return r;
    }
    // SPGrid_Mask::Linear_Offset for non-negative coordinates
    ZMPM_HD static uint64_t linear_offset(int i, int j, int k)
    {
        return deposit((uint32_t)i, XMASK) | deposit((uint32_t)j, YMASK) | deposit((uint32_t)k, ZMASK);
    }
    // page index (offset >> 12) of page coordinates
    ZMPM_HD static uint64_t page_index(int px, int py, int pz)
    {
        return (deposit((uint32_t)px, PAGE_X) | deposit((uint32_t)py, PAGE_Y) | deposit((uint32_t)pz, PAGE_Z)) >> 12;
    }
};
using Layout244 = Layout<7>; // GridState<double,3>
using Layout444 = Layout<6>; // GridState<float,3>

// ----------------------------------------------------------- device flags --
enum : uint32_t { FLAG_NAN = 1u, FLAG_TIMEOUT = 2u, FLAG_OUT_OF_GRID = 4u, FLAG_CFL = 8u };

// Collider state evaluated at the substep's start time.
struct DevCollider {
    int shape, type;
    double friction;
    double a[3], b[3], radius;
    double R[9];
    double omega[3], t[3], dtdt[3];
    double s, dsdt;
};
constexpr int MAX_COLLIDERS = 32;

// Per-particle model parameters (one model copy per particle, as the reference).
struct ModelParams {
    double mu, lambda, kappa, g;
};

} // namespace zmpm
