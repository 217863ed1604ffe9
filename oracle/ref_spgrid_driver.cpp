// TEST INFRASTRUCTURE -- builds against the reference's own SPGrid sources.
//
// This driver is compiled together with the reference files
// Lib/SPGrid/Core/SPGrid_Utilities.cpp and SPGrid_Geometry.cpp, straight from
// the reference tree (oracle/Makefile, target `ref`), into oracle/_ref/.  It
// evaluates the reference's SPGrid_Mask::Linear_Offset / Packed_Add /
// LinearToCoord and SPGrid_Page_Map::Set_Page / Get_Blocks on seeded inputs so
// that tests/golden/ holds outputs of the reference code itself.  The particle
// key, grouping and page-touch loop around those calls follow
// MpmSimulationBase::sortParticlesAndPolluteGrid
// (Lib/MPM/MpmSimulationBase.cpp:1032-1103), which cannot be compiled here
// (it needs Eigen/TBB/OpenVDB).
//
// Usage: ref_spgrid masks|offsets|packed_add|bin <in.bin> <out.bin>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <iostream>

#include <SPGrid/Core/SPGrid_Utilities.h>
#include <SPGrid/Core/SPGrid_Geometry.h>
#include <SPGrid/Core/SPGrid_Mask.h>
#include <SPGrid/Core/SPGrid_Page_Map.h>

using namespace SPGrid;

typedef SPGrid_Mask<7, 7, 3> Mask64; // GridState<double,3>: 128 B
typedef SPGrid_Mask<6, 6, 3> Mask32; // GridState<float,3>: 64 B

static std::vector<char> read_all(const char* path)
{
    std::vector<char> buf;
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(2);
    }
    char tmp[1 << 16];
    size_t n;
    while ((n = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    fclose(f);
    return buf;
}

struct Out {
    FILE* f;
    template <class T>
    void put(const T& v) { fwrite(&v, sizeof(T), 1, f); }
    template <class T>
    void put(const std::vector<T>& v) { fwrite(v.data(), sizeof(T), v.size(), f); }
};

template <class M>
static void masks(Out& o)
{
    uint64_t x = M::xmask, y = M::ymask, z = M::zmask;
    o.put(x);
    o.put(y);
    o.put(z);
    int32_t bits[4] = { (int32_t)M::block_xbits, (int32_t)M::block_ybits, (int32_t)M::block_zbits, (int32_t)M::block_bits };
    for (int i = 0; i < 4; ++i) o.put(bits[i]);
}

template <class M>
static void offsets(const int32_t* c, size_t n, Out& o)
{
    for (size_t i = 0; i < n; ++i) {
        uint64_t off = M::Linear_Offset(c[3 * i], c[3 * i + 1], c[3 * i + 2]);
        o.put(off);
        std::array<int, 3> back = M::LinearToCoord(off);
        for (int d = 0; d < 3; ++d) o.put((int32_t)back[d]);
    }
}

template <class M>
static void packed(const uint64_t* ab, size_t n, Out& o)
{
    for (size_t i = 0; i < n; ++i) o.put((uint64_t)M::Packed_Add(ab[2 * i], ab[2 * i + 1]));
}

static inline int int_floor_f(float x)
{
    int i = (int)x;
    return i - (i > x);
}
static inline int int_floor_d(double x)
{
    int i = (int)x;
    return i - (i > x);
}

template <class M, class T>
static void bin(const double* xyz, int32_t P, double dx_in, Out& o)
{
    const int index_bits = 32 - M::block_bits;
    T dx = (T)dx_in;
    T one_over_dx = (T)1 / dx;
    std::vector<uint64_t> sorter(P), base(P);
    std::vector<int32_t> order(P);
    for (int32_t i = 0; i < P; ++i) {
        int b[3];
        for (int d = 0; d < 3; ++d) {
            T x = (T)xyz[3 * i + d];
            T xs = x * one_over_dx;
            T s = xs - (T)0.5;
            b[d] = sizeof(T) == 4 ? int_floor_f((float)s) : int_floor_d((double)s);
        }
        uint64_t off = M::Linear_Offset(b[0], b[1], b[2]);
        sorter[i] = ((off >> M::data_bits) << index_bits) + (uint64_t)i;
    }
    std::sort(sorter.begin(), sorter.end());
    std::vector<int32_t> groups;
    std::vector<uint64_t> block_offset;
    int last = 0;
    for (int32_t i = 0; i < P; ++i)
        if (i == P - 1 || (sorter[i] >> 32) != (sorter[i + 1] >> 32)) {
            groups.push_back(last);
            groups.push_back(i);
            block_offset.push_back(sorter[i] >> 32);
            last = i + 1;
        }
    SPGrid_Geometry<3> geom(4096, 4096, 4096, M::block_xbits, M::block_ybits, M::block_zbits);
    SPGrid_Page_Map<12> pm(geom);
    pm.Clear();
    for (int32_t i = 0; i < P; ++i) {
        order[i] = (int32_t)(sorter[i] & ((1ll << index_bits) - 1));
        uint64_t off = (sorter[i] >> index_bits) << M::data_bits;
        base[order[i]] = off;
        if (i == P - 1 || (sorter[i] >> 32) != (sorter[i + 1] >> 32)) {
            pm.Set_Page(off);
            int x = 1 << M::block_xbits, y = 1 << M::block_ybits, z = 1 << M::block_zbits;
            for (int a = 0; a < 2; ++a)
                for (int bb = 0; bb < 2; ++bb)
                    for (int c = 0; c < 2; ++c) pm.Set_Page(M::Packed_Add(off, M::Linear_Offset(x * a, y * bb, z * c)));
        }
    }
    pm.Update_Block_Offsets();
    auto blocks = pm.Get_Blocks();
    o.put(sorter);
    o.put(order);
    o.put(base);
    int64_t G = (int64_t)block_offset.size(), B = (int64_t)blocks.second;
    o.put(G);
    o.put(groups);
    o.put(block_offset);
    o.put(B);
    for (int64_t b = 0; b < B; ++b) o.put((uint64_t)blocks.first[b]);
}

int main(int argc, char** argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: %s masks|offsets|packed_add|bin in out\n", argv[0]);
        return 2;
    }
    std::string mode = argv[1];
    std::vector<char> in = read_all(argv[2]);
    Out o{ fopen(argv[3], "wb") };
    if (!o.f) {
        perror(argv[3]);
        return 2;
    }
    if (mode == "masks") {
        masks<Mask64>(o);
        masks<Mask32>(o);
    }
    else if (mode == "offsets") {
        size_t n = in.size() / 12;
        offsets<Mask64>(reinterpret_cast<const int32_t*>(in.data()), n, o);
        offsets<Mask32>(reinterpret_cast<const int32_t*>(in.data()), n, o);
    }
    else if (mode == "packed_add") {
        size_t n = in.size() / 16;
        packed<Mask64>(reinterpret_cast<const uint64_t*>(in.data()), n, o);
        packed<Mask32>(reinterpret_cast<const uint64_t*>(in.data()), n, o);
    }
    else if (mode == "bin") {
        int32_t l2s, P;
        double dx;
        memcpy(&l2s, in.data(), 4);
        memcpy(&P, in.data() + 4, 4);
        memcpy(&dx, in.data() + 8, 8);
        const double* xyz = reinterpret_cast<const double*>(in.data() + 16);
        if (l2s == 7)
            bin<Mask64, double>(xyz, P, dx, o);
        else
            bin<Mask32, float>(xyz, P, dx, o);
    }
    else {
        fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    }
    fclose(o.f);
    return 0;
}
