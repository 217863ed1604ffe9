// Machinery of the fused per-page transfer kernels (Hessian-vector product and
// the Newton update): one CTA per particle group (the particles whose base node
// lies in one SPGrid page), in two phases per chunk of the group's particles.
//
//  phase 1 (thread per particle): the particle's B-spline weights, a gradient
//          gathered from a staged 2x2x2-page window of a grid vector, the
//          per-particle 3x3 algebra, and a record in shared memory: the
//          particle's fractional offsets and the three rows of the 3x3 matrix
//          M_p whose product with grad w_ip is scattered.
//  phase 2 (thread per (cell, row)): the particles of one cell share their 27
//          stencil nodes, so a thread sums row r of M_p grad w_ip over the
//          cell's particles in 27 registers and adds them to the shared window
//          once.  Only occupied cells get threads.
//  flush:  the window [8][3][NPB] is added to the global block-dense vector
//          with one atomic per nonzero entry.
//
// The separable stencil sums use the per-axis index offsets of the 27 nodes
// (node (i,j,k) of a particle with base cell (lx,ly,lz) sits at window offset
// X_i + Y_j + Z_k), so the index arithmetic is one add per node.
#pragma once
#include "xfer.cuh"

namespace zmpm {

constexpr int FUSED_THREADS = 128;

// Quadratic B-spline weight and derivative of stencil offset i (0, 1, 2) for
// the fractional position d = x/dx - base (BSplines.h:55-81).
template <class T>
__device__ __forceinline__ void bspline_all(T d, T w[3], T dw[3])
{
    const T z0 = T(1.5) - d;
    const T d1 = d - T(1);
    const T z2 = d - T(0.5);
    w[0] = T(0.5) * z0 * z0;
    w[1] = T(0.75) - d1 * d1;
    w[2] = T(0.5) * z2 * z2;
    dw[0] = -z0;
    dw[1] = T(-2) * d1;
    dw[2] = z2;
}

// Packed FP32 pairs (sm_100 FFMA2 and friends: two FP32 operations per
// instruction, each rounded as the scalar one).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// bspline_all on a pair of fractional positions.
__device__ __forceinline__ void bspline_all2(float2 d, float2 w[3], float2 dw[3])
{
    const float2 z0 = add2(d, f2(-1.5f)); // d - 1.5 = -(1.5 - d)
    const float2 d1 = add2(d, f2(-1.0f));
    const float2 z2 = add2(d, f2(-0.5f));
    w[0] = mul2(mul2(z0, z0), f2(0.5f));
    w[1] = fma2(mul2(d1, f2(-1.0f)), d1, f2(0.75f));
    w[2] = mul2(mul2(z2, z2), f2(0.5f));
    dw[0] = z0;
    dw[1] = mul2(d1, f2(-2.0f));
    dw[2] = z2;
}

// Per-axis window offsets of the three stencil nodes along each axis, for a
// window of 8 pages of NPB nodes with `comp` scalars per node-page layout
// (node-major: offset counts nodes; component-major: the caller adds r * NPB).
template <class L>
struct StencilOffsets {
    int X[3], Y[3], Z[3]; // in units of nodes of a [8][NPB] window
    __device__ __forceinline__ StencilOffsets(int lx, int ly, int lz)
    {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int wx = lx + i, wy = ly + i, wz = lz + i;
            X[i] = ((wx >= L::BX) ? 4 * L::NPB : 0) + ((wx & (L::BX - 1)) << (L::YB + L::ZB));
            Y[i] = ((wy >= L::BY) ? 2 * L::NPB : 0) + ((wy & (L::BY - 1)) << L::ZB);
            Z[i] = ((wz >= L::BZ) ? L::NPB : 0) + (wz & (L::BZ - 1));
        }
    }
};
// The window's page t and element e of a node offset o = t * NPB + e.
template <int NPB>
__device__ __forceinline__ int window_scalar(int o, int comp, int ncomp)
{
    const int t = o / NPB, e = o - t * NPB;
    return (t * ncomp + comp) * NPB + e;
}

// Input windows of a grid vector: FP32 node-major float4 slabs ([B][NPB][4],
// the copy the Krylov solver keeps for the FP32 product) or FP64
// component-major slabs ([B][3][NPB], the solver's own vectors).
template <int NPB, class TX>
struct VecWindow;
template <int NPB>
struct VecWindow<NPB, float> {
    static constexpr int ELEMS = 8 * NPB * 4;
    static constexpr uint32_t SLAB = NPB * 4 * sizeof(float);
    static constexpr int64_t PAGE = NPB * 4; // elements per page in global memory
    __device__ __forceinline__ static void node(const float* w, int o, float v[3])
    {
        const float4 q = reinterpret_cast<const float4*>(w)[o];
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
    }
};
template <int NPB>
struct VecWindow<NPB, double> {
    static constexpr int ELEMS = 8 * NPB * 3;
    static constexpr uint32_t SLAB = NPB * 3 * sizeof(double);
    static constexpr int64_t PAGE = NPB * 3;
    __device__ __forceinline__ static void node(const double* w, int o, double v[3])
    {
        const int t = o / NPB, e = o - t * NPB;
        const double* p = w + t * 3 * NPB + e;
        v[0] = p[0];
        v[1] = p[NPB];
        v[2] = p[2 * NPB];
    }
};

// Stages the 8 page slabs of `vec` for the window; all threads call it.  The
// mbarrier is initialised once per kernel (by the caller, or here when
// `phase` < 0); a CTA that stages several windows in turn waits on the
// alternating phase parity.
template <int NPB, class TX>
__device__ __forceinline__ void stage_vec_window(TX* win, const TX* __restrict__ vec, const int32_t* nbr, uint64_t* bar, int32_t* flags,
    int phase = -1)
{
    using W = VecWindow<NPB, TX>;
    static_assert(W::SLAB % 16 == 0, "bulk copies move multiples of 16 bytes");
    if (threadIdx.x == 0) {
        if (phase < 0)
            mbar_init(bar, 1);
        else // a persistent kernel: order the vector's generic-proxy writes (other CTAs, before a grid barrier) before the bulk reads
            asm volatile("fence.proxy.async.global;" ::: "memory");
        mbar_expect_tx(bar, 8 * W::SLAB);
#pragma unroll
        for (int t = 0; t < 8; ++t) bulk_g2s(win + t * W::PAGE, vec + (int64_t)nbr[t] * W::PAGE, W::SLAB, bar);
    }
    __syncthreads();
    mbar_wait_bounded(bar, phase < 0 ? 0u : (uint32_t)(phase & 1), flags);
}

// G(r, c) = sum over the 27 stencil nodes of x_r(node) d_c w(node) * dx (the
// caller scales by 1/dx), by separable contraction along z, then y, then x.
template <class L, class T, class TX>
__device__ __forceinline__ void gather_gradient(const TX* win, const StencilOffsets<L>& so, const T w[3][3], const T dw[3][3], T G[9])
{
#pragma unroll
    for (int q = 0; q < 9; ++q) G[q] = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        T C[3] = { 0, 0, 0 }, D[3] = { 0, 0, 0 }, E[3] = { 0, 0, 0 };
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T A[3] = { 0, 0, 0 }, B[3] = { 0, 0, 0 };
            const int oij = so.X[i] + so.Y[j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                TX xv[3];
                VecWindow<L::NPB, TX>::node(win, oij + so.Z[k], xv);
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    A[r] += w[2][k] * (T)xv[r];
                    B[r] += dw[2][k] * (T)xv[r];
                }
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                C[r] += w[1][j] * A[r];
                D[r] += dw[1][j] * A[r];
                E[r] += w[1][j] * B[r];
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            G[3 * r + 0] += dw[0][i] * C[r];
            G[3 * r + 1] += w[0][i] * D[r];
            G[3 * r + 2] += w[0][i] * E[r];
        }
    }
}

// gather_gradient for an FP32 node-major window: components 0 and 1 of each
// node (adjacent in the float4 load) accumulate as one packed pair.
template <class L>
__device__ __forceinline__ void gather_gradient_f32(const float* win, const StencilOffsets<L>& so, const float w[3][3], const float dw[3][3],
    float G[9])
{
    const float4* win4 = reinterpret_cast<const float4*>(win);
    float2 G01[3] = { f2(0.f), f2(0.f), f2(0.f) };
    float G2[3] = { 0.f, 0.f, 0.f };
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float2 C01 = f2(0.f), D01 = f2(0.f), E01 = f2(0.f);
        float C2 = 0.f, D2 = 0.f, E2 = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float2 A01 = f2(0.f), B01 = f2(0.f);
            float A2 = 0.f, B2 = 0.f;
            const int oij = so.X[i] + so.Y[j];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float4 q = win4[oij + so.Z[k]];
                const float2 x01 = f2(q.x, q.y);
                A01 = fma2(x01, f2(w[2][k]), A01);
                B01 = fma2(x01, f2(dw[2][k]), B01);
                A2 = fmaf(q.z, w[2][k], A2);
                B2 = fmaf(q.z, dw[2][k], B2);
            }
            C01 = fma2(A01, f2(w[1][j]), C01);
            D01 = fma2(A01, f2(dw[1][j]), D01);
            E01 = fma2(B01, f2(w[1][j]), E01);
            C2 = fmaf(A2, w[1][j], C2);
            D2 = fmaf(A2, dw[1][j], D2);
            E2 = fmaf(B2, w[1][j], E2);
        }
        G01[0] = fma2(C01, f2(dw[0][i]), G01[0]);
        G01[1] = fma2(D01, f2(w[0][i]), G01[1]);
        G01[2] = fma2(E01, f2(w[0][i]), G01[2]);
        G2[0] = fmaf(C2, dw[0][i], G2[0]);
        G2[1] = fmaf(D2, w[0][i], G2[1]);
        G2[2] = fmaf(E2, w[0][i], G2[2]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        G[c] = G01[c].x;
        G[3 + c] = G01[c].y;
        G[6 + c] = G2[c];
    }
}

// Shared state of a fused kernel: the accumulation window, the particle
// records of the current chunk as 12 arrays of CH values (fractions 0-2, then
// row r of the scattered matrix at 3 + 3 r .. 5 + 3 r; particle-minor, so a
// warp's threads of phase 1 write consecutive words), the cell layout of the
// group and its occupied cells.
constexpr int REC_FIELDS = 12;
// stride of one record field: odd, so the rows r of one particle (fields
// 3 + 3 r + c) fall in different shared-memory banks
template <int CH>
constexpr int rec_stride() { return CH + 1; }
// NF record fields per particle, NC scattered components per node
template <class L, class T, int CH, int NF = REC_FIELDS, int NC = 3>
struct ScatterSmem {
    static constexpr int FS = rec_stride<CH>();
    __align__(16) T acc[8 * NC * L::NPB];
    __align__(16) T rec[NF * FS];
    CellLayout<L> cl;
    int32_t occ[L::NPB];
    int32_t nocc;
    int32_t nbr[8];
};

// The group's occupied cells, in cell order (after build_cell_layout).
template <class SM>
__device__ __forceinline__ void list_occupied(SM& sm)
{
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int base = 0;
#pragma unroll
        for (int c = 0; c < (int)(sizeof(sm.occ) / sizeof(sm.occ[0])); c += 32) {
            const bool on = sm.cl.cnt[c + lane] > 0;
            const unsigned m = __ballot_sync(0xffffffffu, on);
            if (on) sm.occ[base + __popc(m & ((1u << lane) - 1u))] = c + lane;
            base += __popc(m);
        }
        if (lane == 0) sm.nocc = base;
    }
}

// Phase 2 for the chunk of group particles [c0, c1) (group-relative): thread
// item (row r, occupied cell) adds sum_p row_r(M_p) . grad w_ip * dx to the
// window for the cell's particles in the chunk (the rows already carry 1/dx).
// FP32 takes the cell's particles two at a time as packed pairs.
template <class L, class T, int CH>
__device__ __forceinline__ void scatter_rows(ScatterSmem<L, T, CH>& sm, int c0, int c1)
{
    constexpr int NPB = L::NPB;
    // items row-major: the threads of a warp hold consecutive cells of one row,
    // so their window atomics fall in distinct banks
    const int nocc = sm.nocc, items = 3 * nocc;
    for (int q = threadIdx.x; q < items; q += blockDim.x) {
        const int r = q >= nocc ? (q >= 2 * nocc ? 2 : 1) : 0, cidx = q - r * nocc;
        const int ce = sm.occ[cidx];
        const int st = sm.cl.start[ce];
        const int p0 = (st > c0 ? st : c0) - c0;
        const int e1 = st + sm.cl.cnt[ce];
        const int p1 = (e1 < c1 ? e1 : c1) - c0;
        if (p0 >= p1) continue;
        constexpr int FS = ScatterSmem<L, T, CH>::FS;
        const T* fr = sm.rec;
        const T* rrow = sm.rec + (3 + 3 * r) * FS;
        T a[27];
        if constexpr (sizeof(T) == 4) {
            float2 a2[27];
#pragma unroll
            for (int n = 0; n < 27; ++n) a2[n] = f2(0.f);
            for (int p = p0; p < p1; p += 2) {
                // an odd last particle pairs with itself at zero weight
                const int pq = p + 1 < p1 ? p + 1 : p;
                const float sq = p + 1 < p1 ? 1.f : 0.f;
                float2 w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all2(f2(fr[d * FS + p], fr[d * FS + pq]), w[d], dw[d]);
                const float2 s0 = f2(rrow[p], sq * rrow[pq]);
                const float2 s1 = f2(rrow[FS + p], sq * rrow[FS + pq]);
                const float2 s2 = f2(rrow[2 * FS + p], sq * rrow[2 * FS + pq]);
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float2 u = mul2(s0, mul2(w[1][j], w[2][k]));
                        const float2 v = fma2(s2, mul2(w[1][j], dw[2][k]), mul2(s1, mul2(dw[1][j], w[2][k])));
#pragma unroll
                        for (int i = 0; i < 3; ++i) a2[9 * i + 3 * j + k] = fma2(w[0][i], v, fma2(dw[0][i], u, a2[9 * i + 3 * j + k]));
                    }
            }
#pragma unroll
            for (int n = 0; n < 27; ++n) a[n] = a2[n].x + a2[n].y;
        }
        else {
#pragma unroll
            for (int n = 0; n < 27; ++n) a[n] = T(0);
            for (int p = p0; p < p1; ++p) {
                T w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all(fr[d * FS + p], w[d], dw[d]);
                const T s0 = rrow[p], s1 = rrow[FS + p], s2 = rrow[2 * FS + p];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const T u = s0 * (w[1][j] * w[2][k]);
                        const T v = s1 * (dw[1][j] * w[2][k]) + s2 * (w[1][j] * dw[2][k]);
#pragma unroll
                        for (int i = 0; i < 3; ++i) a[9 * i + 3 * j + k] += dw[0][i] * u + w[0][i] * v;
                    }
            }
        }
        const int lx = ce >> (L::YB + L::ZB), ly = (ce >> L::ZB) & (L::BY - 1), lz = ce & (L::BZ - 1);
        const StencilOffsets<L> so(lx, ly, lz);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) atomicAdd(sm.acc + window_scalar<NPB>(so.X[i] + so.Y[j] + so.Z[k], r, 3), a[9 * i + 3 * j + k]);
    }
}

// Phase 2 of the APIC P2G (particlesToGridHelper, MpmSimulationBase.cpp:563-
// 608) for the chunk [c0, c1): item (component c, occupied cell) adds, for the
// cell's particles, w_ip m_p (c = 0) or w_ip (q_r + a_r i + b_r j + c_r k)
// (c = r + 1, the momentum m (v + C (x_i - x_p)) written affinely in the node
// offset (i, j, k)) to the window.  Records: fractions at fields 0-2, the mass
// at 3, row r's (q, a, b, c) at 4 + 4 r .. 7 + 4 r.  FP32 takes the cell's
// particles two at a time as packed pairs.
template <class L, class T, int CH>
__device__ __forceinline__ void scatter_p2g(ScatterSmem<L, T, CH, 16, 4>& sm, int c0, int c1)
{
    constexpr int NPB = L::NPB;
    constexpr int FS = ScatterSmem<L, T, CH, 16, 4>::FS;
    const int nocc = sm.nocc, items = 4 * nocc;
    for (int q = threadIdx.x; q < items; q += blockDim.x) {
        const int c = q / nocc, cidx = q - c * nocc;
        const int ce = sm.occ[cidx];
        const int st = sm.cl.start[ce];
        const int p0 = (st > c0 ? st : c0) - c0;
        const int e1 = st + sm.cl.cnt[ce];
        const int p1 = (e1 < c1 ? e1 : c1) - c0;
        if (p0 >= p1) continue;
        const T* fr = sm.rec;
        const T* row = sm.rec + (c == 0 ? 3 : 4 * c) * FS; // mass, or (q, a, b, c) of row c - 1
        T a[27];
        if constexpr (sizeof(T) == 4) {
            float2 a2[27];
#pragma unroll
            for (int n = 0; n < 27; ++n) a2[n] = f2(0.f);
            for (int p = p0; p < p1; p += 2) {
                const int pq = p + 1 < p1 ? p + 1 : p;
                const float sq = p + 1 < p1 ? 1.f : 0.f;
                float2 w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all2(f2(fr[d * FS + p], fr[d * FS + pq]), w[d], dw[d]);
                const float2 q0 = f2(row[p], sq * row[pq]);
                float2 ax = f2(0.f), by = f2(0.f), cz = f2(0.f);
                if (c != 0) {
                    ax = f2(row[FS + p], sq * row[FS + pq]);
                    by = f2(row[2 * FS + p], sq * row[2 * FS + pq]);
                    cz = f2(row[3 * FS + p], sq * row[3 * FS + pq]);
                }
                const float2 wx1 = w[0][1], wx2 = mul2(w[0][2], f2(2.f)); // i w_i for i = 1, 2
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float2 t = mul2(w[1][j], w[2][k]);
                        // (q + b j + c k) t and a t
                        float2 l = q0;
                        if (j) l = fma2(by, f2((float)j), l);
                        if (k) l = fma2(cz, f2((float)k), l);
                        const float2 u = mul2(l, t), v = mul2(ax, t);
                        a2[3 * j + k] = fma2(w[0][0], u, a2[3 * j + k]);
                        a2[9 + 3 * j + k] = fma2(w[0][1], u, fma2(wx1, v, a2[9 + 3 * j + k]));
                        a2[18 + 3 * j + k] = fma2(w[0][2], u, fma2(wx2, v, a2[18 + 3 * j + k]));
                    }
            }
#pragma unroll
            for (int n = 0; n < 27; ++n) a[n] = a2[n].x + a2[n].y;
        }
        else {
#pragma unroll
            for (int n = 0; n < 27; ++n) a[n] = T(0);
            for (int p = p0; p < p1; ++p) {
                T w[3][3], dw[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d) bspline_all(fr[d * FS + p], w[d], dw[d]);
                const T q0 = row[p];
                const T ax = c ? row[FS + p] : T(0), by = c ? row[2 * FS + p] : T(0), cz = c ? row[3 * FS + p] : T(0);
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const T t = w[1][j] * w[2][k];
                        const T u = (q0 + by * T(j) + cz * T(k)) * t, v = ax * t;
#pragma unroll
                        for (int i = 0; i < 3; ++i) a[9 * i + 3 * j + k] += w[0][i] * u + (T(i) * w[0][i]) * v;
                    }
            }
        }
        const int lx = ce >> (L::YB + L::ZB), ly = (ce >> L::ZB) & (L::BY - 1), lz = ce & (L::BZ - 1);
        const StencilOffsets<L> so(lx, ly, lz);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) atomicAdd(sm.acc + window_scalar<NPB>(so.X[i] + so.Y[j] + so.Z[k], c, 4), a[9 * i + 3 * j + k]);
    }
}

} // namespace zmpm
