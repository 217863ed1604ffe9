// C ABI of the library (include/zmpm.h): context lifecycle, scene plugins,
// state I/O, the substep and the test hooks.  No exception crosses the
// boundary; every entry point returns a zmpm_status_code.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <limits>
#include <new>

#include "internal.cuh"
#include "models.cuh"

using namespace zmpm;

namespace zmpm {
int launch_p2g(Ctx* ctx);
}

namespace {

// Device -> host copy ordered after the context's stream (whose work produced
// the data), complete on return.  The library's stream does not synchronise
// with the legacy default stream, so plain cudaMemcpy would not order it.
cudaError_t d2h_sync(Ctx* ctx, void* dst, const void* src, size_t bytes)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(ctx->stream);
}

int64_t bitlen(uint64_t v)
{
    int64_t n = 0;
    while (v) {
        ++n;
        v >>= 1;
    }
    return n;
}

template <class L>
int64_t key_bits_for(const int pages[3])
{
    uint64_t hi = (L::page_index(pages[0] - 1, pages[1] - 1, pages[2] - 1) << L::BLOCK_BITS) | (uint64_t)(L::NPB - 1);
    return bitlen(hi);
}

} // namespace

namespace zmpm {

// Puts the host scene on the device (first use) with slot = particle index.
int upload(Ctx* ctx)
{
    if (ctx->uploaded) return ZMPM_OK;
    const int64_t P = ctx->P;
    const int64_t cap = std::max<int64_t>(P, 1);
    ctx->Pcap = cap;
    const size_t TH = ctx->mixed ? sizeof(float) : sizeof(double);
    ZMPM_CUDA(ctx->pd.ensure(PD_FIELDS * cap * sizeof(double)));
    ZMPM_CUDA(ctx->pd_alt.ensure(PD_FIELDS * cap * sizeof(double)));
    ZMPM_CUDA(ctx->pi.ensure(PI_FIELDS * cap * sizeof(int32_t)));
    ZMPM_CUDA(ctx->pi_alt.ensure(PI_FIELDS * cap * sizeof(int32_t)));
    ZMPM_CUDA(ctx->slot_of_id.ensure(cap * sizeof(int32_t)));
    ZMPM_CUDA(ctx->base_by_id.ensure(cap * sizeof(short4)));
    ZMPM_CUDA(ctx->base.ensure(cap * sizeof(short4)));
    ZMPM_CUDA(ctx->scratch.ensure(NS * cap * TH));
    ZMPM_CUDA(ctx->frac.ensure(3 * cap * TH));
    ZMPM_CUDA(ctx->stress.ensure(9 * cap * sizeof(double)));
    std::vector<double> hpd((size_t)PD_FIELDS * cap, 0.0);
    std::vector<int32_t> hpi((size_t)PI_FIELDS * cap, 0), sid(cap);
    for (int64_t i = 0; i < P; ++i) {
        for (int d = 0; d < 3; ++d) {
            hpd[(PD_X + d) * cap + i] = ctx->hx[3 * i + d];
            hpd[(PD_V + d) * cap + i] = ctx->hv[3 * i + d];
        }
        for (int q = 0; q < 9; ++q) {
            hpd[(PD_C + q) * cap + i] = ctx->hC[9 * i + q];
            hpd[(PD_F + q) * cap + i] = ctx->hF[9 * i + q];
        }
        hpd[PD_M * cap + i] = ctx->hm[i];
        hpd[PD_VOL * cap + i] = ctx->hvol[i];
        hpd[PD_MU * cap + i] = ctx->hmu[i];
        hpd[PD_LAM * cap + i] = ctx->hlam[i];
        hpd[PD_KAPPA * cap + i] = ctx->hkappa[i];
        hpd[PD_G * cap + i] = ctx->hg[i];
        hpd[PD_YS * cap + i] = ctx->hys[i];
        hpd[PD_XI * cap + i] = ctx->hxi[i];
        hpd[PD_FS * cap + i] = ctx->hfs[i];
        for (int d = 0; d < 3; ++d) hpd[(PD_CRACK + d) * cap + i] = ctx->hcrack[3 * i + d];
        hpd[PD_PF_C * cap + i] = ctx->hpfc[i];
        hpd[PD_PF_K * cap + i] = ctx->hpfk[i];
        hpd[PD_SIGMA_F * cap + i] = ctx->hsigf[i];
        hpd[PD_LOGJP * cap + i] = ctx->hlogjp[i];
        hpd[PD_PF_H * cap + i] = ctx->hpfH[i];
        hpd[PD_PF_L0 * cap + i] = ctx->hpfl0[i];
        hpd[PD_PF_ISC * cap + i] = ctx->hpfisc[i];
        hpd[PD_PF_FP * cap + i] = ctx->hpffp[i];
        hpd[PD_PF_HMAX * cap + i] = ctx->hpfhmax[i];
        hpd[PD_PF_VOL * cap + i] = ctx->hpfvol[i];
        hpd[PD_PF_ALLOW * cap + i] = ctx->hpfallow[i];
        hpi[PI_DAMAGE * cap + i] = ctx->hdamage[i];
        hpi[PI_KIND * cap + i] = ctx->hkind[i];
        hpi[PI_PKIND * cap + i] = ctx->hpkind[i];
        hpi[PI_BROKEN * cap + i] = ctx->hbroken[i];
        hpi[PI_ID * cap + i] = (int32_t)i;
        hpi[PI_VISCO * cap + i] = ctx->hvisco[i];
        for (int q = 0; q < 9; ++q) hpd[(PD_FE + q) * cap + i] = ctx->hFe[9 * i + q];
        hpd[PD_VMU * cap + i] = ctx->hvmu[i];
        hpd[PD_VLAM * cap + i] = ctx->hvlam[i];
        hpd[PD_VD * cap + i] = ctx->hvd[i];
        hpd[PD_VV * cap + i] = ctx->hvv[i];
        for (int q = 0; q < 18; ++q) hpd[(PD_Y + q) * cap + i] = ctx->hy[18 * i + q];
        for (int k = 0; k < 2; ++k) hpd[(PD_OMEGA + k) * cap + i] = ctx->homega[2 * i + k];
        for (int d = 0; d < 3; ++d) hpd[(PD_LASTDV + d) * cap + i] = ctx->hlastdv[3 * i + d];
        sid[i] = (int32_t)i;
    }
    ZMPM_CUDA(cudaMemcpyAsync(ctx->pd.p, hpd.data(), hpd.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->pi.p, hpi.data(), hpi.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->slot_of_id.p, sid.data(), sid.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    ctx->has_damage = false;
    ctx->has_visco = false;
    ctx->all_models = true;
    ctx->has_pf = false;
    ctx->all_pf = P > 0;
    for (int64_t i = 0; i < P; ++i) {
        ctx->has_pf |= ctx->hdamage[i] == ZMPM_DAMAGE_PHASE_FIELD;
        ctx->all_pf &= ctx->hdamage[i] == ZMPM_DAMAGE_PHASE_FIELD;
        ctx->has_damage |= ctx->hdamage[i] == ZMPM_DAMAGE_RANKINE || ctx->hdamage[i] == ZMPM_DAMAGE_RANKINE_REFERENCE;
        ctx->has_visco |= ctx->hvisco[i] != 0;
        ctx->all_models &= ctx->hkind[i] != ZMPM_MODEL_NONE;
    }
    ctx->uploaded = true;
    ctx->binned = false;
    ctx->implicit_ready = false;
    return ZMPM_OK;
}

// Pulls the device state back into the host scene arrays (particle order).
int download(Ctx* ctx)
{
    if (!ctx->uploaded) return ZMPM_OK;
    const int64_t P = ctx->P, cap = ctx->Pcap;
    // fields past pd_active were not moved by the permutation: the host copy stays
    const bool ext = ctx->pd_active == PD_FIELDS, pfx = ctx->pd_active >= PD_PF_END;
    std::vector<double> hpd((size_t)ctx->pd_active * cap);
    std::vector<int32_t> hpi((size_t)PI_FIELDS * cap);
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ZMPM_CUDA(d2h_sync(ctx, hpd.data(), ctx->pd.p, hpd.size() * sizeof(double)));
    ZMPM_CUDA(d2h_sync(ctx, hpi.data(), ctx->pi.p, hpi.size() * sizeof(int32_t)));
    for (int64_t s = 0; s < P; ++s) {
        const int64_t i = hpi[PI_ID * cap + s];
        for (int d = 0; d < 3; ++d) {
            ctx->hx[3 * i + d] = hpd[(PD_X + d) * cap + s];
            ctx->hv[3 * i + d] = hpd[(PD_V + d) * cap + s];
            ctx->hcrack[3 * i + d] = hpd[(PD_CRACK + d) * cap + s];
        }
        for (int q = 0; q < 9; ++q) {
            ctx->hC[9 * i + q] = hpd[(PD_C + q) * cap + s];
            ctx->hF[9 * i + q] = hpd[(PD_F + q) * cap + s];
        }
        ctx->hm[i] = hpd[PD_M * cap + s];
        ctx->hvol[i] = hpd[PD_VOL * cap + s];
        ctx->hmu[i] = hpd[PD_MU * cap + s];
        ctx->hlam[i] = hpd[PD_LAM * cap + s];
        ctx->hkappa[i] = hpd[PD_KAPPA * cap + s];
        ctx->hg[i] = hpd[PD_G * cap + s];
        ctx->hys[i] = hpd[PD_YS * cap + s];
        ctx->hxi[i] = hpd[PD_XI * cap + s];
        ctx->hfs[i] = hpd[PD_FS * cap + s];
        ctx->hpfc[i] = hpd[PD_PF_C * cap + s];
        ctx->hpfk[i] = hpd[PD_PF_K * cap + s];
        ctx->hsigf[i] = hpd[PD_SIGMA_F * cap + s];
        ctx->hlogjp[i] = hpd[PD_LOGJP * cap + s];
        ctx->hdamage[i] = (uint8_t)hpi[PI_DAMAGE * cap + s];
        ctx->hkind[i] = (uint8_t)hpi[PI_KIND * cap + s];
        ctx->hpkind[i] = (uint8_t)hpi[PI_PKIND * cap + s];
        ctx->hbroken[i] = hpi[PI_BROKEN * cap + s];
        ctx->hvisco[i] = (uint8_t)hpi[PI_VISCO * cap + s];
        if (pfx) {
            ctx->hpfH[i] = hpd[PD_PF_H * cap + s];
            ctx->hpfl0[i] = hpd[PD_PF_L0 * cap + s];
            ctx->hpfisc[i] = hpd[PD_PF_ISC * cap + s];
            ctx->hpffp[i] = hpd[PD_PF_FP * cap + s];
            ctx->hpfhmax[i] = hpd[PD_PF_HMAX * cap + s];
            ctx->hpfvol[i] = hpd[PD_PF_VOL * cap + s];
            ctx->hpfallow[i] = hpd[PD_PF_ALLOW * cap + s];
        }
        if (!ext) continue;
        for (int q = 0; q < 9; ++q) ctx->hFe[9 * i + q] = hpd[(PD_FE + q) * cap + s];
        ctx->hvmu[i] = hpd[PD_VMU * cap + s];
        ctx->hvlam[i] = hpd[PD_VLAM * cap + s];
        ctx->hvd[i] = hpd[PD_VD * cap + s];
        ctx->hvv[i] = hpd[PD_VV * cap + s];
        for (int q = 0; q < 18; ++q) ctx->hy[18 * i + q] = hpd[(PD_Y + q) * cap + s];
        for (int k = 0; k < 2; ++k) ctx->homega[2 * i + k] = hpd[(PD_OMEGA + k) * cap + s];
        for (int d = 0; d < 3; ++d) ctx->hlastdv[3 * i + d] = hpd[(PD_LASTDV + d) * cap + s];
    }
    return ZMPM_OK;
}

// Host scene edits go through the host arrays: pull, edit, mark for upload.
int begin_edit(Ctx* ctx)
{
    int rc = download(ctx);
    if (rc) return rc;
    ctx->uploaded = false;
    ctx->binned = false;
    ctx->implicit_ready = false;
    ctx->phase = 0; // an edit ends a substep split into phases
    return ZMPM_OK;
}

} // namespace zmpm

namespace {

void quat_to_R(const double q[4], double R[9])
{
    double w = q[0], x = q[1], y = q[2], z = q[3];
    double n = std::sqrt(w * w + x * x + y * y + z * z);
    if (n == 0) {
        w = 1;
        x = y = z = 0;
        n = 1;
    }
    w /= n;
    x /= n;
    y /= n;
    z /= n;
    R[0] = 1 - 2 * (y * y + z * z);
    R[1] = 2 * (x * y - w * z);
    R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);
    R[4] = 1 - 2 * (x * x + z * z);
    R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);
    R[7] = 2 * (y * z + w * x);
    R[8] = 1 - 2 * (x * x + y * y);
}

// getNumNodes numbering (MpmGrid.h:123-136) of the block-dense grid:
// idx[n] = rank among nodes with m != 0 in page-map then element order.
int node_indices(Ctx* ctx, std::vector<int64_t>& idx, std::vector<double>& hm)
{
    const int64_t nn = ctx->B * ctx->npb();
    hm.resize(nn);
    idx.assign(nn, -1);
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (nn) ZMPM_CUDA(d2h_sync(ctx, hm.data(), ctx->gm.p, nn * sizeof(double)));
    int64_t c = 0;
    for (int64_t n = 0; n < nn; ++n)
        if (hm[n] != 0) idx[n] = c++;
    ctx->N = c;
    return ZMPM_OK;
}

// Particle-index-ordered host arrays <-> slot-ordered device fields, converted
// on the device (one staging copy per array).
__global__ void k_fields_from_host(const double* __restrict__ in, int ncomp, int64_t P, int64_t cap, const int32_t* __restrict__ slot_of_id,
    double* __restrict__ field)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int64_t s = slot_of_id[i];
    for (int c = 0; c < ncomp; ++c) field[c * cap + s] = in[i * ncomp + c];
}
__global__ void k_fields_to_host(double* __restrict__ out, int ncomp, int64_t P, int64_t cap, const int32_t* __restrict__ slot_of_id,
    const double* __restrict__ field)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    const int64_t s = slot_of_id[i];
    for (int c = 0; c < ncomp; ++c) out[i * ncomp + c] = field[c * cap + s];
}

int device_set(Ctx* ctx, const double* x, const double* v, const double* C, const double* F)
{
    const int64_t P = ctx->P, cap = ctx->Pcap;
    if (P == 0) return ZMPM_OK;
    ZMPM_CUDA(ctx->stage.ensure(24 * P * sizeof(double)));
    double* st = ctx->stage.as<double>();
    const double* src[4] = { x, v, C, F };
    const int nc[4] = { 3, 3, 9, 9 };
    const int fld[4] = { PD_X, PD_V, PD_C, PD_F };
    int64_t off = 0;
    for (int a = 0; a < 4; ++a) {
        if (!src[a]) continue;
        ZMPM_CUDA(cudaMemcpyAsync(st + off, src[a], nc[a] * P * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        k_fields_from_host<<<(unsigned)((P + 255) / 256), 256, 0, ctx->stream>>>(st + off, nc[a], P, cap, ctx->slot_of_id.as<int32_t>(),
            ctx->pdf(fld[a]));
        ++g_kernel_launches;
        off += nc[a] * P;
    }
    ZMPM_CUDA(cudaGetLastError());
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->binned = false;
    ctx->implicit_ready = false;
    return ZMPM_OK;
}

int device_get(Ctx* ctx, double* x, double* v, double* C, double* F)
{
    const int64_t P = ctx->P, cap = ctx->Pcap;
    if (P == 0) return ZMPM_OK;
    ZMPM_CUDA(ctx->stage.ensure(24 * P * sizeof(double)));
    double* st = ctx->stage.as<double>();
    double* dst[4] = { x, v, C, F };
    const int nc[4] = { 3, 3, 9, 9 };
    const int fld[4] = { PD_X, PD_V, PD_C, PD_F };
    int64_t off = 0;
    for (int a = 0; a < 4; ++a) {
        if (!dst[a]) continue;
        k_fields_to_host<<<(unsigned)((P + 255) / 256), 256, 0, ctx->stream>>>(st + off, nc[a], P, cap, ctx->slot_of_id.as<int32_t>(),
            ctx->pdf(fld[a]));
        ++g_kernel_launches;
        ZMPM_CUDA(cudaMemcpyAsync(dst[a], st + off, nc[a] * P * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        off += nc[a] * P;
    }
    ZMPM_CUDA(cudaGetLastError());
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    return ZMPM_OK;
}

int check_ready(Ctx* ctx)
{
    if (!ctx->implicit_ready) {
        ctx->err = "call zmpm_begin_implicit first";
        return ZMPM_NOT_READY;
    }
    return ZMPM_OK;
}

} // namespace

namespace zmpm {

int upload_colliders(Ctx* ctx, double time, int slot)
{
    const int n = (int)ctx->colliders.size();
    if (n == 0) return ZMPM_OK;
    std::vector<DevCollider> h(n);
    for (int i = 0; i < n; ++i) {
        const zmpm_collider& c = ctx->colliders[i];
        DevCollider& d = h[i];
        d.shape = c.shape;
        d.type = c.type;
        d.friction = c.friction;
        for (int k = 0; k < 3; ++k) {
            d.a[k] = c.a[k];
            d.b[k] = c.b[k];
            d.omega[k] = c.angular_velocity[k];
            d.t[k] = c.translation[k] + time * c.translation_velocity[k];
            d.dtdt[k] = c.translation_velocity[k];
        }
        d.radius = c.radius;
        quat_to_R(c.rotation, d.R);
        d.s = c.scale + time * c.scale_velocity;
        d.dsdt = c.scale_velocity;
    }
    ZMPM_CUDA(cudaMemcpyAsync(ctx->dcolliders.as<DevCollider>() + (size_t)slot * MAX_COLLIDERS, h.data(), n * sizeof(DevCollider),
        cudaMemcpyHostToDevice, ctx->stream));
    return ZMPM_OK;
}

} // namespace zmpm

extern "C" {

const char* zmpm_status_string(int s)
{
    switch (s) {
    case ZMPM_OK: return "ok";
    case ZMPM_CFL_VIOLATION: return "a particle moved more than one cell (CFL violation)";
    case ZMPM_NEWTON_NOT_CONVERGED: return "Newton did not converge";
    case ZMPM_NAN_DETECTED: return "NaN detected";
    case ZMPM_TIMEOUT: return "a bounded device wait gave up";
    case ZMPM_BAD_ARG: return "bad argument";
    case ZMPM_OUT_OF_GRID: return "particle outside the grid";
    case ZMPM_CUDA_ERROR: return "CUDA error";
    case ZMPM_NO_MEMORY: return "out of memory";
    case ZMPM_NOT_READY: return "not ready";
    case ZMPM_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

void zmpm_default_solver(zmpm_solver* s, int32_t linear_solver, int32_t precision)
{
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->linear_solver = linear_solver;
    s->newton_max_iterations = 3;
    s->newton_tolerance = 1e-5;
    s->krylov_max_iterations = 20;
    s->linear_solve_tolerance_scale = 1;
    s->integrator = ZMPM_NEWTON;
    s->admm_iterations = 100; // AdmmSimulationFoam.h:65-70
    s->admm_rho_scale = 0.5;
    s->admm_local_tolerance = 1e-8;
    s->admm_global_tolerance = 1e-6;
    s->admm_global_max_iterations = 10000;
    s->trial_collision = 1; // useTrialCollision, MpmSimulationBase.cpp:61
    if (linear_solver == ZMPM_MINRES)
        s->krylov_tolerance = 1;
    else
        s->krylov_tolerance = 16 * (precision == ZMPM_FP64 ? 2.220446049250313e-16 : 1.1920928955078125e-07);
}

int zmpm_create(const zmpm_config* cfg, zmpm_ctx** out)
{
    if (!cfg || !out || !(cfg->dx > 0) || cfg->grid_log2 < 4 || cfg->grid_log2 > 12) return ZMPM_BAD_ARG;
    if (cfg->precision != ZMPM_FP64 && cfg->precision != ZMPM_MIXED) return ZMPM_BAD_ARG;
    zmpm_ctx* ctx = new (std::nothrow) zmpm_ctx();
    if (!ctx) return ZMPM_NO_MEMORY;
    *out = nullptr;
    ctx->cfg = *cfg;
    ctx->mixed = cfg->precision == ZMPM_MIXED;
    ctx->layout = cfg->layout == ZMPM_LAYOUT_AUTO ? (ctx->mixed ? 2 : 1) : cfg->layout;
    if (ctx->layout != 1 && ctx->layout != 2) {
        delete ctx;
        return ZMPM_BAD_ARG;
    }
    ctx->device = cfg->device;
    ctx->grid_log2 = cfg->grid_log2;
    auto fail = [&](cudaError_t e) {
        ctx->err = cudaGetErrorString(e);
        delete ctx;
        return ZMPM_CUDA_ERROR;
    };
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) return fail(e);
    const int n = 1 << ctx->grid_log2;
    if (ctx->layout == 1) {
        ctx->pages[0] = n / Layout244::BX;
        ctx->pages[1] = n / Layout244::BY;
        ctx->pages[2] = n / Layout244::BZ;
        ctx->key_bits = (int)key_bits_for<Layout244>(ctx->pages);
    }
    else {
        ctx->pages[0] = n / Layout444::BX;
        ctx->pages[1] = n / Layout444::BY;
        ctx->pages[2] = n / Layout444::BZ;
        ctx->key_bits = (int)key_bits_for<Layout444>(ctx->pages);
    }
    ctx->table_size = (int64_t)ctx->pages[0] * ctx->pages[1] * ctx->pages[2];
    if ((e = ctx->page_first.ensure(ctx->table_size * sizeof(int32_t))) != cudaSuccess) return fail(e);
    if ((e = ctx->page_block.ensure(ctx->table_size * sizeof(int32_t))) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(ctx->page_first.p, 0x7f, ctx->table_size * sizeof(int32_t))) != cudaSuccess) return fail(e);
    if ((e = ctx->counters.ensure(sizeof(DevCounters))) != cudaSuccess) return fail(e);
    if ((e = ctx->scal.ensure(sizeof(SolverScalars))) != cudaSuccess) return fail(e);
    if ((e = ctx->gsync.ensure(sizeof(GridSync))) != cudaSuccess) return fail(e);
    if ((e = ctx->red.ensure(RED_N * RED_MAX_CTAS * sizeof(double))) != cudaSuccess) return fail(e);
    // two collider states: at t, and at t + dt for the explicit substep's trial collision
    if ((e = ctx->dcolliders.ensure(2 * MAX_COLLIDERS * sizeof(DevCollider))) != cudaSuccess) return fail(e);
    cudaMemset(ctx->counters.p, 0, sizeof(DevCounters));
    cudaMemset(ctx->scal.p, 0, sizeof(SolverScalars));
    // the context's stream does not order itself after the legacy stream's memsets
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e);
    *out = ctx;
    return ZMPM_OK;
}

int zmpm_destroy(zmpm_ctx* ctx)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    DBuf* bufs[] = { &ctx->pd, &ctx->pd_alt, &ctx->pi, &ctx->pi_alt, &ctx->slot_of_id, &ctx->base_by_id, &ctx->base, &ctx->Fn, &ctx->scratch,
        &ctx->frac, &ctx->stress, &ctx->keys, &ctx->keys_alt, &ctx->flags_i32, &ctx->scan_i32, &ctx->scan_scr, &ctx->radix_scr, &ctx->group_start,
        &ctx->group_page, &ctx->group_nbr, &ctx->emit_flag, &ctx->emit_scan, &ctx->page_first, &ctx->page_block, &ctx->block_page,
        &ctx->block_index, &ctx->gm, &ctx->gmv, &ctx->vn, &ctx->dv, &ctx->vstar, &ctx->facc, &ctx->res, &ctx->proj, &ctx->collided,
        &ctx->node_idx, &ctx->red, &ctx->scal, &ctx->counters, &ctx->dcolliders, &ctx->adm_F, &ctx->adm_gvn, &ctx->adm_B, &ctx->adm_pre,
        &ctx->adm_rhs, &ctx->adm_w, &ctx->adj, &ctx->kvf, &ctx->vstarf, &ctx->pfn, &ctx->pfsc, &ctx->gsync };
    for (DBuf* b : bufs) b->release();
    for (auto& b : ctx->kv) b.release();
    for (auto* v : { &ctx->ckpt_pd, &ctx->ckpt_pi, &ctx->ckpt_sid })
        for (auto& b : *v) b.release();
    ctx->stage.release();
    for (cudaEvent_t e : ctx->hvp_ev) cudaEventDestroy(e);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ZMPM_OK;
}

const char* zmpm_last_error(const zmpm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t zmpm_num_particles(const zmpm_ctx* ctx) { return ctx ? ctx->P : -1; }

double zmpm_time(const zmpm_ctx* ctx) { return ctx ? ctx->time : 0.0; }

int zmpm_add_particles(zmpm_ctx* ctx, int64_t n, const double* x, const double* v, const double* m, const double* vol, int64_t* lower)
{
    if (!ctx || n < 0 || (n && (!x || !m || !vol))) return ZMPM_BAD_ARG;
    if (ctx->P + n >= ((int64_t)1 << (ctx->layout == 1 ? Layout244::INDEX_BITS : Layout444::INDEX_BITS))) {
        ctx->err = "particle count exceeds the key's index bits (MpmSimulationBase.cpp:1037-1038)";
        return ZMPM_BAD_ARG;
    }
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    if (lower) *lower = ctx->P;
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) {
            ctx->hx.push_back(x[3 * i + d]);
            ctx->hv.push_back(v ? v[3 * i + d] : 0.0);
            ctx->hcrack.push_back(0.0);
        }
        for (int q = 0; q < 9; ++q) {
            ctx->hC.push_back(0.0);
            ctx->hF.push_back((q % 4 == 0) ? 1.0 : 0.0);
        }
        ctx->hm.push_back(m[i]);
        ctx->hvol.push_back(vol[i]);
        ctx->hmu.push_back(0);
        ctx->hlam.push_back(0);
        ctx->hkappa.push_back(0);
        ctx->hg.push_back(1);
        ctx->hys.push_back(0);
        ctx->hxi.push_back(0);
        ctx->hfs.push_back(0);
        ctx->hpfc.push_back(1.0);
        ctx->hpfk.push_back(0.001);
        ctx->hsigf.push_back(0.0);
        ctx->hlogjp.push_back(0.0);
        ctx->hdamage.push_back(ZMPM_DAMAGE_NONE);
        ctx->hkind.push_back(ZMPM_MODEL_NONE);
        ctx->hpkind.push_back(ZMPM_PLASTIC_NONE);
        ctx->hbroken.push_back(0);
        ctx->hvisco.push_back(0);
        for (int q = 0; q < 9; ++q) ctx->hFe.push_back((q % 4 == 0) ? 1.0 : 0.0);
        ctx->hvmu.push_back(0);
        ctx->hvlam.push_back(0);
        ctx->hvd.push_back(1);
        ctx->hvv.push_back(1);
        for (int q = 0; q < 18; ++q) ctx->hy.push_back(0.0);
        ctx->homega.push_back(1.0);
        ctx->homega.push_back(1.0);
        for (int d = 0; d < 3; ++d) ctx->hlastdv.push_back(0.0);
        ctx->hpfH.push_back(0.0);
        ctx->hpfl0.push_back(0.0);
        ctx->hpfisc.push_back(0.0);
        ctx->hpffp.push_back(1.0);
        ctx->hpfhmax.push_back(std::numeric_limits<double>::max());
        ctx->hpfvol.push_back(vol[i]);
        ctx->hpfallow.push_back(1.0);
    }
    ctx->P += n;
    return ZMPM_OK;
}

int zmpm_add_fbased_force(zmpm_ctx* ctx, int64_t lo, int64_t hi, int32_t model, double E, double nu)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    if (model < ZMPM_MODEL_NONE || model > ZMPM_MODEL_FIXED_COROTATED) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    // NeoHookeanBorden::setLameParameters / StvkWithHenckyIsotropic::setLameParameters
    double lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
    double mu = E / (2 * (1 + nu));
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hkind[i] = (uint8_t)model;
        ctx->hmu[i] = mu;
        ctx->hlam[i] = lambda;
        ctx->hkappa[i] = 0.666666 * mu + lambda;
        ctx->hg[i] = 1;
    }
    return ZMPM_OK;
}

int zmpm_set_lame(zmpm_ctx* ctx, int64_t lo, int64_t hi, const double* mu, const double* lambda)
{
    if (!ctx || !mu || !lambda || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hmu[i] = mu[i - lo];
        ctx->hlam[i] = lambda[i - lo];
        ctx->hkappa[i] = 0.666666 * mu[i - lo] + lambda[i - lo];
    }
    return ZMPM_OK;
}

int zmpm_add_plasticity(zmpm_ctx* ctx, int64_t lo, int64_t hi, int32_t kind, double ys, double xi, double fs)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    if (kind != ZMPM_PLASTIC_NONE && kind != ZMPM_PLASTIC_VON_MISES) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hpkind[i] = (uint8_t)kind;
        ctx->hys[i] = ys;
        ctx->hxi[i] = xi;
        ctx->hfs[i] = fs;
    }
    return ZMPM_OK;
}

// sin of an angle in degrees with the reference's constant for pi
// (PlasticityApplier.cpp:17, :255)
static double sin_degrees(double angle) { return std::sin(angle / 180.0 * 3.141592653); }

int zmpm_add_drucker_prager(zmpm_ctx* ctx, int64_t lo, int64_t hi, double friction_angle, double beta, double cohesion,
    int32_t volume_correction)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i)
        if (ctx->hkind[i] != ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
            ctx->err = "Drucker-Prager needs StvkWithHenckyIsotropic particles";
            return ZMPM_BAD_ARG;
        }
    // DruckerPragerStvkHencky::DruckerPragerStvkHencky, PlasticityApplier.cpp:247-255
    const double sin_phi = sin_degrees(friction_angle);
    const double alpha = std::sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi);
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hpkind[i] = ZMPM_PLASTIC_DRUCKER_PRAGER;
        ctx->hys[i] = alpha;
        ctx->hxi[i] = beta;
        ctx->hfs[i] = cohesion;
        ctx->hbroken[i] = volume_correction ? 1 : 0;
        ctx->hlogjp[i] = 0.0;
    }
    return ZMPM_OK;
}

int zmpm_add_cam_clay(zmpm_ctx* ctx, int64_t lo, int64_t hi, double log_jp, double friction_angle, double beta, double xi, int32_t hardening)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i)
        if (ctx->hkind[i] != ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
            ctx->err = "Cam-Clay needs NeoHookeanBorden particles";
            return ZMPM_BAD_ARG;
        }
    // NonAssociativeCamClay::NonAssociativeCamClay with dim = 3, PlasticityApplier.cpp:10-20
    const double sin_phi = sin_degrees(friction_angle);
    const double mc = std::sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi);
    const double M = mc * 3.0 / std::sqrt(2.0 / (6.0 - 3.0));
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hpkind[i] = ZMPM_PLASTIC_CAM_CLAY;
        ctx->hys[i] = M;
        ctx->hxi[i] = beta;
        ctx->hfs[i] = xi;
        ctx->hbroken[i] = hardening ? 1 : 0;
        ctx->hlogjp[i] = log_jp;
    }
    return ZMPM_OK;
}

int zmpm_get_log_jp(zmpm_ctx* ctx, double* log_jp)
{
    if (!ctx || !log_jp) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    std::memcpy(log_jp, ctx->hlogjp.data(), ctx->P * sizeof(double));
    return ZMPM_OK;
}

int zmpm_add_damage(zmpm_ctx* ctx, int64_t lo, int64_t hi, int32_t kind, double sigma_f, double residual_phase)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi) return ZMPM_BAD_ARG;
    if (kind != ZMPM_DAMAGE_NONE && kind != ZMPM_DAMAGE_RANKINE && kind != ZMPM_DAMAGE_RANKINE_REFERENCE) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hdamage[i] = (uint8_t)kind;
        ctx->hsigf[i] = sigma_f;
        ctx->hpfk[i] = residual_phase;
        ctx->hpfc[i] = 1.0;
    }
    return ZMPM_OK;
}

int zmpm_get_damage(zmpm_ctx* ctx, double* c)
{
    if (!ctx || !c) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    for (int64_t i = 0; i < ctx->P; ++i) c[i] = ctx->hpfc[i];
    return ZMPM_OK;
}

// PhaseField::Get_Sigma_C_Based_On_Max_Deformation (PhaseField.h:58-68):
// 1 / psi((1 + percentage) I) with NeoHookeanBorden::psi (NeoHookeanBorden.cpp:38-51).
static double pf_one_over_sigma_c(double mu, double kappa, double g, double percentage)
{
    const double f = 1 + percentage, J = f * (f * f);
    const double a = std::pow(J, -1.0 / 3.0);
    double tr = 0;
    for (int i = 0; i < 3; ++i) tr += (a * f) * (a * f);
    const double psi_dev = mu / 2 * (tr - 3);
    const double psi_vol = kappa / 2 * ((J * J - 1) / 2 - std::log(J));
    const double psi_pos = (J >= 1) ? psi_vol + psi_dev : psi_dev;
    const double psi_neg = (J >= 1) ? 0.0 : psi_vol;
    return 1.0 / (g * psi_pos + psi_neg);
}

int zmpm_add_phase_field(zmpm_ctx* ctx, int64_t lo, int64_t hi, double percentage, double l0, int32_t allow_damage, double residual_phase)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi || !(l0 >= 0)) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = lo; i < hi; ++i)
        if (ctx->hkind[i] != ZMPM_MODEL_NEOHOOKEAN_BORDEN) {
            ctx->err = "the phase field needs NeoHookeanBorden particles";
            return ZMPM_BAD_ARG;
        }
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hdamage[i] = ZMPM_DAMAGE_PHASE_FIELD;
        ctx->hpfk[i] = residual_phase;
        ctx->hpfc[i] = 1.0;
        ctx->hpfH[i] = 0.0;
        ctx->hpfl0[i] = l0;
        ctx->hpfisc[i] = pf_one_over_sigma_c(ctx->hmu[i], ctx->hkappa[i], ctx->hg[i], percentage);
        ctx->hpffp[i] = 1.0;
        ctx->hpfhmax[i] = std::numeric_limits<double>::max();
        ctx->hpfvol[i] = ctx->hvol[i];
        ctx->hpfallow[i] = allow_damage ? 1.0 : 0.0;
    }
    if (hi > lo) ctx->pd_active = std::max(ctx->pd_active, (int)PD_PF_END);
    return ZMPM_OK;
}

int zmpm_set_phase_field_solver(zmpm_ctx* ctx, double parabolic_M, int32_t lumping, double delete_threshold, int32_t cg_max_iterations,
    double cg_tolerance)
{
    if (!ctx || !(parabolic_M >= 0) || cg_max_iterations < 0 || !(cg_tolerance >= 0) || !(delete_threshold == delete_threshold))
        return ZMPM_BAD_ARG;
    ctx->pf_M = parabolic_M;
    ctx->pf_lumping = lumping != 0;
    ctx->pf_delete = delete_threshold;
    ctx->pf_cg_max = cg_max_iterations;
    ctx->pf_cg_tol = cg_tolerance;
    return ZMPM_OK;
}

int zmpm_get_phase_field(zmpm_ctx* ctx, double* c, double* H, double* pf_Fp, double* vol)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    for (int64_t i = 0; i < ctx->P; ++i) {
        if (c) c[i] = ctx->hpfc[i];
        if (H) H[i] = ctx->hpfH[i];
        if (pf_Fp) pf_Fp[i] = ctx->hpffp[i];
        if (vol) vol[i] = ctx->hpfvol[i];
    }
    return ZMPM_OK;
}

int zmpm_set_phase_field_sigma_c(zmpm_ctx* ctx, const double* one_over_sigma_c)
{
    if (!ctx || !one_over_sigma_c) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    for (int64_t i = 0; i < ctx->P; ++i) ctx->hpfisc[i] = one_over_sigma_c[i];
    return ZMPM_OK;
}

int zmpm_add_viscoelastic(zmpm_ctx* ctx, int64_t lo, int64_t hi, double E, double nu, double vd, double vv)
{
    if (!ctx || lo < 0 || hi > ctx->P || lo > hi || !(vd > 0) || !(vv > 0)) return ZMPM_BAD_ARG;
    for (int64_t i = lo; i < hi; ++i)
        if (ctx->hkind[i] != ZMPM_MODEL_STVK_HENCKY_ISOTROPIC) {
            ctx->err = "viscoelastic particles must use StvkWithHenckyIsotropic";
            return ZMPM_BAD_ARG;
        }
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    // StvkWithHencky::setLameParameters, StvkWithHencky.cpp:16-20
    const double lambda = E * nu / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
    for (int64_t i = lo; i < hi; ++i) {
        ctx->hvisco[i] = 1;
        ctx->hvmu[i] = mu;
        ctx->hvlam[i] = lambda;
        ctx->hvd[i] = vd;
        ctx->hvv[i] = vv;
        for (int q = 0; q < 9; ++q) ctx->hFe[9 * i + q] = (q % 4 == 0) ? 1.0 : 0.0;
    }
    if (hi > lo) ctx->has_visco = true;
    ctx->pd_active = PD_FIELDS;
    return ZMPM_OK;
}

int zmpm_get_viscoelastic_strain(zmpm_ctx* ctx, double* Fe)
{
    if (!ctx || !Fe) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    std::memcpy(Fe, ctx->hFe.data(), 9 * ctx->P * sizeof(double));
    return ZMPM_OK;
}

int zmpm_set_viscoelastic_strain(zmpm_ctx* ctx, const double* Fe)
{
    if (!ctx || !Fe) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = begin_edit(ctx);
    if (rc) return rc;
    std::memcpy(ctx->hFe.data(), Fe, 9 * ctx->P * sizeof(double));
    return ZMPM_OK;
}

int zmpm_add_collision_object(zmpm_ctx* ctx, const zmpm_collider* o, int32_t* id)
{
    if (!ctx || !o) return ZMPM_BAD_ARG;
    if ((int)ctx->colliders.size() >= MAX_COLLIDERS) return ZMPM_BAD_ARG;
    if (o->shape < ZMPM_HALF_SPACE || o->shape > ZMPM_BOX || o->type < ZMPM_STICKY || o->type > ZMPM_GHOST || !(o->scale != 0)) return ZMPM_BAD_ARG;
    if (id) *id = (int32_t)ctx->colliders.size();
    ctx->colliders.push_back(*o);
    return ZMPM_OK;
}

int zmpm_set_collision_object(zmpm_ctx* ctx, int32_t id, const zmpm_collider* o)
{
    if (!ctx || !o || id < 0 || id >= (int32_t)ctx->colliders.size()) return ZMPM_BAD_ARG;
    ctx->colliders[id] = *o;
    return ZMPM_OK;
}

int zmpm_get_stream(zmpm_ctx* ctx, void** stream)
{
    if (!ctx || !stream) return ZMPM_BAD_ARG;
    *stream = (void*)ctx->stream;
    return ZMPM_OK;
}

int zmpm_set_spin_limit(zmpm_ctx* ctx, int64_t polls)
{
    if (!ctx || polls < 0) return ZMPM_BAD_ARG;
    ctx->spin_limit = polls == 0 ? (1ll << 22) : polls;
    return ZMPM_OK;
}

int zmpm_set_profiling(zmpm_ctx* ctx, int32_t on)
{
    if (!ctx) return ZMPM_BAD_ARG;
    ctx->profiling = on != 0;
    return ZMPM_OK;
}

int zmpm_get_particles(zmpm_ctx* ctx, double* x, double* v, double* C, double* F)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->uploaded) return device_get(ctx, x, v, C, F);
    const int64_t P = ctx->P;
    if (x) std::memcpy(x, ctx->hx.data(), 3 * P * sizeof(double));
    if (v) std::memcpy(v, ctx->hv.data(), 3 * P * sizeof(double));
    if (C) std::memcpy(C, ctx->hC.data(), 9 * P * sizeof(double));
    if (F) std::memcpy(F, ctx->hF.data(), 9 * P * sizeof(double));
    return ZMPM_OK;
}

int zmpm_set_particles(zmpm_ctx* ctx, const double* x, const double* v, const double* C, const double* F)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->uploaded) return device_set(ctx, x, v, C, F);
    const int64_t P = ctx->P;
    if (x) std::memcpy(ctx->hx.data(), x, 3 * P * sizeof(double));
    if (v) std::memcpy(ctx->hv.data(), v, 3 * P * sizeof(double));
    if (C) std::memcpy(ctx->hC.data(), C, 9 * P * sizeof(double));
    if (F) std::memcpy(ctx->hF.data(), F, 9 * P * sizeof(double));
    return ZMPM_OK;
}

int zmpm_get_plastic_state(zmpm_ctx* ctx, double* ys, int32_t* broken)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    for (int64_t i = 0; i < ctx->P; ++i) {
        if (ys) ys[i] = ctx->hys[i];
        if (broken) broken[i] = ctx->hbroken[i];
    }
    return ZMPM_OK;
}

// ---------------------------------------------------------------- substep --
// FractureSimulation::reinitialize -> deleteParticles (FractureSimulation.h:
// 166-207) ahead of the binning; with a threshold <= 0 no particle qualifies.
static int delete_phase_field_particles(zmpm_ctx* ctx)
{
    if (!ctx->has_pf || !(ctx->pf_delete > 0)) return ZMPM_OK;
    return launch_phase_field_delete(ctx);
}

// Kernels of one Newton loop body when the solve runs as a graph: the update
// (MIXED: the FP32 pass and the gated FP64 stress / force pair, one of which
// returns at once), residual with the Krylov start vectors, Newton check with
// the Krylov start, the persistent linear solve, step, advance.
static int64_t newton_body_launches(const zmpm_ctx* ctx) { return ctx->mixed ? 8 : 6; }

static int begin_implicit_impl(zmpm_ctx* ctx, double dt, bool damage = true)
{
    int rc = upload(ctx);
    if (rc) return rc;
    ctx->dt = dt;
    ctx->implicit_ready = false;
    rc = delete_phase_field_particles(ctx);
    if (rc) return rc;
    rc = run_binning(ctx);
    if (rc) return rc;
    rc = run_p2g(ctx, damage);
    if (rc) return rc;
    ctx->implicit_ready = true;
    return ZMPM_OK;
}

// Argument checks and uploads shared by zmpm_substep and the phase entry points.
static int substep_prepare(zmpm_ctx* ctx, double dt, const zmpm_solver* s)
{
    if (!ctx || !s || !(dt > 0) || s->newton_max_iterations < 0 || s->krylov_max_iterations < 0) return ZMPM_BAD_ARG;
    const bool admm = s->integrator == ZMPM_ADMM, expl = s->integrator == ZMPM_EXPLICIT;
    if (!admm && !expl && s->integrator != ZMPM_NEWTON) return ZMPM_BAD_ARG;
    if (s->mls_mpm && !expl) {
        ctx->err = "mls_mpm requires the explicit integrator (MpmSimulationBase.cpp:102-106)";
        return ZMPM_BAD_ARG;
    }
    ctx->mls = expl && s->mls_mpm;
    if (admm && (s->admm_iterations < 0 || s->admm_global_max_iterations < 0 || !(s->admm_rho_scale > 0))) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    if (admm) {
        // AdmmSimulation indexes F (and Fe) by particle, so every particle needs an F-based model
        int rc = upload(ctx);
        if (rc) return rc;
        if (!ctx->all_models) {
            ctx->err = "ADMM needs an F-based model on every particle";
            return ZMPM_BAD_ARG;
        }
        if (ctx->pd_active != PD_FIELDS) { // ADMM state moves with the particles from now on
            int rc = begin_edit(ctx);
            if (rc) return rc;
            ctx->pd_active = PD_FIELDS;
        }
    }
    else if (ctx->has_visco && !expl) {
        ctx->err = "viscoelastic particles need the ADMM or explicit integrator (StvkWithHencky has no stress differential)";
        return ZMPM_BAD_ARG;
    }
    {
        int rc = upload(ctx);
        if (rc) return rc;
    }
    if (admm)
        for (int64_t i = 0; i < ctx->P; ++i)
            if (ctx->hpkind[i] == ZMPM_PLASTIC_CAM_CLAY) {
                ctx->err = "the ADMM F-step has no Cam-Clay projection (AdmmSimulationFoam.h:617-633 lists none)";
                return ZMPM_UNSUPPORTED;
            }
    if (ctx->has_pf && admm) {
        ctx->err = "the phase-field solve belongs to FractureSimulation; AdmmSimulation does not run it";
        return ZMPM_BAD_ARG;
    }
    if (ctx->has_pf && !ctx->all_pf) {
        ctx->err = "the phase-field solve needs the phase field on every particle (FractureSimulation.h:318-342 reads it for all)";
        return ZMPM_BAD_ARG;
    }
    ctx->pf_iters = 0;
    ctx->pf_res = 0;
    return ZMPM_OK;
}

// Phase 1 of a substep: reinitialize + particlesToGrid (+ the fracture hook and
// the Newton start), or the explicit substep up to the grid update.
static int substep_to_grid(zmpm_ctx* ctx, double dt, const zmpm_solver& s)
{
    const bool admm = s.integrator == ZMPM_ADMM, expl = s.integrator == ZMPM_EXPLICIT;
    ZMPM_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
    if (expl) {
        int rc = upload(ctx);
        if (rc) return rc;
        ctx->dt = dt;
        ctx->implicit_ready = false;
        rc = delete_phase_field_particles(ctx);
        if (rc) return rc;
        rc = run_binning(ctx);
        if (rc) return rc;
        ctx->graph_used = false;
        return run_explicit(ctx, s);
    }
    return begin_implicit_impl(ctx, dt, !admm);
}

// Reads the substep's device counters and scalars back (synchronises the
// stream) and fills the statistics; `g2p_done`: the substep ended with G2P
// (the time advances, and the CFL flag and the device time are final).
static int substep_finish(zmpm_ctx* ctx, double dt, const zmpm_solver& s, zmpm_stats* st, int64_t launches0, bool g2p_done)
{
    const bool admm = s.integrator == ZMPM_ADMM, expl = s.integrator == ZMPM_EXPLICIT;
    if (g2p_done) ZMPM_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    SolverScalars hs;
    DevCounters hc;
    ZMPM_CUDA(cudaMemcpyAsync(&hs, ctx->scal.p, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(&hc, ctx->counters.p, sizeof(hc), cudaMemcpyDeviceToHost, ctx->stream));
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    // the solve's graph stays instantiated until the next solve replaces it
    // (after launching its own graph) or zmpm_destroy: destroying it here sat
    // in the GPU's idle time between substeps
    float ms = 0;
    if (g2p_done) {
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        ctx->time += dt;
        ctx->implicit_ready = false;
    }
    st->newton_iterations = hs.newton_iters;
    st->krylov_iterations = hs.krylov_iters;
    st->hvp_count = hs.hvp_count;
    st->newton_converged = hs.converged;
    st->newton_residual_initial = hs.res_initial;
    st->newton_residual_final = hs.res_final;
    st->cfl_violation = (g2p_done && (hc.flags & FLAG_CFL)) ? 1 : 0;
    st->status_flags = ((hc.flags & FLAG_NAN) || !(hs.res_final == hs.res_final) ? 1 : 0) | ((hc.flags & FLAG_TIMEOUT) ? 2 : 0);
    st->num_particles = ctx->P;
    st->num_groups = ctx->G;
    st->num_blocks = ctx->B;
    st->num_nodes = hc.N;
    st->ms_total = ms;
    st->phase_field_iterations = ctx->pf_iters;
    st->phase_field_residual = ctx->pf_res;
    st->fp64_residual = hs.fp64_res;
    st->rankine_first_not_max = hc.first_not_max;
    st->svd_fp64_reevaluations = hc.svd_fp64;
    if (!admm && !expl) ctx->fp64_res_run = hs.fp64_res ? ctx->fp64_res_run + 1 : 0;
    // ADMM iteration: collision, local step, force scatter, operator, start,
    // Krylov start, persistent MINRES, dv update, dual update, advance
    if (ctx->graph_used && admm)
        g_kernel_launches += 10 * (int64_t)hs.nit;
    else if (ctx->graph_used)
        g_kernel_launches += newton_body_launches(ctx) * (int64_t)hs.nit;
    ctx->graph_used = false;
    st->kernel_launches = (int32_t)(g_kernel_launches - launches0);
    ctx->N = hc.N;
    if (ctx->prof_newton > 0) {
        // the linear solves that iterated: their persistent kernels' time and
        // Krylov iterations
        double tot = 0;
        int n = 0;
        for (int j = 0; j < ctx->prof_newton && j < 64; ++j) {
            float e = 0;
            if (hs.kcount[j] > 0 && cudaEventElapsedTime(&e, ctx->hvp_ev[2 * j], ctx->hvp_ev[2 * j + 1]) == cudaSuccess) {
                tot += e;
                n += hs.kcount[j];
            }
        }
        st->ms_hvp = tot;
        st->hvp_timed = n;
    }
    if (hc.flags & FLAG_TIMEOUT) {
        ctx->err = "a bounded device wait gave up";
        return ZMPM_TIMEOUT;
    }
    if (st->status_flags & 1) return ZMPM_NAN_DETECTED;
    return st->cfl_violation ? ZMPM_CFL_VIOLATION : ZMPM_OK;
}

int zmpm_substep(zmpm_ctx* ctx, double dt, const zmpm_solver* s, zmpm_stats* st)
{
    int rc = substep_prepare(ctx, dt, s);
    if (rc) return rc;
    const bool admm = s->integrator == ZMPM_ADMM, expl = s->integrator == ZMPM_EXPLICIT;
    zmpm_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    const int64_t launches0 = g_kernel_launches;
    ctx->phase = 0;
    rc = substep_to_grid(ctx, dt, *s);
    if (rc) return rc;
    if (!expl) {
        rc = admm ? run_admm(ctx, *s) : run_newton(ctx, *s);
        if (rc) return rc;
    }
    rc = run_g2p(ctx);
    if (rc) return rc;
    return substep_finish(ctx, dt, *s, st, launches0, true);
}

// ------------------------------------------------------------ substep phases --
int zmpm_particles_to_grid(zmpm_ctx* ctx, double dt, const zmpm_solver* s)
{
    int rc = substep_prepare(ctx, dt, s);
    if (rc) return rc;
    if (s->integrator == ZMPM_EXPLICIT) {
        ctx->err = "the phase entry points run the implicit (Newton or ADMM) substep";
        return ZMPM_UNSUPPORTED;
    }
    ctx->phase = 0;
    rc = substep_to_grid(ctx, dt, *s);
    if (rc) return rc;
    ctx->phase = 1;
    ctx->phase_solver = *s;
    ctx->phase_launches0 = g_kernel_launches;
    return ZMPM_OK;
}

int zmpm_backward_euler_step(zmpm_ctx* ctx, zmpm_stats* st)
{
    if (!ctx) return ZMPM_BAD_ARG;
    if (ctx->phase != 1 || !ctx->implicit_ready) {
        ctx->err = "zmpm_backward_euler_step follows zmpm_particles_to_grid";
        return ZMPM_NOT_READY;
    }
    cudaSetDevice(ctx->device);
    const zmpm_solver& s = ctx->phase_solver;
    zmpm_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    int rc = s.integrator == ZMPM_ADMM ? run_admm(ctx, s) : run_newton(ctx, s);
    if (rc) return rc;
    ctx->phase = 2;
    return substep_finish(ctx, ctx->dt, s, st, ctx->phase_launches0, false);
}

int zmpm_grid_to_particles(zmpm_ctx* ctx, int32_t apply_plasticity, zmpm_stats* st)
{
    if (!ctx) return ZMPM_BAD_ARG;
    if (ctx->phase != 2) {
        ctx->err = "zmpm_grid_to_particles follows zmpm_backward_euler_step";
        return ZMPM_NOT_READY;
    }
    cudaSetDevice(ctx->device);
    zmpm_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    const int64_t launches0 = g_kernel_launches;
    int rc = run_g2p(ctx, apply_plasticity != 0);
    if (rc) return rc;
    ctx->phase = 0;
    return substep_finish(ctx, ctx->dt, ctx->phase_solver, st, launches0, true);
}

int zmpm_apply_plasticity(zmpm_ctx* ctx)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = upload(ctx);
    if (rc) return rc;
    rc = launch_plasticity(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaGetLastError());
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    return ZMPM_OK;
}

// ---------------------------------------------------------------- adjoint --
int zmpm_adjoint_substep(zmpm_ctx* ctx, double dt, const zmpm_solver* s, double tol, double* gx, double* gv, double* gC, double* gF,
    double* gE, zmpm_stats* st)
{
    if (!ctx || !s || !(dt > 0) || !(tol > 0) || s->newton_max_iterations < 0 || s->krylov_max_iterations < 0) return ZMPM_BAD_ARG;
    if (s->integrator != ZMPM_NEWTON) {
        ctx->err = "the adjoint differentiates the Newton substep";
        return ZMPM_UNSUPPORTED;
    }
    ctx->mls = false;
    for (int64_t i = 0; i < ctx->P; ++i) {
        // von Mises with a constant yield stress (xi = 0) has an adjoint; hardening
        // would need the yield stress as adjoint state, the other return maps,
        // damage and the viscoelastic strain have none
        const bool vm = ctx->hpkind[i] == ZMPM_PLASTIC_VON_MISES && ctx->hxi[i] == 0.0 && ctx->hkind[i] == ZMPM_MODEL_STVK_HENCKY_ISOTROPIC;
        if ((ctx->hpkind[i] != ZMPM_PLASTIC_NONE && !vm) || ctx->hdamage[i] != ZMPM_DAMAGE_NONE || ctx->hvisco[i]) {
            ctx->err = "the adjoint supports elastic particles and von Mises (StvkWithHenckyIsotropic, xi = 0) only";
            return ZMPM_UNSUPPORTED;
        }
    }
    cudaSetDevice(ctx->device);
    zmpm_stats local;
    if (!st) st = &local;
    std::memset(st, 0, sizeof(*st));
    const int64_t launches0 = g_kernel_launches;
    int rc = upload(ctx);
    if (rc) return rc;
    ctx->dt = dt;
    ctx->implicit_ready = false;
    rc = run_binning(ctx);
    if (rc) return rc;
    const int64_t P = ctx->P, cap = ctx->Pcap;
    cudaStream_t sm = ctx->stream;
    ZMPM_CUDA(ctx->adj.ensure((size_t)AJ_FIELDS * cap * sizeof(double)));
    double* aj = ctx->adj.as<double>();
    // the state before the substep (pool fields x, v, C, F are the first 24) in slot order
    ZMPM_CUDA(cudaMemcpyAsync(aj, ctx->pd.p, 24 * cap * sizeof(double), cudaMemcpyDeviceToDevice, sm));
    ZMPM_CUDA(cudaMemsetAsync(aj + AJ_GX * cap, 0, 24 * cap * sizeof(double), sm));
    if (P) {
        ZMPM_CUDA(ctx->stage.ensure(25 * P * sizeof(double))); // 24 gradient components + dL/dE
        double* stg = ctx->stage.as<double>();
        const double* src[4] = { gx, gv, gC, gF };
        const int nc[4] = { 3, 3, 9, 9 }, fld[4] = { AJ_GX, AJ_GV, AJ_GC, AJ_GF };
        int64_t off = 0;
        for (int a = 0; a < 4; ++a) {
            if (!src[a]) continue;
            ZMPM_CUDA(cudaMemcpyAsync(stg + off, src[a], nc[a] * P * sizeof(double), cudaMemcpyHostToDevice, sm));
            k_fields_from_host<<<(unsigned)((P + 255) / 256), 256, 0, sm>>>(stg + off, nc[a], P, cap, ctx->slot_of_id.as<int32_t>(),
                aj + (int64_t)fld[a] * cap);
            ++g_kernel_launches;
            off += nc[a] * P;
        }
    }
    // forward: P2G, Newton, the Hessian at the converged solution, G2P
    rc = run_p2g(ctx, true);
    if (rc) return rc;
    rc = run_newton(ctx, *s);
    if (rc) return rc;
    rc = launch_update(ctx, false);
    if (rc) return rc;
    rc = run_g2p(ctx);
    if (rc) return rc;
    SolverScalars hs;
    ZMPM_CUDA(cudaMemcpyAsync(&hs, ctx->scal.p, sizeof(hs), cudaMemcpyDeviceToHost, sm));
    ZMPM_CUDA(cudaStreamSynchronize(sm));
    if (ctx->graph_exec) {
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
    }
    if (ctx->graph_used)
        g_kernel_launches += newton_body_launches(ctx) * (int64_t)hs.nit;
    st->newton_iterations = hs.newton_iters;
    st->newton_converged = hs.converged;
    st->fp64_residual = hs.fp64_res;
    ctx->fp64_res_run = hs.fp64_res ? ctx->fp64_res_run + 1 : 0;
    st->newton_residual_initial = hs.res_initial;
    st->newton_residual_final = hs.res_final;
    // reverse: G2P, the adjoint solve, force / P2G / E
    const int64_t nn = ctx->B * ctx->npb();
    ZMPM_CUDA(cudaMemsetAsync(ctx->res.p, 0, 3 * nn * sizeof(double), sm));
    rc = launch_adj_g2p(ctx, ctx->res.as<double>());
    if (rc) return rc;
    rc = run_adjoint_solve(ctx, tol, 100000);
    if (rc) return rc;
    rc = launch_adj_particle(ctx, ctx->kv[0].as<double>());
    if (rc) return rc;
    SolverScalars ha;
    ZMPM_CUDA(cudaMemcpyAsync(&ha, ctx->scal.p, sizeof(ha), cudaMemcpyDeviceToHost, sm));
    // gradients back to particle-index order
    if (P) {
        double* stg = ctx->stage.as<double>();
        double* dst[4] = { gx, gv, gC, gF };
        const int nc[4] = { 3, 3, 9, 9 }, fld[4] = { AJ_OX, AJ_OV, AJ_OC, AJ_OF };
        int64_t off = 0;
        for (int a = 0; a < 4; ++a) {
            if (!dst[a]) continue;
            k_fields_to_host<<<(unsigned)((P + 255) / 256), 256, 0, sm>>>(stg + off, nc[a], P, cap, ctx->slot_of_id.as<int32_t>(),
                aj + (int64_t)fld[a] * cap);
            ++g_kernel_launches;
            ZMPM_CUDA(cudaMemcpyAsync(dst[a], stg + off, nc[a] * P * sizeof(double), cudaMemcpyDeviceToHost, sm));
            off += nc[a] * P;
        }
        if (gE) {
            std::vector<double> e(P);
            k_fields_to_host<<<(unsigned)((P + 255) / 256), 256, 0, sm>>>(stg + off, 1, P, cap, ctx->slot_of_id.as<int32_t>(), aj + AJ_OE * cap);
            ++g_kernel_launches;
            ZMPM_CUDA(cudaMemcpyAsync(e.data(), stg + off, P * sizeof(double), cudaMemcpyDeviceToHost, sm));
            ZMPM_CUDA(cudaStreamSynchronize(sm));
            for (int64_t i = 0; i < P; ++i) gE[i] += e[i];
        }
    }
    ZMPM_CUDA(cudaStreamSynchronize(sm));
    DevCounters hc;
    ZMPM_CUDA(d2h_sync(ctx, &hc, ctx->counters.p, sizeof(hc)));
    st->krylov_iterations = ha.krylov_iters;
    st->hvp_count = ha.hvp_count;
    st->cfl_violation = (hc.flags & FLAG_CFL) ? 1 : 0;
    st->status_flags = (hc.flags & FLAG_NAN ? 1 : 0) | (hc.flags & FLAG_TIMEOUT ? 2 : 0);
    st->num_particles = P;
    st->num_groups = ctx->G;
    st->num_blocks = ctx->B;
    st->num_nodes = hc.N;
    st->kernel_launches = (int32_t)(g_kernel_launches - launches0);
    ctx->time += dt;
    if (hc.flags & FLAG_TIMEOUT) {
        ctx->err = "a bounded device wait gave up";
        return ZMPM_TIMEOUT;
    }
    return st->cfl_violation ? ZMPM_CFL_VIOLATION : ZMPM_OK;
}

// ------------------------------------------------------------ checkpoints --
int zmpm_checkpoint_save(zmpm_ctx* ctx, int32_t slot)
{
    if (!ctx || slot < 0 || slot > 4096) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = upload(ctx);
    if (rc) return rc;
    const size_t n = (size_t)slot + 1;
    if (ctx->ckpt_pd.size() < n) {
        ctx->ckpt_pd.resize(n);
        ctx->ckpt_pi.resize(n);
        ctx->ckpt_sid.resize(n);
        ctx->ckpt_time.resize(n, 0.0);
        ctx->ckpt_P.resize(n, -1);
    }
    const int64_t cap = ctx->Pcap;
    ZMPM_CUDA(ctx->ckpt_pd[slot].ensure((size_t)PD_FIELDS * cap * sizeof(double)));
    ZMPM_CUDA(ctx->ckpt_pi[slot].ensure((size_t)PI_FIELDS * cap * sizeof(int32_t)));
    ZMPM_CUDA(ctx->ckpt_sid[slot].ensure((size_t)cap * sizeof(int32_t)));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->ckpt_pd[slot].p, ctx->pd.p, (size_t)ctx->pd_active * cap * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->ckpt_pi[slot].p, ctx->pi.p, (size_t)PI_FIELDS * cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->ckpt_sid[slot].p, ctx->slot_of_id.p, (size_t)cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->ckpt_time[slot] = ctx->time;
    ctx->ckpt_P[slot] = ctx->P * 1000 + ctx->pd_active; // particle count and active fields of the saved pool
    return ZMPM_OK;
}

int zmpm_checkpoint_load(zmpm_ctx* ctx, int32_t slot)
{
    if (!ctx || slot < 0 || (size_t)slot >= ctx->ckpt_pd.size() || ctx->ckpt_P[slot] < 0) return ZMPM_BAD_ARG;
    if (ctx->ckpt_P[slot] != ctx->P * 1000 + ctx->pd_active || !ctx->uploaded) {
        ctx->err = "the checkpoint was saved with a different particle set";
        return ZMPM_BAD_ARG;
    }
    cudaSetDevice(ctx->device);
    const int64_t cap = ctx->Pcap;
    ZMPM_CUDA(cudaMemcpyAsync(ctx->pd.p, ctx->ckpt_pd[slot].p, (size_t)ctx->pd_active * cap * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->pi.p, ctx->ckpt_pi[slot].p, (size_t)PI_FIELDS * cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaMemcpyAsync(ctx->slot_of_id.p, ctx->ckpt_sid[slot].p, (size_t)cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->time = ctx->ckpt_time[slot];
    ctx->binned = false;
    ctx->implicit_ready = false;
    return ZMPM_OK;
}

// ------------------------------------------------------------------ hooks --
int zmpm_bin(zmpm_ctx* ctx, int64_t* counts)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = upload(ctx);
    if (rc) return rc;
    rc = run_binning(ctx);
    if (rc) return rc;
    if (counts) {
        counts[0] = ctx->P;
        counts[1] = ctx->G;
        counts[2] = ctx->B;
    }
    return ZMPM_OK;
}

int zmpm_bin_fetch(zmpm_ctx* ctx, zmpm_bin_result* out)
{
    if (!ctx || !out) return ZMPM_BAD_ARG;
    if (!ctx->binned) return ZMPM_NOT_READY;
    cudaSetDevice(ctx->device);
    const int64_t P = ctx->P, G = ctx->G, B = ctx->B;
    const int index_bits = ctx->layout == 1 ? Layout244::INDEX_BITS : Layout444::INDEX_BITS;
    const int log2s = ctx->layout == 1 ? Layout244::LOG2_STRUCT : Layout444::LOG2_STRUCT;
    std::vector<uint64_t> keys(P), bidx(B);
    std::vector<int32_t> gs(G + 1);
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (P) ZMPM_CUDA(d2h_sync(ctx, keys.data(), ctx->keys.p, P * sizeof(uint64_t)));
    if (G) ZMPM_CUDA(d2h_sync(ctx, gs.data(), ctx->group_start.p, (G + 1) * sizeof(int32_t)));
    if (B) ZMPM_CUDA(d2h_sync(ctx, bidx.data(), ctx->block_index.p, B * sizeof(uint64_t)));
    for (int64_t i = 0; i < P; ++i) {
        const uint64_t k = keys[i];
        const int32_t id = (int32_t)(k & ((1ull << index_bits) - 1));
        if (out->particle_sorter) out->particle_sorter[i] = k;
        if (out->particle_order) out->particle_order[i] = id;
        if (out->particle_base_offset) out->particle_base_offset[id] = (k >> index_bits) << log2s;
    }
    for (int64_t g = 0; g < G; ++g) {
        if (out->particle_group) {
            out->particle_group[2 * g] = gs[g];
            out->particle_group[2 * g + 1] = gs[g + 1] - 1;
        }
        if (out->block_offset) out->block_offset[g] = keys[gs[g + 1] - 1] >> 32;
    }
    for (int64_t b = 0; b < B; ++b)
        if (out->page_offsets) out->page_offsets[b] = bidx[b] << 12;
    return ZMPM_OK;
}

int zmpm_begin_implicit(zmpm_ctx* ctx, double dt, int64_t* num_nodes)
{
    if (!ctx || !(dt > 0)) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    ctx->phase = 0;
    int rc = begin_implicit_impl(ctx, dt);
    if (rc) return rc;
    std::vector<int64_t> idx;
    std::vector<double> hm;
    rc = node_indices(ctx, idx, hm);
    if (rc) return rc;
    ctx->scratch_valid = false;
    if (num_nodes) *num_nodes = ctx->N;
    return ZMPM_OK;
}

namespace {
// Converts a block-dense vector field [B][3][NPB] to node-index order [N][3].
void dense_to_tv(const Ctx* ctx, const std::vector<int64_t>& idx, const std::vector<double>& dense, double* tv)
{
    const int npb = ctx->npb();
    for (size_t n = 0; n < idx.size(); ++n) {
        if (idx[n] < 0) continue;
        int64_t b = n / npb, e = n % npb;
        for (int d = 0; d < 3; ++d) tv[3 * idx[n] + d] = dense[(b * 3 + d) * npb + e];
    }
}
void tv_to_dense(const Ctx* ctx, const std::vector<int64_t>& idx, const double* tv, std::vector<double>& dense)
{
    const int npb = ctx->npb();
    dense.assign(3 * idx.size(), 0.0);
    for (size_t n = 0; n < idx.size(); ++n) {
        if (idx[n] < 0) continue;
        int64_t b = n / npb, e = n % npb;
        for (int d = 0; d < 3; ++d) dense[(b * 3 + d) * npb + e] = tv[3 * idx[n] + d];
    }
}
int fetch_vec(Ctx* ctx, const DBuf& buf, std::vector<double>& h)
{
    h.resize(3 * ctx->B * ctx->npb());
    if (!h.empty()) ZMPM_CUDA(d2h_sync(ctx, h.data(), buf.p, h.size() * sizeof(double)));
    return ZMPM_OK;
}
} // namespace

int zmpm_get_grid(zmpm_ctx* ctx, double* m, double* v, int32_t* coord)
{
    if (!ctx) return ZMPM_BAD_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    std::vector<int64_t> idx;
    std::vector<double> hm, hv;
    rc = node_indices(ctx, idx, hm);
    if (rc) return rc;
    rc = fetch_vec(ctx, ctx->vn, hv);
    if (rc) return rc;
    std::vector<int4> bp(ctx->B);
    if (ctx->B) ZMPM_CUDA(d2h_sync(ctx, bp.data(), ctx->block_page.p, ctx->B * sizeof(int4)));
    const int npb = ctx->npb();
    const int bx = ctx->layout == 1 ? 2 : 4, by = 4, bz = 4, yb = 2, zb = 2;
    for (size_t n = 0; n < idx.size(); ++n) {
        if (idx[n] < 0) continue;
        int64_t b = n / npb, e = n % npb;
        if (m) m[idx[n]] = hm[n];
        if (coord) {
            coord[3 * idx[n]] = bp[b].x * bx + (int)(e >> (yb + zb));
            coord[3 * idx[n] + 1] = bp[b].y * by + (int)((e >> zb) & (by - 1));
            coord[3 * idx[n] + 2] = bp[b].z * bz + (int)(e & (bz - 1));
        }
    }
    if (v) dense_to_tv(ctx, idx, hv, v);
    return ZMPM_OK;
}

int zmpm_get_initial_dv(zmpm_ctx* ctx, double* dv, int32_t* collided)
{
    if (!ctx) return ZMPM_BAD_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    std::vector<int64_t> idx;
    std::vector<double> hm, hd;
    rc = node_indices(ctx, idx, hm);
    if (rc) return rc;
    rc = fetch_vec(ctx, ctx->dv, hd);
    if (rc) return rc;
    if (dv) dense_to_tv(ctx, idx, hd, dv);
    if (collided) {
        std::vector<int8_t> hc(idx.size());
        if (!hc.empty()) ZMPM_CUDA(d2h_sync(ctx, hc.data(), ctx->collided.p, hc.size()));
        for (size_t n = 0; n < idx.size(); ++n)
            if (idx[n] >= 0) collided[idx[n]] = hc[n];
    }
    return ZMPM_OK;
}

int zmpm_residual(zmpm_ctx* ctx, const double* dvin, double* r, double* norm)
{
    if (!ctx || !dvin) return ZMPM_BAD_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    std::vector<int64_t> idx;
    std::vector<double> hm, hvn, hdv, hres;
    rc = node_indices(ctx, idx, hm);
    if (rc) return rc;
    rc = fetch_vec(ctx, ctx->vn, hvn);
    if (rc) return rc;
    tv_to_dense(ctx, idx, dvin, hdv);
    std::vector<double> hvs(hdv.size());
    for (size_t i = 0; i < hdv.size(); ++i) hvs[i] = hdv[i] + hvn[i];
    for (size_t n = 0; n < idx.size(); ++n)
        if (idx[n] < 0) {
            int64_t b = n / ctx->npb(), e = n % ctx->npb();
            for (int d = 0; d < 3; ++d) hvs[(b * 3 + d) * ctx->npb() + e] = 0.0;
        }
    const size_t bytes = hdv.size() * sizeof(double);
    if (bytes) {
        ZMPM_CUDA(cudaMemcpyAsync(ctx->dv.p, hdv.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
        ZMPM_CUDA(cudaMemcpyAsync(ctx->vstar.p, hvs.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
        ctx->vstarf_valid = false;
        ZMPM_CUDA(cudaMemsetAsync(ctx->facc.p, 0, bytes, ctx->stream));
    }
    ZMPM_CUDA(cudaMemsetAsync(ctx->scal.p, 0, sizeof(SolverScalars), ctx->stream));
    rc = launch_update(ctx);
    if (rc) return rc;
    rc = launch_residual(ctx);
    if (rc) return rc;
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ZMPM_CUDA(cudaGetLastError());
    rc = fetch_vec(ctx, ctx->res, hres);
    if (rc) return rc;
    if (r) dense_to_tv(ctx, idx, hres, r);
    if (norm) {
        // computeNorm (BackwardEuler.h:127-140)
        double s = 0;
        const int npb = ctx->npb();
        for (size_t n = 0; n < idx.size(); ++n) {
            if (idx[n] < 0) continue;
            int64_t b = n / npb, e = n % npb;
            double q = 0;
            for (int d = 0; d < 3; ++d) {
                double v = hres[(b * 3 + d) * npb + e];
                q += v * v;
            }
            s += q / hm[n];
        }
        *norm = std::sqrt(s);
    }
    ctx->scratch_valid = true;
    return ZMPM_OK;
}

int zmpm_multiply(zmpm_ctx* ctx, const double* x, double* b, int32_t fp32)
{
    if (!ctx || !x || !b) return ZMPM_BAD_ARG;
    int rc = check_ready(ctx);
    if (rc) return rc;
    if (!ctx->scratch_valid) {
        ctx->err = "call zmpm_residual first (the Hessian is evaluated at its state)";
        return ZMPM_NOT_READY;
    }
    if ((fp32 != 0) != ctx->mixed) {
        ctx->err = "fp32 Hessian products are the MIXED precision path; FP64 contexts evaluate them in FP64";
        return ZMPM_UNSUPPORTED;
    }
    cudaSetDevice(ctx->device);
    std::vector<int64_t> idx;
    std::vector<double> hm, hx, hb;
    rc = node_indices(ctx, idx, hm);
    if (rc) return rc;
    tv_to_dense(ctx, idx, x, hx);
    const size_t bytes = hx.size() * sizeof(double);
    double* dx_ = ctx->kv[0].as<double>();
    double* dq = ctx->kv[1].as<double>();
    if (bytes) {
        ZMPM_CUDA(cudaMemcpyAsync(dx_, hx.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
        ZMPM_CUDA(cudaMemsetAsync(ctx->kv[9].p, 0, bytes, ctx->stream));
    }
    rc = launch_hvp(ctx, dx_, ctx->kv[9].as<double>(), ctx->mixed);
    if (rc) return rc;
    rc = finalize_multiply(ctx, dx_, dq);
    if (rc) return rc;
    ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
    ZMPM_CUDA(cudaGetLastError());
    rc = fetch_vec(ctx, ctx->kv[1], hb);
    if (rc) return rc;
    dense_to_tv(ctx, idx, hb, b);
    return ZMPM_OK;
}

} // extern "C"
