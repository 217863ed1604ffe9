// Host-side files: restart state and BGEO particle output.
//
// Restart ("ZMPMSTAT" version 1, native little-endian):
//   char[8] magic, uint32 version, uint32 0x01020304 (byte-order check),
//   zmpm_config, int64 P, double time, int32 pd_active,
//   double parabolic_M, delete_threshold, cg_tolerance; int32 lumping, cg_max,
//   int32 ncolliders, zmpm_collider[ncolliders],
//   int32 nfields, then per field: uint16 name length, name, uint8 type
//   (0 f64, 1 u8, 2 i32), int32 components, P * components values.
// Reading matches fields by name and requires every field the library knows.
//
// Restart directory (the reference's layout, SimulationBase.h:146-199): the
// state file restart_<frame>.dat (restart_<frame>_<substep>.dat for
// substep > 0), last_written.txt holding the frame, binary_ver.txt holding
// ZMPM_BINARY_VER.
//
// BGEO (Houdini binary geometry, version 5, big-endian) with points only:
//   int32 magic 'Bgeo', char 'V', int32 5, int32 points, primitives (0), point
//   groups (0), primitive groups (0), point attributes, vertex attributes (0),
//   primitive attributes (0), detail attributes (0); per point attribute:
//   uint16 name length, name, uint16 components, int32 type (5: vector),
//   components x int32 default (0); per point: x, y, z, w = 1, then the
//   attribute floats; trailer bytes 0x00 0xff.
#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cerrno>
#include <cstring>
#include <exception>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "internal.cuh"

namespace zmpm {
namespace {

struct Field {
    const char* name;
    int type;  // 0 f64, 1 u8, 2 i32
    int comps;
    void* vec; // std::vector<double>*, std::vector<uint8_t>* or std::vector<int32_t>*
};

std::vector<Field> state_fields(Ctx* c)
{
    return {
        { "X", 0, 3, &c->hx }, { "V", 0, 3, &c->hv }, { "C", 0, 9, &c->hC }, { "F", 0, 9, &c->hF },
        { "crack_normal", 0, 3, &c->hcrack }, { "mass", 0, 1, &c->hm }, { "element_measure", 0, 1, &c->hvol },
        { "mu", 0, 1, &c->hmu }, { "lambda", 0, 1, &c->hlam }, { "kappa", 0, 1, &c->hkappa }, { "g", 0, 1, &c->hg },
        { "plastic_a", 0, 1, &c->hys }, { "plastic_b", 0, 1, &c->hxi }, { "plastic_c", 0, 1, &c->hfs },
        { "phase_c", 0, 1, &c->hpfc }, { "residual_phase", 0, 1, &c->hpfk }, { "sigma_f", 0, 1, &c->hsigf },
        { "log_jp", 0, 1, &c->hlogjp }, { "model_kind", 1, 1, &c->hkind }, { "plastic_kind", 1, 1, &c->hpkind },
        { "damage_kind", 1, 1, &c->hdamage }, { "visco", 1, 1, &c->hvisco }, { "plastic_flag", 2, 1, &c->hbroken },
        { "Fe", 0, 9, &c->hFe }, { "visco_mu", 0, 1, &c->hvmu }, { "visco_lambda", 0, 1, &c->hvlam },
        { "viscosity_d", 0, 1, &c->hvd }, { "viscosity_v", 0, 1, &c->hvv }, { "admm_y", 0, 18, &c->hy },
        { "admm_omega", 0, 2, &c->homega }, { "admm_last_dv", 0, 3, &c->hlastdv }, { "pf_H", 0, 1, &c->hpfH },
        { "pf_l0", 0, 1, &c->hpfl0 }, { "pf_one_over_sigma_c", 0, 1, &c->hpfisc }, { "pf_Fp", 0, 1, &c->hpffp },
        { "pf_H_max", 0, 1, &c->hpfhmax }, { "pf_vol", 0, 1, &c->hpfvol }, { "pf_allow_damage", 0, 1, &c->hpfallow },
    };
}

size_t type_size(int t) { return t == 0 ? 8 : (t == 1 ? 1 : 4); }

void* field_data(const Field& f)
{
    if (f.type == 0) return static_cast<std::vector<double>*>(f.vec)->data();
    if (f.type == 1) return static_cast<std::vector<uint8_t>*>(f.vec)->data();
    return static_cast<std::vector<int32_t>*>(f.vec)->data();
}

void field_resize(const Field& f, size_t n)
{
    if (f.type == 0)
        static_cast<std::vector<double>*>(f.vec)->resize(n);
    else if (f.type == 1)
        static_cast<std::vector<uint8_t>*>(f.vec)->resize(n);
    else
        static_cast<std::vector<int32_t>*>(f.vec)->resize(n);
}

struct File {
    FILE* f = nullptr;
    bool ok = true;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) { ok = f != nullptr; }
    ~File()
    {
        if (f) std::fclose(f);
    }
    void put(const void* p, size_t n)
    {
        if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false;
    }
    void get(void* p, size_t n)
    {
        if (ok && n && std::fread(p, 1, n, f) != n) ok = false;
    }
    template <class T>
    void put(const T& v)
    {
        put(&v, sizeof(T));
    }
    template <class T>
    T get()
    {
        T v{};
        get(&v, sizeof(T));
        return v;
    }
    // big-endian 32-bit and 16-bit words (BGEO)
    void put_be32(uint32_t v)
    {
        const unsigned char b[4] = { (unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v };
        put(b, 4);
    }
    void put_be16(uint16_t v)
    {
        const unsigned char b[2] = { (unsigned char)(v >> 8), (unsigned char)v };
        put(b, 2);
    }
    void put_bef(float x)
    {
        uint32_t u;
        std::memcpy(&u, &x, 4);
        put_be32(u);
    }
};

const char STATE_MAGIC[8] = { 'Z', 'M', 'P', 'M', 'S', 'T', 'A', 'T' };

// Per-CTA partial maxima of |v|, x and -x (7 values per CTA).
constexpr int SPEED_THREADS = 256;
__global__ void __launch_bounds__(SPEED_THREADS) k_max_speed(const double* __restrict__ pd, int64_t cap, int64_t P, double* __restrict__ part)
{
    __shared__ double red[7][SPEED_THREADS];
    double m[7];
    m[0] = 0;
    for (int k = 1; k < 7; ++k) m[k] = -(double)FLT_MAX; // numeric_limits<float>::lowest(), as the reference
    for (int64_t s = (int64_t)blockIdx.x * SPEED_THREADS + threadIdx.x; s < P; s += (int64_t)gridDim.x * SPEED_THREADS) {
        double v2 = 0;
        for (int d = 0; d < 3; ++d) {
            const double v = pd[(PD_V + d) * cap + s], x = pd[(PD_X + d) * cap + s];
            v2 += v * v;
            m[1 + d] = fmax(m[1 + d], x);
            m[4 + d] = fmax(m[4 + d], -x);
        }
        m[0] = fmax(m[0], sqrt(v2));
    }
    for (int k = 0; k < 7; ++k) red[k][threadIdx.x] = m[k];
    __syncthreads();
    for (int o = SPEED_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int k = 0; k < 7; ++k) red[k][threadIdx.x] = fmax(red[k][threadIdx.x], red[k][threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x < 7) part[7 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

void rotation_of(const double q[4], double R[9])
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
    const double r[9] = { 1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y), 2 * (x * y + w * z), 1 - 2 * (x * x + z * z),
        2 * (y * z - w * x), 2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y) };
    for (int i = 0; i < 9; ++i) R[i] = r[i];
}

// AnalyticCollisionObject::evalMaxSpeed (CollisionObject.cpp:159-196) at `time`
// against the particles' box [pmin, pmax]; the level-set bounds are those of
// AnalyticLevelSet::getBounds (sphere, box; a half space has none).
int collider_max_speed(const zmpm_collider& c, double time, const double pmin[3], const double pmax[3], double& speed, std::string& err)
{
    const double* om = c.angular_velocity;
    const double* dbdt = c.translation_velocity;
    const double dsdt = c.scale_velocity;
    if (!(dsdt != 0 || std::sqrt(om[0] * om[0] + om[1] * om[1] + om[2] * om[2]) != 0)) {
        speed = std::sqrt(dbdt[0] * dbdt[0] + dbdt[1] * dbdt[1] + dbdt[2] * dbdt[2]);
        return ZMPM_OK;
    }
    double lo[3], hi[3];
    if (c.shape == ZMPM_SPHERE)
        for (int d = 0; d < 3; ++d) {
            lo[d] = c.a[d] - c.radius;
            hi[d] = c.a[d] + c.radius;
        }
    else if (c.shape == ZMPM_BOX)
        for (int d = 0; d < 3; ++d) {
            lo[d] = c.a[d];
            hi[d] = c.b[d];
        }
    else {
        err = "a rotating or scaling half space has no bounds (AnalyticLevelSet::getBounds)";
        return ZMPM_BAD_ARG;
    }
    double R[9], b[3];
    rotation_of(c.rotation, R);
    const double s = c.scale + time * dsdt, one_over_s = 1 / s;
    for (int d = 0; d < 3; ++d) b[d] = c.translation[d] + time * dbdt[d];
    std::vector<std::array<double, 3>> corners;
    for (int i = 0; i < 8; ++i) {
        double x[3], X[3];
        for (int d = 0; d < 3; ++d) x[d] = (i & (1 << d)) ? pmin[d] : pmax[d];
        for (int r = 0; r < 3; ++r) X[r] = (R[r] * (x[0] - b[0]) + R[3 + r] * (x[1] - b[1]) + R[6 + r] * (x[2] - b[2])) * one_over_s;
        bool a = false, bb = false;
        for (int d = 0; d < 3; ++d) {
            a = a || lo[d] < X[d];
            bb = bb || X[d] < hi[d];
        }
        if (a && bb) corners.push_back({ x[0], x[1], x[2] });
    }
    for (int i = 0; i < 8; ++i) {
        double X[3], x[3];
        for (int d = 0; d < 3; ++d) X[d] = (i & (1 << d)) ? lo[d] : hi[d];
        for (int r = 0; r < 3; ++r) x[r] = (R[3 * r] * X[0] + R[3 * r + 1] * X[1] + R[3 * r + 2] * X[2]) * s + b[r];
        bool a = false, bb = false;
        for (int d = 0; d < 3; ++d) {
            a = a || pmin[d] < x[d];
            bb = bb || x[d] < pmax[d];
        }
        if (a && bb) corners.push_back({ x[0], x[1], x[2] });
    }
    speed = 0;
    for (const auto& x : corners) {
        const double xb[3] = { x[0] - b[0], x[1] - b[1], x[2] - b[2] };
        const double v[3] = { om[1] * xb[2] - om[2] * xb[1] + (dsdt * one_over_s) * xb[0] + dbdt[0],
            om[2] * xb[0] - om[0] * xb[2] + (dsdt * one_over_s) * xb[1] + dbdt[1],
            om[0] * xb[1] - om[1] * xb[0] + (dsdt * one_over_s) * xb[2] + dbdt[2] };
        speed = std::max(speed, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
    return ZMPM_OK;
}

} // namespace
} // namespace zmpm

using namespace zmpm;

extern "C" {

int zmpm_write_state(zmpm_ctx* ctx, const char* path)
{
    if (!ctx || !path) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    File f(path, "wb");
    if (!f.ok) {
        ctx->err = std::string("cannot open ") + path;
        return ZMPM_BAD_ARG;
    }
    f.put(STATE_MAGIC, 8);
    f.put<uint32_t>(1);
    f.put<uint32_t>(0x01020304u);
    f.put(ctx->cfg);
    f.put<int64_t>(ctx->P);
    f.put<double>(ctx->time);
    f.put<int32_t>(ctx->pd_active);
    f.put<double>(ctx->pf_M);
    f.put<double>(ctx->pf_delete);
    f.put<double>(ctx->pf_cg_tol);
    f.put<int32_t>(ctx->pf_lumping ? 1 : 0);
    f.put<int32_t>(ctx->pf_cg_max);
    f.put<int32_t>((int32_t)ctx->colliders.size());
    for (const auto& c : ctx->colliders) f.put(c);
    const auto fields = state_fields(ctx);
    f.put<int32_t>((int32_t)fields.size());
    for (const auto& fd : fields) {
        const uint16_t n = (uint16_t)std::strlen(fd.name);
        f.put<uint16_t>(n);
        f.put(fd.name, n);
        f.put<uint8_t>((uint8_t)fd.type);
        f.put<int32_t>(fd.comps);
        f.put(field_data(fd), (size_t)ctx->P * fd.comps * type_size(fd.type));
    }
    if (!f.ok) {
        ctx->err = std::string("write failed: ") + path;
        return ZMPM_BAD_ARG;
    }
    return ZMPM_OK;
}

int zmpm_read_state(zmpm_ctx* ctx, const char* path)
{
    if (!ctx || !path) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    File f(path, "rb");
    if (!f.ok) {
        ctx->err = std::string("cannot open ") + path;
        return ZMPM_BAD_ARG;
    }
    char magic[8];
    f.get(magic, 8);
    const uint32_t version = f.get<uint32_t>(), order = f.get<uint32_t>();
    if (!f.ok || std::memcmp(magic, STATE_MAGIC, 8) != 0 || version != 1 || order != 0x01020304u) {
        ctx->err = "not a version-1 restart file of this byte order";
        return ZMPM_BAD_ARG;
    }
    const zmpm_config cfg = f.get<zmpm_config>();
    if (cfg.dx != ctx->cfg.dx || cfg.grid_log2 != ctx->cfg.grid_log2) {
        ctx->err = "restart file has another dx or grid size";
        return ZMPM_BAD_ARG;
    }
    const int64_t P = f.get<int64_t>();
    const double time = f.get<double>();
    const int32_t pd_active = f.get<int32_t>();
    const double pf_M = f.get<double>(), pf_delete = f.get<double>(), pf_tol = f.get<double>();
    const int32_t pf_lumping = f.get<int32_t>(), pf_max = f.get<int32_t>();
    const int32_t ncol = f.get<int32_t>();
    if (!f.ok || P < 0 || ncol < 0 || ncol > MAX_COLLIDERS || !(pd_active == PD_CORE || pd_active == PD_PF_END || pd_active == PD_FIELDS)) {
        ctx->err = "corrupt restart header";
        return ZMPM_BAD_ARG;
    }
    // the particle index must fit the binning key, as zmpm_add_particles requires
    if (P >= ((int64_t)1 << (ctx->layout == 1 ? Layout244::INDEX_BITS : Layout444::INDEX_BITS))) {
        ctx->err = "particle count exceeds the key's index bits (MpmSimulationBase.cpp:1037-1038)";
        return ZMPM_BAD_ARG;
    }
    // every particle holds at least one byte of every field: P cannot exceed the bytes left
    const long here = std::ftell(f.f);
    if (here < 0 || std::fseek(f.f, 0, SEEK_END) != 0) {
        ctx->err = "restart file is not seekable";
        return ZMPM_BAD_ARG;
    }
    const long end = std::ftell(f.f);
    if (end < here || std::fseek(f.f, here, SEEK_SET) != 0 || P > (int64_t)(end - here)) {
        ctx->err = "restart file is shorter than its particle count";
        return ZMPM_BAD_ARG;
    }
    std::vector<zmpm_collider> cols(ncol);
    for (auto& c : cols) c = f.get<zmpm_collider>();
    // stage the arrays as bytes so that a failed read leaves ctx intact
    const auto fields = state_fields(ctx);
    std::vector<std::vector<unsigned char>> staged(fields.size());
    std::vector<bool> seen(fields.size(), false);
    const int32_t nf = f.get<int32_t>();
    for (int32_t k = 0; k < nf && f.ok; ++k) {
        const uint16_t n = f.get<uint16_t>();
        std::string name(n, '\0');
        f.get(&name[0], n);
        const int type = f.get<uint8_t>();
        const int32_t comps = f.get<int32_t>();
        size_t idx = fields.size();
        for (size_t i = 0; i < fields.size(); ++i)
            if (name == fields[i].name) idx = i;
        if (!f.ok || idx == fields.size() || fields[idx].type != type || fields[idx].comps != comps || seen[idx]) {
            ctx->err = "unknown or mistyped field in restart file: " + name;
            return ZMPM_BAD_ARG;
        }
        seen[idx] = true;
        const size_t bytes = (size_t)P * comps * type_size(type);
        if (bytes > (size_t)(end - here)) {
            ctx->err = "restart file is shorter than its field " + name;
            return ZMPM_BAD_ARG;
        }
        try {
            staged[idx].resize(bytes);
        }
        catch (const std::exception&) {
            ctx->err = "no host memory to stage the restart file";
            return ZMPM_NO_MEMORY;
        }
        f.get(staged[idx].data(), staged[idx].size());
    }
    for (size_t i = 0; i < fields.size(); ++i)
        if (!seen[i]) {
            ctx->err = std::string("restart file lacks field ") + fields[i].name;
            return ZMPM_BAD_ARG;
        }
    if (!f.ok) {
        ctx->err = "truncated restart file";
        return ZMPM_BAD_ARG;
    }
    int rc = begin_edit(ctx);
    if (rc) return rc;
    try {
        for (size_t i = 0; i < fields.size(); ++i) {
            field_resize(fields[i], (size_t)P * fields[i].comps);
            if (!staged[i].empty()) std::memcpy(field_data(fields[i]), staged[i].data(), staged[i].size());
        }
    }
    catch (const std::exception&) {
        ctx->err = "no host memory for the restart file's particles";
        return ZMPM_NO_MEMORY;
    }
    ctx->P = P;
    ctx->time = time;
    ctx->pd_active = pd_active;
    ctx->pf_M = pf_M;
    ctx->pf_delete = pf_delete;
    ctx->pf_cg_tol = pf_tol;
    ctx->pf_lumping = pf_lumping != 0;
    ctx->pf_cg_max = pf_max;
    ctx->colliders = cols;
    ctx->uploaded = false;
    ctx->binned = false;
    ctx->implicit_ready = false;
    return ZMPM_OK;
}

int zmpm_write_bgeo(zmpm_ctx* ctx, const char* path, int32_t fields)
{
    if (!ctx || !path || (fields & ~(ZMPM_BGEO_VELOCITY | ZMPM_BGEO_PHASE_FIELD))) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    int rc = download(ctx);
    if (rc) return rc;
    File f(path, "wb");
    if (!f.ok) {
        ctx->err = std::string("cannot open ") + path;
        return ZMPM_BAD_ARG;
    }
    const bool vel = fields & ZMPM_BGEO_VELOCITY, pf = fields & ZMPM_BGEO_PHASE_FIELD;
    struct Attr {
        const char* name;
        int comps;
    };
    std::vector<Attr> attrs;
    if (vel) attrs.push_back({ "v", 3 });
    if (pf) {
        attrs.push_back({ "pf", 1 });
        attrs.push_back({ "sigmaC", 1 });
    }
    f.put_be32(('B' << 24) | ('g' << 16) | ('e' << 8) | 'o');
    f.put<char>('V');
    f.put_be32(5);
    f.put_be32((uint32_t)ctx->P);
    f.put_be32(0); // primitives
    f.put_be32(0); // point groups
    f.put_be32(0); // primitive groups
    f.put_be32((uint32_t)attrs.size());
    f.put_be32(0); // vertex attributes
    f.put_be32(0); // primitive attributes
    f.put_be32(0); // detail attributes
    for (const auto& a : attrs) {
        const uint16_t n = (uint16_t)std::strlen(a.name);
        f.put_be16(n);
        f.put(a.name, n);
        f.put_be16((uint16_t)a.comps);
        f.put_be32(5); // vector
        for (int i = 0; i < a.comps; ++i) f.put_be32(0);
    }
    for (int64_t i = 0; i < ctx->P; ++i) {
        for (int d = 0; d < 3; ++d) f.put_bef((float)ctx->hx[3 * i + d]);
        f.put_bef(1.0f);
        if (vel)
            for (int d = 0; d < 3; ++d) f.put_bef((float)ctx->hv[3 * i + d]);
        if (pf) {
            const bool has = ctx->hdamage[i] == ZMPM_DAMAGE_PHASE_FIELD;
            // FractureSimulation.h:124-143: c, and sigma_C = 1 / (1 / sigma_C); 1 for particles without a phase field
            f.put_bef(has ? (float)ctx->hpfc[i] : 1.0f);
            f.put_bef(has ? 1.0f / (float)ctx->hpfisc[i] : 1.0f);
        }
    }
    f.put<unsigned char>(0x00);
    f.put<unsigned char>(0xff);
    if (!f.ok) {
        ctx->err = std::string("write failed: ") + path;
        return ZMPM_BAD_ARG;
    }
    return ZMPM_OK;
}

int zmpm_max_particle_speed(zmpm_ctx* ctx, double* speed, double* min_corner, double* max_corner)
{
    if (!ctx) return ZMPM_BAD_ARG;
    cudaSetDevice(ctx->device);
    double m[7];
    m[0] = 0;
    for (int k = 1; k < 7; ++k) m[k] = -(double)FLT_MAX;
    if (ctx->uploaded && ctx->P > 0) {
        const int64_t P = ctx->P;
        const int nb = (int)std::min<int64_t>(1024, (P + SPEED_THREADS - 1) / SPEED_THREADS);
        ZMPM_CUDA(ctx->stage.ensure(7 * nb * sizeof(double)));
        k_max_speed<<<nb, SPEED_THREADS, 0, ctx->stream>>>(ctx->pd.as<double>(), ctx->Pcap, P, ctx->stage.as<double>());
        ++g_kernel_launches;
        std::vector<double> part(7 * nb);
        ZMPM_CUDA(cudaMemcpyAsync(part.data(), ctx->stage.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        ZMPM_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int b = 0; b < nb; ++b)
            for (int k = 0; k < 7; ++k) m[k] = std::max(m[k], part[7 * b + k]);
    }
    else
        for (int64_t i = 0; i < ctx->P; ++i) {
            double v2 = 0;
            for (int d = 0; d < 3; ++d) {
                v2 += ctx->hv[3 * i + d] * ctx->hv[3 * i + d];
                m[1 + d] = std::max(m[1 + d], ctx->hx[3 * i + d]);
                m[4 + d] = std::max(m[4 + d], -ctx->hx[3 * i + d]);
            }
            m[0] = std::max(m[0], std::sqrt(v2));
        }
    if (speed) *speed = m[0];
    for (int d = 0; d < 3; ++d) {
        if (max_corner) max_corner[d] = m[1 + d];
        if (min_corner) min_corner[d] = -m[4 + d];
    }
    return ZMPM_OK;
}

int zmpm_calculate_dt(zmpm_ctx* ctx, double max_dt, double* dt)
{
    if (!ctx || !dt || !(max_dt > 0)) return ZMPM_BAD_ARG;
    double v, lo[3], hi[3];
    int rc = zmpm_max_particle_speed(ctx, &v, lo, hi);
    if (rc) return rc;
    const double grow = (2 + 2) * ctx->cfg.dx; // (interpolation_degree + 2) dx
    for (int d = 0; d < 3; ++d) {
        lo[d] -= grow;
        hi[d] += grow;
    }
    for (const auto& c : ctx->colliders) {
        double sc = 0;
        rc = collider_max_speed(c, ctx->time, lo, hi, sc, ctx->err);
        if (rc) return rc;
        v = std::max(v, sc);
    }
    *dt = v ? ctx->cfg.cfl * ctx->cfg.dx / v : max_dt;
    return ZMPM_OK;
}

// SimulationBase::outputFileName (SimulationBase.h:192-199).
static std::string restart_path(const char* dir, int32_t frame, int32_t substep)
{
    std::string p = std::string(dir) + "/restart_" + std::to_string(frame);
    if (substep > 0) p += "_" + std::to_string(substep);
    return p + ".dat";
}

static bool write_text(const std::string& path, long long v)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    const bool ok = std::fprintf(f, "%lld", v) > 0;
    return (std::fclose(f) == 0) && ok;
}

// The integer in a text file; false when the file is missing or holds none.
static bool read_text(const std::string& path, long long& v)
{
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    const bool ok = std::fscanf(f, "%lld", &v) == 1;
    std::fclose(f);
    return ok;
}

int zmpm_write_restart(zmpm_ctx* ctx, const char* output_dir, int32_t frame, int32_t substep)
{
    if (!ctx || !output_dir || frame < 0 || substep < 0) return ZMPM_BAD_ARG;
    struct stat sb;
    if (stat(output_dir, &sb) != 0) {
        if (mkdir(output_dir, 0755) != 0 && errno != EEXIST) {
            ctx->err = std::string("cannot create ") + output_dir;
            return ZMPM_BAD_ARG;
        }
    }
    else if (!S_ISDIR(sb.st_mode)) {
        ctx->err = std::string(output_dir) + " is not a directory";
        return ZMPM_BAD_ARG;
    }
    int rc = zmpm_write_state(ctx, restart_path(output_dir, frame, substep).c_str());
    if (rc) return rc;
    const std::string d(output_dir);
    if (!write_text(d + "/last_written.txt", frame) || !write_text(d + "/binary_ver.txt", ZMPM_BINARY_VER)) {
        ctx->err = "cannot write last_written.txt / binary_ver.txt in " + d;
        return ZMPM_BAD_ARG;
    }
    return ZMPM_OK;
}

int zmpm_read_restart(zmpm_ctx* ctx, const char* output_dir, int32_t frame, int32_t substep, int32_t* last_written_frame)
{
    if (!ctx || !output_dir || frame < 0 || substep < 0) return ZMPM_BAD_ARG;
    const std::string d(output_dir);
    long long ver = 0, last = -1;
    if (!read_text(d + "/binary_ver.txt", ver)) ver = 0; // as the reference: a missing version file reads as 0
    if (ver > ZMPM_BINARY_VER) {
        ctx->err = "the restart data is of binary version " + std::to_string(ver) + ", newer than this library's " +
                   std::to_string(ZMPM_BINARY_VER);
        return ZMPM_BAD_ARG;
    }
    if (!read_text(d + "/last_written.txt", last)) last = -1;
    if (last_written_frame) *last_written_frame = (int32_t)last;
    return zmpm_read_state(ctx, restart_path(output_dir, frame, substep).c_str());
}

} // extern "C"
