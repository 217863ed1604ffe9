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
// BGEO (Houdini binary geometry, version 5, big-endian) with points only:
//   int32 magic 'Bgeo', char 'V', int32 5, int32 points, primitives (0), point
//   groups (0), primitive groups (0), point attributes, vertex attributes (0),
//   primitive attributes (0), detail attributes (0); per point attribute:
//   uint16 name length, name, uint16 components, int32 type (5: vector),
//   components x int32 default (0); per point: x, y, z, w = 1, then the
//   attribute floats; trailer bytes 0x00 0xff.
#include <cstdio>
#include <cstring>
#include <string>
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
        staged[idx].resize((size_t)P * comps * type_size(type));
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
    for (size_t i = 0; i < fields.size(); ++i) {
        field_resize(fields[i], (size_t)P * fields[i].comps);
        if (!staged[i].empty()) std::memcpy(field_data(fields[i]), staged[i].data(), staged[i].size());
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

} // extern "C"
