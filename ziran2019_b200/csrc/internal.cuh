// Context and launch interface shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/zmpm.h"
#include "common.cuh"

namespace zmpm {

// Kernels launched by this library on the calling host thread (reported per
// substep in zmpm_stats.kernel_launches).
extern thread_local int64_t g_kernel_launches;

// ------------------------------------------------------------ primitives --
int64_t scan_scratch_elems(int64_t n);
template <class T>
void exclusive_scan(const T* in, T* out, int64_t n, T* total, T* scratch, cudaStream_t st);
int64_t radix_scratch_elems(int64_t n);
uint64_t* radix_sort(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int nbits, int32_t* scratch, cudaStream_t st);

// ---------------------------------------------------------- device buffer --
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    cudaError_t ensure(size_t n)
    {
        if (n <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t want = n + n / 4 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) bytes = want;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// Counters the device writes and the host reads once per substep.
struct DevCounters {
    int64_t G, B, N;           // groups, pages, active nodes
    int32_t flags;             // FLAG_*
    int32_t pad;
    int64_t first_not_max;     // Rankine (reference order): particles whose first eigenvalue is not the largest
    int64_t svd_fp64;          // MIXED: FP32 constitutive updates redone in FP64 (near-degenerate singular values)
};

// Scalar state of the Newton / Krylov loop, kept on the device so no host
// round trip is needed inside a solve.  Double-buffered where a kernel's CTAs
// read the previous value while CTA 0 writes the next one.
struct SolverScalars {
    int32_t newton_done;       // 1 once the Newton norm fell below tolerance (or NaN)
    int32_t kactive;           // 1 while the current linear solve iterates
    int32_t kit;               // Krylov iteration index of the current linear solve
    int32_t nit;               // Newton iteration index (= Newton loop bodies run)
    int32_t krylov_bodies;     // Krylov loop bodies run (graph launch accounting)
    uint32_t ticket;           // CTAs of the running kernel that finished (last_cta); 0 between kernels
    int32_t newton_iters;      // linear solves run
    int32_t krylov_iters;      // summed Krylov iterations
    int32_t hvp_count;
    int32_t converged;
    int32_t fp64_res;          // MIXED: 1 once the Newton residual is evaluated in FP64 (its FP32 form stalled)
    int32_t skip_step;         // 1: this Newton iteration takes no step (the residual is re-evaluated first)
    int32_t kcount[64];        // Krylov iterations of each Newton iteration
    double res_initial, res_final;
    double rel_tol, local_tol;
    double rnorm;              // current preconditioned residual norm of the linear solve
    // CG
    double zTrk;
    // MINRES (Minres.h:16-24), double buffered by iteration parity
    double mr[2][12];
    // delta, epsilon, gamma, t and beta of the last MINRES iteration: its
    // search direction and x update run in the next operator pass (or at the
    // solve's end)
    double pend[5];
};
enum MinresSlot { MR_GC0, MR_GS0, MR_GC1, MR_GS1, MR_GC2, MR_GS2, MR_RHS0, MR_RHS1, MR_BETA_KP1 };

// State of the bounded grid-wide barrier of a persistent (cooperative) kernel,
// zeroed before each launch.
struct GridSync {
    unsigned count;  // CTAs arrived at the current barrier
    unsigned pad0[31];
    unsigned gen;    // barriers completed (polled by the waiting CTAs, on its own 128-byte line)
    unsigned abort;  // 1 once a CTA's wait gave up
    unsigned pad1[30];
};

// Field indices of the particle pools.
// Fields from PD_CORE on (phase-field state, then viscoelastic strain and ADMM
// state) are moved by the binning permutation only once a context uses them
// (Ctx::pd_active: PD_CORE, PD_PF_END or PD_FIELDS).
// Plasticity parameters by kind: von Mises PD_YS = yield stress, PD_XI = xi,
// PD_FS = fail stress, PI_BROKEN = broken; Drucker-Prager PD_YS = alpha,
// PD_XI = beta, PD_FS = cohesion, PI_BROKEN = volume_correction; Cam-Clay
// PD_YS = M, PD_XI = beta, PD_FS = xi, PI_BROKEN = hardeningOn.  PD_LOGJP is
// log Jp of the last two.
enum PdField { PD_X = 0, PD_V = 3, PD_C = 6, PD_F = 15, PD_M = 24, PD_VOL = 25, PD_MU = 26, PD_LAM = 27, PD_KAPPA = 28,
    PD_G = 29, PD_YS = 30, PD_XI = 31, PD_FS = 32, PD_CRACK = 33, PD_PF_C = 36, PD_PF_K = 37, PD_SIGMA_F = 38, PD_LOGJP = 39, PD_CORE = 40,
    PD_PF_H = 40, PD_PF_L0 = 41, PD_PF_ISC = 42, PD_PF_FP = 43, PD_PF_HMAX = 44, PD_PF_VOL = 45, PD_PF_ALLOW = 46, PD_PF_END = 47,
    PD_FE = 47, PD_VMU = 56, PD_VLAM = 57, PD_VD = 58, PD_VV = 59, PD_Y = 60, PD_OMEGA = 78, PD_LASTDV = 80, PD_FIELDS = 83 };
enum PiField { PI_KIND = 0, PI_PKIND = 1, PI_BROKEN = 2, PI_ID = 3, PI_DAMAGE = 4, PI_VISCO = 5, PI_FIELDS = 6 };

// Adjoint particle arrays [AJ_FIELDS][Pcap] (FP64, slot order): the state
// before the substep (same field order as the pool's first 24 fields), the
// incoming gradients and the outgoing ones.
enum AdjField { AJ_X0 = 0, AJ_V0 = 3, AJ_C0 = 6, AJ_F0 = 15, AJ_GX = 24, AJ_GV = 27, AJ_GC = 30, AJ_GF = 39, AJ_OX = 48, AJ_OV = 51,
    AJ_OC = 54, AJ_OF = 63, AJ_OE = 72, AJ_FIELDS = 73 };

// Reduction slots: per-CTA partial sums written by node kernels.
constexpr int RED_MAX_CTAS = 1024;
enum RedSlot { RED_A = 0, RED_B = 1, RED_C = 2, RED_N = 3 };

struct Ctx {
    zmpm_config cfg;
    int layout = 1;            // 1: 2x4x4 pages, 2: 4x4x4 pages
    bool mixed = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    double time = 0;

    // grid extent
    int grid_log2 = 10;
    int pages[3] = { 0, 0, 0 }; // pages per axis
    int64_t table_size = 0;
    int key_bits = 0;           // significant key bits above the particle index

    // host copy of the scene until the first upload
    int64_t P = 0;
    bool uploaded = false;
    std::vector<double> hx, hv, hC, hF, hcrack, hm, hvol, hmu, hlam, hkappa, hg, hys, hxi, hfs, hpfc, hpfk, hsigf, hlogjp;
    std::vector<uint8_t> hkind, hpkind, hdamage, hvisco;
    std::vector<int32_t> hbroken;
    std::vector<double> hFe, hvmu, hvlam, hvd, hvv, hy, homega, hlastdv; // viscoelastic + ADMM state
    std::vector<double> hpfH, hpfl0, hpfisc, hpffp, hpfhmax, hpfvol, hpfallow; // phase-field state (PhaseField.h:13-22)
    // FractureSimulation members of the phase-field solve (FractureSimulation.h:48-63)
    double pf_M = 0, pf_delete = 0, pf_cg_tol = 1e-6;
    bool pf_lumping = true;
    int pf_cg_max = 100;
    bool has_pf = false;
    bool all_pf = false;
    int32_t pf_iters = 0;   // CG iterations and final |r| of the last phase-field solve
    double pf_res = 0;
    DBuf pfn;   // phase-field node arrays [B][PN_FIELDS][NPB]
    DBuf pfsc;  // PfScalars of the phase-field CG
    bool has_damage = false;
    bool has_visco = false;
    bool mls = false;                     // the running explicit substep uses MLS-MPM (G2P gradV = C)
    int fp64_res_run = 0;                 // MIXED: consecutive Newton solves that needed the FP64 residual; while
                                          // nonzero the next solve starts with it, except every 16th (an FP32 retry)
    bool all_models = true;               // every particle has an F-based model
    int pd_active = PD_CORE;              // pd fields the binning permutation moves
    std::vector<zmpm_collider> colliders;

    // particles in slot order, structure of arrays (capacity Pcap).  The
    // double fields live in one pool [PD_FIELDS][Pcap] and the integer fields
    // in another, so the binning permutation moves all state in one kernel.
    int64_t Pcap = 0;
    DBuf pd, pd_alt, pi, pi_alt;
    DBuf slot_of_id;   // particle index -> slot
    DBuf base_by_id;   // short4 base node per particle index (binning)
    DBuf base;         // short4 base node per slot
    DBuf Fn;           // [9][Pcap] F at the start of the Newton solve
    DBuf scratch;      // Hessian scratch [NS][Pcap] in the HVP precision
    DBuf stress;       // [9][Pcap] V0 P(F) Fn^T of the current Newton iterate
    cudaGraphExec_t graph_exec = nullptr; // last solve graph, released when the next one is launched
    bool graph_used = false;              // the last Newton solve ran as a graph
    DBuf frac;         // [3][Pcap] fractional offsets in cells (FP32 HVP)
    double* pdf(int f) const { return pd.as<double>() + (int64_t)f * Pcap; }
    int32_t* pif(int f) const { return pi.as<int32_t>() + (int64_t)f * Pcap; }

    // binning
    DBuf keys, keys_alt, flags_i32, scan_i32, scan_scr, radix_scr;
    DBuf group_start, group_page, group_nbr, emit_flag, emit_scan;
    DBuf page_first, page_block;          // dense page tables
    DBuf block_page, block_index;         // per page: packed coords, page index
    int64_t G = 0, B = 0, N = 0;
    bool binned = false;

    // grid, block-dense: scalars [B][NPB], vectors [B][3][NPB]
    DBuf gm, gmv, vn, dv, vstar, facc, res, proj, collided, node_idx;
    // Krylov vectors
    DBuf kv[10];
    DBuf vstarf;                          // MIXED: FP32 node-major copy of vstar ([B][NPB][4]), the particle kernels' gather input
    bool vstarf_valid = false;            // vstarf holds the current vstar (the Newton solve keeps it; other integrators refresh it)
    DBuf kvf;                             // FP32 node-major copies of MINRES's two Z vectors ([2][B][NPB][4]), read by the FP32 product
    DBuf red;                             // reduction partials [4][RED_MAX_CTAS]
    DBuf scal;                            // SolverScalars
    DBuf counters;                        // DevCounters
    DBuf dcolliders;
    DevCounters hcounters;
    bool implicit_ready = false;
    bool scratch_valid = false;
    bool profiling = false;
    std::vector<cudaEvent_t> hvp_ev;      // [newton][krylov][2] when profiling
    int prof_newton = 0;
    DBuf stage;                           // host <-> device particle transfers
    double dt = 0;

    // ADMM (per substep): local variables F, Fe [18][Pcap]; grad vn [9][Pcap];
    // global-operator coefficients B [6][Pcap] (HVP precision); node
    // preconditioner, right-hand side and transfer weights
    DBuf adm_F, adm_gvn, adm_B, adm_pre, adm_rhs, adm_w;
    DBuf adj;                             // adjoint particle arrays [AJ_FIELDS][Pcap]
    std::vector<DBuf> ckpt_pd, ckpt_pi, ckpt_sid; // device checkpoints
    std::vector<double> ckpt_time;
    std::vector<int64_t> ckpt_P;
    bool admm_used = false;               // the last substep ran ADMM (launch accounting)
    DBuf gsync;                           // GridSync of the persistent Krylov kernels
    std::map<const void*, int> coop_blocks; // cooperative grid size of each persistent kernel (all CTAs co-resident)
    long long spin_limit = 1ll << 22;     // polls before a grid-barrier wait gives up (zmpm_set_spin_limit)
    // substep phases: 1 after zmpm_particles_to_grid, 2 after zmpm_backward_euler_step
    int phase = 0;
    zmpm_solver phase_solver{};
    int64_t phase_launches0 = 0;
    int admm_iters = 0;

    int npb() const { return layout == 1 ? 32 : 64; }
};

#define ZMPM_CUDA(expr)                                                                            \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            ctx->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                         \
            return ZMPM_CUDA_ERROR;                                                                \
        }                                                                                          \
    } while (0)

// ---------------------------------------------------------------- passes --
int run_binning(Ctx* ctx);
int run_p2g(Ctx* ctx, bool damage = true);            // P2G (+ damage hook) + grid normalisation + Newton setup
int run_newton(Ctx* ctx, const zmpm_solver& s);       // backward-Euler Newton
int run_g2p(Ctx* ctx, bool plastic = true);            // G2P + evolveStrain (+ applyPlasticity)
int refresh_vstar_f32(Ctx* ctx);                       // MIXED: vstarf from vstar
int launch_plasticity(Ctx* ctx);                       // applyPlasticity alone
int upload_colliders(Ctx* ctx, double time, int slot = 0);    // slot 1: the state at t + dt
int upload(Ctx* ctx);      // host scene arrays -> device pools (once per edit)
int download(Ctx* ctx);    // device pools -> host scene arrays (particle order)
int begin_edit(Ctx* ctx);  // download, then mark the device copy stale
int run_explicit(Ctx* ctx, const zmpm_solver& s);      // symplectic substep up to G2P
int launch_explicit_stress(Ctx* ctx);
int run_phase_field(Ctx* ctx, int32_t* iterations, double* residual); // FractureSimulation::solvePhaseFieldSystem after P2G
int launch_phase_field_delete(Ctx* ctx);                               // FractureSimulation::deleteParticles before binning                  // V0 tau(F) (+ V0 tau(Fe)) into the stress buffer
int launch_update(Ctx* ctx, bool gated = true);       // G2P(vn+dv) -> stress -> force P2G
int launch_adj_g2p(Ctx* ctx, double* vsbar);           // adjoint of G2P (adjoint.cu)
int launch_adj_particle(Ctx* ctx, const double* lam);  // adjoint of the force term, P2G and E
int run_adjoint_solve(Ctx* ctx, double tol, int max_iterations); // (M + dt^2 K) lambda = P dL/dv*
int launch_residual(Ctx* ctx);                         // r = dt m g + dt f - m dv (projected), norm partials
int launch_hvp(Ctx* ctx, const double* x, double* out, bool fp32); // out += dt^2 K x (no inertia)
// FP32 product inside the MINRES loop of a MIXED context, on the FP32 copies x0 / x1 (even / odd iterations)
int launch_damage(Ctx* ctx);                           // Rankine damage after P2G
int run_admm(Ctx* ctx, const zmpm_solver& s);         // AdmmSimulation::admmStep
// particle kernels of the ADMM substep (admm.cu)
int launch_admm_dvinit(Ctx* ctx);                      // scatter last_dv w and w
int launch_admm_init(Ctx* ctx, double rho);            // local variables, omega, y rescale, B
int launch_admm_pre(Ctx* ctx);                         // preconditioner += grad w^T B grad w
int launch_admm_local(Ctx* ctx, double rho, double local_tol); // F step + rhs stress
int launch_admm_op(Ctx* ctx, const double* x, double* out); // out += sum (grad x B) grad w
int launch_admm_dual(Ctx* ctx, double rho);            // y += rho omega (F - (I + dt grad v) Fn)
int launch_admm_lastdv(Ctx* ctx);                      // last_dv = sum dv w / (dt sum w)
int launch_force_scatter(Ctx* ctx, double* out, bool mls = false);       // out -= sum_p stress_p grad w_ip (stress buffer)
int finalize_multiply(Ctx* ctx, const double* x, double* q); // q = project(m x + q)
int ensure_node_buffers(Ctx* ctx);
int compute_node_indices(Ctx* ctx);                    // getNumNodes numbering (hooks)

} // namespace zmpm

struct zmpm_ctx : zmpm::Ctx {};
