// Internal to the library: the solver object, error handling, launchers and
// drivers shared by the C-ABI translation units (capi.cu, mixed.cu).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>  // header-only; a no-op unless a profiler attaches

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/gato_b200.h"
#include "adjoint.cuh"
#include "kernels.cuh"
#include "multi.cuh"
#include "pcg_cluster.cuh"
#include "rollout.cuh"
#include "plant_tables.h"

using namespace gato;

// message of the last failure on this thread (gato_last_error)
extern thread_local std::string g_err;

namespace {

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(GATO_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                 \
    } while (0)

#define CKL()                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            return fail(GATO_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                   \
    } while (0)

#define RC(x)                \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

// ---------------------------------------------------------------------------
// host model construction in FP64: the same rules as the FP64 oracle,
// including zeroing transform entries below 1e-6, which reproduces the
// reference's generated tables.
constexpr double SNAP = 1e-6;

void rpy_R(const double* rpy, double* R)
{
    const double cr = cos(rpy[0]), sr = sin(rpy[0]), cp = cos(rpy[1]), sp = sin(rpy[1]),
                 cy = cos(rpy[2]), sy = sin(rpy[2]);
    // Rz(y) Ry(p) Rx(r)
    R[0] = cy * cp;
    R[1] = cy * sp * sr - sy * cr;
    R[2] = cy * sp * cr + sy * sr;
    R[3] = sy * cp;
    R[4] = sy * sp * sr + cy * cr;
    R[5] = sy * sp * cr - cy * sr;
    R[6] = -sp;
    R[7] = cp * sr;
    R[8] = cp * cr;
}

template <int NQ, typename T>
void build_dev_model(const gato_model_t& m, DevModel<NQ, T>* out)
{
    memset(out, 0, sizeof(*out));
    for (int i = 0; i < NQ; ++i) {
        double R[9], E[9], C[9];
        rpy_R(m.joint_rpy[i], R);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) E[3 * r + c] = R[3 * c + r];
        const double* p = m.joint_xyz[i];
        const double px[9] = {0, -p[2], p[1], p[2], 0, -p[0], -p[1], p[0], 0};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double s = 0;
                for (int k = 0; k < 3; ++k) s += E[3 * r + k] * px[3 * k + c];
                C[3 * r + c] = -s;
            }
        for (int k = 0; k < 9; ++k) {
            out->E0[i][k] = (T)(fabs(E[k]) < SNAP ? 0.0 : E[k]);
            out->C0[i][k] = (T)(fabs(C[k]) < SNAP ? 0.0 : C[k]);
            out->R0[i][k] = (T)(fabs(R[k]) < SNAP ? 0.0 : R[k]);
        }
        for (int k = 0; k < 3; ++k) out->P[i][k] = (T)p[k];
        double Ib[6] = {0, 0, 0, 0, 0, 0}, h[3] = {0, 0, 0}, mass = 0;
        for (int bdy = 0; bdy < 2; ++bdy) {
            const double* bd = m.link_inertial[i][bdy];
            const double mm = bd[0];
            if (mm == 0.0) continue;
            const double cx = bd[1], cy = bd[2], cz = bd[3];
            const double c2 = cx * cx + cy * cy + cz * cz;
            Ib[0] += bd[4] + mm * (c2 - cx * cx);
            Ib[1] += bd[5] - mm * cx * cy;
            Ib[2] += bd[6] - mm * cx * cz;
            Ib[3] += bd[7] + mm * (c2 - cy * cy);
            Ib[4] += bd[8] - mm * cy * cz;
            Ib[5] += bd[9] + mm * (c2 - cz * cz);
            h[0] += mm * cx;
            h[1] += mm * cy;
            h[2] += mm * cz;
            mass += mm;
        }
        for (int k = 0; k < 6; ++k) out->Ibar[i][k] = (T)Ib[k];
        for (int k = 0; k < 3; ++k) out->h[i][k] = (T)h[k];
        out->mass[i] = (T)mass;
        const double mg = m.limit_margin;
        out->qlo[i] = (T)(-m.q_limit[i] - mg);
        out->qhi[i] = (T)(m.q_limit[i] + mg);
        out->vlo[i] = (T)(-m.qd_limit[i] - mg);
        out->vhi[i] = (T)(m.qd_limit[i] + mg);
        out->ulo[i] = (T)(-m.u_limit[i] - mg);
        out->uhi[i] = (T)(m.u_limit[i] + mg);
    }
    out->gravity = (T)m.gravity;
    out->barrier_style = m.barrier_style;
}

// The dynamic shared-memory limit is a per-kernel attribute shared by every
// solver on the device, so it is always raised to the device's opt-in
// maximum: a solver with a small N must not lower it below what a solver
// with a larger N already relies on.
template <class K>
int set_smem(K kernel, size_t bytes, int device_limit)
{
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, kernel));
    const int dyn_limit = device_limit - (int)fa.sharedSizeBytes;  // minus static shared memory
    if (bytes > (size_t)dyn_limit)
        return fail(GATO_ERR_UNSUPPORTED, "kernel needs %zu bytes of shared memory, device has %d",
                    bytes, dyn_limit);
    if (bytes > 48 * 1024)
        CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_limit));
    return GATO_OK;
}

// (joints, scalar, reduction scalar) of a solver instance
template <int NQ_, typename T_, typename Acc_>
struct Tag {
    static constexpr int NQ = NQ_;
    using T = T_;
    using Acc = Acc_;
};

}  // namespace

// ===========================================================================
struct gato_solver {
    int nq = 0, N = 0, B = 0, form = 0, precision = 0, device = 0;
    size_t esz = 4;  // bytes of the solver scalar
    gato_model_t model;
    gato_params_t params;
    double dt = 0.01;
    int adapt_rho = 1;
    int use_fext = 0;
    void* wdiag = nullptr;  // [B][nx+nu] diagonal cost weights, allocated on first use
    int use_wdiag = 0;
    int max_smem = 0;
    int nsm = 148;  // SMs of the device
    // device memory, scalar-typed buffers as raw pointers
    void *xu = nullptr, *xs = nullptr, *goal = nullptr, *fext = nullptr;
    void *Q = nullptr, *R = nullptr, *q = nullptr, *r = nullptr, *A = nullptr, *Bm = nullptr,
         *c = nullptr, *Qi = nullptr, *Ri = nullptr;
    void *S = nullptr, *P = nullptr, *gamma = nullptr, *lambda = nullptr, *dz = nullptr;
    void *rho = nullptr, *drho = nullptr, *mu = nullptr, *tol = nullptr, *drho_init_d = nullptr;
    void *sim_x = nullptr, *sim_u = nullptr, *sim_out = nullptr;
    double *merit_terms = nullptr, *merit_init = nullptr, *merit_init0 = nullptr,
           *merit_final = nullptr;
    int *pcg_iters = nullptr, *conv = nullptr, *sqp_iters = nullptr, *done = nullptr,
        *ls_count = nullptr, *h_pcg = nullptr, *status = nullptr;
    int* work = nullptr;  // [4]: counters and wait flag of the persistent PCG
    int wait_tries = PCG_STAGE_WAIT_TRIES, wait_tries_dz = PCG_STAGE_WAIT_TRIES;
    int p32 = 0;  // FP64 solvers: apply P^-1 in FP32 (gato_set_fp32_preconditioner)
    float *h_ls_min = nullptr, *h_ls_step = nullptr;
    // adjoint work buffers, allocated by the first gato_adjoint call
    void *adj_lam = nullptr, *adj_mu = nullptr, *adj_v = nullptr, *adj_scale = nullptr,
         *adj_tol = nullptr;
    int *adj_conv = nullptr, *adj_done = nullptr, *adj_iters = nullptr;
    // rollout work buffers, allocated by the first gato_rollout* call
    void *rl_goal = nullptr, *rl_gx = nullptr, *rl_ga = nullptr, *rl_gu = nullptr,
         *rl_dl = nullptr, *rl_gxs = nullptr, *rl_ggoal = nullptr, *rl_gw = nullptr,
         *rl_rho = nullptr;
    cudaGraphExec_t rexec = nullptr;  // forward rollout graph
    std::vector<const void*> rkey;
    int rver = -1;
    // host
    std::vector<double> rho_init, drho_init;
    int* pin_i = nullptr;  // pinned host ints (B)
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // fused-form graph cache
    cudaGraphExec_t gexec = nullptr;
    const void* gkey[4] = {nullptr, nullptr, nullptr, nullptr};
    int gver = -1;
    int version = 0;  // bumped when a value baked into kernel arguments changes
    std::vector<void*> allocs;
    alignas(16) unsigned char dev_model[sizeof(DevModel<8, double>)];
    // optional per-launch event timing (never during graph capture)
    struct ProfEntry {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<ProfEntry>* prof = nullptr;

    int alloc_bytes(void** p, size_t bytes)
    {
        void* v = nullptr;
        bytes = std::max<size_t>(bytes, 16);
        CK(cudaMalloc(&v, bytes));
        CK(cudaMemset(v, 0, bytes));
        allocs.push_back(v);
        *p = v;
        return GATO_OK;
    }
    template <class U>
    int alloc(U** p, size_t count)
    {
        return alloc_bytes((void**)p, count * sizeof(U));
    }
    int alloc_t(void** p, size_t count) { return alloc_bytes(p, count * esz); }
    // host scalar array -> device scalar array
    int upload(void* dst, const double* src, size_t n)
    {
        if (esz == sizeof(double)) {
            CK(cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice));
        } else {
            std::vector<float> t(src, src + n);
            CK(cudaMemcpy(dst, t.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        }
        return GATO_OK;
    }
};

namespace {

template <class F>
int dispatch(gato_solver* s, F&& f)
{
    if (s->nq == 7) {
        if (s->precision == GATO_PREC_FP64) return f(Tag<7, double, double>());
        if (s->precision == GATO_PREC_MIXED) return f(Tag<7, float, double>());
        return f(Tag<7, float, float>());
    }
    if (s->precision == GATO_PREC_FP64) return f(Tag<6, double, double>());
    if (s->precision == GATO_PREC_MIXED) return f(Tag<6, float, double>());
    return f(Tag<6, float, float>());
}

template <class Tg>
Batch<Tg::NQ, typename Tg::T> make_batch(gato_solver* s, void* xu, const void* xs, const void* goal)
{
    using T = typename Tg::T;
    Batch<Tg::NQ, T> b;
    b.B = s->B;
    b.N = s->N;
    b.solve_ratio = (float)s->params.solve_ratio;
    b.max_pcg_iters = s->params.max_pcg_iters;
    b.abs_tol = 1e-6f;
    b.adapt_rho = s->adapt_rho;
    b.cp.dt = (T)s->dt;
    b.cp.q_cost = (T)s->params.q_cost;
    b.cp.qd_cost = (T)s->params.qd_cost;
    b.cp.u_cost = (T)s->params.u_cost;
    b.cp.N_cost = (T)s->params.N_cost;
    b.cp.q_lim_cost = (T)s->params.q_lim_cost;
    b.cp.vel_lim_cost = (T)s->params.vel_lim_cost;
    b.cp.ctrl_lim_cost = (T)s->params.ctrl_lim_cost;
    b.xu = (T*)xu;
    b.xs = (const T*)xs;
    b.goal = (const T*)goal;
    b.fext = (const T*)s->fext;
    b.use_fext = s->use_fext;
    b.cp.wdiag = s->use_wdiag ? (const T*)s->wdiag : nullptr;
    b.Q = (T*)s->Q;
    b.R = (T*)s->R;
    b.q = (T*)s->q;
    b.r = (T*)s->r;
    b.A = (T*)s->A;
    b.Bm = (T*)s->Bm;
    b.c = (T*)s->c;
    b.Qi = (T*)s->Qi;
    b.Ri = (T*)s->Ri;
    b.S = (T*)s->S;
    b.P = (T*)s->P;
    b.gamma = (T*)s->gamma;
    b.lambda = (T*)s->lambda;
    b.dz = (T*)s->dz;
    b.rho = (T*)s->rho;
    b.drho = (T*)s->drho;
    b.mu = (T*)s->mu;
    b.tol = (T*)s->tol;
    b.merit_terms = s->merit_terms;
    b.merit_init = s->merit_init;
    b.merit_init0 = s->merit_init0;
    b.merit_final = s->merit_final;
    b.pcg_iters = s->pcg_iters;
    b.conv = s->conv;
    b.sqp_iters = s->sqp_iters;
    b.done = s->done;
    b.work = s->work;
    b.ls_count = s->ls_count;
    b.status = s->status;
    b.wait_tries = s->wait_tries;
    b.wait_tries_dz = s->wait_tries_dz;
    b.h_pcg = s->h_pcg;
    b.h_ls_min = s->h_ls_min;
    b.h_ls_step = s->h_ls_step;
    return b;
}

constexpr int WPB = 4;  // warps per block of the per-knot kernels
constexpr int PCG_THREADS = 256;
constexpr int FUSED_THREADS = 256;
constexpr int LS_THREADS = 128;

inline int cdiv(int a, int b) { return (a + b - 1) / b; }

// An NVTX range over a host scope (solve, SQP iteration, stage launch): the
// stage structure shows in Nsight timelines.  Graph replays run no host code,
// so there the ranges mark the capture.
struct Nvtx {
    explicit Nvtx(const char* name) { nvtxRangePushA(name); }
    ~Nvtx() { nvtxRangePop(); }
    Nvtx(const Nvtx&) = delete;
    Nvtx& operator=(const Nvtx&) = delete;
};

const char* const KERNEL_GROUP_NAMES[GATO_KERNEL_COUNT] = {
    "kkt", "schur", "pcg", "dz", "merit", "line_search", "fused_iter", "check", "merit_sum"};

// Brackets one launch with an NVTX range named by its kernel group, and with
// events when profiling is on.
struct ProfScope {
    gato_solver* s;
    cudaStream_t st;
    int id;
    Nvtx range;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(gato_solver* s_, cudaStream_t st_, int id_)
        : s(s_), st(st_), id(id_), range(KERNEL_GROUP_NAMES[id_])
    {
        if (!s->prof) return;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, st);
    }
    ~ProfScope()
    {
        if (!s->prof) return;
        cudaEventRecord(b, st);
        s->prof->push_back({id, a, b});
    }
};

template <class Tg>
const DevModel<Tg::NQ, typename Tg::T>& dmodel(gato_solver* s)
{
    return *reinterpret_cast<const DevModel<Tg::NQ, typename Tg::T>*>(s->dev_model);
}

template <class Tg>
bool pcg_stage_fits(gato_solver* s)
{
    return pcg_smem_bytes<Tg::NQ, typename Tg::T>(s->N, true) <= (size_t)s->max_smem;
}

template <class Tg>
bool fused_stage_fits(gato_solver* s)
{
    FusedLayout<Tg::NQ, typename Tg::T> lay{s->N, FUSED_THREADS / WARP, true};
    return lay.bytes() <= (size_t)s->max_smem;
}

// --- stage launchers ---------------------------------------------------------
template <class Tg>
int launch_merit(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                 int nalpha, int use_dz, int skip)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    ProfScope ps_(s, st, GATO_KERNEL_MERIT);
    const size_t sm = WPB * MeritSmem<NQ>::SIZE * sizeof(T);
    dim3 grid(cdiv(s->N * nalpha, WPB), s->B);
    k_merit<NQ, T><<<grid, WPB * WARP, sm, st>>>(bt, dmodel<Tg>(s), nalpha, use_dz, skip);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_merit_sum(gato_solver* s, cudaStream_t st, double* out, double* out2)
{
    ProfScope ps_(s, st, GATO_KERNEL_MERIT_SUM);
    k_merit_sum<typename Tg::Acc><<<cdiv(s->B, 128), 128, 0, st>>>(s->B, s->N, s->merit_terms,
                                                                    out, out2, s->status);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_kkt(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    ProfScope ps_(s, st, GATO_KERNEL_KKT);
    const size_t sm = WPB * KktSmem<NQ>::SIZE * sizeof(T);
    k_kkt<NQ, T><<<dim3(cdiv(s->N - 1, WPB), s->B), WPB * WARP, sm, st>>>(bt, dmodel<Tg>(s));
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_schur(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    ProfScope ps_(s, st, GATO_KERNEL_SCHUR);
    k_schur_inv<NQ, T><<<dim3(cdiv(s->N, WPB), s->B), WPB * WARP, 0, st>>>(bt);
    CKL();
    const size_t sm = WPB * SchurSmem<NQ>::SIZE * sizeof(T);
    k_schur<NQ, T><<<dim3(cdiv(s->N, WPB), s->B), WPB * WARP, sm, st>>>(bt);
    CKL();
    const size_t sm2 = WPB * 4 * (2 * NQ) * (2 * NQ) * sizeof(T);
    k_schur_off<NQ, T><<<dim3(cdiv(s->N - 1, WPB), s->B), WPB * WARP, sm2, st>>>(bt);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_pcg(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt, int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    ProfScope ps_(s, st, GATO_KERNEL_PCG);
    const bool stage = pcg_stage_fits<Tg>(s);
    const size_t sm = pcg_smem_bytes<NQ, T>(s->N, stage);
    k_pcg<NQ, T, typename Tg::Acc><<<s->B, PCG_THREADS, sm, st>>>(bt, stage, row);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_dz(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    ProfScope ps_(s, st, GATO_KERNEL_DZ);
    const size_t sm = WPB * 3 * (2 * NQ) * sizeof(T);
    k_dz<NQ, T><<<dim3(cdiv(s->N, WPB), s->B), WPB * WARP, sm, st>>>(bt);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_ls(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt, int row,
              int skip)
{
    ProfScope ps_(s, st, GATO_KERNEL_LINE_SEARCH);
    k_line_search<Tg::NQ, typename Tg::T, typename Tg::Acc><<<s->B, LS_THREADS, 0, st>>>(bt, row,
                                                                                      skip);
    CKL();
    return GATO_OK;
}

// FP32 runs the persistent k_pcg_rows_stream (one CTA per SM, the next
// problem's matrices prefetched into shared memory) when its stage fits
template <class Tg>
bool pcg_stream_fits(const gato_solver* s)
{
    if constexpr (sizeof(typename Tg::T) == 4)
        return RowPcg<Tg::NQ, 2>::fits(s->N) &&
               PcgStage<Tg::NQ>::smem_bytes(s->N) + 64 <= (size_t)s->max_smem;
    else
        return false;
}

// ... and the step recovery's A_k, Qi_k blocks too (iiwa14 up to N = 32)
template <class Tg>
bool pcg_stream_dz_fits(const gato_solver* s)
{
    if constexpr (sizeof(typename Tg::T) == 4)
        return pcg_stream_fits<Tg>(s) &&
               PcgStage<Tg::NQ>::smem_bytes_dz(s->N) + 64 <= (size_t)s->max_smem;
    else
        return false;
}

// register-resident PCG + dz of every problem
template <class Tg>
void launch_pcg_rows(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                     int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    if constexpr (sizeof(T) == 4) {
        if (pcg_stream_fits<Tg>(s)) {
            const int grid = std::min(s->B, s->nsm);
            const int dz = pcg_stream_dz_fits<Tg>(s);
            k_pcg_rows_stream<NQ, Acc><<<grid, RowPcg<NQ, 2>::threads(s->N),
                                         dz ? PcgStage<NQ>::smem_bytes_dz(s->N)
                                            : PcgStage<NQ>::smem_bytes(s->N),
                                         st>>>(bt, row, dz);
            return;
        }
    }
    constexpr int RPT = pcg_rows_per_thread<T>();
    if constexpr (sizeof(T) == 8) {
        if (s->p32) {
            k_pcg_rows_p32<NQ><<<s->B, RowPcg<NQ, RPT>::threads(s->N),
                                 RowPcg<NQ, RPT>::smem_bytes_p32(s->N), st>>>(bt, row);
            return;
        }
    }
    k_pcg_rows<NQ, T, Acc, RPT><<<s->B, RowPcg<NQ, RPT>::threads(s->N),
                                   RowPcg<NQ, RPT>::template smem_bytes<T>(s->N), st>>>(bt, row);
}

// cluster PCG + step for horizons beyond one CTA's registers (N > ~36)
template <class Tg>
int launch_pcg_cluster(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                       int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    constexpr int RPT = cluster_rows_per_thread<T>();
    using CP = ClusterPcg<NQ, RPT>;
    ProfScope ps_(s, st, GATO_KERNEL_PCG);
    const int C = CP::ctas(s->N);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(s->B * C);
    cfg.blockDim = dim3(CP::threads(s->N));
    cfg.dynamicSmemBytes = CP::template smem_bytes<T>(s->N);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_pcg_cluster<NQ, T, Acc, RPT>, bt, row));
    return GATO_OK;
}

// KKT blocks and Schur system of every problem, CTA per problem, S and P^-1
// to global memory, as the two halves of k_fused_iter (k_fused_kkt, then
// k_fused_schur), each compiled for its own occupancy
template <class Tg>
int launch_kkt_schur(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                     int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    ProfScope ps_(s, st, GATO_KERNEL_FUSED_ITER);
    FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, false};
    k_fused_kkt<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s), row);
    k_fused_schur<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s), row);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_fused_iter(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                      int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    // rows of S and P^-1 per thread in k_pcg_rows: two (each window value
    // loaded from shared memory feeds two rows)
    constexpr int RPT = pcg_rows_per_thread<T>();
    // Up to 1.5 problems per SM, one CTA per problem would leave SMs idle
    // and make every problem's KKT blocks and Schur complement serial chains
    // of knots, so both run knot-parallel, a warp per knot (k_kkt, then the
    // plain form's k_schur_inv, k_schur, k_schur_off).  Measured, iiwa14
    // N = 32, solves/s fused -> split: B = 1 1,020 -> 1,372; B = 96 75.0K ->
    // 90.7K; B = 192 110.2K -> 113.2K; B = 256 125.6K -> 116.8K.
    const int with_kkt = 2 * s->B > 3 * s->nsm;
    if (!with_kkt) RC(launch_kkt<Tg>(s, st, bt));
    if (rows_pcg_fits<NQ, T>(s->N)) {
        // KKT + Schur into global memory, then the register-resident PCG + dz
        if (with_kkt) {
            RC(launch_kkt_schur<Tg>(s, st, bt, row));
        } else {
            RC(launch_schur<Tg>(s, st, bt));
        }
        ProfScope ps2_(s, st, GATO_KERNEL_PCG);
        launch_pcg_rows<Tg>(s, st, bt, row);
        CKL();
        return GATO_OK;
    }
    if (ClusterPcg<NQ, cluster_rows_per_thread<T>()>::fits(s->N)) {
        if (with_kkt) {
            RC(launch_kkt_schur<Tg>(s, st, bt, row));
        } else {
            RC(launch_schur<Tg>(s, st, bt));
        }
        return launch_pcg_cluster<Tg>(s, st, bt, row);
    }
    ProfScope ps_(s, st, GATO_KERNEL_FUSED_ITER);
    const bool stage = fused_stage_fits<Tg>(s);
    FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, stage};
    k_fused_iter<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s), stage,
                                                                      row, 1, with_kkt);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_merit_ls(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                    int mode, int row)
{
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    ProfScope ps_(s, st, mode == 1 ? GATO_KERNEL_LINE_SEARCH : GATO_KERNEL_MERIT);
    const int items = (mode == 1 ? NUM_ALPHAS : 1) * s->N;
    const int threads = std::min(256, cdiv(items, WARP) * WARP);
    k_merit_ls<Tg::NQ, T, Acc><<<s->B, threads, items * sizeof(Acc), st>>>(bt, dmodel<Tg>(s),
                                                                           mode, row);
    CKL();
    return GATO_OK;
}

template <class Tg>
int launch_check(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt)
{
    ProfScope ps_(s, st, GATO_KERNEL_CHECK);
    k_check<Tg::NQ, typename Tg::T><<<1, 1024, 0, st>>>(bt);
    CKL();
    return GATO_OK;
}

template <class Tg>
int configure_kernels(gato_solver* s)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    RC(set_smem(k_pcg<NQ, T, Acc>, pcg_smem_bytes<NQ, T>(s->N, pcg_stage_fits<Tg>(s)),
                s->max_smem));
    FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, fused_stage_fits<Tg>(s)};
    if (lay.bytes() > (size_t)s->max_smem)
        return fail(GATO_ERR_UNSUPPORTED, "N=%d needs %zu bytes of shared memory", s->N,
                    lay.bytes());
    RC(set_smem(k_fused_iter<NQ, T, Acc>, lay.bytes(), s->max_smem));
    RC(set_smem(k_fused_kkt<NQ, T, Acc>, lay.bytes(), s->max_smem));
    RC(set_smem(k_fused_schur<NQ, T, Acc>, lay.bytes(), s->max_smem));
    constexpr int RPT = pcg_rows_per_thread<T>();
    if (rows_pcg_fits<NQ, T>(s->N)) {  // longer horizons take the cluster PCG
        RC(set_smem(k_pcg_rows<NQ, T, Acc, RPT>, RowPcg<NQ, RPT>::template smem_bytes<T>(s->N),
                    s->max_smem));
        if constexpr (sizeof(T) == 8)
            RC(set_smem(k_pcg_rows_p32<NQ>, RowPcg<NQ, RPT>::smem_bytes_p32(s->N), s->max_smem));
    }
    if constexpr (sizeof(T) == 4) {
        if (pcg_stream_fits<Tg>(s))
            RC(set_smem(k_pcg_rows_stream<NQ, Acc>,
                        pcg_stream_dz_fits<Tg>(s) ? PcgStage<NQ>::smem_bytes_dz(s->N)
                                                  : PcgStage<NQ>::smem_bytes(s->N),
                        s->max_smem));
    }
    return GATO_OK;
}

// --- solve drivers -------------------------------------------------------------
// Reference driver shape (gato/bsqp/bsqp.cuh:103-197): stage kernels and a
// host convergence check after every PCG.
template <class Tg>
int solve_plain(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal,
                int* host_sqp, int* host_conv, int* host_status, int* ls_rows)
{
    const int B = s->B, N = s->N;
    const Dims<Tg::NQ> d{N};
    auto bt = make_batch<Tg>(s, xu, xs, goal);
    CK(cudaMemsetAsync(s->dz, 0, s->esz * (size_t)B * d.traj(), st));
    CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * B, st));
    CK(cudaMemsetAsync(s->status, 0, sizeof(int) * B, st));
    std::fill(host_status, host_status + B, 0);
    RC(launch_merit<Tg>(s, st, bt, 1, 0, 0));
    RC(launch_merit_sum<Tg>(s, st, s->merit_init, s->merit_init0));
    std::fill(host_sqp, host_sqp + B, 0);
    std::fill(host_conv, host_conv + B, 0);
    int rows = 0;
    for (int it = 0; it < s->params.max_sqp_iters; ++it) {
        Nvtx r_("sqp_iteration");
        RC(launch_kkt<Tg>(s, st, bt));
        RC(launch_schur<Tg>(s, st, bt));
        RC(launch_pcg<Tg>(s, st, bt, it));
        RC(launch_dz<Tg>(s, st, bt));
        CK(cudaMemcpyAsync(s->pin_i, s->pcg_iters, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        int solved = 0;
        for (int b = 0; b < B; ++b) {
            if (!host_conv[b] && s->pin_i[b] >= s->params.max_pcg_iters)
                host_status[b] |= GATO_STATUS_PCG_MAX_ITER;
            if (s->pin_i[b] == 0) {
                host_conv[b] = 1;
                host_sqp[b] += 1;
            }
            if (host_conv[b]) solved++;
            else host_sqp[b] += 1;
        }
        if ((float)solved >= (float)B * (float)s->params.solve_ratio) break;
        memcpy(s->pin_i, host_conv, sizeof(int) * B);
        CK(cudaMemcpyAsync(s->conv, s->pin_i, sizeof(int) * B, cudaMemcpyHostToDevice, st));
        RC(launch_merit<Tg>(s, st, bt, NUM_ALPHAS, 1, 0));
        RC(launch_ls<Tg>(s, st, bt, it, 0));
        rows++;
    }
    RC(launch_merit<Tg>(s, st, bt, 1, 0, 0));
    RC(launch_merit_sum<Tg>(s, st, s->merit_final, nullptr));
    CK(cudaMemcpyAsync(s->drho, s->drho_init_d, s->esz * B, cudaMemcpyDeviceToDevice, st));
    *ls_rows = rows;
    return GATO_OK;
}

// Device-side control flow: enqueues the whole solve (no host round trip).
template <class Tg>
int enqueue_fused(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal)
{
    const int B = s->B, N = s->N;
    const Dims<Tg::NQ> d{N};
    auto bt = make_batch<Tg>(s, xu, xs, goal);
    CK(cudaMemsetAsync(s->dz, 0, s->esz * (size_t)B * d.traj(), st));
    CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * B, st));
    CK(cudaMemsetAsync(s->sqp_iters, 0, sizeof(int) * B, st));
    CK(cudaMemsetAsync(s->done, 0, sizeof(int), st));
    CK(cudaMemsetAsync(s->ls_count, 0, sizeof(int), st));
    CK(cudaMemsetAsync(s->status, 0, sizeof(int) * B, st));
    RC(launch_merit_ls<Tg>(s, st, bt, 0, 0));
    for (int it = 0; it < s->params.max_sqp_iters; ++it) {
        Nvtx r_("sqp_iteration");
        RC(launch_fused_iter<Tg>(s, st, bt, it));
        RC(launch_check<Tg>(s, st, bt));
        RC(launch_merit_ls<Tg>(s, st, bt, 1, it));
    }
    RC(launch_merit_ls<Tg>(s, st, bt, 2, 0));
    CK(cudaMemcpyAsync(s->drho, s->drho_init_d, s->esz * B, cudaMemcpyDeviceToDevice, st));
    return GATO_OK;
}

template <class Tg>
int solve_fused(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal)
{
    const bool stale = s->gexec == nullptr || s->gkey[0] != xu || s->gkey[1] != xs ||
                       s->gkey[2] != goal || s->gkey[3] != (const void*)st || s->gver != s->version;
    if (stale) {
        if (s->gexec) {
            cudaGraphExecDestroy(s->gexec);
            s->gexec = nullptr;
        }
        cudaStream_t cap;
        CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_fused<Tg>(s, cap, xu, xs, goal);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&s->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        s->gkey[0] = xu;
        s->gkey[1] = xs;
        s->gkey[2] = goal;
        s->gkey[3] = (const void*)st;
        s->gver = s->version;
    }
    CK(cudaGraphLaunch(s->gexec, st));
    return GATO_OK;
}

// Reports (and clears) an expired bounded wait in a device kernel.  The
// caller has synchronised the solver's stream.
int check_device_waits(gato_solver* s)
{
    int flag = 0;
    CK(cudaMemcpy(&flag, s->work + 2, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        CK(cudaMemset(s->work + 2, 0, sizeof(int)));
        return fail(GATO_ERR_TIMEOUT, "PCG: the wait for a problem's matrices in shared memory expired");
    }
    return GATO_OK;
}

// hstat: status bits found on the host (plain form) or null
int read_stats(gato_solver* s, const int* hsqp, const int* hconv, const int* hstat, int rows,
               gato_stats_t* stats)
{
    RC(check_device_waits(s));
    const int B = s->B;
    if (stats->status) {
        CK(cudaMemcpy(stats->status, s->status, sizeof(int) * B, cudaMemcpyDeviceToHost));
        for (int b = 0; b < B; ++b)
            stats->status[b] |= (hstat ? hstat[b] : 0) |
                                (hconv[b] ? GATO_STATUS_CONVERGED : GATO_STATUS_MAX_ITER);
    }
    const int iters = std::max(1, s->params.max_sqp_iters);
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    stats->sqp_time_us = 1000.0 * ms;
    stats->ls_num_iters = rows;
    if (stats->sqp_iters) memcpy(stats->sqp_iters, hsqp, sizeof(int) * B);
    if (stats->kkt_converged) memcpy(stats->kkt_converged, hconv, sizeof(int) * B);
    std::vector<double> tmp(B);
    if (stats->final_merit) {
        CK(cudaMemcpy(tmp.data(), s->merit_final, sizeof(double) * B, cudaMemcpyDeviceToHost));
        for (int b = 0; b < B; ++b) stats->final_merit[b] = (float)tmp[b];
    }
    if (stats->initial_merit) {
        CK(cudaMemcpy(tmp.data(), s->merit_init0, sizeof(double) * B, cudaMemcpyDeviceToHost));
        for (int b = 0; b < B; ++b) stats->initial_merit[b] = (float)tmp[b];
    }
    if (stats->pcg_iters)
        CK(cudaMemcpy(stats->pcg_iters, s->h_pcg, sizeof(int) * (size_t)iters * B,
                      cudaMemcpyDeviceToHost));
    if (stats->ls_min_merit)
        CK(cudaMemcpy(stats->ls_min_merit, s->h_ls_min, sizeof(float) * (size_t)iters * B,
                      cudaMemcpyDeviceToHost));
    if (stats->ls_step_size)
        CK(cudaMemcpy(stats->ls_step_size, s->h_ls_step, sizeof(float) * (size_t)iters * B,
                      cudaMemcpyDeviceToHost));
    return GATO_OK;
}

template <class Tg>
int do_solve(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal,
             gato_stats_t* stats)
{
    Nvtx r_(s->form == GATO_FORM_PLAIN ? "gato_solve(plain)" : "gato_solve(fused)");
    const int B = s->B;
    std::vector<int> hsqp(B), hconv(B), hstat(B, 0);
    int rows = 0;
    CK(cudaEventRecord(s->ev0, st));
    if (s->form == GATO_FORM_PLAIN)
        RC(solve_plain<Tg>(s, st, xu, xs, goal, hsqp.data(), hconv.data(), hstat.data(), &rows));
    else
        RC(solve_fused<Tg>(s, st, xu, xs, goal));
    CK(cudaEventRecord(s->ev1, st));
    if (!stats) return GATO_OK;
    CK(cudaStreamSynchronize(st));
    if (s->form != GATO_FORM_PLAIN) {
        CK(cudaMemcpy(&rows, s->ls_count, sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hsqp.data(), s->sqp_iters, sizeof(int) * B, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hconv.data(), s->conv, sizeof(int) * B, cudaMemcpyDeviceToHost));
    }
    return read_stats(s, hsqp.data(), hconv.data(), hstat.data(), rows, stats);
}

// --- adjoint ---------------------------------------------------------------------
template <typename T>
__global__ void k_fill(T* p, int n, T v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

int adj_alloc(gato_solver* s)
{
    if (s->adj_lam) return GATO_OK;
    const size_t B = s->B, nx = 2 * s->nq, nu = s->nq, N = s->N;
    const size_t traj = (nx + nu) * N - nu, vecp = (N + 2) * nx;
    RC(s->alloc_t(&s->adj_mu, B * vecp));
    RC(s->alloc_t(&s->adj_v, B * traj));
    RC(s->alloc_t(&s->adj_scale, B));
    RC(s->alloc_t(&s->adj_tol, B));
    RC(s->alloc(&s->adj_conv, B));
    RC(s->alloc(&s->adj_done, 1));
    RC(s->alloc(&s->adj_iters, 2 * B));
    RC(s->alloc_t(&s->adj_lam, B * vecp));  // last: it marks the set as complete
    return GATO_OK;
}

// PCG on (S, P^-1, bt.gamma) from bt.lambda, then the step into bt.dz
// (residuals into bt.q, bt.r): the fused form's register PCG when it fits,
// else the plain PCG and step kernels.
template <class Tg>
int pcg_and_step(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    constexpr int RPT = pcg_rows_per_thread<T>();
    if (rows_pcg_fits<NQ, T>(s->N)) {
        ProfScope ps_(s, st, GATO_KERNEL_PCG);
        launch_pcg_rows<Tg>(s, st, bt, -1);
        CKL();
        return GATO_OK;
    }
    if (ClusterPcg<NQ, cluster_rows_per_thread<T>()>::fits(s->N))
        return launch_pcg_cluster<Tg>(s, st, bt, -1);
    RC(launch_pcg<Tg>(s, st, bt, -1));
    return launch_dz<Tg>(s, st, bt);
}

// Implicit gradient of a loss of the returned trajectory xu through the QP
// of the solver at xu (the adjoint of the converged subproblem): KKT blocks
// recomputed at xu (dynamics derivatives are not stored), Schur system, the
// forward QP step dz (warm-started from the solver's lambda, which is left
// unchanged), the adjoint RHS and its PCG, then the parameter gradients.
template <class Tg>
int adjoint_impl(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal,
                 const void* dl, void* g_xs, void* g_goal, void* g_wdiag, double tol,
                 int max_iters, int32_t* h_iters)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    const int B = s->B, N = s->N;
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    Nvtx r_("gato_adjoint");
    RC(adj_alloc(s));
    auto bt = make_batch<Tg>(s, xu, xs, goal);
    bt.conv = s->adj_conv;
    bt.done = s->adj_done;
    bt.tol = (T*)s->adj_tol;
    bt.h_pcg = nullptr;
    bt.max_pcg_iters = max_iters;
    bt.abs_tol = 1e-30f;  // relative stopping only; an all-zero RHS still stops at once
    CK(cudaMemsetAsync(s->adj_conv, 0, sizeof(int) * B, st));
    CK(cudaMemsetAsync(s->adj_done, 0, sizeof(int), st));
    k_fill<T><<<cdiv(B, 256), 256, 0, st>>>((T*)s->adj_tol, B, (T)tol);
    CKL();
    RC(launch_kkt<Tg>(s, st, bt));
    RC(launch_schur<Tg>(s, st, bt));
    // forward QP step at xu into s->dz
    CK(cudaMemcpyAsync(s->adj_lam, s->lambda, s->esz * (size_t)B * d.vecp(),
                       cudaMemcpyDeviceToDevice, st));
    auto bf = bt;
    bf.lambda = (T*)s->adj_lam;
    bf.pcg_iters = s->adj_iters;
    RC(pcg_and_step<Tg>(s, st, bf));
    // adjoint system: RHS into q, r, gamma; PCG from zero; v into adj_v
    k_adj_rhs<NQ, T><<<B, 256, (size_t)N * (nx + nu) * sizeof(T), st>>>(bt, (const T*)dl,
                                                                        (T*)s->adj_scale);
    CKL();
    CK(cudaMemsetAsync(s->adj_mu, 0, s->esz * (size_t)B * d.vecp(), st));
    auto ba = bt;
    ba.lambda = (T*)s->adj_mu;
    ba.dz = (T*)s->adj_v;
    ba.pcg_iters = s->adj_iters + B;
    RC(pcg_and_step<Tg>(s, st, ba));
    constexpr int GW = 8;
    const size_t gsm = (size_t)GW * (DynSmem<NQ>::SIZE + nx + nx + nu) * sizeof(T);
    k_adj_grad<NQ, T><<<B, GW * WARP, gsm, st>>>(bt, dmodel<Tg>(s), (const T*)s->adj_scale,
                                                 (const T*)s->adj_v, (const T*)s->adj_mu,
                                                 (T*)g_xs, (T*)g_goal, (T*)g_wdiag);
    CKL();
    if (h_iters) {
        CK(cudaMemcpyAsync(h_iters, s->adj_iters, sizeof(int) * 2 * B, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return GATO_OK;
}

// The QP step of the SQP at xu alone: KKT blocks, Schur system, PCG from the
// solver's lambda (left unchanged) with relative tolerance tol (0: no
// tolerance stop, exactly max_iters iterations unless the residual is exactly
// zero) and the step recovery, dz into dz_out.
template <class Tg>
int qp_step_impl(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal,
                 void* dz_out, double tol, int max_iters, int32_t* h_iters)
{
    using T = typename Tg::T;
    const int B = s->B;
    const Dims<Tg::NQ> d{s->N};
    RC(adj_alloc(s));
    auto bt = make_batch<Tg>(s, xu, xs, goal);
    bt.conv = s->adj_conv;
    bt.done = s->adj_done;
    bt.tol = (T*)s->adj_tol;
    bt.h_pcg = nullptr;
    bt.max_pcg_iters = max_iters;
    bt.abs_tol = tol > 0 ? 1e-30f : 0.0f;
    CK(cudaMemsetAsync(s->adj_conv, 0, sizeof(int) * B, st));
    CK(cudaMemsetAsync(s->adj_done, 0, sizeof(int), st));
    k_fill<T><<<cdiv(B, 256), 256, 0, st>>>((T*)s->adj_tol, B, (T)tol);
    CKL();
    RC(launch_kkt<Tg>(s, st, bt));
    RC(launch_schur<Tg>(s, st, bt));
    CK(cudaMemcpyAsync(s->adj_lam, s->lambda, s->esz * (size_t)B * d.vecp(),
                       cudaMemcpyDeviceToDevice, st));
    auto bf = bt;
    bf.lambda = (T*)s->adj_lam;
    bf.pcg_iters = s->adj_iters;
    bf.dz = (T*)dz_out;
    RC(pcg_and_step<Tg>(s, st, bf));
    if (h_iters) {
        CK(cudaMemcpyAsync(h_iters, s->adj_iters, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return GATO_OK;
}

// --- closed-loop rollout ---------------------------------------------------------
int rollout_alloc(gato_solver* s)
{
    if (s->rl_rho) return GATO_OK;
    const size_t B = s->B, nx = 2 * s->nq, nu = s->nq, N = s->N;
    const size_t traj = (nx + nu) * N - nu;
    RC(s->alloc_t(&s->rl_goal, B * 6 * N));
    RC(s->alloc_t(&s->rl_gx, B * nx));
    RC(s->alloc_t(&s->rl_ga, B * nx));
    RC(s->alloc_t(&s->rl_gu, B * nu));
    RC(s->alloc_t(&s->rl_dl, B * traj));
    RC(s->alloc_t(&s->rl_gxs, B * nx));
    RC(s->alloc_t(&s->rl_ggoal, B * 6 * N));
    RC(s->alloc_t(&s->rl_gw, B * (nx + nu)));
    RC(s->alloc_t(&s->rl_rho, B));  // last: it marks the set as complete
    return GATO_OK;
}

template <class Tg>
int enqueue_rollout(gato_solver* s, cudaStream_t st, int steps, const void* goal_traj, void* xu,
                    const void* noise, void* x, void* u, void* ckpt_xu, void* ckpt_rho)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    const int B = s->B, N = s->N, nx = 2 * NQ, nu = NQ;
    const int traj = (nx + nu) * N - nu, stride = 6 * (N + steps);
    const size_t smem_sim = WPB * (DynSmem<NQ>::SIZE + 3 * NQ) * sizeof(T);
    for (int t = 0; t < steps; ++t) {
        T* xt = (T*)x + (size_t)t * B * nx;
        k_goal_window<T><<<cdiv(B * 6 * N, 256), 256, 0, st>>>((const T*)goal_traj, stride, t, N,
                                                                B, (T*)s->rl_goal);
        CKL();
        k_set_x0<T><<<cdiv(B * nx, 256), 256, 0, st>>>((T*)xu, xt, B, traj, nx);
        CKL();
        RC(enqueue_fused<Tg>(s, st, xu, xt, s->rl_goal));
        if (ckpt_xu)
            CK(cudaMemcpyAsync((T*)ckpt_xu + (size_t)t * B * traj, xu, sizeof(T) * B * traj,
                               cudaMemcpyDeviceToDevice, st));
        if (ckpt_rho)
            CK(cudaMemcpyAsync((T*)ckpt_rho + (size_t)t * B, s->rho, sizeof(T) * B,
                               cudaMemcpyDeviceToDevice, st));
        k_sim_step<NQ, T><<<cdiv(B, WPB), WPB * WARP, smem_sim, st>>>(
            dmodel<Tg>(s), B, (T)s->dt, xt, (const T*)xu, traj,
            noise ? (const T*)noise + (size_t)t * B * nu : nullptr, (const T*)s->fext,
            s->use_fext, xt + (size_t)B * nx, (T*)u + (size_t)t * B * nu);
        CKL();
        k_shift<T><<<B, 128, sizeof(T) * traj, st>>>((T*)xu, xt + (size_t)B * nx, N, nx, nu);
        CKL();
    }
    return GATO_OK;
}

template <class Tg>
int enqueue_rollout_backward(gato_solver* s, cudaStream_t st, int steps, const void* goal_traj,
                             const void* x, const void* u, const void* ckpt_xu,
                             const void* ckpt_rho, const void* dl_dx, void* g_x0, void* g_goal,
                             void* g_wdiag, double tol, int max_iters)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    const int B = s->B, N = s->N, nx = 2 * NQ, nu = NQ;
    const int traj = (nx + nu) * N - nu, stride = 6 * (N + steps);
    const size_t smem_vjp = WPB * (DynSmem<NQ>::SIZE + 3 * NQ + nx) * sizeof(T);
    CK(cudaMemcpyAsync(s->rl_rho, s->rho, sizeof(T) * B, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->rl_gx, (const T*)dl_dx + (size_t)steps * B * nx, sizeof(T) * B * nx,
                       cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(g_goal, 0, sizeof(T) * (size_t)B * stride, st));
    CK(cudaMemsetAsync(g_wdiag, 0, sizeof(T) * (size_t)B * (nx + nu), st));
    for (int t = steps - 1; t >= 0; --t) {
        const T* xt = (const T*)x + (size_t)t * B * nx;
        k_sim_vjp<NQ, T><<<cdiv(B, WPB), WPB * WARP, smem_vjp, st>>>(
            dmodel<Tg>(s), B, (T)s->dt, xt, (const T*)u + (size_t)t * B * nu,
            (const T*)s->rl_gx, (const T*)s->fext, s->use_fext, (T*)s->rl_ga, (T*)s->rl_gu);
        CKL();
        k_scatter_u0<T><<<cdiv(B * traj, 256), 256, 0, st>>>((T*)s->rl_dl, (const T*)s->rl_gu, B,
                                                           traj, nx, nu);
        CKL();
        CK(cudaMemcpyAsync(s->rho, (const T*)ckpt_rho + (size_t)t * B, sizeof(T) * B,
                           cudaMemcpyDeviceToDevice, st));
        k_goal_window<T><<<cdiv(B * 6 * N, 256), 256, 0, st>>>((const T*)goal_traj, stride, t, N,
                                                                B, (T*)s->rl_goal);
        CKL();
        RC(adjoint_impl<Tg>(s, st, (void*)((const T*)ckpt_xu + (size_t)t * B * traj), xt,
                            s->rl_goal, s->rl_dl, s->rl_gxs, s->rl_ggoal, s->rl_gw, tol,
                            max_iters, nullptr));
        CK(cudaMemcpyAsync(s->rl_gx, (const T*)dl_dx + (size_t)t * B * nx, sizeof(T) * B * nx,
                           cudaMemcpyDeviceToDevice, st));
        k_add3<T><<<cdiv(B * nx, 256), 256, 0, st>>>((T*)s->rl_gx, (const T*)s->rl_ga,
                                                   (const T*)s->rl_gxs, B * nx);
        CKL();
        k_accum<T><<<cdiv(B * (nx + nu), 256), 256, 0, st>>>((T*)g_wdiag, (const T*)s->rl_gw,
                                                            B * (nx + nu));
        CKL();
        k_goal_accum<T><<<cdiv(B * 6 * N, 256), 256, 0, st>>>((T*)g_goal, (const T*)s->rl_ggoal,
                                                               stride, t, N, B);
        CKL();
    }
    CK(cudaMemcpyAsync(g_x0, s->rl_gx, sizeof(T) * B * nx, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->rho, s->rl_rho, sizeof(T) * B, cudaMemcpyDeviceToDevice, st));
    return GATO_OK;
}

// captures `enqueue` into a graph on a private stream and launches it on st
template <class F>
int capture_and_launch(cudaStream_t st, F&& enqueue, cudaGraphExec_t* exec)
{
    cudaStream_t cap;
    CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    CK(cudaGraphLaunch(*exec, st));
    return GATO_OK;
}

// sim_forward: one warp per problem (simForwardBatchedKernel,
// gato/bsqp/kernels/sim.cuh:14-49).
template <int NQ, typename T>
__global__ void k_sim_forward(DevModel<NQ, T> M, int B, T dt, const T* xk, const T* uk,
                              const T* fext, int use_fext, T* out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x * (blockDim.x / WARP) + warp_id();
    if (b >= B) return;
    T* s = smem + warp_id() * DynSmem<NQ>::SIZE;
    const T* q = xk;
    const T* qd = xk + NQ;
    dyn_load_transforms<NQ, T>(M, q, s);
    __syncwarp();
    T mc[NQ];
    dyn_forward<NQ, T>(M, s, q, qd, uk, use_fext ? fext + 6 * b : nullptr, false, mc);
    const int l = lane_id();
    if (l < 2 * NQ) {
        T v;
        if (l < NQ)
            v = q[l] + dt * qd[l] + T(0.5) * s[DynSmem<NQ>::QDD + l] * dt * dt;
        else
            v = qd[l - NQ] + dt * s[DynSmem<NQ>::QDD + l - NQ];
        out[(size_t)b * 2 * NQ + l] = v;
    }
}

cudaStream_t as_stream(void* st) { return (cudaStream_t)st; }

int check_handle(const gato_solver* s)
{
    if (!s) return fail(GATO_ERR_ARG, "null solver handle");
    return GATO_OK;
}

int bind_device(const gato_solver* s)
{
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != s->device) CK(cudaSetDevice(s->device));
    return GATO_OK;
}

int check_single(const gato_solver* s)
{
    if (s->precision == GATO_PREC_FP64)
        return fail(GATO_ERR_ARG, "FP64 solver: use the _f64 entry points");
    return GATO_OK;
}

int check_double(const gato_solver* s)
{
    if (s->precision != GATO_PREC_FP64)
        return fail(GATO_ERR_ARG, "_f64 entry point on a single-precision solver");
    return GATO_OK;
}

int solve_host_any(gato_solver* s, void* h_xu, double dt, const void* h_xs, const void* h_goal,
                   gato_stats_t* stats)
{
    RC(bind_device(s));
    if (dt != s->dt) {
        s->dt = dt;
        s->version++;
    }
    const int nx = 2 * s->nq, nu = s->nq;
    const size_t traj = (size_t)(nx + nu) * s->N - nu;
    cudaStream_t st = s->own_stream;
    CK(cudaMemcpyAsync(s->xu, h_xu, s->esz * traj * s->B, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->xs, h_xs, s->esz * nx * s->B, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->goal, h_goal, s->esz * 6 * s->N * s->B, cudaMemcpyHostToDevice, st));
    RC(dispatch(s, [&](auto tg) {
        return do_solve<decltype(tg)>(s, st, s->xu, s->xs, s->goal, stats);
    }));
    CK(cudaMemcpyAsync(h_xu, s->xu, s->esz * traj * s->B, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return GATO_OK;
}

int set_batch(gato_solver_t* s, void* d, const float* h, std::vector<double>* dflt, int as_default)
{
    RC(check_handle(s));
    if (!h) return fail(GATO_ERR_ARG, "null host array");
    RC(bind_device(s));
    std::vector<double> v(h, h + s->B);
    RC(s->upload(d, v.data(), s->B));
    if (dflt && as_default) *dflt = v;
    return GATO_OK;
}

int lambda_count(const gato_solver* s) { return s->B * (s->N + 2) * 2 * s->nq; }

}  // namespace

