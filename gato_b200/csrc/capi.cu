// C ABI of the solver (include/gato_b200.h): solver object, the plain and
// fused drivers, CUDA-graph capture, stage entry points and sim_forward.
#include <cuda_runtime.h>

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

namespace {

thread_local std::string g_err;

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
    if (bytes > (size_t)device_limit)
        return fail(GATO_ERR_UNSUPPORTED, "kernel needs %zu bytes of shared memory, device has %d",
                    bytes, device_limit);
    if (bytes > 48 * 1024)
        CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                device_limit));
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
        *ls_count = nullptr, *h_pcg = nullptr;
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
    b.ls_count = s->ls_count;
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

// Brackets one launch with events when profiling is on.
struct ProfScope {
    gato_solver* s;
    cudaStream_t st;
    int id;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(gato_solver* s_, cudaStream_t st_, int id_) : s(s_), st(st_), id(id_)
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
                                                                    out, out2);
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

// cluster PCG + step for horizons beyond one CTA's registers (N > ~36)
template <class Tg>
int launch_pcg_cluster(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                       int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
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

template <class Tg>
int launch_fused_iter(gato_solver* s, cudaStream_t st, const Batch<Tg::NQ, typename Tg::T>& bt,
                      int row)
{
    constexpr int NQ = Tg::NQ;
    using T = typename Tg::T;
    using Acc = typename Tg::Acc;
    // rows of S and P^-1 per thread in k_pcg_rows: two in FP32 (each window
    // value loaded from shared memory feeds two rows), one in FP64 (registers)
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
    if (RowPcg<NQ, RPT>::fits(s->N)) {
        // KKT + Schur into global memory, then the register-resident PCG + dz
        {
            ProfScope ps_(s, st, GATO_KERNEL_FUSED_ITER);
            FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, false};
            k_fused_iter<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s),
                                                                              0, row, 0);
            CKL();
        }
        ProfScope ps2_(s, st, GATO_KERNEL_PCG);
        k_pcg_rows<NQ, T, Acc, RPT><<<s->B, RowPcg<NQ, RPT>::threads(s->N),
                                       RowPcg<NQ, RPT>::template smem_bytes<T>(s->N), st>>>(bt,
                                                                                            row);
        CKL();
        return GATO_OK;
    }
    if (ClusterPcg<NQ, RPT>::fits(s->N)) {
        {
            ProfScope ps_(s, st, GATO_KERNEL_FUSED_ITER);
            FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, false};
            k_fused_iter<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s),
                                                                              0, row, 0);
            CKL();
        }
        return launch_pcg_cluster<Tg>(s, st, bt, row);
    }
    ProfScope ps_(s, st, GATO_KERNEL_FUSED_ITER);
    const bool stage = fused_stage_fits<Tg>(s);
    FusedLayout<NQ, T> lay{s->N, FUSED_THREADS / WARP, stage};
    k_fused_iter<NQ, T, Acc><<<s->B, FUSED_THREADS, lay.bytes(), st>>>(bt, dmodel<Tg>(s), stage,
                                                                      row, 1);
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
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
    RC(set_smem(k_pcg_rows<NQ, T, Acc, RPT>, RowPcg<NQ, RPT>::template smem_bytes<T>(s->N),
                s->max_smem));
    return GATO_OK;
}

// --- solve drivers -------------------------------------------------------------
// Reference driver shape (gato/bsqp/bsqp.cuh:103-197): stage kernels and a
// host convergence check after every PCG.
template <class Tg>
int solve_plain(gato_solver* s, cudaStream_t st, void* xu, const void* xs, const void* goal,
                int* host_sqp, int* host_conv, int* ls_rows)
{
    const int B = s->B, N = s->N;
    const Dims<Tg::NQ> d{N};
    auto bt = make_batch<Tg>(s, xu, xs, goal);
    CK(cudaMemsetAsync(s->dz, 0, s->esz * (size_t)B * d.traj(), st));
    CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * B, st));
    RC(launch_merit<Tg>(s, st, bt, 1, 0, 0));
    RC(launch_merit_sum<Tg>(s, st, s->merit_init, s->merit_init0));
    std::fill(host_sqp, host_sqp + B, 0);
    std::fill(host_conv, host_conv + B, 0);
    int rows = 0;
    for (int it = 0; it < s->params.max_sqp_iters; ++it) {
        RC(launch_kkt<Tg>(s, st, bt));
        RC(launch_schur<Tg>(s, st, bt));
        RC(launch_pcg<Tg>(s, st, bt, it));
        RC(launch_dz<Tg>(s, st, bt));
        CK(cudaMemcpyAsync(s->pin_i, s->pcg_iters, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        int solved = 0;
        for (int b = 0; b < B; ++b) {
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
    RC(launch_merit_ls<Tg>(s, st, bt, 0, 0));
    for (int it = 0; it < s->params.max_sqp_iters; ++it) {
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

int read_stats(gato_solver* s, const int* hsqp, const int* hconv, int rows, gato_stats_t* stats)
{
    const int B = s->B;
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
    const int B = s->B;
    std::vector<int> hsqp(B), hconv(B);
    int rows = 0;
    CK(cudaEventRecord(s->ev0, st));
    if (s->form == GATO_FORM_PLAIN)
        RC(solve_plain<Tg>(s, st, xu, xs, goal, hsqp.data(), hconv.data(), &rows));
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
    return read_stats(s, hsqp.data(), hconv.data(), rows, stats);
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
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
    if (RowPcg<NQ, RPT>::fits(s->N)) {
        ProfScope ps_(s, st, GATO_KERNEL_PCG);
        k_pcg_rows<NQ, T, Acc, RPT><<<s->B, RowPcg<NQ, RPT>::threads(s->N),
                                       RowPcg<NQ, RPT>::template smem_bytes<T>(s->N), st>>>(bt,
                                                                                            -1);
        CKL();
        return GATO_OK;
    }
    if (ClusterPcg<NQ, RPT>::fits(s->N)) return launch_pcg_cluster<Tg>(s, st, bt, -1);
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

// ===========================================================================
extern "C" {

const char* gato_last_error(void) { return g_err.c_str(); }

const char* gato_version(void) { return "gato_b200 0.2 (sm_100a)"; }

int gato_builtin_model(int plant, gato_model_t* out)
{
    if (!out) return fail(GATO_ERR_ARG, "null model pointer");
    if (gato_plant_fill(plant, out) != 0) return fail(GATO_ERR_ARG, "unknown plant %d", plant);
    return GATO_OK;
}

int gato_create(const gato_model_t* model, int N, int batch, const gato_params_t* params,
                int form, int precision, gato_solver_t** out)
{
    if (!out) return fail(GATO_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (!model || !params) return fail(GATO_ERR_ARG, "null model or params");
    if (model->nq != 6 && model->nq != 7)
        return fail(GATO_ERR_UNSUPPORTED, "nq=%d: built for 6 or 7 joints", model->nq);
    if (N < 2 || N > 256) return fail(GATO_ERR_ARG, "N=%d out of range [2, 256]", N);
    if (batch < 1 || batch > 65535) return fail(GATO_ERR_ARG, "batch=%d out of range", batch);
    if (form != GATO_FORM_PLAIN && form != GATO_FORM_FUSED)
        return fail(GATO_ERR_ARG, "unknown form %d", form);
    if (precision != GATO_PREC_FP32 && precision != GATO_PREC_MIXED &&
        precision != GATO_PREC_FP64)
        return fail(GATO_ERR_ARG, "unknown precision %d", precision);
    if (params->max_sqp_iters < 0 || params->max_pcg_iters < 0)
        return fail(GATO_ERR_ARG, "negative iteration limits");
    if (!(params->dt > 0.0)) return fail(GATO_ERR_ARG, "dt must be positive");
    std::unique_ptr<gato_solver> s(new gato_solver);
    gato_solver* p = s.get();
    p->nq = model->nq;
    p->N = N;
    p->B = batch;
    p->form = form;
    p->precision = precision;
    p->esz = precision == GATO_PREC_FP64 ? sizeof(double) : sizeof(float);
    p->model = *model;
    p->params = *params;
    p->dt = params->dt;
    CK(cudaGetDevice(&p->device));
    CK(cudaDeviceGetAttribute(&p->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
    dispatch(p, [&](auto tg) {
        using Tg = decltype(tg);
        build_dev_model<Tg::NQ, typename Tg::T>(*model,
                                                (DevModel<Tg::NQ, typename Tg::T>*)p->dev_model);
        return 0;
    });
    const int nx = 2 * p->nq, nu = p->nq;
    const size_t B = batch;
    const size_t traj = (size_t)(nx + nu) * N - nu, vecp = (size_t)(N + 2) * nx,
                 b3d = (size_t)3 * nx * nx * N;
    const int iters = std::max(1, params->max_sqp_iters);
    RC(p->alloc_t(&p->xu, B * traj));
    RC(p->alloc_t(&p->xs, B * nx));
    RC(p->alloc_t(&p->goal, B * 6 * N));
    RC(p->alloc_t(&p->fext, B * 6));
    RC(p->alloc_t(&p->Q, B * N * nx * nx));
    RC(p->alloc_t(&p->R, B * N * nu * nu));
    RC(p->alloc_t(&p->q, B * N * nx));
    RC(p->alloc_t(&p->r, B * N * nu));
    RC(p->alloc_t(&p->A, B * N * nx * nx));
    RC(p->alloc_t(&p->Bm, B * N * nx * nu));
    RC(p->alloc_t(&p->c, B * N * nx));
    RC(p->alloc_t(&p->Qi, B * N * nx * nx));
    RC(p->alloc_t(&p->Ri, B * N * nu * nu));
    RC(p->alloc_t(&p->S, B * b3d));
    RC(p->alloc_t(&p->P, B * b3d));
    RC(p->alloc_t(&p->gamma, B * vecp));
    RC(p->alloc_t(&p->lambda, B * vecp));
    RC(p->alloc_t(&p->dz, B * traj));
    RC(p->alloc_t(&p->rho, B));
    RC(p->alloc_t(&p->drho, B));
    RC(p->alloc_t(&p->mu, B));
    RC(p->alloc_t(&p->tol, B));
    RC(p->alloc_t(&p->drho_init_d, B));
    RC(p->alloc_t(&p->sim_x, nx));
    RC(p->alloc_t(&p->sim_u, nu));
    RC(p->alloc_t(&p->sim_out, B * nx));
    RC(p->alloc(&p->merit_terms, B * NUM_ALPHAS * N));
    RC(p->alloc(&p->merit_init, B));
    RC(p->alloc(&p->merit_init0, B));
    RC(p->alloc(&p->merit_final, B));
    RC(p->alloc(&p->pcg_iters, B));
    RC(p->alloc(&p->conv, B));
    RC(p->alloc(&p->sqp_iters, B));
    RC(p->alloc(&p->done, 1));
    RC(p->alloc(&p->ls_count, 1));
    RC(p->alloc(&p->h_pcg, (size_t)iters * B));
    RC(p->alloc(&p->h_ls_min, (size_t)iters * B));
    RC(p->alloc(&p->h_ls_step, (size_t)iters * B));
    CK(cudaMallocHost(&p->pin_i, sizeof(int) * B));
    CK(cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&p->ev0));
    CK(cudaEventCreate(&p->ev1));
    // BSQP constructor defaults (bsqp.cuh:46-58): drho = 1, rho/mu/tol from
    // the parameters (float in the reference's FP32 build)
    const bool f64 = precision == GATO_PREC_FP64;
    auto as_t = [&](double v) { return f64 ? v : (double)(float)v; };
    p->rho_init.assign(B, as_t(params->rho));
    p->drho_init.assign(B, 1.0);
    std::vector<double> mu(B, as_t(params->mu)), tol(B, as_t(params->pcg_tol));
    RC(p->upload(p->rho, p->rho_init.data(), B));
    RC(p->upload(p->drho, p->drho_init.data(), B));
    RC(p->upload(p->drho_init_d, p->drho_init.data(), B));
    RC(p->upload(p->mu, mu.data(), B));
    RC(p->upload(p->tol, tol.data(), B));
    RC(dispatch(p, [&](auto tg) { return configure_kernels<decltype(tg)>(p); }));
    CK(cudaDeviceSynchronize());
    *out = s.release();
    return GATO_OK;
}

void gato_destroy(gato_solver_t* s)
{
    if (!s) return;
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(s->device);
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->rexec) cudaGraphExecDestroy(s->rexec);
    for (void* v : s->allocs) cudaFree(v);
    if (s->pin_i) cudaFreeHost(s->pin_i);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (cur >= 0) cudaSetDevice(cur);
    delete s;
}

int gato_sizes(const gato_solver_t* s, int* nx, int* nu, int* traj_size, int* goal_size,
               int* lambda_size)
{
    RC(check_handle(s));
    const int x = 2 * s->nq, u = s->nq;
    if (nx) *nx = x;
    if (nu) *nu = u;
    if (traj_size) *traj_size = (x + u) * s->N - u;
    if (goal_size) *goal_size = 6 * s->N;
    if (lambda_size) *lambda_size = (s->N + 2) * x;
    return GATO_OK;
}

int gato_solve(gato_solver_t* s, void* stream, float* d_xu, const float* d_xs,
               const float* d_goal, gato_stats_t* stats)
{
    RC(check_handle(s));
    RC(check_single(s));
    if (!d_xu || !d_xs || !d_goal) return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    return dispatch(s, [&](auto tg) {
        return do_solve<decltype(tg)>(s, as_stream(stream), d_xu, d_xs, d_goal, stats);
    });
}

int gato_solve_f64(gato_solver_t* s, void* stream, double* d_xu, const double* d_xs,
                   const double* d_goal, gato_stats_t* stats)
{
    RC(check_handle(s));
    RC(check_double(s));
    if (!d_xu || !d_xs || !d_goal) return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    return dispatch(s, [&](auto tg) {
        return do_solve<decltype(tg)>(s, as_stream(stream), d_xu, d_xs, d_goal, stats);
    });
}

int gato_solve_host(gato_solver_t* s, float* h_xu, float dt, const float* h_xs,
                    const float* h_goal, gato_stats_t* stats)
{
    RC(check_handle(s));
    RC(check_single(s));
    if (!h_xu || !h_xs || !h_goal) return fail(GATO_ERR_ARG, "null host buffer");
    if (!(dt > 0.0f)) return fail(GATO_ERR_ARG, "dt must be positive");
    return solve_host_any(s, h_xu, (double)dt, h_xs, h_goal, stats);
}

int gato_solve_host_f64(gato_solver_t* s, double* h_xu, double dt, const double* h_xs,
                        const double* h_goal, gato_stats_t* stats)
{
    RC(check_handle(s));
    RC(check_double(s));
    if (!h_xu || !h_xs || !h_goal) return fail(GATO_ERR_ARG, "null host buffer");
    if (!(dt > 0.0)) return fail(GATO_ERR_ARG, "dt must be positive");
    return solve_host_any(s, h_xu, dt, h_xs, h_goal, stats);
}

int gato_profile_solve(gato_solver_t* s, void* stream, float* d_xu, const float* d_xs,
                       const float* d_goal, double* ms_by_kernel, int32_t* launches_by_kernel)
{
    RC(check_handle(s));
    RC(check_single(s));
    if (!d_xu || !d_xs || !d_goal || !ms_by_kernel || !launches_by_kernel)
        return fail(GATO_ERR_ARG, "null pointer");
    RC(bind_device(s));
    cudaStream_t st = as_stream(stream);
    std::vector<gato_solver::ProfEntry> entries;
    s->prof = &entries;
    std::vector<int> hs(s->B), hc(s->B);
    int rows = 0;
    int rc = dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        if (s->form == GATO_FORM_PLAIN)
            return solve_plain<Tg>(s, st, d_xu, d_xs, d_goal, hs.data(), hc.data(), &rows);
        return enqueue_fused<Tg>(s, st, d_xu, d_xs, d_goal);
    });
    s->prof = nullptr;
    cudaError_t e = cudaStreamSynchronize(st);
    for (int k = 0; k < GATO_KERNEL_COUNT; ++k) {
        ms_by_kernel[k] = 0.0;
        launches_by_kernel[k] = 0;
    }
    for (auto& en : entries) {
        float ms = 0.0f;
        if (rc == 0 && e == cudaSuccess && cudaEventElapsedTime(&ms, en.a, en.b) == cudaSuccess) {
            ms_by_kernel[en.id] += ms;
            launches_by_kernel[en.id] += 1;
        }
        cudaEventDestroy(en.a);
        cudaEventDestroy(en.b);
    }
    if (rc) return rc;
    if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "profile solve: %s", cudaGetErrorString(e));
    return GATO_OK;
}

int gato_set_f_ext_batch(gato_solver_t* s, const float* h_f_ext)
{
    RC(check_handle(s));
    if (!h_f_ext) return fail(GATO_ERR_ARG, "null f_ext");
    RC(bind_device(s));
    std::vector<double> v(h_f_ext, h_f_ext + 6 * (size_t)s->B);
    RC(s->upload(s->fext, v.data(), v.size()));
    int any = 0;
    for (double x : v) any |= (x != 0.0);
    if (any != s->use_fext) {
        s->use_fext = any;
        s->version++;
    }
    return GATO_OK;
}

int gato_set_cost_diag_batch(gato_solver_t* s, const float* h_wdiag)
{
    RC(check_handle(s));
    RC(bind_device(s));
    const int use = h_wdiag != nullptr;
    if (use) {
        const size_t n = (size_t)3 * s->nq * s->B;
        std::vector<double> v(h_wdiag, h_wdiag + n);
        for (double x : v)
            if (!std::isfinite(x)) return fail(GATO_ERR_ARG, "non-finite cost weight");
        if (!s->wdiag) RC(s->alloc_t(&s->wdiag, n));
        RC(s->upload(s->wdiag, v.data(), n));
    }
    if (use != s->use_wdiag) {
        s->use_wdiag = use;
        s->version++;
    }
    return GATO_OK;
}

int gato_set_rho_penalty_batch(gato_solver_t* s, const float* h_rho, int set_as_reset_default)
{
    RC(check_handle(s));
    return set_batch(s, s->rho, h_rho, &s->rho_init, set_as_reset_default);
}

int gato_set_drho_batch(gato_solver_t* s, const float* h_drho, int set_as_reset_default)
{
    RC(check_handle(s));
    RC(set_batch(s, s->drho, h_drho, &s->drho_init, set_as_reset_default));
    if (set_as_reset_default) RC(s->upload(s->drho_init_d, s->drho_init.data(), s->B));
    return GATO_OK;
}

int gato_set_mu_batch(gato_solver_t* s, const float* h_mu)
{
    RC(check_handle(s));
    return set_batch(s, s->mu, h_mu, nullptr, 0);
}

int gato_set_pcg_tol_batch(gato_solver_t* s, const float* h_tol)
{
    RC(check_handle(s));
    return set_batch(s, s->tol, h_tol, nullptr, 0);
}

int gato_set_dt(gato_solver_t* s, float dt)
{
    RC(check_handle(s));
    if (!(dt > 0.0f)) return fail(GATO_ERR_ARG, "dt must be positive");
    if ((double)dt != s->dt) {
        s->dt = dt;
        s->version++;
    }
    return GATO_OK;
}

int gato_reset_dual(gato_solver_t* s)
{
    RC(check_handle(s));
    RC(bind_device(s));
    CK(cudaMemset(s->lambda, 0, s->esz * lambda_count(s)));
    return GATO_OK;
}

int gato_reset_rho(gato_solver_t* s)
{
    RC(check_handle(s));
    RC(bind_device(s));
    RC(s->upload(s->rho, s->rho_init.data(), s->B));
    RC(s->upload(s->drho, s->drho_init.data(), s->B));
    return GATO_OK;
}

int gato_set_rho_adaptation(gato_solver_t* s, int enabled)
{
    RC(check_handle(s));
    if ((enabled != 0) != (s->adapt_rho != 0)) {
        s->adapt_rho = enabled != 0;
        s->version++;
    }
    return GATO_OK;
}

int gato_get_lambda(gato_solver_t* s, float* h_lambda)
{
    RC(check_handle(s));
    if (!h_lambda) return fail(GATO_ERR_ARG, "null lambda");
    RC(bind_device(s));
    const int n = lambda_count(s);
    if (s->esz == sizeof(float)) {
        CK(cudaMemcpy(h_lambda, s->lambda, sizeof(float) * n, cudaMemcpyDeviceToHost));
    } else {
        std::vector<double> t(n);
        CK(cudaMemcpy(t.data(), s->lambda, sizeof(double) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) h_lambda[i] = (float)t[i];
    }
    return GATO_OK;
}

int gato_set_lambda(gato_solver_t* s, const float* h_lambda)
{
    RC(check_handle(s));
    if (!h_lambda) return fail(GATO_ERR_ARG, "null lambda");
    RC(bind_device(s));
    const int n = lambda_count(s);
    std::vector<double> t(h_lambda, h_lambda + n);
    return s->upload(s->lambda, t.data(), n);
}

int gato_get_lambda_f64(gato_solver_t* s, double* h_lambda)
{
    RC(check_handle(s));
    RC(check_double(s));
    if (!h_lambda) return fail(GATO_ERR_ARG, "null lambda");
    RC(bind_device(s));
    CK(cudaMemcpy(h_lambda, s->lambda, sizeof(double) * lambda_count(s), cudaMemcpyDeviceToHost));
    return GATO_OK;
}

int gato_set_lambda_f64(gato_solver_t* s, const double* h_lambda)
{
    RC(check_handle(s));
    RC(check_double(s));
    if (!h_lambda) return fail(GATO_ERR_ARG, "null lambda");
    RC(bind_device(s));
    CK(cudaMemcpy(s->lambda, h_lambda, sizeof(double) * lambda_count(s), cudaMemcpyHostToDevice));
    return GATO_OK;
}

int gato_get_rho(gato_solver_t* s, float* h_rho)
{
    RC(check_handle(s));
    if (!h_rho) return fail(GATO_ERR_ARG, "null rho");
    RC(bind_device(s));
    if (s->esz == sizeof(float)) {
        CK(cudaMemcpy(h_rho, s->rho, sizeof(float) * s->B, cudaMemcpyDeviceToHost));
    } else {
        std::vector<double> t(s->B);
        CK(cudaMemcpy(t.data(), s->rho, sizeof(double) * s->B, cudaMemcpyDeviceToHost));
        for (int i = 0; i < s->B; ++i) h_rho[i] = (float)t[i];
    }
    return GATO_OK;
}

int gato_sim_forward(gato_solver_t* s, const float* h_xk, const float* h_uk, float dt,
                     float* h_xkp1)
{
    RC(check_handle(s));
    if (!h_xk || !h_uk || !h_xkp1) return fail(GATO_ERR_ARG, "null host buffer");
    RC(bind_device(s));
    const int nx = 2 * s->nq, nu = s->nq;
    cudaStream_t st = s->own_stream;
    std::vector<double> x(h_xk, h_xk + nx), u(h_uk, h_uk + nu);
    RC(s->upload(s->sim_x, x.data(), nx));
    RC(s->upload(s->sim_u, u.data(), nu));
    RC(dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        using T = typename Tg::T;
        const size_t sm = WPB * DynSmem<Tg::NQ>::SIZE * sizeof(T);
        k_sim_forward<Tg::NQ, T><<<cdiv(s->B, WPB), WPB * WARP, sm, st>>>(
            dmodel<Tg>(s), s->B, (T)dt, (const T*)s->sim_x, (const T*)s->sim_u, (const T*)s->fext,
            s->use_fext, (T*)s->sim_out);
        CKL();
        return (int)GATO_OK;
    }));
    const size_t n = (size_t)nx * s->B;
    if (s->esz == sizeof(float)) {
        CK(cudaMemcpyAsync(h_xkp1, s->sim_out, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    } else {
        std::vector<double> t(n);
        CK(cudaMemcpyAsync(t.data(), s->sim_out, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t i = 0; i < n; ++i) h_xkp1[i] = (float)t[i];
    }
    return GATO_OK;
}

// --- stage entry points (single-precision solvers) ---------------------------
int gato_stage_setup_kkt(gato_solver_t* s, void* stream, const float* d_xu, const float* d_xs,
                         const float* d_goal, float* d_Q, float* d_R, float* d_q, float* d_r,
                         float* d_A, float* d_B, float* d_c)
{
    RC(check_handle(s));
    RC(check_single(s));
    RC(bind_device(s));
    return dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        using T = typename Tg::T;
        auto bt = make_batch<Tg>(s, (void*)d_xu, d_xs, d_goal);
        bt.Q = (T*)d_Q; bt.R = (T*)d_R; bt.q = (T*)d_q; bt.r = (T*)d_r; bt.A = (T*)d_A;
        bt.Bm = (T*)d_B; bt.c = (T*)d_c;
        return launch_kkt<Tg>(s, as_stream(stream), bt);
    });
}

int gato_stage_form_schur(gato_solver_t* s, void* stream, float* d_Q, float* d_R,
                          const float* d_q, const float* d_r, const float* d_A, const float* d_B,
                          const float* d_c, float* d_S, float* d_Pinv, float* d_gamma)
{
    RC(check_handle(s));
    RC(check_single(s));
    RC(bind_device(s));
    cudaStream_t st = as_stream(stream);
    const int nx = 2 * s->nq, nu = s->nq;
    const size_t nQ = (size_t)s->B * s->N * nx * nx, nR = (size_t)s->B * s->N * nu * nu;
    RC(dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        using T = typename Tg::T;
        auto bt = make_batch<Tg>(s, s->xu, s->xs, s->goal);
        bt.Q = (T*)d_Q; bt.R = (T*)d_R; bt.q = (T*)d_q; bt.r = (T*)d_r; bt.A = (T*)d_A;
        bt.Bm = (T*)d_B; bt.c = (T*)d_c; bt.S = (T*)d_S; bt.P = (T*)d_Pinv;
        bt.gamma = (T*)d_gamma;
        return launch_schur<Tg>(s, st, bt);
    }));
    // the reference leaves (Q + rho I_q)^-1 and R^-1 in d_Q / d_R
    CK(cudaMemcpyAsync(d_Q, s->Qi, sizeof(float) * nQ, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(d_R, s->Ri, sizeof(float) * nR, cudaMemcpyDeviceToDevice, st));
    return GATO_OK;
}

int gato_stage_pcg(gato_solver_t* s, void* stream, const float* d_S, const float* d_Pinv,
                   const float* d_gamma, float* d_lambda, int32_t* d_iters)
{
    RC(check_handle(s));
    RC(check_single(s));
    RC(bind_device(s));
    cudaStream_t st = as_stream(stream);
    CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * s->B, st));
    return dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        using T = typename Tg::T;
        auto bt = make_batch<Tg>(s, s->xu, s->xs, s->goal);
        bt.S = (T*)d_S; bt.P = (T*)d_Pinv; bt.gamma = (T*)d_gamma; bt.lambda = (T*)d_lambda;
        bt.pcg_iters = d_iters;
        return launch_pcg<Tg>(s, st, bt, -1);
    });
}

int gato_adjoint(gato_solver_t* s, void* stream, const float* d_xu, const float* d_xs,
                 const float* d_goal, const float* d_dl_dxu, float* d_g_xs, float* d_g_goal,
                 float* d_g_wdiag, double tol, int max_iters, int32_t* h_iters)
{
    RC(check_handle(s));
    RC(check_single(s));
    if (!d_xu || !d_xs || !d_goal || !d_dl_dxu || !d_g_xs || !d_g_goal || !d_g_wdiag)
        return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    if (tol <= 0) tol = 1e-12;  // FP32 CG stagnates before this: it runs to its floor
    if (max_iters <= 0) max_iters = 4 * s->N * s->nq;
    return dispatch(s, [&](auto tg) {
        return adjoint_impl<decltype(tg)>(s, as_stream(stream), (void*)d_xu, d_xs, d_goal,
                                          d_dl_dxu, d_g_xs, d_g_goal, d_g_wdiag, tol, max_iters,
                                          h_iters);
    });
}

int gato_adjoint_f64(gato_solver_t* s, void* stream, const double* d_xu, const double* d_xs,
                     const double* d_goal, const double* d_dl_dxu, double* d_g_xs,
                     double* d_g_goal, double* d_g_wdiag, double tol, int max_iters,
                     int32_t* h_iters)
{
    RC(check_handle(s));
    RC(check_double(s));
    if (!d_xu || !d_xs || !d_goal || !d_dl_dxu || !d_g_xs || !d_g_goal || !d_g_wdiag)
        return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    if (tol <= 0) tol = 1e-20;
    if (max_iters <= 0) max_iters = 4 * s->N * s->nq;
    return dispatch(s, [&](auto tg) {
        return adjoint_impl<decltype(tg)>(s, as_stream(stream), (void*)d_xu, d_xs, d_goal,
                                          d_dl_dxu, d_g_xs, d_g_goal, d_g_wdiag, tol, max_iters,
                                          h_iters);
    });
}

int gato_rollout(gato_solver_t* s, void* stream, int steps, const void* d_goal_traj, void* d_xu,
                 const void* d_noise, void* d_x, void* d_u, void* d_ckpt_xu, void* d_ckpt_rho)
{
    RC(check_handle(s));
    if (s->form != GATO_FORM_FUSED) return fail(GATO_ERR_UNSUPPORTED, "rollout needs the fused form");
    if (steps < 1) return fail(GATO_ERR_ARG, "steps must be positive");
    if (!d_goal_traj || !d_xu || !d_x || !d_u) return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    RC(rollout_alloc(s));
    cudaStream_t st = as_stream(stream);
    std::vector<const void*> key = {d_goal_traj, d_xu, d_noise, d_x, d_u, d_ckpt_xu, d_ckpt_rho,
                                    (const void*)st, (const void*)(intptr_t)steps};
    if (s->rexec && key == s->rkey && s->rver == s->version) {
        CK(cudaGraphLaunch(s->rexec, st));
        return GATO_OK;
    }
    if (s->rexec) {
        cudaGraphExecDestroy(s->rexec);
        s->rexec = nullptr;
    }
    RC(dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        return capture_and_launch(st, [&](cudaStream_t cap) {
            return enqueue_rollout<Tg>(s, cap, steps, d_goal_traj, d_xu, d_noise, d_x, d_u,
                                       d_ckpt_xu, d_ckpt_rho);
        }, &s->rexec);
    }));
    s->rkey = key;
    s->rver = s->version;
    return GATO_OK;
}

int gato_rollout_backward(gato_solver_t* s, void* stream, int steps, const void* d_goal_traj,
                          const void* d_x, const void* d_u, const void* d_ckpt_xu,
                          const void* d_ckpt_rho, const void* d_dl_dx, void* d_g_x0,
                          void* d_g_goal_traj, void* d_g_wdiag, double tol, int max_iters)
{
    RC(check_handle(s));
    if (s->form != GATO_FORM_FUSED) return fail(GATO_ERR_UNSUPPORTED, "rollout needs the fused form");
    if (steps < 1) return fail(GATO_ERR_ARG, "steps must be positive");
    if (!d_goal_traj || !d_x || !d_u || !d_ckpt_xu || !d_ckpt_rho || !d_dl_dx || !d_g_x0 ||
        !d_g_goal_traj || !d_g_wdiag)
        return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    RC(rollout_alloc(s));
    RC(adj_alloc(s));
    const bool f64 = s->precision == GATO_PREC_FP64;
    if (tol <= 0) tol = f64 ? 1e-20 : 1e-12;
    if (max_iters <= 0) max_iters = 4 * s->N * s->nq;
    cudaStream_t st = as_stream(stream);
    cudaGraphExec_t exec = nullptr;
    int rc = dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        return capture_and_launch(st, [&](cudaStream_t cap) {
            return enqueue_rollout_backward<Tg>(s, cap, steps, d_goal_traj, d_x, d_u, d_ckpt_xu,
                                                d_ckpt_rho, d_dl_dx, d_g_x0, d_g_goal_traj,
                                                d_g_wdiag, tol, max_iters);
        }, &exec);
    });
    if (exec) {
        cudaStreamSynchronize(st);
        cudaGraphExecDestroy(exec);
    }
    return rc;
}

}  // extern "C"

// --- batched PCG with no device allocation -------------------------------------
// A model-predictive controller that re-solves every millisecond cannot call
// cudaMalloc inside its control loop: the call may synchronise the whole
// device and its latency has no bound.  Hosts whose device memory belongs to
// another allocator (a framework's pool, a pre-reserved real-time budget)
// cannot let a library allocate either.  gato_pcg_static runs the PCG stage
// of gato_stage_pcg on caller-owned buffers without a solver handle.  The
// only device scratch that PCG kernel needs besides its operands (one
// "already converged" flag and one stopping tolerance per problem) lives in
// the file-scope array below instead of solver-owned buffers.
namespace {

constexpr int PCG_STATIC_MAX_BATCH = GATO_PCG_STATIC_MAX_BATCH;
// [0, 4*MAX): int converged flags, [4*MAX, 8*MAX): float tolerances (64 KiB)
constexpr size_t PCG_STATIC_SCRATCH_BYTES =
    (size_t)PCG_STATIC_MAX_BATCH * (sizeof(int) + sizeof(float));
static __device__ __align__(256) unsigned char g_pcg_scratch[PCG_STATIC_SCRATCH_BYTES];

constexpr int PCG_STATIC_MAX_DEVICES = 64;
struct PcgStaticDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_pcg_scratch
    int max_smem = 0;
};
PcgStaticDevice g_pcg_static[PCG_STATIC_MAX_DEVICES];
std::mutex g_pcg_static_mu;

// flags := 0 (no problem is skipped), tolerances := pcg_tol
__global__ void k_pcg_static_init(int* conv, float* tol, int B, float pcg_tol)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < B) {
        conv[b] = 0;
        tol[b] = pcg_tol;
    }
}

// One-time set-up per device, run with that device current: look up the
// device address of the scratch array and raise the PCG kernels' shared
// memory limit (the same value configure_kernels sets).
int pcg_static_setup(int dev, PcgStaticDevice** out)
{
    std::lock_guard<std::mutex> lock(g_pcg_static_mu);
    PcgStaticDevice& d = g_pcg_static[dev];
    if (!d.ready) {
        void* p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_pcg_scratch));
        int sm = 0;
        CK(cudaDeviceGetAttribute(&sm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        CK(cudaFuncSetAttribute(k_pcg<6, float, float>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        CK(cudaFuncSetAttribute(k_pcg<7, float, float>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        d.scratch = static_cast<unsigned char*>(p);
        d.max_smem = sm;
        d.ready = true;
    }
    *out = &d;
    return GATO_OK;
}

template <int NQ>
int pcg_static_launch(const PcgStaticDevice& d, cudaStream_t st, int N, int B, float pcg_tol,
                      int max_pcg_iters, const float* S, const float* Pinv, const float* gamma,
                      float* lambda, int32_t* iters)
{
    int* conv = reinterpret_cast<int*>(d.scratch);
    float* tol = reinterpret_cast<float*>(d.scratch + (size_t)PCG_STATIC_MAX_BATCH * sizeof(int));
    const bool stage = pcg_smem_bytes<NQ, float>(N, true) <= (size_t)d.max_smem;
    const size_t sm = pcg_smem_bytes<NQ, float>(N, stage);
    if (sm > (size_t)d.max_smem)
        return fail(GATO_ERR_UNSUPPORTED, "N=%d needs %zu bytes of shared memory", N, sm);
    Batch<NQ, float> bt{};
    bt.B = B;
    bt.N = N;
    bt.max_pcg_iters = max_pcg_iters;
    bt.abs_tol = 1e-6f;
    bt.S = const_cast<float*>(S);
    bt.P = const_cast<float*>(Pinv);
    bt.gamma = const_cast<float*>(gamma);
    bt.lambda = lambda;
    bt.pcg_iters = iters;
    bt.conv = conv;
    bt.tol = tol;
    k_pcg_static_init<<<cdiv(B, 256), 256, 0, st>>>(conv, tol, B, pcg_tol);
    CKL();
    k_pcg<NQ, float, float><<<B, PCG_THREADS, sm, st>>>(bt, stage, -1);
    CKL();
    return GATO_OK;
}

}  // namespace

extern "C" int gato_pcg_static(void* stream, int nq, int N, int batch, float pcg_tol,
                               int max_pcg_iters, const float* d_S, const float* d_Pinv,
                               const float* d_gamma, float* d_lambda, int32_t* d_iters)
{
    if (nq != 6 && nq != 7) return fail(GATO_ERR_UNSUPPORTED, "nq=%d: built for 6 or 7", nq);
    if (N < 2 || N > 256) return fail(GATO_ERR_ARG, "N=%d out of range [2, 256]", N);
    if (batch < 1 || batch > PCG_STATIC_MAX_BATCH)
        return fail(GATO_ERR_ARG, "batch=%d out of range [1, %d] of the static scratch", batch,
                    PCG_STATIC_MAX_BATCH);
    if (max_pcg_iters < 0) return fail(GATO_ERR_ARG, "negative max_pcg_iters");
    if (!d_S || !d_Pinv || !d_gamma || !d_lambda || !d_iters)
        return fail(GATO_ERR_ARG, "null device buffer");
    if (((uintptr_t)d_S | (uintptr_t)d_Pinv) & 15)
        return fail(GATO_ERR_ARG, "S and Pinv must be 16-byte aligned");
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= PCG_STATIC_MAX_DEVICES)
        return fail(GATO_ERR_UNSUPPORTED, "device %d beyond the %d supported", dev,
                    PCG_STATIC_MAX_DEVICES);
    PcgStaticDevice* d = nullptr;
    RC(pcg_static_setup(dev, &d));
    cudaStream_t st = as_stream(stream);
    if (nq == 6)
        return pcg_static_launch<6>(*d, st, N, batch, pcg_tol, max_pcg_iters, d_S, d_Pinv,
                                    d_gamma, d_lambda, d_iters);
    return pcg_static_launch<7>(*d, st, N, batch, pcg_tol, max_pcg_iters, d_S, d_Pinv, d_gamma,
                                d_lambda, d_iters);
}

// --- mixed batches (several plants and horizons in one solve) -------------------
struct gato_mixed {
    int ncls = 0, precision = 0, device = 0, nsm = 0;
    gato_solver* cls[MULTI_MAX_CLASSES] = {};
    int2* d_items = nullptr;  // every problem, longest horizon first
    int nitems = 0;
    int2* d_rows = nullptr;   // problems whose PCG fits one CTA's registers
    int nrows = 0;
    int* d_heads = nullptr;   // one work-queue counter per launch of a solve
    int nheads = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<const void*> gkey;
    long gver = -1;
    int kg = 16, ppb = 1, occ = 2;  // KKT lanes per knot, problems per CTA, CTAs per SM
};

namespace {

template <typename T, typename Acc>
void mixed_args(gato_mixed* mx, void* const* xu, const void* const* xs, const void* const* goal,
                MultiArgs<T>& ma)
{
    ma = MultiArgs<T>{};
    for (int c = 0; c < mx->ncls; ++c) {
        gato_solver* s = mx->cls[c];
        ma.nq[c] = s->nq;
        if (s->nq == 7) {
            ma.b7[c] = make_batch<Tag<7, T, Acc>>(s, xu[c], xs[c], goal[c]);
            ma.m7 = dmodel<Tag<7, T, Acc>>(s);
        } else {
            ma.b6[c] = make_batch<Tag<6, T, Acc>>(s, xu[c], xs[c], goal[c]);
            ma.m6 = dmodel<Tag<6, T, Acc>>(s);
        }
    }
}

template <typename T>
bool rows_fit(const gato_solver* s)
{
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
    return s->nq == 7 ? RowPcg<7, RPT>::fits(s->N) : RowPcg<6, RPT>::fits(s->N);
}

template <typename T, typename Acc, int KG, int PPB, int MINB>
int launch_q_fused(gato_mixed* mx, cudaStream_t st, const MultiArgs<T>& ma, int it)
{
    int team_bytes = 0;
    for (int c = 0; c < mx->ncls; ++c) {
        const gato_solver* s = mx->cls[c];
        const int w = 8 / PPB;
        const size_t by = s->nq == 7 ? FusedLayout<7, T>{s->N, w, false}.bytes()
                                     : FusedLayout<6, T>{s->N, w, false}.bytes();
        team_bytes = std::max(team_bytes, (int)((by + 255) & ~(size_t)255));
    }
    const size_t smem = (size_t)PPB * team_bytes;
    auto kern = k_q_fused_iter<T, Acc, KG, PPB, MINB>;
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem));
    const int grid = std::max(1, std::min(mx->nsm * std::max(occ, 1), cdiv(ma.nitems, PPB)));
    kern<<<grid, 256, smem, st>>>(ma, it, team_bytes);
    CKL();
    return GATO_OK;
}

template <typename T, typename Acc>
int launch_q_fused_any(gato_mixed* mx, cudaStream_t st, const MultiArgs<T>& ma, int it)
{
    const int sel = (mx->kg == 32 ? 4 : 0) + (mx->ppb == 2 ? 2 : 0) + (mx->occ == 4 ? 1 : 0);
    switch (sel) {
        case 0: return launch_q_fused<T, Acc, 16, 1, 2>(mx, st, ma, it);
        case 1: return launch_q_fused<T, Acc, 16, 1, 4>(mx, st, ma, it);
        case 2: return launch_q_fused<T, Acc, 16, 2, 2>(mx, st, ma, it);
        case 3: return launch_q_fused<T, Acc, 16, 2, 4>(mx, st, ma, it);
        case 4: return launch_q_fused<T, Acc, 32, 1, 2>(mx, st, ma, it);
        case 5: return launch_q_fused<T, Acc, 32, 1, 4>(mx, st, ma, it);
        case 6: return launch_q_fused<T, Acc, 32, 2, 2>(mx, st, ma, it);
        default: return launch_q_fused<T, Acc, 32, 2, 4>(mx, st, ma, it);
    }
}

template <typename T, typename Acc>
int enqueue_mixed(gato_mixed* mx, cudaStream_t st, void* const* xu, const void* const* xs,
                  const void* const* goal)
{
    constexpr int RPT = sizeof(T) == 4 ? 2 : 1;
    MultiArgs<T> ma;
    mixed_args<T, Acc>(mx, xu, xs, goal, ma);
    int nmax = 0, rows_smem = 0;
    bool has_long = false;
    for (int c = 0; c < mx->ncls; ++c) {
        gato_solver* s = mx->cls[c];
        const Dims<7> d7{s->N};
        const size_t traj = (size_t)(3 * s->nq) * s->N - s->nq;
        (void)d7;
        CK(cudaMemsetAsync(s->dz, 0, s->esz * (size_t)s->B * traj, st));
        CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * s->B, st));
        CK(cudaMemsetAsync(s->sqp_iters, 0, sizeof(int) * s->B, st));
        CK(cudaMemsetAsync(s->done, 0, sizeof(int), st));
        CK(cudaMemsetAsync(s->ls_count, 0, sizeof(int), st));
        nmax = std::max(nmax, s->N);
        if (rows_fit<T>(s)) {
            const size_t by = s->nq == 7 ? RowPcg<7, RPT>::template smem_bytes<T>(s->N)
                                         : RowPcg<6, RPT>::template smem_bytes<T>(s->N);
            rows_smem = std::max(rows_smem, (int)by);
        } else {
            has_long = true;
        }
    }
    CK(cudaMemsetAsync(mx->d_heads, 0, sizeof(int) * mx->nheads, st));
    int slot = 0;
    auto queue = [&](int2* items, int n) {
        MultiArgs<T> a = ma;
        a.items = items;
        a.nitems = n;
        a.head = mx->d_heads + slot++;
        return a;
    };
    const size_t merit_smem = (size_t)NUM_ALPHAS * nmax * sizeof(Acc);
    int occ_m = 0, occ_r = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_q_merit_ls<T, Acc>, 256,
                                                     merit_smem));
    const int grid_m = std::max(1, std::min(mx->nsm * std::max(occ_m, 1), mx->nitems));
    const int rows_threads = RowPcg<7, RPT>::MAX_THREADS;
    if (mx->nrows) {
        if (rows_smem > 48 * 1024)
            CK(cudaFuncSetAttribute(k_q_pcg_rows<T, Acc>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, rows_smem));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_r, k_q_pcg_rows<T, Acc>,
                                                         rows_threads, rows_smem));
    }
    const int grid_r = std::max(1, std::min(mx->nsm * std::max(occ_r, 1), mx->nrows));
    const int iters = mx->cls[0]->params.max_sqp_iters;
    k_q_merit_ls<T, Acc><<<grid_m, 256, merit_smem, st>>>(queue(mx->d_items, mx->nitems), 0, 0);
    CKL();
    for (int it = 0; it < iters; ++it) {
        RC((launch_q_fused_any<T, Acc>(mx, st, queue(mx->d_items, mx->nitems), it)));
        if (has_long) {
            CK(cudaEventRecord(mx->fork, st));
            CK(cudaStreamWaitEvent(mx->side, mx->fork, 0));
            for (int c = 0; c < mx->ncls; ++c) {
                gato_solver* s = mx->cls[c];
                if (rows_fit<T>(s)) continue;
                if (s->nq == 7)
                    RC((launch_pcg_cluster<Tag<7, T, Acc>>(s, mx->side, ma.b7[c], it)));
                else
                    RC((launch_pcg_cluster<Tag<6, T, Acc>>(s, mx->side, ma.b6[c], it)));
            }
            CK(cudaEventRecord(mx->join, mx->side));
        }
        if (mx->nrows) {
            k_q_pcg_rows<T, Acc><<<grid_r, rows_threads, rows_smem, st>>>(
                queue(mx->d_rows, mx->nrows), it);
            CKL();
        }
        if (has_long) CK(cudaStreamWaitEvent(st, mx->join, 0));
        k_q_check<T><<<mx->ncls, 1024, 0, st>>>(ma);
        CKL();
        k_q_merit_ls<T, Acc><<<grid_m, 256, merit_smem, st>>>(queue(mx->d_items, mx->nitems), 1,
                                                              it);
        CKL();
    }
    k_q_merit_ls<T, Acc><<<grid_m, 256, merit_smem, st>>>(queue(mx->d_items, mx->nitems), 2, 0);
    CKL();
    for (int c = 0; c < mx->ncls; ++c) {
        gato_solver* s = mx->cls[c];
        CK(cudaMemcpyAsync(s->drho, s->drho_init_d, s->esz * s->B, cudaMemcpyDeviceToDevice, st));
    }
    return GATO_OK;
}

int mixed_enqueue(gato_mixed* mx, cudaStream_t st, void* const* xu, const void* const* xs,
                  const void* const* goal)
{
    if (mx->precision == GATO_PREC_FP64) return enqueue_mixed<double, double>(mx, st, xu, xs, goal);
    if (mx->precision == GATO_PREC_MIXED) return enqueue_mixed<float, double>(mx, st, xu, xs, goal);
    return enqueue_mixed<float, float>(mx, st, xu, xs, goal);
}

long mixed_version(const gato_mixed* mx)
{
    long v = (mx->kg * 7 + mx->ppb) * 5 + mx->occ;
    for (int c = 0; c < mx->ncls; ++c) v = v * 131 + mx->cls[c]->version;
    return v;
}

int mixed_solve(gato_mixed* mx, cudaStream_t st, void* const* xu, const void* const* xs,
                const void* const* goal)
{
    std::vector<const void*> key;
    for (int c = 0; c < mx->ncls; ++c) {
        key.push_back(xu[c]);
        key.push_back(xs[c]);
        key.push_back(goal[c]);
    }
    key.push_back((const void*)st);
    const long ver = mixed_version(mx);
    if (!mx->gexec || key != mx->gkey || ver != mx->gver) {
        if (mx->gexec) {
            cudaGraphExecDestroy(mx->gexec);
            mx->gexec = nullptr;
        }
        cudaStream_t cap;
        CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        CK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        int rc = mixed_enqueue(mx, cap, xu, xs, goal);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        cudaStreamDestroy(cap);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&mx->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(GATO_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        mx->gkey = key;
        mx->gver = ver;
    }
    for (int c = 0; c < mx->ncls; ++c) CK(cudaEventRecord(mx->cls[c]->ev0, st));
    CK(cudaEventRecord(mx->ev0, st));
    CK(cudaGraphLaunch(mx->gexec, st));
    CK(cudaEventRecord(mx->ev1, st));
    for (int c = 0; c < mx->ncls; ++c) CK(cudaEventRecord(mx->cls[c]->ev1, st));
    return GATO_OK;
}

int check_mixed(const gato_mixed* mx)
{
    if (!mx) return fail(GATO_ERR_ARG, "null mixed-batch handle");
    return GATO_OK;
}

}  // namespace

extern "C" {

int gato_mixed_create(const gato_class_t* classes, int nclasses, const gato_params_t* params,
                      int precision, gato_mixed_t** out)
{
    if (!out) return fail(GATO_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (!classes || !params) return fail(GATO_ERR_ARG, "null classes or params");
    if (nclasses < 1 || nclasses > MULTI_MAX_CLASSES)
        return fail(GATO_ERR_ARG, "%d classes: 1 to %d supported", nclasses, MULTI_MAX_CLASSES);
    std::unique_ptr<gato_mixed> mx(new gato_mixed);
    mx->ncls = nclasses;
    mx->precision = precision;
    auto cleanup = [&]() {
        for (int c = 0; c < nclasses; ++c)
            if (mx->cls[c]) gato_destroy(mx->cls[c]);
    };
    for (int c = 0; c < nclasses; ++c) {
        gato_model_t m;
        int rc = gato_builtin_model(classes[c].plant, &m);
        if (rc) {
            cleanup();
            return rc;
        }
        rc = gato_create(&m, classes[c].N, classes[c].count, params, GATO_FORM_FUSED, precision,
                         &mx->cls[c]);
        if (rc) {
            cleanup();
            return rc;
        }
    }
    const bool f64 = precision == GATO_PREC_FP64;
    std::vector<int> order(nclasses);
    for (int c = 0; c < nclasses; ++c) order[c] = c;
    // longest horizon (then larger plant) first: the work queue hands out the
    // most expensive problems before the cheap ones fill the tail
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const gato_solver *sa = mx->cls[a], *sb = mx->cls[b];
        return sa->N != sb->N ? sa->N > sb->N : sa->nq > sb->nq;
    });
    std::vector<int2> all, rows;
    for (int c : order)
        for (int b = 0; b < mx->cls[c]->B; ++b) {
            all.push_back(make_int2(c, b));
            const bool fit = f64 ? rows_fit<double>(mx->cls[c]) : rows_fit<float>(mx->cls[c]);
            if (fit) rows.push_back(make_int2(c, b));
        }
    mx->nitems = (int)all.size();
    mx->nrows = (int)rows.size();
    mx->nheads = 3 * std::max(1, params->max_sqp_iters) + 2;
    int err = GATO_OK;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && !err) err = fail(GATO_ERR_CUDA, "%s", cudaGetErrorString(e));
    };
    ck(cudaGetDevice(&mx->device));
    ck(cudaDeviceGetAttribute(&mx->nsm, cudaDevAttrMultiProcessorCount, mx->device));
    ck(cudaMalloc(&mx->d_items, sizeof(int2) * std::max(1, mx->nitems)));
    ck(cudaMalloc(&mx->d_rows, sizeof(int2) * std::max(1, mx->nrows)));
    ck(cudaMalloc(&mx->d_heads, sizeof(int) * mx->nheads));
    if (!err) ck(cudaMemcpy(mx->d_items, all.data(), sizeof(int2) * all.size(),
                            cudaMemcpyHostToDevice));
    if (!err && !rows.empty())
        ck(cudaMemcpy(mx->d_rows, rows.data(), sizeof(int2) * rows.size(), cudaMemcpyHostToDevice));
    ck(cudaStreamCreateWithFlags(&mx->side, cudaStreamNonBlocking));
    ck(cudaEventCreateWithFlags(&mx->fork, cudaEventDisableTiming));
    ck(cudaEventCreateWithFlags(&mx->join, cudaEventDisableTiming));
    ck(cudaEventCreate(&mx->ev0));
    ck(cudaEventCreate(&mx->ev1));
    if (err) {
        gato_mixed_destroy(mx.release());
        return err;
    }
    *out = mx.release();
    return GATO_OK;
}

int gato_mixed_destroy(gato_mixed_t* mx)
{
    if (!mx) return GATO_OK;
    if (mx->gexec) cudaGraphExecDestroy(mx->gexec);
    for (int c = 0; c < mx->ncls; ++c)
        if (mx->cls[c]) gato_destroy(mx->cls[c]);
    cudaFree(mx->d_items);
    cudaFree(mx->d_rows);
    cudaFree(mx->d_heads);
    if (mx->side) cudaStreamDestroy(mx->side);
    if (mx->fork) cudaEventDestroy(mx->fork);
    if (mx->join) cudaEventDestroy(mx->join);
    if (mx->ev0) cudaEventDestroy(mx->ev0);
    if (mx->ev1) cudaEventDestroy(mx->ev1);
    delete mx;
    return GATO_OK;
}

int gato_mixed_class(gato_mixed_t* mx, int c, gato_solver_t** out)
{
    RC(check_mixed(mx));
    if (!out || c < 0 || c >= mx->ncls) return fail(GATO_ERR_ARG, "class %d out of range", c);
    *out = mx->cls[c];
    return GATO_OK;
}

int gato_mixed_solve(gato_mixed_t* mx, void* stream, void* const* d_xu, const void* const* d_xs,
                     const void* const* d_goal)
{
    RC(check_mixed(mx));
    if (!d_xu || !d_xs || !d_goal) return fail(GATO_ERR_ARG, "null pointer array");
    for (int c = 0; c < mx->ncls; ++c)
        if (!d_xu[c] || !d_xs[c] || !d_goal[c]) return fail(GATO_ERR_ARG, "null buffer, class %d", c);
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != mx->device) CK(cudaSetDevice(mx->device));
    return mixed_solve(mx, as_stream(stream), d_xu, d_xs, d_goal);
}

int gato_mixed_stats(gato_mixed_t* mx, int c, gato_stats_t* stats)
{
    RC(check_mixed(mx));
    if (c < 0 || c >= mx->ncls || !stats) return fail(GATO_ERR_ARG, "bad class or stats");
    gato_solver* s = mx->cls[c];
    const int B = s->B;
    std::vector<int> hsqp(B), hconv(B);
    int rows = 0;
    CK(cudaEventSynchronize(mx->ev1));
    CK(cudaMemcpy(&rows, s->ls_count, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hsqp.data(), s->sqp_iters, sizeof(int) * B, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hconv.data(), s->conv, sizeof(int) * B, cudaMemcpyDeviceToHost));
    return read_stats(s, hsqp.data(), hconv.data(), rows, stats);
}

int gato_mixed_elapsed_ms(gato_mixed_t* mx, float* ms)
{
    RC(check_mixed(mx));
    if (!ms) return fail(GATO_ERR_ARG, "null output");
    CK(cudaEventSynchronize(mx->ev1));
    CK(cudaEventElapsedTime(ms, mx->ev0, mx->ev1));
    return GATO_OK;
}

int gato_mixed_config(gato_mixed_t* mx, int lanes_per_knot, int problems_per_block,
                      int ctas_per_sm)
{
    RC(check_mixed(mx));
    if ((lanes_per_knot != 16 && lanes_per_knot != 32) ||
        (problems_per_block != 1 && problems_per_block != 2) ||
        (ctas_per_sm != 2 && ctas_per_sm != 4))
        return fail(GATO_ERR_ARG, "lanes per knot 16|32, problems per block 1|2, CTAs per SM 2|4");
    mx->kg = lanes_per_knot;
    mx->ppb = problems_per_block;
    mx->occ = ctas_per_sm;
    return GATO_OK;
}

int gato_mixed_tune(gato_mixed_t* mx, void* stream, void* const* d_xu, const void* const* d_xs,
                    const void* const* d_goal, float* ms_out)
{
    RC(check_mixed(mx));
    cudaStream_t st = as_stream(stream);
    const int cand[8][3] = {{16, 1, 2}, {16, 1, 4}, {16, 2, 2}, {16, 2, 4},
                            {32, 1, 2}, {32, 1, 4}, {32, 2, 2}, {32, 2, 4}};
    // the solve changes XU, lambda, rho and drho: keep copies, restore them
    // before every trial and at the end
    std::vector<void*> saved;
    auto save = [&](const void* src, size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToDevice, st);
        saved.push_back(p);
        return p;
    };
    struct Keep {
        void *xu, *lam, *rho, *drho;
        size_t nxu, nlam, nb;
    };
    std::vector<Keep> keep(mx->ncls);
    for (int c = 0; c < mx->ncls; ++c) {
        gato_solver* s = mx->cls[c];
        const size_t traj = (size_t)(3 * s->nq) * s->N - s->nq, vecp = (size_t)(s->N + 2) * 2 * s->nq;
        Keep& k = keep[c];
        k.nxu = s->esz * s->B * traj;
        k.nlam = s->esz * s->B * vecp;
        k.nb = s->esz * s->B;
        k.xu = save(d_xu[c], k.nxu);
        k.lam = save(s->lambda, k.nlam);
        k.rho = save(s->rho, k.nb);
        k.drho = save(s->drho, k.nb);
        if (!k.xu || !k.lam || !k.rho || !k.drho) {
            for (void* p : saved) cudaFree(p);
            return fail(GATO_ERR_NOMEM, "tuning copies");
        }
    }
    auto restore = [&]() {
        for (int c = 0; c < mx->ncls; ++c) {
            gato_solver* s = mx->cls[c];
            cudaMemcpyAsync(d_xu[c], keep[c].xu, keep[c].nxu, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(s->lambda, keep[c].lam, keep[c].nlam, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(s->rho, keep[c].rho, keep[c].nb, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(s->drho, keep[c].drho, keep[c].nb, cudaMemcpyDeviceToDevice, st);
        }
    };
    int best = 0, rc = GATO_OK;
    float best_ms = 1e30f;
    for (int i = 0; i < 8 && rc == GATO_OK; ++i) {
        mx->kg = cand[i][0];
        mx->ppb = cand[i][1];
        mx->occ = cand[i][2];
        float t = 0.0f;
        for (int rep = 0; rep < 2 && rc == GATO_OK; ++rep) {  // the first run warms up
            restore();
            rc = mixed_solve(mx, st, d_xu, d_xs, d_goal);
            if (rc == GATO_OK) rc = gato_mixed_elapsed_ms(mx, &t);
        }
        if (ms_out) ms_out[i] = t;
        if (rc == GATO_OK && t < best_ms) {
            best_ms = t;
            best = i;
        }
    }
    restore();
    cudaStreamSynchronize(st);
    for (void* p : saved) cudaFree(p);
    mx->kg = cand[best][0];
    mx->ppb = cand[best][1];
    mx->occ = cand[best][2];
    return rc;
}

}  // extern "C"
