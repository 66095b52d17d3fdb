// C ABI of the solver (include/gato_b200.h): solver object lifetime, solves,
// setters, stage entry points, adjoint, rollout, sim_forward and the
// no-allocation PCG.
#include "solver.cuh"

thread_local std::string g_err;

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
    CK(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device));
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
    RC(p->alloc(&p->work, 4));
    RC(p->alloc(&p->ls_count, 1));
    RC(p->alloc(&p->status, B));
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

static int profile_any(gato_solver_t* s, void* stream, void* d_xu, const void* d_xs,
                       const void* d_goal, double* ms_by_kernel, int32_t* launches_by_kernel)
{
    if (!d_xu || !d_xs || !d_goal || !ms_by_kernel || !launches_by_kernel)
        return fail(GATO_ERR_ARG, "null pointer");
    RC(bind_device(s));
    cudaStream_t st = as_stream(stream);
    std::vector<gato_solver::ProfEntry> entries;
    s->prof = &entries;
    std::vector<int> hs(s->B), hc(s->B), hst(s->B);
    int rows = 0;
    int rc = dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        if (s->form == GATO_FORM_PLAIN)
            return solve_plain<Tg>(s, st, d_xu, d_xs, d_goal, hs.data(), hc.data(), hst.data(),
                                   &rows);
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
    return check_device_waits(s);
}

int gato_profile_solve(gato_solver_t* s, void* stream, float* d_xu, const float* d_xs,
                       const float* d_goal, double* ms_by_kernel, int32_t* launches_by_kernel)
{
    RC(check_handle(s));
    RC(check_single(s));
    return profile_any(s, stream, d_xu, d_xs, d_goal, ms_by_kernel, launches_by_kernel);
}

int gato_profile_solve_f64(gato_solver_t* s, void* stream, double* d_xu, const double* d_xs,
                           const double* d_goal, double* ms_by_kernel,
                           int32_t* launches_by_kernel)
{
    RC(check_handle(s));
    RC(check_double(s));
    return profile_any(s, stream, d_xu, d_xs, d_goal, ms_by_kernel, launches_by_kernel);
}

int gato_set_fp32_preconditioner(gato_solver_t* s, int enabled)
{
    RC(check_handle(s));
    RC(check_double(s));
    if ((enabled != 0) != (s->p32 != 0)) {
        s->p32 = enabled != 0;
        s->version++;
    }
    return GATO_OK;
}

int gato_set_wait_limits(gato_solver_t* s, int copy_tries, int step_copy_tries)
{
    RC(check_handle(s));
    s->wait_tries = copy_tries < 0 ? PCG_STAGE_WAIT_TRIES : copy_tries;
    s->wait_tries_dz = step_copy_tries < 0 ? PCG_STAGE_WAIT_TRIES : step_copy_tries;
    s->version++;  // kernel arguments of the cached graph change
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

// v: the weights widened to double, or null to return to the scalar weights
static int set_cost_diag(gato_solver_t* s, const std::vector<double>* v)
{
    RC(check_handle(s));
    RC(bind_device(s));
    const int use = v != nullptr;
    if (use) {
        const size_t n = (size_t)3 * s->nq * s->B;
        for (double x : *v)
            if (!std::isfinite(x)) return fail(GATO_ERR_ARG, "non-finite cost weight");
        if (!s->wdiag) RC(s->alloc_t(&s->wdiag, n));
        RC(s->upload(s->wdiag, v->data(), n));
    }
    if (use != s->use_wdiag) {
        s->use_wdiag = use;
        s->version++;
    }
    return GATO_OK;
}

int gato_set_cost_diag_batch(gato_solver_t* s, const float* h_wdiag)
{
    RC(check_handle(s));
    if (!h_wdiag) return set_cost_diag(s, nullptr);
    std::vector<double> v(h_wdiag, h_wdiag + (size_t)3 * s->nq * s->B);
    return set_cost_diag(s, &v);
}

int gato_set_cost_diag_batch_f64(gato_solver_t* s, const double* h_wdiag)
{
    RC(check_handle(s));
    if (!h_wdiag) return set_cost_diag(s, nullptr);
    std::vector<double> v(h_wdiag, h_wdiag + (size_t)3 * s->nq * s->B);
    return set_cost_diag(s, &v);
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

int gato_select_hypothesis(gato_solver_t* s, void* stream, const void* d_x_last,
                           const void* d_u_last, const void* d_x_curr, double dt, void* d_xu,
                           void* d_err, int32_t* d_best)
{
    RC(check_handle(s));
    if (!d_x_last || !d_u_last || !d_x_curr || !d_err || !d_best)
        return fail(GATO_ERR_ARG, "null device buffer");
    if (!(dt > 0.0)) return fail(GATO_ERR_ARG, "dt must be positive");
    RC(bind_device(s));
    cudaStream_t st = as_stream(stream);
    return dispatch(s, [&](auto tg) {
        using Tg = decltype(tg);
        using T = typename Tg::T;
        const size_t sm = WPB * DynSmem<Tg::NQ>::SIZE * sizeof(T);
        k_hyp_error<Tg::NQ, T><<<cdiv(s->B, WPB), WPB * WARP, sm, st>>>(
            dmodel<Tg>(s), s->B, (T)dt, (const T*)d_x_last, (const T*)d_u_last,
            (const T*)d_x_curr, (const T*)s->fext, s->use_fext, (T*)d_err);
        CKL();
        k_hyp_argmin<T><<<1, 1024, 0, st>>>(s->B, (const T*)d_err, d_best);
        CKL();
        if (d_xu) {
            const int traj = (3 * s->nq) * s->N - s->nq;
            const size_t n = (size_t)s->B * traj;
            const int grid = (int)std::min<size_t>(cdiv((int)std::min<size_t>(n, 1u << 30), 256),
                                                   4 * (size_t)s->nsm);
            k_hyp_broadcast<T><<<grid, 256, 0, st>>>(s->B, traj, d_best, (T*)d_xu);
            CKL();
        }
        return (int)GATO_OK;
    });
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

static int qp_step_any(gato_solver_t* s, void* stream, void* d_xu, const void* d_xs,
                       const void* d_goal, void* d_dz, double tol, int max_iters,
                       int32_t* h_iters)
{
    if (!d_xu || !d_xs || !d_goal || !d_dz) return fail(GATO_ERR_ARG, "null device buffer");
    RC(bind_device(s));
    if (tol < 0) tol = (double)s->params.pcg_tol;
    if (max_iters <= 0) max_iters = s->params.max_pcg_iters;
    return dispatch(s, [&](auto tg) {
        return qp_step_impl<decltype(tg)>(s, as_stream(stream), d_xu, d_xs, d_goal, d_dz, tol,
                                          max_iters, h_iters);
    });
}

int gato_qp_step(gato_solver_t* s, void* stream, const float* d_xu, const float* d_xs,
                 const float* d_goal, float* d_dz, double tol, int max_iters, int32_t* h_iters)
{
    RC(check_handle(s));
    RC(check_single(s));
    return qp_step_any(s, stream, (void*)d_xu, d_xs, d_goal, d_dz, tol, max_iters, h_iters);
}

int gato_qp_step_f64(gato_solver_t* s, void* stream, const double* d_xu, const double* d_xs,
                     const double* d_goal, double* d_dz, double tol, int max_iters,
                     int32_t* h_iters)
{
    RC(check_handle(s));
    RC(check_double(s));
    return qp_step_any(s, stream, (void*)d_xu, d_xs, d_goal, d_dz, tol, max_iters, h_iters);
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

