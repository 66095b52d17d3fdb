// C ABI of mixed batches (gato_mixed_*, include/gato_b200.h): several plants
// and horizons solved together by persistent work-queue launches.
#include "solver.cuh"

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
    return s->nq == 7 ? rows_pcg_fits<7, T>(s->N) : rows_pcg_fits<6, T>(s->N);
}

template <typename T, typename Acc, int KG, int PPB, int MINB>
int launch_q_kkt(gato_mixed* mx, cudaStream_t st, const MultiArgs<T>& ma, int it)
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
    auto kern = k_q_kkt<T, Acc, KG, PPB, MINB>;
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem));
    const int grid = std::max(1, std::min(mx->nsm * std::max(occ, 1), cdiv(ma.nitems, PPB)));
    kern<<<grid, 256, smem, st>>>(ma, it, team_bytes);
    CKL();
    return GATO_OK;
}

// the Schur half: one problem per CTA, its own queue counter (ma.head)
template <typename T, typename Acc>
int launch_q_schur(gato_mixed* mx, cudaStream_t st, const MultiArgs<T>& ma, int it)
{
    size_t smem = 0;
    for (int c = 0; c < mx->ncls; ++c) {
        const gato_solver* s = mx->cls[c];
        const size_t by = s->nq == 7 ? FusedLayout<7, T>{s->N, 8, false}.bytes()
                                     : FusedLayout<6, T>{s->N, 8, false}.bytes();
        smem = std::max(smem, by);
    }
    auto kern = k_q_schur<T, Acc>;
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem));
    const int grid = std::max(1, std::min(mx->nsm * std::max(occ, 1), ma.nitems));
    kern<<<grid, 256, smem, st>>>(ma, it);
    CKL();
    return GATO_OK;
}

template <typename T, typename Acc>
int launch_q_kkt_any(gato_mixed* mx, cudaStream_t st, const MultiArgs<T>& ma, int it)
{
    const int sel = (mx->kg == 32 ? 4 : 0) + (mx->ppb == 2 ? 2 : 0) + (mx->occ == 4 ? 1 : 0);
    switch (sel) {
        case 0: return launch_q_kkt<T, Acc, 16, 1, 2>(mx, st, ma, it);
        case 1: return launch_q_kkt<T, Acc, 16, 1, 4>(mx, st, ma, it);
        case 2: return launch_q_kkt<T, Acc, 16, 2, 2>(mx, st, ma, it);
        case 3: return launch_q_kkt<T, Acc, 16, 2, 4>(mx, st, ma, it);
        case 4: return launch_q_kkt<T, Acc, 32, 1, 2>(mx, st, ma, it);
        case 5: return launch_q_kkt<T, Acc, 32, 1, 4>(mx, st, ma, it);
        case 6: return launch_q_kkt<T, Acc, 32, 2, 2>(mx, st, ma, it);
        default: return launch_q_kkt<T, Acc, 32, 2, 4>(mx, st, ma, it);
    }
}

template <typename T, typename Acc>
int enqueue_mixed(gato_mixed* mx, cudaStream_t st, void* const* xu, const void* const* xs,
                  const void* const* goal)
{
    constexpr int RPT = pcg_rows_per_thread<T>();
    MultiArgs<T> ma;
    mixed_args<T, Acc>(mx, xu, xs, goal, ma);
    int nmax = 0, rows_smem = 0;
    bool has_long = false;
    for (int c = 0; c < mx->ncls; ++c) {
        gato_solver* s = mx->cls[c];
        const size_t traj = (size_t)(3 * s->nq) * s->N - s->nq;
        CK(cudaMemsetAsync(s->dz, 0, s->esz * (size_t)s->B * traj, st));
        CK(cudaMemsetAsync(s->conv, 0, sizeof(int) * s->B, st));
        CK(cudaMemsetAsync(s->sqp_iters, 0, sizeof(int) * s->B, st));
        CK(cudaMemsetAsync(s->done, 0, sizeof(int), st));
        CK(cudaMemsetAsync(s->ls_count, 0, sizeof(int), st));
        CK(cudaMemsetAsync(s->status, 0, sizeof(int) * s->B, st));
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
        RC((launch_q_kkt_any<T, Acc>(mx, st, queue(mx->d_items, mx->nitems), it)));
        RC((launch_q_schur<T, Acc>(mx, st, queue(mx->d_items, mx->nitems), it)));
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
    mx->nheads = 4 * std::max(1, params->max_sqp_iters) + 2;  // KKT, Schur, PCG, merit per iteration
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
    return read_stats(s, hsqp.data(), hconv.data(), nullptr, rows, stats);
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
