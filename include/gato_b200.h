/*
 * gato_b200 — C ABI of the batched SQP trajectory-optimisation solver for
 * NVIDIA B200 (sm_100a).
 *
 * This header is the drop-in boundary for the reference's pybind11 module
 * `bsqpN{N}_{plant}` (python/bindings.cu) and the solver class it wraps
 * (gato/bsqp/bsqp.cuh).  Every entry point below names the reference
 * interface it replaces.  The ABI uses plain C types only: pointers, sizes,
 * int status codes.  No C++ or torch types cross it.
 *
 * Conventions
 *   - n = 2*nq (state size), m = nq (control size), N knots, B problems.
 *   - XU trajectory per problem: [x_0 u_0 x_1 u_1 ... x_{N-1}], length
 *     (n+m)*N - m (gato/utils/linalg.cuh:624-634).
 *   - goal per problem: 6 floats per knot [px py pz r p y]; only xyz is used.
 *   - lambda per problem: (N+2)*n floats, one zero block padding each end
 *     (gato/utils/linalg.cuh:648-660).
 *   - Functions taking `d_` pointers expect device memory; `h_` pointers are
 *     host memory.  All return GATO_OK (0) or a negative error code;
 *     gato_last_error() gives the message of the last failure on the calling
 *     thread.
 *   - A solver handle is bound to the CUDA device that was current when it was
 *     created.  Calls on one handle must not overlap; distinct handles are
 *     independent.
 */
#ifndef GATO_B200_H
#define GATO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GATO_MAX_NQ 8

enum {
    GATO_OK = 0,
    GATO_ERR_ARG = -1,       /* invalid argument (size, pointer, enum) */
    GATO_ERR_CUDA = -2,      /* a CUDA runtime call failed */
    GATO_ERR_UNSUPPORTED = -3,
    GATO_ERR_NOMEM = -4,
    GATO_ERR_TIMEOUT = -5    /* a bounded device wait expired */
};

enum { GATO_PLANT_IIWA14 = 0, GATO_PLANT_INDY7 = 1 };

/* Solver forms.  Both run the same SQP method with the same batch semantics. */
enum {
    GATO_FORM_PLAIN = 0,  /* one kernel per stage, host convergence check per
                             SQP iteration (the reference's driver shape) */
    GATO_FORM_FUSED = 1   /* one persistent kernel per SQP stage group, device
                             side convergence, whole solve in a CUDA graph */
};

/* Arithmetic of the device path. */
enum {
    GATO_PREC_FP32 = 0,   /* everything FP32 (the reference's arithmetic) */
    GATO_PREC_MIXED = 1,  /* FP32 math, FP64 PCG inner products, alpha/beta
                             recurrences and merit reductions */
    GATO_PREC_FP64 = 2    /* everything FP64 (the reference's USE_DOUBLES build,
                             gato/settings.h:7-11, python/bindings.cu:244-252);
                             solves take double buffers (the _f64 entry points) */
};

/*
 * Robot description: a serial chain of revolute joints, each rotating about
 * the z axis of its joint frame (URDF <axis xyz="0 0 1"/>).  Joint i's frame is
 * placed in link i-1's frame by (joint_xyz, joint_rpy) exactly as the URDF
 * <origin> tag.  Up to two rigid bodies are fixed to each link (a link plus a
 * fixed child such as a flange); mass 0 marks an unused slot.
 * Replaces the compile-time GRiD tables of gato/dynamics/{iiwa14,indy7}/
 * *_grid.cuh (init_XImats, iiwa14_grid.cuh:1210-2098) and the limit tables of
 * gato/dynamics/iiwa14/iiwa14_plant.cuh:37-88.
 */
typedef struct gato_model {
    int nq;
    double joint_xyz[GATO_MAX_NQ][3];
    double joint_rpy[GATO_MAX_NQ][3];
    /* per link, per body: mass, com x y z, ixx ixy ixz iyy iyz izz (about the
       com, in the link frame's axes) */
    double link_inertial[GATO_MAX_NQ][2][10];
    double q_limit[GATO_MAX_NQ];   /* |q| limit (symmetric)   */
    double qd_limit[GATO_MAX_NQ];  /* |qd| limit (symmetric)  */
    double u_limit[GATO_MAX_NQ];   /* |u| limit (symmetric)   */
    double limit_margin;           /* added to the upper limit, subtracted from
                                      the lower: -0.1 tightens by 0.1 */
    double gravity;                /* 9.81 */
    int barrier_style;             /* 0: exact diagonal barrier Hessian
                                        (iiwa14_plant.cuh:113-155)
                                     1: outer product of barrier gradients
                                        (indy7_plant.cuh:141-147, 385-415) */
} gato_model_t;

/* Solver settings; the field meaning follows the BSQP constructor
   (gato/bsqp/bsqp.cuh:43-59, python/bsqp/interface.py:7-32). */
typedef struct gato_params {
    double dt;
    int max_sqp_iters;
    double kkt_tol;          /* accepted for interface parity; unused by the
                                method, as in bsqp.cuh:153 */
    int max_pcg_iters;
    double pcg_tol;
    double solve_ratio;
    double mu;
    double q_cost;
    double qd_cost;
    double u_cost;
    double N_cost;
    double q_lim_cost;
    double vel_lim_cost;
    double ctrl_lim_cost;
    double rho;
} gato_params_t;

/* Per-problem status word of a solve (gato_stats_t.status), a bit set.  The
   reference reports only kkt_converged, step_size = -1 on a failed line
   search and its rho reset (gato/bsqp/kernels/line_search.cuh:75-81,
   gato/bsqp/bsqp.cuh:153-156); these bits add what a caller needs to tell a
   failed problem from a slow one. */
enum {
    GATO_STATUS_CONVERGED = 1,    /* a PCG took zero iterations: the
                                     reference's kkt_converged */
    GATO_STATUS_MAX_ITER = 2,     /* the solve ended with the problem not
                                     converged (SQP iterations exhausted, or
                                     the batch stopped at solve_ratio) */
    GATO_STATUS_LS_FAIL = 4,      /* at least one line search found no step
                                     size that lowered the merit (step -1) */
    GATO_STATUS_NONFINITE = 8,    /* a non-finite merit: the problem's state,
                                     or every trial step of a line search */
    GATO_STATUS_PCG_MAX_ITER = 16 /* at least one PCG ran to max_pcg_iters */
};

/* Per-solve statistics, all host memory supplied by the caller; any pointer
   may be NULL.  Replaces the dict built in python/bindings.cu:96-147.
   Arrays indexed [iteration][problem] hold max_sqp_iters*B entries; the first
   ls_num_iters rows are valid. */
typedef struct gato_stats {
    double sqp_time_us;      /* device time of the solve (CUDA events) */
    int ls_num_iters;        /* SQP iterations that ran the line search */
    int32_t* sqp_iters;      /* [B] */
    int32_t* kkt_converged;  /* [B] */
    float* final_merit;      /* [B] */
    float* initial_merit;    /* [B] */
    int32_t* pcg_iters;      /* [max_sqp_iters][B] */
    float* ls_min_merit;     /* [max_sqp_iters][B] */
    float* ls_step_size;     /* [max_sqp_iters][B] */
    int32_t* status;         /* [B] GATO_STATUS_* bits (no counterpart in
                                the reference's dict) */
} gato_stats_t;

typedef struct gato_solver gato_solver_t;

/* Message of the last failing call on this thread ("" if none). */
const char* gato_last_error(void);

/* Version string of the library. */
const char* gato_version(void);

/* Fills *out with a built-in robot.  Replaces the compile-time plant choice
   PLANT_IIWA14 / PLANT_INDY7 (gato/settings.h:35-41). */
int gato_builtin_model(int plant, gato_model_t* out);

/* Creates a solver for `batch` problems of horizon N on the current device.
   Replaces BSQP<T,B>::BSQP (gato/bsqp/bsqp.cuh:43-59) and PyBSQP::PyBSQP
   (python/bindings.cu:27-56); N and batch are runtime values here
   (2 <= N <= 256, 1 <= batch <= 65536).  `form` is a GATO_FORM_* value and
   `precision` a GATO_PREC_* value. */
int gato_create(const gato_model_t* model, int N, int batch,
                const gato_params_t* params, int form, int precision,
                gato_solver_t** out);

/* Frees the solver and its device memory.  Replaces BSQP::~BSQP
   (bsqp.cuh:61, 258-297). */
void gato_destroy(gato_solver_t* s);

/* Sizes of the solver's per-problem vectors (floats). */
int gato_sizes(const gato_solver_t* s, int* nx, int* nu, int* traj_size,
               int* goal_size, int* lambda_size);

/* Runs the SQP solve on device buffers, stream-ordered on `stream`
   (a cudaStream_t, 0 = legacy default stream).  d_xu [B][traj] is updated in
   place; d_xs [B][nx] is the initial state; d_goal [B][6N] the end-effector
   goals.  Statistics are copied into *stats (may be NULL); when stats is
   non-NULL the call synchronises the stream before returning.
   Replaces BSQP<T,B>::solve (gato/bsqp/bsqp.cuh:103-197). */
int gato_solve(gato_solver_t* s, void* stream, float* d_xu, const float* d_xs,
               const float* d_goal, gato_stats_t* stats);

/* Same solve from host buffers: copies the inputs in, solves and copies XU
   back into h_xu.  Replaces PyBSQP::solve (python/bindings.cu:68-148). */
int gato_solve_host(gato_solver_t* s, float* h_xu, float dt, const float* h_xs,
                    const float* h_goal, gato_stats_t* stats);

/* The two solves above for GATO_PREC_FP64 solvers (double buffers), as the
   BSQP_{B}_double classes of the reference's USE_DOUBLES build. */
int gato_solve_f64(gato_solver_t* s, void* stream, double* d_xu, const double* d_xs,
                   const double* d_goal, gato_stats_t* stats);
int gato_solve_host_f64(gato_solver_t* s, double* h_xu, double dt, const double* h_xs,
                        const double* h_goal, gato_stats_t* stats);

/* Kernel groups reported by gato_profile_solve. */
enum {
    GATO_KERNEL_KKT = 0,
    GATO_KERNEL_SCHUR = 1,
    GATO_KERNEL_PCG = 2,
    GATO_KERNEL_DZ = 3,
    GATO_KERNEL_MERIT = 4,
    GATO_KERNEL_LINE_SEARCH = 5,
    GATO_KERNEL_FUSED_ITER = 6,
    GATO_KERNEL_CHECK = 7,
    GATO_KERNEL_MERIT_SUM = 8,
    GATO_KERNEL_COUNT = 9
};

/* Runs one solve like gato_solve (fused form without its CUDA graph) and
   brackets every kernel launch with CUDA events on `stream`; fills
   ms_by_kernel / launches_by_kernel [GATO_KERNEL_COUNT] with the summed
   device time and launch count per kernel group, and synchronises the stream.
   The reference only times the whole solve on the host (bsqp.cuh:109-190). */
int gato_profile_solve(gato_solver_t* s, void* stream, float* d_xu, const float* d_xs,
                       const float* d_goal, double* ms_by_kernel, int32_t* launches_by_kernel);
/* The same for FP64 solvers (double buffers). */
int gato_profile_solve_f64(gato_solver_t* s, void* stream, double* d_xu, const double* d_xs,
                           const double* d_goal, double* ms_by_kernel,
                           int32_t* launches_by_kernel);

/* Per-problem diagonal cost weights (no counterpart in the reference, whose
   weights are the scalars qd_cost and u_cost): h_wdiag [B][nx+nu] =
   [Qd_0..Qd_{nx-1}, Rd_0..Rd_{nu-1}] per problem; the stage cost gains
   1/2 Qd_i x_i^2 and 1/2 Rd_i u_i^2 in place of 1/2 qd_cost |qd|^2 and
   1/2 u_cost |u|^2, so Qd = [0, qd_cost], Rd = u_cost is the reference's
   cost.  NULL returns to the scalar weights.  These are the Q/R diagonals
   that gato_adjoint differentiates. */
int gato_set_cost_diag_batch(gato_solver_t* s, const float* h_wdiag);
/* The same with FP64 weights, kept at full precision by FP64 solvers (FP32
   and mixed solvers round them to float). */
int gato_set_cost_diag_batch_f64(gato_solver_t* s, const double* h_wdiag);
/* Batched setters (host arrays of B floats, or 6*B for f_ext; FP64 solvers
   widen them).
   Replace BSQP::set_f_ext_batch / set_rho_penalty_batch / set_drho_batch /
   set_mu_batch / set_pcg_tol_batch (gato/bsqp/bsqp.cuh:63-83) and their
   bindings (python/bindings.cu:150-178). */
int gato_set_f_ext_batch(gato_solver_t* s, const float* h_f_ext);
int gato_set_rho_penalty_batch(gato_solver_t* s, const float* h_rho,
                               int set_as_reset_default);
int gato_set_drho_batch(gato_solver_t* s, const float* h_drho,
                        int set_as_reset_default);
int gato_set_mu_batch(gato_solver_t* s, const float* h_mu);
int gato_set_pcg_tol_batch(gato_solver_t* s, const float* h_tol);

/* Sets the time step used by gato_solve (gato_solve_host takes it per call,
   as PyBSQP::solve does). */
int gato_set_dt(gato_solver_t* s, float dt);

/* Bounds of the device-side waits of the PCG kernels that bring S and P^-1
   into shared memory by bulk copy, the persistent FP32 PCG and the FP64 PCG
   (no counterpart in the reference, which has no bulk copies): how many
   mbarrier try_wait calls (each suspends the waiting thread for at most about
   a microsecond) a CTA makes before it gives up on a problem's S / P^-1
   copy (copy_tries) and, FP32 only, on the step recovery's A_k / Qi_k copy
   (step_copy_tries).  A wait that gives up lets the copies in flight land,
   and the next synchronising call on the handle returns GATO_ERR_TIMEOUT
   (the results of that solve are not valid).  A negative value restores
   the default (about four million tries: seconds); 0 gives up at once, which
   is how the tests exercise this path. */
int gato_set_wait_limits(gato_solver_t* s, int copy_tries, int step_copy_tries);

/* FP64 solvers only (no counterpart in the reference): nonzero applies the
   preconditioner P^-1 in FP32 inside the FP64 PCG (its rows rounded to FP32
   in shared memory, applied to an FP32 copy of the residual) while S, the
   residual, every inner product and the CG recurrence stay FP64.  P^-1 only
   steers the iteration, so the solution keeps FP64's accuracy up to where
   the PCG stops; iteration counts can differ from the FP64 oracle's where its
   stop is marginal.  It applies where the one-CTA-per-problem PCG runs (the
   fused form, gato_adjoint, gato_qp_step_f64, up to N = 36 for iiwa14 and 42
   for indy7); the plain form's PCG and the cluster PCG of longer horizons are
   unaffected.  Default off. */
int gato_set_fp32_preconditioner(gato_solver_t* s, int enabled);

/* Zeroes the dual warm start.  Replaces BSQP::reset_dual (bsqp.cuh:85). */
int gato_reset_dual(gato_solver_t* s);
/* Restores rho and drho to their reset defaults.  Replaces BSQP::reset_rho
   (bsqp.cuh:87-91). */
int gato_reset_rho(gato_solver_t* s);
/* Enables/disables rho adaptation.  Replaces BSQP::set_rho_adaptation
   (bsqp.cuh:93). */
int gato_set_rho_adaptation(gato_solver_t* s, int enabled);

/* Copies the dual warm start lambda [B][(N+2)*nx] out of / into the solver
   (host memory).  The reference keeps it device-internal (bsqp.cuh:81). */
int gato_get_lambda(gato_solver_t* s, float* h_lambda);
int gato_set_lambda(gato_solver_t* s, const float* h_lambda);
int gato_get_lambda_f64(gato_solver_t* s, double* h_lambda);
int gato_set_lambda_f64(gato_solver_t* s, const double* h_lambda);
/* Copies the current penalty rho [B] out (host memory). */
int gato_get_rho(gato_solver_t* s, float* h_rho);

/* One integrator step of every problem from the same (x_k, u_k) under each
   problem's own f_ext: h_xkp1 [B][nx] from h_xk [nx], h_uk [nu].
   Replaces BSQP::sim_forward / PyBSQP::sim_forward (bsqp.cuh:95,
   python/bindings.cu:180-194, gato/bsqp/kernels/sim.cuh:14-86). */
int gato_sim_forward(gato_solver_t* s, const float* h_xk, const float* h_uk,
                     float dt, float* h_xkp1);

/* Batch-hypothesis selection of the reference's MPC loop
   (python/bsqp/mpc_controller.py:295-309 evaluate_best_trajectory and the
   warm-start broadcast at 241-242), on the device and stream-ordered: every
   problem b simulates (d_x_last [nx], d_u_last [nu]) for dt under its own
   wrench hypothesis (the f_ext batch of gato_set_f_ext_batch), d_err [B]
   receives |x_b - d_x_curr|_2 and d_best [1] the index of the smallest
   error (numpy.argmin order: a NaN error counts as smallest, ties go to the
   lower index); when d_xu [B][traj] is non-NULL every row is overwritten
   with row best, the chosen trajectory as every problem's next warm start.
   Buffers in the solver's scalar type; no host synchronisation.  The
   reference's force-estimator update that consumes d_err stays on the host
   (examples/force_estimator.py). */
int gato_select_hypothesis(gato_solver_t* s, void* stream, const void* d_x_last,
                           const void* d_u_last, const void* d_x_curr, double dt,
                           void* d_xu, void* d_err, int32_t* d_best);

/*
 * Stage-level entry points on device buffers, for parity testing and custom
 * drivers.  Layouts follow the reference's batch layouts:
 *   Q [B][N][n*n], R [B][N][m*m], q [B][N][n], r [B][N][m], A [B][N][n*n],
 *   B [B][N][n*m], c [B][N][n] (column-major blocks, gato/types.cuh:65-73);
 *   S, Pinv [B][N][3*n*n] row-major block rows; gamma [B][(N+2)*n].
 */
/* Replaces setupKKTSystemBatched (gato/bsqp/kernels/setup_kkt.cuh:130-157). */
int gato_stage_setup_kkt(gato_solver_t* s, void* stream, const float* d_xu,
                         const float* d_xs, const float* d_goal, float* d_Q,
                         float* d_R, float* d_q, float* d_r, float* d_A,
                         float* d_B, float* d_c);
/* Replaces formSchurSystemBatched (gato/bsqp/kernels/schur_linsys.cuh:295-308).
   Reads Q,R,q,r,A,B,c; writes S, Pinv, gamma, and overwrites d_Q/d_R with
   the inverses (Q+rho*I_q)^-1 and R^-1 as the reference does. */
int gato_stage_form_schur(gato_solver_t* s, void* stream, float* d_Q,
                          float* d_R, const float* d_q, const float* d_r,
                          const float* d_A, const float* d_B,
                          const float* d_c, float* d_S, float* d_Pinv,
                          float* d_gamma);
/* Replaces solvePCGBatched (gato/bsqp/kernels/pcg.cuh:157-166).  d_lambda is
   the warm start in, solution out; d_iters [B] receives iteration counts. */
int gato_stage_pcg(gato_solver_t* s, void* stream, const float* d_S,
                   const float* d_Pinv, const float* d_gamma, float* d_lambda,
                   int32_t* d_iters);

/* The QP step of one SQP iteration at d_xu, without line search: KKT
   blocks, Schur complement, PCG warm-started from the solver's lambda (which
   is left unchanged) and step recovery; d_dz [B][traj] receives dz.  No
   counterpart in the reference, whose step stays inside the solve
   (gato/bsqp/bsqp.cuh:116-140); it is the map gato_adjoint differentiates,
   exposed so that its derivative can be checked by finite differences on the
   device.  tol: relative PCG tolerance (< 0: the solver's pcg_tol; 0: no
   tolerance stop, every problem runs max_iters iterations unless its
   residual reaches exactly zero); max_iters <= 0: the solver's
   max_pcg_iters.  h_iters (optional, host [B]) receives the PCG counts. */
int gato_qp_step(gato_solver_t* s, void* stream, const float* d_xu,
                 const float* d_xs, const float* d_goal, float* d_dz, double tol,
                 int max_iters, int32_t* h_iters);
int gato_qp_step_f64(gato_solver_t* s, void* stream, const double* d_xu,
                     const double* d_xs, const double* d_goal, double* d_dz,
                     double tol, int max_iters, int32_t* h_iters);

/* Adjoint of the converged subproblem (no counterpart in the reference).
   For a loss l of the trajectory d_xu returned by gato_solve (same x_s and
   goals), gives dl/dx_s [B][nx], dl/dgoal [B][6N] (rpy entries 0) and
   dl/d(Qd, Rd) [B][nx+nu] (the diagonal weights of
   gato_set_cost_diag_batch; with scalar weights, Qd = [0, qd_cost],
   Rd = u_cost) from d_dl_dxu [B][(nx+nu)N-nu].  The trajectory is treated
   as xu + dz(theta), dz the solution of the QP formed at xu (exact at a
   converged solve): the KKT blocks are recomputed at xu, the transposed KKT
   system (the QP's own, it is symmetric) is solved through the same Schur
   complement and PCG, and the solver's lambda and rho are left unchanged.
   tol <= 0 / max_iters <= 0 select the defaults (relative PCG tolerance
   1e-12 in FP32 / 1e-20 in FP64, 4*N*nq iterations).  h_iters (optional,
   host [2][B]) receives the PCG iterations of the forward QP step and of the
   adjoint.  The first call allocates the adjoint's work buffers. */
int gato_adjoint(gato_solver_t* s, void* stream, const float* d_xu,
                 const float* d_xs, const float* d_goal, const float* d_dl_dxu,
                 float* d_g_xs, float* d_g_goal, float* d_g_wdiag, double tol,
                 int max_iters, int32_t* h_iters);
int gato_adjoint_f64(gato_solver_t* s, void* stream, const double* d_xu,
                     const double* d_xs, const double* d_goal,
                     const double* d_dl_dxu, double* d_g_xs, double* d_g_goal,
                     double* d_g_wdiag, double tol, int max_iters,
                     int32_t* h_iters);

/* Closed-loop receding-horizon rollout (no counterpart in the reference's
   solver; its MPC loop is Python around one solve per step,
   python/bsqp/mpc_controller.py).  Fused-form solvers only; buffers in the
   solver's scalar type.  For t = 0 .. steps-1: solve from x[t] with the goal
   window d_goal_traj[b][6t, 6t+6N) ([B][6(N+steps)]), warm start d_xu
   ([B][traj], its x_0 set to x[t]); apply u[t] = u_0 + noise[t]
   (d_noise [steps][B][nu] or NULL) to the same dynamics for one dt into
   x[t+1] (d_x [steps+1][B][nx], x[0] given); shift the warm start by one
   knot.  d_ckpt_xu [steps][B][traj] and d_ckpt_rho [steps][B] (or NULL)
   keep each step's solution and rho for gato_rollout_backward.  All steps
   run as one CUDA graph (captured on the first call, replayed while the
   pointers and step count stay the same). */
int gato_rollout(gato_solver_t* s, void* stream, int steps, const void* d_goal_traj,
                 void* d_xu, const void* d_noise, void* d_x, void* d_u,
                 void* d_ckpt_xu, void* d_ckpt_rho);
/* Reverse pass of a rollout for a loss of the states: from d_dl_dx
   [steps+1][B][nx] gives dl/dx[0] [B][nx], dl/dgoal_traj [B][6(N+steps)] and
   dl/d(Qd, Rd) [B][nx+nu] by chaining the simulator's step Jacobians with
   gato_adjoint of every step (the controls' dependence on the state and on
   the weights through each step's QP), from the checkpoints of
   gato_rollout; dynamics derivatives are recomputed, the solver's rho is
   restored afterwards.  tol / max_iters as in gato_adjoint.  Runs as one
   CUDA graph and waits for it. */
int gato_rollout_backward(gato_solver_t* s, void* stream, int steps,
                          const void* d_goal_traj, const void* d_x, const void* d_u,
                          const void* d_ckpt_xu, const void* d_ckpt_rho,
                          const void* d_dl_dx, void* d_g_x0, void* d_g_goal_traj,
                          void* d_g_wdiag, double tol, int max_iters);

/* No counterpart in the reference.  The PCG of gato_stage_pcg (FP32 arithmetic
   and reductions, every problem solved), with ONE relative tolerance pcg_tol
   for all problems (gato_stage_pcg uses the per-problem tolerances of
   gato_set_pcg_tol_batch), on caller-owned device buffers, with
   no solver handle and no device allocation, for callers that may not
   allocate: a control loop re-solving every millisecond cannot afford
   cudaMalloc's device-wide synchronisation, and some hosts hand all device
   memory to their own allocator.  Same buffer layout as gato_stage_pcg;
   d_S and d_Pinv 16-byte aligned; nq 6 or 7, 2 <= N <= 256,
   1 <= batch <= GATO_PCG_STATIC_MAX_BATCH (larger batches return
   GATO_ERR_ARG).  The per-problem scratch (converged flags and tolerances,
   GATO_PCG_STATIC_MAX_BATCH * 8 bytes) is one static device array in the
   library; every call re-initialises the part it uses on `stream` before the
   solve, so nothing has to start at zero.  Because the scratch is shared,
   calls on one device must not overlap: two calls in flight at once (other
   streams or host threads) race on it.  The first call on each device does
   a one-time set-up (scratch address lookup, kernel attribute) with that
   device current; make that first call before any stream capture begins.
   The set-up is kept per device for the life of the process: after a
   cudaDeviceReset of that device (which invalidates the looked-up address
   and the kernel attribute) do not call this entry point again in the same
   process. */
#define GATO_PCG_STATIC_MAX_BATCH 8192
int gato_pcg_static(void* stream, int nq, int N, int batch, float pcg_tol,
                    int max_pcg_iters, const float* d_S, const float* d_Pinv,
                    const float* d_gamma, float* d_lambda, int32_t* d_iters);

/* ---- Mixed batches (no counterpart in the reference, which builds one
   module per plant and horizon and one class per power-of-two batch; a mixed
   workload there is one call per module).  Problems are grouped into classes
   (plant, N, count); each class is an ordinary fused-form solver (buffers,
   lambda, rho, setters: gato_mixed_class), and every stage of an SQP
   iteration runs as ONE persistent launch over all classes that takes
   problems from a device work queue, longest horizon first; long horizons
   take the cluster PCG on a parallel branch.  The whole solve is one CUDA
   graph.  All classes share the parameters and precision. */
typedef struct {
    int plant; /* GATO_PLANT_* */
    int N;     /* knots */
    int count; /* problems of this class */
} gato_class_t;
typedef struct gato_mixed gato_mixed_t;

int gato_mixed_create(const gato_class_t* classes, int nclasses,
                      const gato_params_t* params, int precision,
                      gato_mixed_t** out);
int gato_mixed_destroy(gato_mixed_t* mx);
/* the solver of class c (owned by mx): setters, lambda, rho, stats buffers */
int gato_mixed_class(gato_mixed_t* mx, int c, gato_solver_t** out);
/* d_xu / d_xs / d_goal: host arrays of nclasses device pointers (the
   solver scalar type), laid out per class as for gato_solve. */
int gato_mixed_solve(gato_mixed_t* mx, void* stream, void* const* d_xu,
                     const void* const* d_xs, const void* const* d_goal);
/* per-class statistics of the last solve (waits for it) */
int gato_mixed_stats(gato_mixed_t* mx, int c, gato_stats_t* stats);
/* device time of the last solve in ms (waits for it) */
int gato_mixed_elapsed_ms(gato_mixed_t* mx, float* ms);
/* KKT-stage launch shape: lanes per knot (16: two knots per warp, 32: one),
   problems per CTA (1 or 2) and CTAs per SM (2 or 4: registers per thread
   traded for resident warps) */
int gato_mixed_config(gato_mixed_t* mx, int lanes_per_knot,
                      int problems_per_block, int ctas_per_sm);
/* Autotuner: times the solve of these inputs under each launch shape
   (lanes per knot x problems per CTA x CTAs per SM, in the order (16,1,2)
   (16,1,4) (16,2,2) (16,2,4) (32,1,2) (32,1,4) (32,2,2) (32,2,4); ms_out[8]
   optional), restores XU, lambda, rho and drho after every trial, and keeps
   the fastest shape.  Allocates temporary copies. */
int gato_mixed_tune(gato_mixed_t* mx, void* stream, void* const* d_xu,
                    const void* const* d_xs, const void* const* d_goal,
                    float* ms_out);

#ifdef __cplusplus
}
#endif

#endif /* GATO_B200_H */
