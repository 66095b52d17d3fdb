/*
 * C ABI over the reference's own dynamics, plant-cost and integrator device
 * functions, compiled for the host in FP64 through the single-thread shim in
 * stub/.  Test infrastructure only (builds oracle/_ref/libgrid_ref_<plant>.so):
 * it runs the reference's code so the oracle's restatement can be pinned to
 * it, and generates the golden fixtures under tests/golden.
 *
 * Functions wrapped (paths in the reference tree):
 *   gato/dynamics/<plant>/<plant>_plant.cuh  forwardDynamics,
 *       forwardDynamicsAndGradient, trackingcost,
 *       trackingCostGradientAndHessian
 *   gato/dynamics/<plant>/<plant>_grid.cuh   end-effector pose and gradient
 *   gato/dynamics/integrator.cuh             compute_linearized_dynamics,
 *       compute_integrator_error
 */
#include <cuda_runtime.h>

shim_uint3 threadIdx = {0, 0, 0};
shim_uint3 blockIdx = {0, 0, 0};
shim_uint3 blockDim = {1, 1, 1};
shim_uint3 gridDim = {1, 1, 1};

#include "settings.h"
#include "constants.h"
#include "dynamics/integrator.cuh"

#include <vector>

typedef double Td;

static grid::robotModel<Td>* model()
{
    static grid::robotModel<Td>* m = grid::init_robotModel<Td>();
    return m;
}

static std::vector<Td>& scratch()
{
    static std::vector<Td> s(1 << 16, 0.0);
    return s;
}

#if defined(PLANT_IIWA14)
#define EE_POSE(out, q, tmp, mdl) grid::end_effector_pose_device<Td>(out, q, tmp, mdl)
#define EE_GRAD(out, q, tmp, mdl) grid::end_effector_pose_gradient_device<Td>(out, q, tmp, mdl)
#else
#define EE_POSE(out, q, tmp, mdl) grid::end_effector_positions_device<Td>(out, q, tmp, mdl)
#define EE_GRAD(out, q, tmp, mdl) grid::end_effector_positions_gradient_device<Td>(out, q, tmp, mdl)
#endif

extern "C" {

int ref_nq() { return grid::NQ; }
int ref_knot_points() { return KNOT_POINTS; }

/* qdd = FD(q, qd, u[, f_ext]) */
void ref_fd(const Td* q, const Td* qd, const Td* u, const Td* fext, Td* qdd)
{
    Td* s = scratch().data();
    Td sq[16], sqd[16], su[16], sf[6];
    for (int i = 0; i < grid::NQ; ++i) { sq[i] = q[i]; sqd[i] = qd[i]; su[i] = u[i]; }
    if (fext) {
        for (int i = 0; i < 6; ++i) sf[i] = fext[i];
        gato::plant::forwardDynamics<Td>(qdd, sq, sqd, su, s, model(), sf);
    } else {
        gato::plant::forwardDynamics<Td>(qdd, sq, sqd, su, s, model());
    }
}

/* qdd and df_du = [dqdd/dq | dqdd/dqd | Minv] (nq x 3nq column-major) */
void ref_fd_grad(const Td* q, const Td* qd, const Td* u, const Td* fext, Td* qdd, Td* df_du)
{
    Td* s = scratch().data();
    Td sf[6];
    if (fext) {
        for (int i = 0; i < 6; ++i) sf[i] = fext[i];
        gato::plant::forwardDynamicsAndGradient<Td>(df_du, qdd, q, qd, u, s, model(), sf);
    } else {
        gato::plant::forwardDynamicsAndGradient<Td>(df_du, qdd, q, qd, u, s, model());
    }
}

/* end-effector pose (6) and its gradient (6 x nq, column j at 6*j) */
void ref_ee(const Td* q, Td* pose, Td* grad)
{
    Td* s = scratch().data();
    Td sq[16];
    for (int i = 0; i < grid::NQ; ++i) sq[i] = q[i];
    EE_POSE(pose, sq, s, model());
    if (grad) EE_GRAD(grad, sq, s, model());
}

/* trackingcost at a knot; terminal selects the N_cost weight and drops the
   control terms (blockIdx.x == KNOT_POINTS-1 in the merit kernel) */
Td ref_tracking_cost(const Td* xu, const Td* goal, int terminal, Td q_cost, Td qd_cost, Td u_cost,
                    Td N_cost, Td q_lim_cost, Td vel_lim_cost, Td ctrl_lim_cost)
{
    Td* s = scratch().data();
    Td sxu[64], sg[6];
    int len = terminal ? 2 * grid::NQ : 3 * grid::NQ;
    for (int i = 0; i < len; ++i) sxu[i] = xu[i];
    for (int i = 0; i < 6; ++i) sg[i] = goal[i];
    blockIdx.x = terminal ? KNOT_POINTS - 1 : 0;
    Td c = gato::plant::trackingcost<Td>(2 * grid::NQ, grid::NQ, KNOT_POINTS, sxu, sg, s, model(),
                                      q_cost, qd_cost, u_cost, N_cost, q_lim_cost, vel_lim_cost,
                                      ctrl_lim_cost);
    blockIdx.x = 0;
    return c;
}

/* trackingCostGradientAndHessian at a non-terminal KKT knot */
void ref_cost_grad_hess(const Td* xu, const Td* goal, Td q_cost, Td qd_cost, Td u_cost, Td N_cost,
                        Td q_lim_cost, Td vel_lim_cost, Td ctrl_lim_cost, Td* Q, Td* qv, Td* R, Td* rv)
{
    Td* s = scratch().data();
    Td sxu[64], sg[6];
    for (int i = 0; i < 3 * grid::NQ; ++i) sxu[i] = xu[i];
    for (int i = 0; i < 6; ++i) sg[i] = goal[i];
    blockIdx.x = 0;
    gato::plant::trackingCostGradientAndHessian<Td>(2 * grid::NQ, grid::NQ, sxu, sg, Q, qv, R, rv,
                                                   s, model(), q_cost, qd_cost, u_cost, N_cost,
                                                   q_lim_cost, vel_lim_cost, ctrl_lim_cost);
}

/* compute_linearized_dynamics with the integrator error: from
   xux = [x_k u_k x_{k+1}] gives A (nx x nx), B (nx x nu) column-major and
   c = x_{k+1} - f(x_k, u_k) */
void ref_linearized_dynamics(const Td* xux, const Td* fext, Td dt, Td* A, Td* B, Td* c)
{
    Td* s = scratch().data();
    Td sx[64], sf[6];
    for (int i = 0; i < 5 * grid::NQ; ++i) sx[i] = xux[i];
    if (fext) {
        for (int i = 0; i < 6; ++i) sf[i] = fext[i];
        gato::plant::compute_linearized_dynamics<Td, 2, false, true>(sx, A, B, c, s, model(), dt, sf);
    } else {
        gato::plant::compute_linearized_dynamics<Td, 2, false, true>(sx, A, B, c, s, model(), dt);
    }
}

/* compute_integrator_error: L1 norm of x_{k+1} - f(x_k, u_k) */
Td ref_integrator_error(const Td* xux, const Td* fext, Td dt)
{
    Td* s = scratch().data();
    Td sx[64], sf[6];
    for (int i = 0; i < 5 * grid::NQ; ++i) sx[i] = xux[i];
    if (fext) {
        for (int i = 0; i < 6; ++i) sf[i] = fext[i];
        return gato::plant::compute_integrator_error<Td, 2, false>(sx, sx + 3 * grid::NQ, s, model(),
                                                                 dt, sf);
    }
    return gato::plant::compute_integrator_error<Td, 2, false>(sx, sx + 3 * grid::NQ, s, model(), dt);
}

}  // extern "C"
