/*
 * FP64 host oracle of the batched SQP solve — TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker the CUDA path is compared against.  It is used by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never
 * by the product path (gato_b200/), which fails loudly without its CUDA
 * library.
 *
 * It restates the reference's algorithm serially in double precision:
 *   - rigid-body dynamics by textbook spatial algebra (RNEA, CRBA, forward-mode
 *     derivatives of the RNEA recursions), replacing the GRiD-generated
 *     functions the reference calls (gato/dynamics/iiwa14/iiwa14_grid.cuh:
 *     2211-2292 load_update_XImats_helpers, 4740- direct_minv_inner,
 *     3730- inverse_dynamics_inner, 5339-5352 forward_dynamics_finish,
 *     5547- inverse_dynamics_gradient_inner, 2596-2698 end_effector_pose,
 *     2855-2966 end_effector_pose_gradient).  Its results are pinned against
 *     the reference's own GRiD code compiled for the host (oracle/_ref, see
 *     oracle/Makefile) through tests/golden fixtures;
 *   - the plant cost functions (gato/dynamics/iiwa14/iiwa14_plant.cuh:103-450,
 *     gato/dynamics/indy7/indy7_plant.cuh:141-415);
 *   - the trapezoidal integrator (gato/dynamics/integrator.cuh:20-257);
 *   - every solver kernel and the host driver (gato/bsqp/kernels/,
 *     gato/bsqp/bsqp.cuh:103-197), each function below citing the lines it
 *     follows, including the reference's quirks.
 *
 * Problems of a batch run in lockstep exactly like the reference driver; the
 * per-problem stages are spread over std::thread workers.
 */
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <chrono>
#include <atomic>
#include <functional>
#include <thread>

#include "../gato_b200/csrc/plant_tables.h"

namespace orc {

/* ------------------------------------------------------------------ */
/* constants of gato/settings.h:15-21; they are `float` constants in the
   reference, so the rounded float values are used even in FP64            */
static const double RHO_INIT = (double)1e-3f;
static const double RHO_FACTOR = (double)1.2f;
static const double RHO_MIN = (double)1e-8f;
static const double RHO_MAX = 10.0;
static const int NUM_ALPHAS = 8;

/* ------------------------------------------------------------------ */
/* 3x3 and 6x6 helpers (row-major)                                      */
static void mat3_mul(const double* A, const double* B, double* C)
{
    double t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += A[3 * i + k] * B[3 * k + j];
            t[3 * i + j] = s;
        }
    memcpy(C, t, sizeof(t));
}
static void mat3_T(const double* A, double* B)
{
    double t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[3 * i + j] = A[3 * j + i];
    memcpy(B, t, sizeof(t));
}
static void skew(const double* v, double* S)
{
    S[0] = 0;     S[1] = -v[2]; S[2] = v[1];
    S[3] = v[2];  S[4] = 0;     S[5] = -v[0];
    S[6] = -v[1]; S[7] = v[0];  S[8] = 0;
}
static void rpy_to_R(const double* rpy, double* R)
{
    double cr = cos(rpy[0]), sr = sin(rpy[0]);
    double cp = cos(rpy[1]), sp = sin(rpy[1]);
    double cy = cos(rpy[2]), sy = sin(rpy[2]);
    double Rx[9] = {1, 0, 0, 0, cr, -sr, 0, sr, cr};
    double Ry[9] = {cp, 0, sp, 0, 1, 0, -sp, 0, cp};
    double Rz[9] = {cy, -sy, 0, sy, cy, 0, 0, 0, 1};
    double t[9];
    mat3_mul(Ry, Rx, t);
    mat3_mul(Rz, t, R);
}

typedef double M6[36];
static void m6_mv(const double* A, const double* x, double* y)
{
    double t[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0;
        for (int k = 0; k < 6; ++k) s += A[6 * i + k] * x[k];
        t[i] = s;
    }
    memcpy(y, t, sizeof(t));
}
static void m6_mtv(const double* A, const double* x, double* y)
{
    double t[6];
    for (int i = 0; i < 6; ++i) {
        double s = 0;
        for (int k = 0; k < 6; ++k) s += A[6 * k + i] * x[k];
        t[i] = s;
    }
    memcpy(y, t, sizeof(t));
}
static void m6_mul(const double* A, const double* B, double* C)
{
    double t[36];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += A[6 * i + k] * B[6 * k + j];
            t[6 * i + j] = s;
        }
    memcpy(C, t, sizeof(t));
}
/* motion cross product v x m u */
static void crm(const double* v, const double* u, double* out)
{
    const double *w = v, *vl = v + 3, *wu = u, *vu = u + 3;
    double t[6];
    t[0] = w[1] * wu[2] - w[2] * wu[1];
    t[1] = w[2] * wu[0] - w[0] * wu[2];
    t[2] = w[0] * wu[1] - w[1] * wu[0];
    t[3] = w[1] * vu[2] - w[2] * vu[1] + vl[1] * wu[2] - vl[2] * wu[1];
    t[4] = w[2] * vu[0] - w[0] * vu[2] + vl[2] * wu[0] - vl[0] * wu[2];
    t[5] = w[0] * vu[1] - w[1] * vu[0] + vl[0] * wu[1] - vl[1] * wu[0];
    memcpy(out, t, sizeof(t));
}
/* force cross product v x f f */
static void crf(const double* v, const double* f, double* out)
{
    const double *w = v, *vl = v + 3, *n = f, *fl = f + 3;
    double t[6];
    t[0] = w[1] * n[2] - w[2] * n[1] + vl[1] * fl[2] - vl[2] * fl[1];
    t[1] = w[2] * n[0] - w[0] * n[2] + vl[2] * fl[0] - vl[0] * fl[2];
    t[2] = w[0] * n[1] - w[1] * n[0] + vl[0] * fl[1] - vl[1] * fl[0];
    t[3] = w[1] * fl[2] - w[2] * fl[1];
    t[4] = w[2] * fl[0] - w[0] * fl[2];
    t[5] = w[0] * fl[1] - w[1] * fl[0];
    memcpy(out, t, sizeof(t));
}

/* ------------------------------------------------------------------ */
/* Robot model                                                          */
struct Model {
    int nq;
    double E0[GATO_MAX_NQ][9];   /* child-from-parent rotation of the joint
                                    frame at q=0 (R_urdf^T) */
    double R0[GATO_MAX_NQ][9];   /* R_urdf */
    double P[GATO_MAX_NQ][3];    /* joint origin in the parent frame */
    M6 XT[GATO_MAX_NQ];          /* fixed part of the joint transform */
    M6 I[GATO_MAX_NQ];           /* spatial inertia about the link origin */
    double qlo[GATO_MAX_NQ], qhi[GATO_MAX_NQ];
    double vlo[GATO_MAX_NQ], vhi[GATO_MAX_NQ];
    double ulo[GATO_MAX_NQ], uhi[GATO_MAX_NQ];
    double gravity;
    int barrier_style;
};

static double SNAP = 1e-6;
static void build_model(const gato_model_t* src, Model* m)
{
    memset(m, 0, sizeof(*m));
    m->nq = src->nq;
    m->gravity = src->gravity;
    m->barrier_style = src->barrier_style;
    for (int i = 0; i < src->nq; ++i) {
        /* entries below SNAP are zeroed, which reproduces the reference's
           generated transform tables (URDF angles such as -1.5707962635746238
           leave 1e-8 residues that those tables drop) */
        rpy_to_R(src->joint_rpy[i], m->R0[i]);
        mat3_T(m->R0[i], m->E0[i]);
        for (int k = 0; k < 3; ++k) m->P[i][k] = src->joint_xyz[i][k];
        {
            double px[9], Epx[9];
            skew(m->P[i], px);
            mat3_mul(m->E0[i], px, Epx);
            double* X = m->XT[i];
            memset(X, 0, sizeof(M6));
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) {
                    X[6 * r + q] = m->E0[i][3 * r + q];
                    X[6 * (r + 3) + q + 3] = m->E0[i][3 * r + q];
                    X[6 * (r + 3) + q] = -Epx[3 * r + q];
                }
            for (int k = 0; k < 36; ++k)
                if (fabs(X[k]) < SNAP) X[k] = 0.0;
            for (int k = 0; k < 9; ++k) {
                if (fabs(m->R0[i][k]) < SNAP) m->R0[i][k] = 0.0;
                if (fabs(m->E0[i][k]) < SNAP) m->E0[i][k] = 0.0;
            }
        }
        double* I = m->I[i];
        for (int b = 0; b < 2; ++b) {
            const double* bd = src->link_inertial[i][b];
            double mass = bd[0];
            if (mass == 0.0) continue;
            const double* c = bd + 1;
            double Ic[9] = {bd[4], bd[5], bd[6], bd[5], bd[7], bd[8], bd[6], bd[8], bd[9]};
            double cx[9];
            skew(c, cx);
            double cc[9];
            mat3_mul(cx, cx, cc);
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) {
                    I[6 * r + q] += Ic[3 * r + q] - mass * cc[3 * r + q];
                    I[6 * r + q + 3] += mass * cx[3 * r + q];
                    I[6 * (r + 3) + q] += -mass * cx[3 * r + q];
                }
            for (int r = 0; r < 3; ++r) I[6 * (r + 3) + r + 3] += mass;
        }
        /* JOINT_LIMITS() etc. with JOINT_LIMIT_MARGIN (iiwa14_plant.cuh:30-70) */
        m->qlo[i] = -src->q_limit[i] - src->limit_margin;
        m->qhi[i] = src->q_limit[i] + src->limit_margin;
        m->vlo[i] = -src->qd_limit[i] - src->limit_margin;
        m->vhi[i] = src->qd_limit[i] + src->limit_margin;
        m->ulo[i] = -src->u_limit[i] - src->limit_margin;
        m->uhi[i] = src->u_limit[i] + src->limit_margin;
    }
}

/* Plücker motion transform parent->link i at joint angle q:
   X = rot(Rz(q)^T) * XT with the fixed part XT = [E0 0; -E0 P x, E0]. */
static void joint_X(const Model& m, int i, double q, double* X)
{
    double c = cos(q), s = sin(q);
    double RzT[9] = {c, s, 0, -s, c, 0, 0, 0, 1};
    memset(X, 0, 36 * sizeof(double));
    for (int blk = 0; blk < 2; ++blk)
        for (int r = 0; r < 3; ++r)
            for (int col = 0; col < 6; ++col) {
                double acc = 0;
                for (int k = 0; k < 3; ++k) acc += RzT[3 * r + k] * m.XT[i][6 * (3 * blk + k) + col];
                X[6 * (3 * blk + r) + col] = acc;
            }
}

/* ------------------------------------------------------------------ */
/* Inverse dynamics (RNEA).  fext: spatial force on the last link, in its
   frame, subtracted from its net force (iiwa14_fext.cuh:160-171).       */
struct RneaState {
    M6 X[GATO_MAX_NQ];
    double v[GATO_MAX_NQ][6], a[GATO_MAX_NQ][6], f[GATO_MAX_NQ][6];
};

static void rnea(const Model& m, const double* q, const double* qd, const double* qdd,
                 const double* fext, double* tau, RneaState* st)
{
    RneaState local;
    RneaState& S = st ? *st : local;
    const int n = m.nq;
    double vp[6] = {0, 0, 0, 0, 0, 0};
    double ap[6] = {0, 0, 0, 0, 0, m.gravity};
    for (int i = 0; i < n; ++i) {
        joint_X(m, i, q[i], S.X[i]);
        double* v = S.v[i];
        double* a = S.a[i];
        m6_mv(S.X[i], vp, v);
        v[2] += qd[i];
        m6_mv(S.X[i], ap, a);
        a[2] += qdd ? qdd[i] : 0.0;
        double sqd[6] = {0, 0, qd[i], 0, 0, 0};
        double t[6];
        crm(v, sqd, t);
        for (int k = 0; k < 6; ++k) a[k] += t[k];
        double Iv[6], Ia[6];
        m6_mv(m.I[i], v, Iv);
        m6_mv(m.I[i], a, Ia);
        crf(v, Iv, t);
        for (int k = 0; k < 6; ++k) S.f[i][k] = Ia[k] + t[k];
        if (i == n - 1 && fext)
            for (int k = 0; k < 6; ++k) S.f[i][k] -= fext[k];
        memcpy(vp, v, sizeof(vp));
        memcpy(ap, a, sizeof(ap));
    }
    for (int i = n - 1; i >= 0; --i) {
        if (tau) tau[i] = S.f[i][2];
        if (i > 0) {
            double t[6];
            m6_mtv(S.X[i], S.f[i], t);
            for (int k = 0; k < 6; ++k) S.f[i - 1][k] += t[k];
        }
    }
}

/* Joint-space inertia matrix by the composite-rigid-body algorithm;
   M is nq x nq row-major (symmetric). */
static void crba(const Model& m, const double* q, double* M)
{
    const int n = m.nq;
    M6 X[GATO_MAX_NQ], Ic[GATO_MAX_NQ];
    for (int i = 0; i < n; ++i) {
        joint_X(m, i, q[i], X[i]);
        memcpy(Ic[i], m.I[i], sizeof(M6));
    }
    for (int i = n - 1; i > 0; --i) {
        M6 t, XT;
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) XT[6 * r + c] = X[i][6 * c + r];
        m6_mul(Ic[i], X[i], t);
        m6_mul(XT, t, t);
        for (int k = 0; k < 36; ++k) Ic[i - 1][k] += t[k];
    }
    for (int i = 0; i < n; ++i) {
        double F[6];
        for (int k = 0; k < 6; ++k) F[k] = Ic[i][6 * k + 2];
        M[n * i + i] = F[2];
        for (int j = i; j > 0; --j) {
            m6_mtv(X[j], F, F);
            M[n * (j - 1) + i] = F[2];
            M[n * i + (j - 1)] = F[2];
        }
    }
}

/* SPD inverse by Cholesky (n <= 8); row-major in/out. */
static void spd_inverse(int n, const double* A, double* Ainv)
{
    double L[64] = {0};
    for (int j = 0; j < n; ++j) {
        double s = A[n * j + j];
        for (int k = 0; k < j; ++k) s -= L[8 * j + k] * L[8 * j + k];
        L[8 * j + j] = sqrt(s);
        for (int i = j + 1; i < n; ++i) {
            double t = A[n * i + j];
            for (int k = 0; k < j; ++k) t -= L[8 * i + k] * L[8 * j + k];
            L[8 * i + j] = t / L[8 * j + j];
        }
    }
    for (int c = 0; c < n; ++c) {
        double y[8], x[8];
        for (int i = 0; i < n; ++i) {
            double t = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) t -= L[8 * i + k] * y[k];
            y[i] = t / L[8 * i + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double t = y[i];
            for (int k = i + 1; k < n; ++k) t -= L[8 * k + i] * x[k];
            x[i] = t / L[8 * i + i];
        }
        for (int i = 0; i < n; ++i) Ainv[n * i + c] = x[i];
    }
}

/* Forward dynamics qdd = M^-1 (u - c(q, qd, fext)); Minv optional out. */
static void fd(const Model& m, const double* q, const double* qd, const double* u,
               const double* fext, double* qdd, double* Minv_out)
{
    const int n = m.nq;
    double c[GATO_MAX_NQ], M[64], Minv[64];
    rnea(m, q, qd, nullptr, fext, c, nullptr);
    crba(m, q, M);
    spd_inverse(n, M, Minv);
    for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int k = 0; k < n; ++k) s += Minv[n * i + k] * (u[k] - c[k]);
        qdd[i] = s;
    }
    if (Minv_out) memcpy(Minv_out, Minv, sizeof(double) * n * n);
}

/* Forward-mode derivatives of the RNEA recursions.  dtau_dq, dtau_dqd are
   nq x nq row-major ([row i = joint torque i][col j = derivative j]).
   fext enters only through the accumulated link forces. */
static void rnea_derivatives(const Model& m, const double* q, const double* qd,
                             const double* qdd, const double* fext, double* dtau_dq,
                             double* dtau_dqd)
{
    const int n = m.nq;
    RneaState S;
    rnea(m, q, qd, qdd, fext, nullptr, &S); /* S.f holds accumulated forces */
    const double Sv[6] = {0, 0, 1, 0, 0, 0};
    for (int wrt = 0; wrt < 2; ++wrt) {
        for (int j = 0; j < n; ++j) {
            double dv[GATO_MAX_NQ][6], da[GATO_MAX_NQ][6], df[GATO_MAX_NQ][6];
            double dvp[6] = {0}, dap[6] = {0};
            double vp[6] = {0}, ap[6] = {0, 0, 0, 0, 0, m.gravity};
            for (int i = 0; i < n; ++i) {
                double t[6], u[6];
                m6_mv(S.X[i], dvp, dv[i]);
                m6_mv(S.X[i], dap, da[i]);
                if (wrt == 0 && i == j) {
                    m6_mv(S.X[i], vp, u);
                    crm(u, Sv, t);
                    for (int k = 0; k < 6; ++k) dv[i][k] += t[k];
                    m6_mv(S.X[i], ap, u);
                    crm(u, Sv, t);
                    for (int k = 0; k < 6; ++k) da[i][k] += t[k];
                }
                if (wrt == 1 && i == j) dv[i][2] += 1.0;
                double sqd[6] = {0, 0, qd[i], 0, 0, 0};
                crm(dv[i], sqd, t);
                for (int k = 0; k < 6; ++k) da[i][k] += t[k];
                if (wrt == 1 && i == j) {
                    crm(S.v[i], Sv, t);
                    for (int k = 0; k < 6; ++k) da[i][k] += t[k];
                }
                double Iv[6], Idv[6], Ida[6], t2[6];
                m6_mv(m.I[i], S.v[i], Iv);
                m6_mv(m.I[i], dv[i], Idv);
                m6_mv(m.I[i], da[i], Ida);
                crf(dv[i], Iv, t);
                crf(S.v[i], Idv, t2);
                for (int k = 0; k < 6; ++k) df[i][k] = Ida[k] + t[k] + t2[k];
                memcpy(dvp, dv[i], sizeof(dvp));
                memcpy(dap, da[i], sizeof(dap));
                memcpy(vp, S.v[i], sizeof(vp));
                memcpy(ap, S.a[i], sizeof(ap));
            }
            for (int i = n - 1; i >= 0; --i) {
                double* out = wrt == 0 ? dtau_dq : dtau_dqd;
                out[n * i + j] = df[i][2];
                if (i > 0) {
                    double t[6];
                    m6_mtv(S.X[i], df[i], t);
                    for (int k = 0; k < 6; ++k) df[i - 1][k] += t[k];
                    if (wrt == 0 && i == j) {
                        double sf[6];
                        crf(Sv, S.f[i], sf);
                        m6_mtv(S.X[i], sf, t);
                        for (int k = 0; k < 6; ++k) df[i - 1][k] += t[k];
                    }
                }
            }
        }
    }
}

/* qdd and its derivatives in the reference's df_du layout
   (iiwa14_plant.cuh:207-224): nq x 3nq column-major = [dqdd/dq | dqdd/dqd | Minv] */
static void fd_grad(const Model& m, const double* q, const double* qd, const double* u,
                    const double* fext, double* qdd, double* df_du)
{
    const int n = m.nq;
    double Minv[64], dq[64], dqd[64];
    fd(m, q, qd, u, fext, qdd, Minv);
    rnea_derivatives(m, q, qd, qdd, fext, dq, dqd);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double s1 = 0, s2 = 0;
            for (int k = 0; k < n; ++k) {
                s1 += Minv[n * r + k] * dq[n * k + c];
                s2 += Minv[n * r + k] * dqd[n * k + c];
            }
            df_du[c * n + r] = -s1;
            df_du[n * n + c * n + r] = -s2;
            df_du[2 * n * n + c * n + r] = Minv[n * r + c];
        }
}

/* End-effector position: origin of the last link frame in the base frame
   (iiwa14_grid.cuh:2596-2672 takes the translation of the chained
   homogeneous transforms).  J: 3 x nq, column j at J[3*j]. */
static void ee_pos(const Model& m, const double* q, double* p, double* J)
{
    const int n = m.nq;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, o[3] = {0, 0, 0};
    double z[GATO_MAX_NQ][3], org[GATO_MAX_NQ][3];
    for (int i = 0; i < n; ++i) {
        double t[3];
        for (int r = 0; r < 3; ++r)
            t[r] = R[3 * r] * m.P[i][0] + R[3 * r + 1] * m.P[i][1] + R[3 * r + 2] * m.P[i][2];
        for (int r = 0; r < 3; ++r) o[r] += t[r];
        double c = cos(q[i]), s = sin(q[i]);
        double Rz[9] = {c, -s, 0, s, c, 0, 0, 0, 1}, Rj[9];
        mat3_mul(m.R0[i], Rz, Rj);
        mat3_mul(R, Rj, R);
        for (int r = 0; r < 3; ++r) {
            z[i][r] = R[3 * r + 2];
            org[i][r] = o[r];
        }
    }
    for (int r = 0; r < 3; ++r) p[r] = o[r];
    if (J) {
        for (int j = 0; j < n; ++j) {
            double d[3] = {o[0] - org[j][0], o[1] - org[j][1], o[2] - org[j][2]};
            J[3 * j + 0] = z[j][1] * d[2] - z[j][2] * d[1];
            J[3 * j + 1] = z[j][2] * d[0] - z[j][0] * d[2];
            J[3 * j + 2] = z[j][0] * d[1] - z[j][1] * d[0];
        }
    }
}

/* ------------------------------------------------------------------ */
/* Barrier functions (iiwa14_plant.cuh:103-155; indy7_plant.cuh:141-147) */
static double barrier(double q, double lo, double hi)
{
    double dmin = q - lo, dmax = hi - q;
    dmin = (dmin <= 1e-10) ? 1e-10 : dmin;
    dmax = (dmax <= 1e-10) ? 1e-10 : dmax;
    return -log(dmin) - log(dmax);
}
static double barrier_grad(int style, double q, double lo, double hi)
{
    double dmin = q - lo, dmax = hi - q;
    if (style == 0) {
        const double eps = 1e-6;
        if (dmin >= 0) { if (dmin < eps) dmin = eps; } else { if (dmin > -eps) dmin = -eps; }
        if (dmax >= 0) { if (dmax < eps) dmax = eps; } else { if (dmax > -eps) dmax = -eps; }
        return -1.0 / dmin + 1.0 / dmax;
    }
    dmin = (dmin <= 1e-6) ? 1e-6 : dmin;
    dmax = (dmax <= 1e-6) ? 1e-6 : dmax;
    return -1.0 / dmin + 1.0 / dmax;
}
static double barrier_hess(double q, double lo, double hi)
{
    const double eps = 1e-6;
    double amin = fabs(q - lo), amax = fabs(hi - q);
    if (amin < eps) amin = eps;
    if (amax < eps) amax = eps;
    return 1.0 / (amin * amin) + 1.0 / (amax * amax);
}

struct Params {
    double dt;
    int max_sqp_iters;
    double kkt_tol;
    int max_pcg_iters;
    double pcg_tol, solve_ratio, mu, q_cost, qd_cost, u_cost, N_cost, q_lim_cost,
        vel_lim_cost, ctrl_lim_cost, rho;
    /* one problem's diagonal weights [Qd (nx), Rd (nu)] or null: the stage
       cost gains 1/2 Qd_i x_i^2 and 1/2 Rd_i u_i^2 in place of the uniform
       qd_cost / u_cost terms (an extension; Qd = [0, qd_cost], Rd = u_cost is
       the reference's cost) */
    const double* wd = nullptr;
};
static Params to_params(const gato_params_t* p)
{
    Params r;
    r.dt = p->dt;
    r.max_sqp_iters = p->max_sqp_iters;
    r.kkt_tol = p->kkt_tol;
    r.max_pcg_iters = p->max_pcg_iters;
    r.pcg_tol = p->pcg_tol;
    r.solve_ratio = p->solve_ratio;
    r.mu = p->mu;
    r.q_cost = p->q_cost;
    r.qd_cost = p->qd_cost;
    r.u_cost = p->u_cost;
    r.N_cost = p->N_cost;
    r.q_lim_cost = p->q_lim_cost;
    r.vel_lim_cost = p->vel_lim_cost;
    r.ctrl_lim_cost = p->ctrl_lim_cost;
    r.rho = p->rho;
    return r;
}

/* trackingcost (iiwa14_plant.cuh:275-327).  xu holds x (and u when
   has_u); `terminal` selects N_cost (blockIdx.x == KNOT_POINTS-1 in the
   merit kernel). */
static double tracking_cost(const Model& m, const Params& P, const double* xu, bool has_u,
                            const double* goal, bool terminal)
{
    const int nq = m.nq;
    double s = 0;
    for (int i = 0; i < nq; ++i) {
        double qd = xu[i + nq];
        s += 0.5 * (P.wd ? P.wd[nq + i] : P.qd_cost) * qd * qd;
        if (P.wd) s += 0.5 * P.wd[i] * xu[i] * xu[i];
        s += P.q_lim_cost * barrier(xu[i], m.qlo[i], m.qhi[i]);
        s += P.vel_lim_cost * barrier(qd, m.vlo[i], m.vhi[i]);
    }
    if (has_u)
        for (int i = 0; i < nq; ++i) {
            double u = xu[2 * nq + i];
            s += 0.5 * (P.wd ? P.wd[2 * nq + i] : P.u_cost) * u * u;
            s += P.ctrl_lim_cost * barrier(u, m.ulo[i], m.uhi[i]);
        }
    double p[3];
    ee_pos(m, xu, p, nullptr);
    double w = terminal ? P.N_cost : P.q_cost;
    for (int i = 0; i < 3; ++i) {
        double e = p[i] - goal[i];
        s += 0.5 * w * e * e;
    }
    return s;
}

/* trackingCostGradientAndHessian (iiwa14_plant.cuh:338-424,
   indy7_plant.cuh:325-420).  The weight is always q_cost in the KKT setup
   (the blockIdx.x == KNOT_POINTS-1 test never fires there). */
static void tracking_grad_hess(const Model& m, const Params& P, const double* xu,
                               const double* goal, bool computeR, double* Q, double* qv,
                               double* R, double* rv)
{
    const int nq = m.nq, nx = 2 * nq, nu = nq;
    double p[3], J[3 * GATO_MAX_NQ];
    ee_pos(m, xu, p, J);
    double e[3] = {p[0] - goal[0], p[1] - goal[1], p[2] - goal[2]};
    const double w = P.q_cost;
    double ge[GATO_MAX_NQ], bg[GATO_MAX_NQ];
    for (int i = 0; i < nq; ++i) {
        ge[i] = J[3 * i] * e[0] + J[3 * i + 1] * e[1] + J[3 * i + 2] * e[2];
        bg[i] = barrier_grad(m.barrier_style, xu[i], m.qlo[i], m.qhi[i]);
    }
    for (int i = 0; i < nx; ++i) {
        if (i < nq) {
            qv[i] = ge[i] * w + P.q_lim_cost * bg[i];
            if (P.wd) qv[i] += P.wd[i] * xu[i];
        } else {
            qv[i] = (P.wd ? P.wd[i] : P.qd_cost) * xu[i] +
                    P.vel_lim_cost * barrier_grad(m.barrier_style, xu[i], m.vlo[i - nq], m.vhi[i - nq]);
        }
    }
    if (computeR)
        for (int i = 0; i < nu; ++i)
            rv[i] = (P.wd ? P.wd[nx + i] : P.u_cost) * xu[nx + i] +
                    P.ctrl_lim_cost * barrier_grad(m.barrier_style, xu[nx + i], m.ulo[i], m.uhi[i]);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) {
            double val;
            if (i < nq && j < nq) {
                val = ge[i] * ge[j] * w;
                if (m.barrier_style == 0) {
                    if (i == j) val += P.q_lim_cost * barrier_hess(xu[i], m.qlo[i], m.qhi[i]);
                } else {
                    val += P.q_lim_cost * bg[i] * bg[j];
                }
                if (P.wd && i == j) val += P.wd[i];
            } else {
                val = (i == j) ? (P.wd ? P.wd[i] : P.qd_cost) : 0.0;
                if (i == j) {
                    if (m.barrier_style == 0)
                        val += P.vel_lim_cost * barrier_hess(xu[i], m.vlo[i - nq], m.vhi[i - nq]);
                    else {
                        double g = barrier_grad(1, xu[i], m.vlo[i - nq], m.vhi[i - nq]);
                        val += P.vel_lim_cost * g * g;
                    }
                }
            }
            Q[i * nx + j] = val;
        }
    if (computeR)
        for (int i = 0; i < nu; ++i)
            for (int j = 0; j < nu; ++j) {
                double val = (i == j) ? (P.wd ? P.wd[nx + i] : P.u_cost) : 0.0;
                if (i == j) {
                    double uu = xu[nx + i];
                    if (m.barrier_style == 0)
                        val += P.ctrl_lim_cost * barrier_hess(uu, m.ulo[i], m.uhi[i]);
                    else {
                        double g = barrier_grad(1, uu, m.ulo[i], m.uhi[i]);
                        val += P.ctrl_lim_cost * g * g;
                    }
                }
                R[i * nu + j] = val;
            }
}

/* trapezoidal step (integrator.cuh:34-37) */
static void integrate(int nq, const double* x, const double* qdd, double dt, double* xn)
{
    for (int i = 0; i < nq; ++i) {
        xn[nq + i] = x[nq + i] + dt * qdd[i];
        xn[i] = x[i] + dt * x[nq + i] + 0.5 * qdd[i] * dt * dt;
    }
}

/* ------------------------------------------------------------------ */
/* Batch layouts (gato/constants.h:10-26)                               */
struct Dims {
    int nq, nx, nu, N;
    int traj() const { return (nx + nu) * N - nu; }
    int vecp() const { return (N + 2) * nx; }
    int b3d() const { return 3 * nx * nx * N; }
};

/* setupKKTSystemBatchedKernel for one problem (setup_kkt.cuh:52-107).
   Q,A: N*nx*nx; R: N*nu*nu; q,c: N*nx; r: N*nu; B: N*nx*nu. */
static void setup_kkt(const Model& m, const Params& P, const Dims& d, double dt,
                      const double* xu, const double* xs, const double* goal,
                      const double* fext, double* Q, double* R, double* q, double* r,
                      double* A, double* B, double* c)
{
    const int nq = d.nq, nx = d.nx, nu = d.nu, N = d.N;
    for (int k = 0; k < N - 1; ++k) {
        const double* xuk = xu + k * (nx + nu);
        const double* xk1 = xuk + nx + nu;
        double qdd[GATO_MAX_NQ], df[3 * GATO_MAX_NQ * GATO_MAX_NQ];
        fd_grad(m, xuk, xuk + nq, xuk + nx, fext, qdd, df);
        /* integrator_error_inner (integrator.cuh:48-62): c_{k+1} = x_{k+1} - f(x_k,u_k) */
        double xn[2 * GATO_MAX_NQ];
        integrate(nq, xuk, qdd, dt, xn);
        double* ck = c + (k + 1) * nx;
        for (int i = 0; i < nx; ++i) ck[i] = xk1[i] - xn[i];
        /* integrator_gradient_inner, type 2 (integrator.cuh:143-184) */
        const double h = 0.5 * dt * dt;
        double* Ak = A + k * nx * nx;
        for (int i = 0; i < nx * nx; ++i) {
            int col = i / nx, row = i % nx, rq = row % nq;
            double g = df[col * nq + rq];
            double val = (row == col) ? 1.0 : 0.0;
            if (row < nq) {
                if (col >= nq && row == col - nq) val += dt;
                val += h * g;
            } else {
                val += dt * g;
            }
            Ak[i] = val;
        }
        double* Bk = B + k * nx * nu;
        for (int i = 0; i < nx * nu; ++i) {
            int col = i / nx, row = i % nx, rq = row % nq;
            double g = df[nx * nq + col * nq + rq];
            Bk[i] = (row < nq) ? h * g : dt * g;
        }
        const double* gk = goal + 6 * k;
        tracking_grad_hess(m, P, xuk, gk, true, Q + k * nx * nx, q + k * nx, R + k * nu * nu,
                           r + k * nu);
        if (k == N - 2) {
            /* trackingCostGradientAndHessian_lastblock (iiwa14_plant.cuh:426-450):
               the terminal blocks are evaluated at x_{N-2} against goal_{N-1}. */
            tracking_grad_hess(m, P, xuk, gk + 6, false, Q + (k + 1) * nx * nx, q + (k + 1) * nx,
                               nullptr, nullptr);
            for (int i = 0; i < nx; ++i) c[i] = xu[i] - xs[i];
        }
    }
}

/* pivot-free Gauss-Jordan inverse (gato/utils/linalg.cuh:364-400);
   A column-major dim x dim, out column-major. */
static void gj_inverse(int dim, const double* A, double* out)
{
    std::vector<double> W(2 * dim * dim);
    for (int i = 0; i < dim * dim; ++i) W[i] = A[i];
    for (int i = 0; i < dim * dim; ++i) W[dim * dim + i] = 0;
    for (int i = 0; i < dim; ++i) W[dim * dim + i * dim + i] = 1.0;
    /* augmented [A | I] stored column-major with 2*dim columns */
    for (int piv = 0; piv < dim; ++piv) {
        std::vector<double> col(dim), row(2 * dim + 1);
        for (int r = 0; r < dim; ++r) col[r] = W[piv * dim + r];
        double pv = col[piv];
        for (int cidx = piv; cidx < 2 * dim; ++cidx) {
            for (int r = 0; r < dim; ++r) {
                double& e = W[cidx * dim + r];
                if (r == piv) continue;
                e -= col[r] / pv * W[cidx * dim + piv];
            }
        }
        for (int cidx = piv; cidx < 2 * dim; ++cidx) W[cidx * dim + piv] /= pv;
    }
    for (int i = 0; i < dim * dim; ++i) out[i] = W[dim * dim + i];
}

/* column-major helpers */
static inline double& cm(double* M, int ld, int r, int c) { return M[c * ld + r]; }

/* formSchurSystemBatchedKernel1 + 2 for one problem
   (schur_linsys.cuh:54-260).  Reads raw Q (the intended semantics of the
   read of d_Q_batch[k+1] / d_Q_batch[0], which the reference's kernel 1 can
   race with its own in-place inverse writes).  Overwrites Q and R with
   (Q+rho I_q)^-1 and R^-1 (schur_linsys.cuh:100-104).  S, Pinv: N blocks rows
   of nx x 3nx row-major; gamma padded (N+2)*nx. */
static void form_schur(const Dims& d, double rho, double* Q, double* R, const double* q,
                       const double* r, const double* A, const double* B, const double* c,
                       double* S, double* Pinv, double* gamma)
{
    const int nx = d.nx, nu = d.nu, N = d.N, n2 = nx * nx, BR = 3 * nx * nx, RD = 3 * nx;
    std::vector<double> Qraw(Q, Q + N * n2);
    std::vector<double> Qinv(N * n2), Rinv(N * nu * nu), T(N * n2);
    for (int k = 0; k < N; ++k) {
        std::vector<double> Qt(Qraw.begin() + k * n2, Qraw.begin() + (k + 1) * n2);
        for (int i = 0; i < nx / 2; ++i) Qt[i * nx + i] += rho; /* addScaledIdentity, q half */
        gj_inverse(nx, Qt.data(), &Qinv[k * n2]);
        if (k < N - 1) gj_inverse(nu, R + k * nu * nu, &Rinv[k * nu * nu]);
    }
    std::fill(S, S + d.b3d(), 0.0);
    std::fill(Pinv, Pinv + d.b3d(), 0.0);
    std::fill(gamma, gamma + d.vecp(), 0.0);
    for (int k = 0; k < N - 1; ++k) {
        const double* Ak = A + k * n2;
        const double* Bk = B + k * nx * nu;
        const double* Qi = &Qinv[k * n2];
        const double* Qi1 = &Qinv[(k + 1) * n2];
        const double* Ri = &Rinv[k * nu * nu];
        std::vector<double> AQ(n2), BR_(nx * nu), th(n2);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) {
                double s = 0;
                for (int t = 0; t < nx; ++t) s += Ak[t * nx + i] * Qi[j * nx + t];
                AQ[j * nx + i] = s;
            }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nu; ++j) {
                double s = 0;
                for (int t = 0; t < nu; ++t) s += Bk[t * nx + i] * Ri[j * nu + t];
                BR_[j * nx + i] = s;
            }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) {
                double s = Qi1[j * nx + i];
                for (int t = 0; t < nx; ++t) s += AQ[t * nx + i] * Ak[t * nx + j];
                for (int t = 0; t < nu; ++t) s += BR_[t * nx + i] * Bk[t * nx + j];
                th[j * nx + i] = s;
            }
        /* gamma_{k+1} = c_{k+1} - Qinv_{k+1} q_{k+1} + AQinv q_k + BRinv r_k */
        double* g = gamma + (k + 2) * nx;
        const double* ck = c + (k + 1) * nx;
        for (int i = 0; i < nx; ++i) {
            double s = ck[i];
            for (int t = 0; t < nx; ++t) s -= Qi1[t * nx + i] * q[(k + 1) * nx + t];
            for (int t = 0; t < nx; ++t) s += AQ[t * nx + i] * q[k * nx + t];
            for (int t = 0; t < nu; ++t) s += BR_[t * nx + i] * r[k * nu + t];
            g[i] = s;
        }
        /* S blocks (schur_linsys.cuh:136-147) */
        double* Sright = S + k * BR + 2 * nx;
        double* Sleft = S + (k + 1) * BR;
        double* Smain = Sleft + nx;
        for (int y = 0; y < nx; ++y)
            for (int x = 0; x < nx; ++x) {
                Sright[y * RD + x] = AQ[y * nx + x];
                Sleft[y * RD + x] = AQ[x * nx + y];
                Smain[y * RD + x] = -th[x * nx + y];
            }
        /* P^-1 main = -(theta + rho I_q)^-1 (schur_linsys.cuh:150-164) */
        std::vector<double> thr(th);
        for (int i = 0; i < nx / 2; ++i) thr[i * nx + i] += rho;
        gj_inverse(nx, thr.data(), &T[(k + 1) * n2]);
        double* Pm = Pinv + (k + 1) * BR + nx;
        for (int y = 0; y < nx; ++y)
            for (int x = 0; x < nx; ++x) Pm[y * RD + x] = -T[(k + 1) * n2 + x * nx + y];
    }
    { /* last block: Q_0 terms (schur_linsys.cuh:166-210) */
        std::vector<double> Qt(Qraw.begin(), Qraw.begin() + n2);
        for (int i = 0; i < nx / 2; ++i) Qt[i * nx + i] += rho;
        double* Pm = Pinv + nx;
        double* Sm = S + nx;
        for (int y = 0; y < nx; ++y)
            for (int x = 0; x < nx; ++x) {
                Pm[y * RD + x] = -Qt[x * nx + y];
                Sm[y * RD + x] = -Qinv[x * nx + y];
            }
        double* g = gamma + nx;
        for (int i = 0; i < nx; ++i) {
            double s = c[i];
            for (int t = 0; t < nx; ++t) s -= Qinv[t * nx + i] * q[t];
            g[i] = s;
        }
    }
    /* kernel 2 (schur_linsys.cuh:213-260) */
    for (int k = 0; k < N - 1; ++k) {
        std::vector<double> Ta(n2), Tb(n2), ph(n2), sc(n2), X(n2);
        const double* Pa = Pinv + (k + 1) * BR + nx;
        const double* Pb = Pinv + k * BR + nx;
        const double* Sl = S + (k + 1) * BR;
        for (int y = 0; y < nx; ++y)
            for (int x = 0; x < nx; ++x) {
                Ta[x * nx + y] = Pa[y * RD + x];
                Tb[x * nx + y] = Pb[y * RD + x];
                ph[x * nx + y] = Sl[y * RD + x];
            }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) {
                double s = 0;
                for (int t = 0; t < nx; ++t) s += ph[t * nx + i] * Tb[j * nx + t];
                sc[j * nx + i] = s;
            }
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx; ++j) {
                double s = 0;
                for (int t = 0; t < nx; ++t) s += Ta[t * nx + i] * sc[j * nx + t];
                X[j * nx + i] = s;
            }
        double* Pright = Pinv + k * BR + 2 * nx;
        double* Pleft = Pinv + (k + 1) * BR;
        for (int y = 0; y < nx; ++y)
            for (int x = 0; x < nx; ++x) {
                Pright[y * RD + x] = -X[y * nx + x];
                Pleft[y * RD + x] = -X[x * nx + y];
            }
    }
    memcpy(Q, Qinv.data(), sizeof(double) * N * n2);
    memcpy(R, Rinv.data(), sizeof(double) * (N - 1) * nu * nu);
}

/* btdMatrixVectorProduct over padded vectors (linalg.cuh:174-221) */
static void btd_mv(const Dims& d, const double* M, const double* x, double* y)
{
    const int nx = d.nx, RD = 3 * nx;
    for (int br = 0; br < d.N; ++br) {
        const double* blk = M + br * 3 * nx * nx;
        const double* v = x + br * nx;
        for (int r = 0; r < nx; ++r) {
            double s = 0;
            for (int cc = 0; cc < RD; ++cc) s += blk[r * RD + cc] * v[cc];
            y[(br + 1) * nx + r] = s;
        }
    }
}
static double dotv(int n, const double* a, const double* b)
{
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* solvePCGBatchedKernel for one problem (pcg.cuh:23-147); returns the
   iteration count; x (padded lambda) is updated unless the initial residual
   already meets the absolute tolerance. */
static int pcg(const Dims& d, const double* S, const double* Pinv, const double* gamma,
               double* x, double eps, int max_iters)
{
    const int L = d.vecp();
    const double abs_tol = 1e-6;
    std::vector<double> r(L, 0.0), z(L, 0.0), p(L, 0.0), Ap(L, 0.0), xs(x, x + L);
    btd_mv(d, S, xs.data(), r.data());
    for (int i = 0; i < L; ++i) r[i] = gamma[i] - r[i];
    btd_mv(d, Pinv, r.data(), z.data());
    p = z;
    double rho = dotv(L, r.data(), z.data());
    if (fabs(rho) < abs_tol) return 0;
    double rho_init = fabs(rho);
    int it = 0;
    for (int i = 0; i < max_iters; ++i) {
        ++it;
        btd_mv(d, S, p.data(), Ap.data());
        double alpha = rho / dotv(L, p.data(), Ap.data());
        for (int j = 0; j < L; ++j) {
            xs[j] += alpha * p[j];
            r[j] -= alpha * Ap[j];
        }
        btd_mv(d, Pinv, r.data(), z.data());
        double rho_new = dotv(L, r.data(), z.data());
        if (fabs(rho_new) < abs_tol + eps * rho_init) break;
        double beta = rho_new / rho;
        rho = rho_new;
        for (int j = 0; j < L; ++j) p[j] = z[j] + beta * p[j];
    }
    memcpy(x, xs.data(), sizeof(double) * L);
    return it;
}

/* computeDzBatchedKernel for one problem (schur_linsys.cuh:312-431).
   q and r are overwritten with the KKT residuals. */
static void compute_dz(const Dims& d, const double* lambda, const double* Qinv,
                       const double* Rinv, double* q, double* r, const double* A,
                       const double* B, double* dz)
{
    const int nx = d.nx, nu = d.nu, N = d.N;
    for (int k = 0; k < N; ++k) {
        const double* lk = lambda + (k + 1) * nx;
        const double* lk1 = lambda + (k + 2) * nx;
        double res[2 * GATO_MAX_NQ];
        for (int i = 0; i < nx; ++i) {
            double s = 0;
            if (k < N - 1)
                for (int t = 0; t < nx; ++t) s += lk1[t] * A[k * nx * nx + i * nx + t];
            res[i] = q[k * nx + i] - lk[i] + s;
        }
        double* dzk = dz + k * (nx + nu);
        for (int i = 0; i < nx; ++i) {
            double s = 0;
            for (int t = 0; t < nx; ++t) s += Qinv[k * nx * nx + t * nx + i] * res[t];
            dzk[i] = -s;
        }
        for (int i = 0; i < nx; ++i) q[k * nx + i] = res[i];
        if (k < N - 1) {
            double ru[GATO_MAX_NQ];
            for (int i = 0; i < nu; ++i) {
                double s = 0;
                for (int t = 0; t < nx; ++t) s += lk1[t] * B[k * nx * nu + i * nx + t];
                ru[i] = r[k * nu + i] + s;
            }
            for (int i = 0; i < nu; ++i) {
                double s = 0;
                for (int t = 0; t < nu; ++t) s += Rinv[k * nu * nu + t * nu + i] * ru[t];
                dzk[nx + i] = -s;
            }
            for (int i = 0; i < nu; ++i) r[k * nu + i] = ru[i];
        } else {
            for (int i = 0; i < nu; ++i) r[k * nu + i] = 0.0;
        }
    }
}

/* computeMeritBatchedKernel for one problem and one step alpha
   (merit.cuh:34-91). */
static double merit(const Model& m, const Params& P, const Dims& d, double dt, double mu,
                    const double* xu, const double* dz, double alpha, const double* xs,
                    const double* goal, const double* fext)
{
    const int nq = d.nq, nx = d.nx, nu = d.nu, N = d.N;
    double total = 0;
    for (int k = 0; k < N; ++k) {
        double s[3 * GATO_MAX_NQ * 2];
        int len = (k == N - 1) ? nx : 2 * nx + nu;
        for (int i = 0; i < len; ++i) s[i] = xu[k * (nx + nu) + i] + alpha * dz[k * (nx + nu) + i];
        double cost = tracking_cost(m, P, s, k < N - 1, goal + 6 * k, k == N - 1);
        double cons = 0;
        if (k < N - 1) {
            /* compute_integrator_error (integrator.cuh:211-233) */
            double qdd[GATO_MAX_NQ], xn[2 * GATO_MAX_NQ];
            fd(m, s, s + nq, s + nx, fext, qdd, nullptr);
            integrate(nq, s, qdd, dt, xn);
            for (int i = 0; i < nx; ++i) cons += fabs(s[nx + nu + i] - xn[i]);
        } else {
            for (int i = 0; i < nx; ++i) cons += fabs(xu[i] + alpha * dz[i] - xs[i]);
        }
        total += cost + mu * cons;
    }
    return total;
}

/* ------------------------------------------------------------------ */
/* dynamic parallel-for over [0, n) on `threads` workers */
static void parallel_for(int threads, int n, const std::function<void(int)>& fn)
{
    if (threads <= 1 || n <= 1) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
    };
    std::vector<std::thread> pool;
    int t = std::min(threads, n);
    for (int k = 1; k < t; ++k) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

/* ------------------------------------------------------------------ */
/* Solver with the reference driver's batch semantics (bsqp.cuh:103-197) */
struct Solver {
    Model model;
    Params P;
    Dims d;
    int Bn;
    bool adapt_rho = true;
    std::vector<double> lambda, rho, drho, mu, tol, fext;
    std::vector<double> wdiag;  // [Bn][nx+nu] when set
    std::vector<double> rho_init, drho_init;
    int threads = 1;
    /* ORC_ROUND_* flags: stage outputs rounded to FP32 where they are stored
       (orc_solver_set_round_f32) */
    int round_f32 = 0;
};

/* Rounding of stored stage outputs to FP32, with every operation in FP64:
   the arithmetic of an ideal FP32 solver (each stored value the nearest
   float to the exact one).  Measures the accuracy floor of any solver that
   keeps these arrays in FP32; it is not a model of the reference's
   rounding. */
enum {
    ORC_ROUND_KKT = 1,    /* Q, R, q, r, A, B, c after the KKT set-up */
    ORC_ROUND_SCHUR = 2,  /* S, P^-1, gamma, (Q+rho I)^-1, R^-1 */
    ORC_ROUND_LAMBDA = 4, /* lambda after the PCG */
    ORC_ROUND_XU = 8,     /* XU after the line-search update */
    ORC_ROUND_S = 16,     /* S alone */
    ORC_ROUND_PINV = 32,  /* P^-1 alone */
    ORC_ROUND_GAMMA = 64  /* gamma alone */
};
static void round_f32(double* p, size_t n)
{
    for (size_t i = 0; i < n; ++i) p[i] = (double)(float)p[i];
}

/* per-problem status bits, the GATO_STATUS_* values of include/gato_b200.h */
enum { ST_CONVERGED = 1, ST_MAX_ITER = 2, ST_LS_FAIL = 4, ST_NONFINITE = 8, ST_PCG_MAX = 16 };

struct SolveOut {
    int ls_num_iters;
    std::vector<int> sqp_iters, kkt_converged, pcg_iters, status;
    std::vector<double> final_merit, initial_merit, ls_min_merit, ls_step_size;
};

static void solve(Solver& S, double dt, double* xu, const double* xs, const double* goal,
                  SolveOut& out)
{
    const Model& m = S.model;
    const Dims& d = S.d;
    /* the parameters of problem b (its diagonal weights when set) */
    std::vector<Params> Pb(S.Bn, S.P);
    if (!S.wdiag.empty())
        for (int b = 0; b < S.Bn; ++b) Pb[b].wd = &S.wdiag[(size_t)b * (d.nx + d.nu)];
    const Params& P = S.P;
    const int Bn = S.Bn, nx = d.nx, nu = d.nu, N = d.N, T = d.traj(), L = d.vecp();
    std::vector<double> Q(Bn * N * nx * nx), R(Bn * N * nu * nu), q(Bn * N * nx),
        r(Bn * N * nu), A(Bn * N * nx * nx), Bm(Bn * N * nx * nu), c(Bn * N * nx),
        Sm(Bn * d.b3d()), Pi(Bn * d.b3d()), gam(Bn * L), dz(Bn * T, 0.0), merit_init(Bn),
        merit_a(Bn * NUM_ALPHAS);
    std::vector<int> conv(Bn, 0), sqp_it(Bn, 0), pcg_it(Bn, 0), status(Bn, 0);
    out.pcg_iters.clear();
    out.ls_min_merit.clear();
    out.ls_step_size.clear();
    out.ls_num_iters = 0;
    const int nthr = S.threads;
    auto fext_of = [&](int b) { return &S.fext[6 * b]; };
    parallel_for(nthr, Bn, [&](int b) {
        merit_init[b] = merit(m, Pb[b], d, dt, S.mu[b], xu + b * T, &dz[b * T], 1.0, xs + b * nx,
                              goal + b * 6 * N, fext_of(b));
    });
    out.initial_merit = merit_init;
    for (int b = 0; b < Bn; ++b)
        if (!std::isfinite(merit_init[b])) status[b] |= ST_NONFINITE;
    for (int it = 0; it < P.max_sqp_iters; ++it) {
        parallel_for(nthr, Bn, [&](int b) {
            double* Qb = &Q[b * N * nx * nx];
            double* Rb = &R[b * N * nu * nu];
            double* qb = &q[b * N * nx];
            double* rb = &r[b * N * nu];
            double* Ab = &A[b * N * nx * nx];
            double* Bb = &Bm[b * N * nx * nu];
            double* cb = &c[b * N * nx];
            setup_kkt(m, Pb[b], d, dt, xu + b * T, xs + b * nx, goal + b * 6 * N, fext_of(b), Qb,
                      Rb, qb, rb, Ab, Bb, cb);
            if (S.round_f32 & ORC_ROUND_KKT) {
                round_f32(Qb, (size_t)N * nx * nx);
                round_f32(Rb, (size_t)N * nu * nu);
                round_f32(qb, (size_t)N * nx);
                round_f32(rb, (size_t)N * nu);
                round_f32(Ab, (size_t)N * nx * nx);
                round_f32(Bb, (size_t)N * nx * nu);
                round_f32(cb, (size_t)N * nx);
            }
            form_schur(d, S.rho[b], Qb, Rb, qb, rb, Ab, Bb, cb, &Sm[b * d.b3d()],
                       &Pi[b * d.b3d()], &gam[b * L]);
            if (S.round_f32 & ORC_ROUND_SCHUR) {
                round_f32(&Sm[b * d.b3d()], d.b3d());
                round_f32(&Pi[b * d.b3d()], d.b3d());
                round_f32(&gam[b * L], L);
                round_f32(Qb, (size_t)N * nx * nx);
                round_f32(Rb, (size_t)N * nu * nu);
            }
            if (S.round_f32 & ORC_ROUND_S) round_f32(&Sm[b * d.b3d()], d.b3d());
            if (S.round_f32 & ORC_ROUND_PINV) round_f32(&Pi[b * d.b3d()], d.b3d());
            if (S.round_f32 & ORC_ROUND_GAMMA) round_f32(&gam[b * L], L);
            pcg_it[b] = conv[b] ? 0
                                : pcg(d, &Sm[b * d.b3d()], &Pi[b * d.b3d()], &gam[b * L],
                                      &S.lambda[b * L], S.tol[b], P.max_pcg_iters);
            if (S.round_f32 & ORC_ROUND_LAMBDA) round_f32(&S.lambda[b * L], L);
            compute_dz(d, &S.lambda[b * L], Qb, Rb, qb, rb, Ab, Bb, &dz[b * T]);
        });
        out.pcg_iters.insert(out.pcg_iters.end(), pcg_it.begin(), pcg_it.end());
        int num_solved = 0;
        for (int b = 0; b < Bn; ++b) {
            if (!conv[b] && pcg_it[b] >= P.max_pcg_iters) status[b] |= ST_PCG_MAX;
            if (pcg_it[b] == 0) {
                conv[b] = 1;
                sqp_it[b] += 1;
            }
            if (conv[b]) num_solved++;
            else sqp_it[b] += 1;
        }
        if (num_solved >= Bn * P.solve_ratio) break;
        std::vector<double> step(Bn);
        parallel_for(nthr, Bn, [&](int b) {
            double* xb = xu + b * T;
            double best = 1e38;
            int bj = 0;
            for (int j = 0; j < NUM_ALPHAS; ++j) {
                double a = 1.0 / (double)(1 << j);
                double v = merit(m, Pb[b], d, dt, S.mu[b], xb, &dz[b * T], a, xs + b * nx,
                                 goal + b * 6 * N, fext_of(b));
                merit_a[b * NUM_ALPHAS + j] = v;
                if (v < best) { best = v; bj = j; }
            }
            /* lineSearchAndUpdateBatchedKernel (line_search.cuh:27-97) */
            bool ok = best < merit_init[b];
            bool any_finite = false;
            for (int j = 0; j < NUM_ALPHAS; ++j) any_finite |= std::isfinite(merit_a[b * NUM_ALPHAS + j]);
            if (!ok) status[b] |= ST_LS_FAIL;
            if (!any_finite) status[b] |= ST_NONFINITE;
            if (S.adapt_rho) {
                double mult = ok ? std::min(S.drho[b] / RHO_FACTOR, 1.0 / RHO_FACTOR)
                                 : std::max(S.drho[b] * RHO_FACTOR, RHO_FACTOR);
                S.drho[b] = mult;
                S.rho[b] = std::max(S.rho[b] * mult, RHO_MIN);
                S.rho[b] = std::min(S.rho[b], RHO_MAX);
            }
            if (!ok) {
                if (S.rho[b] > RHO_MAX) S.rho[b] = RHO_INIT;
                step[b] = -1;
            } else {
                double a = 1.0 / (double)(1 << bj);
                merit_init[b] = best;
                step[b] = a;
                for (int i = 0; i < T; ++i) xb[i] += a * dz[b * T + i];
                if (S.round_f32 & ORC_ROUND_XU) round_f32(xb, T);
            }
        });
        out.ls_num_iters++;
        out.ls_min_merit.insert(out.ls_min_merit.end(), merit_init.begin(), merit_init.end());
        out.ls_step_size.insert(out.ls_step_size.end(), step.begin(), step.end());
    }
    std::fill(dz.begin(), dz.end(), 0.0);
    parallel_for(nthr, Bn, [&](int b) {
        merit_init[b] = merit(m, Pb[b], d, dt, S.mu[b], xu + b * T, &dz[b * T], 1.0, xs + b * nx,
                              goal + b * 6 * N, fext_of(b));
    });
    out.final_merit = merit_init;
    out.sqp_iters = sqp_it;
    out.kkt_converged = conv;
    for (int b = 0; b < Bn; ++b) {
        if (!std::isfinite(merit_init[b])) status[b] |= ST_NONFINITE;
        status[b] |= conv[b] ? ST_CONVERGED : ST_MAX_ITER;
    }
    out.status = status;
    S.drho = S.drho_init;
}

}  // namespace orc

/* ==================================================================== */
/* C ABI for ctypes                                                       */
using namespace orc;

extern "C" {

void orc_set_snap(double v) { SNAP = v; }

int orc_builtin_model(int plant, gato_model_t* out) { return gato_plant_fill(plant, out); }

void* orc_model_create(const gato_model_t* src)
{
    Model* m = new Model;
    build_model(src, m);
    return m;
}
void orc_model_destroy(void* h) { delete (Model*)h; }

void orc_rnea(void* h, const double* q, const double* qd, const double* qdd,
              const double* fext, double* tau)
{
    rnea(*(Model*)h, q, qd, qdd, fext, tau, nullptr);
}
void orc_mass_matrix(void* h, const double* q, double* M) { crba(*(Model*)h, q, M); }
void orc_fd(void* h, const double* q, const double* qd, const double* u, const double* fext,
            double* qdd)
{
    fd(*(Model*)h, q, qd, u, fext, qdd, nullptr);
}
void orc_fd_grad(void* h, const double* q, const double* qd, const double* u,
                 const double* fext, double* qdd, double* df_du)
{
    fd_grad(*(Model*)h, q, qd, u, fext, qdd, df_du);
}
void orc_rnea_grad(void* h, const double* q, const double* qd, const double* qdd,
                   const double* fext, double* dq, double* dqd)
{
    rnea_derivatives(*(Model*)h, q, qd, qdd, fext, dq, dqd);
}
void orc_ee_pos(void* h, const double* q, double* p, double* J)
{
    ee_pos(*(Model*)h, q, p, J);
}

double orc_tracking_cost(void* h, const gato_params_t* p, const double* xu, int has_u,
                         const double* goal, int terminal, const double* wdiag)
{
    Params P = to_params(p);
    P.wd = wdiag;
    return tracking_cost(*(Model*)h, P, xu, has_u != 0, goal, terminal != 0);
}

void orc_setup_kkt(void* h, int N, const gato_params_t* p, double dt, const double* xu,
                   const double* xs, const double* goal, const double* fext, double* Q,
                   double* R, double* q, double* r, double* A, double* B, double* c,
                   const double* wdiag)
{
    Model& m = *(Model*)h;
    Dims d{m.nq, 2 * m.nq, m.nq, N};
    Params P = to_params(p);
    P.wd = wdiag;
    setup_kkt(m, P, d, dt, xu, xs, goal, fext, Q, R, q, r, A, B, c);
}

void orc_form_schur(int nq, int N, double rho, double* Q, double* R, const double* q,
                    const double* r, const double* A, const double* B, const double* c,
                    double* S, double* Pinv, double* gamma)
{
    Dims d{nq, 2 * nq, nq, N};
    form_schur(d, rho, Q, R, q, r, A, B, c, S, Pinv, gamma);
}

int orc_pcg(int nq, int N, const double* S, const double* Pinv, const double* gamma,
            double* lambda, double eps, int max_iters)
{
    Dims d{nq, 2 * nq, nq, N};
    return pcg(d, S, Pinv, gamma, lambda, eps, max_iters);
}

void orc_compute_dz(int nq, int N, const double* lambda, const double* Qinv,
                    const double* Rinv, double* q, double* r, const double* A, const double* B,
                    double* dz)
{
    Dims d{nq, 2 * nq, nq, N};
    compute_dz(d, lambda, Qinv, Rinv, q, r, A, B, dz);
}

double orc_merit(void* h, int N, const gato_params_t* p, double dt, double mu,
                 const double* xu, const double* dz, double alpha, const double* xs,
                 const double* goal, const double* fext, const double* wdiag)
{
    Model& m = *(Model*)h;
    Dims d{m.nq, 2 * m.nq, m.nq, N};
    Params P = to_params(p);
    P.wd = wdiag;
    return merit(m, P, d, dt, mu, xu, dz, alpha, xs, goal, fext);
}

/* compute_integrator_error (integrator.cuh:211-233): |x_{k+1} - f(x_k,u_k)|_1
   for xux = [x_k u_k x_{k+1}] */
double orc_integrator_error(void* h, const double* xux, const double* fext, double dt)
{
    Model& m = *(Model*)h;
    const int nq = m.nq, nx = 2 * nq;
    double qdd[GATO_MAX_NQ], xn[2 * GATO_MAX_NQ];
    fd(m, xux, xux + nq, xux + nx, fext, qdd, nullptr);
    integrate(nq, xux, qdd, dt, xn);
    double e = 0;
    for (int i = 0; i < nx; ++i) e += fabs(xux[nx + nq + i] - xn[i]);
    return e;
}

void orc_integrate(int nq, const double* x, const double* qdd, double dt, double* xn)
{
    integrate(nq, x, qdd, dt, xn);
}

/* ---- batched solver ---- */
void* orc_solver_create(const gato_model_t* src, int N, int batch, const gato_params_t* p)
{
    Solver* S = new Solver;
    build_model(src, &S->model);
    S->P = to_params(p);
    S->d = Dims{src->nq, 2 * src->nq, src->nq, N};
    S->Bn = batch;
    S->lambda.assign((size_t)batch * S->d.vecp(), 0.0);
    S->rho.assign(batch, S->P.rho);
    S->rho_init = S->rho;
    S->drho.assign(batch, 1.0);
    S->drho_init = S->drho;
    S->mu.assign(batch, S->P.mu);
    S->tol.assign(batch, S->P.pcg_tol);
    S->fext.assign(6 * (size_t)batch, 0.0);
    return S;
}
void orc_solver_destroy(void* h) { delete (Solver*)h; }
void orc_solver_set_threads(void* h, int n) { ((Solver*)h)->threads = n < 1 ? 1 : n; }
void orc_solver_set_rho(void* h, const double* rho, int as_default)
{
    Solver* S = (Solver*)h;
    S->rho.assign(rho, rho + S->Bn);
    if (as_default) S->rho_init = S->rho;
}
void orc_solver_set_drho(void* h, const double* v, int as_default)
{
    Solver* S = (Solver*)h;
    S->drho.assign(v, v + S->Bn);
    if (as_default) S->drho_init = S->drho;
}
void orc_solver_set_mu(void* h, const double* v)
{
    Solver* S = (Solver*)h;
    S->mu.assign(v, v + S->Bn);
}
void orc_solver_set_tol(void* h, const double* v)
{
    Solver* S = (Solver*)h;
    S->tol.assign(v, v + S->Bn);
}
void orc_solver_set_fext(void* h, const double* v)
{
    Solver* S = (Solver*)h;
    S->fext.assign(v, v + 6 * S->Bn);
}
void orc_solver_set_cost_diag(void* h, const double* v)
{
    Solver* S = (Solver*)h;
    if (v)
        S->wdiag.assign(v, v + (size_t)S->Bn * (S->d.nx + S->d.nu));
    else
        S->wdiag.clear();
}
void orc_solver_set_adapt(void* h, int on) { ((Solver*)h)->adapt_rho = on != 0; }
/* flags: ORC_ROUND_* (0 = exact FP64 throughout, the default) */
void orc_solver_set_round_f32(void* h, int flags) { ((Solver*)h)->round_f32 = flags; }
void orc_solver_reset_dual(void* h)
{
    Solver* S = (Solver*)h;
    std::fill(S->lambda.begin(), S->lambda.end(), 0.0);
}
void orc_solver_reset_rho(void* h)
{
    Solver* S = (Solver*)h;
    S->rho = S->rho_init;
    S->drho = S->drho_init;
}
void orc_solver_get_lambda(void* h, double* out)
{
    Solver* S = (Solver*)h;
    memcpy(out, S->lambda.data(), sizeof(double) * S->lambda.size());
}
void orc_solver_set_lambda(void* h, const double* in)
{
    Solver* S = (Solver*)h;
    memcpy(S->lambda.data(), in, sizeof(double) * S->lambda.size());
}
void orc_solver_get_rho(void* h, double* out)
{
    Solver* S = (Solver*)h;
    memcpy(out, S->rho.data(), sizeof(double) * S->Bn);
}

/* Runs one solve.  Outputs (may be NULL): sqp_iters[B], kkt_converged[B],
   final_merit[B], initial_merit[B], pcg_iters[max_iters*B],
   ls_min_merit[max_iters*B], ls_step_size[max_iters*B], status[B]; returns
   ls_num_iters; *seconds gets the wall time of the solve. */
int orc_solver_solve(void* h, double dt, double* xu, const double* xs, const double* goal,
                     int* sqp_iters, int* kkt_converged, double* final_merit,
                     double* initial_merit, int* pcg_iters, double* ls_min_merit,
                     double* ls_step_size, double* seconds, int* status)
{
    Solver* S = (Solver*)h;
    SolveOut out;
    auto t0 = std::chrono::steady_clock::now();
    solve(*S, dt, xu, xs, goal, out);
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    const int Bn = S->Bn;
    if (sqp_iters) memcpy(sqp_iters, out.sqp_iters.data(), sizeof(int) * Bn);
    if (kkt_converged) memcpy(kkt_converged, out.kkt_converged.data(), sizeof(int) * Bn);
    if (final_merit) memcpy(final_merit, out.final_merit.data(), sizeof(double) * Bn);
    if (initial_merit) memcpy(initial_merit, out.initial_merit.data(), sizeof(double) * Bn);
    int nrows = out.ls_num_iters;
    if (pcg_iters) memcpy(pcg_iters, out.pcg_iters.data(), sizeof(int) * Bn * nrows);
    if (ls_min_merit) memcpy(ls_min_merit, out.ls_min_merit.data(), sizeof(double) * Bn * nrows);
    if (ls_step_size) memcpy(ls_step_size, out.ls_step_size.data(), sizeof(double) * Bn * nrows);
    if (status) memcpy(status, out.status.data(), sizeof(int) * Bn);
    return nrows;
}

}  // extern "C"
