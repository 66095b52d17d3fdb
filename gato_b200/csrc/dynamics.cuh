// Warp-level rigid-body dynamics for one knot point (FP32 or FP64).
//
// One warp evaluates one (q, qd, u) sample.  Lanes take independent columns
// of the work so that no lane waits on another inside a recursion:
//   * joint-space inertia: lane j < NQ runs a unit-acceleration RNEA
//     (qd = 0, qdd = e_j, no gravity) and ends holding column j of M;
//     lane 2NQ runs the bias RNEA c(q, qd, g, f_ext) in the same instruction
//     stream;
//   * M^-1: pivot-free Gauss-Jordan across lanes, lane j holding column j of
//     [M | I] (lanes NQ..2NQ-1 end with the columns of M^-1);
//   * derivatives: lane j < 2NQ differentiates the RNEA recursions with
//     respect to x_j (q_j for j < NQ, qd_{j-NQ} otherwise) in forward mode,
//     recomputing the nominal pass in registers.
// Replaces the GRiD-generated functions the reference calls
// (gato/dynamics/iiwa14/iiwa14_grid.cuh:2211-2292, 3730-, 4740-, 5339-5352,
// 5547-; gato/dynamics/iiwa14/iiwa14_plant.cuh:157-268) with an algorithm of
// its own; in FP64 the results agree with the reference to 1e-10.
#pragma once

#include "common.cuh"

namespace gato {

// Layout of the warp-private shared scratch used by one knot evaluation.
template <int NQ>
struct DynSmem {
    static constexpr int SIN = 0;               // sin q (NQ)
    static constexpr int COS = NQ;              // cos q (NQ)
    static constexpr int EC = 2 * NQ;           // per joint: E (9) then C (9)
    static constexpr int MINV = EC + 18 * NQ;   // M^-1 column-major NQ x NQ
    static constexpr int QDD = MINV + NQ * NQ;  // qdd (NQ)
    static constexpr int SIZE = QDD + NQ;
};

// ---------------------------------------------------------------------------
// spatial algebra on register 6-vectors [angular; linear]

// y = X x with X = [E 0; C E]
template <typename T>
__device__ __forceinline__ void x_mul(const T* E, const T* C, const T* x, T* y)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        y[r] = E[3 * r] * x[0] + E[3 * r + 1] * x[1] + E[3 * r + 2] * x[2];
        y[3 + r] = C[3 * r] * x[0] + C[3 * r + 1] * x[1] + C[3 * r + 2] * x[2] +
                   E[3 * r] * x[3] + E[3 * r + 1] * x[4] + E[3 * r + 2] * x[5];
    }
}
// y = X^T f
template <typename T>
__device__ __forceinline__ void xt_mul(const T* E, const T* C, const T* f, T* y)
{
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        y[r] = E[r] * f[0] + E[3 + r] * f[1] + E[6 + r] * f[2] + C[r] * f[3] + C[3 + r] * f[4] +
               C[6 + r] * f[5];
        y[3 + r] = E[r] * f[3] + E[3 + r] * f[4] + E[6 + r] * f[5];
    }
}
// crm(u) e_z
template <typename T>
__device__ __forceinline__ void add_cz(T* y, const T* u, T s)
{
    y[0] += s * u[1];
    y[1] -= s * u[0];
    y[3] += s * u[4];
    y[4] -= s * u[3];
}
// y += crf(v) f
template <typename T>
__device__ __forceinline__ void add_crf(T* y, const T* v, const T* f)
{
    y[0] += v[1] * f[2] - v[2] * f[1] + v[4] * f[5] - v[5] * f[4];
    y[1] += v[2] * f[0] - v[0] * f[2] + v[5] * f[3] - v[3] * f[5];
    y[2] += v[0] * f[1] - v[1] * f[0] + v[3] * f[4] - v[4] * f[3];
    y[3] += v[1] * f[5] - v[2] * f[4];
    y[4] += v[2] * f[3] - v[0] * f[5];
    y[5] += v[0] * f[4] - v[1] * f[3];
}
// f = I_i v  (spatial inertia about the link origin)
template <int NQ, typename T>
__device__ __forceinline__ void i_mul(const DevModel<NQ, T>& M, int i, const T* v, T* f)
{
    const T* I = M.Ibar[i];
    const T* h = M.h[i];
    const T m = M.mass[i];
    f[0] = I[0] * v[0] + I[1] * v[1] + I[2] * v[2] + (h[1] * v[5] - h[2] * v[4]);
    f[1] = I[1] * v[0] + I[3] * v[1] + I[4] * v[2] + (h[2] * v[3] - h[0] * v[5]);
    f[2] = I[2] * v[0] + I[4] * v[1] + I[5] * v[2] + (h[0] * v[4] - h[1] * v[3]);
    f[3] = m * v[3] - (h[1] * v[2] - h[2] * v[1]);
    f[4] = m * v[4] - (h[2] * v[0] - h[0] * v[2]);
    f[5] = m * v[5] - (h[0] * v[1] - h[1] * v[0]);
}

// ---------------------------------------------------------------------------
// per-knot set-up: sin/cos and the joint transforms X_i(q_i) into scratch.
// Must be followed by __syncwarp() before use.
template <int NQ, typename T, int G = 32>
__device__ __forceinline__ void dyn_load_transforms(const DevModel<NQ, T>& M, const T* q, T* s)
{
    const int l = lane_id() & (G - 1);
    if (l < NQ) {
        T sn, cs;
        gsincos(q[l], &sn, &cs);
        s[DynSmem<NQ>::SIN + l] = sn;
        s[DynSmem<NQ>::COS + l] = cs;
        T* E = s + DynSmem<NQ>::EC + 18 * l;
        T* C = E + 9;
        const T* E0 = M.E0[l];
        const T* C0 = M.C0[l];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            E[c] = cs * E0[c] + sn * E0[3 + c];
            E[3 + c] = -sn * E0[c] + cs * E0[3 + c];
            E[6 + c] = E0[6 + c];
            C[c] = cs * C0[c] + sn * C0[3 + c];
            C[3 + c] = -sn * C0[c] + cs * C0[3 + c];
            C[6 + c] = C0[6 + c];
        }
    }
}

// RNEA with per-lane inputs: tau = ID(q, qd_l, qdd_l) with base acceleration
// grav_l along z and, when use_fext, f_ext subtracted from the last link's
// force (iiwa14_fext.cuh:160-171).  qd_l/qdd_l are read through the flags so
// that lanes can run unit-acceleration passes in the same instruction stream.
template <int NQ, typename T>
__device__ __forceinline__ void rnea_lane(const DevModel<NQ, T>& M, const T* s, const T* qd,
                                          T qd_scale, int unit_j, T grav, bool use_fext,
                                          const T* fext, T* tau)
{
    T v[6] = {0, 0, 0, 0, 0, 0};
    T a[6] = {0, 0, 0, 0, 0, grav};
    T f[NQ][6];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const T* E = s + DynSmem<NQ>::EC + 18 * i;
        const T* C = E + 9;
        T vn[6], an[6], t[6];
        x_mul(E, C, v, vn);
        const T qdi = qd_scale * qd[i];
        vn[2] += qdi;
        x_mul(E, C, a, an);
        an[2] += (i == unit_j) ? T(1.0) : T(0.0);
        add_cz(an, vn, qdi);
        i_mul(M, i, an, f[i]);
        i_mul(M, i, vn, t);
        add_crf(f[i], vn, t);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            v[k] = vn[k];
            a[k] = an[k];
        }
    }
    if (use_fext) {
#pragma unroll
        for (int k = 0; k < 6; ++k) f[NQ - 1][k] -= fext[k];
    }
#pragma unroll
    for (int i = NQ - 1; i >= 0; --i) {
        tau[i] = f[i][2];
        if (i > 0) {
            const T* E = s + DynSmem<NQ>::EC + 18 * i;
            const T* C = E + 9;
            T t[6];
            xt_mul(E, C, f[i], t);
#pragma unroll
            for (int k = 0; k < 6; ++k) f[i - 1][k] += t[k];
        }
    }
}

// In-place pivot-free Gauss-Jordan across lanes: lane c holds column c of an
// augmented [A | I] (DIM rows); lanes DIM..2DIM-1 end with the columns of
// A^-1.  Follows the elimination order of gato/utils/linalg.cuh:364-400
// (FP64 also its arithmetic, col_r -= (p_r / p_k) col_k).  FP32 forms one
// factor f = col_k / p_k per pivot and updates row pairs with packed FMAs,
// col_r = fma(-p_r, f, col_r): the same elimination with one rounding moved,
// at about a third of the arithmetic instructions.
// G is the lane-group width (16: two independent systems per warp).
template <int DIM, typename T, int G = 32>
__device__ __forceinline__ void warp_gj(T (&col)[DIM])
{
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        T pk[DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r) pk[r] = __shfl_sync(FULL, col[r], k, G);
        const T rcp = T(1.0) / pk[k];
        const T rowk = col[k];
        if constexpr (sizeof(T) == 4) {
            const float f = rcp * rowk;
            const float2 nf = make_float2(-f, -f);
#pragma unroll
            for (int r = 0; r + 1 < DIM; r += 2) {
                const float2 c = __ffma2_rn(make_float2(pk[r], pk[r + 1]), nf,
                                            make_float2(col[r], col[r + 1]));
                if (r != k) col[r] = c.x;
                if (r + 1 != k) col[r + 1] = c.y;
            }
            if (DIM % 2 == 1 && DIM - 1 != k) col[DIM - 1] = fmaf(-pk[DIM - 1], f, col[DIM - 1]);
        } else {
#pragma unroll
            for (int r = 0; r < DIM; ++r)
                if (r != k) col[r] -= (pk[r] * rcp) * rowk;
        }
        col[k] = rowk * rcp;
    }
}

// Forward dynamics of one knot: qdd into scratch (QDD) and, when with_minv,
// M^-1 column-major into scratch (MINV).  Needs dyn_load_transforms first.
// Returns, in lanes NQ..2NQ-1, column (lane-NQ) of M^-1 in minv_col.
template <int NQ, typename T, int G = 32>
__device__ __forceinline__ void dyn_forward(const DevModel<NQ, T>& M, T* s, const T* q,
                                            const T* qd, const T* u, const T* fext,
                                            bool with_minv, T (&minv_col)[NQ])
{
    static_assert(2 * NQ < G, "the bias lane must lie inside the lane group");
    const int l = lane_id() & (G - 1);
    const bool bias = (l == 2 * NQ);
    T tau[NQ];
    rnea_lane<NQ, T>(M, s, qd, bias ? T(1.0) : T(0.0), (l < NQ) ? l : -1, bias ? M.gravity : T(0.0),
                  bias && fext != nullptr, fext, tau);
    // [M | I] across lanes 0..2NQ-1
    T col[NQ];
#pragma unroll
    for (int r = 0; r < NQ; ++r) col[r] = (l < NQ) ? tau[r] : ((l - NQ == r) ? T(1.0) : T(0.0));
    warp_gj<NQ, T, G>(col);
    // bias c from lane 2NQ; qdd_r = (M^-1 column r) . (u - c)  (M^-1 symmetric)
    T qdd = T(0.0);
#pragma unroll
    for (int r = 0; r < NQ; ++r) {
        const T cr = __shfl_sync(FULL, tau[r], 2 * NQ, G);
        qdd += col[r] * (u[r] - cr);
    }
    if (l >= NQ && l < 2 * NQ) {
        s[DynSmem<NQ>::QDD + (l - NQ)] = qdd;
        if (with_minv) {
#pragma unroll
            for (int r = 0; r < NQ; ++r) s[DynSmem<NQ>::MINV + (l - NQ) * NQ + r] = col[r];
        }
    }
#pragma unroll
    for (int r = 0; r < NQ; ++r) minv_col[r] = col[r];
    __syncwarp();
}

// Forward-mode derivative of the RNEA recursions at (q, qd, qdd) with f_ext:
// lane j < 2NQ returns column j of [dtau/dq | dtau/dqd] in dtau.
template <int NQ, typename T, int G = 32>
__device__ __forceinline__ void rnea_derivative_lane(const DevModel<NQ, T>& M, const T* s,
                                                     const T* qd, const T* qdd,
                                                     const T* fext, T* dtau)
{
    const int l = lane_id() & (G - 1);
    const bool wq = l < NQ;
    const int j = wq ? l : l - NQ;
    T v[6] = {0, 0, 0, 0, 0, 0};
    T a[6] = {0, 0, 0, 0, 0, M.gravity};
    T dv[6] = {0, 0, 0, 0, 0, 0};
    T da[6] = {0, 0, 0, 0, 0, 0};
    T f[NQ][6], df[NQ][6];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const T* E = s + DynSmem<NQ>::EC + 18 * i;
        const T* C = E + 9;
        T xv[6], xa[6], vn[6], an[6], dvn[6], dan[6], iv[6], idv[6];
        x_mul(E, C, v, xv);
        x_mul(E, C, a, xa);
        x_mul(E, C, dv, dvn);
        x_mul(E, C, da, dan);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            vn[k] = xv[k];
            an[k] = xa[k];
        }
        vn[2] += qd[i];
        an[2] += qdd[i];
        add_cz(an, vn, qd[i]);
        if (i == j) {
            if (wq) {
                add_cz(dvn, xv, T(1.0));
                add_cz(dan, xa, T(1.0));
            } else {
                dvn[2] += T(1.0);
            }
        }
        add_cz(dan, dvn, qd[i]);
        if (i == j && !wq) add_cz(dan, vn, T(1.0));
        i_mul(M, i, an, f[i]);
        i_mul(M, i, vn, iv);
        add_crf(f[i], vn, iv);
        i_mul(M, i, dan, df[i]);
        i_mul(M, i, dvn, idv);
        add_crf(df[i], dvn, iv);
        add_crf(df[i], vn, idv);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            v[k] = vn[k];
            a[k] = an[k];
            dv[k] = dvn[k];
            da[k] = dan[k];
        }
    }
    if (fext != nullptr) {
#pragma unroll
        for (int k = 0; k < 6; ++k) f[NQ - 1][k] -= fext[k];
    }
#pragma unroll
    for (int i = NQ - 1; i >= 0; --i) {
        dtau[i] = df[i][2];
        if (i > 0) {
            const T* E = s + DynSmem<NQ>::EC + 18 * i;
            const T* C = E + 9;
            T t[6];
            xt_mul(E, C, df[i], t);
#pragma unroll
            for (int k = 0; k < 6; ++k) df[i - 1][k] += t[k];
            if (wq && i == j) {
                const T cf[6] = {-f[i][1], f[i][0], T(0.0), -f[i][4], f[i][3], T(0.0)};
                xt_mul(E, C, cf, t);
#pragma unroll
                for (int k = 0; k < 6; ++k) df[i - 1][k] += t[k];
            }
            xt_mul(E, C, f[i], t);
#pragma unroll
            for (int k = 0; k < 6; ++k) f[i - 1][k] += t[k];
        }
    }
}

// End-effector position (origin of the last link frame, as
// iiwa14_grid.cuh:2596-2672) computed redundantly by every lane; lane j < NQ
// also gets the position Jacobian column dp/dq_j = z_j x (p - o_j)
// (iiwa14_grid.cuh:2855-2966).  Needs dyn_load_transforms (sin/cos).
template <int NQ, typename T, int G = 32>
__device__ __forceinline__ void fk_lane(const DevModel<NQ, T>& M, const T* s, T* p, T* J)
{
    const int l = lane_id() & (G - 1);
    T R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    T o[3] = {0, 0, 0};
    T zj[3] = {0, 0, 0}, oj[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const T* R0 = M.R0[i];
        const T* P = M.P[i];
#pragma unroll
        for (int r = 0; r < 3; ++r) o[r] += R[3 * r] * P[0] + R[3 * r + 1] * P[1] + R[3 * r + 2] * P[2];
        const T sn = s[DynSmem<NQ>::SIN + i], cs = s[DynSmem<NQ>::COS + i];
        T Rj[9];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            Rj[3 * r] = cs * R0[3 * r] + sn * R0[3 * r + 1];
            Rj[3 * r + 1] = -sn * R0[3 * r] + cs * R0[3 * r + 1];
            Rj[3 * r + 2] = R0[3 * r + 2];
        }
        T Rn[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                Rn[3 * r + c] = R[3 * r] * Rj[c] + R[3 * r + 1] * Rj[3 + c] + R[3 * r + 2] * Rj[6 + c];
#pragma unroll
        for (int k = 0; k < 9; ++k) R[k] = Rn[k];
        if (i == l) {
            zj[0] = R[2];
            zj[1] = R[5];
            zj[2] = R[8];
            oj[0] = o[0];
            oj[1] = o[1];
            oj[2] = o[2];
        }
    }
    p[0] = o[0];
    p[1] = o[1];
    p[2] = o[2];
    if (J != nullptr) {
        const T d0 = o[0] - oj[0], d1 = o[1] - oj[1], d2 = o[2] - oj[2];
        J[0] = zj[1] * d2 - zj[2] * d1;
        J[1] = zj[2] * d0 - zj[0] * d2;
        J[2] = zj[0] * d1 - zj[1] * d0;
    }
}

// ---------------------------------------------------------------------------
// joint-limit barriers (gato/dynamics/iiwa14/iiwa14_plant.cuh:103-155,
// gato/dynamics/indy7/indy7_plant.cuh:141-147)
template <typename T>
__device__ __forceinline__ T barrier(T q, T lo, T hi)
{
    T dmin = q - lo, dmax = hi - q;
    dmin = (dmin <= T(1e-10)) ? T(1e-10) : dmin;
    dmax = (dmax <= T(1e-10)) ? T(1e-10) : dmax;
    return -glog(dmin) - glog(dmax);
}
template <typename T>
__device__ __forceinline__ T barrier_grad(int style, T q, T lo, T hi)
{
    T dmin = q - lo, dmax = hi - q;
    if (style == 0) {
        const T eps = T(1e-6);
        if (dmin >= T(0.0)) { if (dmin < eps) dmin = eps; } else { if (dmin > -eps) dmin = -eps; }
        if (dmax >= T(0.0)) { if (dmax < eps) dmax = eps; } else { if (dmax > -eps) dmax = -eps; }
        return -T(1.0) / dmin + T(1.0) / dmax;
    }
    dmin = (dmin <= T(1e-6)) ? T(1e-6) : dmin;
    dmax = (dmax <= T(1e-6)) ? T(1e-6) : dmax;
    return -T(1.0) / dmin + T(1.0) / dmax;
}
template <typename T>
__device__ __forceinline__ T barrier_hess(T q, T lo, T hi)
{
    const T eps = T(1e-6);
    T amin = gabs(q - lo), amax = gabs(hi - q);
    if (amin < eps) amin = eps;
    if (amax < eps) amax = eps;
    return T(1.0) / (amin * amin) + T(1.0) / (amax * amax);
}

}  // namespace gato
