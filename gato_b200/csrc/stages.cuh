// Warp- and block-level stages of one SQP iteration.  Each function states
// the reference kernel it replaces.  Batch layouts follow gato/constants.h and
// gato/utils/linalg.cuh:547-674 (column-major n x n blocks per knot,
// row-major n x 3n block rows for S and P^-1, padded (N+2)*n dual vectors).
#pragma once

#include "common.cuh"
#include "dynamics.cuh"

namespace gato {

// ---------------------------------------------------------------------------
// KKT blocks of one knot (setupKKTSystemBatchedKernel,
// gato/bsqp/kernels/setup_kkt.cuh:52-107), one warp.
// xuk points at x_k (followed by u_k, x_{k+1}); smem is warp-private scratch
// of at least KktSmem<NQ>::SIZE floats.  Writes A_k, B_k, c_{k+1}, Q_k, q_k,
// R_k, r_k and, for k == N-2, Q_{N-1}, q_{N-1} (evaluated at x_{N-2}, the
// reference's terminal-block quirk, iiwa14_plant.cuh:426-450) and
// c_0 = x_0 - x_s.
template <int NQ>
struct KktSmem {
    static constexpr int XU = DynSmem<NQ>::SIZE;        // x_k u_k x_{k+1}
    static constexpr int G = XU + 5 * NQ;               // ge_j then bg_j
    static constexpr int SIZE = G + 2 * NQ;
};

// G = 16 runs two knots per warp, one per half-warp (all lanes of the warp
// must call together); `valid` = false evaluates without writing.
template <int NQ, typename T, int G = 32>
__device__ void kkt_knot(const DevModel<NQ, T>& M, const CostParams<T>& cp, int N, int k,
                         const T* __restrict__ xu, const T* __restrict__ xs,
                         const T* __restrict__ goal, const T* fext, T* __restrict__ Q,
                         T* __restrict__ R, T* __restrict__ qv, T* __restrict__ rv,
                         T* __restrict__ A, T* __restrict__ Bm, T* __restrict__ c,
                         T* s, bool valid = true)
{
    using D = Dims<NQ>;
    constexpr int nx = D::nx, nu = D::nu;
    const int l = valid ? (lane_id() & (G - 1)) : (lane_id() & (G - 1)) + G * 64;
    const int lg = lane_id() & (G - 1);
    const T* xuk = xu + k * D::nxu;
    T* sx = s + KktSmem<NQ>::XU;
    for (int i = lg; i < 2 * nx + nu; i += G) sx[i] = xuk[i];
    __syncwarp();
    const T* q = sx;
    const T* qd = sx + NQ;
    const T* u = sx + nx;
    const T* xk1 = sx + nx + nu;
    dyn_load_transforms<NQ, T, G>(M, q, s);
    __syncwarp();
    T minv_col[NQ];
    dyn_forward<NQ, T, G>(M, s, q, qd, u, fext, true, minv_col);
    T qdd[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qdd[i] = s[DynSmem<NQ>::QDD + i];
    T dtau[NQ];
    rnea_derivative_lane<NQ, T, G>(M, s, qd, qdd, fext, dtau);
    const T dt = cp.dt;
    const T h2 = T(0.5) * dt * dt;
    // integrator_gradient_inner, trapezoidal (integrator.cuh:143-184)
    if (l < nx) {
        T dq[NQ];
#pragma unroll
        for (int r = 0; r < NQ; ++r) {
            T acc = T(0.0);
#pragma unroll
            for (int t = 0; t < NQ; ++t) acc += s[DynSmem<NQ>::MINV + t * NQ + r] * dtau[t];
            dq[r] = -acc;
        }
        T* Ak = A + k * D::nx2 + l * nx;
#pragma unroll
        for (int r = 0; r < NQ; ++r) {
            T v = (r == l) ? T(1.0) : T(0.0);
            if (l == r + NQ) v += dt;
            Ak[r] = v + h2 * dq[r];
            Ak[NQ + r] = ((NQ + r == l) ? T(1.0) : T(0.0)) + dt * dq[r];
        }
        // integrator_error_inner (integrator.cuh:48-62): c_{k+1} = x_{k+1} - f(x_k, u_k)
        T xn;
        if (l < NQ)
            xn = q[l] + dt * qd[l] + T(0.5) * qdd[l] * dt * dt;
        else
            xn = qd[l - NQ] + dt * qdd[l - NQ];
        c[(k + 1) * nx + l] = xk1[l] - xn;
    }
    if (l >= NQ && l < 2 * NQ) {
        const int j = l - NQ;
        T* Bk = Bm + k * nx * nu + j * nx;
#pragma unroll
        for (int r = 0; r < NQ; ++r) {
            Bk[r] = h2 * minv_col[r];
            Bk[NQ + r] = dt * minv_col[r];
        }
    }
    // tracking cost gradient and Hessian (iiwa14_plant.cuh:338-424,
    // indy7_plant.cuh:325-420); the weight is q_cost at every KKT knot
    T p[3], J[3];
    fk_lane<NQ, T, G>(M, s, p, J);
    const T w = cp.q_cost;
    T* sg = s + KktSmem<NQ>::G;
    const int style = M.barrier_style;
    const T* gk = goal + 6 * k;
    for (int pass = 0; pass < ((k == N - 2) ? 2 : 1); ++pass) {
        const T* gg = gk + 6 * pass;
        const T e0 = p[0] - gg[0], e1 = p[1] - gg[1], e2 = p[2] - gg[2];
        if (lg < NQ) {
            sg[lg] = J[0] * e0 + J[1] * e1 + J[2] * e2;
            sg[NQ + lg] = barrier_grad(style, q[lg], M.qlo[lg], M.qhi[lg]);
        }
        __syncwarp();
        const int kk = k + pass;
        T* Qk = Q + kk * D::nx2;
        T* qk = qv + kk * nx;
        if (l < nx) {
            const int i = l;
            T g;
            if (i < NQ) {
                g = sg[i] * w + cp.q_lim_cost * sg[NQ + i];
                if (cp.wdiag) g += cp.wdiag[i] * sx[i];
            } else {
                g = (cp.wdiag ? cp.wdiag[i] : cp.qd_cost) * sx[i] +
                    cp.vel_lim_cost * barrier_grad(style, sx[i], M.vlo[i - NQ], M.vhi[i - NQ]);
            }
            qk[i] = g;
            // column i of Q (symmetric)
            for (int jr = 0; jr < nx; ++jr) {
                T val;
                if (i < NQ && jr < NQ) {
                    val = sg[jr] * sg[i] * w;
                    if (style == 0) {
                        if (i == jr) val += cp.q_lim_cost * barrier_hess(q[i], M.qlo[i], M.qhi[i]);
                    } else {
                        val += cp.q_lim_cost * sg[NQ + i] * sg[NQ + jr];
                    }
                    if (cp.wdiag && i == jr) val += cp.wdiag[i];
                } else {
                    val = (i == jr) ? (cp.wdiag ? cp.wdiag[i] : cp.qd_cost) : T(0.0);
                    if (i == jr) {
                        if (style == 0) {
                            val += cp.vel_lim_cost * barrier_hess(sx[i], M.vlo[i - NQ], M.vhi[i - NQ]);
                        } else {
                            const T gv = barrier_grad(1, sx[i], M.vlo[i - NQ], M.vhi[i - NQ]);
                            val += cp.vel_lim_cost * gv * gv;
                        }
                    }
                }
                Qk[i * nx + jr] = val;
            }
        }
        if (pass == 0 && l < nu) {
            const T uu = u[l];
            const T uw = cp.wdiag ? cp.wdiag[nx + l] : cp.u_cost;
            rv[k * nu + l] = uw * uu + cp.ctrl_lim_cost * barrier_grad(style, uu, M.ulo[l], M.uhi[l]);
            T* Rk = R + k * nu * nu + l * nu;
            for (int jr = 0; jr < nu; ++jr) {
                T val = (jr == l) ? uw : T(0.0);
                if (jr == l) {
                    if (style == 0) {
                        val += cp.ctrl_lim_cost * barrier_hess(uu, M.ulo[l], M.uhi[l]);
                    } else {
                        const T gu = barrier_grad(1, uu, M.ulo[l], M.uhi[l]);
                        val += cp.ctrl_lim_cost * gu * gu;
                    }
                }
                Rk[jr] = val;
            }
        }
        __syncwarp();
    }
    if (k == N - 2 && l < nx) c[l] = xu[l] - xs[l];
}

// ---------------------------------------------------------------------------
// small dense helpers on warp-private shared memory (column-major)

// Loads [A | I] for a DIM x DIM matrix held column-major at src, adding rho to
// the first DIM/2 diagonal entries when rho_half != 0 (addScaledIdentity,
// gato/utils/linalg.cuh:84-96), inverts across lanes and stores A^-1
// column-major to dst.  dst may alias src.
template <int DIM, typename T>
__device__ __forceinline__ void warp_invert(const T* src, T rho_half, T* dst)
{
    const int l = lane_id();
    T col[DIM];
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
        T v;
        if (l < DIM) {
            v = src[l * DIM + r];
            if (r == l && r < DIM / 2) v += rho_half;
        } else {
            v = (l - DIM == r) ? T(1.0) : T(0.0);
        }
        col[r] = v;
    }
    __syncwarp();
    warp_gj<DIM, T>(col);
    if (l >= DIM && l < 2 * DIM) {
#pragma unroll
        for (int r = 0; r < DIM; ++r) dst[(l - DIM) * DIM + r] = col[r];
    }
    __syncwarp();
}

// out (m x n) = A (m x kdim) * B (kdim x n) [+ C if accumulate]; column-major,
// leading dimensions equal to the row counts.  Lane j of each half-warp
// computes column j: the lower half-warp rows [0, R0), the upper [R0, MR), so
// 2 NC lanes share the work (one column per lane would leave more than half
// of the warp idle at NC = 14).  Every entry is the same FMA sequence over t
// as with one lane per column.  transB selects B^T (B stored n x kdim).
template <int MR, int KD, int NC, bool TRANSB, bool ACC, typename T>
__device__ __forceinline__ void warp_gemm(T* out, const T* A, const T* B)
{
    static_assert(NC <= 16, "one column per lane of a half-warp");
    if constexpr (sizeof(T) == 4 && MR % 2 == 0) {
        // FP32: row pairs in packed FMAs (each entry still one fmaf per t, in
        // order), the lower half-warp taking the first R0 rows, R0 even so
        // that every pair is an aligned float2 (A and out 8-byte aligned)
        constexpr int R0 = ((MR / 2) + 1) & ~1, P0 = R0 / 2;
        const int l = lane_id();
        const int j = l & 15, hi = l >> 4;
        const int r0 = hi ? R0 : 0, np = hi ? (MR - R0) / 2 : P0;
        if (j < NC) {
            float2 acc[P0];
#pragma unroll
            for (int q = 0; q < P0; ++q)
                acc[q] = (ACC && q < np) ? *reinterpret_cast<const float2*>(out + j * MR + r0 + 2 * q)
                                         : make_float2(0.f, 0.f);
#pragma unroll
            for (int t = 0; t < KD; ++t) {
                const float b = TRANSB ? B[t * NC + j] : B[j * KD + t];
                const float2 bb = make_float2(b, b);
#pragma unroll
                for (int q = 0; q < P0; ++q)
                    if (q < np)
                        acc[q] = __ffma2_rn(
                            *reinterpret_cast<const float2*>(A + t * MR + r0 + 2 * q), bb, acc[q]);
            }
#pragma unroll
            for (int q = 0; q < P0; ++q)
                if (q < np) *reinterpret_cast<float2*>(out + j * MR + r0 + 2 * q) = acc[q];
        }
        __syncwarp();
        return;
    }
    constexpr int R0 = (MR + 1) / 2;
    const int l = lane_id();
    const int j = l & 15, r0 = (l >> 4) ? R0 : 0;
    if (j < NC) {
        T acc[R0];
#pragma unroll
        for (int i = 0; i < R0; ++i)
            acc[i] = (ACC && r0 + i < MR) ? out[j * MR + r0 + i] : T(0.0);
#pragma unroll
        for (int t = 0; t < KD; ++t) {
            const T b = TRANSB ? B[t * NC + j] : B[j * KD + t];
#pragma unroll
            for (int i = 0; i < R0; ++i)
                if (MR % 2 == 0 || r0 + i < MR) acc[i] += A[t * MR + r0 + i] * b;
        }
#pragma unroll
        for (int i = 0; i < R0; ++i)
            if (MR % 2 == 0 || r0 + i < MR) out[j * MR + r0 + i] = acc[i];
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Schur complement of one knot (formSchurSystemBatchedKernel1,
// gato/bsqp/kernels/schur_linsys.cuh:54-164), one warp, given the
// inverses Qi_k = (Q_k + rho I_q)^-1, Qi_{k+1} and Ri_k = R_k^-1 already in
// global memory.  Writes S row k right block (phi^T), S row k+1 left (phi)
// and main (-theta), P^-1 row k+1 main (-(theta + rho I_q)^-1) and
// gamma_{k+1}.
template <int NQ>
struct SchurSmem {
    static constexpr int n = 2 * NQ, m = NQ, n2 = n * n;
    static constexpr int A = 0;
    static constexpr int B = A + n2;
    static constexpr int QI = B + n * m;
    static constexpr int QI1 = QI + n2;
    static constexpr int RI = QI1 + n2;
    static constexpr int PHI = RI + ((m * m + 1) & ~1);  // even offsets: float2 operands
    static constexpr int BRI = PHI + n2;
    static constexpr int TH = BRI + n * m;
    static constexpr int V = TH + n2;   // q_k, q_{k+1}, r_k, c_{k+1}
    static constexpr int SIZE = (V + 3 * n + m + 1) & ~1;
};

template <int NQ, typename T>
__device__ void schur_knot(int k, T rho, const T* __restrict__ Qi,
                           const T* __restrict__ Ri, const T* __restrict__ qv,
                           const T* __restrict__ rv, const T* __restrict__ A,
                           const T* __restrict__ Bm, const T* __restrict__ c,
                           T* __restrict__ S, T* __restrict__ P,
                           T* __restrict__ gamma, T* s)
{
    using L = SchurSmem<NQ>;
    constexpr int n = L::n, m = L::m, n2 = L::n2, RD = 3 * n;
    const int l = lane_id();
    // every global load of the knot is issued before the first store to
    // shared memory, so the warp waits for one round trip, not one per
    // strided pass
    constexpr int P2 = (n2 + WARP - 1) / WARP, PB = (n * m + WARP - 1) / WARP,
                  PR = (m * m + WARP - 1) / WARP;
    T ga[P2], gq[P2], gq1[P2], gb[PB], gr[PR], gv[4];
#pragma unroll
    for (int it = 0; it < P2; ++it) {
        const int i = l + it * WARP;
        if (i < n2) {
            ga[it] = A[k * n2 + i];
            gq[it] = Qi[k * n2 + i];
            gq1[it] = Qi[(k + 1) * n2 + i];
        }
    }
#pragma unroll
    for (int it = 0; it < PB; ++it) {
        const int i = l + it * WARP;
        if (i < n * m) gb[it] = Bm[k * n * m + i];
    }
#pragma unroll
    for (int it = 0; it < PR; ++it) {
        const int i = l + it * WARP;
        if (i < m * m) gr[it] = Ri[k * m * m + i];
    }
    if (l < n) {
        gv[0] = qv[k * n + l];
        gv[1] = qv[(k + 1) * n + l];
        gv[2] = c[(k + 1) * n + l];
    }
    if (l < m) gv[3] = rv[k * m + l];
#pragma unroll
    for (int it = 0; it < P2; ++it) {
        const int i = l + it * WARP;
        if (i < n2) {
            s[L::A + i] = ga[it];
            s[L::QI + i] = gq[it];
            s[L::QI1 + i] = gq1[it];
        }
    }
#pragma unroll
    for (int it = 0; it < PB; ++it) {
        const int i = l + it * WARP;
        if (i < n * m) s[L::B + i] = gb[it];
    }
#pragma unroll
    for (int it = 0; it < PR; ++it) {
        const int i = l + it * WARP;
        if (i < m * m) s[L::RI + i] = gr[it];
    }
    if (l < n) {
        s[L::V + l] = gv[0];
        s[L::V + n + l] = gv[1];
        s[L::V + 2 * n + m + l] = gv[2];
    }
    if (l < m) s[L::V + 2 * n + l] = gv[3];
    __syncwarp();
    // phi = A Qi_k, BRi = B Ri, theta = Qi_{k+1} + phi A^T + BRi B^T
    warp_gemm<n, n, n, false, false, T>(s + L::PHI, s + L::A, s + L::QI);
    warp_gemm<n, m, m, false, false, T>(s + L::BRI, s + L::B, s + L::RI);
    for (int i = l; i < n2; i += WARP) s[L::TH + i] = s[L::QI1 + i];
    __syncwarp();
    warp_gemm<n, n, n, true, true, T>(s + L::TH, s + L::PHI, s + L::A);
    warp_gemm<n, m, n, true, true, T>(s + L::TH, s + L::BRI, s + L::B);
    // gamma_{k+1} = c_{k+1} - Qi_{k+1} q_{k+1} + phi q_k + BRi r_k
    if (l < n) {
        T g = s[L::V + 2 * n + m + l];
#pragma unroll
        for (int t = 0; t < n; ++t)
            g += -s[L::QI1 + t * n + l] * s[L::V + n + t] + s[L::PHI + t * n + l] * s[L::V + t];
#pragma unroll
        for (int t = 0; t < m; ++t) g += s[L::BRI + t * n + l] * s[L::V + 2 * n + t];
        gamma[(k + 2) * n + l] = g;
    }
    // S blocks, row-major block rows (schur_linsys.cuh:136-147)
    T* Sright = S + k * 3 * n2 + 2 * n;
    T* Sleft = S + (k + 1) * 3 * n2;
    T* Smain = Sleft + n;
    for (int i = l; i < n2; i += WARP) {
        const int y = i / n, x = i % n;
        Sright[y * RD + x] = s[L::PHI + y * n + x];
        Sleft[y * RD + x] = s[L::PHI + x * n + y];
        Smain[y * RD + x] = -s[L::TH + x * n + y];
    }
    __syncwarp();
    // P^-1 row k+1 main = -(theta + rho I_q)^-1
    warp_invert<n, T>(s + L::TH, rho, s + L::QI);
    T* Pm = P + (k + 1) * 3 * n2 + n;
    for (int i = l; i < n2; i += WARP) {
        const int y = i / n, x = i % n;
        Pm[y * RD + x] = -s[L::QI + x * n + y];
    }
    __syncwarp();
}

// Block row 0 of S and P^-1 and gamma_0 (schur_linsys.cuh:166-210).
template <int NQ, typename T>
__device__ void schur_first(T rho, const T* __restrict__ Q, const T* __restrict__ Qi,
                            const T* __restrict__ qv, const T* __restrict__ c,
                            T* __restrict__ S, T* __restrict__ P,
                            T* __restrict__ gamma)
{
    constexpr int n = 2 * NQ, n2 = n * n, RD = 3 * n;
    const int l = lane_id();
    for (int i = l; i < n2; i += WARP) {
        const int y = i / n, x = i % n;
        T qt = Q[x * n + y];
        if (x == y && x < n / 2) qt += rho;
        P[y * RD + n + x] = -qt;
        S[y * RD + n + x] = -Qi[x * n + y];
    }
    if (l < n) {
        T g = c[l];
#pragma unroll
        for (int t = 0; t < n; ++t) g -= Qi[t * n + l] * qv[t];
        gamma[n + l] = g;
    }
}

// P^-1 off-diagonal blocks of one knot pair (formSchurSystemBatchedKernel2,
// schur_linsys.cuh:213-260): X = Pm_{k+1} phi_k Pm_k, P row k+1 left = -X,
// P row k right = -X^T.  smem: 4 n x n blocks.
template <int NQ, typename T>
__device__ void schur_offdiag(int k, const T* __restrict__ S, T* __restrict__ P, T* s)
{
    constexpr int n = 2 * NQ, n2 = n * n, RD = 3 * n;
    const int l = lane_id();
    T* Ta = s;
    T* Tb = s + n2;
    T* ph = s + 2 * n2;
    T* sc = s + 3 * n2;
    const T* Pa = P + (k + 1) * 3 * n2 + n;
    const T* Pb = P + k * 3 * n2 + n;
    const T* Sl = S + (k + 1) * 3 * n2;
    constexpr int P2 = (n2 + WARP - 1) / WARP;
    T ga[P2], gb[P2], gp[P2];  // all loads first, as in schur_knot
#pragma unroll
    for (int it = 0; it < P2; ++it) {
        const int i = l + it * WARP;
        if (i < n2) {
            const int y = i / n, x = i % n;
            ga[it] = Pa[y * RD + x];
            gb[it] = Pb[y * RD + x];
            gp[it] = Sl[y * RD + x];
        }
    }
#pragma unroll
    for (int it = 0; it < P2; ++it) {
        const int i = l + it * WARP;
        if (i < n2) {
            const int y = i / n, x = i % n;
            Ta[x * n + y] = ga[it];
            Tb[x * n + y] = gb[it];
            ph[x * n + y] = gp[it];
        }
    }
    __syncwarp();
    warp_gemm<n, n, n, false, false, T>(sc, ph, Tb);
    warp_gemm<n, n, n, false, false, T>(ph, Ta, sc);
    T* Pright = P + k * 3 * n2 + 2 * n;
    T* Pleft = P + (k + 1) * 3 * n2;
    for (int i = l; i < n2; i += WARP) {
        const int y = i / n, x = i % n;
        Pright[y * RD + x] = -ph[y * n + x];
        Pleft[y * RD + x] = -ph[x * n + y];
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Step recovery of one knot (computeDzBatchedKernel,
// gato/bsqp/kernels/schur_linsys.cuh:312-431), one warp:
//   res_x = q_k - lambda_k + A_k^T lambda_{k+1},  dz_x = -Qi_k res_x
//   res_u = r_k + B_k^T lambda_{k+1},             dz_u = -Ri_k res_u
// q and r are overwritten with the residuals.
template <int NQ, typename T>
__device__ void dz_knot(int N, int k, const T* __restrict__ lam, const T* __restrict__ Qi,
                        const T* __restrict__ Ri, T* __restrict__ qv, T* __restrict__ rv,
                        const T* __restrict__ A, const T* __restrict__ Bm,
                        T* __restrict__ dz, T* s)
{
    constexpr int n = 2 * NQ, m = NQ, n2 = n * n;
    const int l = lane_id();
    const T* lk = lam + (k + 1) * n;
    const T* lk1 = lam + (k + 2) * n;
    T* res = s;
    T* resu = s + n;
    if (l < n) {
        T acc = T(0.0);
        if (k < N - 1) {
#pragma unroll
            for (int t = 0; t < n; ++t) acc += lk1[t] * A[k * n2 + l * n + t];
        }
        res[l] = qv[k * n + l] - lk[l] + acc;
    }
    if (l < m) {
        if (k < N - 1) {
            T acc = T(0.0);
#pragma unroll
            for (int t = 0; t < n; ++t) acc += lk1[t] * Bm[k * n * m + l * n + t];
            resu[l] = rv[k * m + l] + acc;
        } else {
            resu[l] = T(0.0);
        }
    }
    __syncwarp();
    T* dzk = dz + k * (n + m);
    if (l < n) {
        T acc = T(0.0);
#pragma unroll
        for (int t = 0; t < n; ++t) acc += Qi[k * n2 + t * n + l] * res[t];
        dzk[l] = -acc;
        qv[k * n + l] = res[l];
    }
    if (l < m) {
        if (k < N - 1) {
            T acc = T(0.0);
#pragma unroll
            for (int t = 0; t < m; ++t) acc += Ri[k * m * m + t * m + l] * resu[t];
            dzk[n + l] = -acc;
        }
        rv[k * m + l] = resu[l];
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Merit contribution of one knot at step alpha (computeMeritBatchedKernel,
// gato/bsqp/kernels/merit.cuh:34-91), one warp; returns cost + mu * defect
// in every lane.  dz may be null (alpha = 0 path of the initial merit).
template <int NQ>
struct MeritSmem {
    static constexpr int XU = DynSmem<NQ>::SIZE;
    static constexpr int SIZE = XU + 5 * NQ;
};

template <int NQ, typename T>
__device__ T merit_knot(const DevModel<NQ, T>& M, const CostParams<T>& cp, int N, int k, T alpha,
                            T mu, const T* __restrict__ xu, const T* __restrict__ dz,
                            const T* __restrict__ xs, const T* __restrict__ goal,
                            const T* fext, T* s)
{
    using D = Dims<NQ>;
    constexpr int nx = D::nx, nu = D::nu;
    const int l = lane_id();
    const bool last = (k == N - 1);
    const int len = last ? nx : 2 * nx + nu;
    T* sx = s + MeritSmem<NQ>::XU;
    const T* xuk = xu + k * D::nxu;
    const T* dzk = dz ? dz + k * D::nxu : nullptr;
    for (int i = l; i < len; i += WARP) sx[i] = xuk[i] + (dzk ? alpha * dzk[i] : T(0.0));
    __syncwarp();
    const T* q = sx;
    const T* qd = sx + NQ;
    dyn_load_transforms<NQ, T>(M, q, s);
    __syncwarp();
    // trackingcost (iiwa14_plant.cuh:275-327): per-joint terms, then the
    // end-effector error with N_cost at the last knot
    T term = T(0.0);
    if (l < NQ) {
        const T v = qd[l];
        term += T(0.5) * (cp.wdiag ? cp.wdiag[NQ + l] : cp.qd_cost) * v * v;
        if (cp.wdiag) term += T(0.5) * cp.wdiag[l] * q[l] * q[l];
        term += cp.q_lim_cost * barrier(q[l], M.qlo[l], M.qhi[l]);
        term += cp.vel_lim_cost * barrier(v, M.vlo[l], M.vhi[l]);
        if (!last) {
            const T uu = sx[nx + l];
            term += T(0.5) * (cp.wdiag ? cp.wdiag[nx + l] : cp.u_cost) * uu * uu;
            term += cp.ctrl_lim_cost * barrier(uu, M.ulo[l], M.uhi[l]);
        }
    }
    T p[3];
    fk_lane<NQ, T>(M, s, p, nullptr);
    const T w = last ? cp.N_cost : cp.q_cost;
    if (l < 3) {
        const T e = p[l] - goal[6 * k + l];
        term += T(0.5) * w * e * e;
    }
    T defect = T(0.0);
    if (!last) {
        T minv_col[NQ];
        dyn_forward<NQ, T>(M, s, q, qd, sx + nx, fext, false, minv_col);
        // compute_integrator_error (integrator.cuh:211-233), L1 norm
        if (l < nx) {
            const T dt = cp.dt;
            T xn;
            if (l < NQ)
                xn = q[l] + dt * qd[l] + T(0.5) * s[DynSmem<NQ>::QDD + l] * dt * dt;
            else
                xn = qd[l - NQ] + dt * s[DynSmem<NQ>::QDD + l - NQ];
            defect = gabs(sx[nx + nu + l] - xn);
        }
    } else if (l < nx) {
        defect = gabs(xu[l] + (dz ? alpha * dz[l] : T(0.0)) - xs[l]);
    }
    const T cost = warp_sum(term);
    const T cons = warp_sum(defect);
    __syncwarp();
    return cost + mu * cons;
}

}  // namespace gato
