/*
 * Algorithmic floating-point operation counts of the reference's per-knot
 * device functions, obtained by instantiating them (through the same host
 * shim as grid_ref_wrap.cpp) with a scalar type that counts every add,
 * subtract, multiply, divide and elementary function it performs.  Test and
 * measurement infrastructure only: the counts are the numerators of the
 * benchmark's roofline figures.  Builds oracle/_ref/flop_count_<plant>,
 * which prints one JSON object.
 *
 * Counted per knot (paths in the reference tree):
 *   kkt_dynamics   gato/dynamics/integrator.cuh compute_linearized_dynamics
 *                  (forward dynamics and its gradient, A, B, c)
 *   kkt_cost       gato/dynamics/<plant>/<plant>_plant.cuh
 *                  trackingCostGradientAndHessian
 *   merit_cost     trackingcost (one knot, one step size)
 *   merit_defect   gato/dynamics/integrator.cuh compute_integrator_error
 */
#include <cuda_runtime.h>

#include <cmath>

shim_uint3 threadIdx = {0, 0, 0};
shim_uint3 blockIdx = {0, 0, 0};
shim_uint3 blockDim = {1, 1, 1};
shim_uint3 gridDim = {1, 1, 1};

// counts an operation unless it is evaluated at compile time (the
// reference's constexpr limit tables)
#define FC_COUNT()                                  \
    do {                                            \
        if (!__builtin_is_constant_evaluated()) ++ops_counter(); \
    } while (0)

inline unsigned long long& ops_counter()
{
    static unsigned long long n = 0;
    return n;
}

struct Fc {
    double v;
    constexpr Fc() : v(0) {}
    constexpr Fc(double x) : v(x) {}
    constexpr Fc& operator+=(Fc o) { FC_COUNT(); v += o.v; return *this; }
    constexpr Fc& operator-=(Fc o) { FC_COUNT(); v -= o.v; return *this; }
    constexpr Fc& operator*=(Fc o) { FC_COUNT(); v *= o.v; return *this; }
    constexpr Fc& operator/=(Fc o) { FC_COUNT(); v /= o.v; return *this; }
    explicit constexpr operator double() const { return v; }
};
constexpr Fc operator+(Fc a, Fc b) { FC_COUNT(); return Fc(a.v + b.v); }
constexpr Fc operator-(Fc a, Fc b) { FC_COUNT(); return Fc(a.v - b.v); }
constexpr Fc operator*(Fc a, Fc b) { FC_COUNT(); return Fc(a.v * b.v); }
constexpr Fc operator/(Fc a, Fc b) { FC_COUNT(); return Fc(a.v / b.v); }
constexpr Fc operator-(Fc a) { return Fc(-a.v); }
constexpr Fc operator+(Fc a) { return a; }
constexpr bool operator<(Fc a, Fc b) { return a.v < b.v; }
constexpr bool operator>(Fc a, Fc b) { return a.v > b.v; }
constexpr bool operator<=(Fc a, Fc b) { return a.v <= b.v; }
constexpr bool operator>=(Fc a, Fc b) { return a.v >= b.v; }
constexpr bool operator==(Fc a, Fc b) { return a.v == b.v; }
constexpr bool operator!=(Fc a, Fc b) { return a.v != b.v; }
inline Fc sin(Fc a) { ++ops_counter(); return Fc(std::sin(a.v)); }
inline Fc cos(Fc a) { ++ops_counter(); return Fc(std::cos(a.v)); }
inline Fc sqrt(Fc a) { ++ops_counter(); return Fc(std::sqrt(a.v)); }
inline Fc log(Fc a) { ++ops_counter(); return Fc(std::log(a.v)); }
inline Fc atan2(Fc a, Fc b) { ++ops_counter(); return Fc(std::atan2(a.v, b.v)); }
inline Fc abs(Fc a) { return Fc(std::fabs(a.v)); }

#include "settings.h"
#include "constants.h"
#include "dynamics/integrator.cuh"

#include <cstdio>
#include <vector>

typedef Fc Tc;

static grid::robotModel<Tc>* model()
{
    static grid::robotModel<Tc>* m = grid::init_robotModel<Tc>();
    return m;
}

int main()
{
    const int nq = grid::NQ, nx = 2 * nq;
    std::vector<Tc> s(1 << 16);
    Tc xux[64], A[256], Bm[256], c[32], Q[256], qv[32], R[64], rv[16], goal[6];
    for (int i = 0; i < 64; ++i) xux[i] = 0.1 * ((i * 37) % 11 - 5);
    for (int i = 0; i < 6; ++i) goal[i] = 0.05 * (i + 1);
    const Tc dt = 0.01;
    model();

    ops_counter() = 0;
    gato::plant::compute_linearized_dynamics<Tc, 2, false, true>(xux, A, Bm, c, s.data(),
                                                                 model(), dt);
    const unsigned long long kkt_dyn = ops_counter();

    ops_counter() = 0;
    blockIdx.x = 0;
    gato::plant::trackingCostGradientAndHessian<Tc>(nx, nq, xux, goal, Q, qv, R, rv, s.data(),
                                                    model(), 2.0, 1e-4, 1e-6, 50.0, 1e-3, 1e-4,
                                                    1e-6);
    const unsigned long long kkt_cost = ops_counter();

    ops_counter() = 0;
    gato::plant::trackingcost<Tc>(nx, nq, KNOT_POINTS, xux, goal, s.data(), model(), 2.0, 1e-4,
                                  1e-6, 50.0, 1e-3, 1e-4, 1e-6);
    const unsigned long long merit_cost = ops_counter();

    ops_counter() = 0;
    gato::plant::compute_integrator_error<Tc, 2, false>(xux, xux + 3 * nq, s.data(), model(), dt);
    const unsigned long long merit_defect = ops_counter();

    std::printf("{\"nq\": %d, \"kkt_dynamics\": %llu, \"kkt_cost\": %llu, \"merit_cost\": %llu, "
                "\"merit_defect\": %llu}\n",
                nq, kkt_dyn, kkt_cost, merit_cost, merit_defect);
    return 0;
}
