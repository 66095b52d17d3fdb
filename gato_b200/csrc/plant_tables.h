/*
 * Built-in robot descriptions, transcribed from the URDFs the reference's
 * GRiD dynamics were generated from.  Data only.
 *
 *   iiwa14: examples/iiwa_description/iiwa14.urdf, joints A1..A7 (lines 70-292),
 *           links L1..L7 (lines 90-304), fixed child `contact` merged into L7
 *           (joint EE lines 322-328, link lines 333-337).  Limits as in
 *           gato/dynamics/iiwa14/iiwa14_plant.cuh:37-70.
 *   indy7:  examples/indy7_description/indy7.urdf, joints joint0..joint5
 *           (lines 208-248), links link1..link6 (lines 70-187).  Limits as in
 *           gato/dynamics/indy7/indy7_plant.cuh:66-96.
 *
 * Included by the CUDA library and by the FP64 oracle.
 */
#ifndef GATO_PLANT_TABLES_H
#define GATO_PLANT_TABLES_H

#include <string.h>
#include "../../include/gato_b200.h"

static inline void gato_plant_clear(gato_model_t* m)
{
    memset(m, 0, sizeof(*m));
    m->limit_margin = -0.1;
    m->gravity = 9.81;
}

static inline void gato_plant_iiwa14(gato_model_t* m)
{
    static const double xyz[7][3] = {
        {0.0, 0.0, 0.1575}, {0.0, 0.0, 0.2025}, {0.2045, 0.0, 0.0},
        {0.0, 0.0, 0.2155}, {0.0, 0.1845, 0.0}, {0.0, -0.0607, 0.2155},
        {0.081, 0.0, 0.0607}};
    static const double rpy[7][3] = {
        {0.0, 0.0, 0.0},
        {2.3561944901923457, -1.5707962635746238, 2.3561944901923457},
        {1.5707963267948948, -4.371139000186238e-8, 1.5707963705062866},
        {1.5707963705062866, -0.0, 0.0},
        {-1.5707963705062866, 0.0, -0.0},
        {2.3561944901923457, -1.5707962635746238, 2.3561944901923457},
        {1.5707963267948948, -4.371139000186238e-8, 1.5707963705062866}};
    /* mass, com xyz, ixx ixy ixz iyy iyz izz */
    static const double body[7][10] = {
        {3.94781, 0.0, 0.0, 0.0, 0.00455, 0.0, -0.0, 0.00454, -0.00001, 0.00029},
        {4.50275, 0.0003, 0.059, 0.042, 0.00032, 0.0, 0.0, 0.00010, 0.0, 0.00042},
        {2.45520, 0.0, 0.03, 0.13, 0.00223, -0.00005, 0.00007, 0.00219, 0.00007, 0.00073},
        {2.61155, 0.0, 0.067, 0.034, 0.03844, 0.00088, -0.00112, 0.01144, -0.00111, 0.04958},
        {3.41000, 0.0001, 0.021, 0.076, 0.00277, -0.00001, 0.00001, 0.00284, 0.0, 0.00012},
        {3.38795, 0.0, 0.0006, 0.0004, 0.00050, -0.00005, -0.00003, 0.00281, -0.00004, 0.00232},
        {0.35432, 0.0, 0.0, 0.02, 0.00795, 0.00022, -0.00029, 0.01083, -0.00029, 0.00294}};
    /* fixed link `contact`, 0.04 m along L7's z axis */
    static const double contact[10] = {0.057, 0.0, 0.0, 0.04, 0.0000354, 0.0, 0.0, 0.0000354, 0.0, 0.0000354};
    static const double qlim[7] = {2.96706, 2.09440, 2.96706, 2.09440, 2.96706, 2.09440, 3.05433};
    static const double vlim[7] = {1.48353, 1.48353, 1.74533, 1.30900, 2.26893, 2.35619, 2.35619};
    static const double ulim[7] = {320.0, 320.0, 176.0, 176.0, 110.0, 40.0, 40.0};
    gato_plant_clear(m);
    m->nq = 7;
    for (int i = 0; i < 7; ++i) {
        for (int k = 0; k < 3; ++k) {
            m->joint_xyz[i][k] = xyz[i][k];
            m->joint_rpy[i][k] = rpy[i][k];
        }
        for (int k = 0; k < 10; ++k) m->link_inertial[i][0][k] = body[i][k];
        m->q_limit[i] = qlim[i];
        m->qd_limit[i] = vlim[i];
        m->u_limit[i] = ulim[i];
    }
    for (int k = 0; k < 10; ++k) m->link_inertial[6][1][k] = contact[k];
    m->barrier_style = 0;
}

static inline void gato_plant_indy7(gato_model_t* m)
{
    static const double xyz[6][3] = {
        {0.0, 0.0, 0.0775}, {0.0, -0.109, 0.222}, {-0.45, 0.0, -0.0305},
        {-0.267, 0.0, -0.075}, {0.0, -0.114, 0.083}, {-0.168, 0.0, 0.069}};
    static const double rpy[6][3] = {
        {0.0, 0.0, 0.0}, {1.570796327, 1.570796327, 0.0}, {0.0, 0.0, 0.0},
        {-1.570796327, 0.0, 1.570796327}, {1.570796327, 1.570796327, 0.0},
        {-1.570796327, 0.0, 1.570796327}};
    /* The reference's indy7 dynamics place each link's centre of mass at the
       link origin and use the URDF inertia about that origin: its spatial
       inertias (indy7_grid.cuh, init_XImats blocks I[0..5]) carry no
       mass-offset terms, so the URDF <inertial><origin> offsets (e.g.
       -0.00023749 -0.04310313 0.13245396 for link1) do not enter.  The com
       columns below are therefore zero, which reproduces the reference. */
    static const double body[6][10] = {
        {11.44444535, 0.0, 0.0, 0.0, 0.35065005, 0.00011931, -0.00037553, 0.304798, -0.10984447, 0.06003147},
        {5.84766553, 0.0, 0.0, 0.0, 0.03599743, -4.693e-05, -0.05240346, 0.72293306, 1.76e-06, 0.70024119},
        {2.68206064, 0.0, 0.0, 0.0, 0.0161721, -0.00011817, 0.03341882, 0.11364055, -4.371e-05, 0.10022522},
        {2.12987371, 0.0, 0.0, 0.0, 0.02798891, 3.893e-05, -4.768e-05, 0.01443076, -0.01266296, 0.01496211},
        {2.22412271, 0.0, 0.0, 0.0, 0.01105297, 5.517e-05, -0.01481977, 0.03698291, -3.74e-05, 0.02754795},
        {0.38254932, 0.0, 0.0, 0.0, 0.00078982, -3.4e-07, 8.3e-07, 0.00079764, -5.08e-06, 0.00058319}};
    static const double qlim[6] = {3.0543, 3.0543, 3.0543, 3.0543, 3.0543, 3.7520};
    static const double vlim[6] = {2.61, 2.61, 2.61, 3.14, 3.14, 3.14};
    static const double ulim[6] = {431.97, 431.97, 197.23, 79.79, 79.79, 79.79};
    gato_plant_clear(m);
    m->nq = 6;
    for (int i = 0; i < 6; ++i) {
        for (int k = 0; k < 3; ++k) {
            m->joint_xyz[i][k] = xyz[i][k];
            m->joint_rpy[i][k] = rpy[i][k];
        }
        for (int k = 0; k < 10; ++k) m->link_inertial[i][0][k] = body[i][k];
        m->q_limit[i] = qlim[i];
        m->qd_limit[i] = vlim[i];
        m->u_limit[i] = ulim[i];
    }
    m->barrier_style = 1;
}

static inline int gato_plant_fill(int plant, gato_model_t* m)
{
    if (plant == GATO_PLANT_IIWA14) { gato_plant_iiwa14(m); return 0; }
    if (plant == GATO_PLANT_INDY7) { gato_plant_indy7(m); return 0; }
    return -1;
}

#endif /* GATO_PLANT_TABLES_H */
