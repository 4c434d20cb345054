/*
 * nbody_oracle.c -- CPU oracle for the N-body step (the sibling pair sum of KTT's Nbody example).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls this file; the tests
 * use it as the checker of coul_nbody_step.
 *
 * What it restates (KTT 2.1.0): Examples/Nbody/NbodyReference.cu:36-75 (and the tuned
 * Examples/Nbody/Nbody.cu:103-145, 365-408): for every body i,
 *     a_i = sum_j m_j (p_j - p_i) * invr^3,  invr = 1 / sqrt(|p_j - p_i|^2 + softeningSqr)
 * over all j including j = i (whose difference is zero), then
 *     p_i' = p_i + dt v_i + damping dt^2 a_i,   v_i' = v_i + dt a_i,
 * the mass kept in the position's fourth component and 0 in the velocity's.  Here in FP64 (the FP32
 * inputs widened), for all bodies or for a selected subset of bodies i (the j sum is always complete),
 * parallel over i with OpenMP.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#define ORACLE_API __attribute__((visibility("default")))

ORACLE_API int oracle_nbody_step(const float* pos4, const float* vel4, int64_t n, float dt, float damping, float eps2,
                                 const int64_t* idx, int64_t nidx, double* pos_out4, double* vel_out4, double* acc_out3)
{
    if (n < 0 || pos4 == NULL || vel4 == NULL)
        return 1;
    const int64_t count = idx ? nidx : n;
    const double h = (double)dt, d = (double)damping, e2 = (double)eps2;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t k = 0; k < count; ++k) {
        const int64_t i = idx ? idx[k] : k;
        const double px = pos4[4 * i], py = pos4[4 * i + 1], pz = pos4[4 * i + 2];
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double dx = (double)pos4[4 * j] - px;
            const double dy = (double)pos4[4 * j + 1] - py;
            const double dz = (double)pos4[4 * j + 2] - pz;
            const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz + e2);
            const double f = (double)pos4[4 * j + 3] * inv * inv * inv;
            ax += f * dx;
            ay += f * dy;
            az += f * dz;
        }
        const double vx = vel4[4 * i], vy = vel4[4 * i + 1], vz = vel4[4 * i + 2];
        if (acc_out3) {
            acc_out3[3 * k] = ax;
            acc_out3[3 * k + 1] = ay;
            acc_out3[3 * k + 2] = az;
        }
        if (pos_out4) {
            pos_out4[4 * k] = px + h * vx + d * h * h * ax;
            pos_out4[4 * k + 1] = py + h * vy + d * h * h * ay;
            pos_out4[4 * k + 2] = pz + h * vz + d * h * h * az;
            pos_out4[4 * k + 3] = pos4[4 * i + 3];
        }
        if (vel_out4) {
            vel_out4[4 * k] = vx + h * ax;
            vel_out4[4 * k + 1] = vy + h * ay;
            vel_out4[4 * k + 2] = vz + h * az;
            vel_out4[4 * k + 3] = 0.0;
        }
    }
    return 0;
}
