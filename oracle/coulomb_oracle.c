/*
 * coulomb_oracle.c -- CPU oracle for the direct Coulomb summation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libcoulktt / ktt_b200)
 * links, loads or calls this file.  It is used by the test-suite as the
 * checker, by __graft_entry__.smoke() as the checker, and by bench.py as the
 * timed CPU baseline ("port" of KTT's reference computation).
 *
 * What it restates (file:line refer to the KTT 2.1.0 source tree):
 *   - Examples/CoulombSum3d/CoulombSum3dReference.cu:11-26 : one grid point
 *     per work item, coordinate = gridSpacing * index, x-fastest layout
 *     out[(z*G + y)*G + x], V = sum_j w_j * rsqrt(dx^2 + dy^2 + dz^2).
 *   - Examples/CoulombSum2d/CoulombSum2dReference.cl:8-20 : 2D slice where the
 *     atom's .z field already holds the squared z distance (dz^2), and the
 *     output is assigned (=), not accumulated.
 *   - Examples/JSON/generate-coulomb-output.c:22-31 : the CPU generator of the
 *     known-answer file Coulomb3d.bin (FP32, q / sqrtf(r^2)); restated in
 *     coulomb_oracle_fp32.c so it can be compiled with its own flags.
 *
 * Everything here is FP64: the FP32 inputs are widened to double, grid
 * coordinates are first formed in FP32 exactly as the GPU path forms them
 * (fmaf(index, h, origin), a single rounding; for origin 0 this equals KTT's
 * gridSpacing * index), then widened.  1/sqrt is computed as 1.0/sqrt(r2) in
 * double.  A grid point that coincides with an atom (r2 == 0) contributes
 * +inf/nan exactly like the reference kernels; the tests avoid such inputs.
 *
 * Adjoint (no counterpart in KTT; FP64 definition of the gradient the GPU
 * adjoint computes): L = 0.5 * sum_i w_i (V_i - T_i)^2,
 *   dL/dq_j = sum_i w_i res_i / r_ij,
 *   dL/dr_j = q_j * sum_i w_i res_i (r_i - r_j) / r_ij^3 .
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_API __attribute__((visibility("default")))

typedef struct {
    double* x;
    double* y;
    double* z;
    double* q;
    int64_t n;
} atoms_soa;

static int atoms_from_xyzq(const float* xyzq, int64_t n, atoms_soa* a)
{
    a->n = n;
    a->x = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    a->y = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    a->z = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    a->q = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (!a->x || !a->y || !a->z || !a->q)
        return -1;
    for (int64_t j = 0; j < n; ++j) {
        a->x[j] = (double)xyzq[4 * j + 0];
        a->y[j] = (double)xyzq[4 * j + 1];
        a->z[j] = (double)xyzq[4 * j + 2];
        a->q[j] = (double)xyzq[4 * j + 3];
    }
    return 0;
}

static void atoms_free(atoms_soa* a)
{
    free(a->x);
    free(a->y);
    free(a->z);
    free(a->q);
}

/* Grid coordinate exactly as the GPU path forms it: one FP32 fma. */
static inline double grid_coord(int64_t index, float h, float origin)
{
    return (double)fmaf((float)index, h, origin);
}

ORACLE_API int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

ORACLE_API void oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Potential and conditioning sum at one point. */
static inline void point_sum(const atoms_soa* a, double px, double py, double pz, double* v, double* sabs)
{
    double acc = 0.0, accabs = 0.0;
#pragma omp simd reduction(+ : acc, accabs)
    for (int64_t j = 0; j < a->n; ++j) {
        const double dx = px - a->x[j];
        const double dy = py - a->y[j];
        const double dz = pz - a->z[j];
        const double inv = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        acc += a->q[j] * inv;
        accabs += fabs(a->q[j]) * inv;
    }
    *v = acc;
    if (sabs)
        *sabs = accabs;
}

/*
 * Full 3D map, FP64.  atoms: n x float4 (x, y, z, q).  out: nx*ny*nz doubles,
 * x fastest.  origin may be NULL (= 0,0,0, KTT convention).
 */
ORACLE_API int oracle_grid3d(const float* xyzq, int64_t n, float h, const float* origin, int nx, int ny, int nz,
                             double* out)
{
    atoms_soa a;
    if (nx < 0 || ny < 0 || nz < 0 || n < 0)
        return -1;
    if (atoms_from_xyzq(xyzq, n, &a))
        return -2;
    const float ox = origin ? origin[0] : 0.0f, oy = origin ? origin[1] : 0.0f, oz = origin ? origin[2] : 0.0f;
    const int64_t rows = (int64_t)ny * nz;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t r = 0; r < rows; ++r) {
        const int64_t z = r / ny, y = r % ny;
        const double py = grid_coord(y, h, oy), pz = grid_coord(z, h, oz);
        for (int64_t x = 0; x < nx; ++x) {
            double v;
            point_sum(&a, grid_coord(x, h, ox), py, pz, &v, NULL);
            out[r * nx + x] = v;
        }
    }
    atoms_free(&a);
    return 0;
}

/*
 * Selected points of a 3D map, FP64.  idx: linear indices (x fastest) into the
 * nx*ny*nz grid.  sumabs (optional) receives sum_j |q_j| / r_ij, the
 * condition number of the sum at that point (used for the cancellation-aware
 * error report).
 */
ORACLE_API int oracle_points3d(const float* xyzq, int64_t n, float h, const float* origin, int nx, int ny, int nz,
                               const int64_t* idx, int64_t npts, double* out, double* sumabs)
{
    atoms_soa a;
    if (atoms_from_xyzq(xyzq, n, &a))
        return -2;
    const float ox = origin ? origin[0] : 0.0f, oy = origin ? origin[1] : 0.0f, oz = origin ? origin[2] : 0.0f;
    const int64_t total = (int64_t)nx * ny * nz;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (int64_t p = 0; p < npts; ++p) {
        const int64_t li = idx[p];
        if (li < 0 || li >= total) {
            bad |= 1;
            continue;
        }
        const int64_t x = li % nx, y = (li / nx) % ny, z = li / ((int64_t)nx * ny);
        point_sum(&a, grid_coord(x, h, ox), grid_coord(y, h, oy), grid_coord(z, h, oz), &out[p],
                  sumabs ? &sumabs[p] : NULL);
    }
    atoms_free(&a);
    return bad ? -3 : 0;
}

/*
 * 2D slice with KTT's 2D argument convention: atoms n x float4 (x, y, dz2, q)
 * where dz2 is the precomputed squared z distance of the atom to the slice
 * (CoulombSum2dReference.cl:16).  out[y*nx + x] = sum_j q_j / sqrt(dx^2 + dy^2 + dz2_j).
 */
ORACLE_API int oracle_slice2d(const float* xyc_q, int64_t n, float h, int nx, int ny, double* out)
{
    atoms_soa a;
    if (atoms_from_xyzq(xyc_q, n, &a))
        return -2;
#pragma omp parallel for schedule(dynamic, 2)
    for (int64_t y = 0; y < ny; ++y) {
        const double py = grid_coord(y, h, 0.0f);
        for (int64_t x = 0; x < nx; ++x) {
            const double px = grid_coord(x, h, 0.0f);
            double acc = 0.0;
#pragma omp simd reduction(+ : acc)
            for (int64_t j = 0; j < a.n; ++j) {
                const double dx = px - a.x[j];
                const double dy = py - a.y[j];
                acc += a.q[j] / sqrt(dx * dx + dy * dy + a.z[j]);
            }
            out[y * nx + x] = acc;
        }
    }
    atoms_free(&a);
    return 0;
}

/*
 * FP64 adjoint of L = 0.5 * sum_i w_i (V_i - T_i)^2 on an nx*ny*nz grid.
 * V is recomputed here in FP64 from the atoms.  Outputs (any may be NULL):
 *   loss   : L
 *   dq[j]  : dL/dq_j                 for the atoms listed in sel (or all if sel==NULL)
 *   dr[3j] : dL/d(x_j, y_j, z_j)     same selection
 * nsel = number of selected atoms; outputs are indexed by selection order.
 * vout (optional): the FP64 map V.
 */
ORACLE_API int oracle_adjoint3d(const float* xyzq, int64_t n, float h, const float* origin, int nx, int ny, int nz,
                                const float* weight, const float* target, const int64_t* sel, int64_t nsel,
                                double* loss, double* dq, double* dr, double* vout)
{
    atoms_soa a;
    if (atoms_from_xyzq(xyzq, n, &a))
        return -2;
    const float ox = origin ? origin[0] : 0.0f, oy = origin ? origin[1] : 0.0f, oz = origin ? origin[2] : 0.0f;
    const int64_t total = (int64_t)nx * ny * nz;
    double* res = (double*)malloc(sizeof(double) * (size_t)(total > 0 ? total : 1));
    if (!res) {
        atoms_free(&a);
        return -2;
    }
    double lsum = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : lsum)
    for (int64_t li = 0; li < total; ++li) {
        const int64_t x = li % nx, y = (li / nx) % ny, z = li / ((int64_t)nx * ny);
        double v;
        point_sum(&a, grid_coord(x, h, ox), grid_coord(y, h, oy), grid_coord(z, h, oz), &v, NULL);
        if (vout)
            vout[li] = v;
        const double w = weight ? (double)weight[li] : 1.0;
        const double r = v - (double)target[li];
        res[li] = w * r;
        lsum += 0.5 * w * r * r;
    }
    if (loss)
        *loss = lsum;
    const int64_t m = sel ? nsel : n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t s = 0; s < m; ++s) {
        const int64_t j = sel ? sel[s] : s;
        if (j < 0 || j >= n)
            continue;
        double gq = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
        for (int64_t z = 0; z < nz; ++z) {
            const double pz = grid_coord(z, h, oz) - a.z[j];
            for (int64_t y = 0; y < ny; ++y) {
                const double py = grid_coord(y, h, oy) - a.y[j];
                const double* rr = res + (z * ny + y) * nx;
#pragma omp simd reduction(+ : gq, gx, gy, gz)
                for (int64_t x = 0; x < nx; ++x) {
                    const double px = grid_coord(x, h, ox) - a.x[j];
                    const double inv = 1.0 / sqrt(px * px + py * py + pz * pz);
                    const double t = rr[x] * inv;
                    const double t3 = t * inv * inv;
                    gq += t;
                    gx += t3 * px;
                    gy += t3 * py;
                    gz += t3 * pz;
                }
            }
        }
        if (dq)
            dq[s] = gq;
        if (dr) {
            dr[3 * s + 0] = a.q[j] * gx;
            dr[3 * s + 1] = a.q[j] * gy;
            dr[3 * s + 2] = a.q[j] * gz;
        }
    }
    free(res);
    atoms_free(&a);
    return 0;
}

/*
 * FP64 change of the loss when one atom moves or changes charge, given the
 * FP64 map V of the unperturbed system: used for central finite differences
 * of L without recomputing the whole map.  new_xyzq is the perturbed atom j.
 */
ORACLE_API int oracle_loss_perturbed(const float* xyzq, int64_t n, int64_t j, const double* new_xyzq, float h,
                                     const float* origin, int nx, int ny, int nz, const float* weight,
                                     const float* target, const double* v, double* loss)
{
    if (j < 0 || j >= n)
        return -1;
    const float ox = origin ? origin[0] : 0.0f, oy = origin ? origin[1] : 0.0f, oz = origin ? origin[2] : 0.0f;
    const double ax = xyzq[4 * j], ay = xyzq[4 * j + 1], az = xyzq[4 * j + 2], aq = xyzq[4 * j + 3];
    const double bx = new_xyzq[0], by = new_xyzq[1], bz = new_xyzq[2], bq = new_xyzq[3];
    const int64_t total = (int64_t)nx * ny * nz;
    double lsum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : lsum)
    for (int64_t li = 0; li < total; ++li) {
        const int64_t x = li % nx, y = (li / nx) % ny, z = li / ((int64_t)nx * ny);
        const double px = grid_coord(x, h, ox), py = grid_coord(y, h, oy), pz = grid_coord(z, h, oz);
        const double d0x = px - ax, d0y = py - ay, d0z = pz - az;
        const double d1x = px - bx, d1y = py - by, d1z = pz - bz;
        const double vnew = v[li] - aq / sqrt(d0x * d0x + d0y * d0y + d0z * d0z) +
                            bq / sqrt(d1x * d1x + d1y * d1y + d1z * d1z);
        const double w = weight ? (double)weight[li] : 1.0;
        const double r = vnew - (double)target[li];
        lsum += 0.5 * w * r * r;
    }
    *loss = lsum;
    return 0;
}
