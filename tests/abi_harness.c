/* abi_harness.c -- drives the C ABI of include/maille_gpu.h from C, the way a foreign-language
 * binding does (plain pointers and sizes, no Python): builds a Tet4 box of n x n x n cells (six
 * tetrahedra per cell, the cell split and orientation of the reference's bench mesh helper,
 * benches/common/mod.rs:13-53), then
 *   1. a linear static solve: z = 0 clamped, a downward load on every z = 1 node;
 *   2. a transient thermal step: T = 100 on z = 0, T = 0 at t = 0, 5 backward-Euler increments.
 * Prints one line per call: the status and a few results. Exit code 0 when every call returned
 * MAILLE_OK, or when no CUDA device is visible and every call said so (MAILLE_CUDA_ERROR);
 * 1 otherwise.
 *
 *   gcc -I include tests/abi_harness.c -L maille_b200 -lmaille_gpu -Wl,-rpath,$PWD/maille_b200
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "maille_gpu.h"

static int64_t node_id(int n, int i, int j, int k) { return i + (int64_t)(n + 1) * (j + (int64_t)(n + 1) * k); }

/* the six axis paths from (0,0,0) to (1,1,1) of a cell, in the helper's order */
static const int kPaths[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

static double signed_volume6(const double* x, const int64_t* t) {
    double a[3], b[3], c[3];
    for (int d = 0; d < 3; ++d) {
        a[d] = x[3 * t[1] + d] - x[3 * t[0] + d];
        b[d] = x[3 * t[2] + d] - x[3 * t[0] + d];
        c[d] = x[3 * t[3] + d] - x[3 * t[0] + d];
    }
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 4;
    const int64_t nn = (int64_t)(n + 1) * (n + 1) * (n + 1), ne = 6LL * n * n * n;
    double* coords = malloc(sizeof(double) * 3 * nn);
    int64_t* conn = malloc(sizeof(int64_t) * 4 * ne);
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                const int64_t v = node_id(n, i, j, k);
                coords[3 * v] = (double)i / n;
                coords[3 * v + 1] = (double)j / n;
                coords[3 * v + 2] = (double)k / n;
            }
    int64_t e = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int t = 0; t < 6; ++t, ++e) {
                    int p[3] = {i, j, k};
                    int64_t* tet = conn + 4 * e;
                    tet[0] = node_id(n, p[0], p[1], p[2]);
                    for (int s = 0; s < 3; ++s) {
                        p[kPaths[t][s]] += 1;
                        tet[s + 1] = node_id(n, p[0], p[1], p[2]);
                    }
                    if (signed_volume6(coords, tet) < 0.0) {
                        const int64_t tmp = tet[1];
                        tet[1] = tet[2];
                        tet[2] = tmp;
                    }
                }
    const int devices = maille_gpu_device_count();
    int ok = 1;

    /* 1. linear static */
    double* young = malloc(sizeof(double) * ne);
    double* poisson = malloc(sizeof(double) * ne);
    for (int64_t q = 0; q < ne; ++q) {
        young[q] = 210000.0;
        poisson[q] = 0.3;
    }
    uint8_t* fixed3 = calloc(3 * nn, 1);
    double* imposed3 = calloc(3 * nn, sizeof(double));
    double* f3 = calloc(3 * nn, sizeof(double));
    for (int64_t v = 0; v < nn; ++v) {
        if (coords[3 * v + 2] == 0.0) fixed3[3 * v] = fixed3[3 * v + 1] = fixed3[3 * v + 2] = 1;
        if (coords[3 * v + 2] == 1.0) f3[3 * v + 2] = -1.0;
    }
    MailleElasticProblem ep = {nn, coords, 4, ne, conn, young, poisson, fixed3, imposed3, f3,
                               1e-12, 10000, MAILLE_FP64, MAILLE_ORDER_AUTO, 0};
    double* u = calloc(3 * nn, sizeof(double));
    double* r = calloc(3 * nn, sizeof(double));
    MailleElasticResult er = {0};
    er.u = u;
    er.reactions = r;
    const int32_t s1 = maille_gpu_elastic_solve(&ep, &er);
    double umin = 0.0, rz = 0.0;
    for (int64_t v = 0; v < nn; ++v) {
        if (u[3 * v + 2] < umin) umin = u[3 * v + 2];
        rz += r[3 * v + 2];
    }
    printf("elastic status %d iterations %d min uz %.6e reaction z %.6e%s%s\n", s1, er.iterations, umin, rz,
           s1 ? " error: " : "", s1 ? maille_gpu_last_error() : "");

    /* 2. transient thermal */
    double* k = malloc(sizeof(double) * ne);
    double* rc = malloc(sizeof(double) * ne);
    for (int64_t q = 0; q < ne; ++q) {
        k[q] = 1.0;
        rc[q] = 1.0;
    }
    uint8_t* fixed = calloc(nn, 1);
    double* imposed = calloc(nn, sizeof(double));
    double* t0 = calloc(nn, sizeof(double));
    for (int64_t v = 0; v < nn; ++v)
        if (coords[3 * v + 2] == 0.0) {
            fixed[v] = 1;
            imposed[v] = 100.0;
        }
    const int32_t steps = 5;
    MailleThermalProblem tp = {nn, coords, 4, ne, conn, k, rc, fixed, imposed, NULL, 0, NULL, NULL, NULL, t0,
                               0.02, 1.0, steps, 1e-12, 10000, MAILLE_ORDER_AUTO, 0, MAILLE_FP64};
    double* temps = calloc((size_t)(steps + 1) * nn, sizeof(double));
    double* react = calloc((size_t)(steps + 1) * nn, sizeof(double));
    MailleThermalResult tr = {0};
    tr.temperatures = temps;
    tr.reactions = react;
    const int32_t s2 = maille_gpu_thermal_transient(&tp, &tr);
    double tmin = 1e300, tmax = -1e300, heat = 0.0;
    for (int64_t v = 0; v < nn; ++v) {
        const double t = temps[(size_t)steps * nn + v];
        if (t < tmin) tmin = t;
        if (t > tmax) tmax = t;
        heat += react[(size_t)steps * nn + v];
    }
    printf("thermal status %d iterations %lld final T in [%.6f, %.6f] heat in %.6e%s%s\n", s2,
           (long long)tr.iterations_total, tmin, tmax, heat, s2 ? " error: " : "", s2 ? maille_gpu_last_error() : "");

    if (devices > 0)
        ok = s1 == MAILLE_OK && s2 == MAILLE_OK && umin < 0.0 && fabs(rz - (double)((n + 1) * (n + 1))) < 1e-6 &&
             tmin > -1.0 && tmax < 101.0 && heat > 0.0; /* consistent capacity may undershoot a little */
    else
        ok = s1 == MAILLE_CUDA_ERROR && s2 == MAILLE_CUDA_ERROR;
    printf("devices %d -> %s\n", devices, ok ? "ok" : "FAILED");
    free(coords);
    free(conn);
    free(young);
    free(poisson);
    free(fixed3);
    free(imposed3);
    free(f3);
    free(u);
    free(r);
    free(k);
    free(rc);
    free(fixed);
    free(imposed);
    free(t0);
    free(temps);
    free(react);
    return ok ? 0 : 1;
}
