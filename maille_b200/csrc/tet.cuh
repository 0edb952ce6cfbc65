// tet.cuh -- Tet4 / Tet10 geometry on the device, shared by the element kernels (kernels.cu,
// thermal.cu): shape values and derivatives at a barycentric point (shape.rs:95-153) and the
// Jacobian with its determinant and inverse (Mapping3d::new, shape.rs:164-190).
#pragma once

#include <cuda_runtime.h>

namespace maille {

// dN/dxi of Tet4 (constant) or Tet10 at barycentric l (shape.rs:95-153).
template <int NPE>
__host__ __device__ __forceinline__ void dshape(const double* l, int a, double d[3]) {
    const double dl[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
    if (NPE == 4) {
        d[0] = dl[a][0];
        d[1] = dl[a][1];
        d[2] = dl[a][2];
    } else if (a < 4) {
        const double f = 4.0 * l[a] - 1.0;
        d[0] = f * dl[a][0];
        d[1] = f * dl[a][1];
        d[2] = f * dl[a][2];
    } else {
        const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
        const int p = E[a - 4][0], q = E[a - 4][1];
#pragma unroll
        for (int c = 0; c < 3; ++c) d[c] = 4.0 * (l[p] * dl[q][c] + l[q] * dl[p][c]);
    }
}

template <int NPE>
__host__ __device__ __forceinline__ double shape_value(const double* l, int a) {
    if (NPE == 4) return l[a];
    if (a < 4) return l[a] * (2.0 * l[a] - 1.0);
    const int E[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
    return 4.0 * l[E[a - 4][0]] * l[E[a - 4][1]];
}

// Jacobian J[i][r] = sum_k dN_k/dxi_i x_k[r], determinant by cofactors and J^-1 (Mapping3d::new,
// shape.rs:164-190).
template <int NPE>
__host__ __device__ __forceinline__ double jacobian(const double (*xyz)[3], const double* l, double inv[9]) {
    double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int k = 0; k < NPE; ++k) {
        double d[3];
        dshape<NPE>(l, k, d);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int r = 0; r < 3; ++r) j[i][r] += d[i] * xyz[k][r];
    }
    auto cof = [&](int r, int c) {
        const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        return j[r1][c1] * j[r2][c2] - j[r1][c2] * j[r2][c1];
    };
    const double det = j[0][0] * cof(0, 0) + j[0][1] * cof(0, 1) + j[0][2] * cof(0, 2);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) inv[3 * r + c] = cof(c, r) / det;
    return det;
}

}  // namespace maille
