// Device functions of the magnetic-field side shared by several translation units.
// FP64, reference-exact: include only from files compiled with -fmad=false.
#pragma once
#include "common.cuh"

namespace mhd
{
// uns::reconstruct_cell_vector (src/uns/geometry/Reconstruct.cpp:8-46): area-weighted least squares
// b . n_f = flux_f / A_f, the 3x3 normal matrix built and inverted per cell.
__device__ __forceinline__ V3 cell_vector(const MeshView &m, const double *__restrict__ flux, int32_t c)
{
    // the full (not symmetrised) matrix: its two triangles round differently and both enter det
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, r[3] = {0, 0, 0};
    for (int32_t k = m.c2f_ptr[c]; k < m.c2f_ptr[c + 1]; ++k)
    {
        const int32_t f = m.c2f_idx[k];
        const double A = m.face_area_mag[f];
        if (A <= 0) continue;
        const double s = m.c2f_sgn[k];
        const V3 n = (s / A) * ld3(m.face_area, f);
        const double nv[3] = {n.x, n.y, n.z};
        const double phi = s * flux[f];
        for (int i = 0; i < 3; ++i)
        {
            r[i] += nv[i] * phi;
            for (int j = 0; j < 3; ++j) M[i][j] += A * nv[i] * nv[j];
        }
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double sc = dmax(dmax(dmax(M[0][0], M[1][1]), M[2][2]), 1e-300);
    if (fabs(det) < 1e-12 * sc * sc * sc) return mk(0, 0, 0);
    double I[3][3];
    I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
    I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
    I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
    I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
    I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
    I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
    I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
    I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
    I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    return mk(I[0][0] * r[0] + I[0][1] * r[1] + I[0][2] * r[2], I[1][0] * r[0] + I[1][1] * r[1] + I[1][2] * r[2],
              I[2][0] * r[0] + I[2][1] * r[1] + I[2][2] * r[2]);
}

// (d1^T star2 phi)_e: the resistive current flux of ImplicitInduction::apply_F (ImplicitInduction.cpp:133-137)
// at edge e, its faces in ascending order (e2f rows), each term sgn * (star2_f phi_f)
__device__ __forceinline__ double resistive_p0(const MeshView &m, const double *__restrict__ phi, int32_t e)
{
    double p0 = 0.0;
    for (int32_t k = m.e2f_ptr[e]; k < m.e2f_ptr[e + 1]; ++k)
    {
        const int32_t f = m.e2f_idx[k];
        p0 += m.e2f_sgn[k] * (m.star2[f] * phi[f]);
    }
    return p0;
}
} // namespace mhd
