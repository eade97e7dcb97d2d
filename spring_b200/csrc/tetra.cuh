// Linear-tetrahedron helpers shared by the 3-phonon, isotope, iterative-BTE,
// 4-phonon and path-mode kernels.
//
// FindgAndIver (src/Kappa/Src/TetrahedronIntegration_m.f90:93-218): the
// weight g and vertex weights I of a tetrahedron whose sorted vertex energies
// are M[0..3], at the energy Mqs.  kappa.x takes the cases with >= / <= bounds;
// LineWidth.x (src/LineWidth/Src/TetrahedronIntegration_m.f90:113-169) and
// kappa_iter.x use strict bounds.  my_sort (:18-90) is a stable ascending sort
// of the four vertices (ties keep the original order).
#pragma once

namespace spring {
namespace tet {

// Stable ascending order of four keys: p[] receives original vertex indices.
static __device__ __forceinline__ void sort4(const double* M, int* p) {
    p[0] = 0; p[1] = 1; p[2] = 2; p[3] = 3;
#define SPRING_SWP(i, j)                                                                    \
    {                                                                                       \
        const double a_ = M[p[i]], b_ = M[p[j]];                                            \
        if (b_ < a_ || (b_ == a_ && p[j] < p[i])) { int t_ = p[i]; p[i] = p[j]; p[j] = t_; } \
    }
    SPRING_SWP(0, 1) SPRING_SWP(2, 3) SPRING_SWP(0, 2) SPRING_SWP(1, 3) SPRING_SWP(1, 2)
#undef SPRING_SWP
}

// FindgAndIver on already sorted energies M[0..3].
template <bool STRICT>
static __device__ __forceinline__ bool g_iver(double Mqs, const double* M, double& g, double* I) {
    bool c1, c2, c3;
    if (!STRICT) {
        c1 = (Mqs >= M[0]) && (Mqs < M[1]);
        c2 = (Mqs >= M[1]) && (Mqs < M[2]);
        c3 = (Mqs >= M[2]) && (Mqs <= M[3]);
    } else {
        c1 = (Mqs > M[0]) && (Mqs < M[1]);
        c2 = (Mqs > M[1]) && (Mqs < M[2]);
        c3 = (Mqs > M[2]) && (Mqs < M[3]);
    }
    if (c1) {
        g = (3.0 * ((Mqs - M[0]) * (Mqs - M[0]))) / ((M[1] - M[0]) * (M[2] - M[0]) * (M[3] - M[0]));
        I[0] = (((Mqs - M[1]) / (M[0] - M[1])) + ((Mqs - M[2]) / (M[0] - M[2])) + ((Mqs - M[3]) / (M[0] - M[3]))) / 3.0;
        for (int v = 1; v < 4; ++v) I[v] = ((Mqs - M[0]) / (M[v] - M[0])) / 3.0;
        return true;
    }
    if (c2) {
        g = (3.0 / ((M[1] - M[2]) * (M[3] - M[0]))) *
            ((((Mqs - M[0]) * (Mqs - M[2])) / (M[2] - M[0])) - (((Mqs - M[1]) * (Mqs - M[3])) / (M[1] - M[3])));
        const double den = g * (M[3] - M[0]);
        I[0] = (((Mqs - M[3]) / (M[0] - M[3])) / 3.0) +
               ((((Mqs - M[2]) / (M[0] - M[2])) * ((Mqs - M[0]) / (M[2] - M[0])) * ((Mqs - M[2]) / (M[1] - M[2]))) / den);
        const double t1 = (Mqs - M[3]) / (M[1] - M[3]);
        I[1] = (((Mqs - M[2]) / (M[1] - M[2])) / 3.0) + (((t1 * t1) * ((Mqs - M[1]) / (M[2] - M[1]))) / den);
        const double t2 = (Mqs - M[0]) / (M[2] - M[0]);
        I[2] = (((Mqs - M[1]) / (M[2] - M[1])) / 3.0) + (((t2 * t2) * ((Mqs - M[2]) / (M[1] - M[2]))) / den);
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) / 3.0) +
               ((((Mqs - M[1]) / (M[3] - M[1])) * ((Mqs - M[3]) / (M[1] - M[3])) * ((Mqs - M[1]) / (M[2] - M[1]))) / den);
        return true;
    }
    if (c3) {
        g = (3.0 * ((Mqs - M[3]) * (Mqs - M[3]))) / ((M[3] - M[0]) * (M[3] - M[1]) * (M[3] - M[2]));
        for (int v = 0; v < 3; ++v) I[v] = ((Mqs - M[3]) / (M[v] - M[3])) / 3.0;
        I[3] = (((Mqs - M[0]) / (M[3] - M[0])) + ((Mqs - M[1]) / (M[3] - M[1])) + ((Mqs - M[2]) / (M[3] - M[2]))) / 3.0;
        return true;
    }
    g = 0.0;
    I[0] = I[1] = I[2] = I[3] = 0.0;
    return false;
}

static __device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tet
}  // namespace spring
