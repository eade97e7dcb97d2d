// LineWidth.x path mode on the device (src/LineWidth/Src).
//
//  - Path points: q_points_highsymm (CreateMesh_mod.f90:85-172), on the host.
//  - For every path point q0 and grid point q1: q2 = G - (q0 + q1) with the
//    first G of (0,1,-1,2,-2)^3 (first component fastest) whose fractional
//    coordinates x (G x = q2, LU-factored G) lie in [-1/2, 1/2]^3 on
//    zero-centred segments or [0, 1]^3 otherwise (ScatterProbAllq1,
//    Linewidth_m.f90:48-231; CheckIfWithinBZ :458-497).
//  - Phonons at every q2 (get_phonon_singleq, DynaMat_mod.f90:712-892) with the
//    batched device eigensolver.
//  - V3 -> W for every (path point, q1): ScatterMatEl / ScatterProbability
//    (Linewidth_m.f90:500-660), W = |Phi|^2 / (w0 w1 w2 Nq) * Sctr3THz2, zero
//    below mode 4 where q0, q1 or q2 is Gamma (|q| < 5e-5, integer q1 == 0).
//    Phi uses the same basis-block regrouping as the grid kernels.
//  - Linewidth: CalculateLwTetrahedron (Linewidth_m.f90:326-417, strict case
//    bounds, q2 phonons read per vertex q1) through the shared tetrahedron
//    kernel, or the Gaussian CalculateLinewidth (:234-323) with its branch start
//    reset for every q1.
// Roofline: FP64 FMA (V3, ~42 kflop per (path point, q1) for the 2-atom cell)
// plus Nq 6x6 eigensolves per path point; the delta sums are FP64 ALU.
#include <algorithm>
#include <cmath>
#include <vector>

#include "spring_internal.cuh"

namespace spring {
namespace {

constexpr double ZERO_PREC = 5.0e-5;  // zero_prec, src/LineWidth/Src/constants.f90:36

struct PathQ2Args {
    int nq, n0, n1, n2;
    int p_first;
    double ru[9];     // G(r, c) / mesh(c) at [r * 3 + c]
    double shift[3];  // mesh shift / 2
    double G[9];      // G(r, c) at [r * 3 + c]
    double lu[9];     // LU factors of G (unit lower L below the diagonal, U on and above) at [r * 3 + c]
    int piv[3];       // row interchanges, 0-based
};

// dgetrs('N') on the 3x3 factors: row interchanges, unit-lower then upper
// triangular solves in the column order of the reference BLAS dtrsm, no
// contracted multiply-adds.
__device__ __forceinline__ void lu_solve3(const PathQ2Args& a, double* x) {
    for (int i = 0; i < 3; ++i) {
        const int ip = a.piv[i];
        if (ip != i) {
            const double t = x[i];
            x[i] = x[ip];
            x[ip] = t;
        }
    }
    for (int k = 0; k < 3; ++k)
        if (x[k] != 0.0)
            for (int i = k + 1; i < 3; ++i) x[i] = __dsub_rn(x[i], __dmul_rn(x[k], a.lu[i * 3 + k]));
    for (int k = 2; k >= 0; --k)
        if (x[k] != 0.0) {
            x[k] = __ddiv_rn(x[k], a.lu[k * 3 + k]);
            for (int i = 0; i < k; ++i) x[i] = __dsub_rn(x[i], __dmul_rn(x[k], a.lu[i * 3 + k]));
        }
}

// One thread per (slot, q1): the q1 vector of the segment's mesh, q2 and whether it was found.
__global__ void k_path_q2(PathQ2Args a, int n_slots, const double* __restrict__ q0v, const int* __restrict__ zc,
                          const double* __restrict__ qpnt_zc, double* __restrict__ q1v, double* __restrict__ q2v,
                          int* __restrict__ exists) {
    const int sgn[5] = {0, 1, -1, 2, -2};
    const long long total = (long long)n_slots * a.nq;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int slot = (int)(i / a.nq), g = (int)(i % a.nq);
        const int p = a.p_first + slot;
        const bool zero_c = zc[p] != 0;
        double q1[3];
        if (zero_c) {
            for (int r = 0; r < 3; ++r) q1[r] = qpnt_zc[3 * g + r];
        } else {  // make_tetrahedron(..., .false.): integer coordinates in [0, N)
            const int v[3] = {g % a.n0, (g / a.n0) % a.n1, g / (a.n0 * a.n1)};
            for (int r = 0; r < 3; ++r) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s = __dadd_rn(s, __dmul_rn(a.ru[r * 3 + k], (double)v[k] + a.shift[k]));
                q1[r] = s;
            }
        }
        const double* q0 = q0v + 3 * p;
        double q2[3] = {0.0, 0.0, 0.0};
        bool found = false;
        for (int c3 = 0; c3 < 5 && !found; ++c3)
            for (int c2 = 0; c2 < 5 && !found; ++c2)
                for (int c1 = 0; c1 < 5 && !found; ++c1) {
                    const double idx[3] = {(double)sgn[c1], (double)sgn[c2], (double)sgn[c3]};
                    double x[3], t[3];
                    for (int r = 0; r < 3; ++r) {
                        const double gv = __dadd_rn(__dadd_rn(__dmul_rn(a.G[r * 3], idx[0]), __dmul_rn(a.G[r * 3 + 1], idx[1])),
                                                    __dmul_rn(a.G[r * 3 + 2], idx[2]));
                        t[r] = __dsub_rn(gv, __dadd_rn(q0[r], q1[r]));
                        x[r] = t[r];
                    }
                    lu_solve3(a, x);
                    bool in;
                    if (zero_c)
                        in = fabs(x[0]) <= 0.5 && fabs(x[1]) <= 0.5 && fabs(x[2]) <= 0.5;
                    else
                        in = x[0] >= 0.0 && x[1] >= 0.0 && x[2] >= 0.0 && x[0] <= 1.0 && x[1] <= 1.0 && x[2] <= 1.0;
                    if (in) {
                        found = true;
                        q2[0] = t[0]; q2[1] = t[1]; q2[2] = t[2];
                    }
                }
        for (int r = 0; r < 3; ++r) {
            q1v[3 * i + r] = q1[r];
            q2v[3 * i + r] = q2[r];
        }
        exists[i] = found ? 1 : 0;
    }
}

// Rows whose q2 was not found keep zero frequencies and occupations (the reference's
// omegaq2All / nBEq2All stay at their zero initialisation).
__global__ void k_path_clear_missing(long long rows, int n, int nT, const int* __restrict__ exists,
                                     double* __restrict__ om2, double* __restrict__ nbe2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows * n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / n;
        if (exists[r]) continue;
        om2[i] = 0.0;
        for (int t = 0; t < nT; ++t) nbe2[(size_t)t * rows * n + i] = 0.0;
    }
}

struct V3PArgs {
    int nb, n, na, nq, sb, nsb;
    int p_first;
    double nqd, sctr;
};

__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

// One CTA per (q1 and s0 block, slot): Phi regrouped as in the grid kernels, then W.
__global__ void __launch_bounds__(128) k_v3_path(V3PArgs a, const int* __restrict__ exists, const double* __restrict__ q0v,
                                                 const double* __restrict__ q1v, const double* __restrict__ q2v,
                                                 const int* __restrict__ qint, const double* __restrict__ fc3,
                                                 const double* __restrict__ posr, const int* __restrict__ btyp,
                                                 const double* __restrict__ mrs, const double2* __restrict__ ev0,
                                                 const double* __restrict__ om0, const double2* __restrict__ evg,
                                                 const double* __restrict__ omg, const double2* __restrict__ ev2,
                                                 const double* __restrict__ om2, double* __restrict__ out_w) {
    extern __shared__ double2 smem2[];
    const int n = a.n, na = a.na, nn = n * n, sb = a.sb;
    double2* sE0 = smem2;
    double2* sE1 = sE0 + nn;
    double2* sE2 = sE1 + nn;
    double2* sD = sE2 + nn;
    double2* sT1 = sD + 3 * nn;
    double2* sT2 = sT1 + 3 * nn;
    double2* sPhi = sT2 + 3 * nn;
    double2* sPP = sPhi + sb * nn;
    double2* sP = sPP + na * na;
    double* sFC = reinterpret_cast<double*>(sP + 2 * na);
    int* sBt = reinterpret_cast<int*>(sFC + ((na * na * 27 + 1) & ~1));

    const int tid = threadIdx.x, nt = blockDim.x;
    const int q1 = blockIdx.x / a.nsb;
    const int s0b = (blockIdx.x % a.nsb) * sb;
    const int slot = blockIdx.y;
    const int p = a.p_first + slot;
    const size_t row = (size_t)slot * a.nq + q1;
    const int nphi = min(sb, n - s0b) * nn;
    const size_t n3 = (size_t)n * nn;
    double* W = out_w + row * n3;
    if (!exists[row]) return;  // W stays zero

    const double* q1p = q1v + 3 * row;
    const double* q2p = q2v + 3 * row;
    for (int i = tid; i < nn; i += nt) {
        sE0[i] = ev0[(size_t)p * nn + i];
        sE1[i] = evg[(size_t)q1 * nn + i];
        sE2[(i % n) * n + i / n] = ev2[row * nn + i];  // [row][s]: read along s2 below
    }
    for (int i = tid; i < nphi; i += nt) sPhi[i] = make_double2(0.0, 0.0);

    for (int mu = 0; mu < a.nb; ++mu) {
        const double* f = fc3 + (size_t)mu * na * na * 27;
        for (int i = tid; i < na * na * 27; i += nt) sFC[i] = f[i];
        for (int i = tid; i < na; i += nt) sBt[i] = btyp[mu * na + i];
        for (int i = tid; i < 2 * na; i += nt) {
            const int N = i % na;
            const double* qv = i < na ? q1p : q2p;
            const double* Rv = posr + ((size_t)mu * na + N) * 3;
            const double qr = qv[0] * Rv[0] + qv[1] * Rv[1] + qv[2] * Rv[2];
            double sn, cs;
            sincos(qr, &sn, &cs);
            sP[i] = make_double2(cs, sn);
        }
        __syncthreads();
        for (int i = tid; i < na * na; i += nt) {
            const int N1 = i / na, N2 = i % na;
            const double2 p1 = sP[N1], p2 = sP[na + N2];
            const double m = mrs[sBt[N1]] * mrs[sBt[N2]];
            sPP[i] = make_double2(m * (p1.x * p2.x - p1.y * p2.y), m * (p1.x * p2.y + p1.y * p2.x));
        }
        __syncthreads();
        for (int o = tid; o < 3 * nn; o += nt) {
            const int al = o / nn, r = (o / n) % n, cidx = o % n;
            const int nu = r / 3, be = r % 3, eta = cidx / 3, ga = cidx % 3;
            const int abc = (al * 3 + be) * 3 + ga;
            double2 acc = make_double2(0.0, 0.0);
            for (int N1 = 0; N1 < na; ++N1) {
                if (sBt[N1] != nu) continue;
                for (int N2 = 0; N2 < na; ++N2) {
                    if (sBt[N2] != eta) continue;
                    const double fv = sFC[(N1 * na + N2) * 27 + abc];
                    const double2 pp = sPP[N1 * na + N2];
                    acc.x = fma(fv, pp.x, acc.x);
                    acc.y = fma(fv, pp.y, acc.y);
                }
            }
            sD[o] = acc;
        }
        __syncthreads();
        for (int o = tid; o < 3 * nn; o += nt) {
            const int ar = o / n, s2 = o % n;
            const double2* drow = sD + ar * n;
            const double2* e2 = sE2 + s2;
            double2 acc = make_double2(0.0, 0.0);
            for (int k = 0; k < n; ++k) cfma(acc, drow[k], e2[k * n]);
            sT1[o] = acc;
        }
        __syncthreads();
        for (int o = tid; o < 3 * nn; o += nt) {
            const int al = o / nn, s1 = (o / n) % n, s2 = o % n;
            const double2* e1 = sE1 + s1 * n;
            const double2* t1 = sT1 + al * nn + s2;
            double2 acc = make_double2(0.0, 0.0);
            for (int k = 0; k < n; ++k) cfma(acc, e1[k], t1[k * n]);
            sT2[o] = acc;
        }
        __syncthreads();
        const double mm = mrs[mu];
        for (int o = tid; o < nphi; o += nt) {
            const int s0 = s0b + o / nn, r12 = o % nn;
            double2 acc = sPhi[o];
            for (int al = 0; al < 3; ++al) {
                double2 w = sE0[s0 * n + 3 * mu + al];
                w.x *= mm;
                w.y *= mm;
                cfma(acc, w, sT2[al * nn + r12]);
            }
            sPhi[o] = acc;
        }
        __syncthreads();
    }

    const double* qp0 = q0v + 3 * p;
    const bool gq0 = fabs(qp0[0]) < ZERO_PREC && fabs(qp0[1]) < ZERO_PREC && fabs(qp0[2]) < ZERO_PREC;
    const bool gq1 = qint[3 * q1] == 0 && qint[3 * q1 + 1] == 0 && qint[3 * q1 + 2] == 0;
    const bool gq2 = fabs(q2p[0]) < ZERO_PREC && fabs(q2p[1]) < ZERO_PREC && fabs(q2p[2]) < ZERO_PREC;
    for (int o = tid; o < nphi; o += nt) {
        const int s0 = s0b + o / nn, s1 = (o / n) % n, s2 = o % n;
        double w = 0.0;
        if (!((gq0 && s0 < 3) || (gq1 && s1 < 3) || (gq2 && s2 < 3))) {
            const double2 ph = sPhi[o];
            const double abs2 = ph.x * ph.x + ph.y * ph.y;
            const double den = __dmul_rn(__dmul_rn(__dmul_rn(om0[(size_t)p * n + s0], omg[(size_t)q1 * n + s1]),
                                                   om2[row * n + s2]),
                                         a.nqd);
            w = __dmul_rn(__ddiv_rn(abs2, den), a.sctr);
        }
        W[(s0 * n + s1) * n + s2] = w;
    }
}

// Gaussian CalculateLinewidth: one thread per (q1, s0, slot), every s1, s2 and temperature.
template <int NTM>
__global__ void __launch_bounds__(128) k_gauss_path(int n, int nq, int n_path, int p_first, int nT, long long ntab,
                                                    double os, double os2, const int* __restrict__ exists,
                                                    const int* __restrict__ qint, const double* __restrict__ W,
                                                    const double* __restrict__ om0, const double* __restrict__ omg,
                                                    const double* __restrict__ nbeg, const double* __restrict__ om2,
                                                    const double* __restrict__ nbe2, double* __restrict__ out_lw) {
    __shared__ double sacc[NTM];
    const int s0 = blockIdx.y, slot = blockIdx.z, p = p_first + slot;
    for (int i = threadIdx.x; i < NTM; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    double acc[NTM];
#pragma unroll
    for (int t = 0; t < NTM; ++t) acc[t] = 0.0;
    const size_t n3 = (size_t)n * n * n;
    const double pre = os * ONEBYSQRT2PI;
    const double w0 = om0[(size_t)p * n + s0];
    for (int q1 = blockIdx.x * blockDim.x + threadIdx.x; q1 < nq; q1 += gridDim.x * blockDim.x) {
        const size_t row = (size_t)slot * nq + q1;
        if (!exists[row]) continue;
        const int st1 = (qint[3 * q1] == 0 && qint[3 * q1 + 1] == 0 && qint[3 * q1 + 2] == 0) ? 3 : 0;
        const double* o2 = om2 + row * n;
        const int st2 = (fabs(o2[0]) < ZERO_PREC && fabs(o2[1]) < ZERO_PREC && fabs(o2[2]) < ZERO_PREC) ? 3 : 0;
        const double* Wq = W + row * n3 + (size_t)s0 * n * n;
        for (int s1 = st1; s1 < n; ++s1) {
            const double w1 = omg[(size_t)q1 * n + s1];
            for (int s2 = st2; s2 < n; ++s2) {
                const double w2 = o2[s2];
                const double d1 = w0 - w1 - w2, d2 = w0 + w1 - w2, d3 = w0 - w1 + w2;
                const double e1 = pre * exp(-0.5 * os2 * (d1 * d1));
                const double e2 = pre * exp(-0.5 * os2 * (d2 * d2));
                const double e3 = pre * exp(-0.5 * os2 * (d3 * d3));
                const double Wv = Wq[s1 * n + s2];
#pragma unroll
                for (int t = 0; t < NTM; ++t) {
                    if (t >= nT) break;
                    const double n1 = nbeg[((size_t)t * nq + q1) * n + s1];
                    const double n2 = nbe2[((size_t)t * ntab + row) * n + s2];
                    acc[t] += Wv * (((n1 + n2 + 1.0) * e1) + ((n1 - n2) * (e2 - e3)));
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < NTM; ++t) {
        double v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&sacc[t], v);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nT; t += blockDim.x)
        if (sacc[t] != 0.0) atomicAdd(&out_lw[((size_t)t * n_path + p) * n + s0], sacc[t]);
}

size_t v3p_smem(int n, int na, int sb) {
    const int nn = n * n;
    return sizeof(double2) * (3 * nn + 9 * nn + sb * nn + na * na + 2 * na) +
           sizeof(double) * ((na * na * 27 + 1) & ~1) + sizeof(int) * na + 16;
}

// 3x3 LU with partial pivoting as LAPACK dgetrf computes it for this size: the
// pivot is the first largest |a| of the column, the column below it is scaled by
// the reciprocal of the pivot and the trailing block updated by a(i,j) - l(i) u(j).
void lu3(const double* G, double* lu, int* piv) {
    double A[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) A[r][c] = G[r + 3 * c];
    for (int k = 0; k < 3; ++k) {
        int p = k;
        for (int i = k + 1; i < 3; ++i)
            if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
        piv[k] = p;
        if (p != k)
            for (int c = 0; c < 3; ++c) std::swap(A[k][c], A[p][c]);
        if (A[k][k] != 0.0) {
            const double r = 1.0 / A[k][k];
            for (int i = k + 1; i < 3; ++i) A[i][k] *= r;
        }
        for (int j = k + 1; j < 3; ++j)
            for (int i = k + 1; i < 3; ++i) A[i][j] = A[i][j] + (-A[k][j]) * A[i][k];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) lu[r * 3 + c] = A[r][c];
}

}  // namespace

int path_points(const double* G, int n_nodes, const double* qhs, double* qpoints, double* dist, int* zc) {
    int sp = 0;
    double sd = 0.0, dd = 0.0;
    for (int nd = 0; nd + 1 < n_nodes; ++nd) {
        const double* a = qhs + 4 * nd;
        const double* b = qhs + 4 * (nd + 1);
        const int npt = (int)b[3];
        bool neg = false, sa = true, sb = true;
        for (int k = 0; k < 3; ++k) {
            neg = neg || a[k] < 0.0 || b[k] < 0.0;
            sa = sa && std::fabs(a[k]) <= 0.5;
            sb = sb && std::fabs(b[k]) <= 0.5;
        }
        const bool zero_c = neg || sa || sb;
        double s[3], e[3], d[3], vh[3];
        for (int r = 0; r < 3; ++r) {
            s[r] = G[r] * a[0] + G[r + 3] * a[1] + G[r + 6] * a[2];
            e[r] = G[r] * b[0] + G[r + 3] * b[1] + G[r + 6] * b[2];
            d[r] = e[r] - s[r];
        }
        const double vlen = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int r = 0; r < 3; ++r) vh[r] = d[r] / vlen;
        const double step = npt != 0 ? vlen / npt : 0.0;
        for (int ii = 1; ii <= npt; ++ii) {
            dd = sd + ii * step;
            const double t = ii * step;
            if (qpoints)
                for (int r = 0; r < 3; ++r) qpoints[3 * sp + r] = s[r] + t * vh[r];
            if (dist) dist[sp] = dd;
            if (zc) zc[sp] = zero_c ? 1 : 0;
            ++sp;
        }
        sd = dd;
    }
    return sp;
}

namespace {
PathQ2Args path_q2_args(spring_ctx* c) {
    PathQ2Args qa{};
    qa.nq = c->nq;
    qa.n0 = c->mesh[0];
    qa.n1 = c->mesh[1];
    qa.n2 = c->mesh[2];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            qa.ru[r * 3 + k] = c->G[r + 3 * k] / double(c->mesh[k]);
            qa.G[r * 3 + k] = c->G[r + 3 * k];
        }
    for (int k = 0; k < 3; ++k) qa.shift[k] = (double)c->mesh_shift[k] * 0.5;
    lu3(c->G, qa.lu, qa.piv);
    return qa;
}
}  // namespace

void path_release(PathPlan& p) {
    dfree(p.q0v); dfree(p.q1v); dfree(p.q2v); dfree(p.w); dfree(p.lw); dfree(p.p3); dfree(p.zc); dfree(p.ex);
    free_phonons(p.php);
    free_phonons(p.ph2);
    p.n_path = 0;
    p.slots = 0;
}

int path_prepare(spring_ctx* c, PathPlan& p, int n_path, const double* h_q0, const int* h_zc) {
    const int n = c->ndof, nq = c->nq;
    const size_t n3 = (size_t)n * n * n;
    // slots: path points per batch (W grid + q2 phonons of a slot)
    const size_t per_slot = (size_t)nq * (n3 * sizeof(double) + (size_t)n * n * sizeof(double2) +
                                          (size_t)n * sizeof(double) * (6 + c->nT) + 8 * sizeof(double));
    const size_t budget = (size_t)512 << 20;
    p.n_path = n_path;
    p.slots = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_path, budget / per_slot));
    const long long rows_max = (long long)p.slots * nq;
    SPRING_CHECK(dalloc(c, p.q0v, (size_t)3 * n_path, "path q0"));
    SPRING_CHECK(dalloc(c, p.zc, (size_t)n_path, "path flags"));
    SPRING_CHECK(dalloc(c, p.q1v, (size_t)3 * rows_max, "path q1"));
    SPRING_CHECK(dalloc(c, p.q2v, (size_t)3 * rows_max, "path q2"));
    SPRING_CHECK(dalloc(c, p.ex, (size_t)rows_max, "path q2 flags"));
    SPRING_CHECK(dalloc(c, p.w, (size_t)rows_max * n3, "path W"));
    SPRING_CHECK(dalloc(c, p.lw, (size_t)c->nT * n_path * n, "path linewidth"));
    SPRING_CHECK(dalloc(c, p.p3, (size_t)n_path * n, "path scratch"));
    SPRING_CHECK(alloc_phonons(c, p.php, n_path));
    SPRING_CHECK(alloc_phonons(c, p.ph2, (int)rows_max));
    SPRING_CHECK(h2d(c, p.q0v.p, h_q0, sizeof(double) * 3 * n_path, "path q0"));
    SPRING_CHECK(h2d(c, p.zc.p, h_zc, sizeof(int) * n_path, "path flags"));
    const size_t smem = v3p_smem(n, c->na3, n <= 12 ? n : 6);
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "path V3 tile needs %zu bytes of shared memory", smem);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_v3_path, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return SPRING_OK;
}

int path_enqueue(spring_ctx* c, PathPlan& p, int delta_mode, double sigma) {
    const int n = c->ndof, nq = c->nq, n_path = p.n_path;
    const size_t n3 = (size_t)n * n * n;
    const PathQ2Args qa0 = path_q2_args(c);
    SPRING_CHECK(zero(c, p.lw.p, sizeof(double) * c->nT * n_path * n, "path linewidth"));
    SPRING_CHECK(run_phonons(c, p.php, p.q0v.p, n_path));
    V3PArgs va{};
    va.nb = c->nb;
    va.n = n;
    va.na = c->na3;
    va.nq = nq;
    va.sb = n <= 12 ? n : 6;
    va.nsb = (n + va.sb - 1) / va.sb;
    va.nqd = double(nq);
    va.sctr = host_constants().Sctr3THz2;
    const size_t smem = v3p_smem(n, c->na3, va.sb);
    for (int p0 = 0; p0 < n_path; p0 += p.slots) {
        const int ns = std::min(p.slots, n_path - p0);
        const long long rows = (long long)ns * nq;
        PathQ2Args qa = qa0;
        qa.p_first = p0;
        const int threads = 128;
        const int blocks = (int)std::min<long long>((rows + threads - 1) / threads, 148LL * 32);
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "path: injected launch failure");
        k_path_q2<<<blocks, threads, 0, c->stream>>>(qa, ns, p.q0v.p, p.zc.p, c->d_qpnt.p, p.q1v.p, p.q2v.p, p.ex.p);
        SPRING_CHECK(launch_check(c, "k_path_q2"));
        SPRING_CHECK(run_phonons(c, p.ph2, p.q2v.p, (int)rows, 1));  // single points (get_phonon_singleq)
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "path: injected launch failure");
        k_path_clear_missing<<<blocks, threads, 0, c->stream>>>(rows, n, c->nT, p.ex.p, p.ph2.omega.p, p.ph2.nbe.p);
        SPRING_CHECK(launch_check(c, "k_path_clear_missing"));
        SPRING_CHECK(zero(c, p.w.p, sizeof(double) * rows * n3, "path W"));
        va.p_first = p0;
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "path: injected launch failure");
        k_v3_path<<<dim3((unsigned)(nq * va.nsb), ns), 128, smem, c->stream>>>(
            va, p.ex.p, p.q0v.p, p.q1v.p, p.q2v.p, c->d_qint.p, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p,
            c->d_mass_rs.p, p.php.evec.p, p.php.omega.p, c->ph_grid.evec.p, c->ph_grid.omega.p, p.ph2.evec.p,
            p.ph2.omega.p, p.w.p);
        SPRING_CHECK(launch_check(c, "k_v3_path"));
        if (delta_mode == SPRING_DELTA_TETRA) {
            SPRING_CHECK(run_tetra3_path(c, p0, ns, n_path, p.w.p, p.php.omega.p, p.ph2.omega.p, p.ph2.nbe.p, rows,
                                         p.lw.p, p.p3.p));
        } else {
            const double os = 1.0 / sigma;
            dim3 grid((unsigned)std::max(1, std::min((nq + 127) / 128, 64)), n, ns);
            if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "path: injected launch failure");
#define SPRING_GAUSS_PATH(NTM)                                                                                    \
    k_gauss_path<NTM><<<grid, 128, 0, c->stream>>>(n, nq, n_path, p0, c->nT, rows, os, os * os, p.ex.p, c->d_qint.p, \
                                                   p.w.p, p.php.omega.p, c->ph_grid.omega.p, c->ph_grid.nbe.p,   \
                                                   p.ph2.omega.p, p.ph2.nbe.p, p.lw.p)
            if (c->nT == 1) SPRING_GAUSS_PATH(1);
            else if (c->nT <= 3) SPRING_GAUSS_PATH(3);
            else SPRING_GAUSS_PATH(9);
#undef SPRING_GAUSS_PATH
            SPRING_CHECK(launch_check(c, "k_gauss_path"));
        }
    }
    return SPRING_OK;
}

int path_fetch(spring_ctx* c, PathPlan& p, double* h_lw, double* h_omega) {
    if (h_lw) SPRING_CHECK(d2h(c, h_lw, p.lw.p, sizeof(double) * c->nT * p.n_path * c->ndof, "path linewidth"));
    if (h_omega) SPRING_CHECK(d2h(c, h_omega, p.php.omega.p, sizeof(double) * p.n_path * c->ndof, "path omega"));
    return SPRING_OK;
}

int run_path(spring_ctx* c, int n_path, const double* h_q0, const int* h_zc, int delta_mode, double sigma,
             double* h_lw, double* h_omega) {
    PathPlan p;
    int rc = path_prepare(c, p, n_path, h_q0, h_zc);
    if (rc == SPRING_OK) rc = path_enqueue(c, p, delta_mode, sigma);
    if (rc == SPRING_OK) rc = path_fetch(c, p, h_lw, h_omega);
    cudaStreamSynchronize(c->stream);
    path_release(p);
    return rc;
}

}  // namespace spring
