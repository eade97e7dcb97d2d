// Four-phonon scattering on the device.
//
//  - Enumeration, MomentumConsrv4th + Permutation4th
//    (src/Kappa/Src/QuasiMomentumConsrv4th_m.f90:32-312).  The sequential covering loop
//    has a closed form: (q1,q2) is visited in grid order and the first ordering of a
//    grid multiset {q1,q2,q3} met by the loop covers every other ordering, so (q1,q2)
//    is a representative iff its key q1*Nq+q2 is the smallest of the orderings of its
//    multiset; quartet numbers come from a scan.  Each representative then writes its
//    Allq1q2q3 cells in the reference's order (direct entry, then the five
//    permutations with the reference's "no new permutation" test on the integer
//    vectors), so the arrays are bit-identical to the reference algorithm's.
//  - V4 -> W4, ScatterMatEl4 / ScatterProbability4 (src/Kappa/Src/FourthOrder_m.f90:286-473),
//    regrouped like V3: D_mu[a][nu b][eta c][ro d] = sum over slots of each basis block of
//    FC4 e^{i q1.R1} e^{i q2.R2} e^{i q3.R3} m^-1/2 m^-1/2 m^-1/2, then four Ndof^5
//    contractions with e3, e2, e1, e0.  FP64.  Two-atom cells (Ndof 6).
//  - Rates.  Tetrahedron: TetrahedronIntegration4th / SumOverPolarization /
//    FindFandOmegaVer_4th (src/Kappa/Src/Tetrahedron4th_sep.f90:37-425), with the
//    reference's reading of the stored quartet W through `per` for every permutation
//    type; Gaussian: the same three channels with delta(w0 - M) (build-side form),
//    summed over every ordered grid (q1, q2) - each distinct ordering of a quartet's
//    grid points once - with W taken from the quartet's own W4.
// Roofline: FP64 FMA for V4 (222 kflop phase-folded FC4 + 249 kflop contractions per
// quartet); FP64 ALU for the tetrahedron sums.
#include <algorithm>
#include <cub/cub.cuh>

#include "spring_internal.cuh"
#include "tetra.cuh"

namespace spring {
namespace {

constexpr int NB = 2, N = 6, NA_MAX = 8, QB = 2;
constexpr double EXP_CUT = 40.0;  // exp(-40) = 4e-18 of a delta's peak: terms below it are dropped

__device__ __forceinline__ int imod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// q3 = G - (q0 + q1 + q2) with the first G of (0,+1,-1)^3 inside [-N/2, N/2]^3 (componentwise).
__device__ __forceinline__ int partner4(const int* q0, const int* q1, const int* q2, const int* nn, int* q3) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int b = nn[d] / 2;
        const int v = -(q0[d] + q1[d] + q2[d]);
        int w = v;
        if (w > b || w < -b) {
            w = v + nn[d];
            if (w > b || w < -b) w = v - nn[d];
        }
        q3[d] = w;
    }
    return imod(q3[0], nn[0]) + nn[0] * (imod(q3[1], nn[1]) + nn[1] * imod(q3[2], nn[2]));
}

struct Mesh3 {
    int n[3];
};

__global__ void k_enum4_flags(int nq, Mesh3 m, const int* __restrict__ q0, const int* __restrict__ qint,
                              int* __restrict__ g3o, int* __restrict__ rep) {
    const long long total = (long long)nq * nq;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int g1 = (int)(i / nq), g2 = (int)(i % nq);
        int q3[3];
        const int g3 = partner4(q0, qint + 3 * g1, qint + 3 * g2, m.n, q3);
        g3o[i] = g3;
        const long long k = i, L = nq;
        const long long o[5] = {g1 * L + g3, g2 * L + g1, g2 * L + g3, g3 * L + g1, g3 * L + g2};
        bool r = true;
#pragma unroll
        for (int j = 0; j < 5; ++j) r = r && (k <= o[j]);
        rep[i] = r ? 1 : 0;
    }
}

__global__ void k_enum4_write(int nq, Mesh3 m, const int* __restrict__ q0, const int* __restrict__ qint,
                              const int* __restrict__ g3a, const int* __restrict__ rep, const int* __restrict__ pos,
                              int* __restrict__ all, int* __restrict__ perm, long long cap, int4* __restrict__ quart,
                              unsigned long long* __restrict__ total) {
    const int per[5][3] = {{0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const long long tot = (long long)nq * nq;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        if (!rep[i]) continue;
        const int g1 = (int)(i / nq), g2 = (int)(i % nq), g3 = g3a[i];
        const int cnt = pos[i] + 1;
        if (quart) quart[cnt - 1] = make_int4(g1, g2, g3, 0);
        if (perm && cnt <= cap) {
            perm[3 * (size_t)(cnt - 1)] = g1 + 1;
            perm[3 * (size_t)(cnt - 1) + 1] = g2 + 1;
            perm[3 * (size_t)(cnt - 1) + 2] = g3 + 1;
        }
        int Q[3][3];
        partner4(q0, qint + 3 * g1, qint + 3 * g2, m.n, Q[2]);
        for (int d = 0; d < 3; ++d) {
            Q[0][d] = qint[3 * g1 + d];
            Q[1][d] = qint[3 * g2 + d];
        }
        const int G[3] = {g1, g2, g3};
        if (all) {
            int* e = all + 3 * ((size_t)g1 * nq + g2);
            e[0] = 0; e[1] = cnt; e[2] = g3 + 1;
        }
        int pg[5][3];
        unsigned long long newc = 0;
        for (int pp = 0; pp < 5; ++pp) {
            for (int k = 0; k < 3; ++k) pg[pp][k] = G[per[pp][k]];
            bool nonew = true;
            for (int k = 0; k < 3; ++k)
                for (int d = 0; d < 3; ++d)
                    if (Q[per[pp][k]][d] != Q[k][d]) nonew = false;
            for (int qq = 0; qq < pp; ++qq)
                nonew = nonew || (pg[pp][0] == pg[qq][0] && pg[pp][1] == pg[qq][1] && pg[pp][2] == pg[qq][2]);
            if (!nonew) {
                ++newc;
                if (all) {
                    int* e = all + 3 * ((size_t)pg[pp][0] * nq + pg[pp][1]);
                    e[0] = pp + 1; e[1] = cnt; e[2] = pg[pp][2] + 1;
                }
            }
        }
        atomicAdd(total, 1ull + newc);
    }
}

// ------------------------------------------------------------------------- V4
struct V4Args {
    int nq, nT, nq0, q0, na, nquart;
    double mfac, onebysigma, onebysigma2;
    int pol_lo[4], pol_hi[4];
};

struct V4Smem {
    double2 e[QB][4][36];          // e0 (times m_mu^-1/2 by row), e1, e2, e3: [s][row]
    double2 ppp[QB][NA_MAX * NA_MAX * NA_MAX];
    double2 A[QB][648];            // D4 [a][nb][ec][rd], then T2 [a nb][s2][s3]
    double2 B[QB][648];            // T1 [a nb ec][s3], then T3 [a][s1][s2 s3]
    double2 phi[QB][1296];         // Phi, then W (as doubles in .x)
    double lw[MAX_NDOF][10];       // [s0][T] rate accumulators (T <= 9), last column unused
    double ph[QB][3][NA_MAX][2];
    double wq[QB][3][N];           // omega of the quartet's three grid points
    double nq[QB][9][3][N];        // their occupations per temperature
    int g[QB][4];                  // g1 g2 g3 valid
};

template <int EPI>
__global__ void __launch_bounds__(256, 2)
k_v4(V4Args a, const int4* __restrict__ quart, const double* __restrict__ fc4, const double* __restrict__ posr,
     const int* __restrict__ btyp, const int* __restrict__ off, const double* __restrict__ mrs,
     const double* __restrict__ qpnt, const int* __restrict__ q0int, const double2* __restrict__ ev0,
     const double* __restrict__ om0, const double* __restrict__ ob0, const double* __restrict__ nbe0,
     const double2* __restrict__ evg, const double* __restrict__ omg, const double* __restrict__ obg,
     const double* __restrict__ nbeg, double* __restrict__ out_rate, double* __restrict__ out_w) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V4Smem& S = *reinterpret_cast<V4Smem*>(smem_raw);
    const int tid = threadIdx.x, nt = blockDim.x;
    const int na = a.na;
    const bool gq0 = q0int[0] == 0 && q0int[1] == 0 && q0int[2] == 0;
    if (EPI == 0)
        for (int i = tid; i < MAX_NDOF * 10; i += nt) (&S.lw[0][0])[i] = 0.0;
    for (int grp = blockIdx.x; grp * QB < a.nquart; grp += gridDim.x) {
        __syncthreads();
        if (tid < QB) {
            const int k = grp * QB + tid;
            const bool v = k < a.nquart;
            const int4 q = v ? quart[k] : make_int4(0, 0, 0, 0);
            S.g[tid][0] = q.x; S.g[tid][1] = q.y; S.g[tid][2] = q.z; S.g[tid][3] = v;
        }
        __syncthreads();
        for (int i = tid; i < QB * 4 * 36; i += nt) {
            const int p = i / 144, w = (i / 36) % 4, k = i % 36;
            double2 v = w == 0 ? ev0[k] : evg[(size_t)S.g[p][w - 1] * 36 + k];
            if (w == 0) {
                const double mm = mrs[(k % 6) / 3];
                v.x *= mm;
                v.y *= mm;
            }
            S.e[p][w][k] = v;
        }
        for (int i = tid; i < QB * 1296; i += nt) S.phi[i / 1296][i % 1296] = make_double2(0.0, 0.0);
        for (int mu = 0; mu < NB; ++mu) {
            for (int i = tid; i < QB * 3 * na; i += nt) {
                const int p = i / (3 * na), k = (i / na) % 3, Nn = i % na;
                const int gg = S.g[p][k];
                const double* R = posr + ((size_t)mu * na + Nn) * 3;
                const double qr = qpnt[3 * gg] * R[0] + qpnt[3 * gg + 1] * R[1] + qpnt[3 * gg + 2] * R[2];
                double sn, cs;
                sincos(qr, &sn, &cs);
                const double mm = mrs[btyp[mu * na + Nn]];
                S.ph[p][k][Nn][0] = mm * cs;
                S.ph[p][k][Nn][1] = mm * sn;
            }
            __syncthreads();
            for (int i = tid; i < QB * na * na * na; i += nt) {
                const int p = i / (na * na * na), n1 = (i / (na * na)) % na, n2 = (i / na) % na, n3 = i % na;
                const double* x = S.ph[p][0][n1];
                const double* y = S.ph[p][1][n2];
                const double* z = S.ph[p][2][n3];
                const double xr = x[0] * y[0] - x[1] * y[1], xi = x[0] * y[1] + x[1] * y[0];
                S.ppp[p][(n1 * na + n2) * na + n3] = make_double2(xr * z[0] - xi * z[1], xr * z[1] + xi * z[0]);
            }
            __syncthreads();
            // D4: thread per (pair, abcd); all eight (nu, eta, ro) blocks in registers
            const int* o = off + mu * (NB + 1);
            for (int u = tid; u < QB * 81; u += nt) {
                const int p = u / 81, r = u % 81;
                double2 acc[NB][NB][NB];
#pragma unroll
                for (int x = 0; x < NB; ++x)
#pragma unroll
                    for (int y = 0; y < NB; ++y)
#pragma unroll
                        for (int z = 0; z < NB; ++z) acc[x][y][z] = make_double2(0.0, 0.0);
                const double* f = fc4 + (size_t)mu * na * na * na * 81 + r;
#pragma unroll
                for (int nu = 0; nu < NB; ++nu)
                    for (int n1 = o[nu]; n1 < o[nu + 1]; ++n1)
#pragma unroll
                        for (int eta = 0; eta < NB; ++eta)
                            for (int n2 = o[eta]; n2 < o[eta + 1]; ++n2)
#pragma unroll
                                for (int ro = 0; ro < NB; ++ro)
                                    for (int n3 = o[ro]; n3 < o[ro + 1]; ++n3) {
                                        const int s = (n1 * na + n2) * na + n3;
                                        const double fv = __ldg(f + (size_t)s * 81);
                                        const double2 q = S.ppp[p][s];
                                        acc[nu][eta][ro].x = fma(fv, q.x, acc[nu][eta][ro].x);
                                        acc[nu][eta][ro].y = fma(fv, q.y, acc[nu][eta][ro].y);
                                    }
                const int al = r / 27, be = (r / 9) % 3, ga = (r / 3) % 3, de = r % 3;
#pragma unroll
                for (int nu = 0; nu < NB; ++nu)
#pragma unroll
                    for (int eta = 0; eta < NB; ++eta)
#pragma unroll
                        for (int ro = 0; ro < NB; ++ro)
                            S.A[p][((al * 6 + nu * 3 + be) * 6 + eta * 3 + ga) * 6 + ro * 3 + de] = acc[nu][eta][ro];
            }
            __syncthreads();
            // T1[a nb ec][s3] = sum_rd D4[a nb ec][rd] e3(rd, s3)
            for (int u = tid; u < QB * 108; u += nt) {
                const int p = u / 108, row = u % 108;
                double2 acc[N];
#pragma unroll
                for (int s = 0; s < N; ++s) acc[s] = make_double2(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const double2 d = S.A[p][row * 6 + k];
#pragma unroll
                    for (int s = 0; s < N; ++s) {
                        const double2 e = S.e[p][3][s * 6 + k];
                        acc[s].x = fma(d.x, e.x, fma(-d.y, e.y, acc[s].x));
                        acc[s].y = fma(d.x, e.y, fma(d.y, e.x, acc[s].y));
                    }
                }
#pragma unroll
                for (int s = 0; s < N; ++s) S.B[p][row * 6 + s] = acc[s];
            }
            __syncthreads();
            // T2[a nb][s2][s3] = sum_ec e2(ec, s2) T1[a nb ec][s3]
            for (int u = tid; u < QB * 108; u += nt) {
                const int p = u / 108, ab = (u % 108) / 6, s2 = u % 6;
                double2 acc[N];
#pragma unroll
                for (int s = 0; s < N; ++s) acc[s] = make_double2(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const double2 e = S.e[p][2][s2 * 6 + k];
#pragma unroll
                    for (int s = 0; s < N; ++s) {
                        const double2 t = S.B[p][(ab * 6 + k) * 6 + s];
                        acc[s].x = fma(e.x, t.x, fma(-e.y, t.y, acc[s].x));
                        acc[s].y = fma(e.x, t.y, fma(e.y, t.x, acc[s].y));
                    }
                }
#pragma unroll
                for (int s = 0; s < N; ++s) S.A[p][(ab * 6 + s2) * 6 + s] = acc[s];
            }
            __syncthreads();
            // T3[a][s1][s2 s3] = sum_nb e1(nb, s1) T2[a nb][s2 s3]
            for (int u = tid; u < QB * 108; u += nt) {
                const int p = u / 108, al = (u % 108) / 36, s1 = (u % 36) / 6, s2 = u % 6;
                double2 acc[N];
#pragma unroll
                for (int s = 0; s < N; ++s) acc[s] = make_double2(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const double2 e = S.e[p][1][s1 * 6 + k];
#pragma unroll
                    for (int s = 0; s < N; ++s) {
                        const double2 t = S.A[p][((al * 6 + k) * 6 + s2) * 6 + s];
                        acc[s].x = fma(e.x, t.x, fma(-e.y, t.y, acc[s].x));
                        acc[s].y = fma(e.x, t.y, fma(e.y, t.x, acc[s].y));
                    }
                }
#pragma unroll
                for (int s = 0; s < N; ++s) S.B[p][((al * 6 + s1) * 6 + s2) * 6 + s] = acc[s];
            }
            __syncthreads();
            // Phi[s0][s1 s2 s3] += sum_a e0'(mu a, s0) T3[a][s1 s2 s3]
            for (int u = tid; u < QB * 216; u += nt) {
                const int p = u / 216, s0 = (u % 216) / 36, s12 = u % 36;
#pragma unroll
                for (int s = 0; s < N; ++s) {
                    double2 acc = S.phi[p][(s0 * 36 + s12) * 6 + s];
#pragma unroll
                    for (int al = 0; al < 3; ++al) {
                        const double2 e = S.e[p][0][s0 * 6 + mu * 3 + al];
                        const double2 t = S.B[p][(al * 36 + s12) * 6 + s];
                        acc.x = fma(e.x, t.x, fma(-e.y, t.y, acc.x));
                        acc.y = fma(e.x, t.y, fma(e.y, t.x, acc.y));
                    }
                    S.phi[p][(s0 * 36 + s12) * 6 + s] = acc;
                }
            }
            __syncthreads();
        }
        // W4 = |Phi|^2 (1/w0)(1/w1)(1/w2)(1/w3) Sctr4THz2/Nq^2, zero for Gamma acoustic modes
        for (int i = tid; i < QB * 1296; i += nt) {
            const int p = i / 1296, k = i % 1296;
            const int s0 = k / 216, s1 = (k / 36) % 6, s2 = (k / 6) % 6, s3 = k % 6;
            const int g1 = S.g[p][0], g2 = S.g[p][1], g3 = S.g[p][2];
            const bool z = (gq0 && s0 < 3) || (g1 == 0 && s1 < 3) || (g2 == 0 && s2 < 3) || (g3 == 0 && s3 < 3);
            const double2 v = S.phi[p][k];
            const double a2 = v.x * v.x + v.y * v.y;
            const double W = z ? 0.0 : (a2 * (ob0[s0] * obg[(size_t)g1 * N + s1] * obg[(size_t)g2 * N + s2] *
                                              obg[(size_t)g3 * N + s3])) * a.mfac;
            S.phi[p][k].x = W;
            if (EPI == 1 && S.g[p][3]) out_w[(size_t)(grp * QB + p) * 1296 + k] = W;
        }
        if (EPI == 0) {
            __syncthreads();
            // Gaussian: every distinct ordering (qa, qb, qc) of the quartet's grid points.  The
            // frequencies and occupations of the three points are staged; each (mode quad, ordering)
            // is screened in FP32 against the window where a delta weight exceeds exp(-40) of its
            // peak, and only the rest is evaluated in FP64.
            for (int i = tid; i < QB * 3 * N; i += nt) {
                const int p = i / (3 * N), k = (i / N) % 3, sx = i % N;
                const int gg = S.g[p][k];
                S.wq[p][k][sx] = omg[(size_t)gg * N + sx];
                for (int t = 0; t < a.nT; ++t) S.nq[p][t][k][sx] = nbeg[(size_t)t * a.nq * N + (size_t)gg * N + sx];
            }
            __syncthreads();
            const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
            const double pre = a.onebysigma * ONEBYSQRT2PI;
            const float Rf = (float)(sqrt(2.0 * EXP_CUT) / a.onebysigma * 1.0001 + 1e-3);
            for (int i = tid; i < QB * 1296; i += nt) {
                const int p = i / 1296, k = i % 1296;
                if (!S.g[p][3]) continue;
                const int s0 = k / 216, sa = (k / 36) % 6, sb = (k / 6) % 6, sc = k % 6;
                if (s0 < (gq0 ? 3 : a.pol_lo[0]) || s0 > a.pol_hi[0]) continue;  // SumOverPolarization s0Strt
                if (sa < a.pol_lo[1] || sa > a.pol_hi[1] || sb < a.pol_lo[2] || sb > a.pol_hi[2] ||
                    sc < a.pol_lo[3] || sc > a.pol_hi[3])
                    continue;
                const int* G = S.g[p];
                const double w0 = om0[s0];
                const float f0 = (float)w0;
                for (int pi = 0; pi < 6; ++pi) {
                    const int ia = perms[pi][0], ib = perms[pi][1], ic = perms[pi][2];
                    const int ga = G[ia], gb = G[ib];
                    bool dup = false;
                    for (int pj = 0; pj < pi; ++pj)
                        dup = dup || (G[perms[pj][0]] == ga && G[perms[pj][1]] == gb);
                    if (dup) continue;
                    const double wa = S.wq[p][ia][sa], wb = S.wq[p][ib][sb], wc = S.wq[p][ic][sc];
                    const float fa = (float)wa, fb = (float)wb, fc = (float)wc;
                    if (fabsf(f0 - (fa + fb + fc)) >= Rf && fabsf(f0 - (fb + fc - fa)) >= Rf &&
                        fabsf(f0 - (fc - fa - fb)) >= Rf)
                        continue;
                    int m[3];
                    m[ia] = sa;
                    m[ib] = sb;
                    m[ic] = sc;
                    const double Wv = S.phi[p][((s0 * 6 + m[0]) * 6 + m[1]) * 6 + m[2]].x;
                    if (Wv == 0.0) continue;
                    const double d1 = w0 - (wa + wb + wc), d2 = w0 - (wb + wc - wa), d3 = w0 - (wc - wa - wb);
                    const double x1 = 0.5 * a.onebysigma2 * (d1 * d1), x2 = 0.5 * a.onebysigma2 * (d2 * d2),
                                 x3 = 0.5 * a.onebysigma2 * (d3 * d3);
                    const double e1 = x1 < EXP_CUT ? pre * exp(-x1) : 0.0;
                    const double e2 = x2 < EXP_CUT ? pre * exp(-x2) : 0.0;
                    const double e3 = x3 < EXP_CUT ? pre * exp(-x3) : 0.0;
                    if (e1 == 0.0 && e2 == 0.0 && e3 == 0.0) continue;
                    for (int t = 0; t < a.nT; ++t) {
                        const double na_ = S.nq[p][t][ia][sa], nbb = S.nq[p][t][ib][sb], nc = S.nq[p][t][ic][sc];
                        const double n0 = nbe0[(size_t)t * a.nq0 * N + s0];
                        const double v = ONEBYSIX * (Wv * (na_ * nbb * nc / n0)) * e1 +
                                         0.5 * (Wv * ((1.0 + na_) * nbb * nc / n0)) * e2 +
                                         0.5 * (Wv * ((1.0 + na_) * (1.0 + nbb) * nc / n0)) * e3;
                        atomicAdd(&S.lw[s0][t], v);
                    }
                }
            }
        }
    }
    if (EPI == 0) {
        __syncthreads();
        for (int i = tid; i < N * a.nT; i += nt) {
            const int s0 = i / a.nT, t = i % a.nT;
            if (S.lw[s0][t] != 0.0) atomicAdd(&out_rate[((size_t)t * a.nq0 + a.q0) * N + s0], S.lw[s0][t]);
        }
    }
}

// ------------------------------------------------------------------------- tetrahedron
struct T4Args {
    int nq, nT, nq0, q0, ntet, nquart;
    int pol_lo[4], pol_hi[4];
};

// one thread per (q1, tetrahedron of q2, s1, s2, s3); all s0 and temperatures in the thread
__global__ void __launch_bounds__(128) k_tetra4(T4Args a, const int4* __restrict__ tet, const int* __restrict__ all,
                                                const double* __restrict__ Wq, const int* __restrict__ q0int,
                                                const double* __restrict__ om0, const double* __restrict__ nbe0,
                                                const double* __restrict__ omg, const double* __restrict__ nbeg,
                                                double* __restrict__ out) {
    __shared__ double sacc[N * 10];
    const int per[5][3] = {{0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int i = threadIdx.x; i < N * 10; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    const bool gq0 = q0int[0] == 0 && q0int[1] == 0 && q0int[2] == 0;
    const int s0a = gq0 ? 3 : a.pol_lo[0];
    const int n1r = a.pol_hi[1] - a.pol_lo[1] + 1, n2r = a.pol_hi[2] - a.pol_lo[2] + 1, n3r = a.pol_hi[3] - a.pol_lo[3] + 1;
    const long long items = (long long)a.nq * a.ntet * n1r * n2r * n3r;
    double acc[N][9];
#pragma unroll
    for (int s = 0; s < N; ++s)
#pragma unroll
        for (int t = 0; t < 9; ++t) acc[s][t] = 0.0;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int s3 = a.pol_lo[3] + (int)(it % n3r);
        const int s2 = a.pol_lo[2] + (int)((it / n3r) % n2r);
        const int s1 = a.pol_lo[1] + (int)((it / ((long long)n3r * n2r)) % n1r);
        const long long r = it / ((long long)n3r * n2r * n1r);
        const int t = (int)(r % a.ntet), q1 = (int)(r / a.ntet);
        const int4 tv = tet[t];
        const int v2[4] = {tv.x, tv.y, tv.z, tv.w};
        int v3[4], typ[4], pos[4];
        double M[3][4];
        const double w1 = omg[(size_t)q1 * N + s1];
        bool ok = true;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int* e = all + 3 * ((size_t)q1 * a.nq + v2[v]);
            typ[v] = e[0];
            pos[v] = e[1] - 1;
            v3[v] = e[2] - 1;
            ok = ok && typ[v] >= 0 && typ[v] <= 5 && pos[v] >= 0 && pos[v] < a.nquart && v3[v] >= 0 && v3[v] < a.nq;
        }
        if (!ok) continue;  // every cell is written by the enumeration; an unwritten one is skipped, not read
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double w2 = omg[(size_t)v2[v] * N + s2], w3 = omg[(size_t)v3[v] * N + s3];
            M[0][v] = (w1 + w2 + w3);
            M[1][v] = (w2 + w3 - w1);
            M[2][v] = (w3 - w1 - w2);
        }
        int pm[3][4];
        double Sm[3][4];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            tet::sort4(M[ch], pm[ch]);
#pragma unroll
            for (int v = 0; v < 4; ++v) Sm[ch][v] = M[ch][pm[ch][v]];
        }
        int wofs[4];  // mode offset of (s1,s2,s3) read through the reference's permutation
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int before[3] = {s1, s2, s3};
            int af[3];
            for (int k = 0; k < 3; ++k) af[k] = typ[v] == 0 ? before[k] : before[per[typ[v] - 1][k]];
            wofs[v] = (af[0] * N + af[1]) * N + af[2];
        }
        for (int s0 = s0a; s0 <= a.pol_hi[0]; ++s0) {
            const double Mqs = om0[s0];
            double Wv[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) Wv[v] = Wq[(size_t)pos[v] * 1296 + s0 * 216 + wofs[v]];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                double g, I[4];
                const bool e = tet::g_iver<false>(Mqs, Sm[ch], g, I);
#pragma unroll
                for (int v = 0; v < 4; ++v) if (isnan(I[v])) I[v] = 0.0;
                if (isnan(g)) g = 0.0;
                if (!e) continue;
                const double wt = ch == 0 ? ONEBYSIX : 0.5;
                for (int T = 0; T < a.nT; ++T) {
                    const double* nb = nbeg + (size_t)T * a.nq * N;
                    const double n0 = nbe0[(size_t)T * a.nq0 * N + s0];
                    const double n1 = nb[(size_t)q1 * N + s1];
                    double sum = 0.0;
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int q = pm[ch][v];
                        const double n2 = nb[(size_t)v2[q] * N + s2], n3 = nb[(size_t)v3[q] * N + s3];
                        const double f = ch == 0 ? (n1 * n2 * n3 / n0)
                                                 : (ch == 1 ? ((1.0 + n1) * n2 * n3 / n0)
                                                            : ((1.0 + n1) * (1.0 + n2) * n3 / n0));
                        sum += I[v] * (Wv[q] * f);
                    }
                    acc[s0][T] += wt * g * (ONEBYSIX * sum);
                }
            }
        }
    }
#pragma unroll
    for (int s = 0; s < N; ++s)
#pragma unroll
        for (int T = 0; T < 9; ++T) {
            double v = acc[s][T];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&sacc[s * 10 + T], v);
        }
    __syncthreads();
    for (int i = threadIdx.x; i < N * a.nT; i += blockDim.x) {
        const int s = i / a.nT, T = i % a.nT;
        if (sacc[s * 10 + T] != 0.0) atomicAdd(&out[((size_t)T * a.nq0 + a.q0) * N + s], sacc[s * 10 + T]);
    }
}

// Enumerate the quartets of q0 into device buffers (grid-pair scratch owned by the caller).
struct Enum4Bufs {
    DBuf<int> g3, rep, pos, all;
    DBuf<int4> quart;
    DBuf<unsigned long long> total;
};

int enumerate4(spring_ctx* c, int q0, Enum4Bufs& b, bool want_all, int* d_perm, long long cap, long long* h_counts) {
    const long long tot = (long long)c->nq * c->nq;
    if (tot > 0x7fffffffLL) return fail(c, SPRING_ERR_UNSUPPORTED, "Nq^2 exceeds 2^31");
    SPRING_CHECK(dalloc(c, b.g3, tot, "quartet scratch"));
    SPRING_CHECK(dalloc(c, b.rep, tot, "quartet scratch"));
    SPRING_CHECK(dalloc(c, b.pos, tot, "quartet scratch"));
    SPRING_CHECK(dalloc(c, b.total, 1, "quartet scratch"));
    if (want_all) SPRING_CHECK(dalloc(c, b.all, tot * 3, "Allq1q2q3"));
    Mesh3 m{{c->mesh[0], c->mesh[1], c->mesh[2]}};
    const int* q0v = c->d_irr_int.p + 3 * q0;
    const int threads = 256, blocks = (int)std::min<long long>((tot + threads - 1) / threads, 148LL * 32);
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "enumerate4: injected launch failure");
    k_enum4_flags<<<blocks, threads, 0, c->stream>>>(c->nq, m, q0v, c->d_qint.p, b.g3.p, b.rep.p);
    SPRING_CHECK(launch_check(c, "k_enum4_flags"));
    SPRING_CHECK(run_exclusive_scan(c, b.rep.p, b.pos.p, (int)tot));
    int last[2];
    SPRING_CHECK(d2h(c, &last[0], b.pos.p + tot - 1, sizeof(int), "quartet count"));
    SPRING_CHECK(d2h(c, &last[1], b.rep.p + tot - 1, sizeof(int), "quartet count"));
    const long long nquart = (long long)last[0] + last[1];
    SPRING_CHECK(dalloc(c, b.quart, std::max<long long>(nquart, 1), "quartet list"));
    SPRING_CHECK(zero(c, b.total.p, sizeof(unsigned long long), "quartet count"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "enumerate4: injected launch failure");
    k_enum4_write<<<blocks, threads, 0, c->stream>>>(c->nq, m, q0v, c->d_qint.p, b.g3.p, b.rep.p, b.pos.p,
                                                     want_all ? b.all.p : nullptr, d_perm, cap, b.quart.p, b.total.p);
    SPRING_CHECK(launch_check(c, "k_enum4_write"));
    unsigned long long total = 0;
    SPRING_CHECK(d2h(c, &total, b.total.p, sizeof total, "quartet total"));
    h_counts[0] = nquart;
    h_counts[1] = (long long)total;
    return SPRING_OK;
}

void free4(Enum4Bufs& b) {
    dfree(b.g3); dfree(b.rep); dfree(b.pos); dfree(b.all); dfree(b.quart); dfree(b.total);
}

}  // namespace

int run_enumerate4_fortran(spring_ctx* c, int q0, int* d_all, int* d_perm, long long cap, long long* h_counts) {
    Enum4Bufs b;
    int rc = enumerate4(c, q0, b, d_all != nullptr, d_perm, cap, h_counts);
    if (rc == SPRING_OK && d_all) {
        const size_t bytes = sizeof(int) * 3 * (size_t)c->nq * c->nq;
        cudaError_t e = cudaMemcpyAsync(d_all, b.all.p, bytes, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) rc = cuda_fail(c, e, "Allq1q2q3 copy");
    }
    cudaStreamSynchronize(c->stream);
    free4(b);
    return rc;
}

// Quartet list of q0 (0-based) in buffers kept by the context: (g1, g2, g3, 0) sorted by (g1, g2).
int run_enum4_list(spring_ctx* c, int q0, const int4** d_quart, long long* nquart) {
    if (!c->e4) c->e4 = new Enum4Bufs();
    Enum4Bufs& b = *static_cast<Enum4Bufs*>(c->e4);
    long long cnt[2] = {0, 0};
    SPRING_CHECK(enumerate4(c, q0, b, false, nullptr, 0, cnt));
    *d_quart = b.quart.p;
    *nquart = cnt[0];
    return SPRING_OK;
}

void free_enum4(spring_ctx* c) {
    if (!c->e4) return;
    Enum4Bufs* b = static_cast<Enum4Bufs*>(c->e4);
    free4(*b);
    delete b;
    c->e4 = nullptr;
}

int run_lw4(spring_ctx* c, int q0_first, int n_q0, int delta_mode, double sigma, const int* pol4, double* d_rate) {
    if (c->nb != NB || c->na4 > NA_MAX || c->nT > 9)
        return fail(c, SPRING_ERR_UNSUPPORTED, "four-phonon path handles two-atom cells, Na4 <= %d, <= 9 temperatures",
                    NA_MAX);
    V4Args a{};
    a.nq = c->nq;
    a.nT = c->nT;
    a.nq0 = c->nq0;
    a.na = c->na4;
    a.mfac = host_constants().Sctr4THz2 / (double(c->nq) * double(c->nq));
    a.onebysigma = delta_mode == SPRING_DELTA_GAUSS ? 1.0 / sigma : 0.0;
    a.onebysigma2 = a.onebysigma * a.onebysigma;
    for (int k = 0; k < 4; ++k) {
        a.pol_lo[k] = pol4 ? pol4[2 * k] - 1 : 0;
        a.pol_hi[k] = pol4 ? pol4[2 * k + 1] - 1 : N - 1;
    }
    const size_t smem = sizeof(V4Smem);
    cudaFuncSetAttribute(k_v4<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_v4<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    Enum4Bufs b;
    DBuf<double> wq;
    int rc = SPRING_OK;
    for (int q0 = q0_first; rc == SPRING_OK && q0 < q0_first + n_q0; ++q0) {
        long long cnt[2];
        rc = enumerate4(c, q0, b, delta_mode == SPRING_DELTA_TETRA, nullptr, 0, cnt);
        if (rc != SPRING_OK) break;
        a.q0 = q0;
        a.nquart = (int)cnt[0];
        const int groups = (a.nquart + QB - 1) / QB;
        const int grid = std::max(1, std::min(groups, 148 * 2));
        const double2* ev0 = c->ph_irr.evec.p + (size_t)q0 * 36;
        const double* om0 = c->ph_irr.omega.p + (size_t)q0 * N;
        const double* ob0 = c->ph_irr.oneby.p + (size_t)q0 * N;
        const double* nbe0 = c->ph_irr.nbe.p + (size_t)q0 * N;
        const int* q0i = c->d_irr_int.p + 3 * q0;
        if (delta_mode == SPRING_DELTA_GAUSS) {
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "v4: injected launch failure"); break; }
            k_v4<0><<<grid, 256, smem, c->stream>>>(a, b.quart.p, c->d_fc4.p, c->d_fc4_posr.p, c->d_fc4_btyp.p,
                                                    c->d_fc4_off.p, c->d_mass_rs.p, c->d_qpnt.p, q0i, ev0, om0, ob0,
                                                    nbe0, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p,
                                                    c->ph_grid.nbe.p, d_rate, nullptr);
            rc = launch_check(c, "k_v4<gauss>");
        } else {
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            const size_t need = (size_t)a.nquart * 1296 * sizeof(double);
            if (need > free_b / 2) {
                rc = fail(c, SPRING_ERR_UNSUPPORTED, "tetrahedron four-phonon W of one q0 needs %zu bytes", need);
                break;
            }
            if ((rc = dalloc(c, wq, (size_t)a.nquart * 1296, "quartet W")) != SPRING_OK) break;
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "v4: injected launch failure"); break; }
            k_v4<1><<<grid, 256, smem, c->stream>>>(a, b.quart.p, c->d_fc4.p, c->d_fc4_posr.p, c->d_fc4_btyp.p,
                                                    c->d_fc4_off.p, c->d_mass_rs.p, c->d_qpnt.p, q0i, ev0, om0, ob0,
                                                    nbe0, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p,
                                                    c->ph_grid.nbe.p, nullptr, wq.p);
            if ((rc = launch_check(c, "k_v4<wstore>")) != SPRING_OK) break;
            T4Args t{};
            t.nq = c->nq;
            t.nT = c->nT;
            t.nq0 = c->nq0;
            t.q0 = q0;
            t.ntet = 6 * c->nq;
            t.nquart = a.nquart;
            for (int k = 0; k < 4; ++k) {
                t.pol_lo[k] = a.pol_lo[k];
                t.pol_hi[k] = a.pol_hi[k];
            }
            const long long items = (long long)c->nq * t.ntet * (t.pol_hi[1] - t.pol_lo[1] + 1) *
                                    (t.pol_hi[2] - t.pol_lo[2] + 1) * (t.pol_hi[3] - t.pol_lo[3] + 1);
            const int tb = (int)std::max<long long>(1, std::min<long long>((items + 511) / 512, 148LL * 16));
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "tetra4: injected launch failure"); break; }
            k_tetra4<<<tb, 128, 0, c->stream>>>(t, reinterpret_cast<const int4*>(c->d_tetra.p), b.all.p, wq.p, q0i, om0,
                                                nbe0, c->ph_grid.omega.p, c->ph_grid.nbe.p, d_rate);
            rc = launch_check(c, "k_tetra4");
        }
    }
    cudaStreamSynchronize(c->stream);
    free4(b);
    dfree(wq);
    return rc;
}

}  // namespace spring
