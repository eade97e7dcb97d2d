// Point-defect scattering rate: T-matrix with the tetrahedron Green's function
// (ScatterRatePointDefect, src/Kappa/Src/point_defect_m.f90:139-376; the vertex coefficients of
// src/Kappa/Src/GreensFunc_m.f90:35-587).
//
// For an irreducible mode (q0, s0) with energy E0 = omega0^2, the reference sums over the
// tetrahedra of a second mesh (qMesh_pd) and every branch s
//   G(E0) = 1/NT sum_tet sum_s sum_v Coeff_v(E0) e_{q_v s} e_{q_v s}^H,
//   Coeff_v = d_v - i pi c_v     (d: real part by degeneracy type, c: delta-function weights),
// forms V = V_FC - E0 V_M, T = (1 - V G)^-1 V (or V + V G V) and the rate from the optical theorem,
// rho V_cell (-Im e0^H T e0) / omega0, or from a second tetrahedron sum of |e_qs^H T e0|^2.
//
// Regrouped for the GPU:
//   1. k_pd_weights, one thread per (item, q, s) of the defect mesh: w(q, s) = sum over the 24
//      tetrahedra that contain q of the coefficient at q's vertex (each tetrahedron's four energies
//      sorted in registers); no atomics, so the sums are deterministic;
//   2. k_pd_green, one CTA per item: G(a, b) = 1/NT sum_{q,s} w(q, s) e_a conj(e_b);
//   3. k_pd_tmatrix, one CTA per item: (1 - V G) T = V by Gaussian elimination with partial pivoting
//      in shared memory, then e0^H T e0, or T e0 for
//   4. k_pd_tetra (OptcTherm = .false.): -1/NT sum_{q,s} Im w(q, s) |e_qs^H T e0|^2.
// The delta weights c_v enter both G (as Im w) and step 4 (c = -Im w / pi).  FP64 throughout.
#include <algorithm>
#include <vector>

#include "spring_internal.cuh"

namespace spring {
namespace {

constexpr double PI_D = 3.141592653589793;
constexpr double ZERO_PREC_PD = 5.0e-5;  // degeneracy tolerance of GFcoeffv_RealPart
constexpr double CMP_PREC_PD = 1.0e-8;   // case bounds of DiracDeltaCoeffVertices_1984

__device__ __forceinline__ double sqd(double x) { return x * x; }
__device__ __forceinline__ double cbd(double x) { return x * x * x; }

// Real part of the vertex coefficients (GFcoeffv_RealPart, GreensFunc_m.f90:153-269) for sorted
// energies W[0..3]; the form follows the pattern of equal energies (within 5e-5).
__device__ void gf_real(const double* W, double E, double* d) {
    for (int v = 0; v < 4; ++v) d[v] = 0.0;
    bool chk[4] = {true, true, true, true};
    int same = 0, types = 0, p0a = 0, p0b = 0, p1a = 0;
    for (int i = 0; i < 4; ++i) {
        if (!chk[i]) continue;
        bool first = true;
        for (int j = i + 1; j < 4; ++j)
            if (fabs(W[i] - W[j]) < ZERO_PREC_PD) {
                if (same == 0) { p0a = i; p0b = j; }
                if (same == 1) p1a = i;
                ++same;
                if (first) { first = false; ++types; }
                chk[j] = false;
            }
    }
    if (same == 0) {  // all distinct (Type D, :450-496): vertex v with the others in cyclic order
        for (int v = 0; v < 4; ++v) {
            const double g1 = E - W[v], g2 = E - W[(v + 1) & 3], g3 = E - W[(v + 2) & 3], g4 = E - W[(v + 3) & 3];
            const double r2 = g2 / g1, r3 = g3 / g1, r4 = g4 / g1;
            const double q = 1.0 / ((1.0 - r2) * (1.0 - r3) * (1.0 - r4)) +
                             (1.0 / (sqd(1.0 - g1 / g2) * (1.0 - g3 / g2) * (1.0 - g4 / g2))) * (log(fabs(r2)) / r2) +
                             (1.0 / (sqd(1.0 - g1 / g3) * (1.0 - g2 / g3) * (1.0 - g4 / g3))) * (log(fabs(r3)) / r3) +
                             (1.0 / (sqd(1.0 - g1 / g4) * (1.0 - g2 / g4) * (1.0 - g3 / g4))) * (log(fabs(r4)) / r4);
            d[v] = q / g1;
        }
    } else if (same == 1) {  // one equal pair (l, m) (Type 0, :272-333)
        const int l = p0a, m = p0b;
        int j = -1, k = -1;
        for (int v = 0; v < 4; ++v)
            if (v != l && v != m) {
                if (j < 0) j = v;
                else k = v;
            }
        const double tj = (E - W[j]) / (W[m] - W[j]), tk = (E - W[k]) / (W[m] - W[k]);
        const double dlm = (cbd(E - W[j]) / ((W[j] - W[k]) * cbd(W[j] - W[m]))) * log(fabs(E - W[j])) +
                           (cbd(E - W[k]) / ((W[k] - W[j]) * cbd(W[k] - W[m]))) * log(fabs(E - W[k])) +
                           ((E - W[m]) / ((W[m] - W[j]) * (W[m] - W[k]))) *
                               (0.5 + tj + tk + (tj * tj + tk * tk + tj * tk) * log(fabs(E - W[m])));
        d[l] = dlm;
        d[m] = dlm;
        for (int t = 0; t < 2; ++t) {
            const int i = t == 0 ? j : k, o = t == 0 ? k : j;
            d[i] = (sqd(E - W[i]) / (sqd(W[i] - W[m]) * (W[o] - W[i]))) *
                       (1.0 + ((2.0 * (E - W[m]) / (W[i] - W[m])) + ((E - W[o]) / (W[i] - W[o]))) * log(fabs(E - W[i]))) +
                   (sqd(E - W[m]) / (sqd(W[m] - W[i]) * (W[o] - W[m]))) *
                       (1.0 + ((2.0 * (E - W[i]) / (W[m] - W[i])) + ((E - W[o]) / (W[m] - W[o]))) * log(fabs(E - W[m]))) +
                   (cbd(E - W[o]) / (sqd(W[o] - W[i]) * sqd(W[o] - W[m]))) * log(fabs(E - W[o]));
        }
    } else if (same == 2 && types == 1 && p0a == p1a && (p0a == 0 || p0a == 1)) {
        // three equal: vertices 1-3 (Type 1, :336-371) or 2-4 (Type 3, :374-409)
        const bool low = p0a == 0;
        const int a = low ? 0 : 1, b = low ? 3 : 0;  // a: one of the three, b: the odd one
        const double ga = E - W[a], gb = E - W[b];
        const double rba = gb / ga, rab = ga / gb;
        const double q = 11.0 / (6.0 * (1.0 - rba)) - 5.0 / (2.0 * sqd(1.0 - rba)) + 1.0 / cbd(1.0 - rba) +
                         log(fabs(rba)) / (sqd(sqd(1.0 - rab)) * rba);
        const double db = ((3.0 / sqd(1.0 - rba) - 6.0 / cbd(1.0 - rba) + 3.0 / sqd(sqd(1.0 - rba))) * (log(fabs(rab)) / rab) +
                           1.0 / cbd(1.0 - rab) + 2.5 * rba / sqd(1.0 - rba) - 2.0 * rba / cbd(1.0 - rba)) / gb;
        for (int v = 0; v < 4; ++v) d[v] = v == b ? db : q / ga;
    } else if (same == 2 && types == 2) {  // two equal pairs, 1 = 2 and 3 = 4 (Type 2, :412-447)
        const double g1 = E - W[0], g3 = E - W[2];
        const double r31 = g3 / g1, r13 = g1 / g3;
        const double q12 = 2.5 / sqd(1.0 - r31) - 2.0 / cbd(1.0 - r31) + r13 / cbd(1.0 - r13) +
                           3.0 * (1.0 / cbd(1.0 - r13) - 1.0 / sqd(sqd(1.0 - r13))) * (log(fabs(r31)) / r31);
        const double q34 = 2.5 / sqd(1.0 - r13) - 2.0 / cbd(1.0 - r13) + r31 / cbd(1.0 - r31) +
                           3.0 * (1.0 / cbd(1.0 - r31) - 1.0 / sqd(sqd(1.0 - r31))) * (log(fabs(r13)) / r13);
        d[0] = d[1] = q12 / g1;
        d[2] = d[3] = q34 / g3;
    } else if (same == 3) {  // all four equal
        for (int v = 0; v < 4; ++v) d[v] = 0.25 / (E - W[0]);
    }
}

// Delta-function weights at the sorted vertices (DiracDeltaCoeffVertices_1984, :499-587).
__device__ void gf_delta(const double* Ev, double E, double* c) {
    const double E1 = Ev[0], E2 = Ev[1], E3 = Ev[2], E4 = Ev[3];
    if ((E1 - E) <= CMP_PREC_PD && (E - E2) <= CMP_PREC_PD) {
        const double t = cbd(E - E1);
        c[0] = ((E2 - E) / (E2 - E1) + (E3 - E) / (E3 - E1) + (E4 - E) / (E4 - E1)) *
               (sqd(E - E1) / ((E4 - E1) * (E3 - E1) * (E2 - E1)));
        c[1] = t / (sqd(E2 - E1) * (E3 - E1) * (E4 - E1));
        c[2] = t / ((E2 - E1) * sqd(E3 - E1) * (E4 - E1));
        c[3] = t / ((E2 - E1) * (E3 - E1) * sqd(E4 - E1));
    } else if ((E2 - E) <= CMP_PREC_PD && (E - E3) <= CMP_PREC_PD) {
        // the six products that recur in the four weights
        const double A = ((E3 - E) * (E - E2)) / ((E4 - E2) * (E3 - E2)) + ((E4 - E) * (E - E1)) / ((E4 - E1) * (E4 - E2)) +
                         ((E3 - E) * (E - E1)) / ((E3 - E2) * (E4 - E1));
        const double B = ((E4 - E) * (E - E1)) / ((E4 - E2) * (E3 - E1)) + ((E4 - E) * (E - E2)) / ((E4 - E2) * (E3 - E2)) +
                         ((E3 - E) * (E - E1)) / ((E3 - E1) * (E3 - E2));
        const double C = ((E3 - E) * (E - E2)) / ((E4 - E2) * (E3 - E1)) + ((E4 - E) * (E - E2)) / ((E4 - E2) * (E4 - E1)) +
                         ((E3 - E) * (E - E1)) / ((E3 - E1) * (E4 - E1));
        const double D = ((E3 - E) * (E - E2)) / ((E3 - E2) * (E3 - E1)) + ((E4 - E) * (E - E1)) / ((E4 - E1) * (E3 - E1)) +
                         ((E4 - E) * (E - E2)) / ((E3 - E2) * (E4 - E1));
        c[0] = 0.5 * (((E3 - E) / sqd(E3 - E1)) * A + ((E4 - E) / sqd(E4 - E1)) * B);
        c[1] = 0.5 * (((E3 - E) / sqd(E3 - E2)) * C + ((E4 - E) / sqd(E4 - E2)) * D);
        c[2] = 0.5 * (((E - E2) / sqd(E3 - E2)) * C + ((E - E1) / sqd(E3 - E1)) * A);
        c[3] = 0.5 * (((E - E2) / sqd(E4 - E2)) * D + ((E - E1) / sqd(E4 - E1)) * B);
    } else if ((E3 - E) <= CMP_PREC_PD && (E - E4) <= CMP_PREC_PD) {
        const double t = cbd(E4 - E);
        c[0] = t / (sqd(E4 - E1) * (E4 - E2) * (E4 - E3));
        c[1] = t / ((E4 - E1) * sqd(E4 - E2) * (E4 - E3));
        c[2] = t / ((E4 - E1) * (E4 - E2) * sqd(E4 - E3));
        c[3] = ((E - E3) / (E4 - E3) + (E - E2) / (E4 - E2) + (E - E1) / (E4 - E1)) *
               (sqd(E4 - E) / ((E4 - E1) * (E4 - E2) * (E4 - E3)));
    } else {
        c[0] = c[1] = c[2] = c[3] = 0.0;
    }
}

struct PdArgs {
    int n, nq, i0_first, n_items;
    double inv_nt, rho_vol;
};

// w(item, q, s) = sum over the tetrahedra containing q of Coeff at q's vertex (item = (q0, s0)).
__global__ void __launch_bounds__(128) k_pd_weights(PdArgs a, const int* __restrict__ inc, const int4* __restrict__ tet,
                                                    const double* __restrict__ w2, const double* __restrict__ om0,
                                                    double2* __restrict__ wgt) {
    const long long total = (long long)a.n_items * a.nq * a.n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int item = (int)(t / ((long long)a.nq * a.n));
        const int r = (int)(t % ((long long)a.nq * a.n));
        const int q = r / a.n, s = r % a.n;
        const int i0 = a.i0_first + item / a.n, s0 = item % a.n;
        const double w0 = om0[(size_t)i0 * a.n + s0], E = w0 * w0;
        double2 acc = make_double2(0.0, 0.0);
        for (int k = 0; k < 24; ++k) {
            const int code = inc[(size_t)q * 24 + k];
            const int4 tv = tet[code >> 2];
            const int vert[4] = {tv.x, tv.y, tv.z, tv.w};
            double W[4];
            int slot[4];
            for (int v = 0; v < 4; ++v) {
                W[v] = w2[(size_t)vert[v] * a.n + s];
                slot[v] = v;
            }
            // stable insertion sort of the four energies with their slots (my_sort_GF)
            for (int i = 1; i < 4; ++i)
                for (int j = i; j > 0 && W[j - 1] > W[j]; --j) {
                    const double x = W[j]; W[j] = W[j - 1]; W[j - 1] = x;
                    const int y = slot[j]; slot[j] = slot[j - 1]; slot[j - 1] = y;
                }
            double d[4], c[4];
            gf_real(W, E, d);
            gf_delta(W, E, c);
            const int mine = code & 3;
            for (int v = 0; v < 4; ++v)
                if (slot[v] == mine) {
                    const double re = isnan(d[v]) ? 0.0 : d[v];
                    const double im = isnan(c[v]) ? 0.0 : -PI_D * c[v];
                    acc.x += re;
                    acc.y += im;
                }
        }
        wgt[t] = acc;
    }
}

// G(item)(a, b) = 1/NT sum_{q, s} w e_a conj(e_b); entries split over J thread groups.
__global__ void __launch_bounds__(256) k_pd_green(PdArgs a, const double2* __restrict__ wgt,
                                                  const double2* __restrict__ evec, double2* __restrict__ G) {
    extern __shared__ double2 pd_red[];
    const int item = blockIdx.x, n = a.n, E = n * n;
    if (E > (int)blockDim.x) {  // large cells: each thread sums whole entries
        const double2* w = wgt + (size_t)item * a.nq * n;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
            const int ra = e % n, cb = e / n;
            double2 acc = make_double2(0.0, 0.0);
            for (int qs = 0; qs < a.nq * n; ++qs) {
                const double2 x = w[qs];
                const double2 ea = evec[(size_t)qs * n + ra], eb = evec[(size_t)qs * n + cb];
                const double2 p = make_double2(ea.x * eb.x + ea.y * eb.y, ea.y * eb.x - ea.x * eb.y);
                acc.x += x.x * p.x - x.y * p.y;
                acc.y += x.x * p.y + x.y * p.x;
            }
            G[(size_t)item * E + e] = make_double2(acc.x * a.inv_nt, acc.y * a.inv_nt);
        }
        return;
    }
    const int J = max(1, (int)blockDim.x / E);
    const int e = threadIdx.x % E, j = threadIdx.x / E;
    const int ra = e % n, cb = e / n;  // G(ra, cb), column-major
    double2 acc = make_double2(0.0, 0.0);
    if (j < J && threadIdx.x < J * E) {
        const double2* w = wgt + (size_t)item * a.nq * n;
        for (int qs = j; qs < a.nq * n; qs += J) {
            const double2 x = w[qs];
            if (x.x == 0.0 && x.y == 0.0) continue;
            const double2* ev = evec + (size_t)qs * n;  // e_{q,s}(row) = evec[q][s][row]
            const double2 ea = ev[ra], eb = ev[cb];
            const double2 p = make_double2(ea.x * eb.x + ea.y * eb.y, ea.y * eb.x - ea.x * eb.y);  // ea conj(eb)
            acc.x += x.x * p.x - x.y * p.y;
            acc.y += x.x * p.y + x.y * p.x;
        }
    }
    if (threadIdx.x < J * E) pd_red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < E) {
        double2 s = make_double2(0.0, 0.0);
        for (int jj = 0; jj < J; ++jj) {
            s.x += pd_red[jj * E + threadIdx.x].x;
            s.y += pd_red[jj * E + threadIdx.x].y;
        }
        G[(size_t)item * E + threadIdx.x] = make_double2(s.x * a.inv_nt, s.y * a.inv_nt);
    }
}

__device__ __forceinline__ double2 cmulp(double2 x, double2 y) {
    return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}

// T-matrix of one item.  rate(item) from the optical theorem, and T e0 (for the tetrahedron form).
// Shared: M (n x n), R (n x n, right-hand side V then T), V (n x n real), e0 (n), piv info.
__global__ void __launch_bounds__(128) k_pd_tmatrix(PdArgs a, const double2* __restrict__ G, const double* __restrict__ vfc,
                                                    const double* __restrict__ vm, const double2* __restrict__ ev0,
                                                    const double* __restrict__ om0, const int* __restrict__ gamma0,
                                                    int mat_inv_full, double* __restrict__ rate, double2* __restrict__ te0) {
    extern __shared__ double2 pd_sm[];
    const int n = a.n, E = n * n, tid = threadIdx.x, T = blockDim.x;
    double2* M = pd_sm;         // 1 - V G
    double2* R = M + E;         // V, then T
    double2* VG = R + E;        // V G
    double* V = reinterpret_cast<double*>(VG + E);
    __shared__ int s_piv, s_sing;
    const int item = blockIdx.x;
    const int i0 = a.i0_first + item / n, s0 = item % n;
    const double w0 = om0[(size_t)i0 * n + s0], E0 = w0 * w0;
    const bool skip = gamma0[i0] && s0 < 3;
    for (int i = tid; i < E; i += T) V[i] = vfc[i] - E0 * vm[i];
    __syncthreads();
    const double2* Gi = G + (size_t)item * E;
    for (int i = tid; i < E; i += T) {  // VG(r, c) = sum_k V(r, k) G(k, c), column-major
        const int r = i % n, c = i / n;
        double2 s = make_double2(0.0, 0.0);
        for (int k = 0; k < n; ++k) {
            const double v = V[r + n * k];
            const double2 g = Gi[k + n * c];
            s.x += v * g.x;
            s.y += v * g.y;
        }
        VG[i] = s;
        M[i] = make_double2((r == c ? 1.0 : 0.0) - s.x, -s.y);
        R[i] = make_double2(V[i], 0.0);
    }
    if (tid == 0) s_sing = 0;
    __syncthreads();
    if (mat_inv_full) {  // Gaussian elimination with partial pivoting on [M | R]
        for (int k = 0; k < n; ++k) {
            if (tid == 0) {
                int p = k;
                double best = -1.0;
                for (int i = k; i < n; ++i) {
                    const double2 x = M[i + n * k];
                    const double m = hypot(x.x, x.y);
                    if (m > best) { best = m; p = i; }
                }
                s_piv = p;
                if (best == 0.0) s_sing = 1;
            }
            __syncthreads();
            if (s_sing) break;
            const int p = s_piv;
            if (p != k)
                for (int c = tid; c < 2 * n; c += T) {
                    double2* X = c < n ? M : R;
                    const int cc = c % n;
                    const double2 t = X[k + n * cc];
                    X[k + n * cc] = X[p + n * cc];
                    X[p + n * cc] = t;
                }
            __syncthreads();
            const double2 piv = M[k + n * k];
            const double den = piv.x * piv.x + piv.y * piv.y;
            for (int w = tid; w < (n - 1) * 2 * n; w += T) {  // rows i != k, columns of [M | R]
                int i = w / (2 * n);
                if (i >= k) ++i;
                const int c = w % (2 * n);
                double2* X = c < n ? M : R;
                const int cc = c % n;
                if (c < n && cc <= k) continue;  // M columns left of k+1 are not needed again
                const double2 mi = M[i + n * k];
                const double2 f = make_double2((mi.x * piv.x + mi.y * piv.y) / den, (mi.y * piv.x - mi.x * piv.y) / den);
                const double2 xk = X[k + n * cc];
                const double2 pr = cmulp(f, xk);
                X[i + n * cc].x -= pr.x;
                X[i + n * cc].y -= pr.y;
            }
            __syncthreads();
        }
        if (!s_sing)
            for (int w = tid; w < E; w += T) {  // divide each row of R by its pivot
                const int i = w % n;
                const double2 piv = M[i + n * i];
                const double den = piv.x * piv.x + piv.y * piv.y;
                const double2 x = R[w];
                R[w] = make_double2((x.x * piv.x + x.y * piv.y) / den, (x.y * piv.x - x.x * piv.y) / den);
            }
        __syncthreads();
    }
    if (!mat_inv_full || s_sing) {  // T = V + V G V
        for (int i = tid; i < E; i += T) {
            const int r = i % n, c = i / n;
            double2 s = make_double2(V[r + n * c], 0.0);
            for (int k = 0; k < n; ++k) {
                const double2 x = VG[r + n * k];
                const double v = V[k + n * c];
                s.x += x.x * v;
                s.y += x.y * v;
            }
            R[i] = s;
        }
        __syncthreads();
    }
    // T e0 and e0^H T e0
    const double2* e0 = ev0 + ((size_t)i0 * n + s0) * n;
    double2* Te = M;  // reuse
    for (int r = tid; r < n; r += T) {
        double2 s = make_double2(0.0, 0.0);
        for (int k = 0; k < n; ++k) {
            const double2 p = cmulp(R[r + n * k], e0[k]);
            s.x += p.x;
            s.y += p.y;
        }
        Te[r] = s;
        if (te0) te0[(size_t)item * n + r] = skip ? make_double2(0.0, 0.0) : s;
    }
    __syncthreads();
    if (tid == 0) {
        double im = 0.0;
        for (int r = 0; r < n; ++r) im += e0[r].x * Te[r].y - e0[r].y * Te[r].x;  // Im(conj(e0) . Te)
        rate[item] = skip ? 0.0 : a.rho_vol * (-im / w0);
    }
}

// Tetrahedron form of the rate: -1/NT sum_{q,s} Im w |e_qs^H T e0|^2 rho V / omega0 (one CTA per item).
__global__ void __launch_bounds__(256) k_pd_tetra(PdArgs a, const double2* __restrict__ wgt, const double2* __restrict__ evec,
                                                  const double2* __restrict__ te0, const double* __restrict__ om0,
                                                  const int* __restrict__ gamma0, double* __restrict__ rate) {
    __shared__ double red[256];
    const int item = blockIdx.x, n = a.n;
    const int i0 = a.i0_first + item / n, s0 = item % n;
    const double2* w = wgt + (size_t)item * a.nq * n;
    const double2* t = te0 + (size_t)item * n;
    double acc = 0.0;
    for (int qs = threadIdx.x; qs < a.nq * n; qs += blockDim.x) {
        const double im = w[qs].y;
        if (im == 0.0) continue;
        const double2* e = evec + (size_t)qs * n;
        double2 d = make_double2(0.0, 0.0);
        for (int r = 0; r < n; ++r) {  // conj(e) . T e0
            d.x += e[r].x * t[r].x + e[r].y * t[r].y;
            d.y += e[r].x * t[r].y - e[r].y * t[r].x;
        }
        acc -= im * (d.x * d.x + d.y * d.y);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double w0 = om0[(size_t)i0 * n + s0];
        rate[item] = (gamma0[i0] && s0 < 3) ? 0.0 : a.rho_vol * red[0] * a.inv_nt / w0;
    }
}

// LW_Allq0(T, q0, s) += 0.5 rate(q0, s) for every temperature.
__global__ void k_pd_add(int n, int nq0, int nT, int i0_first, int n_q0, const double* __restrict__ rate,
                         double* __restrict__ lw) {
    const int per = n_q0 * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nT * per; i += gridDim.x * blockDim.x) {
        const int T = i / per, j = i % per;
        lw[((size_t)T * nq0 + i0_first) * n + j] += 0.5 * rate[j];
    }
}

}  // namespace

int set_point_defect(spring_ctx* c, const int* qmesh, int na_p, const int* num_p, const int* idx_p, const double* fc_p,
                     const double* mass_def, double rho, int mat_inv_full, int optc_therm) {
    PointDefectDev& P = c->pd;
    if (!qmesh) {
        P.on = false;
        return SPRING_OK;
    }
    const int nb = c->nb, n = c->ndof;
    for (int k = 0; k < 3; ++k)
        if (qmesh[k] < 1) return fail(c, SPRING_ERR_ARG, "qMesh_pd must be positive");
    if (!num_p || !idx_p || !fc_p || !mass_def || na_p < 1) return fail(c, SPRING_ERR_ARG, "point defect: NULL inputs");
    for (int mu = 0; mu < nb; ++mu) {
        if (num_p[mu] < 0 || num_p[mu] > na_p) return fail(c, SPRING_ERR_ARG, "perturbed FC2 atm_num out of range");
        if (!(mass_def[mu] > 0.0)) return fail(c, SPRING_ERR_ARG, "Mass_def must be positive");
    }
    // PerturbationMatrix (point_defect_m.f90:40-108): home-cell blocks, pristine vs perturbed
    const double wthz = host_constants().wTHz;
    auto ifc2 = [&](int na, const int* num, const int* idx, const double* fc, int mu, int nu, int al, int be) {
        for (int N = 0; N < num[mu]; ++N) {
            const int* e = idx + 4 * (N + (size_t)na * mu);
            if (e[3] - 1 == nu && e[0] == 0 && e[1] == 0 && e[2] == 0) return fc[be + 3 * al + 9 * N + (size_t)9 * na * mu];
        }
        return 0.0;
    };
    std::vector<double> vfc((size_t)n * n, 0.0), vm((size_t)n * n, 0.0);
    for (int nu = 0; nu < nb; ++nu)
        for (int be = 0; be < 3; ++be)
            for (int mu = 0; mu < nb; ++mu)
                for (int al = 0; al < 3; ++al) {
                    const int row = 3 * mu + al, col = 3 * nu + be;
                    const double p = ifc2(c->na2, c->h_fc2_num.data(), c->h_fc2_idx.data(), c->h_fc2.data(), mu, nu, al, be);
                    const double d = ifc2(na_p, num_p, idx_p, fc_p, mu, nu, al, be);
                    vfc[row + (size_t)n * col] = (d - p) / std::sqrt(c->mass[mu] * c->mass[nu]) * (wthz * wthz);
                    if (mu == nu && al == be) vm[row + (size_t)n * col] = (mass_def[mu] - c->mass[mu]) / c->mass[mu];
                }
    const int nq = qmesh[0] * qmesh[1] * qmesh[2];
    SPRING_CHECK(dalloc(c, P.vfc, (size_t)n * n, "point-defect V"));
    SPRING_CHECK(dalloc(c, P.vm, (size_t)n * n, "point-defect V"));
    SPRING_CHECK(h2d(c, P.vfc.p, vfc.data(), sizeof(double) * n * n, "point-defect V"));
    SPRING_CHECK(h2d(c, P.vm.p, vm.data(), sizeof(double) * n * n, "point-defect V"));
    // the defect mesh (make_tetrahedron with ZeroCentered, the run's shift) and its phonons
    SPRING_CHECK(dalloc(c, P.qint, (size_t)nq * 3, "defect mesh"));
    SPRING_CHECK(dalloc(c, P.qpnt, (size_t)nq * 3, "defect mesh"));
    SPRING_CHECK(dalloc(c, P.tet, (size_t)nq * 24, "defect mesh"));
    SPRING_CHECK(run_make_mesh_on(c, qmesh, c->mesh_shift, 1, P.qint.p, P.qpnt.p, P.tet.p));
    std::vector<int> tet((size_t)nq * 24);
    SPRING_CHECK(d2h(c, tet.data(), P.tet.p, sizeof(int) * tet.size(), "defect tetrahedra"));
    // every grid point is a vertex of 24 tetrahedra: (tet << 2 | slot) per incidence
    std::vector<int> inc((size_t)nq * 24), fill(nq, 0);
    for (int t = 0; t < 6 * nq; ++t)
        for (int v = 0; v < 4; ++v) {
            const int q = tet[4 * (size_t)t + v];
            if (q < 0 || q >= nq || fill[q] >= 24) return fail(c, SPRING_ERR_UNSUPPORTED, "defect mesh: irregular tetrahedra");
            inc[(size_t)q * 24 + fill[q]++] = (t << 2) | v;
        }
    for (int q = 0; q < nq; ++q)
        if (fill[q] != 24) return fail(c, SPRING_ERR_UNSUPPORTED, "defect mesh: irregular tetrahedra");
    SPRING_CHECK(dalloc(c, P.inc, inc.size(), "defect incidences"));
    SPRING_CHECK(h2d(c, P.inc.p, inc.data(), sizeof(int) * inc.size(), "defect incidences"));
    SPRING_CHECK(alloc_phonons(c, P.ph, nq));
    SPRING_CHECK(run_phonons(c, P.ph, P.qpnt.p, nq, 0));
    P.nq = nq;
    P.rho = rho;
    P.mat_inv_full = mat_inv_full != 0;
    P.optc_therm = optc_therm != 0;
    P.on = true;
    return SPRING_OK;
}

int run_point_defect(spring_ctx* c, int i0_first, int n_q0, double* d_rate) {
    PointDefectDev& P = c->pd;
    const int n = c->ndof, nq = P.nq;
    // omega^2 of the defect mesh
    std::vector<double> om((size_t)nq * n);
    SPRING_CHECK(d2h(c, om.data(), P.ph.omega.p, sizeof(double) * om.size(), "defect phonons"));
    for (double& w : om) w = w * w;
    SPRING_CHECK(dalloc(c, P.w2, om.size(), "defect energies"));
    SPRING_CHECK(h2d(c, P.w2.p, om.data(), sizeof(double) * om.size(), "defect energies"));
    // Gamma flags of the irreducible points
    std::vector<int> g0(c->nq0);
    for (int i = 0; i < c->nq0; ++i)
        g0[i] = c->h_irr_int[3 * i] == 0 && c->h_irr_int[3 * i + 1] == 0 && c->h_irr_int[3 * i + 2] == 0;
    SPRING_CHECK(dalloc(c, P.gamma0, c->nq0, "Gamma flags"));
    SPRING_CHECK(h2d(c, P.gamma0.p, g0.data(), sizeof(int) * c->nq0, "Gamma flags"));
    // items in blocks so that the weights stay within ~1 GB
    const size_t per_item = (size_t)nq * n * sizeof(double2);
    const int blk_q0 = (int)std::max<size_t>(1, std::min<size_t>(n_q0, ((size_t)1 << 30) / (per_item * n)));
    int rc = SPRING_OK;
    for (int b = 0; b < n_q0 && rc == SPRING_OK; b += blk_q0) {
        const int nb0 = std::min(blk_q0, n_q0 - b), items = nb0 * n;
        PdArgs a{};
        a.n = n;
        a.nq = nq;
        a.i0_first = i0_first + b;
        a.n_items = items;
        a.inv_nt = 1.0 / (6.0 * nq);
        a.rho_vol = P.rho * c->vol;
        if ((rc = dalloc(c, P.wgt, (size_t)items * nq * n, "defect weights")) != SPRING_OK) break;
        if ((rc = dalloc(c, P.G, (size_t)items * n * n, "defect Green's functions")) != SPRING_OK) break;
        if ((rc = dalloc(c, P.te0, (size_t)items * n, "defect T e0")) != SPRING_OK) break;
        if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "point defect: injected launch failure"); break; }
        const long long tot = (long long)items * nq * n;
        k_pd_weights<<<(int)std::min<long long>((tot + 127) / 128, 148LL * 32), 128, 0, c->stream>>>(
            a, P.inc.p, reinterpret_cast<const int4*>(P.tet.p), P.w2.p, c->ph_irr.omega.p, P.wgt.p);
        if ((rc = launch_check(c, "k_pd_weights")) != SPRING_OK) break;
        const int E = n * n, J = std::max(1, 256 / E), gthreads = E > 256 ? 256 : J * E;
        k_pd_green<<<items, gthreads, sizeof(double2) * gthreads, c->stream>>>(a, P.wgt.p, P.ph.evec.p, P.G.p);
        if ((rc = launch_check(c, "k_pd_green")) != SPRING_OK) break;
        const size_t sm = sizeof(double2) * 3 * E + sizeof(double) * E;
        if (sm > 48 * 1024) cudaFuncSetAttribute(k_pd_tmatrix, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pd_tmatrix<<<items, 128, sm, c->stream>>>(a, P.G.p, P.vfc.p, P.vm.p, c->ph_irr.evec.p, c->ph_irr.omega.p,
                                                   P.gamma0.p, P.mat_inv_full ? 1 : 0, d_rate + (size_t)b * n, P.te0.p);
        if ((rc = launch_check(c, "k_pd_tmatrix")) != SPRING_OK) break;
        if (!P.optc_therm) {
            k_pd_tetra<<<items, 256, 0, c->stream>>>(a, P.wgt.p, P.ph.evec.p, P.te0.p, c->ph_irr.omega.p, P.gamma0.p,
                                                    d_rate + (size_t)b * n);
            if ((rc = launch_check(c, "k_pd_tetra")) != SPRING_OK) break;
        }
    }
    return rc;
}

int run_point_defect_add(spring_ctx* c, int i0_first, int n_q0, const double* d_rate) {
    const int total = c->nT * n_q0 * c->ndof;
    if (total == 0) return SPRING_OK;
    k_pd_add<<<(total + 255) / 256, 256, 0, c->stream>>>(c->ndof, c->nq0, c->nT, i0_first, n_q0, d_rate, c->d_lw_all.p);
    return launch_check(c, "k_pd_add");
}

}  // namespace spring
