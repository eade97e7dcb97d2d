// Harmonic phonons on the device: get_phonon (src/Kappa/Src/DynaMat_mod.f90:486-709)
// for a batch of q-points, one CTA per q-point.
//   1. D(q) and dD/dq_k from FC2 (DynMatgv_SR, DynaMat_mod.f90:98-190).
//   2. Hermitian eigensolve in FP64 by cyclic complex Jacobi with round-robin
//      (parallel) pair ordering: n/2 disjoint rotations per step, column
//      updates then row updates, until the off-diagonal mass is below 1e-30 of
//      the diagonal's or a sweep finds no element above 1e-16 sqrt|a_pp a_qq|
//      (threshold Jacobi).  Eigenvalues ascending like LAPACK zheevd.  The
//      eigenvector phase (gauge) is the eigensolver's own: only gauge-invariant
//      quantities are comparable with LAPACK's.
//   3. omega = sqrt|lambda| (negative for imaginary modes), v = Re(e^H dD e)/(2 omega),
//      nBE for every temperature, 1/(omega wTHz); Gamma acoustic modes zeroed.
//   4. On a Gamma-centred mesh only one point of each (q, -q) pair is solved: the
//      other gets e(-q) = conj(e(q)) (D(-q) = D(q)* for real force constants),
//      the same omega, 1/omega and nBE, and v(-q) = -v(q).  The irreducible
//      points run in the same launch.
// FP64 ALU bound (~10 n^3 flops per sweep).
#include <algorithm>
#include <vector>

#include "spring_internal.cuh"

namespace spring {
namespace {

struct PhArgs {
    int nb, n, na2;
    double latvec[9];
    double wTHz, vg_ms, BEConv;
    int nT;
    const double2* dd;  // dipole-dipole D and dD/dq per work item ([4][n][n]), or null
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

constexpr int MAX_SWEEPS = 30;

// Outputs of one set of q-points: [q][s][row] eigenvectors, [q][s] scalars, [T][nq][s] nBE,
// [q][s][3] velocities; q vectors qpts[q][3].
struct PhSet {
    const double* qpts;
    double2* evec;
    double* omega;
    double* oneby;
    double* nbe;
    double* vel;
    int nq;
};

// Work item i < n_a: point list_a[i] (or i when list_a is null) of set SA; else point i - n_a of set SB.
__global__ void __launch_bounds__(128, 8) k_phonons(PhArgs a, PhSet SA, const int* __restrict__ list_a, int n_a,
                                                    PhSet SB, int n_b, const double* __restrict__ fc2,
                                                    const int* __restrict__ idx, const int* __restrict__ num,
                                                    const double* __restrict__ mrs, const double* __restrict__ temps) {
    extern __shared__ double2 sm[];
    const int n = a.n;
    const int m = n + (n & 1);  // even size for round-robin pairing (index n is a dummy)
    double2* A = sm;             // [n][n]
    double2* V = A + n * n;      // [n][n]
    double2* dD = V + n * n;     // [3][n][n]
    double2* rotE = dD + 3 * n * n;               // [m/2] e^{i phi}
    double* rotC = reinterpret_cast<double*>(rotE + m / 2);  // [m/2]
    double* rotS = rotC + m / 2;                             // [m/2]
    double* red = rotS + m / 2;                              // [2] reduction
    int* rotP = reinterpret_cast<int*>(red + 2);             // [m/2]
    int* rotQ = rotP + m / 2;                                // [m/2]
    int* rank = rotQ + m / 2;                                // [n]
    __shared__ int nrot;                                     // rotations applied in this sweep
    double* lam = reinterpret_cast<double*>(rank + n + (n & 1));  // [n]

    const int tid = threadIdx.x, nt = blockDim.x;
    for (int item = blockIdx.x; item < n_a + n_b; item += gridDim.x) {
        const bool in_a = item < n_a;
        const PhSet& P = in_a ? SA : SB;
        const int q = in_a ? (list_a ? list_a[item] : item) : item - n_a;
        const int nq = P.nq;
        double2* __restrict__ evec = P.evec;
        double* __restrict__ omega = P.omega;
        double* __restrict__ oneby = P.oneby;
        double* __restrict__ nbe = P.nbe;
        double* __restrict__ vel = P.vel;
        const double qx = P.qpts[3 * q], qy = P.qpts[3 * q + 1], qz = P.qpts[3 * q + 2];
        for (int i = tid; i < 5 * n * n; i += nt) A[i] = make_double2(0.0, 0.0);  // A, V, dD
        __syncthreads();
        // --- D(q), dD/dq: thread per (mu, alpha, beta); neighbours in reference order
        for (int w = tid; w < a.nb * 9; w += nt) {
            const int mu = w / 9, al = (w / 3) % 3, be = w % 3;
            const int row = 3 * mu + al;
            for (int N = 0; N < num[mu]; ++N) {
                const int* e = idx + 4 * (N + a.na2 * mu);
                const int nu = e[3] - 1;
                double R[3];
                for (int r = 0; r < 3; ++r)
                    R[r] = a.latvec[r] * e[0] + a.latvec[r + 3] * e[1] + a.latvec[r + 6] * e[2];
                const double qr = qx * R[0] + qy * R[1] + qz * R[2];
                double sn, cs;
                sincos(qr, &sn, &cs);
                const double f = fc2[((mu * a.na2 + N) * 3 + al) * 3 + be];  // fC(1,be,al,N,mu)
                const double mf = mrs[mu] * mrs[nu];
                const int col = 3 * nu + be;
                double2 t = make_double2(f * cs * mf, f * sn * mf);
                A[row * n + col] = cadd(A[row * n + col], t);
                for (int k = 0; k < 3; ++k)  // (i R_k) * t
                    dD[(k * n + row) * n + col] = cadd(dD[(k * n + row) * n + col], make_double2(-t.y * R[k], t.x * R[k]));
            }
        }
        __syncthreads();
        if (a.dd) {  // + DynEw, dDynEw/dq (LongEw); then the lower triangle from the upper one, as zheevd('U')
            const double2* d = a.dd + (size_t)item * 4 * n * n;
            for (int i = tid; i < 4 * n * n; i += nt) {
                double2& t = i < n * n ? A[i] : dD[i - n * n];
                t = cadd(t, d[i]);
            }
            __syncthreads();
            for (int i = tid; i < n * n; i += nt) {
                const int r = i / n, cc = i % n;
                if (r > cc) A[i] = conj2(A[cc * n + r]);
                else if (r == cc) A[i].y = 0.0;
            }
        }
        for (int i = tid; i < n; i += nt) V[i * n + i] = make_double2(1.0, 0.0);
        __syncthreads();

        // --- cyclic complex Jacobi
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            if (nt == 32) {  // one warp: lane-parallel sums
                double off = 0.0, dg = 0.0;
                for (int w = tid; w < n * n; w += 32) {
                    const int i = w / n, j = w % n;
                    const double2 z = A[w];
                    if (i == j) dg += z.x * z.x;
                    else if (j > i) off += z.x * z.x + z.y * z.y;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    off += __shfl_xor_sync(0xffffffffu, off, o);
                    dg += __shfl_xor_sync(0xffffffffu, dg, o);
                }
                if (tid == 0) {
                    nrot = 0;
                    red[0] = off;
                    red[1] = dg;
                }
            } else if (tid == 0) {
                nrot = 0;
                double off = 0.0, dg = 0.0;
                for (int i = 0; i < n; ++i) {
                    dg += A[i * n + i].x * A[i * n + i].x;
                    for (int j = i + 1; j < n; ++j) off += A[i * n + j].x * A[i * n + j].x + A[i * n + j].y * A[i * n + j].y;
                }
                red[0] = off;
                red[1] = dg;
            }
            __syncthreads();
            const bool done = red[0] <= 1e-30 * red[1] || red[0] == 0.0;
            __syncthreads();
            if (done) break;
            for (int r = 0; r < m - 1; ++r) {
                for (int k = tid; k < m / 2; k += nt) {
                    int p, qq;
                    if (k == 0) { p = r; qq = m - 1; }
                    else { p = (r + k) % (m - 1); qq = (r - k + (m - 1)) % (m - 1); }
                    if (p > qq) { int t = p; p = qq; qq = t; }
                    double c = 1.0, s = 0.0;
                    double2 ee = make_double2(1.0, 0.0);
                    bool valid = qq < n;
                    if (valid) {
                        const double2 z = A[p * n + qq];
                        const double rr = hypot(z.x, z.y);
                        if (rr > 1e-300 && rr > 1e-16 * sqrt(fabs(A[p * n + p].x * A[qq * n + qq].x))) {
                            const double app = A[p * n + p].x, aqq = A[qq * n + qq].x;
                            const double tau = (aqq - app) / (2.0 * rr);
                            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                            c = 1.0 / sqrt(1.0 + t * t);
                            s = t * c;
                            ee = make_double2(z.x / rr, z.y / rr);
                        } else {
                            valid = false;
                        }
                    }
                    if (valid) atomicAdd(&nrot, 1);
                    rotP[k] = valid ? p : -1;
                    rotQ[k] = qq;
                    rotC[k] = c;
                    rotS[k] = s;
                    rotE[k] = ee;
                }
                __syncthreads();
                // A <- A U and V <- V U (columns p, q of every row)
                for (int w = tid; w < 2 * n * (m / 2); w += nt) {
                    const int k = w % (m / 2), i = (w / (m / 2)) % n;
                    double2* M = (w / (m / 2)) >= n ? V : A;
                    const int p = rotP[k];
                    if (p < 0) continue;
                    const int qq = rotQ[k];
                    const double c = rotC[k], s = rotS[k];
                    const double2 eb = conj2(rotE[k]);
                    const double2 x = M[i * n + p], y = M[i * n + qq];
                    const double2 ey = cmul(eb, y);
                    M[i * n + p] = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
                    M[i * n + qq] = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
                }
                __syncthreads();
                // A <- U^H A (rows p, q of every column)
                for (int w = tid; w < n * (m / 2); w += nt) {
                    const int k = w % (m / 2), j = w / (m / 2);
                    const int p = rotP[k];
                    if (p < 0) continue;
                    const int qq = rotQ[k];
                    const double c = rotC[k], s = rotS[k];
                    const double2 e = rotE[k];
                    const double2 x = A[p * n + j], y = A[qq * n + j];
                    const double2 ey = cmul(e, y);
                    A[p * n + j] = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
                    A[qq * n + j] = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
                }
                __syncthreads();
                for (int k = tid; k < m / 2; k += nt) {
                    const int p = rotP[k];
                    if (p < 0) continue;
                    const int qq = rotQ[k];
                    A[p * n + qq] = make_double2(0.0, 0.0);
                    A[qq * n + p] = make_double2(0.0, 0.0);
                    A[p * n + p].y = 0.0;
                    A[qq * n + qq].y = 0.0;
                }
                __syncthreads();
            }
            if (nrot == 0) break;  // nothing above the threshold: converged (nrot read after the last barrier)
            __syncthreads();
        }
        // --- ascending order (stable): rank of each eigenvalue
        for (int i = tid; i < n; i += nt) {
            const double li = A[i * n + i].x;
            int rk = 0;
            for (int j = 0; j < n; ++j) {
                const double lj = A[j * n + j].x;
                rk += (lj < li) || (lj == li && j < i);
            }
            rank[i] = rk;
            lam[rk] = li;
        }
        __syncthreads();
        const bool gamma = fabs(qx) < CMP_PREC && fabs(qy) < CMP_PREC && fabs(qz) < CMP_PREC;
        // eigenvectors: evec[q][s][row] = V[row][col with rank s]
        for (int w = tid; w < n * n; w += nt) {
            const int col = w / n, row = w % n;
            evec[((size_t)q * n + rank[col]) * n + row] = V[row * n + col];
        }
        // per-mode quantities
        for (int col = tid; col < n; col += nt) {
            const int s = rank[col];
            const double lv = A[col * n + col].x;
            double W = sqrt(fabs(lv));
            if (fabs(lv) > EPS_F32 && lv < 0.0) W = -W;
            omega[(size_t)q * n + s] = W * a.wTHz;
            const bool zero_mode = gamma && s < 3;
            double v3[3] = {0.0, 0.0, 0.0};
            if (!zero_mode) {
                for (int k = 0; k < 3; ++k) {
                    double2 acc = make_double2(0.0, 0.0);
                    for (int i = 0; i < n; ++i) {
                        double2 t = make_double2(0.0, 0.0);
                        for (int j = 0; j < n; ++j) t = cadd(t, cmul(dD[(k * n + i) * n + j], V[j * n + col]));
                        acc = cadd(acc, cmul(conj2(V[i * n + col]), t));
                    }
                    v3[k] = acc.x / (2.0 * W) * a.vg_ms;
                }
            }
            for (int k = 0; k < 3; ++k) vel[((size_t)q * n + s) * 3 + k] = v3[k];
            oneby[(size_t)q * n + s] = zero_mode ? 0.0 : 1.0 / (W * a.wTHz);
            for (int t = 0; t < a.nT; ++t)
                nbe[((size_t)t * nq + q) * n + s] = zero_mode ? 0.0 : 1.0 / (exp(a.BEConv * fabs(W) / temps[t]) - 1.0);
        }
        __syncthreads();
    }
}

// Two-atom cells (n = 6): eight lanes per q-point, four points per one-warp block, each group
// with its own shared-memory state (16 KB per block: 13 blocks, 52 points, per SM).  The same steps as k_phonons (phases once
// per (mu, N), then D and dD/dq in reference neighbour order; the same round-robin Jacobi rotations
// and stopping rules; ordering, velocities, nBE), with every control decision warp-uniform: the
// groups synchronise with full-warp barriers, a converged or idle group only skips work, and the
// sweep loop ends when every group of the warp has converged.
constexpr int PH6_LANES = 8, PH6_PTS = 4, PH6_NA2 = 32;
struct Ph6 {
    double2 A[36], V[36], dD[3 * 36];
    double2 ph[2 * PH6_NA2];  // e^{i q.R} per (mu, N)
    double2 rotE[3];
    double rotC[3], rotS[3], lam[6];
    int rotP[3], rotQ[3], rank[6], nrot;
};

__global__ void __launch_bounds__(32) k_phonons_n6(PhArgs a, PhSet SA, const int* __restrict__ list_a, int n_a,
                                                  PhSet SB, int n_b, const double* __restrict__ fc2,
                                                  const int* __restrict__ idx, const int* __restrict__ num,
                                                  const double* __restrict__ mrs, const double* __restrict__ temps) {
    constexpr int n = 6, m = 6, L = PH6_LANES;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ Ph6 sh[PH6_PTS];
    const int gi = threadIdx.x / L, gl = threadIdx.x % L;
    Ph6& S = sh[gi];
    const int total = n_a + n_b;
    for (int base = blockIdx.x * PH6_PTS; base < total; base += gridDim.x * PH6_PTS) {
        const int item = base + gi;
        const bool act = item < total;
        const bool in_a = item < n_a;
        const PhSet& P = in_a ? SA : SB;
        const int q = act ? (in_a ? (list_a ? list_a[item] : item) : item - n_a) : 0;
        double qx = 0.0, qy = 0.0, qz = 0.0;
        if (act) {
            qx = P.qpts[3 * q];
            qy = P.qpts[3 * q + 1];
            qz = P.qpts[3 * q + 2];
            for (int w = gl; w < 4 * 36; w += L) {
                if (w < 36) S.A[w] = make_double2(0.0, 0.0);
                else S.dD[w - 36] = make_double2(0.0, 0.0);
            }
            for (int w = gl; w < 36; w += L) S.V[w] = make_double2(w % 7 == 0 ? 1.0 : 0.0, 0.0);
            for (int w = gl; w < 2 * a.na2; w += L) {
                const int mu = w / a.na2, N = w % a.na2;
                if (N < num[mu]) {
                    const int* e = idx + 4 * (N + a.na2 * mu);
                    double R[3];
                    for (int r = 0; r < 3; ++r)
                        R[r] = a.latvec[r] * e[0] + a.latvec[r + 3] * e[1] + a.latvec[r + 6] * e[2];
                    const double qr = qx * R[0] + qy * R[1] + qz * R[2];
                    double sn, cs;
                    sincos(qr, &sn, &cs);
                    S.ph[mu * PH6_NA2 + N] = make_double2(cs, sn);
                }
            }
        }
        __syncwarp();
        // D(q), dD/dq: lane per (mu, alpha, beta); neighbours in reference order
        if (act)
            for (int w = gl; w < 18; w += L) {
                const int mu = w / 9, al = (w / 3) % 3, be = w % 3;
                const int row = 3 * mu + al;
                for (int N = 0; N < num[mu]; ++N) {
                    const int* e = idx + 4 * (N + a.na2 * mu);
                    const int nu = e[3] - 1;
                    double R[3];
                    for (int r = 0; r < 3; ++r)
                        R[r] = a.latvec[r] * e[0] + a.latvec[r + 3] * e[1] + a.latvec[r + 6] * e[2];
                    const double2 pe = S.ph[mu * PH6_NA2 + N];
                    const double f = fc2[((mu * a.na2 + N) * 3 + al) * 3 + be];  // fC(1,be,al,N,mu)
                    const double mf = mrs[mu] * mrs[nu];
                    const int col = 3 * nu + be;
                    const double2 t = make_double2(f * pe.x * mf, f * pe.y * mf);
                    S.A[row * n + col] = cadd(S.A[row * n + col], t);
                    for (int k = 0; k < 3; ++k)  // (i R_k) * t
                        S.dD[(k * n + row) * n + col] =
                            cadd(S.dD[(k * n + row) * n + col], make_double2(-t.y * R[k], t.x * R[k]));
                }
            }
        __syncwarp();
        if (act && a.dd) {  // + DynEw, dDynEw/dq (LongEw)
            const double2* d = a.dd + (size_t)item * 4 * 36;
            for (int w = gl; w < 4 * 36; w += L) {
                double2& t = w < 36 ? S.A[w] : S.dD[w - 36];
                t = cadd(t, d[w]);
            }
        }
        __syncwarp();
        if (act && a.dd)  // the lower triangle from the upper one, as zheevd('U') reads it
            for (int w = gl; w < 36; w += L) {
                const int r = w / n, cc = w % n;
                if (r > cc) S.A[w] = conj2(S.A[cc * n + r]);
                else if (r == cc) S.A[w].y = 0.0;
            }
        __syncwarp();

        // --- cyclic complex Jacobi, one group per point
        bool gdone = !act;
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            double off = 0.0, dg = 0.0;
            if (!gdone)
                for (int w = gl; w < 36; w += L) {
                    const int i = w / n, j = w % n;
                    const double2 z = S.A[w];
                    if (i == j) dg += z.x * z.x;
                    else if (j > i) off += z.x * z.x + z.y * z.y;
                }
            for (int o = L / 2; o > 0; o >>= 1) {  // within the group; every lane gets the same sums
                off += __shfl_xor_sync(FULL, off, o);
                dg += __shfl_xor_sync(FULL, dg, o);
            }
            if (!gdone && (off <= 1e-30 * dg || off == 0.0)) gdone = true;
            if (__all_sync(FULL, gdone)) break;
            if (gl == 0) S.nrot = 0;
            __syncwarp();
            for (int r = 0; r < m - 1; ++r) {
                if (!gdone && gl < m / 2) {
                    const int k = gl;
                    int p, qq;
                    if (k == 0) { p = r; qq = m - 1; }
                    else { p = (r + k) % (m - 1); qq = (r - k + (m - 1)) % (m - 1); }
                    if (p > qq) { const int t = p; p = qq; qq = t; }
                    double c = 1.0, sn = 0.0;
                    double2 ee = make_double2(1.0, 0.0);
                    bool valid = false;
                    const double2 z = S.A[p * n + qq];
                    const double rr = hypot(z.x, z.y);
                    if (rr > 1e-300 && rr > 1e-16 * sqrt(fabs(S.A[p * n + p].x * S.A[qq * n + qq].x))) {
                        const double app = S.A[p * n + p].x, aqq = S.A[qq * n + qq].x;
                        const double tau = (aqq - app) / (2.0 * rr);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                        ee = make_double2(z.x / rr, z.y / rr);
                        valid = true;
                        atomicAdd(&S.nrot, 1);
                    }
                    S.rotP[k] = valid ? p : -1;
                    S.rotQ[k] = qq;
                    S.rotC[k] = c;
                    S.rotS[k] = sn;
                    S.rotE[k] = ee;
                }
                __syncwarp();
                if (!gdone)  // A <- A U and V <- V U (columns p, q of every row)
                    for (int w = gl; w < 2 * n * (m / 2); w += L) {
                        const int k = w % (m / 2), i = (w / (m / 2)) % n;
                        double2* M = (w / (m / 2)) >= n ? S.V : S.A;
                        const int p = S.rotP[k];
                        if (p < 0) continue;
                        const int qq = S.rotQ[k];
                        const double c = S.rotC[k], sn = S.rotS[k];
                        const double2 eb = conj2(S.rotE[k]);
                        const double2 x = M[i * n + p], y = M[i * n + qq];
                        const double2 ey = cmul(eb, y);
                        M[i * n + p] = make_double2(c * x.x - sn * ey.x, c * x.y - sn * ey.y);
                        M[i * n + qq] = make_double2(sn * x.x + c * ey.x, sn * x.y + c * ey.y);
                    }
                __syncwarp();
                if (!gdone)  // A <- U^H A (rows p, q of every column)
                    for (int w = gl; w < n * (m / 2); w += L) {
                        const int k = w % (m / 2), j = w / (m / 2);
                        const int p = S.rotP[k];
                        if (p < 0) continue;
                        const int qq = S.rotQ[k];
                        const double c = S.rotC[k], sn = S.rotS[k];
                        const double2 e = S.rotE[k];
                        const double2 x = S.A[p * n + j], y = S.A[qq * n + j];
                        const double2 ey = cmul(e, y);
                        S.A[p * n + j] = make_double2(c * x.x - sn * ey.x, c * x.y - sn * ey.y);
                        S.A[qq * n + j] = make_double2(sn * x.x + c * ey.x, sn * x.y + c * ey.y);
                    }
                __syncwarp();
                if (!gdone && gl < m / 2) {
                    const int p = S.rotP[gl];
                    if (p >= 0) {
                        const int qq = S.rotQ[gl];
                        S.A[p * n + qq] = make_double2(0.0, 0.0);
                        S.A[qq * n + p] = make_double2(0.0, 0.0);
                        S.A[p * n + p].y = 0.0;
                        S.A[qq * n + qq].y = 0.0;
                    }
                }
                __syncwarp();
            }
            if (!gdone && S.nrot == 0) gdone = true;  // nothing above the threshold: converged
            __syncwarp();
        }
        // --- ascending order (stable): rank of each eigenvalue
        if (act && gl < n) {
            const double li = S.A[gl * n + gl].x;
            int rk = 0;
            for (int j = 0; j < n; ++j) {
                const double lj = S.A[j * n + j].x;
                rk += (lj < li) || (lj == li && j < gl);
            }
            S.rank[gl] = rk;
            S.lam[rk] = li;
        }
        __syncwarp();
        if (act) {
            const int nq = P.nq;
            const bool gamma = fabs(qx) < CMP_PREC && fabs(qy) < CMP_PREC && fabs(qz) < CMP_PREC;
            for (int w = gl; w < 36; w += L) {
                const int col = w / n, row = w % n;
                P.evec[((size_t)q * n + S.rank[col]) * n + row] = S.V[row * n + col];
            }
            if (gl < n) {
                const int col = gl, s = S.rank[col];
                const double lv = S.A[col * n + col].x;
                double W = sqrt(fabs(lv));
                if (fabs(lv) > EPS_F32 && lv < 0.0) W = -W;
                P.omega[(size_t)q * n + s] = W * a.wTHz;
                const bool zero_mode = gamma && s < 3;
                double v3[3] = {0.0, 0.0, 0.0};
                if (!zero_mode) {
                    for (int k = 0; k < 3; ++k) {
                        double2 acc = make_double2(0.0, 0.0);
                        for (int i = 0; i < n; ++i) {
                            double2 t = make_double2(0.0, 0.0);
                            for (int j = 0; j < n; ++j) t = cadd(t, cmul(S.dD[(k * n + i) * n + j], S.V[j * n + col]));
                            acc = cadd(acc, cmul(conj2(S.V[i * n + col]), t));
                        }
                        v3[k] = acc.x / (2.0 * W) * a.vg_ms;
                    }
                }
                for (int k = 0; k < 3; ++k) P.vel[((size_t)q * n + s) * 3 + k] = v3[k];
                P.oneby[(size_t)q * n + s] = zero_mode ? 0.0 : 1.0 / (W * a.wTHz);
                for (int t = 0; t < a.nT; ++t)
                    P.nbe[((size_t)t * nq + q) * n + s] =
                        zero_mode ? 0.0 : 1.0 / (exp(a.BEConv * fabs(W) / temps[t]) - 1.0);
            }
        }
        __syncwarp();
    }
}

// Points of the other half of the (q, -q) pairs: copies of their partner with conjugate
// eigenvectors and reversed velocities.
__global__ void k_phonons_tr(int n, int nT, int nq, const int* __restrict__ fill, const int* __restrict__ partner,
                             double2* __restrict__ evec, double* __restrict__ omega, double* __restrict__ oneby,
                             double* __restrict__ nbe, double* __restrict__ vel, int n_fill) {
    const int per = n * n + n * (3 + nT + 2);
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < (long long)n_fill * per;
         w += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(w / per), k = (int)(w % per);
        const int g = fill[i], p = partner[g];
        if (k < n * n) {
            const double2 e = evec[(size_t)p * n * n + k];
            evec[(size_t)g * n * n + k] = make_double2(e.x, -e.y);
        } else {
            const int r = k - n * n, s = r % n, what = r / n;  // 0..2 velocity, 3 omega, 4 1/omega, 5.. nBE
            if (what < 3) vel[((size_t)g * n + s) * 3 + what] = -vel[((size_t)p * n + s) * 3 + what];
            else if (what == 3) omega[(size_t)g * n + s] = omega[(size_t)p * n + s];
            else if (what == 4) oneby[(size_t)g * n + s] = oneby[(size_t)p * n + s];
            else {
                const int t = what - 5;
                nbe[((size_t)t * nq + g) * n + s] = nbe[((size_t)t * nq + p) * n + s];
            }
        }
    }
}

PhArgs ph_args(spring_ctx* c) {
    PhArgs a;
    a.nb = c->nb;
    a.n = c->ndof;
    a.na2 = c->na2;
    for (int i = 0; i < 9; ++i) a.latvec[i] = c->latvec[i];
    HostConst k = host_constants();
    a.wTHz = k.wTHz;
    a.vg_ms = k.vg_ms;
    a.BEConv = k.BEConv;
    a.nT = c->nT;
    a.dd = nullptr;
    return a;
}

size_t ph_smem(int n) {
    const int m = n + (n & 1);
    return sizeof(double2) * (5 * n * n + m / 2) + sizeof(double) * (2 * (m / 2) + 2) +
           sizeof(int) * (2 * (m / 2) + n + (n & 1)) + sizeof(double) * n + 16;
}

int launch_phonons(spring_ctx* c, const PhSet& A, const int* list_a, int n_a, const PhSet& B, int n_b,
                   int gamma_mode = 0) {
    PhArgs a = ph_args(c);
    SPRING_CHECK(launch_ewald(c, A.qpts, A.nq, list_a, n_a, B.qpts, B.nq, n_b, gamma_mode, &a.dd));
    const int n = c->ndof;
    const size_t smem = ph_smem(n);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_phonons, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int threads = n <= 6 ? 32 : 128;
    const int items = n_a + n_b;
    if (items == 0) return SPRING_OK;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "phonons: injected launch failure");
    if (n == 6 && a.nb == 2 && a.na2 <= PH6_NA2) {
        const int blocks = std::min((items + PH6_PTS - 1) / PH6_PTS, 148 * 13);
        k_phonons_n6<<<blocks, PH6_LANES * PH6_PTS, 0, c->stream>>>(a, A, list_a, n_a, B, n_b, c->d_fc2.p,
                                                                   c->d_fc2_idx.p, c->d_fc2_num.p, c->d_mass_rs.p,
                                                                   c->d_temps.p);
        return launch_check(c, "k_phonons_n6");
    }
    const int blocks = items < 148 * 32 ? items : 148 * 32;
    k_phonons<<<blocks, threads, smem, c->stream>>>(a, A, list_a, n_a, B, n_b, c->d_fc2.p, c->d_fc2_idx.p,
                                                    c->d_fc2_num.p, c->d_mass_rs.p, c->d_temps.p);
    return launch_check(c, "k_phonons");
}

PhSet ph_set(Phonons& ph, const double* q, int nq) {
    return PhSet{q, ph.evec.p, ph.omega.p, ph.oneby.p, ph.nbe.p, ph.vel.p, nq};
}

}  // namespace

int run_phonons(spring_ctx* c, Phonons& ph, const double* d_q, int nq, int gamma_mode) {
    const PhSet A = ph_set(ph, d_q, nq);
    return launch_phonons(c, A, nullptr, nq, A, 0, gamma_mode);
}

// Grid and irreducible phonons in one launch; on a Gamma-centred mesh only one point of each
// (q, -q) pair of the grid is solved and the other filled by time reversal.
int run_phonons_mesh(spring_ctx* c) {
    const int nq = c->nq;
    const PhSet G = ph_set(c->ph_grid, c->d_qpnt.p, nq), I = ph_set(c->ph_irr, c->d_irr_q.p, c->nq0);
    const bool tr = c->mesh_shift[0] == 0 && c->mesh_shift[1] == 0 && c->mesh_shift[2] == 0 &&
                    !(c->ew.on && c->ew.even);
    if (!tr) {
        SPRING_CHECK(launch_phonons(c, G, nullptr, nq, G, 0));
        return launch_phonons(c, I, nullptr, c->nq0, I, 0);
    }
    if (c->tr_nq != nq) {  // partner of every grid point and the two lists (built once per mesh)
        std::vector<int> partner(nq), solve, fill;
        for (int g = 0; g < nq; ++g) {
            const int x = g % c->mesh[0], y = (g / c->mesh[0]) % c->mesh[1], z = g / (c->mesh[0] * c->mesh[1]);
            const int xm = (c->mesh[0] - x) % c->mesh[0], ym = (c->mesh[1] - y) % c->mesh[1],
                      zm = (c->mesh[2] - z) % c->mesh[2];
            const int p = xm + c->mesh[0] * (ym + c->mesh[1] * zm);
            partner[g] = p;
            (g <= p ? solve : fill).push_back(g);
        }
        SPRING_CHECK(dalloc(c, c->d_tr_partner, nq, "time-reversal partners"));
        SPRING_CHECK(dalloc(c, c->d_tr_solve, std::max<size_t>(solve.size(), 1), "time-reversal lists"));
        SPRING_CHECK(dalloc(c, c->d_tr_fill, std::max<size_t>(fill.size(), 1), "time-reversal lists"));
        SPRING_CHECK(h2d(c, c->d_tr_partner.p, partner.data(), sizeof(int) * nq, "time-reversal partners"));
        SPRING_CHECK(h2d(c, c->d_tr_solve.p, solve.data(), sizeof(int) * solve.size(), "time-reversal lists"));
        SPRING_CHECK(h2d(c, c->d_tr_fill.p, fill.data(), sizeof(int) * fill.size(), "time-reversal lists"));
        c->tr_nsolve = (int)solve.size();
        c->tr_nfill = (int)fill.size();
        c->tr_nq = nq;
    }
    SPRING_CHECK(launch_phonons(c, G, c->d_tr_solve.p, c->tr_nsolve, I, c->nq0));
    if (c->tr_nfill == 0) return SPRING_OK;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "phonons: injected launch failure");
    const int n = c->ndof;
    const long long work = (long long)c->tr_nfill * (n * n + n * (5 + c->nT));
    k_phonons_tr<<<(int)std::min<long long>((work + 255) / 256, 148LL * 16), 256, 0, c->stream>>>(
        n, c->nT, nq, c->d_tr_fill.p, c->d_tr_partner.p, G.evec, G.omega, G.oneby, G.nbe, G.vel, c->tr_nfill);
    return launch_check(c, "k_phonons_tr");
}

}  // namespace spring
