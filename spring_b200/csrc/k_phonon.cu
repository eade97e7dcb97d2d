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
// FP64 ALU bound (~10 n^3 flops per sweep); negligible next to the scattering path.
#include "spring_internal.cuh"

namespace spring {
namespace {

struct PhArgs {
    int nb, n, na2;
    double latvec[9];
    double wTHz, vg_ms, BEConv;
    int nT;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }

constexpr int MAX_SWEEPS = 30;

__global__ void __launch_bounds__(128, 8) k_phonons(PhArgs a, const double* __restrict__ qpts, const double* __restrict__ fc2,
                          const int* __restrict__ idx, const int* __restrict__ num, const double* __restrict__ mrs,
                          const double* __restrict__ temps, double2* __restrict__ evec, double* __restrict__ omega,
                          double* __restrict__ oneby, double* __restrict__ nbe, double* __restrict__ vel, int nq) {
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
    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        const double qx = qpts[3 * q], qy = qpts[3 * q + 1], qz = qpts[3 * q + 2];
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
        for (int i = tid; i < n; i += nt) V[i * n + i] = make_double2(1.0, 0.0);
        __syncthreads();

        // --- cyclic complex Jacobi
        for (int sweep = 0; sweep < MAX_SWEEPS; ++sweep) {
            if (tid == 0) {
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

}  // namespace

int run_phonons(spring_ctx* c, Phonons& ph, const double* d_q, int nq) {
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
    const int n = c->ndof, m = n + (n & 1);
    size_t smem = sizeof(double2) * (5 * n * n + m / 2) + sizeof(double) * (2 * (m / 2) + 2) +
                  sizeof(int) * (2 * (m / 2) + n + (n & 1)) + sizeof(double) * n + 16;
    if (smem > 48 * 1024) {
        cudaFuncSetAttribute(k_phonons, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    const int threads = n <= 6 ? 32 : 128;
    const int blocks = nq < 148 * 32 ? nq : 148 * 32;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "phonons: injected launch failure");
    k_phonons<<<blocks, threads, smem, c->stream>>>(a, d_q, c->d_fc2.p, c->d_fc2_idx.p, c->d_fc2_num.p,
                                                    c->d_mass_rs.p, c->d_temps.p, ph.evec.p, ph.omega.p, ph.oneby.p,
                                                    ph.nbe.p, ph.vel.p, nq);
    return launch_check(c, "k_phonons");
}

}  // namespace spring
