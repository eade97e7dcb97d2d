// The two-atom V3 work (groups of 8 pairs, 288 threads) shared by the per-call
// kernel (k_v3s.cu) and the batched persistent kernel (k_batch.cu); the layout
// and the citations are described in k_v3s.cu.
#pragma once
#include "spring_internal.cuh"

namespace spring {
namespace {
namespace s3 {


constexpr int NB = 2, N = 6, NA = 7, PP = 8, THREADS = PP * 36, RS = 7;  // RS: padded row stride
constexpr int MAXT = 9;
constexpr double EXP_UNDERFLOW = 745.2;

struct S3Args {
    int nq, nT, nq0, q0_first, pair_first, pair_end, ngroups;
    const int* plist;  // null: pairs pair_first .. pair_end - 1; else the pairs plist[pair_first .. pair_end - 1]
    double mfac, onebysigma, onebysigma2;
    int pol_lo[3], pol_hi[3];
};

// Shared memory of one CTA (about 106 KB: two CTAs per SM).  The phases live in
// A and the phase products in B until D and T1 overwrite them.
struct Smem {
    double2 e[PP][3][N * RS];        // e0 (times m_mu^-1/2 per row), e1, e2: [s][row]
    double2 A[PP][36 * RS];          // phases (stages 1-2), D (3-4), T2 (5-6)
    double2 B[PP][36 * RS];          // phase products (2-3), T1 (4-5)
    double fc[NB * NA * NA * 27];
    double posr[NB * NA * 3];
    double lw[PP][MAXT + 1][N];
    double mrs[NB];
    int off[NB * (NB + 1)];
    int btyp[NB * NA];
    int g1[PP], g2[PP], q0[PP], p0[PP], valid[PP];
};

__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

// Inputs and outputs of one launch of the specialised kernel.
struct S3Ptrs {
    const int2* pairs;
    const int* pair_q0;
    const double* fc3;
    const double* posr;
    const int* btyp;
    const int* off;
    const double* mrs;
    const double* qpnt;
    const int* q0_int;
    const int* q0_grid;
    const double2* ev0;
    const double* om0;
    const double* ob0;
    const double2* evg;
    const double* omg;
    const double* obg;
    const double* nbeg;
    double* out_lw;
    double* out_p3;
    double* out_w;
    // EPI 2 (the Gaussian BTE operator): entries appended at *item_ctr (those past item_cap are
    // counted, not written)
    void* out_items;
    unsigned long long* item_ctr;
    long long item_cap;
};

// One entry of the Gaussian BTE scattering operator (EPI 2): row r0 = q0 slot * 6 + s0, grid modes
// k1 = g1 * 6 + s1 and k2 = g2 * 6 + s2 of an enumerated pair, and the temperature-free parts of
// its coefficient c = (n1 - n2) P + (1 + n1 + n2) Q: P = 4 W (d(w0 + w1 - w2) - d(w0 + w2 - w1)),
// Q = 4 W d(w0 - w1 - w2) (halved, and the second delta of P absent, when q1 = q2).
struct BteEntry {
    int r0, k1, k2, pad;
    double P, Q;
};
static_assert(sizeof(BteEntry) == 32, "BTE entry");
constexpr double EXP_CUT_BTE = 40.0;  // exp(-40) = 4e-18 of a delta's peak: terms below are dropped

// Stage the cell's constants (FC3, neighbour positions and basis, masses, slot groups).
__device__ __forceinline__ void v3s_stage(Smem& S, const S3Ptrs& P) {
    const int tid = threadIdx.x;
    for (int i = tid; i < NB * NA * NA * 27; i += THREADS) S.fc[i] = P.fc3[i];
    for (int i = tid; i < NB * NA * 3; i += THREADS) S.posr[i] = P.posr[i];
    if (tid < NB) S.mrs[tid] = P.mrs[tid];
    if (tid < NB * (NB + 1)) S.off[tid] = P.off[tid];
    if (tid < NB * NA) S.btyp[tid] = P.btyp[tid];
}

// One group of PP pairs (called by all THREADS threads after v3s_stage).
template <int EPI>
__device__ __forceinline__ void v3s_group(Smem& S, const S3Args& a, const S3Ptrs& P, int grp) {
    const int2* __restrict__ pairs = P.pairs;
    const int* __restrict__ pair_q0 = P.pair_q0;
    const double* __restrict__ qpnt = P.qpnt;
    const int* __restrict__ q0_int = P.q0_int;
    const int* __restrict__ q0_grid = P.q0_grid;
    const double2* __restrict__ ev0 = P.ev0;
    const double* __restrict__ om0 = P.om0;
    const double* __restrict__ ob0 = P.ob0;
    const double2* __restrict__ evg = P.evg;
    const double* __restrict__ omg = P.omg;
    const double* __restrict__ obg = P.obg;
    const double* __restrict__ nbeg = P.nbeg;
    double* __restrict__ out_lw = P.out_lw;
    double* __restrict__ out_p3 = P.out_p3;
    double* __restrict__ out_w = P.out_w;
    // phases [p][which][mu][N] inside A[p]; phase products [p][mu][N1][N2] inside B[p]
    auto PH = [&](int p, int which, int mu, int n) -> double2& { return S.A[p][(which * NB + mu) * NA + n]; };
    auto PPR = [&](int p, int mu, int n1, int n2) -> double2& { return S.B[p][(mu * NA + n1) * NA + n2]; };
    const int tid = threadIdx.x;
    __syncthreads();  // previous group done with every buffer; constants staged
    // --- 0: pair descriptors
    if (tid < PP) {
        const int idx = a.pair_first + grp * PP + tid;
        const int v = idx < a.pair_end;
        S.valid[tid] = v;
        if (v) {
            const int pr = a.plist ? a.plist[idx] : idx;
            const int2 g = pairs[pr];
            const int q = pair_q0[pr];
            S.g1[tid] = g.x;
            S.g2[tid] = g.y;
            S.q0[tid] = q;
            S.p0[tid] = q0_grid ? q0_grid[q] : q;
        }
    }
    if (EPI == 0)
        for (int i = tid; i < PP * (MAXT + 1) * N; i += THREADS) (&S.lw[0][0][0])[i] = 0.0;
    __syncthreads();
    // --- 1: eigenvectors and neighbour phases
    for (int i = tid; i < PP * 3 * 36; i += THREADS) {
        const int p = i / 108, w = (i / 36) % 3, k = i % 36, s = k / 6, row = k % 6;
        if (!S.valid[p]) continue;
        double2 v;
        if (w == 0) {
            v = ev0[(size_t)S.p0[p] * 36 + k];
            const double m = S.mrs[row / 3];
            v.x *= m;
            v.y *= m;
        } else {
            v = evg[(size_t)(w == 1 ? S.g1[p] : S.g2[p]) * 36 + k];
        }
        S.e[p][w][s * RS + row] = v;
    }
    if (tid < PP * 2 * NB * NA) {
        const int p = tid / 28, j = tid % 28, which = j / 14, mu = (j / 7) % 2, Nn = j % 7;
        if (S.valid[p]) {
            const int g = which ? S.g2[p] : S.g1[p];
            const double* R = S.posr + (mu * NA + Nn) * 3;
            const double qr = qpnt[3 * g] * R[0] + qpnt[3 * g + 1] * R[1] + qpnt[3 * g + 2] * R[2];
            double sn, cs;
            sincos(qr, &sn, &cs);
            PH(p, which, mu, Nn) = make_double2(cs, sn);
        }
    }
    __syncthreads();
    // --- 2: phase products with neighbour masses
    for (int i = tid; i < PP * NB * NA * NA; i += THREADS) {
        const int p = i / 98, mu = (i / 49) % 2, n1 = (i / 7) % 7, n2 = i % 7;
        const double2 x = PH(p, 0, mu, n1), y = PH(p, 1, mu, n2);
        const double m = S.mrs[S.btyp[mu * NA + n1]] * S.mrs[S.btyp[mu * NA + n2]];
        PPR(p, mu, n1, n2) = make_double2(m * (x.x * y.x - x.y * y.y), m * (x.x * y.y + x.y * y.x));
    }
    __syncthreads();
    // --- 3: D[mu a][nu b][eta c]; one thread per (pair, mu, abc), all four (nu, eta) blocks
    for (int i = tid; i < PP * NB * 27; i += THREADS) {
        const int p = i / 54, mu = (i / 27) % 2, abc = i % 27;
        const int al = abc / 9, be = (abc / 3) % 3, ga = abc % 3;
        double2 acc[NB][NB];
#pragma unroll
        for (int u = 0; u < NB; ++u)
#pragma unroll
            for (int v = 0; v < NB; ++v) acc[u][v] = make_double2(0.0, 0.0);
        const int* o = S.off + mu * (NB + 1);
#pragma unroll
        for (int nu = 0; nu < NB; ++nu)
            for (int n1 = o[nu]; n1 < o[nu + 1]; ++n1)
#pragma unroll
                for (int eta = 0; eta < NB; ++eta)
                    for (int n2 = o[eta]; n2 < o[eta + 1]; ++n2) {
                        const double f = S.fc[((mu * NA + n1) * NA + n2) * 27 + abc];
                        const double2 q = PPR(p, mu, n1, n2);
                        acc[nu][eta].x = fma(f, q.x, acc[nu][eta].x);
                        acc[nu][eta].y = fma(f, q.y, acc[nu][eta].y);
                    }
#pragma unroll
        for (int nu = 0; nu < NB; ++nu)
#pragma unroll
            for (int eta = 0; eta < NB; ++eta)
                S.A[p][((mu * 3 + al) * 6 + nu * 3 + be) * RS + eta * 3 + ga] = acc[nu][eta];
    }
    __syncthreads();
    const int p = tid / 36, j = tid % 36;
    const int hi = j / 6, lo = j % 6;
    // --- 4: T1[ma][nb][s2] = sum_c D[ma][nb][c] e2(c, s2)      (thread: row r = j)
    {
        double2 acc[N];
#pragma unroll
        for (int s = 0; s < N; ++s) acc[s] = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double2 d = S.A[p][j * RS + k];
#pragma unroll
            for (int s = 0; s < N; ++s) cfma(acc[s], d, S.e[p][2][s * RS + k]);
        }
#pragma unroll
        for (int s = 0; s < N; ++s) S.B[p][j * RS + s] = acc[s];
    }
    __syncthreads();
    // --- 5: T2[ma][s1][s2] = sum_nb e1(nb, s1) T1[ma][nb][s2]    (thread: ma = hi, s1 = lo)
    {
        double2 acc[N];
#pragma unroll
        for (int s = 0; s < N; ++s) acc[s] = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double2 e = S.e[p][1][lo * RS + k];
#pragma unroll
            for (int s = 0; s < N; ++s) cfma(acc[s], e, S.B[p][(hi * 6 + k) * RS + s]);
        }
#pragma unroll
        for (int s = 0; s < N; ++s) S.A[p][j * RS + s] = acc[s];
    }
    __syncthreads();
    // --- 6: Phi[s0][s1][s2] = sum_ma e0'(ma, s0) T2[ma][s1][s2]  (thread: s0 = hi, s1 = lo)
    double2 phi[N];
#pragma unroll
    for (int s = 0; s < N; ++s) phi[s] = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double2 e = S.e[p][0][hi * RS + k];
#pragma unroll
        for (int s = 0; s < N; ++s) cfma(phi[s], e, S.A[p][(k * 6 + lo) * RS + s]);
    }
    // --- 7: W and epilogue
    double bP[N], bQ[N];  // EPI 2: this thread's operator entries (s2)
#pragma unroll
    for (int s2 = 0; s2 < N; ++s2) bP[s2] = bQ[s2] = 0.0;
    if (S.valid[p]) {
        const int g1 = S.g1[p], g2 = S.g2[p], q0 = S.q0[p], p0 = S.p0[p];
        const int s0 = hi, s1 = lo;
        const bool gq0 = q0_int[3 * q0] == 0 && q0_int[3 * q0 + 1] == 0 && q0_int[3 * q0 + 2] == 0;
        const bool gq1 = g1 == 0, gq2 = g2 == 0;
        const double o01 = ob0[(size_t)p0 * N + s0] * obg[(size_t)g1 * N + s1];
        double W[N];
#pragma unroll
        for (int s2 = 0; s2 < N; ++s2) {
            const bool zero = (gq0 && s0 < 3) || (gq1 && s1 < 3) || (gq2 && s2 < 3);
            const double abs2 = phi[s2].x * phi[s2].x + phi[s2].y * phi[s2].y;
            W[s2] = zero ? 0.0 : abs2 * (o01 * obg[(size_t)g2 * N + s2]) * a.mfac;
        }
        if (EPI == 2) {
            // entries of the Gaussian BTE operator (appended below, outside this branch)
            const double w0 = om0[(size_t)p0 * N + s0];
            const double w1 = omg[(size_t)g1 * N + s1];
            const double pre = a.onebysigma * ONEBYSQRT2PI;
            const bool self = g1 == g2;
#pragma unroll
            for (int s2 = 0; s2 < N; ++s2) {
                if (W[s2] == 0.0) continue;
                const double w2 = omg[(size_t)g2 * N + s2];
                const double da = w0 + w1 - w2, db = w0 + w2 - w1, dm = w0 - w1 - w2;
                const double xa = 0.5 * a.onebysigma2 * (da * da), xb = 0.5 * a.onebysigma2 * (db * db),
                             xm = 0.5 * a.onebysigma2 * (dm * dm);
                const double ea = xa < EXP_CUT_BTE ? pre * exp(-xa) : 0.0;
                const double eb = (!self && xb < EXP_CUT_BTE) ? pre * exp(-xb) : 0.0;
                const double em = xm < EXP_CUT_BTE ? pre * exp(-xm) : 0.0;
                bP[s2] = 4.0 * W[s2] * (ea - eb);
                bQ[s2] = 4.0 * W[s2] * (self ? 0.5 : 1.0) * em;
            }
        } else if (EPI == 1) {
            const int slot = q0 - a.q0_first;
            double* w1 = out_w + ((size_t)slot * a.nq + g1) * 216 + (s0 * N + s1) * N;
#pragma unroll
            for (int s2 = 0; s2 < N; ++s2) w1[s2] = W[s2];
            if (g1 != g2) {
                double* w2 = out_w + ((size_t)slot * a.nq + g2) * 216 + s0 * N * N + s1;
#pragma unroll
                for (int s2 = 0; s2 < N; ++s2) w2[s2 * N] = W[s2];
            }
        } else {
            const bool in01 = s0 >= a.pol_lo[0] && s0 <= a.pol_hi[0] && s1 >= a.pol_lo[1] && s1 <= a.pol_hi[1] &&
                              !(gq1 && s1 < 3);
            if (in01) {
                const double w0 = om0[(size_t)p0 * N + s0];
                const double w1 = omg[(size_t)g1 * N + s1];
                const double pre = a.onebysigma * ONEBYSQRT2PI;
                double e1v[N], edv[N], esum = 0.0;
#pragma unroll
                for (int s2 = 0; s2 < N; ++s2) {
                    e1v[s2] = edv[s2] = 0.0;
                    if (s2 < a.pol_lo[2] || s2 > a.pol_hi[2] || (gq2 && s2 < 3)) continue;
                    const double w2 = omg[(size_t)g2 * N + s2];
                    const double d1 = w0 - w1 - w2, d2 = w0 + w1 - w2, d3 = w0 - w1 + w2;
                    const double x1 = 0.5 * a.onebysigma2 * (d1 * d1);
                    const double x2 = 0.5 * a.onebysigma2 * (d2 * d2);
                    const double x3 = 0.5 * a.onebysigma2 * (d3 * d3);
                    const double ea = x1 < EXP_UNDERFLOW ? pre * exp(-x1) : 0.0;
                    const double eb = x2 < EXP_UNDERFLOW ? pre * exp(-x2) : 0.0;
                    const double ec = x3 < EXP_UNDERFLOW ? pre * exp(-x3) : 0.0;
                    e1v[s2] = ea;
                    edv[s2] = eb - ec;
                    esum += (ea + eb) + ec;
                }
                if (esum != 0.0) {
                    for (int t = 0; t < a.nT; ++t) {
                        const double n1 = nbeg[((size_t)t * a.nq + g1) * N + s1];
                        double v = 0.0;
#pragma unroll
                        for (int s2 = 0; s2 < N; ++s2) {
                            const double n2 = nbeg[((size_t)t * a.nq + g2) * N + s2];
                            v += W[s2] * (((n1 + n2 + 1.0) * e1v[s2]) + ((n1 - n2) * edv[s2]));
                        }
                        atomicAdd(&S.lw[p][t][s0], v);
                    }
                    atomicAdd(&S.lw[p][MAXT][s0], esum);
                }
            }
        }
    }
    if (EPI == 2) {
        // append this thread's nonzero entries: one atomic per warp for the warp's block
        const bool on = S.valid[p] != 0;
        int cnt = 0;
        if (on)
#pragma unroll
            for (int s2 = 0; s2 < N; ++s2) cnt += (bP[s2] != 0.0 || bQ[s2] != 0.0) ? 1 : 0;
        const int lane = tid & 31;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned long long base = 0;
        if (lane == 31 && total > 0) base = atomicAdd(P.item_ctr, (unsigned long long)total);
        base = __shfl_sync(0xffffffffu, base, 31);
        if (cnt > 0) {
            unsigned long long pos = base + (unsigned long long)(incl - cnt);
            const int g1 = S.g1[p], g2 = S.g2[p];
            const int r0 = (S.q0[p] - a.q0_first) * N + hi;  // row: q0 slot of this launch, s0
            BteEntry* out = static_cast<BteEntry*>(P.out_items);
#pragma unroll
            for (int s2 = 0; s2 < N; ++s2) {
                const double bp = bP[s2], bq = bQ[s2];
                if (bp == 0.0 && bq == 0.0) continue;
                if ((long long)pos < P.item_cap) {
                    BteEntry e;
                    e.r0 = r0;
                    e.k1 = g1 * N + lo;
                    e.k2 = g2 * N + s2;
                    e.pad = 0;
                    e.P = bp;
                    e.Q = bq;
                    out[pos] = e;
                }
                ++pos;
            }
        }
    }
    if (EPI == 0) {
        __syncthreads();
        for (int i = tid; i < PP * (a.nT + 1) * N; i += THREADS) {
            const int pp_ = i / ((a.nT + 1) * N), t = (i / N) % (a.nT + 1), s0 = i % N;
            if (!S.valid[pp_]) continue;
            const int tt = t < a.nT ? t : MAXT;
            const double v = S.lw[pp_][tt][s0];
            if (v == 0.0) continue;
            const double mult = S.g1[pp_] != S.g2[pp_] ? 2.0 : 1.0;
            if (t < a.nT)
                atomicAdd(&out_lw[((size_t)t * a.nq0 + S.q0[pp_]) * N + s0], mult * v);
            else
                atomicAdd(&out_p3[(size_t)S.q0[pp_] * N + s0], mult * v);
        }
    }
}

}  // namespace s3
}  // namespace
}  // namespace spring
