// The any-cell V3 work item (one pair, one s0 block) shared by the per-call
// kernel (k_v3.cu) and the batched persistent kernel (k_batch.cu).  Reference
// citations and the regrouping are described in k_v3.cu.
#pragma once
#include "spring_internal.cuh"

namespace spring {
namespace {

struct V3Args {
    int nb, n, na, nq;
    int sb;            // s0 block size
    int nsb;           // number of s0 blocks
    int q0_first;
    int pair_first;    // first pair of the range
    double mfac;       // Sctr3THz2 / Nq
    // GAUSS
    double onebysigma, onebysigma2;
    int nT, nq0;
    int pol_lo[3], pol_hi[3];
};

constexpr double EXP_UNDERFLOW = 745.2;  // exp(-x) == 0 in FP64 for x above this

__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

// Inputs of one V3 work range: pairs and their q0, FC3 and the crystal, the q0 and grid phonons,
// and the outputs.
struct V3Ptrs {
    const int2* pairs;
    const int* pair_q0;
    const double* fc3;
    const double* posr;
    const int* btyp;
    const double* mrs;
    const double* qpnt;
    const int* irr_int;
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
};

// One (pair, s0-block) work item: Phi of the pair for s0 in [s0b, s0b + sb), then W and the
// epilogue (EPI 0: Gaussian sums into out_lw / out_p3; EPI 1: W and its transpose into out_w).
// Called by every thread of the CTA; smem2 holds v3_smem() bytes.
template <int EPI>
__device__ __forceinline__ void v3_item(const V3Args& a, const V3Ptrs& P, int pr, int s0b, double2* smem2) {
    const int2* __restrict__ pairs = P.pairs;
    const int* __restrict__ pair_q0 = P.pair_q0;
    const double* __restrict__ fc3 = P.fc3;
    const double* __restrict__ posr = P.posr;
    const int* __restrict__ btyp = P.btyp;
    const double* __restrict__ mrs = P.mrs;
    const double* __restrict__ qpnt = P.qpnt;
    const int* __restrict__ irr_int = P.irr_int;
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

    const int n = a.n, na = a.na, nn = n * n;
    const int sb = a.sb;
    double2* sE0 = smem2;              // [s][row]
    double2* sE1 = sE0 + nn;
    double2* sE2 = sE1 + nn;           // [row][s] (transposed: stage (d) reads it along s2)
    double2* sD = sE2 + nn;            // [a][nu b][eta c]
    double2* sT1 = sD + 3 * nn;        // [a][nu b][s2]
    double2* sT2 = sD;                 // [a][s1][s2]: D is dead once T1 is formed
    double2* sPhi = sT1 + 3 * nn;      // [s0 - s0b][s1][s2]
    double2* sPP = sPhi + sb * nn;     // [N1][N2] phase products with masses
    double2* sP = sPP + na * na;       // [2][na] phases of q1 and q2
    double* sFC = reinterpret_cast<double*>(sP + 2 * na);  // [N1][N2][27]
    double* sLw = sFC + ((na * na * 27 + 1) & ~1);         // [nT + 1][sb]
    int* sBt = reinterpret_cast<int*>(sLw + (a.nT + 1) * sb + 1);  // [na]
    int* sCnt = sBt + na;              // [nb] slots of each basis type
    int* sIdx = sCnt + a.nb;           // [nb][na] those slots, ascending

    const int tid = threadIdx.x, nt = blockDim.x;
    const int2 pq = pairs[pr];
    const int g1 = pq.x, g2 = pq.y;
    const int q0 = pair_q0[pr];
    const int p0 = q0_grid ? q0_grid[q0] : q0;  // row of the q0 phonons
    const int nphi = min(sb, n - s0b) * nn;  // the last s0 block may be partial

    for (int i = tid; i < nn; i += nt) {
        sE0[i] = ev0[(size_t)p0 * nn + i];
        sE1[i] = evg[(size_t)g1 * nn + i];
        sE2[(i % n) * n + i / n] = evg[(size_t)g2 * nn + i];
    }
    for (int i = tid; i < nphi; i += nt) sPhi[i] = make_double2(0.0, 0.0);

    for (int mu = 0; mu < a.nb; ++mu) {
        // (a) stage FC3 of mu, basis of each neighbour slot, and the neighbour phases
        const double* f = fc3 + (size_t)mu * na * na * 27;
        for (int i = tid; i < na * na * 27; i += nt) sFC[i] = f[i];
        for (int i = tid; i < na; i += nt) sBt[i] = btyp[mu * na + i];
        for (int i = tid; i < 2 * na; i += nt) {
            const int N = i % na;
            const int g = i < na ? g1 : g2;
            const double* Rv = posr + ((size_t)mu * na + N) * 3;
            const double qr = qpnt[3 * g] * Rv[0] + qpnt[3 * g + 1] * Rv[1] + qpnt[3 * g + 2] * Rv[2];
            double sn, cs;
            sincos(qr, &sn, &cs);
            sP[i] = make_double2(cs, sn);
        }
        __syncthreads();
        // the slots of each basis type (the D sums below visit only these, in the same order)
        if (tid < a.nb) {
            int cnt = 0;
            for (int N = 0; N < na; ++N)
                if (sBt[N] == tid) sIdx[tid * na + cnt++] = N;
            sCnt[tid] = cnt;
        }
        // (b) phase products with the neighbour masses
        for (int i = tid; i < na * na; i += nt) {
            const int N1 = i / na, N2 = i % na;
            const double2 p1 = sP[N1], p2 = sP[na + N2];
            const double m = mrs[sBt[N1]] * mrs[sBt[N2]];
            sPP[i] = make_double2(m * (p1.x * p2.x - p1.y * p2.y), m * (p1.x * p2.y + p1.y * p2.x));
        }
        __syncthreads();
        // (c) D[a][nu b][eta c] = sum over slots of basis nu / eta of FC * phase
        for (int o = tid; o < 3 * nn; o += nt) {
            const int al = o / nn, r = (o / n) % n, cidx = o % n;
            const int nu = r / 3, be = r % 3, eta = cidx / 3, ga = cidx % 3;
            const int abc = (al * 3 + be) * 3 + ga;
            double2 acc = make_double2(0.0, 0.0);
            const int c1 = sCnt[nu], c2 = sCnt[eta];
            for (int i1 = 0; i1 < c1; ++i1) {
                const int N1 = sIdx[nu * na + i1];
                for (int i2 = 0; i2 < c2; ++i2) {
                    const int N2 = sIdx[eta * na + i2];
                    const double fv = sFC[(N1 * na + N2) * 27 + abc];
                    const double2 pp = sPP[N1 * na + N2];
                    acc.x = fma(fv, pp.x, acc.x);
                    acc.y = fma(fv, pp.y, acc.y);
                }
            }
            sD[o] = acc;
        }
        __syncthreads();
        // (d) T1[a][r][s2] = sum_c D[a][r][c] e2(c, s2); one thread per (r, s2), all three a, so each
        // e2 value read serves three products (consecutive threads read consecutive s2: no bank
        // conflict)
        for (int o = tid; o < nn; o += nt) {
            const int r = o / n, s2 = o % n;
            const double2* d0 = sD + r * n;
            const double2* e2 = sE2 + s2;
            double2 acc0 = make_double2(0.0, 0.0), acc1 = acc0, acc2 = acc0;
            for (int k = 0; k < n; ++k) {
                const double2 e = e2[k * n];
                cfma(acc0, d0[k], e);
                cfma(acc1, d0[nn + k], e);
                cfma(acc2, d0[2 * nn + k], e);
            }
            sT1[o] = acc0;
            sT1[nn + o] = acc1;
            sT1[2 * nn + o] = acc2;
        }
        __syncthreads();
        // (e) T2[a][s1][s2] = sum_r e1(r, s1) T1[a][r][s2]; one thread per (s1, s2), all three a
        for (int o = tid; o < nn; o += nt) {
            const int s1 = o / n, s2 = o % n;
            const double2* e1 = sE1 + s1 * n;
            const double2* t1 = sT1 + s2;
            double2 acc0 = make_double2(0.0, 0.0), acc1 = acc0, acc2 = acc0;
            for (int k = 0; k < n; ++k) {
                const double2 w = e1[k];
                cfma(acc0, w, t1[k * n]);
                cfma(acc1, w, t1[nn + k * n]);
                cfma(acc2, w, t1[2 * nn + k * n]);
            }
            sT2[o] = acc0;
            sT2[nn + o] = acc1;
            sT2[2 * nn + o] = acc2;
        }
        __syncthreads();
        // (f) Phi[s0][s1][s2] += sum_a m_mu^-1/2 e0(mu a, s0) T2[a][s1][s2]
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

    // W and epilogue
    const bool gq0 = irr_int[3 * q0] == 0 && irr_int[3 * q0 + 1] == 0 && irr_int[3 * q0 + 2] == 0;
    const bool gq1 = g1 == 0, gq2 = g2 == 0;
    if (EPI == 0) {
        for (int i = tid; i < (a.nT + 1) * sb; i += nt) sLw[i] = 0.0;
        __syncthreads();
    }
    for (int o = tid; o < nphi; o += nt) {
        const int s0 = s0b + o / nn, s1 = (o / n) % n, s2 = o % n;
        double W = 0.0;
        if (!((gq0 && s0 < 3) || (gq1 && s1 < 3) || (gq2 && s2 < 3))) {
            const double2 p = sPhi[o];
            const double abs2 = p.x * p.x + p.y * p.y;
            W = abs2 * (ob0[(size_t)p0 * n + s0] * obg[(size_t)g1 * n + s1] * obg[(size_t)g2 * n + s2]) * a.mfac;
        }
        if (EPI == 1) {
            const int slot = q0 - a.q0_first;
            const size_t n3 = (size_t)n * nn;
            out_w[((size_t)slot * a.nq + g1) * n3 + (s0 * n + s1) * n + s2] = W;
            if (g1 != g2) out_w[((size_t)slot * a.nq + g2) * n3 + (s0 * n + s2) * n + s1] = W;
        } else {
            if (s0 < a.pol_lo[0] || s0 > a.pol_hi[0] || s1 < a.pol_lo[1] || s1 > a.pol_hi[1] || s2 < a.pol_lo[2] ||
                s2 > a.pol_hi[2] || (gq1 && s1 < 3) || (gq2 && s2 < 3))
                continue;
            const double w0 = om0[(size_t)p0 * n + s0];
            const double w1 = omg[(size_t)g1 * n + s1];
            const double w2 = omg[(size_t)g2 * n + s2];
            const double d1 = w0 - w1 - w2, d2 = w0 + w1 - w2, d3 = w0 - w1 + w2;
            const double pre = a.onebysigma * ONEBYSQRT2PI;
            const double x1 = 0.5 * a.onebysigma2 * (d1 * d1);
            const double x2 = 0.5 * a.onebysigma2 * (d2 * d2);
            const double x3 = 0.5 * a.onebysigma2 * (d3 * d3);
            const double e1v = x1 < EXP_UNDERFLOW ? pre * exp(-x1) : 0.0;
            const double e2v = x2 < EXP_UNDERFLOW ? pre * exp(-x2) : 0.0;
            const double e3v = x3 < EXP_UNDERFLOW ? pre * exp(-x3) : 0.0;
            const double esum = e1v + e2v + e3v;
            if (esum == 0.0) continue;
            for (int t = 0; t < a.nT; ++t) {
                const double n1 = nbeg[((size_t)t * a.nq + g1) * n + s1];
                const double n2 = nbeg[((size_t)t * a.nq + g2) * n + s2];
                const double v = W * (((n1 + n2 + 1.0) * e1v) + ((n1 - n2) * (e2v - e3v)));
                atomicAdd(&sLw[t * sb + (s0 - s0b)], v);
            }
            atomicAdd(&sLw[a.nT * sb + (s0 - s0b)], esum);
        }
    }
    if (EPI == 0) {
        __syncthreads();
        const double mult = g1 != g2 ? 2.0 : 1.0;
        for (int i = tid; i < (a.nT + 1) * sb; i += nt) {
            const int t = i / sb, s0 = s0b + i % sb;
            if (s0 >= n || sLw[i] == 0.0) continue;
            if (t < a.nT)
                atomicAdd(&out_lw[((size_t)t * a.nq0 + q0) * n + s0], mult * sLw[i]);
            else
                atomicAdd(&out_p3[(size_t)q0 * n + s0], mult * sLw[i]);
        }
    }
}



inline size_t v3_smem(int n, int na, int sb, int nT) {
    const int nn = n * n;
    return sizeof(double2) * (3 * nn + 6 * nn + sb * nn + na * na + 2 * na) +
           sizeof(double) * (((na * na * 27 + 1) & ~1) + (nT + 1) * sb + 1) + sizeof(int) * (na + n / 3 * (na + 1)) +
           16;
}

inline int v3_block(int n) {
    // s0 block: the whole range for small cells; chunks for Ndof 24
    return n <= 12 ? n : 6;
}


}  // namespace
}  // namespace spring
