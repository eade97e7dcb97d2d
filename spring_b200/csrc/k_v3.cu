// Three-phonon matrix elements V3 -> W (FP64) and their Gaussian delta sum.
//
// Reference: ScatterProbAllq1 / ScatterMatEl / ScatterProbability
// (src/Kappa/Src/ThirdOrder_m.f90:41-166, 278-386, 389-439) and the Gaussian
// linewidth CalculateLinewidth (:442-543).
//
// The reference evaluates Phi(s2,s1,s) in a 9-deep loop (~Na3^2*27*Ndof^3
// complex MACs per pair).  Here the sum is factored into three contractions
// per basis atom mu (FC3 is real, phases are per neighbour slot):
//   E1[N1 b][s1] = e^{i q1.R_N1} m_nu^-1/2 e1(nu b, s1)        (nu = basis of N1)
//   E2[N2 c][s2] = e^{i q2.R_N2} m_eta^-1/2 e2(eta c, s2)
//   Y[(N1 a) b][s2] = sum_{N2 c} FC3(c,b,a,N2,N1,mu) E2[N2 c][s2]   (real x complex GEMM, K = 3 Na3)
//   Z[a][s1][s2]    = sum_{N1 b} E1[N1 b][s1] Y[(N1 a) b][s2]
//   Phi[s0][s1][s2] += sum_a m_mu^-1/2 e0(mu a, s0) Z[a][s1][s2]
// W = |Phi|^2 (1/w0)(1/w1)(1/w2) Sctr3THz2/Nq, zero for Gamma acoustic modes.
//
// One CTA handles one (pair, block of s0) work item, so that Phi fits in shared
// memory for Ndof up to 24.  Two epilogues:
//   GAUSS: the pair's contribution to Gamma(q0,s0) for every temperature, fused
//          (W never leaves the SM).  The reference sums over every grid q1; the
//          q2-side term of a pair equals its q1-side term exactly (swap s1<->s2),
//          so each pair is weighted by 2 (1 when q1 == q2).
//   WGRID: W for q1 and its s1<->s2 transpose for q2, i.e. the reference's
//          Sctrq1(s2,s1,s0,q) for every grid q, for the tetrahedron integration.
// Roofline: FP64 FMA pipe (about 110 kflop per pair for Ndof 6), plus FP64 exp
// in the GAUSS epilogue (3 per mode triple).
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

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int EPI>
__global__ void __launch_bounds__(128) k_v3(V3Args a, const int2* __restrict__ pairs, const int* __restrict__ pair_q0,
                                            const double* __restrict__ fc3t, const double* __restrict__ posr,
                                            const int* __restrict__ btyp, const double* __restrict__ mrs,
                                            const double* __restrict__ qpnt, const int* __restrict__ irr_int,
                                            const double2* __restrict__ ev0, const double* __restrict__ om0,
                                            const double* __restrict__ ob0, const double2* __restrict__ evg,
                                            const double* __restrict__ omg, const double* __restrict__ obg,
                                            const double* __restrict__ nbeg, double* __restrict__ out_lw,
                                            double* __restrict__ out_p3, double* __restrict__ out_w) {
    extern __shared__ double smem_d[];
    const int n = a.n, K = 3 * a.na, R = 9 * a.na;
    const int sb = a.sb;
    double* sFC = smem_d;                                  // [K][R] (padded to an even count)
    double2* sE1 = reinterpret_cast<double2*>(sFC + ((K * R + 1) & ~1));  // [K][n]
    double2* sE2 = sE1 + K * n;                            // [K][n]
    double2* sY = sE2 + K * n;                             // [R][n]
    double2* sZ = sY + R * n;                              // [3][n][n]
    double2* sPhi = sZ + 3 * n * n;                        // [sb][n][n]
    double2* sP1 = sPhi + sb * n * n;                      // [na]
    double2* sP2 = sP1 + a.na;                             // [na]
    double* sLw = reinterpret_cast<double*>(sP2 + a.na);  // [nT][sb] + [sb]

    const int tid = threadIdx.x, nt = blockDim.x;
    const int work = blockIdx.x;
    const int pr = a.pair_first + work / a.nsb;
    const int s0b = (work % a.nsb) * sb;
    const int2 pq = pairs[pr];
    const int g1 = pq.x, g2 = pq.y;
    const int q0 = pair_q0[pr];
    const double q1x = qpnt[3 * g1], q1y = qpnt[3 * g1 + 1], q1z = qpnt[3 * g1 + 2];
    const double q2x = qpnt[3 * g2], q2y = qpnt[3 * g2 + 1], q2z = qpnt[3 * g2 + 2];
    const double2* e0 = ev0 + (size_t)q0 * n * n;   // [s][row]
    const double2* e1 = evg + (size_t)g1 * n * n;
    const double2* e2 = evg + (size_t)g2 * n * n;
    const int nphi = min(sb, n - s0b) * n * n;  // the last s0 block may be partial

    for (int i = tid; i < nphi; i += nt) sPhi[i] = make_double2(0.0, 0.0);

    for (int mu = 0; mu < a.nb; ++mu) {
        // stage FC3 of mu and the neighbour phases
        const double* f = fc3t + (size_t)mu * K * R;
        for (int i = tid; i < K * R; i += nt) sFC[i] = f[i];
        for (int i = tid; i < 2 * a.na; i += nt) {
            const int N = i % a.na;
            const double* Rv = posr + ((size_t)mu * a.na + N) * 3;
            const double qr = i < a.na ? (q1x * Rv[0] + q1y * Rv[1] + q1z * Rv[2])
                                       : (q2x * Rv[0] + q2y * Rv[1] + q2z * Rv[2]);
            double sn, cs;
            sincos(qr, &sn, &cs);
            (i < a.na ? sP1 : sP2)[N] = make_double2(cs, sn);
        }
        __syncthreads();
        // E1, E2: [k = N*3 + b][s]
        for (int i = tid; i < 2 * K * n; i += nt) {
            const int which = i / (K * n), j = i % (K * n);
            const int k = j / n, s = j % n;
            const int N = k / 3, b = k % 3;
            const int nu = btyp[mu * a.na + N];
            const double2 ph = (which ? sP2 : sP1)[N];
            const double2 ev = (which ? e2 : e1)[s * n + 3 * nu + b];
            const double m = mrs[nu];
            (which ? sE2 : sE1)[j] = make_double2(m * (ph.x * ev.x - ph.y * ev.y), m * (ph.x * ev.y + ph.y * ev.x));
        }
        __syncthreads();
        // Y[r][s2] = sum_k FC[k][r] E2[k][s2]
        for (int o = tid; o < R * n; o += nt) {
            const int r = o / n, s2 = o % n;
            double yr = 0.0, yi = 0.0;
            for (int k = 0; k < K; ++k) {
                const double fv = sFC[k * R + r];
                const double2 e = sE2[k * n + s2];
                yr = fma(fv, e.x, yr);
                yi = fma(fv, e.y, yi);
            }
            sY[o] = make_double2(yr, yi);
        }
        __syncthreads();
        // Z[al][s1][s2] = sum_{N1, b} E1[N1*3+b][s1] Y[(N1*3+al)*3+b][s2]
        for (int o = tid; o < 3 * n * n; o += nt) {
            const int al = o / (n * n), s1 = (o / n) % n, s2 = o % n;
            double zr = 0.0, zi = 0.0;
            for (int N1 = 0; N1 < a.na; ++N1)
                for (int b = 0; b < 3; ++b) {
                    const double2 x = sE1[(N1 * 3 + b) * n + s1];
                    const double2 y = sY[((N1 * 3 + al) * 3 + b) * n + s2];
                    zr = fma(x.x, y.x, zr);
                    zr = fma(-x.y, y.y, zr);
                    zi = fma(x.x, y.y, zi);
                    zi = fma(x.y, y.x, zi);
                }
            sZ[o] = make_double2(zr, zi);
        }
        __syncthreads();
        // Phi[s0][s1][s2] += sum_al m_mu^-1/2 e0(3 mu + al, s0) Z[al][s1][s2]
        const double mm = mrs[mu];
        for (int o = tid; o < nphi; o += nt) {
            const int s0 = s0b + o / (n * n), r12 = o % (n * n);
            double2 acc = sPhi[o];
            for (int al = 0; al < 3; ++al) {
                double2 w = e0[s0 * n + 3 * mu + al];
                w.x *= mm;
                w.y *= mm;
                const double2 z = sZ[al * n * n + r12];
                acc.x = fma(w.x, z.x, acc.x);
                acc.x = fma(-w.y, z.y, acc.x);
                acc.y = fma(w.x, z.y, acc.y);
                acc.y = fma(w.y, z.x, acc.y);
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
        const int s0 = s0b + o / (n * n), s1 = (o / n) % n, s2 = o % n;
        double W = 0.0;
        if (!((gq0 && s0 < 3) || (gq1 && s1 < 3) || (gq2 && s2 < 3))) {
            const double2 p = sPhi[o];
            const double abs2 = p.x * p.x + p.y * p.y;
            W = abs2 * (ob0[(size_t)q0 * n + s0] * obg[(size_t)g1 * n + s1] * obg[(size_t)g2 * n + s2]) * a.mfac;
        }
        if (EPI == 1) {
            const int slot = q0 - a.q0_first;
            const size_t n3 = (size_t)n * n * n;
            out_w[((size_t)slot * a.nq + g1) * n3 + (s0 * n + s1) * n + s2] = W;
            if (g1 != g2) out_w[((size_t)slot * a.nq + g2) * n3 + (s0 * n + s2) * n + s1] = W;
        } else {
            if (s0 < a.pol_lo[0] || s0 > a.pol_hi[0] || s1 < a.pol_lo[1] || s1 > a.pol_hi[1] || s2 < a.pol_lo[2] ||
                s2 > a.pol_hi[2] || (gq1 && s1 < 3) || (gq2 && s2 < 3))
                continue;
            const double w0 = om0[(size_t)q0 * n + s0];
            const double w1 = omg[(size_t)g1 * n + s1];
            const double w2 = omg[(size_t)g2 * n + s2];
            const double d1 = w0 - w1 - w2, d2 = w0 + w1 - w2, d3 = w0 - w1 + w2;
            const double pre = a.onebysigma * ONEBYSQRT2PI;
            const double e1v = pre * exp(-0.5 * a.onebysigma2 * (d1 * d1));
            const double e2v = pre * exp(-0.5 * a.onebysigma2 * (d2 * d2));
            const double e3v = pre * exp(-0.5 * a.onebysigma2 * (d3 * d3));
            for (int t = 0; t < a.nT; ++t) {
                const double n1 = nbeg[((size_t)t * a.nq + g1) * n + s1];
                const double n2 = nbeg[((size_t)t * a.nq + g2) * n + s2];
                const double v = W * (((n1 + n2 + 1.0) * e1v) + ((n1 - n2) * (e2v - e3v)));
                atomicAdd(&sLw[t * sb + (s0 - s0b)], v);
            }
            atomicAdd(&sLw[a.nT * sb + (s0 - s0b)], e1v + e2v + e3v);
        }
    }
    if (EPI == 0) {
        __syncthreads();
        const double mult = g1 != g2 ? 2.0 : 1.0;
        for (int i = tid; i < (a.nT + 1) * sb; i += nt) {
            const int t = i / sb, s0 = s0b + i % sb;
            if (s0 >= n) continue;
            if (t < a.nT)
                atomicAdd(&out_lw[((size_t)t * a.nq0 + q0) * n + s0], mult * sLw[i]);
            else
                atomicAdd(&out_p3[(size_t)q0 * n + s0], mult * sLw[i]);
        }
    }
}

size_t v3_smem(int n, int na, int sb, int nT) {
    const int K = 3 * na, R = 9 * na;
    return sizeof(double) * ((K * R + 1) & ~1) + sizeof(double2) * (2 * K * n + R * n + 3 * n * n + sb * n * n + 2 * na) +
           sizeof(double) * (nT + 1) * sb;
}

int v3_block(int n) {
    // s0 block: the whole range for small cells; chunks for Ndof 24
    return n <= 12 ? n : 6;
}

template <int EPI>
int launch_v3(spring_ctx* c, int q0_first, int n_q0, V3Args a, double* lw, double* p3, double* w) {
    a.nb = c->nb;
    a.n = c->ndof;
    a.na = c->na3;
    a.nq = c->nq;
    a.nq0 = c->nq0;
    a.nT = c->nT;
    a.q0_first = q0_first;
    a.sb = v3_block(c->ndof);
    a.nsb = (c->ndof + a.sb - 1) / a.sb;
    a.mfac = host_constants().Sctr3THz2 / double(c->nq);
    const int p0 = c->h_pairoff[q0_first], p1 = c->h_pairoff[q0_first + n_q0];
    a.pair_first = p0;
    const size_t smem = v3_smem(a.n, a.na, a.sb, a.nT);
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "V3 tile needs %zu bytes of shared memory", smem);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_v3<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long items = (long long)(p1 - p0) * a.nsb;
    if (items == 0) return SPRING_OK;
    if (items > 0x7fffffffLL) return fail(c, SPRING_ERR_UNSUPPORTED, "too many V3 work items");
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3: injected launch failure");
    k_v3<EPI><<<(unsigned)items, 128, smem, c->stream>>>(
        a, c->d_pairs.p, c->d_pair_q0.p, c->d_fc3t.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p, c->d_qpnt.p,
        c->d_irr_int.p, c->ph_irr.evec.p, c->ph_irr.omega.p, c->ph_irr.oneby.p, c->ph_grid.evec.p, c->ph_grid.omega.p,
        c->ph_grid.oneby.p, c->ph_grid.nbe.p, lw, p3, w);
    return launch_check(c, EPI == 0 ? "k_v3<gauss>" : "k_v3<wgrid>");
}

}  // namespace

int run_v3_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3) {
    V3Args a{};
    a.onebysigma = 1.0 / sigma;
    a.onebysigma2 = a.onebysigma * a.onebysigma;
    for (int k = 0; k < 3; ++k) {
        a.pol_lo[k] = pol.lo[k];
        a.pol_hi[k] = pol.hi[k];
    }
    return launch_v3<0>(c, q0_first, n_q0, a, d_lw, d_p3, nullptr);
}

int run_v3_wgrid(spring_ctx* c, int q0_first, int n_q0, double* d_w) {
    V3Args a{};
    return launch_v3<1>(c, q0_first, n_q0, a, nullptr, nullptr, d_w);
}

}  // namespace spring
