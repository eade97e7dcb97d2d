// Three-phonon matrix elements V3 -> W (FP64) and their Gaussian delta sum.
//
// Reference: ScatterProbAllq1 / ScatterMatEl / ScatterProbability
// (src/Kappa/Src/ThirdOrder_m.f90:41-166, 278-386, 389-439) and the Gaussian
// linewidth CalculateLinewidth (:442-543).
//
// The reference evaluates Phi(s2,s1,s) in a 9-deep loop (~Na3^2*27*Ndof^3
// complex MACs per pair).  Here the sum is regrouped: the neighbour phases
// depend on the neighbour slot while the eigenvectors depend only on its basis
// atom, so the phases are folded into the force constants first,
//   D_mu[a][nu b][eta c] = sum_{N1 in nu, N2 in eta} FC3(c,b,a,N2,N1,mu)
//                          e^{i q1.R_N1} e^{i q2.R_N2} m_nu^-1/2 m_eta^-1/2,
// and the eigenvectors enter through three Ndof^4 contractions:
//   T1[a][nu b][s2] = sum_{eta c} D_mu[a][nu b][eta c] e2(eta c, s2)
//   T2[a][s1][s2]   = sum_{nu b}  e1(nu b, s1) T1[a][nu b][s2]
//   Phi[s0][s1][s2] += sum_a m_mu^-1/2 e0(mu a, s0) T2[a][s1][s2]
// 4*27*sum_mu Na3^2 + 3*8*Ndof^4 flops per pair (41.7 kflop for the 2-atom cell).
// W = |Phi|^2 (1/w0)(1/w1)(1/w2) Sctr3THz2/Nq, zero for Gamma acoustic modes.
//
// One CTA handles one (pair, block of s0) work item, so that every tensor fits
// in shared memory up to Ndof = 24.  Two epilogues:
//   GAUSS: the pair's contribution to Gamma(q0,s0) for every temperature, fused
//          (W never leaves the SM).  The reference sums over every grid q1; the
//          q2-side term of a pair equals its q1-side term exactly (swap s1<->s2),
//          so each pair is weighted by 2 (1 when q1 == q2).  exp() is skipped
//          where it underflows to 0 (argument below -745.2), which leaves every
//          sum bit-identical to evaluating it.
//   WGRID: W for q1 and its s1<->s2 transpose for q2, i.e. the reference's
//          Sctrq1(s2,s1,s0,q) for every grid q, for the tetrahedron integration.
// Roofline: FP64 FMA pipe; inputs per pair are two eigenvector sets (2 Ndof^2
// complex, L2-resident), outputs a few atomics (GAUSS) or 2 Ndof^3 doubles (WGRID).
#include <algorithm>

#include "v3item.cuh"

namespace spring {
namespace {

// range != null: the pair range is read on the device, pairs range[0] .. range[n_q0] (clamped to
// the list's capacity); the grid then covers the bound and CTAs past the range return at once.
template <int EPI>
__global__ void __launch_bounds__(128) k_v3(V3Args a_, V3Ptrs P_, const int* __restrict__ range, int n_q0, int cap) {
    extern __shared__ double2 smem2[];
    V3Args a = a_;  // local copies: the device function takes references
    const V3Ptrs P = P_;
    const int work = blockIdx.x;
    if (range) {
        a.pair_first = min(range[0], cap);
        const int pr = a.pair_first + work / a.nsb;
        if (pr >= min(range[n_q0], cap)) return;
    }
    v3_item<EPI>(a, P, a.pair_first + work / a.nsb, (work % a.nsb) * a.sb, smem2);
}

template <int EPI>
int launch_v3(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, V3Args a, double* lw,
              double* p3, double* w) {
    a.nb = c->nb;
    a.n = c->ndof;
    a.na = c->na3;
    a.nq = c->nq;
    a.nq0 = ps.n0;
    a.nT = c->nT;
    a.q0_first = q0_first;
    a.sb = v3_block(c->ndof);
    a.nsb = (c->ndof + a.sb - 1) / a.sb;
    a.mfac = host_constants().Sctr3THz2 / double(c->nq);
    // Host offsets when they were read already; otherwise the range is read on the device and the
    // grid covers the bound of at most Nq/2 + 8 pairs per q0 (no readback, no wait).
    const int* range = nullptr;
    long long npairs;
    if (ps.h_ok) {
        a.pair_first = ps.h_pairoff[q0_first];
        npairs = ps.h_pairoff[q0_first + n_q0] - a.pair_first;
    } else {
        range = ps.pairoff.p + q0_first;
        npairs = std::min<long long>((long long)n_q0 * (c->nq / 2 + 8), ps.cap);
    }
    const size_t smem = v3_smem(a.n, a.na, a.sb, a.nT);
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "V3 tile needs %zu bytes of shared memory", smem);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_v3<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long items = npairs * a.nsb;
    if (items == 0) return SPRING_OK;
    if (items > 0x7fffffffLL) return fail(c, SPRING_ERR_UNSUPPORTED, "too many V3 work items");
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3: injected launch failure");
    const V3Ptrs P{ps.pairs.p, ps.pair_q0.p, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p,
                   c->d_qpnt.p, v.q0_int, v.q0_grid, v.evec, v.omega, v.oneby, c->ph_grid.evec.p,
                   c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p, lw, p3, w};
    k_v3<EPI><<<(unsigned)items, 128, smem, c->stream>>>(a, P, range, n_q0, ps.cap);
    return launch_check(c, EPI == 0 ? "k_v3<gauss>" : "k_v3<wgrid>");
}

}  // namespace

Q0View irr_view(spring_ctx* c) {
    return Q0View{c->d_irr_int.p, nullptr, c->ph_irr.evec.p, c->ph_irr.omega.p, c->ph_irr.oneby.p};
}

int run_v3_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3) {
    bool handled = false;
    if (c->precision != SPRING_FP64) {
        SPRING_CHECK(run_v3tc_gauss(c, q0_first, n_q0, sigma, pol, d_lw, d_p3, &handled));
        if (handled) return SPRING_OK;
    }
    if (!c->force_generic_v3) {
        // optional: only the pairs with a mode triple inside the Gaussian's exp(-40) window (the
        // tensor-core path's pre-screen), every weight of the others being below that cut
        const int* plist = nullptr;
        int nlist = 0;
        if (c->fp64_prescreen && c->nb == 2 && c->na3 <= 8) {
            SPRING_CHECK(run_v3_prescreen(c, q0_first, n_q0, sigma, &plist, &nlist));
            if (nlist == 0) return SPRING_OK;
        }
        SPRING_CHECK(launch_v3s(c, c->ps_irr, irr_view(c), q0_first, n_q0, 0, sigma, &pol, d_lw, d_p3, nullptr,
                                &handled, plist, nlist));
    }
    if (handled) return SPRING_OK;
    V3Args a{};
    a.onebysigma = 1.0 / sigma;
    a.onebysigma2 = a.onebysigma * a.onebysigma;
    for (int k = 0; k < 3; ++k) {
        a.pol_lo[k] = pol.lo[k];
        a.pol_hi[k] = pol.hi[k];
    }
    return launch_v3<0>(c, c->ps_irr, irr_view(c), q0_first, n_q0, a, d_lw, d_p3, nullptr);
}

int run_v3_wgrid(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, double* d_w) {
    bool handled = false;
    if (!c->force_generic_v3)
        SPRING_CHECK(launch_v3s(c, ps, v, q0_first, n_q0, 1, 0.0, nullptr, nullptr, nullptr, d_w, &handled));
    if (handled) return SPRING_OK;
    V3Args a{};
    return launch_v3<1>(c, ps, v, q0_first, n_q0, a, nullptr, nullptr, d_w);
}

}  // namespace spring
