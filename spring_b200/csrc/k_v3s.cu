// V3 -> W for two-atom cells (Ndof = 6) with 7-slot neighbour clusters: the
// shapes of the rocksalt benchmark crystal, with every extent a compile-time
// constant.  Same mathematics and epilogues as k_v3.cu (see there for the
// reference citations); this kernel differs only in how the work is laid out:
//
//   - 8 pairs per CTA and 288 threads, so each contraction stage gives every
//     thread exactly one 6-wide output row (36 rows per pair and stage);
//   - the phases are folded into FC3 first (D_mu[a][nu b][eta c], one thread per
//     (pair, mu, abc) looping over the slot pairs of each basis block, the slots
//     being grouped by basis atom on the host), then three 6x6 complex
//     contractions T1 = D e2, T2 = e1^T T1, Phi = e0^T T2;
//   - Phi stays in registers and feeds the epilogue directly;
//   - rows in shared memory are padded to 7 complex so that the 128-bit loads of
//     8 consecutive threads hit distinct banks;
//   - the grid is persistent (FC3 is staged once per CTA).
// Roofline: FP64 FMA (41.7 kflop per pair) with shared-memory operands.
#include <algorithm>

#include "v3sitem.cuh"

namespace spring {
namespace {

using namespace s3;

// range != null: the pair range is read on the device, pairs range[0] .. range[n_q0] (the pair
// offsets of the enumeration, clamped to the list's capacity), instead of a.pair_first/pair_end.
template <int EPI>
__global__ void __launch_bounds__(THREADS, 2) k_v3s(S3Args a_, S3Ptrs P_, const int* __restrict__ range, int n_q0,
                                                    int cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    S3Args a = a_;  // local copies: the device functions take references
    const S3Ptrs P = P_;
    if (range) {
        a.pair_first = min(range[0], cap);
        a.pair_end = min(range[n_q0], cap);
        a.ngroups = (a.pair_end - a.pair_first + PP - 1) / PP;
    }
    v3s_stage(S, P);
    for (int grp = blockIdx.x; grp < a.ngroups; grp += gridDim.x) v3s_group<EPI>(S, a, P, grp);
}

}  // namespace

// Launch the specialised kernel when the cell fits it; *handled tells the caller.
int launch_v3s(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, int epi, double sigma,
               const Pol* pol, double* lw, double* p3, double* w, bool* handled, const int* plist, int nlist) {
    *handled = false;
    if (c->nb != NB || c->na3 != NA || c->nT > MAXT) return SPRING_OK;
    *handled = true;
    S3Args a{};
    a.nq = c->nq;
    a.nT = c->nT;
    a.nq0 = ps.n0;
    a.q0_first = q0_first;
    // Host offsets when they were read already; otherwise the kernel reads its range on the device
    // and the grid is sized by the bound of at most Nq/2 + 8 pairs per q0 (no readback, no wait).
    const int* range = nullptr;
    a.plist = plist;
    if (plist) {  // an explicit list of pairs (the Gaussian window's pre-screen)
        a.pair_first = 0;
        a.pair_end = nlist;
        a.ngroups = (nlist + PP - 1) / PP;
    } else if (ps.h_ok) {
        a.pair_first = ps.h_pairoff[q0_first];
        a.pair_end = ps.h_pairoff[q0_first + n_q0];
        a.ngroups = (a.pair_end - a.pair_first + PP - 1) / PP;
    } else {
        range = ps.pairoff.p + q0_first;
        const long long bound = std::min<long long>((long long)n_q0 * (c->nq / 2 + 8), ps.cap);
        a.ngroups = (int)((bound + PP - 1) / PP);
    }
    a.mfac = host_constants().Sctr3THz2 / double(c->nq);
    if (epi == 0) {
        a.onebysigma = 1.0 / sigma;
        a.onebysigma2 = a.onebysigma * a.onebysigma;
        for (int k = 0; k < 3; ++k) {
            a.pol_lo[k] = pol->lo[k];
            a.pol_hi[k] = pol->hi[k];
        }
    }
    if (a.ngroups == 0) return SPRING_OK;
    const size_t smem = sizeof(Smem);
    auto kern = epi == 0 ? k_v3s<0> : k_v3s<1>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    const int grid = std::min(a.ngroups, dev_sms * 2);
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3: injected launch failure");
    const S3Ptrs P{ps.pairs.p, ps.pair_q0.p, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_fc3_off.p,
                   c->d_mass_rs.p, c->d_qpnt.p, v.q0_int, v.q0_grid, v.evec, v.omega, v.oneby, c->ph_grid.evec.p,
                   c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p, lw, p3, w};
    kern<<<grid, THREADS, smem, c->stream>>>(a, P, range, n_q0, ps.cap);
    return launch_check(c, epi == 0 ? "k_v3s<gauss>" : "k_v3s<wgrid>");
}

// Entries of the Gaussian BTE operator (EPI 2) of pair set ps, q0 block [q0_first, +n_q0): every
// mode triple with a delta weight above the exp(-40) cut is appended to `items` (capacity cap) at
// *ctr (zeroed by the caller); *ctr ends as the number of entries, those past cap not written.
int launch_v3s_bte(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, double sigma,
                   void* items, unsigned long long* ctr, long long cap, bool* handled) {
    *handled = false;
    if (c->nb != NB || c->na3 != NA) return SPRING_OK;
    *handled = true;
    S3Args a{};
    a.nq = c->nq;
    a.nT = c->nT;
    a.nq0 = ps.n0;
    a.q0_first = q0_first;
    a.plist = nullptr;
    SPRING_CHECK(pairoff_host(c, ps));
    a.pair_first = ps.h_pairoff[q0_first];
    a.pair_end = ps.h_pairoff[q0_first + n_q0];
    a.ngroups = (a.pair_end - a.pair_first + PP - 1) / PP;
    a.mfac = host_constants().Sctr3THz2 / double(c->nq);
    a.onebysigma = 1.0 / sigma;
    a.onebysigma2 = a.onebysigma * a.onebysigma;
    if (a.ngroups == 0) return SPRING_OK;
    const size_t smem = sizeof(Smem);
    cudaFuncSetAttribute(k_v3s<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device);
    const int grid = std::min(a.ngroups, dev_sms * 2);
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3: injected launch failure");
    S3Ptrs P{ps.pairs.p, ps.pair_q0.p, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_fc3_off.p,
             c->d_mass_rs.p, c->d_qpnt.p, v.q0_int, v.q0_grid, v.evec, v.omega, v.oneby, c->ph_grid.evec.p,
             c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p, nullptr, nullptr, nullptr};
    P.out_items = items;
    P.item_ctr = ctr;
    P.item_cap = cap;
    k_v3s<2><<<grid, THREADS, smem, c->stream>>>(a, P, nullptr, n_q0, ps.cap);
    return launch_check(c, "k_v3s<bte>");
}

}  // namespace spring
