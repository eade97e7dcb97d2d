// Momentum-conserving pair enumeration on the device (3-phonon).
//
// Reference: MomentumConsrv3rd (src/Kappa/Src/QuasiMomentumConsrv3rd_m.f90:13-158).
// The reference walks q1 in grid order, finds q2 = G - (q0 + q1) with G the
// first of (0,+1,-1)^3 * N (c1 fastest) that puts q2 inside [-N/2, N/2]^3,
// records the pair, and marks q2 as covered when the integer vectors of q1 and
// q2 differ.  That sequential loop has a closed form that every thread can
// evaluate for itself:
//   - the first admissible G is chosen component by component (the search is
//     lexicographic over independent per-component conditions);
//   - q1 -> p(q1) = grid(-q0 - q1) is an involution, and p(q1) != q1 implies
//     the integer vectors differ, so q1 is a pair representative iff p(q1) >= q1;
//   - the pair number of a representative is 1 + the number of representatives
//     before it (an exclusive scan).
// The outputs (Allq1q2, q1q2_permuted, counts), including the even-mesh case
// where q1 == p(q1) but the integer vectors differ (the reference then
// overwrites the direct entry with flag 0), are bit-identical to the
// reference algorithm's.  HBM bound: 8 bytes per pair written.
#include <algorithm>
#include <cub/cub.cuh>

#include "spring_internal.cuh"

namespace spring {
namespace {

__device__ __forceinline__ int imod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// q2 integer vector for (q0, q1) and its grid index.
__device__ __forceinline__ int partner3(const int* q0, const int* q1, int n0, int n1, int n2, int* q2) {
    const int nn[3] = {n0, n1, n2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int b = nn[d] / 2;
        const int v = -(q0[d] + q1[d]);
        int w = v;
        if (w > b || w < -b) {
            w = v + nn[d];
            if (w > b || w < -b) w = v - nn[d];
        }
        q2[d] = w;
    }
    return imod(q2[0], n0) + n0 * (imod(q2[1], n1) + n1 * imod(q2[2], n2));
}

// Every (q0, q1): partner and representative flag.
__global__ void k_enum3_flags(int nq, int nq0, int n0, int n1, int n2, const int* __restrict__ irr,
                              const int* __restrict__ qint, int* __restrict__ partner, int* __restrict__ rep) {
    const long long total = (long long)nq0 * nq;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int q0 = (int)(i / nq), g = (int)(i % nq);
        int q2[3];
        const int p = partner3(irr + 3 * q0, qint + 3 * g, n0, n1, n2, q2);
        partner[i] = p;
        rep[i] = p >= g ? 1 : 0;
    }
}

// Pairs beyond `cap` are not written.  cap is the proven bound (at most Nq/2 + 8 pairs per q0), so
// nothing is dropped; pairoff_host fails with an error if the total ever exceeded it, and kernels
// that read their pair range on the device clamp it to cap.
__global__ void k_enum3_pairs(int nq, int nq0, int cap, const int* __restrict__ partner, const int* __restrict__ rep,
                              const int* __restrict__ pos, int2* __restrict__ pairs, int* __restrict__ pair_q0,
                              int* __restrict__ pairoff) {
    const long long total = (long long)nq0 * nq;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int q0 = (int)(i / nq), g = (int)(i % nq);
        if (g == 0) pairoff[q0] = pos[i];
        if (i == total - 1) pairoff[nq0] = pos[i] + rep[i];
        if (rep[i] && pos[i] < cap) {
            pairs[pos[i]] = make_int2(g, partner[i]);
            pair_q0[pos[i]] = q0;
        }
    }
}

// Fortran-layout outputs for one q0 (1-based indices).
__global__ void k_enum3_fortran(int nq, int n0, int n1, int n2, const int* __restrict__ q0v,
                                const int* __restrict__ qint, const int* __restrict__ partner,
                                const int* __restrict__ pos, int base, int* __restrict__ allq1q2,
                                int* __restrict__ perm, int* __restrict__ counts) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
        int q2[3];
        const int* q1 = qint + 3 * g;
        const int p = partner3(q0v, q1, n0, n1, n2, q2);
        const bool flag = q1[0] != q2[0] || q1[1] != q2[1] || q1[2] != q2[2];
        int4 e;
        if (p >= g) {
            const int cnt = pos[g] - base + 1;
            e = (p == g && flag) ? make_int4(0, cnt, g + 1, g + 1) : make_int4(1, cnt, g + 1, p + 1);
            perm[2 * (cnt - 1)] = g + 1;
            perm[2 * (cnt - 1) + 1] = p + 1;
            atomicAdd(&counts[0], 1);
            atomicAdd(&counts[1], flag ? 2 : 1);
        } else {
            e = make_int4(0, pos[p] - base + 1, g + 1, p + 1);
        }
        reinterpret_cast<int4*>(allq1q2)[g] = e;
    }
}

}  // namespace

int run_exclusive_scan(spring_ctx* c, const int* d_in, int* d_out, int n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, d_in, d_out, n, c->stream);
    SPRING_CHECK(dalloc(c, c->d_scan_tmp, (bytes + sizeof(int) - 1) / sizeof(int), "scan scratch"));
    cudaError_t e = cub::DeviceScan::ExclusiveSum(c->d_scan_tmp.p, bytes, d_in, d_out, n, c->stream);
    c->launches += 1;
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, "exclusive scan");
}

int pairoff_host(spring_ctx* c, const PairSet& ps) {
    if (ps.h_ok) return SPRING_OK;
    ps.h_pairoff.assign(ps.n0 + 1, 0);
    SPRING_CHECK(d2h(c, ps.h_pairoff.data(), ps.pairoff.p, sizeof(int) * (ps.n0 + 1), "pair offsets"));
    if (ps.h_pairoff[ps.n0] > ps.cap) return fail(c, SPRING_ERR_CUDA, "enumerate3: %d pairs exceed the list's %d",
                                                 ps.h_pairoff[ps.n0], ps.cap);
    ps.h_ok = true;
    return SPRING_OK;
}

int run_enumerate3(spring_ctx* c, PairSet& ps) {
    ps.done = false;
    const long long total = (long long)ps.n0 * c->nq;
    if (total > 0x7fffffffLL) return fail(c, SPRING_ERR_UNSUPPORTED, "Nq0 * Nq exceeds 2^31");
    DBuf<int>& rep = c->d_scr_rep;
    SPRING_CHECK(dalloc(c, ps.partner, total, "partner map"));
    int rc = dalloc(c, rep, total, "representative flags");
    if (rc == SPRING_OK) rc = dalloc(c, ps.pairpos, total, "pair positions");
    const int threads = 256;
    const int blocks = (int)std::min<long long>((total + threads - 1) / threads, 148LL * 32);
    if (rc == SPRING_OK && launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "enumerate3: injected launch failure");
    if (rc == SPRING_OK) {
        k_enum3_flags<<<blocks, threads, 0, c->stream>>>(c->nq, ps.n0, c->mesh[0], c->mesh[1], c->mesh[2],
                                                         ps.q0_int, c->d_qint.p, ps.partner.p, rep.p);
        rc = launch_check(c, "k_enum3_flags");
    }
    if (rc == SPRING_OK) rc = run_exclusive_scan(c, rep.p, ps.pairpos.p, (int)total);
    // The pair list is sized without a readback: q1 is a representative iff its partner p(q1) >= q1,
    // so each q0 has at most (Nq + F) / 2 of them, F <= 8 the points with p(q1) = q1 (two solutions
    // of 2 x = c mod N per dimension).  The writes are guarded all the same, and pairoff_host checks
    // the total when the offsets are first read.
    const long long bound = std::min<long long>(total, (long long)ps.n0 * (c->nq / 2 + 8));
    const int cap = (int)std::max<long long>(bound, 1);
    if (rc == SPRING_OK) rc = dalloc(c, ps.pairoff, ps.n0 + 1, "pair offsets");
    if (rc == SPRING_OK) rc = dalloc(c, ps.pairs, cap, "pair list");
    if (rc == SPRING_OK) rc = dalloc(c, ps.pair_q0, cap, "pair list");
    if (rc == SPRING_OK && launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "enumerate3: injected launch failure");
    if (rc == SPRING_OK) {
        k_enum3_pairs<<<blocks, threads, 0, c->stream>>>(c->nq, ps.n0, cap, ps.partner.p, rep.p, ps.pairpos.p,
                                                         ps.pairs.p, ps.pair_q0.p, ps.pairoff.p);
        rc = launch_check(c, "k_enum3_pairs");
    }
    ps.cap = cap;
    ps.h_ok = false;
    if (rc == SPRING_OK) {
        ps.done = true;
        ps.gen += 1;
    }
    return rc;
}

int run_enumerate3_fortran(spring_ctx* c, int q0, int* d_allq1q2, int* d_perm, int* d_counts) {
    PairSet& ps = c->ps_irr;
    if (!ps.done) SPRING_CHECK(run_enumerate3(c, ps));
    SPRING_CHECK(pairoff_host(c, ps));
    const int* p = ps.pairpos.p + (size_t)q0 * c->nq;
    const int base = ps.h_pairoff[q0];
    SPRING_CHECK(zero(c, d_counts, 2 * sizeof(int), "counts"));
    const int threads = 256, blocks = (c->nq + threads - 1) / threads;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "enumerate3: injected launch failure");
    k_enum3_fortran<<<blocks, threads, 0, c->stream>>>(c->nq, c->mesh[0], c->mesh[1], c->mesh[2],
                                                       ps.q0_int + 3 * q0, c->d_qint.p,
                                                       ps.partner.p + (size_t)q0 * c->nq, p, base, d_allq1q2, d_perm,
                                                       d_counts);
    return launch_check(c, "k_enum3_fortran");
}

}  // namespace spring
