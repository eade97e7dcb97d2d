// Iterative (non-RTA) Boltzmann transport of kappa_iter.x on the device.
//
// Reference (src/Kappa/Src_iterative): the time-reversal irreducible set
// (Irr_q_point_m.f90:216-335), W+ = W (n1 - n2) and W- = W (1 + n1 + n2) per
// pair (Quasi_momentum_consrv.f90:567-621, Sctr3THz2 with pi/4), 1/tau from the
// tetrahedron sums TetrahedronWplus / TetrahedronWminus (:701-1208, strict case
// bounds, a vertex set counts only when |sum I - 1| < 5e-5), CreateFzero,
// TetrahedronIterPlus / Minus (TetrahedronDeltaSum.f90:22-607), multiplyTaudFnew,
// kappa (HelperSubroutines.f90:118-347) and the loop of main.f90:295-361.
//
// Representatives of the time-reversal pairs {q, -q} are the smaller grid
// index (the reference takes the first one met while building tetrahedra);
// F(-q) = -F(q).  The W of a vertex comes from kappa.x's W grid of the same q0,
// which stores both orientations of every pair; 4 W there is kappa_iter's W.
//   plus  channel, vertex x:  partner -p(x),  M = w(-p(x),s2) - w(x,s1),
//                             W+ = 4 W3(q0; x s1; p(x) s2) (n(x,s1) - n(p(x),s2)),
//                             dF term (F(-p(x),s2) - F(x,s1));
//   minus channel, vertex v:  partner u = -p(-v), M = w(v,s1) + w(u,s2),
//                             W- = 4 W3(q0; -v s1; p(-v) s2) (1 + n(-v,s1) + n(p(-v),s2)),
//                             dF term 0.5 (F(u,s2) + F(v,s1));
// with p(x) = grid(-q0 - x).  One thread per (q0, tetrahedron, s1, s2) sorts each
// channel's vertex energies once (stable) and loops over s0.  The W grids of
// every q0 are computed once and kept in HBM when they fit a 40 GB budget, and
// otherwise recomputed batch by batch on every pass.
// Roofline: FP64 ALU (divisions of the tetrahedron weights), like k_tetra3.
#include <algorithm>
#include <cmath>
#include <cub/cub.cuh>

#include "spring_internal.cuh"
#include "tetra.cuh"
#include "v3sitem.cuh"

namespace spring {
namespace {

constexpr int NS0 = 6;
constexpr double ZERO_PREC = 5.0e-5;
constexpr double FUNIT_E = 1.054571817 / 1.380649;  // FunitE_11m_K (Src_iterative/constants.f90:56)
constexpr double KW_MK = 1.054571817 * 0.001;       // kW_mK (:58)

struct PassArgs {
    int n, nq, ntet, q0_first, s0a, s0n;
    const int* tr_grid;   // [ntr]
    const int* tr_pos;    // [nq]
    const int* tr_sgn;    // [nq]
    const int* neg;       // [nq]
    const int* partner;   // [ntr][nq]
    const double* wgrid;  // [slot][nq][n^3] for q0_first ..
    const double* omega;  // [nq][n]
    const double* nbe;    // [nq][n] at this temperature
    const double* F;      // [ntr][n][3] (MODE 1)
    double* out;          // MODE 0: inv_tau [ntr][n]; MODE 1: dF [ntr][n][3]
};

template <int MODE>
__global__ void __launch_bounds__(128) k_bte_pass(PassArgs a, const int4* __restrict__ tet) {
    constexpr int NC = MODE == 0 ? 1 : 3;
    __shared__ double sacc[NS0 * 3];
    const int slot = blockIdx.y;
    const int q0 = a.q0_first + slot;
    const int n = a.n;
    const size_t n3 = (size_t)n * n * n;
    const int g0 = a.tr_grid[q0];
    const int* p = a.partner + (size_t)q0 * a.nq;
    const double* W3 = a.wgrid + (size_t)slot * a.nq * n3;
    for (int i = threadIdx.x; i < NS0 * 3; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    double acc[NS0][NC];
#pragma unroll
    for (int s = 0; s < NS0; ++s)
#pragma unroll
        for (int k = 0; k < NC; ++k) acc[s][k] = 0.0;

    const long long items = (long long)a.ntet * n * n;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int s2 = (int)(it % n), s1 = (int)((it / n) % n), t = (int)(it / ((long long)n * n));
        const int4 tv = tet[t];
        const int x[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            int part[4], wrow[4];
            double M[4], Wf[4];  // Wf: the occupation factor; W3 is read per s0
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (ch == 0) {
                    const int px = p[x[v]];
                    part[v] = a.neg[px];
                    wrow[v] = x[v];
                    M[v] = a.omega[(size_t)part[v] * n + s2] - a.omega[(size_t)x[v] * n + s1];
                    Wf[v] = a.nbe[(size_t)x[v] * n + s1] - a.nbe[(size_t)px * n + s2];
                } else {
                    const int y = a.neg[x[v]];
                    const int py = p[y];
                    part[v] = a.neg[py];
                    wrow[v] = y;
                    M[v] = a.omega[(size_t)x[v] * n + s1] + a.omega[(size_t)part[v] * n + s2];
                    Wf[v] = 1.0 + a.nbe[(size_t)y * n + s1] + a.nbe[(size_t)py * n + s2];
                }
            }
            int pm[4];
            tet::sort4(M, pm);
            double S[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) S[v] = M[pm[v]];
            // F terms per vertex (MODE 1): plus F(part,s2) - F(x,s1); minus F(part,s2) + F(x,s1)
            double Fc[4][NC];
            if (MODE == 1) {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int xv = x[pm[v]], pv = part[pm[v]];
                    const double sx = a.tr_sgn[xv], sp = a.tr_sgn[pv];
                    const double* f1 = a.F + ((size_t)a.tr_pos[xv] * n + s1) * 3;
                    const double* f2 = a.F + ((size_t)a.tr_pos[pv] * n + s2) * 3;
#pragma unroll
                    for (int k = 0; k < NC; ++k)
                        Fc[v][k] = ch == 0 ? (sp * f2[k] - sx * f1[k]) : (sp * f2[k] + sx * f1[k]);
                }
            }
#pragma unroll
            for (int si = 0; si < NS0; ++si) {
                if (si >= a.s0n) break;
                const int s0 = a.s0a + si;
                const double Mqs = a.omega[(size_t)g0 * n + s0];
                double g, I[4];
                if (!tet::g_iver<true>(Mqs, S, g, I)) continue;
                if (!(fabs(I[0] + I[1] + I[2] + I[3] - 1.0) < ZERO_PREC)) continue;
                const double pre = ch == 0 ? ONEBYSIX * g : 0.5 * ONEBYSIX * g;
                double tv[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) tv[k] = 0.0;
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int q = pm[v];
                    const double Wv = 4.0 * W3[(size_t)wrow[q] * n3 + (s0 * n + s1) * n + s2] * Wf[q];
                    if (MODE == 0) {
                        tv[0] += I[v] * Wv;
                    } else {
#pragma unroll
                        for (int k = 0; k < NC; ++k) tv[k] += (I[v] * Wv) * Fc[v][k];
                    }
                }
#pragma unroll
                for (int k = 0; k < NC; ++k) acc[si][k] += pre * tv[k];
            }
        }
    }
#pragma unroll
    for (int s = 0; s < NS0; ++s)
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const double v = tet::warp_sum(acc[s][k]);
            if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&sacc[s * 3 + k], v);
        }
    __syncthreads();
    for (int i = threadIdx.x; i < NS0 * NC; i += blockDim.x) {
        const int s = i / NC, k = i % NC;
        if (s >= a.s0n || sacc[s * 3 + k] == 0.0) continue;
        const int s0 = a.s0a + s;
        if (MODE == 0) atomicAdd(&a.out[(size_t)q0 * n + s0], sacc[s * 3]);
        else atomicAdd(&a.out[((size_t)q0 * n + s0) * 3 + k], sacc[s * 3 + k]);
    }
}

// F0 = FunitE w v / (1/tau T^2) where |1/tau| > zero_prec (CreateFzero).
__global__ void k_bte_f0(int ntr, int n, const int* tr_grid, const double* omega, const double* vel,
                         const double* inv_tau, double T, double* F0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntr * n; i += gridDim.x * blockDim.x) {
        const int q = i / n, s = i % n, g0 = tr_grid[q];
        const double it = inv_tau[i];
        for (int k = 0; k < 3; ++k) {
            double f = 0.0;
            if (!(g0 == 0 && s < 3) && fabs(it) > ZERO_PREC)
                f = FUNIT_E * omega[(size_t)g0 * n + s] * vel[((size_t)g0 * n + s) * 3 + k] / (it * (T * T));
            F0[(size_t)i * 3 + k] = f;
        }
    }
}

// multiplyTaudFnew then F = F0 + dF.
__global__ void k_bte_update(int ntr, int n, const int* tr_grid, const double* inv_tau, const double* F0,
                             double* dF, double* F) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntr * n; i += gridDim.x * blockDim.x) {
        const int q = i / n, s = i % n;
        const double it = inv_tau[i];
        const bool scale = !(tr_grid[q] == 0 && s < 3) && fabs(it) > ZERO_PREC;
        for (int k = 0; k < 3; ++k) {
            double d = dF[(size_t)i * 3 + k];
            if (scale) d /= it;
            F[(size_t)i * 3 + k] = F0[(size_t)i * 3 + k] + d;
        }
    }
}

// kappa = kW_mK / (Nq V) sum_{q, s} deg w n (n+1) v (x) F   (one CTA, tree reduction)
__global__ void __launch_bounds__(256) k_bte_kappa(int ntr, int n, int nq, double vol, const int* tr_grid,
                                                   const int* deg, const double* omega, const double* nbe,
                                                   const double* vel, const double* F, double* kappa) {
    __shared__ double red[256][9];
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < ntr * n; i += blockDim.x) {
        const int q = i / n, s = i % n, g0 = tr_grid[q];
        if (g0 == 0 && s < 3) continue;
        const double w = omega[(size_t)g0 * n + s], nb = nbe[(size_t)g0 * n + s];
        const double pre = double(deg[q]) * w * nb * (nb + 1.0);
        const double* v = vel + ((size_t)g0 * n + s) * 3;
        const double* f = F + (size_t)i * 3;
        for (int x = 0; x < 3; ++x)
            for (int y = 0; y < 3; ++y) acc[3 * x + y] += pre * (v[x] * f[y]);
    }
    for (int k = 0; k < 9; ++k) red[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int k = 0; k < 9; ++k) red[threadIdx.x][k] += red[threadIdx.x + h][k];
        __syncthreads();
    }
    if (threadIdx.x < 9) kappa[threadIdx.x] = KW_MK * (1.0 / (double(nq) * vol)) * red[0][threadIdx.x];
}

int grid_x(long long items, int threads, int slots) {
    long long want = (items + (long long)threads * 4 - 1) / ((long long)threads * 4);
    long long cap = (148LL * 16 + slots - 1) / slots;
    if (want > cap) want = cap;
    return (int)(want < 1 ? 1 : want);
}

// Time-reversal set on the host from the grid addresses.
int build_tr_set(spring_ctx* c) {
    const int nq = c->nq;
    std::vector<int> qint((size_t)nq * 3);
    SPRING_CHECK(d2h(c, qint.data(), c->d_qint.p, sizeof(int) * qint.size(), "grid addresses"));
    auto gidx = [&](int x, int y, int z) {
        auto m = [](int a, int n) { int r = a % n; return r < 0 ? r + n : r; };
        return m(x, c->mesh[0]) + c->mesh[0] * (m(y, c->mesh[1]) + c->mesh[1] * m(z, c->mesh[2]));
    };
    std::vector<int> neg(nq), rep(nq);
    for (int q = 0; q < nq; ++q) {
        neg[q] = gidx(-qint[3 * q], -qint[3 * q + 1], -qint[3 * q + 2]);
        rep[q] = std::min(q, neg[q]);
    }
    std::vector<int> grid;
    for (int q = 0; q < nq; ++q)
        if (rep[q] == q) grid.push_back(q);
    const int ntr = (int)grid.size();
    std::vector<int> slot(nq, -1), pos(nq), sgn(nq), deg(ntr, 0), tint((size_t)ntr * 3);
    for (int i = 0; i < ntr; ++i) {
        slot[grid[i]] = i;
        for (int d = 0; d < 3; ++d) tint[3 * i + d] = qint[3 * grid[i] + d];
    }
    for (int q = 0; q < nq; ++q) {
        pos[q] = slot[rep[q]];
        sgn[q] = q == rep[q] ? 1 : -1;
        deg[pos[q]] += 1;
    }
    SPRING_CHECK(dalloc(c, c->d_tr_int, tint.size(), "time-reversal set"));
    SPRING_CHECK(dalloc(c, c->d_tr_grid, ntr, "time-reversal set"));
    SPRING_CHECK(dalloc(c, c->d_tr_pos, nq, "time-reversal set"));
    SPRING_CHECK(dalloc(c, c->d_tr_sgn, nq, "time-reversal set"));
    SPRING_CHECK(dalloc(c, c->d_tr_deg, ntr, "time-reversal set"));
    SPRING_CHECK(dalloc(c, c->d_neg, nq, "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_tr_int.p, tint.data(), sizeof(int) * tint.size(), "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_tr_grid.p, grid.data(), sizeof(int) * ntr, "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_tr_pos.p, pos.data(), sizeof(int) * nq, "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_tr_sgn.p, sgn.data(), sizeof(int) * nq, "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_tr_deg.p, deg.data(), sizeof(int) * ntr, "time-reversal set"));
    SPRING_CHECK(h2d(c, c->d_neg.p, neg.data(), sizeof(int) * nq, "time-reversal set"));
    c->ntr = ntr;
    c->ps_tr.n0 = ntr;
    c->ps_tr.q0_int = c->d_tr_int.p;
    c->ps_tr.q0_grid = c->d_tr_grid.p;
    c->ps_tr.done = false;
    dfree(c->d_wtr);
    return SPRING_OK;
}

// ---------------------------------------------------------------- Gaussian operator
// The iterative BTE with Gaussian delta weights in place of the tetrahedra (build-side form): per
// enumerated pair (q0 of the time-reversal set, q1, q2 = p(q1)) and mode triple with a weight above
// the exp(-40) cut, one operator entry (r0, k1, k2, P, Q); with c = (n1 - n2) P + (1 + n1 + n2) Q,
//   1/tau(r0) = sum c,   dF(r0) = -sum c (F(k1) + F(k2)),
// which is the reference's two channels (TetrahedronWplus / Wminus and TetrahedronIterPlus / Minus,
// Quasi_momentum_consrv.f90:701-1208, TetrahedronDeltaSum.f90:22-607) summed over every grid q1 with
// d(w0 - M): the plus channel at q1 and at q2 gives (n1 - n2) d(w0 + w1 - w2) + (n2 - n1) d(w0 + w2 - w1)
// and the minus channel at -q1 and -q2 gives (1 + n1 + n2) d(w0 - w1 - w2), each times 4 W3 and -(F1 + F2)
// because F(-q) = -F(q).  The entries are sorted by row once and kept in HBM (CSR); an iteration is one
// pass over them.
__global__ void k_bteg_keys(long long n, const s3::BteEntry* __restrict__ e, int* __restrict__ key,
                            int* __restrict__ idx, int* __restrict__ rowcnt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        key[i] = e[i].r0;
        idx[i] = (int)i;
        atomicAdd(&rowcnt[e[i].r0], 1);
    }
}
__global__ void k_bteg_gather(long long n, const s3::BteEntry* __restrict__ e, const int* __restrict__ idx,
                              int2* __restrict__ kk, double2* __restrict__ pq) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const s3::BteEntry x = e[idx[i]];
        kk[i] = make_int2(x.k1, x.k2);
        pq[i] = make_double2(x.P, x.Q);
    }
}
// c = (n1 - n2) P + (1 + n1 + n2) Q at one temperature
__global__ void k_bteg_coef(long long n, const int2* __restrict__ kk, const double2* __restrict__ pq,
                            const double* __restrict__ nbe, double* __restrict__ cf) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int2 k = kk[i];
        const double2 v = pq[i];
        const double n1 = nbe[k.x], n2 = nbe[k.y];
        cf[i] = (n1 - n2) * v.x + (1.0 + n1 + n2) * v.y;
    }
}
// F at every grid mode from the time-reversal slots: Fg[g][s] = sgn(g) F[pos(g)][s], padded to four
// doubles (32 bytes, one L2 sector) per mode for the row pass's gathers.
__global__ void k_bteg_expand(int nq, int n, const int* __restrict__ pos, const int* __restrict__ sgn,
                              const double* __restrict__ F, double* __restrict__ Fg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq * n; i += gridDim.x * blockDim.x) {
        const int g = i / n, sx = i % n;
        const double sg = sgn[g];
        const double* f = F + ((size_t)pos[g] * n + sx) * 3;
        double2* o = reinterpret_cast<double2*>(Fg + 4 * (size_t)i);
        o[0] = make_double2(sg * f[0], sg * f[1]);
        o[1] = make_double2(sg * f[2], 0.0);
    }
}
// One warp per row: MODE 0 inv_tau[r] = sum c; MODE 1 dF[r] = -sum c (Fg[k1] + Fg[k2]) (Fg: four
// doubles per mode, the fourth zero).
template <int MODE>
__global__ void __launch_bounds__(256) k_bteg_rows(int rows, const int* __restrict__ rowoff, const int2* __restrict__ kk,
                                                  const double* __restrict__ cf, const double* __restrict__ Fg,
                                                  double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += (gridDim.x * blockDim.x) >> 5) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int i = rowoff[r] + lane; i < rowoff[r + 1]; i += 32) {
            const double c = cf[i];
            if (MODE == 0) {
                a0 += c;
            } else {
                const int2 k = kk[i];
                const double2* f1 = reinterpret_cast<const double2*>(Fg + 4 * (size_t)k.x);
                const double2* f2 = reinterpret_cast<const double2*>(Fg + 4 * (size_t)k.y);
                const double2 u1 = f1[0], v1 = f1[1], u2 = f2[0], v2 = f2[1];
                a0 -= c * (u1.x + u2.x);
                a1 -= c * (u1.y + u2.y);
                a2 -= c * (v1.x + v2.x);
            }
        }
        a0 = tet::warp_sum(a0);
        if (MODE == 1) {
            a1 = tet::warp_sum(a1);
            a2 = tet::warp_sum(a2);
        }
        if (lane == 0) {
            if (MODE == 0) {
                out[r] = a0;
            } else {
                out[3 * (size_t)r] = a0;
                out[3 * (size_t)r + 1] = a1;
                out[3 * (size_t)r + 2] = a2;
            }
        }
    }
}

}  // namespace

int run_bte_gauss(spring_ctx* c, double sigma, double eps_k, int max_iter, double* h_kappa, double* h_kappa_rta,
                  int* h_iters, double* h_stats) {
    if (c->nb != 2 || c->na3 != 7) return fail(c, SPRING_ERR_UNSUPPORTED, "Gaussian iterative kappa: two-atom cells with 7-atom FC3 clusters");
    if (c->ntr == 0) SPRING_CHECK(build_tr_set(c));
    if (!c->ps_tr.done) SPRING_CHECK(run_enumerate3(c, c->ps_tr));
    SPRING_CHECK(pairoff_host(c, c->ps_tr));
    const int n = c->ndof, ntr = c->ntr, nq = c->nq, rows = ntr * n;
    const Q0View view{c->d_tr_int.p, c->d_tr_grid.p, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p};
    const long long npairs = c->ps_tr.h_pairoff[ntr];
    const int threads = 256;
    auto blocks_for = [&](long long m) { return (int)std::max<long long>(1, std::min<long long>((m + threads - 1) / threads, 148LL * 16)); };
    // ---- the operator: entries, sorted by row (kept until sigma, the phonons or the pairs change)
    if (!(c->bteg_sigma == sigma && c->bteg_gen == c->ph_gen && c->bteg_pairs == c->ps_tr.gen && c->bteg_n > 0 &&
          c->bteg_prec == c->precision)) {
        c->bteg_n = 0;
        DBuf<s3::BteEntry> ent;
        DBuf<unsigned long long> ctr;
        SPRING_CHECK(dalloc(c, ctr, 1, "operator count"));
        long long cap = std::max<long long>(1 << 20, npairs * 216 / 40);  // the window passes ~1-2% of the triples
        long long cnt = 0;
        for (int attempt = 0; attempt < 2; ++attempt) {
            int rc = dalloc(c, ent, (size_t)cap, "BTE operator entries");
            if (rc == SPRING_OK) rc = zero(c, ctr.p, sizeof(unsigned long long), "operator count");
            bool handled = false;
            // BF16 / BF16x3 contexts: the tensor-core pass writes the entries; FP64: the FP64 pass
            if (rc == SPRING_OK) rc = run_v3tc_bte(c, 0, ntr, sigma, ent.p, ctr.p, cap, &handled);
            if (rc == SPRING_OK && !handled)
                rc = launch_v3s_bte(c, c->ps_tr, view, 0, ntr, sigma, ent.p, ctr.p, cap, &handled);
            unsigned long long h = 0;
            if (rc == SPRING_OK) rc = d2h(c, &h, ctr.p, sizeof h, "operator count");
            if (rc != SPRING_OK) { dfree(ent); dfree(ctr); return rc; }
            cnt = (long long)h;
            if (cnt <= cap) break;
            dfree(ent);
            cap = cnt + cnt / 16 + 1024;
        }
        dfree(ctr);
        if (cnt > cap) { dfree(ent); return fail(c, SPRING_ERR_CUDA, "BTE operator: entry count changed between runs"); }
        if (cnt > 0x7fffffffLL) { dfree(ent); return fail(c, SPRING_ERR_UNSUPPORTED, "BTE operator above 2^31 entries"); }
        DBuf<int> key, keys, idx, idxs, cntr;
        int rc = dalloc(c, key, std::max<long long>(cnt, 1), "operator keys");
        if (rc == SPRING_OK) rc = dalloc(c, keys, std::max<long long>(cnt, 1), "operator keys");
        if (rc == SPRING_OK) rc = dalloc(c, idx, std::max<long long>(cnt, 1), "operator keys");
        if (rc == SPRING_OK) rc = dalloc(c, idxs, std::max<long long>(cnt, 1), "operator keys");
        if (rc == SPRING_OK) rc = dalloc(c, cntr, rows + 1, "operator rows");
        if (rc == SPRING_OK) rc = dalloc(c, c->d_bteg_row, rows + 1, "operator rows");
        if (rc == SPRING_OK) rc = zero(c, cntr.p, sizeof(int) * (rows + 1), "operator rows");
        if (rc == SPRING_OK && cnt > 0) {
            k_bteg_keys<<<blocks_for(cnt), threads, 0, c->stream>>>(cnt, ent.p, key.p, idx.p, cntr.p);
            rc = launch_check(c, "k_bteg_keys");
        }
        if (rc == SPRING_OK) rc = run_exclusive_scan(c, cntr.p, c->d_bteg_row.p, rows + 1);
        if (rc == SPRING_OK && cnt > 0) {
            int bits = 1;
            while ((1 << bits) <= rows) ++bits;
            size_t tb = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, keys.p, idx.p, idxs.p, (int)cnt, 0, bits, c->stream);
            DBuf<uint8_t> tmp;
            rc = dalloc(c, tmp, std::max<size_t>(tb, 1), "operator sort");
            if (rc == SPRING_OK) {
                const cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, keys.p, idx.p, idxs.p, (int)cnt,
                                                                      0, bits, c->stream);
                c->launches += 1;
                if (e != cudaSuccess) rc = cuda_fail(c, e, "operator sort");
            }
            if (rc == SPRING_OK) rc = dalloc(c, c->d_bteg_kk, cnt, "BTE operator");
            if (rc == SPRING_OK) rc = dalloc(c, c->d_bteg_pq, cnt, "BTE operator");
            if (rc == SPRING_OK) {
                k_bteg_gather<<<blocks_for(cnt), threads, 0, c->stream>>>(cnt, ent.p, idxs.p, c->d_bteg_kk.p, c->d_bteg_pq.p);
                rc = launch_check(c, "k_bteg_gather");
            }
            cudaStreamSynchronize(c->stream);
            dfree(tmp);
        }
        cudaStreamSynchronize(c->stream);
        dfree(ent); dfree(key); dfree(keys); dfree(idx); dfree(idxs); dfree(cntr);
        if (rc != SPRING_OK) return rc;
        c->bteg_n = cnt;
        c->bteg_sigma = sigma;
        c->bteg_gen = c->ph_gen;
        c->bteg_pairs = c->ps_tr.gen;
        c->bteg_prec = c->precision;
    }
    const long long cnt = c->bteg_n;
    if (h_stats) {
        h_stats[0] = (double)cnt;
        h_stats[1] = (double)npairs;
    }
    // ---- iterations per temperature
    DBuf<double> inv_tau, F0, F, dF, kap, cf, Fg;
    int rc = dalloc(c, inv_tau, (size_t)rows, "1/tau");
    if (rc == SPRING_OK) rc = dalloc(c, F0, (size_t)rows * 3, "F0");
    if (rc == SPRING_OK) rc = dalloc(c, F, (size_t)rows * 3, "F");
    if (rc == SPRING_OK) rc = dalloc(c, dF, (size_t)rows * 3, "dF");
    if (rc == SPRING_OK) rc = dalloc(c, kap, 9, "kappa");
    if (rc == SPRING_OK) rc = dalloc(c, cf, std::max<long long>(cnt, 1), "operator coefficients");
    if (rc == SPRING_OK) rc = dalloc(c, Fg, (size_t)nq * n * 4, "F on the grid");
    const int rblocks = std::max(1, std::min((rows + 7) / 8, 148 * 16));
    const int eblocks = std::max(1, std::min((rows + threads - 1) / threads, 148 * 8));
    auto kappa_of = [&](int T, const double* Fv, double* out9) -> int {
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure");
        k_bte_kappa<<<1, 256, 0, c->stream>>>(ntr, n, nq, c->vol, c->d_tr_grid.p, c->d_tr_deg.p, c->ph_grid.omega.p,
                                              c->ph_grid.nbe.p + (size_t)T * nq * n, c->ph_grid.vel.p, Fv, kap.p);
        SPRING_CHECK(launch_check(c, "k_bte_kappa"));
        return d2h(c, out9, kap.p, sizeof(double) * 9, "kappa");
    };
    for (int T = 0; rc == SPRING_OK && T < c->nT; ++T) {
        const double* nbeT = c->ph_grid.nbe.p + (size_t)T * nq * n;
        if (cnt > 0) {
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
            k_bteg_coef<<<blocks_for(cnt), threads, 0, c->stream>>>(cnt, c->d_bteg_kk.p, c->d_bteg_pq.p, nbeT, cf.p);
            if ((rc = launch_check(c, "k_bteg_coef")) != SPRING_OK) break;
        }
        if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
        k_bteg_rows<0><<<rblocks, 256, 0, c->stream>>>(rows, c->d_bteg_row.p, c->d_bteg_kk.p, cf.p, nullptr, inv_tau.p);
        if ((rc = launch_check(c, "k_bteg_rows<tau>")) != SPRING_OK) break;
        if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
        k_bte_f0<<<eblocks, threads, 0, c->stream>>>(ntr, n, c->d_tr_grid.p, c->ph_grid.omega.p, c->ph_grid.vel.p,
                                                    inv_tau.p, c->temps[T], F0.p);
        if ((rc = launch_check(c, "k_bte_f0")) != SPRING_OK) break;
        if (cudaMemcpyAsync(F.p, F0.p, sizeof(double) * rows * 3, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
            rc = fail(c, SPRING_ERR_CUDA, "F copy");
            break;
        }
        double k0[9], kold[9], knew[9];
        if ((rc = kappa_of(T, F.p, k0)) != SPRING_OK) break;
        std::copy(k0, k0 + 9, kold);
        std::copy(k0, k0 + 9, knew);
        int iter = 0;
        for (;;) {
            ++iter;
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
            k_bteg_expand<<<blocks_for((long long)nq * n), threads, 0, c->stream>>>(nq, n, c->d_tr_pos.p, c->d_tr_sgn.p,
                                                                                     F.p, Fg.p);
            if ((rc = launch_check(c, "k_bteg_expand")) != SPRING_OK) break;
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
            k_bteg_rows<1><<<rblocks, 256, 0, c->stream>>>(rows, c->d_bteg_row.p, c->d_bteg_kk.p, cf.p, Fg.p, dF.p);
            if ((rc = launch_check(c, "k_bteg_rows<dF>")) != SPRING_OK) break;
            if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure"); break; }
            k_bte_update<<<eblocks, threads, 0, c->stream>>>(ntr, n, c->d_tr_grid.p, inv_tau.p, F0.p, dF.p, F.p);
            if ((rc = launch_check(c, "k_bte_update")) != SPRING_OK) break;
            if ((rc = kappa_of(T, F.p, knew)) != SPRING_OK) break;
            double d = 0.0;
            for (int k = 0; k < 9; ++k) d = std::max(d, std::fabs(knew[k] - kold[k]));
            if (d < eps_k || iter > max_iter) break;
            std::copy(knew, knew + 9, kold);
        }
        if (rc != SPRING_OK) break;
        if (h_kappa) std::copy(knew, knew + 9, h_kappa + 9 * T);
        if (h_kappa_rta) std::copy(k0, k0 + 9, h_kappa_rta + 9 * T);
        if (h_iters) h_iters[T] = iter;
    }
    dfree(inv_tau); dfree(F0); dfree(F); dfree(dF); dfree(kap); dfree(cf); dfree(Fg);
    return rc;
}

int run_bte(spring_ctx* c, double eps_k, int max_iter, double* h_kappa, double* h_kappa_rta, int* h_iters) {
    if (c->ntr == 0) SPRING_CHECK(build_tr_set(c));
    if (!c->ps_tr.done) SPRING_CHECK(run_enumerate3(c, c->ps_tr));
    const int n = c->ndof, ntr = c->ntr, nq = c->nq;
    const size_t slot = (size_t)nq * n * n * n;
    const Q0View view{c->d_tr_int.p, c->d_tr_grid.p, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p};
    // W grids: all of them resident when they fit the budget, else batches recomputed per pass
    const size_t budget = (size_t)40 << 30;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const bool cache_all = slot * ntr * sizeof(double) <= std::min(budget, free_b / 2);
    int batch = ntr;
    if (cache_all) {
        if (!c->d_wtr.p || c->d_wtr.n < slot * ntr) {
            SPRING_CHECK(dalloc(c, c->d_wtr, slot * ntr, "time-reversal W grids"));
            SPRING_CHECK(run_v3_wgrid(c, c->ps_tr, view, 0, ntr, c->d_wtr.p));
        }
    } else {
        batch = (int)std::max<size_t>(1, ((size_t)96 << 20) / (slot * sizeof(double)));
        batch = std::min(batch, ntr);
        SPRING_CHECK(dalloc(c, c->d_w, slot * batch, "W buffer"));
    }
    DBuf<double> inv_tau, F0, F, dF, kap;
    int rc = dalloc(c, inv_tau, (size_t)ntr * n, "1/tau");
    if (rc == SPRING_OK) rc = dalloc(c, F0, (size_t)ntr * n * 3, "F0");
    if (rc == SPRING_OK) rc = dalloc(c, F, (size_t)ntr * n * 3, "F");
    if (rc == SPRING_OK) rc = dalloc(c, dF, (size_t)ntr * n * 3, "dF");
    if (rc == SPRING_OK) rc = dalloc(c, kap, 9, "kappa");

    auto pass = [&](int mode, int T) -> int {
        PassArgs pa;
        pa.n = n;
        pa.nq = nq;
        pa.ntet = 6 * nq;
        pa.tr_grid = c->d_tr_grid.p;
        pa.tr_pos = c->d_tr_pos.p;
        pa.tr_sgn = c->d_tr_sgn.p;
        pa.neg = c->d_neg.p;
        pa.partner = c->ps_tr.partner.p;
        pa.omega = c->ph_grid.omega.p;
        pa.nbe = c->ph_grid.nbe.p + (size_t)T * nq * n;
        pa.F = F.p;
        pa.out = mode == 0 ? inv_tau.p : dF.p;
        const long long items = (long long)pa.ntet * n * n;
        for (int b = 0; b < ntr; b += batch) {
            const int nb = std::min(batch, ntr - b);
            if (!cache_all) SPRING_CHECK(run_v3_wgrid(c, c->ps_tr, view, b, nb, c->d_w.p));
            pa.q0_first = b;
            pa.wgrid = cache_all ? c->d_wtr.p + slot * b : c->d_w.p;
            dim3 grid(grid_x(items, 128, nb), nb);
            for (int s0a = 0; s0a < n; s0a += NS0) {
                pa.s0a = s0a;
                pa.s0n = std::min(NS0, n - s0a);
                if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure");
                if (mode == 0) k_bte_pass<0><<<grid, 128, 0, c->stream>>>(pa, reinterpret_cast<const int4*>(c->d_tetra.p));
                else k_bte_pass<1><<<grid, 128, 0, c->stream>>>(pa, reinterpret_cast<const int4*>(c->d_tetra.p));
                SPRING_CHECK(launch_check(c, mode == 0 ? "k_bte_pass<tau>" : "k_bte_pass<dF>"));
            }
        }
        return SPRING_OK;
    };
    auto kappa_of = [&](int T, const double* Fv, double* out9) -> int {
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "bte: injected launch failure");
        k_bte_kappa<<<1, 256, 0, c->stream>>>(ntr, n, nq, c->vol, c->d_tr_grid.p, c->d_tr_deg.p, c->ph_grid.omega.p,
                                              c->ph_grid.nbe.p + (size_t)T * nq * n, c->ph_grid.vel.p, Fv, kap.p);
        SPRING_CHECK(launch_check(c, "k_bte_kappa"));
        return d2h(c, out9, kap.p, sizeof(double) * 9, "kappa");
    };
    const int threads = 256, blocks = std::max(1, std::min((ntr * n + threads - 1) / threads, 148 * 8));
    for (int T = 0; rc == SPRING_OK && T < c->nT; ++T) {
        rc = zero(c, inv_tau.p, sizeof(double) * ntr * n, "1/tau");
        if (rc == SPRING_OK) rc = pass(0, T);
        if (rc == SPRING_OK && !launch_injected(c)) {
            k_bte_f0<<<blocks, threads, 0, c->stream>>>(ntr, n, c->d_tr_grid.p, c->ph_grid.omega.p, c->ph_grid.vel.p,
                                                        inv_tau.p, c->temps[T], F0.p);
            rc = launch_check(c, "k_bte_f0");
        }
        if (rc == SPRING_OK)
            rc = cudaMemcpyAsync(F.p, F0.p, sizeof(double) * ntr * n * 3, cudaMemcpyDeviceToDevice, c->stream) ==
                         cudaSuccess ? SPRING_OK : fail(c, SPRING_ERR_CUDA, "F copy");
        double k0[9], kold[9], knew[9];
        if (rc == SPRING_OK) rc = kappa_of(T, F.p, k0);
        if (rc != SPRING_OK) break;
        std::copy(k0, k0 + 9, kold);
        std::copy(k0, k0 + 9, knew);
        int iter = 0;
        for (;;) {
            ++iter;
            rc = zero(c, dF.p, sizeof(double) * ntr * n * 3, "dF");
            if (rc == SPRING_OK) rc = pass(1, T);
            if (rc == SPRING_OK && !launch_injected(c)) {
                k_bte_update<<<blocks, threads, 0, c->stream>>>(ntr, n, c->d_tr_grid.p, inv_tau.p, F0.p, dF.p, F.p);
                rc = launch_check(c, "k_bte_update");
            }
            if (rc == SPRING_OK) rc = kappa_of(T, F.p, knew);
            if (rc != SPRING_OK) break;
            double d = 0.0;
            for (int k = 0; k < 9; ++k) d = std::max(d, std::fabs(knew[k] - kold[k]));
            if (d < eps_k || iter > max_iter) break;
            std::copy(knew, knew + 9, kold);
        }
        if (rc != SPRING_OK) break;
        if (h_kappa) std::copy(knew, knew + 9, h_kappa + 9 * T);
        if (h_kappa_rta) std::copy(k0, k0 + 9, h_kappa_rta + 9 * T);
        if (h_iters) h_iters[T] = iter;
    }
    dfree(inv_tau); dfree(F0); dfree(F); dfree(dF); dfree(kap);
    return rc;
}

}  // namespace spring
