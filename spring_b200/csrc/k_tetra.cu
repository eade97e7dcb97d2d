// Linear-tetrahedron delta sums on the device.
//
// 3-phonon: CalculateLwTetrahedron (src/Kappa/Src/ThirdOrder_m.f90:169-275)
// with FindFandOmegaAtVertices / FindgAndIver / my_sort / FindIverxFver
// (src/Kappa/Src/TetrahedronIntegration_m.f90:18-295).
// Isotope: CalculateIsoW + CalculateIsoLwTetra (src/Kappa/Src/IsotopicScatter.f90:36-168),
// and a Gaussian form delta(omega0 - omega1).
//
// One thread per (q0, tetrahedron, s1, s2).  The vertex energies of the three
// channels (w1+w2, w2-w1, w1-w2) do not depend on s0, so each channel is sorted
// once per thread (stable: ties keep the original vertex order, which is what
// my_sort's first-uncovered search produces) and reused for every s0 and
// temperature.  Case bounds, formulas and the order of the vertex sum follow
// the reference; only the summation order over tetrahedra differs (partial
// sums per thread, then warp/CTA reduction).
// Roofline: FP64 ALU (about 60 flops and 10 divisions per tetrahedron, mode
// triple and channel); W is read from the L2-resident W grid.
#include "spring_internal.cuh"
#include "tetra.cuh"

namespace spring {
namespace {

constexpr int NS0 = 6;  // s0 values per pass (register accumulators)

struct TetArgs {
    int n, nq, nq0, nT, ntet;
    long long ntab;  // rows of the q2 table (path mode)
    int q0_first;
    int s0a, s0n;  // s0 pass: [s0a, s0a + s0n)
    int lo1, n1, lo2, n2;
};

// Q2TAB = false: kappa.x, the q2 of vertex q1 is the grid partner p(q1) of this q0.
// Q2TAB = true: LineWidth.x path mode, the q2 phonons of vertex q1 come from a
// per-q1 table (omega_q2All / nBE_q2All of Linewidth_m.f90:48-231), [slot][q1][s]
// and [T][row][s] with row = slot * Nq + q1 of a table of `ntab` rows.
template <int NTM, bool STRICT, bool Q2TAB>
__global__ void __launch_bounds__(128) k_tetra3(TetArgs a, const int4* __restrict__ tet, const int* __restrict__ partner,
                                                const double* __restrict__ wgrid, const double* __restrict__ om0,
                                                const double* __restrict__ omg, const double* __restrict__ nbeg,
                                                const double* __restrict__ om2t, const double* __restrict__ nbe2t,
                                                double* __restrict__ out_lw, double* __restrict__ out_p3) {
    __shared__ double sacc[NS0 * (NTM + 1)];
    const int slot = blockIdx.y;
    const int q0 = a.q0_first + slot;
    const int n = a.n;
    const size_t n3 = (size_t)n * n * n;
    const int* part = Q2TAB ? nullptr : partner + (size_t)q0 * a.nq;
    const size_t row0 = (size_t)slot * a.nq;  // first row of this slot in the q2 table
    const double* W = wgrid + (size_t)slot * a.nq * n3;
    for (int i = threadIdx.x; i < NS0 * (NTM + 1); i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();

    double acc[NS0][NTM + 1];
#pragma unroll
    for (int s = 0; s < NS0; ++s)
#pragma unroll
        for (int t = 0; t <= NTM; ++t) acc[s][t] = 0.0;

    const long long items = (long long)a.ntet * a.n1 * a.n2;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int s2 = a.lo2 + (int)(it % a.n2);
        const int s1 = a.lo1 + (int)((it / a.n2) % a.n1);
        const int t = (int)(it / ((long long)a.n1 * a.n2));
        const int4 tv = tet[t];
        const int v1[4] = {tv.x, tv.y, tv.z, tv.w};
        int v2[4];
        double o1[4], o2[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            v2[v] = Q2TAB ? v1[v] : part[v1[v]];
            o1[v] = omg[(size_t)v1[v] * n + s1];
            o2[v] = Q2TAB ? om2t[(row0 + v1[v]) * n + s2] : omg[(size_t)v2[v] * n + s2];
        }
        double M1[4], M2[4], M3[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            M1[v] = o1[v] + o2[v];
            M2[v] = o2[v] - o1[v];
            M3[v] = o1[v] - o2[v];
        }
        int p1[4], p2[4], p3[4];
        tet::sort4(M1, p1);
        tet::sort4(M2, p2);
        tet::sort4(M3, p3);
        double S1[4], S2[4], S3[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            S1[v] = M1[p1[v]];
            S2[v] = M2[p2[v]];
            S3[v] = M3[p3[v]];
        }
        // occupation factors per vertex and temperature
        double fa[NTM][4], fb[NTM][4];  // n1+n2+1 and n1-n2
#pragma unroll
        for (int T = 0; T < NTM; ++T)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (T < a.nT) {
                    const double n1 = nbeg[((size_t)T * a.nq + v1[v]) * n + s1];
                    const double n2 = Q2TAB ? nbe2t[((size_t)T * a.ntab + row0 + v1[v]) * n + s2]
                                            : nbeg[((size_t)T * a.nq + v2[v]) * n + s2];
                    fa[T][v] = n1 + n2 + 1.0;
                    fb[T][v] = n1 - n2;
                } else {
                    fa[T][v] = fb[T][v] = 0.0;
                }
            }
#pragma unroll
        for (int si = 0; si < NS0; ++si) {
            if (si >= a.s0n) break;
            const int s0 = a.s0a + si;
            const double Mqs = om0[(size_t)q0 * n + s0];
            double Wv[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) Wv[v] = W[(size_t)v1[v] * n3 + (s0 * n + s1) * n + s2];
            double g, I[4];
            // channel 1: F = W (n1 + n2 + 1), M = w1 + w2, added
            bool e = tet::g_iver<STRICT>(Mqs, S1, g, I);
            acc[si][NTM] += g;
            if (e) {
#pragma unroll
                for (int T = 0; T < NTM; ++T) {
                    double s = 0.0;
#pragma unroll
                    for (int v = 0; v < 4; ++v) s += I[v] * (Wv[p1[v]] * fa[T][p1[v]]);
                    acc[si][T] += g * (ONEBYSIX * s);
                }
            }
            // channel 2: F = W (n1 - n2), M = w2 - w1, added
            e = tet::g_iver<STRICT>(Mqs, S2, g, I);
            acc[si][NTM] += g;
            if (e) {
#pragma unroll
                for (int T = 0; T < NTM; ++T) {
                    double s = 0.0;
#pragma unroll
                    for (int v = 0; v < 4; ++v) s += I[v] * (Wv[p2[v]] * fb[T][p2[v]]);
                    acc[si][T] += g * (ONEBYSIX * s);
                }
            }
            // channel 3: F = W (n1 - n2), M = w1 - w2, subtracted
            e = tet::g_iver<STRICT>(Mqs, S3, g, I);
            acc[si][NTM] += g;
            if (e) {
#pragma unroll
                for (int T = 0; T < NTM; ++T) {
                    double s = 0.0;
#pragma unroll
                    for (int v = 0; v < 4; ++v) s += I[v] * (Wv[p3[v]] * fb[T][p3[v]]);
                    acc[si][T] -= g * (ONEBYSIX * s);
                }
            }
        }
    }
    // reduce: warp, then CTA (shared), then global
#pragma unroll
    for (int s = 0; s < NS0; ++s)
#pragma unroll
        for (int T = 0; T <= NTM; ++T) {
            const double v = tet::warp_sum(acc[s][T]);
            if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&sacc[s * (NTM + 1) + T], v);
        }
    __syncthreads();
    for (int i = threadIdx.x; i < NS0 * (NTM + 1); i += blockDim.x) {
        const int s = i / (NTM + 1), T = i % (NTM + 1);
        if (s >= a.s0n) continue;
        const int s0 = a.s0a + s;
        if (T < NTM) {
            if (T < a.nT) atomicAdd(&out_lw[((size_t)T * a.nq0 + q0) * n + s0], sacc[i]);
        } else {
            atomicAdd(&out_p3[(size_t)q0 * n + s0], sacc[i]);
        }
    }
}

// ---- isotope ------------------------------------------------------------
// W_iso(s1,s0,q1) = pi w0(s0)^2 / 2 / Nq * sum_b g2(b) |e1(b,s1)^H e0(b,s0)|^2  -> [slot][q1][s0][s1]
__global__ void k_iso_w(int n, int nb, int nq, int q0_first, int nslot, double scale, const double* __restrict__ g2,
                        const double2* __restrict__ ev0, const double* __restrict__ om0, const double2* __restrict__ evg,
                        double* __restrict__ wiso) {
    const long long total = (long long)nslot * nq * n * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int s1 = (int)(i % n), s0 = (int)((i / n) % n);
        const int q1 = (int)((i / ((long long)n * n)) % nq);
        const int slot = (int)(i / ((long long)n * n * nq));
        const int q0 = q0_first + slot;
        const double2* a0 = ev0 + ((size_t)q0 * n + s0) * n;
        const double2* a1 = evg + ((size_t)q1 * n + s1) * n;
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) {
            double dr = 0.0, di = 0.0;
            for (int c = 0; c < 3; ++c) {  // conj(e1) * e0
                const double2 x = a1[3 * b + c], y = a0[3 * b + c];
                dr += x.x * y.x + x.y * y.y;
                di += x.x * y.y - x.y * y.x;
            }
            acc += g2[b] * (dr * dr + di * di);
        }
        const double M = om0[(size_t)q0 * n + s0];
        wiso[i] = acc * scale * (M * M) * 0.5 / double(nq);
    }
}

__global__ void __launch_bounds__(128) k_iso_tetra(int n, int nq, int nq0, int ntet, int q0_first, int nT,
                                                   const int4* __restrict__ tet, const double* __restrict__ wiso,
                                                   const double* __restrict__ om0, const double* __restrict__ omg,
                                                   double* __restrict__ out) {
    __shared__ double sacc[MAX_NDOF];
    const int slot = blockIdx.y, q0 = q0_first + slot;
    for (int i = threadIdx.x; i < MAX_NDOF; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    const double* Wi = wiso + (size_t)slot * nq * n * n;
    const long long items = (long long)ntet * n;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int s1 = (int)(it % n), t = (int)(it / n);
        const int4 tv = tet[t];
        const int v1[4] = {tv.x, tv.y, tv.z, tv.w};
        double M[4];
        for (int v = 0; v < 4; ++v) M[v] = omg[(size_t)v1[v] * n + s1];
        int p[4];
        tet::sort4(M, p);
        double S[4];
        for (int v = 0; v < 4; ++v) S[v] = M[p[v]];
        for (int s0 = 0; s0 < n; ++s0) {
            double g, I[4];
            const bool e = tet::g_iver<false>(om0[(size_t)q0 * n + s0], S, g, I);
            for (int v = 0; v < 4; ++v) if (isnan(I[v])) I[v] = 0.0;
            if (isnan(g)) g = 0.0;
            double s = 0.0;
            if (e)
                for (int v = 0; v < 4; ++v) s += I[v] * Wi[((size_t)v1[p[v]] * n + s0) * n + s1];
            const double c = g * (ONEBYSIX * s);
            if (c != 0.0) atomicAdd(&sacc[s0], c);
        }
    }
    __syncthreads();
    for (int s0 = threadIdx.x; s0 < n; s0 += blockDim.x)
        for (int T = 0; T < nT; ++T) atomicAdd(&out[((size_t)T * nq0 + q0) * n + s0], sacc[s0]);
}

__global__ void __launch_bounds__(128) k_iso_gauss(int n, int nq, int nq0, int q0_first, int nT, double os, double os2,
                                                   const double* __restrict__ wiso, const double* __restrict__ om0,
                                                   const double* __restrict__ omg, double* __restrict__ out) {
    __shared__ double sacc[MAX_NDOF];
    const int slot = blockIdx.y, q0 = q0_first + slot;
    for (int i = threadIdx.x; i < MAX_NDOF; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    const double* Wi = wiso + (size_t)slot * nq * n * n;
    const long long items = (long long)nq * n;
    for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        const int s1 = (int)(it % n), q1 = (int)(it / n);
        const double w1 = omg[(size_t)q1 * n + s1];
        for (int s0 = 0; s0 < n; ++s0) {
            const double d = om0[(size_t)q0 * n + s0] - w1;
            const double c = Wi[((size_t)q1 * n + s0) * n + s1] * os * ONEBYSQRT2PI * exp(-0.5 * os2 * d * d);
            if (c != 0.0) atomicAdd(&sacc[s0], c);
        }
    }
    __syncthreads();
    for (int s0 = threadIdx.x; s0 < n; s0 += blockDim.x)
        for (int T = 0; T < nT; ++T) atomicAdd(&out[((size_t)T * nq0 + q0) * n + s0], sacc[s0]);
}

int grid_x(long long items, int threads, int slots) {
    long long want = (items + (long long)threads * 4 - 1) / ((long long)threads * 4);
    long long cap = (148LL * 16 + slots - 1) / slots;
    if (want > cap) want = cap;
    return (int)(want < 1 ? 1 : want);
}

template <bool STRICT, bool Q2TAB>
int launch_tetra3(spring_ctx* c, TetArgs a, int n_q0, const Pol& pol, const double* d_w, const int* part,
                  const double* om0, const double* omg, const double* nbeg, const double* om2t, const double* nbe2t,
                  double* d_lw, double* d_p3) {
    a.lo1 = pol.lo[1];
    a.n1 = pol.hi[1] - pol.lo[1] + 1;
    a.lo2 = pol.lo[2];
    a.n2 = pol.hi[2] - pol.lo[2] + 1;
    const long long items = (long long)a.ntet * a.n1 * a.n2;
    const int threads = 128;
    dim3 grid(grid_x(items, threads, n_q0), n_q0);
    const int4* tet = reinterpret_cast<const int4*>(c->d_tetra.p);
    for (int s0a = pol.lo[0]; s0a <= pol.hi[0]; s0a += NS0) {
        a.s0a = s0a;
        a.s0n = std::min(NS0, pol.hi[0] - s0a + 1);
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "tetra3: injected launch failure");
        if (c->nT == 1) {
            k_tetra3<1, STRICT, Q2TAB><<<grid, threads, 0, c->stream>>>(a, tet, part, d_w, om0, omg, nbeg, om2t, nbe2t,
                                                                        d_lw, d_p3);
        } else if (c->nT <= 3) {
            k_tetra3<3, STRICT, Q2TAB><<<grid, threads, 0, c->stream>>>(a, tet, part, d_w, om0, omg, nbeg, om2t, nbe2t,
                                                                        d_lw, d_p3);
        } else if (c->nT <= 9) {
            k_tetra3<9, STRICT, Q2TAB><<<grid, threads, 0, c->stream>>>(a, tet, part, d_w, om0, omg, nbeg, om2t, nbe2t,
                                                                        d_lw, d_p3);
        } else {
            return fail(c, SPRING_ERR_UNSUPPORTED, "tetrahedron integration supports at most 9 temperatures per call");
        }
        SPRING_CHECK(launch_check(c, Q2TAB ? "k_tetra3<path>" : "k_tetra3"));
    }
    return SPRING_OK;
}

}  // namespace

int run_tetra3(spring_ctx* c, int q0_first, int n_q0, const double* d_w, const Pol& pol, double* d_lw, double* d_p3) {
    TetArgs a{};
    a.n = c->ndof;
    a.nq = c->nq;
    a.nq0 = c->nq0;
    a.nT = c->nT;
    a.ntet = 6 * c->nq;
    a.q0_first = q0_first;
    return launch_tetra3<false, false>(c, a, n_q0, pol, d_w, c->ps_irr.partner.p, c->ph_irr.omega.p,
                                       c->ph_grid.omega.p, c->ph_grid.nbe.p, nullptr, nullptr, d_lw, d_p3);
}

int run_tetra3_path(spring_ctx* c, int p_first, int n_slots, int n_path, const double* d_w, const double* om0,
                    const double* om2t, const double* nbe2t, long long ntab, double* d_lw, double* d_scratch) {
    TetArgs a{};
    a.n = c->ndof;
    a.nq = c->nq;
    a.nq0 = n_path;
    a.nT = c->nT;
    a.ntet = 6 * c->nq;
    a.q0_first = p_first;
    a.ntab = ntab;
    Pol pol;
    for (int k = 0; k < 3; ++k) {
        pol.lo[k] = 0;
        pol.hi[k] = c->ndof - 1;
    }
    return launch_tetra3<true, true>(c, a, n_slots, pol, d_w, nullptr, om0, c->ph_grid.omega.p, c->ph_grid.nbe.p,
                                     om2t, nbe2t, d_lw, d_scratch);
}

int run_iso(spring_ctx* c, int q0_first, int n_q0, int delta_mode, double sigma, const double* g2, double* d_rate) {
    const size_t per = (size_t)c->nq * c->ndof * c->ndof;
    size_t budget = (size_t)64 << 20;
    int slots = (int)std::max<size_t>(1, budget / (per * sizeof(double)));
    slots = std::min(slots, n_q0);
    SPRING_CHECK(dalloc(c, c->d_wiso, per * slots, "isotope W"));
    DBuf<double> dg2;
    SPRING_CHECK(dalloc(c, dg2, c->nb, "g2"));
    int rc = h2d(c, dg2.p, g2, sizeof(double) * c->nb, "g2");
    const int threads = 128;
    for (int b = 0; rc == SPRING_OK && b < n_q0; b += slots) {
        const int ns = std::min(slots, n_q0 - b);
        const long long tot = (long long)ns * per;
        const int blocks = (int)std::min<long long>((tot + threads - 1) / threads, 148LL * 64);
        if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "iso: injected launch failure"); break; }
        k_iso_w<<<blocks, threads, 0, c->stream>>>(c->ndof, c->nb, c->nq, q0_first + b, ns, PI, dg2.p,
                                                   c->ph_irr.evec.p, c->ph_irr.omega.p, c->ph_grid.evec.p, c->d_wiso.p);
        rc = launch_check(c, "k_iso_w");
        if (rc != SPRING_OK) break;
        if (launch_injected(c)) { rc = fail(c, SPRING_ERR_INJECTED, "iso: injected launch failure"); break; }
        if (delta_mode == SPRING_DELTA_TETRA) {
            const long long items = 6LL * c->nq * c->ndof;
            dim3 grid(grid_x(items, threads, ns), ns);
            k_iso_tetra<<<grid, threads, 0, c->stream>>>(c->ndof, c->nq, c->nq0, 6 * c->nq, q0_first + b, c->nT,
                                                         reinterpret_cast<const int4*>(c->d_tetra.p), c->d_wiso.p,
                                                         c->ph_irr.omega.p, c->ph_grid.omega.p, d_rate);
            rc = launch_check(c, "k_iso_tetra");
        } else {
            const long long items = (long long)c->nq * c->ndof;
            dim3 grid(grid_x(items, threads, ns), ns);
            k_iso_gauss<<<grid, threads, 0, c->stream>>>(c->ndof, c->nq, c->nq0, q0_first + b, c->nT, 1.0 / sigma,
                                                         1.0 / (sigma * sigma), c->d_wiso.p, c->ph_irr.omega.p,
                                                         c->ph_grid.omega.p, d_rate);
            rc = launch_check(c, "k_iso_gauss");
        }
    }
    cudaStreamSynchronize(c->stream);
    dfree(dg2);
    return rc;
}

}  // namespace spring
