// Dipole-dipole (Ewald) part of the dynamical matrix and of its q-derivative, for the phonon
// kernels (LongEw = .true., &FCInfo Force_dd).
//
// Per q-point, the reference adds DynMatgv_Ew (src/Kappa/Src/DynaMat_mod.f90:285-380) to the
// short-range D(q):
//   Cq = KSpaceEW(q) - RealSpaceEW(q) - CConst,  CqZ = CombineZStar(Cq) - delta CSumq0,
//   D_ew(3mu+a, 3nu+b) = eV_A2 CqZ(b, a, nu, mu) / sqrt(m_mu m_nu)
// (EwaldSum_mod.f90:37-563), and at q = 0 DynMat_NA along qhat (DynaMat_mod.f90:383-483) with the
// q-derivative by central differences of DynMat_Ew at +-h/2 (h = |qhat| / 8); qhat is the next
// point of the list minus this one (the previous one for the last point), as in get_phonon
// (DynaMat_mod.f90:548-590), or q + (0.0034, 0, 0.001234) for single points (get_phonon_singleq,
// src/LineWidth/Src/DynaMat_mod.f90:770-800).
//
// Layout of the work: one CTA per q-point.  The real-space sum is q-independent apart from its
// phase, so its Born-charge-folded terms HZ_R are precomputed on the host (host/ewald.hpp) and the
// kernel forms sum_R e^{iqR} HZ_R and sum_R iR e^{iqR} HZ_R.  The reciprocal-space sum is staged in
// shared memory 64 G-vectors at a time (K = G + q, exp(-K.eps.K / 4 Lmb^2) / K.eps.K, the
// derivative factors and e^{iK.tau_mu} per atom), and each thread accumulates one (nu, mu, a, b)
// entry and its three derivatives over its share of the chunk; the Born charges are applied once
// per q after the sum (CombineZStar is linear).  FP64 throughout.
// Output dd[item][0][row][col] = D_ew, dd[item][1 + k][row][col] = dD_ew/dq_k.
#include <algorithm>
#include <string>

#include "spring_internal.cuh"
#include "../host/ewald.hpp"

namespace spring {
namespace {

constexpr int EW_THREADS = 128;
constexpr int GC = 64;   // G-vectors per staged chunk
constexpr int RC = 128;  // R-points per staged chunk

struct EwArgs {
    int nb, n, E, J, ng, nr, gamma_mode;
    double inv4l2, q4, vol, ev_a2;
    double eps[9];
    double qdir[3];
    const double* g;     // [NG][3]
    const double* r;     // [NR][3]
    const double* hz;    // [NR][E]
    const double2* cc;   // [E]
    const double* tau;   // [nb][3]
    const double* z;     // Zstar(3,3,nb)
    const double* mrs;   // 1/sqrt(m) per basis atom
};

struct EwSmem {
    double2* raw;   // [J][4][E]
    double2* comb;  // [4][E]
    double* gs;     // [GC][8]: K, KG, KpLmb, epsK
    double2* ph;    // [GC][nb]: e^{i K.tau_mu}
    double2* rph;   // [RC]: e^{i q.R}
};

__device__ __forceinline__ void decode(int e, int nb, int& b, int& al, int& nu, int& mu) {
    b = e % 3;
    al = (e / 3) % 3;
    nu = (e / 9) % nb;
    mu = e / (9 * nb);
}

// D_ew(q) (and, with grad, its three derivatives) into comb[k][e], e in the (b, a, nu, mu) order,
// already scaled: comb = eV_A2 (CqZ) / sqrt(m m).  Every thread of the CTA calls it.
__device__ void ew_eval(const EwArgs& a, const double q[3], bool grad, const EwSmem& S) {
    const int tid = threadIdx.x, T = blockDim.x, E = a.E, J = a.J, nc = grad ? 4 : 1;
    for (int w = tid; w < J * 4 * E; w += T) S.raw[w] = make_double2(0.0, 0.0);
    const bool qnz = fabs(q[0]) > CMP_PREC || fabs(q[1]) > CMP_PREC || fabs(q[2]) > CMP_PREC;
    for (int g0 = 0; g0 < a.ng; g0 += GC) {
        __syncthreads();
        const int gn = min(GC, a.ng - g0);
        for (int i = tid; i < gn; i += T) {  // stage the chunk (KSpaceEW_gv, EwaldSum_mod.f90:375-437)
            const double* G = a.g + 3 * (g0 + i);
            double* s = S.gs + 8 * i;
            const bool use = qnz || fabs(G[0]) > CMP_PREC || fabs(G[1]) > CMP_PREC || fabs(G[2]) > CMP_PREC;
            if (!use) {
                for (int k = 0; k < 8; ++k) s[k] = 0.0;
                for (int mu = 0; mu < a.nb; ++mu) S.ph[i * a.nb + mu] = make_double2(0.0, 0.0);
                continue;
            }
            const double K[3] = {G[0] + q[0], G[1] + q[1], G[2] + q[2]};
            double eK[3];
            for (int j = 0; j < 3; ++j) eK[j] = K[0] * a.eps[3 * j] + K[1] * a.eps[1 + 3 * j] + K[2] * a.eps[2 + 3 * j];
            const double KeK = K[0] * eK[0] + K[1] * eK[1] + K[2] * eK[2];
            s[0] = K[0];
            s[1] = K[1];
            s[2] = K[2];
            s[3] = exp(-KeK * a.inv4l2) / KeK;
            s[4] = 1.0 / KeK + a.q4;
            for (int ii = 0; ii < 3; ++ii)  // dot(eps(:, ii), K) + dot(K, eps(ii, :))
                s[5 + ii] = (a.eps[3 * ii] * K[0] + a.eps[1 + 3 * ii] * K[1] + a.eps[2 + 3 * ii] * K[2]) +
                            (K[0] * a.eps[ii] + K[1] * a.eps[ii + 3] + K[2] * a.eps[ii + 6]);
            for (int mu = 0; mu < a.nb; ++mu) {
                double sn, cs;
                sincos(K[0] * a.tau[3 * mu] + K[1] * a.tau[3 * mu + 1] + K[2] * a.tau[3 * mu + 2], &sn, &cs);
                S.ph[i * a.nb + mu] = make_double2(cs, sn);
            }
        }
        __syncthreads();
        const bool one = E * J <= T;
        for (int w = tid; one ? w < E * J : w < E; w += T) {
            const int j = one ? w / E : 0, e = one ? w % E : w;
            const int step = one ? J : 1;
            int b, al, nu, mu;
            decode(e, a.nb, b, al, nu, mu);
            double tmn[3];
            for (int k = 0; k < 3; ++k) tmn[k] = a.tau[3 * mu + k] - a.tau[3 * nu + k];
            double2 acc[4] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0),
                              make_double2(0.0, 0.0)};
            for (int i = j; i < gn; i += step) {
                const double* s = S.gs + 8 * i;
                const double2 pm = S.ph[i * a.nb + mu], pn = S.ph[i * a.nb + nu];
                // e^{iK.(tau_mu - tau_nu)} = pm conj(pn)
                const double2 ph = make_double2(pm.x * pn.x + pm.y * pn.y, pm.y * pn.x - pm.x * pn.y);
                const double2 Kmn = make_double2(s[3] * ph.x, s[3] * ph.y);
                const double kk = s[al] * s[b];
                const double2 Kab = make_double2(kk * Kmn.x, kk * Kmn.y);
                acc[0].x += Kab.x;
                acc[0].y += Kab.y;
                if (grad)
                    for (int d = 0; d < 3; ++d) {
                        // Kab (i tmn_d - epsK_d KpLmb) + Kmn d(K_a K_b)/dK_d
                        const double f = s[5 + d] * s[4];
                        const double km = (al == d ? s[b] : 0.0) + (b == d ? s[al] : 0.0);
                        acc[1 + d].x += -Kab.y * tmn[d] - Kab.x * f + Kmn.x * km;
                        acc[1 + d].y += Kab.x * tmn[d] - Kab.y * f + Kmn.y * km;
                    }
            }
            for (int k = 0; k < nc; ++k) {
                double2& r = S.raw[(j * 4 + k) * E + e];
                r.x += acc[k].x;
                r.y += acc[k].y;
            }
        }
    }
    __syncthreads();
    // CombineZStar of the reciprocal part, times 4 pi / vol
    const double ks = 4.0 * 3.141592653589793 / a.vol;
    for (int w = tid; w < nc * E; w += T) {
        const int k = w / E, e = w % E;
        int b, al, nu, mu;
        decode(e, a.nb, b, al, nu, mu);
        const double* Zm = a.z + 9 * mu;
        const double* Zn = a.z + 9 * nu;
        double2 s = make_double2(0.0, 0.0);
        for (int ap = 0; ap < 3; ++ap)
            for (int bp = 0; bp < 3; ++bp) {
                const int src = bp + 3 * ap + 9 * nu + 9 * a.nb * mu;
                double2 v = make_double2(0.0, 0.0);
                for (int j = 0; j < J; ++j) {
                    const double2 x = S.raw[(j * 4 + k) * E + src];
                    v.x += x.x;
                    v.y += x.y;
                }
                const double zz = Zm[ap + 3 * al] * Zn[bp + 3 * b];
                s.x += zz * v.x;
                s.y += zz * v.y;
            }
        S.comb[k * E + e] = make_double2(ks * s.x, ks * s.y);
    }
    // minus the real-space part: sum_R e^{iqR} HZ_R (and i R_k e^{iqR} HZ_R)
    for (int r0 = 0; r0 < a.nr; r0 += RC) {
        __syncthreads();
        const int rn = min(RC, a.nr - r0);
        for (int i = tid; i < rn; i += T) {
            const double* R = a.r + 3 * (r0 + i);
            double sn, cs;
            sincos(q[0] * R[0] + q[1] * R[1] + q[2] * R[2], &sn, &cs);
            S.rph[i] = make_double2(cs, sn);
        }
        __syncthreads();
        for (int w = tid; w < nc * E; w += T) {
            const int k = w / E, e = w % E;
            double2 acc = make_double2(0.0, 0.0);
            for (int i = 0; i < rn; ++i) {
                const double h = a.hz[(size_t)(r0 + i) * E + e];
                const double2 p = S.rph[i];
                if (k == 0) {
                    acc.x += p.x * h;
                    acc.y += p.y * h;
                } else {
                    const double Rk = a.r[3 * (r0 + i) + k - 1];
                    acc.x -= Rk * p.y * h;  // i R_k e^{iqR} h
                    acc.y += Rk * p.x * h;
                }
            }
            double2& c = S.comb[k * E + e];
            c.x -= acc.x;
            c.y -= acc.y;
        }
    }
    __syncthreads();
    for (int w = tid; w < nc * E; w += T) {
        const int k = w / E, e = w % E;
        int b, al, nu, mu;
        decode(e, a.nb, b, al, nu, mu);
        double2 c = S.comb[k * E + e];
        if (k == 0) {
            c.x += a.cc[e].x;
            c.y += a.cc[e].y;
        }
        const double f = a.ev_a2 * a.mrs[mu] * a.mrs[nu];
        S.comb[k * E + e] = make_double2(f * c.x, f * c.y);
    }
    __syncthreads();
}

// comb[src] (src 0: D_ew, 1..3: its derivatives) into slot dst of the item's output
__device__ __forceinline__ void put(const EwArgs& a, const EwSmem& S, int src, int dst, double2* out) {
    const int n = a.n;
    for (int e = threadIdx.x; e < a.E; e += blockDim.x) {
        int b, al, nu, mu;
        decode(e, a.nb, b, al, nu, mu);
        out[(dst * n + 3 * mu + al) * n + 3 * nu + b] = S.comb[src * a.E + e];
    }
}

// Work item i < n_a: point list_a[i] (or i) of list A (nqa points), else point i - n_a of list B.
__global__ void __launch_bounds__(EW_THREADS) k_ewald(EwArgs a, const double* __restrict__ qa, int nqa,
                                                      const int* __restrict__ list_a, int n_a,
                                                      const double* __restrict__ qb, int nqb, int n_b,
                                                      double2* __restrict__ dd) {
    extern __shared__ __align__(16) unsigned char ew_smem[];
    EwSmem S;
    S.raw = reinterpret_cast<double2*>(ew_smem);
    S.comb = S.raw + (size_t)a.J * 4 * a.E;
    S.gs = reinterpret_cast<double*>(S.comb + 4 * a.E);
    S.ph = reinterpret_cast<double2*>(S.gs + 8 * GC);
    S.rph = S.ph + GC * a.nb;
    const int n = a.n;
    for (int item = blockIdx.x; item < n_a + n_b; item += gridDim.x) {
        const bool in_a = item < n_a;
        const double* Q = in_a ? qa : qb;
        const int nq = in_a ? nqa : nqb;
        const int qi = in_a ? (list_a ? list_a[item] : item) : item - n_a;
        const double q[3] = {Q[3 * qi], Q[3 * qi + 1], Q[3 * qi + 2]};
        double2* out = dd + (size_t)item * 4 * n * n;
        const bool gamma = fabs(q[0]) < CMP_PREC && fabs(q[1]) < CMP_PREC && fabs(q[2]) < CMP_PREC;
        if (!gamma) {
            ew_eval(a, q, true, S);
            for (int k = 0; k < 4; ++k) put(a, S, k, k, out);
            __syncthreads();
            continue;
        }
        double qh[3];
        for (int k = 0; k < 3; ++k) {
            if (a.gamma_mode == 1 || nq == 1) qh[k] = q[k] + a.qdir[k];
            else if (qi != nq - 1) qh[k] = Q[3 * (qi + 1) + k] - q[k];
            else qh[k] = q[k] - Q[3 * (qi - 1) + k];
        }
        const double h = sqrt(qh[0] * qh[0] + qh[1] * qh[1] + qh[2] * qh[2]) / 8.0;
        // DynMat_NA: D_ew(0) plus 4 pi eV_A2 (qh.Z_mu)_a (qh.Z_nu)_b / (vol qh.eps.qh sqrt(m m))
        const double zero[3] = {0.0, 0.0, 0.0};
        ew_eval(a, zero, false, S);
        double den = 0.0;
        for (int j = 0; j < 3; ++j)
            den += (qh[0] * a.eps[3 * j] + qh[1] * a.eps[1 + 3 * j] + qh[2] * a.eps[2 + 3 * j]) * qh[j];
        const double fna = 4.0 * 3.141592653589793 * a.ev_a2 / (a.vol * den);
        for (int e = threadIdx.x; e < a.E; e += blockDim.x) {
            int b, al, nu, mu;
            decode(e, a.nb, b, al, nu, mu);
            double t1 = 0.0, t2 = 0.0;
            for (int j = 0; j < 3; ++j) {
                t1 += qh[j] * a.z[al + 3 * j + 9 * mu];  // dot_product(q, Zstar(alpha, :, mu))
                t2 += qh[j] * a.z[b + 3 * j + 9 * nu];
            }
            const double na = (t1 * t2) * (a.mrs[mu] * a.mrs[nu]) * fna;
            const double2 d0 = S.comb[e];
            out[(3 * mu + al) * n + 3 * nu + b] = make_double2(d0.x + na, d0.y);
        }
        __syncthreads();
        for (int k = 0; k < 3; ++k) {  // (DynEw(q + h/2 e_k) - DynEw(q - h/2 e_k)) / h
            double qp[3] = {q[0], q[1], q[2]};
            qp[k] += 0.5 * h;
            ew_eval(a, qp, false, S);
            put(a, S, 0, 1 + k, out);
            __syncthreads();
            double qm[3] = {q[0], q[1], q[2]};
            qm[k] -= 0.5 * h;
            ew_eval(a, qm, false, S);
            for (int e = threadIdx.x; e < a.E; e += blockDim.x) {
                int b, al, nu, mu;
                decode(e, a.nb, b, al, nu, mu);
                double2& o = out[((1 + k) * n + 3 * mu + al) * n + 3 * nu + b];
                const double2 m = S.comb[e];
                o = make_double2((o.x - m.x) / h, (o.y - m.y) / h);
            }
            __syncthreads();
        }
    }
}

size_t ew_smem_bytes(int nb, int J) {
    const int E = 9 * nb * nb;
    return sizeof(double2) * ((size_t)J * 4 * E + 4 * E) + sizeof(double) * 8 * GC + sizeof(double2) * (GC * nb + RC);
}

}  // namespace

int set_dipole(spring_ctx* c, const double* atm_pos, const double* eps, const double* zstar, int decide,
               double prec_ew, double lmb, const int* gmesh, const int* rmesh, const int* sup_cell) {
    EwaldDev& D = c->ew;
    if (!eps) {  // switch the term off
        D.on = false;
        return SPRING_OK;
    }
    if (!atm_pos || !zstar || !rmesh || (!decide && !gmesh))
        return fail(c, SPRING_ERR_ARG, "dipole term: atm_pos, BornZ and Rmesh (and Gmesh unless decided) needed");
    const int sc_default[3] = {5, 5, 5};
    spring_ewald::Setup S;
    std::string err;
    if (spring_ewald::setup(c->latvec, c->nb, atm_pos, eps, zstar, decide, prec_ew, lmb, gmesh, rmesh,
                            sup_cell ? sup_cell : sc_default, S, err) != 0)
        return fail(c, SPRING_ERR_ARG, "%s", err.c_str());
    const int E = 9 * c->nb * c->nb;
    std::vector<double2> cc(E);
    for (int e = 0; e < E; ++e) cc[e] = make_double2(S.cc[2 * e], S.cc[2 * e + 1]);
    SPRING_CHECK(dalloc(c, D.g, S.gpts.size(), "Ewald G points"));
    SPRING_CHECK(dalloc(c, D.r, S.rpts.size(), "Ewald R points"));
    SPRING_CHECK(dalloc(c, D.hz, S.hz.size(), "Ewald real-space table"));
    SPRING_CHECK(dalloc(c, D.cc, E, "Ewald constant"));
    SPRING_CHECK(dalloc(c, D.tau, S.tau.size(), "Ewald basis"));
    SPRING_CHECK(dalloc(c, D.z, S.zstar.size(), "Born charges"));
    SPRING_CHECK(h2d(c, D.g.p, S.gpts.data(), sizeof(double) * S.gpts.size(), "Ewald G points"));
    SPRING_CHECK(h2d(c, D.r.p, S.rpts.data(), sizeof(double) * S.rpts.size(), "Ewald R points"));
    SPRING_CHECK(h2d(c, D.hz.p, S.hz.data(), sizeof(double) * S.hz.size(), "Ewald real-space table"));
    SPRING_CHECK(h2d(c, D.cc.p, cc.data(), sizeof(double2) * E, "Ewald constant"));
    SPRING_CHECK(h2d(c, D.tau.p, S.tau.data(), sizeof(double) * S.tau.size(), "Ewald basis"));
    SPRING_CHECK(h2d(c, D.z.p, S.zstar.data(), sizeof(double) * S.zstar.size(), "Born charges"));
    D.lmb = S.lmb;
    D.vol = S.vol;
    for (int i = 0; i < 9; ++i) D.eps[i] = S.eps[i];
    for (int k = 0; k < 3; ++k) {
        D.gmesh[k] = S.gmesh[k];
        D.rmesh[k] = S.rmesh[k];
    }
    D.ng = S.ng();
    D.nr = S.nr();
    // an even mesh is not symmetric under R -> -R (fold_indx keeps +N/2): D(-q) = conj D(q) then
    // holds only to the sum's tail, and every grid point is solved directly
    D.even = false;
    for (int k = 0; k < 3; ++k) D.even = D.even || (S.gmesh[k] % 2 == 0) || (S.rmesh[k] % 2 == 0);
    D.on = true;
    return SPRING_OK;
}

// dd[item][4][n][n] for the items of one phonon launch (same item order as the phonon kernels).
int launch_ewald(spring_ctx* c, const double* qa, int nqa, const int* list_a, int n_a, const double* qb, int nqb,
                 int n_b, int gamma_mode, const double2** dd_out) {
    *dd_out = nullptr;
    EwaldDev& D = c->ew;
    if (!D.on) return SPRING_OK;
    const int items = n_a + n_b, n = c->ndof;
    if (items == 0) return SPRING_OK;
    SPRING_CHECK(dalloc(c, D.dd, (size_t)items * 4 * n * n, "dipole-dipole matrices"));
    EwArgs a{};
    a.nb = c->nb;
    a.n = n;
    a.E = 9 * c->nb * c->nb;
    a.J = std::max(1, EW_THREADS / a.E);
    a.ng = D.ng;
    a.nr = D.nr;
    a.gamma_mode = gamma_mode;
    a.inv4l2 = 1.0 / (4.0 * D.lmb * D.lmb);
    a.q4 = 0.25 / (D.lmb * D.lmb);
    a.vol = D.vol;
    a.ev_a2 = (1.602176634 * 2.99792458) * (1.602176634 * 2.99792458) * 6.241509074460763 * 0.1;
    for (int i = 0; i < 9; ++i) a.eps[i] = D.eps[i];
    a.qdir[0] = 0.0034;
    a.qdir[1] = 0.0;
    a.qdir[2] = 0.001234;
    a.g = D.g.p;
    a.r = D.r.p;
    a.hz = D.hz.p;
    a.cc = D.cc.p;
    a.tau = D.tau.p;
    a.z = D.z.p;
    a.mrs = c->d_mass_rs.p;
    const size_t smem = ew_smem_bytes(a.nb, a.J);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_ewald, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "ewald: injected launch failure");
    const int blocks = std::min(items, 148 * 8);
    k_ewald<<<blocks, EW_THREADS, smem, c->stream>>>(a, qa, nqa, list_a, n_a, qb, nqb, n_b, D.dd.p);
    SPRING_CHECK(launch_check(c, "k_ewald"));
    *dd_out = D.dd.p;
    return SPRING_OK;
}

}  // namespace spring
