// RTA thermal conductivity and linewidth bookkeeping on the device.
//   kappa_noIter_symm (src/Kappa/Src/ThermalConductivity.f90:167-292) with the
//   rotation-averaged v(x)v of GrVelKronProdSymm (VelocityKronProd_symm.f90:34-91),
//   or kappa_noIter over the full grid (ThermalConductivity.f90:36-164).
// kappa_ab = kW_m_k / (T^2 V Nq) * sum_{q,s} w^2 n (n+1) tau (v(x)v)_ab,  tau = 0.5/Gamma;
// Gamma-point acoustic modes are skipped.  Up to 64 CTAs per temperature each reduce a slice of
// the mode points (per thread, then as a tree in shared memory) into a partial sum; k_kappa_sum adds
// the partial sums in block order, so the result does not depend on scheduling.  Negligible cost.
#include <algorithm>

#include "spring_internal.cuh"

namespace spring {
namespace {

__global__ void k_axpy_lw(int n, int nq0, int nT, int q0_first, int n_q0, double a, const double* __restrict__ x,
                          double* __restrict__ y) {
    const int per = n_q0 * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nT * per; i += gridDim.x * blockDim.x) {
        const int T = i / per, j = i % per;
        const size_t o = ((size_t)T * nq0 + q0_first) * n + j;
        y[o] += a * x[o];
    }
}

struct KapArgs {
    int n, nq, nq0, nsym, symm, s_lo, s_hi;
    double kwmk, vol;
};

__global__ void __launch_bounds__(256) k_kappa(KapArgs a, const double* __restrict__ temps,
                                               const int* __restrict__ irr_int, const int* __restrict__ mult,
                                               const double* __restrict__ rxyz, const int* __restrict__ qint,
                                               const int* __restrict__ pos, const double* __restrict__ om,
                                               const double* __restrict__ nbe, const double* __restrict__ vel,
                                               const double* __restrict__ lw, double* __restrict__ part) {
    __shared__ double red[256][9];
    __shared__ double smode[MAX_NDOF * 9];
    const int T = blockIdx.y, nbk = gridDim.x;
    const double temp = temps[T];
    const int npts = a.symm ? a.nq0 : a.nq;
    for (int i = threadIdx.x; i < a.n * 9; i += blockDim.x) smode[i] = 0.0;
    __syncthreads();
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < npts * a.n; it += nbk * blockDim.x) {
        const int q = it / a.n, s = it % a.n;
        const int* qi = a.symm ? irr_int + 3 * q : qint + 3 * q;
        const bool gamma = qi[0] == 0 && qi[1] == 0 && qi[2] == 0;
        const int strt = gamma ? 3 : a.s_lo;
        if (s < strt || s > a.s_hi) continue;
        const int ip = a.symm ? q : pos[q] - 1;
        const double w = om[(size_t)q * a.n + s];
        const double nb = nbe[((size_t)T * npts + q) * a.n + s];
        const double tau = 0.5 / lw[((size_t)T * a.nq0 + ip) * a.n + s];
        const double pre = (w * w) * nb * (nb + 1.0) * tau;
        const double* v = vel + ((size_t)q * a.n + s) * 3;
        double kr[9];
        if (a.symm) {
            for (int k = 0; k < 9; ++k) kr[k] = 0.0;
            for (int ns = 0; ns < a.nsym; ++ns) {
                const double* R = rxyz + 9 * ns;  // column-major 3x3
                double rv[3];
                for (int i = 0; i < 3; ++i) rv[i] = R[i] * v[0] + R[i + 3] * v[1] + R[i + 6] * v[2];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) kr[3 * i + j] += rv[i] * rv[j];
            }
            const double p = 1.0 / double(a.nsym / mult[q]);
            for (int k = 0; k < 9; ++k) kr[k] *= p;
        } else {
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) kr[3 * i + j] = v[i] * v[j];
        }
        for (int k = 0; k < 9; ++k) {
            const double kq = pre * kr[k];
            acc[k] += kq;
            atomicAdd(&smode[s * 9 + k], kq);
        }
    }
    for (int k = 0; k < 9; ++k) red[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int k = 0; k < 9; ++k) red[threadIdx.x][k] += red[threadIdx.x + h][k];
        __syncthreads();
    }
    // this block's partial sums: [T][block][kappa 9, then mode n x 9]
    double* out = part + ((size_t)T * nbk + blockIdx.x) * (9 + a.n * 9);
    if (threadIdx.x < 9) out[threadIdx.x] = red[0][threadIdx.x];
    for (int i = threadIdx.x; i < a.n * 9; i += blockDim.x) out[9 + i] = smode[i];
}

// kappa[T][9] and mode[T][n][9] (mode may be null): the blocks' partial sums in block order, times
// the prefactor.
__global__ void k_kappa_sum(KapArgs a, int nbk, const double* __restrict__ temps, const double* __restrict__ part,
                            double* __restrict__ kappa, double* __restrict__ mode) {
    const int T = blockIdx.x;
    const int w = 9 + a.n * 9;
    const double temp = temps[T];
    const double f2 = a.kwmk / ((temp * temp) * a.vol) / double(a.nq);
    for (int i = threadIdx.x; i < w; i += blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nbk; ++b) acc += part[((size_t)T * nbk + b) * w + i];
        if (i < 9) kappa[T * 9 + i] = acc * f2;
        else if (mode) mode[(size_t)T * a.n * 9 + (i - 9)] = acc * f2;
    }
}

}  // namespace

int run_axpy_lw(spring_ctx* c, double a, const double* d_x, double* d_y, int q0_first, int n_q0) {
    const int total = c->nT * n_q0 * c->ndof;
    if (total == 0) return SPRING_OK;
    const int threads = 256, blocks = (total + threads - 1) / threads;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "axpy: injected launch failure");
    k_axpy_lw<<<blocks, threads, 0, c->stream>>>(c->ndof, c->nq0, c->nT, q0_first, n_q0, a, d_x, d_y);
    return launch_check(c, "k_axpy_lw");
}

int run_kappa_rta(spring_ctx* c, int symm, int nsym, const double* d_rxyz, int s_lo, int s_hi, double* d_kappa,
                  double* d_mode) {
    KapArgs a;
    a.n = c->ndof;
    a.nq = c->nq;
    a.nq0 = c->nq0;
    a.nsym = nsym;
    a.symm = symm;
    a.s_lo = s_lo;
    a.s_hi = s_hi;
    a.kwmk = host_constants().kW_m_k;
    a.vol = c->vol;
    const Phonons& ph = symm ? c->ph_irr : c->ph_grid;
    // blocks per temperature: about two mode points per thread, at most 64 blocks
    const int npts = (symm ? c->nq0 : c->nq) * c->ndof;
    const int nbk = std::max(1, std::min(64, (npts + 511) / 512));
    SPRING_CHECK(dalloc(c, c->d_kap_part, (size_t)c->nT * nbk * (9 + c->ndof * 9), "kappa partial sums"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "kappa: injected launch failure");
    k_kappa<<<dim3(nbk, c->nT), 256, 0, c->stream>>>(a, c->d_temps.p, c->d_irr_int.p, c->d_mult.p, d_rxyz,
                                                      c->d_qint.p, c->d_pos.p, ph.omega.p, ph.nbe.p, ph.vel.p,
                                                      c->d_lw_all.p, c->d_kap_part.p);
    SPRING_CHECK(launch_check(c, "k_kappa"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "kappa: injected launch failure");
    k_kappa_sum<<<c->nT, 256, 0, c->stream>>>(a, nbk, c->d_temps.p, c->d_kap_part.p, d_kappa, d_mode);
    return launch_check(c, "k_kappa_sum");
}

}  // namespace spring
