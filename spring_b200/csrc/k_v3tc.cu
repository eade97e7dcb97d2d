// Three-phonon V3 on the 5th-generation tensor cores (tcgen05, BF16 in, FP32
// accumulate), with the Gaussian linewidth sum.  Two-atom cells.
//
// Same quantity as ScatterMatEl / ScatterProbability + CalculateLinewidth
// (src/Kappa/Src/ThirdOrder_m.f90:278-439, 442-543), regrouped so that the
// bulk of the work is a GEMM with a shared operand:
//   U_q[mu][N b][s]      = e^{i q.R_{mu N}} m_{nu(N)}^-1/2 e_q(nu(N) b, s)         (per grid q)
//   Z_q1[mu][a s1][N2 c] = sum_{N1 b} FC3[mu][N1][N2][a b c] U_q1[mu][N1 b][s1]     (per grid q1)
//   Y[mu][a s1][s2]      = sum_{N2 c} Z_q1[mu][a s1][N2 c] U_q2[mu][N2 c][s2]       (per pair: tensor cores)
//   Phi[s0][s1][s2]      = sum_{mu a} m_mu^-1/2 e0(mu a, s0) Y[mu][a s1][s2]        (per pair: epilogue)
// Pairs are grouped by q1, so one tile is up to 16 pairs sharing Z_q1: the MMA
// computes Y^T for rows 8 pair + s2 at once, M = 128, N = 48 (8 columns per
// s1: Re/Im of a and two zero rows, s1 in the order 0 3 1 4 2 5), K = 48 (Re/Im
// of (N2, c), 42 used), one accumulator per basis atom mu in tensor memory.  The complex product is written as a real one:
//   A[(pair, s2)][k] = [Re U_q2 | Im U_q2],   B[(re, a s1)][k] = [Re Z | -Im Z],
//   B[(im, a s1)][k] = [Im Z | Re Z].
// Precision: SPRING_BF16 rounds A and B to BF16 once; SPRING_BF16X3 splits each
// into hi + lo BF16 parts and accumulates hi*hi + hi*lo + lo*hi (compensated).
// Frequencies, occupations, the delta weights and every sum stay FP64.  Pairs with
// no mode triple inside the delta window are dropped before the tiles are cut
// (k_tc_keys, about half of them).  One pass: k_v3tc computes Y on the tensor
// cores and screens each mode triple in FP32 against the window where a delta
// weight can exceed exp(-40) of its peak (4e-18); for the ~1-3 % inside it the
// epilogue warp forms |Phi|^2 (FP32), stages it in shared memory and, 64 at a
// time (two per lane), evaluates W, the FP64 delta weights and the phase-space
// and linewidth sums (or, for the iterative BTE, the operator entries).
// Roofline: tensor pipe for Y (about 74 kflop issued per pair per split pass);
// in practice the per-tile pipeline (TMA requests, FP32 screening issue) and the
// L2 latency of the mode records read by the staged evaluations.
#include <algorithm>
#include <vector>
#include <cub/cub.cuh>
#include <cuda.h>
#include <cuda_bf16.h>

#include "spring_internal.cuh"
#include "tc.cuh"

namespace spring {
namespace {

constexpr int NMODE = 6;     // Ndof of the two-atom cell
constexpr int KP = 48;       // padded K: Re/Im of (N2, c), 2 * 3 * Na3 <= 48
constexpr int EPT = 16;      // pairs per tile: one 8-row core-matrix group each (rows 8e .. 8e+5 of 128)
constexpr uint32_t LBO = 128, SBO = (KP / 8) * 128;
constexpr int B_BYTES = (48 / 8) * SBO;   // 4608
constexpr int AIMG = 8 * KP;              // bf16 elements of one (q, mu, hi/lo) A image: 8 rows x 48 (768 bytes)
constexpr int BIMG = 48 * KP;             // bf16 elements of one (q1, mu, hi/lo) B image (4608 bytes)
constexpr double EXP_CUT = 40.0;
// Poll limit of the waits that drain work already issued (TMA copies, MMAs) before shared and
// tensor memory are released: these always complete, the limit only bounds a broken device.
constexpr long long MAX_SPINS = 1LL << 26;

// bf16 hi/lo split of an FP64 value
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    const float f = (float)x;
    hi = __float2bfloat16_rn(f);
    lo = __float2bfloat16_rn(f - __bfloat162float(hi));
}

// FP32 delta-window test of one mode triple, shared by the pair pre-screen and the tensor-core
// pass so that both decide alike.  From the FP32 omegas, (d, b) = (w0 - w2, w0 + w2) of (s0, s2)
// (tc_window_vals); the triple is kept when ||w1| - |d|| < R or |b - w1| < R.  R is the half-width
// where a delta weight falls to exp(-40) of its peak, times 1.0001, plus 1e-3 rad/ps: far above the
// FP32 rounding of the omegas (~1e-5 rad/ps), so every triple with a weight above the cut passes.
__device__ __forceinline__ float2 tc_window_vals(float w0, float w2) { return make_float2(w0 - w2, w0 + w2); }
__device__ __forceinline__ bool tc_window(float d, float b, float w1, float rf) {
    return fabsf(fabsf(w1) - fabsf(d)) < rf || fabsf(b - w1) < rf;
}

// Phases e^{i q.R_{mu N}} of one grid point and basis atom, N < na, into ph[N] (threads 0..na-1).
__device__ __forceinline__ void q_phases(int q, int mu, int na, const double* __restrict__ posr,
                                         const double* __restrict__ qpnt, double2* ph) {
    const int N = threadIdx.x;
    if (N < na) {
        const double* R = posr + ((size_t)mu * na + N) * 3;
        const double qr = qpnt[3 * q] * R[0] + qpnt[3 * q + 1] * R[1] + qpnt[3 * q + 2] * R[2];
        double sn, cs;
        sincos(qr, &sn, &cs);
        ph[N] = make_double2(cs, sn);
    }
}

// U of one grid point, basis mu, slot k = N*3 + b, branch s (FP64), from the phases of (q, mu)
__device__ __forceinline__ double2 u_value(const double2* ph, int q, int mu, int k, int s, int na,
                                          const int* __restrict__ btyp, const double* __restrict__ mrs,
                                          const double2* __restrict__ evg) {
    const int N = k / 3, b = k % 3;
    const double cs = ph[N].x, sn = ph[N].y;
    const int nu = btyp[mu * na + N];
    const double m = mrs[nu];
    const double2 e = evg[((size_t)q * NMODE + s) * NMODE + nu * 3 + b];
    return make_double2(m * (cs * e.x - sn * e.y), m * (cs * e.y + sn * e.x));
}

// A table: per (q, hi/lo, mu) the 768-byte shared-memory image of one 8-row group of the canonical
// K-major layout, element (row s, k) at (k/8)*64 + s*8 + k%8, rows 6 and 7 zero.  Hi parts first,
// so a BF16 launch copies the two hi images as one block.  One CTA per (q, mu), images built in
// shared memory and written as 16-byte vectors.
__global__ void __launch_bounds__(128) k_tc_tab_a(int nq, int na, const double* __restrict__ posr,
                                                  const int* __restrict__ btyp, const double* __restrict__ mrs,
                                                  const double* __restrict__ qpnt, const double2* __restrict__ evg,
                                                  __nv_bfloat16* __restrict__ tab) {
    __shared__ double2 ph[8];
    __shared__ __align__(16) __nv_bfloat16 img[2][AIMG];
    const int q = blockIdx.x / 2, mu = blockIdx.x % 2;
    const int KR = 3 * na;
    q_phases(q, mu, na, posr, qpnt, ph);
    __syncthreads();
    for (int i = threadIdx.x; i < 8 * KP; i += blockDim.x) {
        const int k = i % KP, s = i / KP;
        double x = 0.0;
        if (k < 2 * KR && s < NMODE) {
            const double2 u = u_value(ph, q, mu, k % KR, s, na, btyp, mrs, evg);
            x = k < KR ? u.x : u.y;
        }
        __nv_bfloat16 hi, lo;
        split_bf16(x, hi, lo);
        const int off = (k / 8) * 64 + s * 8 + k % 8;
        img[0][off] = hi;
        img[1][off] = lo;
    }
    __syncthreads();
    constexpr int V = AIMG * 2 / 16;  // 16-byte vectors per image
    uint4* out = reinterpret_cast<uint4*>(tab + (size_t)q * 4 * AIMG + mu * AIMG);
    for (int i = threadIdx.x; i < 2 * V; i += blockDim.x)
        out[(i / V) * 2 * V + i % V] = reinterpret_cast<const uint4*>(&img[0][0])[i];
}

// B table: per (q1, hi/lo, mu) the 4608-byte shared-memory image of the 48 x 48 B operand in the
// canonical K-major layout: element (row n, k) at (n/8)*384 + (k/8)*64 + (n%8)*8 + k%8.  Row
// n = 8 slot(s1) + 3 part + a (part 0: Re output, 1: Im output) with slot(s1) = 2 (s1 % 3) + s1 / 3,
// so that the accumulator columns of s1 = g and g + 3 are the 16 columns from 16 g; rows 8 slot + 6,
// 8 slot + 7 and the K padding are zero.  Hi parts first.  One CTA per (q1, mu).
__host__ __device__ constexpr int b_slot(int s1) { return 2 * (s1 % 3) + s1 / 3; }
__device__ __forceinline__ size_t bimg(int n, int k) {
    return (size_t)(n / 8) * 384 + (size_t)(k / 8) * 64 + (n % 8) * 8 + k % 8;
}
__global__ void __launch_bounds__(128) k_tc_tab_b(int nq, int na, const double* __restrict__ fc3,
                                                  const double* __restrict__ posr, const int* __restrict__ btyp,
                                                  const double* __restrict__ mrs, const double* __restrict__ qpnt,
                                                  const double2* __restrict__ evg, __nv_bfloat16* __restrict__ tab) {
    __shared__ double2 sU[24 * NMODE];                   // [N b][s]
    __shared__ __align__(16) __nv_bfloat16 img[2][BIMG];  // hi, lo images of this (q1, mu), built here
    __shared__ double2 ph[8];
    __shared__ double sF[8 * 8 * 27];  // FC3 of mu, staged once: the CTA loops over grid points
    const int mu = blockIdx.x % 2;
    const int KR = 3 * na;
    for (int i = threadIdx.x; i < na * na * 27; i += blockDim.x) sF[i] = fc3[(size_t)mu * na * na * 27 + i];
    for (int q = blockIdx.x / 2; q < nq; q += gridDim.x / 2) {
        __syncthreads();  // the previous point's image has been written out
        q_phases(q, mu, na, posr, qpnt, ph);
        for (int i = threadIdx.x; i < (int)(sizeof(img) / 16); i += blockDim.x)  // padding rows and K stay zero
            reinterpret_cast<uint4*>(&img[0][0])[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (int i = threadIdx.x; i < KR * NMODE; i += blockDim.x)
            sU[i] = u_value(ph, q, mu, i / NMODE, i % NMODE, na, btyp, mrs, evg);
        __syncthreads();
        // Z[(a, s1)][(N2, c)] = sum_{N1, b} FC3[mu][N1][N2][a b c] U[N1 b][s1]: one thread per
        // (a, N2, c, s1 half), each FC3 value (staged in shared memory) used for three s1.
        for (int i = threadIdx.x; i < 3 * KR * 2; i += blockDim.x) {
            const int half = i % 2, t = i / 2, al = t / KR, k2 = t % KR;  // k2 = N2*3 + c
            const int N2 = k2 / 3, ga = k2 % 3;
            double zr[3] = {0.0, 0.0, 0.0}, zi[3] = {0.0, 0.0, 0.0};
            for (int N1 = 0; N1 < na; ++N1) {  // k1 = N1*3 + b in order
                const double* f = sF + (N1 * na + N2) * 27 + al * 9 + ga;
                const double2* u1 = sU + N1 * 3 * NMODE + half * 3;
#pragma unroll
                for (int be = 0; be < 3; ++be) {
                    const double fv = f[be * 3];
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const double2 u = u1[be * NMODE + j];
                        zr[j] = fma(fv, u.x, zr[j]);
                        zi[j] = fma(fv, u.y, zi[j]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int r = 8 * b_slot(half * 3 + j) + al, ri = r + 3;  // Re and Im output rows of (a, s1)
                __nv_bfloat16 h, l;
                // row r (Re output): [Re Z | -Im Z];  row ri (Im output): [Im Z | Re Z]
                split_bf16(zr[j], h, l);
                img[0][bimg(r, k2)] = h;               img[1][bimg(r, k2)] = l;
                img[0][bimg(ri, KR + k2)] = h;         img[1][bimg(ri, KR + k2)] = l;
                split_bf16(-zi[j], h, l);
                img[0][bimg(r, KR + k2)] = h;          img[1][bimg(r, KR + k2)] = l;
                split_bf16(zi[j], h, l);
                img[0][bimg(ri, k2)] = h;              img[1][bimg(ri, k2)] = l;
            }
        }
        __syncthreads();
        constexpr int V = BIMG * 2 / 16;  // 16-byte vectors per image
        uint4* out = reinterpret_cast<uint4*>(tab + (size_t)q * 4 * BIMG + mu * BIMG);
        for (int i = threadIdx.x; i < 2 * V; i += blockDim.x)
            out[(i / V) * 2 * V + i % V] = reinterpret_cast<const uint4*>(&img[0][0])[i];
    }
}

// q0 mode records, 64 bytes per (q0, s0): e0' = m_mu^-1/2 e0(mu a, s0) as float2[6], omega0, 1/omega0.
struct Q0Rec {
    float2 e0[NMODE];
    double w, ob;
};
static_assert(sizeof(Q0Rec) == 64, "q0 record");
__global__ void k_tc_q0tab(int nq0, const double2* __restrict__ ev0, const double* __restrict__ om0,
                           const double* __restrict__ ob0, const double* __restrict__ mrs, Q0Rec* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq0 * NMODE; i += gridDim.x * blockDim.x) {
        const int q = i / NMODE, s0 = i % NMODE;
        Q0Rec r;
        for (int k = 0; k < NMODE; ++k) {
            const double2 e = ev0[((size_t)q * NMODE + s0) * NMODE + k];
            const double m = mrs[k / 3];
            r.e0[k] = make_float2((float)(m * e.x), (float)(m * e.y));
        }
        r.w = om0[(size_t)q * NMODE + s0];
        r.ob = ob0[(size_t)q * NMODE + s0];
        out[i] = r;
    }
}

// Grid mode records, `rs` doubles per (q, s) (a multiple of 4, so 32-byte aligned): omega,
// 1/omega, nBE[T].
__global__ void k_tc_modes(int nq, int nT, int rs, const double* __restrict__ omg, const double* __restrict__ obg,
                           const double* __restrict__ nbeg, double* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)nq * NMODE * rs;
         i += (long long)gridDim.x * blockDim.x) {
        const long long qs = i / rs;
        const int k = (int)(i % rs);
        double v = 0.0;
        if (k == 0) v = omg[qs];
        else if (k == 1) v = obg[qs];
        else if (k - 2 < nT) v = nbeg[(size_t)(k - 2) * nq * NMODE + qs];
        out[i] = v;
    }
}

// ------------------------------------------------------------------ tiles
// Sort keys of the pairs: q1 for a pair with at least one mode triple inside the delta window,
// nq (sorted after every q1, and left out of the tiles) for a pair with none.  The test is the
// tensor-core pass's own, so a pair left out would have produced no item there.  About half the
// pairs of a 24^3 mesh (Gaussian width 0.38 rad/ps) have no triple in the window.
// The pairs of q0 block [q0_first, q0_first + n_q0) are read from the device offsets; slots
// i >= their count (up to nmax) get key nq too.  The count goes to *n_out for the host to check
// against nmax; no pair at or beyond `cap` (the list's size) is read.
__global__ void k_tc_keys(int nmax, int cap, int q0_first, int n_q0, int nq, const int* __restrict__ pairoff,
                          const int2* __restrict__ pairs, const int* __restrict__ pair_q0,
                          const double* __restrict__ om0, const double* __restrict__ omg, float rf,
                          int* __restrict__ keys, int* __restrict__ vals, int* __restrict__ cnt,
                          int* __restrict__ n_out) {
    const int p0 = pairoff[q0_first], n = pairoff[q0_first + n_q0] - p0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nmax; i += gridDim.x * blockDim.x) {
        if (i >= n || p0 + i >= cap) {
            keys[i] = nq;
            vals[i] = -1;
            continue;
        }
        const int2 pq = pairs[p0 + i];
        const double* w0d = om0 + (size_t)pair_q0[p0 + i] * NMODE;
        const double* w1d = omg + (size_t)pq.x * NMODE;
        const double* w2d = omg + (size_t)pq.y * NMODE;
        float w0[NMODE], w1[NMODE], w2[NMODE];
#pragma unroll
        for (int s = 0; s < NMODE; ++s) {
            w0[s] = (float)w0d[s];
            w1[s] = (float)w1d[s];
            w2[s] = (float)w2d[s];
        }
        bool any = false;
#pragma unroll
        for (int s0 = 0; s0 < NMODE; ++s0)
#pragma unroll
            for (int s2 = 0; s2 < NMODE; ++s2) {
                const float2 v = tc_window_vals(w0[s0], w2[s2]);
#pragma unroll
                for (int s1 = 0; s1 < NMODE; ++s1) any |= tc_window(v.x, v.y, w1[s1], rf);
            }
        keys[i] = any ? pq.x : nq;
        vals[i] = p0 + i;
        if (any) atomicAdd(&cnt[pq.x], 1);
    }
}
// Tiles (out[0]) and tiled pairs (out[2]) from the last entries of the exclusive scans.
__global__ void k_tc_totals(int nq, const int* __restrict__ toff, const int* __restrict__ ntl,
                            const int* __restrict__ seg, const int* __restrict__ cnt, int* __restrict__ out) {
    out[0] = toff[nq - 1] + ntl[nq - 1];
    out[2] = seg[nq - 1] + cnt[nq - 1];
}
__global__ void k_tc_ntiles(int nq, const int* __restrict__ cnt, int* __restrict__ nt) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x)
        nt[g] = (cnt[g] + EPT - 1) / EPT;
}
__global__ void k_tc_tiles(int nq, const int* __restrict__ cnt, const int* __restrict__ seg, const int* __restrict__ toff,
                           int4* __restrict__ tiles) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
        const int c = cnt[g];
        for (int t = 0; t * EPT < c; ++t) tiles[toff[g] + t] = make_int4(g, seg[g] + t * EPT, min(EPT, c - t * EPT), 0);
    }
}
// Entry records in q1 order: (q0, q2, pair-folding weight, q0 is Gamma); entries with key nq
// (outside the window or past the block's pairs, all after the tiled ones) are skipped.
__global__ void k_tc_entrec(int n, int nq, const int* __restrict__ entries, const int* __restrict__ keys_s,
                            const int2* __restrict__ pairs, const int* __restrict__ pair_q0,
                            const int* __restrict__ irr_int, int4* __restrict__ rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (keys_s[i] >= nq) continue;
        const int pi = entries[i];
        const int2 pq = pairs[pi];
        const int q0 = pair_q0[pi];
        const int g0 = irr_int[3 * q0] == 0 && irr_int[3 * q0 + 1] == 0 && irr_int[3 * q0 + 2] == 0;
        rec[i] = make_int4(q0, pq.y, pq.x != pq.y ? 2 : 1, g0);
    }
}

// ------------------------------------------------------------------ main kernels
struct TcArgs {
    int nq, nq0, nT, ntiles, tiles_per_cta, rs;
    int q0_first;            // first q0 of the block (operator rows are counted from it)
    long long bte_cap;       // operator entries the output holds (entry mode)
    int lo[3], hi[3];
    double half_os2, pre, mfac;
    float rf;             // delta window of the FP32 screen (tc_window)
    long long max_spins;  // poll limit of every wait of one warp on another (the pipeline waits)
};

constexpr int NOP = 2;  // operand stages (A and B images; free once the tile's MMAs completed)
constexpr int NEP = 4;  // epilogue stages (frequencies and one 128-column accumulator each)
static_assert(NOP <= NEP, "operand stages beyond the accumulator stages would wait on the epilogue anyway");

// An active mode triple, staged in shared memory by the epilogue warp that found it: |Phi|^2 in
// FP32, k0 = (q0 * 6 + s0) | (wt == 2) << 30 | (W = 0) << 29, k1 = q1 * 6 + s1, k2 = q2 * 6 + s2.
struct TcStage {
    float phi2;
    int k0, k1, k2;
};
constexpr int STG_CAP = 160;  // staged triples per epilogue warp: fewer than 64 left + up to 96 from one chunk

// One entry of the Gaussian iterative-BTE operator (row r0 = (q0 - q0_first) * 6 + s0, grid modes
// k1, k2; c = (n1 - n2) P + (1 + n1 + n2) Q), in the layout the operator sort reads.
struct TcBteEntry {
    int r0, k1, k2, pad;
    double P, Q;
};
static_assert(sizeof(TcBteEntry) == 32, "operator entry");

struct OpStage {
    alignas(128) uint8_t A[2][EPT * 1536];    // [hi, lo]: per pair its two mu images (pair stride 1536)
    alignas(128) uint8_t B[2 * 2 * B_BYTES];  // [hi, lo][mu]: rows (re/im, a, s1)
    int q1;                                   // q1 whose B images are resident
};
struct EpStage {
    alignas(128) Q0Rec q0r[EPT][NMODE];        // per pair its six q0 records (e0' only: 16-byte async copies)
    alignas(16) float2 cb[EPT][NMODE][NMODE];  // per pair, s2, s0: tc_window_vals of the FP32 omegas
    alignas(8) float w1s[NMODE];               // omega of q1 in FP32, s1 in slot order 0 3 1 4 2 5
    int4 ent[EPT];                             // (q0, q2, weight, q0 is Gamma)
    int q1, ne;
};
constexpr int EPI_WARPS = 12;      // warps 0-11: epilogue; warps w, w+4, w+8 share TMEM lanes, two s1 each
struct TcSmem {
    OpStage op[NOP];
    EpStage ep[NEP];
    alignas(16) TcStage stg[EPI_WARPS][STG_CAP];
    alignas(8) uint64_t ready[NEP], full[NEP], empty[NEP], opfree[NOP], opready[NOP];
    uint32_t tslot;
    int abort;  // set by any warp whose pipeline wait ran out
    int fdone;  // tiles the frequency warp filled (written when it leaves its loop)
};
static_assert(sizeof(TcSmem) <= 227 * 1024, "tensor-core V3 shared memory");

constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int TC_THREADS = EPI_THREADS + 96;  // warp 12: TMA copies; warp 13: MMA issue; warp 14: frequencies
constexpr int TC_COLS = NEP * 128;
constexpr int NT_FAST = 4;  // mode records of 8 doubles carry the occupations of up to 4 temperatures

// FP64 part of n <= 32 staged triples, one per lane: W = wt mfac |Phi|^2 / (omega0 omega1 omega2),
// the three Gaussian delta weights, then the phase-space and linewidth sums with atomics:
// P3 += wt (g1 + g2 + g3), Gamma_T += W [(n1 + n2 + 1) g1 + (n1 - n2)(g2 - g3)].  The q0 record
// (omega, 1/omega) and the mode records (omega, 1/omega, nBE[T]) of q1 and q2 are read whole, so
// a triple needs one memory round trip.  FAST: records of 8 doubles, n_temps <= 4.
// exp(-x) of the arguments below the cut (g = 0 for the others), each lane computing only its own:
// the warp runs as many exponentials as the lane that needs most (usually one of the three, the
// deltas of a triple being 2 omega1 or 2 omega2 apart).  One call site of exp.
__device__ __forceinline__ void tc_gauss3(double x1, double x2, double x3, double& g1, double& g2, double& g3) {
    unsigned need = (x1 < EXP_CUT ? 1u : 0u) | (x2 < EXP_CUT ? 2u : 0u) | (x3 < EXP_CUT ? 4u : 0u);
    g1 = g2 = g3 = 0.0;
    while (__any_sync(0xffffffffu, need != 0u)) {
        if (need != 0u) {
            const int k = __ffs(need) - 1;
            need &= need - 1u;
            const double g = exp(-(k == 0 ? x1 : (k == 1 ? x2 : x3)));
            if (k == 0) g1 = g;
            else if (k == 1) g2 = g;
            else g3 = g;
        }
    }
}

// One round of operator entries (iterative BTE): n <= 32 staged triples, one per lane.
__device__ __forceinline__ void tc_bte_round(const TcStage* st, int n, int rs, double half_os2, double pre, double mfac,
                                             const Q0Rec* __restrict__ q0rec, const double* __restrict__ modes,
                                             TcBteEntry* bte, unsigned long long* bte_ctr, long long bte_cap,
                                             int q0_first) {
    const int lane = threadIdx.x & 31;
    // operator entries: P = 4 W (g(w0 + w1 - w2) - g(w0 + w2 - w1)), Q = 4 W g(w0 - w1 - w2), the
    // second term of P dropped and Q halved when q1 = q2; one entry per triple with P or Q nonzero
    double Pv = 0.0, Qv = 0.0;
    TcStage s{};
    double xm = EXP_CUT, xa = EXP_CUT, xb = EXP_CUT, W = 0.0;  // EXP_CUT: no weight
    bool self = true;
    if (lane < n) {
        s = st[lane];
        const int o = s.k0 & 0x1fffffff;
        const double2 r0 = *reinterpret_cast<const double2*>(&q0rec[o].w);
        const double2 a = *reinterpret_cast<const double2*>(modes + (size_t)s.k1 * rs);
        const double2 b = *reinterpret_cast<const double2*>(modes + (size_t)s.k2 * rs);
        if (!((s.k0 >> 29) & 1)) {
            const double w0 = r0.x, w1 = a.x, w2 = b.x;
            const double dm = w0 - w1 - w2, da = w0 + w1 - w2, db = w0 - w1 + w2;
            xm = half_os2 * (dm * dm);
            xa = half_os2 * (da * da);
            xb = half_os2 * (db * db);
            self = !((s.k0 >> 30) & 1);
            if (self) xb = EXP_CUT;  // the second term of P is dropped when q1 = q2
            W = (double)s.phi2 * (r0.y * b.y * a.y) * mfac;
        }
    }
    double gm, ga, gb;
    tc_gauss3(xm, xa, xb, gm, ga, gb);
    if (W != 0.0) {
        const double em = xm < EXP_CUT ? pre * gm : 0.0;
        const double ea = xa < EXP_CUT ? pre * ga : 0.0;
        const double eb = xb < EXP_CUT ? pre * gb : 0.0;
        Pv = 4.0 * W * (ea - eb);
        Qv = 4.0 * W * (self ? 0.5 : 1.0) * em;
    }
    const bool has = Pv != 0.0 || Qv != 0.0;
    const unsigned bal = __ballot_sync(0xffffffffu, has);
    unsigned long long base = 0;
    if (lane == 0 && bal != 0u) base = atomicAdd(bte_ctr, (unsigned long long)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (has) {
        const unsigned long long pos = base + (unsigned long long)__popc(bal & ((1u << lane) - 1u));
        if ((long long)pos < bte_cap) {
            TcBteEntry e;
            e.r0 = (s.k0 & 0x1fffffff) - q0_first * NMODE;
            e.k1 = s.k1;
            e.k2 = s.k2;
            e.pad = 0;
            e.P = Pv;
            e.Q = Qv;
            bte[pos] = e;
        }
    }
    __syncwarp();
}

// One staged triple of the linewidth sums, loaded: its entry, the q0 record (omega, 1/omega), the mode
// records of q1 and q2 (omega, 1/omega, up to four occupations when FAST) and the three Gaussian
// arguments (EXP_CUT, no weight, for an empty slot).
struct TcEv {
    TcStage s;
    double2 r0, a, b, a1, a2, b1, b2;
    double x1, x2, x3;
};
template <bool FAST>
__device__ __forceinline__ void tc_ev_load(TcEv& v, const TcStage* st, int i, int n, int rs,
                                           const Q0Rec* __restrict__ q0rec, const double* __restrict__ modes) {
    v.x1 = v.x2 = v.x3 = EXP_CUT;
    if (i >= n) return;
    v.s = st[i];
    const int o = v.s.k0 & 0x1fffffff;
    v.r0 = *reinterpret_cast<const double2*>(&q0rec[o].w);
    const double2* pa = reinterpret_cast<const double2*>(modes + (size_t)v.s.k1 * rs);
    const double2* pb = reinterpret_cast<const double2*>(modes + (size_t)v.s.k2 * rs);
    v.a = pa[0];
    v.b = pb[0];
    if (FAST) {
        v.a1 = pa[1];
        v.a2 = pa[2];
        v.b1 = pb[1];
        v.b2 = pb[2];
    }
}
__device__ __forceinline__ void tc_ev_args(TcEv& v, int i, int n, double half_os2) {
    if (i >= n) return;
    const double w0 = v.r0.x, w1 = v.a.x, w2 = v.b.x;
    const double d1 = w0 - w1 - w2, d2 = w0 + w1 - w2, d3 = w0 - w1 + w2;
    v.x1 = half_os2 * (d1 * d1);
    v.x2 = half_os2 * (d2 * d2);
    v.x3 = half_os2 * (d3 * d3);
}
template <bool FAST>
__device__ __forceinline__ void tc_ev_sum(const TcEv& v, double g1, double g2, double g3, int nq0, int nT, int rs,
                                          double pre, double mfac, const double* __restrict__ modes, double* out_lw,
                                          double* out_p3) {
    const TcStage& s = v.s;
    const int o = s.k0 & 0x1fffffff;
    const double e1 = v.x1 < EXP_CUT ? pre * g1 : 0.0;
    const double e2 = v.x2 < EXP_CUT ? pre * g2 : 0.0;
    const double e3 = v.x3 < EXP_CUT ? pre * g3 : 0.0;
    const double wt = (s.k0 >> 30) & 1 ? 2.0 : 1.0;
    const double p3 = e1 + e2 + e3;
    if (p3 != 0.0) atomicAdd(&out_p3[o], wt * p3);
    if ((s.k0 >> 29) & 1) return;  // W = 0 for the Gamma acoustic modes of q0
    const double W = (double)s.phi2 * (v.r0.y * v.b.y * v.a.y) * mfac * wt;
    const double we1 = W * e1, wf2 = W * (e2 - e3);
    if (FAST) {
        const double n1[NT_FAST] = {v.a1.x, v.a1.y, v.a2.x, v.a2.y}, n2[NT_FAST] = {v.b1.x, v.b1.y, v.b2.x, v.b2.y};
#pragma unroll
        for (int T = 0; T < NT_FAST; ++T)
            if (T < nT) {
                const double x = ((n1[T] + n2[T] + 1.0) * we1) + ((n1[T] - n2[T]) * wf2);
                if (x != 0.0) atomicAdd(&out_lw[(size_t)T * nq0 * NMODE + o], x);
            }
    } else {
        const double* m1 = modes + (size_t)s.k1 * rs + 2;
        const double* m2 = modes + (size_t)s.k2 * rs + 2;
        for (int T = 0; T < nT; ++T) {
            const double x = ((m1[T] + m2[T] + 1.0) * we1) + ((m1[T] - m2[T]) * wf2);
            if (x != 0.0) atomicAdd(&out_lw[(size_t)T * nq0 * NMODE + o], x);
        }
    }
}

// FP64 part of n <= 64 staged triples, entries lane and lane + 32 of each lane (the loads of both
// issued before either is evaluated): MODE 0 the linewidth and phase-space sums, W = wt mfac
// |Phi|^2 / (omega0 omega1 omega2), P3 += wt (g1 + g2 + g3), Gamma_T += W [(n1 + n2 + 1) g1 +
// (n1 - n2)(g2 - g3)] with atomics; MODE 1 operator entries.  FAST: mode records of 8 doubles,
// n_temps <= 4.
template <bool FAST, int MODE>
__device__ __forceinline__ void tc_drain(const TcStage* st, int n, int nq0, int nT, int rs, double half_os2, double pre,
                                         double mfac, const Q0Rec* __restrict__ q0rec, const double* __restrict__ modes,
                                         double* out_lw, double* out_p3, TcBteEntry* bte, unsigned long long* bte_ctr,
                                         long long bte_cap, int q0_first) {
    const int lane = threadIdx.x & 31;
    if (MODE == 1) {
        tc_bte_round(st, min(n, 32), rs, half_os2, pre, mfac, q0rec, modes, bte, bte_ctr, bte_cap, q0_first);
        if (n > 32)
            tc_bte_round(st + 32, n - 32, rs, half_os2, pre, mfac, q0rec, modes, bte, bte_ctr, bte_cap, q0_first);
        return;
    }
    TcEv v0, v1;
    tc_ev_load<FAST>(v0, st, lane, n, rs, q0rec, modes);
    tc_ev_load<FAST>(v1, st, lane + 32, n, rs, q0rec, modes);
    tc_ev_args(v0, lane, n, half_os2);
    tc_ev_args(v1, lane + 32, n, half_os2);
    double g1, g2, g3;
    tc_gauss3(v0.x1, v0.x2, v0.x3, g1, g2, g3);
    if (lane < n) tc_ev_sum<FAST>(v0, g1, g2, g3, nq0, nT, rs, pre, mfac, modes, out_lw, out_p3);
    if (__any_sync(0xffffffffu, lane + 32 < n)) {
        tc_gauss3(v1.x1, v1.x2, v1.x3, g1, g2, g3);
        if (lane + 32 < n) tc_ev_sum<FAST>(v1, g1, g2, g3, nq0, nT, rs, pre, mfac, modes, out_lw, out_p3);
    }
    __syncwarp();  // every lane has read its entries before the warp stages new ones over them
}

// Warp-specialised tensor-core pass.  For tile j the copy warp loads operand stage j % 2 (TMA
// gathers of the A images, four pairs' table rows per request, hi and lo parts as separate
// requests; one bulk copy of the B images when q1 changed), completing on opready[j % 2], and the
// frequency warp epilogue stage j % 4 (entry records and the tile's omegas, plain loads issued one
// tile ahead; the pairs' e0' as asynchronous copies), completing on ready[j % 4].  The MMA warp
// issues tile j's MMAs once its operands landed and the epilogue released accumulator j % 4
// (empty), and commits them to full[j % 4] and opfree[j % 2]: the frequency warp's fill is off the
// operand loop (copy -> MMA -> opfree -> copy), which runs two tiles deep.  Each
// epilogue warp works on its own: it reads its 32 accumulator rows, screens its 12 mode triples per
// row in FP32 against the delta window, forms |Phi|^2 of the active ones (about 1-3 %) from the
// stage's q0 records, stages them in its shared-memory buffer, releases the stage, and evaluates
// the FP64 delta weights and sums of the staged triples 64 at a time, two per lane (tc_drain).
// MODE 0: linewidth and phase-space sums; MODE 1: entries of the iterative-BTE operator.
template <bool SPLIT, bool FAST, int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1)
k_v3tc(TcArgs a, const __grid_constant__ CUtensorMap tmA, const int4* __restrict__ tiles, const int4* __restrict__ entrec,
       const __nv_bfloat16* __restrict__ tabB, const double* __restrict__ om0, const double* __restrict__ omg,
       const Q0Rec* __restrict__ q0rec, const double* __restrict__ modes, double* __restrict__ out_lw,
       double* __restrict__ out_p3, TcBteEntry* __restrict__ bte, unsigned long long* __restrict__ bte_ctr,
       int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smraw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int H = SPLIT ? 2 : 1;
    constexpr int PB = 1536;  // pair stride of the A images = their 8-row group stride
    const int t0 = blockIdx.x * a.tiles_per_cta;
    const int t1 = min(a.ntiles, t0 + a.tiles_per_cta);
    const int nt = t1 - t0;
    if ((tc::smem_u32(smraw) & 127u) != 0u) {  // TMA destinations below assume a 128-byte aligned base
        if (tid == 0) atomicExch(err, 2);
        return;
    }

    if (tid == 0) {
        S.abort = 0;
        S.fdone = 0;
        for (int k = 0; k < NOP; ++k) {
            S.op[k].q1 = -1;
            tc::mbar_init(tc::smem_u32(&S.opfree[k]), 1);
            tc::mbar_init(tc::smem_u32(&S.opready[k]), 32);  // copy-warp lanes (and the copies' bytes)
        }
        for (int k = 0; k < NEP; ++k) {
            tc::mbar_init(tc::smem_u32(&S.ready[k]), 64);  // frequency-warp lanes and their copies
            tc::mbar_init(tc::smem_u32(&S.full[k]), 1);
            tc::mbar_init(tc::smem_u32(&S.empty[k]), EPI_WARPS);
        }
        tc::mbar_fence_init();
    }
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tslot), TC_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = S.tslot;
    int filled = -1;  // copy warp: last tile whose operand copies were issued

    if (warp == EPI_WARPS) {
        // ------------------------------------------------------------ copy warp
        // Operand stage j % 2 for tile j, after the MMAs of tile j-2 released it (so the previous
        // phase of opready[j % 2] has completed): TMA gathers of the A images and, when q1 changed,
        // the B images; each issuing lane adds its own bytes to opready before its copy, then every
        // lane arrives.  Tile and entry records are loaded ahead into registers.
        const int4 z4 = make_int4(0, 0, 0, 0);
        int4 recA = nt > 0 ? tiles[t0] : z4, recB = nt > 1 ? tiles[t0 + 1] : z4;
        int4 entA = lane < recA.z ? entrec[recA.y + lane] : z4;
        for (int j = 0; j < nt; ++j) {
            const int os = j % NOP;
            const bool ok = j < NOP || tc::mbar_wait(tc::smem_u32(&S.opfree[os]), (uint32_t)(((j - NOP) / NOP) & 1),
                                                     a.max_spins);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    *(volatile int*)&S.abort = 1;
                }
                break;
            }
            OpStage& O = S.op[os];
            const int q1 = recA.x, ne = recA.z;
            // lane l < 4 H gathers group g = l / H (pairs 4g .. 4g+3, beyond ne repeating pair 0),
            // part l % H; lane 31 copies the B images when q1 changed.
            const int g = (lane / H) & 3, part = lane % H;
            int rows[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) rows[k] = __shfl_sync(0xffffffffu, entA.y, 4 * g + k < ne ? 4 * g + k : 0);
            const uint32_t rb = tc::smem_u32(&S.opready[os]);
            if (lane < 4 * H && 4 * g < ne) {
                tc::mbar_expect_tx(rb, 4u * PB);
                tc::gather4_g2s(tc::smem_u32(&O.A[part][g * 4 * PB]), &tmA, part * (PB / 8), rows[0], rows[1], rows[2],
                                rows[3], rb);
            }
            if (lane == 31 && O.q1 != q1) {
                O.q1 = q1;
                tc::mbar_expect_tx(rb, (uint32_t)(2 * H * B_BYTES));
                tc::bulk_g2s(tc::smem_u32(&O.B[0]), tabB + (size_t)q1 * 4 * BIMG, (uint32_t)(2 * H * B_BYTES), rb);
            }
            tc::mbar_arrive(rb);
            filled = j;
            const int4 entB = (j + 1 < nt && lane < recB.z) ? entrec[recB.y + lane] : z4;
            const int4 recC = j + 2 < nt ? tiles[t0 + j + 2] : z4;
            recA = recB;
            recB = recC;
            entA = entB;
        }
    } else if (warp == EPI_WARPS + 2) {
        // ------------------------------------------------------------ frequency warp
        // Epilogue stage j % 4 for tile j, after the epilogue of tile j-4 released it: entry
        // records, the pairs' e0' (lane l copies those of pair l % 16 for s0 = 3 (l / 16) .. + 2 as
        // nine 16-byte asynchronous copies), the q1 omegas and, per pair, s2 and s0, the window
        // values (w0 - w2, w0 + w2) of the FP32 screen.  Lane l prepares pair l % 16 for s2 = 3 (l / 16)
        // .. 3 (l / 16) + 2 from omegas loaded during the fill of tile j-1; no warp barrier follows
        // a load: each lane arrives on ready itself, after its own stores and before it issues new
        // loads, and once more when its copies have landed.
        const int4 z4 = make_int4(0, 0, 0, 0);
        int4 recA = nt > 0 ? tiles[t0] : z4, recB = nt > 1 ? tiles[t0 + 1] : z4, recC = nt > 2 ? tiles[t0 + 2] : z4;
        int4 entA = lane < recA.z ? entrec[recA.y + lane] : z4;
        int4 entB = lane < recB.z ? entrec[recB.y + lane] : z4;
        double2 w0v[3], wq1[3];
        double w2v[3];
        const int pw = lane & 15, hw = lane >> 4;
        auto load_w = [&](const int4& ent, const int4& rec) {
            const int q0 = __shfl_sync(0xffffffffu, ent.x, pw);
            const int q2 = __shfl_sync(0xffffffffu, ent.y, pw);
            if (pw < rec.z) {
                const double2* src = reinterpret_cast<const double2*>(om0 + (size_t)q0 * NMODE);
                w0v[0] = src[0];
                w0v[1] = src[1];
                w0v[2] = src[2];
                const double* s2p = omg + (size_t)q2 * NMODE + 3 * hw;
                w2v[0] = s2p[0];
                w2v[1] = s2p[1];
                w2v[2] = s2p[2];
            }
            if (lane == 0) {
                const double2* src = reinterpret_cast<const double2*>(omg + (size_t)rec.x * NMODE);
                wq1[0] = src[0];
                wq1[1] = src[1];
                wq1[2] = src[2];
            }
        };
        if (nt > 0) load_w(entA, recA);
        int j = 0;
        for (; j < nt; ++j) {
            const int es = j % NEP;
            const bool ok = j < NEP || tc::mbar_wait(tc::smem_u32(&S.empty[es]), (uint32_t)(((j - NEP) / NEP) & 1),
                                                     a.max_spins);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    *(volatile int*)&S.abort = 1;
                }
                break;
            }
            EpStage& E = S.ep[es];
            const int q1 = recA.x, ne = recA.z;
            const uint32_t rb = tc::smem_u32(&S.ready[es]);
            {
                const int q0p = __shfl_sync(0xffffffffu, entA.x, pw);
                if (pw < ne) {
                    const char* src = reinterpret_cast<const char*>(q0rec + (size_t)q0p * NMODE + 3 * hw);
                    const uint32_t dst = tc::smem_u32(&E.q0r[pw][3 * hw]);
#pragma unroll
                    for (int k = 0; k < 9; ++k)  // e0' of three s0: 48 of each record's 64 bytes
                        tc::cp_async16(dst + (k / 3) * 64 + (k % 3) * 16, src + (k / 3) * 64 + (k % 3) * 16);
                }
            }
            if (lane == 0) {
                E.ne = ne;
                E.q1 = q1;
                const double w1[NMODE] = {wq1[0].x, wq1[0].y, wq1[1].x, wq1[1].y, wq1[2].x, wq1[2].y};
#pragma unroll
                for (int s1 = 0; s1 < NMODE; ++s1) E.w1s[b_slot(s1)] = (float)w1[s1];
            }
            if (lane < ne) E.ent[lane] = entA;
            if (pw < ne) {
                const float w0[NMODE] = {(float)w0v[0].x, (float)w0v[0].y, (float)w0v[1].x,
                                         (float)w0v[1].y, (float)w0v[2].x, (float)w0v[2].y};
                float4* d = reinterpret_cast<float4*>(&E.cb[pw][3 * hw][0]);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const float w2 = (float)w2v[i];
#pragma unroll
                    for (int s0 = 0; s0 < NMODE; s0 += 2) {
                        const float2 u = tc_window_vals(w0[s0], w2), v = tc_window_vals(w0[s0 + 1], w2);
                        d[i * 3 + s0 / 2] = make_float4(u.x, u.y, v.x, v.y);
                    }
                }
            }
            tc::mbar_arrive(rb);           // each lane releases its own stores
            tc::cp_async_mbar_arrive(rb);  // and, once they land, its copies
            // loads for later fills
            if (j + 1 < nt) load_w(entB, recB);
            const int4 entC = (j + 2 < nt && lane < recC.z) ? entrec[recC.y + lane] : z4;
            const int4 recD = j + 3 < nt ? tiles[t0 + j + 3] : z4;
            recA = recB;
            recB = recC;
            recC = recD;
            entA = entB;
            entB = entC;
        }
        if (lane == 0) S.fdone = j;
    } else if (warp == EPI_WARPS + 1) {
        // ------------------------------------------------------------ MMA warp
        // Tile j's MMAs once the epilogue has drained its accumulator (tile j-4, empty) and its
        // operands have landed (opready); its operands stay until the commit to opfree.
        int issued = -1;
        if (lane == 0) {
            for (int j = 0; j < nt; ++j) {
                const int es = j % NEP, os = j % NOP;
                const bool acc_free = j < NEP || tc::mbar_wait(tc::smem_u32(&S.empty[es]),
                                                               (uint32_t)(((j - NEP) / NEP) & 1), a.max_spins);
                if (!acc_free || !tc::mbar_wait(tc::smem_u32(&S.opready[os]), (uint32_t)((j / NOP) & 1), a.max_spins)) {
                    atomicExch(err, 1);
                    *(volatile int*)&S.abort = 1;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t idesc = tc::idesc_bf16(128, 48);
                const uint32_t pa = tc::smem_u32(&S.op[os].A[0][0]), pl = tc::smem_u32(&S.op[os].A[1][0]);
                const uint32_t pb = tc::smem_u32(&S.op[os].B[0]);
#pragma unroll
                for (int mu = 0; mu < 2; ++mu) {
                    const uint32_t d = tm + (uint32_t)(es * 128 + mu * 64);
#pragma unroll
                    for (int kk = 0; kk < KP / 16; ++kk) {
                        const uint32_t ko = (uint32_t)kk * 2u * LBO;
                        const uint64_t ah = tc::sdesc(pa + mu * 768 + ko, LBO, PB);
                        const uint64_t bh = tc::sdesc(pb + mu * B_BYTES + ko, LBO, SBO);
                        tc::mma_bf16(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                        if (SPLIT) {
                            const uint64_t al = tc::sdesc(pl + mu * 768 + ko, LBO, PB);
                            const uint64_t bl = tc::sdesc(pb + (2 + mu) * B_BYTES + ko, LBO, SBO);
                            tc::mma_bf16(d, ah, bl, idesc, 1u);
                            tc::mma_bf16(d, al, bh, idesc, 1u);
                        }
                    }
                }
                tc::mma_commit(tc::smem_u32(&S.full[es]));
                tc::mma_commit(tc::smem_u32(&S.opfree[os]));
                issued = j;
            }
            // the last commit tracks every MMA issued: wait (bounded) before TMEM is released
            if (issued >= 0)
                tc::mbar_wait(tc::smem_u32(&S.full[issued % NEP]), (uint32_t)((issued / NEP) & 1), MAX_SPINS);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue warps
        // Warp (wq, g): TMEM lanes 32 wq .. 32 wq + 31 (pairs 4 wq .. 4 wq + 3, s2 = lane % 8), the
        // q1 branches s1 = g and g + 3 (accumulator columns 16 g .. 16 g + 15 of each mu) and every
        // s0; slot bit 6 sl + s0 stands for (s0, s1 = g + 3 sl).  One acoustic and one optical s1
        // per warp keeps the active triples even across the three warps of a lane quarter.
        const int wq = warp & 3, g = warp >> 2;
        const int e = 4 * wq + lane / 8, s2 = lane % 8, s2c = s2 < NMODE ? s2 : 0;
        TcStage* stg = S.stg[warp];
        int count = 0;  // staged triples (warp-uniform); fewer than 64 between tiles
        // slots allowed by the mode ranges, and by the Gamma acoustic rule when q1 = Gamma (amask_g:
        // s1 = g < 3 drops out)
        unsigned amask_n = 0u;
#pragma unroll
        for (int sl = 0; sl < 2; ++sl) {
            const int s1 = g + 3 * sl;
#pragma unroll
            for (int s0 = 0; s0 < NMODE; ++s0)
                if (s1 >= a.lo[1] && s1 <= a.hi[1] && s0 >= a.lo[0] && s0 <= a.hi[0]) amask_n |= 1u << (6 * sl + s0);
        }
        const unsigned amask_g = amask_n & ~0x3fu;
        const unsigned lt = (1u << lane) - 1u;
        for (int j = 0; j < nt; ++j) {
            const int es = j % NEP, u = j / NEP;
            const EpStage& E = S.ep[es];
            const bool ok = tc::mbar_wait(tc::smem_u32(&S.ready[es]), (uint32_t)(u & 1), a.max_spins) &&
                            tc::mbar_wait(tc::smem_u32(&S.full[es]), (uint32_t)(u & 1), a.max_spins);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    *(volatile int*)&S.abort = 1;
                }
                break;
            }
            tc::fence_after_sync();
            float y[2][16];  // per mu, this row's Y for s1 = g (columns 0-7) and g + 3 (8-15): Re a, Im a, 0, 0
            const uint32_t ta = tm + ((uint32_t)(wq * 32) << 16) + (uint32_t)(es * 128 + 16 * g);
            tc::tmem_ld16(ta, y[0]);
            tc::tmem_ld16(ta + 64, y[1]);
            // The window screen and the item positions need only the stage's shared-memory records:
            // they run while the accumulator loads are in flight.
            const int ne = E.ne, q1 = E.q1;
            const int4 en = E.ent[e];
            const float4* cbp = reinterpret_cast<const float4*>(&E.cb[e][s2c][0]);
            const float4 c01 = cbp[0], c23 = cbp[1], c45 = cbp[2];
            const float2 w1 = *reinterpret_cast<const float2*>(&E.w1s[2 * g]);
            const bool row_on = s2 < NMODE && e < ne && s2 >= a.lo[2] && s2 <= a.hi[2] && !(en.y == 0 && s2 < 3);
            const unsigned amask = q1 == 0 ? amask_g : amask_n;
            unsigned act = 0u;
            if (row_on) {
                const float cc[NMODE] = {c01.x, c01.z, c23.x, c23.z, c45.x, c45.z};
                const float bb[NMODE] = {c01.y, c01.w, c23.y, c23.w, c45.y, c45.w};
#pragma unroll
                for (int s0 = 0; s0 < NMODE; ++s0) {
                    act |= tc_window(cc[s0], bb[s0], w1.x, a.rf) ? (1u << s0) : 0u;
                    act |= tc_window(cc[s0], bb[s0], w1.y, a.rf) ? (1u << (6 + s0)) : 0u;
                }
                act &= amask;
            }
            // Stage the active triples: positions from four bit-plane ballots of the lanes' counts
            // (at most 12), then each lane writes its own, |Phi|^2 = |sum_k e0'(k, s0) Y_k|^2 in FP32
            // from the stage's q0 record of the lane's pair (the two basis atoms' terms summed
            // separately).  When the tile's triples would not fit beside those left from earlier
            // tiles (fewer than 64; rare), they go in four chunks of at most 3 per lane, each after
            // full rounds are evaluated to make room.
            const int kw = en.z == 2 ? (1 << 30) : 0;
            const int k0b = en.x * NMODE, k2 = en.y * NMODE + s2;
            const bool g0 = en.w != 0;
            const Q0Rec* qr = E.q0r[e];
            auto stage_bits = [&](unsigned m, int pos) {
                while (m != 0u) {
                    const int bit = __ffs(m) - 1;  // bit 6 sl + s0
                    m &= m - 1u;
                    const int sl = bit >= NMODE ? 1 : 0, s0 = bit - NMODE * sl;
                    const float4* cq = reinterpret_cast<const float4*>(qr[s0].e0);
                    const float4 c01 = cq[0], c23 = cq[1], c45 = cq[2];
                    const float cx[NMODE] = {c01.x, c01.z, c23.x, c23.z, c45.x, c45.z};
                    const float cy[NMODE] = {c01.y, c01.w, c23.y, c23.w, c45.y, c45.w};
                    float pr[2] = {0.0f, 0.0f}, pim[2] = {0.0f, 0.0f};
#pragma unroll
                    for (int k = 0; k < NMODE; ++k) {
                        const int mu = k / 3, al = k % 3;
                        const float yr = sl ? y[mu][8 + al] : y[mu][al], yi = sl ? y[mu][11 + al] : y[mu][3 + al];
                        pr[mu] = fmaf(cx[k], yr, fmaf(-cy[k], yi, pr[mu]));
                        pim[mu] = fmaf(cx[k], yi, fmaf(cy[k], yr, pim[mu]));
                    }
                    const float p = pr[0] + pr[1], q = pim[0] + pim[1];
                    const int k0 = (k0b + s0) | kw | (g0 && s0 < 3 ? (1 << 29) : 0);
                    stg[pos++] = TcStage{p * p + q * q, k0, q1 * NMODE + g + 3 * sl, k2};
                }
            };
            const int cnt = __popc(act);
            int pre = 0, tot = 0;
#pragma unroll
            for (int bp = 0; bp < 4; ++bp) {
                const unsigned bal = __ballot_sync(0xffffffffu, (cnt >> bp) & 1);
                pre += __popc(bal & lt) << bp;
                tot += __popc(bal) << bp;
            }
            tc::tmem_ld_wait();
            tc::tmem_regs_ready<16>(y[0]);
            tc::tmem_regs_ready<16>(y[1]);
            if (count + tot <= STG_CAP) {
                stage_bits(act, count + pre);
                count += tot;
            } else {
#pragma unroll 1
                for (int c = 0; c < 4; ++c) {
                    const unsigned m = act & (7u << (3 * c));
                    const int cm = __popc(m);
                    const unsigned b0 = __ballot_sync(0xffffffffu, cm & 1), b1 = __ballot_sync(0xffffffffu, cm & 2);
                    const int nc = __popc(b0) + 2 * __popc(b1);
                    while (count + nc > STG_CAP) {
                        count -= 32;
                        tc_drain<FAST, MODE>(stg + count, 32, a.nq0, a.nT, a.rs, a.half_os2, a.pre, a.mfac, q0rec, modes,
                                       out_lw, out_p3, bte, bte_ctr, a.bte_cap, a.q0_first);
                    }
                    stage_bits(m, count + __popc(b0 & lt) + 2 * __popc(b1 & lt));
                    count += nc;
                    __syncwarp();
                }
            }
            // every read of the stage is done: release it, then evaluate full rounds
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(tc::smem_u32(&S.empty[es]));
            while (count >= 64) {
                count -= 64;
                tc_drain<FAST, MODE>(stg + count, 64, a.nq0, a.nT, a.rs, a.half_os2, a.pre, a.mfac, q0rec, modes, out_lw,
                               out_p3, bte, bte_ctr, a.bte_cap, a.q0_first);
            }
        }
        if (count > 0)
            tc_drain<FAST, MODE>(stg, count, a.nq0, a.nT, a.rs, a.half_os2, a.pre, a.mfac, q0rec, modes, out_lw, out_p3, bte, bte_ctr, a.bte_cap, a.q0_first);
    }
    // Every role has left its loop (each of its waits is bounded).  After a time-out copies may be
    // in flight into shared memory, unconsumed: the copy warp's operand copies of up to NOP tiles
    // (a copy of tile t is only issued once the MMAs of tile t - NOP completed, so those tiles are
    // filled - NOP + 1 .. filled) and the frequency warp's e0' copies of up to NEP tiles (a fill of
    // tile t follows the epilogue of tile t - NEP, so those tiles are fdone - NEP .. fdone - 1).
    // Every such phase completes by itself once its copies land (each filling lane arrived, its
    // copies' arrivals are asynchronous): the copy warp waits for them before the CTA releases its
    // shared memory.  The MMA warp already waited for its last commit, so no MMA writes tensor memory
    // after the release below.
    tc::fence_before_sync();
    __syncthreads();
    if (warp == EPI_WARPS && lane == 0 && *(volatile int*)&S.abort) {
        for (int t = max(0, filled - NOP + 1); t <= filled; ++t)
            tc::mbar_wait(tc::smem_u32(&S.opready[t % NOP]), (uint32_t)((t / NOP) & 1), MAX_SPINS);
        const int fd = S.fdone;
        for (int t = max(0, fd - NEP); t < fd; ++t)
            tc::mbar_wait(tc::smem_u32(&S.ready[t % NEP]), (uint32_t)((t / NEP) & 1), MAX_SPINS);
    }
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tm, TC_COLS);
}

// Tensor map of the A table as a 2-D array of 8-byte elements: rows = grid points, 384 columns
// (the [hi, lo][mu] images of one point, 3072 bytes), box 192 x 1 (one part of one row).
int make_tmap_a(spring_ctx* c, CUtensorMap* tm) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return fail(c, SPRING_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<Encode>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)(4 * AIMG / 4), (cuuint64_t)c->nq};
    const cuuint64_t strides[1] = {(cuuint64_t)(4 * AIMG * 2)};
    const cuuint32_t box[2] = {(cuuint32_t)(2 * AIMG * 2 / 8), 1u};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, c->d_tc_a.p, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, SPRING_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SPRING_OK;
}

// The q0 set a pass runs over: its pairs, its q0 phonons ([q0][s] and [q0][s][row]) and integer
// coordinates, and a tag for the tile cache (0: the irreducible set, 1: the time-reversal set).
struct TcQ0 {
    const PairSet* ps;
    const double2* ev0;
    const double* om0;
    const double* ob0;
    const int* q0_int;
    int nq0, set;
};
TcQ0 irr_src(spring_ctx* c) {
    return TcQ0{&c->ps_irr, c->ph_irr.evec.p, c->ph_irr.omega.p, c->ph_irr.oneby.p, c->d_irr_int.p, c->nq0, 0};
}

template <bool SPLIT, bool FAST, int MODE>
int launch_tc(spring_ctx* c, TcArgs& a, const TcQ0& src, double* d_lw, double* d_p3, TcBteEntry* bte,
              unsigned long long* bte_ctr) {
    const size_t smem = sizeof(TcSmem);
    alignas(64) CUtensorMap tmA;
    SPRING_CHECK(make_tmap_a(c, &tmA));
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "tensor-core V3 needs %zu bytes of shared memory", smem);
    cudaFuncSetAttribute(k_v3tc<SPLIT, FAST, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc: injected launch failure");
    k_v3tc<SPLIT, FAST, MODE><<<c->tc_grid, TC_THREADS, smem, c->stream>>>(
        a, tmA, c->d_tc_tiles.p, c->d_tc_rec.p, reinterpret_cast<const __nv_bfloat16*>(c->d_tc_b.p), src.om0,
        c->ph_grid.omega.p, reinterpret_cast<const Q0Rec*>(c->d_tc_q0.p), c->d_tc_modes.p, d_lw, d_p3, bte, bte_ctr,
        c->d_tc_cnt_cta.p);
    return launch_check(c, SPLIT ? "k_v3tc<bf16x3>" : "k_v3tc<bf16>");
}

// Pairs of q0 block [q0, q0 + n0) with a mode triple inside the delta window `rf`, sorted by q1
// (stable radix sort over nmax >= their count slots), cut into tiles of at most EPT pairs of one
// q1, with the entry record of every sorted pair.  Cached until the pair list, the phonons or the
// window change.  build_tiles_begin queues the keys,
// the sort, the tile counts and an asynchronous readback of their total (c->tc_pending);
// build_tiles_end waits for it and cuts the tiles, so that work queued between the two (the
// operand tables) runs while the host waits.
int build_tiles_begin(spring_ctx* c, const TcQ0& src, int q0, int n0, int nmax, float rf) {
    const PairSet& ps = *src.ps;
    c->tc_pending = false;
    if (c->tc_set == src.set && c->tc_gen == ps.gen && c->tc_q0 == q0 && c->tc_n0 == n0 && c->tc_ph_gen == c->ph_gen &&
        c->tc_rf == rf)
        return SPRING_OK;
    c->tc_gen = -1;  // no valid tiles until build_tiles_end has cut them
    const int n = nmax, nq = c->nq;
    DBuf<int>&keys = c->d_tc_keys, &keys_s = c->d_tc_keys_s, &vals = c->d_tc_vals, &cnt = c->d_tc_cnt,
              &seg = c->d_tc_seg, &ntl = c->d_tc_ntl, &toff = c->d_tc_toff;
    int rc = SPRING_OK;
    auto step = [&](int r) { if (rc == SPRING_OK) rc = r; };
    step(dalloc(c, keys, std::max(n, 1), "tile keys"));
    step(dalloc(c, keys_s, std::max(n, 1), "tile keys"));
    step(dalloc(c, vals, std::max(n, 1), "tile values"));
    step(dalloc(c, c->d_tc_entries, std::max(n, 1), "tile entries"));
    step(dalloc(c, c->d_tc_rec, std::max(n, 1), "entry records"));
    step(dalloc(c, cnt, nq, "tile counts"));
    step(dalloc(c, seg, nq, "tile segments"));
    step(dalloc(c, ntl, nq, "tile counts"));
    step(dalloc(c, toff, nq, "tile offsets"));
    step(dalloc(c, c->d_scr_sum, 3, "tile and pair counts"));
    if (rc == SPRING_OK) rc = zero(c, cnt.p, sizeof(int) * nq, "tile counts");
    if (rc == SPRING_OK) rc = zero(c, c->d_scr_sum.p, 3 * sizeof(int), "tile and pair counts");
    const int threads = 256;
    if (rc == SPRING_OK && n > 0) {
        if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "tiles: injected launch failure");
        else {
            k_tc_keys<<<std::min((n + threads - 1) / threads, 148 * 8), threads, 0, c->stream>>>(
                n, ps.cap, q0, n0, nq, ps.pairoff.p, ps.pairs.p, ps.pair_q0.p, src.om0, c->ph_grid.omega.p,
                rf, keys.p, vals.p, cnt.p, c->d_scr_sum.p + 1);
            rc = launch_check(c, "k_tc_keys");
        }
    }
    int bits = 1;
    while ((1 << bits) <= nq) ++bits;  // keys run to nq (pairs outside the window)
    if (rc == SPRING_OK && n > 0) {
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, keys_s.p, vals.p, c->d_tc_entries.p, n, 0, bits, c->stream);
        DBuf<uint8_t>& tmp = c->d_tc_sort;
        rc = dalloc(c, tmp, std::max<size_t>(bytes, 1), "sort scratch");
        if (rc == SPRING_OK) {
            cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keys.p, keys_s.p, vals.p, c->d_tc_entries.p, n,
                                                            0, bits, c->stream);
            c->launches += 1;
            if (e != cudaSuccess) rc = cuda_fail(c, e, "pair sort");
        }
    }
    if (rc == SPRING_OK) rc = run_exclusive_scan(c, cnt.p, seg.p, nq);
    if (rc == SPRING_OK) {
        if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "tiles: injected launch failure");
        else {
            k_tc_ntiles<<<(nq + threads - 1) / threads, threads, 0, c->stream>>>(nq, cnt.p, ntl.p);
            rc = launch_check(c, "k_tc_ntiles");
        }
    }
    if (rc == SPRING_OK) rc = run_exclusive_scan(c, ntl.p, toff.p, nq);
    if (rc == SPRING_OK) {
        k_tc_totals<<<1, 1, 0, c->stream>>>(nq, toff.p, ntl.p, seg.p, cnt.p, c->d_scr_sum.p);
        rc = launch_check(c, "k_tc_totals");
    }
    if (rc == SPRING_OK) rc = d2h_pin_async(c, c->d_scr_sum.p, 3 * sizeof(int), "tile and pair counts");
    if (rc != SPRING_OK) return rc;
    c->tc_pending = true;
    c->tc_set = src.set;
    c->tc_q0 = q0;
    c->tc_n0 = n0;
    c->tc_nmax = nmax;
    c->tc_rf = rf;
    return SPRING_OK;
}

int build_tiles_end(spring_ctx* c, const TcQ0& src) {
    if (!c->tc_pending) return SPRING_OK;
    c->tc_pending = false;
    const PairSet& ps = *src.ps;
    const int n = c->tc_nmax, nq = c->nq;
    DBuf<int>&cnt = c->d_tc_cnt, &seg = c->d_tc_seg, &toff = c->d_tc_toff;
    const int threads = 256;
    int rc = pin_wait(c, "tile count");
    const int ntiles = rc == SPRING_OK ? c->h_pin[0] : 0;
    if (rc == SPRING_OK && c->h_pin[1] > n)
        rc = fail(c, SPRING_ERR_CUDA, "tiles: %d pairs in the q0 block exceed the %d slots", c->h_pin[1], n);
    if (rc == SPRING_OK) rc = dalloc(c, c->d_tc_tiles, std::max(ntiles, 1), "tiles");
    if (rc == SPRING_OK) {
        if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "tiles: injected launch failure");
        else {
            k_tc_tiles<<<(nq + threads - 1) / threads, threads, 0, c->stream>>>(nq, cnt.p, seg.p, toff.p, c->d_tc_tiles.p);
            rc = launch_check(c, "k_tc_tiles");
        }
    }
    if (rc == SPRING_OK && n > 0) {
        if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "tiles: injected launch failure");
        else {
            k_tc_entrec<<<std::min((n + threads - 1) / threads, 148 * 8), threads, 0, c->stream>>>(
                n, nq, c->d_tc_entries.p, c->d_tc_keys_s.p, ps.pairs.p, ps.pair_q0.p, src.q0_int, c->d_tc_rec.p);
            rc = launch_check(c, "k_tc_entrec");
        }
    }
    if (rc != SPRING_OK) return rc;
    c->tc_ntiles = ntiles;
    c->tc_npairs = c->h_pin[2];
    c->tc_gen = ps.gen;
    c->tc_ph_gen = c->ph_gen;
    return SPRING_OK;
}

}  // namespace

int run_v3_prescreen(spring_ctx* c, int q0_first, int n_q0, double sigma, const int** d_list, int* n) {
    const PairSet& ps = c->ps_irr;
    const int nmax = (int)std::min<long long>(ps.cap, (long long)n_q0 * (c->nq / 2 + 8));
    const double os = 1.0 / sigma;
    const float rf = (float)(sqrt(EXP_CUT / (0.5 * (os * os))) * 1.0001 + 1e-3);
    const TcQ0 src = irr_src(c);
    SPRING_CHECK(build_tiles_begin(c, src, q0_first, n_q0, nmax, rf));
    SPRING_CHECK(build_tiles_end(c, src));
    *d_list = c->d_tc_entries.p;  // sorted by q1; the pairs with a triple in the window come first
    *n = c->tc_npairs;
    return SPRING_OK;
}

namespace {

// q0 phonons of the time-reversal set, gathered from the grid phonons
__global__ void k_tc_gather_q0(int n0, const int* __restrict__ grid, const double2* __restrict__ evg,
                               const double* __restrict__ omg, const double* __restrict__ obg, double2* __restrict__ ev0,
                               double* __restrict__ om0, double* __restrict__ ob0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n0 * NMODE * NMODE; i += gridDim.x * blockDim.x) {
        const int q = i / (NMODE * NMODE), r = i % (NMODE * NMODE);
        const size_t g = (size_t)grid[q];
        ev0[i] = evg[g * NMODE * NMODE + r];
        if (r < NMODE) {
            om0[q * NMODE + r] = omg[g * NMODE + r];
            ob0[q * NMODE + r] = obg[g * NMODE + r];
        }
    }
}

int tr_src(spring_ctx* c, TcQ0* out) {
    const int n0 = c->ntr;
    if (c->tr_ph_gen != c->ph_gen || c->d_tr_ev.n < (size_t)n0 * NMODE * NMODE) {
        SPRING_CHECK(dalloc(c, c->d_tr_ev, (size_t)n0 * NMODE * NMODE, "time-reversal q0 phonons"));
        SPRING_CHECK(dalloc(c, c->d_tr_om, (size_t)n0 * NMODE, "time-reversal q0 phonons"));
        SPRING_CHECK(dalloc(c, c->d_tr_ob, (size_t)n0 * NMODE, "time-reversal q0 phonons"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc: injected launch failure");
        k_tc_gather_q0<<<std::max(1, std::min((n0 * NMODE * NMODE + 255) / 256, 148 * 8)), 256, 0, c->stream>>>(
            n0, c->d_tr_grid.p, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p, c->d_tr_ev.p, c->d_tr_om.p,
            c->d_tr_ob.p);
        SPRING_CHECK(launch_check(c, "k_tc_gather_q0"));
        c->tr_ph_gen = c->ph_gen;
    }
    *out = TcQ0{&c->ps_tr, c->d_tr_ev.p, c->d_tr_om.p, c->d_tr_ob.p, c->d_tr_int.p, n0, 1};
    return SPRING_OK;
}

// The tensor-core pass over q0 block [q0_first, q0_first + n_q0) of `src`: MODE 0 adds the
// linewidths and phase space into d_lw / d_p3, MODE 1 appends operator entries to bte (its count
// in *bte_ctr, which may exceed bte_cap: then only bte_cap were written).
template <int MODE>
int run_v3tc_core(spring_ctx* c, const TcQ0& src, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw,
                  double* d_p3, TcBteEntry* bte, unsigned long long* bte_ctr, long long bte_cap) {
    const PairSet& ps = *src.ps;
    const int nq = c->nq;
    // slots for the block's pairs without reading their count: at most Nq/2 + 8 per q0
    const int nmax = (int)std::min<long long>(ps.cap, (long long)n_q0 * (nq / 2 + 8));
    SPRING_CHECK(dalloc(c, c->d_tc_a, (size_t)nq * 4 * AIMG, "V3 A table"));
    SPRING_CHECK(dalloc(c, c->d_tc_b, (size_t)nq * 4 * BIMG, "V3 B table"));
    SPRING_CHECK(dalloc(c, c->d_tc_q0, (size_t)src.nq0 * NMODE * sizeof(Q0Rec) / sizeof(double), "V3 q0 records"));
    const int rs = (2 + c->nT + 3) / 4 * 4;
    SPRING_CHECK(dalloc(c, c->d_tc_modes, (size_t)nq * NMODE * rs, "V3 mode records"));
    const double os = 1.0 / sigma;
    const double half_os2 = 0.5 * (os * os);
    const float rf = (float)(sqrt(EXP_CUT / half_os2) * 1.0001 + 1e-3);
    const int threads = 256;
    // The operand tables depend only on the phonons: they run on a side stream, forked after every
    // earlier launch on the main stream, beside the tile build, and are joined before the pass.
    if (!c->stream2) {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(c, e, "side stream");
    }
    {
        cudaError_t e = cudaEventRecord(c->ev_fork, c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream2, c->ev_fork, 0);
        if (e != cudaSuccess) return cuda_fail(c, e, "side stream fork");
    }
    auto tables = [&]() -> int {
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
        k_tc_tab_a<<<nq * 2, 128, 0, c->stream>>>(nq, c->na3, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p,
                                                   c->d_qpnt.p, c->ph_grid.evec.p,
                                                   reinterpret_cast<__nv_bfloat16*>(c->d_tc_a.p));
        SPRING_CHECK(launch_check(c, "k_tc_tab_a"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
        k_tc_tab_b<<<std::min(nq, 148 * 6) * 2, 128, 0, c->stream>>>(nq, c->na3, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p,
                                                   c->d_qpnt.p, c->ph_grid.evec.p,
                                                   reinterpret_cast<__nv_bfloat16*>(c->d_tc_b.p));
        SPRING_CHECK(launch_check(c, "k_tc_tab_b"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
        k_tc_q0tab<<<std::max(1, std::min((src.nq0 * NMODE + threads - 1) / threads, 148 * 4)), threads, 0, c->stream>>>(
            src.nq0, src.ev0, src.om0, src.ob0, c->d_mass_rs.p, reinterpret_cast<Q0Rec*>(c->d_tc_q0.p));
        SPRING_CHECK(launch_check(c, "k_tc_q0tab"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
        k_tc_modes<<<(int)std::min<long long>(((long long)nq * NMODE * rs + threads - 1) / threads, 148LL * 8), threads, 0,
                     c->stream>>>(nq, c->nT, rs, c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p,
                                  c->d_tc_modes.p);
        SPRING_CHECK(launch_check(c, "k_tc_modes"));
        return SPRING_OK;
    };
    cudaStream_t main_stream = c->stream;
    c->stream = c->stream2;  // launches (and their profiling events) go to the side stream
    const int trc = tables();
    c->stream = main_stream;
    {
        const cudaError_t e = cudaEventRecord(c->ev_join, c->stream2);
        if (trc != SPRING_OK) {
            cudaStreamWaitEvent(c->stream, c->ev_join, 0);
            return trc;
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "side stream join");
    }
    int brc = build_tiles_begin(c, src, q0_first, n_q0, nmax, rf);
    if (brc == SPRING_OK) brc = build_tiles_end(c, src);  // the tile count was read while the tables ran
    {
        const cudaError_t e = cudaStreamWaitEvent(c->stream, c->ev_join, 0);  // join the tables
        if (brc != SPRING_OK) return brc;
        if (e != cudaSuccess) return cuda_fail(c, e, "side stream join");
    }
    if (c->tc_ntiles == 0) return SPRING_OK;  // no pair has a mode triple inside the window

    TcArgs a{};
    a.nq = nq;
    a.nq0 = src.nq0;
    a.nT = c->nT;
    a.ntiles = c->tc_ntiles;
    a.q0_first = q0_first;
    a.bte_cap = bte_cap;
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = pol.lo[k];
        a.hi[k] = pol.hi[k];
    }
    a.half_os2 = half_os2;
    a.rf = rf;
    a.max_spins = c->tc_max_spins >= 0 ? c->tc_max_spins : MAX_SPINS;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int ctas = std::max(1, std::min(a.ntiles, sms));
    a.tiles_per_cta = (a.ntiles + ctas - 1) / ctas;
    c->tc_grid = (a.ntiles + a.tiles_per_cta - 1) / a.tiles_per_cta;
    a.rs = rs;
    a.pre = os * ONEBYSQRT2PI;
    a.mfac = host_constants().Sctr3THz2 / double(nq);
    SPRING_CHECK(dalloc(c, c->d_tc_cnt_cta, 1, "V3 status"));
    SPRING_CHECK(zero(c, c->d_tc_cnt_cta.p, sizeof(int), "V3 status"));
    const bool split = c->precision == SPRING_BF16X3, fast = rs == 8 && c->nT <= NT_FAST;
    int lrc;
    if (MODE == 1)
        lrc = split ? launch_tc<true, false, 1>(c, a, src, d_lw, d_p3, bte, bte_ctr)
                    : launch_tc<false, false, 1>(c, a, src, d_lw, d_p3, bte, bte_ctr);
    else if (split)
        lrc = fast ? launch_tc<true, true, 0>(c, a, src, d_lw, d_p3, bte, bte_ctr)
                   : launch_tc<true, false, 0>(c, a, src, d_lw, d_p3, bte, bte_ctr);
    else
        lrc = fast ? launch_tc<false, true, 0>(c, a, src, d_lw, d_p3, bte, bte_ctr)
                   : launch_tc<false, false, 0>(c, a, src, d_lw, d_p3, bte, bte_ctr);
    SPRING_CHECK(lrc);
    SPRING_CHECK(d2h_pin_async(c, c->d_tc_cnt_cta.p, sizeof(int), "V3 status"));
    SPRING_CHECK(pin_wait(c, "V3 status"));
    const int herr = c->h_pin[0];
    if (herr == 2) return fail(c, SPRING_ERR_CUDA, "tensor-core V3: shared memory base not 128-byte aligned");
    if (herr) return fail(c, SPRING_ERR_TIMEOUT, "tensor-core V3: a pipeline wait ran out after %lld polls", a.max_spins);
    return SPRING_OK;
}

}  // namespace

int run_v3tc_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3,
                   bool* handled) {
    *handled = false;
    if (c->nb != 2 || c->na3 > 8) return SPRING_OK;
    *handled = true;
    return run_v3tc_core<0>(c, irr_src(c), q0_first, n_q0, sigma, pol, d_lw, d_p3, nullptr, nullptr, 0);
}

int run_v3tc_bte(spring_ctx* c, int q0_first, int n_q0, double sigma, void* entries, unsigned long long* ctr,
                 long long cap, bool* handled) {
    *handled = false;
    if (c->nb != 2 || c->na3 > 8 || c->precision == SPRING_FP64) return SPRING_OK;
    *handled = true;
    TcQ0 src;
    SPRING_CHECK(tr_src(c, &src));
    Pol all;
    for (int k = 0; k < 3; ++k) {
        all.lo[k] = 0;
        all.hi[k] = NMODE - 1;
    }
    return run_v3tc_core<1>(c, src, q0_first, n_q0, sigma, all, nullptr, nullptr, static_cast<TcBteEntry*>(entries),
                            ctr, cap);
}

}  // namespace spring
