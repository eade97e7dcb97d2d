// Four-phonon V4 on the 5th-generation tensor cores (tcgen05, BF16 in, FP32 accumulate), with the
// Gaussian four-phonon scattering rate.  Two-atom cells.
//
// Same quantity as ScatterMatEl4 / ScatterProbability4 (src/Kappa/Src/FourthOrder_m.f90:286-473)
// and the build-side Gaussian form of the three channels of Tetrahedron4th_sep.f90:329-343, with the
// sum regrouped so that the bulk of it is a GEMM with an operand shared by many quartets.  With
// a = (N, b) a neighbour slot and Cartesian index of the cluster of basis atom mu, P_mu(q, N) =
// e^{i q.R_{mu N}}, and E_q[nu c][s] = m_nu^-1/2 e_q(nu c, s):
//   C_mu[s0][a1][a2][a3]     = sum_al FC4(de,ga,be,al,N3,N2,N1,mu) m_mu^-1/2 e0(mu al, s0)   (per q0)
//   X_mu[s0 s1][a2][a3]      = sum_a1 C_mu[s0][a1][a2][a3] P_mu(q1,N1) E_q1[nu(N1) b][s1]    (per q0, q1)
//   X'[s0 s1 c d][nu2 nu3]   = sum_mu sum_{N2 in nu2, N3 in nu3} X_mu[s0 s1][N2 c][N3 d]
//                               P_mu(q2,N2) P_mu(q3,N3)                                      (per quartet)
//   Phi[s0][s1][s2][s3]      = sum_{nu2 c, nu3 d} X'[s0 s1 c d][nu2 nu3] E_q2[nu2 c][s2] E_q3[nu3 d][s3]
// Quartets are grouped by (q0, q1): a tile is up to 128 quartets of one q1.  X' is the tensor-core
// part: one GEMM per block (nu2, nu3) with the quartets' phase products as the A rows (K = the
// block's (mu, N2, N3) entries, Re and Im halves) and X as the shared B operand (rows = Re/Im of
// (s0 s1 c d)), M = 128 quartets, N = 64 per block, one chunk (s0, three s1) at a time into one of
// two tensor-memory buffers.  The complex product is written as a real one:
//   A[q][k] = [Re P | Im P],  B[(re, r)][k] = [Re X | -Im X],  B[(im, r)][k] = [Im X | Re X].
// The epilogue (FP32, two threads per quartet, three s3 each) contracts E_q3 and E_q2, screens every
// mode quad in FP32 against the windows of its seven delta terms, and evaluates the terms inside
// them in FP64: W = |Phi|^2 (1/w0)(1/w1)(1/w2)(1/w3) Sctr4THz2/Nq^2 and
//   rate(s0) += W [ w1 n1 n2 n3 d(w0 - w1 - w2 - w3)
//                 + sum_k w2_k (1 + n_k) n_i n_j d(w0 + w_k - w_i - w_j)
//                 + sum_k w3_k (1 + n_i)(1 + n_j) n_k d(w0 + w_i + w_j - w_k) ] / n0,
// the three channels of every distinct ordering of the quartet's grid points (1/6, 1/2, 1/2 each)
// gathered by which point plays the first (channel 2) or last (channel 3) role; for three distinct
// points all seven weights are 1.  Precision: SPRING_BF16 rounds A and B to BF16 once;
// SPRING_BF16X3 splits both into hi + lo parts and accumulates hi*hi + hi*lo + lo*hi.
// Roofline: the FP32 epilogue (about 62 kflop of contraction per quartet) bounds the kernel; the
// tensor pipe carries the X' GEMM (about 0.25 Mflop algorithmic per quartet, issued three times
// for BF16x3).
#include <algorithm>
#include <vector>
#include <cub/cub.cuh>
#include <cuda_bf16.h>

#include "spring_internal.cuh"
#include "tc.cuh"

namespace spring {
namespace {

constexpr int NM = 6;           // Ndof of the two-atom cell
constexpr int NA4 = 8;          // largest FC4 cluster handled
constexpr int KA = 3 * NA4;     // slots x Cartesian of one cluster
constexpr int QT = 128;         // quartets per tile (TMEM lanes)
constexpr int NBLK = 4;         // (nu2, nu3) blocks
constexpr int CROWS = 64;       // B rows of one (chunk, block): 3 s1 x 3 c x (re, im) x 3 d = 54, padded
constexpr int NCHUNK = 12;      // chunks of a tile: (s0, s1 in {0,1,2} or {3,4,5})
constexpr int KLIST = 128;      // entries of one block's K list
constexpr int EPI_WARPS = 8;    // two threads per quartet row
constexpr int V4_THREADS = EPI_WARPS * 32 + 64;  // + copy warp (8) + MMA warp (9)
constexpr int TCOLS = 512;      // two buffers of 4 blocks x 64 columns
constexpr double EXP_CUT = 40.0;
constexpr long long MAX_SPINS = 1LL << 26;  // drains of work already issued
constexpr int E2S = 37;         // float2 stride of one quartet's E_q2 in shared memory (36 used)

// Row of the B image (= accumulator column inside a block's 64) of value i = c*6 + ri*3 + d
// (ri = 0 Re, 1 Im) of s1 slot j: the first 16 values of each j at 16 j, the last two at 48 + 2 j,
// so that the epilogue reads them with one 16-column and one 2-column load at aligned columns.
__host__ __device__ __forceinline__ int brow(int j, int i) { return i < 16 ? 16 * j + i : 48 + 2 * j + (i - 16); }

// The block structure of the X' GEMM (host-built from the FC4 cluster's basis types).
struct Blk4 {
    int kb[NBLK];                // complex K entries of each block
    int kpad[NBLK];              // real K of each block, 2 kb rounded up to 16
    int koff[NBLK];              // offset of each block's K range (bf16 elements of one row)
    int ktot;                    // sum of kpad
    short klist[NBLK][KLIST];    // entries mu * 256 + N2 * 16 + N3
};

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    const float f = (float)x;
    hi = __float2bfloat16_rn(f);
    lo = __float2bfloat16_rn(f - __bfloat162float(hi));
}

// ------------------------------------------------------------------ per-grid tables
// Phases P_mu(q, N) = e^{i q.R_{mu N}} (FP64) [q][mu][NA4], and E_q[nu c][s] = m_nu^-1/2 e_q(nu c, s)
// (FP32) [q][nu c][s], and the FP32 omegas [q][s].
__global__ void k4_grid_tabs(int nq, int na, const double* __restrict__ posr, const double* __restrict__ qpnt,
                             const double2* __restrict__ evg, const double* __restrict__ mrs,
                             const double* __restrict__ omg, double2* __restrict__ ph, float2* __restrict__ etab,
                             float* __restrict__ wf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq * 64; i += gridDim.x * blockDim.x) {
        const int q = i / 64, k = i % 64;
        if (k < 2 * NA4) {
            const int mu = k / NA4, N = k % NA4;
            double2 v = make_double2(0.0, 0.0);
            if (N < na) {
                const double* R = posr + ((size_t)mu * na + N) * 3;
                const double qr = qpnt[3 * q] * R[0] + qpnt[3 * q + 1] * R[1] + qpnt[3 * q + 2] * R[2];
                double sn, cs;
                sincos(qr, &sn, &cs);
                v = make_double2(cs, sn);
            }
            ph[(size_t)q * 2 * NA4 + k] = v;
        } else if (k < 2 * NA4 + 36) {
            const int j = k - 2 * NA4, row = j / NM, s = j % NM;  // row = nu * 3 + c
            const double2 e = evg[((size_t)q * NM + s) * NM + row];
            const double m = mrs[row / 3];
            etab[(size_t)q * 36 + j] = make_float2((float)(m * e.x), (float)(m * e.y));
        } else if (k < 2 * NA4 + 36 + NM) {
            const int s = k - 2 * NA4 - 36;
            wf[(size_t)q * NM + s] = (float)omg[(size_t)q * NM + s];
        }
    }
}

// Mode records [q][s][rs]: omega, 1/omega, then n(T) for every temperature (FP64), so that the
// FP64 terms of a mode quad read each grid mode with one contiguous load.
__global__ void k4_modes(int nq, int nT, int rs, const double* __restrict__ omg, const double* __restrict__ obg,
                         const double* __restrict__ nbeg, double* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)nq * NM * rs;
         i += (long long)gridDim.x * blockDim.x) {
        const long long qs = i / rs;
        const int k = (int)(i % rs);
        double v = 0.0;
        if (k == 0) v = omg[qs];
        else if (k == 1) v = obg[qs];
        else if (k - 2 < nT) v = nbeg[(size_t)(k - 2) * nq * NM + qs];
        out[i] = v;
    }
}

// C_mu[s0][a1][a2][a3] of one q0 (FP32 complex), a = N * 3 + b over the slots of mu's cluster
// (slots grouped by basis atom, zero beyond na), [mu][s0][a1][a2][a3] with extent KA each.
__global__ void k4_c0(int na, const double* __restrict__ fc4, const double2* __restrict__ ev0,
                      const double* __restrict__ mrs, float2* __restrict__ cq) {
    const int total = 2 * NM * KA * KA * KA;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int a3 = i % KA, a2 = (i / KA) % KA, a1 = (i / (KA * KA)) % KA, s0 = (i / (KA * KA * KA)) % NM,
                  mu = i / (NM * KA * KA * KA);
        const int N1 = a1 / 3, be = a1 % 3, N2 = a2 / 3, ga = a2 % 3, N3 = a3 / 3, de = a3 % 3;
        double re = 0.0, im = 0.0;
        if (N1 < na && N2 < na && N3 < na) {
            const double* f = fc4 + ((((size_t)mu * na + N1) * na + N2) * na + N3) * 81 + be * 9 + ga * 3 + de;
            const double m = mrs[mu];
#pragma unroll
            for (int al = 0; al < 3; ++al) {
                const double2 e = ev0[s0 * NM + mu * 3 + al];
                const double fv = f[al * 27] * m;
                re = fma(fv, e.x, re);
                im = fma(fv, e.y, im);
            }
        }
        cq[i] = make_float2((float)re, (float)im);
    }
}

// B images of one q1: for chunk ch = (s0, s1 half) and part (hi, lo), the blocks' canonical K-major
// images (LBO 128, SBO kpad/8 * 128) one after the other, rows brow(j, c*6 + ri*3 + d) (j = s1 % 3,
// ri = 0 Re / 1 Im row of the real product), columns [Re P | Im P] of the block's entries.  One
// CTA per (q1, s0) builds the two chunks of s0 in shared memory (from X_mu[s0 s1][a2][a3] =
// sum_a1 C_mu[s0][a1][a2][a3] D_mu(q1)[a1][s1]) and writes them as 16-byte vectors.
// map[mu][N2][N3] = block * 256 + entry of (mu, N2, N3), or -1.
__global__ void __launch_bounds__(256) k4_bimg(int nq, int na, int H, int s0mask, Blk4 bk, const int* __restrict__ qcnt,
                                               const short* __restrict__ map, const float2* __restrict__ cq,
                                               const double2* __restrict__ ph, const float2* __restrict__ etab,
                                               const int* __restrict__ btyp, __nv_bfloat16* __restrict__ img) {
    extern __shared__ __align__(16) unsigned char sm4[];
    const int q1 = blockIdx.x / NM, s0 = blockIdx.x % NM;
    if (qcnt[q1] == 0 || !((s0mask >> s0) & 1)) return;  // no quartet of q0 starts at q1, or s0 not wanted
    const int cimg = CROWS * bk.ktot;               // bf16 elements of one (chunk, part) image
    __nv_bfloat16* simg = reinterpret_cast<__nv_bfloat16*>(sm4);  // [2 chunks][H][cimg]
    float2* sD = reinterpret_cast<float2*>(sm4 + (size_t)2 * H * cimg * 2);  // [mu][a1][s1]
    for (int i = threadIdx.x; i < 2 * H * cimg / 8; i += blockDim.x)
        reinterpret_cast<uint4*>(simg)[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int i = threadIdx.x; i < 2 * KA * NM; i += blockDim.x) {
        const int mu = i / (KA * NM), a1 = (i / NM) % KA, s1 = i % NM;
        const int N1 = a1 / 3, b = a1 % 3;
        float2 v = make_float2(0.f, 0.f);
        if (N1 < na) {
            const double2 p = ph[(size_t)q1 * 2 * NA4 + mu * NA4 + N1];
            const float2 e = etab[(size_t)q1 * 36 + (btyp[mu * na + N1] * 3 + b) * NM + s1];
            v = make_float2((float)(p.x * e.x - p.y * e.y), (float)(p.x * e.y + p.y * e.x));
        }
        sD[i] = v;
    }
    __syncthreads();
    const int KR = 3 * na;
    for (int o = threadIdx.x; o < 2 * KR * KR; o += blockDim.x) {
        const int mu = o / (KR * KR), a2 = (o / KR) % KR, a3 = o % KR;
        const int N2 = a2 / 3, c = a2 % 3, N3 = a3 / 3, d = a3 % 3;
        const int m = map[(mu * NA4 + N2) * NA4 + N3];
        if (m < 0) continue;
        const int b = m >> 8, kk = m & 255;
        float xr[NM], xi[NM];
#pragma unroll
        for (int s = 0; s < NM; ++s) xr[s] = xi[s] = 0.f;
        const float2* cp = cq + (((size_t)mu * NM + s0) * KA * KA * KA) + (size_t)a2 * KA + a3;
        const float2* dp = sD + mu * KA * NM;
        for (int a1 = 0; a1 < KR; ++a1) {
            const float2 cv = cp[(size_t)a1 * KA * KA];
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                const float2 dv = dp[a1 * NM + s];
                xr[s] = fmaf(cv.x, dv.x, fmaf(-cv.y, dv.y, xr[s]));
                xi[s] = fmaf(cv.x, dv.y, fmaf(cv.y, dv.x, xi[s]));
            }
        }
        const uint32_t sbo = (uint32_t)(bk.kpad[b] / 8) * 128u;
        const int base = CROWS * bk.koff[b];  // elements of the block inside a chunk image
        const int kre = kk, kim = bk.kb[b] + kk;
#pragma unroll
        for (int s = 0; s < NM; ++s) {
            const int ch = s / 3, j = s % 3;
            const int nre = brow(j, c * 6 + d), nim = brow(j, c * 6 + 3 + d);
            __nv_bfloat16 h, l;
            __nv_bfloat16* I0 = simg + (size_t)(ch * H) * cimg + base;
            __nv_bfloat16* I1 = I0 + cimg;  // lo part (H == 2)
            auto put = [&](int n, int k, double v) {
                const uint32_t off = tc::kmajor_offset(n, k, 128u, sbo) / 2;
                split_bf16(v, h, l);
                I0[off] = h;
                if (H == 2) I1[off] = l;
            };
            put(nre, kre, xr[s]);
            put(nre, kim, -xi[s]);
            put(nim, kre, xi[s]);
            put(nim, kim, xr[s]);
        }
    }
    __syncthreads();
    // chunks 2 s0 and 2 s0 + 1 of q1, [q1][chunk][part][cimg]
    uint4* dst = reinterpret_cast<uint4*>(img + ((size_t)q1 * NCHUNK + 2 * s0) * H * cimg);
    for (int i = threadIdx.x; i < 2 * H * cimg / 8; i += blockDim.x) dst[i] = reinterpret_cast<const uint4*>(simg)[i];
}

// ------------------------------------------------------------------ tiles
__global__ void k4_count(long long n, const int4* __restrict__ quart, int* __restrict__ cnt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        atomicAdd(&cnt[quart[i].x], 1);
}
__global__ void k4_ntiles(int nq, const int* __restrict__ cnt, int* __restrict__ nt) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x)
        nt[g] = (cnt[g] + QT - 1) / QT;
}
// Tiles (q1, first quartet, count, 0): the quartets are sorted by q1, so the first of q1 is the
// exclusive scan of the counts.
__global__ void k4_tiles(int nq, const int* __restrict__ cnt, const int* __restrict__ seg,
                         const int* __restrict__ toff, int4* __restrict__ tiles) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
        const int c = cnt[g];
        for (int t = 0; t * QT < c; ++t) tiles[toff[g] + t] = make_int4(g, seg[g] + t * QT, min(QT, c - t * QT), 0);
    }
}
__global__ void k4_total(int nq, const int* __restrict__ toff, const int* __restrict__ nt, int* __restrict__ out) {
    out[0] = toff[nq - 1] + nt[nq - 1];
}

// ------------------------------------------------------------------ the tensor-core pass
struct V4Args {
    int nq, nT, nq0, q0, ntiles, tiles_per_cta, H, gq0;
    int rs;                      // doubles per mode record (omega, 1/omega, n(T)), even
    int nch;                     // chunks per tile: two for every branch s0 of the mask
    int chunk[NCHUNK];           // the chunks, in order (chunk c is s0 = c / 2, s1 = 3 (c % 2) .. + 2)
    double mfac, half_os2, pre;  // Sctr4THz2 / Nq^2; 1 / (2 sigma^2); 1 / (sigma sqrt(2 pi))
    float rf;                    // FP32 window half-width of a delta term
    long long max_spins;
};

// Shared memory: A (H parts x QT x ktot bf16), one B part (CROWS x ktot bf16), E_q2 of every quartet
// (a private copy for each of its two threads), then this tail.
struct V4Sm {
    alignas(8) uint64_t afull, afree, bfull, bfree, tfull[2], tempty[2];
    uint32_t tslot;
    int abort;
    double w0[NM], ob0[NM], n0inv[9][NM];
    float w0f[NM];
    double rate[NM][9];  // this CTA's sums for q0, flushed once at the end
};

__global__ void __launch_bounds__(V4_THREADS, 1)
k_v4tc(V4Args a, Blk4 bk, const int4* __restrict__ tiles, const int4* __restrict__ quart,
       const __nv_bfloat16* __restrict__ img, const double2* __restrict__ ph, const float2* __restrict__ etab,
       const float* __restrict__ wf, const double* __restrict__ om0, const double* __restrict__ ob0,
       const double* __restrict__ nbe0, const double* __restrict__ rec, double* __restrict__ out_rate,
       int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smraw[];
    const int H = a.H;
    const size_t abytes = (size_t)H * QT * bk.ktot * 2, bbytes = (size_t)CROWS * bk.ktot * 2;
    uint8_t* sA = smraw;
    uint8_t* sB = smraw + abytes;
    float2* sE2 = reinterpret_cast<float2*>(smraw + abytes + bbytes);
    V4Sm& S = *reinterpret_cast<V4Sm*>(smraw + abytes + bbytes + (size_t)2 * QT * E2S * 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t0 = blockIdx.x * a.tiles_per_cta;
    const int t1 = min(a.ntiles, t0 + a.tiles_per_cta);
    const int nt = max(0, t1 - t0);
    if ((tc::smem_u32(smraw) & 127u) != 0u) {
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    // A (both parts) zero once: the padding columns stay zero, the rows of a short tile finite
    for (int i = tid; i < (int)(abytes / 16); i += blockDim.x) reinterpret_cast<uint4*>(sA)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        S.abort = 0;
        tc::mbar_init(tc::smem_u32(&S.afull), EPI_WARPS * 32);
        tc::mbar_init(tc::smem_u32(&S.afree), 1);
        tc::mbar_init(tc::smem_u32(&S.bfull), 1);
        tc::mbar_init(tc::smem_u32(&S.bfree), 1);
        for (int k = 0; k < 2; ++k) {
            tc::mbar_init(tc::smem_u32(&S.tfull[k]), 1);
            tc::mbar_init(tc::smem_u32(&S.tempty[k]), EPI_WARPS);
        }
        tc::mbar_fence_init();
    }
    for (int i = tid; i < NM * 9; i += blockDim.x) (&S.rate[0][0])[i] = 0.0;
    for (int i = tid; i < NM; i += blockDim.x) {
        S.w0[i] = om0[i];
        S.w0f[i] = (float)om0[i];
        S.ob0[i] = ob0[i];
        for (int t = 0; t < a.nT; ++t) S.n0inv[t][i] = 1.0 / nbe0[(size_t)t * a.nq0 * NM + i];
    }
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tslot), TCOLS);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = S.tslot;
    int issued_copies = 0;  // copy warp: chunk copies issued

    if (warp == EPI_WARPS) {
        // ------------------------------------------------------------ copy warp
        // One B buffer holding one part: part u = chunk * H + part is copied once the MMAs of part
        // u - 1 released the buffer.
        if (lane == 0) {
            const uint32_t bytes = (uint32_t)bbytes;
            for (int t = 0; t < nt; ++t) {
                const int q1 = tiles[t0 + t].x;
                for (int ch = 0; ch < a.nch * H; ++ch) {
                    const int u = t * a.nch * H + ch;
                    if (u > 0 && !tc::mbar_wait(tc::smem_u32(&S.bfree), (uint32_t)((u - 1) & 1), a.max_spins)) {
                        atomicExch(err, 1);
                        *(volatile int*)&S.abort = 1;
                        t = nt;
                        break;
                    }
                    const uint32_t fb = tc::smem_u32(&S.bfull);
                    tc::mbar_expect_tx(fb, bytes);
                    const int cpart = a.chunk[ch / H] * H + ch % H;  // (chunk, part) of the image
                    tc::bulk_g2s(tc::smem_u32(sB), img + ((size_t)q1 * NCHUNK * H + cpart) * CROWS * bk.ktot, bytes, fb);
                    tc::mbar_arrive(fb);
                    issued_copies = u + 1;
                }
            }
        }
        __syncwarp();
    } else if (warp == EPI_WARPS + 1) {
        // ------------------------------------------------------------ MMA warp
        // Chunk k into accumulator buffer k % 2 once the epilogue drained it (chunk k - 2); part 0
        // (B hi) takes A hi and, for BF16x3, A lo; part 1 (B lo) takes A hi.  bfree after every part,
        // tfull after the chunk, afree after the tile's last chunk.
        int last_u = -1;  // last part whose MMAs were committed (to bfree)
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16(QT, CROWS);
            bool ok = true;
            for (int t = 0; ok && t < nt; ++t) {
                ok = tc::mbar_wait(tc::smem_u32(&S.afull), (uint32_t)(t & 1), a.max_spins);
                for (int ch = 0; ok && ch < a.nch; ++ch) {
                    const int k = t * a.nch + ch, buf = k & 1;
                    ok = k < 2 || tc::mbar_wait(tc::smem_u32(&S.tempty[buf]), (uint32_t)(((k >> 1) - 1) & 1),
                                                a.max_spins);
                    for (int part = 0; ok && part < H; ++part) {
                        const int u = k * H + part;
                        ok = tc::mbar_wait(tc::smem_u32(&S.bfull), (uint32_t)(u & 1), a.max_spins);
                        if (!ok) break;
                        tc::fence_after_sync();
                        for (int b = 0; b < NBLK; ++b) {
                            const uint32_t d = tm + (uint32_t)(buf * 256 + b * CROWS);
                            const uint32_t sbo = (uint32_t)(bk.kpad[b] / 8) * 128u;
                            const uint32_t ah = tc::smem_u32(sA) + (uint32_t)(QT * bk.koff[b] * 2);
                            const uint32_t al = ah + (uint32_t)(QT * bk.ktot * 2);
                            const uint32_t bb = tc::smem_u32(sB) + (uint32_t)(CROWS * bk.koff[b] * 2);
                            for (int kk = 0; kk < bk.kpad[b] / 16; ++kk) {
                                const uint32_t ko = (uint32_t)kk * 256u;
                                const uint64_t bd = tc::sdesc(bb + ko, 128u, sbo);
                                tc::mma_bf16(d, tc::sdesc(ah + ko, 128u, sbo), bd, idesc, (part > 0 || kk > 0) ? 1u : 0u);
                                if (H == 2 && part == 0) tc::mma_bf16(d, tc::sdesc(al + ko, 128u, sbo), bd, idesc, 1u);
                            }
                        }
                        tc::mma_commit(tc::smem_u32(&S.bfree));
                        last_u = u;
                    }
                    if (!ok) break;
                    tc::mma_commit(tc::smem_u32(&S.tfull[buf]));
                    if (ch == a.nch - 1) tc::mma_commit(tc::smem_u32(&S.afree));
                }
            }
            if (!ok) {
                atomicExch(err, 1);
                *(volatile int*)&S.abort = 1;
            }
            // the last commit tracks every MMA issued: wait for it before tensor memory is released
            if (last_u >= 0) tc::mbar_wait(tc::smem_u32(&S.bfree), (uint32_t)(last_u & 1), MAX_SPINS);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue warps
        // Thread (row r, half h): quartet r of the tile, s3 = 3h .. 3h+2.  It builds its half of the
        // quartet's A row (blocks h and h + 2) and its own copy of E_q2, so that no thread reads what
        // another wrote; the only synchronisation is through the mbarriers (every wait bounded).
        const int wq = warp & 3, h = warp >> 2;      // TMEM lanes 32 wq .. +31; s3 = 3h .. 3h+2
        const int r = wq * 32 + lane;                 // quartet row of the tile
        const int pol_lo0 = a.gq0 ? 3 : 0;
        float2* myE2 = sE2 + (size_t)(h * QT + r) * E2S;
        for (int t = 0; t < nt; ++t) {
            // ---- tile set-up: wait until the MMAs of the previous tile no longer read A
            bool ok = t == 0 || tc::mbar_wait(tc::smem_u32(&S.afree), (uint32_t)((t - 1) & 1), a.max_spins);
            if (__any_sync(0xffffffffu, !ok)) {
                if (lane == 0) {
                    atomicExch(err, 1);
                    *(volatile int*)&S.abort = 1;
                }
                break;
            }
            const int4 tr = tiles[t0 + t];
            const bool valid = r < tr.z;
            int4 qd = make_int4(tr.x, 0, 0, 0);
            if (valid) qd = quart[tr.y + r];
            const int g1 = qd.x, g2 = qd.y, g3 = qd.z;
            // A row: this thread's two blocks (h = 0: blocks 0, 2; h = 1: blocks 1, 3)
            if (valid) {
                for (int bi = 0; bi < 2; ++bi) {
                    const int b = h + 2 * bi;
                    const uint32_t sbo = (uint32_t)(bk.kpad[b] / 8) * 128u;
                    __nv_bfloat16* Ah = reinterpret_cast<__nv_bfloat16*>(sA) + QT * bk.koff[b];
                    __nv_bfloat16* Al = Ah + QT * bk.ktot;
#pragma unroll 4
                    for (int j = 0; j < bk.kb[b]; ++j) {
                        const int e = bk.klist[b][j];
                        const int mu = e >> 8, N2 = (e >> 4) & 15, N3 = e & 15;
                        const double2 p2 = ph[(size_t)g2 * 2 * NA4 + mu * NA4 + N2];
                        const double2 p3 = ph[(size_t)g3 * 2 * NA4 + mu * NA4 + N3];
                        const double pr = p2.x * p3.x - p2.y * p3.y, pim = p2.x * p3.y + p2.y * p3.x;
                        __nv_bfloat16 hh, ll;
                        const uint32_t ore = tc::kmajor_offset(r, j, 128u, sbo) / 2;
                        const uint32_t oim = tc::kmajor_offset(r, bk.kb[b] + j, 128u, sbo) / 2;
                        split_bf16(pr, hh, ll);
                        Ah[ore] = hh;
                        if (H == 2) Al[ore] = ll;
                        split_bf16(pim, hh, ll);
                        Ah[oim] = hh;
                        if (H == 2) Al[oim] = ll;
                    }
                }
#pragma unroll 6
                for (int j = 0; j < 36; ++j) myE2[j] = etab[(size_t)g2 * 36 + j];
            }
            tc::fence_async_smem();
            tc::mbar_arrive(tc::smem_u32(&S.afull));
            // per-quartet registers: E_q3 of this thread's s3, FP32 omegas, Gamma flags, term weights
            float2 e3[6][3];
            float w1f[NM], w2f[NM], w3f[3];
#pragma unroll
            for (int x = 0; x < 6; ++x)
#pragma unroll
                for (int y = 0; y < 3; ++y)
                    e3[x][y] = valid ? etab[(size_t)g3 * 36 + x * NM + 3 * h + y] : make_float2(0.f, 0.f);
#pragma unroll
            for (int s = 0; s < NM; ++s) {
                w1f[s] = wf[(size_t)g1 * NM + s];
                w2f[s] = valid ? wf[(size_t)g2 * NM + s] : 0.f;
            }
#pragma unroll
            for (int y = 0; y < 3; ++y) w3f[y] = valid ? wf[(size_t)g3 * NM + 3 * h + y] : 0.f;
            // term weights in units of 1/6 (channel 1) and 1/2 (channels 2, 3): the distinct orderings
            // of (g1, g2, g3) by their first two points (every one of the six when they differ)
            int c1 = 0, c2[3] = {0, 0, 0}, c3[3] = {0, 0, 0};
            {
                const int G[3] = {g1, g2, g3};
                const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
#pragma unroll
                for (int pi = 0; pi < 6; ++pi) {
                    bool dup = false;
#pragma unroll
                    for (int pj = 0; pj < pi; ++pj)
                        dup = dup || (G[perms[pj][0]] == G[perms[pi][0]] && G[perms[pj][1]] == G[perms[pi][1]]);
                    if (dup) continue;
                    c1 += 1;
                    c2[perms[pi][0]] += 1;
                    c3[perms[pi][2]] += 1;
                }
            }
            const bool gam1 = g1 == 0, gam2 = g2 == 0, gam3 = g3 == 0;
            // ---- chunks
            for (int ch = 0; ch < a.nch; ++ch) {
                const int k = t * a.nch + ch, buf = k & 1;
                const int s0 = a.chunk[ch] >> 1, s1b = 3 * (a.chunk[ch] & 1);
                ok = tc::mbar_wait(tc::smem_u32(&S.tfull[buf]), (uint32_t)((k >> 1) & 1), a.max_spins);
                if (__any_sync(0xffffffffu, !ok)) {
                    if (lane == 0) {
                        atomicExch(err, 1);
                        *(volatile int*)&S.abort = 1;
                    }
                    t = nt;
                    break;
                }
                tc::fence_after_sync();
                double acc[9];
#pragma unroll
                for (int T = 0; T < 9; ++T) acc[T] = 0.0;
                const uint32_t tb = tm + ((uint32_t)(wq * 32) << 16) + (uint32_t)(buf * 256);
#pragma unroll 1
                for (int j = 0; j < 3; ++j) {
                    const int s1 = s1b + j;
                    const bool act = valid && s0 >= pol_lo0 && !(gam1 && s1 < 3);
                    float2 phi[NM][3];
#pragma unroll
                    for (int x = 0; x < NM; ++x)
#pragma unroll
                        for (int y = 0; y < 3; ++y) phi[x][y] = make_float2(0.f, 0.f);
#pragma unroll
                    for (int nu2 = 0; nu2 < 2; ++nu2) {
                        // blocks (nu2, 0) = 2 nu2 and (nu2, 1) = 2 nu2 + 1: the 18 values of slot j
                        // (value i = c*6 + ri*3 + d at column brow(j, i))
                        float xv[2][18];
                        __syncwarp();
#pragma unroll
                        for (int nu3 = 0; nu3 < 2; ++nu3) {
                            const uint32_t cb = tb + (uint32_t)((2 * nu2 + nu3) * CROWS);
                            tc::tmem_ld16(cb + (uint32_t)(16 * j), xv[nu3]);
                            tc::tmem_ld2(cb + (uint32_t)(48 + 2 * j), xv[nu3] + 16);
                        }
                        tc::tmem_ld_wait();
                        if (j == 2 && nu2 == 1) {  // this warp's reads of the buffer are done
                            tc::fence_before_sync();
                            __syncwarp();
                            if (lane == 0) tc::mbar_arrive(tc::smem_u32(&S.tempty[buf]));
                        }
                        if (act) {
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                // Z[s3] = sum_{nu3 d} X'[c d][nu2 nu3] E3[nu3 d][s3]; value c*6 + ri*3 + d
                                float2 z[3];
#pragma unroll
                                for (int y = 0; y < 3; ++y) z[y] = make_float2(0.f, 0.f);
#pragma unroll
                                for (int nu3 = 0; nu3 < 2; ++nu3)
#pragma unroll
                                    for (int d = 0; d < 3; ++d) {
                                        const float xr = xv[nu3][c * 6 + d], xi = xv[nu3][c * 6 + 3 + d];
#pragma unroll
                                        for (int y = 0; y < 3; ++y) {
                                            const float2 e = e3[nu3 * 3 + d][y];
                                            z[y].x = fmaf(xr, e.x, fmaf(-xi, e.y, z[y].x));
                                            z[y].y = fmaf(xr, e.y, fmaf(xi, e.x, z[y].y));
                                        }
                                    }
                                // Phi[s2][s3] += E2[nu2 c][s2] Z[s3]
                                const float2* e2p = myE2 + (nu2 * 3 + c) * NM;
#pragma unroll
                                for (int s2 = 0; s2 < NM; ++s2) {
                                    const float2 e = e2p[s2];
#pragma unroll
                                    for (int y = 0; y < 3; ++y) {
                                        phi[s2][y].x = fmaf(e.x, z[y].x, fmaf(-e.y, z[y].y, phi[s2][y].x));
                                        phi[s2][y].y = fmaf(e.x, z[y].y, fmaf(e.y, z[y].x, phi[s2][y].y));
                                    }
                                }
                            }
                        }
                    }
                    if (!act) continue;
                    // ---- screen every (s2, s3) of this (s0, s1) against the seven windows:
                    // with u = w0 - w1, v = w0 + w1, P = w2 + w3, M = w2 - w3 the terms are u - P, v - P,
                    // u + P, u + M, u - M, v - M, v + M; min(|x - y|, |x + y|) = ||x| - |y||
                    const double* r1 = rec + ((size_t)g1 * NM + s1) * a.rs;
                    const double2 m1 = *reinterpret_cast<const double2*>(r1);
                    const float u = S.w0f[s0] - w1f[s1], v = S.w0f[s0] + w1f[s1];
                    const float au = fabsf(u), av = fabsf(v);
                    // FP32 screen of the 18 (s2, s3) of this thread (unrolled: registers only), then
                    // one copy of the FP64 code for the quads inside a window (a rolled loop keeps the
                    // kernel's code within the instruction cache)
                    unsigned am = 0u;
                    float a2s[NM * 3];
#pragma unroll
                    for (int s2 = 0; s2 < NM; ++s2)
#pragma unroll
                        for (int y = 0; y < 3; ++y) {
                            a2s[3 * s2 + y] = phi[s2][y].x * phi[s2][y].x + phi[s2][y].y * phi[s2][y].y;
                            if ((gam2 && s2 < 3) || (gam3 && 3 * h + y < 3)) continue;
                            const float P = w2f[s2] + w3f[y], M = w2f[s2] - w3f[y];
                            const float aM = fabsf(M);
                            const bool any = fabsf(au - fabsf(P)) < a.rf || fabsf(v - P) < a.rf ||
                                             fabsf(au - aM) < a.rf || fabsf(av - aM) < a.rf;
                            if (any) am |= 1u << (3 * s2 + y);
                        }
#pragma unroll 1
                    while (am != 0u) {
                        const int bq = __ffs(am) - 1;
                        am &= am - 1u;
                        const int s2 = bq / 3, s3 = 3 * h + bq % 3;
                        const float a2 = a2s[bq];
                        // FP64: W and the seven terms, from the mode records (omega, 1/omega, n(T))
                        // of q2 and q3, one load each; the q1 record was read for this s1
                        const double* r2 = rec + ((size_t)g2 * NM + s2) * a.rs;
                        const double* r3 = rec + ((size_t)g3 * NM + s3) * a.rs;
                        const double2 m2 = *reinterpret_cast<const double2*>(r2);
                        const double2 m3 = *reinterpret_cast<const double2*>(r3);
                        // occupations of up to four temperatures, loaded with the records (rs >= 6)
                        double2 n2a = make_double2(0.0, 0.0), n2b = n2a, n3a = n2a, n3b = n2a;
                        if (a.nT <= 4) {
                            n2a = *reinterpret_cast<const double2*>(r2 + 2);
                            n3a = *reinterpret_cast<const double2*>(r3 + 2);
                            if (a.nT > 2) {
                                n2b = *reinterpret_cast<const double2*>(r2 + 4);
                                n3b = *reinterpret_cast<const double2*>(r3 + 4);
                            }
                        }
                        const double W0 = S.w0[s0], W1 = m1.x, W2 = m2.x, W3 = m3.x;
                        const double Wv = (double)a2 * S.ob0[s0] * m1.y * m2.y * m3.y * a.mfac;
                        const double dd[7] = {W0 - W1 - W2 - W3, W0 + W1 - W2 - W3, W0 + W2 - W1 - W3,
                                              W0 + W3 - W1 - W2, W0 + W2 + W3 - W1, W0 + W1 + W3 - W2,
                                              W0 + W1 + W2 - W3};
                        const int cw[7] = {c1, c2[0], c2[1], c2[2], c3[0], c3[1], c3[2]};
                        double gm[7], xs[7];
                        unsigned need = 0u;  // the terms of this quad inside the cut
#pragma unroll
                        for (int m = 0; m < 7; ++m) {
                            gm[m] = 0.0;
                            xs[m] = a.half_os2 * (dd[m] * dd[m]);
                            if (cw[m] != 0 && xs[m] < EXP_CUT) need |= 1u << m;
                        }
                        if (need == 0u) continue;
                        // one exp call site for whichever terms a lane needs (lanes needing different
                        // terms run it together); the values are those of the term-by-term form
                        while (need != 0u) {
                            const int m = __ffs(need) - 1;
                            need &= need - 1u;
                            double x = xs[0];
                            int c = cw[0];
#pragma unroll
                            for (int k = 1; k < 7; ++k)
                                if (m == k) {
                                    x = xs[k];
                                    c = cw[k];
                                }
                            const double wt = m == 0 ? c * ONEBYSIX : c * 0.5;
                            const double g = (a.pre * exp(-x)) * wt * Wv;
#pragma unroll
                            for (int k = 0; k < 7; ++k)
                                if (m == k) gm[k] = g;
                        }
                        // occupation factors of the seven terms, per temperature:
                        // n1 n2 n3, (1+n1) n2 n3, (1+n2) n1 n3, (1+n3) n1 n2, (1+n2)(1+n3) n1,
                        // (1+n1)(1+n3) n2, (1+n1)(1+n2) n3, over n0
#pragma unroll
                        for (int T = 0; T < 9; ++T) {
                            if (T >= a.nT) break;
                            double n2, n3;
                            if (a.nT <= 4 && T < 4) {
                                n2 = T == 0 ? n2a.x : T == 1 ? n2a.y : T == 2 ? n2b.x : n2b.y;
                                n3 = T == 0 ? n3a.x : T == 1 ? n3a.y : T == 2 ? n3b.x : n3b.y;
                            } else {
                                n2 = r2[2 + T];
                                n3 = r3[2 + T];
                            }
                            const double n1 = r1[2 + T];
                            const double p1 = 1.0 + n1, p2 = 1.0 + n2, p3 = 1.0 + n3;
                            const double f = gm[0] * (n1 * n2 * n3) + gm[1] * (p1 * n2 * n3) + gm[2] * (p2 * n1 * n3) +
                                             gm[3] * (p3 * n1 * n2) + gm[4] * (p2 * p3 * n1) + gm[5] * (p1 * p3 * n2) +
                                             gm[6] * (p1 * p2 * n3);
                            acc[T] += f * S.n0inv[T][s0];
                        }
                    }
                }
                // this chunk's sums of s0: warp reduction, one shared-memory add per warp
#pragma unroll
                for (int T = 0; T < 9; ++T) {
                    if (T >= a.nT) break;
                    double vv = acc[T];
                    for (int o = 16; o > 0; o >>= 1) vv += __shfl_down_sync(0xffffffffu, vv, o);
                    if (lane == 0 && vv != 0.0) atomicAdd(&S.rate[s0][T], vv);
                }
            }
        }
    }
    // Drain: after a time-out the last chunk copy may be in flight unconsumed; the copy warp waits
    // for it before shared memory is released (its bytes always land).  The MMA warp already waited
    // for its last commit.
    tc::fence_before_sync();
    __syncthreads();
    if (warp == EPI_WARPS && lane == 0 && *(volatile int*)&S.abort && issued_copies > 0)
        tc::mbar_wait(tc::smem_u32(&S.bfull), (uint32_t)((issued_copies - 1) & 1), MAX_SPINS);
    // this CTA's rates of q0
    if (tid < NM * a.nT) {
        const int sx = tid / a.nT, T = tid % a.nT;
        const double vv = S.rate[sx][T];
        if (vv != 0.0) atomicAdd(&out_rate[((size_t)T * a.nq0 + a.q0) * NM + sx], vv);
    }
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tm, TCOLS);
}

}  // namespace

// Block structure of the X' GEMM from the FC4 cluster of each basis atom: block (nu2, nu3) holds
// every (mu, N2, N3) whose slots N2, N3 have basis types nu2, nu3.
static int v4_blocks(spring_ctx* c, Blk4& bk, std::vector<short>& map) {
    std::vector<int> btyp((size_t)2 * c->na4);
    SPRING_CHECK(d2h(c, btyp.data(), c->d_fc4_btyp.p, sizeof(int) * btyp.size(), "FC4 basis"));
    std::vector<int> num(2);
    map.assign((size_t)2 * NA4 * NA4, (short)-1);
    for (int b = 0; b < NBLK; ++b) bk.kb[b] = 0;
    for (int mu = 0; mu < 2; ++mu)
        for (int N2 = 0; N2 < c->na4; ++N2)
            for (int N3 = 0; N3 < c->na4; ++N3) {
                const int b = btyp[mu * c->na4 + N2] * 2 + btyp[mu * c->na4 + N3];
                if (bk.kb[b] >= KLIST) return fail(c, SPRING_ERR_UNSUPPORTED, "tensor-core V4: block too large");
                bk.klist[b][bk.kb[b]] = (short)(mu * 256 + N2 * 16 + N3);
                map[((size_t)mu * NA4 + N2) * NA4 + N3] = (short)(b * 256 + bk.kb[b]);
                bk.kb[b] += 1;
            }
    bk.ktot = 0;
    for (int b = 0; b < NBLK; ++b) {
        bk.kpad[b] = std::max(16, (2 * bk.kb[b] + 15) / 16 * 16);
        bk.koff[b] = bk.ktot;
        bk.ktot += bk.kpad[b];
    }
    return SPRING_OK;
}

int run_v4tc_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const int* h_mask, double* d_rate,
                   bool* handled) {
    *handled = false;
    if (c->nb != 2 || c->na4 > NA4 || c->nT > 9 || c->precision == SPRING_FP64) return SPRING_OK;
    *handled = true;
    const int nq = c->nq, H = c->precision == SPRING_BF16X3 ? 2 : 1;
    Blk4 bk{};
    std::vector<short> hmap;
    SPRING_CHECK(v4_blocks(c, bk, hmap));
    const size_t abytes = (size_t)H * QT * bk.ktot * 2, bbytes = (size_t)CROWS * bk.ktot * 2;
    const size_t smem = abytes + bbytes + (size_t)2 * QT * E2S * 8 + sizeof(V4Sm);
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "tensor-core V4 needs %zu bytes of shared memory", smem);
    const size_t bimg_smem = (size_t)2 * H * CROWS * bk.ktot * 2 + (size_t)2 * KA * NM * 8;
    if (bimg_smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "V4 operand images need %zu bytes", bimg_smem);
    // per-grid tables and per-call buffers (kept in the context)
    SPRING_CHECK(dalloc(c, c->d_v4_ph, (size_t)nq * 2 * NA4, "V4 phases"));
    SPRING_CHECK(dalloc(c, c->d_v4_etab, (size_t)nq * 36, "V4 eigenvector table"));
    SPRING_CHECK(dalloc(c, c->d_v4_wf, (size_t)nq * NM, "V4 omegas"));
    SPRING_CHECK(dalloc(c, c->d_v4_c, (size_t)2 * NM * KA * KA * KA, "V4 C table"));
    SPRING_CHECK(dalloc(c, c->d_v4_map, hmap.size(), "V4 block map"));
    const size_t img_elems = (size_t)nq * NCHUNK * H * CROWS * bk.ktot;
    SPRING_CHECK(dalloc(c, c->d_v4_img, (img_elems * 2 + 15) / 16, "V4 operand images"));
    SPRING_CHECK(dalloc(c, c->d_v4_cnt, nq, "V4 tile counts"));
    SPRING_CHECK(dalloc(c, c->d_v4_seg, nq, "V4 tile counts"));
    SPRING_CHECK(dalloc(c, c->d_v4_ntl, nq, "V4 tile counts"));
    SPRING_CHECK(dalloc(c, c->d_v4_toff, nq, "V4 tile counts"));
    SPRING_CHECK(dalloc(c, c->d_v4_stat, 2, "V4 status"));
    const int rs = (2 + c->nT + 1) / 2 * 2;
    SPRING_CHECK(dalloc(c, c->d_v4_rec, (size_t)nq * NM * rs, "V4 mode records"));
    SPRING_CHECK(h2d(c, c->d_v4_map.p, hmap.data(), sizeof(short) * hmap.size(), "V4 block map"));
    const int threads = 256;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc tables: injected launch failure");
    k4_grid_tabs<<<(int)std::min<long long>(((long long)nq * 64 + threads - 1) / threads, 148LL * 16), threads, 0,
                   c->stream>>>(nq, c->na4, c->d_fc4_posr.p, c->d_qpnt.p, c->ph_grid.evec.p, c->d_mass_rs.p,
                                c->ph_grid.omega.p, c->d_v4_ph.p, c->d_v4_etab.p, c->d_v4_wf.p);
    SPRING_CHECK(launch_check(c, "k4_grid_tabs"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc tables: injected launch failure");
    k4_modes<<<(int)std::min<long long>(((long long)nq * NM * rs + threads - 1) / threads, 148LL * 16), threads, 0,
               c->stream>>>(nq, c->nT, rs, c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p, c->d_v4_rec.p);
    SPRING_CHECK(launch_check(c, "k4_modes"));
    cudaFuncSetAttribute(k_v4tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k4_bimg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bimg_smem);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const double os = 1.0 / sigma;
    V4Args a{};
    a.nq = nq;
    a.nT = c->nT;
    a.nq0 = c->nq0;
    a.H = H;
    a.rs = rs;
    a.mfac = host_constants().Sctr4THz2 / (double(nq) * double(nq));
    a.half_os2 = 0.5 * os * os;
    a.pre = os * ONEBYSQRT2PI;
    a.rf = (float)(std::sqrt(EXP_CUT / a.half_os2) * 1.0001 + 1e-3);
    a.max_spins = c->tc_max_spins >= 0 ? c->tc_max_spins : MAX_SPINS;
    for (int q0 = q0_first; q0 < q0_first + n_q0; ++q0) {
        const int mask = h_mask ? (h_mask[q0 - q0_first] & 0x3f) : 0x3f;
        a.nch = 0;
        for (int s0 = 0; s0 < NM; ++s0)
            if ((mask >> s0) & 1) {
                a.chunk[a.nch++] = 2 * s0;
                a.chunk[a.nch++] = 2 * s0 + 1;
            }
        if (a.nch == 0) continue;
        const int4* d_quart = nullptr;
        long long nquart = 0;
        SPRING_CHECK(run_enum4_list(c, q0, &d_quart, &nquart));
        if (nquart == 0) continue;
        // tiles of up to 128 quartets of one q1
        SPRING_CHECK(zero(c, c->d_v4_cnt.p, sizeof(int) * nq, "V4 tile counts"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc tiles: injected launch failure");
        k4_count<<<(int)std::min<long long>((nquart + threads - 1) / threads, 148LL * 16), threads, 0, c->stream>>>(
            nquart, d_quart, c->d_v4_cnt.p);
        SPRING_CHECK(launch_check(c, "k4_count"));
        SPRING_CHECK(run_exclusive_scan(c, c->d_v4_cnt.p, c->d_v4_seg.p, nq));
        k4_ntiles<<<(nq + threads - 1) / threads, threads, 0, c->stream>>>(nq, c->d_v4_cnt.p, c->d_v4_ntl.p);
        SPRING_CHECK(launch_check(c, "k4_ntiles"));
        SPRING_CHECK(run_exclusive_scan(c, c->d_v4_ntl.p, c->d_v4_toff.p, nq));
        k4_total<<<1, 1, 0, c->stream>>>(nq, c->d_v4_toff.p, c->d_v4_ntl.p, c->d_v4_stat.p);
        SPRING_CHECK(launch_check(c, "k4_total"));
        // C of q0 and the operand images of every q1 that starts a quartet (while the count is read)
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc tables: injected launch failure");
        k4_c0<<<std::min((2 * NM * KA * KA * KA + threads - 1) / threads, 148 * 8), threads, 0, c->stream>>>(
            c->na4, c->d_fc4.p, c->ph_irr.evec.p + (size_t)q0 * 36, c->d_mass_rs.p, c->d_v4_c.p);
        SPRING_CHECK(launch_check(c, "k4_c0"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc tables: injected launch failure");
        k4_bimg<<<nq * NM, 256, bimg_smem, c->stream>>>(
            nq, c->na4, H, mask, bk, c->d_v4_cnt.p, c->d_v4_map.p, c->d_v4_c.p, c->d_v4_ph.p, c->d_v4_etab.p,
            c->d_fc4_btyp.p, reinterpret_cast<__nv_bfloat16*>(c->d_v4_img.p));
        SPRING_CHECK(launch_check(c, "k4_bimg"));
        int ntiles = 0;
        SPRING_CHECK(d2h(c, &ntiles, c->d_v4_stat.p, sizeof(int), "V4 tile count"));
        if (ntiles == 0) continue;
        SPRING_CHECK(dalloc(c, c->d_v4_tiles, ntiles, "V4 tiles"));
        k4_tiles<<<(nq + threads - 1) / threads, threads, 0, c->stream>>>(nq, c->d_v4_cnt.p, c->d_v4_seg.p,
                                                                          c->d_v4_toff.p, c->d_v4_tiles.p);
        SPRING_CHECK(launch_check(c, "k4_tiles"));
        int q0int[3];
        std::copy(c->h_irr_int.begin() + 3 * q0, c->h_irr_int.begin() + 3 * q0 + 3, q0int);
        a.q0 = q0;
        a.gq0 = q0int[0] == 0 && q0int[1] == 0 && q0int[2] == 0;
        a.ntiles = ntiles;
        const int ctas = std::max(1, std::min(ntiles, sms));
        a.tiles_per_cta = (ntiles + ctas - 1) / ctas;
        const int grid = (ntiles + a.tiles_per_cta - 1) / a.tiles_per_cta;
        SPRING_CHECK(zero(c, c->d_v4_stat.p + 1, sizeof(int), "V4 status"));
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v4tc: injected launch failure");
        k_v4tc<<<grid, V4_THREADS, smem, c->stream>>>(
            a, bk, c->d_v4_tiles.p, d_quart, reinterpret_cast<const __nv_bfloat16*>(c->d_v4_img.p), c->d_v4_ph.p,
            c->d_v4_etab.p, c->d_v4_wf.p, c->ph_irr.omega.p + (size_t)q0 * NM, c->ph_irr.oneby.p + (size_t)q0 * NM,
            c->ph_irr.nbe.p + (size_t)q0 * NM, c->d_v4_rec.p, d_rate, c->d_v4_stat.p + 1);
        SPRING_CHECK(launch_check(c, H == 2 ? "k_v4tc<bf16x3>" : "k_v4tc<bf16>"));
        int st = 0;
        SPRING_CHECK(d2h(c, &st, c->d_v4_stat.p + 1, sizeof(int), "V4 status"));
        if (st == 2) return fail(c, SPRING_ERR_CUDA, "tensor-core V4: shared memory base not 128-byte aligned");
        if (st) return fail(c, SPRING_ERR_TIMEOUT, "tensor-core V4: a pipeline wait ran out after %lld polls",
                            a.max_spins);
    }
    return SPRING_OK;
}

}  // namespace spring
