// Three-phonon V3 on the 5th-generation tensor cores (tcgen05, BF16 in, FP32
// accumulate), fused with the Gaussian linewidth sum.  Two-atom cells.
//
// Same quantity as ScatterMatEl / ScatterProbability + CalculateLinewidth
// (src/Kappa/Src/ThirdOrder_m.f90:278-439, 442-543), regrouped so that the
// bulk of the work is a GEMM with a shared operand:
//   U_q[mu][N b][s]      = e^{i q.R_{mu N}} m_{nu(N)}^-1/2 e_q(nu(N) b, s)         (per grid q)
//   Z_q1[mu][a s1][N2 c] = sum_{N1 b} FC3[mu][N1][N2][a b c] U_q1[mu][N1 b][s1]     (per grid q1)
//   Y[mu][a s1][s2]      = sum_{N2 c} Z_q1[mu][a s1][N2 c] U_q2[mu][N2 c][s2]       (per pair: tensor cores)
//   Phi[s0][s1][s2]      = sum_{mu a} m_mu^-1/2 e0(mu a, s0) Y[mu][a s1][s2]        (per pair: epilogue)
// Pairs are grouped by q1, so one tile is up to 16 pairs sharing Z_q1: the MMA
// computes Y^T for rows 8 pair + s2 at once, M = 128, N = 48 (36 used:
// Re/Im of (a, s1)), K = 48 (Re/Im of (N2, c), 42 used), one accumulator per
// basis atom mu in tensor memory.  The complex product is written as a real one:
//   A[(pair, s2)][k] = [Re U_q2 | Im U_q2],   B[(re, a s1)][k] = [Re Z | -Im Z],
//   B[(im, a s1)][k] = [Im Z | Re Z].
// Precision: SPRING_BF16 rounds A and B to BF16 once; SPRING_BF16X3 splits each
// into hi + lo BF16 parts and accumulates hi*hi + hi*lo + lo*hi (compensated).
// Frequencies, occupations, the delta weights and every sum stay FP64.  The
// epilogue screens each mode triple in FP32 against the window where a delta
// weight can exceed exp(-40) of its peak (4e-18) and evaluates Phi, W and the
// FP64 deltas only for the triples inside it (about 1-2 % of them).
// Roofline: tensor pipe for Y (about 74 kflop issued per pair per split pass),
// L2 bandwidth for gathering the U_q2 rows, FP32/FP64 ALU for the screen.
#include <algorithm>
#include <cub/cub.cuh>
#include <cuda_bf16.h>

#include "spring_internal.cuh"
#include "tc.cuh"

namespace spring {
namespace {

constexpr int NMODE = 6;     // Ndof of the two-atom cell
constexpr int KP = 48;       // padded K: Re/Im of (N2, c), 2 * 3 * Na3 <= 48
constexpr int EPT = 16;      // pairs per tile: one 8-row core-matrix group each (rows 8e .. 8e+5 of 128)
constexpr int BROWS = 36;    // used B rows
constexpr int QSMAX = 12 + 6 * 9;  // packed phonons of one grid point: omega[6], 1/omega[6], nBE[T][6]
constexpr int Q0ROW = 50;    // packed q0 row in doubles (48 used; 400-byte stride spreads the banks)
constexpr uint32_t LBO = 128, SBO = (KP / 8) * 128;
constexpr int A_BYTES = (128 / 8) * SBO;  // 12288
constexpr int B_BYTES = (48 / 8) * SBO;   // 4608
constexpr int AIMG = 8 * KP;              // bf16 elements of one (q, mu, hi/lo) A image: 8 rows x 48 (768 bytes)
constexpr int BIMG = 48 * KP;             // bf16 elements of one (q1, mu, hi/lo) B image (4608 bytes)
constexpr int AREC = 4 * AIMG * 2 / 8;    // doubles taken by the four A images of a grid record (384)
constexpr int PBMAX = QSMAX * 8 + 4 * 768;  // bytes of the largest pair block in shared memory
constexpr double EXP_CUT = 40.0;
constexpr long long MAX_SPINS = 1LL << 26;

// bf16 hi/lo split of an FP64 value
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    const float f = (float)x;
    hi = __float2bfloat16_rn(f);
    lo = __float2bfloat16_rn(f - __bfloat162float(hi));
}

// U of one grid point, basis mu, slot k = N*3 + b, branch s (FP64)
__device__ __forceinline__ double2 u_value(int q, int mu, int k, int s, int na, const double* __restrict__ posr,
                                          const int* __restrict__ btyp, const double* __restrict__ mrs,
                                          const double* __restrict__ qpnt, const double2* __restrict__ evg) {
    const int N = k / 3, b = k % 3;
    const double* R = posr + ((size_t)mu * na + N) * 3;
    const double qr = qpnt[3 * q] * R[0] + qpnt[3 * q + 1] * R[1] + qpnt[3 * q + 2] * R[2];
    double sn, cs;
    sincos(qr, &sn, &cs);
    const int nu = btyp[mu * na + N];
    const double m = mrs[nu];
    const double2 e = evg[((size_t)q * NMODE + s) * NMODE + nu * 3 + b];
    return make_double2(m * (cs * e.x - sn * e.y), m * (cs * e.y + sn * e.x));
}

// A operand images, stored in the grid records after the packed row (qs doubles): per (hi/lo, mu)
// the 768-byte shared-memory image of one 8-row group of the canonical K-major layout, element
// (row s, k) at (k/8)*64 + s*8 + k%8, rows 6 and 7 zero.  Hi parts first, so a BF16 launch copies
// the row and the two hi images as one block.
__global__ void k_tc_tab_a(int nq, int na, int qs, const double* __restrict__ posr, const int* __restrict__ btyp,
                           const double* __restrict__ mrs, const double* __restrict__ qpnt,
                           const double2* __restrict__ evg, double* __restrict__ rec) {
    const int KR = 3 * na;
    const long long total = (long long)nq * 2 * 8 * KP;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % KP), s = (int)((i / KP) % 8), mu = (int)((i / (KP * 8)) % 2);
        const int q = (int)(i / (KP * 8 * 2));
        double x = 0.0;
        if (k < 2 * KR && s < NMODE) {
            const double2 u = u_value(q, mu, k % KR, s, na, posr, btyp, mrs, qpnt, evg);
            x = k < KR ? u.x : u.y;
        }
        __nv_bfloat16 hi, lo;
        split_bf16(x, hi, lo);
        __nv_bfloat16* img = reinterpret_cast<__nv_bfloat16*>(rec + (size_t)q * (qs + AREC) + qs);
        const int off = mu * AIMG + (k / 8) * 64 + s * 8 + k % 8;
        img[off] = hi;
        img[2 * AIMG + off] = lo;
    }
}

// B table: per (q1, hi/lo, mu) the 4608-byte shared-memory image of the 48 x 48 B operand in the
// canonical K-major layout: element (row n, k) at (n/8)*384 + (k/8)*64 + (n%8)*8 + k%8; rows 36-47
// and the K padding are zero.  Hi parts first.  One CTA per (q1, mu).
__device__ __forceinline__ size_t bimg(int n, int k) {
    return (size_t)(n / 8) * 384 + (size_t)(k / 8) * 64 + (n % 8) * 8 + k % 8;
}
__global__ void __launch_bounds__(128) k_tc_tab_b(int nq, int na, const double* __restrict__ fc3,
                                                  const double* __restrict__ posr, const int* __restrict__ btyp,
                                                  const double* __restrict__ mrs, const double* __restrict__ qpnt,
                                                  const double2* __restrict__ evg, __nv_bfloat16* __restrict__ tab) {
    __shared__ double2 sU[24 * NMODE];  // [N b][s]
    const int q = blockIdx.x / 2, mu = blockIdx.x % 2;
    const int KR = 3 * na;
    for (int i = threadIdx.x; i < KR * NMODE; i += blockDim.x)
        sU[i] = u_value(q, mu, i / NMODE, i % NMODE, na, posr, btyp, mrs, qpnt, evg);
    __syncthreads();
    const double* f = fc3 + (size_t)mu * na * na * 27;
    __nv_bfloat16* out = tab + (size_t)q * 4 * BIMG + mu * BIMG;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
    for (int i = threadIdx.x; i < 48 * KP; i += blockDim.x) {  // zero rows 36-47 and the K padding
        const int n = i / KP, k = i % KP;
        if (n >= BROWS || k >= 2 * KR) {
            out[bimg(n, k)] = zero;
            out[2 * BIMG + bimg(n, k)] = zero;
        }
    }
    for (int i = threadIdx.x; i < 18 * KR; i += blockDim.x) {
        const int r = i / KR, k2 = i % KR;  // r = a*6 + s1, k2 = N2*3 + c
        const int al = r / NMODE, s1 = r % NMODE, N2 = k2 / 3, ga = k2 % 3;
        double zr = 0.0, zi = 0.0;
        for (int k1 = 0; k1 < KR; ++k1) {
            const int N1 = k1 / 3, be = k1 % 3;
            const double fv = f[((size_t)N1 * na + N2) * 27 + (al * 3 + be) * 3 + ga];
            const double2 u = sU[k1 * NMODE + s1];
            zr = fma(fv, u.x, zr);
            zi = fma(fv, u.y, zi);
        }
        __nv_bfloat16 h, l;
        // row r (Re output): [Re Z | -Im Z];  row 18 + r (Im output): [Im Z | Re Z]
        split_bf16(zr, h, l);
        out[bimg(r, k2)] = h;                  out[2 * BIMG + bimg(r, k2)] = l;
        out[bimg(18 + r, KR + k2)] = h;        out[2 * BIMG + bimg(18 + r, KR + k2)] = l;
        split_bf16(-zi, h, l);
        out[bimg(r, KR + k2)] = h;             out[2 * BIMG + bimg(r, KR + k2)] = l;
        split_bf16(zi, h, l);
        out[bimg(18 + r, k2)] = h;             out[2 * BIMG + bimg(18 + r, k2)] = l;
    }
}

// Packed q0 rows (Q0ROW doubles): e0' = m_mu^-1/2 e0(mu a, s0) as float2 [s0][row] (288 bytes), then
// omega0[6] and 1/omega0[6].
__global__ void k_tc_q0tab(int nq0, const double2* __restrict__ ev0, const double* __restrict__ om0,
                           const double* __restrict__ ob0, const double* __restrict__ mrs, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nq0 * 48; i += gridDim.x * blockDim.x) {
        const int q = i / 48, k = i % 48;
        double* row = out + (size_t)q * Q0ROW;
        if (k < 36) {
            const double2 e = ev0[(size_t)q * 36 + k];
            const double m = mrs[(k % NMODE) / 3];
            reinterpret_cast<float2*>(row)[k] = make_float2((float)(m * e.x), (float)(m * e.y));
        } else if (k < 42) {
            row[k] = om0[(size_t)q * NMODE + k - 36];
        } else {
            row[k] = ob0[(size_t)q * NMODE + k - 42];
        }
    }
}

// Packed grid rows at the head of each grid record (qs = 12 + 6 x the kernel's temperature bucket
// doubles): omega[6], 1/omega[6], nBE[T][6] (zero beyond the n_temps in use).
__global__ void k_tc_qtab(int nq, int nT, int qs, const double* __restrict__ omg, const double* __restrict__ obg,
                          const double* __restrict__ nbeg, double* __restrict__ rec) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)nq * qs;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / qs), k = (int)(i % qs);
        double v;
        if (k < 6) v = omg[(size_t)q * NMODE + k];
        else if (k < 12) v = obg[(size_t)q * NMODE + k - 6];
        else if ((k - 12) / NMODE < nT) v = nbeg[((size_t)((k - 12) / NMODE) * nq + q) * NMODE + (k - 12) % NMODE];
        else v = 0.0;
        rec[(size_t)q * (qs + AREC) + k] = v;
    }
}

// ------------------------------------------------------------------ tiles
__global__ void k_tc_keys(int n, int p0, const int2* __restrict__ pairs, int* __restrict__ keys, int* __restrict__ vals,
                          int* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int g1 = pairs[p0 + i].x;
        keys[i] = g1;
        vals[i] = p0 + i;
        atomicAdd(&cnt[g1], 1);
    }
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
// Entry records in q1 order: (q0, q2, pair-folding weight, q0 is Gamma).
__global__ void k_tc_entrec(int n, const int* __restrict__ entries, const int2* __restrict__ pairs,
                            const int* __restrict__ pair_q0, const int* __restrict__ irr_int, int4* __restrict__ rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int pi = entries[i];
        const int2 pq = pairs[pi];
        const int q0 = pair_q0[pi];
        const int g0 = irr_int[3 * q0] == 0 && irr_int[3 * q0 + 1] == 0 && irr_int[3 * q0 + 2] == 0;
        rec[i] = make_int4(q0, pq.y, pq.x != pq.y ? 2 : 1, g0);
    }
}

// ------------------------------------------------------------------ main kernel
struct TcArgs {
    int nq, nq0, nT, qs, ntiles, tiles_per_cta;
    int lo[3], hi[3];
    double mfac, half_os2, pre;
};

// One pipeline stage: the operands of one tile and everything its epilogue reads.
struct TcStage {
    // pair blocks, PB bytes apart: q2 row (QS doubles), then the A images [hi, lo][mu] of q2;
    // pair e's images are rows 8e .. 8e+5 of the M = 128 operand (8-row group stride PB)
    alignas(128) uint8_t P[EPT * PBMAX];
    alignas(128) uint8_t B[2 * 2 * B_BYTES];  // [hi, lo][mu]: rows (re/im, a, s1)
    alignas(16) double q0d[EPT][Q0ROW];       // packed q0 rows
    alignas(16) double q1d[QSMAX];            // packed q1 row
    int4 ent[EPT];                            // (q0, q2, weight, q0 is Gamma)
    int q1, ne;
};

// An active mode triple handed from the screening thread to any epilogue thread:
// (Re, Im) Y[mu][a] for its s1, and (pair, s2, s0, s1).
struct QItem {
    float yr[6], yi[6];
    int meta;  // e | s2 << 8 | s0 << 12 | s1 << 16
    int pad[3];
};
constexpr int QCAP = 512;

struct TcSmem {
    TcStage st[2];
    QItem q[QCAP];                  // active triples of the tile being reduced
    alignas(16) int4 pf[2][EPT];    // entry records, prefetched one tile ahead
    alignas(16) int4 trec[4];       // tile records, prefetched two tiles ahead
    alignas(8) uint64_t ready[2], full[2], empty[2], pfb[2], trb[4];
    uint32_t tslot;
    int qn, qmore;
    int abort_e;  // an epilogue wait gave up (set by any epilogue thread, read by all after a barrier)
};

constexpr int EPI_WARPS = 12;      // warps 0-11: epilogue; warps w, w+4, w+8 share TMEM lanes, two s0 each
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int TC_THREADS = EPI_THREADS + 32;  // warp 12: bulk copies and MMA issue

// Warp-specialised, double-buffered.  The producer warp fills stage s with TMA bulk copies of
// ready-made shared-memory images, two per pair (the q2 grid record: packed row + A images; the
// packed q0 row) and two when q1 changes (the B images, the q1 row), completing on ready[s].  At
// its next iteration it first issues that tile's MMAs into the stage's TMEM columns (lane 0,
// committed to full[s]) and then fills the other stage, so the MMAs of tile j overlap the
// epilogue of tile j-1.  The epilogue warps reduce the tile, then arrive on empty[s].  Entry and
// tile records are prefetched ahead on their own mbarriers.
template <int NTM, bool SPLIT>
__global__ void __launch_bounds__(TC_THREADS, 1)
k_v3tc(TcArgs a, const int4* __restrict__ tiles, const int4* __restrict__ entrec, const double* __restrict__ rec,
       const __nv_bfloat16* __restrict__ tabB, const double* __restrict__ q0tab, double* __restrict__ out_lw,
       double* __restrict__ out_p3, int* __restrict__ err) {
    extern __shared__ __align__(128) uint8_t smraw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int H = SPLIT ? 2 : 1;
    constexpr int QS = 12 + 6 * NTM;       // packed grid row (the records are laid out for NTM)
    constexpr int RSD = QS + AREC;         // grid record stride in doubles
    constexpr int PB = QS * 8 + H * 1536;  // pair block bytes: the row and the hi (and lo) A images
    static_assert(PB <= PBMAX && PB % 16 == 0, "pair block");
    const int t0 = blockIdx.x * a.tiles_per_cta;
    const int t1 = min(a.ntiles, t0 + a.tiles_per_cta);
    const int nt = t1 - t0;

    if (tid == 0) {
        S.st[0].q1 = S.st[1].q1 = -1;
        S.abort_e = 0;
        S.qn = S.qmore = 0;
        for (int k = 0; k < 2; ++k) {
            tc::mbar_init(tc::smem_u32(&S.ready[k]), 1);
            tc::mbar_init(tc::smem_u32(&S.full[k]), 1);
            tc::mbar_init(tc::smem_u32(&S.empty[k]), EPI_WARPS);
            tc::mbar_init(tc::smem_u32(&S.pfb[k]), 1);
        }
        for (int k = 0; k < 4; ++k) tc::mbar_init(tc::smem_u32(&S.trb[k]), 1);
        tc::mbar_fence_init();
    }
    if (tid < 2 && tid < nt) S.trec[tid] = tiles[t0 + tid];
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tslot), 256);
    tc::fence_before_sync();
    __syncthreads();
    if (nt > 0 && tid < S.trec[0].z) S.pf[0][tid] = entrec[S.trec[0].y + tid];
    tc::fence_after_sync();
    __syncthreads();
    const uint32_t tm = S.tslot;

    if (warp == EPI_WARPS) {
        // ------------------------------------------------------------ producer warp
        bool abort = false;
        int filled = -1, issued = -1;  // last tile whose copies / MMAs were issued
        for (int j = 0; j <= nt && !abort; ++j) {
            if (j >= 1) {
                // (a) MMAs of tile j-1 once its operands have landed; its TMEM columns were freed when
                // the stage's previous tile (j-3) was drained, which the fill of j-1 waited for
                const int jm = j - 1, s = jm & 1, u = jm >> 1;
                TcStage& G = S.st[s];
                bool ok = true;
                if (lane == 0) {
                    ok = tc::mbar_wait(tc::smem_u32(&S.ready[s]), (uint32_t)(u & 1), MAX_SPINS);
                    if (ok) {
                        tc::fence_after_sync();
                        const uint32_t idesc = tc::idesc_bf16(128, 48);
                        const uint32_t pa = tc::smem_u32(&G.P[QS * 8]), pb = tc::smem_u32(&G.B[0]);
                        for (int mu = 0; mu < 2; ++mu) {
                            const uint32_t d = tm + (uint32_t)(s * 128 + mu * 64);
                            for (int kk = 0; kk < KP / 16; ++kk) {
                                const uint32_t ko = (uint32_t)kk * 2u * LBO;
                                const uint64_t ah = tc::sdesc(pa + mu * 768 + ko, LBO, PB);
                                const uint64_t bh = tc::sdesc(pb + mu * B_BYTES + ko, LBO, SBO);
                                tc::mma_bf16(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                                if (SPLIT) {
                                    const uint64_t al = tc::sdesc(pa + (2 + mu) * 768 + ko, LBO, PB);
                                    const uint64_t bl = tc::sdesc(pb + (2 + mu) * B_BYTES + ko, LBO, SBO);
                                    tc::mma_bf16(d, ah, bl, idesc, 1u);
                                    tc::mma_bf16(d, al, bh, idesc, 1u);
                                }
                            }
                        }
                        tc::mma_commit(tc::smem_u32(&S.full[s]));
                        issued = jm;
                    }
                }
                issued = __shfl_sync(0xffffffffu, issued, 0);
                if (__any_sync(0xffffffffu, !ok)) {
                    if (lane == 0) atomicExch(err, 1);
                    abort = true;
                    break;
                }
            }
            if (j < nt) {
                // (b) fill stage j & 1 with tile j
                const int s = j & 1, u = j >> 1;
                TcStage& G = S.st[s];
                // every lane waits, so each one observes the completed copies it reads or overwrites
                bool ok = true;
                if (u > 0) ok = tc::mbar_wait(tc::smem_u32(&S.empty[s]), (uint32_t)((u - 1) & 1), MAX_SPINS);
                if (ok && j > 0) ok = tc::mbar_wait(tc::smem_u32(&S.pfb[j & 1]), (uint32_t)(((j - 1) >> 1) & 1), MAX_SPINS);
                if (ok && j >= 2) ok = tc::mbar_wait(tc::smem_u32(&S.trb[j & 3]), (uint32_t)(((j - 2) >> 2) & 1), MAX_SPINS);
                if (ok && j + 1 < nt && j >= 1)
                    ok = tc::mbar_wait(tc::smem_u32(&S.trb[(j + 1) & 3]), (uint32_t)(((j - 1) >> 2) & 1), MAX_SPINS);
                if (__any_sync(0xffffffffu, !ok)) {
                    if (lane == 0) atomicExch(err, 1);
                    abort = true;
                    break;
                }
                const int4 tile = S.trec[j & 3];
                const int q1 = tile.x, ne = tile.z;
                const int4* ent = S.pf[j & 1];
                const bool newb = G.q1 != q1;
                if (lane < ne) G.ent[lane] = ent[lane];
                __syncwarp();
                const uint32_t rb = tc::smem_u32(&S.ready[s]);
                if (lane == 0) {
                    G.ne = ne;
                    G.q1 = q1;
                    uint32_t bytes = (uint32_t)ne * (uint32_t)(PB + 384);
                    if (newb) bytes += (uint32_t)(2 * H * B_BYTES + QS * 8);
                    tc::mbar_arrive_tx(rb, bytes);
                }
                __syncwarp();
                if (lane < ne) {
                    const int4 en = ent[lane];
                    tc::bulk_g2s(tc::smem_u32(&G.P[lane * PB]), rec + (size_t)en.y * RSD, (uint32_t)PB, rb);
                    tc::bulk_g2s(tc::smem_u32(&G.q0d[lane][0]), q0tab + (size_t)en.x * Q0ROW, 384u, rb);
                }
                if (newb && lane == 30)
                    tc::bulk_g2s(tc::smem_u32(&G.B[0]), tabB + (size_t)q1 * 4 * BIMG, (uint32_t)(2 * H * B_BYTES), rb);
                if (newb && lane == 31) tc::bulk_g2s(tc::smem_u32(&G.q1d[0]), rec + (size_t)q1 * RSD, (uint32_t)QS * 8u, rb);
                // prefetch: entry records of tile j+1, tile record j+2
                if (lane == 0 && j + 1 < nt) {
                    const int4 nx = S.trec[(j + 1) & 3];
                    const uint32_t pb = tc::smem_u32(&S.pfb[(j + 1) & 1]);
                    tc::mbar_arrive_tx(pb, (uint32_t)nx.z * 16u);
                    tc::bulk_g2s(tc::smem_u32(&S.pf[(j + 1) & 1][0]), entrec + nx.y, (uint32_t)nx.z * 16u, pb);
                }
                if (lane == 0 && j + 2 < nt) {
                    const uint32_t tb = tc::smem_u32(&S.trb[(j + 2) & 3]);
                    tc::mbar_arrive_tx(tb, 16u);
                    tc::bulk_g2s(tc::smem_u32(&S.trec[(j + 2) & 3]), tiles + t0 + j + 2, 16u, tb);
                }
                filled = j;
            }
        }
        if (abort && lane == 0) {
            // Error path: wait (bounded) for the copies and MMAs still in flight before the CTA
            // releases its shared memory and TMEM.
            for (int t = issued + 1; t <= filled; ++t)
                tc::mbar_wait(tc::smem_u32(&S.ready[t & 1]), (uint32_t)((t >> 1) & 1), MAX_SPINS);
            if (filled >= 0 && filled + 1 < nt)
                tc::mbar_wait(tc::smem_u32(&S.pfb[(filled + 1) & 1]), (uint32_t)((filled >> 1) & 1), MAX_SPINS);
            for (int t = max(2, filled + 1); t <= filled + 2 && t < nt; ++t)
                tc::mbar_wait(tc::smem_u32(&S.trb[t & 3]), (uint32_t)(((t - 2) >> 2) & 1), MAX_SPINS);
            if (issued >= 0)
                tc::mbar_wait(tc::smem_u32(&S.full[issued & 1]), (uint32_t)((issued >> 1) & 1), MAX_SPINS);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int wq = warp & 3, grp = warp >> 2;  // lane quarter, s0 pair (2 grp, 2 grp + 1)
        const int e = 4 * wq + lane / 8, s2 = lane % 8;
        const float Rf = (float)(sqrt(EXP_CUT / a.half_os2) * 1.0001 + 1e-3);
        const int etid = tid;  // 0 .. EPI_THREADS-1
        for (int j = 0; j < nt; ++j) {
            const int s = j & 1, u = j >> 1;
            TcStage& G = S.st[s];
            // every thread waits on both barriers: the copies and the accumulator it reads
            if (!(tc::mbar_wait(tc::smem_u32(&S.ready[s]), (uint32_t)(u & 1), MAX_SPINS) &&
                  tc::mbar_wait(tc::smem_u32(&S.full[s]), (uint32_t)(u & 1), MAX_SPINS)))
                S.abort_e = 1;
            tc::named_bar(2, EPI_THREADS);
            if (S.abort_e) {
                if (etid == 0) atomicExch(err, 1);
                break;
            }
            tc::fence_after_sync();
            float y[2][48];
            {
                const uint32_t ta = tm + ((uint32_t)(wq * 32) << 16) + (uint32_t)(s * 128);
                tc::tmem_ld16(ta, y[0]);
                tc::tmem_ld16(ta + 16, y[0] + 16);
                tc::tmem_ld16(ta + 32, y[0] + 32);
                tc::tmem_ld16(ta + 64, y[1]);
                tc::tmem_ld16(ta + 80, y[1] + 16);
                tc::tmem_ld16(ta + 96, y[1] + 32);
                tc::tmem_ld_wait();
            }
            const int ne = G.ne;
            const bool valid = s2 < NMODE && e < ne;
            const int4 en = valid ? G.ent[e] : make_int4(0, 0, 0, 0);
            const bool row_on = valid && s2 >= a.lo[2] && s2 <= a.hi[2] && !(en.y == 0 && s2 < 3);
            const bool gq1 = G.q1 == 0;
            const double* q1d = G.q1d;
            const double* q2d = reinterpret_cast<const double*>(&G.P[(valid ? e : 0) * PB]);
            const double* q0d = G.q0d[valid ? e : 0];
            const double w2 = q2d[valid ? s2 : 0];
            // FP32 screen: bit 6*jj + s1 marks (s0 = 2 grp + jj, s1) inside the delta window
            unsigned act = 0u;
            if (row_on) {
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int s0 = grp * 2 + jj;
                    if (s0 < a.lo[0] || s0 > a.hi[0]) continue;
                    const double w0 = q0d[36 + s0];
                    const float af = (float)(w0 - w2), bf = (float)(w0 + w2);
#pragma unroll
                    for (int s1 = 0; s1 < NMODE; ++s1) {
                        const float w1 = (float)q1d[s1];
                        const bool in = fabsf(af - w1) < Rf || fabsf(af + w1) < Rf || fabsf(bf - w1) < Rf;
                        const bool allowed = s1 >= a.lo[1] && s1 <= a.hi[1] && !(gq1 && s1 < 3);
                        act |= (in && allowed) ? (1u << (jj * NMODE + s1)) : 0u;
                    }
                }
            }
            // Compaction: the screened triples of the whole tile go to a shared queue (several passes if
            // it fills), and all epilogue threads evaluate them one per thread, so the FP64 work runs
            // with full warps; each triple's contribution goes straight to the output.
            for (;;) {
                if (act) {
                    const int n = __popc(act);
                    const int base = atomicAdd(&S.qn, n);
                    for (int i = 0; i < n && base + i < QCAP; ++i) {
                        const int bit = __ffs(act) - 1;
                        act &= act - 1u;
                        const int jj = bit / NMODE, s1 = bit % NMODE;
                        QItem& it = S.q[base + i];
#pragma unroll
                        for (int k = 0; k < 6; ++k) {
                            float r = 0.0f, im = 0.0f;
#pragma unroll
                            for (int c1 = 0; c1 < NMODE; ++c1) {
                                r = (c1 == s1) ? y[k / 3][(k % 3) * NMODE + c1] : r;
                                im = (c1 == s1) ? y[k / 3][18 + (k % 3) * NMODE + c1] : im;
                            }
                            it.yr[k] = r;
                            it.yi[k] = im;
                        }
                        it.meta = e | (s2 << 8) | ((grp * 2 + jj) << 12) | (s1 << 16);
                    }
                    if (act) S.qmore = 1;
                }
                tc::named_bar(2, EPI_THREADS);
                const int cnt = min(S.qn, QCAP);
                for (int i = etid; i < cnt; i += EPI_THREADS) {
                    const QItem& it = S.q[i];
                    const int ie = it.meta & 0xff, is2 = (it.meta >> 8) & 0xf, s0 = (it.meta >> 12) & 0xf,
                              s1 = (it.meta >> 16) & 0xf;
                    const int4 ien = G.ent[ie];
                    const double* p0 = G.q0d[ie];
                    const double* p2 = reinterpret_cast<const double*>(&G.P[ie * PB]);
                    const double w0 = p0[36 + s0], w1d = q1d[s1], w2d = p2[is2];
                    const double d1 = w0 - w1d - w2d, d2 = w0 + w1d - w2d, d3 = w0 - w1d + w2d;
                    const double x1 = a.half_os2 * (d1 * d1), x2 = a.half_os2 * (d2 * d2), x3 = a.half_os2 * (d3 * d3);
                    const double e1 = x1 < EXP_CUT ? a.pre * exp(-x1) : 0.0;
                    const double e2 = x2 < EXP_CUT ? a.pre * exp(-x2) : 0.0;
                    const double e3 = x3 < EXP_CUT ? a.pre * exp(-x3) : 0.0;
                    const double wt = (double)ien.z;
                    const double p3 = e1 + e2 + e3;
                    if (p3 != 0.0) atomicAdd(&out_p3[(size_t)ien.x * NMODE + s0], wt * p3);
                    if (ien.w != 0 && s0 < 3) continue;  // W = 0 for the Gamma acoustic modes of q0
                    const float2* e0 = reinterpret_cast<const float2*>(p0) + s0 * NMODE;
                    float pr = 0.0f, pim = 0.0f;
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const float2 c = e0[k];
                        pr = fmaf(c.x, it.yr[k], fmaf(-c.y, it.yi[k], pr));
                        pim = fmaf(c.x, it.yi[k], fmaf(c.y, it.yr[k], pim));
                    }
                    const double W = (double)(pr * pr + pim * pim) * (p0[42 + s0] * p2[6 + is2] * q1d[6 + s1]) * a.mfac;
                    const double we1 = wt * W * e1, wf2 = wt * W * (e2 - e3);
                    for (int T = 0; T < a.nT; ++T) {
                        const double n1 = q1d[12 + 6 * T + s1], n2 = p2[12 + 6 * T + is2];
                        const double v = ((n1 + n2 + 1.0) * we1) + ((n1 - n2) * wf2);
                        if (v != 0.0) atomicAdd(&out_lw[((size_t)T * a.nq0 + ien.x) * NMODE + s0], v);
                    }
                }
                const int more = S.qmore;
                tc::named_bar(2, EPI_THREADS);
                if (etid == 0) {
                    S.qn = 0;
                    S.qmore = 0;
                }
                tc::named_bar(2, EPI_THREADS);
                if (!more) break;
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(tc::smem_u32(&S.empty[s]));
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tm, 256);
}

template <int NTM, bool SPLIT>
int launch_tc(spring_ctx* c, TcArgs a, double* lw, double* p3) {
    const size_t smem = sizeof(TcSmem);
    if (smem > 227 * 1024) return fail(c, SPRING_ERR_UNSUPPORTED, "tensor-core V3 needs %zu bytes of shared memory", smem);
    cudaFuncSetAttribute(k_v3tc<NTM, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    const int ctas = std::max(1, std::min(a.ntiles, sms));
    a.tiles_per_cta = (a.ntiles + ctas - 1) / ctas;
    const int grid = (a.ntiles + a.tiles_per_cta - 1) / a.tiles_per_cta;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc: injected launch failure");
    k_v3tc<NTM, SPLIT><<<grid, TC_THREADS, smem, c->stream>>>(
        a, c->d_tc_tiles.p, c->d_tc_rec.p, c->d_tc_q.p, reinterpret_cast<const __nv_bfloat16*>(c->d_tc_b.p),
        c->d_tc_q0.p, lw, p3, c->d_tc_err.p);
    return launch_check(c, SPLIT ? "k_v3tc<bf16x3>" : "k_v3tc<bf16>");
}

// Pairs of [p0, p1) sorted by q1 (stable radix sort), cut into tiles of at most EPT
// pairs of one q1, with the entry record of every sorted pair.
int build_tiles(spring_ctx* c, int p0, int p1) {
    const PairSet& ps = c->ps_irr;
    if (c->tc_gen == ps.gen && c->tc_p0 == p0 && c->tc_p1 == p1) return SPRING_OK;
    const int n = p1 - p0, nq = c->nq;
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
    if (rc == SPRING_OK) rc = zero(c, cnt.p, sizeof(int) * nq, "tile counts");
    const int threads = 256;
    if (rc == SPRING_OK && n > 0) {
        if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "tiles: injected launch failure");
        else {
            k_tc_keys<<<std::min((n + threads - 1) / threads, 148 * 8), threads, 0, c->stream>>>(n, p0, ps.pairs.p, keys.p,
                                                                                                   vals.p, cnt.p);
            rc = launch_check(c, "k_tc_keys");
        }
    }
    int bits = 1;
    while ((1 << bits) < nq) ++bits;
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
    int last[2] = {0, 0};
    if (rc == SPRING_OK) rc = d2h(c, &last[0], toff.p + nq - 1, sizeof(int), "tile count");
    if (rc == SPRING_OK) rc = d2h(c, &last[1], ntl.p + nq - 1, sizeof(int), "tile count");
    const int ntiles = last[0] + last[1];
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
                n, c->d_tc_entries.p, ps.pairs.p, ps.pair_q0.p, c->d_irr_int.p, c->d_tc_rec.p);
            rc = launch_check(c, "k_tc_entrec");
        }
    }
    if (rc != SPRING_OK) return rc;
    c->tc_ntiles = ntiles;
    c->tc_gen = ps.gen;
    c->tc_p0 = p0;
    c->tc_p1 = p1;
    return SPRING_OK;
}

}  // namespace

int run_v3tc_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3,
                   bool* handled) {
    *handled = false;
    if (c->nb != 2 || c->na3 > 8 || c->nT > 9) return SPRING_OK;
    const PairSet& ps = c->ps_irr;
    const int p0 = ps.h_pairoff[q0_first], p1 = ps.h_pairoff[q0_first + n_q0];
    *handled = true;
    if (p1 == p0) return SPRING_OK;
    const int nq = c->nq;
    const int ntm = c->nT == 1 ? 1 : (c->nT <= 3 ? 3 : 9);  // temperature bucket of the kernel instance
    const int qs = 12 + 6 * ntm;
    SPRING_CHECK(dalloc(c, c->d_tc_b, (size_t)nq * 4 * BIMG, "V3 B table"));
    SPRING_CHECK(dalloc(c, c->d_tc_q0, (size_t)c->nq0 * Q0ROW, "V3 q0 rows"));
    SPRING_CHECK(dalloc(c, c->d_tc_q, (size_t)nq * (qs + AREC), "V3 grid records"));
    SPRING_CHECK(dalloc(c, c->d_tc_err, 1, "V3 status"));
    SPRING_CHECK(zero(c, c->d_tc_err.p, sizeof(int), "V3 status"));
    SPRING_CHECK(build_tiles(c, p0, p1));
    const int threads = 256;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
    {
        const long long tot = (long long)nq * 2 * 8 * KP;
        k_tc_tab_a<<<(int)std::min<long long>((tot + threads - 1) / threads, 148LL * 16), threads, 0, c->stream>>>(
            nq, c->na3, qs, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p, c->d_qpnt.p, c->ph_grid.evec.p,
            c->d_tc_q.p);
        SPRING_CHECK(launch_check(c, "k_tc_tab_a"));
    }
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
    k_tc_tab_b<<<nq * 2, 128, 0, c->stream>>>(nq, c->na3, c->d_fc3.p, c->d_fc3_posr.p, c->d_fc3_btyp.p, c->d_mass_rs.p,
                                               c->d_qpnt.p, c->ph_grid.evec.p,
                                               reinterpret_cast<__nv_bfloat16*>(c->d_tc_b.p));
    SPRING_CHECK(launch_check(c, "k_tc_tab_b"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
    k_tc_q0tab<<<std::max(1, std::min((c->nq0 * 48 + threads - 1) / threads, 148 * 4)), threads, 0, c->stream>>>(
        c->nq0, c->ph_irr.evec.p, c->ph_irr.omega.p, c->ph_irr.oneby.p, c->d_mass_rs.p, c->d_tc_q0.p);
    SPRING_CHECK(launch_check(c, "k_tc_q0tab"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "v3tc tables: injected launch failure");
    k_tc_qtab<<<std::max(1, (int)std::min<long long>(((long long)nq * qs + threads - 1) / threads, 148LL * 8)), threads,
                0, c->stream>>>(nq, c->nT, qs, c->ph_grid.omega.p, c->ph_grid.oneby.p, c->ph_grid.nbe.p, c->d_tc_q.p);
    SPRING_CHECK(launch_check(c, "k_tc_qtab"));

    TcArgs a{};
    a.nq = nq;
    a.nq0 = c->nq0;
    a.nT = c->nT;
    a.qs = qs;
    a.ntiles = c->tc_ntiles;
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = pol.lo[k];
        a.hi[k] = pol.hi[k];
    }
    a.mfac = host_constants().Sctr3THz2 / double(nq);
    const double os = 1.0 / sigma;
    a.half_os2 = 0.5 * (os * os);
    a.pre = os * ONEBYSQRT2PI;
    const bool split = c->precision == SPRING_BF16X3;
    int rc;
    if (c->nT == 1) rc = split ? launch_tc<1, true>(c, a, d_lw, d_p3) : launch_tc<1, false>(c, a, d_lw, d_p3);
    else if (c->nT <= 3) rc = split ? launch_tc<3, true>(c, a, d_lw, d_p3) : launch_tc<3, false>(c, a, d_lw, d_p3);
    else rc = split ? launch_tc<9, true>(c, a, d_lw, d_p3) : launch_tc<9, false>(c, a, d_lw, d_p3);
    SPRING_CHECK(rc);
    int herr = 0;
    SPRING_CHECK(d2h(c, &herr, c->d_tc_err.p, sizeof(int), "V3 status"));
    if (herr) return fail(c, SPRING_ERR_CUDA, "tensor-core V3: an mbarrier wait timed out");
    return SPRING_OK;
}

}  // namespace spring
