// The surrogate network of the screened four-phonon path: 5 -> 128 -> 128 -> 128 -> 1,
// SiLU after every hidden layer, trained on the device in FP32 with Adam on a
// mean-squared-error loss, evaluated in FP32 or with BF16-rounded weights and
// activations.  No counterpart in the reference (which computes every
// four-phonon rate exactly); its error is measured against the exact path.
//
// Kernels: a tiled FP32 GEMM C = op(A) op(B) (+ bias) used for the forward pass
// (Z = A W^T + b), the weight gradients (dZ^T A) and the backpropagated
// activations (dZ W); element-wise SiLU and its derivative; the loss; a
// column sum for the bias gradients; Adam; and the BF16 inference kernel on
// the tensor cores (k_mlp_bf16, mma.sync BF16 with FP32 accumulation).  Parameters are one flat FP32 vector:
// W1 (128x5, row-major), b1, W2 (128x128), b2, W3, b3, W4 (1x128), b4.
// Roofline: tiny GEMMs (B x 128 x 128), latency- and launch-bound; the data of a
// training run fits in L2.
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>
#include <numeric>
#include <random>
#include <vector>

#include "spring_internal.cuh"

namespace spring {
namespace {

constexpr int NL = 4;
constexpr int SZ[NL + 1] = {SPRING_MLP_INPUTS, 128, 128, 128, 1};
constexpr int TILE = 32, KT = 16;

int w_off(int l) {  // offset of W_l (l = 0..3) in the flat vector
    int k = 0;
    for (int i = 0; i < l; ++i) k += SZ[i + 1] * SZ[i] + SZ[i + 1];
    return k;
}
int b_off(int l) { return w_off(l) + SZ[l + 1] * SZ[l]; }

// C[M x N] = op(A)[M x K] op(B)[K x N] (+ bias[N]); A(i,k) = TA ? A[k*lda+i] : A[i*lda+k],
// B(k,j) = TB ? B[j*ldb+k] : B[k*ldb+j].  256 threads, a 32 x 32 tile, 2 x 2 outputs per thread.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                               const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                               const float* __restrict__ bias) {
    __shared__ float As[KT][TILE + 1];
    __shared__ float Bs[KT][TILE + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.y * TILE, j0 = blockIdx.x * TILE;
    float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
    for (int k0 = 0; k0 < K; k0 += KT) {
        for (int t = threadIdx.x; t < KT * TILE; t += blockDim.x) {
            const int kk = t / TILE, ii = t % TILE;
            const int i = i0 + ii, k = k0 + kk;
            As[kk][ii] = (i < M && k < K) ? (TA ? A[(size_t)k * lda + i] : A[(size_t)i * lda + k]) : 0.f;
            const int j = j0 + ii;
            Bs[kk][ii] = (j < N && k < K) ? (TB ? B[(size_t)j * ldb + k] : B[(size_t)k * ldb + j]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KT; ++kk) {
            const float a0 = As[kk][ty], a1 = As[kk][ty + 16];
            const float b0 = Bs[kk][tx], b1 = Bs[kk][tx + 16];
            acc[0][0] = fmaf(a0, b0, acc[0][0]);
            acc[0][1] = fmaf(a0, b1, acc[0][1]);
            acc[1][0] = fmaf(a1, b0, acc[1][0]);
            acc[1][1] = fmaf(a1, b1, acc[1][1]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
            if (i < M && j < N) C[(size_t)i * ldc + j] = acc[a][b] + (bias ? bias[j] : 0.f);
        }
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

__global__ void k_silu(int n, const float* __restrict__ z, float* __restrict__ a, int round_bf16) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = z[i] * sigm(z[i]);
        a[i] = round_bf16 ? __bfloat162float(__float2bfloat16_rn(v)) : v;
    }
}
__global__ void k_silu_bwd(int n, const float* __restrict__ z, const float* __restrict__ da, float* __restrict__ dz) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float s = sigm(z[i]);
        dz[i] = da[i] * s * (1.0f + z[i] * (1.0f - s));
    }
}
__global__ void k_round_bf16(int n, const float* __restrict__ x, float* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = __bfloat162float(__float2bfloat16_rn(x[i]));
}
// d loss / d out = 2 (out - y) / n; loss += (out - y)^2 / n
__global__ void k_mse(int n, const float* __restrict__ out, const float* __restrict__ y, float* __restrict__ dout,
                      float* __restrict__ loss) {
    float acc = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float r = out[i] - y[i];
        dout[i] = 2.0f * r / n;
        acc += r * r / n;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.f) atomicAdd(loss, acc);
}
__global__ void k_colsum(int M, int N, const float* __restrict__ d, float* __restrict__ g) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int i = 0; i < M; ++i) s += d[(size_t)i * N + j];
        g[j] = s;
    }
}
__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        m[i] = b1 * m[i] + (1.f - b1) * gi;
        v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
        p[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
    }
}
__global__ void k_gather(int nb, int in, const int* __restrict__ idx, const float* __restrict__ X,
                         const float* __restrict__ y, float* __restrict__ Xb, float* __restrict__ yb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb * in; i += gridDim.x * blockDim.x) {
        const int r = i / in, c = i % in, src = idx[r];
        Xb[i] = X[(size_t)src * in + c];
        if (c == 0) yb[r] = y[src];
    }
}

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8)); }

template <bool TA, bool TB>
int gemm(spring_ctx* c, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
         const float* bias) {
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "mlp: injected launch failure");
    dim3 grid((N + TILE - 1) / TILE, (M + TILE - 1) / TILE);
    k_sgemm<TA, TB><<<grid, 256, 0, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, bias);
    return launch_check(c, "k_sgemm");
}

#define MLP_LAUNCH(name, n, ...)                                                                  \
    do {                                                                                          \
        if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "mlp: injected launch failure"); \
        name<<<blocks_for(n), 256, 0, c->stream>>>(__VA_ARGS__);                                  \
        SPRING_CHECK(launch_check(c, #name));                                                     \
    } while (0)

// Activation buffers for batches of up to `nb` rows: Z_l and A_l of every layer, two gradient buffers.
int ensure_buffers(spring_ctx* c, int nb) {
    Mlp& m = c->mlp;
    if (m.cap >= nb) return SPRING_OK;
    size_t per = 0;
    for (int l = 1; l <= NL; ++l) per += 2 * (size_t)SZ[l];
    per += 2 * 128 + SZ[0] + 2;
    SPRING_CHECK(dalloc(c, m.act, per * nb, "network activations"));
    m.cap = nb;
    return SPRING_OK;
}

struct Bufs {
    float *x, *y, *z[NL + 1], *a[NL + 1], *d0, *d1;
};
Bufs carve(spring_ctx* c, int nb) {
    Bufs b{};
    float* p = c->mlp.act.p;
    b.x = p; p += (size_t)nb * SZ[0];
    b.y = p; p += nb;
    b.a[0] = b.x;
    for (int l = 1; l <= NL; ++l) {
        b.z[l] = p; p += (size_t)nb * SZ[l];
        b.a[l] = p; p += (size_t)nb * SZ[l];
    }
    b.d0 = p; p += (size_t)nb * 128;
    b.d1 = p; p += (size_t)nb * 128;
    return b;
}

// ---- BF16 inference on the tensor cores: the whole network per warp, in registers.
// mma.sync m16n8k16 (BF16 operands, FP32 accumulation): a warp takes 16 rows; each hidden layer is
// 16 column tiles x 8 K steps of MMAs with the weights (BF16, row-major W[out][in] in shared memory)
// as the B operand; the FP32 accumulators get the bias and SiLU and are packed to BF16 as the next
// layer's A fragments (the C layout of two adjacent 8-column tiles is the A layout of one 16-wide K
// step).  The input layer pads K 5 -> 16, the output layer N 1 -> 8.
constexpr int MW = 4;  // warps per CTA (64 rows)
struct MlpBf16Smem {
    __nv_bfloat16 w1[128][16];
    __nv_bfloat16 w2[128][128 + 8];  // rows padded by 16 bytes: conflict-free B fragment loads
    __nv_bfloat16 w3[128][128 + 8];
    __nv_bfloat16 w4[8][128 + 8];
    float b[3][128];
    float b4;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One hidden layer of K = 16 * KT inputs: acc[16 tiles][4] = A W^T (+ bias, SiLU) -> A fragments.
template <int KT>
__device__ __forceinline__ void mlp_layer(const uint32_t (&a)[KT][4], const __nv_bfloat16* w, int ldw,
                                          const float* bias, uint32_t (&out)[8][4], int g, int t) {
    float acc[16][4];
#pragma unroll
    for (int n = 0; n < 16; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt)
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const __nv_bfloat16* row = w + (size_t)(8 * n + g) * ldw + 16 * kt + 2 * t;
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + 8);
            mma_bf16_16816(acc[n], a[kt], b0, b1);
        }
#pragma unroll
    for (int n = 0; n < 16; ++n) {
        const float c0 = bias[8 * n + 2 * t], c1 = bias[8 * n + 2 * t + 1];
        float v[4] = {acc[n][0] + c0, acc[n][1] + c1, acc[n][2] + c0, acc[n][3] + c1};
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = v[i] * (1.0f / (1.0f + expf(-v[i])));
        // C tile n -> A step n / 2: even tiles give a0a1 / a2a3, odd tiles a4a5 / a6a7
        out[n / 2][(n & 1) * 2 + 0] = pack_bf16(v[0], v[1]);
        out[n / 2][(n & 1) * 2 + 1] = pack_bf16(v[2], v[3]);
    }
}

__global__ void __launch_bounds__(MW * 32) k_mlp_bf16(int n, const float* __restrict__ X, const float* __restrict__ P,
                                                      int o1, int o2, int o3, int o4, float* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char mlp_sm[];
    MlpBf16Smem& S = *reinterpret_cast<MlpBf16Smem*>(mlp_sm);
    const int tid = threadIdx.x;
    for (int i = tid; i < 128 * 16; i += blockDim.x) {
        const int r = i / 16, k = i % 16;
        S.w1[r][k] = __float2bfloat16_rn(k < SPRING_MLP_INPUTS ? P[o1 + r * SPRING_MLP_INPUTS + k] : 0.f);
    }
    for (int i = tid; i < 128 * 128; i += blockDim.x) {
        const int r = i / 128, k = i % 128;
        S.w2[r][k] = __float2bfloat16_rn(P[o2 + i]);
        S.w3[r][k] = __float2bfloat16_rn(P[o3 + i]);
    }
    for (int i = tid; i < 8 * 128; i += blockDim.x) {
        const int r = i / 128, k = i % 128;
        S.w4[r][k] = __float2bfloat16_rn(r == 0 ? P[o4 + k] : 0.f);
    }
    for (int i = tid; i < 3 * 128; i += blockDim.x) {
        const int l = i / 128, j = i % 128;
        const int ob = (l == 0 ? o1 + 128 * SPRING_MLP_INPUTS : (l == 1 ? o2 : o3) + 128 * 128);
        S.b[l][j] = P[ob + j];
    }
    if (tid == 0) S.b4 = P[o4 + 128];
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    for (int r0 = (blockIdx.x * MW + warp) * 16; r0 < n; r0 += gridDim.x * MW * 16) {
        // input fragment: rows r0 + g and r0 + g + 8, columns 2t, 2t + 1 (the rest of K is zero)
        uint32_t a0[1][4];
        float x[2][2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int row = r0 + g + 8 * h, col = 2 * t + c;
                x[h][c] = (row < n && col < SPRING_MLP_INPUTS) ? X[(size_t)row * SPRING_MLP_INPUTS + col] : 0.f;
            }
        a0[0][0] = pack_bf16(x[0][0], x[0][1]);
        a0[0][1] = pack_bf16(x[1][0], x[1][1]);
        a0[0][2] = 0u;  // columns 8 .. 15
        a0[0][3] = 0u;
        uint32_t h1[8][4], h2[8][4];
        mlp_layer<1>(a0, &S.w1[0][0], 16, S.b[0], h1, g, t);
        mlp_layer<8>(h1, &S.w2[0][0], 128 + 8, S.b[1], h2, g, t);
        mlp_layer<8>(h2, &S.w3[0][0], 128 + 8, S.b[2], h1, g, t);
        // output layer: one column (a tile of 8, the other weights zero)
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < 8; ++kt) {
            const __nv_bfloat16* row = &S.w4[g][16 * kt + 2 * t];
            mma_bf16_16816(acc, h1[kt], *reinterpret_cast<const uint32_t*>(row),
                           *reinterpret_cast<const uint32_t*>(row + 8));
        }
        if (t == 0) {  // column 0 of rows g and g + 8
            if (r0 + g < n) y[r0 + g] = acc[0] + S.b4;
            if (r0 + g + 8 < n) y[r0 + g + 8] = acc[2] + S.b4;
        }
    }
}

// forward over nb rows already in b.x; output in b.z[NL] (and b.a[NL])
int forward(spring_ctx* c, const Bufs& b, int nb, const float* params, int round_bf16) {
    for (int l = 1; l <= NL; ++l) {
        const int in = SZ[l - 1], out = SZ[l];
        SPRING_CHECK((gemm<false, true>(c, nb, out, in, b.a[l - 1], in, params + w_off(l - 1), in, b.z[l], out,
                                        params + b_off(l - 1))));
        if (l < NL) MLP_LAUNCH(k_silu, (long long)nb * out, nb * out, b.z[l], b.a[l], round_bf16);
    }
    return SPRING_OK;
}

// loss and gradient (into m.g) over nb rows in b.x / b.y
int backward(spring_ctx* c, const Bufs& b, int nb, float* d_loss) {
    Mlp& m = c->mlp;
    const float* P = m.p.p;
    float* G = m.g.p;
    MLP_LAUNCH(k_mse, nb, nb, b.z[NL], b.y, b.d0, d_loss);
    float* dz = b.d0;
    float* spare = b.d1;
    for (int l = NL; l >= 1; --l) {
        const int in = SZ[l - 1], out = SZ[l];
        SPRING_CHECK((gemm<true, false>(c, out, in, nb, dz, out, b.a[l - 1], in, G + w_off(l - 1), in, nullptr)));
        MLP_LAUNCH(k_colsum, out, nb, out, dz, G + b_off(l - 1));
        if (l > 1) {
            SPRING_CHECK((gemm<false, false>(c, nb, in, out, dz, out, P + w_off(l - 1), in, spare, in, nullptr)));
            MLP_LAUNCH(k_silu_bwd, (long long)nb * in, nb * in, b.z[l - 1], spare, spare);
            std::swap(dz, spare);
        }
    }
    return SPRING_OK;
}

}  // namespace

int mlp_num_params() { return w_off(NL); }

int run_mlp_init(spring_ctx* c, unsigned long long seed) {
    const int n = mlp_num_params();
    std::vector<float> p(n, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < NL; ++l) {  // He-uniform weights, zero biases
        const int in = SZ[l], out = SZ[l + 1];
        const float lim = std::sqrt(6.0f / in) * (l == NL - 1 ? 0.5f : 1.0f);
        std::uniform_real_distribution<float> u(-lim, lim);
        for (int k = 0; k < out * in; ++k) p[w_off(l) + k] = u(rng);
    }
    return run_mlp_set(c, p.data());
}

int run_mlp_set(spring_ctx* c, const float* params) {
    Mlp& m = c->mlp;
    const int n = mlp_num_params();
    SPRING_CHECK(dalloc(c, m.p, n, "network parameters"));
    SPRING_CHECK(dalloc(c, m.g, n, "network gradient"));
    SPRING_CHECK(dalloc(c, m.m, n, "Adam moments"));
    SPRING_CHECK(dalloc(c, m.v, n, "Adam moments"));
    SPRING_CHECK(dalloc(c, m.scal, 1, "loss"));
    SPRING_CHECK(h2d(c, m.p.p, params, sizeof(float) * n, "network parameters"));
    SPRING_CHECK(zero(c, m.m.p, sizeof(float) * n, "Adam moments"));
    SPRING_CHECK(zero(c, m.v.p, sizeof(float) * n, "Adam moments"));
    m.step = 0;
    m.set = true;
    return SPRING_OK;
}

int run_mlp_loss_grad(spring_ctx* c, int n, const float* hX, const float* hy, float* loss, float* grad) {
    SPRING_CHECK(ensure_buffers(c, n));
    Bufs b = carve(c, n);
    SPRING_CHECK(h2d(c, b.x, hX, sizeof(float) * n * SZ[0], "network inputs"));
    SPRING_CHECK(h2d(c, b.y, hy, sizeof(float) * n, "network targets"));
    SPRING_CHECK(zero(c, c->mlp.scal.p, sizeof(float), "loss"));
    SPRING_CHECK(forward(c, b, n, c->mlp.p.p, 0));
    SPRING_CHECK(backward(c, b, n, c->mlp.scal.p));
    if (loss) SPRING_CHECK(d2h(c, loss, c->mlp.scal.p, sizeof(float), "loss"));
    if (grad) SPRING_CHECK(d2h(c, grad, c->mlp.g.p, sizeof(float) * mlp_num_params(), "network gradient"));
    return SPRING_OK;
}

int run_mlp_train(spring_ctx* c, int n, const float* hX, const float* hy, int epochs, int batch, float lr,
                  unsigned long long seed, float* epoch_loss) {
    Mlp& m = c->mlp;
    const int np = mlp_num_params();
    batch = std::min(batch, n);
    DBuf<float> X, y;
    DBuf<int> idx;
    int rc = dalloc(c, X, (size_t)n * SZ[0], "training inputs");
    if (rc == SPRING_OK) rc = dalloc(c, y, n, "training targets");
    if (rc == SPRING_OK) rc = dalloc(c, idx, n, "training order");
    if (rc == SPRING_OK) rc = ensure_buffers(c, batch);
    if (rc == SPRING_OK) rc = h2d(c, X.p, hX, sizeof(float) * n * SZ[0], "training inputs");
    if (rc == SPRING_OK) rc = h2d(c, y.p, hy, sizeof(float) * n, "training targets");
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    Bufs b = carve(c, batch);
    for (int ep = 0; rc == SPRING_OK && ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        rc = h2d(c, idx.p, order.data(), sizeof(int) * n, "training order");
        if (rc == SPRING_OK) rc = zero(c, m.scal.p, sizeof(float), "loss");
        int nbat = 0;
        for (int s0 = 0; rc == SPRING_OK && s0 + batch <= n; s0 += batch, ++nbat) {
            auto body = [&]() -> int {
                MLP_LAUNCH(k_gather, (long long)batch * SZ[0], batch, SZ[0], idx.p + s0, X.p, y.p, b.x, b.y);
                SPRING_CHECK(forward(c, b, batch, m.p.p, 0));
                SPRING_CHECK(backward(c, b, batch, m.scal.p));
                m.step += 1;
                const float bc1 = 1.f - std::pow(b1, (float)m.step), bc2 = 1.f - std::pow(b2, (float)m.step);
                MLP_LAUNCH(k_adam, np, np, m.p.p, m.g.p, m.m.p, m.v.p, lr, b1, b2, eps, bc1, bc2);
                return SPRING_OK;
            };
            rc = body();
        }
        if (rc == SPRING_OK && epoch_loss) {
            float l = 0.f;
            rc = d2h(c, &l, m.scal.p, sizeof(float), "loss");
            epoch_loss[ep] = nbat ? l / nbat : 0.f;
        }
    }
    cudaStreamSynchronize(c->stream);
    dfree(X); dfree(y); dfree(idx);
    return rc;
}

int run_mlp_predict(spring_ctx* c, int n, const float* hX, float* hy, int bf16) {
    Mlp& m = c->mlp;
    if (bf16) {  // BF16 on the tensor cores, FP32 accumulation
        DBuf<float> dx, dy;
        int rc = dalloc(c, dx, (size_t)std::max(n, 1) * SZ[0], "network inputs");
        if (rc == SPRING_OK) rc = dalloc(c, dy, std::max(n, 1), "network outputs");
        if (rc == SPRING_OK) rc = h2d(c, dx.p, hX, sizeof(float) * n * SZ[0], "network inputs");
        if (rc == SPRING_OK && n > 0) {
            if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "mlp: injected launch failure");
            else {
                const int grid = std::max(1, std::min((n + MW * 16 - 1) / (MW * 16), 148 * 8));
                cudaFuncSetAttribute(k_mlp_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpBf16Smem));
                k_mlp_bf16<<<grid, MW * 32, sizeof(MlpBf16Smem), c->stream>>>(n, dx.p, m.p.p, w_off(0), w_off(1),
                                                                                w_off(2), w_off(3), dy.p);
                rc = launch_check(c, "k_mlp_bf16");
            }
        }
        if (rc == SPRING_OK && n > 0) rc = d2h(c, hy, dy.p, sizeof(float) * n, "network outputs");
        cudaStreamSynchronize(c->stream);
        dfree(dx);
        dfree(dy);
        return rc;
    }
    const int np = mlp_num_params();
    const int chunk = std::min(n, 1 << 16);
    SPRING_CHECK(ensure_buffers(c, chunk));
    DBuf<float> pr;
    const float* P = m.p.p;
    int rc = SPRING_OK;
    if (bf16) {  // BF16 weights (and, in the forward, BF16-rounded activations)
        rc = dalloc(c, pr, np, "rounded parameters");
        if (rc == SPRING_OK) {
            if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "mlp: injected launch failure");
            else {
                k_round_bf16<<<blocks_for(np), 256, 0, c->stream>>>(np, m.p.p, pr.p);
                rc = launch_check(c, "k_round_bf16");
            }
        }
        P = pr.p;
    }
    Bufs b = carve(c, chunk);
    for (int s0 = 0; rc == SPRING_OK && s0 < n; s0 += chunk) {
        const int nb = std::min(chunk, n - s0);
        rc = h2d(c, b.x, hX + (size_t)s0 * SZ[0], sizeof(float) * nb * SZ[0], "network inputs");
        if (rc == SPRING_OK && bf16) {
            if (launch_injected(c)) rc = fail(c, SPRING_ERR_INJECTED, "mlp: injected launch failure");
            else {
                k_round_bf16<<<blocks_for((long long)nb * SZ[0]), 256, 0, c->stream>>>(nb * SZ[0], b.x, b.x);
                rc = launch_check(c, "k_round_bf16");
            }
        }
        if (rc == SPRING_OK) rc = forward(c, b, nb, P, bf16);
        if (rc == SPRING_OK) rc = d2h(c, hy + s0, b.z[NL], sizeof(float) * nb, "network outputs");
    }
    cudaStreamSynchronize(c->stream);
    dfree(pr);
    return rc;
}

void free_mlp(Mlp& m) {
    dfree(m.p); dfree(m.g); dfree(m.m); dfree(m.v); dfree(m.act); dfree(m.scal);
    m.cap = 0;
    m.set = false;
}

}  // namespace spring
