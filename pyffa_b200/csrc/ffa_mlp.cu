// ffa_mlp.cu -- the learned sector map: a residual MLP on the tensor cores.
//
// y = x + x Ws + bs + f(x),  f = L4 . SiLU . L3 . SiLU . L2 . SiLU . L1,
// widths 6 -> 256 -> 256 -> 256 -> 6.  Weights are float32 masters, rounded to
// bfloat16 where they enter an MMA; products accumulate in float32
// (mma.sync m16n8k16 bf16 -> f32).  The skip layer (Ws, bs) stays float32.
//
// Training: a tiled tensor-core GEMM (op(A) op(B) + bias, operands staged in
// shared memory as bf16 from float32) and element-wise kernels for SiLU, its
// derivative, the loss gradient, bias gradients and Adam.
// Inference: one fused kernel per 128 particles that applies the map
// n_apply times in a row with the state in shared memory and the hidden
// activations in registers as MMA operand fragments (an accumulator tile of
// one layer is, lane for lane, an operand tile of the next: no shuffles).
#include <cuda_bf16.h>

#include "ffa_internal.cuh"

namespace {

// ----------------------------------------------------------- parameters
constexpr int H = FFA_MLP_HIDDEN;      // 256
constexpr int KIN = 16;                // input width padded to one k tile
constexpr int NOUT = 8;                // output width padded to one n tile
// float32 parameter block (offsets in floats)
constexpr int64_t P_W1 = 0;                       // [KIN][H]
constexpr int64_t P_B1 = P_W1 + KIN * H;
constexpr int64_t P_W2 = P_B1 + H;                // [H][H]
constexpr int64_t P_B2 = P_W2 + H * H;
constexpr int64_t P_W3 = P_B2 + H;                // [H][H]
constexpr int64_t P_B3 = P_W3 + H * H;
constexpr int64_t P_W4 = P_B3 + H;                // [H][NOUT]
constexpr int64_t P_B4 = P_W4 + H * NOUT;
constexpr int64_t P_WS = P_B4 + NOUT;             // [NOUT][NOUT] (6 x 6 used)
constexpr int64_t P_BS = P_WS + NOUT * NOUT;
constexpr int64_t P_TOTAL = P_BS + NOUT;
static_assert(P_TOTAL == FFA_MLP_PARAMS, "parameter block layout");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

__device__ __forceinline__ float dsilu(float z)
{
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ------------------------------------------------------------ GEMM (training)
// C[M][N] = op(A)[M][K] op(B)[K][N] (+ bias[N]); op(A)[m][k] = A[m*lda + k]
// or, with transA, A[k*lda + m]; op(B)[k][n] = B[k*ldb + n] or, with transB,
// B[n*ldb + k].  64 x 64 block tile, K staged 32 at a time as bf16 in shared
// memory (A row-major in k, B n-major in k: both fragment loads are 32-bit
// words), four warps of 32 x 32.
constexpr int GT_M = 64, GT_N = 64, GT_K = 32, GT_PAD = 8;

__global__ void __launch_bounds__(128) gemm_tc(const float *__restrict__ A, int lda, int transA,
                                               const float *__restrict__ B, int ldb, int transB,
                                               float *__restrict__ C, int ldc, int M, int N, int K,
                                               const float *__restrict__ bias)
{
    __shared__ __align__(16) __nv_bfloat16 sA[GT_M][GT_K + GT_PAD];
    __shared__ __align__(16) __nv_bfloat16 sB[GT_N][GT_K + GT_PAD];
    const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int r = lane >> 2, c2 = (lane & 3) * 2;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += GT_K) {
        for (int e = threadIdx.x; e < GT_M * GT_K; e += blockDim.x) {
            const int mm = e / GT_K, kk = e - mm * GT_K;
            const int gm = m0 + mm, gk = k0 + kk;
            float v = 0.0f;
            if (gm < M && gk < K) v = transA ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk];
            sA[mm][kk] = __float2bfloat16_rn(v);
        }
        for (int e = threadIdx.x; e < GT_N * GT_K; e += blockDim.x) {
            const int nn = e / GT_K, kk = e - nn * GT_K;
            const int gn = n0 + nn, gk = k0 + kk;
            float v = 0.0f;
            if (gn < N && gk < K) v = transB ? B[(int64_t)gn * ldb + gk] : B[(int64_t)gk * ldb + gn];
            sB[nn][kk] = __float2bfloat16_rn(v);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GT_K; kk += 16) {
            uint32_t a[2][4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = wm + i * 16 + r;
                a[i][0] = *reinterpret_cast<const uint32_t *>(&sA[row][kk + c2]);
                a[i][1] = *reinterpret_cast<const uint32_t *>(&sA[row + 8][kk + c2]);
                a[i][2] = *reinterpret_cast<const uint32_t *>(&sA[row][kk + c2 + 8]);
                a[i][3] = *reinterpret_cast<const uint32_t *>(&sA[row + 8][kk + c2 + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = wn + j * 8 + r;
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&sB[col][kk + c2]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&sB[col][kk + c2 + 8]);
#pragma unroll
                for (int i = 0; i < 2; ++i) mma_bf16(acc[i][j], a[i], b0, b1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int gm = m0 + wm + i * 16 + r + ((q & 2) ? 8 : 0);
                const int gn = n0 + wn + j * 8 + c2 + (q & 1);
                if (gm < M && gn < N) C[(int64_t)gm * ldc + gn] = acc[i][j][q] + (bias ? bias[gn] : 0.0f);
            }
}

// ------------------------------------------------------- element-wise (training)
__global__ void silu_kernel(const float *z, float *h, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        h[i] = silu(z[i]);
}

__global__ void dsilu_kernel(float *dh, const float *z, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dh[i] *= dsilu(z[i]);
}

// y = x + x Ws + bs + f; d = 2 (y - t) / (B n_fit) on the fitted outputs;
// per-block partial of the squared error.  x, t: [B][8] float32, f: [B][8].
__global__ void out_grad_kernel(const float *x, const float *t, const float *f, const float *P, float *y, float *d,
                                int64_t B, int n_fit, double *loss_part)
{
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B; i += (int64_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < NOUT; ++c) {
            float v = 0.0f;
            if (c < 6) {
                v = x[i * NOUT + c] + f[i * NOUT + c] + P[P_BS + c];
                for (int k = 0; k < 6; ++k) v += x[i * NOUT + k] * P[P_WS + k * NOUT + c];
            }
            y[i * NOUT + c] = v;
            float g = 0.0f;
            if (c < n_fit) {
                const float e = v - t[i * NOUT + c];
                acc += (double)e * (double)e;
                g = 2.0f * e / (float)(B * n_fit);
            }
            d[i * NOUT + c] = g;
        }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_part[blockIdx.x] = sh[0];
}

// column sums g[c] = sum_i d[i][c]: one block per 32 columns, eight warps
// over interleaved rows, then a fixed-order reduction (deterministic).
__global__ void __launch_bounds__(256) colsum_kernel(const float *d, int64_t B, int ncol, int ld, float *g)
{
    __shared__ float sh[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    float s = 0.0f;
    if (c < ncol)
        for (int64_t i = w; i < B; i += 8) s += d[i * ld + c];
    sh[w][lane] = s;
    __syncthreads();
    if (w == 0 && c < ncol) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += sh[k][lane];
        g[c] = t;
    }
}

// skip-layer gradient gWs[k][c] = sum_i x[i][k] d[i][c] (k, c < 6): block k,
// 256 threads over rows, fixed-order reduction.
__global__ void __launch_bounds__(256) skip_grad_kernel(const float *x, const float *d, int64_t B, float *G)
{
    __shared__ float sh[256][NOUT + 1];
    const int k = blockIdx.x;
    float s[NOUT];
#pragma unroll
    for (int c = 0; c < NOUT; ++c) s[c] = 0.0f;
    if (k < 6)
        for (int64_t i = threadIdx.x; i < B; i += blockDim.x) {
            const float xk = x[i * NOUT + k];
#pragma unroll
            for (int c = 0; c < 6; ++c) s[c] += xk * d[i * NOUT + c];
        }
#pragma unroll
    for (int c = 0; c < NOUT; ++c) sh[threadIdx.x][c] = s[c];
    __syncthreads();
    if (threadIdx.x < NOUT) {
        float t = 0.0f;
        for (int i = 0; i < (int)blockDim.x; ++i) t += sh[i][threadIdx.x];
        G[P_WS + k * NOUT + threadIdx.x] = t;
    }
}

__global__ void adam_kernel(float *P, const float *G, float *m, float *v, int64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, const uint8_t *mask)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask && !mask[i]) continue;
        const float g = G[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ------------------------------------------------------- fused inference
// 8 warps x 16 particles.  Shared: W2^T as bf16 [n][k + 8] (k padded against
// bank conflicts), W1^T [n][16], W4^T [8][k + 8], biases, skip layer, the
// state of the block's 128 particles.  W3^T bf16 [n][k] is read from global
// (L1 / L2 resident: 128 KB shared by every block).
constexpr int KP = H + 8;
constexpr int INF_WARPS = 8;
constexpr size_t INF_SMEM = sizeof(__nv_bfloat16) * ((size_t)H * KP + (size_t)H * KIN + (size_t)NOUT * KP) +
                            sizeof(float) * (3 * H + NOUT + NOUT * NOUT + NOUT + INF_WARPS * 16 * NOUT) +
                            sizeof(int) * 2 * INF_WARPS * 16;

__global__ void pack_weights_kernel(const float *P, __nv_bfloat16 *w1t, __nv_bfloat16 *w2t, __nv_bfloat16 *w3t,
                                    __nv_bfloat16 *w4t)
{
    // transposed bf16 copies: w?t[n][k] = W?[k][n]
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < H * KIN) { const int n = tid / KIN, k = tid % KIN; w1t[tid] = __float2bfloat16_rn(P[P_W1 + k * H + n]); }
    if (tid < H * H) {
        const int n = tid / H, k = tid % H;
        w2t[tid] = __float2bfloat16_rn(P[P_W2 + k * H + n]);
        w3t[tid] = __float2bfloat16_rn(P[P_W3 + k * H + n]);
    }
    if (tid < NOUT * H) { const int n = tid / H, k = tid % H; w4t[tid] = __float2bfloat16_rn(P[P_W4 + k * NOUT + n]); }
}

// one hidden layer: in (16 k tiles of A fragments) -> out, bias + SiLU
template <bool GLOBAL_B>
__device__ __forceinline__ void hidden_layer(const uint32_t (&in)[16][4], uint32_t (&out)[16][4],
                                             const __nv_bfloat16 *W, int ldw, const float *bias, int lane)
{
    const int r = lane >> 2, c2 = (lane & 3) * 2;
#pragma unroll
    for (int nt = 0; nt < H / 8; ++nt) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16 *wr = W + (int64_t)(nt * 8 + r) * ldw;
#pragma unroll
        for (int kt = 0; kt < H / 16; ++kt) {
            uint32_t b0, b1;
            if (GLOBAL_B) {
                b0 = __ldg(reinterpret_cast<const unsigned int *>(wr + kt * 16 + c2));
                b1 = __ldg(reinterpret_cast<const unsigned int *>(wr + kt * 16 + c2 + 8));
            } else {
                b0 = *reinterpret_cast<const uint32_t *>(wr + kt * 16 + c2);
                b1 = *reinterpret_cast<const uint32_t *>(wr + kt * 16 + c2 + 8);
            }
            mma_bf16(acc, in[kt], b0, b1);
        }
        const float bb0 = bias[nt * 8 + c2], bb1 = bias[nt * 8 + c2 + 1];
        const uint32_t lo = pack_bf16(silu(acc[0] + bb0), silu(acc[1] + bb1));   // row r
        const uint32_t hi = pack_bf16(silu(acc[2] + bb0), silu(acc[3] + bb1));   // row r + 8
        if ((nt & 1) == 0) { out[nt >> 1][0] = lo; out[nt >> 1][1] = hi; }
        else { out[nt >> 1][2] = lo; out[nt >> 1][3] = hi; }
    }
}

__global__ void __launch_bounds__(INF_WARPS * 32, 1)
    mlp_infer_kernel(const float *P, const __nv_bfloat16 *w1t, const __nv_bfloat16 *w2t, const __nv_bfloat16 *w3t,
                     const __nv_bfloat16 *w4t, float *state, int32_t *applied, int64_t n, int n_apply, float radius2)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16 *sW2 = reinterpret_cast<__nv_bfloat16 *>(smraw);
    __nv_bfloat16 *sW1 = sW2 + (size_t)H * KP;
    __nv_bfloat16 *sW4 = sW1 + (size_t)H * KIN;
    float *sB = reinterpret_cast<float *>(sW4 + (size_t)NOUT * KP);   // b1 b2 b3
    float *sB4 = sB + 3 * H;
    float *sWs = sB4 + NOUT;
    float *sBs = sWs + NOUT * NOUT;
    float *sX = sBs + NOUT;                                             // [128][8]
    int *sAct = reinterpret_cast<int *>(sX + INF_WARPS * 16 * NOUT);   // [128]
    int *sCnt = sAct + INF_WARPS * 16;                                  // [128]
    for (int e = threadIdx.x; e < H * H; e += blockDim.x) {
        const int nn = e / H, k = e - nn * H;
        sW2[nn * KP + k] = w2t[e];
    }
    for (int e = threadIdx.x; e < H * KIN; e += blockDim.x) sW1[e] = w1t[e];
    for (int e = threadIdx.x; e < NOUT * H; e += blockDim.x) {
        const int nn = e / H, k = e - nn * H;
        sW4[nn * KP + k] = w4t[e];
    }
    for (int e = threadIdx.x; e < H; e += blockDim.x) {
        sB[e] = P[P_B1 + e];
        sB[H + e] = P[P_B2 + e];
        sB[2 * H + e] = P[P_B3 + e];
    }
    if (threadIdx.x < NOUT) { sB4[threadIdx.x] = P[P_B4 + threadIdx.x]; sBs[threadIdx.x] = P[P_BS + threadIdx.x]; }
    if (threadIdx.x < NOUT * NOUT) sWs[threadIdx.x] = P[P_WS + threadIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = lane >> 2, c2 = (lane & 3) * 2;
    const int64_t p0 = (int64_t)blockIdx.x * (INF_WARPS * 16) + warp * 16;
    float *x = sX + warp * 16 * NOUT;
    int *act = sAct + warp * 16, *cnt = sCnt + warp * 16;
    for (int e = lane; e < 16 * NOUT; e += 32) {
        const int64_t p = p0 + e / NOUT;
        x[e] = p < n ? state[p * NOUT + (e % NOUT)] : 0.0f;
    }
    if (lane < 16) { act[lane] = (p0 + lane) < n; cnt[lane] = 0; }
    __syncthreads();
    uint32_t a[16][4], b[16][4];
    for (int it = 0; it < n_apply; ++it) {
        if (lane < 16 && radius2 > 0.0f) {
            const float *xs = x + lane * NOUT;
            const bool inside = xs[0] * xs[0] + xs[1] * xs[1] <= radius2 && xs[2] * xs[2] + xs[3] * xs[3] <= radius2 &&
                                fabsf(xs[4]) <= 1.0f;
            if (!inside) act[lane] = 0;
        }
        __syncwarp();
        // layer 1: one k tile of the (6-wide, zero-padded) input
        {
            uint32_t in[4];
            in[0] = (c2 < 6) ? pack_bf16(x[r * NOUT + c2], x[r * NOUT + c2 + 1]) : 0u;
            in[1] = (c2 < 6) ? pack_bf16(x[(r + 8) * NOUT + c2], x[(r + 8) * NOUT + c2 + 1]) : 0u;
            in[2] = 0u;
            in[3] = 0u;
#pragma unroll
            for (int nt = 0; nt < H / 8; ++nt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                const __nv_bfloat16 *wr = sW1 + (nt * 8 + r) * KIN;
                mma_bf16(acc, in, *reinterpret_cast<const uint32_t *>(wr + c2),
                         *reinterpret_cast<const uint32_t *>(wr + c2 + 8));
                const float bb0 = sB[nt * 8 + c2], bb1 = sB[nt * 8 + c2 + 1];
                const uint32_t lo = pack_bf16(silu(acc[0] + bb0), silu(acc[1] + bb1));
                const uint32_t hi = pack_bf16(silu(acc[2] + bb0), silu(acc[3] + bb1));
                if ((nt & 1) == 0) { a[nt >> 1][0] = lo; a[nt >> 1][1] = hi; }
                else { a[nt >> 1][2] = lo; a[nt >> 1][3] = hi; }
            }
        }
        hidden_layer<false>(a, b, sW2, KP, sB + H, lane);
        hidden_layer<true>(b, a, w3t, H, sB + 2 * H, lane);
        // layer 4 and the residual: rows r and r + 8, columns c2, c2 + 1
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        const __nv_bfloat16 *wr = sW4 + r * KP;
#pragma unroll
        for (int kt = 0; kt < H / 16; ++kt)
            mma_bf16(acc, a[kt], *reinterpret_cast<const uint32_t *>(wr + kt * 16 + c2),
                     *reinterpret_cast<const uint32_t *>(wr + kt * 16 + c2 + 8));
        float y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = r + ((q & 2) ? 8 : 0), col = c2 + (q & 1);
            float v = x[row * NOUT + col];
            if (col < 6) {
                float lin = sBs[col];
                for (int k = 0; k < 6; ++k) lin += x[row * NOUT + k] * sWs[k * NOUT + col];
                v += lin + (acc[q] + sB4[col]);
            }
            y[q] = v;
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = r + ((q & 2) ? 8 : 0), col = c2 + (q & 1);
            if (col < 4 && act[row]) x[row * NOUT + col] = y[q];   // e and the spare column stay
        }
        if (lane < 16) cnt[lane] += act[lane];
        __syncwarp();
    }
    for (int e = lane; e < 16 * NOUT; e += 32) {
        const int64_t p = p0 + e / NOUT;
        if (p < n) state[p * NOUT + (e % NOUT)] = x[e];
    }
    if (applied && lane < 16 && p0 + lane < n) applied[p0 + lane] = cnt[lane];
}

int blocks_for(int64_t n, int tb) { return (int)((n + tb - 1) / tb < 4096 ? (n + tb - 1) / tb : 4096); }

}  // namespace

// ------------------------------------------------------------------ C ABI

static_assert(2 * (H * KIN + 2 * H * H + NOUT * H) == FFA_MLP_WPACK_BYTES, "inference weight pack size");

extern "C" int ffa_mlp_gemm(const float *A, int lda, int transA, const float *B, int ldb, int transB, float *C,
                            int ldc, int M, int N, int K, const float *bias, void *stream)
{
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return FFA_ERR_INVALID;
    dim3 grid((unsigned)((N + GT_N - 1) / GT_N), (unsigned)((M + GT_M - 1) / GT_M));
    if (grid.y > 65535) return FFA_ERR_UNSUPPORTED;
    gemm_tc<<<grid, 128, 0, (cudaStream_t)stream>>>(A, lda, transA, B, ldb, transB, C, ldc, M, N, K, bias);
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

extern "C" int ffa_mlp_train_step(const ffa_mlp_train_desc *d, void *stream)
{
    if (!d || !d->params || !d->grads || !d->adam_m || !d->adam_v || !d->x || !d->target || !d->work ||
        !d->loss_part || d->batch <= 0 || d->n_fit < 1 || d->n_fit > 6 || (d->lr > 0.0f && d->step < 1))
        return FFA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t B = d->batch;
    if (B > 65535LL * GT_M || B * H > INT32_MAX) return FFA_ERR_UNSUPPORTED;
    float *P = d->params, *G = d->grads;
    float *z1 = d->work, *h1 = z1 + B * H, *z2 = h1 + B * H, *h2 = z2 + B * H, *z3 = h2 + B * H, *h3 = z3 + B * H;
    float *f = h3 + B * H, *y = f + B * NOUT, *dd = y + B * NOUT, *dh = dd + B * NOUT, *dz = dh + B * H;
    const int ew = blocks_for(B * H, 256);
    const int Bi = (int)B;
    auto gemm = [&](const float *A_, int lda_, int tA_, const float *B_, int ldb_, int tB_, float *C_, int ldc_,
                    int M_, int N_, int K_, const float *bias_) {
        const dim3 grid((unsigned)((N_ + GT_N - 1) / GT_N), (unsigned)((M_ + GT_M - 1) / GT_M));
        gemm_tc<<<grid, 128, 0, s>>>(A_, lda_, tA_, B_, ldb_, tB_, C_, ldc_, M_, N_, K_, bias_);
    };
    // forward
    gemm(d->x, NOUT, 0, P + P_W1, H, 0, z1, H, Bi, H, 6, P + P_B1);
    silu_kernel<<<ew, 256, 0, s>>>(z1, h1, B * H);
    gemm(h1, H, 0, P + P_W2, H, 0, z2, H, Bi, H, H, P + P_B2);
    silu_kernel<<<ew, 256, 0, s>>>(z2, h2, B * H);
    gemm(h2, H, 0, P + P_W3, H, 0, z3, H, Bi, H, H, P + P_B3);
    silu_kernel<<<ew, 256, 0, s>>>(z3, h3, B * H);
    gemm(h3, H, 0, P + P_W4, NOUT, 0, f, NOUT, Bi, NOUT, H, P + P_B4);
    out_grad_kernel<<<148, 256, 0, s>>>(d->x, d->target, f, P, y, dd, B, d->n_fit, d->loss_part);
    // backward
    FFA_CHECK_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * P_TOTAL, s));
    skip_grad_kernel<<<NOUT, 256, 0, s>>>(d->x, dd, B, G);
    colsum_kernel<<<1, 256, 0, s>>>(dd, B, NOUT, NOUT, G + P_BS);
    gemm(h3, H, 1, dd, NOUT, 0, G + P_W4, NOUT, H, NOUT, Bi, nullptr);
    colsum_kernel<<<1, 256, 0, s>>>(dd, B, NOUT, NOUT, G + P_B4);
    gemm(dd, NOUT, 0, P + P_W4, NOUT, 1, dh, H, Bi, H, NOUT, nullptr);
    const float *zs[3] = {z3, z2, z1};
    const float *hin[3] = {h2, h1, d->x};
    const int64_t wofs[3] = {P_W3, P_W2, P_W1}, bofs[3] = {P_B3, P_B2, P_B1};
    const int ldin[3] = {H, H, NOUT}, kin[3] = {H, H, 6};
    for (int l = 0; l < 3; ++l) {
        dsilu_kernel<<<ew, 256, 0, s>>>(dh, zs[l], B * H);   // dh -> dz in place
        gemm(hin[l], ldin[l], 1, dh, H, 0, G + wofs[l], H, kin[l], H, Bi, nullptr);
        colsum_kernel<<<H / 32, 256, 0, s>>>(dh, B, H, H, G + bofs[l]);
        if (l < 2) {
            gemm(dh, H, 0, P + wofs[l], H, 1, dz, H, Bi, H, H, nullptr);
            float *t = dh;
            dh = dz;
            dz = t;
        }
    }
    if (d->lr > 0.0f) {
        const float c1 = 1.0f - powf(d->beta1, (float)d->step), c2 = 1.0f - powf(d->beta2, (float)d->step);
        adam_kernel<<<blocks_for(P_TOTAL, 256), 256, 0, s>>>(P, G, d->adam_m, d->adam_v, P_TOTAL, d->lr, d->beta1,
                                                             d->beta2, d->eps, c1, c2, d->mask);
    }
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

extern "C" int ffa_mlp_pack(const float *params, void *wpack, void *stream)
{
    if (!params || !wpack || (reinterpret_cast<uintptr_t>(wpack) & 15)) return FFA_ERR_INVALID;
    __nv_bfloat16 *w1t = reinterpret_cast<__nv_bfloat16 *>(wpack);
    __nv_bfloat16 *w2t = w1t + H * KIN, *w3t = w2t + H * H, *w4t = w3t + H * H;
    pack_weights_kernel<<<(H * H + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, w1t, w2t, w3t, w4t);
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

extern "C" int ffa_mlp_infer(const ffa_mlp_infer_desc *d, void *stream)
{
    if (!d || !d->params || !d->wpack || !d->state || d->n < 0 || d->n_apply < 0 ||
        (reinterpret_cast<uintptr_t>(d->wpack) & 15))
        return FFA_ERR_INVALID;
    if (d->n == 0) return FFA_OK;
    const int64_t blocks = (d->n + INF_WARPS * 16 - 1) / (INF_WARPS * 16);
    if (blocks > INT32_MAX) return FFA_ERR_UNSUPPORTED;
    const __nv_bfloat16 *w1t = reinterpret_cast<const __nv_bfloat16 *>(d->wpack);
    const __nv_bfloat16 *w2t = w1t + H * KIN, *w3t = w2t + H * H, *w4t = w3t + H * H;
    FFA_CHECK_CUDA(cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM));
    mlp_infer_kernel<<<(unsigned)blocks, INF_WARPS * 32, INF_SMEM, (cudaStream_t)stream>>>(
        d->params, w1t, w2t, w3t, w4t, d->state, d->applied, d->n, d->n_apply, d->radius2);
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}
