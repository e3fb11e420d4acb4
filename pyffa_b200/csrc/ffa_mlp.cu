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
constexpr int64_t P_WQ = P_BS + NOUT;             // [16][NOUT] (15 x 6 used)
constexpr int64_t P_TOTAL = P_WQ + 16 * NOUT;
// quadratic skip features: s_i s_j for i <= j < 5, in this order
__device__ __constant__ int8_t QI[15] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4};
__device__ __constant__ int8_t QJ[15] = {0, 1, 2, 3, 4, 1, 2, 3, 4, 2, 3, 4, 3, 4, 4};

// the 15 quadratic features of a register-resident state, in QI / QJ order
__device__ __forceinline__ void quad_features(const float *x, float *q)
{
    q[0] = x[0] * x[0]; q[1] = x[0] * x[1]; q[2] = x[0] * x[2]; q[3] = x[0] * x[3]; q[4] = x[0] * x[4];
    q[5] = x[1] * x[1]; q[6] = x[1] * x[2]; q[7] = x[1] * x[3]; q[8] = x[1] * x[4];
    q[9] = x[2] * x[2]; q[10] = x[2] * x[3]; q[11] = x[2] * x[4];
    q[12] = x[3] * x[3]; q[13] = x[3] * x[4];
    q[14] = x[4] * x[4];
}
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

__device__ __forceinline__ float tanh_approx(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// SiLU(z) = z sigmoid(z) = h + h tanh(h), h = z / 2 (training and inference
// evaluate it the same way)
__device__ __forceinline__ float silu(float z)
{
    const float h = 0.5f * z;
    return fmaf(h, tanh_approx(h), h);
}

// d SiLU / dz = sigmoid(z) (1 + z (1 - sigmoid(z))) = (1 + t)(1 + h (1 - t)) / 2
__device__ __forceinline__ float dsilu(float z)
{
    const float h = 0.5f * z, t = tanh_approx(h);
    return 0.5f * (1.0f + t) * fmaf(h, 1.0f - t, 1.0f);
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
                                               const float *__restrict__ bias, int k_chunk)
{
    __shared__ __align__(16) __nv_bfloat16 sA[GT_M][GT_K + GT_PAD];
    __shared__ __align__(16) __nv_bfloat16 sB[GT_N][GT_K + GT_PAD];
    const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
    // split K: block z covers [kb, ke) and writes its partial product to
    // C + z * M * N (row stride N) when gridDim.z > 1
    const int kb = blockIdx.z * k_chunk, ke = min(K, kb + k_chunk);
    if (gridDim.z > 1) {
        C += (int64_t)blockIdx.z * M * N;
        ldc = N;
        bias = nullptr;
    }
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
    for (int k0 = kb; k0 < ke; k0 += GT_K) {
        // staging: the index that is contiguous in global memory runs fastest
        // across threads (coalesced loads), converted to bfloat16
        // fixed trip counts (128 threads): the loads of a stage are issued together
        if (!transA) {
#pragma unroll
            for (int it = 0; it < GT_M * GT_K / 128; ++it) {
                const int e = threadIdx.x + 128 * it;
                const int mm = e / GT_K, kk = e - mm * GT_K;
                const int gm = m0 + mm, gk = k0 + kk;
                sA[mm][kk] = __float2bfloat16_rn((gm < M && gk < ke) ? A[(int64_t)gm * lda + gk] : 0.0f);
            }
        } else {
#pragma unroll
            for (int it = 0; it < GT_M * GT_K / 128; ++it) {
                const int e = threadIdx.x + 128 * it;
                const int kk = e / GT_M, mm = e - kk * GT_M;
                const int gm = m0 + mm, gk = k0 + kk;
                sA[mm][kk] = __float2bfloat16_rn((gm < M && gk < ke) ? A[(int64_t)gk * lda + gm] : 0.0f);
            }
        }
        if (transB) {
#pragma unroll
            for (int it = 0; it < GT_N * GT_K / 128; ++it) {
                const int e = threadIdx.x + 128 * it;
                const int nn = e / GT_K, kk = e - nn * GT_K;
                const int gn = n0 + nn, gk = k0 + kk;
                sB[nn][kk] = __float2bfloat16_rn((gn < N && gk < ke) ? B[(int64_t)gn * ldb + gk] : 0.0f);
            }
        } else {
#pragma unroll
            for (int it = 0; it < GT_N * GT_K / 128; ++it) {
                const int e = threadIdx.x + 128 * it;
                const int kk = e / GT_N, nn = e - kk * GT_N;
                const int gn = n0 + nn, gk = k0 + kk;
                sB[nn][kk] = __float2bfloat16_rn((gn < N && gk < ke) ? B[(int64_t)gk * ldb + gn] : 0.0f);
            }
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

// C[m][n] = sum over the splits of part[z][m][n], in split order
__global__ void split_sum_kernel(const float *__restrict__ part, int splits, int M, int N, float *__restrict__ C,
                                 int ldc, const float *__restrict__ bias)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * N) return;
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(int64_t)z * M * N + i];
    C[(int64_t)(i / N) * ldc + (i % N)] = s + (bias ? bias[i % N] : 0.0f);
}

constexpr int SPLITS_MAX = 16;
constexpr int64_t SPLIT_WORK = (int64_t)SPLITS_MAX * H * H;   // floats
static_assert(SPLIT_WORK == FFA_MLP_SPLIT_WORK, "training split-K work area");

// ------------------------------------------------------- element-wise (training)
// layer 1: z1 = x W1 + b1 with the float32 input and bfloat16-rounded W1, the
// values the inference kernel's split-input product forms
__global__ void layer1_kernel(const float *__restrict__ x, const float *__restrict__ P, float *__restrict__ z1,
                              int64_t B)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B * H; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / H;
        const int n = (int)(i - r * H);
        float z = P[P_B1 + n];
#pragma unroll
        for (int k = 0; k < 6; ++k)
            z = fmaf(x[r * NOUT + k], __bfloat162float(__float2bfloat16_rn(P[P_W1 + k * H + n])), z);
        z1[i] = z;
    }
}

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
                for (int m = 0; m < 15; ++m) v += x[i * NOUT + QI[m]] * x[i * NOUT + QJ[m]] * P[P_WQ + m * NOUT + c];
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
// Column sums g[c] = sum_i d[i][c] (bias gradients) in two fixed-order
// passes: block (x, y) sums 32 columns over the rows [y rows_per, (y + 1)
// rows_per) into part[y][c] (8 warps, 4 rows each per step), then one
// thread per column adds the partial sums in row-chunk order.
__global__ void __launch_bounds__(256) colsum_part_kernel(const float *__restrict__ d, int64_t B, int ncol, int ld,
                                                          int64_t rows_per, float *__restrict__ part)
{
    __shared__ float sh[8][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    const int64_t i0 = blockIdx.y * rows_per, i1 = min(B, i0 + rows_per);
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
    if (c < ncol) {
        int64_t i = i0 + w;
        for (; i + 24 < i1; i += 32) {
            s0 += d[i * ld + c];
            s1 += d[(i + 8) * ld + c];
            s2 += d[(i + 16) * ld + c];
            s3 += d[(i + 24) * ld + c];
        }
        for (; i < i1; i += 8) s0 += d[i * ld + c];
    }
    sh[w][lane] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    if (w == 0 && c < ncol) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += sh[k][lane];
        part[(int64_t)blockIdx.y * ncol + c] = t;
    }
}

// one warp per column: lane l adds chunks l, l + 32, ..., then a fixed
// shuffle tree (the same order every call)
__global__ void colsum_final_kernel(const float *__restrict__ part, int chunks, int ncol, float *__restrict__ g)
{
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (c >= ncol) return;
    float t = 0.0f;
    for (int y = lane; y < chunks; y += 32) t += part[(int64_t)y * ncol + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) g[c] = t;
}

// skip-layer gradients: block k < 8 forms gWs[k][c] = sum_i x[i][k] d[i][c],
// block 8 + m forms gWq[m][c] = sum_i x[i][QI[m]] x[i][QJ[m]] d[i][c]
// (c < 6), 256 threads over rows, fixed-order reduction
__global__ void __launch_bounds__(256) skip_grad_kernel(const float *x, const float *d, int64_t B, float *G)
{
    __shared__ float sh[256][NOUT + 1];
    const int k = blockIdx.x;
    const bool quad = k >= NOUT;
    const int m = k - NOUT;
    float s[NOUT];
#pragma unroll
    for (int c = 0; c < NOUT; ++c) s[c] = 0.0f;
    if ((!quad && k < 6) || (quad && m < 15))
        for (int64_t i = threadIdx.x; i < B; i += blockDim.x) {
            const float xk = quad ? x[i * NOUT + QI[m]] * x[i * NOUT + QJ[m]] : x[i * NOUT + k];
#pragma unroll
            for (int c = 0; c < 6; ++c) s[c] += xk * d[i * NOUT + c];
        }
#pragma unroll
    for (int c = 0; c < NOUT; ++c) sh[threadIdx.x][c] = s[c];
    __syncthreads();
    if (threadIdx.x < NOUT) {
        float t = 0.0f;
        for (int i = 0; i < (int)blockDim.x; ++i) t += sh[i][threadIdx.x];
        G[(quad ? P_WQ + m * NOUT : P_WS + k * NOUT) + threadIdx.x] = t;
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

// Adam with the step read from the device: learning rate lr_table[*counter],
// bias corrections of step *counter + 1
__global__ void adam_sched_kernel(float *P, const float *G, float *m, float *v, int64_t n, const float *lr_table,
                                  const int32_t *counter, float b1, float b2, float eps, const uint8_t *mask)
{
    const int k = *counter;
    const float lr = lr_table[k], t = (float)(k + 1);
    const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
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

__global__ void counter_advance_kernel(int32_t *counter) { *counter += 1; }

// ------------------------------------------------------- fused inference
// 8 warps x 16 particles.  Shared: W2^T as bf16 [n][k + 8] (k padded against
// bank conflicts), W1^T [n][16], W4^T [8][k + 8], biases, skip layer, the
// state of the block's 128 particles.  W3^T bf16 [n][k] is read from global
// (L1 / L2 resident: 128 KB shared by every block).
// ------------------------------------------------------- fused inference
// tcgen05 tensor cores, one 128-state tile per CTA at a time (persistent grid,
// one CTA per SM).  Every layer is one 128 x N accumulator in tensor memory:
// D0 = columns 0..255, D1 = columns 256..511, layers 1..4 alternate D0, D1.
// Warp roles: warp 0 streams W2 / W3 from global (L2-resident) into a ring
// of three 32 KB shared-memory slots with cp.async.bulk; warp 1 owns tensor
// memory and issues the MMAs (one thread); warps 2..17 are the epilogue, four
// threads per state (its tensor-memory lane), one per 16-column quarter of
// each 64-column chunk.  They read the accumulator row, add the bias, apply
// SiLU, round to bfloat16 and write the next layer's A operand one chunk at
// a time (the next chunk's tensor-memory load in flight meanwhile), so the
// next layer's MMAs on chunk c start while chunk c + 1 is still being
// written.  The state, the domain check and the float32 skip connection stay
// in the registers of the quarter-0 thread for all n_apply maps.
//
// Shared-memory operand layouts (K-major):
//  - A (activations, 128 x 256) and W2 / W3 / W4 (B operand, N x 256): four
//    64-column chunks, each row 128 B with the 128-byte swizzle (16-byte
//    unit j of row m stored at unit j ^ (m mod 8)), rows consecutive,
//    chunk bases 1024-aligned; descriptor SBO = 1024 B; the K = 16 slices of
//    a chunk start 32 B apart;
//  - X (layer-1 input, 128 x 16) and W1 (256 x 16): no swizzle, 8 x 8 core
//    matrices of 128 B, the two K halves 128 B apart (LBO) and 8-row groups
//    256 B apart (SBO).
// The inference weight pack in global memory holds W1, W4, W2, W3 in exactly
// these layouts, so each ring slot is one linear bulk copy.
constexpr int TC_M = 128;
constexpr int TC_CHUNK = 64;                                 // K columns per chunk
constexpr uint32_t A_CHUNK_BYTES = TC_M * 128;               // 16 KB
constexpr uint32_t W_CHUNK_BYTES = H * 128;                  // 32 KB
constexpr uint32_t W4_CHUNK_BYTES = 16 * 128;                // 2 KB
constexpr int RING = 3;
// weight pack (bytes)
constexpr uint32_t PK_W1 = 0;                                // 256 x 16 bf16, core matrices
constexpr uint32_t PK_W4 = PK_W1 + H * KIN * 2;              // 4 chunks x 16 rows
constexpr uint32_t PK_W2 = PK_W4 + 4 * W4_CHUNK_BYTES;       // 4 chunks x 256 rows
constexpr uint32_t PK_W3 = PK_W2 + 4 * W_CHUNK_BYTES;
constexpr uint32_t PK_TOTAL = PK_W3 + 4 * W_CHUNK_BYTES;
// shared memory (bytes from the 1024-aligned base)
constexpr uint32_t SM_A = 0;
constexpr uint32_t SM_RING = SM_A + 4 * A_CHUNK_BYTES;
constexpr uint32_t SM_W4 = SM_RING + RING * W_CHUNK_BYTES;
constexpr uint32_t SM_W1 = SM_W4 + 4 * W4_CHUNK_BYTES;
constexpr uint32_t SM_X = SM_W1 + H * KIN * 2;
constexpr uint32_t SM_BIAS = SM_X + TC_M * KIN * 2;          // b1 b2 b3 (halved), float
constexpr uint32_t SM_TAIL = SM_BIAS + 3 * H * 4;            // b4[8] Ws[64] bs[8] Wq[128]
constexpr uint32_t SM_BAR = SM_TAIL + 208 * 4;               // mbarriers (8 B each)
constexpr int NBAR = 1 + 4 + 1 + 2 * RING + 1;               // x_ready, a_ready[4], d_full, full[], empty[], drain
constexpr uint32_t SM_MISC = SM_BAR + NBAR * 8;              // tmem base, abort flag
constexpr uint32_t SM_TOTAL = SM_MISC + 16;
constexpr size_t TC_SMEM = SM_TOTAL + 1024;                  // + alignment slack
constexpr uint64_t WAIT_NS = 2000000000ull;                  // a pipeline wait gives up after 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `bar` with `parity` for at most WAIT_NS, whatever
// the abort flag says (teardown: copies and MMAs in flight must land).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity))
        if (global_ns() - t0 > WAIT_NS) return false;
    return true;
}

// Waits for the phase of `bar` with `parity`; gives up (and raises the
// block's abort flag) after WAIT_NS or when another thread has raised it.
// try_wait suspends the thread for a while by itself; the clock and the flag
// are read once every 64 polls.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true) {
#pragma unroll 1
        for (int i = 0; i < 64; ++i)
            if (mbar_test(bar, parity)) return true;
        if (*abort_flag) return false;
        if (global_ns() - t0 > WAIT_NS) {
            *abort_flag = 1;
            return false;
        }
    }
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// smem matrix descriptor: start, leading / stride byte offsets, layout
// (0: no swizzle, 2: 128-byte swizzle), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout)
{
    return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

// instruction descriptor, kind::f16: bfloat16 A and B (K-major), float32 D
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

#define TMEM_LD32(taddr, v)                                                                                  \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15," \
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"              \
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),      \
                   "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),  \
                   "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),             \
                   "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),             \
                   "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])              \
                 : "r"(taddr))

#define TMEM_LD16(taddr, v)                                                                                  \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}," \
                 " [%16];"                                                                                   \
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),      \
                   "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),  \
                   "=r"(v[14]), "=r"(v[15])                                                                  \
                 : "r"(taddr))

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// keeps the compiler from moving uses of tcgen05.ld results above the wait
#define REG_FENCE16(v)                                                                                       \
    asm volatile("" : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]),   \
                 "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]),      \
                 "+r"(v[14]), "+r"(v[15]))
#define REG_FENCE32(v)  \
    REG_FENCE16(v);     \
    REG_FENCE16((v + 16))

// byte offset of element (row, k) in a 128-byte-swizzled chunked operand
// with `rows` rows per chunk
__host__ __device__ __forceinline__ uint32_t swz_off(int row, int k, int rows)
{
    return (uint32_t)((k >> 6) * rows * 128 + row * 128 + ((((k & 63) >> 3) ^ (row & 7)) << 4) + ((k & 7) << 1));
}

// byte offset of element (row, k) of a no-swizzle K = 16 operand
__host__ __device__ __forceinline__ uint32_t core_off(int row, int k)
{
    return (uint32_t)((((row >> 3) * 2 + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// float32 parameters -> the inference weight pack (bfloat16, layouts above)
__global__ void pack_weights_kernel(const float *__restrict__ P, unsigned char *__restrict__ wp)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < H * H) {
        const int n = tid / H, k = tid % H;
        *reinterpret_cast<__nv_bfloat16 *>(wp + PK_W2 + swz_off(n, k, H)) = __float2bfloat16_rn(P[P_W2 + k * H + n]);
        *reinterpret_cast<__nv_bfloat16 *>(wp + PK_W3 + swz_off(n, k, H)) = __float2bfloat16_rn(P[P_W3 + k * H + n]);
    }
    if (tid < H * KIN) {
        // columns 0..5 and 6..11 both hold W1 rows 0..5 (high / low input parts)
        const int n = tid / KIN, k = tid % KIN;
        const float v = k < 12 ? P[P_W1 + (k % 6) * H + n] : 0.0f;
        *reinterpret_cast<__nv_bfloat16 *>(wp + PK_W1 + core_off(n, k)) = __float2bfloat16_rn(v);
    }
    if (tid < 16 * H) {
        const int n = tid / H, k = tid % H;
        const float v = n < NOUT ? P[P_W4 + k * NOUT + n] : 0.0f;
        *reinterpret_cast<__nv_bfloat16 *>(wp + PK_W4 + swz_off(n, k, 16)) = __float2bfloat16_rn(v);
    }
}

// SiLU of 8 accumulator values (bias pre-halved), packed to 4 bfloat16 pairs
__device__ __forceinline__ uint4 silu8(const uint32_t *v, const float *hb)
{
    float h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = fmaf(__uint_as_float(v[i]), 0.5f, hb[i]);
    uint4 o;
    o.x = pack_bf16(fmaf(h[0], tanh_approx(h[0]), h[0]), fmaf(h[1], tanh_approx(h[1]), h[1]));
    o.y = pack_bf16(fmaf(h[2], tanh_approx(h[2]), h[2]), fmaf(h[3], tanh_approx(h[3]), h[3]));
    o.z = pack_bf16(fmaf(h[4], tanh_approx(h[4]), h[4]), fmaf(h[5], tanh_approx(h[5]), h[5]));
    o.w = pack_bf16(fmaf(h[6], tanh_approx(h[6]), h[6]), fmaf(h[7], tanh_approx(h[7]), h[7]));
    return o;
}

constexpr int TC_THREADS = 32 * (2 + 16);

__global__ void __launch_bounds__(TC_THREADS, 1)
    mlp_infer_tc_kernel(const float *__restrict__ P, const unsigned char *__restrict__ wp, float *__restrict__ state,
                        int32_t *__restrict__ applied, int32_t *__restrict__ error, int64_t n, int n_apply,
                        float radius2)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t s0 = smem_u32(sm);
    float *sbias = reinterpret_cast<float *>(sm + SM_BIAS);
    float *stail = reinterpret_cast<float *>(sm + SM_TAIL);   // b4[0..7], Ws[8..71], bs[72..79], Wq[80..207]
    const uint32_t bar0 = s0 + SM_BAR;
    const uint32_t BAR_X = bar0, BAR_A = bar0 + 8, BAR_D = bar0 + 40, BAR_FULL = bar0 + 48,
                   BAR_EMPTY = bar0 + 48 + 8 * RING, BAR_DRAIN = bar0 + 48 + 16 * RING;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(sm + SM_MISC);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + SM_MISC + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ntiles = (n + TC_M - 1) / TC_M;

    // resident operands and constants
    for (int i = threadIdx.x; i < (int)(H * KIN * 2 / 16); i += blockDim.x)
        reinterpret_cast<uint4 *>(sm + SM_W1)[i] = reinterpret_cast<const uint4 *>(wp + PK_W1)[i];
    for (int i = threadIdx.x; i < (int)(4 * W4_CHUNK_BYTES / 16); i += blockDim.x)
        reinterpret_cast<uint4 *>(sm + SM_W4)[i] = reinterpret_cast<const uint4 *>(wp + PK_W4)[i];
    for (int i = threadIdx.x; i < 3 * H; i += blockDim.x) sbias[i] = 0.5f * P[(i < H ? P_B1 : i < 2 * H ? P_B2 : P_B3) + (i % H)];
    for (int i = threadIdx.x; i < 208; i += blockDim.x)
        stail[i] = i < 8 ? P[P_B4 + i] : i < 72 ? P[P_WS + (i - 8)] : i < 80 ? P[P_BS + (i - 72)] : P[P_WQ + (i - 80)];
    if (threadIdx.x == 0) {
        mbar_init(BAR_X, 4);
        for (int c = 0; c < 4; ++c) mbar_init(BAR_A + 8 * c, 16);
        mbar_init(BAR_D, 1);
        for (int s = 0; s < RING; ++s) {
            mbar_init(BAR_FULL + 8 * s, 1);
            mbar_init(BAR_EMPTY + 8 * s, 1);
        }
        mbar_init(BAR_DRAIN, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tmem_holder;

    if (warp == 0) {
        // ---------------------------------------------------- weight stream
        if (lane == 0) {
            uint32_t q = 0;
            for (int64_t tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x)
                for (int it = 0; it < n_apply && !*abort_flag; ++it)
                    for (int l = 0; l < 2; ++l)
                        for (int c = 0; c < 4; ++c, ++q) {
                            const uint32_t slot = q % RING, use = q / RING;
                            if (!mbar_wait(BAR_EMPTY + 8 * slot, (use & 1) ^ 1, abort_flag)) break;
                            mbar_expect_tx(BAR_FULL + 8 * slot, W_CHUNK_BYTES);
                            bulk_load(s0 + SM_RING + slot * W_CHUNK_BYTES,
                                      wp + (l == 0 ? PK_W2 : PK_W3) + c * W_CHUNK_BYTES, W_CHUNK_BYTES,
                                      BAR_FULL + 8 * slot);
                        }
            // drain: every issued copy has landed before the block exits
            const uint32_t issued = q;
            for (uint32_t r = issued > RING ? issued - RING : 0; r < issued; ++r)
                if (!mbar_wait_bounded(BAR_FULL + 8 * (r % RING), (r / RING) & 1)) *abort_flag = 1;
        }
    } else if (warp == 1) {
        // ---------------------------------------------------- MMA issue
        if (lane == 0) {
            const uint32_t ID256 = idesc_bf16(TC_M, H), ID16 = idesc_bf16(TC_M, 16);
            const uint32_t D0 = tmem, D1 = tmem + 256;
            uint32_t q = 0, nx = 0, na = 0;
            bool ok = true;
            for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x)
                for (int it = 0; it < n_apply && ok; ++it) {
                    // layer 1: X (128 x 16) x W1^T -> D0
                    ok = mbar_wait(BAR_X, nx++ & 1, abort_flag);
                    if (!ok) break;
                    tc_after_sync();
                    umma(D0, sdesc(s0 + SM_X, 128, 256, 0), sdesc(s0 + SM_W1, 128, 256, 0), ID256, 0);
                    umma_commit(BAR_D);
                    // layers 2, 3: A (128 x 256) x W^T (streamed) -> D1, D0
                    for (int l = 0; l < 2 && ok; ++l) {
                        const uint32_t D = l == 0 ? D1 : D0;
                        for (int c = 0; c < 4; ++c, ++q) {
                            const uint32_t slot = q % RING, use = q / RING;
                            ok = mbar_wait(BAR_A + 8 * c, na & 1, abort_flag) &&
                                 mbar_wait(BAR_FULL + 8 * slot, use & 1, abort_flag);
                            if (!ok) break;
                            tc_after_sync();
                            const uint32_t a0 = s0 + SM_A + c * A_CHUNK_BYTES;
                            const uint32_t b0 = s0 + SM_RING + slot * W_CHUNK_BYTES;
#pragma unroll
                            for (int kk = 0; kk < 4; ++kk)
                                umma(D, sdesc(a0 + 32 * kk, 16, 1024, 2), sdesc(b0 + 32 * kk, 16, 1024, 2), ID256,
                                     (c | kk) != 0);
                            umma_commit(BAR_EMPTY + 8 * slot);
                        }
                        ++na;
                        if (ok) umma_commit(BAR_D);
                    }
                    if (!ok) break;
                    // layer 4: A (128 x 256) x W4^T (16 x 256, resident) -> D1 columns 0..15
                    for (int c = 0; c < 4; ++c) {
                        ok = mbar_wait(BAR_A + 8 * c, na & 1, abort_flag);
                        if (!ok) break;
                        tc_after_sync();
                        const uint32_t a0 = s0 + SM_A + c * A_CHUNK_BYTES;
                        const uint32_t b0 = s0 + SM_W4 + c * W4_CHUNK_BYTES;
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            umma(D1, sdesc(a0 + 32 * kk, 16, 1024, 2), sdesc(b0 + 32 * kk, 16, 1024, 2), ID16,
                                 (c | kk) != 0);
                    }
                    ++na;
                    if (ok) umma_commit(BAR_D);
                }
            // drain: every MMA issued has completed before tensor memory is freed
            umma_commit(BAR_DRAIN);
            if (!mbar_wait_bounded(BAR_DRAIN, 0)) *abort_flag = 1;
        }
    } else {
        // ---------------------------------------------------- epilogue
        // warps 2..17: tensor-memory lane quarter warp % 4, column quarter
        // (warp - 2) / 4 of every 64-column chunk; the quarter-0 thread of a
        // row owns that state
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;          // column quarter 0..3
        const int row = quarter * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16) + 16 * half;
        uint32_t nd = 0;
        bool ok = true;
        for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            const int64_t p = tile * TC_M + row;
            float x[NOUT];
            if (p < n) {
                const float4 u = reinterpret_cast<const float4 *>(state)[2 * p];
                const float4 w = reinterpret_cast<const float4 *>(state)[2 * p + 1];
                x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w; x[4] = w.x; x[5] = w.y; x[6] = w.z; x[7] = w.w;
            } else {
#pragma unroll
                for (int i = 0; i < NOUT; ++i) x[i] = 0.0f;
            }
            bool act = p < n;
            int cnt = 0;
            for (int it = 0; it < n_apply && ok; ++it) {
                if (half == 0) {
                    if (radius2 > 0.0f)
                        act = act && (x[0] * x[0] + x[1] * x[1] <= radius2) &&
                              (x[2] * x[2] + x[3] * x[3] <= radius2) && (fabsf(x[4]) <= 1.0f);
                    // layer-1 input row: s0..s5 split into bfloat16 high and low
                    // parts (columns 0..5 and 6..11; W1 is stacked twice), so
                    // the product sees the float32 state, zero padding to 16
                    float xl[6];
#pragma unroll
                    for (int k = 0; k < 6; ++k) xl[k] = x[k] - __bfloat162float(__float2bfloat16_rn(x[k]));
                    uint4 lo, hi;
                    lo.x = pack_bf16(x[0], x[1]);
                    lo.y = pack_bf16(x[2], x[3]);
                    lo.z = pack_bf16(x[4], x[5]);
                    lo.w = pack_bf16(xl[0], xl[1]);
                    hi.x = pack_bf16(xl[2], xl[3]);
                    hi.y = pack_bf16(xl[4], xl[5]);
                    hi.z = 0u;
                    hi.w = 0u;
                    *reinterpret_cast<uint4 *>(sm + SM_X + core_off(row, 0)) = lo;
                    *reinterpret_cast<uint4 *>(sm + SM_X + core_off(row, 8)) = hi;
                    fence_async_smem();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(BAR_X);
                }
                // hidden layers: D0 (layer 1), D1 (layer 2), D0 (layer 3)
                for (int l = 0; l < 3 && ok; ++l) {
                    ok = __all_sync(0xffffffffu, mbar_wait(BAR_D, nd++ & 1, abort_flag));
                    if (!ok) break;
                    tc_after_sync();
                    const uint32_t src = lane_base + ((l == 1) ? 256u : 0u);
                    const float *hb = sbias + l * H + 16 * half;
                    unsigned char *arow = sm + SM_A + row * 128;
                    uint32_t va[16], vb[16];
                    TMEM_LD16(src, va);
                    tmem_wait_ld();
                    REG_FENCE16(va);
                    // chunk c is converted while chunk c + 1 is in flight
#define EPI_CHUNK(c, cur, nxt)                                                                           \
    {                                                                                                    \
        if ((c) < 3) TMEM_LD16(src + ((c) + 1) * TC_CHUNK, nxt);                                         \
        _Pragma("unroll") for (int j = 0; j < 2; ++j)                                                    \
        {                                                                                                \
            const uint4 o = silu8(cur + 8 * j, hb + (c) * TC_CHUNK + 8 * j);                            \
            *reinterpret_cast<uint4 *>(arow + (c) * A_CHUNK_BYTES + (((2 * half + j) ^ (row & 7)) << 4)) = o; \
        }                                                                                                \
        fence_async_smem();                                                                              \
        if ((c) < 3) {                                                                                   \
            tmem_wait_ld();                                                                              \
            REG_FENCE16(nxt);                                                                            \
        }                                                                                                \
        tc_before_sync();                                                                                \
        __syncwarp();                                                                                    \
        if (lane == 0) mbar_arrive(BAR_A + 8 * (c));                                                     \
    }
                    EPI_CHUNK(0, va, vb)
                    EPI_CHUNK(1, vb, va)
                    EPI_CHUNK(2, va, vb)
                    EPI_CHUNK(3, vb, va)
#undef EPI_CHUNK
                }
                if (!ok) break;
                // layer 4 and the residual update
                ok = __all_sync(0xffffffffu, mbar_wait(BAR_D, nd++ & 1, abort_flag));
                if (!ok) break;
                if (half == 0) {
                    tc_after_sync();
                    uint32_t f[16];
                    TMEM_LD16(lane_base + 256, f);
                    tmem_wait_ld();
                    REG_FENCE16(f);
                    tc_before_sync();
                    if (act) {
                        float y[4], q[15];
                        quad_features(x, q);
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            float lin = stail[72 + c];
#pragma unroll
                            for (int k = 0; k < 6; ++k) lin = fmaf(x[k], stail[8 + k * NOUT + c], lin);
#pragma unroll
                            for (int m = 0; m < 15; ++m) lin = fmaf(q[m], stail[80 + m * NOUT + c], lin);
                            y[c] = x[c] + (lin + (__uint_as_float(f[c]) + stail[c]));
                        }
#pragma unroll
                        for (int c = 0; c < 4; ++c) x[c] = y[c];
                        ++cnt;
                    }
                }
            }
            if (half == 0 && p < n && ok) {
                reinterpret_cast<float4 *>(state)[2 * p] = make_float4(x[0], x[1], x[2], x[3]);
                reinterpret_cast<float4 *>(state)[2 * p + 1] = make_float4(x[4], x[5], x[6], x[7]);
                if (applied) applied[p] = cnt;
            }
        }
    }
    // teardown: the MMA thread has drained its MMAs, the epilogue its loads
    tc_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
    if (threadIdx.x == 0 && *abort_flag && error) atomicExch(error, 1);
}

// ------------------------------------------------ paired-tile inference
// Two 128-state tiles per CTA in flight (slots 0 and 1), each with one
// 256-column accumulator (D_s = tensor-memory columns 256 s .. 256 s + 255),
// its own activation operand A_s and layer-1 input X_s in shared memory.
// The epilogue warps alternate between the slots layer by layer,
//   E(0, l)  E(1, l)  E(0, l + 1)  E(1, l + 1) ...
// and the MMA thread issues in the same order, so the tensor cores run one
// slot's layer while the epilogue converts the other slot's.  The MMAs of a
// slot's next layer overwrite its accumulator: they wait for d_free[s], which
// the epilogue warps signal once their last tensor-memory load of D_s has
// completed (before the last chunk is converted), besides the A_s chunks.
// W2 / W3 stream through a ring of two 32 KB slots, once per slot and layer.
// A CTA's tiles are t, t + G (a pair), t + 2G, t + 3G, ... (G = grid size);
// an unpaired last tile runs in slot 0 alone.
constexpr int RING2 = 2;
constexpr uint32_t S2_A = 0;                                   // A_0, A_1: 64 KB each
constexpr uint32_t S2_RING = S2_A + 2 * 4 * A_CHUNK_BYTES;
constexpr uint32_t S2_W4 = S2_RING + RING2 * W_CHUNK_BYTES;
constexpr uint32_t S2_W1 = S2_W4 + 4 * W4_CHUNK_BYTES;
constexpr uint32_t S2_X = S2_W1 + H * KIN * 2;                 // X_0, X_1: 4 KB each
constexpr uint32_t S2_XB = TC_M * KIN * 2;
constexpr uint32_t S2_BIAS = S2_X + 2 * S2_XB;
constexpr uint32_t S2_TAIL = S2_BIAS + 3 * H * 4;
constexpr uint32_t S2_BAR = S2_TAIL + 208 * 4;
// x_ready[2], a_ready[2][4], d_full[2], d_free[2], full[RING2], empty[RING2], drain
constexpr int NBAR2 = 2 + 8 + 2 + 2 + 2 * RING2 + 1;
constexpr uint32_t S2_MISC = S2_BAR + NBAR2 * 8;
constexpr uint32_t S2_TOTAL = S2_MISC + 16;
constexpr size_t TC2_SMEM = S2_TOTAL + 1024;
static_assert(TC2_SMEM <= 232448, "paired inference: shared memory per block");

__global__ void __launch_bounds__(TC_THREADS, 1)
    mlp_infer_tc2_kernel(const float *__restrict__ P, const unsigned char *__restrict__ wp, float *__restrict__ state,
                         int32_t *__restrict__ applied, int32_t *__restrict__ error, int64_t n, int n_apply,
                         float radius2)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t s0 = smem_u32(sm);
    float *sbias = reinterpret_cast<float *>(sm + S2_BIAS);
    float *stail = reinterpret_cast<float *>(sm + S2_TAIL);   // b4[0..7], Ws[8..71], bs[72..79], Wq[80..207]
    const uint32_t bar0 = s0 + S2_BAR;
    const uint32_t BAR_X = bar0, BAR_A = bar0 + 16, BAR_D = bar0 + 80, BAR_F = bar0 + 96, BAR_FULL = bar0 + 112,
                   BAR_EMPTY = BAR_FULL + 8 * RING2, BAR_DRAIN = BAR_EMPTY + 8 * RING2;
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(sm + S2_MISC);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + S2_MISC + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ntiles = (n + TC_M - 1) / TC_M, G = gridDim.x;

    for (int i = threadIdx.x; i < (int)(H * KIN * 2 / 16); i += blockDim.x)
        reinterpret_cast<uint4 *>(sm + S2_W1)[i] = reinterpret_cast<const uint4 *>(wp + PK_W1)[i];
    for (int i = threadIdx.x; i < (int)(4 * W4_CHUNK_BYTES / 16); i += blockDim.x)
        reinterpret_cast<uint4 *>(sm + S2_W4)[i] = reinterpret_cast<const uint4 *>(wp + PK_W4)[i];
    for (int i = threadIdx.x; i < 3 * H; i += blockDim.x) sbias[i] = 0.5f * P[(i < H ? P_B1 : i < 2 * H ? P_B2 : P_B3) + (i % H)];
    for (int i = threadIdx.x; i < 208; i += blockDim.x)
        stail[i] = i < 8 ? P[P_B4 + i] : i < 72 ? P[P_WS + (i - 8)] : i < 80 ? P[P_BS + (i - 72)] : P[P_WQ + (i - 80)];
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(BAR_X + 8 * s, 4);
            for (int c = 0; c < 4; ++c) mbar_init(BAR_A + 8 * (4 * s + c), 16);
            mbar_init(BAR_D + 8 * s, 1);
            mbar_init(BAR_F + 8 * s, 16);
        }
        for (int r = 0; r < RING2; ++r) {
            mbar_init(BAR_FULL + 8 * r, 1);
            mbar_init(BAR_EMPTY + 8 * r, 1);
        }
        mbar_init(BAR_DRAIN, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tmem_holder;

    if (warp == 0) {
        // ---------------------------------------------------- weight stream
        // consumption order of the MMA thread: per map, W2 for slot 0, W2 for
        // slot 1, W3 for slot 0, W3 for slot 1, four chunks each
        if (lane == 0) {
            uint32_t q = 0;
            for (int64_t t0 = blockIdx.x; t0 < ntiles && !*abort_flag; t0 += 2 * G) {
                const int ns = t0 + G < ntiles ? 2 : 1;
                for (int it = 0; it < n_apply && !*abort_flag; ++it)
                    for (int l = 0; l < 2; ++l)
                        for (int s = 0; s < ns; ++s)
                            for (int c = 0; c < 4; ++c, ++q) {
                                const uint32_t slot = q % RING2, use = q / RING2;
                                if (!mbar_wait(BAR_EMPTY + 8 * slot, (use & 1) ^ 1, abort_flag)) break;
                                mbar_expect_tx(BAR_FULL + 8 * slot, W_CHUNK_BYTES);
                                bulk_load(s0 + S2_RING + slot * W_CHUNK_BYTES,
                                          wp + (l == 0 ? PK_W2 : PK_W3) + c * W_CHUNK_BYTES, W_CHUNK_BYTES,
                                          BAR_FULL + 8 * slot);
                            }
            }
            // drain: every issued copy has landed before the block exits
            const uint32_t issued = q;
            for (uint32_t r = issued > RING2 ? issued - RING2 : 0; r < issued; ++r)
                if (!mbar_wait_bounded(BAR_FULL + 8 * (r % RING2), (r / RING2) & 1)) *abort_flag = 1;
        }
    } else if (warp == 1) {
        // ---------------------------------------------------- MMA issue
        if (lane == 0) {
            const uint32_t ID256 = idesc_bf16(TC_M, H), ID16 = idesc_bf16(TC_M, 16);
            uint32_t q = 0, nx[2] = {0, 0}, na[2] = {0, 0}, nb[2] = {0, 0};
            bool ok = true;
            for (int64_t t0 = blockIdx.x; t0 < ntiles && ok; t0 += 2 * G) {
                const int ns = t0 + G < ntiles ? 2 : 1;
                for (int it = 0; it < n_apply && ok; ++it)
                    for (int layer = 0; layer < 4 && ok; ++layer)
                        for (int s = 0; s < ns && ok; ++s) {
                            const uint32_t D = tmem + 256 * s;
                            // the accumulator's previous contents have been read
                            if (nb[s] > 0) ok = mbar_wait(BAR_F + 8 * s, (nb[s] - 1) & 1, abort_flag);
                            ++nb[s];
                            if (!ok) break;
                            if (layer == 0) {
                                // layer 1: X_s (128 x 16) x W1^T -> D_s
                                ok = mbar_wait(BAR_X + 8 * s, nx[s]++ & 1, abort_flag);
                                if (!ok) break;
                                tc_after_sync();
                                umma(D, sdesc(s0 + S2_X + s * S2_XB, 128, 256, 0), sdesc(s0 + S2_W1, 128, 256, 0), ID256, 0);
                            } else if (layer < 3) {
                                // layers 2, 3: A_s (128 x 256) x W^T (streamed) -> D_s
                                for (int c = 0; c < 4; ++c, ++q) {
                                    const uint32_t slot = q % RING2, use = q / RING2;
                                    ok = mbar_wait(BAR_A + 8 * (4 * s + c), na[s] & 1, abort_flag) &&
                                         mbar_wait(BAR_FULL + 8 * slot, use & 1, abort_flag);
                                    if (!ok) break;
                                    tc_after_sync();
                                    const uint32_t a0 = s0 + S2_A + (4 * s + c) * A_CHUNK_BYTES;
                                    const uint32_t b0 = s0 + S2_RING + slot * W_CHUNK_BYTES;
#pragma unroll
                                    for (int kk = 0; kk < 4; ++kk)
                                        umma(D, sdesc(a0 + 32 * kk, 16, 1024, 2), sdesc(b0 + 32 * kk, 16, 1024, 2),
                                             ID256, (c | kk) != 0);
                                    umma_commit(BAR_EMPTY + 8 * slot);
                                }
                                ++na[s];
                            } else {
                                // layer 4: A_s x W4^T (16 x 256, resident) -> D_s columns 0..15
                                for (int c = 0; c < 4; ++c) {
                                    ok = mbar_wait(BAR_A + 8 * (4 * s + c), na[s] & 1, abort_flag);
                                    if (!ok) break;
                                    tc_after_sync();
                                    const uint32_t a0 = s0 + S2_A + (4 * s + c) * A_CHUNK_BYTES;
                                    const uint32_t b0 = s0 + S2_W4 + c * W4_CHUNK_BYTES;
#pragma unroll
                                    for (int kk = 0; kk < 4; ++kk)
                                        umma(D, sdesc(a0 + 32 * kk, 16, 1024, 2), sdesc(b0 + 32 * kk, 16, 1024, 2),
                                             ID16, (c | kk) != 0);
                                }
                                ++na[s];
                            }
                            if (ok) umma_commit(BAR_D + 8 * s);
                        }
            }
            // drain: every MMA issued has completed before tensor memory is freed
            umma_commit(BAR_DRAIN);
            if (!mbar_wait_bounded(BAR_DRAIN, 0)) *abort_flag = 1;
        }
    } else {
        // ---------------------------------------------------- epilogue
        // warps 2..17: tensor-memory lane quarter warp % 4, column quarter
        // (warp - 2) / 4 of every 64-column chunk; the quarter-0 thread of a
        // row owns that row's state in both slots
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;          // column quarter 0..3
        const int row = quarter * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16) + 16 * half;
        uint32_t nd[2] = {0, 0};
        bool ok = true;
        // layer-1 input row of slot s (quarter-0 threads): the domain test, then
        // s0..s5 split into bfloat16 high and low parts (columns 0..5 and 6..11;
        // W1 is stacked twice), zero padding to 16
        auto write_x = [&](const float *x, bool &act, int s) {
            if (radius2 > 0.0f)
                act = act && (x[0] * x[0] + x[1] * x[1] <= radius2) && (x[2] * x[2] + x[3] * x[3] <= radius2) &&
                      (fabsf(x[4]) <= 1.0f);
            float xl[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) xl[k] = x[k] - __bfloat162float(__float2bfloat16_rn(x[k]));
            uint4 lo, hi;
            lo.x = pack_bf16(x[0], x[1]);
            lo.y = pack_bf16(x[2], x[3]);
            lo.z = pack_bf16(x[4], x[5]);
            lo.w = pack_bf16(xl[0], xl[1]);
            hi.x = pack_bf16(xl[2], xl[3]);
            hi.y = pack_bf16(xl[4], xl[5]);
            hi.z = 0u;
            hi.w = 0u;
            unsigned char *xb = sm + S2_X + s * S2_XB;
            *reinterpret_cast<uint4 *>(xb + core_off(row, 0)) = lo;
            *reinterpret_cast<uint4 *>(xb + core_off(row, 8)) = hi;
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(BAR_X + 8 * s);
        };
        // layer 4 of slot s: the fitted outputs, the float32 skip connection
        auto update = [&](float *x, bool act, int &cnt, const uint32_t *f) {
            if (!act) return;
            float y[4], q[15];
            quad_features(x, q);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float lin = stail[72 + c];
#pragma unroll
                for (int k = 0; k < 6; ++k) lin = fmaf(x[k], stail[8 + k * NOUT + c], lin);
#pragma unroll
                for (int m = 0; m < 15; ++m) lin = fmaf(q[m], stail[80 + m * NOUT + c], lin);
                y[c] = x[c] + (lin + (__uint_as_float(f[c]) + stail[c]));
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) x[c] = y[c];
            ++cnt;
        };
        for (int64_t t0 = blockIdx.x; t0 < ntiles && ok; t0 += 2 * G) {
            const int ns = t0 + G < ntiles ? 2 : 1;
            const int64_t p0 = t0 * TC_M + row, p1 = (t0 + G) * TC_M + row;
            float x0[NOUT], x1[NOUT];
            bool act0 = p0 < n, act1 = ns == 2 && p1 < n;
            int cnt0 = 0, cnt1 = 0;
            if (half == 0) {
#pragma unroll
                for (int i = 0; i < NOUT; ++i) x0[i] = x1[i] = 0.0f;
                if (act0) {
                    const float4 u = reinterpret_cast<const float4 *>(state)[2 * p0];
                    const float4 w = reinterpret_cast<const float4 *>(state)[2 * p0 + 1];
                    x0[0] = u.x; x0[1] = u.y; x0[2] = u.z; x0[3] = u.w; x0[4] = w.x; x0[5] = w.y; x0[6] = w.z; x0[7] = w.w;
                }
                if (act1) {
                    const float4 u = reinterpret_cast<const float4 *>(state)[2 * p1];
                    const float4 w = reinterpret_cast<const float4 *>(state)[2 * p1 + 1];
                    x1[0] = u.x; x1[1] = u.y; x1[2] = u.z; x1[3] = u.w; x1[4] = w.x; x1[5] = w.y; x1[6] = w.z; x1[7] = w.w;
                }
                write_x(x0, act0, 0);
                if (ns == 2) write_x(x1, act1, 1);
            }
            for (int it = 0; it < n_apply && ok; ++it) {
                // hidden layers 1..3 of slot 0, then slot 1
                for (int l = 0; l < 3 && ok; ++l)
                    for (int s = 0; s < ns && ok; ++s) {
                        ok = __all_sync(0xffffffffu, mbar_wait(BAR_D + 8 * s, nd[s]++ & 1, abort_flag));
                        if (!ok) break;
                        tc_after_sync();
                        const uint32_t src = lane_base + 256u * s;
                        const float *hb = sbias + l * H + 16 * half;
                        unsigned char *arow = sm + S2_A + s * (4 * A_CHUNK_BYTES) + row * 128;
                        const uint32_t bar_a = BAR_A + 8 * (4 * s), bar_f = BAR_F + 8 * s;
                        uint32_t va[16], vb[16];
                        TMEM_LD16(src, va);
                        tmem_wait_ld();
                        REG_FENCE16(va);
                        // chunk c is converted while chunk c + 1 is in flight; once
                        // chunk 3 has landed, D_s is free for the next layer's MMAs
#define EPI2_CHUNK(c, cur, nxt)                                                                          \
    {                                                                                                    \
        if ((c) < 3) TMEM_LD16(src + ((c) + 1) * TC_CHUNK, nxt);                                         \
        _Pragma("unroll") for (int j = 0; j < 2; ++j)                                                    \
        {                                                                                                \
            const uint4 o = silu8(cur + 8 * j, hb + (c) * TC_CHUNK + 8 * j);                            \
            *reinterpret_cast<uint4 *>(arow + (c) * A_CHUNK_BYTES + (((2 * half + j) ^ (row & 7)) << 4)) = o; \
        }                                                                                                \
        fence_async_smem();                                                                              \
        if ((c) < 3) {                                                                                   \
            tmem_wait_ld();                                                                              \
            REG_FENCE16(nxt);                                                                            \
        }                                                                                                \
        tc_before_sync();                                                                                \
        __syncwarp();                                                                                    \
        if (lane == 0) {                                                                                 \
            mbar_arrive(bar_a + 8 * (c));                                                                \
            if ((c) == 2) mbar_arrive(bar_f);                                                            \
        }                                                                                                \
    }
                        EPI2_CHUNK(0, va, vb)
                        EPI2_CHUNK(1, vb, va)
                        EPI2_CHUNK(2, va, vb)
                        EPI2_CHUNK(3, vb, va)
#undef EPI2_CHUNK
                    }
                if (!ok) break;
                // layer 4 and the residual update per slot, then that slot's
                // layer-1 input of the next map
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    if (s >= ns || !ok) break;
                    ok = __all_sync(0xffffffffu, mbar_wait(BAR_D + 8 * s, nd[s]++ & 1, abort_flag));
                    if (!ok) break;
                    uint32_t f[16];
                    if (half == 0) {
                        tc_after_sync();
                        TMEM_LD16(lane_base + 256u * s, f);
                        tmem_wait_ld();
                        REG_FENCE16(f);
                    }
                    tc_before_sync();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(BAR_F + 8 * s);
                    if (half == 0) {
                        if (s == 0) {
                            update(x0, act0, cnt0, f);
                            if (it + 1 < n_apply) write_x(x0, act0, 0);
                        } else {
                            update(x1, act1, cnt1, f);
                            if (it + 1 < n_apply) write_x(x1, act1, 1);
                        }
                    }
                }
            }
            if (half == 0 && ok) {
                if (p0 < n) {
                    reinterpret_cast<float4 *>(state)[2 * p0] = make_float4(x0[0], x0[1], x0[2], x0[3]);
                    reinterpret_cast<float4 *>(state)[2 * p0 + 1] = make_float4(x0[4], x0[5], x0[6], x0[7]);
                    if (applied) applied[p0] = cnt0;
                }
                if (ns == 2 && p1 < n) {
                    reinterpret_cast<float4 *>(state)[2 * p1] = make_float4(x1[0], x1[1], x1[2], x1[3]);
                    reinterpret_cast<float4 *>(state)[2 * p1 + 1] = make_float4(x1[4], x1[5], x1[6], x1[7]);
                    if (applied) applied[p1] = cnt1;
                }
            }
        }
    }
    // teardown: the MMA thread has drained its MMAs, the epilogue its loads
    tc_before_sync();
    __syncthreads();
    if (warp == 1) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
    if (threadIdx.x == 0 && *abort_flag && error) atomicExch(error, 1);
}

// ------------------------------------------------- GEMM (training, tcgen05)
// The training products of at least 128 x 128 x 64 on the 5th-generation
// tensor cores: C[M][N] = op(A) op(B) (+ bias) with the operands and the
// meaning of transA / transB of gemm_tc.  One CTA of sixteen warps per
// 128 x 128 output tile (and per K split, gridDim.z, as in gemm_tc); K is
// staged 64 at a time: every thread loads its 16 + 16 float32 of the step
// from global memory along the index that is contiguous there (into
// registers, one step ahead), rounds to bfloat16 (as gemm_tc does) and
// stores into a 128-byte-swizzled K-major tile (A: 128 m-rows, B: 128
// n-rows, 128 bytes of k each), two stages; one thread issues the four
// K = 16 MMAs of a stage into a 128-column TMEM accumulator and commits them
// to that stage's mbarrier, which frees the stage for the store two steps
// later.  Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its 32 output
// rows) and 32 columns, adds the bias and stores float32.  Waits are
// bounded: on a timeout the tile is written as NaN and g_gemm_timeouts is
// counted.
constexpr int G5_BM = 128, G5_BN = 128, G5_BK = 64, G5_STAGES = 2, G5_THREADS = 512;
constexpr uint32_t G5_TILE = 128 * 128;                               // one operand stage: 16 KB
constexpr uint32_t G5_SM_A = 0;
constexpr uint32_t G5_SM_B = G5_SM_A + G5_STAGES * G5_TILE;
constexpr uint32_t G5_SM_BAR = G5_SM_B + G5_STAGES * G5_TILE;        // one mbarrier per stage
constexpr uint32_t G5_SM_MISC = G5_SM_BAR + 8 * G5_STAGES;            // tmem base, abort flag
constexpr size_t G5_SMEM = G5_SM_MISC + 16 + 1024;                    // + alignment slack
constexpr uint32_t G5_TMEM_COLS = 128;
constexpr int G5_PER = G5_BM * G5_BK / G5_THREADS;                    // floats per thread per operand: 16
static_assert(G5_PER == 16, "staging split");

__device__ int g_gemm_timeouts;

// This thread's share of rows [r0, r0 + 128) x k [k0, k0 + 64) of op(X)
// (X[r ld + k] when kcont, else X[k ld + r]) into registers; rows >= nrows
// and k >= kend read as 0.  kcont: 8 threads per row, two runs of 8
// consecutive k each (a row's 256 bytes over 8 lanes); otherwise one row per
// thread and 16 consecutive k (every load 32 consecutive rows of one k).
__device__ __forceinline__ void g5_load(float v[G5_PER], const float *__restrict__ X, int ld, bool kcont, bool vec,
                                        int r0, int nrows, int k0, int kend)
{
    const int t = threadIdx.x;
    if (kcont) {
#pragma unroll
        for (int it = 0; it < 2; ++it) {
            const int id = t + G5_THREADS * it;
            const int gr = r0 + (id >> 3), gk = k0 + 8 * (id & 7);
            if (gr < nrows && vec && gk + 8 <= kend) {
                const float4 *src = reinterpret_cast<const float4 *>(X + (int64_t)gr * ld + gk);
                const float4 a = __ldg(src), b = __ldg(src + 1);
                v[8 * it + 0] = a.x; v[8 * it + 1] = a.y; v[8 * it + 2] = a.z; v[8 * it + 3] = a.w;
                v[8 * it + 4] = b.x; v[8 * it + 5] = b.y; v[8 * it + 6] = b.z; v[8 * it + 7] = b.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    v[8 * it + j] = (gr < nrows && gk + j < kend) ? __ldg(X + (int64_t)gr * ld + gk + j) : 0.0f;
            }
        }
    } else {
        const int gr = r0 + (t & 127), kq = k0 + 16 * (t >> 7);
        const bool rok = gr < nrows;
#pragma unroll
        for (int j = 0; j < G5_PER; ++j) v[j] = (rok && kq + j < kend) ? __ldg(X + (int64_t)(kq + j) * ld + gr) : 0.0f;
    }
}

// the registers of g5_load as bfloat16 into a 128-byte-swizzled K-major stage
__device__ __forceinline__ void g5_store(unsigned char *dst, const float v[G5_PER], bool kcont)
{
    const int t = threadIdx.x;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        int row, c;
        if (kcont) {
            const int id = t + G5_THREADS * h;
            row = id >> 3;
            c = id & 7;
        } else {
            row = t & 127;
            c = 2 * (t >> 7) + h;
        }
        *reinterpret_cast<uint4 *>(dst + row * 128 + ((c ^ (row & 7)) << 4)) =
            make_uint4(pack_bf16(v[8 * h], v[8 * h + 1]), pack_bf16(v[8 * h + 2], v[8 * h + 3]),
                       pack_bf16(v[8 * h + 4], v[8 * h + 5]), pack_bf16(v[8 * h + 6], v[8 * h + 7]));
    }
}

__global__ void __launch_bounds__(G5_THREADS) gemm_tc05(const float *__restrict__ A, int lda, int transA,
                                                        const float *__restrict__ B, int ldb, int transB,
                                                        float *__restrict__ C, int ldc, int M, int N, int K,
                                                        const float *__restrict__ bias, int k_chunk, int vecA, int vecB)
{
    extern __shared__ unsigned char g5_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(g5_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t s0 = smem_u32(sm);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(sm + G5_SM_MISC);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + G5_SM_MISC + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * G5_BM, n0 = blockIdx.x * G5_BN;
    const int kb = blockIdx.z * k_chunk, ke = min(K, kb + k_chunk);
    if (gridDim.z > 1) {
        C += (int64_t)blockIdx.z * M * N;
        ldc = N;
        bias = nullptr;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < G5_STAGES; ++s) mbar_init(s0 + G5_SM_BAR + 8 * s, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(G5_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    const int nk = ke > kb ? (ke - kb + G5_BK - 1) / G5_BK : 0;
    const bool kcA = !transA, kcB = transB != 0;
    float va[G5_PER], vb[G5_PER];
    if (nk > 0) {                                  // the first K step's loads overlap the set-up barrier
        g5_load(va, A, lda, kcA, vecA != 0, m0, M, kb, ke);
        g5_load(vb, B, ldb, kcB, vecB != 0, n0, N, kb, ke);
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tmem_holder;
    constexpr uint32_t IDESC = idesc_bf16(G5_BM, G5_BN);
    int issued = 0;                                // commits made (thread 0)
    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % G5_STAGES;
        const uint32_t bar = s0 + G5_SM_BAR + 8 * s;
        if (kt >= G5_STAGES) {
            // the MMAs that read this stage two steps ago have completed
            if (threadIdx.x == 0) mbar_wait(bar, ((kt / G5_STAGES) - 1) & 1, abort_flag);
            __syncthreads();
            if (*abort_flag) break;                // read by every thread after the barrier
        }
        g5_store(sm + G5_SM_A + s * G5_TILE, va, kcA);
        g5_store(sm + G5_SM_B + s * G5_TILE, vb, kcB);
        if (kt + 1 < nk) {                         // next K step in flight during the MMAs
            const int k1 = kb + (kt + 1) * G5_BK;
            g5_load(va, A, lda, kcA, vecA != 0, m0, M, k1, ke);
            g5_load(vb, B, ldb, kcB, vecB != 0, n0, N, k1, ke);
        }
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_after_sync();
            const uint32_t a0 = s0 + G5_SM_A + s * G5_TILE, b0 = s0 + G5_SM_B + s * G5_TILE;
#pragma unroll
            for (int kk = 0; kk < G5_BK / 16; ++kk)
                umma(tmem, sdesc(a0 + 32 * kk, 16, 1024, 2), sdesc(b0 + 32 * kk, 16, 1024, 2), IDESC, (kt | kk) != 0);
            umma_commit(bar);
            ++issued;
        }
    }
    // the last commit covers every MMA of the tile
    if (threadIdx.x == 0 && issued > 0) {
        const int last = issued - 1;
        const uint32_t bar = s0 + G5_SM_BAR + 8 * (last % G5_STAGES);
        if (*abort_flag) mbar_wait_bounded(bar, (last / G5_STAGES) & 1);   // drain what is in flight
        else mbar_wait(bar, (last / G5_STAGES) & 1, abort_flag);
    }
    __syncthreads();
    tc_after_sync();
    const bool failed = *abort_flag != 0;
    // warp w: TMEM lanes 32 (w % 4) .. + 31 (its output rows), columns 32 (w / 4) .. + 31
    const int quarter = warp & 3, cg = warp >> 2;
    const int row = m0 + 32 * quarter + lane;
    const bool vecC = ((ldc & 3) == 0) && ((reinterpret_cast<uintptr_t>(C) & 15) == 0);
    uint32_t v[32];
    if (nk > 0 && !failed) {
        TMEM_LD32(tmem + ((uint32_t)(32 * quarter) << 16) + 32 * cg, v);
        tmem_wait_ld();
        REG_FENCE32(v);
    } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = failed ? 0x7FC00000u : 0u;
    }
    const int gn0 = n0 + 32 * cg;
    if (row < M && gn0 < N) {
        float *dst = C + (int64_t)row * ldc + gn0;
        if (vecC && gn0 + 32 <= N) {
#pragma unroll
            for (int j = 0; j < 32; j += 4) {
                float4 o = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]), __uint_as_float(v[j + 2]),
                                       __uint_as_float(v[j + 3]));
                if (bias) {
                    o.x += bias[gn0 + j]; o.y += bias[gn0 + j + 1]; o.z += bias[gn0 + j + 2]; o.w += bias[gn0 + j + 3];
                }
                *reinterpret_cast<float4 *>(dst + j) = o;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (gn0 + j < N) dst[j] = __uint_as_float(v[j]) + (bias ? bias[gn0 + j] : 0.0f);
        }
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(G5_TMEM_COLS));
    }
    if (threadIdx.x == 0 && failed) atomicAdd(&g_gemm_timeouts, 1);
}

bool g5_fits(int M, int N, int K) { return M >= G5_BM && N >= G5_BN && K >= G5_BK; }

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// one GEMM launch: the tcgen05 kernel for products of at least one full
// tile, gemm_tc for the narrow ones (N = 8 outputs, K = 8 inputs, M = 6)
cudaError_t launch_gemm(const float *A, int lda, int tA, const float *B, int ldb, int tB, float *C, int ldc, int M,
                        int N, int K, const float *bias, int k_chunk, int splits, cudaStream_t s)
{
    if (g5_fits(M, N, K)) {
        // once per process (one process per GPU); set outside any graph
        // capture: the first training step runs directly before the capture
        static bool attr = false;
        if (!attr) {
            const cudaError_t e = cudaFuncSetAttribute(gemm_tc05, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)G5_SMEM);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        const dim3 grid((unsigned)((N + G5_BN - 1) / G5_BN), (unsigned)((M + G5_BM - 1) / G5_BM), (unsigned)splits);
        const int vA = !tA && (lda & 3) == 0 && aligned16(A), vB = tB && (ldb & 3) == 0 && aligned16(B);
        gemm_tc05<<<grid, G5_THREADS, G5_SMEM, s>>>(A, lda, tA, B, ldb, tB, C, ldc, M, N, K, bias, k_chunk, vA, vB);
    } else {
        const dim3 grid((unsigned)((N + GT_N - 1) / GT_N), (unsigned)((M + GT_M - 1) / GT_M), (unsigned)splits);
        gemm_tc<<<grid, 128, 0, s>>>(A, lda, tA, B, ldb, tB, C, ldc, M, N, K, bias, k_chunk);
    }
    return cudaGetLastError();
}

int blocks_for(int64_t n, int tb) { return (int)((n + tb - 1) / tb < 4096 ? (n + tb - 1) / tb : 4096); }

}  // namespace

// ------------------------------------------------------------------ C ABI


static_assert(PK_TOTAL == FFA_MLP_WPACK_BYTES, "inference weight pack size");
static_assert(TC_SMEM <= 232448, "inference kernel shared memory");


extern "C" int ffa_mlp_gemm(const float *A, int lda, int transA, const float *B, int ldb, int transB, float *C,
                            int ldc, int M, int N, int K, const float *bias, void *stream)
{
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return FFA_ERR_INVALID;
    if ((M + GT_M - 1) / GT_M > 65535) return FFA_ERR_UNSUPPORTED;
    return launch_gemm(A, lda, transA ? 1 : 0, B, ldb, transB ? 1 : 0, C, ldc, M, N, K, bias, K, 1,
                       (cudaStream_t)stream) == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

extern "C" int ffa_mlp_gemm_timeouts(int32_t *count)
{
    if (!count) return FFA_ERR_INVALID;
    int v = 0;
    FFA_CHECK_CUDA(cudaMemcpyFromSymbol(&v, g_gemm_timeouts, sizeof(int)));
    const int zero = 0;
    FFA_CHECK_CUDA(cudaMemcpyToSymbol(g_gemm_timeouts, &zero, sizeof(int)));
    *count = v;
    return FFA_OK;
}

extern "C" int ffa_mlp_train_step(const ffa_mlp_train_desc *d, void *stream)
{
    if (!d || !d->params || !d->grads || !d->adam_m || !d->adam_v || !d->x || !d->target || !d->work ||
        !d->loss_part || d->batch <= 0 || d->n_fit < 1 || d->n_fit > 6)
        return FFA_ERR_INVALID;
    const bool sched = d->lr_table != nullptr;
    if (sched != (d->counter != nullptr)) return FFA_ERR_INVALID;
    if (!sched && d->lr > 0.0f && d->step < 1) return FFA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t B = d->batch;
    if (B > 65535LL * GT_M || B * H > INT32_MAX) return FFA_ERR_UNSUPPORTED;
    float *P = d->params, *G = d->grads;
    float *z1 = d->work, *h1 = z1 + B * H, *z2 = h1 + B * H, *h2 = z2 + B * H, *z3 = h2 + B * H, *h3 = z3 + B * H;
    float *f = h3 + B * H, *y = f + B * NOUT, *dd = y + B * NOUT, *dh = dd + B * NOUT, *dz = dh + B * H;
    const int ew = blocks_for(B * H, 256);
    const int Bi = (int)B;
    float *part = dz + B * H;                                    // split-K partials
    // split K over `splits` blocks per output tile (chunks a multiple of
    // `kq`), partials in the split-K area, summed in a fixed order (+ bias)
    auto gemm_split = [&](const float *A_, int lda_, int tA_, const float *B_, int ldb_, int tB_, float *C_, int ldc_,
                          int M_, int N_, int K_, const float *bias_, int splits, int kq) {
        const int kc = ((K_ + splits - 1) / splits + kq - 1) / kq * kq;
        splits = (K_ + kc - 1) / kc;
        if (splits <= 1) {
            launch_gemm(A_, lda_, tA_, B_, ldb_, tB_, C_, ldc_, M_, N_, K_, bias_, K_, 1, s);
        } else {
            launch_gemm(A_, lda_, tA_, B_, ldb_, tB_, part, N_, M_, N_, K_, nullptr, kc, splits, s);
            split_sum_kernel<<<(M_ * N_ + 255) / 256, 256, 0, s>>>(part, splits, M_, N_, C_, ldc_, bias_);
        }
    };
    auto max_splits = [&](int M_, int N_, int cap) {
        const int64_t room = SPLIT_WORK / ((int64_t)M_ * N_);
        return (int)(room < cap ? room : cap);
    };
    // products: the tcgen05 kernel whole; the narrow ones (N = 8 outputs)
    // split in K chunks of 64, as the partial-product area allows
    auto gemm = [&](const float *A_, int lda_, int tA_, const float *B_, int ldb_, int tB_, float *C_, int ldc_,
                    int M_, int N_, int K_, const float *bias_) {
        int splits = 1;
        if (!g5_fits(M_, N_, K_) && K_ >= 128) {
            splits = (K_ + 63) / 64;
            const int cap = max_splits(M_, N_, 64);
            splits = splits < cap ? splits : cap;
        }
        gemm_split(A_, lda_, tA_, B_, ldb_, tB_, C_, ldc_, M_, N_, K_, bias_, splits < 1 ? 1 : splits, GT_K);
    };
    // weight gradients (K = batch): chunks of 512 on the tcgen05 path (up to
    // 16 splits), 256 on gemm_tc (up to 64)
    auto gemm_wgrad = [&](const float *A_, int lda_, const float *B_, int ldb_, float *C_, int ldc_, int M_, int N_) {
        const bool tc05 = g5_fits(M_, N_, (int)B);
        const int64_t per = tc05 ? 512 : 256;
        int splits = (int)((B + per - 1) / per);
        const int cap = max_splits(M_, N_, tc05 ? SPLITS_MAX : 64);
        splits = splits < 1 ? 1 : splits > cap ? cap : splits;
        gemm_split(A_, lda_, 1, B_, ldb_, 0, C_, ldc_, M_, N_, (int)B, nullptr, splits, tc05 ? G5_BK : GT_K);
    };
    // bias gradients: column sums in two fixed-order passes (scratch: the
    // split-K area, free between products)
    auto colsum = [&](const float *d_, int ncol, int ld_, float *g_) {
        int chunks = (int)((B + 127) / 128);
        chunks = chunks > 64 ? 64 : chunks;
        const int64_t rows_per = (B + chunks - 1) / chunks;
        chunks = (int)((B + rows_per - 1) / rows_per);
        colsum_part_kernel<<<dim3((unsigned)((ncol + 31) / 32), (unsigned)chunks), 256, 0, s>>>(d_, B, ncol, ld_,
                                                                                              rows_per, part);
        colsum_final_kernel<<<(ncol + 7) / 8, 256, 0, s>>>(part, chunks, ncol, g_);
    };
    // forward
    layer1_kernel<<<ew, 256, 0, s>>>(d->x, P, z1, B);
    silu_kernel<<<ew, 256, 0, s>>>(z1, h1, B * H);
    gemm(h1, H, 0, P + P_W2, H, 0, z2, H, Bi, H, H, P + P_B2);
    silu_kernel<<<ew, 256, 0, s>>>(z2, h2, B * H);
    gemm(h2, H, 0, P + P_W3, H, 0, z3, H, Bi, H, H, P + P_B3);
    silu_kernel<<<ew, 256, 0, s>>>(z3, h3, B * H);
    gemm(h3, H, 0, P + P_W4, NOUT, 0, f, NOUT, Bi, NOUT, H, P + P_B4);
    out_grad_kernel<<<148, 256, 0, s>>>(d->x, d->target, f, P, y, dd, B, d->n_fit, d->loss_part);
    // backward
    FFA_CHECK_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * P_TOTAL, s));
    skip_grad_kernel<<<NOUT + 16, 256, 0, s>>>(d->x, dd, B, G);
    colsum(dd, NOUT, NOUT, G + P_BS);
    gemm_wgrad(h3, H, dd, NOUT, G + P_W4, NOUT, H, NOUT);
    colsum(dd, NOUT, NOUT, G + P_B4);
    gemm(dd, NOUT, 0, P + P_W4, NOUT, 1, dh, H, Bi, H, NOUT, nullptr);
    const float *zs[3] = {z3, z2, z1};
    const float *hin[3] = {h2, h1, d->x};
    const int64_t wofs[3] = {P_W3, P_W2, P_W1}, bofs[3] = {P_B3, P_B2, P_B1};
    const int ldin[3] = {H, H, NOUT}, kin[3] = {H, H, 6};
    for (int l = 0; l < 3; ++l) {
        dsilu_kernel<<<ew, 256, 0, s>>>(dh, zs[l], B * H);   // dh -> dz in place
        gemm_wgrad(hin[l], ldin[l], dh, H, G + wofs[l], H, kin[l], H);
        colsum(dh, H, H, G + bofs[l]);
        if (l < 2) {
            gemm(dh, H, 0, P + wofs[l], H, 1, dz, H, Bi, H, H, nullptr);
            float *t = dh;
            dh = dz;
            dz = t;
        }
    }
    if (sched) {
        adam_sched_kernel<<<blocks_for(P_TOTAL, 256), 256, 0, s>>>(P, G, d->adam_m, d->adam_v, P_TOTAL, d->lr_table,
                                                                   d->counter, d->beta1, d->beta2, d->eps, d->mask);
        counter_advance_kernel<<<1, 1, 0, s>>>(d->counter);
    } else if (d->lr > 0.0f) {
        const float c1 = 1.0f - powf(d->beta1, (float)d->step), c2 = 1.0f - powf(d->beta2, (float)d->step);
        adam_kernel<<<blocks_for(P_TOTAL, 256), 256, 0, s>>>(P, G, d->adam_m, d->adam_v, P_TOTAL, d->lr, d->beta1,
                                                             d->beta2, d->eps, c1, c2, d->mask);
    }
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}


extern "C" int ffa_mlp_pack(const float *params, void *wpack, void *stream)
{
    if (!params || !wpack || (reinterpret_cast<uintptr_t>(wpack) & 15)) return FFA_ERR_INVALID;
    pack_weights_kernel<<<(H * H + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params, reinterpret_cast<unsigned char *>(wpack));
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

extern "C" int ffa_mlp_infer(const ffa_mlp_infer_desc *d, void *stream)
{
    if (!d || !d->params || !d->wpack || !d->state || d->n < 0 || d->n_apply < 0 ||
        (reinterpret_cast<uintptr_t>(d->wpack) & 15) || (reinterpret_cast<uintptr_t>(d->state) & 15))
        return FFA_ERR_INVALID;
    if (d->n == 0 || d->n_apply == 0) {
        if (d->applied && d->n > 0) FFA_CHECK_CUDA(cudaMemsetAsync(d->applied, 0, sizeof(int32_t) * d->n, (cudaStream_t)stream));
        return FFA_OK;
    }
    int dev = 0, sms = 0;
    FFA_CHECK_CUDA(cudaGetDevice(&dev));
    FFA_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t tiles = (d->n + TC_M - 1) / TC_M;
    const int grid = (int)(tiles < sms ? tiles : sms);
    if (tiles > sms) {
        // more tiles than SMs: two tiles in flight per SM
        FFA_CHECK_CUDA(cudaFuncSetAttribute(mlp_infer_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)TC2_SMEM));
        mlp_infer_tc2_kernel<<<grid, TC_THREADS, TC2_SMEM, (cudaStream_t)stream>>>(
            d->params, reinterpret_cast<const unsigned char *>(d->wpack), d->state, d->applied, d->error, d->n,
            d->n_apply, d->radius2);
    } else {
        FFA_CHECK_CUDA(cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)TC_SMEM));
        mlp_infer_tc_kernel<<<grid, TC_THREADS, TC_SMEM, (cudaStream_t)stream>>>(
            d->params, reinterpret_cast<const unsigned char *>(d->wpack), d->state, d->applied, d->error, d->n,
            d->n_apply, d->radius2);
    }
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}
