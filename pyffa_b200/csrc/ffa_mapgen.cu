// ffa_mapgen.cu -- z-Taylor coefficient tables of a scaling FFA map.
//
// The reference builds every table entry term by term on the CPU
// (Generate_Bmaps, src/FFAG_HighOrder.py:828-911): for each radius and each
// Laplacian term it re-evaluates the flutter derivatives on the whole theta
// grid, ~18 minutes per 1301 x 6000 map on 8 processes.  All r-dependence of
// an entry factors out of the theta-dependence, so here the host reduces the
// term algebra to a few weights per (component, order, radius, derivative
// order p), and the device does the two array passes that are left:
//   1. flutter_kernel: G^(p)(theta_j) for p < n_deriv, one thread per theta
//      node (sigmoid-derivative polynomials, src/FFAG_HighOrder.py:212-350);
//   2. mean_kernel: the sector mean of G (the reference's MeanF);
//   3. expand_kernel: T[c][n][i][j] = sum_p w[c][n][i][p] G^(p)[(j - shift_i)
//      mod n_theta] / mean(G): an HBM-write-bound pass, coalesced along theta.
#include "ffa_internal.cuh"

namespace {

constexpr int MG_TB = 256;

__global__ void flutter_kernel(const ffa_mapgen_desc d)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.n_theta) return;
    const int P = d.n_deriv;
    const double x = d.theta[j];
    double acc[FFA_MAPGEN_MAX_DERIV];
    for (int p = 0; p < P; ++p) acc[p] = 0.0;
    for (int sgi = 0; sgi < d.n_seg; ++sgi) {
        const double k = d.seg_k[sgi], yc = d.seg_y[sgi];
        // sigmoid(x, x0, k) = 1 / (1 + exp(-k (x - x0))); the exit edge uses -k
        const double s1 = 1.0 / (1.0 + exp(-k * (x - d.seg_x0[sgi])));
        const double s2 = 1.0 / (1.0 + exp(-(-k) * (x - d.seg_x1[sgi])));
        double d1[FFA_MAPGEN_MAX_DERIV], d2[FFA_MAPGEN_MAX_DERIV];
        const double *pp = d.sig_poly + (int64_t)sgi * 2 * P * (P + 1);
        for (int i = 0; i < P; ++i) {
            // Horner without contraction, in the reference's order (polyval_manual)
            const double *c1 = pp + (int64_t)i * (P + 1);
            const double *c2 = pp + (int64_t)(P + i) * (P + 1);
            double v1 = 0.0, v2 = 0.0;
            for (int a = 0; a < i + 2; ++a) {
                v1 = __dadd_rn(__dmul_rn(v1, s1), c1[a]);
                v2 = __dadd_rn(__dmul_rn(v2, s2), c2[a]);
            }
            d1[i] = v1;
            d2[i] = v2;
        }
        // order 0: the shape itself; order p: Leibniz sum over the two edges
        acc[0] = __dadd_rn(acc[0], __dmul_rn(__dmul_rn(yc, s1), s2));
        for (int p = 1; p < P; ++p) {
            double res = 0.0, bin = 1.0;
            for (int i = 0; i <= p; ++i) {
                res = __dadd_rn(res, __dmul_rn(__dmul_rn(bin, d1[i]), d2[p - i]));
                bin = bin * (double)(p - i) / (double)(i + 1);
            }
            acc[p] = __dadd_rn(acc[p], __dmul_rn(yc, res));
        }
    }
    for (int p = 0; p < P; ++p) d.gder[(int64_t)p * d.n_theta + j] = acc[p];
}

// Sector mean of G^(0): one block, fixed-order tree (deterministic).
__global__ void mean_kernel(const ffa_mapgen_desc d)
{
    __shared__ double part[MG_TB];
    double s = 0.0;
    for (int64_t j = threadIdx.x; j < d.n_theta; j += blockDim.x) s += d.gder[j];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = MG_TB / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) d.gmean[0] = part[0] / (double)d.n_theta;
}

__global__ void expand_kernel(const ffa_mapgen_desc d)
{
    extern __shared__ double wsh[];        // this row's weights [3][n_orders][n_deriv]
    const int64_t i = blockIdx.y;
    const int P = d.n_deriv, NO = d.n_orders;
    for (int t = threadIdx.x; t < 3 * NO * P; t += blockDim.x) {
        const int c = t / (NO * P), n = (t / P) % NO, p = t % P;
        wsh[t] = d.weights[(((int64_t)c * NO + n) * d.n_r + i) * P + p];
    }
    __syncthreads();
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.n_theta) return;
    int64_t src = (j - (int64_t)d.shift[i]) % d.n_theta;
    if (src < 0) src += d.n_theta;
    double g[FFA_MAPGEN_MAX_DERIV];
    for (int p = 0; p < P; ++p) g[p] = __ldg(d.gder + (int64_t)p * d.n_theta + src);
    const double inv_mean = 1.0 / d.gmean[0];
    double *out[3] = {d.bz, d.br, d.bfi};
    for (int c = 0; c < 3; ++c) {
        for (int n = 0; n < NO; ++n) {
            const double *w = wsh + (c * NO + n) * P;
            double v = 0.0;
            for (int p = 0; p < P; ++p) v += w[p] * g[p];
            out[c][((int64_t)n * d.n_r + i) * d.n_theta + j] = v * inv_mean;
        }
    }
}

}  // namespace

extern "C" int ffa_mapgen(const ffa_mapgen_desc *d, void *stream)
{
    if (!d) return FFA_ERR_INVALID;
    if (d->n_seg < 0 || d->n_seg > FFA_MAX_SEG || d->n_deriv < 1 || d->n_deriv > FFA_MAPGEN_MAX_DERIV ||
        d->n_orders < 1 || d->n_r < 1 || d->n_r > 65535 || d->n_theta < 2)
        return FFA_ERR_INVALID;
    if (!d->sig_poly || !d->theta || !d->weights || !d->shift || !d->gder || !d->gmean || !d->bz || !d->br ||
        !d->bfi)
        return FFA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned gx = (unsigned)((d->n_theta + MG_TB - 1) / MG_TB);
    flutter_kernel<<<gx, MG_TB, 0, s>>>(*d);
    FFA_CHECK_CUDA(cudaGetLastError());
    mean_kernel<<<1, MG_TB, 0, s>>>(*d);
    FFA_CHECK_CUDA(cudaGetLastError());
    const size_t smem = sizeof(double) * 3 * d->n_orders * d->n_deriv;
    if (smem > 48 * 1024) return FFA_ERR_UNSUPPORTED;
    expand_kernel<<<dim3(gx, (unsigned)d->n_r), MG_TB, smem, s>>>(*d);
    FFA_CHECK_CUDA(cudaGetLastError());
    return FFA_OK;
}
