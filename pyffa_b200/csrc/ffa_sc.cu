// ffa_sc.cu -- 2.5D slice-by-slice space charge on the GPU.
//
// One update (FFAG_Bunch.Build_2_5D_SliceGrid_sbs, src/FFAG_Bunch.py:1157-1352)
// runs as a chain of stream-ordered kernels with every intermediate scalar
// kept on the device, so the host never waits inside an update:
//   pass1   per particle: gamma, fi mod 2pi, closed-orbit lookup r0 / pr0,
//           x = r - r0; per-block partial count, sum(gamma) and the extreme
//           azimuths under 4 trial shifts   (GetLocalCoordinates_2p5,
//           src/FFAG_SC_new.py:74-147; divide_arc2 :534-567; lookup
//           src/FFAG_Bunch.py:1227-1244)
//   reduce1 one block: arc [fi_s, fi_e], slice width, mean gamma
//           (merge_multiple_arcs :577-606 for one rank)
//   pass2   slice index and the moment sums   (ComputeSliceBoundsAndCoordsSBS_merged
//           :449-531)
//   reduce2 one block: box mean +- sigma_ratio * sigma, bunch length, cell
//           charge   (src/FFAG_Bunch.py:1265-1294)
//   deposit CIC weights accumulated as 2^-40 fixed-point integers with 64-bit
//           atomics: the sum is exact, so the charge cube is identical for any
//           particle order and launch (DistributeChargeSBS_Njit :244-312
//           accumulates float32 in particle order)
//   solve   per slice: 2D FFT, multiply by the periodic 1/(eps0 k^2) kernel
//           (make_fft_kernel_open_numba :731-760) or by the FFT of the
//           open-boundary Green's function on the doubled grid (Hockney),
//           inverse FFT.  The FFTs are batched radix-2 transforms of whole
//           lines held in shared memory, one kernel per axis, with the cube
//           resident in L2 between passes.
//   field   central differences of the potential / gamma^2
//           (compute_field_from_potential_numba_SBS :672-728)
//   gather  bilinear field at each particle, projected on the orbit
//           direction (interpolate_fields_to_particles_SBS_numba :870-972)
//   roll    the two extrapolation endpoints (src/FFAG_track.py:341-400)
// Block partial sums use a fixed grid and fixed reduction order, so every
// update is bit-for-bit reproducible run to run.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ffa_internal.cuh"

namespace {

using ffa::PI;

constexpr int SC_TB = 256;
constexpr int SC_BLOCKS = 592;             // 4 per SM on 148 SMs; fixed for determinism
constexpr double FIX_SCALE = 1099511627776.0;  // 2^40
constexpr double EPS0 = 8.854187817e-12;

struct SCState {
    ffa_sc_diag diag;
    double amin[4], amax[4];
    double sum_gamma;
    double inv_dx, inv_dz;
    int32_t degenerate;   // dx <= 0 or dz <= 0: fields are not updated
    int32_t bad;          // degenerate or bunch length <= 0: gathered field = 0
};

struct Partial1 {
    double sum_gamma;
    double amin[4], amax[4];
    long long count;
};

struct Partial2 {
    double sx, sz, sx2, sz2;
};

__device__ __forceinline__ double fast_mod(double a, double b) { return a - b * floor(a / b); }

__device__ __forceinline__ double py_mod(double a, double b)
{
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}

__device__ __forceinline__ double gamma_of(const ffa_state_soa &S, int64_t i, int boris, double c, double E0_J)
{
    if (boris) {
        const double rd = S.r[i] * S.f5[i];
        const double v2 = S.vr[i] * S.vr[i] + S.vz[i] * S.vz[i] + rd * rd;
        return 1.0 / sqrt(1.0 - v2 / (c * c));
    }
    return S.f5[i] / E0_J;
}

// Bilinear_interp_2D_vect_uniform (src/FFAG_MathTools.py:828-936) for one point
__device__ __forceinline__ double seo_lookup(const double *Z, double X0, double dX, int64_t NX, double Y0,
                                             double dY, int64_t NY, double x, double y)
{
    int64_t i = (int64_t)floor((x - X0) / dX);
    int64_t j = (int64_t)floor((y - Y0) / dY);
    if (i < 0) i = 0; else if (i >= NX - 1) i = NX - 2;
    if (j < 0) j = 0; else if (j >= NY - 1) j = NY - 2;
    const double tx = (x - (X0 + (double)i * dX)) / dX, ty = (y - (Y0 + (double)j * dY)) / dY;
    const double z00 = Z[i * NY + j], z01 = Z[i * NY + j + 1], z10 = Z[(i + 1) * NY + j], z11 = Z[(i + 1) * NY + j + 1];
    return (1 - tx) * (1 - ty) * z00 + (1 - tx) * ty * z01 + tx * (1 - ty) * z10 + tx * ty * z11;
}

template <typename T>
__device__ T block_sum(T v, T *sh)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
    return r;  // valid in thread 0
}

__device__ double block_min(double v, double *sh)
{
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 1e300;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fmin(r, sh[k]);
    return r;
}

__device__ double block_max(double v, double *sh)
{
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = -1e300;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fmax(r, sh[k]);
    return r;
}

// ----------------------------------------------------------------- passes

__global__ void __launch_bounds__(SC_TB) sc_pass1(ffa_state_soa S, int64_t n, ffa_sc_desc d, double *x_out,
                                                  double *pr0_out, int32_t *slice, int64_t *cell, Partial1 *part)
{
    __shared__ double shd[32];
    __shared__ long long shl[32];
    const double shifts[4] = {0.0, PI, PI * 0.5, PI * 1.5};
    double sg = 0.0;
    long long cnt = 0;
    double mn[4] = {1e30, 1e30, 1e30, 1e30}, mx[4] = {-1e30, -1e30, -1e30, -1e30};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        slice[i] = -1;
        cell[i] = -1;
        if (S.surv[i] == 0) continue;
        const double g = gamma_of(S, i, d.boris, d.speed_c, d.E0_J);
        const double fi = S.fi[i];
        const double fm = fi - 2 * PI * floor(fi / (2 * PI));
        const double Ek = (g - 1) * d.E0_rest_MeV;
        const double r0 = seo_lookup(d.seo_r, d.Ek0, d.dEk, d.nE, d.fi0, d.dfi, d.nfi, Ek, fm);
        pr0_out[i] = seo_lookup(d.seo_pr, d.Ek0, d.dEk, d.nE, d.fi0, d.dfi, d.nfi, Ek, fm);
        x_out[i] = S.r[i] - r0;
        sg += g;
        ++cnt;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double v = fast_mod(fm + shifts[k], 2 * PI);
            mn[k] = fmin(mn[k], v);
            mx[k] = fmax(mx[k], v);
        }
    }
    const double bsg = block_sum(sg, shd);
    const long long bcnt = block_sum(cnt, shl);
    double bmn[4], bmx[4];
    for (int k = 0; k < 4; ++k) {
        bmn[k] = block_min(mn[k], shd);
        bmx[k] = block_max(mx[k], shd);
    }
    if (threadIdx.x == 0) {
        Partial1 &P = part[blockIdx.x];
        P.sum_gamma = bsg;
        P.count = bcnt;
        for (int k = 0; k < 4; ++k) { P.amin[k] = bmn[k]; P.amax[k] = bmx[k]; }
    }
}

// One block of SC_TB threads: each thread folds a fixed strided subset of the
// block partials, then a fixed-shape tree -- the same order on every run.
__global__ void __launch_bounds__(SC_TB) sc_reduce1(const Partial1 *part, int nblk, ffa_sc_desc d, SCState *st)
{
    __shared__ double shd[32];
    __shared__ long long shl[32];
    double sg = 0.0;
    long long cnt = 0;
    double mn[4] = {1e30, 1e30, 1e30, 1e30}, mx[4] = {-1e30, -1e30, -1e30, -1e30};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        sg += part[b].sum_gamma;
        cnt += part[b].count;
        for (int k = 0; k < 4; ++k) {
            mn[k] = fmin(mn[k], part[b].amin[k]);
            mx[k] = fmax(mx[k], part[b].amax[k]);
        }
    }
    sg = block_sum(sg, shd);
    cnt = block_sum(cnt, shl);
    for (int k = 0; k < 4; ++k) {
        mn[k] = block_min(mn[k], shd);
        mx[k] = block_max(mx[k], shd);
    }
    if (threadIdx.x != 0) return;
    const double shifts[4] = {0.0, PI, PI * 0.5, PI * 1.5};
    int best = 0;
    double best_span = mx[0] - mn[0];
    for (int k = 1; k < 4; ++k)
        if (mx[k] - mn[k] < best_span) { best_span = mx[k] - mn[k]; best = k; }
    double arc_s = mn[best] - shifts[best], arc_e = mx[best] - shifts[best];
    if (arc_e < arc_s) arc_e += 2 * PI;
    double fi_s = py_mod(arc_s, 2 * PI), fi_e = py_mod(arc_e, 2 * PI);
    if (fi_e <= fi_s) fi_e += 2 * PI;
    ffa_sc_diag &D = st->diag;
    D.fi_s = fi_s;
    D.fi_e = fi_e;
    D.slice_step = (fi_e - fi_s) / (d.ns - 1);
    D.count = cnt;
    D.mean_gamma_m1 = cnt > 0 ? sg / (double)cnt - 1.0 : 0.0;
    st->sum_gamma = sg;
}

__global__ void __launch_bounds__(SC_TB) sc_pass2(ffa_state_soa S, int64_t n, ffa_sc_desc d, const double *x,
                                                  int32_t *slice, const SCState *st, Partial2 *part)
{
    __shared__ double shd[32];
    const double fi_s = st->diag.fi_s, step = st->diag.slice_step;
    double sx = 0, sz = 0, sx2 = 0, sz2 = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (S.surv[i] == 0) continue;
        const double xi = x[i], zi = S.z[i];
        sx += xi;
        sz += zi;
        sx2 += xi * xi;
        sz2 += zi * zi;
        double fi = S.fi[i];
        fi = fi - 2 * PI * floor(fi / (2 * PI));
        if (fi < fi_s) fi += 2 * PI;
        int64_t s = (int64_t)((fi - fi_s) / step);
        if (s < 0) s = 0; else if (s >= d.ns) s = d.ns - 1;
        slice[i] = (int32_t)s;
    }
    const double a = block_sum(sx, shd), b = block_sum(sz, shd), c = block_sum(sx2, shd), e = block_sum(sz2, shd);
    if (threadIdx.x == 0) part[blockIdx.x] = Partial2{a, b, c, e};
}

__global__ void __launch_bounds__(SC_TB) sc_reduce2(const Partial2 *part, int nblk, ffa_sc_desc d, SCState *st,
                                                    int64_t *status)
{
    __shared__ double shd[32];
    double sx = 0, sz = 0, sx2 = 0, sz2 = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        sx += part[b].sx; sz += part[b].sz; sx2 += part[b].sx2; sz2 += part[b].sz2;
    }
    sx = block_sum(sx, shd);
    sz = block_sum(sz, shd);
    sx2 = block_sum(sx2, shd);
    sz2 = block_sum(sz2, shd);
    if (threadIdx.x != 0) return;
    ffa_sc_diag &D = st->diag;
    const long long cnt = D.count;
    double mx = 0, mz = 0, sgx = 0, sgz = 0;
    if (cnt > 1) {
        mx = sx / (double)cnt;
        mz = sz / (double)cnt;
        const double vx = sx2 / (double)cnt - mx * mx, vz = sz2 / (double)cnt - mz * mz;
        sgx = sqrt(vx > 0.0 ? vx : 0.0);
        sgz = sqrt(vz > 0.0 ? vz : 0.0);
    }
    // np.interp(mean Ek, Ek axis, perimeter)
    const double xe = D.mean_gamma_m1 * d.E0_rest_MeV;
    const double *xp = d.seo_Ek, *fp = d.seo_perimeter;
    double perim;
    if (xe <= xp[0]) perim = fp[0];
    else if (xe >= xp[d.nE - 1]) perim = fp[d.nE - 1];
    else {
        int64_t lo = 0, hi = d.nE - 1;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) / 2;
            if (xp[mid] <= xe) lo = mid; else hi = mid;
        }
        perim = (fp[hi] - fp[lo]) / (xp[hi] - xp[lo]) * (xe - xp[lo]) + fp[lo];
    }
    const double BL = perim * (D.fi_e - D.fi_s) / PI / 2.0;
    const double scale = d.sigma_ratio;
    D.mean_x = mx; D.mean_z = mz; D.sigma_x = sgx; D.sigma_z = sgz;
    D.xmin = mx - scale * sgx; D.xmax = mx + scale * sgx;
    D.zmin = mz - scale * sgz; D.zmax = mz + scale * sgz;
    D.dx = (D.xmax - D.xmin) / d.nx;
    D.dz = (D.zmax - D.zmin) / d.nz;
    D.bunch_length = BL;
    st->degenerate = (D.dx <= 0.0 || D.dz <= 0.0) ? 1 : 0;
    st->bad = (st->degenerate || BL <= 0.0) ? 1 : 0;
    st->inv_dx = 1.0 / D.dx;
    st->inv_dz = 1.0 / D.dz;
    D.q_density = st->bad ? 0.0 : (d.q_macro / BL * d.ns) * (1.0 / (D.dx * D.dz));
    D.degenerate = st->degenerate;
    if (st->degenerate && status) atomicAdd((unsigned long long *)&status[FFA_STATUS_SC_DEGENERATE], 1ull);
}

__global__ void __launch_bounds__(SC_TB) sc_deposit(ffa_state_soa S, int64_t n, ffa_sc_desc d, const double *x,
                                                    const int32_t *slice, int64_t *cell, const SCState *st,
                                                    unsigned long long *acc)
{
    if (st->bad) return;
    const double xmin = st->diag.xmin, zmin = st->diag.zmin, inv_dx = st->inv_dx, inv_dz = st->inv_dz;
    const int nx = d.nx, nz = d.nz;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = slice[i];
        if (s < 0) continue;
        const double rx = (x[i] - xmin) * inv_dx, rz = (S.z[i] - zmin) * inv_dz;
        int64_t ix = (int64_t)floor(rx), iz = (int64_t)floor(rz);
        double fx = rx - (double)ix, fz = rz - (double)iz;
        if (ix < 0) { ix = 0; fx = 0.0; } else if (ix >= nx - 1) { ix = nx - 2; fx = 1.0; }
        if (iz < 0) { iz = 0; fz = 0.0; } else if (iz >= nz - 1) { iz = nz - 2; fz = 1.0; }
        const int64_t c0 = ((int64_t)s * nz + iz) * nx + ix;
        cell[i] = c0;
        atomicAdd(acc + c0, (unsigned long long)llrint((1.0 - fx) * (1.0 - fz) * FIX_SCALE));
        atomicAdd(acc + c0 + 1, (unsigned long long)llrint(fx * (1.0 - fz) * FIX_SCALE));
        atomicAdd(acc + c0 + nx, (unsigned long long)llrint((1.0 - fx) * fz * FIX_SCALE));
        atomicAdd(acc + c0 + nx + 1, (unsigned long long)llrint(fx * fz * FIX_SCALE));
    }
}

// fixed point -> float32 charge cube, and the complex work buffer of the
// solver (the reference copies rho into a complex64 array, imaginary 0)
__global__ void sc_convert(const unsigned long long *acc, ffa_sc_desc d, const SCState *st, float *rho,
                           float2 *work, int NZ, int NX)
{
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    const int64_t wsz = (int64_t)d.ns * NZ * NX;
    const double q = st->diag.q_density / FIX_SCALE;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < wsz; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e / ((int64_t)NZ * NX);
        const int64_t rem = e - s * NZ * NX;
        const int j = (int)(rem / NX), i = (int)(rem - (int64_t)j * NX);
        float v = 0.0f;
        if (j < d.nz && i < d.nx) {
            const int64_t c = (s * d.nz + j) * d.nx + i;
            v = st->bad ? 0.0f : (float)((double)acc[c] * q);
            rho[c] = v;
        }
        work[e] = make_float2(v, 0.0f);
    }
    (void)cube;
}

// ---------------------------------------------------------------- FFTs

template <typename T> struct C2;
template <> struct C2<float> { using t = float2; };
template <> struct C2<double> { using t = double2; };

// Batched radix-2 transforms of complete lines in shared memory.
// Lines run along x (axis 1, contiguous) or z (axis 0, stride NX); a CTA
// holds LINES lines of length n (bit-reversed on load, in-place butterflies,
// one barrier per stage).  Loads and stores are coalesced for both axes:
// along x consecutive threads read consecutive elements of a line, along z
// consecutive threads read the same element of consecutive lines.
// Forward: exp(-2 pi i jk/n); inverse: exp(+2 pi i jk/n), unnormalised.
template <typename T, int LINES>
__global__ void __launch_bounds__(256) fft_axis(typename C2<T>::t *data, int nslices, int NZ, int NX, int axis,
                                                int logn, const typename C2<T>::t *tw, int inverse)
{
    using V = typename C2<T>::t;
    extern __shared__ unsigned char smraw[];
    V *sm = reinterpret_cast<V *>(smraw);
    const int n = 1 << logn;
    const int ld = n + 1;  // padded line pitch
    V *base;
    int64_t lstride, estride;
    if (axis == 1) {
        const int64_t line0 = (int64_t)blockIdx.x * LINES;  // over nslices * NZ rows
        base = data + line0 * NX;
        lstride = NX;
        estride = 1;
    } else {
        const int tiles = NX / LINES;
        const int64_t s = blockIdx.x / tiles;
        const int t = blockIdx.x - (int)(s * tiles);
        base = data + s * (int64_t)NZ * NX + (int64_t)t * LINES;
        lstride = 1;
        estride = NX;
    }
    const int total = LINES * n;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int l, k;
        if (axis == 1) { l = e >> logn; k = e & (n - 1); }
        else { k = e / LINES; l = e - k * LINES; }
        const unsigned rk = __brev((unsigned)k) >> (32 - logn);
        sm[l * ld + rk] = base[l * lstride + (int64_t)k * estride];
    }
    // twiddles exp(-2 pi i k / n), k < n / 2, staged once per block
    V *tws = sm + LINES * ld;
    for (int k = threadIdx.x; k < (n >> 1); k += blockDim.x) tws[k] = tw[k];
    __syncthreads();
    const T sgn = inverse ? (T)1 : (T)-1;
    const int hb = logn - 1;                  // log2(n / 2)
    for (int s = 1; s <= logn; ++s) {
        const int half = 1 << (s - 1);
        const int twshift = logn - s;         // twiddle index j * (n >> s)
        for (int b = threadIdx.x; b < LINES * (n >> 1); b += blockDim.x) {
            const int l = b >> hb;
            const int bb = b & ((n >> 1) - 1);
            const int grp = bb >> (s - 1);
            const int j = bb & (half - 1);
            const int i0 = grp * (half << 1) + j, i1 = i0 + half;
            const V w = tws[j << twshift];
            const T wr = w.x, wi = sgn * (-w.y);  // table holds exp(-2 pi i k/n)
            V *p = sm + l * ld;
            const V a = p[i0], c = p[i1];
            const T xr = c.x * wr - c.y * wi, xi = c.x * wi + c.y * wr;
            p[i1].x = a.x - xr;
            p[i1].y = a.y - xi;
            p[i0].x = a.x + xr;
            p[i0].y = a.y + xi;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int l, k;
        if (axis == 1) { l = e >> logn; k = e & (n - 1); }
        else { k = e / LINES; l = e - k * LINES; }
        base[l * lstride + (int64_t)k * estride] = sm[l * ld + k];
    }
}

// multiply by the periodic kernel 1/(eps0 k^2), built in float32 exactly as
// make_fft_kernel_open_numba (k = 0 term zero; bin n/2 counts as +n/2)
__global__ void sc_mul_periodic(float2 *work, ffa_sc_desc d, const SCState *st)
{
    if (st->bad) return;
    const int nx = d.nx, nz = d.nz;
    const float dkx = (float)(2.0 * PI / (nx * st->diag.dx));
    const float dkz = (float)(2.0 * PI / (nz * st->diag.dz));
    const int64_t tot = (int64_t)d.ns * nz * nx;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t rem = e % ((int64_t)nz * nx);
        const int j = (int)(rem / nx), i = (int)(rem - (int64_t)j * nx);
        const float kx = (float)((double)dkx * (double)(i <= nx / 2 ? i : i - nx));
        const float kz = (float)((double)dkz * (double)(j <= nz / 2 ? j : j - nz));
        const float kz2 = __fmul_rn(kz, kz);
        const float k2 = __fadd_rn(__fmul_rn(kx, kx), kz2);
        const float kern = (k2 == 0.0f) ? 0.0f : (float)(1.0 / (EPS0 * (double)k2));
        float2 v = work[e];
        v.x = __fmul_rn(v.x, kern);
        v.y = __fmul_rn(v.y, kern);
        work[e] = v;
    }
}

// Open-boundary Green's function on the doubled (NZ, NX) grid, float64:
// G = -ln(x^2 + z^2) / (4 pi eps0), the cell average at the origin.
__global__ void sc_green_fill(double2 *g, int NZ, int NX, const SCState *st)
{
    if (st->bad) return;
    const double dx = st->diag.dx, dz = st->diag.dz;
    const double K = -1.0 / (4.0 * PI * EPS0);
    const int nx = NX / 2, nz = NZ / 2;
    const int64_t tot = (int64_t)NZ * NX;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / NX), i = (int)(e - (int64_t)j * NX);
        const double z = dz * (double)(j <= nz ? j : NZ - j);
        const double x = dx * (double)(i <= nx ? i : NX - i);
        double v;
        if (i == 0 && j == 0) {
            const double a = 0.5 * dx, b = 0.5 * dz;
            const double F = a * b * (log(a * a + b * b) - 3.0) + a * a * atan(b / a) + b * b * atan(a / b);
            v = K * (F / (a * b));
        } else {
            v = K * log(x * x + z * z);
        }
        g[e] = make_double2(v * dx * dz, 0.0);
    }
}

__global__ void sc_green_finish(const double2 *g, float *gk, int64_t tot, const SCState *st)
{
    if (st->bad) return;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        gk[e] = (float)g[e].x;  // real and even: the transform is real
}

__global__ void sc_mul_green(float2 *work, int ns, int64_t plane, const float *gk, const SCState *st)
{
    if (st->bad) return;
    const int64_t tot = (int64_t)ns * plane;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const float k = gk[e % plane];
        float2 v = work[e];
        v.x *= k;
        v.y *= k;
        work[e] = v;
    }
}

// potential = real part / (NX NZ), corner (nz, nx) of the work grid
__global__ void sc_potential(const float2 *work, ffa_sc_desc d, int NZ, int NX, const SCState *st, float *phi)
{
    const int64_t tot = (int64_t)d.ns * d.nz * d.nx;
    const float scale = (float)(1.0 / ((double)NX * (double)NZ));
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e / ((int64_t)d.nz * d.nx);
        const int64_t rem = e - s * d.nz * d.nx;
        const int j = (int)(rem / d.nx), i = (int)(rem - (int64_t)j * d.nx);
        phi[e] = st->bad ? 0.0f : __fmul_rn(work[(s * NZ + j) * NX + i].x, scale);
    }
}

// compute_field_from_potential_numba_SBS for every cell (each cell takes the
// value of the last loop of the reference that writes it)
__global__ void sc_field(const float *phi, ffa_sc_desc d, const SCState *st, float *Ex, float *Ez)
{
    if (st->degenerate) return;
    const int nx = d.nx, nz = d.nz;
    const double dr = st->diag.dx, dz = st->diag.dz, BL = st->diag.bunch_length;
    const double g = st->diag.mean_gamma_m1 + 1.0;
    const double ig2 = 1.0 / (g * g);
    const double inv2dr = 0.5 / dr, inv2dz = 0.5 / dz;
    const int64_t tot = (int64_t)d.ns * nz * nx;
    const bool zero = (dr == 0.0 || dz == 0.0 || BL == 0);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        if (zero) { Ex[e] = 0.0f; Ez[e] = 0.0f; continue; }
        const int64_t s = e / ((int64_t)nz * nx);
        const int64_t rem = e - s * nz * nx;
        const int j = (int)(rem / nx), i = (int)(rem - (int64_t)j * nx);
        const float *P = phi + s * nz * nx;
#define PH(jj, ii) P[(int64_t)(jj) * nx + (ii)]
        double ex, ez;
        if (i == 0 || i == nx - 1) {
            const int jp = j + 1 < nz - 1 ? j + 1 : nz - 1, jm = j - 1 > 0 ? j - 1 : 0;
            ex = (i == 0) ? -(double)__fsub_rn(PH(j, 1), PH(j, 0)) / dr * ig2
                          : -(double)__fsub_rn(PH(j, nx - 1), PH(j, nx - 2)) / dr * ig2;
            ez = -(double)__fsub_rn(PH(jp, i), PH(jm, i)) / dz * ig2;
        } else if (j == 0) {
            ex = -(double)__fsub_rn(PH(0, i + 1), PH(0, i - 1)) * inv2dr * ig2;
            ez = -(double)__fsub_rn(PH(1, i), PH(0, i)) / dz * ig2;
        } else if (j == nz - 1) {
            ex = -(double)__fsub_rn(PH(nz - 1, i + 1), PH(nz - 1, i - 1)) * inv2dr * ig2;
            ez = -(double)__fsub_rn(PH(nz - 1, i), PH(nz - 2, i)) / dz * ig2;
        } else {
            ex = -(double)__fsub_rn(PH(j, i + 1), PH(j, i - 1)) * inv2dr * ig2;
            ez = -(double)__fsub_rn(PH(j + 1, i), PH(j - 1, i)) * inv2dz * ig2;
        }
#undef PH
        Ex[e] = (float)ex;
        Ez[e] = (float)ez;
    }
}

__global__ void __launch_bounds__(SC_TB) sc_gather(ffa_state_soa S, int64_t n, ffa_sc_desc d, const double *x,
                                                   const double *pr0, const int32_t *slice, const SCState *st,
                                                   const float *Ex, const float *Ez)
{
    if (st->degenerate) return;
    const int nx = d.nx, nz = d.nz;
    const double x0 = st->diag.xmin, z0 = st->diag.zmin, dx = st->diag.dx, dz = st->diag.dz;
    const bool bad = st->bad != 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int s = slice[i];
        if (s < 0) continue;
        if (bad) { S.esc_r[i] = 0.0; S.esc_z[i] = 0.0; S.esc_fi[i] = 0.0; continue; }
        const float *EX = Ex + (int64_t)s * nz * nx, *EZ = Ez + (int64_t)s * nz * nx;
        const double t = (x[i] - x0) / dx, u = (S.z[i] - z0) / dz;
        int64_t i0 = (int64_t)floor(t), j0 = (int64_t)floor(u);
        if (i0 < 0) i0 = 0; else if (i0 > nx - 2) i0 = nx - 2;
        if (j0 < 0) j0 = 0; else if (j0 > nz - 2) j0 = nz - 2;
        const double al = t - (double)i0, be = u - (double)j0;
        const double w00 = (1.0 - al) * (1.0 - be), w10 = al * (1.0 - be), w01 = (1.0 - al) * be, w11 = al * be;
        const double er = w00 * EX[j0 * nx + i0] + w10 * EX[j0 * nx + i0 + 1] + w01 * EX[(j0 + 1) * nx + i0] +
                          w11 * EX[(j0 + 1) * nx + i0 + 1];
        const double ez = w00 * EZ[j0 * nx + i0] + w10 * EZ[j0 * nx + i0 + 1] + w01 * EZ[(j0 + 1) * nx + i0] +
                          w11 * EZ[(j0 + 1) * nx + i0 + 1];
        const double p = pr0[i];
        const double rt = sqrt(1 + p * p);
        S.esc_r[i] = er * (1 / rt);
        S.esc_z[i] = ez;
        S.esc_fi[i] = er * (-p / rt);
    }
}

// extrapolation endpoints after an update (src/FFAG_track.py:341-400)
__global__ void sc_roll(ffa_state_soa S, int64_t n, int first)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t alive = S.surv[i] != 0;
        if (first) {
            S.sc_pre[i] = alive;
            S.sc_pp[i] = 0;
            if (alive) { S.e_pre_r[i] = S.esc_r[i]; S.e_pre_z[i] = S.esc_z[i]; S.e_pre_fi[i] = S.esc_fi[i]; }
            S.e_pp_r[i] = S.e_pre_r[i]; S.e_pp_z[i] = S.e_pre_z[i]; S.e_pp_fi[i] = S.e_pre_fi[i];
        } else {
            S.sc_pp[i] = S.sc_pre[i];
            S.sc_pre[i] = alive;
            S.e_pp_r[i] = S.e_pre_r[i]; S.e_pp_z[i] = S.e_pre_z[i]; S.e_pp_fi[i] = S.e_pre_fi[i];
            if (alive) { S.e_pre_r[i] = S.esc_r[i]; S.e_pre_z[i] = S.esc_z[i]; S.e_pre_fi[i] = S.esc_fi[i]; }
        }
    }
}

int ilog2(int v)
{
    int l = 0;
    while ((1 << l) < v) ++l;
    return (1 << l) == v ? l : -1;
}

}  // namespace

struct ffa_sc_plan {
    ffa_sc_desc d;
    int NZ, NX;           // solver grid (doubled for Hockney)
    int lognz, lognx;
    double *x, *pr0;
    int32_t *slice;
    int64_t *cell;
    Partial1 *p1;
    Partial2 *p2;
    SCState *st;
    unsigned long long *acc;
    float *rho, *phi, *ex, *ez;
    float2 *work;
    float2 *twx32, *twz32;
    double2 *gwork, *twx64, *twz64;
    float *gk;
};

namespace {

void free_plan(ffa_sc_plan *p)
{
    if (!p) return;
    void *ptrs[] = {p->x, p->pr0, p->slice, p->cell, p->p1, p->p2, p->st, p->acc, p->rho, p->phi, p->ex, p->ez,
                    p->work, p->twx32, p->twz32, p->gwork, p->twx64, p->twz64, p->gk};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    free(p);
}

template <typename V>
int upload_twiddles(int n, V **out)
{
    V *h = (V *)malloc(sizeof(V) * (n / 2));
    if (!h) return FFA_ERR_NOMEM;
    for (int k = 0; k < n / 2; ++k) {
        const double a = -2.0 * PI * (double)k / (double)n;
        h[k].x = (decltype(h[k].x))cos(a);
        h[k].y = (decltype(h[k].y))sin(a);
    }
    if (cudaMalloc(out, sizeof(V) * (n / 2)) != cudaSuccess) { free(h); return FFA_ERR_NOMEM; }
    const cudaError_t e = cudaMemcpy(*out, h, sizeof(V) * (n / 2), cudaMemcpyHostToDevice);
    free(h);
    return e == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

template <typename T, int LINES>
cudaError_t fft2d(typename C2<T>::t *data, int nslices, int NZ, int NX, int lognz, int lognx,
                  const typename C2<T>::t *twz, const typename C2<T>::t *twx, int inverse, cudaStream_t s)
{
    using V = typename C2<T>::t;
    // lines (padded pitch) + the n / 2 twiddles
    const size_t smx = sizeof(V) * (LINES * (NX + 1) + NX / 2), smz = sizeof(V) * (LINES * (NZ + 1) + NZ / 2);
    cudaFuncSetAttribute(fft_axis<T, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(smx > smz ? smx : smz));
    if (!inverse) {
        fft_axis<T, LINES><<<(unsigned)((int64_t)nslices * NZ / LINES), 256, smx, s>>>(data, nslices, NZ, NX, 1, lognx, twx, 0);
        fft_axis<T, LINES><<<(unsigned)((int64_t)nslices * (NX / LINES)), 256, smz, s>>>(data, nslices, NZ, NX, 0, lognz, twz, 0);
    } else {
        fft_axis<T, LINES><<<(unsigned)((int64_t)nslices * (NX / LINES)), 256, smz, s>>>(data, nslices, NZ, NX, 0, lognz, twz, 1);
        fft_axis<T, LINES><<<(unsigned)((int64_t)nslices * NZ / LINES), 256, smx, s>>>(data, nslices, NZ, NX, 1, lognx, twx, 1);
    }
    return cudaGetLastError();
}

}  // namespace

extern "C" {

int ffa_sc_plan_create(const ffa_sc_desc *desc, void *stream, ffa_sc_plan **out)
{
    (void)stream;
    if (!desc || !out) return FFA_ERR_INVALID;
    *out = nullptr;
    const ffa_sc_desc &d = *desc;
    if (d.ns < 2 || d.nx < 16 || d.nz < 16 || d.n_max < 0 || d.nE < 2 || d.nfi < 2 || !d.seo_Ek || !d.seo_r ||
        !d.seo_pr || !d.seo_perimeter || !(d.dEk > 0) || !(d.dfi > 0))
        return FFA_ERR_INVALID;
    const int lx = ilog2(d.nx), lz = ilog2(d.nz);
    if (lx < 0 || lz < 0 || d.nx > 512 || d.nz > 512) return FFA_ERR_UNSUPPORTED;  // powers of two, <= 512
    ffa_sc_plan *p = (ffa_sc_plan *)calloc(1, sizeof(ffa_sc_plan));
    if (!p) return FFA_ERR_NOMEM;
    p->d = d;
    p->NX = d.hockney ? 2 * d.nx : d.nx;
    p->NZ = d.hockney ? 2 * d.nz : d.nz;
    p->lognx = ilog2(p->NX);
    p->lognz = ilog2(p->NZ);
    const int64_t n = d.n_max > 0 ? d.n_max : 1;
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    const int64_t wsz = (int64_t)d.ns * p->NZ * p->NX;
    bool ok = cudaMalloc(&p->x, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&p->pr0, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&p->slice, sizeof(int32_t) * n) == cudaSuccess &&
              cudaMalloc(&p->cell, sizeof(int64_t) * n) == cudaSuccess &&
              cudaMalloc(&p->p1, sizeof(Partial1) * SC_BLOCKS) == cudaSuccess &&
              cudaMalloc(&p->p2, sizeof(Partial2) * SC_BLOCKS) == cudaSuccess &&
              cudaMalloc(&p->st, sizeof(SCState)) == cudaSuccess &&
              cudaMalloc(&p->acc, sizeof(unsigned long long) * cube) == cudaSuccess &&
              cudaMalloc(&p->rho, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&p->phi, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&p->ex, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&p->ez, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&p->work, sizeof(float2) * wsz) == cudaSuccess;
    if (ok && d.hockney)
        ok = cudaMalloc(&p->gwork, sizeof(double2) * (int64_t)p->NZ * p->NX) == cudaSuccess &&
             cudaMalloc(&p->gk, sizeof(float) * (int64_t)p->NZ * p->NX) == cudaSuccess;
    if (!ok) { free_plan(p); return FFA_ERR_NOMEM; }
    int rc = upload_twiddles(p->NX, &p->twx32);
    if (rc == FFA_OK) rc = upload_twiddles(p->NZ, &p->twz32);
    if (rc == FFA_OK && d.hockney) rc = upload_twiddles(p->NX, &p->twx64);
    if (rc == FFA_OK && d.hockney) rc = upload_twiddles(p->NZ, &p->twz64);
    if (rc != FFA_OK) { free_plan(p); return rc; }
    if (cudaMemset(p->st, 0, sizeof(SCState)) != cudaSuccess || cudaMemset(p->slice, 0xff, sizeof(int32_t) * n) != cudaSuccess ||
        cudaMemset(p->cell, 0xff, sizeof(int64_t) * n) != cudaSuccess) {
        free_plan(p);
        return FFA_ERR_CUDA;
    }
    *out = p;
    return FFA_OK;
}

int ffa_sc_plan_destroy(ffa_sc_plan *plan)
{
    free_plan(plan);
    return FFA_OK;
}

int ffa_sc_step(ffa_sc_plan *p, ffa_state_soa *S, int64_t n, int32_t roll, int32_t first, void *stream,
                int64_t *status, ffa_sc_diag *diag)
{
    if (!p || !S || !S->r || !S->vr || !S->z || !S->vz || !S->fi || !S->f5 || !S->surv || !S->esc_r || !S->esc_z ||
        !S->esc_fi || n < 0)
        return FFA_ERR_INVALID;
    if (n > p->d.n_max) return FFA_ERR_INVALID;
    if (roll && (!S->sc_pre || !S->sc_pp || !S->e_pre_r || !S->e_pre_z || !S->e_pre_fi || !S->e_pp_r ||
                 !S->e_pp_z || !S->e_pp_fi))
        return FFA_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const ffa_sc_desc &d = p->d;
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    const int64_t wsz = (int64_t)d.ns * p->NZ * p->NX;
    const unsigned ew = 148 * 8;  // elementwise grids
    FFA_CHECK_CUDA(cudaMemsetAsync(p->acc, 0, sizeof(unsigned long long) * cube, s));
    sc_pass1<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, p->x, p->pr0, p->slice, p->cell, p->p1);
    sc_reduce1<<<1, SC_TB, 0, s>>>(p->p1, SC_BLOCKS, d, p->st);
    sc_pass2<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, p->x, p->slice, p->st, p->p2);
    sc_reduce2<<<1, SC_TB, 0, s>>>(p->p2, SC_BLOCKS, d, p->st, status);
    sc_deposit<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, p->x, p->slice, p->cell, p->st, p->acc);
    sc_convert<<<ew, 256, 0, s>>>(p->acc, d, p->st, p->rho, p->work, p->NZ, p->NX);
    FFA_CHECK_CUDA(cudaGetLastError());
    if (d.hockney) {
        sc_green_fill<<<ew, 256, 0, s>>>(p->gwork, p->NZ, p->NX, p->st);
        FFA_CHECK_CUDA((fft2d<double, 8>(p->gwork, 1, p->NZ, p->NX, p->lognz, p->lognx, p->twz64, p->twx64, 0, s)));
        sc_green_finish<<<ew, 256, 0, s>>>(p->gwork, p->gk, (int64_t)p->NZ * p->NX, p->st);
    }
    FFA_CHECK_CUDA((fft2d<float, 16>(p->work, d.ns, p->NZ, p->NX, p->lognz, p->lognx, p->twz32, p->twx32, 0, s)));
    if (d.hockney) sc_mul_green<<<ew, 256, 0, s>>>(p->work, d.ns, (int64_t)p->NZ * p->NX, p->gk, p->st);
    else sc_mul_periodic<<<ew, 256, 0, s>>>(p->work, d, p->st);
    FFA_CHECK_CUDA((fft2d<float, 16>(p->work, d.ns, p->NZ, p->NX, p->lognz, p->lognx, p->twz32, p->twx32, 1, s)));
    sc_potential<<<ew, 256, 0, s>>>(p->work, d, p->NZ, p->NX, p->st, p->phi);
    sc_field<<<ew, 256, 0, s>>>(p->phi, d, p->st, p->ex, p->ez);
    sc_gather<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, p->x, p->pr0, p->slice, p->st, p->ex, p->ez);
    if (roll) sc_roll<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, first);
    FFA_CHECK_CUDA(cudaGetLastError());
    if (diag) FFA_CHECK_CUDA(cudaMemcpyAsync(diag, &p->st->diag, sizeof(ffa_sc_diag), cudaMemcpyDeviceToDevice, s));
    (void)wsz;
    return FFA_OK;
}

int ffa_sc_buffers(const ffa_sc_plan *p, const float **rho, const float **phi, const float **ex, const float **ez,
                   const int32_t **slice_idx, const int64_t **cell_idx)
{
    if (!p) return FFA_ERR_INVALID;
    if (rho) *rho = p->rho;
    if (phi) *phi = p->phi;
    if (ex) *ex = p->ex;
    if (ez) *ez = p->ez;
    if (slice_idx) *slice_idx = p->slice;
    if (cell_idx) *cell_idx = p->cell;
    return FFA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Space-charge update without any allocation.
//
// Some callers of this library cannot allocate device memory once they are
// running: a host code that reserves its whole device budget at start-up
// and hands it out from its own pool, or a tracking loop embedded in a
// control or online-model system where a cudaMalloc in the middle of a run
// could fail or stall every stream on the device.  ffa_sc_step_static runs
// the same update as ffa_sc_plan_create + ffa_sc_step, but takes its scratch
// from one fixed array compiled into the library, so it calls no cudaMalloc,
// cudaFree or other allocating routine.
//
// Limits (the array holds ~31 MB on every device that loads the library,
// until the process exits): at most FFA_SC_STATIC_MAX_PARTICLES particles,
// ns * nz * nx <= FFA_SC_STATIC_MAX_CELLS, nx and nz <= 128, periodic
// boundary only.  Larger sizes are rejected with FFA_ERR_INVALID (particle
// count) or FFA_ERR_UNSUPPORTED (grid, open boundary) before anything runs.
//
// The array is shared by every call on a device and keeps the previous
// call's contents; the charge accumulator is cleared at the start of each
// call, every other region is fully rewritten before it is read.  Calls
// whose work overlaps on the GPU (different streams, or host threads)
// race on the array and must be serialised by the caller.
// The first call on a device looks up the array's device address (with that
// device current) and fills the FFT twiddle tables; make that first call
// before capturing any stream.
// ------------------------------------------------------------------------
namespace {

constexpr int64_t ST_MAX_N = FFA_SC_STATIC_MAX_PARTICLES;
constexpr int64_t ST_MAX_CELLS = FFA_SC_STATIC_MAX_CELLS;
constexpr int ST_MAX_GRID = 128;

constexpr size_t a256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t ST_OFF_X = 0;
constexpr size_t ST_OFF_PR0 = ST_OFF_X + a256(sizeof(double) * ST_MAX_N);
constexpr size_t ST_OFF_SLICE = ST_OFF_PR0 + a256(sizeof(double) * ST_MAX_N);
constexpr size_t ST_OFF_CELL = ST_OFF_SLICE + a256(sizeof(int32_t) * ST_MAX_N);
constexpr size_t ST_OFF_P1 = ST_OFF_CELL + a256(sizeof(int64_t) * ST_MAX_N);
constexpr size_t ST_OFF_P2 = ST_OFF_P1 + a256(sizeof(Partial1) * SC_BLOCKS);
constexpr size_t ST_OFF_STATE = ST_OFF_P2 + a256(sizeof(Partial2) * SC_BLOCKS);
constexpr size_t ST_OFF_ACC = ST_OFF_STATE + a256(sizeof(SCState));
constexpr size_t ST_OFF_RHO = ST_OFF_ACC + a256(sizeof(unsigned long long) * ST_MAX_CELLS);
constexpr size_t ST_OFF_PHI = ST_OFF_RHO + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_EX = ST_OFF_PHI + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_EZ = ST_OFF_EX + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_WORK = ST_OFF_EZ + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_TWX = ST_OFF_WORK + a256(sizeof(float2) * ST_MAX_CELLS);
constexpr size_t ST_OFF_TWZ = ST_OFF_TWX + a256(sizeof(float2) * ST_MAX_GRID / 2);
constexpr size_t ST_BYTES = ST_OFF_TWZ + a256(sizeof(float2) * ST_MAX_GRID / 2);

// Twiddles exp(-2 pi i k / n) of both axes, one set per device; the table of
// an axis is rebuilt when a call uses a different length.
struct StaticDev {
    unsigned char *base;  // device address of the array (from cudaGetSymbolAddress)
    int twx_n, twz_n;
};

constexpr int ST_MAX_DEVICES = 64;
StaticDev g_static_dev[ST_MAX_DEVICES];

__global__ void st_twiddles(float2 *tw, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n / 2) return;
    const double a = -2.0 * PI * (double)k / (double)n;
    tw[k] = make_float2((float)cos(a), (float)sin(a));
}

}  // namespace

static __device__ __align__(256) unsigned char ffa_sc_static_scratch[ST_BYTES];

extern "C" int ffa_sc_step_static(const ffa_sc_desc *desc, ffa_state_soa *S, int64_t n, int32_t roll,
                                  int32_t first, void *stream, int64_t *status, ffa_sc_diag *diag)
{
    if (!desc || !S || !S->r || !S->vr || !S->z || !S->vz || !S->fi || !S->f5 || !S->surv || !S->esc_r ||
        !S->esc_z || !S->esc_fi || n < 0)
        return FFA_ERR_INVALID;
    const ffa_sc_desc &d = *desc;
    if (d.ns < 2 || d.nx < 16 || d.nz < 16 || d.nE < 2 || d.nfi < 2 || !d.seo_Ek || !d.seo_r || !d.seo_pr ||
        !d.seo_perimeter || !(d.dEk > 0) || !(d.dfi > 0))
        return FFA_ERR_INVALID;
    if (n > ST_MAX_N) return FFA_ERR_INVALID;  // more particles than the static scratch holds
    const int lx = ilog2(d.nx), lz = ilog2(d.nz);
    if (d.hockney || lx < 0 || lz < 0 || d.nx > ST_MAX_GRID || d.nz > ST_MAX_GRID ||
        (int64_t)d.ns * d.nz * d.nx > ST_MAX_CELLS)
        return FFA_ERR_UNSUPPORTED;
    if (roll && (!S->sc_pre || !S->sc_pp || !S->e_pre_r || !S->e_pre_z || !S->e_pre_fi || !S->e_pp_r ||
                 !S->e_pp_z || !S->e_pp_fi))
        return FFA_ERR_INVALID;
    int dev = 0;
    FFA_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= ST_MAX_DEVICES) return FFA_ERR_UNSUPPORTED;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    StaticDev &sd = g_static_dev[dev];
    if (!sd.base) {
        // host code must not use the array's name as a device address: ask
        // the runtime for the address on this (current) device once
        void *ptr = nullptr;
        FFA_CHECK_CUDA(cudaGetSymbolAddress(&ptr, ffa_sc_static_scratch));
        sd.base = static_cast<unsigned char *>(ptr);
        sd.twx_n = sd.twz_n = 0;
    }
    unsigned char *b = sd.base;
    double *x = reinterpret_cast<double *>(b + ST_OFF_X);
    double *pr0 = reinterpret_cast<double *>(b + ST_OFF_PR0);
    int32_t *slice = reinterpret_cast<int32_t *>(b + ST_OFF_SLICE);
    int64_t *cell = reinterpret_cast<int64_t *>(b + ST_OFF_CELL);
    Partial1 *p1 = reinterpret_cast<Partial1 *>(b + ST_OFF_P1);
    Partial2 *p2 = reinterpret_cast<Partial2 *>(b + ST_OFF_P2);
    SCState *st = reinterpret_cast<SCState *>(b + ST_OFF_STATE);
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(b + ST_OFF_ACC);
    float *rho = reinterpret_cast<float *>(b + ST_OFF_RHO);
    float *phi = reinterpret_cast<float *>(b + ST_OFF_PHI);
    float *ex = reinterpret_cast<float *>(b + ST_OFF_EX);
    float *ez = reinterpret_cast<float *>(b + ST_OFF_EZ);
    float2 *work = reinterpret_cast<float2 *>(b + ST_OFF_WORK);
    float2 *twx = reinterpret_cast<float2 *>(b + ST_OFF_TWX);
    float2 *twz = reinterpret_cast<float2 *>(b + ST_OFF_TWZ);
    if (sd.twx_n != d.nx) {
        st_twiddles<<<1, 64, 0, s>>>(twx, d.nx);
        sd.twx_n = d.nx;
    }
    if (sd.twz_n != d.nz) {
        st_twiddles<<<1, 64, 0, s>>>(twz, d.nz);
        sd.twz_n = d.nz;
    }
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    const unsigned ew = 148 * 8;
    FFA_CHECK_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * cube, s));
    sc_pass1<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, x, pr0, slice, cell, p1);
    sc_reduce1<<<1, SC_TB, 0, s>>>(p1, SC_BLOCKS, d, st);
    sc_pass2<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, x, slice, st, p2);
    sc_reduce2<<<1, SC_TB, 0, s>>>(p2, SC_BLOCKS, d, st, status);
    sc_deposit<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, x, slice, cell, st, acc);
    sc_convert<<<ew, 256, 0, s>>>(acc, d, st, rho, work, d.nz, d.nx);
    FFA_CHECK_CUDA(cudaGetLastError());
    FFA_CHECK_CUDA((fft2d<float, 16>(work, d.ns, d.nz, d.nx, lz, lx, twz, twx, 0, s)));
    sc_mul_periodic<<<ew, 256, 0, s>>>(work, d, st);
    FFA_CHECK_CUDA((fft2d<float, 16>(work, d.ns, d.nz, d.nx, lz, lx, twz, twx, 1, s)));
    sc_potential<<<ew, 256, 0, s>>>(work, d, d.nz, d.nx, st, phi);
    sc_field<<<ew, 256, 0, s>>>(phi, d, st, ex, ez);
    sc_gather<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, x, pr0, slice, st, ex, ez);
    if (roll) sc_roll<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, first);
    FFA_CHECK_CUDA(cudaGetLastError());
    if (diag) FFA_CHECK_CUDA(cudaMemcpyAsync(diag, &st->diag, sizeof(ffa_sc_diag), cudaMemcpyDeviceToDevice, s));
    return FFA_OK;
}
