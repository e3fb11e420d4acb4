// ffa_sc.cu -- 2.5D slice-by-slice space charge on the GPU.
//
// One update (FFAG_Bunch.Build_2_5D_SliceGrid_sbs, src/FFAG_Bunch.py:1157-1352)
// runs as a short chain of stream-ordered kernels with every intermediate
// scalar kept on the device, so the host never waits inside an update:
//   pass1   per particle: gamma, fi mod 2pi, closed-orbit lookup r0 / pr0,
//           x = r - r0, the moment sums and the extreme azimuths under 4
//           trial shifts (GetLocalCoordinates_2p5, src/FFAG_SC_new.py:74-147;
//           divide_arc2 :534-567; lookup src/FFAG_Bunch.py:1227-1244; sums of
//           ComputeSliceBoundsAndCoordsSBS_merged :449-531).  The last block
//           to finish folds the block partials in a fixed order: arc
//           [fi_s, fi_e], slice width, mean gamma (merge_multiple_arcs
//           :577-606 for one rank), box mean +- sigma_ratio * sigma, bunch
//           length and cell charge (src/FFAG_Bunch.py:1265-1294).
//   deposit slice index, then CIC weights accumulated as 2^-40 fixed-point
//           integers with 64-bit atomics: the sum is exact, so the charge cube
//           is identical for any particle order and launch
//           (DistributeChargeSBS_Njit :244-312 accumulates float32 in
//           particle order)
//   green   open boundary only: the transform of the free-space Green's
//           function on the doubled grid, float64, as a sum of cosines
//   solve   ONE block per slice, the slice resident in shared memory: real
//           FFT of the charge (rows paired as real and imaginary parts),
//           per column the z transform, the kernel multiply (periodic
//           1/(eps0 k^2) of make_fft_kernel_open_numba :731-760, or the Green
//           transform) and the inverse, inverse real FFT of the rows, and the
//           central-difference field / gamma^2
//           (compute_field_from_potential_numba_SBS :672-728)
//   gather  bilinear field at each particle, projected on the orbit
//           direction (interpolate_fields_to_particles_SBS_numba :870-972),
//           and the roll of the two extrapolation endpoints
//           (src/FFAG_track.py:341-400) in the same pass
// Grids the fused solve does not cover (nx != nz, or sizes other than 32, 64
// and 128) take a chain of batched line FFTs through a global work cube.
// Block partial sums use a fixed grid and fixed reduction order, so every
// update is bit-for-bit reproducible run to run.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cooperative_groups.h>

#include "ffa_internal.cuh"

namespace {

namespace cg = cooperative_groups;
using ffa::PI;

constexpr int SC_TB = 256;
constexpr int SC_BLOCKS = 444;             // pass1: 3 per SM on 148 SMs (one wave); fixed for determinism
constexpr double FIX_SCALE = 1099511627776.0;  // 2^40
constexpr double EPS0 = 8.854187817e-12;

struct SCState {
    ffa_sc_diag diag;
    double inv_dx, inv_dz;
    int32_t degenerate;   // dx <= 0 or dz <= 0: fields are not updated
    int32_t bad;          // degenerate or bunch length <= 0: gathered field = 0
};

// per-block partial sums of pass1
struct Partial {
    double sum_gamma;
    double amin[4], amax[4];
    double sx, sz, sx2, sz2;
    long long count;
};

__device__ __forceinline__ double fast_mod(double a, double b) { return a - b * floor(a / b); }

__device__ __forceinline__ double py_mod(double a, double b)
{
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
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

// Warp tree (shuffle down) then warp 0's values folded in warp order by
// thread 0: the same order on every run.
template <typename T, typename Op>
__device__ __forceinline__ T warp_fold(T v, Op op)
{
    for (int off = 16; off > 0; off >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, off));
    return v;
}

struct OpSum { template <typename T> __device__ T operator()(T a, T b) const { return a + b; } };
struct OpMin { __device__ double operator()(double a, double b) const { return fmin(a, b); } };
struct OpMax { __device__ double operator()(double a, double b) const { return fmax(a, b); } };

// Block reduction of one Partial per thread (valid in thread 0).  Per value:
// warp tree, then thread 0 folds the warps' results starting from the
// identity (0, +1e300 / -1e300 for min / max), in warp order.
__device__ Partial block_partial(const Partial &p)
{
    constexpr int NW = SC_TB / 32;
    __shared__ double sh[NW][13];
    __shared__ long long shc[NW];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    double v[13];
    v[0] = warp_fold(p.sum_gamma, OpSum());
    for (int k = 0; k < 4; ++k) {
        v[1 + k] = warp_fold(p.amin[k], OpMin());
        v[5 + k] = warp_fold(p.amax[k], OpMax());
    }
    v[9] = warp_fold(p.sx, OpSum());
    v[10] = warp_fold(p.sz, OpSum());
    v[11] = warp_fold(p.sx2, OpSum());
    v[12] = warp_fold(p.sz2, OpSum());
    const long long c = warp_fold(p.count, OpSum());
    __syncthreads();
    if (l == 0) {
        for (int k = 0; k < 13; ++k) sh[w][k] = v[k];
        shc[w] = c;
    }
    __syncthreads();
    Partial r;
    r.sum_gamma = 0.0; r.sx = r.sz = r.sx2 = r.sz2 = 0.0; r.count = 0;
    for (int k = 0; k < 4; ++k) { r.amin[k] = 1e300; r.amax[k] = -1e300; }
    if (threadIdx.x == 0) {
        for (int q = 0; q < NW; ++q) {
            r.sum_gamma += sh[q][0];
            for (int k = 0; k < 4; ++k) {
                r.amin[k] = fmin(r.amin[k], sh[q][1 + k]);
                r.amax[k] = fmax(r.amax[k], sh[q][5 + k]);
            }
            r.sx += sh[q][9]; r.sz += sh[q][10]; r.sx2 += sh[q][11]; r.sz2 += sh[q][12];
            r.count += shc[q];
        }
    }
    return r;
}

// The final state from the block partials, by one block: each thread folds a
// fixed strided subset of the partials, then the block reduction above.
__device__ void finalize_state(const Partial *part, int nblk, const ffa_sc_desc &d, SCState *st, int64_t *status)
{
    Partial a;
    a.sum_gamma = 0.0; a.sx = a.sz = a.sx2 = a.sz2 = 0.0; a.count = 0;
    for (int k = 0; k < 4; ++k) { a.amin[k] = 1e30; a.amax[k] = -1e30; }
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        const Partial *q = part + b;
        a.sum_gamma += __ldcg(&q->sum_gamma);
        a.count += __ldcg(&q->count);
        for (int k = 0; k < 4; ++k) {
            a.amin[k] = fmin(a.amin[k], __ldcg(&q->amin[k]));
            a.amax[k] = fmax(a.amax[k], __ldcg(&q->amax[k]));
        }
        a.sx += __ldcg(&q->sx); a.sz += __ldcg(&q->sz); a.sx2 += __ldcg(&q->sx2); a.sz2 += __ldcg(&q->sz2);
    }
    const Partial t = block_partial(a);
    if (threadIdx.x != 0) return;
    ffa_sc_diag &D = st->diag;
    // arc: the trial shift with the smallest span (merge_multiple_arcs)
    const double shifts[4] = {0.0, PI, PI * 0.5, PI * 1.5};
    int best = 0;
    double best_span = t.amax[0] - t.amin[0];
    for (int k = 1; k < 4; ++k)
        if (t.amax[k] - t.amin[k] < best_span) { best_span = t.amax[k] - t.amin[k]; best = k; }
    double arc_s = t.amin[best] - shifts[best], arc_e = t.amax[best] - shifts[best];
    if (arc_e < arc_s) arc_e += 2 * PI;
    double fi_s = py_mod(arc_s, 2 * PI), fi_e = py_mod(arc_e, 2 * PI);
    if (fi_e <= fi_s) fi_e += 2 * PI;
    const long long cnt = t.count;
    D.fi_s = fi_s;
    D.fi_e = fi_e;
    D.slice_step = (fi_e - fi_s) / (d.ns - 1);
    D.count = cnt;
    D.mean_gamma_m1 = cnt > 0 ? t.sum_gamma / (double)cnt - 1.0 : 0.0;
    // box from the moments
    double mx = 0, mz = 0, sgx = 0, sgz = 0;
    if (cnt > 1) {
        mx = t.sx / (double)cnt;
        mz = t.sz / (double)cnt;
        const double vx = t.sx2 / (double)cnt - mx * mx, vz = t.sz2 / (double)cnt - mz * mz;
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

// ----------------------------------------------------------------- passes

// `done` counts finished blocks; it must be zero at launch (it sits in the
// slot after the charge accumulator, which is cleared before every update).
__global__ void __launch_bounds__(SC_TB, 3) sc_pass1(ffa_state_soa S, int64_t n, ffa_sc_desc d, double *x_out,
                                                     double *pr0_out, Partial *part, unsigned long long *done,
                                                     SCState *st, int64_t *status)
{
    const double shifts[4] = {0.0, PI, PI * 0.5, PI * 1.5};
    Partial p;
    p.sum_gamma = 0.0; p.sx = p.sz = p.sx2 = p.sz2 = 0.0; p.count = 0;
    for (int k = 0; k < 4; ++k) { p.amin[k] = 1e30; p.amax[k] = -1e30; }
    // one live particle into the partial sums, in the thread's fixed order
    auto take = [&](int64_t i, double r, double vr, double z, double vz, double fi, double f5) {
        double g;
        if (d.boris) {
            const double rd = r * f5;
            const double v2 = vr * vr + vz * vz + rd * rd;
            g = 1.0 / sqrt(1.0 - v2 / (d.speed_c * d.speed_c));
        } else {
            g = f5 / d.E0_J;
        }
        const double fm = fi - 2 * PI * floor(fi / (2 * PI));
        const double Ek = (g - 1) * d.E0_rest_MeV;
        const double r0 = seo_lookup(d.seo_r, d.Ek0, d.dEk, d.nE, d.fi0, d.dfi, d.nfi, Ek, fm);
        pr0_out[i] = seo_lookup(d.seo_pr, d.Ek0, d.dEk, d.nE, d.fi0, d.dfi, d.nfi, Ek, fm);
        const double xi = r - r0, zi = z;
        x_out[i] = xi;
        p.sum_gamma += g;
        ++p.count;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double v = fast_mod(fm + shifts[k], 2 * PI);
            p.amin[k] = fmin(p.amin[k], v);
            p.amax[k] = fmax(p.amax[k], v);
        }
        p.sx += xi;
        p.sz += zi;
        p.sx2 += xi * xi;
        p.sz2 += zi * zi;
    };
    // every load of a particle issued before its survival test
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t a = S.surv[i];
        const double r = S.r[i], vr = S.vr[i], z = S.z[i], vz = S.vz[i], fi = S.fi[i], f5 = S.f5[i];
        if (a != 0) take(i, r, vr, z, vz, fi, f5);
    }
    const Partial b = block_partial(p);
    __shared__ int last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(done, 1ull) == (unsigned long long)(gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    finalize_state(part, gridDim.x, d, st, status);
}

// slice index of every live particle (-1 otherwise), then the CIC deposit.
// The integer sums do not depend on the order of the atomics, so any grid
// gives the same cube; two particles per pass keep two particles' loads in
// flight per thread.
__global__ void __launch_bounds__(SC_TB) sc_deposit(ffa_state_soa S, int64_t n, ffa_sc_desc d, const double *x,
                                                    int32_t *slice, int64_t *cell, const SCState *st,
                                                    unsigned long long *acc)
{
    const int bad = st->bad;
    const double fi_s = st->diag.fi_s, step = st->diag.slice_step;
    const double xmin = st->diag.xmin, zmin = st->diag.zmin, inv_dx = st->inv_dx, inv_dz = st->inv_dz;
    const int nx = d.nx, nz = d.nz;
    auto one = [&](int64_t i, uint8_t alive, double fi, double xi, double zi) {
        if (alive == 0) {
            slice[i] = -1;
            cell[i] = -1;
            return;
        }
        fi = fi - 2 * PI * floor(fi / (2 * PI));
        if (fi < fi_s) fi += 2 * PI;
        int64_t s = (int64_t)((fi - fi_s) / step);
        if (s < 0) s = 0; else if (s >= d.ns) s = d.ns - 1;
        slice[i] = (int32_t)s;
        if (bad) {
            cell[i] = -1;
            return;
        }
        const double rx = (xi - xmin) * inv_dx, rz = (zi - zmin) * inv_dz;
        int64_t ix = (int64_t)floor(rx), iz = (int64_t)floor(rz);
        double fx = rx - (double)ix, fz = rz - (double)iz;
        if (ix < 0) { ix = 0; fx = 0.0; } else if (ix >= nx - 1) { ix = nx - 2; fx = 1.0; }
        if (iz < 0) { iz = 0; fz = 0.0; } else if (iz >= nz - 1) { iz = nz - 2; fz = 1.0; }
        const int64_t c0 = (s * nz + iz) * nx + ix;
        cell[i] = c0;
        atomicAdd(acc + c0, (unsigned long long)llrint((1.0 - fx) * (1.0 - fz) * FIX_SCALE));
        atomicAdd(acc + c0 + 1, (unsigned long long)llrint(fx * (1.0 - fz) * FIX_SCALE));
        atomicAdd(acc + c0 + nx, (unsigned long long)llrint((1.0 - fx) * fz * FIX_SCALE));
        atomicAdd(acc + c0 + nx + 1, (unsigned long long)llrint(fx * fz * FIX_SCALE));
    };
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 2 * stride) {
        const int64_t k = i + stride < n ? i + stride : i;
        const uint8_t a0 = S.surv[i], a1 = S.surv[k];
        const double f0 = S.fi[i], f1 = S.fi[k], x0 = x[i], x1 = x[k], z0 = S.z[i], z1 = S.z[k];
        one(i, a0, f0, x0, z0);
        if (k != i) one(k, a1, f1, x1, z1);
    }
}

// --------------------------------------------------- open-boundary Green's
//
// G(x, z) = -ln(x^2 + z^2) / (4 pi eps0) on the doubled (NZ, NX) grid with
// x = dx * min(i, NX - i), z = dz * min(j, NZ - j) (the cell average at the
// origin), times dx dz.  G is real and even in both indices, so its 2D DFT is
// real, even, and a double cosine sum over the first quadrant:
//   T[j][kx]  = sum_{i=0}^{NX/2} w_i G[j][i] cos(2 pi i kx / NX)
//   Gk[kz][kx] = sum_{j=0}^{NZ/2} w_j T[j][kx] cos(2 pi j kz / NZ)
// with w = 1 at 0 and N/2, 2 elsewhere.  Both sums in float64; the solve
// reads the (NZ/2 + 1) x (NX/2 + 1) quadrant of Gk rounded to float32.
__device__ __forceinline__ double green_point(int j, int i, double dx, double dz)
{
    const double K = -1.0 / (4.0 * PI * EPS0);
    double v;
    if (i == 0 && j == 0) {
        const double a = 0.5 * dx, b = 0.5 * dz;
        const double F = a * b * (log(a * a + b * b) - 3.0) + a * a * atan(b / a) + b * b * atan(a / b);
        v = K * (F / (a * b));
    } else {
        const double x = dx * (double)i, z = dz * (double)j;
        v = K * log(x * x + z * z);
    }
    return v * dx * dz;
}

// Both sums are small dense products, (hz + 1) x (hx + 1) outputs of
// hx + 1 (rows) or hz + 1 (columns) terms, tiled: a block computes 32 x 32
// outputs (each thread one kx and four rows j or kz), with the shared
// operand staged in GT-term chunks through shared memory and the cosine
// table of the summed axis in shared memory; every output is summed over
// increasing i (or j) as one chain of multiply-adds.
constexpr int GT = 64;

// w_i G[j][i] over the first quadrant (j <= NZ/2, i <= NX/2), row-major,
// every point once
__global__ void __launch_bounds__(256) sc_green_points(int NZ, int NX, const SCState *st, double *G)
{
    if (st->bad) return;
    const int hx = NX / 2, hz = NZ / 2;
    const double dx = st->diag.dx, dz = st->diag.dz;
    const int64_t tot = (int64_t)(hz + 1) * (hx + 1);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(e / (hx + 1)), i = (int)(e - (int64_t)j * (hx + 1));
        G[e] = ((i == 0 || i == hx) ? 1.0 : 2.0) * green_point(j, i, dx, dz);
    }
}

__global__ void __launch_bounds__(256) sc_green_rows(int NZ, int NX, const SCState *st, const double *G, double *T)
{
    if (st->bad) return;
    __shared__ double g[GT][33];     // w_i G[j][i] for a chunk of i and the block's 32 rows j (padded)
    extern __shared__ double cx[];   // cos(2 pi m / NX), m < NX
    const int hx = NX / 2, hz = NZ / 2;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int kx = blockIdx.x * 32 + tx, jb = blockIdx.y * 32;
    for (int m = threadIdx.x; m < NX; m += blockDim.x) cx[m] = cospi(2.0 * (double)m / (double)NX);
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i0 = 0; i0 <= hx; i0 += GT) {
        __syncthreads();
        for (int e = threadIdx.x; e < GT * 32; e += blockDim.x) {
            const int ii = e & (GT - 1), jj = e / GT, i = i0 + ii, j = jb + jj;
            g[ii][jj] = (i <= hx && j <= hz) ? G[(int64_t)j * (hx + 1) + i] : 0.0;
        }
        __syncthreads();
        const int in = min(GT, hx + 1 - i0);
        for (int ii = 0; ii < in; ++ii) {
            const double c = cx[((i0 + ii) * kx) & (NX - 1)];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] += g[ii][ty * 4 + q] * c;
        }
    }
    if (kx > hx) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int j = jb + ty * 4 + q;
        if (j <= hz) T[(int64_t)j * (hx + 1) + kx] = a[q];
    }
}

__global__ void __launch_bounds__(256) sc_green_cols(int NZ, int NX, const SCState *st, const double *T, float *gk)
{
    if (st->bad) return;
    __shared__ double t[GT][32];     // w_j T[j][kx] for a chunk of j and the block's 32 columns kx
    extern __shared__ double cz[];   // cos(2 pi m / NZ), m < NZ
    const int hx = NX / 2, hz = NZ / 2;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int kx = blockIdx.x * 32 + tx, kzb = blockIdx.y * 32 + ty * 4;
    for (int m = threadIdx.x; m < NZ; m += blockDim.x) cz[m] = cospi(2.0 * (double)m / (double)NZ);
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j0 = 0; j0 <= hz; j0 += GT) {
        __syncthreads();
        for (int e = threadIdx.x; e < GT * 32; e += blockDim.x) {
            const int jj = e >> 5, xx = e & 31, j = j0 + jj, x = blockIdx.x * 32 + xx;
            t[jj][xx] = (j <= hz && x <= hx) ? ((j == 0 || j == hz) ? 1.0 : 2.0) * T[(int64_t)j * (hx + 1) + x] : 0.0;
        }
        __syncthreads();
        const int jn = min(GT, hz + 1 - j0);
        for (int jj = 0; jj < jn; ++jj) {
            const double v = t[jj][tx];
            const int j = j0 + jj;
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] += v * cz[(j * (kzb + q)) & (NZ - 1)];
        }
    }
    if (kx > hx) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int kz = kzb + q;
        if (kz <= hz) gk[(int64_t)kz * (hx + 1) + kx] = (float)a[q];
    }
}

// ------------------------------------------------------- fused slice solve
//
// Line transforms in registers.  A line of N = N1 * N2 points is held by a
// group of N1 threads of one warp, N2 points per thread; the four-step
// factorisation
//   X[k2 + N2 k1] = sum_n1 W_N1^(n1 k1) W_N^(n1 k2) sum_n2 x[n1 + N1 n2] W_N2^(n2 k2)
// runs the inner DFTs of length N2 in registers (thread n1 holds
// x[n1 + N1 n2]), multiplies by the twiddles, exchanges through a
// per-group shared-memory scratch (row k2, pitch N1 + 1, conflict-free both
// ways), and runs the outer DFTs of length N1 in registers: thread t ends
// with X[(t + N1 q) + N2 k1].  The inverse runs the same two steps in reverse
// order, so a forward transform followed by an inverse leaves every thread
// with its own input points again.

template <int N> struct Split;
template <> struct Split<32> { static constexpr int N1 = 4, N2 = 8; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<128> { static constexpr int N1 = 8, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };

constexpr int SOLVE_TB = 512;

// group scratch stride (float2): N2 rows of N1 + 1, padded so that the
// groups sharing a half-warp land on disjoint banks
template <int N1, int N2>
__host__ __device__ constexpr int scratch_stride()
{
    return N2 * (N1 + 1) + (((N1 % 16) - (N2 * (N1 + 1)) % 16 + 16) % 16);
}

// cos(2 pi m / 16)
__device__ __forceinline__ float cos16(int m)
{
    switch (m & 15) {
    case 0: return 1.0f;
    case 1: case 15: return 0.92387953251128674f;
    case 2: case 14: return 0.70710678118654752f;
    case 3: case 13: return 0.38268343236508977f;
    case 4: case 12: return 0.0f;
    case 5: case 11: return -0.38268343236508977f;
    case 6: case 10: return -0.70710678118654752f;
    case 7: case 9: return -0.92387953251128674f;
    default: return -1.0f;
    }
}

// b * W_R^m, W = exp(-2 pi i m / R) forward, exp(+2 pi i m / R) inverse;
// m is a constant after unrolling, so the branches and constants fold
template <int R, bool INV>
__device__ __forceinline__ float2 rot(float2 b, int m)
{
    const int m16 = (m * (16 / R)) & 15;
    if (m16 == 0) return b;
    if (m16 == 8) return make_float2(-b.x, -b.y);
    if (m16 == 4) return INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
    if (m16 == 12) return INV ? make_float2(b.y, -b.x) : make_float2(-b.y, b.x);
    const float c = cos16(m16), sn = cos16(m16 - 4);
    const float wi = INV ? sn : -sn;
    return make_float2(b.x * c - b.y * wi, b.x * wi + b.y * c);
}

template <int R>
__host__ __device__ constexpr int brev_c(int k)
{
    int r = 0;
    for (int b = 1, rb = R >> 1; b < R; b <<= 1, rb >>= 1)
        if (k & b) r |= rb;
    return r;
}

template <int R> struct Log2;
template <> struct Log2<4> { static constexpr int v = 2; };
template <> struct Log2<8> { static constexpr int v = 3; };
template <> struct Log2<16> { static constexpr int v = 4; };

// in-register DFT of length R (radix-2, decimation in time), natural order in and out
template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&v)[R])
{
    float2 t[R];
#pragma unroll
    for (int k = 0; k < R; ++k) t[k] = v[brev_c<R>(k)];
#pragma unroll
    for (int st = 0; st < Log2<R>::v; ++st) {
        const int h = 1 << st;
#pragma unroll
        for (int g = 0; g < R; g += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; ++j) {
                const float2 a = t[g + j];
                const float2 b = rot<R, INV>(t[g + j + h], j * (R / (2 * h)));
                t[g + j] = make_float2(a.x + b.x, a.y + b.y);
                t[g + j + h] = make_float2(a.x - b.x, a.y - b.y);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = t[k];
}

__device__ __forceinline__ float2 cmul(float2 a, float2 w) { return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x); }
__device__ __forceinline__ float2 cmulc(float2 a, float2 w) { return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y); }

// forward: in v[n2] = x[t + N1 n2]; out v[q N1 + k1] = X[(t + N1 q) + N2 k1].
// tw[m] = exp(-2 pi i m / N).  Every lane of the warp must call it.
template <int N1, int N2>
__device__ __forceinline__ void fft_fwd(float2 (&v)[N2], int t, float2 *S, const float2 *tw)
{
    constexpr int N = N1 * N2;
    dft<N2, false>(v);
    __syncwarp();
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) S[k2 * (N1 + 1) + t] = cmul(v[k2], tw[(t * k2) & (N - 1)]);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < N2 / N1; ++q) {
        float2 u[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) u[n1] = S[(t + N1 * q) * (N1 + 1) + n1];
        dft<N1, false>(u);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) v[q * N1 + k1] = u[k1];
    }
}

// inverse (unnormalised): in v[q N1 + k1] = X[(t + N1 q) + N2 k1]; out
// v[n2] = x[t + N1 n2].  Every lane of the warp must call it.
template <int N1, int N2>
__device__ __forceinline__ void fft_inv(float2 (&v)[N2], int t, float2 *S, const float2 *tw)
{
    constexpr int N = N1 * N2;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < N2 / N1; ++q) {
        float2 u[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) u[k1] = v[q * N1 + k1];
        dft<N1, true>(u);
        const int k2 = t + N1 * q;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) S[k2 * (N1 + 1) + n1] = cmulc(u[n1], tw[(n1 * k2) & (N - 1)]);
    }
    __syncwarp();
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) v[k2] = S[k2 * (N1 + 1) + t];
    dft<N2, true>(v);
}

// Thread -> (line group, point) map for lines of N1 threads.  Lines in one
// half-warp are N1 apart so that their column points fall on disjoint banks.
template <int N1>
struct Grp {
    int t, gid, line;
    __device__ Grp()
    {
        const int tid = threadIdx.x;
        const int h = tid >> 4;
        const int e = (tid & 15) / N1;
        t = tid & (N1 - 1);
        gid = tid / N1;
        line = (h / N1) * 16 + (h % N1) + N1 * e;
    }
};

template <int NX, int NZ, bool HOCK>
constexpr size_t solve_smem()
{
    constexpr int nz = HOCK ? NZ / 2 : NZ;
    constexpr int P = NX / 2 + 1;
    constexpr int SX = scratch_stride<Split<NX>::N1, Split<NX>::N2>();
    constexpr int SZ = scratch_stride<Split<NZ>::N1, Split<NZ>::N2>();
    constexpr int GX = SOLVE_TB / Split<NX>::N1 * SX, GZ = SOLVE_TB / Split<NZ>::N1 * SZ;
    return sizeof(float2) * (size_t)(nz * P + NX + NZ + (GX > GZ ? GX : GZ));
}

// One cluster of two blocks per slice (block 2 s + r, r = 0, 1; each pass
// over lines gives line 2 m + r to block r).  Charge rows (2p, 2p + 1) are the real and imaginary
// parts of one complex line; their x transforms give the two half spectra
// (kx = 0 .. NX/2).  Each half-spectrum column then goes through the z
// transform, the kernel and the inverse z transform in registers, and row
// pairs come back through one inverse complex line transform each.  The
// inverse takes the real parts of the kx = 0 and kx = NX/2 bins, which is
// what the real part of a full complex inverse transform keeps.  Output: the
// potential (scaled by 1 / (NX NZ) as the normalised inverse does) and the
// field cubes; the charge cube as float32 on the way in.
template <int NX, int NZ, bool HOCK>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SOLVE_TB, 1)
    sc_solve_fused(const unsigned long long *__restrict__ acc, const SCState *st, const float *__restrict__ gk,
                   float *__restrict__ rho, float *__restrict__ phi, float *__restrict__ Ex, float *__restrict__ Ez)
{
    // a cluster of two CTAs per slice: each holds the whole half spectrum,
    // transforms every second line of each pass, and stores its results in
    // its own and its partner's shared memory
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    constexpr int nx = HOCK ? NX / 2 : NX, nz = HOCK ? NZ / 2 : NZ;
    constexpr int P = NX / 2 + 1;     // half-spectrum pitch (float2)
    constexpr int NCOL = NX / 2 + 1;
    constexpr int X1 = Split<NX>::N1, X2 = Split<NX>::N2, Z1 = Split<NZ>::N1, Z2 = Split<NZ>::N2;
    constexpr int SX = scratch_stride<X1, X2>(), SZ = scratch_stride<Z1, Z2>();
    extern __shared__ float4 sm_solve[];
    float2 *spec = reinterpret_cast<float2 *>(sm_solve);
    float2 *twx = spec + nz * P;
    float2 *twz = twx + NX;
    float2 *scr = twz + NZ;
    float2 *peer = cluster.map_shared_rank(spec, rank ^ 1);
    const int tid = threadIdx.x;
    const int64_t cube0 = (int64_t)(blockIdx.x >> 1) * nz * nx;
    const int degenerate = st->degenerate, bad = st->bad;
    if (bad) {   // the same for both CTAs: neither touches the other's memory
        for (int e = tid + rank * SOLVE_TB; e < nz * nx; e += 2 * SOLVE_TB) {
            rho[cube0 + e] = 0.0f;
            phi[cube0 + e] = 0.0f;
            if (!degenerate) { Ex[cube0 + e] = 0.0f; Ez[cube0 + e] = 0.0f; }
        }
        return;
    }
    const double qd = st->diag.q_density / FIX_SCALE;
    for (int m = tid; m < NX; m += SOLVE_TB) {
        double sv, cv;
        sincospi(2.0 * (double)m / (double)NX, &sv, &cv);
        twx[m] = make_float2((float)cv, (float)(-sv));
    }
    for (int m = tid; m < NZ; m += SOLVE_TB) {
        double sv, cv;
        sincospi(2.0 * (double)m / (double)NZ, &sv, &cv);
        twz[m] = make_float2((float)cv, (float)(-sv));
    }
    cluster.sync();   // both CTAs running (and twiddles ready) before any store to the partner

    // (1) forward row transforms, two real rows per complex line
    {
        const Grp<X1> g;
        float2 *S = scr + g.gid * SX;
        constexpr int NPAIR = nz / 2, G = SOLVE_TB / X1;
        for (int base = 0; base < (NPAIR + 1) / 2; base += G) {
            const int p = 2 * (base + g.line) + rank;
            const bool act = p < NPAIR;
            float2 v[X2];
#pragma unroll
            for (int n2 = 0; n2 < X2; ++n2) {
                const int nn = g.t + X1 * n2;
                float a = 0.0f, b = 0.0f;
                if (act && nn < nx) {
                    const int64_t ca = cube0 + (int64_t)(2 * p) * nx + nn;
                    a = (float)((double)acc[ca] * qd);
                    b = (float)((double)acc[ca + nx] * qd);
                    rho[ca] = a;
                    rho[ca + nx] = b;
                }
                v[n2] = make_float2(a, b);
            }
            fft_fwd<X1, X2>(v, g.t, S, twx);
            // natural order into the scratch, then split the pair:
            // A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / 2i
            __syncwarp();
#pragma unroll
            for (int q = 0; q < X2 / X1; ++q)
#pragma unroll
                for (int k1 = 0; k1 < X1; ++k1) S[(g.t + X1 * q) + X2 * k1] = v[q * X1 + k1];
            __syncwarp();
            if (act) {
                for (int k = g.t; k <= NX / 2; k += X1) {
                    const float2 zk = S[k], zn = S[(NX - k) & (NX - 1)];
                    const float2 A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
                    const float2 B = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
                    spec[(2 * p) * P + k] = A;
                    spec[(2 * p + 1) * P + k] = B;
                    peer[(2 * p) * P + k] = A;
                    peer[(2 * p + 1) * P + k] = B;
                }
            }
        }
    }
    cluster.sync();

    // (2) per half-spectrum column: z transform, kernel, inverse z transform
    {
        const Grp<Z1> g;
        float2 *S = scr + g.gid * SZ;
        constexpr int G = SOLVE_TB / Z1;
        float dkx = 0.0f, dkz = 0.0f;
        if (!HOCK) {
            dkx = (float)(2.0 * PI / (nx * st->diag.dx));
            dkz = (float)(2.0 * PI / (nz * st->diag.dz));
        }
        for (int base = 0; base < (NCOL + 1) / 2; base += G) {
            const int c = 2 * (base + g.line) + rank;
            const bool act = c < NCOL;
            float2 v[Z2];
#pragma unroll
            for (int n2 = 0; n2 < Z2; ++n2) {
                const int row = g.t + Z1 * n2;
                v[n2] = (act && row < nz) ? spec[row * P + c] : make_float2(0.0f, 0.0f);
            }
            fft_fwd<Z1, Z2>(v, g.t, S, twz);
#pragma unroll
            for (int q = 0; q < Z2 / Z1; ++q) {
#pragma unroll
                for (int k1 = 0; k1 < Z1; ++k1) {
                    const int kz = (g.t + Z1 * q) + Z2 * k1;
                    float kern = 0.0f;
                    if (act) {
                        if (HOCK) {
                            kern = __ldg(gk + (kz <= NZ / 2 ? kz : NZ - kz) * NCOL + c);
                        } else {
                            // make_fft_kernel_open_numba in float32: bin n/2 is +n/2
                            const float kxf = (float)((double)dkx * (double)c);
                            const float kzf = (float)((double)dkz * (double)(kz <= nz / 2 ? kz : kz - nz));
                            const float kz2 = __fmul_rn(kzf, kzf);
                            const float k2 = __fadd_rn(__fmul_rn(kxf, kxf), kz2);
                            kern = (k2 == 0.0f) ? 0.0f : (float)(1.0 / (EPS0 * (double)k2));
                        }
                    }
                    float2 &w = v[q * Z1 + k1];
                    w.x = __fmul_rn(w.x, kern);
                    w.y = __fmul_rn(w.y, kern);
                }
            }
            fft_inv<Z1, Z2>(v, g.t, S, twz);
            if (act) {
#pragma unroll
                for (int n2 = 0; n2 < Z2; ++n2) {
                    const int row = g.t + Z1 * n2;
                    if (row < nz) {
                        spec[row * P + c] = v[n2];
                        peer[row * P + c] = v[n2];
                    }
                }
            }
        }
    }
    cluster.sync();

    // (3) inverse row transforms: half spectra A (row 2p), B (row 2p + 1)
    // -> Z[k] = A[k] + i B[k] over all k (Hermitian extension) -> a + i b
    {
        const Grp<X1> g;
        float2 *S = scr + g.gid * SX;
        constexpr int NPAIR = nz / 2, G = SOLVE_TB / X1;
        const float scale = (float)(1.0 / ((double)NX * (double)NZ));
        for (int base = 0; base < (NPAIR + 1) / 2; base += G) {
            const int p = 2 * (base + g.line) + rank;
            const bool act = p < NPAIR;
            float2 v[X2];
#pragma unroll
            for (int q = 0; q < X2 / X1; ++q) {
#pragma unroll
                for (int k1 = 0; k1 < X1; ++k1) {
                    const int k = (g.t + X1 * q) + X2 * k1;
                    float2 A = make_float2(0.0f, 0.0f), B = A;
                    if (act) {
                        const int kk = k <= NX / 2 ? k : NX - k;
                        A = spec[(2 * p) * P + kk];
                        B = spec[(2 * p + 1) * P + kk];
                        if (k > NX / 2) { A.y = -A.y; B.y = -B.y; }
                        else if (k == 0 || k == NX / 2) { A.y = 0.0f; B.y = 0.0f; }
                    }
                    v[q * X1 + k1] = make_float2(A.x - B.y, A.y + B.x);
                }
            }
            fft_inv<X1, X2>(v, g.t, S, twx);
            // the group has read rows 2p, 2p + 1 before fft_inv's first
            // barrier: they now hold the two potential rows (float32)
            if (act) {
                float *pa = reinterpret_cast<float *>(spec + (2 * p) * P);
                float *pb = reinterpret_cast<float *>(spec + (2 * p + 1) * P);
                float *qa = reinterpret_cast<float *>(peer + (2 * p) * P);
                float *qb = reinterpret_cast<float *>(peer + (2 * p + 1) * P);
#pragma unroll
                for (int n2 = 0; n2 < X2; ++n2) {
                    const int nn = g.t + X1 * n2;
                    if (nn < nx) {
                        const float fa = __fmul_rn(v[n2].x, scale), fb = __fmul_rn(v[n2].y, scale);
                        pa[nn] = fa;
                        pb[nn] = fb;
                        qa[nn] = fa;
                        qb[nn] = fb;
                        phi[cube0 + (int64_t)(2 * p) * nx + nn] = fa;
                        phi[cube0 + (int64_t)(2 * p + 1) * nx + nn] = fb;
                    }
                }
            }
        }
    }
    cluster.sync();   // the last stores to the partner: phase 4 reads local memory only

    // (4) compute_field_from_potential_numba_SBS for every cell (each cell
    // takes the value of the last loop of the reference that writes it)
    {
        const double dr = st->diag.dx, dz = st->diag.dz, BL = st->diag.bunch_length;
        const double gm = st->diag.mean_gamma_m1 + 1.0;
        const double ig2 = 1.0 / (gm * gm);
        const double inv2dr = 0.5 / dr, inv2dz = 0.5 / dz;
        const bool zero = (dr == 0.0 || dz == 0.0 || BL == 0);
        for (int e = tid + rank * SOLVE_TB; e < nz * nx; e += 2 * SOLVE_TB) {
            if (zero) { Ex[cube0 + e] = 0.0f; Ez[cube0 + e] = 0.0f; continue; }
            const int j = e / nx, i = e - j * nx;
#define PH(jj, ii) reinterpret_cast<const float *>(spec + (jj) * P)[(ii)]
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
            Ex[cube0 + e] = (float)ex;
            Ez[cube0 + e] = (float)ez;
        }
    }
}

// grids the fused solve is instantiated for: square, 32 / 64 / 128
bool fused_grid(int nx, int nz) { return nx == nz && (nx == 32 || nx == 64 || nx == 128); }

template <int NX, int NZ, bool HOCK>
cudaError_t launch_fused_t(const unsigned long long *acc, const SCState *st, int ns, const float *gk, float *rho,
                           float *phi, float *ex, float *ez, cudaStream_t s)
{
    constexpr size_t smem = solve_smem<NX, NZ, HOCK>();
    static_assert(smem <= 227 * 1024, "slice does not fit in shared memory");
    const cudaError_t e = cudaFuncSetAttribute(sc_solve_fused<NX, NZ, HOCK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
    if (e != cudaSuccess) return e;
    sc_solve_fused<NX, NZ, HOCK><<<2 * ns, SOLVE_TB, smem, s>>>(acc, st, gk, rho, phi, ex, ez);   // 2-CTA clusters
    return cudaGetLastError();
}

cudaError_t launch_fused(int n, bool hockney, const unsigned long long *acc, const SCState *st, int ns,
                         const float *gk, float *rho, float *phi, float *ex, float *ez, cudaStream_t s)
{
    if (!hockney) {
        switch (n) {
        case 32: return launch_fused_t<32, 32, false>(acc, st, ns, gk, rho, phi, ex, ez, s);
        case 64: return launch_fused_t<64, 64, false>(acc, st, ns, gk, rho, phi, ex, ez, s);
        default: return launch_fused_t<128, 128, false>(acc, st, ns, gk, rho, phi, ex, ez, s);
        }
    }
    switch (n) {
    case 32: return launch_fused_t<64, 64, true>(acc, st, ns, gk, rho, phi, ex, ez, s);
    case 64: return launch_fused_t<128, 128, true>(acc, st, ns, gk, rho, phi, ex, ez, s);
    default: return launch_fused_t<256, 256, true>(acc, st, ns, gk, rho, phi, ex, ez, s);
    }
}

// ------------------------------------- batched line FFTs (other grid sizes)

// fixed point -> float32 charge cube, and the complex work cube of the
// solver (the reference copies rho into a complex64 array, imaginary 0)
__global__ void sc_convert(const unsigned long long *acc, ffa_sc_desc d, const SCState *st, float *rho,
                           float2 *work, int NZ, int NX)
{
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
}

// Batched radix-2 transforms of complete lines in shared memory, one kernel
// per axis.  Lines run along x (axis 1, contiguous) or z (axis 0, stride NX);
// a CTA holds LINES lines of length n (bit-reversed on load, in-place
// butterflies, one barrier per stage) and forms the n / 2 twiddles
// exp(-2 pi i k / n) itself.  Loads and stores are coalesced for both axes.
// Forward: exp(-2 pi i jk/n); inverse: exp(+2 pi i jk/n), unnormalised.
template <int LINES>
__global__ void __launch_bounds__(256) fft_axis(float2 *data, int NZ, int NX, int axis, int logn, int inverse)
{
    extern __shared__ float2 smf[];
    float2 *sm = smf;
    const int n = 1 << logn;
    const int ld = n + 1;  // padded line pitch
    float2 *base;
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
    float2 *tws = sm + LINES * ld;
    for (int k = threadIdx.x; k < (n >> 1); k += blockDim.x) {
        double sv, cv;
        sincospi(2.0 * (double)k / (double)n, &sv, &cv);
        tws[k] = make_float2((float)cv, (float)(-sv));
    }
    __syncthreads();
    const float sgn = inverse ? 1.0f : -1.0f;
    const int hb = logn - 1;
    for (int s = 1; s <= logn; ++s) {
        const int half = 1 << (s - 1);
        const int twshift = logn - s;
        for (int b = threadIdx.x; b < LINES * (n >> 1); b += blockDim.x) {
            const int l = b >> hb;
            const int bb = b & ((n >> 1) - 1);
            const int grp = bb >> (s - 1);
            const int j = bb & (half - 1);
            const int i0 = grp * (half << 1) + j, i1 = i0 + half;
            const float2 w = tws[j << twshift];
            const float wr = w.x, wi = sgn * (-w.y);  // table holds exp(-2 pi i k/n)
            float2 *p = sm + l * ld;
            const float2 a = p[i0], c = p[i1];
            const float xr = c.x * wr - c.y * wi, xi = c.x * wi + c.y * wr;
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

// multiply by the Green transform (first-quadrant table, even in both indices)
__global__ void sc_mul_green(float2 *work, int ns, int NZ, int NX, const float *gk, const SCState *st)
{
    if (st->bad) return;
    const int64_t plane = (int64_t)NZ * NX;
    const int64_t tot = (int64_t)ns * plane;
    const int hx = NX / 2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t rem = e % plane;
        const int j = (int)(rem / NX), i = (int)(rem - (int64_t)j * NX);
        const int jj = j <= NZ / 2 ? j : NZ - j, ii = i <= hx ? i : NX - i;
        const float k = gk[(int64_t)jj * (hx + 1) + ii];
        float2 v = work[e];
        v.x = __fmul_rn(v.x, k);
        v.y = __fmul_rn(v.y, k);
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

// compute_field_from_potential_numba_SBS for every cell
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

cudaError_t fft2d(float2 *data, int nslices, int NZ, int NX, int lognz, int lognx, int inverse, cudaStream_t s)
{
    constexpr int LINES = 16;
    // lines (padded pitch) + the n / 2 twiddles
    const size_t smx = sizeof(float2) * (LINES * (NX + 1) + NX / 2), smz = sizeof(float2) * (LINES * (NZ + 1) + NZ / 2);
    const cudaError_t e = cudaFuncSetAttribute(fft_axis<LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(smx > smz ? smx : smz));
    if (e != cudaSuccess) return e;
    const unsigned gx = (unsigned)((int64_t)nslices * NZ / LINES), gz = (unsigned)((int64_t)nslices * (NX / LINES));
    if (!inverse) {
        fft_axis<LINES><<<gx, 256, smx, s>>>(data, NZ, NX, 1, lognx, 0);
        fft_axis<LINES><<<gz, 256, smz, s>>>(data, NZ, NX, 0, lognz, 0);
    } else {
        fft_axis<LINES><<<gz, 256, smz, s>>>(data, NZ, NX, 0, lognz, 1);
        fft_axis<LINES><<<gx, 256, smx, s>>>(data, NZ, NX, 1, lognx, 1);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------- gather + roll

// Bilinear field at each live particle, projected on the closed-orbit
// direction; then, when `roll`, the extrapolation endpoints after the update
// (src/FFAG_track.py:341-400): pre <- the new field for live particles,
// pp <- the old pre, and the masks likewise.
__global__ void __launch_bounds__(SC_TB) sc_gather_roll(ffa_state_soa S, int64_t n, ffa_sc_desc d, const double *x,
                                                        const double *pr0, const int32_t *slice, const SCState *st,
                                                        const float *Ex, const float *Ez, int roll, int first)
{
    const int nx = d.nx, nz = d.nz;
    const int degenerate = st->degenerate, bad = st->bad;
    const double x0 = st->diag.xmin, z0 = st->diag.zmin, dx = st->diag.dx, dz = st->diag.dz;
    auto one = [&](int64_t i, int s, double xi, double zi, double p, uint8_t surv) {
        double er = 0.0, ez = 0.0, ef = 0.0;
        bool fresh = false;
        if (!degenerate && s >= 0) {
            if (!bad) {
                const float *EX = Ex + (int64_t)s * nz * nx, *EZ = Ez + (int64_t)s * nz * nx;
                const double t = (xi - x0) / dx, u = (zi - z0) / dz;
                int64_t i0 = (int64_t)floor(t), j0 = (int64_t)floor(u);
                if (i0 < 0) i0 = 0; else if (i0 > nx - 2) i0 = nx - 2;
                if (j0 < 0) j0 = 0; else if (j0 > nz - 2) j0 = nz - 2;
                const double al = t - (double)i0, be = u - (double)j0;
                const double w00 = (1.0 - al) * (1.0 - be), w10 = al * (1.0 - be), w01 = (1.0 - al) * be, w11 = al * be;
                const double gr = w00 * EX[j0 * nx + i0] + w10 * EX[j0 * nx + i0 + 1] + w01 * EX[(j0 + 1) * nx + i0] +
                                  w11 * EX[(j0 + 1) * nx + i0 + 1];
                const double gz = w00 * EZ[j0 * nx + i0] + w10 * EZ[j0 * nx + i0 + 1] + w01 * EZ[(j0 + 1) * nx + i0] +
                                  w11 * EZ[(j0 + 1) * nx + i0 + 1];
                const double rt = sqrt(1 + p * p);
                er = gr * (1 / rt);
                ez = gz;
                ef = gr * (-p / rt);
            }
            S.esc_r[i] = er;
            S.esc_z[i] = ez;
            S.esc_fi[i] = ef;
            fresh = true;
        }
        if (!roll) return;
        const uint8_t alive = surv != 0;
        if (alive && !fresh) { er = S.esc_r[i]; ez = S.esc_z[i]; ef = S.esc_fi[i]; }
        if (first) {
            S.sc_pre[i] = alive;
            S.sc_pp[i] = 0;
            if (alive) {
                S.e_pre_r[i] = er; S.e_pre_z[i] = ez; S.e_pre_fi[i] = ef;
                S.e_pp_r[i] = er; S.e_pp_z[i] = ez; S.e_pp_fi[i] = ef;
            } else {
                S.e_pp_r[i] = S.e_pre_r[i]; S.e_pp_z[i] = S.e_pre_z[i]; S.e_pp_fi[i] = S.e_pre_fi[i];
            }
        } else {
            S.sc_pp[i] = S.sc_pre[i];
            S.sc_pre[i] = alive;
            S.e_pp_r[i] = S.e_pre_r[i]; S.e_pp_z[i] = S.e_pre_z[i]; S.e_pp_fi[i] = S.e_pre_fi[i];
            if (alive) { S.e_pre_r[i] = er; S.e_pre_z[i] = ez; S.e_pre_fi[i] = ef; }
        }
    };
    // two particles per pass, their first loads issued together
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 2 * stride) {
        const int64_t k = i + stride < n ? i + stride : i;
        const int s0 = slice[i], s1 = slice[k];
        const double xa = x[i], xb = x[k], za = S.z[i], zb = S.z[k], pa = pr0[i], pb = pr0[k];
        const uint8_t va = S.surv[i], vb = S.surv[k];
        one(i, s0, xa, za, pa, va);
        if (k != i) one(k, s1, xb, zb, pb, vb);
    }
}

// Blocks of the per-particle passes whose results do not depend on the
// grid (deposit, gather): two particles per thread, at most 16 blocks per SM
unsigned particle_blocks(int64_t n)
{
    const int64_t b = (n + 2 * SC_TB - 1) / (2 * SC_TB);
    return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

int ilog2(int v)
{
    int l = 0;
    while ((1 << l) < v) ++l;
    return (1 << l) == v ? l : -1;
}

// Device buffers of one update.  `acc` holds cells + 1 values: the slot after
// the charge cube is pass1's block counter, cleared with the cube.
struct SCBufs {
    double *x, *pr0;
    int32_t *slice;
    int64_t *cell;
    Partial *part;
    SCState *st;
    unsigned long long *acc;
    float *rho, *phi, *ex, *ez;
    float2 *work;         // batched-FFT path only
    double *gT;           // open boundary: Green row sums, (NZ/2 + 1) x (NX/2 + 1)
    double *gG;           // open boundary: weighted Green points, same shape
    // open boundary with a plan: the Green transform runs on `side`,
    // concurrently with the deposit (fork after pass1, join before the solve)
    cudaStream_t side;
    cudaEvent_t fork, join;
    float *gk;            // open boundary: Green transform quadrant
};

// The whole update on one stream, no host synchronisation.
int run_update(const ffa_sc_desc &d, const SCBufs &b, ffa_state_soa *S, int64_t n, int roll, int first,
               cudaStream_t s, int64_t *status, ffa_sc_diag *diag)
{
    const int NX = d.hockney ? 2 * d.nx : d.nx, NZ = d.hockney ? 2 * d.nz : d.nz;
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    const unsigned ew = 148 * 8;  // elementwise grids
    FFA_CHECK_CUDA(cudaMemsetAsync(b.acc, 0, sizeof(unsigned long long) * (cube + 1), s));
    sc_pass1<<<SC_BLOCKS, SC_TB, 0, s>>>(*S, n, d, b.x, b.pr0, b.part, b.acc + cube, b.st, status);
    if (d.hockney) {
        const bool par = b.side != nullptr;
        const cudaStream_t g = par ? b.side : s;
        if (par) {
            FFA_CHECK_CUDA(cudaEventRecord(b.fork, s));
            FFA_CHECK_CUDA(cudaStreamWaitEvent(b.side, b.fork, 0));
        }
        const dim3 gg((NX / 2 + 32) / 32, (NZ / 2 + 32) / 32);
        const int64_t quad = (int64_t)(NZ / 2 + 1) * (NX / 2 + 1);
        sc_green_points<<<(unsigned)((quad + 255) / 256), 256, 0, g>>>(NZ, NX, b.st, b.gG);
        sc_green_rows<<<gg, 256, sizeof(double) * NX, g>>>(NZ, NX, b.st, b.gG, b.gT);
        sc_green_cols<<<gg, 256, sizeof(double) * NZ, g>>>(NZ, NX, b.st, b.gT, b.gk);
        FFA_CHECK_CUDA(cudaGetLastError());
        if (par) FFA_CHECK_CUDA(cudaEventRecord(b.join, b.side));
    }
    sc_deposit<<<particle_blocks(n), SC_TB, 0, s>>>(*S, n, d, b.x, b.slice, b.cell, b.st, b.acc);
    FFA_CHECK_CUDA(cudaGetLastError());
    if (d.hockney && b.side) FFA_CHECK_CUDA(cudaStreamWaitEvent(s, b.join, 0));
    if (fused_grid(d.nx, d.nz)) {
        FFA_CHECK_CUDA(launch_fused(d.nx, d.hockney != 0, b.acc, b.st, d.ns, b.gk, b.rho, b.phi, b.ex, b.ez, s));
    } else {
        const int lx = ilog2(NX), lz = ilog2(NZ);
        sc_convert<<<ew, 256, 0, s>>>(b.acc, d, b.st, b.rho, b.work, NZ, NX);
        FFA_CHECK_CUDA(cudaGetLastError());
        FFA_CHECK_CUDA(fft2d(b.work, d.ns, NZ, NX, lz, lx, 0, s));
        if (d.hockney) sc_mul_green<<<ew, 256, 0, s>>>(b.work, d.ns, NZ, NX, b.gk, b.st);
        else sc_mul_periodic<<<ew, 256, 0, s>>>(b.work, d, b.st);
        FFA_CHECK_CUDA(fft2d(b.work, d.ns, NZ, NX, lz, lx, 1, s));
        sc_potential<<<ew, 256, 0, s>>>(b.work, d, NZ, NX, b.st, b.phi);
        sc_field<<<ew, 256, 0, s>>>(b.phi, d, b.st, b.ex, b.ez);
    }
    sc_gather_roll<<<particle_blocks(n), SC_TB, 0, s>>>(*S, n, d, b.x, b.pr0, b.slice, b.st, b.ex, b.ez,
                                                        roll ? 1 : 0, first ? 1 : 0);
    FFA_CHECK_CUDA(cudaGetLastError());
    if (diag) FFA_CHECK_CUDA(cudaMemcpyAsync(diag, &b.st->diag, sizeof(ffa_sc_diag), cudaMemcpyDeviceToDevice, s));
    return FFA_OK;
}

int check_state(const ffa_state_soa *S, int64_t n, int32_t roll)
{
    if (!S || n < 0) return FFA_ERR_INVALID;
    if (n == 0) return FFA_OK;      // an empty bunch: the update gives an empty (degenerate) grid
    if (!S->r || !S->vr || !S->z || !S->vz || !S->fi || !S->f5 || !S->surv || !S->esc_r || !S->esc_z || !S->esc_fi)
        return FFA_ERR_INVALID;
    if (roll && (!S->sc_pre || !S->sc_pp || !S->e_pre_r || !S->e_pre_z || !S->e_pre_fi || !S->e_pp_r ||
                 !S->e_pp_z || !S->e_pp_fi))
        return FFA_ERR_INVALID;
    return FFA_OK;
}

int check_desc(const ffa_sc_desc &d)
{
    if (d.ns < 2 || d.nx < 16 || d.nz < 16 || d.nE < 2 || d.nfi < 2 || !d.seo_Ek || !d.seo_r || !d.seo_pr ||
        !d.seo_perimeter || !(d.dEk > 0) || !(d.dfi > 0))
        return FFA_ERR_INVALID;
    return FFA_OK;
}

}  // namespace

struct ffa_sc_plan {
    ffa_sc_desc d;
    SCBufs b;
};

namespace {

void free_plan(ffa_sc_plan *p)
{
    if (!p) return;
    void *ptrs[] = {p->b.x, p->b.pr0, p->b.slice, p->b.cell, p->b.part, p->b.st, p->b.acc, p->b.rho, p->b.phi,
                    p->b.ex, p->b.ez, p->b.work, p->b.gT, p->b.gG, p->b.gk};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (p->b.fork) cudaEventDestroy(p->b.fork);
    if (p->b.join) cudaEventDestroy(p->b.join);
    if (p->b.side) cudaStreamDestroy(p->b.side);
    free(p);
}

}  // namespace

extern "C" {

int ffa_sc_plan_create(const ffa_sc_desc *desc, void *stream, ffa_sc_plan **out)
{
    (void)stream;
    if (!desc || !out) return FFA_ERR_INVALID;
    *out = nullptr;
    const ffa_sc_desc &d = *desc;
    if (check_desc(d) != FFA_OK || d.n_max < 0) return FFA_ERR_INVALID;
    const int lx = ilog2(d.nx), lz = ilog2(d.nz);
    if (lx < 0 || lz < 0 || d.nx > 512 || d.nz > 512) return FFA_ERR_UNSUPPORTED;  // powers of two, <= 512
    ffa_sc_plan *p = (ffa_sc_plan *)calloc(1, sizeof(ffa_sc_plan));
    if (!p) return FFA_ERR_NOMEM;
    p->d = d;
    const int NX = d.hockney ? 2 * d.nx : d.nx, NZ = d.hockney ? 2 * d.nz : d.nz;
    const int64_t n = d.n_max > 0 ? d.n_max : 1;
    const int64_t cube = (int64_t)d.ns * d.nz * d.nx;
    SCBufs &b = p->b;
    bool ok = cudaMalloc(&b.x, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&b.pr0, sizeof(double) * n) == cudaSuccess &&
              cudaMalloc(&b.slice, sizeof(int32_t) * n) == cudaSuccess &&
              cudaMalloc(&b.cell, sizeof(int64_t) * n) == cudaSuccess &&
              cudaMalloc(&b.part, sizeof(Partial) * SC_BLOCKS) == cudaSuccess &&
              cudaMalloc(&b.st, sizeof(SCState)) == cudaSuccess &&
              cudaMalloc(&b.acc, sizeof(unsigned long long) * (cube + 1)) == cudaSuccess &&
              cudaMalloc(&b.rho, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&b.phi, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&b.ex, sizeof(float) * cube) == cudaSuccess &&
              cudaMalloc(&b.ez, sizeof(float) * cube) == cudaSuccess;
    if (ok && !fused_grid(d.nx, d.nz)) ok = cudaMalloc(&b.work, sizeof(float2) * d.ns * (int64_t)NZ * NX) == cudaSuccess;
    if (ok && d.hockney) {
        const int64_t quad = (int64_t)(NZ / 2 + 1) * (NX / 2 + 1);
        ok = cudaMalloc(&b.gT, sizeof(double) * quad) == cudaSuccess &&
             cudaMalloc(&b.gG, sizeof(double) * quad) == cudaSuccess &&
             cudaMalloc(&b.gk, sizeof(float) * quad) == cudaSuccess &&
             cudaStreamCreateWithFlags(&b.side, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&b.join, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) { free_plan(p); return FFA_ERR_NOMEM; }
    if (cudaMemset(b.st, 0, sizeof(SCState)) != cudaSuccess || cudaMemset(b.slice, 0xff, sizeof(int32_t) * n) != cudaSuccess ||
        cudaMemset(b.cell, 0xff, sizeof(int64_t) * n) != cudaSuccess) {
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
    if (!p) return FFA_ERR_INVALID;
    const int rc = check_state(S, n, roll);
    if (rc != FFA_OK) return rc;
    if (n > p->d.n_max) return FFA_ERR_INVALID;
    return run_update(p->d, p->b, S, n, roll, first, reinterpret_cast<cudaStream_t>(stream), status, diag);
}

int ffa_sc_buffers(const ffa_sc_plan *p, const float **rho, const float **phi, const float **ex, const float **ez,
                   const int32_t **slice_idx, const int64_t **cell_idx)
{
    if (!p) return FFA_ERR_INVALID;
    if (rho) *rho = p->b.rho;
    if (phi) *phi = p->b.phi;
    if (ex) *ex = p->b.ex;
    if (ez) *ez = p->b.ez;
    if (slice_idx) *slice_idx = p->b.slice;
    if (cell_idx) *cell_idx = p->b.cell;
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
// call's contents; the charge accumulator (and the block counter after it)
// is cleared at the start of each call, every other region is fully
// rewritten before it is read, and the FFT twiddles are formed inside the
// kernels, so no table outlives a call.  Calls whose work overlaps on the
// GPU (different streams, or host threads) race on the array and must be
// serialised by the caller.  Every call asks the runtime for the array's
// address on the current device (cudaGetSymbolAddress, which allocates
// nothing), so nothing cached can go stale after a device reset.
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
constexpr size_t ST_OFF_PART = ST_OFF_CELL + a256(sizeof(int64_t) * ST_MAX_N);
constexpr size_t ST_OFF_STATE = ST_OFF_PART + a256(sizeof(Partial) * SC_BLOCKS);
constexpr size_t ST_OFF_ACC = ST_OFF_STATE + a256(sizeof(SCState));
constexpr size_t ST_OFF_RHO = ST_OFF_ACC + a256(sizeof(unsigned long long) * (ST_MAX_CELLS + 1));
constexpr size_t ST_OFF_PHI = ST_OFF_RHO + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_EX = ST_OFF_PHI + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_EZ = ST_OFF_EX + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_OFF_WORK = ST_OFF_EZ + a256(sizeof(float) * ST_MAX_CELLS);
constexpr size_t ST_BYTES = ST_OFF_WORK + a256(sizeof(float2) * ST_MAX_CELLS);

}  // namespace

static __device__ __align__(256) unsigned char ffa_sc_static_scratch[ST_BYTES];

extern "C" int ffa_sc_step_static(const ffa_sc_desc *desc, ffa_state_soa *S, int64_t n, int32_t roll,
                                  int32_t first, void *stream, int64_t *status, ffa_sc_diag *diag)
{
    if (!desc) return FFA_ERR_INVALID;
    int rc = check_state(S, n, roll);
    if (rc != FFA_OK) return rc;
    const ffa_sc_desc &d = *desc;
    if (check_desc(d) != FFA_OK) return FFA_ERR_INVALID;
    if (n > ST_MAX_N) return FFA_ERR_INVALID;  // more particles than the static scratch holds
    const int lx = ilog2(d.nx), lz = ilog2(d.nz);
    if (d.hockney || lx < 0 || lz < 0 || d.nx > ST_MAX_GRID || d.nz > ST_MAX_GRID ||
        (int64_t)d.ns * d.nz * d.nx > ST_MAX_CELLS)
        return FFA_ERR_UNSUPPORTED;
    // host code must not use the array's name as a device address: ask the
    // runtime for its address on the current device
    void *ptr = nullptr;
    FFA_CHECK_CUDA(cudaGetSymbolAddress(&ptr, ffa_sc_static_scratch));
    unsigned char *base = static_cast<unsigned char *>(ptr);
    SCBufs b{};
    b.x = reinterpret_cast<double *>(base + ST_OFF_X);
    b.pr0 = reinterpret_cast<double *>(base + ST_OFF_PR0);
    b.slice = reinterpret_cast<int32_t *>(base + ST_OFF_SLICE);
    b.cell = reinterpret_cast<int64_t *>(base + ST_OFF_CELL);
    b.part = reinterpret_cast<Partial *>(base + ST_OFF_PART);
    b.st = reinterpret_cast<SCState *>(base + ST_OFF_STATE);
    b.acc = reinterpret_cast<unsigned long long *>(base + ST_OFF_ACC);
    b.rho = reinterpret_cast<float *>(base + ST_OFF_RHO);
    b.phi = reinterpret_cast<float *>(base + ST_OFF_PHI);
    b.ex = reinterpret_cast<float *>(base + ST_OFF_EX);
    b.ez = reinterpret_cast<float *>(base + ST_OFF_EZ);
    b.work = reinterpret_cast<float2 *>(base + ST_OFF_WORK);
    return run_update(d, b, S, n, roll, first, reinterpret_cast<cudaStream_t>(stream), status, diag);
}
