// ffa_capi.cu -- extern "C" entry points of libffa_cuda.so (see include/ffa_cuda.h).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ffa_internal.cuh"

using namespace ffa;

namespace {

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// the columns every kernel reads; an empty bunch (n = 0) may leave them NULL
bool state_ok(const ffa_state_soa *st, int64_t n)
{
    if (!st) return false;
    if (n == 0) return true;
    return st->r && st->vr && st->z && st->vz && st->fi && st->f5 && st->rf && st->esc_r && st->esc_z &&
           st->esc_fi && st->inj && st->surv;
}

// ---------------------------------------------------------------- kernels

__global__ void inject_kernel(ffa_state_soa st, int64_t n, int64_t step)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (st.inj_step[i] == step) {
        st.inj[i] = 1;
        st.surv[i] = 1;
    }
}

// AoS rows of 16 doubles -> SoA.  Flags are stored as bytes: a column value
// equal to 1.0 maps to 1; the reference only ever stores 0 or 1 there.
__global__ void aos_to_soa_kernel(const double *__restrict__ aos, int64_t n, ffa_state_soa st)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *row = aos + i * 16;
    st.r[i] = row[0];
    st.vr[i] = row[1];
    st.z[i] = row[2];
    st.vz[i] = row[3];
    st.fi[i] = row[4];
    st.f5[i] = row[5];
    st.inj[i] = row[7] == 1.0 ? 1 : (row[7] != 0.0 ? 2 : 0);
    st.surv[i] = row[8] == 1.0 ? 1 : (row[8] != 0.0 ? 2 : 0);
    st.rf[i] = row[9];
    st.esc_r[i] = row[10];
    st.esc_z[i] = row[11];
    st.esc_fi[i] = row[12];
}

__global__ void soa_to_aos_kernel(ffa_state_soa st, int64_t n, double *__restrict__ aos)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *row = aos + i * 16;
    row[0] = st.r[i];
    row[1] = st.vr[i];
    row[2] = st.z[i];
    row[3] = st.vz[i];
    row[4] = st.fi[i];
    row[5] = st.f5[i];
    row[7] = st.inj[i] == 2 ? row[7] : (double)st.inj[i];
    row[8] = st.surv[i] == 2 ? row[8] : (double)st.surv[i];
    row[9] = st.rf[i];
    row[10] = st.esc_r[i];
    row[11] = st.esc_z[i];
    row[12] = st.esc_fi[i];
}

__global__ void mean_fi_kernel(const double *__restrict__ fi, int64_t n, double *out, int64_t *count)
{
    __shared__ double ssum[32];
    __shared__ long long scnt[32];
    double s = 0.0;
    long long c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double v = fi[i];
        if (!isnan(v)) {
            s += v;
            ++c;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        c += __shfl_down_sync(0xffffffffu, c, off);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { ssum[w] = s; scnt[w] = c; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        s = l < nw ? ssum[l] : 0.0;
        c = l < nw ? scnt[l] : 0;
        for (int off = 16; off > 0; off >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, off);
            c += __shfl_down_sync(0xffffffffu, c, off);
        }
        if (l == 0) {
            atomicAdd(out, s);
            atomicAdd((unsigned long long *)count, (unsigned long long)c);
        }
    }
}

unsigned blocks_for(int64_t n, int tb) { return (unsigned)((n + tb - 1) / tb); }

}  // namespace

extern "C" {

int ffa_fieldmap_create(const ffa_field_desc *d, void *stream, ffa_fieldmap **out)
{
    if (!d || !out) return FFA_ERR_INVALID;
    *out = nullptr;
    if (d->nsectors <= 0 || d->n_spoly < 0 || d->n_spoly > FFA_MAX_POLY || d->n_spolyp < 0 ||
        d->n_spolyp > FFA_MAX_POLY || d->n_convex < 0 || d->n_convex > FFA_MAX_SEG || d->max_order < 0)
        return FFA_ERR_INVALID;
    if (d->max_order > FFA_MAX_ORDER) return FFA_ERR_UNSUPPORTED;
    if (d->max_order > 0 && (d->r_size < 2 || d->fi_size < 2 || !d->bz_stack || !d->bfi_stack || !d->br_stack ||
                             !(d->r_step > 0) || !(d->fi_step > 0)))
        return FFA_ERR_INVALID;
    for (int j = 0; j < d->n_convex; ++j)
        if (!(d->convex[5 * j + 2] != 0.0)) return FFA_ERR_INVALID;
    // the push kernels index the node table with 32-bit offsets (12 values per
    // node at most): larger tables are refused
    if (d->max_order > 0 && (double)d->r_size * (double)d->fi_size * 12.0 >= 2147483647.0)
        return FFA_ERR_UNSUPPORTED;

    ffa_fieldmap *fm = (ffa_fieldmap *)calloc(1, sizeof(ffa_fieldmap));
    if (!fm) return FFA_ERR_NOMEM;
    FieldK &k = fm->k;
    k.nsectors = d->nsectors;
    k.n_spoly = d->n_spoly;
    k.n_spolyp = d->n_spolyp;
    k.n_seg = d->n_convex;
    k.max_order = d->max_order;
    const int nv = 3 * d->max_order;
    k.npad = nv <= 4 ? 4 : (nv <= 8 ? 8 : 12);
    k.B0 = d->B0;
    k.k = d->k;
    k.km1 = d->k - 1.0;
    k.B0k = d->B0 * d->k;
    k.period = 2.0 * PI / (double)d->nsectors;
    k.inv_period = 1.0 / k.period;
    memcpy(k.spoly, d->spoly, sizeof(k.spoly));
    memcpy(k.spolyp, d->spolyp, sizeof(k.spolyp));
    for (int j = 0; j < d->n_convex; ++j) {
        const double *cp = d->convex + 5 * j;
        k.seg_x0[j] = cp[0];
        k.seg_x1[j] = cp[1];
        k.seg_k[j] = 16.0 / cp[2];
        k.seg_y[j] = cp[4] * fabs(cp[3]);
    }
    k.r_min = d->r_min;
    k.r_step = d->r_step;
    k.fi_min = d->fi_min;
    k.fi_step = d->fi_step;
    k.r_size = d->r_size;
    k.fi_size = d->fi_size;
    k.spiral_zero = 1;
    for (int a = 0; a < d->n_spoly; ++a) if (d->spoly[a] != 0.0) k.spiral_zero = 0;
    for (int a = 0; a < d->n_spolyp; ++a) if (d->spolyp[a] != 0.0) k.spiral_zero = 0;
    k.r_ref = (d->r_size > 1 && d->r_step > 0) ? d->r_min + 0.5 * d->r_step * (double)(d->r_size - 1) : 1.0;
    k.inv_r_ref = 1.0 / k.r_ref;
    k.inv_r_step = d->r_step > 0 ? 1.0 / d->r_step : 0.0;
    k.inv_fi_step = d->fi_step > 0 ? 1.0 / d->fi_step : 0.0;
    k.c1 = d->k == 0.0 ? d->B0 : d->B0 * pow(k.r_ref, d->k - 1.0);
    k.kc1 = d->k * k.c1;
    // binomial series of (1 + t)^(k-1) around the map centre (see FieldK)
    k.pw_tlim = -1.0;
    if (d->k != 0.0 && d->r_size > 1 && d->r_step > 0) {
        const double m = d->k - 1.0;
        k.pw_r0 = d->r_min + 0.5 * d->r_step * (double)(d->r_size - 1);
        k.pw_inv_r0 = 1.0 / k.pw_r0;
        k.pw_r0m = pow(k.pw_r0, m);
        double c = 1.0;
        for (int n = 0; n < 16; ++n) {
            k.pw_c[n] = c;
            c = c * (m - n) / (double)(n + 1);
        }
        // c is now the first omitted coefficient: largest |t| whose remainder
        // bound |c| |t|^16 / (1 - |t|) stays below 2^-56 (1 - |t|)^m
        double lo = 0.0, hi = 0.5;
        for (int it = 0; it < 60; ++it) {
            const double t = 0.5 * (lo + hi);
            const double rem = fabs(c) * pow(t, 16) / (1.0 - t);
            if (rem < ldexp(1.0, -56) * pow(1.0 - t, fabs(m))) lo = t; else hi = t;
        }
        k.pw_tlim = lo;
    }
    k.B0f = (float)k.B0;
    k.c1f = (float)k.c1;
    k.kc1f = (float)k.kc1;
    k.km1f = (float)k.km1;
    for (int j = 0; j < d->n_convex; ++j) {
        k.seg_x0f[j] = (float)k.seg_x0[j];
        k.seg_x1f[j] = (float)k.seg_x1[j];
        k.seg_kf[j] = (float)k.seg_k[j];
        k.seg_yf[j] = (float)k.seg_y[j];
        k.seg_ykf[j] = (float)(k.seg_y[j] * k.seg_k[j]);
    }
    for (int j = 0; j < d->n_convex; ++j) {
        k.seg_yk[j] = k.seg_y[j] * k.seg_k[j];
        const double hc = 0.5 * k.seg_k[j] * (k.seg_x1[j] - k.seg_x0[j]);
        k.seg_hc[j] = hc <= 300.0 ? hc : 1e300;
        k.seg_K[j] = hc <= 300.0 ? exp(-hc) : 0.0;
    }
    if (d->max_order > 0) {
        const int64_t plane = d->r_size * d->fi_size;
        if (cudaMalloc(&fm->nodes64, sizeof(double) * plane * k.npad) != cudaSuccess) {
            free(fm);
            return FFA_ERR_NOMEM;
        }
        if (cudaMalloc(&fm->nodes32, sizeof(float) * plane * k.npad) != cudaSuccess) {
            cudaFree(fm->nodes64);
            free(fm);
            return FFA_ERR_NOMEM;
        }
        if (launch_pack_nodes(*d, k.npad, fm->nodes64, fm->nodes32, as_stream(stream)) != cudaSuccess) {
            cudaFree(fm->nodes64);
            cudaFree(fm->nodes32);
            free(fm);
            return FFA_ERR_CUDA;
        }
    }
    k.nodes64 = fm->nodes64;
    k.nodes32 = fm->nodes32;
    *out = fm;
    return FFA_OK;
}

int ffa_fieldmap_set_harmonics(ffa_fieldmap *fm, int32_t n, const double *m, const double *amp,
                               const double *phase, const double *rmin, const double *rmax)
{
    if (!fm || n < 0) return FFA_ERR_INVALID;
    if (n > FFA_MAX_HARMONICS) return FFA_ERR_UNSUPPORTED;
    if (n > 0 && (!m || !amp || !phase || !rmin || !rmax)) return FFA_ERR_INVALID;
    double rows[5 * FFA_MAX_HARMONICS] = {0};
    for (int k = 0; k < n; ++k) {
        if (m[k] != floor(m[k]) || !isfinite(amp[k]) || !isfinite(phase[k])) return FFA_ERR_INVALID;
        rows[5 * k] = m[k];
        rows[5 * k + 1] = amp[k];
        rows[5 * k + 2] = phase[k];
        rows[5 * k + 3] = rmin[k];
        rows[5 * k + 4] = rmax[k];
    }
    if (n > 0) {
        if (!fm->harm && cudaMalloc(&fm->harm, sizeof(rows)) != cudaSuccess) return FFA_ERR_NOMEM;
        FFA_CHECK_CUDA(cudaMemcpy(fm->harm, rows, sizeof(rows), cudaMemcpyHostToDevice));
    }
    fm->k.harm = fm->harm;
    fm->k.n_harm = n;
    return FFA_OK;
}

int ffa_fieldmap_destroy(ffa_fieldmap *fm)
{
    if (!fm) return FFA_OK;
    if (fm->nodes64) cudaFree(fm->nodes64);
    if (fm->nodes32) cudaFree(fm->nodes32);
    if (fm->harm) cudaFree(fm->harm);
    free(fm);
    return FFA_OK;
}

int ffa_inject(ffa_state_soa *st, int64_t n, int64_t step, void *stream)
{
    if (n < 0 || !state_ok(st, n) || (n > 0 && !st->inj_step)) return FFA_ERR_INVALID;
    if (n == 0) return FFA_OK;
    inject_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(*st, n, step);
    FFA_CHECK_CUDA(cudaGetLastError());
    return FFA_OK;
}

static int push_impl(const ffa_fieldmap *fm, const ffa_rf_desc *rf, const ffa_aperture *ap, const ffa_consts *cs,
                     const ffa_step_table *tab, ffa_state_soa *st, int64_t n, int64_t step0, int32_t nsteps,
                     double dt, int32_t sc_step, int32_t flags, void *stream, int64_t *status,
                     const ffa_crossing *xing)
{
    if (!fm || !rf || !ap || !cs || !tab || n < 0 || !state_ok(st, n) || nsteps < 0 || step0 < 0)
        return FFA_ERR_INVALID;
    if (!tab->drf || !tab->acc || step0 + nsteps > tab->nsteps) return FFA_ERR_INVALID;
    if (rf->ngaps < 1 || rf->ngaps > FFA_MAX_GAPS) return FFA_ERR_INVALID;
    if (rf->spiral_nodes &&
        (rf->spiral_nr < 2 || rf->spiral_nphi < 2 || !(rf->spiral_dr > 0.0) || !(rf->spiral_dphi > 0.0) ||
         (int64_t)rf->spiral_nr * rf->spiral_nphi >= ((int64_t)1 << 31)))
        return FFA_ERR_INVALID;
    if (sc_step < 0) return FFA_ERR_INVALID;
    if (sc_step > 0 && st->sc_pre &&
        (!st->sc_pp || !st->e_pre_r || !st->e_pre_z || !st->e_pre_fi || !st->e_pp_r || !st->e_pp_z || !st->e_pp_fi))
        return FFA_ERR_INVALID;
    if (flags & ~(FFA_RK4 | FFA_FP32C | FFA_FP32 | FFA_RF_PHYSICAL_SUM | FFA_SHAPE_MASK)) return FFA_ERR_INVALID;
    if ((flags & FFA_FP32) && ((flags & (FFA_RK4 | FFA_FP32C)) || (sc_step > 0 && st->sc_pre) ||
                               fm->k.n_harm > 0))
        return FFA_ERR_UNSUPPORTED;
    const int tb_sel = (flags >> FFA_SHAPE_TB_SHIFT) & 3, nreg_sel = (flags >> FFA_SHAPE_NREG_SHIFT) & 3;
    if ((flags & FFA_RK4) && (tb_sel | nreg_sel)) return FFA_ERR_UNSUPPORTED;
    if (nreg_sel && (!(flags & FFA_FP32C) || (sc_step > 0 && st->sc_pre) || fm->k.n_harm > 0))
        return FFA_ERR_UNSUPPORTED;
    if (n == 0 || nsteps == 0) return FFA_OK;

    PushK p;
    memset(&p, 0, sizeof(p));
    p.f = fm->k;
    p.rf.enable = rf->enable;
    p.rf.ngaps = rf->ngaps;
    p.rf.physical_sum = (flags & FFA_RF_PHYSICAL_SUM) ? 1 : 0;
    memcpy(p.rf.poly_x, rf->poly_x, sizeof(p.rf.poly_x));
    memcpy(p.rf.poly_y, rf->poly_y, sizeof(p.rf.poly_y));
    memcpy(p.rf.box, rf->box, sizeof(p.rf.box));
    memcpy(p.rf.theta_n, rf->theta_n, sizeof(p.rf.theta_n));
    memcpy(p.rf.rf_shift, rf->rf_shift, sizeof(p.rf.rf_shift));
    for (int g = 0; g < rf->ngaps; ++g) {
        // angular extent of the gap rectangle: a convex polygon that does not
        // contain the origin subtends the angles spanned by its vertices
        double cx = 0.0, cy = 0.0;
        for (int j = 0; j < 4; ++j) { cx += rf->poly_x[g][j]; cy += rf->poly_y[g][j]; }
        const double c0 = atan2(cy, cx);
        double half = 0.0;
        for (int j = 0; j < 4; ++j) {
            double d = atan2(rf->poly_y[g][j], rf->poly_x[g][j]) - c0;
            d -= 2.0 * PI * rint(d / (2.0 * PI));
            half = fmax(half, fabs(d));
        }
        p.rf.win_center[g] = c0;
        p.rf.win_half[g] = half < 1.0 ? half + 1e-9 : 4.0;  // wide gaps: no shortcut
    }
    if (rf->spiral_nodes) {
        p.rf.sp = rf->spiral_nodes;
        p.rf.sp_nr = rf->spiral_nr;
        p.rf.sp_nphi = rf->spiral_nphi;
        p.rf.sp_r0 = rf->spiral_r0;
        p.rf.sp_dr = rf->spiral_dr;
        p.rf.sp_phi0 = rf->spiral_phi0;
        p.rf.sp_dphi = rf->spiral_dphi;
        // phi_max and the window centre as shift_to_nearest_window forms them
        // (src/FFAG_MathTools.py:1072-1073, 1131)
        p.rf.sp_phimax = rf->spiral_phi0 + rf->spiral_dphi * (double)(rf->spiral_nphi - 1);
        p.rf.sp_phic = 0.5 * (rf->spiral_phi0 + p.rf.sp_phimax);
        memcpy(p.rf.gap_az, rf->gap_azimuth, sizeof(p.rf.gap_az));
    }
    p.ap = *ap;
    p.cs = *cs;
    p.st = *st;
    if (sc_step == 0) p.st.sc_pre = nullptr;
    p.drf = tab->drf;
    p.acc = tab->acc;
    p.n = n;
    p.step0 = step0;
    p.nsteps = nsteps;
    p.sc_step = sc_step;
    p.dt = dt;
    {
        const double q = cs->q, c = cs->c, m = cs->m0;
        p.hq = 0.5 * dt * q;
        p.inv_mmcc = 1.0 / (m * m * c * c);
        p.inv_cc = 1.0 / (c * c);
        p.inv_m = 1.0 / m;
        p.hqm = p.hq * p.inv_m;
    }
    p.status = status;
    if (xing) {
        if (xing->ntargets < 1 || xing->ntargets > FFA_MAX_CROSSING_TARGETS) return FFA_ERR_INVALID;
        if (xing->fit_sums) {
            // the fit reads f5 as d(phi)/dt, the Boris state; one target
            if (!xing->fit_instance || !xing->fit_centre || !xing->fit_scale || !xing->fit_last ||
                !xing->fit_has || xing->ntargets != 1)
                return FFA_ERR_INVALID;
            if (flags & FFA_RK4) return FFA_ERR_UNSUPPORTED;
        } else if (!xing->buf || !xing->count || xing->capacity < 0) {
            return FFA_ERR_INVALID;
        }
        for (int t = 0; t < xing->ntargets; ++t)
            if (!(xing->target[t] >= 0.0) || !(xing->target[t] < 2.0 * ffa::PI)) return FFA_ERR_INVALID;
        p.xing = *xing;
    }
    cudaError_t e;
    if (flags & FFA_RK4) e = launch_rk4_f64(p, as_stream(stream), (flags & FFA_FP32C) != 0);
    else if (flags & FFA_FP32) e = launch_boris_f32(p, as_stream(stream), 32 << tb_sel);
    else if (flags & FFA_FP32C) e = launch_boris_f32c(p, as_stream(stream), 32 << tb_sel, nreg_sel);
    else e = launch_boris_f64(p, as_stream(stream), 32 << tb_sel);
    return e == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

int ffa_push_occupancy(int32_t flags, int32_t max_order, int32_t crossing, int32_t *blocks_per_sm,
                       int32_t *threads_per_block)
{
    if (!blocks_per_sm || !threads_per_block || max_order < 0 || max_order > FFA_MAX_ORDER) return FFA_ERR_INVALID;
    if (flags & ~(FFA_RK4 | FFA_FP32C | FFA_RF_PHYSICAL_SUM | FFA_SHAPE_MASK)) return FFA_ERR_INVALID;
    const int tb_sel = (flags >> FFA_SHAPE_TB_SHIFT) & 3, nreg_sel = (flags >> FFA_SHAPE_NREG_SHIFT) & 3;
    if ((flags & FFA_RK4) && (tb_sel | nreg_sel)) return FFA_ERR_UNSUPPORTED;
    if (nreg_sel && !(flags & FFA_FP32C)) return FFA_ERR_UNSUPPORTED;
    const int tb = (flags & FFA_RK4) ? ffa::RK4_TB : (32 << tb_sel);
    int blocks = 0;
    if (push_occupancy((flags & FFA_RK4) != 0, (flags & FFA_FP32C) != 0, max_order, crossing != 0, tb, nreg_sel,
                       &blocks) != cudaSuccess)
        return FFA_ERR_CUDA;
    *blocks_per_sm = blocks;
    *threads_per_block = tb;
    return FFA_OK;
}

int ffa_theta_track(const ffa_fieldmap *fm, const ffa_theta_track_desc *d, void *stream)
{
    if (!fm || !d || d->m < 0 || d->n_points < 2 || !(d->t_end > 0.0) || !d->x0 || !d->x1)
        return FFA_ERR_INVALID;
    if (d->time_mode != 0 && d->time_mode != 1) return FFA_ERR_INVALID;
    if (d->traj && d->traj_cols != 2 && d->traj_cols != 7) return FFA_ERR_INVALID;
    if (d->m == 0) return FFA_OK;
    return launch_theta_track(fm->k, *d, as_stream(stream)) == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}

int ffa_push(const ffa_fieldmap *fm, const ffa_rf_desc *rf, const ffa_aperture *ap, const ffa_consts *cs,
             const ffa_step_table *tab, ffa_state_soa *st, int64_t n, int64_t step0, int32_t nsteps, double dt,
             int32_t sc_step, int32_t flags, void *stream, int64_t *status)
{
    return push_impl(fm, rf, ap, cs, tab, st, n, step0, nsteps, dt, sc_step, flags, stream, status, nullptr);
}

int ffa_push_crossing(const ffa_fieldmap *fm, const ffa_rf_desc *rf, const ffa_aperture *ap, const ffa_consts *cs,
                      const ffa_step_table *tab, ffa_state_soa *st, int64_t n, int64_t step0, int32_t nsteps,
                      double dt, int32_t sc_step, int32_t flags, void *stream, int64_t *status,
                      const ffa_crossing *xing)
{
    if (!xing) return FFA_ERR_INVALID;
    return push_impl(fm, rf, ap, cs, tab, st, n, step0, nsteps, dt, sc_step, flags, stream, status, xing);
}

int ffa_aos_to_soa(const double *aos, int64_t n, ffa_state_soa *st, void *stream)
{
    if (n < 0 || !state_ok(st, n) || (n > 0 && !aos)) return FFA_ERR_INVALID;
    if (n == 0) return FFA_OK;
    aos_to_soa_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(aos, n, *st);
    FFA_CHECK_CUDA(cudaGetLastError());
    return FFA_OK;
}

int ffa_soa_to_aos(const ffa_state_soa *st, int64_t n, double *aos, void *stream)
{
    if (n < 0 || !state_ok(st, n) || (n > 0 && !aos)) return FFA_ERR_INVALID;
    if (n == 0) return FFA_OK;
    soa_to_aos_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(*st, n, aos);
    FFA_CHECK_CUDA(cudaGetLastError());
    return FFA_OK;
}

int ffa_mean_fi(const ffa_state_soa *st, int64_t n, double *out, int64_t *count, void *stream)
{
    if (!st || (n > 0 && !st->fi) || !out || !count || n < 0) return FFA_ERR_INVALID;
    cudaStream_t s = as_stream(stream);
    FFA_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
    FFA_CHECK_CUDA(cudaMemsetAsync(count, 0, sizeof(int64_t), s));
    if (n == 0) return FFA_OK;
    unsigned nb = blocks_for(n, 256);
    if (nb > 1184) nb = 1184;
    mean_fi_kernel<<<nb, 256, 0, s>>>(st->fi, n, out, count);
    FFA_CHECK_CUDA(cudaGetLastError());
    return FFA_OK;
}

}  // extern "C"
