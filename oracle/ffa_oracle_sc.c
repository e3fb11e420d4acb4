/*
 * ffa_oracle_sc.c -- CPU restatement of PyFFA's 2.5D space-charge step
 * (FFAG_Bunch.Build_2_5D_SliceGrid_sbs, src/FFAG_Bunch.py:1157-1352) for one
 * rank, plus the open-boundary (Hockney) variant that the reference does not
 * implement.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA space-charge kernels.
 *
 * The reference's transforms run in FFTW complex64 (pyfftw, not vendored,
 * no version pinned).  This restatement transforms in double precision, so
 * its potential is the more accurate of the two; comparisons at the FFT
 * boundary are tolerance checks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NCOL 16

typedef struct {
    int32_t ns, nx, nz;
    int32_t boris;          /* 1: gamma from |v| (Boris layout); 0: Etot/E0 (RK4) */
    int32_t hockney;        /* 0: reference periodic kernel; 1: open boundary */
    int32_t pad0;
    double sigma_ratio;     /* box half-width in sigmas (grid_size_rfz[3]) */
    double q_macro;         /* marcosize * q */
    double speed_c;
    double E0_rest_MeV;
    /* closed-orbit tables: r0(Ek, fi), pr0(Ek, fi) row-major (nE, nfi) */
    int64_t nE, nfi;
    const double *seo_Ek;   /* nE, uniform */
    const double *seo_fi;   /* nfi, uniform, rad */
    const double *seo_r;
    const double *seo_pr;
    const double *seo_perimeter; /* nE */
} orc_sc_params;

typedef struct {
    double fi_s, fi_e, slice_step;
    double mean_gamma_m1;   /* mean(gamma) - 1 */
    double mean_x, mean_z, sigma_x, sigma_z;
    double xmin, xmax, zmin, zmax, dx, dz;
    double bunch_length;
    double q_density;       /* charge weight per particle per cell area */
    int64_t count;
} orc_sc_diag;

static const double EPS0 = 8.854187817e-12;

/* Python's float %, result with the sign of the divisor. */
static double py_mod(double a, double b)
{
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}

/* fast_mod_njit, src/FFAG_MathTools.py:1548-1551 */
static double fast_mod(double a, double b) { return a - b * floor(a / b); }

/* np.interp for increasing xp */
static double np_interp(double x, const double *xp, const double *fp, int64_t n)
{
    if (x <= xp[0]) return fp[0];
    if (x >= xp[n - 1]) return fp[n - 1];
    int64_t lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) / 2;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    double slope = (fp[hi] - fp[lo]) / (xp[hi] - xp[lo]);
    return slope * (x - xp[lo]) + fp[lo];
}

/* Bilinear_interp_2D_vect_uniform, src/FFAG_MathTools.py:828-936 (one point) */
static double bilinear_uniform(double X0, double dX, int64_t NX, double Y0, double dY, int64_t NY,
                               const double *Z, double x, double y)
{
    int64_t i = (int64_t)floor((x - X0) / dX);
    int64_t j = (int64_t)floor((y - Y0) / dY);
    if (i < 0) i = 0; else if (i >= NX - 1) i = NX - 2;
    if (j < 0) j = 0; else if (j >= NY - 1) j = NY - 2;
    double xx0 = X0 + (double)i * dX, yy0 = Y0 + (double)j * dY;
    double tx = (x - xx0) / dX, ty = (y - yy0) / dY;
    double z00 = Z[i * NY + j], z01 = Z[i * NY + j + 1];
    double z10 = Z[(i + 1) * NY + j], z11 = Z[(i + 1) * NY + j + 1];
    return (1 - tx) * (1 - ty) * z00 + (1 - tx) * ty * z01 + tx * (1 - ty) * z10 + tx * ty * z11;
}

/* ------------------------------------------------- radix-2 complex FFT */

static void fft1d(double *re, double *im, int n, int stride, int inverse)
{
    /* bit reversal */
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i * stride]; re[i * stride] = re[j * stride]; re[j * stride] = t;
            t = im[i * stride]; im[i * stride] = im[j * stride]; im[j * stride] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        double ang = 2.0 * M_PI / len * (inverse ? 1.0 : -1.0);
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; ++k) {
                double wr = cos(ang * k), wi = sin(ang * k);
                int a = (i + k) * stride, b = (i + k + len / 2) * stride;
                double xr = re[b] * wr - im[b] * wi;
                double xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
        }
    }
}

/* 2D transform of an (nz, nx) row-major array; the inverse is normalised by
 * 1/(nx*nz) as pyfftw's FFTW.__call__ does by default. */
static void fft2d(double *re, double *im, int nz, int nx, int inverse)
{
    for (int j = 0; j < nz; ++j) fft1d(re + (int64_t)j * nx, im + (int64_t)j * nx, nx, 1, inverse);
    for (int i = 0; i < nx; ++i) fft1d(re + i, im + i, nz, nx, inverse);
    if (inverse) {
        double s = 1.0 / ((double)nx * (double)nz);
        for (int64_t a = 0; a < (int64_t)nx * nz; ++a) { re[a] *= s; im[a] *= s; }
    }
}

/* make_fft_kernel_open_numba, src/FFAG_SC_new.py:731-760: periodic
 * 1/(eps0 k^2) on the (nz, nx) grid in float32, k = 0 set to 0. */
void orc_periodic_kernel(int nx, int nz, double dx, double dz, float *kernel)
{
    float dkx = (float)(2.0 * M_PI / (nx * dx));
    float dkz = (float)(2.0 * M_PI / (nz * dz));
    float *kx = malloc(sizeof(float) * nx), *kz = malloc(sizeof(float) * nz);
    for (int i = 0; i < nx; ++i) kx[i] = (float)((double)dkx * (double)(i <= nx / 2 ? i : i - nx));
    for (int j = 0; j < nz; ++j) kz[j] = (float)((double)dkz * (double)(j <= nz / 2 ? j : j - nz));
    for (int j = 0; j < nz; ++j) {
        float kz2 = kz[j] * kz[j];
        for (int i = 0; i < nx; ++i) {
            float k2 = kx[i] * kx[i] + kz2;
            kernel[(int64_t)j * nx + i] = (k2 == 0.0f) ? 0.0f : (float)(1.0 / (EPS0 * (double)k2));
        }
    }
    free(kx); free(kz);
}

/* Cell average of ln(x^2 + z^2) over [-a, a] x [-b, b]:
 * the antiderivative F(x,z) = x z (ln(x^2+z^2) - 3) + x^2 atan(z/x) + z^2 atan(x/z)
 * taken over the quadrant [0,a] x [0,b], times 4, over the area 4ab. */
static double cell_avg_log_r2(double a, double b)
{
    double F = a * b * (log(a * a + b * b) - 3.0) + a * a * atan(b / a) + b * b * atan(a / b);
    return F / (a * b);
}

/* Open-boundary potential of one slice: zero-pad rho (nz, nx) to (2nz, 2nx),
 * convolve with G(x,z) = -ln(x^2+z^2)/(4 pi eps0) (cell-averaged at the
 * origin) times the cell area, keep the (nz, nx) corner. */
static void hockney_potential(const float *rho, int nz, int nx, double dx, double dz, double *phi)
{
    int NZ = 2 * nz, NX = 2 * nx;
    int64_t M = (int64_t)NZ * NX;
    double *gr = calloc(M, sizeof(double)), *gi = calloc(M, sizeof(double));
    double *rr = calloc(M, sizeof(double)), *ri = calloc(M, sizeof(double));
    const double K = -1.0 / (4.0 * M_PI * EPS0);
    for (int j = 0; j < NZ; ++j) {
        double z = dz * (double)(j <= nz ? j : NZ - j);
        for (int i = 0; i < NX; ++i) {
            double x = dx * (double)(i <= nx ? i : NX - i);
            double g = (i == 0 && j == 0) ? K * cell_avg_log_r2(0.5 * dx, 0.5 * dz) : K * log(x * x + z * z);
            gr[(int64_t)j * NX + i] = g * dx * dz;
        }
    }
    for (int j = 0; j < nz; ++j)
        for (int i = 0; i < nx; ++i) rr[(int64_t)j * NX + i] = rho[(int64_t)j * nx + i];
    fft2d(gr, gi, NZ, NX, 0);
    fft2d(rr, ri, NZ, NX, 0);
    for (int64_t a = 0; a < M; ++a) {
        double xr = rr[a] * gr[a] - ri[a] * gi[a];
        double xi = rr[a] * gi[a] + ri[a] * gr[a];
        rr[a] = xr; ri[a] = xi;
    }
    fft2d(rr, ri, NZ, NX, 1);
    for (int j = 0; j < nz; ++j)
        for (int i = 0; i < nx; ++i) phi[(int64_t)j * nx + i] = rr[(int64_t)j * NX + i];
    free(gr); free(gi); free(rr); free(ri);
}

/* compute_field_from_potential_numba_SBS, src/FFAG_SC_new.py:672-728 */
static void field_from_potential(const float *phi, int nz, int nx, double dr, double dz,
                                 double BL, double mean_gamma_m1, float *Ex, float *Ez)
{
    double gamma = mean_gamma_m1 + 1.0;
    double ig2 = 1.0 / (gamma * gamma);
#define P(j, i) ((double)phi[(int64_t)(j) * nx + (i)])
#define EX(j, i) Ex[(int64_t)(j) * nx + (i)]
#define EZ(j, i) Ez[(int64_t)(j) * nx + (i)]
    if (dr == 0.0 || dz == 0.0 || BL == 0) {
        for (int64_t a = 0; a < (int64_t)nx * nz; ++a) { Ex[a] = 0.0f; Ez[a] = 0.0f; }
        return;
    }
    double inv2dr = 0.5 / dr, inv2dz = 0.5 / dz;
    for (int j = 1; j < nz - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
            EX(j, i) = (float)(-(double)(phi[(int64_t)j * nx + i + 1] - phi[(int64_t)j * nx + i - 1]) * inv2dr * ig2);
            EZ(j, i) = (float)(-(double)(phi[(int64_t)(j + 1) * nx + i] - phi[(int64_t)(j - 1) * nx + i]) * inv2dz * ig2);
        }
    for (int j = 0; j < nz; ++j) {
        int jp = j + 1 < nz - 1 ? j + 1 : nz - 1, jm = j - 1 > 0 ? j - 1 : 0;
        EX(j, 0) = (float)(-(double)(phi[(int64_t)j * nx + 1] - phi[(int64_t)j * nx + 0]) / dr * ig2);
        EZ(j, 0) = (float)(-(double)(phi[(int64_t)jp * nx + 0] - phi[(int64_t)jm * nx + 0]) / dz * ig2);
        EX(j, nx - 1) = (float)(-(double)(phi[(int64_t)j * nx + nx - 1] - phi[(int64_t)j * nx + nx - 2]) / dr * ig2);
        EZ(j, nx - 1) = (float)(-(double)(phi[(int64_t)jp * nx + nx - 1] - phi[(int64_t)jm * nx + nx - 1]) / dz * ig2);
    }
    for (int i = 1; i < nx - 1; ++i) {
        EX(0, i) = (float)(-(double)(phi[i + 1] - phi[i - 1]) * inv2dr * ig2);
        EZ(0, i) = (float)(-(double)(phi[(int64_t)nx + i] - phi[i]) / dz * ig2);
        EX(nz - 1, i) = (float)(-(double)(phi[(int64_t)(nz - 1) * nx + i + 1] - phi[(int64_t)(nz - 1) * nx + i - 1]) * inv2dr * ig2);
        EZ(nz - 1, i) = (float)(-(double)(phi[(int64_t)(nz - 1) * nx + i] - phi[(int64_t)(nz - 2) * nx + i]) / dz * ig2);
    }
#undef P
#undef EX
#undef EZ
}

/* One space-charge update.  alive: Step_SurviveFlag (nonzero = included).
 * Writes cols 10-12 of the surviving particles, the charge, potential and
 * field cubes (ns, nz, nx) float32, per-particle slice index and cell index
 * (cell = (s*nz + iz)*nx + ix of the deposit's lower-left node; -1 for
 * particles not included), and the diagnostics.  Returns 0, or 1 when the
 * grid degenerates (fields not written, as in the reference). */
int orc_sc_step(double *mat, int64_t N, const uint8_t *alive, const orc_sc_params *p,
                float *rho, float *phi_out, float *Ex, float *Ez,
                int32_t *slice_idx, int64_t *cell_idx, orc_sc_diag *dg)
{
    const int ns = p->ns, nx = p->nx, nz = p->nz;
    const double TWO_PI = 2 * M_PI;
    int64_t *sidx = malloc(sizeof(int64_t) * (N > 0 ? N : 1));
    double *cr = malloc(sizeof(double) * (N > 0 ? N : 1)), *cz = malloc(sizeof(double) * (N > 0 ? N : 1));
    double *cfm = malloc(sizeof(double) * (N > 0 ? N : 1)), *cg = malloc(sizeof(double) * (N > 0 ? N : 1));
    int64_t j = 0;
    double sum_gamma = 0.0;
    const double E0_J = 938.2723e6 * 1.60217662e-19;
    /* GetLocalCoordinates_2p5 / _rk, src/FFAG_SC_new.py:74-147 */
    for (int64_t i = 0; i < N; ++i) {
        slice_idx[i] = -1;
        cell_idx[i] = -1;
        if (!alive[i]) continue;
        const double *row = mat + i * NCOL;
        double gamma;
        if (p->boris) {
            double r_dfidt = row[0] * row[5];
            double v2 = row[1] * row[1] + row[3] * row[3] + r_dfidt * r_dfidt;
            gamma = 1.0 / sqrt(1.0 - v2 / (p->speed_c * p->speed_c));
        } else {
            gamma = row[5] / E0_J;
        }
        cr[j] = row[0];
        cz[j] = row[2];
        cg[j] = gamma;
        cfm[j] = row[4] - TWO_PI * floor(row[4] / TWO_PI);
        sidx[j] = i;
        sum_gamma += gamma;
        ++j;
    }
    int64_t cnt = j;
    /* divide_arc2, src/FFAG_SC_new.py:534-567 */
    const double shifts[4] = {0.0, M_PI, M_PI * 0.5, M_PI * 1.5};
    double mn[4] = {1e30, 1e30, 1e30, 1e30}, mx[4] = {-1e30, -1e30, -1e30, -1e30};
    for (int64_t a = 0; a < cnt; ++a)
        for (int k = 0; k < 4; ++k) {
            double v = fast_mod(cfm[a] + shifts[k], 2 * M_PI);
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
        }
    int best = 0;
    double best_span = mx[0] - mn[0];
    for (int k = 1; k < 4; ++k)
        if (mx[k] - mn[k] < best_span) { best_span = mx[k] - mn[k]; best = k; }
    double arc_s = mn[best] - shifts[best], arc_e = mx[best] - shifts[best];
    /* merge_multiple_arcs with one arc, src/FFAG_SC_new.py:577-606 */
    if (arc_e < arc_s) arc_e += 2 * M_PI;
    double fi_s = py_mod(arc_s, 2 * M_PI), fi_e = py_mod(arc_e, 2 * M_PI);
    if (fi_e <= fi_s) fi_e += 2 * M_PI;
    double slice_step = (fi_e - fi_s) / (ns - 1);
    double mg = cnt > 0 ? sum_gamma / (double)cnt - 1.0 : 0.0;

    /* r0, pr0 lookups (src/FFAG_Bunch.py:1227-1244) and
     * ComputeSliceBoundsAndCoordsSBS_merged (src/FFAG_SC_new.py:449-531) */
    double *cx = malloc(sizeof(double) * (cnt > 0 ? cnt : 1)), *cpr = malloc(sizeof(double) * (cnt > 0 ? cnt : 1));
    int32_t *cs = malloc(sizeof(int32_t) * (cnt > 0 ? cnt : 1));
    double dE = p->seo_Ek[1] - p->seo_Ek[0], dF = p->seo_fi[1] - p->seo_fi[0];
    double sx = 0.0, sz = 0.0, sx2 = 0.0, sz2 = 0.0;
    for (int64_t a = 0; a < cnt; ++a) {
        double Ek = (cg[a] - 1) * p->E0_rest_MeV;
        double r0 = bilinear_uniform(p->seo_Ek[0], dE, p->nE, p->seo_fi[0], dF, p->nfi, p->seo_r, Ek, cfm[a]);
        cpr[a] = bilinear_uniform(p->seo_Ek[0], dE, p->nE, p->seo_fi[0], dF, p->nfi, p->seo_pr, Ek, cfm[a]);
        double x = cr[a] - r0, z = cz[a];
        cx[a] = x;
        sx += x; sz += z; sx2 += x * x; sz2 += z * z;
        double fi = cfm[a];
        if (fi < fi_s) fi += TWO_PI;
        int64_t s = (int64_t)((fi - fi_s) / slice_step);
        if (s < 0) s = 0; else if (s >= ns) s = ns - 1;
        cs[a] = (int32_t)s;
        slice_idx[sidx[a]] = (int32_t)s;
    }
    double mean_x = 0, mean_z = 0, sig_x = 0, sig_z = 0;
    if (cnt > 1) {
        mean_x = sx / (double)cnt;
        mean_z = sz / (double)cnt;
        double vx = sx2 / (double)cnt - mean_x * mean_x, vz = sz2 / (double)cnt - mean_z * mean_z;
        sig_x = sqrt(vx > 0.0 ? vx : 0.0);
        sig_z = sqrt(vz > 0.0 ? vz : 0.0);
    }
    double perim = np_interp(mg * p->E0_rest_MeV, p->seo_Ek, p->seo_perimeter, p->nE);
    double BL = perim * (fi_e - fi_s) / M_PI / 2.0;
    double scale = p->sigma_ratio;
    double xmin = mean_x - scale * sig_x, xmax = mean_x + scale * sig_x;
    double zmin = mean_z - scale * sig_z, zmax = mean_z + scale * sig_z;

    /* DistributeChargeSBS_Njit, src/FFAG_SC_new.py:244-312: slices in order,
     * particles of a slice in index order, float32 accumulation. */
    int64_t cube = (int64_t)ns * nz * nx;
    memset(rho, 0, sizeof(float) * cube);
    double dx = (xmax - xmin) / nx, dz = (zmax - zmin) / nz;
    double q = 0.0;
    int degenerate = (dx <= 0.0 || dz <= 0.0);
    if (!degenerate && BL > 0.0) {
        double inv_dx = 1.0 / dx, inv_dz = 1.0 / dz;
        q = (p->q_macro / BL * ns) * (1.0 / (dx * dz));
        for (int s = 0; s < ns; ++s)
            for (int64_t a = 0; a < cnt; ++a) {
                if (cs[a] != s) continue;
                double rx = (cx[a] - xmin) * inv_dx, rz = (cz[a] - zmin) * inv_dz;
                int64_t ix = (int64_t)floor(rx), iz = (int64_t)floor(rz);
                double fx = rx - (double)ix, fz = rz - (double)iz;
                if (ix < 0) { ix = 0; fx = 0.0; } else if (ix >= nx - 1) { ix = nx - 2; fx = 1.0; }
                if (iz < 0) { iz = 0; fz = 0.0; } else if (iz >= nz - 1) { iz = nz - 2; fz = 1.0; }
                float *R = rho + (int64_t)s * nz * nx;
                R[iz * nx + ix] = (float)((double)R[iz * nx + ix] + (1.0 - fx) * (1.0 - fz) * q);
                R[iz * nx + ix + 1] = (float)((double)R[iz * nx + ix + 1] + fx * (1.0 - fz) * q);
                R[(iz + 1) * nx + ix] = (float)((double)R[(iz + 1) * nx + ix] + (1.0 - fx) * fz * q);
                R[(iz + 1) * nx + ix + 1] = (float)((double)R[(iz + 1) * nx + ix + 1] + fx * fz * q);
                cell_idx[sidx[a]] = ((int64_t)s * nz + iz) * nx + ix;
            }
    }
    dg->fi_s = fi_s; dg->fi_e = fi_e; dg->slice_step = slice_step; dg->mean_gamma_m1 = mg;
    dg->mean_x = mean_x; dg->mean_z = mean_z; dg->sigma_x = sig_x; dg->sigma_z = sig_z;
    dg->xmin = xmin; dg->xmax = xmax; dg->zmin = zmin; dg->zmax = zmax; dg->dx = dx; dg->dz = dz;
    dg->bunch_length = BL; dg->q_density = q; dg->count = cnt;

    int rc = 0;
    if (degenerate) {
        memset(phi_out, 0, sizeof(float) * cube);
        memset(Ex, 0, sizeof(float) * cube);
        memset(Ez, 0, sizeof(float) * cube);
        rc = 1;
    } else {
        int64_t M = (int64_t)nz * nx;
        float *kern = malloc(sizeof(float) * M);
        orc_periodic_kernel(nx, nz, dx, dz, kern);
        double *re = malloc(sizeof(double) * M), *im = malloc(sizeof(double) * M);
        double *ph = malloc(sizeof(double) * M);
        for (int s = 0; s < ns; ++s) {
            const float *R = rho + (int64_t)s * M;
            float *PH = phi_out + (int64_t)s * M;
            if (p->hockney) {
                hockney_potential(R, nz, nx, dx, dz, ph);
                for (int64_t a = 0; a < M; ++a) PH[a] = (float)ph[a];
            } else {
                for (int64_t a = 0; a < M; ++a) { re[a] = R[a]; im[a] = 0.0; }
                fft2d(re, im, nz, nx, 0);
                for (int64_t a = 0; a < M; ++a) { re[a] *= kern[a]; im[a] *= kern[a]; }
                fft2d(re, im, nz, nx, 1);
                for (int64_t a = 0; a < M; ++a) PH[a] = (float)re[a];
            }
            field_from_potential(PH, nz, nx, dx, dz, BL, mg, Ex + (int64_t)s * M, Ez + (int64_t)s * M);
        }
        free(kern); free(re); free(im); free(ph);
        /* interpolate_fields_to_particles_SBS_numba, src/FFAG_SC_new.py:870-972 */
        int bad = (dx <= 0.0) || (dz <= 0.0) || (BL <= 0.0);
        for (int64_t a = 0; a < cnt; ++a) {
            double *row = mat + sidx[a] * NCOL;
            if (bad) { row[10] = 0.0; row[11] = 0.0; row[12] = 0.0; continue; }
            int s = cs[a];
            const float *EXs = Ex + (int64_t)s * M, *EZs = Ez + (int64_t)s * M;
            double t = (cx[a] - xmin) / dx, u = (cz[a] - zmin) / dz;
            int64_t i0 = (int64_t)floor(t), j0 = (int64_t)floor(u);
            if (i0 < 0) i0 = 0; else if (i0 > nx - 2) i0 = nx - 2;
            if (j0 < 0) j0 = 0; else if (j0 > nz - 2) j0 = nz - 2;
            double al = t - (double)i0, be = u - (double)j0;
            double w00 = (1.0 - al) * (1.0 - be), w10 = al * (1.0 - be);
            double w01 = (1.0 - al) * be, w11 = al * be;
            double er = w00 * EXs[j0 * nx + i0] + w10 * EXs[j0 * nx + i0 + 1] + w01 * EXs[(j0 + 1) * nx + i0] + w11 * EXs[(j0 + 1) * nx + i0 + 1];
            double ez = w00 * EZs[j0 * nx + i0] + w10 * EZs[j0 * nx + i0 + 1] + w01 * EZs[(j0 + 1) * nx + i0] + w11 * EZs[(j0 + 1) * nx + i0 + 1];
            double pr0 = cpr[a];
            row[10] = er * (1 / sqrt(1 + pr0 * pr0));
            row[11] = ez;
            row[12] = er * (-pr0 / sqrt(1 + pr0 * pr0));
        }
    }
    free(sidx); free(cr); free(cz); free(cfm); free(cg); free(cx); free(cpr); free(cs);
    return rc;
}
