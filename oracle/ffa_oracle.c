/*
 * ffa_oracle.c -- CPU restatement of PyFFA's multiparticle tracking hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * path is compared against (tests/, __graft_entry__.smoke(), and the
 * cpu_baseline / --impl reference legs of bench.py).  Nothing in the product
 * package links, loads or calls it.
 *
 * Parity pin: the functions below were checked against the reference's own
 * Numba kernels, imported in the development container through single-rank
 * shims, by the golden vectors in tests/golden/ (script: make_golden.py).
 *
 * Every function follows the reference loop it restates, operation for
 * operation and in the same evaluation order, on the reference's N x 16
 * row-major float64 particle matrix (src/FFAG_Bunch.py:23-74):
 *   0 r  1 vr  2 z  3 vz  4 fi (unwrapped)  5 dfi/dt (Boris) | Etot[J] (RK4)
 *   6 inj_t[ns]  7 Inj_flag  8 Survive  9 RF_phase  10-12 Esc r/z/fi
 *   13 Bunch_ID  14 Local_ID  15 Global_ID
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp, no fast-math, no FMA contraction).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NCOL 16
#define MAXG 8
#define MAXSEG 16
#define MAXPOLY 16
#define MAXHARM 16

/* ---------------------------------------------------------------- types */

typedef struct {
    int32_t nsectors;
    int32_t n_spoly;
    int32_t n_spolyp;
    int32_t n_convex;
    int32_t max_order;
    int32_t pad0;
    double B0, k;
    double spoly[MAXPOLY];      /* s(r), highest degree first */
    double spolyp[MAXPOLY];     /* s'(r) */
    double convex[MAXSEG * 5];  /* x0, x1, W0, y01, y02 per segment */
    double r_min, r_step;
    int64_t r_size;
    double fi_min, fi_step;
    int64_t fi_size;
    const double *bz_stack;     /* (max_order+1, r_size, fi_size) */
    const double *bfi_stack;
    const double *br_stack;
    /* field-error harmonics (FFAG_BField_Error, src/FFAG_Field.py:947-993):
     * m, amplitude [T], phase [rad], radial band */
    int32_t n_harm;
    int32_t pad1;
    double harm_m[MAXHARM], harm_amp[MAXHARM], harm_ph[MAXHARM];
    double harm_rmin[MAXHARM], harm_rmax[MAXHARM];
} orc_field;

typedef struct {
    int32_t enable;             /* Emap EnableFlag */
    int32_t ngaps;
    int32_t physical_sum;       /* 0: reference semantics (last gap wins) */
    int32_t pad0;
    double poly_x[MAXG][4], poly_y[MAXG][4];
    double box[MAXG][4];        /* x_min, x_max, y_min, y_max */
    double theta_n[MAXG];       /* gap azimuth + pi/2 */
    double rf_shift[MAXG];      /* rad */
    double acc_Etot_uniform;    /* 1 / gap_width */
    double fc_x0, fc_dx;        /* frequency-curve time axis */
    int64_t fc_n;
    const double *fc_freq;
    const double *fc_volt;
    /* spiral gaps (FFAG_EField_spiral, src/FFAG_Field.py:379-550); er_map
     * NULL: fixed gaps.  Maps (nr, nphi), row-major. */
    const double *er_map, *ezc_map, *ephi_map;
    int64_t nr, nphi;
    double r0, dr, phi0, dphi;
    double gap_az[MAXG];
} orc_emap;

typedef struct {
    int32_t enable;
    int32_t pad0;
    double rmin, rmax, zmin, zmax;
} orc_aperture;

typedef struct {
    double q, c, m0, E0;
} orc_consts;

/* ------------------------------------------------------ small utilities */

/* linear_interpolation_uniform_njit_two_vars, src/FFAG_MathTools.py:1431-1478 */
void orc_freq_curve(const orc_emap *em, double xi, double *freq, double *volt)
{
    int64_t N = em->fc_n;
    int64_t i = (int64_t)floor((xi - em->fc_x0) / em->fc_dx);
    if (i < 0) i = 0;
    else if (i >= N - 1) i = N - 2;
    double x0 = em->fc_x0 + (double)i * em->fc_dx;
    double x1 = x0 + em->fc_dx;
    double y0 = em->fc_freq[i], y1 = em->fc_freq[i + 1];
    double z0 = em->fc_volt[i], z1 = em->fc_volt[i + 1];
    *freq = y0 + (xi - x0) / (x1 - x0) * (y1 - y0);
    *volt = z0 + (xi - x0) / (x1 - x0) * (z1 - z0);
}

/* bharmonics_kernel_1d, src/FFAG_Field.py:1541-1587, for one particle: the
 * Bz sum of the harmonics whose radial band holds r (fi unwrapped), which
 * the caller adds to Bz afterwards; Br and Bfi take nothing. */
static double harmonics_Bz(const orc_field *f, double r, double fi)
{
    if (r <= 0.0) return 0.0;
    double Bz = 0.0;
    for (int k = 0; k < f->n_harm; ++k) {
        if (f->harm_rmin[k] <= r && r <= f->harm_rmax[k])
            Bz += f->harm_amp[k] * cos(f->harm_m[k] * fi + f->harm_ph[k]);
    }
    return Bz;
}

/* GetBfields_Njit body, src/FFAG_Field.py:1333-1426 (alive particles only) */
static void analytic_B(const orc_field *f, double ri, double fii, double zi,
                       double *Bz, double *Br, double *Bfi)
{
    double val = 0.0;
    for (int a = 0; a < f->n_spoly; ++a) val = val * ri + f->spoly[a];
    double spiral = val;
    val = 0.0;
    for (int a = 0; a < f->n_spolyp; ++a) val = val * ri + f->spolyp[a];
    double spiral_p = val;

    double B0r, B0r_p;
    if (f->k == 0.0) {
        B0r = f->B0;
        B0r_p = 0.0;
    } else {
        B0r = f->B0 * pow(ri, f->k);
        B0r_p = f->B0 * f->k * pow(ri, f->k - 1.0);
    }
    double period = 2.0 * M_PI / (double)f->nsectors;
    double fs = fii - spiral;
    fs -= period * floor(fs / period);

    double B0F = 0.0, B0Fp = 0.0;
    for (int j = 0; j < f->n_convex; ++j) {
        const double *cp = &f->convex[5 * j];
        double x0 = cp[0], x1 = cp[1], W0 = cp[2], y01 = cp[3], y02 = cp[4];
        double y_convex = y02 * fabs(y01);
        double k_sig = 16.0 / W0;
        double s1 = 1.0 / (1.0 + exp(-k_sig * (fs - x0)));
        double s2 = 1.0 / (1.0 + exp(k_sig * (fs - x1)));
        double y_local = y_convex * s1 * s2;
        B0F += y_local;
        double s1p = k_sig * s1 * (1.0 - s1);
        double s2p = -k_sig * s2 * (1.0 - s2);
        B0Fp += y_convex * (s1p * s2 + s1 * s2p);
    }
    *Bz = B0r * B0F;
    *Bfi = B0r * B0Fp / ri * zi;
    *Br = (B0r_p * B0F - B0r * B0Fp * spiral_p) * zi;
}

/* Bmap_add_all_orders body, src/FFAG_MathTools.py:1139-1188
 * (int() truncation, index clamped, weights not clamped -> extrapolation) */
static void high_order_B(const orc_field *f, double x, double y, double z,
                         double *oBz, double *oBfi, double *oBr)
{
    int64_t NX = f->r_size, NY = f->fi_size;
    int64_t i = (int64_t)((x - f->r_min) / f->r_step);
    int64_t j = (int64_t)((y - f->fi_min) / f->fi_step);
    if (i < 0) i = 0;
    else if (i >= NX - 1) i = NX - 2;
    if (j < 0) j = 0;
    else if (j >= NY - 1) j = NY - 2;
    double tx = (x - (f->r_min + (double)i * f->r_step)) / f->r_step;
    double ty = (y - (f->fi_min + (double)j * f->fi_step)) / f->fi_step;
    double w00 = (1.0 - tx) * (1.0 - ty), w01 = (1.0 - tx) * ty;
    double w10 = tx * (1.0 - ty), w11 = tx * ty;
    int64_t i1 = i + 1, j1 = j + 1;
    double z2 = z * z;
    double z_even = z2, z_odd = z_even * z;
    for (int n = 1; n <= f->max_order; ++n) {
        const double *BZ = f->bz_stack + (int64_t)n * NX * NY;
        const double *BF = f->bfi_stack + (int64_t)n * NX * NY;
        const double *BR = f->br_stack + (int64_t)n * NX * NY;
        double bz = w00 * BZ[i * NY + j] + w01 * BZ[i * NY + j1] + w10 * BZ[i1 * NY + j] + w11 * BZ[i1 * NY + j1];
        double bfi = w00 * BF[i * NY + j] + w01 * BF[i * NY + j1] + w10 * BF[i1 * NY + j] + w11 * BF[i1 * NY + j1];
        double br = w00 * BR[i * NY + j] + w01 * BR[i * NY + j1] + w10 * BR[i1 * NY + j] + w11 * BR[i1 * NY + j1];
        *oBz += bz * z_even;
        *oBfi += bfi * z_odd;
        *oBr += br * z_odd;
        if (n != f->max_order) {
            z_even *= z2;
            z_odd *= z2;
        }
    }
}

/* emap_kernel for one gap, src/FFAG_Utils.py:984-1036.
 * Returns 1 when (r, fi) is inside the gap rectangle and writes Er, Efi. */
static int gap_field(const orc_emap *em, int g, double acc_Etot, double r, double fi,
                     double *Er, double *Efi)
{
    double x = r * cos(fi);
    double y = r * sin(fi);
    if (x < em->box[g][0] || x > em->box[g][1] || y < em->box[g][2] || y > em->box[g][3])
        return 0;
    double prev = 0.0;
    for (int j = 0; j < 4; ++j) {
        double x0 = em->poly_x[g][j], y0 = em->poly_y[g][j];
        double x1 = em->poly_x[g][(j + 1) % 4], y1 = em->poly_y[g][(j + 1) % 4];
        double cross = (x1 - x0) * (y - y0) - (y1 - y0) * (x - x0);
        if (j == 0) prev = cross;
        else if (cross * prev < 0.0) return 0;
    }
    double dtheta = em->theta_n[g] - fi;
    *Er = acc_Etot * cos(dtheta);
    *Efi = acc_Etot * sin(dtheta);
    return 1;
}

/* Spiral gaps: interpolate_spiral_emap_unique_gap_kernel (src/FFAG_MathTools.py:
 * 1042-1114) for one point -- the first gap whose shifted azimuth
 * (shift_to_nearest_window, :1118-1135) lies on the map's phi axis, then
 * Bilinear_interp_2D_vect_uniform_3fields (:940-1039) with rf_amp = V0 /
 * gap_width.  Returns the gap (-1: none, and no field). */
int orc_spiral_lookup(const orc_emap *em, double rf_amp, double r, double fi, double z, double *Er, double *Ez,
                      double *Efi)
{
    const double twopi = 2.0 * M_PI;
    const double phi_min = em->phi0;
    const double phi_max = em->phi0 + em->dphi * (double)(em->nphi - 1);
    const double phi_center = 0.5 * (phi_min + phi_max);
    int hit = -1;
    double phl = 0.0;
    *Er = 0.0;
    *Ez = 0.0;
    *Efi = 0.0;
    for (int g = 0; g < em->ngaps; ++g) {
        double phi = fi - em->gap_az[g];
        double k = nearbyint((phi_center - phi) / twopi);
        double local = phi + k * twopi;
        if (local >= phi_min && local <= phi_max) {
            hit = g;
            phl = local;
            break;
        }
    }
    if (hit < 0) return -1;
    int64_t i = (int64_t)floor((r - em->r0) / em->dr);
    int64_t j = (int64_t)floor((phl - em->phi0) / em->dphi);
    if (i < 0) i = 0;
    else if (i >= em->nr - 1) i = em->nr - 2;
    if (j < 0) j = 0;
    else if (j >= em->nphi - 1) j = em->nphi - 2;
    double xx0 = em->r0 + (double)i * em->dr;
    double yy0 = em->phi0 + (double)j * em->dphi;
    double tx = (r - xx0) / em->dr;
    double ty = (phl - yy0) / em->dphi;
    double w00 = (1.0 - tx) * (1.0 - ty), w01 = (1.0 - tx) * ty, w10 = tx * (1.0 - ty), w11 = tx * ty;
    const int64_t a = i * em->nphi + j, b = a + em->nphi;
    double er = w00 * em->er_map[a] + w01 * em->er_map[a + 1] + w10 * em->er_map[b] + w11 * em->er_map[b + 1];
    double ez = w00 * em->ezc_map[a] + w01 * em->ezc_map[a + 1] + w10 * em->ezc_map[b] + w11 * em->ezc_map[b + 1];
    double ef = w00 * em->ephi_map[a] + w01 * em->ephi_map[a + 1] + w10 * em->ephi_map[b] +
                w11 * em->ephi_map[b + 1];
    *Er = rf_amp * er;
    *Ez = rf_amp * ez * z;
    *Efi = rf_amp * ef;
    return hit;
}

/* The spiral field times the RF factor of cylindrical_to_cartesian
 * (src/FFAG_MathTools.py:1984) with the hit gap's rf_shift. */
static void spiral_field(const orc_emap *em, double rf_amp, double r, double fi, double z, double rf_phase,
                         double *Er, double *Ez, double *Efi)
{
    int hit = orc_spiral_lookup(em, rf_amp, r, fi, z, Er, Ez, Efi);
    if (hit < 0) return;
    double s = sin(rf_phase + em->rf_shift[hit]);
    *Er = *Er * s;
    *Ez = *Ez * s;
    *Efi = *Efi * s;
}

/* Interpolation2D_EMap (src/FFAG_Field.py:284-306) followed by the RF factor of
 * cylindrical_to_cartesian / RK4_equations_of_motion_njit:
 *   E_cyl = E_gap * sin(RF_phase + rf_shift[gap]).
 * Reference semantics: each gap's call overwrites E, so only the last gap's
 * field survives (E = 0 outside the last gap).  physical_sum adds every gap. */
static void rf_field(const orc_emap *em, double acc_Etot, double r, double fi, double z, double rf_phase,
                     double *Er, double *Ez, double *Efi)
{
    *Er = 0.0;
    *Ez = 0.0;
    *Efi = 0.0;
    if (!em->enable) return;
    if (em->er_map) {
        spiral_field(em, acc_Etot, r, fi, z, rf_phase, Er, Ez, Efi);
        return;
    }
    if (!em->physical_sum) {
        int g = em->ngaps - 1;
        double er = 0.0, ef = 0.0;
        if (gap_field(em, g, acc_Etot, r, fi, &er, &ef)) {
            double s = sin(rf_phase + em->rf_shift[g]);
            *Er = er * s;
            *Efi = ef * s;
        }
    } else {
        for (int g = 0; g < em->ngaps; ++g) {
            double er = 0.0, ef = 0.0;
            if (gap_field(em, g, acc_Etot, r, fi, &er, &ef)) {
                double s = sin(rf_phase + em->rf_shift[g]);
                *Er += er * s;
                *Efi += ef * s;
            }
        }
    }
}

/* ------------------------------------------------------------ Boris step */

/* One Boris_solve call, src/FFAG_track.py:948-1049:
 *   fast_mod_parallel (MathTools:1553), GetBfields_Njit (Field:1333),
 *   Bmap_add_all_orders (MathTools:1139), Interpolation1D_freq_curve
 *   (Field:309), emap_kernel (Utils:984), cylindrical_to_cartesian
 *   (MathTools:1969), boris_push_cartesian_njit (MathTools:1877),
 *   convert_cartesian_to_cylindrical (MathTools:2017).
 * Field-error harmonics are disabled in every workload here (no-op). */
void orc_boris_step(double t, double *mat, int64_t N, double dt,
                    const orc_field *f, const orc_emap *em, const orc_aperture *ap,
                    const orc_consts *cs)
{
    double freq, volt;
    orc_freq_curve(em, t, &freq, &volt);
    double acc_Etot = em->acc_Etot_uniform * volt;
    double dRF = freq * M_PI * 2.0 * dt;
    double period = M_PI * 2.0 / (double)f->nsectors;
    const double q = cs->q, c = cs->c, m = cs->m0;

#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        double *row = mat + i * NCOL;
        double r = row[0], rdot = row[1], z = row[2], zdot = row[3];
        double fi = row[4], fidot = row[5];
        int alive = (row[7] == 1.0) && (row[8] == 1.0);
        double fi_mod = fi - period * floor(fi / period);

        double Bz = 0.0, Br = 0.0, Bfi = 0.0;
        if (alive) {
            analytic_B(f, r, fi_mod, z, &Bz, &Br, &Bfi);
            if (f->max_order >= 1) high_order_B(f, r, fi_mod, z, &Bz, &Bfi, &Br);
        }
        if (f->n_harm > 0) Bz += harmonics_Bz(f, r, fi);   /* src/FFAG_track.py:1007 */
        double Er = 0.0, Ez = 0.0, Efi = 0.0;
        rf_field(em, acc_Etot, r, fi, z, row[9], &Er, &Ez, &Efi);
        Ez += row[11];
        Er += row[10];
        Efi += row[12];

        double sinFi = sin(fi), cosFi = cos(fi);
        double x = r * cosFi, y = r * sinFi;
        double vx = rdot * cosFi - r * fidot * sinFi;
        double vy = rdot * sinFi + r * fidot * cosFi;
        double vz = zdot;
        double x_new = x, y_new = y, z_new = z;
        double vx_new = vx, vy_new = vy, vz_new = vz;

        if (alive) {
            double Ex = Er * cosFi - Efi * sinFi;
            double Ey = Er * sinFi + Efi * cosFi;
            double Bx = -(Br * cosFi - Bfi * sinFi);
            double By = -(Br * sinFi + Bfi * cosFi);
            double Bzc = -Bz;
            if (ap->enable) {
                if (r > ap->rmax || r < ap->rmin || z > ap->zmax || z < ap->zmin) row[8] = 0.0;
            }
            double v2 = vx * vx + vy * vy + vz * vz;
            double gamma = 1.0 / sqrt(1 - v2 / (c * c));
            double px = gamma * m * vx, py = gamma * m * vy, pz = gamma * m * vz;
            px += 0.5 * dt * q * Ex;
            py += 0.5 * dt * q * Ey;
            pz += 0.5 * dt * q * Ez;
            double p2 = px * px + py * py + pz * pz;
            double gamma_minus = sqrt(1 + p2 / (m * m * c * c));
            double coeff_b = 0.5 * dt * q / (gamma_minus * m);
            double tx = coeff_b * Bx, ty = coeff_b * By, tz = coeff_b * Bzc;
            double pxp = px + (py * tz - pz * ty);
            double pyp = py + (pz * tx - px * tz);
            double pzp = pz + (px * ty - py * tx);
            double t2 = tx * tx + ty * ty + tz * tz;
            double s = 2.0 / (1.0 + t2);
            double sx = s * tx, sy = s * ty, sz = s * tz;
            px += (pyp * sz - pzp * sy);
            py += (pzp * sx - pxp * sz);
            pz += (pxp * sy - pyp * sx);
            px += 0.5 * dt * q * Ex;
            py += 0.5 * dt * q * Ey;
            pz += 0.5 * dt * q * Ez;
            double p2n = px * px + py * py + pz * pz;
            double gamma_new = sqrt(1 + p2n / (m * m * c * c));
            vx_new = px / (gamma_new * m);
            vy_new = py / (gamma_new * m);
            vz_new = pz / (gamma_new * m);
            x_new = x + vx_new * dt;
            y_new = y + vy_new * dt;
            z_new = z + vz_new * dt;
        }

        double r_new = sqrt(x_new * x_new + y_new * y_new);
        double fi_before = atan2(y, x);
        double fi_after = atan2(y_new, x_new);
        double dfi = fi_after - fi_before;
        if (dfi > M_PI) dfi -= 2 * M_PI;
        else if (dfi < -M_PI) dfi += 2 * M_PI;
        double fi_new = fi + dfi;
        double cn = cos(fi_new), sn = sin(fi_new);
        double vr = vx_new * cn + vy_new * sn;
        double vfi = -vx_new * sn + vy_new * cn;
        row[0] = r_new;
        row[1] = vr;
        row[2] = z_new;
        row[3] = vz_new;
        row[4] = fi_new;
        row[5] = r_new > 1e-12 ? vfi / r_new : 0.0;
        row[9] += dRF;
    }
}

/* ------------------------------------------------------------- RK4 step */

/* FunctionForAccelerationBunch_dt (src/FFAG_track.py:1743-1801) +
 * RK4_equations_of_motion_njit (src/FFAG_MathTools.py:2205-2266) for one
 * particle row.  Writes the 7 used derivative slots (cols 0-5, 9). */
static void rk4_rhs_row(const double *row, double dRF_rate, double acc_Etot,
                        const orc_field *f, const orc_emap *em, const orc_consts *cs,
                        double *d /* [7]: 0..5 and rf */, int *wrote_motion)
{
    double r = row[0], rdot = row[1], z = row[2], zdot = row[3], fi = row[4], Et = row[5];
    const double q = cs->q, c = cs->c, E0 = cs->E0;
    double period = M_PI * 2.0 / (double)f->nsectors;
    int alive = (row[7] == 1.0) && (row[8] == 1.0);
    if (!alive) {
        *wrote_motion = 0;
        d[6] = dRF_rate;
        return;
    }
    double fi_mod = fi - period * floor(fi / period);
    double Bz = 0.0, Br = 0.0, Bfi = 0.0;
    analytic_B(f, r, fi_mod, z, &Bz, &Br, &Bfi);
    if (f->max_order >= 1) high_order_B(f, r, fi_mod, z, &Bz, &Bfi, &Br);
    if (f->n_harm > 0) Bz += harmonics_Bz(f, r, fi);       /* src/FFAG_track.py:1782 */
    double Er = 0.0, Ez = 0.0, Efi = 0.0;
    rf_field(em, acc_Etot, r, fi, z, row[9], &Er, &Ez, &Efi);
    Ez += row[11];
    Er += row[10];
    Efi += row[12];

    double ig = E0 / Et;
    double inv_gamma2 = ig * ig;
    double beta2 = 1.0 - inv_gamma2;
    double v2 = beta2 * (c * c);
    double vperp2 = v2 - rdot * rdot - zdot * zdot;
    double fidot = sqrt(vperp2) / r;
    double E_dot_v = rdot * Er + (r * fidot) * Efi + zdot * Ez;
    double qc2E = q * (c * c) / Et;
    d[0] = rdot;
    d[1] = (r * fidot * fidot + qc2E * (Er - r * fidot * Bz + zdot * Bfi) - q * rdot / Et * E_dot_v);
    d[2] = zdot;
    d[3] = (qc2E * (Ez + r * fidot * Br - rdot * Bfi) - q * zdot / Et * E_dot_v);
    d[4] = fidot;
    d[5] = q * E_dot_v;
    d[6] = dRF_rate;
    *wrote_motion = 1;
}

/* rk4_step_malloc (src/FFAG_track.py:51-61) + RK4_Post_Step_njit
 * (src/FFAG_MathTools.py:2269-2299).  For skipped (not injected or lost)
 * particles the reference leaves the motion slots of its shared derivative
 * buffer untouched; the post step then only adds the RF-phase increment, so
 * those slots never reach the output and are not modelled here. */
void orc_rk4_step(double t, double *mat, int64_t N, double h,
                  const orc_field *f, const orc_emap *em, const orc_consts *cs)
{
    double fr[4], vo[4], ts[4] = {t, t + 0.5 * h, t + 0.5 * h, t + h};
    double rate[4], acc[4];
    for (int s = 0; s < 4; ++s) {
        orc_freq_curve(em, ts[s], &fr[s], &vo[s]);
        rate[s] = fr[s] * M_PI * 2.0;
        acc[s] = em->acc_Etot_uniform * vo[s];
    }
    static const int cols[7] = {0, 1, 2, 3, 4, 5, 9};

#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        double *row = mat + i * NCOL;
        int alive = (row[7] == 1.0) && (row[8] == 1.0);
        double k[4][7];
        if (!alive) {
            double dr9 = (h * rate[0] + 2 * (h * rate[1]) + 2 * (h * rate[2]) + h * rate[3]) / 6;
            row[9] += dr9;
            continue;
        }
        double stage[NCOL];
        double d[7];
        int wrote;
        memcpy(stage, row, sizeof(stage));
        for (int s = 0; s < 4; ++s) {
            if (s > 0) {
                double w = (s == 3) ? 1.0 : 0.5;
                for (int a = 0; a < 7; ++a)
                    stage[cols[a]] = (s == 3) ? row[cols[a]] + k[s - 1][a] : row[cols[a]] + w * k[s - 1][a];
            }
            rk4_rhs_row(stage, rate[s], acc[s], f, em, cs, d, &wrote);
            for (int a = 0; a < 7; ++a) k[s][a] = h * d[a];
        }
        double dr[7];
        for (int a = 0; a < 7; ++a) dr[a] = (k[0][a] + 2 * k[1][a] + 2 * k[2][a] + k[3][a]) / 6;
        for (int a = 0; a < 6; ++a) row[a] += dr[a];
        row[9] += dr[6];
    }
}

/* ------------------------------------------------------ tracking loops */

/* InjectParticles, src/FFAG_Bunch.py:265-303: particles (sorted by inj_t)
 * from *head onwards with inj_t in [(t-dt)*1e9, t*1e9] are injected. */
static int64_t lower_bound(const double *mat, int64_t lo, int64_t hi, double v)
{
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (mat[mid * NCOL + 6] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static int64_t upper_bound(const double *mat, int64_t lo, int64_t hi, double v)
{
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (mat[mid * NCOL + 6] <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

void orc_inject(double *mat, int64_t N, double t, double dt, int64_t *head)
{
    double high = t * 1e9;
    double low = (t - dt) * 1e9;
    int64_t s = lower_bound(mat, *head, N, low);
    int64_t e = upper_bound(mat, *head, N, high);
    if (e - s > 0) {
        for (int64_t i = s; i < e; ++i) {
            mat[i * NCOL + 7] = 1.0;
            mat[i * NCOL + 8] = 1.0;
        }
        *head = e;
    }
}

/* The step loop of rk4_solve_dt_bunch3_withSC_boris / _withSC
 * (src/FFAG_track.py:297-579, 65-294) with space charge disabled: inject,
 * push, t += dt.  The SC extrapolation masks are all false without SC, so
 * cols 10-12 keep their values.  Returns the final time. */
double orc_track(int solver /*1 Boris, 0 RK4*/, double *mat, int64_t N, double t_start,
                 double dt, int64_t nsteps, int64_t *head,
                 const orc_field *f, const orc_emap *em, const orc_aperture *ap,
                 const orc_consts *cs)
{
    double t = t_start;
    for (int64_t s = 0; s < nsteps; ++s) {
        orc_inject(mat, N, t, dt, head);
        if (solver == 1) orc_boris_step(t, mat, N, dt, f, em, ap, cs);
        else orc_rk4_step(t, mat, N, dt, f, em, cs);
        t = t + dt;
    }
    return t;
}

/* splitmix64 (Steele, Lea and Flood, OOPSLA 2014) as a hash */
static uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* orc_track with rounding noise (test infrastructure): after every step the
 * last bit of r, vr, z, vz, fi and f5 of every particle is flipped or kept,
 * as a hash of (seed, step0 + step, particle, column) decides -- a model of
 * a second float64 implementation whose roundings differ from this one's
 * at every step.  How far the dynamics carries that noise over many steps
 * is the scale against which two correct implementations are compared. */
double orc_track_noisy(int solver, double *mat, int64_t N, double t_start, double dt, int64_t nsteps,
                       int64_t *head, const orc_field *f, const orc_emap *em, const orc_aperture *ap,
                       const orc_consts *cs, uint64_t seed, int64_t step0)
{
    double t = t_start;
    for (int64_t s = 0; s < nsteps; ++s) {
        orc_inject(mat, N, t, dt, head);
        if (solver == 1) orc_boris_step(t, mat, N, dt, f, em, ap, cs);
        else orc_rk4_step(t, mat, N, dt, f, em, cs);
        t = t + dt;
        const uint64_t key = mix64(seed ^ mix64((uint64_t)(step0 + s)));
        for (int64_t i = 0; i < N; ++i) {
            const uint64_t h = mix64(key ^ (uint64_t)i);
            for (int c = 0; c < 6; ++c) {
                double *x = mat + i * NCOL + c;
                uint64_t u;
                memcpy(&u, x, 8);
                u ^= (h >> c) & 1ull;
                memcpy(x, &u, 8);
            }
        }
    }
    return t;
}

/* FunctionForSEO (src/FFAG_track.py:1698-1740): d/dtheta of (r, pr, z, pz)
 * at fixed momentum P, mid-plane field and its z-linear terms. */
static void seo_rhs(const orc_field *f, double t, const double *x, double P, double q, double *d)
{
    double fi = fmod(t, 2.0 * M_PI);
    double fim = fmod(fi, 2.0 * M_PI / (double)f->nsectors);
    double r = x[0], pr = x[1], z = x[2], pz = x[3];
    double Bz, Br, Bfi;
    analytic_B(f, r, fim, z, &Bz, &Br, &Bfi);
    double pfi = sqrt(1 - pr * pr - pz * pz);
    d[0] = r * pr / pfi;
    d[1] = pfi - q / P * (r * Bz - r * pz / pfi * Bfi);
    d[2] = r * pz / pfi;
    d[3] = q / P * (r * Br - r * pr / pfi * Bfi);
}

/* rk4_solve / rk4_solve_vect (src/FFAG_track.py:582-640) in the azimuth:
 * m trajectories x0[m][5] = r, pr, z, pz, P over n_points - 1 steps of
 * h = t_end / (n_points - 1); stage azimuths i*h (time_mode 0) or a running
 * sum (time_mode 1).  x1[m][4] the end state, traj[m][n_points][nc] when
 * not NULL: r, pr (nc = 2) or r, pr, z, pz, Bz, Br, Bfi at each point (nc = 7). */
static void theta_record(const orc_field *f, const double *x, double ts, double *row, int nc)
{
    row[0] = x[0];
    row[1] = x[1];
    if (nc == 7) {
        row[2] = x[2];
        row[3] = x[3];
        double fim = fmod(fmod(ts, 2.0 * M_PI), 2.0 * M_PI / (double)f->nsectors);
        analytic_B(f, x[0], fim, x[2], &row[4], &row[5], &row[6]);
    }
}

void orc_theta_track(const orc_field *f, const double *x0, int64_t m, int n_points, int time_mode,
                     double t_end, double q, double *x1, double *traj, int nc)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double x[4] = {x0[5 * i], x0[5 * i + 1], x0[5 * i + 2], x0[5 * i + 3]};
        double P = x0[5 * i + 4];
        double h = t_end / (double)(n_points - 1);
        double *tr = traj ? traj + i * (int64_t)n_points * nc : NULL;
        if (tr) theta_record(f, x, 0.0, tr, nc);
        double t = 0.0;
        for (int s = 0; s < n_points - 1; ++s) {
            if (time_mode == 0) t = (double)s * h;
            double k1[4], k2[4], k3[4], k4[4], y[4], d[4];
            seo_rhs(f, t, x, P, q, d);
            for (int c = 0; c < 4; ++c) { k1[c] = h * d[c]; y[c] = x[c] + 0.5 * k1[c]; }
            seo_rhs(f, t + 0.5 * h, y, P, q, d);
            for (int c = 0; c < 4; ++c) { k2[c] = h * d[c]; y[c] = x[c] + 0.5 * k2[c]; }
            seo_rhs(f, t + 0.5 * h, y, P, q, d);
            for (int c = 0; c < 4; ++c) { k3[c] = h * d[c]; y[c] = x[c] + k3[c]; }
            seo_rhs(f, t + h, y, P, q, d);
            for (int c = 0; c < 4; ++c) {
                k4[c] = h * d[c];
                x[c] = x[c] + (k1[c] + 2 * k2[c] + 2 * k3[c] + k4[c]) / 6;
            }
            if (time_mode != 0) t = t + h;
            if (tr) theta_record(f, x, time_mode != 0 ? t : (double)(s + 1) * h, tr + (int64_t)(s + 1) * nc, nc);
        }
        for (int c = 0; c < 4; ++c) x1[4 * i + c] = x[c];
    }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
