// ffa_push.cu -- fused multi-step particle pushers for sm_100a.
//
// One thread owns one particle for the whole launch: the state lives in
// registers across `nsteps` time steps, so HBM sees one read and one write of
// the structure-of-arrays state per launch.  Per step the thread does what the
// reference does in ~8 full-array passes:
//   fast_mod_parallel        src/FFAG_MathTools.py:1553-1557
//   GetBfields_Njit          src/FFAG_Field.py:1333-1426
//   Bmap_add_all_orders      src/FFAG_MathTools.py:1139-1188
//   emap_kernel (per gap)    src/FFAG_Utils.py:984-1036
//   cylindrical_to_cartesian src/FFAG_MathTools.py:1969-2014
//   boris_push_cartesian_njit src/FFAG_MathTools.py:1877-1966
//   convert_cartesian_to_cylindrical src/FFAG_MathTools.py:2017-2060
// (RK4: FunctionForAccelerationBunch_dt src/FFAG_track.py:1743-1801 four times,
//  RK4_equations_of_motion_njit and RK4_Post_Step_njit
//  src/FFAG_MathTools.py:2205-2299.)
//
// The Boris step is taken in the particle's own frame (r-hat, fi-hat, z-hat)
// instead of the fixed Cartesian frame.  The Boris update commutes with
// rotations, so this is the reference's step up to rounding: the reference
// rotates x, v, E, B into Cartesian axes, pushes, and rotates back with the
// azimuth change atan2(y', x') - atan2(y, x); here the azimuth change is
// atan2 of the displacement in the local frame.  It saves one atan2 and two
// sin/cos pairs per step and is the more accurate of the two.  Particles that
// are skipped (not injected or lost) take the reference's exact Cartesian
// round trip, which perturbs r, vr and dfi/dt by rounding every step.
// Expressions otherwise keep the reference's evaluation order; the compiler may
// fuse a multiply and an add into one FMA (at most an ulp per operation).
#include "ffa_internal.cuh"

namespace ffa {

// ----------------------------------------------------------- field (fp64)

__device__ __forceinline__ void analytic_b64(const FieldK &f, double ri, double ir, double fim, double zi,
                                             double &Bz, double &Br, double &Bfi)
{
    // theta' = (fi mod P) - s(r), reduced mod P again.  Without a spiral
    // (all-zero coefficients evaluate to exactly 0) the callers' fim is
    // reduced already: the second reduction would only map a fim within an
    // ulp of P to about 0 (a step lands there with probability ~1e-16), so
    // it is skipped with the polynomials.
    double spiral_p = 0.0;
    double fs = fim;
    if (!f.spiral_zero) {
        double spiral = 0.0;
        for (int a = 0; a < f.n_spoly; ++a) spiral = spiral * ri + f.spoly[a];
        for (int a = 0; a < f.n_spolyp; ++a) spiral_p = spiral_p * ri + f.spolyp[a];
        fs = fim - spiral;
        fs -= f.period * floor(fs * f.inv_period);
    }
    double B0r, B0r_p;
    if (f.k == 0.0) {
        B0r = f.B0;
        B0r_p = 0.0;
    } else {
        // r^k = r^(k-1) * r: one power instead of two.  Near the map centre
        // the binomial series of (1 + t)^(k-1) (16 terms, truncation below
        // 2^-56, a few ulp of rounding); elsewhere exp((k-1) ln r), whose
        // error is a few ulp of (k-1) ln r ~ 14, i.e. ~1e-15 relative.
        double pk1;
        const double t = (ri - f.pw_r0) * f.pw_inv_r0;
        if (fabs(t) <= f.pw_tlim) {
            double P = f.pw_c[15];
#pragma unroll
            for (int a = 14; a >= 0; --a) P = P * t + f.pw_c[a];
            pk1 = f.pw_r0m * P;
        } else {
            pk1 = exp(f.km1 * log(ri));
        }
        B0r_p = f.B0k * pk1;
        B0r = f.B0 * (pk1 * ri);
    }
    double B0F = 0.0, B0Fp = 0.0;
    for (int j = 0; j < f.n_seg; ++j) {
        const double ks = f.seg_k[j];
        // Past 37.5 the exponential is below 2^-54, so 1 + e rounds to 1 and
        // the sigmoid is exactly 1 (its derivative exactly 0): the branch
        // skips only exponentials that cannot change the result.  Inside a
        // magnet both of its sigmoids saturate; outside it, one of them.
        const double a1 = ks * (fs - f.seg_x0[j]);
        const double a2 = ks * (fs - f.seg_x1[j]);
        double s1 = 1.0, s2 = 1.0, s1p = 0.0, s2p = 0.0;
        const double v = a1 - f.seg_hc[j];
        if (a1 < 37.5 && a2 > -37.5 && fabs(v) <= 300.0) {
            // Both edges active: one exponential and one division for the
            // pair.  With c = k (x1 - x0), u = exp(a1 - c/2), K = exp(-c/2):
            // exp(-a1) = K / u and exp(a2) = K u, so
            //   s1 = u / (u + K),  s2 = 1 / (1 + K u),
            // both over the common denominator (u + K)(1 + K u), which stays
            // finite for |a1 - c/2|, c/2 <= 300.  Each sigmoid then carries
            // a few ulp instead of one.
            const double u = exp(v), K = f.seg_K[j];
            const double p1 = u + K, p2 = 1.0 + K * u;
            const double R = 1.0 / (p1 * p2);
            s1 = u * p2 * R;
            s2 = p1 * R;
            s1p = ks * s1 * (1.0 - s1);
            s2p = -ks * s2 * (1.0 - s2);
        } else {
            if (a1 < 37.5) {
                s1 = 1.0 / (1.0 + exp(-a1));
                s1p = ks * s1 * (1.0 - s1);
            }
            if (a2 > -37.5) {
                s2 = 1.0 / (1.0 + exp(a2));
                s2p = -ks * s2 * (1.0 - s2);
            }
        }
        const double y = f.seg_y[j];
        B0F += y * s1 * s2;
        B0Fp += y * (s1p * s2 + s1 * s2p);
    }
    Bz = B0r * B0F;
    Bfi = B0r * B0Fp * ir * zi;    // ir = 1 / ri to an ulp
    Br = (B0r_p * B0F - B0r * B0Fp * spiral_p) * zi;
}

// Bilinear lookup of the z-Taylor coefficients: int() truncation, index
// clamped to [0, n-2], weights not clamped (linear extrapolation).
// Node indices are 32-bit (the largest table offset, NX * NY * 12 values, is
// below 2^31): the truncation saturates outside the int range, where the
// clamp applies anyway, and a NaN coordinate truncates to node 0.
__device__ __forceinline__ int trunc_index(double q) { return __double2int_rz(q); }

// 32-byte read-only global loads (sm_100): four doubles, eight floats; the
// address must be 32-byte aligned
__device__ __forceinline__ void ldg_v4(const double *p, double t[4])
{
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(t[0]), "=d"(t[1]), "=d"(t[2]), "=d"(t[3]) : "l"(p));
}

__device__ __forceinline__ void ldg_v8(const float *p, float t[8])
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(t[0]), "=f"(t[1]), "=f"(t[2]), "=f"(t[3]), "=f"(t[4]), "=f"(t[5]), "=f"(t[6]), "=f"(t[7])
        : "l"(p));
}

template <int MAXO>
__device__ __forceinline__ void high_order_b64(const FieldK &f, double x, double y, double z,
                                               double &Bz, double &Bfi, double &Br, int &clamped)
{
    // cell index and weights from (x - x_min) times 1 / step: within an ulp
    // of the reference's quotient; where that moves the index across a node
    // line, the bilinear interpolant is continuous there, so the field
    // changes by rounding only
    const double qx = (x - f.r_min) * f.inv_r_step;
    const double qy = (y - f.fi_min) * f.inv_fi_step;
    const int nr = (int)f.r_size, nf = (int)f.fi_size;
    int i = trunc_index(qx);
    int j = trunc_index(qy);
    if (i < 0) { i = 0; ++clamped; }
    else if (i >= nr - 1) { i = nr - 2; ++clamped; }
    if (j < 0) { j = 0; ++clamped; }
    else if (j >= nf - 1) { j = nf - 2; ++clamped; }
    const double tx = qx - (double)i;
    const double ty = qy - (double)j;
    const double w00 = (1.0 - tx) * (1.0 - ty), w01 = (1.0 - tx) * ty;
    const double w10 = tx * (1.0 - ty), w11 = tx * ty;
    constexpr int NP = (3 * MAXO <= 4) ? 4 : ((3 * MAXO <= 8) ? 8 : 12);
    constexpr int NV = 3 * MAXO;
    const double *nd[4];
    nd[0] = f.nodes64 + (i * nf + j) * NP;    // (i, j)
    nd[1] = nd[0] + NP;                       // (i, j+1)
    nd[2] = nd[0] + nf * NP;                  // (i+1, j)
    nd[3] = nd[2] + NP;                       // (i+1, j+1)
    const double w[4] = {w00, w01, w10, w11};
    // accumulate node by node in the reference's order w00, w01, w10, w11;
    // a node (32, 64 or 96 B) is read in 32-byte loads: half the load
    // instructions of 16-byte pairs, and the L1 throughput they take is the
    // kernel's bound
    double acc[NV > 0 ? NV : 1];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int a = 0; a < NV; a += 4) {
            double t[4];
            ldg_v4(nd[k] + a, t);
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (a + b < NV) acc[a + b] = (k == 0) ? w[0] * t[b] : acc[a + b] + w[k] * t[b];
        }
    }
    const double z2 = z * z;
    double ze = z2, zo = ze * z;
#pragma unroll
    for (int n = 0; n < MAXO; ++n) {
        Bz += acc[3 * n] * ze;
        Bfi += acc[3 * n + 1] * zo;
        Br += acc[3 * n + 2] * zo;
        ze *= z2;
        zo *= z2;
    }
}

// bharmonics_kernel_1d (src/FFAG_Field.py:1541-1587) for one particle: the
// Bz sum of the field-error harmonics (rows m, amp, phase, rmin, rmax of the
// device table h) whose radial band holds r, fi the unwrapped azimuth; the
// caller adds it to Bz after the map as the reference does, Br and Bfi take
// nothing.  Compiled only into the kernel variants launched for a map with
// harmonics, so the others keep their registers.
__device__ __forceinline__ double harmonics_bz(const double *h, int n, double r, double fi)
{
    if (!(r > 0.0)) return 0.0;
    double b = 0.0;
    for (int k = 0; k < n; ++k) {
        const double *row = h + 5 * k;
        if (row[3] <= r && r <= row[4]) b += row[1] * cos(row[0] * fi + row[2]);
    }
    return b;
}

// One gap of emap_kernel: inside test on (x, y) = r (cos fi, sin fi).
__device__ __forceinline__ bool gap_inside(const RFK &rf, int g, double x, double y)
{
    if (x < rf.box[g][0] || x > rf.box[g][1] || y < rf.box[g][2] || y > rf.box[g][3]) return false;
    double prev = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double x0 = rf.poly_x[g][j], y0 = rf.poly_y[g][j];
        const double x1 = rf.poly_x[g][(j + 1) & 3], y1 = rf.poly_y[g][(j + 1) & 3];
        const double cross = (x1 - x0) * (y - y0) - (y1 - y0) * (x - x0);
        if (j == 0) prev = cross;
        else if (cross * prev < 0.0) return false;
    }
    return true;
}

__device__ __forceinline__ bool in_window(const RFK &rf, int g, double fi)
{
    double d = fi - rf.win_center[g];
    d -= (2.0 * PI) * rint(d * (0.5 / PI));   // a flip of rint at a half turn leaves |d| ~ pi, outside
    return fabs(d) <= rf.win_half[g];
}

// Spiral gaps (interpolate_spiral_emap_unique_gap_kernel, src/FFAG_MathTools.py:
// 1042-1114, with shift_to_nearest_window :1118-1135 and
// Bilinear_interp_2D_vect_uniform_3fields :940-1039): the first gap whose
// window holds the particle, the bilinear map value, the RF factor.  The
// roundings are the reference's, one operation at a time (no contraction).
__device__ __forceinline__ double3 rf_spiral64(const RFK &rf, double acc, double r, double fi, double z, double rfph)
{
    const double tw = 2.0 * PI;
    int hit = -1;
    double phl = 0.0;
    for (int g = 0; g < rf.ngaps; ++g) {
        const double d = fi - rf.gap_az[g];
        const double k = rint((rf.sp_phic - d) / tw);
        const double l = __dadd_rn(d, __dmul_rn(k, tw));
        if (l >= rf.sp_phi0 && l <= rf.sp_phimax) {
            hit = g;
            phl = l;
            break;
        }
    }
    if (hit < 0) return make_double3(0.0, 0.0, 0.0);
    int i = (int)floor((r - rf.sp_r0) / rf.sp_dr);
    int j = (int)floor((phl - rf.sp_phi0) / rf.sp_dphi);
    i = i < 0 ? 0 : (i >= rf.sp_nr - 1 ? rf.sp_nr - 2 : i);
    j = j < 0 ? 0 : (j >= rf.sp_nphi - 1 ? rf.sp_nphi - 2 : j);
    const double tx = (r - __dadd_rn(rf.sp_r0, __dmul_rn((double)i, rf.sp_dr))) / rf.sp_dr;
    const double ty = (phl - __dadd_rn(rf.sp_phi0, __dmul_rn((double)j, rf.sp_dphi))) / rf.sp_dphi;
    const double w00 = (1.0 - tx) * (1.0 - ty), w01 = (1.0 - tx) * ty, w10 = tx * (1.0 - ty), w11 = tx * ty;
    // node (i, j): Er, Ez/z as one 16-byte load, Ephi in the next
    const double2 *nd = reinterpret_cast<const double2 *>(rf.sp);
    const int64_t b0 = 2 * ((int64_t)i * rf.sp_nphi + j), b1 = b0 + 2 * (int64_t)rf.sp_nphi;
    const double2 a00 = __ldg(nd + b0), a01 = __ldg(nd + b0 + 2), a10 = __ldg(nd + b1), a11 = __ldg(nd + b1 + 2);
    const double f00 = __ldg(rf.sp + 2 * b0 + 2), f01 = __ldg(rf.sp + 2 * b0 + 6);
    const double f10 = __ldg(rf.sp + 2 * b1 + 2), f11 = __ldg(rf.sp + 2 * b1 + 6);
    const double er = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(w00, a00.x), __dmul_rn(w01, a01.x)),
                                          __dmul_rn(w10, a10.x)), __dmul_rn(w11, a11.x));
    const double ez = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(w00, a00.y), __dmul_rn(w01, a01.y)),
                                          __dmul_rn(w10, a10.y)), __dmul_rn(w11, a11.y));
    const double ef = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(w00, f00), __dmul_rn(w01, f01)),
                                          __dmul_rn(w10, f10)), __dmul_rn(w11, f11));
    const double s = sin(rfph + rf.rf_shift[hit]);
    return make_double3((acc * er) * s, ((acc * ez) * z) * s, (acc * ef) * s);   // Er, Ez, Efi
}

// RF field (cylindrical r, z, fi components) times sin(RF phase +
// rf_shift[gap]).  Fixed gaps, reference semantics: every gap's emap_kernel
// call overwrites the field, so only the last gap contributes (no Ez);
// physical_sum adds all gaps.  Spiral gaps: rf_spiral64.
__device__ __forceinline__ void rf_field64(const RFK &rf, double acc, double r, double fi, double z, double rfph,
                                           double &Er, double &Ez, double &Efi)
{
    Er = 0.0;
    Ez = 0.0;
    Efi = 0.0;
    if (!rf.enable) return;
    if (rf.sp) {
        const double3 e = rf_spiral64(rf, acc, r, fi, z, rfph);
        Er = e.x;
        Ez = e.y;
        Efi = e.z;
        return;
    }
    const int g0 = rf.physical_sum ? 0 : rf.ngaps - 1;
    for (int g = g0; g < rf.ngaps; ++g) {
        if (!in_window(rf, g, fi)) continue;
        double sf, cf;
        sincos(fi, &sf, &cf);
        if (!gap_inside(rf, g, r * cf, r * sf)) continue;
        double sd, cd;
        sincos(rf.theta_n[g] - fi, &sd, &cd);
        const double s = sin(rfph + rf.rf_shift[g]);
        Er += (acc * cd) * s;
        Efi += (acc * sd) * s;
    }
}

// Azimuth change of one step and its sine / cosine, from the new position's
// unit vector in the local frame: sin and cos of the step angle are y / r and
// x / r (r^-1 is at hand from the drift); a step turns the particle by about
// 2 pi / (steps per turn), and for |sin| < 0.02 the angle is the arcsine series
//   asin(s) = s (1 + s^2/6 + 3 s^4/40 + 5 s^6/112 + 35 s^8/1152 + 63 s^10/2816)
// (truncation < 1e-22 relative): no division and no sin/cos series.
__device__ __forceinline__ void step_rotation(double y, double x, double ir, double &a, double &s, double &c)
{
    const double s0 = y * ir;
    if (x > 0.0 && fabs(s0) < 0.02) {
        const double s2 = s0 * s0;
        a = s0 * (1.0 + s2 * (1.0 / 6 + s2 * (3.0 / 40 + s2 * (5.0 / 112 + s2 * (35.0 / 1152 + s2 * (63.0 / 2816))))));
        s = s0;
        c = x * ir;
    } else {
        a = atan2(y, x);
        sincos(a, &s, &c);
    }
}

__device__ __forceinline__ void status_add(int64_t *status, int lost, int bad, int oob)
{
    if (!status) return;
    const unsigned mask = __activemask();
    for (int off = 16; off > 0; off >>= 1) {
        lost += __shfl_down_sync(mask, lost, off);
        bad += __shfl_down_sync(mask, bad, off);
        oob += __shfl_down_sync(mask, oob, off);
    }
    if ((threadIdx.x & 31) == __ffs(mask) - 1) {
        if (lost) atomicAdd((unsigned long long *)&status[FFA_STATUS_LOST], (unsigned long long)lost);
        if (bad) atomicAdd((unsigned long long *)&status[FFA_STATUS_NAN], (unsigned long long)bad);
        if (oob) atomicAdd((unsigned long long *)&status[FFA_STATUS_OUT_OF_MAP], (unsigned long long)oob);
    }
}

// Azimuth-crossing test of detect_azimuth_crossing (src/FFAG_MathTools.py:
// 1633-1695) on the step's pre / post azimuth, and the record append.  The
// reductions mod 2 pi are a - 2 pi floor(a / 2 pi) with no fused multiply-add,
// as in fast_mod_parallel (src/FFAG_MathTools.py:1554-1557); the target comes
// targets come in already reduced to [0, 2 pi).
__device__ __forceinline__ double mod_2pi(double a)
{
    const double tw = 2.0 * PI;
    return __dsub_rn(a, __dmul_rn(tw, floor(a / tw)));
}

// sin and cos of a small angle (|d| below a push step's azimuth advance, a
// few 1e-3 rad) by their Taylor series to d^9 / 9! and d^8 / 8!: truncation
// below 1e-22 for |d| < 0.02.
__device__ __forceinline__ void sincos_small(double d, double &s, double &c)
{
    const double d2 = d * d;
    s = d * (1.0 - d2 * (1.0 / 6 - d2 * (1.0 / 120 - d2 * (1.0 / 5040 - d2 * (1.0 / 362880)))));
    c = 1.0 - d2 * (0.5 - d2 * (1.0 / 24 - d2 * (1.0 / 720 - d2 * (1.0 / 40320))));
}

// One-turn-map sums at a crossing (the fit_sums form of ffa_crossing).  d0
// and d1: the step's start and end azimuth relative to the target (d0 <= 0
// <= d1, reduced mod 2 pi).
__device__ __forceinline__ void fit_accumulate(const ffa_crossing &xc, int64_t i, double dt, double d0, double d1,
                                               const double pre[7], const double post[7])
{
    // Cartesian state in the frame whose x axis points at the target azimuth
    double s0, c0, s1, c1;
    sincos_small(d0, s0, c0);
    sincos_small(d1, s1, c1);
    const double r0 = pre[0], vf0 = r0 * pre[5], r1 = post[0], vf1 = r1 * post[5];
    const double X0 = r0 * c0, Y0 = r0 * s0, VX0 = pre[1] * c0 - vf0 * s0, VY0 = pre[1] * s0 + vf0 * c0;
    const double X1 = r1 * c1, Y1 = r1 * s1, VX1 = post[1] * c1 - vf1 * s1, VY1 = post[1] * s1 + vf1 * c1;
    double tau = Y0 / (Y0 - Y1);
    for (int it = 0; it < 3; ++it) {
        const double t2 = tau * tau, t3 = t2 * tau;
        const double y = (2 * t3 - 3 * t2 + 1) * Y0 + (t3 - 2 * t2 + tau) * VY0 * dt + (3 * t2 - 2 * t3) * Y1 +
                         (t3 - t2) * VY1 * dt;
        const double dy = (6 * t2 - 6 * tau) * Y0 + (3 * t2 - 4 * tau + 1) * VY0 * dt + (6 * tau - 6 * t2) * Y1 +
                          (3 * t2 - 2 * tau) * VY1 * dt;
        tau = tau - y / dy;
    }
    const double t2 = tau * tau, t3 = t2 * tau;
    const double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + tau, h01 = 3 * t2 - 2 * t3, h11 = t3 - t2;
    const int k = xc.fit_instance[i];
    const double *ce = xc.fit_centre + 4 * k, *sc = xc.fit_scale + 4 * k;
    double u[4];
    u[0] = h00 * X0 + h10 * VX0 * dt + h01 * X1 + h11 * VX1 * dt;
    u[1] = VX0 + tau * (VX1 - VX0);
    u[2] = h00 * pre[2] + h10 * pre[3] * dt + h01 * post[2] + h11 * post[3] * dt;
    u[3] = pre[3] + tau * (post[3] - pre[3]);
    for (int c = 0; c < 4; ++c) u[c] = (u[c] - ce[c]) * sc[c];
    double *acc = xc.fit_sums + (int64_t)k * FFA_FIT_SUMS;
    double *w = xc.fit_last + 4 * i;
    if (xc.fit_has[i]) {
        for (int pl = 0; pl < 2; ++pl) {
            const double f0 = w[2 * pl], f1 = w[2 * pl + 1], a = u[2 * pl], b = u[2 * pl + 1];
            double *q = acc + 12 * pl;
            atomicAdd(q + 0, f0 * f0);
            atomicAdd(q + 1, f0 * f1);
            atomicAdd(q + 2, f0);
            atomicAdd(q + 3, f1 * f1);
            atomicAdd(q + 4, f1);
            atomicAdd(q + 5, 1.0);
            atomicAdd(q + 6, a * f0);
            atomicAdd(q + 7, a * f1);
            atomicAdd(q + 8, a);
            atomicAdd(q + 9, b * f0);
            atomicAdd(q + 10, b * f1);
            atomicAdd(q + 11, b);
        }
    }
    atomicAdd(acc + 24, 1.0);
    for (int c = 0; c < 4; ++c) w[c] = u[c];
    xc.fit_has[i] = 1;
}

__device__ __forceinline__ void xing_check(const ffa_crossing &xc, int64_t i, int64_t gs, const double pre[7],
                                           const double post[7], int surv_after, int inj, double esr, double esz,
                                           double esf, double dt)
{
    const double tw = 2.0 * PI;
    const double a = mod_2pi(pre[4]), b = mod_2pi(post[4]);
    for (int t = 0; t < xc.ntargets; ++t) {
        const double target = xc.target[t];
        bool hit;
        double ratio = 0.0;
        if (b >= a) {
            hit = a <= target && target <= b;
            if (hit && b - a > 1e-12) ratio = (target - a) / (b - a);
        } else {
            hit = (target >= a && target < tw) || (target >= 0 && target <= b);
            if (hit) {
                const double span = (b + tw) - a;
                if (span > 1e-12) ratio = ((target <= b ? target + tw : target) - a) / span;
            }
        }
        if (!hit) continue;
        if (xc.fit_sums) {
            double d0 = a - target, d1 = b - target;
            if (b < a) {
                if (target >= a) d1 += tw;
                else d0 -= tw;
            }
            fit_accumulate(xc, i, dt, d0, d1, pre, post);
            continue;
        }
        const unsigned long long k = atomicAdd((unsigned long long *)xc.count, 1ull);
        if ((int64_t)k >= xc.capacity) continue;
        double *rec = xc.buf + (int64_t)k * FFA_CROSSING_RECORD;
        rec[0] = (double)t;
        rec[1] = (double)i;
        rec[2] = (double)gs;
        rec[3] = ratio;
        for (int c = 0; c < 7; ++c) { rec[4 + c] = pre[c]; rec[11 + c] = post[c]; }
        rec[18] = (double)surv_after;
        rec[19] = (double)inj;
        rec[20] = esr; rec[21] = esz; rec[22] = esf;
    }
}

// Linear extrapolation of the space-charge field between updates
// (src/FFAG_track.py:449-478).
struct SCExtrap {
    bool pre = false, pp = false;
    double epr = 0, epz = 0, epf = 0, eqr = 0, eqz = 0, eqf = 0;
    __device__ void load(const ffa_state_soa &S, int64_t i)
    {
        pre = S.sc_pre[i] != 0;
        pp = S.sc_pp[i] != 0;
        if (pre) {
            epr = S.e_pre_r[i]; epz = S.e_pre_z[i]; epf = S.e_pre_fi[i];
            if (pp) { eqr = S.e_pp_r[i]; eqz = S.e_pp_z[i]; eqf = S.e_pp_fi[i]; }
        }
    }
    __device__ void apply(int64_t gs, int sc_step, double &esr, double &esz, double &esf) const
    {
        if (!pre) return;
        const double sf = gs >= sc_step ? (double)(gs % sc_step) / (double)sc_step : 0.0;
        if (pp) {
            esr = epr + sf * (epr - eqr);
            esz = epz + sf * (epz - eqz);
            esf = epf + sf * (epf - eqf);
        } else {
            esr = epr; esz = epz; esf = epf;
        }
    }
};

// ------------------------------------------------- field, float32 kernels
//
// The FP32C Boris pusher spends float32 arithmetic only where float64 is
// expensive: the exponentials of the fringe sigmoids and of the power law
// (expf / log1pf, accurately rounded library functions) and the bilinear
// lookup of the z-Taylor nodes (float32 table).  The constants these values
// are combined with, the products with r and z, and the whole Boris push stay
// float64, so float32 rounding enters the field as an error of relative size
// ~1e-7 that changes from step to step, never as a fixed scale error of the
// bending (a fixed bias of the bending shifts the revolution time and, with
// the RF on, the synchronous phase).
template <int MAXO>
__device__ __forceinline__ void field_mixed(const FieldK &f, double r, double ir, double fim, double z,
                                            double &Bz, double &Br, double &Bfi, int &clamped)
{
    // the table lookup first, so its loads are in flight during the rest
    double hz = 0.0, hf = 0.0, hr = 0.0;
    if constexpr (MAXO >= 1) {
        const double qx = (r - f.r_min) * f.inv_r_step;
        const double qy = (fim - f.fi_min) * f.inv_fi_step;
        const int nr = (int)f.r_size, nf = (int)f.fi_size;
        int i = trunc_index(qx), jj = trunc_index(qy);
        if (i < 0) { i = 0; ++clamped; } else if (i >= nr - 1) { i = nr - 2; ++clamped; }
        if (jj < 0) { jj = 0; ++clamped; } else if (jj >= nf - 1) { jj = nf - 2; ++clamped; }
        const float tx = (float)(qx - (double)i), ty = (float)(qy - (double)jj);
        const float w[4] = {(1.0f - tx) * (1.0f - ty), (1.0f - tx) * ty, tx * (1.0f - ty), tx * ty};
        constexpr int NP = (3 * MAXO <= 4) ? 4 : ((3 * MAXO <= 8) ? 8 : 12);
        constexpr int NV = 3 * MAXO;
        const float *nd[4];
        nd[0] = f.nodes32 + (i * nf + jj) * NP;
        nd[1] = nd[0] + NP;
        nd[2] = nd[0] + nf * NP;
        nd[3] = nd[2] + NP;
        float acc[NV];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if constexpr (NP == 8) {   // 32-byte nodes: one 32-byte load each
                float tv[8];
                ldg_v8(nd[k], tv);
#pragma unroll
                for (int b = 0; b < NV; ++b) acc[b] = (k == 0) ? w[0] * tv[b] : acc[b] + w[k] * tv[b];
            } else {
#pragma unroll
                for (int a = 0; a < NV; a += 4) {
                    const float4 t = __ldg(reinterpret_cast<const float4 *>(nd[k] + a));
                    const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        if (a + b < NV) acc[a + b] = (k == 0) ? w[0] * tv[b] : acc[a + b] + w[k] * tv[b];
                }
            }
        }
        const double z2 = z * z;
        double ze = z2, zo = z2 * z;
#pragma unroll
        for (int n = 0; n < MAXO; ++n) {
            hz += (double)acc[3 * n] * ze;
            hf += (double)acc[3 * n + 1] * zo;
            hr += (double)acc[3 * n + 2] * zo;
            ze *= z2;
            zo *= z2;
        }
    }

    double spiral = 0.0, spiral_p = 0.0;
    if (!f.spiral_zero) {
        for (int a = 0; a < f.n_spoly; ++a) spiral = spiral * r + f.spoly[a];
        for (int a = 0; a < f.n_spolyp; ++a) spiral_p = spiral_p * r + f.spolyp[a];
    }
    double B0r, B0r_p;
    if (f.k == 0.0) {
        B0r = f.B0;
        B0r_p = 0.0;
    } else {
        // (r / r_ref)^(k-1) with r / r_ref = 1 + eps, eps formed in float64
        const float eps = (float)((r - f.r_ref) * f.inv_r_ref);
        const double g = (double)expf((float)(f.km1 * (double)log1pf(eps)));
        B0r_p = f.kc1 * g;
        B0r = f.c1 * g * r;
    }
    double fs = fim;
    if (!f.spiral_zero) {   // as in analytic_b64
        fs = fim - spiral;
        fs -= f.period * floor(fs * f.inv_period);
    }
    double F = 0.0, Fp = 0.0;
    for (int j = 0; j < f.n_seg; ++j) {
        const float a1 = (float)(f.seg_k[j] * (fs - f.seg_x0[j]));
        const float a2 = (float)(f.seg_k[j] * (fs - f.seg_x1[j]));
        // exponents capped at 80 so e stays finite: past it s < 2e-35, which
        // is 0 in every sum below, and e * s would otherwise be inf * 0.
        // Where a sigmoid is saturated at 1 (e < 4e-11) its exponential is
        // skipped and e taken as 0.
        float e1 = 0.0f, e2 = 0.0f;
        if (a1 < 24.0f) e1 = expf(fminf(-a1, 80.0f));
        if (a2 > -24.0f) e2 = expf(fminf(a2, 80.0f));
        const float s1 = __frcp_rn(1.0f + e1), s2 = __frcp_rn(1.0f + e2);
        const float ss = s1 * s2;
        // s1' s2 + s1 s2' = k s1 s2 ((1 - s1) - (1 - s2)) with 1 - s = e s:
        // no cancellation where a sigmoid saturates
        const float dd = e1 * s1 - e2 * s2;
        F += f.seg_y[j] * (double)ss;
        Fp += f.seg_yk[j] * (double)(ss * dd);
    }
    Bz = B0r * F + hz;
    Bfi = B0r * Fp * ir * z + hf;
    Br = (B0r_p * F - B0r * Fp * spiral_p) * z + hr;
}

// ------------------------------------------------------------ Boris fp64

// One-warp blocks, at most 80 registers.  The register file is split over
// the SM's four schedulers (16384 registers each): 80 x 32 = 2560 registers
// per warp gives 6 warps per scheduler, 24 per SM, 3552 on 148 SMs, so the
// 3125 warps of a 1e5-particle bunch are resident in one wave.  At 88
// registers it is 5 per scheduler (2960 warps): the last 165 warps then run
// all their steps as a second, nearly empty wave (measured: 5.09 ms per
// 720-step turn at 88 registers, 3.81 ms at 80).
constexpr int BORIS_TB = 32;

// NREG: the register cap.  80 is the default launch shape; the compensated
// float32 pusher without space charge is also built with 72, 64 and 56
// (more resident warps, more spills) for the launch-shape autotuner.  The
// cap changes register allocation only, not the arithmetic.
template <int MAXO, bool SC, bool XING, bool F32, int NREG = 80, bool HARM = false>
__global__ void __maxnreg__(NREG) boris_f64_kernel(const __grid_constant__ PushK p)
{
    const int64_t t_ = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t_ >= p.n) return;
    const int64_t i = p.st.order ? (int64_t)__ldg(p.st.order + t_) : t_;   // the particle this thread advances
    const FieldK &f = p.f;
    const ffa_state_soa &S = p.st;
    double r = S.r[i], rdot = S.vr[i], z = S.z[i], zdot = S.vz[i], fi = S.fi[i], fidot = S.f5[i];
    double rfph = S.rf[i];
    double esr = S.esc_r[i], esz = S.esc_z[i], esf = S.esc_fi[i];
    int inj = S.inj[i], surv = S.surv[i];
    const int32_t injs = S.inj_step ? S.inj_step[i] : -1;
    SCExtrap ex;
    if (SC) ex.load(S, i);
    const double m = p.cs.m0, dt = p.dt;
    const double hq = p.hq, hqm = p.hqm, inv_m = p.inv_m, inv_cc = p.inv_cc, inv_mmcc = p.inv_mmcc;
    double ir = 1.0 / r;                     // 1 / r, carried from the previous step
    int lost = 0, oob = 0;

    for (int s = 0; s < p.nsteps; ++s) {
        const int64_t gs = p.step0 + s;
        if (injs == gs) { inj = 1; surv = 1; }
        if (SC) ex.apply(gs, p.sc_step, esr, esz, esf);
        const double drf = __ldg(p.drf + gs);
        double pre[7];
        const int surv0 = surv;
        if constexpr (XING) {
            pre[0] = r; pre[1] = rdot; pre[2] = z; pre[3] = zdot; pre[4] = fi; pre[5] = fidot; pre[6] = rfph;
        }
        if ((inj == 1) && (surv == 1)) {
            const double acc = __ldg(p.acc + gs);
            // fi mod the sector; a multiply by 1 / period instead of the
            // division can move floor() only where fi / period is within an
            // ulp of an integer, i.e. between two equal values of the
            // periodic field (0 and the period)
            const double fim = fi - f.period * floor(fi * f.inv_period);
            double Bz, Br, Bfi;
            if constexpr (F32) {
                field_mixed<MAXO>(f, r, ir, fim, z, Bz, Br, Bfi, oob);
            } else {
                // the table lookup first: its loads are in flight while the
                // analytic part computes (measured 3.53 vs 3.64 ms per
                // 1e5-particle turn; 3.30 ms with the zero-spiral skip)
                double hz = 0.0, hf = 0.0, hr = 0.0;
                if constexpr (MAXO >= 1) high_order_b64<MAXO>(f, r, fim, z, hz, hf, hr, oob);
                analytic_b64(f, r, ir, fim, z, Bz, Br, Bfi);
                Bz += hz;
                Bfi += hf;
                Br += hr;
            }
            if constexpr (HARM) Bz += harmonics_bz(f.harm, f.n_harm, r, fi);
            double Er, Ez, Efi;
            rf_field64(p.rf, acc, r, fi, z, rfph, Er, Ez, Efi);
            Ez += esz;
            Er += esr;
            Efi += esf;
            if (p.ap.enable && (r > p.ap.rmax || r < p.ap.rmin || z > p.ap.zmax || z < p.ap.zmin)) {
                surv = 0;
                ++lost;
            }
            // local frame: x along r-hat, y along fi-hat; B enters negated
            const double vx = rdot, vy = r * fidot, vz = zdot;
            const double Bx = -Br, By = -Bfi, Bzc = -Bz;
            const double v2 = vx * vx + vy * vy + vz * vz;
            const double gamma = rsqrt(1 - v2 * inv_cc);
            double px = gamma * m * vx, py = gamma * m * vy, pz = gamma * m * vz;
            px += hq * Er;
            py += hq * Efi;
            pz += hq * Ez;
            const double p2 = px * px + py * py + pz * pz;
            const double cb = hqm * rsqrt(1 + p2 * inv_mmcc);
            const double tx = cb * Bx, ty = cb * By, tz = cb * Bzc;
            const double pxp = px + (py * tz - pz * ty);
            const double pyp = py + (pz * tx - px * tz);
            const double pzp = pz + (px * ty - py * tx);
            const double t2 = tx * tx + ty * ty + tz * tz;
            const double sb = 2.0 / (1.0 + t2);
            const double sx = sb * tx, sy = sb * ty, sz = sb * tz;
            px += (pyp * sz - pzp * sy);
            py += (pzp * sx - pxp * sz);
            pz += (pxp * sy - pyp * sx);
            px += hq * Er;
            py += hq * Efi;
            pz += hq * Ez;
            const double p2n = px * px + py * py + pz * pz;
            const double igm = inv_m * rsqrt(1 + p2n * inv_mmcc);
            const double vxn = px * igm, vyn = py * igm, vzn = pz * igm;
            const double xn = r + vxn * dt, yn = vyn * dt;
            z = z + vzn * dt;
            zdot = vzn;
            const double rr2 = xn * xn + yn * yn;
            const double irn = rsqrt(rr2);
            const double rn = rr2 * irn;
            double dfi, sn, cn;
            step_rotation(yn, xn, irn, dfi, sn, cn);
            fi = fi + dfi;
            rdot = vxn * cn + vyn * sn;
            const double vfi = -vxn * sn + vyn * cn;
            fidot = rn > 1e-12 ? vfi * irn : 0.0;
            r = rn;
            ir = irn;
        } else {
            // skipped particle: the reference's Cartesian round trip
            double sinFi, cosFi;
            sincos(fi, &sinFi, &cosFi);
            const double x = r * cosFi, y = r * sinFi;
            const double vx = rdot * cosFi - r * fidot * sinFi;
            const double vy = rdot * sinFi + r * fidot * cosFi;
            const double rn = sqrt(x * x + y * y);
            rdot = vx * cosFi + vy * sinFi;
            const double vfi = -vx * sinFi + vy * cosFi;
            fidot = rn > 1e-12 ? vfi / rn : 0.0;
            r = rn;
            ir = 1.0 / rn;
        }
        rfph += drf;
        if constexpr (XING) {
            if (surv0 == 1) {
                const double post[7] = {r, rdot, z, zdot, fi, fidot, rfph};
                xing_check(p.xing, i, gs, pre, post, surv, inj, esr, esz, esf, p.dt);
            }
        }
    }
    S.r[i] = r; S.vr[i] = rdot; S.z[i] = z; S.vz[i] = zdot; S.fi[i] = fi; S.f5[i] = fidot;
    S.rf[i] = rfph;
    S.esc_r[i] = esr; S.esc_z[i] = esz; S.esc_fi[i] = esf;
    S.inj[i] = (uint8_t)inj;
    S.surv[i] = (uint8_t)surv;
    status_add(p.status, lost, !(isfinite(r) && isfinite(fi) && isfinite(z)), oob);
}

// ------------------------------------------------------ Boris, float32 push
//
// The float32 pusher: field and Boris update in float32, the positions (r,
// fi, z) and the RF phase accumulated in float64 from float32 increments.
// It carries the normalised momentum u = gamma v / c across the launch
// (float32) and converts from and to the float64 state once per launch.
// Each step the radius increment comes from
//   r' - r = (2 r dx + dx^2 + dy^2) / (r' + r)
// (dx, dy the local-frame displacement, formed in float32, so the increment
// keeps float32's relative accuracy instead of the radius), the azimuth
// increment from the arcsine series of dy / r'.  The RF gap test runs in
// float64 inside the gap's angular window.  Velocities keep float32
// precision: their rounding (~6e-8 of |u| per step) walks over a run, which
// is what limits this pusher's accuracy.  Not built with space charge,
// crossing capture of the steps' states is.

template <int MAXO>
__device__ __forceinline__ void field_f32(const FieldK &f, double r, double fim, float z, float &Bz, float &Br,
                                          float &Bfi, int &clamped)
{
    float hz = 0.0f, hf = 0.0f, hr = 0.0f;
    if constexpr (MAXO >= 1) {
        const double qx = (r - f.r_min) * f.inv_r_step;
        const double qy = (fim - f.fi_min) * f.inv_fi_step;
        const int nr = (int)f.r_size, nf = (int)f.fi_size;
        int i = trunc_index(qx), jj = trunc_index(qy);
        if (i < 0) { i = 0; ++clamped; } else if (i >= nr - 1) { i = nr - 2; ++clamped; }
        if (jj < 0) { jj = 0; ++clamped; } else if (jj >= nf - 1) { jj = nf - 2; ++clamped; }
        const float tx = (float)(qx - (double)i), ty = (float)(qy - (double)jj);
        const float w[4] = {(1.0f - tx) * (1.0f - ty), (1.0f - tx) * ty, tx * (1.0f - ty), tx * ty};
        constexpr int NP = (3 * MAXO <= 4) ? 4 : ((3 * MAXO <= 8) ? 8 : 12);
        constexpr int NV = 3 * MAXO;
        const float *nd[4];
        nd[0] = f.nodes32 + (i * nf + jj) * NP;
        nd[1] = nd[0] + NP;
        nd[2] = nd[0] + nf * NP;
        nd[3] = nd[2] + NP;
        float acc[NV];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if constexpr (NP == 8) {   // 32-byte nodes: one 32-byte load each
                float tv[8];
                ldg_v8(nd[k], tv);
#pragma unroll
                for (int b = 0; b < NV; ++b) acc[b] = (k == 0) ? w[0] * tv[b] : acc[b] + w[k] * tv[b];
            } else {
#pragma unroll
                for (int a = 0; a < NV; a += 4) {
                    const float4 t = __ldg(reinterpret_cast<const float4 *>(nd[k] + a));
                    const float tv[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        if (a + b < NV) acc[a + b] = (k == 0) ? w[0] * tv[b] : acc[a + b] + w[k] * tv[b];
                }
            }
        }
        const float z2 = z * z;
        float ze = z2, zo = z2 * z;
#pragma unroll
        for (int n = 0; n < MAXO; ++n) {
            hz += acc[3 * n] * ze;
            hf += acc[3 * n + 1] * zo;
            hr += acc[3 * n + 2] * zo;
            ze *= z2;
            zo *= z2;
        }
    }
    float spiral_p = 0.0f;
    double fs = fim;
    if (!f.spiral_zero) {   // as in analytic_b64, in float64 (spiral lattices only)
        double spiral = 0.0, sp = 0.0;
        for (int a = 0; a < f.n_spoly; ++a) spiral = spiral * r + f.spoly[a];
        for (int a = 0; a < f.n_spolyp; ++a) sp = sp * r + f.spolyp[a];
        spiral_p = (float)sp;
        fs = fim - spiral;
        fs -= f.period * floor(fs * f.inv_period);
    }
    const float rf = (float)r;
    float B0r, B0r_p;
    if (f.k == 0.0) {
        B0r = f.B0f;
        B0r_p = 0.0f;
    } else {
        const float eps = (float)((r - f.r_ref) * f.inv_r_ref);
        const float g = expf(f.km1f * log1pf(eps));
        B0r_p = f.kc1f * g;
        B0r = f.c1f * g * rf;
    }
    const float fsf = (float)fs;
    float F = 0.0f, Fp = 0.0f;
    for (int j = 0; j < f.n_seg; ++j) {
        const float a1 = f.seg_kf[j] * (fsf - f.seg_x0f[j]);
        const float a2 = f.seg_kf[j] * (fsf - f.seg_x1f[j]);
        float e1 = 0.0f, e2 = 0.0f;   // as in field_mixed
        if (a1 < 24.0f) e1 = expf(fminf(-a1, 80.0f));
        if (a2 > -24.0f) e2 = expf(fminf(a2, 80.0f));
        const float s1 = __frcp_rn(1.0f + e1), s2 = __frcp_rn(1.0f + e2);
        const float ss = s1 * s2;
        const float dd = e1 * s1 - e2 * s2;
        F += f.seg_yf[j] * ss;
        Fp += f.seg_ykf[j] * (ss * dd);
    }
    Bz = B0r * F + hz;
    Bfi = B0r * Fp * __frcp_rn(rf) * z + hf;
    Br = (B0r_p * F - B0r * Fp * spiral_p) * z + hr;
}

template <int MAXO, bool XING>
__global__ void __launch_bounds__(128) boris_f32_kernel(const __grid_constant__ PushK p)
{
    const int64_t t_ = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t_ >= p.n) return;
    const int64_t i = p.st.order ? (int64_t)__ldg(p.st.order + t_) : t_;   // the particle this thread advances
    const FieldK &f = p.f;
    const ffa_state_soa &S = p.st;
    const double c = p.cs.c;
    double r = S.r[i], z = S.z[i], fi = S.fi[i], rfph = S.rf[i];
    float ux, uy, uz;
    {
        const double vr = S.vr[i], vf = r * S.f5[i], vz = S.vz[i];
        const double g = 1.0 / sqrt(1.0 - (vr * vr + vf * vf + vz * vz) * p.inv_cc);
        ux = (float)(g * vr / c);
        uy = (float)(g * vf / c);
        uz = (float)(g * vz / c);
    }
    const double esr = S.esc_r[i], esz = S.esc_z[i], esf = S.esc_fi[i];
    int inj = S.inj[i], surv = S.surv[i];
    const int32_t injs = S.inj_step ? S.inj_step[i] : -1;
    const float aE = (float)(p.hq / (p.cs.m0 * c));   // q dt / (2 m c): E [V/m] -> du
    const float aB = (float)p.hqm;                     // q dt / (2 m): B [T] -> gamma t
    const float cdt = (float)(c * p.dt);
    const float esrf = (float)esr, eszf = (float)esz, esff = (float)esf;
    int lost = 0, oob = 0;
    // vr, vz and dfi/dt of the current momentum in float64 (crossing records)
    auto vstate = [&](double rr, double out[3]) {
        const double ig = 1.0 / sqrt(1.0 + (double)ux * ux + (double)uy * uy + (double)uz * uz);
        out[0] = (double)ux * ig * c;
        out[1] = (double)uz * ig * c;
        out[2] = (double)uy * ig * c / rr;
    };

    for (int s = 0; s < p.nsteps; ++s) {
        const int64_t gs = p.step0 + s;
        if (injs == gs) { inj = 1; surv = 1; }
        const double drf = __ldg(p.drf + gs);
        double pre[7];
        const int surv0 = surv;
        if constexpr (XING) {
            double v[3];
            vstate(r, v);
            pre[0] = r; pre[1] = v[0]; pre[2] = z; pre[3] = v[1]; pre[4] = fi; pre[5] = v[2]; pre[6] = rfph;
        }
        if ((inj == 1) && (surv == 1)) {
            const double acc = __ldg(p.acc + gs);
            const double fim = fi - f.period * floor(fi * f.inv_period);
            float Bz, Br, Bfi;
            field_f32<MAXO>(f, r, fim, (float)z, Bz, Br, Bfi, oob);
            double Erd, Ezd, Efid;
            rf_field64(p.rf, acc, r, fi, z, rfph, Erd, Ezd, Efid);
            const float Er = (float)Erd + esrf, Efi = (float)Efid + esff, Ez = (float)Ezd + eszf;
            if (p.ap.enable && (r > p.ap.rmax || r < p.ap.rmin || z > p.ap.zmax || z < p.ap.zmin)) {
                surv = 0;
                ++lost;
            }
            // local frame, B negated as in the float64 pusher
            const float Bx = -Br, By = -Bfi, Bzc = -Bz;
            ux += aE * Er;
            uy += aE * Efi;
            uz += aE * Ez;
            const float cb = aB * rsqrtf(1.0f + ux * ux + uy * uy + uz * uz);
            const float tx = cb * Bx, ty = cb * By, tz = cb * Bzc;
            const float upx = ux + (uy * tz - uz * ty);
            const float upy = uy + (uz * tx - ux * tz);
            const float upz = uz + (ux * ty - uy * tx);
            const float sb = 2.0f * __frcp_rn(1.0f + tx * tx + ty * ty + tz * tz);
            const float sx = sb * tx, sy = sb * ty, sz = sb * tz;
            ux += (upy * sz - upz * sy);
            uy += (upz * sx - upx * sz);
            uz += (upx * sy - upy * sx);
            ux += aE * Er;
            uy += aE * Efi;
            uz += aE * Ez;
            const float k = cdt * rsqrtf(1.0f + ux * ux + uy * uy + uz * uz);
            const float dx = ux * k, dy = uy * k, dz = uz * k;
            const float rf = (float)r;
            const float xn = rf + dx;
            const float rn2 = xn * xn + dy * dy;
            const float irn = rsqrtf(rn2);
            const float rn = rn2 * irn;
            const float dr = (2.0f * rf * dx + dx * dx + dy * dy) * __frcp_rn(rn + rf);
            const float sn = dy * irn, cn = xn * irn;
            const float s2 = sn * sn;
            const float dfi = sn * (1.0f + s2 * (1.0f / 6 + s2 * (3.0f / 40 + s2 * (5.0f / 112))));
            r += (double)dr;
            fi += (double)dfi;
            z += (double)dz;
            const float nux = ux * cn + uy * sn;
            uy = -ux * sn + uy * cn;
            ux = nux;
        }
        rfph += drf;
        if constexpr (XING) {
            if (surv0 == 1) {
                double v[3];
                vstate(r, v);
                const double post[7] = {r, v[0], z, v[1], fi, v[2], rfph};
                xing_check(p.xing, i, gs, pre, post, surv, inj, esr, esz, esf, p.dt);
            }
        }
    }
    const double ig = 1.0 / sqrt(1.0 + (double)ux * ux + (double)uy * uy + (double)uz * uz);
    S.r[i] = r; S.z[i] = z; S.fi[i] = fi; S.rf[i] = rfph;
    S.vr[i] = (double)ux * ig * c;
    S.vz[i] = (double)uz * ig * c;
    S.f5[i] = (double)uy * ig * c / r;
    S.inj[i] = (uint8_t)inj;
    S.surv[i] = (uint8_t)surv;
    status_add(p.status, lost, !(isfinite(r) && isfinite(fi) && isfinite(z)), oob);
}

// -------------------------------------------------------------- RK4 fp64

struct Y7 {
    double r, vr, z, vz, fi, E, rf;
};

// RK4_equations_of_motion_njit for one live particle at stage state y.
// F32: the field of the FP32C Boris pusher (field_mixed: float32 flutter
// exponentials and map lookup, float64 products with r and z); the
// equations of motion and the RK4 stages stay float64.
template <int MAXO, bool HARM, bool F32>
__device__ __forceinline__ void rk4_rhs64(const PushK &p, const Y7 &y, double rate, double acc,
                                          double esr, double esz, double esf, Y7 &d, int &oob)
{
    const FieldK &f = p.f;
    const double q = p.cs.q, c = p.cs.c, E0 = p.cs.E0;
    const double fim = y.fi - f.period * floor(y.fi / f.period);
    double Bz, Br, Bfi;
    if constexpr (F32) {
        field_mixed<MAXO>(f, y.r, 1.0 / y.r, fim, y.z, Bz, Br, Bfi, oob);
    } else {
        analytic_b64(f, y.r, 1.0 / y.r, fim, y.z, Bz, Br, Bfi);
        if constexpr (MAXO >= 1) high_order_b64<MAXO>(f, y.r, fim, y.z, Bz, Bfi, Br, oob);
    }
    if constexpr (HARM) Bz += harmonics_bz(f.harm, f.n_harm, y.r, y.fi);
    double Er, Ez, Efi;
    rf_field64(p.rf, acc, y.r, y.fi, y.z, y.rf, Er, Ez, Efi);
    Ez += esz;
    Er += esr;
    Efi += esf;
    const double ig = E0 / y.E;
    const double beta2 = 1.0 - ig * ig;
    const double v2 = beta2 * (c * c);
    const double vperp2 = v2 - y.vr * y.vr - y.vz * y.vz;
    const double fidot = sqrt(vperp2) / y.r;
    const double Edv = y.vr * Er + (y.r * fidot) * Efi + y.vz * Ez;
    const double qc2E = q * (c * c) / y.E;
    d.r = y.vr;
    d.vr = y.r * fidot * fidot + qc2E * (Er - y.r * fidot * Bz + y.vz * Bfi) - q * y.vr / y.E * Edv;
    d.z = y.vz;
    d.vz = qc2E * (Ez + y.r * fidot * Br - y.vr * Bfi) - q * y.vz / y.E * Edv;
    d.fi = fidot;
    d.E = q * Edv;
    d.rf = rate;
}

// One-warp blocks (RK4_TB), at most 80 registers (24 warps per SM, spills
// to L1): the 3125 warps of a 1e5-particle bunch are resident in one wave.
// Uncapped the kernel takes 130 registers, 12 warps per SM, 1.76 waves
// (measured on c1: 14.8 ms per 720-step turn uncapped; at 80 registers
// 12.4 ms in 128-thread blocks, 12.3 ms in 32-thread blocks; 11.3 ms with
// the stages as one loop, whose loop body the instruction cache holds).

template <int MAXO, bool SC, bool XING, bool HARM = false, bool F32 = false>
__global__ void __maxnreg__(80) rk4_f64_kernel(const __grid_constant__ PushK p)
{
    const int64_t t_ = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t_ >= p.n) return;
    const int64_t i = p.st.order ? (int64_t)__ldg(p.st.order + t_) : t_;   // the particle this thread advances
    const ffa_state_soa &S = p.st;
    Y7 y{S.r[i], S.vr[i], S.z[i], S.vz[i], S.fi[i], S.f5[i], S.rf[i]};
    double esr = S.esc_r[i], esz = S.esc_z[i], esf = S.esc_fi[i];
    int inj = S.inj[i], surv = S.surv[i];
    const int32_t injs = S.inj_step ? S.inj_step[i] : -1;
    SCExtrap ex;
    if (SC) ex.load(S, i);
    const double h = p.dt;
    int oob = 0;
    for (int s = 0; s < p.nsteps; ++s) {
        const int64_t gs = p.step0 + s;
        if (injs == gs) { inj = 1; surv = 1; }
        if (SC) ex.apply(gs, p.sc_step, esr, esz, esf);
        const double *rate = p.drf + 4 * gs;
        const double *acc = p.acc + 4 * gs;
        const double k1rf = h * __ldg(rate + 0), k2rf = h * __ldg(rate + 1);
        const double k3rf = h * __ldg(rate + 2), k4rf = h * __ldg(rate + 3);
        const double drf = (k1rf + 2 * k2rf + 2 * k3rf + k4rf) / 6;
        Y7 y0;
        if constexpr (XING) y0 = y;
        if (!((inj == 1) && (surv == 1))) {
            y.rf += drf;
            if constexpr (XING) {
                if (surv == 1) {
                    const double pre[7] = {y0.r, y0.vr, y0.z, y0.vz, y0.fi, y0.E, y0.rf};
                    const double post[7] = {y.r, y.vr, y.z, y.vz, y.fi, y.E, y.rf};
                    xing_check(p.xing, i, gs, pre, post, surv, inj, esr, esz, esf, p.dt);
                }
            }
            continue;
        }
        // the four stages as one loop, so the right-hand side is in the code
        // once: stage k is evaluated at y + a K(k-1) with a = 1/2, 1/2, 1, and
        // the increments are summed as K1 + 2 K2 + 2 K3 + K4, in that order
        Y7 d, K, S, ys = y;
#pragma unroll 1
        for (int k = 0; k < 4; ++k) {
            rk4_rhs64<MAXO, HARM, F32>(p, ys, __ldg(rate + k), __ldg(acc + k), esr, esz, esf, d, oob);
            K = {h * d.r, h * d.vr, h * d.z, h * d.vz, h * d.fi, h * d.E, h * d.rf};
            if (k == 0) {
                S = K;
            } else if (k < 3) {
                S = {S.r + 2 * K.r, S.vr + 2 * K.vr, S.z + 2 * K.z, S.vz + 2 * K.vz, S.fi + 2 * K.fi,
                     S.E + 2 * K.E, S.rf + 2 * K.rf};
            } else {
                S = {S.r + K.r, S.vr + K.vr, S.z + K.z, S.vz + K.vz, S.fi + K.fi, S.E + K.E, S.rf + K.rf};
            }
            const double a = k == 2 ? 1.0 : 0.5;
            ys = {y.r + a * K.r, y.vr + a * K.vr, y.z + a * K.z, y.vz + a * K.vz, y.fi + a * K.fi,
                  y.E + a * K.E, y.rf + a * K.rf};
        }
        y.r += S.r / 6;
        y.vr += S.vr / 6;
        y.z += S.z / 6;
        y.vz += S.vz / 6;
        y.fi += S.fi / 6;
        y.E += S.E / 6;
        y.rf += S.rf / 6;
        if constexpr (XING) {
            const double pre[7] = {y0.r, y0.vr, y0.z, y0.vz, y0.fi, y0.E, y0.rf};
            const double post[7] = {y.r, y.vr, y.z, y.vz, y.fi, y.E, y.rf};
            xing_check(p.xing, i, gs, pre, post, surv, inj, esr, esz, esf, p.dt);
        }
    }
    S.r[i] = y.r; S.vr[i] = y.vr; S.z[i] = y.z; S.vz[i] = y.vz; S.fi[i] = y.fi; S.f5[i] = y.E;
    S.rf[i] = y.rf;
    S.esc_r[i] = esr; S.esc_z[i] = esz; S.esc_fi[i] = esf;
    S.inj[i] = (uint8_t)inj;
    S.surv[i] = (uint8_t)surv;
    status_add(p.status, 0, !(isfinite(y.r) && isfinite(y.fi) && isfinite(y.z)), oob);
}

// ------------------------------------------------- closed-orbit tracks

// d/dtheta of (r, pr, z, pz) at fixed momentum P (FunctionForSEO,
// src/FFAG_track.py:1698-1740), same operation order.
__device__ __forceinline__ void seo_rhs(const FieldK &f, double t, const double x[4], double P, double q,
                                        double d[4])
{
    const double tw = 2.0 * PI;
    const double fi = fmod(t, tw);
    const double fim = fmod(fi, f.period);
    const double r = x[0], pr = x[1], z = x[2], pz = x[3];
    double Bz, Br, Bfi;
    analytic_b64(f, r, 1.0 / r, fim, z, Bz, Br, Bfi);
    const double pfi = sqrt(1.0 - pr * pr - pz * pz);
    const double qP = q / P;
    d[0] = r * pr / pfi;
    d[1] = pfi - qP * (r * Bz - r * pz / pfi * Bfi);
    d[2] = r * pz / pfi;
    d[3] = qP * (r * Br - r * pr / pfi * Bfi);
}

__global__ void __launch_bounds__(64) theta_track_kernel(const FieldK f, const ffa_theta_track_desc d)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.m) return;
    double x[4] = {d.x0[5 * i], d.x0[5 * i + 1], d.x0[5 * i + 2], d.x0[5 * i + 3]};
    const double P = d.x0[5 * i + 4], q = d.q;
    const double h = d.t_end / (double)(d.n_points - 1);
    const int nc = d.traj_cols;
    double *tr = d.traj ? d.traj + (int64_t)i * d.n_points * nc : nullptr;
    double t = 0.0;
    // row of point s: the state and, for 7 columns, the field there
    auto record = [&](int s, double ts) {
        double *row = tr + (int64_t)s * nc;
        row[0] = x[0];
        row[1] = x[1];
        if (nc == 7) {
            row[2] = x[2];
            row[3] = x[3];
            const double fim = fmod(fmod(ts, 2.0 * PI), f.period);
            analytic_b64(f, x[0], 1.0 / x[0], fim, x[2], row[4], row[5], row[6]);
        }
    };
    if (tr) record(0, 0.0);
    for (int s = 0; s < d.n_points - 1; ++s) {
        if (d.time_mode == 0) t = (double)s * h;
        double k1[4], k2[4], k3[4], k4[4], y[4], dd[4];
        seo_rhs(f, t, x, P, q, dd);
        for (int c = 0; c < 4; ++c) { k1[c] = h * dd[c]; y[c] = x[c] + 0.5 * k1[c]; }
        seo_rhs(f, t + 0.5 * h, y, P, q, dd);
        for (int c = 0; c < 4; ++c) { k2[c] = h * dd[c]; y[c] = x[c] + 0.5 * k2[c]; }
        seo_rhs(f, t + 0.5 * h, y, P, q, dd);
        for (int c = 0; c < 4; ++c) { k3[c] = h * dd[c]; y[c] = x[c] + k3[c]; }
        seo_rhs(f, t + h, y, P, q, dd);
        for (int c = 0; c < 4; ++c) {
            k4[c] = h * dd[c];
            x[c] = x[c] + (k1[c] + 2 * k2[c] + 2 * k3[c] + k4[c]) / 6;
        }
        if (d.time_mode != 0) t = t + h;
        if (tr) record(s + 1, d.time_mode != 0 ? t : (double)(s + 1) * h);
    }
    for (int c = 0; c < 4; ++c) d.x1[4 * i + c] = x[c];
}

cudaError_t launch_theta_track(const FieldK &f, const ffa_theta_track_desc &d, cudaStream_t s)
{
    theta_track_kernel<<<(unsigned)((d.m + 63) / 64), 64, 0, s>>>(f, d);
    return cudaGetLastError();
}

// ------------------------------------------------------------ node packing

__global__ void pack_nodes_kernel(const double *__restrict__ bz, const double *__restrict__ bfi,
                                  const double *__restrict__ br, int64_t plane, int max_order,
                                  int npad, double *__restrict__ n64, float *__restrict__ n32)
{
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= plane) return;
    for (int v = 0; v < npad; ++v) {
        double val = 0.0;
        const int n = v / 3 + 1, comp = v % 3;
        if (n <= max_order) {
            const double *src = comp == 0 ? bz : (comp == 1 ? bfi : br);
            val = src[(int64_t)n * plane + node];
        }
        n64[node * npad + v] = val;
        n32[node * npad + v] = (float)val;
    }
}

cudaError_t launch_pack_nodes(const ffa_field_desc &d, int npad, double *n64, float *n32, cudaStream_t s)
{
    const int64_t plane = d.r_size * d.fi_size;
    const int tb = 256;
    pack_nodes_kernel<<<(unsigned)((plane + tb - 1) / tb), tb, 0, s>>>(d.bz_stack, d.bfi_stack, d.br_stack,
                                                                        plane, d.max_order, npad, n64, n32);
    return cudaGetLastError();
}

// Field-error harmonics select their own kernel variants (HARM), so that
// the harmonic sum costs the common case nothing.
template <int MAXO, bool SC, bool F32>
static void boris_default(const PushK &p, cudaStream_t s, int tb)
{
    const unsigned g = (unsigned)((p.n + tb - 1) / tb);
    const bool x = xing_on(p);
    if (p.f.n_harm > 0) {
        if (x) boris_f64_kernel<MAXO, SC, true, F32, 80, true><<<g, tb, 0, s>>>(p);
        else boris_f64_kernel<MAXO, SC, false, F32, 80, true><<<g, tb, 0, s>>>(p);
    } else {
        if (x) boris_f64_kernel<MAXO, SC, true, F32><<<g, tb, 0, s>>>(p);
        else boris_f64_kernel<MAXO, SC, false, F32><<<g, tb, 0, s>>>(p);
    }
}

template <int MAXO, bool SC>
static void boris_launch(const PushK &p, cudaStream_t s, int tb, int)
{
    boris_default<MAXO, SC, false>(p, s, tb);
}

template <int MAXO, bool SC, bool F32>
static void rk4_launch_p(const PushK &p, cudaStream_t s)
{
    const int tb = RK4_TB;
    const unsigned g = (unsigned)((p.n + tb - 1) / tb);
    const bool x = xing_on(p);
    if (p.f.n_harm > 0) {
        if (x) rk4_f64_kernel<MAXO, SC, true, true, F32><<<g, tb, 0, s>>>(p);
        else rk4_f64_kernel<MAXO, SC, false, true, F32><<<g, tb, 0, s>>>(p);
    } else {
        if (x) rk4_f64_kernel<MAXO, SC, true, false, F32><<<g, tb, 0, s>>>(p);
        else rk4_f64_kernel<MAXO, SC, false, false, F32><<<g, tb, 0, s>>>(p);
    }
}

template <int MAXO, bool SC>
static void rk4_launch(const PushK &p, cudaStream_t s, bool f32)
{
    if (f32) rk4_launch_p<MAXO, SC, true>(p, s);
    else rk4_launch_p<MAXO, SC, false>(p, s);
}

#define FFA_DISPATCH(FN, p, ...)                                                       \
    do {                                                                               \
        const bool sc_ = (p).st.sc_pre != nullptr && (p).sc_step > 0;                  \
        switch ((p).f.max_order) {                                                     \
        case 0: sc_ ? FN<0, true>(p, __VA_ARGS__) : FN<0, false>(p, __VA_ARGS__); break; \
        case 1: sc_ ? FN<1, true>(p, __VA_ARGS__) : FN<1, false>(p, __VA_ARGS__); break; \
        case 2: sc_ ? FN<2, true>(p, __VA_ARGS__) : FN<2, false>(p, __VA_ARGS__); break; \
        case 3: sc_ ? FN<3, true>(p, __VA_ARGS__) : FN<3, false>(p, __VA_ARGS__); break; \
        default: sc_ ? FN<4, true>(p, __VA_ARGS__) : FN<4, false>(p, __VA_ARGS__); break; \
        }                                                                              \
    } while (0)

cudaError_t launch_boris_f64(const PushK &p, cudaStream_t s, int tb)
{
    FFA_DISPATCH(boris_launch, p, s, tb, 0);
    return cudaGetLastError();
}

cudaError_t launch_rk4_f64(const PushK &p, cudaStream_t s, bool f32)
{
    FFA_DISPATCH(rk4_launch, p, s, f32);
    return cudaGetLastError();
}

template <int MAXO, bool XING, int NREG>
static void boris32_shaped(const PushK &p, cudaStream_t s, int tb)
{
    boris_f64_kernel<MAXO, false, XING, true, NREG><<<(unsigned)((p.n + tb - 1) / tb), tb, 0, s>>>(p);
}

template <int MAXO, bool SC>
static void boris32_launch(const PushK &p, cudaStream_t s, int tb, int nreg_sel)
{
    if constexpr (!SC) {
        if (nreg_sel != 0) {   // the caller has checked: no space charge, no harmonics
            const bool x = xing_on(p);
            switch (nreg_sel) {
            case 1: x ? boris32_shaped<MAXO, true, 72>(p, s, tb) : boris32_shaped<MAXO, false, 72>(p, s, tb); break;
            case 2: x ? boris32_shaped<MAXO, true, 64>(p, s, tb) : boris32_shaped<MAXO, false, 64>(p, s, tb); break;
            default: x ? boris32_shaped<MAXO, true, 56>(p, s, tb) : boris32_shaped<MAXO, false, 56>(p, s, tb); break;
            }
            return;
        }
    }
    boris_default<MAXO, SC, true>(p, s, tb);
}

cudaError_t launch_boris_f32c(const PushK &p, cudaStream_t s, int tb, int nreg_sel)
{
    FFA_DISPATCH(boris32_launch, p, s, tb, nreg_sel);
    return cudaGetLastError();
}

template <int MAXO, bool SC>
static void boris_f32_launch(const PushK &p, cudaStream_t s, int tb, int)
{
    const unsigned g = (unsigned)((p.n + tb - 1) / tb);
    if (xing_on(p)) boris_f32_kernel<MAXO, true><<<g, tb, 0, s>>>(p);
    else boris_f32_kernel<MAXO, false><<<g, tb, 0, s>>>(p);
}

cudaError_t launch_boris_f32(const PushK &p, cudaStream_t s, int tb)
{
    switch (p.f.max_order) {
    case 0: boris_f32_launch<0, false>(p, s, tb, 0); break;
    case 1: boris_f32_launch<1, false>(p, s, tb, 0); break;
    case 2: boris_f32_launch<2, false>(p, s, tb, 0); break;
    case 3: boris_f32_launch<3, false>(p, s, tb, 0); break;
    default: boris_f32_launch<4, false>(p, s, tb, 0); break;
    }
    return cudaGetLastError();
}

// Resident blocks per SM of a push kernel (no space charge), from the runtime.
template <int MAXO, bool X>
static const void *push_kernel_fn(bool rk4, bool f32, int nreg_sel)
{
    if (rk4) return f32 ? (const void *)rk4_f64_kernel<MAXO, false, X, false, true>
                        : (const void *)rk4_f64_kernel<MAXO, false, X>;
    if (!f32) return (const void *)boris_f64_kernel<MAXO, false, X, false>;
    switch (nreg_sel) {
    case 0: return (const void *)boris_f64_kernel<MAXO, false, X, true, 80>;
    case 1: return (const void *)boris_f64_kernel<MAXO, false, X, true, 72>;
    case 2: return (const void *)boris_f64_kernel<MAXO, false, X, true, 64>;
    default: return (const void *)boris_f64_kernel<MAXO, false, X, true, 56>;
    }
}

cudaError_t push_occupancy(bool rk4, bool f32, int max_order, bool xing, int tb, int nreg_sel, int *blocks)
{
    const void *fn;
    switch (max_order) {
    case 0: fn = xing ? push_kernel_fn<0, true>(rk4, f32, nreg_sel) : push_kernel_fn<0, false>(rk4, f32, nreg_sel); break;
    case 1: fn = xing ? push_kernel_fn<1, true>(rk4, f32, nreg_sel) : push_kernel_fn<1, false>(rk4, f32, nreg_sel); break;
    case 2: fn = xing ? push_kernel_fn<2, true>(rk4, f32, nreg_sel) : push_kernel_fn<2, false>(rk4, f32, nreg_sel); break;
    case 3: fn = xing ? push_kernel_fn<3, true>(rk4, f32, nreg_sel) : push_kernel_fn<3, false>(rk4, f32, nreg_sel); break;
    default: fn = xing ? push_kernel_fn<4, true>(rk4, f32, nreg_sel) : push_kernel_fn<4, false>(rk4, f32, nreg_sel); break;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, fn, tb, 0);
}

}  // namespace ffa
