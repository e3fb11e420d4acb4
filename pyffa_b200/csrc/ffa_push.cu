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
// Expressions keep the reference's evaluation order; the compiler may fuse a
// multiply and an add into one FMA, which changes results by at most an ulp.
#include "ffa_internal.cuh"

namespace ffa {

// ----------------------------------------------------------- field (fp64)

__device__ __forceinline__ void analytic_b64(const FieldK &f, double ri, double fim, double zi,
                                             double &Bz, double &Br, double &Bfi)
{
    double spiral = 0.0, spiral_p = 0.0;
    for (int a = 0; a < f.n_spoly; ++a) spiral = spiral * ri + f.spoly[a];
    for (int a = 0; a < f.n_spolyp; ++a) spiral_p = spiral_p * ri + f.spolyp[a];
    double B0r, B0r_p;
    if (f.k == 0.0) {
        B0r = f.B0;
        B0r_p = 0.0;
    } else {
        // r^k = r^(k-1) * r: one pow instead of two.
        double pk1 = pow(ri, f.km1);
        B0r_p = f.B0k * pk1;
        B0r = f.B0 * (pk1 * ri);
    }
    double fs = fim - spiral;
    fs -= f.period * floor(fs / f.period);
    double B0F = 0.0, B0Fp = 0.0;
    for (int j = 0; j < f.n_seg; ++j) {
        double ks = f.seg_k[j];
        double s1 = 1.0 / (1.0 + exp(-ks * (fs - f.seg_x0[j])));
        double s2 = 1.0 / (1.0 + exp(ks * (fs - f.seg_x1[j])));
        double y = f.seg_y[j];
        B0F += y * s1 * s2;
        double s1p = ks * s1 * (1.0 - s1);
        double s2p = -ks * s2 * (1.0 - s2);
        B0Fp += y * (s1p * s2 + s1 * s2p);
    }
    Bz = B0r * B0F;
    Bfi = B0r * B0Fp / ri * zi;
    Br = (B0r_p * B0F - B0r * B0Fp * spiral_p) * zi;
}

// Bilinear lookup of the z-Taylor coefficients: int() truncation, index
// clamped to [0, n-2], weights not clamped (linear extrapolation).
__device__ __forceinline__ void high_order_b64(const FieldK &f, double x, double y, double z,
                                               double &Bz, double &Bfi, double &Br, bool &clamped)
{
    int64_t i = (int64_t)((x - f.r_min) / f.r_step);
    int64_t j = (int64_t)((y - f.fi_min) / f.fi_step);
    clamped = false;
    if (i < 0) { i = 0; clamped = true; }
    else if (i >= f.r_size - 1) { i = f.r_size - 2; clamped = true; }
    if (j < 0) { j = 0; clamped = true; }
    else if (j >= f.fi_size - 1) { j = f.fi_size - 2; clamped = true; }
    double tx = (x - (f.r_min + (double)i * f.r_step)) / f.r_step;
    double ty = (y - (f.fi_min + (double)j * f.fi_step)) / f.fi_step;
    double w00 = (1.0 - tx) * (1.0 - ty), w01 = (1.0 - tx) * ty;
    double w10 = tx * (1.0 - ty), w11 = tx * ty;
    const int np = f.npad;
    const double *n00 = f.nodes64 + (i * f.fi_size + j) * np;
    const double *n01 = n00 + np;
    const double *n10 = n00 + f.fi_size * np;
    const double *n11 = n10 + np;
    double z2 = z * z;
    double ze = z2, zo = ze * z;
#pragma unroll 1
    for (int n = 0; n < f.max_order; ++n) {
        int o = 3 * n;
        double bz = w00 * __ldg(n00 + o) + w01 * __ldg(n01 + o) + w10 * __ldg(n10 + o) + w11 * __ldg(n11 + o);
        double bf = w00 * __ldg(n00 + o + 1) + w01 * __ldg(n01 + o + 1) + w10 * __ldg(n10 + o + 1) + w11 * __ldg(n11 + o + 1);
        double br = w00 * __ldg(n00 + o + 2) + w01 * __ldg(n01 + o + 2) + w10 * __ldg(n10 + o + 2) + w11 * __ldg(n11 + o + 2);
        Bz += bz * ze;
        Bfi += bf * zo;
        Br += br * zo;
        ze *= z2;
        zo *= z2;
    }
}

// One gap of emap_kernel: inside test on (x, y) = r (cos fi, sin fi).
__device__ __forceinline__ bool gap_inside(const RFK &rf, int g, double x, double y)
{
    if (x < rf.box[g][0] || x > rf.box[g][1] || y < rf.box[g][2] || y > rf.box[g][3]) return false;
    double prev = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        double x0 = rf.poly_x[g][j], y0 = rf.poly_y[g][j];
        double x1 = rf.poly_x[g][(j + 1) & 3], y1 = rf.poly_y[g][(j + 1) & 3];
        double cross = (x1 - x0) * (y - y0) - (y1 - y0) * (x - x0);
        if (j == 0) prev = cross;
        else if (cross * prev < 0.0) return false;
    }
    return true;
}

// RF field in cylindrical components times sin(RF phase + rf_shift[gap]).
// Reference semantics: every gap's emap_kernel call overwrites the field, so
// only the last gap contributes; physical_sum adds all gaps.
__device__ __forceinline__ void rf_field64(const RFK &rf, double acc, double x, double y, double fi,
                                           double rfph, double &Er, double &Efi)
{
    Er = 0.0;
    Efi = 0.0;
    if (!rf.enable) return;
    int g0 = rf.physical_sum ? 0 : rf.ngaps - 1;
    for (int g = g0; g < rf.ngaps; ++g) {
        if (!gap_inside(rf, g, x, y)) continue;
        double sd, cd;
        sincos(rf.theta_n[g] - fi, &sd, &cd);
        double s = sin(rfph + rf.rf_shift[g]);
        Er += (acc * cd) * s;
        Efi += (acc * sd) * s;
    }
}

// ------------------------------------------------------------ Boris fp64

__global__ void __launch_bounds__(128) boris_f64_kernel(const PushK p)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const FieldK &f = p.f;
    const ffa_state_soa &S = p.st;
    double r = S.r[i], rdot = S.vr[i], z = S.z[i], zdot = S.vz[i], fi = S.fi[i], fidot = S.f5[i];
    double rfph = S.rf[i];
    double esr = S.esc_r[i], esz = S.esc_z[i], esf = S.esc_fi[i];
    int inj = S.inj[i], surv = S.surv[i];
    const int32_t injs = S.inj_step ? S.inj_step[i] : -1;
    const bool sc_on = p.sc_step > 0 && S.sc_pre != nullptr;
    bool pre = false, pp = false;
    double epr = 0, epz = 0, epf = 0, eqr = 0, eqz = 0, eqf = 0;
    if (sc_on) {
        pre = S.sc_pre[i] != 0;
        pp = S.sc_pp[i] != 0;
        if (pre) {
            epr = S.e_pre_r[i]; epz = S.e_pre_z[i]; epf = S.e_pre_fi[i];
            if (pp) { eqr = S.e_pp_r[i]; eqz = S.e_pp_z[i]; eqf = S.e_pp_fi[i]; }
        }
    }
    const double q = p.cs.q, c = p.cs.c, m = p.cs.m0, dt = p.dt;
    const double hq = 0.5 * dt * q;          // (0.5 * dt) * q
    const double mmcc = m * m * c * c;
    const double cc = c * c;
    int lost = 0, oob = 0;

    for (int s = 0; s < p.nsteps; ++s) {
        const int64_t gs = p.step0 + s;
        if (injs == gs) { inj = 1; surv = 1; }
        if (pre) {
            double sf = gs >= p.sc_step ? (double)(gs % p.sc_step) / (double)p.sc_step : 0.0;
            if (pp) {
                esr = epr + sf * (epr - eqr);
                esz = epz + sf * (epz - eqz);
                esf = epf + sf * (epf - eqf);
            } else {
                esr = epr; esz = epz; esf = epf;
            }
        }
        const double acc = __ldg(p.acc + gs), drf = __ldg(p.drf + gs);
        double sinFi, cosFi;
        sincos(fi, &sinFi, &cosFi);
        const double x = r * cosFi, y = r * sinFi;
        const double vx = rdot * cosFi - r * fidot * sinFi;
        const double vy = rdot * sinFi + r * fidot * cosFi;
        const bool alive = (inj == 1) && (surv == 1);
        if (alive) {
            const double fim = fi - f.period * floor(fi / f.period);
            double Bz, Br, Bfi;
            analytic_b64(f, r, fim, z, Bz, Br, Bfi);
            if (f.max_order >= 1) {
                bool cl;
                high_order_b64(f, r, fim, z, Bz, Bfi, Br, cl);
                oob += cl;
            }
            double Er, Efi;
            rf_field64(p.rf, acc, x, y, fi, rfph, Er, Efi);
            double Ez = 0.0;
            Ez += esz;
            Er += esr;
            Efi += esf;
            const double Ex = Er * cosFi - Efi * sinFi;
            const double Ey = Er * sinFi + Efi * cosFi;
            const double Bx = -(Br * cosFi - Bfi * sinFi);
            const double By = -(Br * sinFi + Bfi * cosFi);
            const double Bzc = -Bz;
            if (p.ap.enable && (r > p.ap.rmax || r < p.ap.rmin || z > p.ap.zmax || z < p.ap.zmin)) {
                surv = 0;
                ++lost;
            }
            const double vz = zdot;
            const double v2 = vx * vx + vy * vy + vz * vz;
            const double gamma = 1.0 / sqrt(1 - v2 / cc);
            double px = gamma * m * vx, py = gamma * m * vy, pz = gamma * m * vz;
            px += hq * Ex;
            py += hq * Ey;
            pz += hq * Ez;
            const double p2 = px * px + py * py + pz * pz;
            const double gm = sqrt(1 + p2 / mmcc);
            const double cb = hq / (gm * m);
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
            px += hq * Ex;
            py += hq * Ey;
            pz += hq * Ez;
            const double p2n = px * px + py * py + pz * pz;
            const double gmn = sqrt(1 + p2n / mmcc);
            const double vxn = px / (gmn * m), vyn = py / (gmn * m), vzn = pz / (gmn * m);
            const double xn = x + vxn * dt, yn = y + vyn * dt;
            z = z + vzn * dt;
            zdot = vzn;
            const double rn = sqrt(xn * xn + yn * yn);
            double dfi = atan2(yn, xn) - atan2(y, x);
            if (dfi > PI) dfi -= 2 * PI;
            else if (dfi < -PI) dfi += 2 * PI;
            fi = fi + dfi;
            double sn, cn;
            sincos(fi, &sn, &cn);
            rdot = vxn * cn + vyn * sn;
            const double vfi = -vxn * sn + vyn * cn;
            fidot = rn > 1e-12 ? vfi / rn : 0.0;
            r = rn;
        } else {
            // Skipped particles still take the reference's cylindrical ->
            // Cartesian -> cylindrical round trip (fi is unchanged exactly).
            const double rn = sqrt(x * x + y * y);
            rdot = vx * cosFi + vy * sinFi;
            const double vfi = -vx * sinFi + vy * cosFi;
            fidot = rn > 1e-12 ? vfi / rn : 0.0;
            r = rn;
        }
        rfph += drf;
    }
    S.r[i] = r; S.vr[i] = rdot; S.z[i] = z; S.vz[i] = zdot; S.fi[i] = fi; S.f5[i] = fidot;
    S.rf[i] = rfph;
    S.esc_r[i] = esr; S.esc_z[i] = esz; S.esc_fi[i] = esf;
    S.inj[i] = (uint8_t)inj;
    S.surv[i] = (uint8_t)surv;
    const bool bad = !(isfinite(r) && isfinite(fi) && isfinite(z));
    if (p.status) {
        // warp-aggregated status counters
        unsigned mask = __activemask();
        int l = lost, b = bad ? 1 : 0, o = oob;
        for (int off = 16; off > 0; off >>= 1) {
            l += __shfl_down_sync(mask, l, off);
            b += __shfl_down_sync(mask, b, off);
            o += __shfl_down_sync(mask, o, off);
        }
        if ((threadIdx.x & 31) == __ffs(mask) - 1) {
            if (l) atomicAdd((unsigned long long *)&p.status[FFA_STATUS_LOST], (unsigned long long)l);
            if (b) atomicAdd((unsigned long long *)&p.status[FFA_STATUS_NAN], (unsigned long long)b);
            if (o) atomicAdd((unsigned long long *)&p.status[FFA_STATUS_OUT_OF_MAP], (unsigned long long)o);
        }
    }
}

// -------------------------------------------------------------- RK4 fp64

struct Y7 {
    double r, vr, z, vz, fi, E, rf;
};

// RK4_equations_of_motion_njit for one live particle at stage state y.
__device__ __forceinline__ void rk4_rhs64(const PushK &p, const Y7 &y, double rate, double acc,
                                          double esr, double esz, double esf, Y7 &d, int &oob)
{
    const FieldK &f = p.f;
    const double q = p.cs.q, c = p.cs.c, E0 = p.cs.E0;
    const double fim = y.fi - f.period * floor(y.fi / f.period);
    double Bz, Br, Bfi;
    analytic_b64(f, y.r, fim, y.z, Bz, Br, Bfi);
    if (f.max_order >= 1) {
        bool cl;
        high_order_b64(f, y.r, fim, y.z, Bz, Bfi, Br, cl);
        oob += cl;
    }
    double Er = 0.0, Efi = 0.0;
    if (p.rf.enable) {
        double sf, cf;
        sincos(y.fi, &sf, &cf);
        rf_field64(p.rf, acc, y.r * cf, y.r * sf, y.fi, y.rf, Er, Efi);
    }
    double Ez = 0.0;
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

__global__ void __launch_bounds__(128) rk4_f64_kernel(const PushK p)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const ffa_state_soa &S = p.st;
    Y7 y{S.r[i], S.vr[i], S.z[i], S.vz[i], S.fi[i], S.f5[i], S.rf[i]};
    double esr = S.esc_r[i], esz = S.esc_z[i], esf = S.esc_fi[i];
    int inj = S.inj[i], surv = S.surv[i];
    const int32_t injs = S.inj_step ? S.inj_step[i] : -1;
    const bool sc_on = p.sc_step > 0 && S.sc_pre != nullptr;
    bool pre = false, pp = false;
    double epr = 0, epz = 0, epf = 0, eqr = 0, eqz = 0, eqf = 0;
    if (sc_on) {
        pre = S.sc_pre[i] != 0;
        pp = S.sc_pp[i] != 0;
        if (pre) {
            epr = S.e_pre_r[i]; epz = S.e_pre_z[i]; epf = S.e_pre_fi[i];
            if (pp) { eqr = S.e_pp_r[i]; eqz = S.e_pp_z[i]; eqf = S.e_pp_fi[i]; }
        }
    }
    const double h = p.dt;
    int oob = 0;
    for (int s = 0; s < p.nsteps; ++s) {
        const int64_t gs = p.step0 + s;
        if (injs == gs) { inj = 1; surv = 1; }
        if (pre) {
            double sf = gs >= p.sc_step ? (double)(gs % p.sc_step) / (double)p.sc_step : 0.0;
            if (pp) {
                esr = epr + sf * (epr - eqr);
                esz = epz + sf * (epz - eqz);
                esf = epf + sf * (epf - eqf);
            } else {
                esr = epr; esz = epz; esf = epf;
            }
        }
        const double *rate = p.drf + 4 * gs;
        const double *acc = p.acc + 4 * gs;
        const double k1rf = h * __ldg(rate + 0), k2rf = h * __ldg(rate + 1);
        const double k3rf = h * __ldg(rate + 2), k4rf = h * __ldg(rate + 3);
        const double drf = (k1rf + 2 * k2rf + 2 * k3rf + k4rf) / 6;
        if (!((inj == 1) && (surv == 1))) {
            y.rf += drf;
            continue;
        }
        Y7 d, k1, k2, k3, k4, ys;
        rk4_rhs64(p, y, __ldg(rate + 0), __ldg(acc + 0), esr, esz, esf, d, oob);
        k1 = {h * d.r, h * d.vr, h * d.z, h * d.vz, h * d.fi, h * d.E, h * d.rf};
        ys = {y.r + 0.5 * k1.r, y.vr + 0.5 * k1.vr, y.z + 0.5 * k1.z, y.vz + 0.5 * k1.vz,
              y.fi + 0.5 * k1.fi, y.E + 0.5 * k1.E, y.rf + 0.5 * k1.rf};
        rk4_rhs64(p, ys, __ldg(rate + 1), __ldg(acc + 1), esr, esz, esf, d, oob);
        k2 = {h * d.r, h * d.vr, h * d.z, h * d.vz, h * d.fi, h * d.E, h * d.rf};
        ys = {y.r + 0.5 * k2.r, y.vr + 0.5 * k2.vr, y.z + 0.5 * k2.z, y.vz + 0.5 * k2.vz,
              y.fi + 0.5 * k2.fi, y.E + 0.5 * k2.E, y.rf + 0.5 * k2.rf};
        rk4_rhs64(p, ys, __ldg(rate + 2), __ldg(acc + 2), esr, esz, esf, d, oob);
        k3 = {h * d.r, h * d.vr, h * d.z, h * d.vz, h * d.fi, h * d.E, h * d.rf};
        ys = {y.r + k3.r, y.vr + k3.vr, y.z + k3.z, y.vz + k3.vz, y.fi + k3.fi, y.E + k3.E, y.rf + k3.rf};
        rk4_rhs64(p, ys, __ldg(rate + 3), __ldg(acc + 3), esr, esz, esf, d, oob);
        k4 = {h * d.r, h * d.vr, h * d.z, h * d.vz, h * d.fi, h * d.E, h * d.rf};
        y.r += (k1.r + 2 * k2.r + 2 * k3.r + k4.r) / 6;
        y.vr += (k1.vr + 2 * k2.vr + 2 * k3.vr + k4.vr) / 6;
        y.z += (k1.z + 2 * k2.z + 2 * k3.z + k4.z) / 6;
        y.vz += (k1.vz + 2 * k2.vz + 2 * k3.vz + k4.vz) / 6;
        y.fi += (k1.fi + 2 * k2.fi + 2 * k3.fi + k4.fi) / 6;
        y.E += (k1.E + 2 * k2.E + 2 * k3.E + k4.E) / 6;
        y.rf += (k1.rf + 2 * k2.rf + 2 * k3.rf + k4.rf) / 6;
    }
    S.r[i] = y.r; S.vr[i] = y.vr; S.z[i] = y.z; S.vz[i] = y.vz; S.fi[i] = y.fi; S.f5[i] = y.E;
    S.rf[i] = y.rf;
    S.esc_r[i] = esr; S.esc_z[i] = esz; S.esc_fi[i] = esf;
    S.inj[i] = (uint8_t)inj;
    S.surv[i] = (uint8_t)surv;
    const int bad = !(isfinite(y.r) && isfinite(y.fi) && isfinite(y.z));
    if (p.status) {
        unsigned mask = __activemask();
        int b = bad, o = oob;
        for (int off = 16; off > 0; off >>= 1) {
            b += __shfl_down_sync(mask, b, off);
            o += __shfl_down_sync(mask, o, off);
        }
        if ((threadIdx.x & 31) == __ffs(mask) - 1) {
            if (b) atomicAdd((unsigned long long *)&p.status[FFA_STATUS_NAN], (unsigned long long)b);
            if (o) atomicAdd((unsigned long long *)&p.status[FFA_STATUS_OUT_OF_MAP], (unsigned long long)o);
        }
    }
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

cudaError_t launch_boris_f64(const PushK &p, cudaStream_t s)
{
    const int tb = 128;
    boris_f64_kernel<<<(unsigned)((p.n + tb - 1) / tb), tb, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_rk4_f64(const PushK &p, cudaStream_t s)
{
    const int tb = 128;
    rk4_f64_kernel<<<(unsigned)((p.n + tb - 1) / tb), tb, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace ffa
