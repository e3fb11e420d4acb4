// ffa_bunch.cu -- seeded bunch generation on the GPU.
//
// One sub-bunch of GenerateInitDistributionDtInjNew
// (src/FFAG_Distribution.py:1152-1345) per call: every particle draws its
// normalised transverse and longitudinal coordinates from the distribution
// shapes of the reference (KV / water-bag / Gauss / hollow water-bag,
// src/FFAG_Distribution.py:76-1149), takes them through the Twiss
// transformation u = sqrt(beta eps) u_n, u' = sqrt(eps / beta) (u'_n -
// alpha u_n) (TwissContainer, :16-73), adds the injection point, and is
// written as one row of the reference's p-format matrix.
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011), a counter-based generator:
// the four 32-bit outputs are a bijection of the 128-bit counter under a
// 64-bit key, so particle i's draws depend only on (seed, sub-bunch, i,
// draw group) and a bunch is the same for any launch shape or split.
// Counter words: (i low, i high, draw group, sub-bunch); key: the seed.
// A uniform is (x + 1/2) 2^-32 from one 32-bit output, in (0, 1); normals
// come in Box-Muller pairs.  Rejection draws (Gauss cut-off, hollow shapes)
// try draw groups 2a, 2a + 1 for attempts a = 0 .. FFA_BUNCH_MAX_ATTEMPTS-1;
// a particle that never passes keeps its last attempt and is counted.
#include <math.h>

#include "ffa_internal.cuh"

namespace {

__host__ __device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint64_t key)
{
    uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        philox_round(c, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

struct Draw {
    int64_t i;
    uint32_t sub;
    uint64_t key;
    // four uniforms in (0, 1) of draw group g
    __device__ void uniforms(uint32_t g, double u[4]) const
    {
        uint32_t c[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), g, sub};
        philox4x32_10(c, key);
#pragma unroll
        for (int k = 0; k < 4; ++k) u[k] = ((double)c[k] + 0.5) * 2.3283064365386963e-10;
    }
};

// Box-Muller: two normals from two uniforms
__device__ __forceinline__ void box_muller(double u1, double u2, double &n1, double &n2)
{
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    n1 = rad * c;
    n2 = rad * s;
}

struct Twiss {
    double u_max, up_coeff, alpha;
    __device__ Twiss(const double t[3], double scale)
    {
        const double a = t[0], b = t[1], e = t[2] * scale;
        u_max = sqrt(b * e);
        up_coeff = sqrt(e / b);
        alpha = a;
    }
    __device__ void apply(double un, double upn, double &u, double &up) const
    {
        u = u_max * un;
        up = up_coeff * (upn - alpha * un);
    }
};

// KVDist1D: x = sin(2 pi (U - 1/2)), x' = +-sqrt(1 - x^2) (normalised)
__device__ __forceinline__ void kv1d(double ua, double ub, double &x, double &xp)
{
    x = sinpi(2.0 * (ua - 0.5));
    xp = (ub < 0.5 ? -1.0 : 1.0) * sqrt(1.0 - x * x);
}

// emittance factor each shape applies to the Twiss it is given
__device__ __forceinline__ double trans_scale(int type)
{
    switch (type) {
    case FFA_DIST_KV: return 4.0;          // KVDist2D: 100 % = 4 x rms
    case FFA_DIST_WATERBAG: return 6.0;    // WaterBagDist2D: KV2D of 6 / 4 x
    default: return 1.0;                   // Gauss; hollow: KV1D(e / 2) x 2
    }
}

__device__ __forceinline__ double long_scale(int type)
{
    switch (type) {
    case FFA_DIST_KV: return 2.0;          // KVDist1D: 100 % = 2 x rms
    case FFA_DIST_WATERBAG: return 4.0;    // WaterBagDist1D: KV1D of 2 x
    default: return 1.0;                   // Gauss, uniform-Gauss; hollow: KV1D(e / 2) x 2
    }
}

__global__ void __launch_bounds__(256) bunch_sample_kernel(const ffa_bunch_desc d, unsigned long long *rejected)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    Draw D{d.id0 + i, (uint32_t)d.sub_bunch, d.seed};
    const Twiss tx(d.twiss[0], trans_scale(d.transverse)), tz(d.twiss[1], trans_scale(d.transverse));
    const Twiss tl(d.twiss[2], long_scale(d.longitudinal));
    double xn = 0, xpn = 0, yn = 0, ypn = 0;
    int bad = 0;
    double u[4], w[4];
    switch (d.transverse) {
    case FFA_DIST_KV:
    case FFA_DIST_WATERBAG: {            // KVDist2D (+ water-bag radius g = U^(1/4))
        D.uniforms(0, u);
        const double rho = sqrt(u[1]);
        double s, c;
        sincospi(2.0 * (u[0] - 0.5), &s, &c);
        xn = rho * c;
        yn = rho * s;
        const double p0 = sqrt(fabs(1.0 - rho * rho));
        sincospi(2.0 * (u[2] - 0.5), &s, &c);
        xpn = p0 * c;
        ypn = p0 * s;
        if (d.transverse == FFA_DIST_WATERBAG) {
            const double g = sqrt(sqrt(u[3]));
            xn *= g; xpn *= g; yn *= g; ypn *= g;
        }
        break;
    }
    case FFA_DIST_HOLLOW_WATERBAG: {     // IndependentHollowWaterBagDist2D
        // per plane KV1D of e / 2 times g in U(0.4, 1); kept where
        // 0.3 <= (x / xm)^2 + (y / ym)^2 <= 1 (xm: the KV1D's u_max)
        bool ok = false;
        for (int a = 0; a < FFA_BUNCH_MAX_ATTEMPTS && !ok; ++a) {
            D.uniforms(2 * a, u);
            D.uniforms(2 * a + 1, w);
            double x1, x1p, y1, y1p;
            kv1d(u[0], u[1], x1, x1p);
            kv1d(u[2], u[3], y1, y1p);
            const double gx = 0.4 + 0.6 * w[0], gy = 0.4 + 0.6 * w[1];
            // in units of the KV1D's u_max the bound reads (gx x1)^2 + (gy y1)^2
            const double q = (gx * x1) * (gx * x1) + (gy * y1) * (gy * y1);
            xn = gx * x1; xpn = gx * x1p; yn = gy * y1; ypn = gy * y1p;
            ok = q >= 0.3 && q <= 1.0;
        }
        bad |= !ok;
        break;
    }
    default: {                           // GaussDist2D, optional cut-off per plane
        bool okx = false, oky = false;
        for (int a = 0; a < FFA_BUNCH_MAX_ATTEMPTS && !(okx && oky); ++a) {
            D.uniforms(2 * a, u);
            double n0, n1, n2, n3;
            box_muller(u[0], u[1], n0, n1);
            box_muller(u[2], u[3], n2, n3);
            const double c2 = d.cut_off * d.cut_off;
            if (!okx) {
                xn = n0; xpn = n1;
                okx = d.cut_off <= 0.0 || n0 * n0 + n1 * n1 <= c2;
            }
            if (!oky) {
                yn = n2; ypn = n3;
                oky = d.cut_off <= 0.0 || n2 * n2 + n3 * n3 <= c2;
            }
        }
        bad |= !(okx && oky);
    }
    }
    // hollow shapes draw KV1D of e / 2: in the reference's Twiss that is the
    // emittance the caller gave times 1/2, times the KV1D's 2 (trans_scale 1)
    double x, xp, y, yp;
    tx.apply(xn, xpn, x, xp);
    tz.apply(yn, ypn, y, yp);

    // longitudinal: (t, dE)
    double tn = 0, en = 0;
    switch (d.longitudinal) {
    case FFA_DIST_KV:
    case FFA_DIST_WATERBAG:
    case FFA_DIST_HOLLOW_WATERBAG: {
        D.uniforms(1u << 30, u);
        kv1d(u[0], u[1], tn, en);
        if (d.longitudinal == FFA_DIST_WATERBAG) {
            const double g = sqrt(u[2]);
            tn *= g; en *= g;
        } else if (d.longitudinal == FFA_DIST_HOLLOW_WATERBAG) {
            const double g = 0.4 + 0.6 * u[2];
            tn *= g; en *= g;
        }
        break;
    }
    case FFA_DIST_UNIFORM_GAUSS: {       // t uniform over the bunch length, dE normal
        D.uniforms(1u << 30, u);
        double n0, n1;
        box_muller(u[1], u[2], n0, n1);
        (void)n1;
        tn = u[0];
        en = n0;
        break;
    }
    default: {
        bool ok = false;
        for (int a = 0; a < FFA_BUNCH_MAX_ATTEMPTS && !ok; ++a) {
            D.uniforms((1u << 30) + a, u);
            box_muller(u[0], u[1], tn, en);
            ok = d.cut_off <= 0.0 || tn * tn + en * en <= d.cut_off * d.cut_off;
        }
        bad |= !ok;
    }
    }
    double t, dE;
    if (d.longitudinal == FFA_DIST_UNIFORM_GAUSS) {
        t = d.uniform_length * (tn - 0.5);
        dE = d.uniform_sigma * en;
    } else {
        tl.apply(tn, en, t, dE);
    }
    double *row = d.out + i * 16;
    row[0] = x + d.centre[0];
    row[1] = xp + d.centre[1];
    row[2] = y + d.centre[2];
    row[3] = yp + d.centre[3];
    row[4] = d.fi;
    row[5] = dE + d.centre[4];
    row[6] = t + d.centre[5];
#pragma unroll
    for (int c = 7; c < 13; ++c) row[c] = 0.0;
    row[13] = d.bunch_id;
    row[14] = (double)(d.id0 + i);
    row[15] = (double)(d.id0 + i);
    if (bad && rejected) atomicAdd(rejected, 1ull);
}

}  // namespace

extern "C" int ffa_bunch_sample(const ffa_bunch_desc *d, unsigned long long *rejected, void *stream)
{
    if (!d || d->n < 0 || d->id0 < 0 || (d->n > 0 && !d->out)) return FFA_ERR_INVALID;
    if (d->transverse < FFA_DIST_GAUSS || d->transverse > FFA_DIST_HOLLOW_WATERBAG) return FFA_ERR_INVALID;
    if (d->longitudinal < FFA_DIST_GAUSS || d->longitudinal > FFA_DIST_UNIFORM_GAUSS) return FFA_ERR_INVALID;
    for (int p = 0; p < 3; ++p)
        if (!(d->twiss[p][1] > 0.0) || !(d->twiss[p][2] >= 0.0)) return FFA_ERR_INVALID;
    if (d->n == 0) return FFA_OK;
    const int tb = 256;
    bunch_sample_kernel<<<(unsigned)((d->n + tb - 1) / tb), tb, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        *d, rejected);
    return cudaGetLastError() == cudaSuccess ? FFA_OK : FFA_ERR_CUDA;
}
