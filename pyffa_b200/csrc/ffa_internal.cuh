// ffa_internal.cuh -- shared device-side definitions of libffa_cuda.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/ffa_cuda.h"

#define FFA_CHECK_CUDA(call)                         \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return FFA_ERR_CUDA;  \
    } while (0)

namespace ffa {

constexpr double PI = 3.141592653589793;

// Kernel-side view of the field (analytic parameters precomputed once and the
// packed z-Taylor node table).  Node (i, j) of the r x fi grid holds, for
// n = 1..max_order, (bz_n, bfi_n, br_n), padded to `npad` values so a node is
// 32 B (float32) or 64 B (float64) aligned for max_order <= 2.
struct FieldK {
    int32_t nsectors, n_spoly, n_spolyp, n_seg, max_order, npad;
    double B0, k, km1, B0k;       // B0, k, k - 1, B0 * k
    double period;                // 2 pi / nsectors
    double inv_period;            // nsectors / (2 pi)
    double spoly[FFA_MAX_POLY];
    double spolyp[FFA_MAX_POLY];
    double seg_x0[FFA_MAX_SEG], seg_x1[FFA_MAX_SEG];
    double seg_k[FFA_MAX_SEG];    // 16 / W0
    double seg_y[FFA_MAX_SEG];    // y02 * |y01|
    double r_min, r_step, fi_min, fi_step;
    int64_t r_size, fi_size;
    const double *nodes64;
    const float *nodes32;
    // float32 field: B0 r^(k-1) = c1 * (1 + eps)^(k-1), eps = (r - r_ref) / r_ref
    int32_t spiral_zero;          // s(r) == 0: skip the spiral polynomials
    int32_t pad1;
    double r_ref, inv_r_ref, inv_r_step, inv_fi_step;
    double c1, kc1;               // B0 r_ref^(k-1), k * c1
    double seg_yk[FFA_MAX_SEG];   // seg_y * seg_k
    // paired sigmoids: half the edge-to-edge exponent c/2 = k (x1 - x0) / 2
    // (a huge value disables the pairing) and exp(-c/2)
    double seg_hc[FFA_MAX_SEG], seg_K[FFA_MAX_SEG];
    // power law near the map centre: r^(k-1) = r0^(k-1) (1 + t)^(k-1),
    // t = (r - r0) / r0, as a 16-term binomial series for |t| <= pw_tlim
    // (truncation below 2^-56 relative); pw_tlim = -1 disables it
    double pw_r0, pw_inv_r0, pw_tlim, pw_r0m;
    double pw_c[16];
    // field-error harmonics: Bz += sum_k amp cos(m fi + phase) over the n_harm
    // rows (m, amp, phase, rmin, rmax) of the device table `harm` with
    // rmin <= r <= rmax (fi unwrapped)
    int32_t n_harm, pad2;
    const double *harm;
    // float32 copies for the float32 pusher
    float B0f, c1f, kc1f, km1f;
    float seg_x0f[FFA_MAX_SEG], seg_x1f[FFA_MAX_SEG], seg_kf[FFA_MAX_SEG], seg_yf[FFA_MAX_SEG], seg_ykf[FFA_MAX_SEG];
};

struct RFK {
    int32_t enable, ngaps, physical_sum, pad0;
    double poly_x[FFA_MAX_GAPS][4];
    double poly_y[FFA_MAX_GAPS][4];
    double box[FFA_MAX_GAPS][4];
    double theta_n[FFA_MAX_GAPS];
    double rf_shift[FFA_MAX_GAPS];
    // Angular window of each gap rectangle as seen from the origin: every
    // point of the rectangle lies within win_half of win_center, so a
    // particle outside the window is outside the gap without the Cartesian
    // test (win_half = pi disables the shortcut).
    double win_center[FFA_MAX_GAPS];
    double win_half[FFA_MAX_GAPS];
    // spiral gaps (sp != NULL): the shared (r, phi) map, its axes, the
    // middle and end of the phi axis, and each gap's azimuth
    const double *sp;
    int32_t sp_nr, sp_nphi;
    double sp_r0, sp_dr, sp_phi0, sp_dphi, sp_phimax, sp_phic;
    double gap_az[FFA_MAX_GAPS];
};

struct PushK {
    FieldK f;
    RFK rf;
    ffa_aperture ap;
    ffa_consts cs;
    ffa_state_soa st;
    const double *drf;
    const double *acc;
    int64_t n, step0;
    int32_t nsteps, sc_step;
    double dt;
    int64_t *status;
    ffa_crossing xing;  // buf and fit_sums both NULL: no crossing capture
    // Boris constants, formed on the host so the kernel reads them from the
    // parameter bank instead of holding them in registers
    double hq;          // (0.5 dt) q
    double hqm;         // hq / m
    double inv_m;       // 1 / m
    double inv_cc;      // 1 / c^2
    double inv_mmcc;    // 1 / (m^2 c^2)
};

inline __host__ __device__ bool xing_on(const PushK &p)
{
    return p.xing.buf != nullptr || p.xing.fit_sums != nullptr;
}

}  // namespace ffa

struct ffa_fieldmap {
    ffa::FieldK k;
    double *nodes64;
    float *nodes32;
    double *harm;         // device, FFA_MAX_HARMONICS rows of 5
};

// Launchers implemented in ffa_push.cu
namespace ffa {
// tb: threads per block; nreg_sel: register cap 80, 72, 64, 56 (0..3)
cudaError_t launch_boris_f64(const PushK &p, cudaStream_t s, int tb);
// RK4 (f32: the FP32C field) in blocks of RK4_TB threads
constexpr int RK4_TB = 32;
cudaError_t launch_rk4_f64(const PushK &p, cudaStream_t s, bool f32);
cudaError_t launch_boris_f32c(const PushK &p, cudaStream_t s, int tb, int nreg_sel);
cudaError_t launch_boris_f32(const PushK &p, cudaStream_t s, int tb);
cudaError_t push_occupancy(bool rk4, bool f32, int max_order, bool xing, int tb, int nreg_sel, int *blocks);
cudaError_t launch_theta_track(const FieldK &f, const ffa_theta_track_desc &d, cudaStream_t s);
cudaError_t launch_pack_nodes(const ffa_field_desc &d, int npad, double *n64, float *n32, cudaStream_t s);
}  // namespace ffa
