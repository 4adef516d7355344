// kmhd_internal.cuh -- shared device utilities and the per-instance plan.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/kmhd_sph.h"

namespace kmhd {

// ---------------------------------------------------------------------------
// Tile geometry shared by host and device.
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kRB = 4;        // radii per column block (one "quad" per field)
constexpr int kThBlk = 64;    // hemisphere latitudes per backward CTA
constexpr int kKC = 16;       // reduction chunk (l for bwd, theta for fwd)
constexpr int kLBlk = 32;     // l rows per parity per forward CTA
constexpr int kMaxVec = 5;    // vectors per field group
constexpr int kMaxScl = 2;    // scalars per field group
constexpr int kMaxProd = 16;
constexpr int kMaxFftFactors = 16;
constexpr int kSeedL = 32;    // degrees between on-the-fly recurrence seeds
constexpr int kWideCtasPerSm = 2;  // resident CTAs per SM of the wide-line FFT cycle (one grid scratch each)
constexpr long long kSelfTestSpinCap = 1ll << 16;  // bounded-wait rounds of the failure self-test

// Plan of one transform instance (device pointers + sizes).
struct Plan {
  int L, nth, nph, nr, nh, nh_pad, nr4, nrb;
  // radial window [r_lo, r_hi) of the cycle launches (0, nr: every radius);
  // r_lo is a multiple of 16, so the window covers whole radial blocks and
  // whole split-GEMM column tiles
  int r_lo, r_hi;
  long long J;
  int nvb, nsb, nvf, nsf, ncb, ncf;
  // tables
  const double* radius;   // [nr]
  const double* colat;    // [nth]
  const double* weight;   // [nth]
  const double* asin_t;   // [nth]
  const double* P;        // Ptab[m][p][kpad][nh_pad]
  const double* dP;
  const long long* poff;  // [(L+1)*2] element offset of (m,p) block in P/dP
  const int* kpad;        // [(L+1)*2]
  const int* jmap;        // [(L+1)][2][L+1] -> rj j, -1 if absent
  // P / dP generated inside the FP64 Legendre kernels (otf = 1) instead of
  // read from P / dP: per-order recurrence and dP coefficients, start values
  // and the forward kernel's block seeds (see pchain)
  int otf;
  const double* cos_t;      // [nh] cos(colat)
  const double2* pco;       // [(L+2)][L+1] (a_l, b_l) of order mo, l >= mo + 2
  const double2* dco;       // [(L+1)][L+1] (e, f): dP_l^m = (e P_l^{m-1} - f P_l^{m+1}) / 2
  const double2* pst;       // [(L+2)][nh_pad] (P_mo^mo, P_{mo+1}^mo)
  const double* pseed;      // [m][s][6][nh_pad] chain states before l = m + kSeedL s
  const long long* pseed_off;  // [L+1] first seed of order m
  int* err;               // device error word of the instance (KMHD_ERR_TIMEOUT from a bounded wait), or null
  // work buffers
  double* SB;             // packed backward spectra [m][p][kpad][nrb*ncolb_blk]
  const long long* sboff; // [(L+1)*2]
  double* rtm_b;          // [m][r][th][record of ncb (cos, sin) pairs, see rec_off, rtm_off]
  double* rtm_f;          // [m][r][th][record of ncf pairs]
  // FFT
  int nfac;
  int fac[kMaxFftFactors];
  const double2* twid;    // [nph] e^{+2 pi i k/nph}
  const int* digrev;      // [nph] frequency index of DIF output slot
  double2* fft_scratch;   // wide lines only: [fft_scratch_ctas][pairs][nph] grid of the line
  int fft_scratch_ctas;
  // products
  int nprod;
  int pkind[kMaxProd], pa[kMaxProd], pb[kMaxProd];
  double pcoef[kMaxProd];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Offset (in doubles) of component c's (cos, sin) pair inside an rtm record of
// one (m, theta, r): [theta/phi pairs of every vector: (th c, th s, ph c, ph s)]
// [r pairs of every vector] [scalar pairs].  The theta/phi block of a vector is
// one 32-byte sector, so tensor-core epilogues write whole sectors.
__host__ __device__ __forceinline__ int rec_off(int c, int nv) {
  if (c < 3 * nv) {
    const int v = c / 3, q = c % 3;
    return q == 0 ? 4 * nv + 2 * v : 4 * v + 2 * (q - 1);
  }
  return 6 * nv + 2 * (c - 3 * nv);
}

// Offset (in doubles) of the rtm record of (m, theta, r) holding nc (cos, sin)
// pairs: layout [m][r][theta][record], so the records of one (m, r) are
// contiguous over theta.
__host__ __device__ __forceinline__ long long rtm_off(const Plan& P, int m, int th, int r, int nc) {
  return (((long long)m * P.nr + r) * P.nth + th) * (2LL * nc);
}

// One step of the Schmidt recurrence of order mo at hemisphere latitude th:
// returns P_l^mo from the chain state (p1, p2) = (P_{l-1}^mo, P_{l-2}^mo) and
// advances it.  P_l^mo = 0 for l < mo (and mo < 0); l = mo, mo + 1 take the
// start values (the fixed-order closed forms times sin^mo, formed as the
// stored tables form them); above, P_l = a_l cos(theta) P_{l-1} - b_l P_{l-2},
// a_l = (2l - 1) / sqrt(l^2 - mo^2), b_l = sqrt((l-1)^2 - mo^2) / sqrt(l^2 - mo^2)
// (schmidt_legendre_m, CORE_src/spherical_harmonics/schmidt_fix_m.f90:86-140,
// with sin^mo carried in the recurrence instead of multiplied in afterwards).
__device__ __forceinline__ double pchain(double& p1, double& p2, const Plan& P, int mo, int l, double ct, int th,
                                        double2 ab) {
  double v;
  if (mo < 0 || l < mo) {
    v = 0.0;
  } else if (l <= mo + 1) {
    const double2 s = P.pst[(long long)mo * P.nh_pad + th];
    v = l == mo ? s.x : s.y;
  } else {
    v = fma(ab.x * ct, p1, -(ab.y * p2));
  }
  p2 = p1;
  p1 = v;
  return v;
}

// Coefficients of degree l for pgen_step: (a_l, b_l) of orders m - 1, m, m + 1
// and the dP factors (e, f); zero where a chain takes no recurrence step.
__device__ __forceinline__ double2 pgen_coef(const Plan& P, int m, int l, int q) {
  if (l > P.L) return make_double2(0.0, 0.0);
  if (q == 3) return __ldg(P.dco + (long long)m * (P.L + 1) + l);
  const int mo = m - 1 + q;
  if (mo < 0 || l < mo + 2) return make_double2(0.0, 0.0);
  return __ldg(P.pco + (long long)mo * (P.L + 1) + l);
}

// P_l^m and dP_l^m/dtheta at (l, th) from the three chains of orders m - 1,
// m, m + 1 (state st), as diff_schmidt_legendre_m
// (schmidt_fix_m.f90:143-175): dP = (e P^{m-1} - f P^{m+1}) / 2.  cf holds
// the four coefficient pairs of degree l (pgen_coef q = 0..3).
__device__ __forceinline__ void pgen_step(double (&st)[6], const Plan& P, int m, int l, double ct, int th,
                                          const double2* cf, double& p, double& dp) {
  const double pm = pchain(st[0], st[1], P, m - 1, l, ct, th, cf[0]);
  p = pchain(st[2], st[3], P, m, l, ct, th, cf[1]);
  const double pp = pchain(st[4], st[5], P, m + 1, l, ct, th, cf[2]);
  const double2 ef = cf[3];
  dp = 0.5 * (ef.x * pm - ef.y * pp);
}
// pgen_step for l >= m + 3, where every chain takes a plain recurrence step
// (order m - 1 < 0 has zero coefficients and state).
__device__ __forceinline__ void pgen_step_fast(double (&st)[6], double ct, const double2* cf, double& p, double& dp) {
  const double pm = fma(cf[0].x * ct, st[0], -(cf[0].y * st[1]));
  st[1] = st[0];
  st[0] = pm;
  p = fma(cf[1].x * ct, st[2], -(cf[1].y * st[3]));
  st[3] = st[2];
  st[2] = p;
  const double pp = fma(cf[2].x * ct, st[4], -(cf[2].y * st[5]));
  st[5] = st[4];
  st[4] = pp;
  dp = 0.5 * (cf[3].x * pm - cf[3].y * pp);
}
__device__ __forceinline__ void pgen_step(double (&st)[6], const Plan& P, int m, int l, double ct, int th,
                                          double& p, double& dp) {
  const double2 cf[4] = {pgen_coef(P, m, l, 0), pgen_coef(P, m, l, 1), pgen_coef(P, m, l, 2), pgen_coef(P, m, l, 3)};
  pgen_step(st, P, m, l, ct, th, cf, p, dp);
}

// Radial blocks (kRB radii each) of the window: first block and count.
__host__ __device__ __forceinline__ int win_rb0(const Plan& P) { return P.r_lo / kRB; }
__host__ __device__ __forceinline__ int win_nrb(const Plan& P) { return (P.r_hi + kRB - 1) / kRB - P.r_lo / kRB; }

__host__ __device__ __forceinline__ int kcount(int L, int m, int p) {
  // number of l in [m, L] with (l - m) % 2 == p
  return p == 0 ? (L - m) / 2 + 1 : (L - m + 1) / 2;
}

__host__ __device__ __forceinline__ double g7_of(int l, int m) {
  // sph_normalizations (CORE_src/spherical_harmonics/spherical_harmonics.f90:121-136)
  if (l == 0) return 1.0;
  if (m == 0) return (double)(2 * l + 1) / (double)(2 * l * (l + 1));
  return (double)(2 * l + 1) / (double)(4 * l * (l + 1));
}
__host__ __device__ __forceinline__ double g6_of(int l, int m) {
  if (l == 0 && m == 0) return 0.5;
  if (m == 0) return (double)(2 * l + 1) / 2.0;
  return (double)(2 * l + 1) / 4.0;
}
__host__ __device__ __forceinline__ double g3_of(int l) {
  // g(j,3) = l(l+1), overridden to 1/2 at l = 0 (schmidt_poly_on_rtm_grid.f90:109)
  return l == 0 ? 0.5 : (double)(l * (l + 1));
}

// Launchers (defined in the .cu files).
cudaError_t launch_tables(const Plan& p, double* colat, double* weight, double* asin_t,
                          double* P, double* dP, cudaStream_t s);
// Divergence of a flux vector's spectra (kmhd_post.cu): S, dS, out are one
// J*nr column each; coef = d1[3 nr], bnd[6], ar2[nr], g3[J]; fin / fout the
// fixed boundary values (null: zero).
cudaError_t launch_div_flux(long long J, int nr, const double* S, const double* dS, double* out, const double* coef,
                            const double* fin, const double* fout, cudaStream_t s, int flux_in = 0,
                            int flux_out = 0);
// Boundary rows of the spectral curl, per side: insulating (the magnetic
// field's condition), else d2S/dr2 = s[0] S(boundary) + s[1] S(neighbour) and
// dT/dr = t[0] T(boundary) + t[1] T(neighbour) + t[2] T(second neighbour).
struct RotBnd {
  int insulating_in, insulating_out;
  int qvac_in, qvac_out;  // pseudo-vacuum (radial field): dpol/dr = tor = 0
  // curl of a field (vorticity, current) rather than of a force: interior
  // rows take the 3-point second derivative of S instead of d(dS/dr)/dr
  int d2_interior;
  // insulating boundary of the current: the potential field's dS/dr =
  // (l+1) S / r (inner) or -l S / r (outer) folded into the second derivative
  // with the fixed-derivative coefficient cdr
  int ins_s_in, ins_s_out;
  double cdr_in, cdr_out;
  double s_in[2], t_in[3], s_out[2], t_out[3];
};
// Curl of a vector (kmhd_post.cu): input S, dS, T, output pol, dpol, tor (one
// J*nr column each); coef as launch_div_flux, then ar1[nr] = 1/r and gl[J] = l.
cudaError_t launch_rot_vec(long long J, int nr, const double* S, const double* dS, const double* T, double* pol,
                           double* dpol, double* tor, const double* coef, const RotBnd& b, cudaStream_t s);
// Curl of the Coriolis term (kmhd_post.cu): vel and vort point at the S
// columns of (S, dS/dr, T) triples with column stride ld; idx[4 J] coupled
// modes, cf[12 J] coefficients, radius[nr] on the device.
cudaError_t launch_rot_coriolis(long long J, int nr, const double* vel, const double* vort, long long ld,
                                double* pol, double* tor, const int* idx, const double* cf, const double* radius,
                                double coef_cor, cudaStream_t s);
// Backward transform at the poles (kmhd_post.cu): v rows r (north) and nr + r
// (south) for every radius, ncb columns with stride ldv (Cartesian vectors).
cudaError_t launch_b_trans_center(const Plan& p, const double* d_rj, long long ld, const int* cols, double* v,
                                  cudaStream_t s);
cudaError_t launch_b_trans_pole(const Plan& p, const double* d_rj, long long ld, const int* cols, double* v,
                                long long ldv, cudaStream_t s);
// Curl of the radial buoyancy (kmhd_post.cu); C null: one scalar.
cudaError_t launch_rot_buoyancy(long long J, int nr, const double* T, double coef_t, const double* C, double coef_c,
                                double* out, const double* radius, cudaStream_t s);
// Set-up of the on-the-fly tables (cos_t, pco, dco, pst, pseed of the plan).
cudaError_t launch_otf_tables(const Plan& p, double* cos_t, double2* pco, double2* dco, double2* pst,
                              double* pseed, const long long* pseed_off, cudaStream_t s);
// P / dP of order m as the on-the-fly kernels generate them, [l - m][nh] (device).
cudaError_t launch_otf_order(const Plan& p, int m, double* P, double* dP, cudaStream_t s);
cudaError_t launch_pack_b(const Plan& p, int nlc_max, const double* d_rj, long long ld,
                          const int* cols, int nv, int ns, cudaStream_t s);
cudaError_t launch_leg_bwd_f64(const Plan& p, cudaStream_t s);
// m_count: run orders m < m_count only (0 = all orders)
cudaError_t launch_leg_fwd_f64(const Plan& p, double* d_rj, long long ld, const int* cols,
                               cudaStream_t s, int m_count = 0);
cudaError_t launch_fft_cycle(const Plan& p, cudaStream_t s);
cudaError_t launch_fft_bwd_grid(const Plan& p, double* fld, cudaStream_t s);
// true when one (r, theta) line of every component fits in shared memory
bool fft_line_fits(const Plan& p);
// failure-path self-test of the FFT's bounded staging wait (kmhd_selftest_wait_timeout)
cudaError_t launch_selftest_fft_wait(int* err, cudaStream_t s);
cudaError_t launch_fft_fwd_grid(const Plan& p, const double* frc, cudaStream_t s);

}  // namespace kmhd
