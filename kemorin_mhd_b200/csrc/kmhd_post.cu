// kmhd_post.cu -- spectral post-processing after the forward transform: the
// divergence of a flux vector's spectra (the reference's u.grad(T) term is
// -div(u T), formed this way after sph_f_trans), the curl of u x B (the
// induction term), the curl and divergence of the momentum forces and the
// curl of the Coriolis term.
//
// Interior rows as cal_sph_nod_vect_div2 (MHD_src/sph_MHD/cal_sph_exp_rotation.f90:254-290),
// fixed-field boundary rows as cal_sph_div_flux_4_fix_in / _fix_out
// (MHD_src/sph_MHD/cal_sph_exp_fixed_scalar.f90:381-456); the FDM coefficients
// are built on the host (kmhd_sph.cu) as the reference builds them.
#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

// One thread per (j, k), j fastest.  coef: d1[3 nr] (offsets -1, 0, +1 of
// row k), bnd[6] (inner: nodes 0, 1, 2; outer: nodes nr-1, nr-2, nr-3),
// ar2[nr] = (1/r)^2, g3[J] = max(l(l+1), 1/2).
// flux_in / flux_out: that boundary has a fixed flux (cal_div_sph_in_fix_flux_2
// / cal_div_sph_out_fix_flux_2, cal_sph_exp_fixed_flux.f90:134-157, 253-276):
// the row takes the given flux in place of the one-sided derivative,
// div = (flux - dS/dr) max(g3, 1/2) / r^2; fin / fout then hold the flux.
__global__ void k_div_flux(long long J, int nr, const double* __restrict__ S, const double* __restrict__ dS,
                           double* __restrict__ out, const double* __restrict__ coef, const double* __restrict__ fin,
                           const double* __restrict__ fout, int flux_in, int flux_out) {
  const double* d1 = coef;
  const double* bnd = coef + 3 * nr;
  const double* ar2 = bnd + 6;
  const double* g3 = ar2 + nr;
  const long long n = J * nr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / J);
    const long long j = i - (long long)k * J;
    double d1s;
    if (k == 0) {
      d1s = flux_in ? (fin ? fin[j] : 0.0) : bnd[0] * (fin ? fin[j] : 0.0) + bnd[1] * S[i + J] + bnd[2] * S[i + 2 * J];
    } else if (k == nr - 1) {
      d1s = flux_out ? (fout ? fout[j] : 0.0)
                     : bnd[5] * S[i - 2 * J] + bnd[4] * S[i - J] + bnd[3] * (fout ? fout[j] : 0.0);
    } else {
      d1s = d1[3 * k] * S[i - J] + d1[3 * k + 1] * S[i] + d1[3 * k + 2] * S[i + J];
    }
    out[i] = (d1s - dS[i]) * g3[j] * ar2[k];
  }
}

// Curl of a vector (S, dS/dr, T) into (pol, dpol/dr, tor), one thread per
// (j, k).  Interior rows as cal_sph_nod_vect_w_div_rot2
// (MHD_src/sph_MHD/cal_sph_exp_rotation.f90:207-248).  Boundary rows per side:
// - insulating (curl of u x B): cal_sph_nod_icb_ins_vp_rot2 /
//   cal_sph_nod_cmb_ins_vp_rot2 (cal_sph_exp_nod_icb_ins.f90:135-160,
//   cal_sph_exp_nod_cmb_ins.f90:131-157), dpol = (l + 1) T / r or -l T / r, tor = 0;
// - velocity conditions (curl of a force, sel_bc_sph_vorticity,
//   select_exp_velocity_bc.f90:215-262): dpol = one-sided dT/dr, tor =
//   -(d2S/dr2 - g3 S / r^2) with RotBnd's coefficients (non-slip:
//   cal_sph_nod_icb_rigid_rot2 / cal_sph_nod_cmb_rigid_rot2, free slip:
//   cal_sph_nod_icb_free_rot2 / cal_sph_nod_cmb_free_rot2).
// coef as k_div_flux, then ar1[nr] = 1/r, gl[J] = l and d2[3 nr] (second
// derivative, offsets -1, 0, +1).
__global__ void k_rot_vec(long long J, int nr, const double* __restrict__ S, const double* __restrict__ dS,
                          const double* __restrict__ T, double* __restrict__ pol, double* __restrict__ dpol,
                          double* __restrict__ tor, const double* __restrict__ coef, const RotBnd b) {
  const double* d1 = coef;
  const double* ar2 = coef + 3 * nr + 6;
  const double* g3 = ar2 + nr;
  const double* ar1 = g3 + J;
  const double* gl = ar1 + nr;
  const double* d2 = gl + J;  // interior 3-point second derivative
  const long long n = J * nr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / J);
    const long long j = i - (long long)k * J;
    const double t = T[i];
    // g_sph_rj(j,3) = l(l+1), 0 at l = 0 (the rj copy has no l = 0 override;
    // the coefficient array holds max(l(l+1), 1/2) for the divergence)
    const double g3j = gl[j] > 0.0 ? g3[j] : 0.0;
    double dp, tr;
    if (k == 0) {
      if (b.qvac_in) {  // pseudo-vacuum (radial field): cal_sph_nod_icb_qvc_vp_rot2
        dp = 0.0;
        tr = 0.0;
      } else if (b.insulating_in) {
        dp = (gl[j] + 1.0) * ar1[0] * t;
        tr = 0.0;
      } else {
        const double s0 = b.ins_s_in ? (gl[j] + 1.0) * ar1[0] * b.cdr_in + b.s_in[0] : b.s_in[0];
        const double d2s = s0 * S[i] + b.s_in[1] * S[i + J];
        dp = b.t_in[0] * t + b.t_in[1] * T[i + J] + b.t_in[2] * T[i + 2 * J];
        tr = -(d2s - g3j * ar2[0] * S[i]);
      }
    } else if (k == nr - 1) {
      if (b.qvac_out) {  // cal_sph_nod_cmb_qvc_vp_rot2
        dp = 0.0;
        tr = 0.0;
      } else if (b.insulating_out) {
        dp = -gl[j] * ar1[k] * t;
        tr = 0.0;
      } else {
        const double s0 = b.ins_s_out ? b.s_out[0] - gl[j] * ar1[k] * b.cdr_out : b.s_out[0];
        const double d2s = b.s_out[1] * S[i - J] + s0 * S[i];
        dp = b.t_out[2] * T[i - 2 * J] + b.t_out[1] * T[i - J] + b.t_out[0] * t;
        tr = -(d2s - g3j * ar2[k] * S[i]);
      }
    } else {
      dp = d1[3 * k] * T[i - J] + d1[3 * k + 1] * t + d1[3 * k + 2] * T[i + J];
      if (b.d2_interior) {  // cal_sph_nod_vect_rot2 (cal_sph_exp_rotation.f90:157-203)
        const double d2s = d2[3 * k] * S[i - J] + d2[3 * k + 1] * S[i] + d2[3 * k + 2] * S[i + J];
        tr = -d2s + g3j * ar2[k] * S[i];
      } else {
        const double d1d = d1[3 * k] * dS[i - J] + d1[3 * k + 1] * dS[i] + d1[3 * k + 2] * dS[i + J];
        tr = -d1d + g3j * ar2[k] * S[i];
      }
    }
    pol[i] = t;
    dpol[i] = dp;
    tor[i] = tr;
  }
}

// Curl of the Coriolis term (pol, tor) from the velocity (vS, vdS, vT) and
// vorticity (wS, wdS, wT) spectra, unit z rotation (r^2/2, r, 1) times
// coef_cor, as sum_rot_coriolis_rlm_10
// (MHD_src/sph_MHD/sum_coriolis_terms_rlm.f90:94-189).  One thread per mode j
// over a range of radii, so the per-mode table -- coupled modes idx[4 j ..]
// = (l-1, m), (l+1, m), (l, -m) and cf[12 j ..] = sw(1,1), sw(2,1), sw(1,3),
// sw(1,2), sw(2,2), tw(1,1), tw(1,2), tw(1,3), tw(2,3), tw(1,4), tw(2,4),
// g_sph_rlm(j,3) -- is read once; every radius's loads and stores are
// coalesced over j (the coupled modes of consecutive j are consecutive).
__global__ void k_rot_coriolis(long long J, int nr, int kchunk, const double* __restrict__ vS,
                               const double* __restrict__ vdS, const double* __restrict__ wS,
                               const double* __restrict__ wdS, const double* __restrict__ wT,
                               double* __restrict__ pol, double* __restrict__ tor, const int* __restrict__ idx,
                               const double* __restrict__ cf, const double* __restrict__ radius, double coef_cor) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= J) return;
  const int4 q = reinterpret_cast<const int4*>(idx)[j];
  const double* c = cf + 12 * j;
  const double sw11 = c[0], sw21 = c[1], sw13 = c[2], sw12 = c[3], sw22 = c[4];
  const double tw11 = c[5], tw12 = c[6], tw13 = c[7], tw23 = c[8], tw14 = c[9], tw24 = c[10], g3 = c[11];
  const int k0 = blockIdx.y * kchunk, k1 = min(nr, k0 + kchunk);
  for (int k = k0; k < k1; ++k) {
    const long long o = (long long)k * J;
    const double r = radius[k], ar = 1.0 / r;
    const double w0 = 0.5 * r * r, w1 = r, w2 = 1.0;
    const double dvp1 = vdS[o + q.x], dvp2 = vdS[o + q.y];
    const double wp_l1 = wS[o + q.z];
    const double vp1 = vS[o + q.x], vp2 = vS[o + q.y];
    const double vp_l1 = vS[o + q.z];
    const double d2vp_l1 = ar * ar * g3 * vp_l1 - wT[o + q.z];
    const double wp1 = wS[o + q.x], wp2 = wS[o + q.y];
    const double dwp1 = wdS[o + q.x] - 2.0 * ar * wp1;
    const double dwp2 = wdS[o + q.y] - 2.0 * ar * wp2;
    const double rp = sw11 * w0 * dvp1 + sw21 * w0 * dvp2 + sw13 * w0 * wp_l1 + sw12 * w1 * vp1 + sw22 * w1 * vp2;
    const double rt = tw11 * w0 * d2vp_l1 - tw12 * w2 * vp_l1 + tw13 * w1 * wp1 + tw23 * w1 * wp2 + tw14 * w0 * dwp1 +
                      tw24 * w0 * dwp2;
    pol[o + j] = -coef_cor * rp * ar * ar;
    tor[o + j] = -coef_cor * rt * ar * ar;
  }
}

// Backward transform at the two poles of every radius, for grids with pole
// points: schmidt_b_trans_pole_vect / schmidt_b_trans_pole_scalar
// (PARALLEL_src/SPH_SHELL_src/schmidt_b_trans_at_pole.f90:88-289).  Only the
// orders 0 (scalars, the vectors' radial part) and +-1 (the horizontal part)
// are nonzero at a pole; the vector comes out in Cartesian components (x, y,
// z at the north pole; z = -radial at the south pole).  Pole values of the
// Schmidt functions in closed form: P_l^0 = 1 / (-1)^l, dP_l^1/dtheta =
// sqrt(l(l+1)/2) / (-1)^l sqrt(l(l+1)/2) (north / south).  One CTA per
// radius, one warp per field, lanes over l, warp sums.  v: rows r (north) and
// nr + r (south), column stride ldv.
__global__ void k_b_trans_pole(Plan P, const double* __restrict__ d_rj, long long ld, const int* __restrict__ cols,
                               double* __restrict__ v, long long ldv) {
  const int r = blockIdx.x, L = P.L;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const double ar = 1.0 / P.radius[r];
  const long long jr = P.J * (long long)r;
  auto jof = [&](int l, int m) {
    const int am = m < 0 ? -m : m;
    return (long long)P.jmap[((long long)am * 2 + (m < 0 ? 1 : 0)) * (L + 1) + l];
  };
  auto wsum = [](double x) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
  };
  for (int f = warp; f < P.nvb + P.nsb; f += nw) {
    if (f < P.nvb) {
      const double* S = d_rj + jr + ld * cols[f];
      const double* dS = S + ld;
      const double* T = S + 2 * ld;
      double zn = 0.0, zs = 0.0, xn = 0.0, yn = 0.0, xs = 0.0, ys = 0.0;
      for (int l = lane; l <= L; l += 32) {
        const double sgn = (l & 1) ? -1.0 : 1.0;
        const double g3 = l == 0 ? 0.5 : (double)l * (double)(l + 1);
        const double s0 = S[jof(l, 0)];
        zn += s0 * g3;
        zs -= s0 * sgn * g3;
        if (l >= 1) {
          const double dpn = sqrt(0.5 * (double)l * (double)(l + 1)), dps = sgn * dpn;
          const long long jm = jof(l, -1), jp = jof(l, 1);
          xn += T[jm] * dpn + dS[jp] * dpn;
          yn += dS[jm] * dpn - T[jp] * dpn;
          xs += T[jm] * dps - dS[jp] * dps;
          ys -= dS[jm] * dps + T[jp] * dps;
        }
      }
      zn = wsum(zn); zs = wsum(zs); xn = wsum(xn); yn = wsum(yn); xs = wsum(xs); ys = wsum(ys);
      if (lane == 0) {
        const int c = 3 * f;
        v[r + ldv * c] = xn * ar;
        v[r + ldv * (c + 1)] = yn * ar;
        v[r + ldv * (c + 2)] = zn * ar * ar;
        v[P.nr + r + ldv * c] = xs * ar;
        v[P.nr + r + ldv * (c + 1)] = ys * ar;
        v[P.nr + r + ldv * (c + 2)] = zs * ar * ar;
      }
    } else {
      const double* s = d_rj + jr + ld * cols[f];
      double sn = 0.0, ss = 0.0;
      for (int l = lane; l <= L; l += 32) {
        const double x = s[jof(l, 0)];
        sn += x;
        ss += (l & 1) ? -x : x;
      }
      sn = wsum(sn);
      ss = wsum(ss);
      if (lane == 0) {
        const int c = 3 * P.nvb + (f - P.nvb);
        v[r + ldv * c] = sn;
        v[P.nr + r + ldv * c] = ss;
      }
    }
  }
}

// Backward transform at the centre of a full-sphere grid (the node at r = 0
// of a mesh with a centre point): schmidt_b_trans_center_vect
// (PARALLEL_src/SPH_SHELL_src/schmidt_b_trans_at_center.f90:64-119).  From
// the poloidal column S of the innermost radius r_1 = radius[0]: component 3
// = 2 S(1, 0) / r_1^2, component 1 = -2 S(1, -1) / r_1^2, component 2 =
// -2 S(1, +1) / r_1^2 (orders -1 / +1 as the code assigns them; its header
// comment names the opposite pairing).  Scalars are left as they are
// (schmidt_b_trans_center_scalar assigns a value to itself).  Thread f: vector f.
__global__ void k_b_trans_center(Plan P, const double* __restrict__ d_rj, long long ld, const int* __restrict__ cols,
                                 double* __restrict__ v) {
  const int f = threadIdx.x;
  if (f >= P.nvb || P.L < 1) return;
  const int L = P.L;
  const double* S = d_rj + ld * cols[f];  // radius index 0: rows 0 .. J - 1
  const double ar = 1.0 / P.radius[0];
  const long long j0 = P.jmap[(0LL * 2 + 0) * (L + 1) + 1];
  const long long jp = P.jmap[(1LL * 2 + 0) * (L + 1) + 1];
  const long long jm = P.jmap[(1LL * 2 + 1) * (L + 1) + 1];
  v[3 * f + 0] = -2.0 * S[jm] * ar * ar;
  v[3 * f + 1] = -2.0 * S[jp] * ar * ar;
  v[3 * f + 2] = 2.0 * S[j0] * ar * ar;
}

// Curl of the radial buoyancy (toroidal part): out = coef_t T r, or
// (coef_t T + coef_c C) r with a second scalar (cal_rot_buoyancy_sph_MHD /
// cal_rot_double_buoyancy_sph_MHD, MHD_src/sph_MHD/cal_rot_buoyancies_sph_MHD.f90:106-165).
__global__ void k_rot_buoyancy(long long J, int nr, const double* __restrict__ T, double coef_t,
                               const double* __restrict__ C, double coef_c, double* __restrict__ out,
                               const double* __restrict__ radius) {
  const long long n = J * nr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / J);
    out[i] = C ? (coef_t * T[i] + coef_c * C[i]) * radius[k] : coef_t * T[i] * radius[k];
  }
}

}  // namespace

cudaError_t launch_rot_vec(long long J, int nr, const double* S, const double* dS, const double* T, double* pol,
                           double* dpol, double* tor, const double* coef, const RotBnd& b, cudaStream_t s) {
  const long long n = J * nr;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (n + 255) / 256;
  const int grid = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  if (grid <= 0) return cudaSuccess;
  k_rot_vec<<<grid, 256, 0, s>>>(J, nr, S, dS, T, pol, dpol, tor, coef, b);
  return cudaGetLastError();
}

cudaError_t launch_rot_buoyancy(long long J, int nr, const double* T, double coef_t, const double* C, double coef_c,
                                double* out, const double* radius, cudaStream_t s) {
  const long long n = J * nr;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (n + 255) / 256;
  const int grid = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  if (grid <= 0) return cudaSuccess;
  k_rot_buoyancy<<<grid, 256, 0, s>>>(J, nr, T, coef_t, C, coef_c, out, radius);
  return cudaGetLastError();
}

cudaError_t launch_b_trans_pole(const Plan& p, const double* d_rj, long long ld, const int* cols, double* v,
                                long long ldv, cudaStream_t s) {
  if (p.nr <= 0 || p.nvb + p.nsb == 0) return cudaSuccess;
  const int warps = p.nvb + p.nsb < 8 ? p.nvb + p.nsb : 8;
  k_b_trans_pole<<<p.nr, 32 * warps, 0, s>>>(p, d_rj, ld, cols, v, ldv);
  return cudaGetLastError();
}

cudaError_t launch_b_trans_center(const Plan& p, const double* d_rj, long long ld, const int* cols, double* v,
                                  cudaStream_t s) {
  if (p.nvb <= 0) return cudaSuccess;
  k_b_trans_center<<<1, 32 * ((p.nvb + 31) / 32), 0, s>>>(p, d_rj, ld, cols, v);
  return cudaGetLastError();
}

cudaError_t launch_rot_coriolis(long long J, int nr, const double* vel, const double* vort, long long ld,
                                double* pol, double* tor, const int* idx, const double* cf, const double* radius,
                                double coef_cor, cudaStream_t s) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long jb = (J + 255) / 256;
  if (jb <= 0 || nr <= 0) return cudaSuccess;
  // enough blocks for 8 per SM; each block walks a contiguous range of radii
  long long ks = (8LL * nsm + jb - 1) / jb;
  if (ks > nr) ks = nr;
  const int kchunk = (int)((nr + ks - 1) / ks);
  const int ky = (nr + kchunk - 1) / kchunk;
  k_rot_coriolis<<<dim3((unsigned)jb, (unsigned)ky), 256, 0, s>>>(J, nr, kchunk, vel, vel + ld, vort, vort + ld,
                                                                   vort + 2 * ld, pol, tor, idx, cf, radius,
                                                                   coef_cor);
  return cudaGetLastError();
}

cudaError_t launch_div_flux(long long J, int nr, const double* S, const double* dS, double* out, const double* coef,
                            const double* fin, const double* fout, cudaStream_t s, int flux_in, int flux_out) {
  const long long n = J * nr;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (n + 255) / 256;
  const int grid = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  if (grid <= 0) return cudaSuccess;
  k_div_flux<<<grid, 256, 0, s>>>(J, nr, S, dS, out, coef, fin, fout, flux_in, flux_out);
  return cudaGetLastError();
}

}  // namespace kmhd
