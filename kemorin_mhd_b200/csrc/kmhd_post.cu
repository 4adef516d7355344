// kmhd_post.cu -- spectral post-processing after the forward transform: the
// divergence of a flux vector's spectra (the reference's u.grad(T) term is
// -div(u T), formed this way after sph_f_trans), the curl of u x B (the
// induction term) and the curl and divergence of the momentum forces.
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
__global__ void k_div_flux(long long J, int nr, const double* __restrict__ S, const double* __restrict__ dS,
                           double* __restrict__ out, const double* __restrict__ coef, const double* __restrict__ fin,
                           const double* __restrict__ fout) {
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
      d1s = bnd[0] * (fin ? fin[j] : 0.0) + bnd[1] * S[i + J] + bnd[2] * S[i + 2 * J];
    } else if (k == nr - 1) {
      d1s = bnd[5] * S[i - 2 * J] + bnd[4] * S[i - J] + bnd[3] * (fout ? fout[j] : 0.0);
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
// coef as k_div_flux, then ar1[nr] = 1/r and gl[J] = l.
__global__ void k_rot_vec(long long J, int nr, const double* __restrict__ S, const double* __restrict__ dS,
                          const double* __restrict__ T, double* __restrict__ pol, double* __restrict__ dpol,
                          double* __restrict__ tor, const double* __restrict__ coef, const RotBnd b) {
  const double* d1 = coef;
  const double* ar2 = coef + 3 * nr + 6;
  const double* g3 = ar2 + nr;
  const double* ar1 = g3 + J;
  const double* gl = ar1 + nr;
  const long long n = J * nr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / J);
    const long long j = i - (long long)k * J;
    const double t = T[i];
    double dp, tr;
    if (k == 0) {
      if (b.insulating_in) {
        dp = (gl[j] + 1.0) * ar1[0] * t;
        tr = 0.0;
      } else {
        const double d2s = b.s_in[0] * S[i] + b.s_in[1] * S[i + J];
        dp = b.t_in[0] * t + b.t_in[1] * T[i + J] + b.t_in[2] * T[i + 2 * J];
        tr = -(d2s - g3[j] * ar2[0] * S[i]);
      }
    } else if (k == nr - 1) {
      if (b.insulating_out) {
        dp = -gl[j] * ar1[k] * t;
        tr = 0.0;
      } else {
        const double d2s = b.s_out[1] * S[i - J] + b.s_out[0] * S[i];
        dp = b.t_out[2] * T[i - 2 * J] + b.t_out[1] * T[i - J] + b.t_out[0] * t;
        tr = -(d2s - g3[j] * ar2[k] * S[i]);
      }
    } else {
      const double d1d = d1[3 * k] * dS[i - J] + d1[3 * k + 1] * dS[i] + d1[3 * k + 2] * dS[i + J];
      dp = d1[3 * k] * T[i - J] + d1[3 * k + 1] * t + d1[3 * k + 2] * T[i + J];
      tr = -d1d + g3[j] * ar2[k] * S[i];
    }
    pol[i] = t;
    dpol[i] = dp;
    tor[i] = tr;
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

cudaError_t launch_div_flux(long long J, int nr, const double* S, const double* dS, double* out, const double* coef,
                            const double* fin, const double* fout, cudaStream_t s) {
  const long long n = J * nr;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long want = (n + 255) / 256;
  const int grid = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  if (grid <= 0) return cudaSuccess;
  k_div_flux<<<grid, 256, 0, s>>>(J, nr, S, dS, out, coef, fin, fout);
  return cudaGetLastError();
}

}  // namespace kmhd
