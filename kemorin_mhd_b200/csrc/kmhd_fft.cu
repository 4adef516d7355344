// kmhd_fft.cu -- longitudinal real FFTs fused with the grid-space products.
//
// One CTA owns one (r, theta) line and keeps every component of it in shared
// memory: inverse FFT -> products -> forward FFT never touch HBM.
// Convention (t_sph_single_FFTW.F90 normalisation with the FFTPACK slot order of
// PARALLEL_src/SPH_SHELL_src/t_sph_FFTPACK5.f90:183-331):
//   x_j = a_0 + sum_{k>=1} (a_k cos(2 pi jk/N) + b_k sin(2 pi jk/N)),
//   a_0 = (1/N) sum x_j, a_k = (2/N) sum x_j cos, b_k = (2/N) sum x_j sin.
// Two real components are carried as one complex sequence z = x_a + i x_b.
// The inverse transform is an in-place mixed-radix decimation in frequency
// (natural spectrum in, digit-reversed grid out); the products are pointwise,
// so they run on the digit-reversed grid; the forward transform is the exact
// transpose (decimation in time, digit-reversed in, natural out).  No
// reordering pass is needed.
// Products: cal_cross_prod_w_coef_smp, cal_vec_scalar_prod_w_coef_smp,
// cal_dot_prod_w_coef_smp (CORE_src/BASE/cal_products_smp.f90) as called by
// nonlinear_terms_in_rtp (MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:64-128).
#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by (sign * i)
template <int SIGN>
__device__ __forceinline__ double2 mul_si(double2 a) {
  return SIGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// In-place R-point DFT, y_q = sum_r x_r e^{SIGN 2 pi i r q / R}.
template <int SIGN>
__device__ __forceinline__ void dft2(double2* x) {
  const double2 a = x[0], b = x[1];
  x[0] = cadd(a, b);
  x[1] = csub(a, b);
}
template <int SIGN>
__device__ __forceinline__ void dft4(double2* x) {
  const double2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
  const double2 c = cadd(x[1], x[3]), d = mul_si<SIGN>(csub(x[1], x[3]));
  x[0] = cadd(a, c);
  x[1] = cadd(b, d);
  x[2] = csub(a, c);
  x[3] = csub(b, d);
}
template <int SIGN>
__device__ __forceinline__ void dft3(double2* x) {
  const double s3 = 0.86602540378443864676 * (double)SIGN;
  const double2 t = cadd(x[1], x[2]);
  const double2 d = csub(x[1], x[2]);
  const double2 u = make_double2(-d.y * s3, d.x * s3);
  const double2 v = make_double2(x[0].x - 0.5 * t.x, x[0].y - 0.5 * t.y);
  x[0] = cadd(x[0], t);
  x[1] = cadd(v, u);
  x[2] = csub(v, u);
}
template <int SIGN>
__device__ __forceinline__ void dft5(double2* x) {
  // direct 5-point DFT with exact-ish constants
  const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
  const double s1 = 0.95105651629515357212 * (double)SIGN, s2 = 0.58778525229247312917 * (double)SIGN;
  const double2 a1 = cadd(x[1], x[4]), b1 = csub(x[1], x[4]);
  const double2 a2 = cadd(x[2], x[3]), b2 = csub(x[2], x[3]);
  const double2 x0 = x[0];
  const double2 t1 = make_double2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  const double2 t2 = make_double2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  const double2 u1 = make_double2(-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x);
  const double2 u2 = make_double2(-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x);
  x[0] = make_double2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
  x[1] = cadd(t1, u1);
  x[4] = csub(t1, u1);
  x[2] = cadd(t2, u2);
  x[3] = csub(t2, u2);
}
template <int SIGN>
__device__ __forceinline__ void dft8(double2* x) {
  // radix-8 = 2 x 4 with internal twiddles e^{SIGN i pi k/4}
  const double h = 0.70710678118654752440;
  double2 e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
  dft4<SIGN>(e);
  dft4<SIGN>(o);
  // o[k] *= e^{SIGN 2 pi i k / 8}
  o[1] = make_double2(h * (o[1].x - (double)SIGN * o[1].y), h * (o[1].y + (double)SIGN * o[1].x));
  o[2] = mul_si<SIGN>(o[2]);
  o[3] = make_double2(h * (-o[3].x - (double)SIGN * o[3].y), h * (-o[3].y + (double)SIGN * o[3].x));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[k] = cadd(e[k], o[k]);
    x[k + 4] = csub(e[k], o[k]);
  }
}

template <int SIGN>
__device__ __forceinline__ void dft_r(double2* x, int R) {
  switch (R) {
    case 2: dft2<SIGN>(x); break;
    case 3: dft3<SIGN>(x); break;
    case 4: dft4<SIGN>(x); break;
    case 5: dft5<SIGN>(x); break;
    default: dft8<SIGN>(x); break;
  }
}

// twiddle e^{SIGN 2 pi i idx / N} from the +sign table
template <int SIGN>
__device__ __forceinline__ double2 twd(const double2* tw, int idx) {
  const double2 w = tw[idx];
  return SIGN > 0 ? w : make_double2(w.x, -w.y);
}

// Inverse (+) DIF over all npair sequences z[p*N + .] in shared memory.
__device__ void fft_dif_plus(double2* z, int npair, int N, const Plan& P, const double2* tw) {
  int span = N;
  for (int f = 0; f < P.nfac; ++f) {
    const int R = P.fac[f];
    const int s = span / R;
    const int nbf = N / R;
    const int stw = N / span;
    for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
      const int pp = it / nbf;
      const int rem = it % nbf;
      const int j = rem % s;
      const int b = rem / s;
      double2* base = z + (long long)pp * N + b * span + j;
      double2 x[8];
      for (int r = 0; r < R; ++r) x[r] = base[r * s];
      dft_r<+1>(x, R);
      base[0] = x[0];
      for (int q = 1; q < R; ++q) base[q * s] = cmul(x[q], twd<+1>(tw, j * q * stw));
    }
    __syncthreads();
    span = s;
  }
}

// Forward (-) DIT, the transpose of fft_dif_plus.
__device__ void fft_dit_minus(double2* z, int npair, int N, const Plan& P, const double2* tw) {
  int spans[kMaxFftFactors];
  int span = N;
  for (int f = 0; f < P.nfac; ++f) {
    spans[f] = span;
    span /= P.fac[f];
  }
  for (int f = P.nfac - 1; f >= 0; --f) {
    const int R = P.fac[f];
    span = spans[f];
    const int s = span / R;
    const int nbf = N / R;
    const int stw = N / span;
    for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
      const int pp = it / nbf;
      const int rem = it % nbf;
      const int j = rem % s;
      const int b = rem / s;
      double2* base = z + (long long)pp * N + b * span + j;
      double2 x[8];
      x[0] = base[0];
      for (int q = 1; q < R; ++q) x[q] = cmul(base[q * s], twd<-1>(tw, j * q * stw));
      dft_r<-1>(x, R);
      for (int r = 0; r < R; ++r) base[r * s] = x[r];
    }
    __syncthreads();
  }
}

// Load the spectra of line (r, theta) from rtm [m][th][r][nc][2] into z.
__device__ void load_line_spectra(double2* z, int npair, const Plan& P, const double* rtm, int nc,
                                  int th, int r) {
  const int N = P.nph, L = P.L;
  // zero the band L < k < N-L
  for (int it = threadIdx.x; it < npair * (N - 2 * L - 1); it += blockDim.x) {
    const int pp = it / (N - 2 * L - 1);
    const int k = L + 1 + it % (N - 2 * L - 1);
    z[(long long)pp * N + k] = make_double2(0.0, 0.0);
  }
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  const double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  for (int it = threadIdx.x; it < (L + 1) * npair; it += blockDim.x) {
    const int m = it / npair, pp = it % npair;
    const double* rec = base + m * strideM + 4 * pp;
    const double a0 = rec[0], b0 = rec[1];
    double a1 = 0.0, b1 = 0.0;
    if (2 * pp + 1 < nc) {
      a1 = rec[2];
      b1 = rec[3];
    }
    double2* zp = z + (long long)pp * N;
    if (m == 0) {
      zp[0] = make_double2(a0, a1);
    } else {
      // X_c = (a_c - i b_c)/2 ; z = X_0 + i X_1 ; z[N-m] = conj(X_0) + i conj(X_1)
      zp[m] = make_double2(0.5 * a0 + 0.5 * b1, 0.5 * a1 - 0.5 * b0);
      zp[N - m] = make_double2(0.5 * a0 - 0.5 * b1, 0.5 * b0 + 0.5 * a1);
    }
  }
}

// Store (a_m, b_m), m <= L, of line (r, theta) from the natural-order forward
// spectra in z into rtm [m][th][r][nc][2].
__device__ void store_line_spectra(const double2* z, int npair, const Plan& P, double* rtm, int nc,
                                   int th, int r) {
  const int N = P.nph, L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  for (int it = threadIdx.x; it < (L + 1) * npair; it += blockDim.x) {
    const int m = it / npair, pp = it % npair;
    const double2* zp = z + (long long)pp * N;
    const double2 zm = zp[m];
    double a0, b0, a1, b1;
    if (m == 0) {
      a0 = zm.x * aN;
      a1 = zm.y * aN;
      b0 = 0.0;
      b1 = 0.0;
    } else {
      const double2 wm = zp[N - m];
      a0 = (zm.x + wm.x) * aN;
      b0 = (wm.y - zm.y) * aN;
      a1 = (zm.y + wm.y) * aN;
      b1 = (zm.x - wm.x) * aN;
    }
    double* rec = base + m * strideM + 4 * pp;
    *reinterpret_cast<double2*>(rec) = make_double2(a0, b0);
    if (2 * pp + 1 < nc) *reinterpret_cast<double2*>(rec + 2) = make_double2(a1, b1);
  }
}

__device__ __forceinline__ double zget(const double2* z, int N, int c, int pos) {
  const double2 v = z[(long long)(c >> 1) * N + pos];
  return (c & 1) ? v.y : v.x;
}

__global__ void __launch_bounds__(512, 1) k_fft_cycle(Plan P) {
  extern __shared__ double2 zs[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npair = npb > npf ? npb : npf;
  double2* tw = zs + (long long)npair * N;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = P.twid[k];
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  load_line_spectra(zs, npb, P, P.rtm_b, P.ncb, th, r);
  __syncthreads();
  fft_dif_plus(zs, npb, N, P, tw);
  // products at every (digit-reversed) grid point
  for (int pos = threadIdx.x; pos < N; pos += blockDim.x) {
    double in[3 * kMaxVec + kMaxScl];
    double out[3 * kMaxVec + kMaxScl];
    for (int c = 0; c < P.ncb; ++c) in[c] = zget(zs, N, c, pos);
    int iv = 0, is = 0;
    for (int q = 0; q < P.nprod; ++q) {
      const int kind = P.pkind[q];
      const double cf = P.pcoef[q];
      const int a = P.pa[q], b = P.pb[q];
      if (kind == KMHD_PROD_CROSS) {
        const double* x = in + 3 * a;
        const double* y = in + 3 * b;
        out[3 * iv + 0] = (x[1] * y[2] - x[2] * y[1]) * cf;
        out[3 * iv + 1] = (x[2] * y[0] - x[0] * y[2]) * cf;
        out[3 * iv + 2] = (x[0] * y[1] - x[1] * y[0]) * cf;
        ++iv;
      } else if (kind == KMHD_PROD_VEC_SCALAR) {
        const double* x = in + 3 * a;
        const double s = in[3 * P.nvb + b];
        out[3 * iv + 0] = x[0] * s * cf;
        out[3 * iv + 1] = x[1] * s * cf;
        out[3 * iv + 2] = x[2] * s * cf;
        ++iv;
      } else if (kind == KMHD_PROD_DOT) {
        const double* x = in + 3 * a;
        const double* y = in + 3 * b;
        out[3 * P.nvf + is] = (x[0] * y[0] + x[1] * y[1] + x[2] * y[2]) * cf;
        ++is;
      } else {
        out[3 * P.nvf + is] = in[3 * P.nvb + a] * in[3 * P.nvb + b] * cf;
        ++is;
      }
    }
    for (int q = 0; q < npf; ++q) {
      const double hi = (2 * q + 1 < P.ncf) ? out[2 * q + 1] : 0.0;
      zs[(long long)q * N + pos] = make_double2(out[2 * q], hi);
    }
  }
  __syncthreads();
  fft_dit_minus(zs, npf, N, P, tw);
  store_line_spectra(zs, npf, P, P.rtm_f, P.ncf, th, r);
}

// Separable backward: spectra -> grid fld[node + nnod*c], node = r + nr*(th + nth*phi).
__global__ void __launch_bounds__(512, 1) k_fft_bwd_grid(Plan P, double* __restrict__ fld) {
  extern __shared__ double2 zs[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2;
  double2* tw = zs + (long long)npb * N;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = P.twid[k];
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  load_line_spectra(zs, npb, P, P.rtm_b, P.ncb, th, r);
  __syncthreads();
  fft_dif_plus(zs, npb, N, P, tw);
  const long long nnod = (long long)P.nr * P.nth * N;
  for (int it = threadIdx.x; it < N * P.ncb; it += blockDim.x) {
    const int c = it / N, pos = it % N;
    const int phi = P.digrev[pos];
    fld[(long long)r + (long long)P.nr * (th + (long long)P.nth * phi) + nnod * c] = zget(zs, N, c, pos);
  }
}

// Separable forward: grid frc -> spectra rtm_f.
__global__ void __launch_bounds__(512, 1) k_fft_fwd_grid(Plan P, const double* __restrict__ frc) {
  extern __shared__ double2 zs[];
  const int N = P.nph;
  const int npf = (P.ncf + 1) / 2;
  double2* tw = zs + (long long)npf * N;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = P.twid[k];
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  const long long nnod = (long long)P.nr * P.nth * N;
  for (int it = threadIdx.x; it < N * npf; it += blockDim.x) {
    const int q = it / N, pos = it % N;
    const int phi = P.digrev[pos];
    const long long node = (long long)r + (long long)P.nr * (th + (long long)P.nth * phi);
    const double lo = frc[node + nnod * (2 * q)];
    const double hi = (2 * q + 1 < P.ncf) ? frc[node + nnod * (2 * q + 1)] : 0.0;
    zs[(long long)q * N + pos] = make_double2(lo, hi);
  }
  __syncthreads();
  fft_dit_minus(zs, npf, N, P, tw);
  store_line_spectra(zs, npf, P, P.rtm_f, P.ncf, th, r);
}

}  // namespace

size_t fft_smem_bytes(const Plan& p, int npair) {
  return sizeof(double2) * ((size_t)npair * p.nph + p.nph);
}

cudaError_t launch_fft_cycle(const Plan& p, cudaStream_t s) {
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  const size_t smem = fft_smem_bytes(p, npair);
  cudaFuncSetAttribute(k_fft_cycle, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_cycle<<<p.nr * p.nth, 512, smem, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_fft_bwd_grid(const Plan& p, double* fld, cudaStream_t s) {
  const size_t smem = fft_smem_bytes(p, (p.ncb + 1) / 2);
  cudaFuncSetAttribute(k_fft_bwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_bwd_grid<<<p.nr * p.nth, 512, smem, s>>>(p, fld);
  return cudaGetLastError();
}

cudaError_t launch_fft_fwd_grid(const Plan& p, const double* frc, cudaStream_t s) {
  const size_t smem = fft_smem_bytes(p, (p.ncf + 1) / 2);
  cudaFuncSetAttribute(k_fft_fwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fft_fwd_grid<<<p.nr * p.nth, 512, smem, s>>>(p, frc);
  return cudaGetLastError();
}

}  // namespace kmhd
