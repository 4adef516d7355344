// kmhd_fft.cu -- longitudinal real FFTs fused with the grid-space products.
//
// Each (r, theta) line is handled by one CTA with every component of the line
// in shared memory, so inverse FFT -> products -> forward FFT never touch HBM.
// Convention (t_sph_single_FFTW.F90 normalisation with the FFTPACK slot order of
// PARALLEL_src/SPH_SHELL_src/t_sph_FFTPACK5.f90:183-331):
//   x_j = a_0 + sum_{k>=1} (a_k cos(2 pi jk/N) + b_k sin(2 pi jk/N)),
//   a_0 = (1/N) sum x_j, a_k = (2/N) sum x_j cos, b_k = (2/N) sum x_j sin.
// Two real components travel as one complex sequence z = x_a + i x_b.  The
// inverse transform is an in-place mixed-radix decimation in frequency
// (natural spectrum in, digit-reversed grid out); the products are pointwise,
// so they run on the digit-reversed grid; the forward transform is its exact
// transpose (decimation in time, digit-reversed in, natural out).  No
// reordering pass exists.  The first inverse pass reads the staged spectra
// directly and skips the band L < k < N-L, which is zero.
// Products: cal_cross_prod_w_coef_smp, cal_vec_scalar_prod_w_coef_smp,
// cal_dot_prod_w_coef_smp (CORE_src/BASE/cal_products_smp.f90) as called by
// nonlinear_terms_in_rtp (MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:64-128).
#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

constexpr int kFftThreads = 256;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <int SIGN>
__device__ __forceinline__ double2 mul_si(double2 a) {  // a * (SIGN i)
  return SIGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// y_q = sum_r x_r e^{SIGN 2 pi i r q / R}, in place, compile-time R.
template <int R, int SIGN>
struct DFT;
template <int SIGN>
struct DFT<2, SIGN> {
  __device__ static void run(double2* x) {
    const double2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  }
};
template <int SIGN>
struct DFT<4, SIGN> {
  __device__ static void run(double2* x) {
    const double2 a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
    const double2 c = cadd(x[1], x[3]), d = mul_si<SIGN>(csub(x[1], x[3]));
    x[0] = cadd(a, c);
    x[1] = cadd(b, d);
    x[2] = csub(a, c);
    x[3] = csub(b, d);
  }
};
template <int SIGN>
struct DFT<3, SIGN> {
  __device__ static void run(double2* x) {
    const double s3 = 0.86602540378443864676 * (double)SIGN;
    const double2 t = cadd(x[1], x[2]);
    const double2 d = csub(x[1], x[2]);
    const double2 u = make_double2(-d.y * s3, d.x * s3);
    const double2 v = make_double2(x[0].x - 0.5 * t.x, x[0].y - 0.5 * t.y);
    x[0] = cadd(x[0], t);
    x[1] = cadd(v, u);
    x[2] = csub(v, u);
  }
};
template <int SIGN>
struct DFT<5, SIGN> {
  __device__ static void run(double2* x) {
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
};
template <int SIGN>
struct DFT<8, SIGN> {
  __device__ static void run(double2* x) {
    const double h = 0.70710678118654752440;
    double2 e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
    DFT<4, SIGN>::run(e);
    DFT<4, SIGN>::run(o);
    o[1] = make_double2(h * (o[1].x - (double)SIGN * o[1].y), h * (o[1].y + (double)SIGN * o[1].x));
    o[2] = mul_si<SIGN>(o[2]);
    o[3] = make_double2(h * (-o[3].x - (double)SIGN * o[3].y), h * (-o[3].y + (double)SIGN * o[3].x));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[k] = cadd(e[k], o[k]);
      x[k + 4] = csub(e[k], o[k]);
    }
  }
};

template <int SIGN>
__device__ __forceinline__ double2 twd(const double2* __restrict__ tw, int idx) {
  const double2 w = __ldg(tw + idx);
  return SIGN > 0 ? w : make_double2(w.x, -w.y);
}

// One in-place DIF (+) pass over npair sequences: butterfly, then twiddle.
template <int R>
__device__ void dif_pass(double2* z, int npair, int N, int span, const double2* __restrict__ tw) {
  const int s = span / R, nbf = N / R, stw = N / span;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, rem = it % nbf;
    const int j = rem % s, b = rem / s;
    double2* base = z + pp * N + b * span + j;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = base[r * s];
    DFT<R, +1>::run(x);
    base[0] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) base[q * s] = cmul(x[q], twd<+1>(tw, j * q * stw));
  }
}

// One in-place DIT (-) pass, the transpose of dif_pass.
template <int R>
__device__ void dit_pass(double2* z, int npair, int N, int span, const double2* __restrict__ tw) {
  const int s = span / R, nbf = N / R, stw = N / span;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, rem = it % nbf;
    const int j = rem % s, b = rem / s;
    double2* base = z + pp * N + b * span + j;
    double2 x[R];
    x[0] = base[0];
#pragma unroll
    for (int q = 1; q < R; ++q) x[q] = cmul(base[q * s], twd<-1>(tw, j * q * stw));
    DFT<R, -1>::run(x);
#pragma unroll
    for (int r = 0; r < R; ++r) base[r * s] = x[r];
  }
}

__device__ void dif_dispatch(int R, double2* z, int npair, int N, int span, const double2* tw) {
  switch (R) {
    case 8: dif_pass<8>(z, npair, N, span, tw); break;
    case 4: dif_pass<4>(z, npair, N, span, tw); break;
    case 2: dif_pass<2>(z, npair, N, span, tw); break;
    case 3: dif_pass<3>(z, npair, N, span, tw); break;
    default: dif_pass<5>(z, npair, N, span, tw); break;
  }
}
__device__ void dit_dispatch(int R, double2* z, int npair, int N, int span, const double2* tw) {
  switch (R) {
    case 8: dit_pass<8>(z, npair, N, span, tw); break;
    case 4: dit_pass<4>(z, npair, N, span, tw); break;
    case 2: dit_pass<2>(z, npair, N, span, tw); break;
    case 3: dit_pass<3>(z, npair, N, span, tw); break;
    default: dit_pass<5>(z, npair, N, span, tw); break;
  }
}

// Complex spectrum of pair pp at frequency k from staged records
// st[(m*nc + c)*2 + {0: a, 1: b}], m <= L.  z = X_{2pp} + i X_{2pp+1},
// X_c[m] = (a - i b)/2 for m > 0, X_c[0] = a, X_c[N-m] = conj(X_c[m]).
__device__ __forceinline__ double2 spec_at(const double* st, int nc, int nv, int pp, int k, int N, int L) {
  int m;
  bool mirror;
  if (k <= L) { m = k; mirror = false; }
  else if (k >= N - L) { m = N - k; mirror = true; }
  else return make_double2(0.0, 0.0);
  const double* rec = st + m * nc * 2;
  const double* r0 = rec + rec_off(2 * pp, nv);
  const double a0 = r0[0], b0 = r0[1];
  double a1 = 0.0, b1 = 0.0;
  if (2 * pp + 1 < nc) {
    const double* r1 = rec + rec_off(2 * pp + 1, nv);
    a1 = r1[0];
    b1 = r1[1];
  }
  if (m == 0) return make_double2(a0, a1);
  return mirror ? make_double2(0.5 * a0 - 0.5 * b1, 0.5 * b0 + 0.5 * a1)
                : make_double2(0.5 * a0 + 0.5 * b1, 0.5 * a1 - 0.5 * b0);
}

// First DIF pass: input from the staged spectra, output into z.
template <int R>
__device__ void dif_first(const double* st, int nc, int nv, double2* z, int npair, int N, int L,
                          const double2* __restrict__ tw) {
  const int s = N / R, nbf = N / R;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, j = it % nbf;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = spec_at(st, nc, nv, pp, j + r * s, N, L);
    DFT<R, +1>::run(x);
    double2* base = z + pp * N + j;
    base[0] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) base[q * s] = cmul(x[q], twd<+1>(tw, j * q));
  }
}
__device__ void dif_first_dispatch(int R, const double* st, int nc, int nv, double2* z, int npair,
                                   int N, int L, const double2* tw) {
  switch (R) {
    case 8: dif_first<8>(st, nc, nv, z, npair, N, L, tw); break;
    case 4: dif_first<4>(st, nc, nv, z, npair, N, L, tw); break;
    case 2: dif_first<2>(st, nc, nv, z, npair, N, L, tw); break;
    case 3: dif_first<3>(st, nc, nv, z, npair, N, L, tw); break;
    default: dif_first<5>(st, nc, nv, z, npair, N, L, tw); break;
  }
}

__device__ void dif_rest(double2* z, int npair, int N, const Plan& P, const double2* tw) {
  int span = N / P.fac[0];
  for (int f = 1; f < P.nfac; ++f) {
    dif_dispatch(P.fac[f], z, npair, N, span, tw);
    __syncthreads();
    span /= P.fac[f];
  }
}

__device__ void dit_all(double2* z, int npair, int N, const Plan& P, const double2* tw) {
  int spans[kMaxFftFactors];
  int span = N;
  for (int f = 0; f < P.nfac; ++f) {
    spans[f] = span;
    span /= P.fac[f];
  }
  for (int f = P.nfac - 1; f >= 0; --f) {
    dit_dispatch(P.fac[f], z, npair, N, spans[f], tw);
    __syncthreads();
  }
}

// Stage the records of line (th, r) for all m into st via cp.async (16 B each).
__device__ void prefetch_line(double* st, const double* rtm, int nc, const Plan& P, int th, int r) {
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  const double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  const int n = (P.L + 1) * nc;
  for (int it = threadIdx.x; it < n; it += blockDim.x) {
    const int m = it / nc, c = it % nc;
    cp_async16(st + (m * nc + c) * 2, base + m * strideM + c * 2);
  }
  cp_async_commit();
}

// Natural-order forward spectra in z -> (a_m, b_m), m <= L, into rtm.
__device__ void store_line(const double2* z, int npair, const Plan& P, double* rtm, int nc, int nv, int th, int r) {
  const int N = P.nph, L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  for (int it = threadIdx.x; it < (L + 1) * npair; it += blockDim.x) {
    const int m = it / npair, pp = it % npair;
    const double2* zp = z + pp * N;
    const double2 zm = zp[m];
    double a0, b0, a1, b1;
    if (m == 0) {
      a0 = zm.x * aN; a1 = zm.y * aN; b0 = 0.0; b1 = 0.0;
    } else {
      const double2 wm = zp[N - m];
      a0 = (zm.x + wm.x) * aN;
      b0 = (wm.y - zm.y) * aN;
      a1 = (zm.y + wm.y) * aN;
      b1 = (zm.x - wm.x) * aN;
    }
    double* rec = base + m * strideM;
    *reinterpret_cast<double2*>(rec + rec_off(2 * pp, nv)) = make_double2(a0, b0);
    if (2 * pp + 1 < nc) *reinterpret_cast<double2*>(rec + rec_off(2 * pp + 1, nv)) = make_double2(a1, b1);
  }
}

// Vector a of the backward fields, selected without dynamic register indexing.
template <int MV>
__device__ __forceinline__ void selvec(const double* in, int a, double& x0, double& x1, double& x2) {
  x0 = in[0]; x1 = in[1]; x2 = in[2];
#pragma unroll
  for (int v = 1; v < MV; ++v)
    if (a == v) { x0 = in[3 * v]; x1 = in[3 * v + 1]; x2 = in[3 * v + 2]; }
}
template <int MS>
__device__ __forceinline__ double selscl(const double* s, int b) {
  double x = s[0];
#pragma unroll
  for (int q = 1; q < MS; ++q)
    if (b == q) x = s[q];
  return x;
}

// Pointwise products on the digit-reversed grid.  MV*/MS* are compile-time
// maxima; the plan's counts are <= them (products are ordered vectors first).
template <int MVB, int MSB, int MVF, int MSF>
__device__ void products(double2* z, int N, const Plan& P) {
  constexpr int MCF = 3 * MVF + MSF;
  const int nvb = P.nvb, nsb = P.nsb, nvf = P.nvf, nsf = P.nsf;
  for (int pos = threadIdx.x; pos < N; pos += blockDim.x) {
    double vin[3 * MVB > 0 ? 3 * MVB : 1], sin_[MSB > 0 ? MSB : 1];
#pragma unroll
    for (int c = 0; c < 3 * MVB; ++c)
      if (c < 3 * nvb) {
        const double2 v = z[(c >> 1) * N + pos];
        vin[c] = (c & 1) ? v.y : v.x;
      }
#pragma unroll
    for (int q = 0; q < MSB; ++q)
      if (q < nsb) {
        const int c = 3 * nvb + q;
        const double2 v = z[(c >> 1) * N + pos];
        sin_[q] = (c & 1) ? v.y : v.x;
      }
    double out[MCF > 0 ? MCF : 1];
#pragma unroll
    for (int i = 0; i < MVF; ++i) {
      if (i < nvf) {
        const int kind = P.pkind[i];
        const double cf = P.pcoef[i];
        double x0, x1, x2;
        selvec<MVB>(vin, P.pa[i], x0, x1, x2);
        if (kind == KMHD_PROD_CROSS) {
          double y0, y1, y2;
          selvec<MVB>(vin, P.pb[i], y0, y1, y2);
          out[3 * i + 0] = (x1 * y2 - x2 * y1) * cf;
          out[3 * i + 1] = (x2 * y0 - x0 * y2) * cf;
          out[3 * i + 2] = (x0 * y1 - x1 * y0) * cf;
        } else {
          const double s = selscl<MSB>(sin_, P.pb[i]);
          out[3 * i + 0] = x0 * s * cf;
          out[3 * i + 1] = x1 * s * cf;
          out[3 * i + 2] = x2 * s * cf;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MSF; ++j) {
      if (j < nsf) {
        const int q = nvf + j;
        const int kind = P.pkind[q];
        const double cf = P.pcoef[q];
        double o;
        if (kind == KMHD_PROD_DOT) {
          double x0, x1, x2, y0, y1, y2;
          selvec<MVB>(vin, P.pa[q], x0, x1, x2);
          selvec<MVB>(vin, P.pb[q], y0, y1, y2);
          o = (x0 * y0 + x1 * y1 + x2 * y2) * cf;
        } else {
          o = selscl<MSB>(sin_, P.pa[q]) * selscl<MSB>(sin_, P.pb[q]) * cf;
        }
        // output component 3*nvf + j: compile-time slot only when nvf == MVF
        out[3 * MVF + j] = o;
      }
    }
    // dense output order: vectors [0, 3*nvf), then scalars; compile-time slots
    const int ncf = 3 * nvf + nsf;
    double dense[MCF > 0 ? MCF : 1];
#pragma unroll
    for (int c = 0; c < MCF; ++c) {
      double v = 0.0;
      if (c < 3 * MVF) v = out[c < 3 * MVF ? c : 0];
      if (c >= 3 * nvf) {
        v = 0.0;
#pragma unroll
        for (int j = 0; j < MSF; ++j)
          if (c == 3 * nvf + j) v = out[3 * MVF + j];
      }
      dense[c] = v;
    }
#pragma unroll
    for (int c = 0; c < MCF; c += 2) {
      if (c < ncf) {
        const double hi = (c + 1 < MCF && c + 1 < ncf) ? dense[c + 1 < MCF ? c + 1 : c] : 0.0;
        z[(c >> 1) * N + pos] = make_double2(dense[c], hi);
      }
    }
  }
}

template <int MVB, int MSB, int MVF, int MSF>
__global__ void __launch_bounds__(kFftThreads) k_fft_cycle(Plan P, int nlines) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npair = npb > npf ? npb : npf;
  double2* z = reinterpret_cast<double2*>(smraw);
  double* st = reinterpret_cast<double*>(z + npair * N);
  int line = blockIdx.x;
  if (line >= nlines) return;
  prefetch_line(st, P.rtm_b, P.ncb, P, line / P.nr, line % P.nr);
  while (line < nlines) {
    const int r = line % P.nr, th = line / P.nr;
    cp_async_wait<0>();
    __syncthreads();
    dif_first_dispatch(P.fac[0], st, P.ncb, P.nvb, z, npb, N, P.L, P.twid);
    __syncthreads();
    const int next = line + gridDim.x;
    if (next < nlines) prefetch_line(st, P.rtm_b, P.ncb, P, next / P.nr, next % P.nr);
    dif_rest(z, npb, N, P, P.twid);
    products<MVB, MSB, MVF, MSF>(z, N, P);
    __syncthreads();
    dit_all(z, npf, N, P, P.twid);
    store_line(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
    line = next;
  }
}

// Separable backward: spectra -> grid fld[node + nnod*c], node = r + nr*(th + nth*phi).
__global__ void __launch_bounds__(kFftThreads) k_fft_bwd_grid(Plan P, double* __restrict__ fld) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2;
  double2* z = reinterpret_cast<double2*>(smraw);
  double* st = reinterpret_cast<double*>(z + npb * N);
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  prefetch_line(st, P.rtm_b, P.ncb, P, th, r);
  cp_async_wait<0>();
  __syncthreads();
  dif_first_dispatch(P.fac[0], st, P.ncb, P.nvb, z, npb, N, P.L, P.twid);
  __syncthreads();
  dif_rest(z, npb, N, P, P.twid);
  const long long nnod = (long long)P.nr * P.nth * N;
  for (int it = threadIdx.x; it < N * P.ncb; it += blockDim.x) {
    const int c = it / N, pos = it % N;
    const int phi = P.digrev[pos];
    const double2 v = z[(c >> 1) * N + pos];
    fld[(long long)r + (long long)P.nr * (th + (long long)P.nth * phi) + nnod * c] = (c & 1) ? v.y : v.x;
  }
}

// Separable forward: grid frc -> spectra rtm_f.
__global__ void __launch_bounds__(kFftThreads) k_fft_fwd_grid(Plan P, const double* __restrict__ frc) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npf = (P.ncf + 1) / 2;
  double2* z = reinterpret_cast<double2*>(smraw);
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  const long long nnod = (long long)P.nr * P.nth * N;
  for (int it = threadIdx.x; it < N * npf; it += blockDim.x) {
    const int q = it / N, pos = it % N;
    const int phi = P.digrev[pos];
    const long long node = (long long)r + (long long)P.nr * (th + (long long)P.nth * phi);
    const double lo = frc[node + nnod * (2 * q)];
    const double hi = (2 * q + 1 < P.ncf) ? frc[node + nnod * (2 * q + 1)] : 0.0;
    z[q * N + pos] = make_double2(lo, hi);
  }
  __syncthreads();
  dit_all(z, npf, N, P, P.twid);
  store_line(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
}

// ---------------------------------------------------------------------------
// Compile-time variant for the common N = 3 2^k: factor order (3, leftover 4 or
// 2, then 8s), spans and strides are constants, 512 threads, and a bank-
// conflict-free shared layout: inside each pair sequence the index is swizzled
// i -> i ^ ((i >> 3) & 7) and pairs are N + 1 entries apart; passes with stride
// >= 8 run the in-block index fastest across threads, the others the butterfly
// block index, so every quarter warp (8 x 16 bytes) hits 8 distinct bank groups.
constexpr int kFftThreadsT = 512;

__host__ __device__ constexpr int tfac_count(int n) {
  int c = 0;
  while (n % 3 == 0) { n /= 3; ++c; }
  while (n % 5 == 0) { n /= 5; ++c; }
  int e = 0;
  while (n % 8 == 0) { n /= 8; ++e; }
  if (n == 2 || n == 4) { ++c; n = 1; }
  return c + e;
}
__host__ __device__ constexpr int tfac_at(int n, int i) {
  int c = 0;
  while (n % 3 == 0) { if (c == i) return 3; n /= 3; ++c; }
  while (n % 5 == 0) { if (c == i) return 5; n /= 5; ++c; }
  int r = n, e = 0;
  while (r % 8 == 0) { r /= 8; ++e; }
  if (r == 2 || r == 4) { if (c == i) return r; ++c; }
  return 8;
}
__host__ __device__ constexpr int tspan_at(int n, int i) {
  int sp = n;
  for (int q = 0; q < i; ++q) sp /= tfac_at(n, q);
  return sp;
}
__device__ __forceinline__ int sw(int i) { return i ^ ((i >> 3) & 7); }

// twiddles w^q, q = 1..R-1, from two table loads (w^1, w^2)
template <int R, int SIGN>
__device__ __forceinline__ void twiddles(const double2* __restrict__ tw, int base, int N, double2* w) {
  if constexpr (R >= 2) w[1] = twd<SIGN>(tw, base);
  if constexpr (R >= 3) w[2] = twd<SIGN>(tw, (2 * base) % N);
  if constexpr (R >= 4) w[3] = cmul(w[1], w[2]);
  if constexpr (R >= 5) w[4] = cmul(w[2], w[2]);
  if constexpr (R >= 6) w[5] = cmul(w[4], w[1]);
  if constexpr (R >= 7) w[6] = cmul(w[4], w[2]);
  if constexpr (R >= 8) w[7] = cmul(w[4], w[3]);
}

template <int N, int I>
__device__ __forceinline__ void tdif(double2* z, int npair, const double2* __restrict__ tw) {
  if constexpr (I < tfac_count(N)) {
    constexpr int R = tfac_at(N, I), span = tspan_at(N, I), s = span / R, nbf = N / R, stw = N / span;
    constexpr int NB = N / span;  // butterfly blocks
    constexpr int NP = N + 1;
    for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
      const int pp = it / nbf, rem = it - pp * nbf;
      int b, j;
      if constexpr (s >= 8) { b = rem / s; j = rem - b * s; }
      else { j = rem / NB; b = rem - j * NB; }
      double2* zp = z + pp * NP;
      const int base = b * span + j;
      double2 x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = zp[sw(base + r * s)];
      DFT<R, +1>::run(x);
      double2 w[R];
      twiddles<R, +1>(tw, j * stw, N, w);
      zp[sw(base)] = x[0];
#pragma unroll
      for (int q = 1; q < R; ++q) zp[sw(base + q * s)] = cmul(x[q], w[q]);
    }
    __syncthreads();
    tdif<N, I + 1>(z, npair, tw);
  }
}

template <int N, int I>
__device__ __forceinline__ void tdit(double2* z, int npair, const double2* __restrict__ tw) {
  if constexpr (I >= 0) {
    constexpr int R = tfac_at(N, I), span = tspan_at(N, I), s = span / R, nbf = N / R, stw = N / span;
    constexpr int NB = N / span;
    constexpr int NP = N + 1;
    for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
      const int pp = it / nbf, rem = it - pp * nbf;
      int b, j;
      if constexpr (s >= 8) { b = rem / s; j = rem - b * s; }
      else { j = rem / NB; b = rem - j * NB; }
      double2* zp = z + pp * NP;
      const int base = b * span + j;
      double2 w[R];
      twiddles<R, -1>(tw, j * stw, N, w);
      double2 x[R];
      x[0] = zp[sw(base)];
#pragma unroll
      for (int q = 1; q < R; ++q) x[q] = cmul(zp[sw(base + q * s)], w[q]);
      DFT<R, -1>::run(x);
#pragma unroll
      for (int r = 0; r < R; ++r) zp[sw(base + r * s)] = x[r];
    }
    __syncthreads();
    tdit<N, I - 1>(z, npair, tw);
  }
}

// staged records of one line: [m][ncs pairs], ncs = nc rounded up to odd
__device__ __forceinline__ int ncs_of(int nc) { return nc | 1; }

__device__ void prefetch_line_t(double* st, const double* rtm, int nc, const Plan& P, int th, int r) {
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  const double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  const int ncs = ncs_of(nc);
  const int n = (P.L + 1) * nc;
  for (int it = threadIdx.x; it < n; it += blockDim.x) {
    const int m = it / nc, c = it - m * nc;
    cp_async16(st + (m * ncs + c) * 2, base + m * strideM + c * 2);
  }
  cp_async_commit();
}

__device__ __forceinline__ double2 spec_at_t(const double* st, int nc, int nv, int pp, int k, int N, int L) {
  int m;
  bool mirror;
  if (k <= L) { m = k; mirror = false; }
  else if (k >= N - L) { m = N - k; mirror = true; }
  else return make_double2(0.0, 0.0);
  const double* rec = st + m * ncs_of(nc) * 2;
  const double* r0 = rec + rec_off(2 * pp, nv);
  const double a0 = r0[0], b0 = r0[1];
  double a1 = 0.0, b1 = 0.0;
  if (2 * pp + 1 < nc) {
    const double* r1 = rec + rec_off(2 * pp + 1, nv);
    a1 = r1[0];
    b1 = r1[1];
  }
  if (m == 0) return make_double2(a0, a1);
  return mirror ? make_double2(0.5 * a0 - 0.5 * b1, 0.5 * b0 + 0.5 * a1)
                : make_double2(0.5 * a0 + 0.5 * b1, 0.5 * a1 - 0.5 * b0);
}

template <int N>
__device__ __forceinline__ void tdif_first(const double* st, int nc, int nv, double2* z, int npair, int L,
                                           const double2* __restrict__ tw) {
  constexpr int R = tfac_at(N, 0), s = N / R, nbf = N / R;
  constexpr int NP = N + 1;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, j = it - pp * nbf;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = spec_at_t(st, nc, nv, pp, j + r * s, N, L);
    DFT<R, +1>::run(x);
    double2 w[R];
    twiddles<R, +1>(tw, j, N, w);
    double2* zp = z + pp * NP;
    zp[sw(j)] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) zp[sw(j + q * s)] = cmul(x[q], w[q]);
  }
}

template <int N>
__device__ void tstore_line(const double2* z, int npair, const Plan& P, double* rtm, int nc, int nv, int th, int r) {
  constexpr int NP = N + 1;
  const int L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  double* base = rtm + ((long long)th * P.nr + r) * nc * 2;
  for (int it = threadIdx.x; it < (L + 1) * npair; it += blockDim.x) {
    const int pp = it / (L + 1), m = it - pp * (L + 1);
    const double2* zp = z + pp * NP;
    const double2 zm = zp[sw(m)];
    double a0, b0, a1, b1;
    if (m == 0) {
      a0 = zm.x * aN; a1 = zm.y * aN; b0 = 0.0; b1 = 0.0;
    } else {
      const double2 wm = zp[sw(N - m)];
      a0 = (zm.x + wm.x) * aN;
      b0 = (wm.y - zm.y) * aN;
      a1 = (zm.y + wm.y) * aN;
      b1 = (zm.x - wm.x) * aN;
    }
    double* rec = base + m * strideM;
    *reinterpret_cast<double2*>(rec + rec_off(2 * pp, nv)) = make_double2(a0, b0);
    if (2 * pp + 1 < nc) *reinterpret_cast<double2*>(rec + rec_off(2 * pp + 1, nv)) = make_double2(a1, b1);
  }
}

template <int N, int MVB, int MSB, int MVF, int MSF>
__device__ void tproducts(double2* z, const Plan& P) {
  constexpr int NP = N + 1;
  constexpr int MCF = 3 * MVF + MSF;
  const int nvb = P.nvb, nsb = P.nsb, nvf = P.nvf, nsf = P.nsf;
  for (int pos = threadIdx.x; pos < N; pos += blockDim.x) {
    const int pq = sw(pos);
    double vin[3 * MVB > 0 ? 3 * MVB : 1], sin_[MSB > 0 ? MSB : 1];
#pragma unroll
    for (int c = 0; c < 3 * MVB; ++c)
      if (c < 3 * nvb) {
        const double2 v = z[(c >> 1) * NP + pq];
        vin[c] = (c & 1) ? v.y : v.x;
      }
#pragma unroll
    for (int q = 0; q < MSB; ++q)
      if (q < nsb) {
        const int c = 3 * nvb + q;
        const double2 v = z[(c >> 1) * NP + pq];
        sin_[q] = (c & 1) ? v.y : v.x;
      }
    double out[MCF > 0 ? MCF : 1];
#pragma unroll
    for (int i = 0; i < MVF; ++i) {
      if (i < nvf) {
        const double cf = P.pcoef[i];
        double x0, x1, x2;
        selvec<MVB>(vin, P.pa[i], x0, x1, x2);
        if (P.pkind[i] == KMHD_PROD_CROSS) {
          double y0, y1, y2;
          selvec<MVB>(vin, P.pb[i], y0, y1, y2);
          out[3 * i + 0] = (x1 * y2 - x2 * y1) * cf;
          out[3 * i + 1] = (x2 * y0 - x0 * y2) * cf;
          out[3 * i + 2] = (x0 * y1 - x1 * y0) * cf;
        } else {
          const double sv = selscl<MSB>(sin_, P.pb[i]);
          out[3 * i + 0] = x0 * sv * cf;
          out[3 * i + 1] = x1 * sv * cf;
          out[3 * i + 2] = x2 * sv * cf;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MSF; ++j) {
      if (j < nsf) {
        const int q = nvf + j;
        const double cf = P.pcoef[q];
        double o;
        if (P.pkind[q] == KMHD_PROD_DOT) {
          double x0, x1, x2, y0, y1, y2;
          selvec<MVB>(vin, P.pa[q], x0, x1, x2);
          selvec<MVB>(vin, P.pb[q], y0, y1, y2);
          o = (x0 * y0 + x1 * y1 + x2 * y2) * cf;
        } else {
          o = selscl<MSB>(sin_, P.pa[q]) * selscl<MSB>(sin_, P.pb[q]) * cf;
        }
        out[3 * MVF + j] = o;
      }
    }
    const int ncf = 3 * nvf + nsf;
    double dense[MCF > 0 ? MCF : 1];
#pragma unroll
    for (int c = 0; c < MCF; ++c) {
      double v = 0.0;
      if (c < 3 * MVF) v = out[c < 3 * MVF ? c : 0];
      if (c >= 3 * nvf) {
        v = 0.0;
#pragma unroll
        for (int j = 0; j < MSF; ++j)
          if (c == 3 * nvf + j) v = out[3 * MVF + j];
      }
      dense[c] = v;
    }
#pragma unroll
    for (int c = 0; c < MCF; c += 2) {
      if (c < ncf) {
        const double hi = (c + 1 < MCF && c + 1 < ncf) ? dense[c + 1 < MCF ? c + 1 : c] : 0.0;
        z[(c >> 1) * NP + pq] = make_double2(dense[c], hi);
      }
    }
  }
}

template <int N, int MVB, int MSB, int MVF, int MSF>
__global__ void __launch_bounds__(kFftThreadsT, 1) k_fft_cycle_t(Plan P, int nlines) {
  extern __shared__ double4 smraw[];
  constexpr int NP = N + 1;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npair = npb > npf ? npb : npf;
  double2* z = reinterpret_cast<double2*>(smraw);
  double* st = reinterpret_cast<double*>(z + npair * NP + 1);  // keep 16-byte alignment
  int line = blockIdx.x;
  if (line >= nlines) return;
  prefetch_line_t(st, P.rtm_b, P.ncb, P, line / P.nr, line % P.nr);
  while (line < nlines) {
    const int r = line % P.nr, th = line / P.nr;
    cp_async_wait<0>();
    __syncthreads();
    tdif_first<N>(st, P.ncb, P.nvb, z, npb, P.L, P.twid);
    __syncthreads();
    const int next = line + gridDim.x;
    if (next < nlines) prefetch_line_t(st, P.rtm_b, P.ncb, P, next / P.nr, next % P.nr);
    tdif<N, 1>(z, npb, P.twid);
    tproducts<N, MVB, MSB, MVF, MSF>(z, P);
    __syncthreads();
    tdit<N, tfac_count(N) - 1>(z, npf, P.twid);
    tstore_line<N>(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
    line = next;
  }
}

size_t smem_cycle_t(const Plan& p) {
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  return sizeof(double2) * ((size_t)npair * (p.nph + 1) + 1) + sizeof(double) * 2 * (size_t)(p.L + 1) * (p.ncb | 1);
}

template <int N, int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_t(const Plan& p, cudaStream_t s) {
  auto kern = k_fft_cycle_t<N, MVB, MSB, MVF, MSF>;
  const size_t smem = smem_cycle_t(p);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kFftThreadsT, smem);
  if (occ < 1) occ = 1;
  const int nlines = p.nr * p.nth;
  int grid = nsm * occ;
  if (grid > nlines) grid = nlines;
  kern<<<grid, kFftThreadsT, smem, s>>>(p, nlines);
  return cudaGetLastError();
}

template <int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_n(const Plan& p, cudaStream_t s, bool* handled) {
  *handled = true;
  if (smem_cycle_t(p) <= 227 * 1024) {
    switch (p.nph) {
      case 96: return run_cycle_t<96, MVB, MSB, MVF, MSF>(p, s);
      case 192: return run_cycle_t<192, MVB, MSB, MVF, MSF>(p, s);
      case 384: return run_cycle_t<384, MVB, MSB, MVF, MSF>(p, s);
      case 768: return run_cycle_t<768, MVB, MSB, MVF, MSF>(p, s);
      case 1536: return run_cycle_t<1536, MVB, MSB, MVF, MSF>(p, s);
      default: break;
    }
  }
  *handled = false;
  return cudaSuccess;
}

size_t smem_cycle(const Plan& p) {
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  return sizeof(double2) * (size_t)npair * p.nph + sizeof(double) * 2 * (size_t)(p.L + 1) * p.ncb;
}

template <int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle(const Plan& p, cudaStream_t s) {
  auto kern = k_fft_cycle<MVB, MSB, MVF, MSF>;
  const size_t smem = smem_cycle(p);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kFftThreads, smem);
  if (occ < 1) occ = 1;
  const int nlines = p.nr * p.nth;
  int grid = nsm * occ;
  if (grid > nlines) grid = nlines;
  kern<<<grid, kFftThreads, smem, s>>>(p, nlines);
  return cudaGetLastError();
}

}  // namespace

size_t fft_smem_bytes(const Plan& p, int npair) {
  (void)npair;
  return smem_cycle(p);
}

cudaError_t launch_fft_cycle(const Plan& p, cudaStream_t s) {
  if (p.nvb == 3 && p.nsb == 1 && p.nvf == 3 && p.nsf == 1) {
    bool handled = false;
    const cudaError_t e = run_cycle_n<3, 1, 3, 1>(p, s, &handled);
    if (handled) return e;
    return run_cycle<3, 1, 3, 1>(p, s);
  }
  if (p.nvb == 2 && p.nsb == 1 && p.nvf == 2 && p.nsf == 1) {
    bool handled = false;
    const cudaError_t e = run_cycle_n<2, 1, 2, 1>(p, s, &handled);
    if (handled) return e;
    return run_cycle<2, 1, 2, 1>(p, s);
  }
  if (p.nvb == 1 && p.nsb == 1 && p.nvf == 1 && p.nsf == 0) {
    bool handled = false;
    const cudaError_t e = run_cycle_n<1, 1, 1, 0>(p, s, &handled);
    if (handled) return e;
    return run_cycle<1, 1, 1, 0>(p, s);
  }
  return run_cycle<kMaxVec, kMaxScl, kMaxVec, kMaxScl>(p, s);
}

cudaError_t launch_fft_bwd_grid(const Plan& p, double* fld, cudaStream_t s) {
  const int npb = (p.ncb + 1) / 2;
  const size_t smem = sizeof(double2) * (size_t)npb * p.nph + sizeof(double) * 2 * (size_t)(p.L + 1) * p.ncb;
  cudaError_t e = cudaFuncSetAttribute(k_fft_bwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_fft_bwd_grid<<<p.nr * p.nth, kFftThreads, smem, s>>>(p, fld);
  return cudaGetLastError();
}

cudaError_t launch_fft_fwd_grid(const Plan& p, const double* frc, cudaStream_t s) {
  const int npf = (p.ncf + 1) / 2;
  const size_t smem = sizeof(double2) * (size_t)npf * p.nph;
  cudaError_t e = cudaFuncSetAttribute(k_fft_fwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_fft_fwd_grid<<<p.nr * p.nth, kFftThreads, smem, s>>>(p, frc);
  return cudaGetLastError();
}

}  // namespace kmhd
