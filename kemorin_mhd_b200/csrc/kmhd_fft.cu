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
#include <algorithm>
#include <utility>

#include <cuda.h>

#include <cstring>

#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

constexpr int kFftThreads = 256;

// mbarrier + TMA tensor load (staging of a line's spectra)
constexpr long long kFftSpinCap = 1ll << 22;  // try_wait rounds (each may suspend for microseconds)
__device__ __forceinline__ unsigned ssa(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool fbar_wait(unsigned long long* b, unsigned parity, long long cap = kFftSpinCap) {
  for (long long it = 0; it < cap; ++it) {
    unsigned ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(ssa(b)), "r"(parity));
    if (ok) return true;
  }
  return false;
}

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

// Twiddles w^(j q), q = 0, 1, ..., of one radix-R butterfly (w = e^{2 pi i / N})
// with a table load every eighth q only: a running product w^(j q) =
// w^(j (q - 1)) w^j, restarted from the table at q = 8, 16, ..., so at most
// seven products separate a twiddle from a table value (within 2e-15 of
// e^{2 pi i j q / N} for N = 48 .. 3072, checked against exact values).
// Used by the first and last passes of the specialised kernels, whose lanes
// read 32 different table entries per load (at L = 511 the FFT kernel takes
// 20.6 ms this way, 21.7 ms restarting every fourth q, 23.5 ms loading every
// twiddle).
template <int SIGN>
struct TwiddleRun {
  const double2* tw;
  int j;
  double2 w1, cur;
  __device__ __forceinline__ TwiddleRun(const double2* __restrict__ t, int jj) : tw(t), j(jj) {
    w1 = twd<SIGN>(tw, j);
    cur = make_double2(1.0, 0.0);
  }
  // w^(j q) for the next q (called for q = 1, 2, ... in order)
  __device__ __forceinline__ double2 next(int q) {
    cur = (q & 7) == 0 ? twd<SIGN>(tw, j * q) : (q == 1 ? w1 : cmul(cur, w1));
    return cur;
  }
};

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
// rs: doubles between the records of consecutive orders (staged: 2 nc; in
// place in rtm: the order stride of the rtm layout)
__device__ __forceinline__ double2 spec_at(const double* st, int nc, int nv, int pp, int k, int N, int L,
                                           long long rs) {
  int m;
  bool mirror;
  if (k <= L) { m = k; mirror = false; }
  else if (k >= N - L) { m = N - k; mirror = true; }
  else return make_double2(0.0, 0.0);
  const double* rec = st + m * rs;
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

// First DIF pass: input from the spectra (staged records, order stride rs =
// 2 nc; or the rtm records in place, rs = their order stride), output into z.
template <int R>
__device__ void dif_first(const double* st, int nc, int nv, double2* z, int npair, int N, int L,
                          const double2* __restrict__ tw, long long rs) {
  const int s = N / R, nbf = N / R;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, j = it % nbf;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = spec_at(st, nc, nv, pp, j + r * s, N, L, rs);
    DFT<R, +1>::run(x);
    double2* base = z + pp * N + j;
    base[0] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) base[q * s] = cmul(x[q], twd<+1>(tw, j * q));
  }
}
__device__ void dif_first_dispatch(int R, const double* st, int nc, int nv, double2* z, int npair,
                                   int N, int L, const double2* tw, long long rs = -1) {
  if (rs < 0) rs = 2LL * nc;
  switch (R) {
    case 8: dif_first<8>(st, nc, nv, z, npair, N, L, tw, rs); break;
    case 4: dif_first<4>(st, nc, nv, z, npair, N, L, tw, rs); break;
    case 2: dif_first<2>(st, nc, nv, z, npair, N, L, tw, rs); break;
    case 3: dif_first<3>(st, nc, nv, z, npair, N, L, tw, rs); break;
    default: dif_first<5>(st, nc, nv, z, npair, N, L, tw, rs); break;
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
  const double* base = rtm + rtm_off(P, 0, th, r, nc);
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
  double* base = rtm + rtm_off(P, 0, th, r, nc);
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
__global__ void __launch_bounds__(kFftThreads) k_fft_cycle(Plan P, int line0, int nlines) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npair = npb > npf ? npb : npf;
  double2* z = reinterpret_cast<double2*>(smraw);
  double* st = reinterpret_cast<double*>(z + npair * N);
  int line = line0 + blockIdx.x;
  if (line >= nlines) return;
  prefetch_line(st, P.rtm_b, P.ncb, P, line % P.nth, line / P.nth);
  while (line < nlines) {
    const int th = line % P.nth, r = line / P.nth;
    cp_async_wait<0>();
    __syncthreads();
    dif_first_dispatch(P.fac[0], st, P.ncb, P.nvb, z, npb, N, P.L, P.twid);
    __syncthreads();
    const int next = line + gridDim.x;
    if (next < nlines) prefetch_line(st, P.rtm_b, P.ncb, P, next % P.nth, next / P.nth);
    dif_rest(z, npb, N, P, P.twid);
    products<MVB, MSB, MVF, MSF>(z, N, P);
    __syncthreads();
    dit_all(z, npf, N, P, P.twid);
    store_line(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
    line = next;
  }
}

// Lines whose grid fits in shared memory but not together with the staged
// spectra of the next line (many fields, e.g. 14 + 16 components at
// Nphi = 1536: 197 KB of grid pairs): the first pass reads the line's spectra
// in place from the rtm records, everything else as k_fft_cycle.
template <int MVB, int MSB, int MVF, int MSF>
__global__ void __launch_bounds__(kFftThreads) k_fft_cycle_direct(Plan P, int line0, int nlines) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  double2* z = reinterpret_cast<double2*>(smraw);
  const long long rs = (long long)P.nth * P.nr * P.ncb * 2;
  for (int line = line0 + blockIdx.x; line < nlines; line += gridDim.x) {
    const int th = line % P.nth, r = line / P.nth;
    dif_first_dispatch(P.fac[0], P.rtm_b + rtm_off(P, 0, th, r, P.ncb), P.ncb, P.nvb, z, npb, N, P.L, P.twid, rs);
    __syncthreads();
    dif_rest(z, npb, N, P, P.twid);
    products<MVB, MSB, MVF, MSF>(z, N, P);
    __syncthreads();
    dit_all(z, npf, N, P, P.twid);
    store_line(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Wide lines (one line of every component does not fit in shared memory, e.g.
// Nphi = 3072 with 10 components): the pairs go through shared memory one at a
// time.  The cycle keeps the line's grid in a per-CTA global scratch
// (pairs x N x 16 bytes, L2-resident), forms the products there and runs the
// forward transforms pair by pair from it.

// First inverse pass of pair pp only: spectra from the staged records, output z[0 .. N).
template <int R>
__device__ void dif_first_one(const double* st, int nc, int nv, int pp, double2* z, int N, int L,
                              const double2* __restrict__ tw, long long rs) {
  const int s = N / R;
  for (int j = threadIdx.x; j < s; j += blockDim.x) {
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = spec_at(st, nc, nv, pp, j + r * s, N, L, rs);
    DFT<R, +1>::run(x);
    z[j] = x[0];
#pragma unroll
    for (int q = 1; q < R; ++q) z[j + q * s] = cmul(x[q], twd<+1>(tw, j * q));
  }
}
__device__ void dif_first_one_dispatch(int R, const double* st, int nc, int nv, int pp, double2* z, int N, int L,
                                       const double2* tw, long long rs) {
  switch (R) {
    case 8: dif_first_one<8>(st, nc, nv, pp, z, N, L, tw, rs); break;
    case 4: dif_first_one<4>(st, nc, nv, pp, z, N, L, tw, rs); break;
    case 2: dif_first_one<2>(st, nc, nv, pp, z, N, L, tw, rs); break;
    case 3: dif_first_one<3>(st, nc, nv, pp, z, N, L, tw, rs); break;
    default: dif_first_one<5>(st, nc, nv, pp, z, N, L, tw, rs); break;
  }
}
// Natural-order forward spectrum of pair q in z -> (a_m, b_m), m <= L, into rtm.
__device__ void store_one(const double2* z, int q, const Plan& P, double* rtm, int nc, int nv, int th, int r) {
  const int N = P.nph, L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  double* base = rtm + rtm_off(P, 0, th, r, nc);
  for (int m = threadIdx.x; m <= L; m += blockDim.x) {
    const double2 zm = z[m];
    double a0, b0, a1, b1;
    if (m == 0) {
      a0 = zm.x * aN; a1 = zm.y * aN; b0 = 0.0; b1 = 0.0;
    } else {
      const double2 wm = z[N - m];
      a0 = (zm.x + wm.x) * aN;
      b0 = (wm.y - zm.y) * aN;
      a1 = (zm.y + wm.y) * aN;
      b1 = (zm.x - wm.x) * aN;
    }
    double* rec = base + m * strideM;
    *reinterpret_cast<double2*>(rec + rec_off(2 * q, nv)) = make_double2(a0, b0);
    if (2 * q + 1 < nc) *reinterpret_cast<double2*>(rec + rec_off(2 * q + 1, nv)) = make_double2(a1, b1);
  }
}

template <int MVB, int MSB, int MVF, int MSF>
__global__ void __launch_bounds__(kFftThreads) k_fft_cycle_wide(Plan P, int line0, int nlines) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npm = npb > npf ? npb : npf;
  double2* z = reinterpret_cast<double2*>(smraw);
  double2* sc = P.fft_scratch + (long long)blockIdx.x * npm * N;
  // the first pass reads the line's spectra in place (rtm records, order
  // stride rs): one line of a wide grid is too large to stage, and a small
  // CTA keeps several resident per SM
  const long long rs = (long long)P.nth * P.nr * P.ncb * 2;
  for (int line = line0 + blockIdx.x; line < nlines; line += gridDim.x) {
    const int th = line % P.nth, r = line / P.nth;
    const double* st = P.rtm_b + rtm_off(P, 0, th, r, P.ncb);
    for (int pp = 0; pp < npb; ++pp) {
      dif_first_one_dispatch(P.fac[0], st, P.ncb, P.nvb, pp, z, N, P.L, P.twid, rs);
      __syncthreads();
      dif_rest(z, 1, N, P, P.twid);
      for (int i = threadIdx.x; i < N; i += blockDim.x) sc[(long long)pp * N + i] = z[i];
      __syncthreads();
    }
    products<MVB, MSB, MVF, MSF>(sc, N, P);
    __syncthreads();
    for (int q = 0; q < npf; ++q) {
      for (int i = threadIdx.x; i < N; i += blockDim.x) z[i] = sc[(long long)q * N + i];
      __syncthreads();
      dit_all(z, 1, N, P, P.twid);
      store_one(z, q, P, P.rtm_f, P.ncf, P.nvf, th, r);
      __syncthreads();
    }
  }
}

// Separable backward for wide lines: one pair at a time straight to the grid.
__global__ void __launch_bounds__(kFftThreads) k_fft_bwd_grid_wide(Plan P, double* __restrict__ fld) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npb = (P.ncb + 1) / 2;
  double2* z = reinterpret_cast<double2*>(smraw);
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  const long long nnod = (long long)P.nr * P.nth * N;
  const double* st = P.rtm_b + rtm_off(P, 0, th, r, P.ncb);  // spectra read in place
  const long long rs = (long long)P.nth * P.nr * P.ncb * 2;
  for (int pp = 0; pp < npb; ++pp) {
    dif_first_one_dispatch(P.fac[0], st, P.ncb, P.nvb, pp, z, N, P.L, P.twid, rs);
    __syncthreads();
    dif_rest(z, 1, N, P, P.twid);
    const int nc2 = 2 * pp + 1 < P.ncb ? 2 : 1;
    for (int it = threadIdx.x; it < N * nc2; it += blockDim.x) {
      const int c = it / N, pos = it % N;
      const int phi = P.digrev[pos];
      const double2 v = z[pos];
      fld[(long long)r + (long long)P.nr * (th + (long long)P.nth * phi) + nnod * (2 * pp + c)] = c ? v.y : v.x;
    }
    __syncthreads();
  }
}

// Separable forward for wide lines: one pair at a time from the grid.
__global__ void __launch_bounds__(kFftThreads) k_fft_fwd_grid_wide(Plan P, const double* __restrict__ frc) {
  extern __shared__ double4 smraw[];
  const int N = P.nph;
  const int npf = (P.ncf + 1) / 2;
  double2* z = reinterpret_cast<double2*>(smraw);
  const int line = blockIdx.x;
  const int r = line % P.nr, th = line / P.nr;
  const long long nnod = (long long)P.nr * P.nth * N;
  for (int q = 0; q < npf; ++q) {
    for (int pos = threadIdx.x; pos < N; pos += blockDim.x) {
      const int phi = P.digrev[pos];
      const long long node = (long long)r + (long long)P.nr * (th + (long long)P.nth * phi);
      const double lo = frc[node + nnod * (2 * q)];
      const double hi = (2 * q + 1 < P.ncf) ? frc[node + nnod * (2 * q + 1)] : 0.0;
      z[pos] = make_double2(lo, hi);
    }
    __syncthreads();
    dit_all(z, 1, N, P, P.twid);
    store_one(z, q, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
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
// staged records of one line: [m][ncs pairs], ncs = nc rounded up to odd
__device__ __forceinline__ int ncs_of(int nc) { return nc | 1; }

// Stages the spectra of one line (NC components, all orders) into shared
// memory with cp.async: thread t copies the 16-byte pieces of component t % NC of orders t / NC, t / NC + T / NC, ...
// (T = the largest multiple of NC not above the thread count), with pointer
// increments instead of divisions.
template <int NC>
__device__ void prefetch_line_c(double* st, const double* rtm, const Plan& P, int th, int r) {
  constexpr int NCS = NC | 1;
  const int per = blockDim.x / NC;  // orders per sweep
  if ((int)threadIdx.x < per * NC) {
    const int c = threadIdx.x % NC;
    int m = threadIdx.x / NC;
    const long long strideM = (long long)P.nth * P.nr * NC * 2;
    const double* src = rtm + rtm_off(P, m, th, r, NC) + 2 * c;
    double* dst = st + (m * NCS + c) * 2;
    const long long sstep = strideM * per;
    for (; m <= P.L; m += per, src += sstep, dst += 2 * NCS * per) cp_async16(dst, src);
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

size_t smem_cycle_f(const Plan& p) {
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  // grid pairs, alignment of the staging to 128 bytes, staged spectra, mbarrier
  return sizeof(double2) * ((size_t)npair * (p.nph + 1)) + 128 + sizeof(double) * 2 * (size_t)(p.L + 1) * (p.ncb | 1) + 16;
}

// cuTensorMapEncodeTiled, resolved through the runtime (no link-time
// dependency on the driver library, so the library also loads on hosts
// without a GPU driver); null when unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<EncodeTiledFn>(nullptr);
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Tensor map of rtm_b for the TMA staging of k_fft_cycle_f: [m][r][theta][record]
// doubles, box (2 (ncb | 1), 1, 1, mbox).  False when the orders do not split
// into whole boxes or the driver refuses the map (the kernel then uses cp.async).
bool make_rtm_map(const Plan& p, CUtensorMap* map, int* mbox) {
  const int nc = p.ncb, ncs2 = 2 * (nc | 1);
  const int mb = p.L + 1 < 256 ? p.L + 1 : 256;
  *mbox = mb;
  if ((p.L + 1) % mb != 0 || !p.rtm_b || (reinterpret_cast<uintptr_t>(p.rtm_b) & 15)) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)(2 * nc), (cuuint64_t)p.nth, (cuuint64_t)p.nr, (cuuint64_t)(p.L + 1)};
  const cuuint64_t strides[3] = {16ull * nc, 16ull * nc * p.nth, 16ull * nc * p.nth * p.nr};
  const cuuint32_t box[4] = {(cuuint32_t)ncs2, 1, 1, (cuuint32_t)mb};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(p.rtm_b), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// Fused-pass variant for N = F0 * M * 4 (F0 in {3, 6, 12, 24}, M in {4, 16}):
// inverse passes radix F0 (reading the staged spectra), radix M, radix 4; the
// last inverse radix-4 pass, the grid products and the first forward radix-4
// pass share one item (4 grid points of every component in registers), so a
// line takes five sweeps over shared memory instead of nine.  The radix-4
// passes of span 4 carry no twiddles.  Swizzle i -> i ^ (((i >> 3) ^ (i >> 6))
// & 7) inside each pair sequence (pairs N + 1 entries apart) keeps every
// quarter warp on 8 distinct 16-byte bank groups in all passes at N = 1536.
constexpr int kFftThreadsF = 384;

__host__ __device__ constexpr int ff_mid(int n) { return (n % 64 == 0 && (n / 64 == 3 || n / 64 == 6 || n / 64 == 12 || n / 64 == 24)) ? 16 : 4; }
__host__ __device__ constexpr int ff_first(int n) { return n / (4 * ff_mid(n)); }
__device__ __forceinline__ int swf(int i) { return i ^ (((i >> 3) ^ (i >> 6)) & 7); }
// 32-byte global store; p 32-byte aligned
__device__ __forceinline__ void st_v4(double* p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

// e^{2 pi i k / 48}: cos and sin of the first quadrant, k = 0..11
__host__ __device__ constexpr double c48q(int k) {
  constexpr double c[12] = {1.0, 0.9914448613738104, 0.9659258262890683, 0.9238795325112867,
                            0.8660254037844386, 0.7933533402912352, 0.7071067811865476, 0.6087614290087207,
                            0.5, 0.3826834323650898, 0.25881904510252074, 0.1305261922200516};
  return c[k];
}
// x * e^{SIGN 2 pi i e / R}, e and R compile-time, R | 48
template <int R, int E, int SIGN>
__device__ __forceinline__ double2 rot(double2 x) {
  constexpr int k = (E * (48 / R)) % 48;
  constexpr int q = k / 12, k0 = k % 12;
  if constexpr (k0 == 0) {
    // multiples of 90 degrees
    if constexpr (q == 0) return x;
    else if constexpr (q == 2) return make_double2(-x.x, -x.y);
    else if constexpr ((q == 1) == (SIGN > 0)) return make_double2(-x.y, x.x);  // * i
    else return make_double2(x.y, -x.x);                                        // * -i
  } else {
    // (c, s) of angle k * 7.5 degrees
    constexpr double c0 = c48q(k0), s0 = c48q(12 - k0);
    constexpr double c = q == 0 ? c0 : q == 1 ? -s0 : q == 2 ? -c0 : s0;
    constexpr double sn = (q == 0 ? s0 : q == 1 ? c0 : q == 2 ? -s0 : -c0) * (double)SIGN;
    return make_double2(x.x * c - x.y * sn, x.x * sn + x.y * c);
  }
}

// DFT of length A*B (Cooley-Tukey, n = B n1 + n2, k = k1 + A k2), in place.
template <int A, int B, int SIGN>
struct DFT2F {
  template <int N2, int K1>
  __device__ static void tw_one(double2* y) {
    y[N2 * A + K1] = rot<A * B, N2 * K1, SIGN>(y[N2 * A + K1]);
  }
  __device__ static void run(double2* x) {
    double2 y[A * B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      double2 t[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) t[n1] = x[B * n1 + n2];
      DFT<A, SIGN>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) y[n2 * A + k1] = t[k1];
    }
    twiddle_all(y, std::make_integer_sequence<int, A * B>{});
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      double2 t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * A + k1];
      DFT<B, SIGN>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
    }
  }
  template <int... I>
  __device__ static void twiddle_all(double2* y, std::integer_sequence<int, I...>) {
    (tw_one<I / A, I % A>(y), ...);
  }
};
template <int SIGN> struct DFT<6, SIGN> { __device__ static void run(double2* x) { DFT2F<3, 2, SIGN>::run(x); } };
template <int SIGN> struct DFT<12, SIGN> { __device__ static void run(double2* x) { DFT2F<3, 4, SIGN>::run(x); } };
template <int SIGN> struct DFT<16, SIGN> { __device__ static void run(double2* x) { DFT2F<4, 4, SIGN>::run(x); } };
template <int SIGN> struct DFT<24, SIGN> { __device__ static void run(double2* x) { DFT2F<3, 8, SIGN>::run(x); } };
template <int SIGN> struct DFT<1, SIGN> { __device__ static void run(double2*) {} };

// DFT of length 3B whose middle third of inputs (n = B .. 2B-1) is zero: the
// first-stage length-3 transforms see (x0, 0, x2).
template <int A, int B, int SIGN>
struct DFT2F_ZM;
template <int B, int SIGN>
struct DFT2F_ZM<3, B, SIGN> {
  template <int N2, int K1>
  __device__ static void tw_one(double2* y) {
    y[N2 * 3 + K1] = rot<3 * B, N2 * K1, SIGN>(y[N2 * 3 + K1]);
  }
  template <int... I>
  __device__ static void twiddle_all(double2* y, std::integer_sequence<int, I...>) {
    (tw_one<I / 3, I % 3>(y), ...);
  }
  __device__ static void run(double2* x) {
    const double s3 = 0.86602540378443864676 * (double)SIGN;
    double2 y[3 * B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      const double2 a = x[n2], c = x[2 * B + n2];
      const double2 v = make_double2(a.x - 0.5 * c.x, a.y - 0.5 * c.y);
      const double2 u = make_double2(c.y * s3, -c.x * s3);  // -(SIGN i sqrt3/2) c
      y[n2 * 3 + 0] = cadd(a, c);
      y[n2 * 3 + 1] = cadd(v, u);
      y[n2 * 3 + 2] = csub(v, u);
    }
    twiddle_all(y, std::make_integer_sequence<int, 3 * B>{});
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      double2 t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * 3 + k1];
      DFT<B, SIGN>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) x[k1 + 3 * k2] = t[k2];
    }
  }
};

// Shared-memory index of entry i of a pair sequence: swf(i).  The passes below
// compute it with the bits that are compile-time constants folded out.
//
// First inverse pass: radix F0 over the whole line (span N, stride S1 = N/F0),
// inputs from the staged spectra.  Twiddles w^(j q) are read straight from the
// table (j q < N here).  When N = 3 (L + 1) (PR), the middle third of the
// inputs (L < k < N - L) is zero and the outer thirds need no range checks.
// st: the line's records, staged (order stride 2 ncs) or, with INPLACE, the
// rtm records themselves (order stride rsg doubles)
template <int N, bool PR, bool INPLACE = false>
__device__ __forceinline__ void ff_dif_first(const double* st, int nc, int nv, double2* z, int npair, int L,
                                             const double2* __restrict__ tw, long long rsg = 0) {
  constexpr int R = ff_first(N), S1 = N / R, NP = N + 1, T3 = R / 3;
  for (int it = threadIdx.x; it < npair * S1; it += blockDim.x) {
    const int pp = it / S1, j = it - pp * S1;
    double2 x[R];
    if constexpr (PR) {
      // N = 3 (L + 1), S1 = (L + 1) / T3: input r < T3 is order m = j + r S1
      // (m = 0 only at j = r = 0); input r >= 2 T3 is the mirror of order
      // m = N - j - r S1 (m = L + 1, a zero, only at j = 0, r = 2 T3); the
      // pair's two components sit at record offsets o0, o1 (o1 < 0: none)
      const int o0 = rec_off(2 * pp, nv), o1 = 2 * pp + 1 < nc ? rec_off(2 * pp + 1, nv) : -1;
      const int rs = 2 * ncs_of(nc);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (r >= T3 && r < 2 * T3) {
          x[r] = make_double2(0.0, 0.0);
          continue;
        }
        const bool mir = r >= 2 * T3;
        const int m = mir ? N - j - r * S1 : j + r * S1;
        const double* rec = INPLACE ? st + (long long)(m <= L ? m : 0) * rsg : st + (m <= L ? m : 0) * rs;
        const double2 c0 = *reinterpret_cast<const double2*>(rec + o0);
        const double2 c1 = o1 >= 0 ? *reinterpret_cast<const double2*>(rec + o1) : make_double2(0.0, 0.0);
        if (mir) {
          x[r] = m <= L ? make_double2(0.5 * c0.x - 0.5 * c1.y, 0.5 * c0.y + 0.5 * c1.x) : make_double2(0.0, 0.0);
        } else {
          x[r] = (r == 0 && m == 0) ? make_double2(c0.x, c1.x)
                                    : make_double2(0.5 * c0.x + 0.5 * c1.y, 0.5 * c1.x - 0.5 * c0.y);
        }
      }
      DFT2F_ZM<3, T3, +1>::run(x);
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r)
        x[r] = INPLACE ? spec_at(st, nc, nv, pp, j + r * S1, N, L, rsg) : spec_at_t(st, nc, nv, pp, j + r * S1, N, L);
      DFT<R, +1>::run(x);
    }
    double2* zp = z + pp * NP;
    TwiddleRun<+1> tr(tw, j);
    if constexpr (S1 % 64 == 0) {
      const int jj = j ^ ((j >> 3) & 7);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const double2 v = q == 0 ? x[0] : cmul(x[q], tr.next(q));
        zp[(jj ^ (((q * S1) >> 6) & 7)) + q * S1] = v;
      }
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) zp[swf(j + q * S1)] = q == 0 ? x[0] : cmul(x[q], tr.next(q));
    }
  }
}

// Last forward pass (transpose of ff_dif_first): radix F0 over the whole line,
// natural-order output.  With PR only the outer thirds of the output (the
// orders 0..L and their mirrors) are stored.
template <int N, bool PR>
__device__ __forceinline__ void ff_dit_last(double2* z, int npair, const double2* __restrict__ tw) {
  constexpr int R = ff_first(N), S1 = N / R, NP = N + 1, T3 = R / 3;
  for (int it = threadIdx.x; it < npair * S1; it += blockDim.x) {
    const int pp = it / S1, j = it - pp * S1;
    double2* zp = z + pp * NP;
    double2 x[R];
    TwiddleRun<-1> tr(tw, j);
    if constexpr (S1 % 64 == 0) {
      const int jj = j ^ ((j >> 3) & 7);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const double2 v = zp[(jj ^ (((q * S1) >> 6) & 7)) + q * S1];
        x[q] = q == 0 ? v : cmul(v, tr.next(q));
      }
      DFT<R, -1>::run(x);
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (!PR || q < T3 || q >= 2 * T3) zp[(jj ^ (((q * S1) >> 6) & 7)) + q * S1] = x[q];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const double2 v = zp[swf(j + q * S1)];
        x[q] = q == 0 ? v : cmul(v, tr.next(q));
      }
      DFT<R, -1>::run(x);
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (!PR || q < T3 || q >= 2 * T3) zp[swf(j + q * S1)] = x[q];
    }
  }
}

// Middle pass of radix M over span SP = N/F0 (stride SP/M = 4): butterfly
// block b fastest across threads.  For SP = 64 the swizzle of element r is
// ((j + 4r) ^ (r/2) ^ (b % 8)) within the block, j < 4.
template <int N, int SIGN>
__device__ __forceinline__ void ff_mid_pass(double2* z, int npair, const double2* __restrict__ tw) {
  constexpr int R = ff_mid(N), SP = N / ff_first(N), s = SP / R, nbf = N / R, NB = N / SP, stw = N / SP;
  constexpr int NP = N + 1;
  for (int it = threadIdx.x; it < npair * nbf; it += blockDim.x) {
    const int pp = it / nbf, rem = it - pp * nbf;
    const int b = rem % NB, j = rem / NB;
    double2* zp = z + pp * NP + b * SP;
    double2 x[R];
    if constexpr (SP == 64 && s == 4) {
      // element e = 4r + j (j < 4): e >> 3 = r / 2, so swf gives
      // 8 (r / 2) + ((j ^ (b % 8)) ^ (r / 2) ^ 4 (r % 2))
      const int jb = j ^ (b & 7);
#define KMHD_MIDX(r) (8 * ((r) >> 1) + (jb ^ (((r) >> 1) ^ (4 * ((r) & 1)))))
      if constexpr (SIGN > 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = zp[KMHD_MIDX(r)];
        DFT<R, +1>::run(x);
#pragma unroll
        for (int q = 0; q < R; ++q) zp[KMHD_MIDX(q)] = q == 0 ? x[0] : cmul(x[q], twd<+1>(tw, j * q * stw));
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double2 v = zp[KMHD_MIDX(r)];
          x[r] = r == 0 ? v : cmul(v, twd<-1>(tw, j * r * stw));
        }
        DFT<R, -1>::run(x);
#pragma unroll
        for (int q = 0; q < R; ++q) zp[KMHD_MIDX(q)] = x[q];
      }
#undef KMHD_MIDX
    } else {
      if constexpr (SIGN > 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = z[pp * NP + swf(b * SP + j + r * s)];
        DFT<R, +1>::run(x);
#pragma unroll
        for (int q = 0; q < R; ++q)
          z[pp * NP + swf(b * SP + j + q * s)] = q == 0 ? x[0] : cmul(x[q], twd<+1>(tw, j * q * stw));
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double2 v = z[pp * NP + swf(b * SP + j + r * s)];
          x[r] = r == 0 ? v : cmul(v, twd<-1>(tw, j * r * stw));
        }
        DFT<R, -1>::run(x);
#pragma unroll
        for (int q = 0; q < R; ++q) z[pp * NP + swf(b * SP + j + q * s)] = x[q];
      }
    }
  }
}

// Grid products of one grid point: vin = backward components (3 MVB vector
// components, then MSB scalars, as laid out in the pairs), out = forward
// components in pair order.
template <int MVB, int MSB, int MVF, int MSF>
__device__ __forceinline__ void point_products(const double* vin_all, const Plan& P, double* dense) {
  constexpr int MCF = 3 * MVF + MSF;
  const int nvb = P.nvb, nvf = P.nvf, nsf = P.nsf;
  double vin[3 * MVB > 0 ? 3 * MVB : 1], sin_[MSB > 0 ? MSB : 1];
#pragma unroll
  for (int c = 0; c < 3 * MVB; ++c) vin[c] = vin_all[c];
#pragma unroll
  for (int q = 0; q < MSB; ++q) sin_[q] = vin_all[3 * nvb + q < 3 * MVB + MSB ? 3 * nvb + q : 0];
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
}

// Products of the standard MHD set at one grid point: backward (u, omega, B; T),
// forward (omega x u, u x B, u T; u . omega), coefficients from the plan.
__device__ __forceinline__ void point_products_mhd(const double* v, const Plan& P, double* o) {
  const double u0 = v[0], u1 = v[1], u2 = v[2], w0 = v[3], w1 = v[4], w2 = v[5];
  const double b0 = v[6], b1 = v[7], b2 = v[8], t = v[9];
  const double c0 = P.pcoef[0], c1 = P.pcoef[1], c2 = P.pcoef[2], c3 = P.pcoef[3];
  o[0] = (w1 * u2 - w2 * u1) * c0;
  o[1] = (w2 * u0 - w0 * u2) * c0;
  o[2] = (w0 * u1 - w1 * u0) * c0;
  o[3] = (u1 * b2 - u2 * b1) * c1;
  o[4] = (u2 * b0 - u0 * b2) * c1;
  o[5] = (u0 * b1 - u1 * b0) * c1;
  o[6] = u0 * t * c2;
  o[7] = u1 * t * c2;
  o[8] = u2 * t * c2;
  o[9] = (u0 * w0 + u1 * w1 + u2 * w2) * c3;
}

// Last inverse radix-4 pass + products + first forward radix-4 pass, for the
// grid points 4b .. 4b+3 of every pair.
template <int N, int MVB, int MSB, int MVF, int MSF, int PK>
__device__ __forceinline__ void ff_fused(double2* z, const Plan& P) {
  constexpr int NP = N + 1;
  constexpr int MCB = 3 * MVB + MSB, MCF = 3 * MVF + MSF;
  constexpr int NPB = (MCB + 1) / 2, NPF = (MCF + 1) / 2;
  constexpr int NPM = NPB > NPF ? NPB : NPF;
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2, ncb = P.ncb, ncf = P.ncf;
  for (int b = threadIdx.x; b < N / 4; b += blockDim.x) {
    const int e0 = (4 * b) ^ (((b >> 1) ^ (b >> 4)) & 7);  // swf(4b + r) = e0 ^ r
    double2 v[NPM][4];
#pragma unroll
    for (int pp = 0; pp < NPB; ++pp) {
      if (pp < npb) {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[pp][r] = z[pp * NP + (e0 ^ r)];
        DFT<4, +1>::run(v[pp]);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double vin[MCB > 0 ? MCB : 1], dense[MCF > 0 ? MCF : 1];
#pragma unroll
      for (int c = 0; c < MCB; ++c) vin[c] = (c < ncb) ? ((c & 1) ? v[c >> 1][r].y : v[c >> 1][r].x) : 0.0;
      if constexpr (PK == 1) point_products_mhd(vin, P, dense);
      else point_products<MVB, MSB, MVF, MSF>(vin, P, dense);
#pragma unroll
      for (int q = 0; q < NPF; ++q)
        v[q][r] = make_double2(2 * q < ncf ? dense[2 * q] : 0.0, 2 * q + 1 < ncf ? dense[2 * q + 1 < MCF ? 2 * q + 1 : 0] : 0.0);
    }
#pragma unroll
    for (int q = 0; q < NPF; ++q) {
      if (q < npf) {
        DFT<4, -1>::run(v[q]);
#pragma unroll
        for (int r = 0; r < 4; ++r) z[q * NP + (e0 ^ r)] = v[q][r];
      }
    }
  }
}

template <int N>
__device__ void ff_store_line(const double2* z, int npair, const Plan& P, double* rtm, int nc, int nv, int th, int r) {
  constexpr int NP = N + 1;
  const int L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * nc * 2;
  double* base = rtm + rtm_off(P, 0, th, r, nc);
  for (int it = threadIdx.x; it < (L + 1) * npair; it += blockDim.x) {
    const int pp = it / (L + 1), m = it - pp * (L + 1);
    const double2* zp = z + pp * NP;
    const double2 zm = zp[swf(m)];
    double a0, b0, a1, b1;
    if (m == 0) {
      a0 = zm.x * aN; a1 = zm.y * aN; b0 = 0.0; b1 = 0.0;
    } else {
      const double2 wm = zp[swf(N - m)];
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

// Store of the line's forward spectra, one thread per order m writing the
// whole rtm record (every component's (cos, sin) pair, assembled in registers)
// as 32-byte stores: each record sector is written once, by one store.  The
// record holds NC = 3 MVF + MSF pairs (NC even: 16 NC bytes, a multiple of 32).
template <int N, int MVF, int MSF>
__device__ void ff_store_records(const double2* z, const Plan& P, double* rtm, int th, int r) {
  constexpr int NP = N + 1;
  constexpr int NC = 3 * MVF + MSF, NPF = (NC + 1) / 2;
  static_assert(NC % 2 == 0, "32-byte record stores need an even component count");
  const int L = P.L;
  const double aN = 1.0 / (double)N;
  const long long strideM = (long long)P.nth * P.nr * NC * 2;
  double* base = rtm + rtm_off(P, 0, th, r, NC);
  for (int m = threadIdx.x; m <= L; m += blockDim.x) {
    double rec[2 * NC];
    const int im = swf(m), iw = swf(N - m);
#pragma unroll
    for (int pp = 0; pp < NPF; ++pp) {
      const double2* zp = z + pp * NP;
      const double2 zm = zp[im];
      double a0, b0, a1, b1;
      if (m == 0) {
        a0 = zm.x * aN; a1 = zm.y * aN; b0 = 0.0; b1 = 0.0;
      } else {
        const double2 wm = zp[iw];
        a0 = (zm.x + wm.x) * aN;
        b0 = (wm.y - zm.y) * aN;
        a1 = (zm.y + wm.y) * aN;
        b1 = (zm.x - wm.x) * aN;
      }
      rec[rec_off(2 * pp, MVF)] = a0;
      rec[rec_off(2 * pp, MVF) + 1] = b0;
      rec[rec_off(2 * pp + 1, MVF)] = a1;
      rec[rec_off(2 * pp + 1, MVF) + 1] = b1;
    }
    double* dst = base + m * strideM;
#pragma unroll
    for (int q = 0; q < 2 * NC; q += 4) st_v4(dst + q, rec[q], rec[q + 1], rec[q + 2], rec[q + 3]);
  }
}

// Staging of the next line's spectra: with a tensor map (tma != 0) thread 0
// issues one TMA tensor load per mbox orders: the map views rtm_b as
// [m][r][theta][record] doubles with a box of (2 ncs, 1, 1, mbox), the two
// doubles past each record zero-filled, which lands the records at the
// conflict-free stride 2 ncs that the first pass reads; completion on an
// mbarrier with a bounded wait.  Otherwise 16-byte cp.async pieces.
// NT threads: fewer threads leave more registers to each for the fused
// products of many fields (the unstaged variants)
template <int N, int MVB, int MSB, int MVF, int MSF, bool PR, int PK, bool STG = true, int NT = kFftThreadsF>
__global__ void __launch_bounds__(NT, 1)
    k_fft_cycle_f(Plan P, int line0, int nlines, const __grid_constant__ CUtensorMap tmap, int tma, int mbox) {
  extern __shared__ double4 smraw[];
  constexpr int NP = N + 1;
  constexpr int NCB = 3 * MVB + MSB, NCS2 = 2 * (NCB | 1);
  const int npb = (P.ncb + 1) / 2, npf = (P.ncf + 1) / 2;
  const int npair = npb > npf ? npb : npf;
  double2* z = reinterpret_cast<double2*>(smraw);
  // staged spectra, 128-byte aligned (TMA destination), then the mbarrier
  double* st = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(z + npair * NP) + 127) & ~static_cast<uintptr_t>(127));
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(st + (P.L + 1) * NCS2);
  int line = line0 + blockIdx.x;
  if (line >= nlines) return;
  if constexpr (!STG) {
    // only the grid fits in shared memory: the first pass reads the line's
    // records in place (order stride nth nr ncb 2)
    const long long rsg = (long long)P.nth * P.nr * P.ncb * 2;
    for (; line < nlines; line += gridDim.x) {
      const int th = line % P.nth, r = line / P.nth;
      ff_dif_first<N, PR, true>(P.rtm_b + rtm_off(P, 0, th, r, P.ncb), P.ncb, P.nvb, z, npb, P.L, P.twid, rsg);
      __syncthreads();
      ff_mid_pass<N, +1>(z, npb, P.twid);
      __syncthreads();
      ff_fused<N, MVB, MSB, MVF, MSF, PK>(z, P);
      __syncthreads();
      ff_mid_pass<N, -1>(z, npf, P.twid);
      __syncthreads();
      ff_dit_last<N, PR>(z, npf, P.twid);
      __syncthreads();
      if constexpr ((3 * MVF + MSF) % 2 == 0) ff_store_records<N, MVF, MSF>(z, P, P.rtm_f, th, r);
      else ff_store_line<N>(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
      __syncthreads();
    }
    return;
  }
  if (tma && threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(ssa(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  auto stage = [&](int ln) {
    const int sth = ln % P.nth, sr = ln / P.nth;
    if (!tma) {
      prefetch_line_c<NCB>(st, P.rtm_b, P, sth, sr);
    } else if (threadIdx.x == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(ssa(bar)),
                   "r"((unsigned)((P.L + 1) * NCS2 * 8)));
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the first pass's reads of st
      for (int m0 = 0; m0 <= P.L; m0 += mbox)
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
            "[%6];\n" ::"r"(ssa(st + m0 * NCS2)),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(0), "r"(sth), "r"(sr), "r"(m0), "r"(ssa(bar))
            : "memory");
    }
  };
  __syncthreads();
  // lines theta fastest: concurrent CTAs touch neighbouring records of one (m, r)
  stage(line);
  unsigned phase = 0;
  while (line < nlines) {
    const int th = line % P.nth, r = line / P.nth;
    if (tma) {
      const bool late = !fbar_wait(bar, phase);
      phase ^= 1u;
      if (__syncthreads_or(late)) {
        // the staging did not complete in time: report it, let the copy land, stop
        if (threadIdx.x == 0) {
          if (P.err) atomicExch(P.err, KMHD_ERR_TIMEOUT);
          (void)fbar_wait(bar, phase ^ 1u);
        }
        return;
      }
    } else {
      cp_async_wait<0>();
      __syncthreads();
    }
    ff_dif_first<N, PR>(st, P.ncb, P.nvb, z, npb, P.L, P.twid);
    __syncthreads();
    const int next = line + gridDim.x;
    if (next < nlines) stage(next);
    ff_mid_pass<N, +1>(z, npb, P.twid);
    __syncthreads();
    ff_fused<N, MVB, MSB, MVF, MSF, PK>(z, P);
    __syncthreads();
    ff_mid_pass<N, -1>(z, npf, P.twid);
    __syncthreads();
    ff_dit_last<N, PR>(z, npf, P.twid);
    __syncthreads();
    if constexpr ((3 * MVF + MSF) % 2 == 0) ff_store_records<N, MVF, MSF>(z, P, P.rtm_f, th, r);
    else ff_store_line<N>(z, npf, P, P.rtm_f, P.ncf, P.nvf, th, r);
    __syncthreads();
    line = next;
  }
}

template <int N, int MVB, int MSB, int MVF, int MSF, bool PR, int PK, bool STG = true, int NT = kFftThreadsF>
cudaError_t run_cycle_fk(const Plan& p, cudaStream_t s) {
  auto kern = k_fft_cycle_f<N, MVB, MSB, MVF, MSF, PR, PK, STG, NT>;
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  const size_t smem = STG ? smem_cycle_f(p) : sizeof(double2) * (size_t)npair * (N + 1);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, smem);
  if (occ < 1) occ = 1;
  // lines (r, theta) of the radial window, theta fastest
  const int line0 = p.r_lo * p.nth, nlines = p.r_hi * p.nth;
  int grid = nsm * occ;
  if (grid > nlines - line0) grid = nlines - line0;
  if (grid <= 0) return cudaSuccess;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  int mbox = 1;
  const int tma = STG && make_rtm_map(p, &map, &mbox) ? 1 : 0;
  kern<<<grid, NT, smem, s>>>(p, line0, nlines, map, tma, mbox);
  return cudaGetLastError();
}

// The specialised passes without staging (the first pass reads the records in
// place), for lines whose grid fits in shared memory but not with the staged
// spectra; generic products.
template <int N, int MVB, int MSB, int MVF, int MSF, int NT = kFftThreadsF>
cudaError_t run_cycle_fu(const Plan& p, cudaStream_t s) {
  const bool pr = p.nph == 3 * (p.L + 1);
  return pr ? run_cycle_fk<N, MVB, MSB, MVF, MSF, true, 0, false, NT>(p, s)
            : run_cycle_fk<N, MVB, MSB, MVF, MSF, false, 0, false, NT>(p, s);
}

// the standard MHD product list, after the vectors-first reordering
inline bool is_mhd_products(const Plan& p) {
  if (p.nvb != 3 || p.nsb != 1 || p.nvf != 3 || p.nsf != 1 || p.nprod != 4) return false;
  const int k[4] = {KMHD_PROD_CROSS, KMHD_PROD_CROSS, KMHD_PROD_VEC_SCALAR, KMHD_PROD_DOT};
  const int a[4] = {1, 0, 0, 0}, b[4] = {0, 2, 0, 1};
  for (int i = 0; i < 4; ++i)
    if (p.pkind[i] != k[i] || p.pa[i] != a[i] || p.pb[i] != b[i]) return false;
  return true;
}

template <int N, int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_f(const Plan& p, cudaStream_t s) {
  const bool pr = p.nph == 3 * (p.L + 1);
  if constexpr (MVB == 3 && MSB == 1 && MVF == 3 && MSF == 1) {
    if (is_mhd_products(p))
      return pr ? run_cycle_fk<N, MVB, MSB, MVF, MSF, true, 1>(p, s) : run_cycle_fk<N, MVB, MSB, MVF, MSF, false, 1>(p, s);
  }
  return pr ? run_cycle_fk<N, MVB, MSB, MVF, MSF, true, 0>(p, s) : run_cycle_fk<N, MVB, MSB, MVF, MSF, false, 0>(p, s);
}

template <int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_n(const Plan& p, cudaStream_t s, bool* handled) {
  *handled = true;
  if (smem_cycle_f(p) <= 227 * 1024) {
    switch (p.nph) {
      case 96: return run_cycle_f<96, MVB, MSB, MVF, MSF>(p, s);
      case 192: return run_cycle_f<192, MVB, MSB, MVF, MSF>(p, s);
      case 384: return run_cycle_f<384, MVB, MSB, MVF, MSF>(p, s);
      case 768: return run_cycle_f<768, MVB, MSB, MVF, MSF>(p, s);
      case 1536: return run_cycle_f<1536, MVB, MSB, MVF, MSF>(p, s);
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
  const int line0 = p.r_lo * p.nth, nlines = p.r_hi * p.nth;
  int grid = nsm * occ;
  if (grid > nlines - line0) grid = nlines - line0;
  if (grid <= 0) return cudaSuccess;
  kern<<<grid, kFftThreads, smem, s>>>(p, line0, nlines);
  return cudaGetLastError();
}

// Failure-path self-test: the staging wait on an mbarrier that nothing
// completes runs out and records KMHD_ERR_TIMEOUT; the kernel returns.
__global__ void k_selftest_fft_wait(int* err) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(ssa(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !fbar_wait(&bar, 0, kSelfTestSpinCap)) atomicExch(err, KMHD_ERR_TIMEOUT);
}

}  // namespace

cudaError_t launch_selftest_fft_wait(int* err, cudaStream_t s) {
  k_selftest_fft_wait<<<1, 32, 0, s>>>(err);
  return cudaGetLastError();
}

bool fft_line_fits(const Plan& p) {
  return smem_cycle(p) <= 227 * 1024 || smem_cycle_f(p) <= 227 * 1024;
}

size_t fft_smem_bytes(const Plan& p, int npair) {
  (void)npair;
  return smem_cycle(p);
}

size_t smem_wide(const Plan& p) { return sizeof(double2) * (size_t)p.nph; }

size_t smem_direct(const Plan& p) {
  const int npair = ((p.ncb > p.ncf ? p.ncb : p.ncf) + 1) / 2;
  return sizeof(double2) * (size_t)npair * p.nph;
}

template <int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_direct(const Plan& p, cudaStream_t s) {
  auto kern = k_fft_cycle_direct<MVB, MSB, MVF, MSF>;
  const size_t smem = smem_direct(p);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kFftThreads, smem);
  if (occ < 1) occ = 1;
  const int line0 = p.r_lo * p.nth, nlines = p.r_hi * p.nth;
  int grid = nsm * occ;
  if (grid > nlines - line0) grid = nlines - line0;
  if (grid <= 0) return cudaSuccess;
  kern<<<grid, kFftThreads, smem, s>>>(p, line0, nlines);
  return cudaGetLastError();
}

template <int MVB, int MSB, int MVF, int MSF>
cudaError_t run_cycle_wide(const Plan& p, cudaStream_t s) {
  auto kern = k_fft_cycle_wide<MVB, MSB, MVF, MSF>;
  const size_t smem = smem_wide(p);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (!p.fft_scratch) return cudaErrorInvalidValue;
  const int line0 = p.r_lo * p.nth, nlines = p.r_hi * p.nth;
  const int grid = std::min(p.fft_scratch_ctas, nlines - line0);
  if (grid <= 0) return cudaSuccess;
  kern<<<grid, kFftThreads, smem, s>>>(p, line0, nlines);
  return cudaGetLastError();
}

cudaError_t launch_fft_cycle(const Plan& p, cudaStream_t s) {
  if (smem_cycle(p) > 227 * 1024 && smem_cycle_f(p) > 227 * 1024) {
    // the specialised passes need (N + 1)-strided pairs: at most 16 pairs more
    if (smem_direct(p) + 16 * 16 <= 227 * 1024) {
      // the reference's full MHD set (u, omega, B, J + T, C -> five vectors + one scalar) at its own counts
      if (p.nph == 1536 && p.nvb == 4 && p.nsb == 2 && p.nvf == 5 && p.nsf == 1)
        return run_cycle_fu<1536, 4, 2, 5, 1>(p, s);
      // the dynamo benchmark set (u, omega, B, J + T -> omega x u, J x B, u x B, u T)
      if (p.nph == 1536 && p.nvb == 4 && p.nsb == 1 && p.nvf == 4 && p.nsf == 0)
        return run_cycle_fu<1536, 4, 1, 4, 0, 256>(p, s);  // 256 threads: 71.8 against 78.8 ms at L=511
      if (p.nph == 1536) return run_cycle_fu<1536, kMaxVec, kMaxScl, kMaxVec, kMaxScl>(p, s);
      if (p.nph == 768) return run_cycle_fu<768, kMaxVec, kMaxScl, kMaxVec, kMaxScl>(p, s);
    }
    if (smem_direct(p) <= 227 * 1024) return run_cycle_direct<kMaxVec, kMaxScl, kMaxVec, kMaxScl>(p, s);
    if (p.nvb == 3 && p.nsb == 1 && p.nvf == 3 && p.nsf == 1) return run_cycle_wide<3, 1, 3, 1>(p, s);
    return run_cycle_wide<kMaxVec, kMaxScl, kMaxVec, kMaxScl>(p, s);
  }
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
  if (smem > 227 * 1024) {
    const size_t sw = smem_wide(p);
    cudaError_t e = cudaFuncSetAttribute(k_fft_bwd_grid_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
    if (e != cudaSuccess) return e;
    k_fft_bwd_grid_wide<<<p.nr * p.nth, kFftThreads, sw, s>>>(p, fld);
    return cudaGetLastError();
  }
  cudaError_t e = cudaFuncSetAttribute(k_fft_bwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_fft_bwd_grid<<<p.nr * p.nth, kFftThreads, smem, s>>>(p, fld);
  return cudaGetLastError();
}

cudaError_t launch_fft_fwd_grid(const Plan& p, const double* frc, cudaStream_t s) {
  const int npf = (p.ncf + 1) / 2;
  const size_t smem = sizeof(double2) * (size_t)npf * p.nph;
  if (smem > 227 * 1024) {
    const size_t sw = sizeof(double2) * (size_t)p.nph;
    cudaError_t e = cudaFuncSetAttribute(k_fft_fwd_grid_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw);
    if (e != cudaSuccess) return e;
    k_fft_fwd_grid_wide<<<p.nr * p.nth, kFftThreads, sw, s>>>(p, frc);
    return cudaGetLastError();
  }
  cudaError_t e = cudaFuncSetAttribute(k_fft_fwd_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_fft_fwd_grid<<<p.nr * p.nth, kFftThreads, smem, s>>>(p, frc);
  return cudaGetLastError();
}

}  // namespace kmhd
