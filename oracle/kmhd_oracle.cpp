// kmhd_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU FP64 restatement of Calypso's spherical-transform cycle as the
// reference computes it on the host with the `symmetric_BLAS` Legendre
// variant (flag 11), OpenMP over flattened (field, radius) blocks and one
// single-threaded DGEMM per thread.  Used by tests/ as the parity oracle and
// by bench.py as the timed CPU baseline.  Nothing in the product links it.
//
// Parity status: UNPINNED against the reference's own outputs.  The reference
// is Fortran 90 and no Fortran compiler exists here; its tree stores no golden
// vectors for this path.  This restatement is pinned instead by mathematical
// invariants (Gauss quadrature exactness, Schmidt orthogonality, fwd(bwd(S))=S,
// analytic single modes) and by independent implementations (scipy Gauss
// nodes and associated Legendre functions) in tests/.
//
// Reference files followed (paths relative to MHD/Fortran_src/):
//   Gauss nodes/weights ....... CORE_src/gauss_integration/gauss_integration.f90:60-133
//   Schmidt P_l^m, dP/dtheta .. CORE_src/spherical_harmonics/schmidt_fix_m.f90:62-175
//   P table on the rtm grid ... CORE_src/SPH_SPECTR_src/schmidt_poly_on_rtm_grid.f90:145-197
//   normalisation g(j,1:17) ... CORE_src/spherical_harmonics/spherical_harmonics.f90:91-140
//                               + l=0 override schmidt_poly_on_rtm_grid.f90:109
//   m stacks .................. PARALLEL_src/SPH_SHELL_src/set_params_sph_trans.f90:64-137
//   even/odd stacks, Ps tables  PARALLEL_src/SPH_SHELL_src/set_legendre_matrices.f90:64-130
//   j / m orderings ........... PARALLEL_src/CONST_SPH_GRID/set_sph_tranform_ordering.f90:64-206
//   bwd driver ................ PARALLEL_src/SPH_SHELL_src/legendre_bwd_sym_matmul.f90:301-426, 430-500
//   bwd pack .................. PARALLEL_src/SPH_SHELL_src/set_sp_rlm_for_leg_matmul.f90:153-276
//   bwd unpack ................ PARALLEL_src/SPH_SHELL_src/cal_vr_rtm_by_matmul.f90:163-352
//   DGEMM semantics ........... PARALLEL_src/SPH_SHELL_src/matmul_for_legendre_trans.F90:144-169, 265-294
//   FFT convention ............ PARALLEL_src/SPH_SHELL_src/t_sph_single_FFTW.F90 (fwd/bwd normalisation)
//                               and t_sph_FFTPACK5.f90:183-331 (slot order a0, a_N/2, a1, b1, ...)
//   grid products ............. MHD_src/sph_MHD/cal_nonlinear_sph_MHD.f90:64-128,
//                               CORE_src/BASE/cal_products_smp.f90:153-172
//   fwd driver ................ PARALLEL_src/SPH_SHELL_src/legendre_fwd_sym_matmul.f90:315-452
//   fwd pack .................. PARALLEL_src/SPH_SHELL_src/set_vr_rtm_for_leg_matmul.f90:170-364
//   fwd unpack ................ PARALLEL_src/SPH_SHELL_src/cal_sp_rlm_by_matmul.f90:172-360
//
// Indices are 64-bit throughout: the reference's int32 buffer offsets
// (ncomp*nnod) overflow at L=511, Nr=257, 10 components.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <complex>
#include <omp.h>

namespace {

typedef long long i64;
typedef void (*fortran_dgemm64_t)(const char*, const char*, const i64*, const i64*,
                                  const i64*, const double*, const double*, const i64*,
                                  const double*, const i64*, const double*, double*,
                                  const i64*, long, long);

fortran_dgemm64_t g_ext_dgemm = nullptr;

// C(m x n) = A(m x k) * B(k x n), column-major, beta = 0.
void dgemm_nn(i64 m, i64 n, i64 k, const double* A, i64 lda, const double* B,
              i64 ldb, double* C, i64 ldc) {
  if (m <= 0 || n <= 0) return;
  if (k <= 0) {
    for (i64 j = 0; j < n; ++j)
      for (i64 i = 0; i < m; ++i) C[i + j * ldc] = 0.0;
    return;
  }
  if (g_ext_dgemm) {
    const double one = 1.0, zero = 0.0;
    g_ext_dgemm("N", "N", &m, &n, &k, &one, A, &lda, B, &ldb, &zero, C, &ldc, 1, 1);
    return;
  }
  // Blocked column-major kernel: 4 columns of C at a time, axpy over rows.
  const i64 KB = 128;
  for (i64 j = 0; j < n; ++j)
    for (i64 i = 0; i < m; ++i) C[i + j * ldc] = 0.0;
  for (i64 k0 = 0; k0 < k; k0 += KB) {
    const i64 k1 = std::min(k, k0 + KB);
    i64 j = 0;
    for (; j + 4 <= n; j += 4) {
      double* c0 = C + (j + 0) * ldc;
      double* c1 = C + (j + 1) * ldc;
      double* c2 = C + (j + 2) * ldc;
      double* c3 = C + (j + 3) * ldc;
      for (i64 kk = k0; kk < k1; ++kk) {
        const double b0 = B[kk + (j + 0) * ldb], b1 = B[kk + (j + 1) * ldb];
        const double b2 = B[kk + (j + 2) * ldb], b3 = B[kk + (j + 3) * ldb];
        const double* a = A + kk * lda;
#pragma omp simd
        for (i64 i = 0; i < m; ++i) {
          const double av = a[i];
          c0[i] += av * b0;
          c1[i] += av * b1;
          c2[i] += av * b2;
          c3[i] += av * b3;
        }
      }
    }
    for (; j < n; ++j) {
      double* c0 = C + j * ldc;
      for (i64 kk = k0; kk < k1; ++kk) {
        const double b0 = B[kk + j * ldb];
        const double* a = A + kk * lda;
#pragma omp simd
        for (i64 i = 0; i < m; ++i) c0[i] += a[i] * b0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Complex FFT (mixed radix 2/3/4/5, iterative Stockham), written from the DFT
// definition; used only to evaluate the FFTPACK real-transform convention.
struct CFFT {
  int n = 0;
  std::vector<int> radix;
  // per stage: twiddles e^{-2 pi i j r / (l R)}, j < l, 1 <= r < R, laid out [j][r-1]
  std::vector<std::vector<std::complex<double>>> stw;
  void init(int n_) {
    n = n_;
    radix.clear();
    int r = n;
    while (r % 4 == 0) { radix.push_back(4); r /= 4; }
    while (r % 2 == 0) { radix.push_back(2); r /= 2; }
    while (r % 3 == 0) { radix.push_back(3); r /= 3; }
    while (r % 5 == 0) { radix.push_back(5); r /= 5; }
    if (r != 1) radix.push_back(r);  // generic DFT stage for any leftover prime
    stw.clear();
    int l = 1;
    for (int R : radix) {
      std::vector<std::complex<double>> t((size_t)l * (R - 1));
      for (int j = 0; j < l; ++j)
        for (int q = 1; q < R; ++q) {
          const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)j * q / (long double)(l * R);
          t[(size_t)j * (R - 1) + (q - 1)] = std::complex<double>((double)cosl(a), (double)sinl(a));
        }
      stw.push_back(std::move(t));
      l *= R;
    }
  }
  // sign = -1: forward e^{-i}, sign = +1: inverse e^{+i}; unnormalised.
  // Stockham autosort: stage input viewed as [R][m][l], output as [m][R][l].
  void run(std::complex<double>* x, std::complex<double>* work, int sign) const {
    std::complex<double>* src = x;
    std::complex<double>* dst = work;
    int l = 1, m = n;
    for (size_t s = 0; s < radix.size(); ++s) {
      const int R = radix[s];
      m /= R;
      const std::complex<double>* tw = stw[s].data();
      for (int q = 0; q < m; ++q) {
        for (int j = 0; j < l; ++j) {
          std::complex<double> in[64];
          for (int r = 0; r < R; ++r) {
            std::complex<double> v = src[j + l * (q + m * r)];
            if (r > 0) {
              std::complex<double> w = tw[(size_t)j * (R - 1) + (r - 1)];
              if (sign > 0) w = std::conj(w);
              v *= w;
            }
            in[r] = v;
          }
          std::complex<double>* out = dst + j + l * (R * q);
          if (R == 2) {
            out[0] = in[0] + in[1];
            out[l] = in[0] - in[1];
          } else if (R == 4) {
            const std::complex<double> a = in[0] + in[2], b = in[0] - in[2];
            const std::complex<double> c = in[1] + in[3];
            const std::complex<double> d = (in[1] - in[3]) * std::complex<double>(0.0, (double)sign);
            out[0] = a + c;
            out[l] = b + d;
            out[2 * l] = a - c;
            out[3 * l] = b - d;
          } else if (R == 3) {
            const double s3 = 0.86602540378443864676 * (double)sign;
            const std::complex<double> t = in[1] + in[2];
            const std::complex<double> u = (in[1] - in[2]) * std::complex<double>(0.0, s3);
            const std::complex<double> v = in[0] - 0.5 * t;
            out[0] = in[0] + t;
            out[l] = v + u;
            out[2 * l] = v - u;
          } else {
            for (int p = 0; p < R; ++p) {
              std::complex<double> acc = 0.0;
              for (int r = 0; r < R; ++r) {
                const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)((r * p) % R) / R;
                acc += in[r] * std::complex<double>((double)cosl(a), (double)(sign * sinl(a)));
              }
              out[p * l] = acc;
            }
          }
        }
      }
      l *= R;
      std::swap(src, dst);
    }
    if (src != x) std::memcpy(x, src, sizeof(std::complex<double>) * n);
  }
};

struct Product { int kind, a, b; double coef; };

struct Oracle {
  int L = 0, nth = 0, nph = 0, nr = 0, nh = 0, nlo = 0;
  int nvb = 0, nsb = 0, nvf = 0, nsf = 0, ncb = 0, ncf = 0;
  int nthreads = 1;
  i64 J = 0, nmslot = 0;
  std::vector<double> radius, ar_1d;                // r, 1/r
  std::vector<double> gpoint, colat, weight, asin_t;
  std::vector<i64> lstack, lstack_even;             // size nmslot+1 (0-based start per slot)
  std::vector<int> jl, jm;                          // rlm j -> (l, m)
  std::vector<double> g3, g6, g7;
  std::vector<double> P_rtm, dP_rtm;                // [j * nth + i]
  std::vector<double> Ps, dPs;                      // [j * nh + i]  (even-then-odd per m slot)
  std::vector<Product> prods;
  CFFT fft;
};

// gauss_integration.f90:60-133.  Only the last n of the reference's n-loop
// survives (each n overwrites all n points), so that n alone is evaluated.
void gauss_points(int n_point, std::vector<double>& w_point, std::vector<double>& w_coefs) {
  w_point.assign(n_point, 0.0);
  w_coefs.assign(n_point, 0.0);
  const double pi = 4.0 * std::atan(1.0);
  const double x1 = 0.0, x2 = 1.0;
  if (n_point == 1) { w_point[0] = 0.5; w_coefs[0] = 1.0; }
  else {
    const int n = n_point;
    const int m = (n + 1 - (n + 1) % 2) / 2;
    const double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
    for (int i = 1; i <= m; ++i) {
      double z = std::cos(pi * ((double)i - 0.25) / ((double)n + 0.5));
      double pp, z1, p1, p2, p3;
      for (;;) {
        p1 = 1.0; p2 = 0.0;
        for (int j = 1; j <= n; ++j) {
          p3 = p2; p2 = p1;
          p1 = ((2.0 * (double)j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
        }
        pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
        z1 = z;
        z = z1 - p1 / pp;
        if (std::fabs(z - z1) < 3.0e-12) break;
      }
      w_point[i - 1] = xm - xl * z;
      w_point[n - i] = xm + xl * z;
      w_coefs[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
      w_coefs[n - i] = w_coefs[i - 1];
    }
  }
  for (int i = 0; i < n_point; ++i) {
    w_point[i] = w_point[i] * 2.0 - 1.0;
    w_coefs[i] = w_coefs[i] * 2.0;
  }
}

// schmidt_fix_m.f90:86-139 (p has ltr+1 entries, df ltr+3).
void schmidt_legendre_m(int ltr, int m, double theta, double* p, double* df) {
  if (m < 0) {
    for (int l = 0; l <= ltr; ++l) p[l] = 0.0;
  } else if (m == 0) {
    p[0] = 1.0;
    p[1] = std::cos(theta);
    for (int l = 2; l <= ltr; ++l)
      p[l] = p[l - 1] * (double)(2 * l - 1) / (double)l * std::cos(theta) -
             p[l - 2] * (double)(l - 1) / (double)l;
  } else {
    df[m] = 1.0;
    for (int k = 1; k <= m; ++k) df[m] = df[m] * (double)(2 * k - 1) / (double)(2 * k);
    df[m + 1] = std::sqrt(2.0 * df[m] * (double)(2 * m + 1)) * std::cos(theta);
    df[m] = std::sqrt(2.0 * df[m]);
    if (m < ltr - 1) {
      for (int l = m + 2; l <= ltr; ++l)
        df[l] = (std::cos(theta) * (double)(2 * l - 1) * df[l - 1] -
                 std::sqrt((double)((l - 1) * (l - 1) - m * m)) * df[l - 2]) /
                std::sqrt((double)(l * l - m * m));
    }
    for (int l = m; l <= ltr; ++l) {
      p[l] = df[l];
      for (int m1 = 1; m1 <= m; ++m1) p[l] = p[l] * std::sin(theta);
    }
  }
}

// schmidt_fix_m.f90:143-175
void diff_schmidt_legendre_m(int ltr, int m, const double* pmn1, const double* pmp1, double* dp) {
  if (m == 0) {
    dp[0] = 0.0;
    for (int l = 1; l <= ltr; ++l) dp[l] = -std::sqrt((double)(l * (l + 1) / 2)) * pmp1[l];
  } else if (m == 1) {
    dp[1] = pmn1[1];
    for (int l = 2; l <= ltr; ++l)
      dp[l] = 0.5 * (std::sqrt((double)(2 * l * (l + 1))) * pmn1[l] -
                     std::sqrt((double)((l - 1) * (l + 2))) * pmp1[l]);
  } else {
    dp[m] = 0.5 * std::sqrt((double)(2 * m)) * pmn1[m];
    for (int l = m + 1; l <= ltr; ++l)
      dp[l] = 0.5 * (std::sqrt((double)((l + m) * (l - m + 1))) * pmn1[l] -
                     std::sqrt((double)((l - m) * (l + m + 1))) * pmp1[l]);
  }
}

void build_tables(Oracle& o) {
  const int L = o.L;
  o.nh = (o.nth + 1) / 2;
  o.nlo = o.nth / 2;
  o.nmslot = 2 * L + 1;
  o.J = (i64)(L + 1) * (L + 1);
  o.ar_1d.resize(o.nr);
  for (int k = 0; k < o.nr; ++k) o.ar_1d[k] = 1.0 / o.radius[k];
  gauss_points(o.nth, o.gpoint, o.weight);
  o.colat.resize(o.nth);
  o.asin_t.resize(o.nth);
  for (int i = 0; i < o.nth; ++i) {
    o.colat[i] = std::acos(o.gpoint[i]);
    o.asin_t[i] = 1.0 / std::sin(o.colat[i]);  // set_params_sph_trans.f90:141-157
  }
  // m slots: m = -L..L (single domain, set_zonal_wavenum_4_legendre); j: per slot, l = |m|..L
  o.lstack.assign(o.nmslot + 1, 0);
  o.lstack_even.assign(o.nmslot + 1, 0);
  o.jl.resize(o.J);
  o.jm.resize(o.J);
  i64 j = 0;
  for (i64 ms = 0; ms < o.nmslot; ++ms) {
    const int m = (int)ms - L;
    const int am = std::abs(m);
    o.lstack[ms + 1] = o.lstack[ms] + (L - am + 1);
    const i64 nj = o.lstack[ms + 1] - o.lstack[ms];
    o.lstack_even[ms + 1] = o.lstack[ms] + (nj + 1) / 2;
    for (int l = am; l <= L; ++l) { o.jl[j] = l; o.jm[j] = m; ++j; }
  }
  o.g3.resize(o.J); o.g6.resize(o.J); o.g7.resize(o.J);
  for (i64 jj = 0; jj < o.J; ++jj) {
    const int l = o.jl[jj], m = o.jm[jj];
    o.g3[jj] = (double)(l * (l + 1));
    if (l == 0 && m == 0) {
      o.g6[jj] = 1.0 / 2.0;
      o.g7[jj] = 1.0;
      o.g3[jj] = 0.5;  // schmidt_poly_on_rtm_grid.f90:109
    } else if (m == 0) {
      o.g6[jj] = (double)(2 * l + 1) / 2.0;
      o.g7[jj] = (double)(2 * l + 1) / (double)(2 * l * (l + 1));
    } else {
      o.g6[jj] = (double)(2 * l + 1) / 4.0;
      o.g7[jj] = (double)(2 * l + 1) / (double)(4 * l * (l + 1));
    }
  }
  // P_rtm(theta, j), dPdt_rtm(theta, j)  (schmidt_poly_on_rtm_grid.f90:145-197)
  o.P_rtm.assign((size_t)o.J * o.nth, 0.0);
  o.dP_rtm.assign((size_t)o.J * o.nth, 0.0);
#pragma omp parallel num_threads(o.nthreads)
  {
    std::vector<double> p(L + 1), dp(L + 1), pmn1(L + 1), pmp1(L + 1), df(L + 3);
#pragma omp for schedule(static)
    for (int i = 0; i < o.nth; ++i) {
      for (i64 ms = 0; ms < o.nmslot; ++ms) {
        const int mm = std::abs((int)ms - L);
        schmidt_legendre_m(L, mm - 1, o.colat[i], pmn1.data(), df.data());
        schmidt_legendre_m(L, mm, o.colat[i], p.data(), df.data());
        schmidt_legendre_m(L, mm + 1, o.colat[i], pmp1.data(), df.data());
        diff_schmidt_legendre_m(L, mm, pmn1.data(), pmp1.data(), dp.data());
        for (i64 jj = o.lstack[ms]; jj < o.lstack[ms + 1]; ++jj) {
          const int l = o.jl[jj];
          o.P_rtm[(size_t)jj * o.nth + i] = p[l];
          o.dP_rtm[(size_t)jj * o.nth + i] = dp[l];
        }
      }
    }
  }
  // Hemisphere tables, even-then-odd per slot (set_legendre_matrices.f90:86-130)
  o.Ps.assign((size_t)o.J * o.nh, 0.0);
  o.dPs.assign((size_t)o.J * o.nh, 0.0);
  for (i64 ms = 0; ms < o.nmslot; ++ms) {
    const i64 jst = o.lstack[ms];
    const i64 ne = o.lstack_even[ms + 1] - o.lstack[ms];
    const i64 no = o.lstack[ms + 1] - o.lstack_even[ms + 1];
    for (i64 e = 0; e < ne; ++e) {
      const i64 jr = jst + 2 * e;
      for (int i = 0; i < o.nh; ++i) {
        o.Ps[(size_t)(jst + e) * o.nh + i] = o.P_rtm[(size_t)jr * o.nth + i];
        o.dPs[(size_t)(jst + e) * o.nh + i] = o.dP_rtm[(size_t)jr * o.nth + i];
      }
    }
    for (i64 q = 0; q < no; ++q) {
      const i64 jr = jst + 2 * q + 1;
      for (int i = 0; i < o.nh; ++i) {
        o.Ps[(size_t)(jst + ne + q) * o.nh + i] = o.P_rtm[(size_t)jr * o.nth + i];
        o.dPs[(size_t)(jst + ne + q) * o.nh + i] = o.dP_rtm[(size_t)jr * o.nth + i];
      }
    }
  }
  o.fft.init(o.nph);
}

// Partition of the flattened (field, radius) index space into nthreads blocks,
// as istack_rtm_kr_smp * nfield does in the reference.
void kr_block(const Oracle& o, int nfield, int ip, i64& kst, i64& nkr) {
  const i64 nr = o.nr;
  const i64 q = nr / o.nthreads, rem = nr % o.nthreads;
  const i64 ist = ip * q + std::min<i64>(ip, rem);
  const i64 ied = ist + q + (ip < rem ? 1 : 0);
  kst = (i64)nfield * ist;
  nkr = (i64)nfield * (ied - ist);
}

// sp_rlm[(j + J*k) * ncb + comp]; rtm[((ms*nr + k)*nth + i) * ncb + comp]
void leg_bwd(const Oracle& o, const double* sp, double* rtm) {
  const int nc = o.ncb;
  const i64 nnod_rtm = (i64)o.nth * o.nr * o.nmslot;
  std::memset(rtm, 0, sizeof(double) * nnod_rtm * nc);
  const int nl = o.nh;
  auto rtm_at = [&](int i, i64 k, i64 ms) -> i64 { return ((ms * o.nr + k) * o.nth + i) * nc; };
#pragma omp parallel num_threads(o.nthreads)
  {
    const int ip = omp_get_thread_num();
    const i64 maxk = (o.L + 2) / 2;
    // ---- vectors (legendre_bwd_sym_matmul.f90:301-426)
    if (o.nvb > 0) {
      i64 kst, nkr;
      kr_block(o, o.nvb, ip, kst, nkr);
      std::vector<double> pol_e(maxk * nkr), dpoldt_e(maxk * nkr), dpoldp_e(maxk * nkr),
          dtordt_e(maxk * nkr), dtordp_e(maxk * nkr), pol_o(maxk * nkr), dpoldt_o(maxk * nkr),
          dpoldp_o(maxk * nkr), dtordt_o(maxk * nkr), dtordp_o(maxk * nkr);
      std::vector<double> symp_r(nl * nkr), asmp_t(nl * nkr), asmp_p(nl * nkr), symn_t(nl * nkr),
          symn_p(nl * nkr), asmp_r(nl * nkr), symp_t(nl * nkr), symp_p(nl * nkr),
          asmn_t(nl * nkr), asmn_p(nl * nkr);
      for (i64 mp = 0; mp < o.nmslot && nkr > 0; ++mp) {
        const i64 mn = o.nmslot - 1 - mp;
        const i64 jst = o.lstack[mp];
        const i64 ne = o.lstack_even[mp + 1] - o.lstack[mp];
        const i64 no = o.lstack[mp + 1] - o.lstack_even[mp + 1];
        // pack (set_sp_rlm_for_leg_matmul.f90:153-229)
        for (i64 kk = 0; kk < nkr; ++kk) {
          const i64 kr_nd = kk + kst;
          const i64 k = kr_nd % o.nr;
          const i64 nd = kr_nd / o.nr;
          const double a1r = o.ar_1d[k];
          const double a2r = o.ar_1d[k] * o.ar_1d[k];
          for (i64 jj = 0; jj < ne; ++jj) {
            const i64 j = jst + 2 * jj;
            const double g3 = o.g3[j], gm = (double)o.jm[j];
            const double* w = sp + ((j + o.J * k) * nc + 3 * nd);
            pol_e[jj + ne * kk] = w[0] * a2r * g3;
            dpoldt_e[jj + ne * kk] = w[1] * a1r;
            dpoldp_e[jj + ne * kk] = w[1] * a1r * gm;
            dtordt_e[jj + ne * kk] = w[2] * a1r;
            dtordp_e[jj + ne * kk] = w[2] * a1r * gm;
          }
          for (i64 jj = 0; jj < no; ++jj) {
            const i64 j = jst + 2 * jj + 1;
            const double g3 = o.g3[j], gm = (double)o.jm[j];
            const double* w = sp + ((j + o.J * k) * nc + 3 * nd);
            pol_o[jj + no * kk] = w[0] * a2r * g3;
            dpoldt_o[jj + no * kk] = w[1] * a1r;
            dpoldp_o[jj + no * kk] = w[1] * a1r * gm;
            dtordt_o[jj + no * kk] = w[2] * a1r;
            dtordp_o[jj + no * kk] = w[2] * a1r * gm;
          }
        }
        const double* Pe = o.Ps.data() + (size_t)jst * nl;
        const double* dPe = o.dPs.data() + (size_t)jst * nl;
        const double* Po = o.Ps.data() + (size_t)(jst + ne) * nl;
        const double* dPo = o.dPs.data() + (size_t)(jst + ne) * nl;
        dgemm_nn(nl, nkr, ne, Pe, nl, pol_e.data(), ne, symp_r.data(), nl);
        dgemm_nn(nl, nkr, ne, dPe, nl, dpoldt_e.data(), ne, asmp_t.data(), nl);
        dgemm_nn(nl, nkr, ne, dPe, nl, dtordt_e.data(), ne, asmp_p.data(), nl);
        dgemm_nn(nl, nkr, ne, Pe, nl, dtordp_e.data(), ne, symn_t.data(), nl);
        dgemm_nn(nl, nkr, ne, Pe, nl, dpoldp_e.data(), ne, symn_p.data(), nl);
        dgemm_nn(nl, nkr, no, Po, nl, pol_o.data(), no, asmp_r.data(), nl);
        dgemm_nn(nl, nkr, no, dPo, nl, dpoldt_o.data(), no, symp_t.data(), nl);
        dgemm_nn(nl, nkr, no, dPo, nl, dtordt_o.data(), no, symp_p.data(), nl);
        dgemm_nn(nl, nkr, no, Po, nl, dtordp_o.data(), no, asmn_t.data(), nl);
        dgemm_nn(nl, nkr, no, Po, nl, dpoldp_o.data(), no, asmn_p.data(), nl);
        // unpack (cal_vr_rtm_by_matmul.f90:163-286)
        for (i64 kk = 0; kk < nkr; ++kk)
          for (int lp = 0; lp < nl; ++lp) {
            const i64 q = lp + nl * kk;
            symn_t[q] = -symn_t[q] * o.asin_t[lp];
            symn_p[q] = -symn_p[q] * o.asin_t[lp];
            asmn_t[q] = -asmn_t[q] * o.asin_t[lp];
            asmn_p[q] = -asmn_p[q] * o.asin_t[lp];
          }
        for (i64 kk = 0; kk < nkr; ++kk) {
          const i64 kr_nd = kk + kst;
          const i64 k = kr_nd % o.nr;
          const i64 nd = kr_nd / o.nr;
          for (int lp = 0; lp < o.nth / 2; ++lp) {
            const int ln = o.nth - 1 - lp;
            const i64 q = lp + nl * kk;
            double* ipp = rtm + rtm_at(lp, k, mp) + 3 * nd;
            double* inp = rtm + rtm_at(lp, k, mn) + 3 * nd;
            double* ipn = rtm + rtm_at(ln, k, mp) + 3 * nd;
            double* inn = rtm + rtm_at(ln, k, mn) + 3 * nd;
            ipp[0] = ipp[0] + symp_r[q] + asmp_r[q];
            ipp[1] = ipp[1] + asmp_t[q] + symp_t[q];
            ipp[2] = ipp[2] - asmp_p[q] - symp_p[q];
            inp[1] = inp[1] + symn_t[q] + asmn_t[q];
            inp[2] = inp[2] + symn_p[q] + asmn_p[q];
            ipn[0] = ipn[0] + symp_r[q] - asmp_r[q];
            ipn[1] = ipn[1] - asmp_t[q] + symp_t[q];
            ipn[2] = ipn[2] + asmp_p[q] - symp_p[q];
            inn[1] = inn[1] + symn_t[q] - asmn_t[q];
            inn[2] = inn[2] + symn_p[q] - asmn_p[q];
          }
          for (int lp = o.nth / 2; lp < nl; ++lp) {
            const i64 q = lp + nl * kk;
            double* ipp = rtm + rtm_at(lp, k, mp) + 3 * nd;
            double* inp = rtm + rtm_at(lp, k, mn) + 3 * nd;
            ipp[0] = ipp[0] + symp_r[q];
            ipp[1] = ipp[1] + symp_t[q];
            ipp[2] = ipp[2] - symp_p[q];
            inp[1] = inp[1] + symn_t[q];
            inp[2] = inp[2] + symn_p[q];
          }
        }
      }
    }
#pragma omp barrier
    // ---- scalars (legendre_bwd_sym_matmul.f90:430-500)
    if (o.nsb > 0) {
      i64 kst, nkr;
      kr_block(o, o.nsb, ip, kst, nkr);
      std::vector<double> scl_e(maxk * nkr), scl_o(maxk * nkr), symp(nl * nkr), asmp(nl * nkr);
      for (i64 mp = 0; mp < o.nmslot && nkr > 0; ++mp) {
        const i64 jst = o.lstack[mp];
        const i64 ne = o.lstack_even[mp + 1] - o.lstack[mp];
        const i64 no = o.lstack[mp + 1] - o.lstack_even[mp + 1];
        for (i64 kk = 0; kk < nkr; ++kk) {
          const i64 kr_nd = kk + kst;
          const i64 k = kr_nd % o.nr;
          const i64 nd = kr_nd / o.nr;
          for (i64 jj = 0; jj < ne; ++jj)
            scl_e[jj + ne * kk] = sp[(jst + 2 * jj + o.J * k) * nc + 3 * o.nvb + nd];
          for (i64 jj = 0; jj < no; ++jj)
            scl_o[jj + no * kk] = sp[(jst + 2 * jj + 1 + o.J * k) * nc + 3 * o.nvb + nd];
        }
        dgemm_nn(nl, nkr, ne, o.Ps.data() + (size_t)jst * nl, nl, scl_e.data(), ne, symp.data(), nl);
        dgemm_nn(nl, nkr, no, o.Ps.data() + (size_t)(jst + ne) * nl, nl, scl_o.data(), no, asmp.data(), nl);
        for (i64 kk = 0; kk < nkr; ++kk) {
          const i64 kr_nd = kk + kst;
          const i64 k = kr_nd % o.nr;
          const i64 nd = kr_nd / o.nr;
          for (int lp = 0; lp < o.nth / 2; ++lp) {
            const int ln = o.nth - 1 - lp;
            const i64 q = lp + nl * kk;
            double* ipp = rtm + rtm_at(lp, k, mp) + 3 * o.nvb + nd;
            double* ipn = rtm + rtm_at(ln, k, mp) + 3 * o.nvb + nd;
            ipp[0] = ipp[0] + symp[q] + asmp[q];
            ipn[0] = ipn[0] + symp[q] - asmp[q];
          }
          for (int lp = o.nth / 2; lp < nl; ++lp) {
            const i64 q = lp + nl * kk;
            double* ipp = rtm + rtm_at(lp, k, mp) + 3 * o.nvb + nd;
            ipp[0] = ipp[0] + symp[q];
          }
        }
      }
    }
  }
}

// rtm (grid, cos/sin per m slot) -> sp_rlm, forward symmetric Legendre.
void leg_fwd(const Oracle& o, const double* rtm, double* sp) {
  const int nc = o.ncf;
  std::memset(sp, 0, sizeof(double) * o.J * o.nr * nc);
  const int nle = o.nh, nlo = o.nlo;
  auto rtm_at = [&](int i, i64 k, i64 ms) -> i64 { return ((ms * o.nr + k) * o.nth + i) * nc; };
#pragma omp parallel num_threads(o.nthreads)
  {
    const int ip = omp_get_thread_num();
    const i64 maxk = (o.L + 2) / 2;
    if (o.nvf > 0) {
      i64 kst, nkr;
      kr_block(o, o.nvf, ip, kst, nkr);
      std::vector<double> symp_r(nkr * nle), asmp_t(nkr * nle), asmp_p(nkr * nle),
          symn_t(nkr * nle), symn_p(nkr * nle), asmp_r(nkr * nle), symp_t(nkr * nle),
          symp_p(nkr * nle), asmn_t(nkr * nle), asmn_p(nkr * nle);
      std::vector<double> pol_e(maxk * nkr), dpoldt_e(maxk * nkr), dpoldp_e(maxk * nkr),
          dtordt_e(maxk * nkr), dtordp_e(maxk * nkr), pol_o(maxk * nkr), dpoldt_o(maxk * nkr),
          dpoldp_o(maxk * nkr), dtordt_o(maxk * nkr), dtordp_o(maxk * nkr);
      for (i64 mp = 0; mp < o.nmslot && nkr > 0; ++mp) {
        const i64 mn = o.nmslot - 1 - mp;
        const i64 jst = o.lstack[mp];
        const i64 ne = o.lstack_even[mp + 1] - o.lstack[mp];
        const i64 no = o.lstack[mp + 1] - o.lstack_even[mp + 1];
        // pack (set_vr_rtm_for_leg_matmul.f90:170-291)
        for (int lp = 0; lp < nlo; ++lp) {
          const int ln = o.nth - 1 - lp;
          const double wp = o.weight[lp], as = o.asin_t[lp];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 kr_nd = kk + kst;
            const i64 k = kr_nd % o.nr;
            const i64 nd = kr_nd / o.nr;
            const double* pp = rtm + rtm_at(lp, k, mp) + 3 * nd;
            const double* pn = rtm + rtm_at(ln, k, mp) + 3 * nd;
            const double* np_ = rtm + rtm_at(lp, k, mn) + 3 * nd;
            const double* nn = rtm + rtm_at(ln, k, mn) + 3 * nd;
            const i64 q = kk + nkr * lp;
            symp_r[q] = (pp[0] + pn[0]) * wp;
            symp_t[q] = (pp[1] + pn[1]) * wp;
            symp_p[q] = (pp[2] + pn[2]) * wp;
            asmp_r[q] = (pp[0] - pn[0]) * wp;
            asmp_t[q] = (pp[1] - pn[1]) * wp;
            asmp_p[q] = (pp[2] - pn[2]) * wp;
            symn_t[q] = (np_[1] + nn[1]) * wp * as;
            symn_p[q] = (np_[2] + nn[2]) * wp * as;
            asmn_t[q] = (np_[1] - nn[1]) * wp * as;
            asmn_p[q] = (np_[2] - nn[2]) * wp * as;
          }
        }
        for (int lp = nlo; lp < nle; ++lp) {
          const double wp = o.weight[lp], as = o.asin_t[lp];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 kr_nd = kk + kst;
            const i64 k = kr_nd % o.nr;
            const i64 nd = kr_nd / o.nr;
            const double* pp = rtm + rtm_at(lp, k, mp) + 3 * nd;
            const double* np_ = rtm + rtm_at(lp, k, mn) + 3 * nd;
            const i64 q = kk + nkr * lp;
            symp_r[q] = pp[0] * wp;
            symp_t[q] = pp[1] * wp;
            symp_p[q] = pp[2] * wp;
            asmp_r[q] = 0.0; asmp_t[q] = 0.0; asmp_p[q] = 0.0;
            symn_t[q] = np_[1] * wp * as;
            symn_p[q] = np_[2] * wp * as;
            asmn_t[q] = 0.0; asmn_p[q] = 0.0;
          }
        }
        const double* Pe = o.Ps.data() + (size_t)jst * nle;
        const double* dPe = o.dPs.data() + (size_t)jst * nle;
        const double* Po = o.Ps.data() + (size_t)(jst + ne) * nle;
        const double* dPo = o.dPs.data() + (size_t)(jst + ne) * nle;
        dgemm_nn(nkr, ne, nle, symp_r.data(), nkr, Pe, nle, pol_e.data(), nkr);
        dgemm_nn(nkr, ne, nle, asmp_t.data(), nkr, dPe, nle, dpoldt_e.data(), nkr);
        dgemm_nn(nkr, ne, nle, symn_p.data(), nkr, Pe, nle, dpoldp_e.data(), nkr);
        dgemm_nn(nkr, ne, nle, symn_t.data(), nkr, Pe, nle, dtordp_e.data(), nkr);
        dgemm_nn(nkr, ne, nle, asmp_p.data(), nkr, dPe, nle, dtordt_e.data(), nkr);
        dgemm_nn(nkr, no, nle, asmp_r.data(), nkr, Po, nle, pol_o.data(), nkr);
        dgemm_nn(nkr, no, nle, symp_t.data(), nkr, dPo, nle, dpoldt_o.data(), nkr);
        dgemm_nn(nkr, no, nle, asmn_p.data(), nkr, Po, nle, dpoldp_o.data(), nkr);
        dgemm_nn(nkr, no, nle, asmn_t.data(), nkr, Po, nle, dtordp_o.data(), nkr);
        dgemm_nn(nkr, no, nle, symp_p.data(), nkr, dPo, nle, dtordt_o.data(), nkr);
        // unpack (cal_sp_rlm_by_matmul.f90:172-292)
        for (i64 jj = 0; jj < ne; ++jj) {
          const i64 j = jst + 2 * jj;
          const double g7 = o.g7[j], gm = (double)o.jm[j];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 k = (kk + kst) % o.nr;
            const double r1 = o.radius[k], r2 = r1 * r1;
            const i64 q = kk + jj * nkr;
            pol_e[q] = pol_e[q] * r2 * g7;
            dpoldt_e[q] = dpoldt_e[q] * r1 * g7;
            dpoldp_e[q] = dpoldp_e[q] * r1 * g7 * gm;
            dtordt_e[q] = dtordt_e[q] * r1 * g7;
            dtordp_e[q] = dtordp_e[q] * r1 * g7 * gm;
          }
        }
        for (i64 jj = 0; jj < no; ++jj) {
          const i64 j = jst + 2 * jj + 1;
          const double g7 = o.g7[j], gm = (double)o.jm[j];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 k = (kk + kst) % o.nr;
            const double r1 = o.radius[k], r2 = r1 * r1;
            const i64 q = kk + jj * nkr;
            pol_o[q] = pol_o[q] * r2 * g7;
            dpoldt_o[q] = dpoldt_o[q] * r1 * g7;
            dpoldp_o[q] = dpoldp_o[q] * r1 * g7 * gm;
            dtordt_o[q] = dtordt_o[q] * r1 * g7;
            dtordp_o[q] = dtordp_o[q] * r1 * g7 * gm;
          }
        }
        for (i64 jj = 0; jj < ne; ++jj) {
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 kr_nd = kk + kst;
            const i64 k = kr_nd % o.nr;
            const i64 nd = kr_nd / o.nr;
            const i64 q = kk + jj * nkr;
            double* ie = sp + ((jst + 2 * jj) + o.J * k) * nc + 3 * nd;
            ie[0] = ie[0] + pol_e[q];
            ie[1] = ie[1] - dpoldp_e[q] + dpoldt_e[q];
            ie[2] = ie[2] - dtordp_e[q] - dtordt_e[q];
            if (jj < no) {
              double* io = sp + ((jst + 2 * jj + 1) + o.J * k) * nc + 3 * nd;
              io[0] = io[0] + pol_o[q];
              io[1] = io[1] - dpoldp_o[q] + dpoldt_o[q];
              io[2] = io[2] - dtordp_o[q] - dtordt_o[q];
            }
          }
        }
      }
    }
#pragma omp barrier
    if (o.nsf > 0) {
      i64 kst, nkr;
      kr_block(o, o.nsf, ip, kst, nkr);
      std::vector<double> symp(nkr * nle), asmp(nkr * nle), scl_e(maxk * nkr), scl_o(maxk * nkr);
      for (i64 mp = 0; mp < o.nmslot && nkr > 0; ++mp) {
        const i64 jst = o.lstack[mp];
        const i64 ne = o.lstack_even[mp + 1] - o.lstack[mp];
        const i64 no = o.lstack[mp + 1] - o.lstack_even[mp + 1];
        for (int lp = 0; lp < nlo; ++lp) {
          const int ln = o.nth - 1 - lp;
          const double wp = o.weight[lp];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 kr_nd = kk + kst;
            const i64 k = kr_nd % o.nr;
            const i64 nd = kr_nd / o.nr;
            const double a = rtm[rtm_at(lp, k, mp) + 3 * o.nvf + nd];
            const double b = rtm[rtm_at(ln, k, mp) + 3 * o.nvf + nd];
            symp[kk + nkr * lp] = (a + b) * wp;
            asmp[kk + nkr * lp] = (a - b) * wp;
          }
        }
        for (int lp = nlo; lp < nle; ++lp) {
          const double wp = o.weight[lp];
          for (i64 kk = 0; kk < nkr; ++kk) {
            const i64 kr_nd = kk + kst;
            const i64 k = kr_nd % o.nr;
            const i64 nd = kr_nd / o.nr;
            symp[kk + nkr * lp] = rtm[rtm_at(lp, k, mp) + 3 * o.nvf + nd] * wp;
            asmp[kk + nkr * lp] = 0.0;
          }
        }
        dgemm_nn(nkr, ne, nle, symp.data(), nkr, o.Ps.data() + (size_t)jst * nle, nle, scl_e.data(), nkr);
        dgemm_nn(nkr, no, nle, asmp.data(), nkr, o.Ps.data() + (size_t)(jst + ne) * nle, nle, scl_o.data(), nkr);
        for (i64 jj = 0; jj < ne; ++jj) {
          const double g6 = o.g6[jst + 2 * jj];
          for (i64 kk = 0; kk < nkr; ++kk) scl_e[kk + jj * nkr] = scl_e[kk + jj * nkr] * g6;
        }
        for (i64 jj = 0; jj < no; ++jj) {
          const double g6 = o.g6[jst + 2 * jj + 1];
          for (i64 kk = 0; kk < nkr; ++kk) scl_o[kk + jj * nkr] = scl_o[kk + jj * nkr] * g6;
        }
        for (i64 kk = 0; kk < nkr; ++kk) {
          const i64 kr_nd = kk + kst;
          const i64 k = kr_nd % o.nr;
          const i64 nd = kr_nd / o.nr;
          for (i64 jj = 0; jj < ne; ++jj) {
            sp[((jst + 2 * jj) + o.J * k) * nc + 3 * o.nvf + nd] += scl_e[kk + jj * nkr];
            if (jj < no) sp[((jst + 2 * jj + 1) + o.J * k) * nc + 3 * o.nvf + nd] += scl_o[kk + jj * nkr];
          }
        }
      }
    }
  }
}

// rtm (slots m=-L..L: cos for m>=0, sin for -m) -> rtp grid, per (r, theta, comp).
// Backward real FFT with the FFTPACK/FFTW-wrapper convention:
//   x_j = a0 + sum_{k=1}^{N/2-1} (a_k cos(2 pi jk/N) + b_k sin(2 pi jk/N))
// fld[(k + nr*(i + nth*p)) + nnod*comp].  Work is blocked per latitude so the
// grid is touched radius-contiguously, as FFTPACK's multiple-sequence RFFTMB
// processes consecutive (r, theta) sequences together.
void fft_bwd(const Oracle& o, const double* rtm, int nc, double* fld) {
  const i64 N = o.nph, nnod = (i64)o.nr * o.nth * N;
  const int np = (nc + 1) / 2;
#pragma omp parallel num_threads(o.nthreads)
  {
    std::vector<std::complex<double>> buf((size_t)o.nr * np * N), w(N);
#pragma omp for schedule(static)
    for (int i = 0; i < o.nth; ++i) {
      for (int k = 0; k < o.nr; ++k)
        for (int pp = 0; pp < np; ++pp) {
          std::complex<double>* z = buf.data() + ((size_t)k * np + pp) * N;
          for (i64 q = 0; q < N; ++q) z[q] = 0.0;
          const int c0 = 2 * pp;
          const bool two = (c0 + 1 < nc);
          for (int m = 0; m <= o.L && m < N / 2; ++m) {
            const i64 msp = o.L + m, msn = o.L - m;
            for (int t = 0; t < (two ? 2 : 1); ++t) {
              const int c = c0 + t;
              const double a = rtm[((msp * o.nr + k) * o.nth + i) * nc + c];
              const double b = (m == 0) ? 0.0 : rtm[((msn * o.nr + k) * o.nth + i) * nc + c];
              std::complex<double> X = (m == 0) ? std::complex<double>(a, 0.0)
                                                : std::complex<double>(0.5 * a, -0.5 * b);
              const std::complex<double> f = (t == 0) ? std::complex<double>(1, 0) : std::complex<double>(0, 1);
              z[m] += f * X;
              if (m > 0) z[N - m] += f * std::conj(X);
            }
          }
          o.fft.run(z, w.data(), +1);
        }
      for (int c = 0; c < nc; ++c)
        for (i64 p = 0; p < N; ++p) {
          double* dst = fld + (i64)o.nr * (i + (i64)o.nth * p) + nnod * c;
          for (int k = 0; k < o.nr; ++k) {
            const std::complex<double> v = buf[((size_t)k * np + c / 2) * N + p];
            dst[k] = (c & 1) ? v.imag() : v.real();
          }
        }
    }
  }
}

// rtp grid -> rtm slots (m <= L kept).  a0 = (1/N) sum x, a_k = (2/N) sum x cos,
// b_k = (2/N) sum x sin.
void fft_fwd(const Oracle& o, const double* frc, int nc, double* rtm) {
  const i64 N = o.nph, nnod = (i64)o.nr * o.nth * N;
  const int np = (nc + 1) / 2;
  std::memset(rtm, 0, sizeof(double) * (i64)o.nth * o.nr * o.nmslot * nc);
#pragma omp parallel num_threads(o.nthreads)
  {
    std::vector<std::complex<double>> buf((size_t)o.nr * np * N), w(N);
#pragma omp for schedule(static)
    for (int i = 0; i < o.nth; ++i) {
      for (int pp = 0; pp < np; ++pp)
        for (i64 p = 0; p < N; ++p) {
          const double* s0 = frc + (i64)o.nr * (i + (i64)o.nth * p) + nnod * (2 * pp);
          const double* s1 = s0 + nnod;
          const bool two = (2 * pp + 1 < nc);
          for (int k = 0; k < o.nr; ++k)
            buf[((size_t)k * np + pp) * N + p] = std::complex<double>(s0[k], two ? s1[k] : 0.0);
        }
      const double aN = 1.0 / (double)N;
      for (int k = 0; k < o.nr; ++k)
        for (int pp = 0; pp < np; ++pp) {
          std::complex<double>* z = buf.data() + ((size_t)k * np + pp) * N;
          o.fft.run(z, w.data(), -1);
          const int c0 = 2 * pp;
          const bool two = (c0 + 1 < nc);
          for (int m = 0; m <= o.L && m < N / 2; ++m) {
            const std::complex<double> zp = z[m], zm = std::conj(z[(N - m) % N]);
            const std::complex<double> X0 = 0.5 * (zp + zm);
            const std::complex<double> X1 = std::complex<double>(0, -0.5) * (zp - zm);
            for (int t = 0; t < (two ? 2 : 1); ++t) {
              const std::complex<double> X = (t == 0) ? X0 : X1;
              const int c = c0 + t;
              const i64 msp = o.L + m, msn = o.L - m;
              if (m == 0) {
                rtm[((msp * o.nr + k) * o.nth + i) * nc + c] = aN * X.real();
              } else {
                rtm[((msp * o.nr + k) * o.nth + i) * nc + c] = 2.0 * aN * X.real();
                rtm[((msn * o.nr + k) * o.nth + i) * nc + c] = -2.0 * aN * X.imag();
              }
            }
          }
        }
    }
  }
}

// cal_nonlinear_sph_MHD.f90:64-128 with cal_products_smp.f90.
void products(const Oracle& o, const double* fld, double* frc) {
  const i64 nnod = (i64)o.nr * o.nth * o.nph;
  int iv = 0, is = 0;
  for (const Product& p : o.prods) {
    if (p.kind == 0 || p.kind == 1) {
      double* out = frc + nnod * (3 * iv);
      ++iv;
      const double* a = fld + nnod * (3 * p.a);
#pragma omp parallel for num_threads(o.nthreads) schedule(static)
      for (i64 n = 0; n < nnod; ++n) {
        if (p.kind == 0) {
          const double* b = fld + nnod * (3 * p.b);
          out[n] = (a[n + nnod] * b[n + 2 * nnod] - a[n + 2 * nnod] * b[n + nnod]) * p.coef;
          out[n + nnod] = (a[n + 2 * nnod] * b[n] - a[n] * b[n + 2 * nnod]) * p.coef;
          out[n + 2 * nnod] = (a[n] * b[n + nnod] - a[n + nnod] * b[n]) * p.coef;
        } else {
          const double s = fld[n + nnod * (3 * o.nvb + p.b)];
          out[n] = a[n] * s * p.coef;
          out[n + nnod] = a[n + nnod] * s * p.coef;
          out[n + 2 * nnod] = a[n + 2 * nnod] * s * p.coef;
        }
      }
    }
  }
  for (const Product& p : o.prods) {
    if (p.kind == 2 || p.kind == 3) {
      double* out = frc + nnod * (3 * o.nvf + is);
      ++is;
#pragma omp parallel for num_threads(o.nthreads) schedule(static)
      for (i64 n = 0; n < nnod; ++n) {
        if (p.kind == 2) {
          const double* a = fld + nnod * (3 * p.a);
          const double* b = fld + nnod * (3 * p.b);
          out[n] = (a[n] * b[n] + a[n + nnod] * b[n + nnod] + a[n + 2 * nnod] * b[n + 2 * nnod]) * p.coef;
        } else {
          out[n] = fld[n + nnod * (3 * o.nvb + p.a)] * fld[n + nnod * (3 * o.nvb + p.b)] * p.coef;
        }
      }
    }
  }
}

}  // namespace

extern "C" {

// Use an external Fortran-ABI (64-bit integer) DGEMM, e.g. OpenBLAS, as the
// reference does with -DBLAS; NULL restores the built-in blocked kernel.
void oracle_set_dgemm(void* fn) { g_ext_dgemm = (fortran_dgemm64_t)fn; }

void* oracle_create(int L, int nth, int nph, int nr, const double* radius, int nvb,
                    int nsb, int nvf, int nsf, int nprod, const int* prod_kind,
                    const int* prod_a, const int* prod_b, const double* prod_coef,
                    int nthreads) {
  Oracle* o = new Oracle();
  o->L = L; o->nth = nth; o->nph = nph; o->nr = nr;
  o->nvb = nvb; o->nsb = nsb; o->nvf = nvf; o->nsf = nsf;
  o->ncb = 3 * nvb + nsb; o->ncf = 3 * nvf + nsf;
  o->nthreads = nthreads > 0 ? nthreads : 1;
  o->radius.assign(radius, radius + nr);
  for (int i = 0; i < nprod; ++i) o->prods.push_back({prod_kind[i], prod_a[i], prod_b[i], prod_coef[i]});
  build_tables(*o);
  return o;
}

void oracle_destroy(void* h) { delete (Oracle*)h; }

long long oracle_J(void* h) { return ((Oracle*)h)->J; }

// Test-only: replace the reference's weights (P'_n evaluated at the previous
// Newton iterate, ~1e-12 relative error) by 2/((1-x^2) P'_n(x)^2) at the final
// node, so invariant tests can separate quadrature error from index errors.
void oracle_refine_weights(void* h) {
  Oracle* o = (Oracle*)h;
  const int n = o->nth;
  for (int i = 0; i < n; ++i) {
    const long double z = o->gpoint[i];
    long double p1 = 1.0L, p2 = 0.0L, p3;
    for (int j = 1; j <= n; ++j) {
      p3 = p2; p2 = p1;
      p1 = ((2.0L * j - 1.0L) * z * p2 - (j - 1.0L) * p3) / (long double)j;
    }
    const long double pp = (long double)n * (z * p1 - p2) / (z * z - 1.0L);
    o->weight[i] = (double)(2.0L / ((1.0L - z * z) * pp * pp));
  }
}

// Tables for tests: colat[nth], weight[nth], P_rtm/dP_rtm[J*nth] (j-major, theta fastest),
// g3/g6/g7[J], jl/jm[J].
void oracle_tables(void* h, double* colat, double* weight, double* P, double* dP, double* g3,
                   double* g6, double* g7, int* jl, int* jm) {
  Oracle* o = (Oracle*)h;
  if (colat) std::memcpy(colat, o->colat.data(), sizeof(double) * o->nth);
  if (weight) std::memcpy(weight, o->weight.data(), sizeof(double) * o->nth);
  if (P) std::memcpy(P, o->P_rtm.data(), sizeof(double) * o->P_rtm.size());
  if (dP) std::memcpy(dP, o->dP_rtm.data(), sizeof(double) * o->dP_rtm.size());
  if (g3) std::memcpy(g3, o->g3.data(), sizeof(double) * o->J);
  if (g6) std::memcpy(g6, o->g6.data(), sizeof(double) * o->J);
  if (g7) std::memcpy(g7, o->g7.data(), sizeof(double) * o->J);
  if (jl) std::memcpy(jl, o->jl.data(), sizeof(int) * o->J);
  if (jm) std::memcpy(jm, o->jm.data(), sizeof(int) * o->J);
}

// d_rj is column-major (ld x ncol); cols[f] is the first column of field f
// (vectors first, 3 columns each, then scalars).  j order of d_rj = rlm order.
static void gather_sp(const Oracle& o, const double* d_rj, long long ld, const int* cols, int nv,
                      int ns, std::vector<double>& sp) {
  const int nc = 3 * nv + ns;
  const i64 nn = o.J * o.nr;
  sp.resize((size_t)nn * nc);
  for (int f = 0; f < nv + ns; ++f) {
    const int ncomp = f < nv ? 3 : 1;
    const int c0 = f < nv ? 3 * f : 3 * nv + (f - nv);
    for (int q = 0; q < ncomp; ++q)
      for (i64 n = 0; n < nn; ++n) sp[n * nc + c0 + q] = d_rj[n + ld * (cols[f] + q)];
  }
}
static void scatter_sp(const Oracle& o, const std::vector<double>& sp, int nv, int ns, double* d_rj,
                       long long ld, const int* cols) {
  const int nc = 3 * nv + ns;
  const i64 nn = o.J * o.nr;
  for (int f = 0; f < nv + ns; ++f) {
    const int ncomp = f < nv ? 3 : 1;
    const int c0 = f < nv ? 3 * f : 3 * nv + (f - nv);
    for (int q = 0; q < ncomp; ++q)
      for (i64 n = 0; n < nn; ++n) d_rj[n + ld * (cols[f] + q)] = sp[n * nc + c0 + q];
  }
}

// Stage timings of the last call in ms: [0] Legendre bwd, [1] FFT bwd, [2] products,
// [3] FFT fwd, [4] Legendre fwd.
static double g_t[5];
void oracle_last_timing(double* t) { std::memcpy(t, g_t, sizeof(g_t)); }

// sph_b_trans: d_rj -> fld_rtp (nnod_rtp x ncb, column-major)
void oracle_b_trans(void* h, const double* d_rj, long long ld, const int* cols, double* fld_rtp) {
  Oracle* o = (Oracle*)h;
  std::vector<double> sp, rtm((size_t)o->nth * o->nr * o->nmslot * o->ncb);
  gather_sp(*o, d_rj, ld, cols, o->nvb, o->nsb, sp);
  double t0 = omp_get_wtime();
  leg_bwd(*o, sp.data(), rtm.data());
  double t1 = omp_get_wtime();
  fft_bwd(*o, rtm.data(), o->ncb, fld_rtp);
  double t2 = omp_get_wtime();
  g_t[0] = 1e3 * (t1 - t0); g_t[1] = 1e3 * (t2 - t1);
}

// sph_f_trans: frc_rtp (nnod_rtp x ncf) -> d_rj
void oracle_f_trans(void* h, const double* frc_rtp, double* d_rj, long long ld, const int* cols) {
  Oracle* o = (Oracle*)h;
  std::vector<double> sp((size_t)o->J * o->nr * o->ncf), rtm((size_t)o->nth * o->nr * o->nmslot * o->ncf);
  double t0 = omp_get_wtime();
  fft_fwd(*o, frc_rtp, o->ncf, rtm.data());
  double t1 = omp_get_wtime();
  leg_fwd(*o, rtm.data(), sp.data());
  double t2 = omp_get_wtime();
  scatter_sp(*o, sp, o->nvf, o->nsf, d_rj, ld, cols);
  g_t[3] = 1e3 * (t1 - t0); g_t[4] = 1e3 * (t2 - t1);
}

// Full cycle: d_rj_in -> bwd -> products -> fwd -> d_rj_out
void oracle_cycle(void* h, const double* d_rj_in, long long ld_in, const int* cols_in,
                  double* d_rj_out, long long ld_out, const int* cols_out) {
  Oracle* o = (Oracle*)h;
  const i64 nnod = (i64)o->nr * o->nth * o->nph;
  std::vector<double> fld((size_t)nnod * o->ncb), frc((size_t)nnod * o->ncf);
  oracle_b_trans(h, d_rj_in, ld_in, cols_in, fld.data());
  double t0 = omp_get_wtime();
  products(*o, fld.data(), frc.data());
  double t1 = omp_get_wtime();
  oracle_f_trans(h, frc.data(), d_rj_out, ld_out, cols_out);
  g_t[2] = 1e3 * (t1 - t0);
}

// Legendre stages alone on the reference rtm layout (for stage tests):
// sp[(j + J*k)*ncb + comp] -> rtm[((ms*nr + k)*nth + i)*ncb + comp] and back.
void oracle_leg_bwd(void* h, const double* sp, double* rtm) { leg_bwd(*(Oracle*)h, sp, rtm); }
void oracle_leg_fwd(void* h, const double* rtm, double* sp) { leg_fwd(*(Oracle*)h, rtm, sp); }

}  // extern "C"
