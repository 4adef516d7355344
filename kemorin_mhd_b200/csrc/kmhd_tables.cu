// kmhd_tables.cu -- FP64 set-up on the device: Gauss-Legendre nodes/weights and
// the equator-symmetric Schmidt P_l^m / dP_l^m/dtheta tables.
//
// Gauss nodes:  const_gauss_points_coefs (CORE_src/gauss_integration/gauss_integration.f90:60-133)
// Schmidt:      schmidt_legendre_m / diff_schmidt_legendre_m
//               (CORE_src/spherical_harmonics/schmidt_fix_m.f90:86-175)
// Table layout: the hemisphere tables of set_symmetric_legendre_lj
//               (PARALLEL_src/SPH_SHELL_src/set_legendre_matrices.f90:86-130), stored per
//               order m >= 0 and parity p = (l-m) mod 2 as Ptab[m][p][k][theta], l = m+2k+p,
//               theta fastest (the +m and -m slots share one table).
#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

// One Newton solve per node, exactly the reference's iteration (only the final
// n of its n-loop survives, so only n = nth is evaluated).
__global__ void k_gauss(int n, double* colat, double* weight, double* asin_t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int mh = (n + 1 - (n + 1) % 2) / 2;
  if (i > mh) return;
  const double pi = 4.0 * atan(1.0);
  const double x1 = 0.0, x2 = 1.0;
  const double xm = 0.5 * (x2 + x1), xl = 0.5 * (x2 - x1);
  double z = cos(pi * ((double)i - 0.25) / ((double)n + 0.5));
  double pp = 1.0, z1, p1, p2, p3;
  for (int it = 0; it < 100; ++it) {  // bounded: the reference loops until |dz| < 3e-12
    p1 = 1.0;
    p2 = 0.0;
    for (int j = 1; j <= n; ++j) {
      p3 = p2;
      p2 = p1;
      p1 = ((2.0 * (double)j - 1.0) * z * p2 - ((double)j - 1.0) * p3) / (double)j;
    }
    pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
    z1 = z;
    z = z1 - p1 / pp;
    if (fabs(z - z1) < 3.0e-12) break;
  }
  const double wc = 2.0 * xl / ((1.0 - z * z) * pp * pp);
  const double pa = xm - xl * z, pb = xm + xl * z;
  // final mapping to (-1, 1): w_point*2 - 1, w_coefs*2
  const double ga = pa * 2.0 - 1.0, gb = pb * 2.0 - 1.0;
  const double ca = acos(ga), cb = acos(gb);
  colat[i - 1] = ca;
  weight[i - 1] = wc * 2.0;
  asin_t[i - 1] = 1.0 / sin(ca);
  colat[n - i] = cb;
  weight[n - i] = wc * 2.0;
  asin_t[n - i] = 1.0 / sin(cb);
}

// Streaming state of the reference's fixed-order recurrence for order mo >= 1:
// df(mo), df(mo+1) in closed form, then the 3-term recurrence in l.
struct SchmidtRec {
  int mo;
  int l;        // next l to produce
  double d1, d2;  // df(l-1), df(l-2)
  double c0, c1;  // df(mo), df(mo+1)
  __device__ void init(int mo_, double ct) {
    mo = mo_;
    l = mo_;
    double df = 1.0;
    for (int k = 1; k <= mo; ++k) df = df * (double)(2 * k - 1) / (double)(2 * k);
    c1 = sqrt(2.0 * df * (double)(2 * mo + 1)) * ct;
    c0 = sqrt(2.0 * df);
    d1 = 0.0;
    d2 = 0.0;
  }
  // returns df(l) and advances
  __device__ double next(double ct) {
    double v;
    if (l == mo) v = c0;
    else if (l == mo + 1) v = c1;
    else
      v = (ct * (double)(2 * l - 1) * d1 - sqrt((double)((l - 1) * (l - 1) - mo * mo)) * d2) /
          sqrt((double)(l * l - mo * mo));
    d2 = d1;
    d1 = v;
    ++l;
    return v;
  }
};

__device__ __forceinline__ double times_sin_m(double v, double st, int m) {
  for (int k = 0; k < m; ++k) v = v * st;  // repeated multiplication, as the reference
  return v;
}

// One thread per (hemisphere latitude i, order m).
__global__ void k_legendre(int L, int nh, int nh_pad, const double* __restrict__ colat,
                           const long long* __restrict__ poff, double* __restrict__ P,
                           double* __restrict__ dP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (i >= nh) return;
  const double th = colat[i];
  const double ct = cos(th), st = sin(th);
  double* Pe = P + poff[2 * m + 0] + i;
  double* Po = P + poff[2 * m + 1] + i;
  double* dPe = dP + poff[2 * m + 0] + i;
  double* dPo = dP + poff[2 * m + 1] + i;
  if (m == 0) {
    // P_l^0 by the Legendre recurrence, P_l^1 for dP = -sqrt(l(l+1)/2) P_l^1
    SchmidtRec r1;
    r1.init(1, ct);
    double pl1 = 0.0, pl2 = 0.0;
    for (int l = 0; l <= L; ++l) {
      double p;
      if (l == 0) p = 1.0;
      else if (l == 1) p = ct;
      else p = pl1 * (double)(2 * l - 1) / (double)l * ct - pl2 * (double)(l - 1) / (double)l;
      pl2 = pl1;
      pl1 = p;
      double dp = 0.0;
      if (l >= 1) {
        const double pmp1 = times_sin_m(r1.next(ct), st, 1);
        dp = -sqrt((double)(l * (l + 1) / 2)) * pmp1;
      }
      const int k = l >> 1;
      if ((l & 1) == 0) { Pe[(long long)k * nh_pad] = p; dPe[(long long)k * nh_pad] = dp; }
      else { Po[(long long)k * nh_pad] = p; dPo[(long long)k * nh_pad] = dp; }
    }
    return;
  }
  // orders m-1 (from l = m), m, m+1 (from l = m+1)
  SchmidtRec rn, rc, rp;
  double pl1 = 0.0, pl2 = 0.0;  // used when m-1 == 0
  const int mn = m - 1;
  if (mn >= 1) {
    rn.init(mn, ct);
    (void)rn.next(ct);  // df(m-1) at l = m-1, not needed
  }
  rc.init(m, ct);
  rp.init(m + 1, ct);
  for (int l = m; l <= L; ++l) {
    double pmn1;
    if (mn == 0) {
      // Legendre P_l^0 at l = m = 1, 2, ...: recompute from l = 0 once
      if (l == m) {
        pl2 = 1.0;     // P_0
        pl1 = ct;      // P_1
        for (int q = 2; q <= l; ++q) {
          const double p = pl1 * (double)(2 * q - 1) / (double)q * ct - pl2 * (double)(q - 1) / (double)q;
          pl2 = pl1;
          pl1 = p;
        }
        pmn1 = (l == 0) ? 1.0 : pl1;
      } else {
        const double p = pl1 * (double)(2 * l - 1) / (double)l * ct - pl2 * (double)(l - 1) / (double)l;
        pl2 = pl1;
        pl1 = p;
        pmn1 = p;
      }
    } else {
      pmn1 = times_sin_m(rn.next(ct), st, mn);
    }
    const double p = times_sin_m(rc.next(ct), st, m);
    double dp;
    if (m == 1) {
      if (l == 1) dp = pmn1;
      else {
        const double pmp1 = times_sin_m(rp.next(ct), st, m + 1);
        dp = 0.5 * (sqrt((double)(2 * l * (l + 1))) * pmn1 - sqrt((double)((l - 1) * (l + 2))) * pmp1);
      }
    } else {
      if (l == m) dp = 0.5 * sqrt((double)(2 * m)) * pmn1;
      else {
        const double pmp1 = times_sin_m(rp.next(ct), st, m + 1);
        dp = 0.5 * (sqrt((double)((l + m) * (l - m + 1))) * pmn1 -
                    sqrt((double)((l - m) * (l + m + 1))) * pmp1);
      }
    }
    const int q = l - m;
    const int k = q >> 1;
    if ((q & 1) == 0) { Pe[(long long)k * nh_pad] = p; dPe[(long long)k * nh_pad] = dp; }
    else { Po[(long long)k * nh_pad] = p; dPo[(long long)k * nh_pad] = dp; }
  }
}

// ---------------------------------------------------------------------------
// On-the-fly P tables (FP64 tier, KMHD_FLAG_P_ON_THE_FLY): O(L^2) coefficients,
// O(L Ntheta) start values and the forward kernel's block seeds replace the
// O(L^2 Ntheta) P / dP tables.

// Recurrence coefficients of order mo (block y, 0..L+1) and dP coefficients of
// order m = mo (mo <= L), one thread per degree l.
__global__ void k_otf_coef(int L, double2* pco, double2* dco) {
  const int mo = blockIdx.y;
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l <= L; l += gridDim.x * blockDim.x) {
    double2 ab = make_double2(0.0, 0.0);
    if (l >= mo + 2) {
      const double s2 = sqrt((double)(l * l - mo * mo));
      ab.x = (double)(2 * l - 1) / s2;
      ab.y = sqrt((double)((l - 1) * (l - 1) - mo * mo)) / s2;
    }
    pco[(long long)mo * (L + 1) + l] = ab;
    if (mo > L) continue;
    // dP = (e P^{m-1} - f P^{m+1}) / 2 with the factors of k_legendre (the
    // m = 0 form -sqrt(l(l+1)/2) P^1 and the m = 1, l = 1 form P^0 included)
    const int m = mo;
    double2 ef = make_double2(0.0, 0.0);
    if (m == 0) {
      if (l >= 1) ef.y = 2.0 * sqrt((double)(l * (l + 1) / 2));
    } else if (m == 1) {
      if (l == 1) ef.x = 2.0;
      else if (l > 1) ef = make_double2(sqrt((double)(2 * l * (l + 1))), sqrt((double)((l - 1) * (l + 2))));
    } else {
      if (l == m) ef.x = sqrt((double)(2 * m));
      else if (l > m) ef = make_double2(sqrt((double)((l + m) * (l - m + 1))), sqrt((double)((l - m) * (l + m + 1))));
    }
    dco[(long long)m * (L + 1) + l] = ef;
  }
}

// Start values (P_mo^mo, P_{mo+1}^mo) per (order mo = block y, latitude), the
// same operations as k_legendre's first two values of the order; cos(colat).
__global__ void k_otf_start(int nh, int nh_pad, const double* __restrict__ colat, double* cos_t, double2* pst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int mo = blockIdx.y;
  if (i >= nh_pad) return;
  double2 v = make_double2(0.0, 0.0);
  if (i < nh) {
    const double th = colat[i];
    const double ct = cos(th), st = sin(th);
    if (mo == 0) {
      v = make_double2(1.0, ct);
      cos_t[i] = ct;
    } else {
      SchmidtRec r;
      r.init(mo, ct);
      v = make_double2(times_sin_m(r.c0, st, mo), times_sin_m(r.c1, st, mo));
    }
  }
  pst[(long long)mo * nh_pad + i] = v;
}

// Chain states (orders m - 1, m, m + 1) before every l0 = m + kSeedL s, one
// thread per (latitude, order m = block y).
__global__ void k_otf_seed(Plan p, double* pseed, const long long* __restrict__ pseed_off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (i >= p.nh_pad) return;
  const int L = p.L;
  const int nsd = (L - m + kSeedL) / kSeedL;
  double* out = pseed + pseed_off[m] * 6 * p.nh_pad + i;
  const bool ok = i < p.nh;
  const double ct = ok ? p.cos_t[i] : 0.0;
  double st[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int sd = 0;
  for (int l = m > 0 ? m - 1 : 0; l <= L && sd < nsd; ++l) {
    if (l == m + kSeedL * sd) {
      for (int q = 0; q < 6; ++q) out[((long long)sd * 6 + q) * p.nh_pad] = st[q];
      ++sd;
    }
    if (ok) {
      double a, b;
      pgen_step(st, p, m, l, ct, i, a, b);
    }
  }
}

// Generated P / dP of one order m, [l - m][latitude] (nh per row): the values
// the on-the-fly kernels use, for kmhd_sph_get_tables.
__global__ void k_otf_order(Plan p, int m, double* __restrict__ P, double* __restrict__ dP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.nh) return;
  double st[6];
  const double* sd = p.pseed + p.pseed_off[m] * 6 * p.nh_pad + i;
  for (int q = 0; q < 6; ++q) st[q] = sd[(long long)q * p.nh_pad];
  const double ct = p.cos_t[i];
  for (int l = m; l <= p.L; ++l) {
    double a, b;
    pgen_step(st, p, m, l, ct, i, a, b);
    P[(long long)(l - m) * p.nh + i] = a;
    dP[(long long)(l - m) * p.nh + i] = b;
  }
}

}  // namespace

cudaError_t launch_otf_order(const Plan& p, int m, double* P, double* dP, cudaStream_t s) {
  k_otf_order<<<(p.nh + 127) / 128, 128, 0, s>>>(p, m, P, dP);
  return cudaGetLastError();
}

cudaError_t launch_otf_tables(const Plan& p, double* cos_t, double2* pco, double2* dco, double2* pst,
                              double* pseed, const long long* pseed_off, cudaStream_t s) {
  k_otf_coef<<<dim3((p.L + 1 + 127) / 128, p.L + 2), 128, 0, s>>>(p.L, pco, dco);
  k_otf_start<<<dim3((p.nh_pad + 127) / 128, p.L + 2), 128, 0, s>>>(p.nh, p.nh_pad, p.colat, cos_t, pst);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  Plan q = p;
  q.cos_t = cos_t;
  q.pco = pco;
  q.dco = dco;
  q.pst = pst;
  k_otf_seed<<<dim3((p.nh_pad + 63) / 64, p.L + 1), 64, 0, s>>>(q, pseed, pseed_off);
  return cudaGetLastError();
}

cudaError_t launch_tables(const Plan& p, double* colat, double* weight, double* asin_t,
                          double* P, double* dP, cudaStream_t s) {
  const int mh = (p.nth + 1) / 2;
  k_gauss<<<(mh + 127) / 128, 128, 0, s>>>(p.nth, colat, weight, asin_t);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (!P) return cudaSuccess;  // on-the-fly P: no tables
  dim3 grid((p.nh + 63) / 64, p.L + 1);
  k_legendre<<<grid, 64, 0, s>>>(p.L, p.nh, p.nh_pad, colat, p.poff, P, dP);
  return cudaGetLastError();
}

}  // namespace kmhd
