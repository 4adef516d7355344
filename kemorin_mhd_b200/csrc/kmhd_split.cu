// kmhd_split.cu -- split-precision Legendre transforms on the tcgen05 tensor cores.
//
// Every Legendre contraction C = A B (A from the FP64 Schmidt tables, B from the
// data) is evaluated as an Ozaki-style sum of INT8 slice products:
//   A' = A D, B' = D^-1 B        D = diag(2^d_k): power-of-two column equilibration of A
//   A'[i][:] = 2^eA[i] sum_s a_s[i][:] 256^(ns-1-s)   balanced base-256 digits a_s in [-128,127]
//   B'[:][c] = 2^eB[c] sum_s b_s[:][c] 256^(ns-1-s)
//   C[i][c] = 2^(eA[i]+eB[c]) sum_{t<=T} 256^(2ns-2-t) G_t,  G_t = sum_{u+v=t} a_u b_v
// Each anti-diagonal group G_t accumulates exactly in an INT32 TMEM accumulator
// (tcgen05.mma kind::i8); the groups are recombined in FP64 in the epilogue.
// Tier "split": ns = 6, T = 6 (26 slice products); tier "fp32acc": ns = 4, T = 3 (10).
//
// The symmetric form of the reference (legendre_bwd_sym_matmul.f90:301-500 and
// legendre_fwd_sym_matmul.f90:315-452) is kept.  The +-m cross terms and the
// P / dP products that meet in one output are concatenated along K so that every
// output element is one accumulator:
//   backward theta/phi:  sym  = [dP_o | (m/sin) P_e] . [b_o ; c_e]-type columns
//                        asym = [dP_e | (m/sin) P_o] . [b_e ; c_o]-type columns
//   backward r, scalars: sym = P_e . a_e,  asym = P_o . a_o
//   forward comp 1, scalars: P_p . X,  comp 2/3: [dP_p | m P_p] . [W ; U]-type columns
// The backward sym and asym halves are computed by the two CTAs of a cluster and
// combined (N = sym + asym, S = sym - asym) through distributed shared memory.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "kmhd_split.cuh"

namespace kmhd {
namespace {

constexpr int kTM = 128;     // rows per tile (MMA M)
constexpr int kTN = 64;      // columns per tile (MMA N)
constexpr int kTK = 32;      // K per chunk (one kind::i8 MMA)
constexpr int kStages = 4;
constexpr int kNT = 8;       // operand types
constexpr int kGemmThreads = 128;
constexpr long long kSpinCap = 1ll << 24;

// types: 0 theta/phi sym, 1 theta/phi asym, 2 r/scalar sym, 3 r/scalar asym (backward)
//        4 F1 even, 5 F1 odd, 6 F2 even, 7 F2 odd (forward)

__host__ __device__ __forceinline__ int pad_to(int x, int q) { return (x + q - 1) / q * q; }

// byte offset of (row, k) in a K-major no-swizzle tile of 8x16-byte core matrices
__host__ __device__ __forceinline__ int tile_off(int row, int k) {
  return (row >> 3) * 256 + ((k >> 4) & 1) * 128 + (row & 7) * 16 + (k & 15);
}

// ---------------------------------------------------------------------------
// PTX wrappers (tcgen05, mbarrier, bulk copy, cluster)
__device__ __forceinline__ unsigned sptr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(sptr(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(sptr(b)), "r"(bytes));
}
// bounded wait on phase parity; returns false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
  for (long long it = 0; it < kSpinCap; ++it) {
    unsigned ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(sptr(b)), "r"(parity));
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(sptr(dst)),
      "l"(src), "r"(bytes), "r"(sptr(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t smem_desc(const void* p, unsigned lbo, unsigned sbo) {
  const uint64_t a = (sptr(p) >> 4) & 0x3FFF;
  return a | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
         (1ull << 46);  // version 1 (sm_100), base offset 0, SWIZZLE_NONE
}
__device__ __forceinline__ void mma_i8(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, unsigned idesc, unsigned acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(sptr(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(unsigned taddr, int* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ double ld_peer_f64(const double* local, unsigned peer) {
  unsigned a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(a) : "r"(sptr(local)), "r"(peer));
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(a));
  return v;
}

// ---------------------------------------------------------------------------
// Digit extraction: v must satisfy |rint(v)| < 2^(8 ns - 2).
__device__ __forceinline__ void digits(double v, int ns, signed char* d) {
  long long x = __double2ll_rn(v);
  for (int s = ns - 1; s >= 1; --s) {
    const long long dd = ((x + 128) & 255) - 128;
    d[s] = (signed char)dd;
    x = (x - dd) >> 8;
  }
  d[0] = (signed char)x;
}

// frexp-style exponent: smallest e with |x| < 2^e (x > 0)
__device__ __forceinline__ int exp_above(double x) {
  int e;
  frexp(x, &e);  // x = f 2^e, f in [0.5, 1)
  return e;
}

// ---------------------------------------------------------------------------
// Operand geometry (host and device)
struct TypeGeo {
  int rows;    // valid rows
  int rpad;    // rows padded to kTM
  int kpart0;  // K of the first concatenated part (padded to kTK), or full K
  int kpad;    // total padded K
};

__host__ __device__ inline TypeGeo type_geo(int t, int L, int m, int nh) {
  const int Ke = kcount(L, m, 0), Ko = kcount(L, m, 1);
  const int Kep = pad_to(Ke, kTK), Kop = pad_to(Ko, kTK), Nhp = pad_to(nh, kTK);
  TypeGeo g;
  switch (t) {
    case 0: g.rows = nh; g.kpart0 = Kop; g.kpad = Kop + Kep; break;
    case 1: g.rows = nh; g.kpart0 = Kep; g.kpad = Kep + Kop; break;
    case 2: g.rows = nh; g.kpart0 = Kep; g.kpad = Kep; break;
    case 3: g.rows = nh; g.kpart0 = Kop; g.kpad = Kop; break;
    case 4: g.rows = Ke; g.kpart0 = Nhp; g.kpad = Nhp; break;
    case 5: g.rows = Ko; g.kpart0 = Nhp; g.kpad = Nhp; break;
    case 6: g.rows = Ke; g.kpart0 = Nhp; g.kpad = 2 * Nhp; break;
    default: g.rows = Ko; g.kpart0 = Nhp; g.kpad = 2 * Nhp; break;
  }
  g.rpad = pad_to(g.rows > 0 ? g.rows : 1, kTM);
  return g;
}

// A element (FP64, before equilibration) of type t at (row, k).
__device__ inline double a_value(const Plan& P, int t, int m, int row, int k) {
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  if (row >= g.rows || k >= g.kpad) return 0.0;
  const int Ke = kcount(P.L, m, 0), Ko = kcount(P.L, m, 1);
  auto Pv = [&](const double* T, int par, int kk, int th) -> double {
    return T[P.poff[2 * m + par] + (long long)kk * P.nh_pad + th];
  };
  if (t <= 3) {  // rows = theta, K = l
    const int th = row;
    const double ms = (double)m * P.asin_t[th];
    if (t == 0) {
      if (k < g.kpart0) return k < Ko ? Pv(P.dP, 1, k, th) : 0.0;
      const int kk = k - g.kpart0;
      return kk < Ke ? ms * Pv(P.P, 0, kk, th) : 0.0;
    }
    if (t == 1) {
      if (k < g.kpart0) return k < Ke ? Pv(P.dP, 0, k, th) : 0.0;
      const int kk = k - g.kpart0;
      return kk < Ko ? ms * Pv(P.P, 1, kk, th) : 0.0;
    }
    if (t == 2) return k < Ke ? Pv(P.P, 0, k, th) : 0.0;
    return k < Ko ? Pv(P.P, 1, k, th) : 0.0;
  }
  const int par = (t == 4 || t == 6) ? 0 : 1;
  if (t <= 5) return k < P.nh ? Pv(P.P, par, row, k) : 0.0;
  if (k < g.kpart0) return k < P.nh ? Pv(P.dP, par, row, k) : 0.0;
  const int th = k - g.kpart0;
  return th < P.nh ? (double)m * Pv(P.P, par, row, th) : 0.0;
}

struct SliceTabs {
  signed char* A;        // A slices
  const long long* aoff; // [(L+1)*kNT] byte offsets
  int* aexp;             // row exponents, [(L+1)*kNT] blocks of rpad
  const long long* aeoff;
  int* dexp;             // column equilibration exponents, blocks of kpad
  const long long* deoff;
  signed char* B;        // B slices (per call)
  const long long* boff;
  int* bexp;             // column exponents, blocks of npad
  const long long* beoff;
  int ns, T;
  int ncolT[kNT];        // valid columns per type
  int npadT[kNT];        // padded columns per type
  int nrT, nrR;          // radius paddings (theta/phi and F2: 16; r and F1: 8)
};

// Column equilibration exponents: dexp = -(smallest e with max_rows |A[:,k]| < 2^e)
__global__ void k_a_dexp(Plan P, SliceTabs S, int t) {
  const int m = blockIdx.y;
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g.kpad) return;
  double mx = 0.0;
  for (int r = 0; r < g.rows; ++r) mx = fmax(mx, fabs(a_value(P, t, m, r, k)));
  S.dexp[S.deoff[m * kNT + t] + k] = mx > 0.0 ? -exp_above(mx) : 0;
}

// Row exponents and digits of A' = A D: one warp per (m, row).
__global__ void k_a_slices(Plan P, SliceTabs S, int t) {
  const int m = blockIdx.y;
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int row = warp;
  if (row >= g.rpad) return;
  const int* dx = S.dexp + S.deoff[m * kNT + t];
  double mx = 0.0;
  for (int k = lane; k < g.kpad; k += 32) mx = fmax(mx, fabs(ldexp(a_value(P, t, m, row, k), dx[k])));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int bits = 8 * S.ns - 2;
  const int e = mx > 0.0 ? exp_above(mx) : 0;
  if (lane == 0) S.aexp[S.aeoff[m * kNT + t] + row] = e - bits;
  signed char* base = S.A + S.aoff[m * kNT + t];
  const int nkc = g.kpad / kTK;
  const int mt = row / kTM, rr = row % kTM;
  for (int k = lane; k < g.kpad; k += 32) {
    signed char d[8];
    const double v = mx > 0.0 ? ldexp(a_value(P, t, m, row, k), dx[k] + bits - e) : 0.0;
    digits(v, S.ns, d);
    const int kc = k / kTK;
    for (int s = 0; s < S.ns; ++s)
      base[((long long)(mt * nkc + kc) * S.ns + s) * (kTM * kTK) + tile_off(rr, k % kTK)] = d[s];
  }
}

// ---------------------------------------------------------------------------
// B operand values.
// Backward theta/phi column (v, r, q); K concatenation as the A type.
__device__ inline double b_bwd_value(const Plan& P, const SliceTabs& S, const double* d_rj, long long ld,
                                     const int* cols, int t, int m, int col, int k) {
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  const int Ke = kcount(P.L, m, 0), Ko = kcount(P.L, m, 1);
  if (t <= 1) {
    const int q = col & 3, r = (col >> 2) % S.nrT, v = (col >> 2) / S.nrT;
    if (v >= P.nvb || r >= P.nr) return 0.0;
    int par, kk;
    const bool first = k < g.kpart0;
    kk = first ? k : k - g.kpart0;
    // type 0: first part odd l (dP_o), second even l (msP_e); type 1 the reverse
    par = (t == 0) ? (first ? 1 : 0) : (first ? 0 : 1);
    if (kk >= (par ? Ko : Ke)) return 0.0;
    const int l = m + 2 * kk + par;
    // quantity selection: first part uses dP columns, second the m/sin P columns
    // q: 0 th cos, 1 th sin, 2 ph cos, 3 ph sin
    // first part  : b+, b-, -c+, -c-
    // second part : c-, -c+, b-, -b+
    int slot, comp;
    double sg = 1.0;
    if (first) {
      comp = (q < 2) ? 1 : 2;  // b = dS/dr (col+1), c = T (col+2)
      slot = q & 1;
      if (q >= 2) sg = -1.0;
    } else {
      switch (q) {
        case 0: comp = 2; slot = 1; break;
        case 1: comp = 2; slot = 0; sg = -1.0; break;
        case 2: comp = 1; slot = 1; break;
        default: comp = 1; slot = 0; sg = -1.0; break;
      }
    }
    if (slot == 1 && m == 0) return 0.0;
    const int j = P.jmap[((long long)m * 2 + slot) * (P.L + 1) + l];
    const double x = d_rj[(long long)j + P.J * r + ld * (cols[v] + comp)];
    return sg * (x * (1.0 / P.radius[r]));
  }
  // r / scalar columns (r, f, slot), f < 4
  const int slot = col & 1, f = (col >> 1) & 3, r = col >> 3;
  if (r >= P.nr || f >= P.nvb + P.nsb) return 0.0;
  const int par = t - 2;
  if (k >= (par ? Ko : Ke)) return 0.0;
  if (slot == 1 && m == 0) return 0.0;
  const int l = m + 2 * k + par;
  const int j = P.jmap[((long long)m * 2 + slot) * (P.L + 1) + l];
  if (f < P.nvb) {
    const double ar = 1.0 / P.radius[r];
    return d_rj[(long long)j + P.J * r + ld * cols[f]] * (ar * ar) * g3_of(l);
  }
  return d_rj[(long long)j + P.J * r + ld * cols[f]];
}

// Forward columns from the grid spectra rtm_f (sym / asym with weights).
__device__ inline double b_fwd_value(const Plan& P, const SliceTabs& S, int t, int m, int col, int k) {
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  const int par = (t == 4 || t == 6) ? 0 : 1;
  const long long strideTh = (long long)P.nr * P.ncf * 2;
  auto sy = [&](int th, int r, int c, int slot, bool want_sym, bool overs) -> double {
    // (N +- S) w [/ sin], equator: N w, asym 0
    const int ro = rec_off(c, P.nvf) + slot;
    const double wp = P.weight[th];
    const double nval = P.rtm_f[((long long)m * P.nth + th) * strideTh + (long long)r * P.ncf * 2 + ro];
    double v;
    if (th < P.nth / 2) {
      const double sval = P.rtm_f[((long long)m * P.nth + (P.nth - 1 - th)) * strideTh + (long long)r * P.ncf * 2 + ro];
      v = want_sym ? (nval + sval) * wp : (nval - sval) * wp;
    } else {
      v = want_sym ? nval * wp : 0.0;
    }
    return overs ? v * P.asin_t[th] : v;
  };
  if (t <= 5) {
    const int slot = col & 1, f = (col >> 1) & 3, r = col >> 3;
    if (r >= P.nr || f >= P.nvf + P.nsf || k >= P.nh) return 0.0;
    if (slot == 1 && m == 0) return 0.0;
    const int c = f < P.nvf ? 3 * f : 3 * P.nvf + (f - P.nvf);
    return sy(k, r, c, slot, par == 0, false);
  }
  const int q = col & 3, r = (col >> 2) % S.nrT, v = (col >> 2) / S.nrT;
  if (v >= P.nvf || r >= P.nr) return 0.0;
  const bool first = k < g.kpart0;
  const int th = first ? k : k - g.kpart0;
  if (th >= P.nh) return 0.0;
  if (m == 0 && !first) return 0.0;
  // W = [a]sym(F_theta) w, W' = [a]sym(F_phi) w      (dP part: asym for even l)
  // U = [a]sym(F_phi) w/sin, U' = [a]sym(F_theta) w/sin (P part: sym for even l)
  const bool dP_sym = (par == 1), P_sym = (par == 0);
  // q: 0 comp2+ = W.c - m U.s ; 1 comp2- = W.s + m U.c ; 2 comp3+ = -W'.c - m U'.s ; 3 comp3- = -W'.s + m U'.c
  if (first) {
    switch (q) {
      case 0: return sy(th, r, 3 * v + 1, 0, dP_sym, false);
      case 1: return sy(th, r, 3 * v + 1, 1, dP_sym, false);
      case 2: return -sy(th, r, 3 * v + 2, 0, dP_sym, false);
      default: return -sy(th, r, 3 * v + 2, 1, dP_sym, false);
    }
  }
  switch (q) {
    case 0: return -sy(th, r, 3 * v + 2, 1, P_sym, true);
    case 1: return sy(th, r, 3 * v + 2, 0, P_sym, true);
    case 2: return -sy(th, r, 3 * v + 1, 1, P_sym, true);
    default: return sy(th, r, 3 * v + 1, 0, P_sym, true);
  }
}

// B slicer: one CTA per (m, type, n-tile).  Pass 1: column maxima of B' = B/D;
// pass 2: digits, written as 16-byte rows of the tile layout.
template <bool FWD>
__global__ void k_b_slices(Plan P, SliceTabs S, int t, const double* __restrict__ d_rj, long long ld,
                           const int* __restrict__ cols) {
  __shared__ int colexp[kTN];
  __shared__ double colmax[kTN];
  const int m = blockIdx.y;
  const int nt = blockIdx.x;
  const TypeGeo g = type_geo(t, P.L, m, P.nh);
  if (nt * kTN >= S.npadT[t]) return;
  const int* dx = S.dexp + S.deoff[m * kNT + t];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  auto val = [&](int c, int k) -> double {
    const int col = nt * kTN + c;
    const double x = FWD ? b_fwd_value(P, S, t, m, col, k) : b_bwd_value(P, S, d_rj, ld, cols, t, m, col, k);
    return ldexp(x, -dx[k]);
  };
  for (int c = warp; c < kTN; c += nw) {
    double mx = 0.0;
    for (int k = lane; k < g.kpad; k += 32) mx = fmax(mx, fabs(val(c, k)));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      colmax[c] = mx;
      colexp[c] = mx > 0.0 ? exp_above(mx) : 0;
    }
  }
  __syncthreads();
  const int bits = 8 * S.ns - 2;
  if (threadIdx.x < kTN) S.bexp[S.beoff[m * kNT + t] + nt * kTN + threadIdx.x] = colexp[threadIdx.x] - bits;
  signed char* base = S.B + S.boff[m * kNT + t];
  const int nkc = g.kpad / kTK;
  const int n16 = g.kpad / 16;
  for (int it = threadIdx.x; it < kTN * n16; it += blockDim.x) {
    const int c = it % kTN, kb = it / kTN;
    const bool nz = colmax[c] > 0.0;
    const int sh = bits - colexp[c];
    alignas(16) signed char row[8][16];
    for (int q = 0; q < 16; ++q) {
      signed char d[8];
      const double v = nz ? ldexp(val(c, kb * 16 + q), sh) : 0.0;
      digits(v, S.ns, d);
      for (int s = 0; s < S.ns; ++s) row[s][q] = d[s];
    }
    const int kc = kb >> 1;
    for (int s = 0; s < S.ns; ++s) {
      signed char* dst = base + ((long long)(nt * nkc + kc) * S.ns + s) * (kTN * kTK) + tile_off(c, (kb & 1) * 16);
      *reinterpret_cast<int4*>(dst) = *reinterpret_cast<const int4*>(row[s]);
    }
  }
}

// ---------------------------------------------------------------------------
// The split GEMM.  One CTA = (m, type, m-tile, n-tile); backward launches pair
// the sym (rank 0) and asym (rank 1) CTAs of one output tile in a cluster.
struct Work {
  int m, t, mt, nt;
};

struct GemmArgs {
  Plan P;
  SliceTabs S;
  const Work* work;
  int nwork;
  int pair;        // 1: backward cluster pairs
  double* d_rj;    // forward output
  long long ld;
  const int* cols;
  int* err;        // device error word
};

__device__ __forceinline__ unsigned make_idesc() {
  // kind::i8: D s32 (2 << 4), A s8 (1 << 7), B s8 (1 << 10), K-major A/B, N = 64, M = 128
  return (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(kTN >> 3) << 17) | ((unsigned)(kTM >> 4) << 24);
}

template <int NS, int TG>
__global__ void __launch_bounds__(kGemmThreads, 1) k_split_gemm(GemmArgs args) {
  extern __shared__ __align__(1024) unsigned char sm[];
  constexpr int A_BYTES = NS * kTM * kTK, B_BYTES = NS * kTN * kTK;
  constexpr int STAGE = A_BYTES + B_BYTES;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + kStages * STAGE);
  unsigned long long* empty = full + kStages;
  unsigned long long* done = empty + kStages;
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(done + 1);
  const Plan& P = args.P;
  const SliceTabs& S = args.S;
  const Work w = args.work[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const TypeGeo g = type_geo(w.t, P.L, w.m, P.nh);
  const int nk = g.rows > 0 ? g.kpad / kTK : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(sptr(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  bool ok = true;

  const signed char* Ag = S.A + S.aoff[w.m * kNT + w.t] + (long long)w.mt * nk * A_BYTES;
  const signed char* Bg = S.B + S.boff[w.m * kNT + w.t] + (long long)w.nt * nk * B_BYTES;

  if (nk > 0) {
    if (warp == 1 && lane == 0) {
      // producer: bulk copies of pre-laid-out slice tiles
      for (int kc = 0; kc < nk; ++kc) {
        const int st = kc % kStages;
        if (kc >= kStages && !mbar_wait(&empty[st], ((kc / kStages) - 1) & 1)) { ok = false; break; }
        mbar_expect_tx(&full[st], STAGE);
        bulk_g2s(sm + st * STAGE, Ag + (long long)kc * A_BYTES, A_BYTES, &full[st]);
        bulk_g2s(sm + st * STAGE + A_BYTES, Bg + (long long)kc * B_BYTES, B_BYTES, &full[st]);
      }
      if (!ok) atomicExch(args.err, KMHD_ERR_TIMEOUT);
    } else if (warp == 0 && lane == 0) {
      const unsigned idesc = make_idesc();
      for (int kc = 0; kc < nk; ++kc) {
        const int st = kc % kStages;
        if (!mbar_wait(&full[st], (kc / kStages) & 1)) { ok = false; break; }
        tc_fence_after();
        const unsigned char* As = sm + st * STAGE;
        const unsigned char* Bs = As + A_BYTES;
#pragma unroll
        for (int u = 0; u < NS; ++u) {
#pragma unroll
          for (int v = 0; v < NS; ++v) {
            const int grp = u + v;
            if (grp > TG) continue;
            // the first product of group grp (smallest u) overwrites, the rest accumulate
            const unsigned first_u = (grp < NS) ? 0 : grp - (NS - 1);
            const unsigned acc = (kc > 0 || (unsigned)u > first_u) ? 1u : 0u;
            mma_i8(tmem + (unsigned)(grp * kTN), smem_desc(As + u * (kTM * kTK), 128, 256),
                   smem_desc(Bs + v * (kTN * kTK), 128, 256), idesc, acc);
          }
        }
        mma_commit(&empty[st]);
      }
      mma_commit(done);
      if (!ok) atomicExch(args.err, KMHD_ERR_TIMEOUT);
    }
    __syncwarp();
    // every thread waits for the accumulators
    if (!mbar_wait(done, 0)) {
      ok = false;
      atomicExch(args.err, KMHD_ERR_TIMEOUT);
    }
    tc_fence_after();
  }

  // ---- epilogue: combine groups, scale, and emit
  const int row = warp * 32 + lane;  // TMEM lane
  const int grow = w.mt * kTM + row;
  const int eA = (grow < g.rows) ? S.aexp[S.aeoff[w.m * kNT + w.t] + grow] : 0;
  const int* eBp = S.bexp + S.beoff[w.m * kNT + w.t] + w.nt * kTN;
  const double wscale = ldexp(1.0, 8 * (2 * NS - 2 - TG));
  double* xbuf = reinterpret_cast<double*>(sm);  // [kTM][kTN + 1] for the cluster exchange
  for (int cb = 0; cb < kTN / 16; ++cb) {
    double val[16];
    if (nk > 0 && ok) {
      int acc[TG + 1][16];
#pragma unroll
      for (int gi = 0; gi <= TG; ++gi)
        tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(gi * kTN + cb * 16), acc[gi]);
      tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        double v = (double)acc[0][c];
#pragma unroll
        for (int gi = 1; gi <= TG; ++gi) v = v * 256.0 + (double)acc[gi][c];
        val[c] = ldexp(v * wscale, eA + eBp[cb * 16 + c]);
      }
    } else {
#pragma unroll
      for (int c = 0; c < 16; ++c) val[c] = 0.0;
    }
    if (args.pair) {
#pragma unroll
      for (int c = 0; c < 16; ++c) xbuf[row * (kTN + 1) + cb * 16 + c] = val[c];
    } else {
      // forward: scatter into d_rj with the r, r^2, g7, g6, m factors
      const int par = (w.t == 4 || w.t == 6) ? 0 : 1;
      const int l = w.m + 2 * grow + par;
      if (grow < g.rows && l <= P.L) {
        const double g7 = g7_of(l, w.m);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int col = w.nt * kTN + cb * 16 + c;
          if (w.t <= 5) {
            const int slot = col & 1, f = (col >> 1) & 3, r = col >> 3;
            if (r >= P.nr || f >= P.nvf + P.nsf || (slot == 1 && w.m == 0)) continue;
            const long long j = P.jmap[((long long)w.m * 2 + slot) * (P.L + 1) + l] + P.J * r;
            if (f < P.nvf) {
              const double r1 = P.radius[r];
              args.d_rj[j + args.ld * args.cols[f]] = val[c] * (r1 * r1) * g7;
            } else {
              args.d_rj[j + args.ld * args.cols[f]] = val[c] * g6_of(l, w.m);
            }
          } else {
            const int q = col & 3, r = (col >> 2) % S.nrT, v = (col >> 2) / S.nrT;
            if (v >= P.nvf || r >= P.nr) continue;
            const int slot = q & 1;
            if (slot == 1 && w.m == 0) continue;
            const long long j = P.jmap[((long long)w.m * 2 + slot) * (P.L + 1) + l] + P.J * r;
            args.d_rj[j + args.ld * (args.cols[v] + 1 + (q >> 1))] = val[c] * P.radius[r] * g7;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));

  if (args.pair) {
    // ---- backward: N = sym + asym (rank 0), S = sym - asym (rank 1)
    cluster_sync();
    const unsigned rank = cluster_rank();
    const unsigned peer = rank ^ 1u;
    const int th = grow;
    if (th < P.nh) {
      const bool pairrow = th < P.nth / 2;
      const int thout = rank == 0 ? th : P.nth - 1 - th;
      const bool write = rank == 0 || pairrow;
      if (write) {
        const long long recb = ((long long)w.m * P.nth + thout) * P.nr * P.ncb * 2;
        for (int c = 0; c < kTN; ++c) {
          const double own = xbuf[row * (kTN + 1) + c];
          const double oth = ld_peer_f64(xbuf + row * (kTN + 1) + c, peer);
          double v;
          if (!pairrow) v = rank == 0 ? own : 0.0;            // equator: sym only
          else v = rank == 0 ? own + oth : oth - own;          // rank 1 holds asym
          const int col = w.nt * kTN + c;
          if (w.t <= 1) {
            const int q = col & 3, r = (col >> 2) % S.nrT, vv = (col >> 2) / S.nrT;
            if (vv >= P.nvb || r >= P.nr) continue;
            P.rtm_b[recb + (long long)r * P.ncb * 2 + 4 * vv + q] = v;
          } else {
            const int slot = col & 1, f = (col >> 1) & 3, r = col >> 3;
            if (r >= P.nr || f >= P.nvb + P.nsb) continue;
            P.rtm_b[recb + (long long)r * P.ncb * 2 + 4 * P.nvb + 2 * f + slot] = v;
          }
        }
      }
    }
    cluster_sync();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
struct SplitState {
  int tier, ns, T;
  SliceTabs S;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  std::vector<long long> aoff, aeoff, deoff, boff, beoff;
  Work* work_b = nullptr;  // backward work (cluster pairs)
  Work* work_f = nullptr;  // forward work
  int nwork_b = 0, nwork_f = 0;
  int* err = nullptr;
  int nlc_max = 0;
};

namespace {

template <typename T>
int salloc(SplitState* s, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) return KMHD_ERR_NOMEM;
  s->allocs.push_back(q);
  s->bytes += (int64_t)(sizeof(T) * (n > 0 ? n : 1));
  *p = (T*)q;
  return KMHD_OK;
}

size_t gemm_smem(int ns) {
  return (size_t)kStages * ns * (kTM + kTN) * kTK + (2 * kStages + 2) * 8 + 64;
}

template <int NS, int TG>
cudaError_t launch_gemm(const GemmArgs& a, int nblocks, bool cluster, cudaStream_t st) {
  auto kern = k_split_gemm<NS, TG>;
  const size_t smem = gemm_smem(NS) > (size_t)(kTM * (kTN + 1) * 8) ? gemm_smem(NS) : (size_t)(kTM * (kTN + 1) * 8) + 256;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblocks);
  cfg.blockDim = dim3(kGemmThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  int na = 0;
  if (cluster) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    na = 1;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, kern, a);
}

cudaError_t run_gemm(const SplitState* s, const GemmArgs& a, int nblocks, bool cluster, cudaStream_t st) {
  if (s->ns == 6) return launch_gemm<6, 6>(a, nblocks, cluster, st);
  return launch_gemm<4, 3>(a, nblocks, cluster, st);
}

}  // namespace

int64_t split_bytes(const SplitState* s) { return s ? s->bytes : 0; }

void split_destroy(SplitState* s) {
  if (!s) return;
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

int split_create(SplitState** out, const Plan& p, int tier, int nslice, cudaStream_t st) {
  *out = nullptr;
  if (p.nvb + p.nsb > 4 || p.nvf + p.nsf > 4) return KMHD_ERR_SIZE;
  SplitState* s = new SplitState();
  s->tier = tier;
  s->ns = tier == KMHD_TIER_SPLIT_I8 ? 6 : 4;
  if (nslice != 0 && nslice != s->ns) { delete s; return KMHD_ERR_SIZE; }
  s->T = tier == KMHD_TIER_SPLIT_I8 ? 6 : 3;
  SliceTabs& S = s->S;
  std::memset(&S, 0, sizeof(S));
  S.ns = s->ns;
  S.T = s->T;
  S.nrT = pad_to(p.nr, 16);
  S.nrR = pad_to(p.nr, 8);
  for (int t = 0; t < kNT; ++t) {
    int n;
    if (t <= 1) n = 4 * p.nvb * S.nrT;
    else if (t <= 3) n = 8 * S.nrR;
    else if (t <= 5) n = 8 * S.nrR;
    else n = 4 * p.nvf * S.nrT;
    S.ncolT[t] = n;
    S.npadT[t] = pad_to(n > 0 ? n : 1, kTN);
  }
  const int L = p.L;
  s->aoff.resize((L + 1) * kNT);
  s->aeoff.resize((L + 1) * kNT);
  s->deoff.resize((L + 1) * kNT);
  s->boff.resize((L + 1) * kNT);
  s->beoff.resize((L + 1) * kNT);
  long long ao = 0, aeo = 0, deo = 0, bo = 0, beo = 0;
  std::vector<Work> wb, wf;
  for (int m = 0; m <= L; ++m)
    for (int t = 0; t < kNT; ++t) {
      const TypeGeo g = type_geo(t, L, m, p.nh);
      const int i = m * kNT + t;
      s->aoff[i] = ao;
      s->aeoff[i] = aeo;
      s->deoff[i] = deo;
      s->boff[i] = bo;
      s->beoff[i] = beo;
      ao += (long long)g.rpad * g.kpad * s->ns;
      aeo += g.rpad;
      deo += g.kpad;
      bo += (long long)S.npadT[t] * g.kpad * s->ns;
      beo += S.npadT[t];
    }
  // work lists: backward pairs (0,1) and (2,3) per (m, m-tile, n-tile); forward 4..7
  for (int m = 0; m <= L; ++m) {
    for (int tp = 0; tp < 4; tp += 2) {
      if ((tp == 0 && p.nvb == 0)) continue;
      const TypeGeo g = type_geo(tp, L, m, p.nh);
      const int nn = S.npadT[tp] / kTN;
      for (int mt = 0; mt < g.rpad / kTM; ++mt)
        for (int nt = 0; nt < nn; ++nt) {
          wb.push_back({m, tp, mt, nt});
          wb.push_back({m, tp + 1, mt, nt});
        }
    }
    for (int t = 4; t < 8; ++t) {
      if (t >= 6 && p.nvf == 0) continue;
      const TypeGeo g = type_geo(t, L, m, p.nh);
      if (g.rows <= 0) continue;
      const int nn = S.npadT[t] / kTN;
      for (int mt = 0; mt < g.rpad / kTM; ++mt)
        for (int nt = 0; nt < nn; ++nt) wf.push_back({m, t, mt, nt});
    }
  }
  int st_ = KMHD_OK;
  long long *aoff_d, *aeoff_d, *deoff_d, *boff_d, *beoff_d;
  if ((st_ = salloc(s, &S.A, (size_t)ao)) || (st_ = salloc(s, &S.aexp, (size_t)aeo)) ||
      (st_ = salloc(s, &S.dexp, (size_t)deo)) || (st_ = salloc(s, &S.B, (size_t)bo)) ||
      (st_ = salloc(s, &S.bexp, (size_t)beo)) || (st_ = salloc(s, &aoff_d, s->aoff.size())) ||
      (st_ = salloc(s, &aeoff_d, s->aeoff.size())) || (st_ = salloc(s, &deoff_d, s->deoff.size())) ||
      (st_ = salloc(s, &boff_d, s->boff.size())) || (st_ = salloc(s, &beoff_d, s->beoff.size())) ||
      (st_ = salloc(s, &s->work_b, wb.size())) || (st_ = salloc(s, &s->work_f, wf.size())) ||
      (st_ = salloc(s, &s->err, 1))) {
    split_destroy(s);
    return st_;
  }
  S.aoff = aoff_d;
  S.aeoff = aeoff_d;
  S.deoff = deoff_d;
  S.boff = boff_d;
  S.beoff = beoff_d;
  s->nwork_b = (int)wb.size();
  s->nwork_f = (int)wf.size();
  auto up = [&](void* d, const void* h, size_t b) { return cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, st); };
  if (up(aoff_d, s->aoff.data(), sizeof(long long) * s->aoff.size()) ||
      up(aeoff_d, s->aeoff.data(), sizeof(long long) * s->aeoff.size()) ||
      up(deoff_d, s->deoff.data(), sizeof(long long) * s->deoff.size()) ||
      up(boff_d, s->boff.data(), sizeof(long long) * s->boff.size()) ||
      up(beoff_d, s->beoff.data(), sizeof(long long) * s->beoff.size()) ||
      (wb.size() && up(s->work_b, wb.data(), sizeof(Work) * wb.size())) ||
      (wf.size() && up(s->work_f, wf.data(), sizeof(Work) * wf.size())) ||
      cudaMemsetAsync(s->err, 0, sizeof(int), st) || cudaMemsetAsync(S.B, 0, (size_t)bo, st)) {
    split_destroy(s);
    return KMHD_ERR_CUDA;
  }
  // A slices from the device P tables
  int maxk = 0, maxr = 0;
  for (int t = 0; t < kNT; ++t) {
    const TypeGeo g = type_geo(t, L, 0, p.nh);
    maxk = std::max(maxk, g.kpad);
    maxr = std::max(maxr, g.rpad);
  }
  for (int t = 0; t < kNT; ++t) {
    k_a_dexp<<<dim3((maxk + 127) / 128, L + 1), 128, 0, st>>>(p, S, t);
    k_a_slices<<<dim3((maxr * 32 + 127) / 128, L + 1), 128, 0, st>>>(p, S, t);
  }
  if (cudaGetLastError() != cudaSuccess) {
    split_destroy(s);
    return KMHD_ERR_CUDA;
  }
  *out = s;
  return KMHD_OK;
}

int split_bwd(SplitState* s, const Plan& p, int, const double* d_rj, long long ld, const int* cols, cudaStream_t st) {
  const SliceTabs& S = s->S;
  int maxn = 0;
  for (int t = 0; t < 4; ++t) maxn = std::max(maxn, S.npadT[t] / kTN);
  for (int t = 0; t < 4; ++t) {
    if (t <= 1 && p.nvb == 0) continue;
    k_b_slices<false><<<dim3(maxn, p.L + 1), 256, 0, st>>>(p, S, t, d_rj, ld, cols);
  }
  if (cudaGetLastError() != cudaSuccess) return KMHD_ERR_CUDA;
  GemmArgs a;
  a.P = p;
  a.S = S;
  a.work = s->work_b;
  a.nwork = s->nwork_b;
  a.pair = 1;
  a.d_rj = nullptr;
  a.ld = 0;
  a.cols = nullptr;
  a.err = s->err;
  if (s->nwork_b > 0 && run_gemm(s, a, s->nwork_b, true, st) != cudaSuccess) return KMHD_ERR_CUDA;
  return KMHD_OK;
}

int split_fwd(SplitState* s, const Plan& p, double* d_rj, long long ld, const int* cols, cudaStream_t st) {
  const SliceTabs& S = s->S;
  int maxn = 0;
  for (int t = 4; t < 8; ++t) maxn = std::max(maxn, S.npadT[t] / kTN);
  for (int t = 4; t < 8; ++t) {
    if (t >= 6 && p.nvf == 0) continue;
    k_b_slices<true><<<dim3(maxn, p.L + 1), 256, 0, st>>>(p, S, t, nullptr, 0, nullptr);
  }
  if (cudaGetLastError() != cudaSuccess) return KMHD_ERR_CUDA;
  GemmArgs a;
  a.P = p;
  a.S = S;
  a.work = s->work_f;
  a.nwork = s->nwork_f;
  a.pair = 0;
  a.d_rj = d_rj;
  a.ld = ld;
  a.cols = cols;
  a.err = s->err;
  if (s->nwork_f > 0 && run_gemm(s, a, s->nwork_f, false, st) != cudaSuccess) return KMHD_ERR_CUDA;
  return KMHD_OK;
}

int split_check_error(SplitState* s, cudaStream_t st) {
  int h = 0;
  if (cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return KMHD_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return KMHD_ERR_CUDA;
  return h;
}

}  // namespace kmhd

// ---------------------------------------------------------------------------
// Self-test of one tcgen05 kind::i8 MMA (M=128, N=64, K=32) with the tile layout
// above and caller-chosen descriptor byte offsets (test support).
namespace kmhd {
namespace {
__global__ void __launch_bounds__(128, 1) k_selftest_mma(const signed char* A, const signed char* B, int* D,
                                                        unsigned lbo, unsigned sbo, int* err) {
  __shared__ __align__(1024) unsigned char sa[kTM * kTK];
  __shared__ __align__(1024) unsigned char sb[kTN * kTK];
  __shared__ unsigned long long bar;
  __shared__ unsigned slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kTM * kTK; i += blockDim.x) sa[tile_off(i / kTK, i % kTK)] = (unsigned char)A[i];
  for (int i = tid; i < kTN * kTK; i += blockDim.x) sb[tile_off(i / kTK, i % kTK)] = (unsigned char)B[i];
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  if (tid == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;\n" ::"r"(sptr(&slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = slot;
  if (tid == 0) {
    mma_i8(tmem, smem_desc(sa, lbo, sbo), smem_desc(sb, lbo, sbo), make_idesc(), 0u);
    mma_commit(&bar);
  }
  __syncwarp();
  if (!mbar_wait(&bar, 0)) atomicExch(err, KMHD_ERR_TIMEOUT);
  tc_fence_after();
  for (int cb = 0; cb < kTN / 16; ++cb) {
    int v[16];
    tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(cb * 16), v);
    tmem_wait_ld();
    for (int c = 0; c < 16; ++c) D[(warp * 32 + lane) * kTN + cb * 16 + c] = v[c];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;\n" ::"r"(tmem));
}
}  // namespace
}  // namespace kmhd

extern "C" int kmhd_selftest_i8_mma(int lbo, int sbo, const signed char* A, const signed char* B, int* D) {
  using namespace kmhd;
  signed char *dA = nullptr, *dB = nullptr;
  int *dD = nullptr, *err = nullptr;
  int st = KMHD_OK;
  if (cudaMalloc(&dA, kTM * kTK) || cudaMalloc(&dB, kTN * kTK) || cudaMalloc(&dD, sizeof(int) * kTM * kTN) ||
      cudaMalloc(&err, sizeof(int)))
    st = KMHD_ERR_NOMEM;
  if (!st) {
    cudaMemcpy(dA, A, kTM * kTK, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, kTN * kTK, cudaMemcpyHostToDevice);
    cudaMemset(err, 0, sizeof(int));
    k_selftest_mma<<<1, 128>>>(dA, dB, dD, (unsigned)lbo, (unsigned)sbo, err);
    int h = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) st = KMHD_ERR_CUDA;
    else {
      cudaMemcpy(D, dD, sizeof(int) * kTM * kTN, cudaMemcpyDeviceToHost);
      cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
      st = h;
    }
  }
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dD);
  cudaFree(err);
  return st;
}
