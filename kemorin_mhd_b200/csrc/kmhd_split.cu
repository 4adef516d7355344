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
// One CTA computes both the backward sym and asym tiles of an output tile and
// combines them (N = sym + asym, S = sym - asym) through its own shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "kmhd_split.cuh"

namespace kmhd {
namespace {

constexpr int kTM = 128;     // rows per tile (MMA M)
constexpr int kTN = 64;      // columns per tile (MMA N)
constexpr int kTK = 32;      // K per chunk (one kind::i8 MMA)
constexpr int kNT = 8;       // operand types
constexpr long long kSpinCap = 1ll << 22;  // try_wait rounds (each may suspend for microseconds)

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
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, long long cap = kSpinCap) {
  for (long long it = 0; it < cap; ++it) {
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
__device__ __forceinline__ void tmem_ld8(unsigned taddr, int* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

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

// 2^e as a double, e in the normal range
__device__ __forceinline__ double pow2(int e) {
  if (e < -1022 || e > 1023) return ldexp(1.0, e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// 32-byte global load (sm_100 256-bit ld.global, read-only path); p must be 32-byte aligned
__device__ __forceinline__ void ld_global_v4(const double* p, double& a, double& b, double& c, double& d) {
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];\n" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
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
  // Forward tiles: byte kc of the 64-byte block bnz[64 (foff[m kNT + t] +
  // n-tile) ..] is set to 1 by the forward slicer when any digit of K chunk kc
  // of that tile is nonzero (at most 64 chunks tracked; types 4..7 only).  A
  // chunk whose B digits are all zero adds nothing to the tile's products, so
  // the GEMM skips it.
  unsigned char* bnz;
  const long long* foff;
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
// Slicers.  Column list of one (m, r): backward: for each vector v: types 0/1
// quantity q (8 columns), for each field f < 4: types 2/3 slots (4 columns);
// forward: types 4/5 (field f, slot) and types 6/7 (vector v, quantity q).
constexpr int kGrpCols = 24;  // derived columns of one slicer field group (at most 6 fields x 2 slots x 2 types)
// slicer CTA size (measured at L = 511 for the forward slicer: 256 threads
// 14.2 ms, 384 18.6 ms, 512 15.0 ms; in a later build 256 13.6 ms, 192
// 14.3 ms, 320 17.4 ms)
constexpr int kSliceThreads = 256;
constexpr int kSlab = 320;    // per-slice staging bytes of one 256-byte tile block (k halves 192 apart)

struct ColRef {
  int t, col;     // operand type and global column index
  int f, q;       // field (vector or scalar slot) and quantity/slot selector
};

// Columns of the radial-component / scalar types (2..5): one 8-column block
// per (group of four fields, radius), group-major like the vector types'
// (vector, radius) blocks: field f, slot s of radius r is column
// ((f / 4) nrR + r) 8 + 2 (f % 4) + s.
__host__ __device__ __forceinline__ int rs_col(const SliceTabs& S, int r, int f, int slot) {
  return (((f >> 2) * S.nrR + r) * 4 + (f & 3)) * 2 + slot;
}
__host__ __device__ __forceinline__ int rs_groups(int nF) { return (nF + 3) >> 2; }

__device__ __forceinline__ ColRef colref_bwd(const Plan& P, const SliceTabs& S, int r, int i) {
  ColRef c;
  if (i < 8 * P.nvb) {
    const int v = i >> 3, t = (i >> 2) & 1, q = i & 3;
    c.t = t; c.f = v; c.q = q; c.col = (v * S.nrT + r) * 4 + q;
  } else {
    const int j = i - 8 * P.nvb, f = j >> 2, t = 2 + ((j >> 1) & 1), slot = j & 1;
    c.t = t; c.f = f; c.q = slot; c.col = rs_col(S, r, f, slot);
  }
  return c;
}
__device__ __forceinline__ ColRef colref_fwd(const Plan& P, const SliceTabs& S, int r, int i) {
  ColRef c;
  const int nf1 = 4 * (P.nvf + P.nsf);
  if (i < nf1) {
    const int f = i >> 2, t = 4 + ((i >> 1) & 1), slot = i & 1;
    c.t = t; c.f = f; c.q = slot; c.col = rs_col(S, r, f, slot);
  } else {
    const int j = i - nf1, v = j >> 3, t = 6 + ((j >> 2) & 1), q = j & 3;
    c.t = t; c.f = v; c.q = q; c.col = (v * S.nrT + r) * 4 + q;
  }
  return c;
}

// Balanced base-256 digits of round(v[i]), |round(v[i])| < 2^(8 NS - 2), for four
// values, packed as bytes (value i in byte i) into one word per slice; w[NS-1]
// holds the least significant digits.  Every digit d_s lies in [-128, 127],
// so x + K with K = 0x80 in each of the NS bytes has the bytes d_s + 128
// (0 < x + K < 2^(8 NS)); a balanced digit's two's-complement byte is that
// byte XOR 0x80.  The rounding to the nearest integer x (ties to even) adds
// 1.5 2^52, whose double then holds 2^52 + 2^51 + x in its mantissa; K is
// folded into the constant subtracted from those bits.
template <int NS>
__device__ __forceinline__ void digits4(const double (&v)[4], uint32_t (&w)[NS]) {
  static_assert(NS == 4 || NS == 6, "slice count");
  constexpr unsigned long long K = NS == 6 ? 0x808080808080ull : 0x80808080ull;
  constexpr long long C = 0x4338000000000000LL - (long long)K;
  uint32_t lo[4], hi[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long y = __double_as_longlong(v[i] + 6755399441055744.0) - C;
    lo[i] = (uint32_t)y ^ 0x80808080u;
    hi[i] = (uint32_t)((unsigned long long)y >> 32) ^ 0x80808080u;
  }
#pragma unroll
  for (int b = 0; b < NS; ++b) {
    const uint32_t* q = b < 4 ? lo : hi;
    const uint32_t sel = (uint32_t)(b & 3) | ((uint32_t)((b & 3) + 4) << 4);
    w[NS - 1 - b] = __byte_perm(__byte_perm(q[0], q[1], sel), __byte_perm(q[2], q[3], sel), 0x5410);
  }
}

// Slicer: one CTA per (field group z, radius r, order m).  Backward groups:
// z < nvb is vector z (types 0/1 from its theta/phi components); z = nvb is
// the radial components and scalars (types 2/3).  Forward groups: z = 0 is the
// radial components and scalars (types 4/5, record words [4 nvf, rec));
// z = 1 + v is vector v (types 6/7, record words [4v, 4v + 4)).
//
// Pass 1 builds the group's derived columns X[col][k] = B[k][col] 2^-dexp[k]
// in shared memory, one thread per theta row (forward) or degree l
// (backward), with the sym/asym combination, weights and factors of each
// column written out explicitly (the same algebra as the FP64 tier's operand
// loaders).  Pass 2 takes the column maxima, pass 3 cuts the digits.
template <bool FWD, int NS>
__global__ void __launch_bounds__(kSliceThreads) k_slice_mr(Plan P, SliceTabs S, const double* __restrict__ d_rj, long long ld,
                                                   const int* __restrict__ cols) {
  extern __shared__ double X[];
  const int z = blockIdx.x, r = P.r_lo + blockIdx.y, m = blockIdx.z;
  const int L = P.L;
  const int Kall = L - m + 1;
  const int nv = FWD ? P.nvf : P.nvb;
  const int nF = FWD ? P.nvf + P.nsf : P.nvb + P.nsb;
  const bool vgrp = FWD ? z > 0 : z < nv;  // vector (theta/phi) group
  const int v = FWD ? z - 1 : z;
  const int t0 = FWD ? (vgrp ? 6 : 4) : (vgrp ? 0 : 2);  // the group's two types: t0, t0 + 1
  const int ncolg = vgrp ? 8 : 4 * nF;                    // local columns: 4 per (type) for vectors
  int i0;
  if (!FWD) i0 = vgrp ? 8 * v : 8 * nv;
  else i0 = vgrp ? 4 * nF + 8 * v : 0;
  const TypeGeo ga = type_geo(t0, L, m, P.nh), gb = type_geo(t0 + 1, L, m, P.nh);
  const int kst = max(ga.kpad, gb.kpad);  // X row stride
  // local column c -> type: vectors 4 (t - t0) + q; radial/scalar 4 f + 2 (t - t0) + slot
  auto ctype = [&](int c) { return t0 + (vgrp ? (c >> 2) : ((c >> 1) & 1)); };
  const int* dxa = S.dexp + S.deoff[m * kNT + t0];
  const int* dxb = S.dexp + S.deoff[m * kNT + t0 + 1];
  const int nx = ncolg * kst;
  // Forward with m > 0 and no theta padding, pass 1 writes every X entry
  // (both parts of the vector types, both slots of every field)
  if (!(FWD && m > 0 && P.nh % kTK == 0)) {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) X[i] = 0.0;
    __syncthreads();
  }
  const double ar = 1.0 / P.radius[r];

  // ---- pass 1: derived columns
  if (FWD) {
    const int rec = 2 * P.ncf;
    const long long strideTh = rec;  // records of one (m, r) are contiguous over theta
    const double* base = P.rtm_f + rtm_off(P, m, 0, r, P.ncf) + (vgrp ? 4 * v : 4 * nv);
    // 256-bit loads need 32-byte aligned records (an even forward component count)
    const bool v4 = ((reinterpret_cast<uintptr_t>(P.rtm_f) | (uintptr_t)(16 * P.ncf)) & 31) == 0;
    double2 nxt = make_double2(0.0, 0.0), sxt = nxt;  // second field of a 256-bit load
    // the thread's second row is loaded (vector groups) or its first sector
    // pair (radial / scalar group: fields 0 and 1) before the first row is
    // processed: twice the loads in flight
    const int th2 = threadIdx.x + blockDim.x;
    const bool pre = v4 && th2 < P.nh && (vgrp || nF >= 2);
    double pn2[4] = {0.0, 0.0, 0.0, 0.0}, ps2[4] = {0.0, 0.0, 0.0, 0.0};
    if (pre) {
      ld_global_v4(base + th2 * strideTh, pn2[0], pn2[1], pn2[2], pn2[3]);
      if (th2 < P.nth / 2)
        ld_global_v4(base + (long long)(P.nth - 1 - th2) * strideTh, ps2[0], ps2[1], ps2[2], ps2[3]);
    }
    for (int th = threadIdx.x; th < P.nh; th += blockDim.x) {
      const bool hasS = th < P.nth / 2;
      const double w = __ldg(P.weight + th);
      const double* pn = base + th * strideTh;
      const double* ps = base + (long long)(P.nth - 1 - th) * strideTh;
      const double sa = pow2(-__ldg(dxa + th)), sb = pow2(-__ldg(dxb + th));
      if (vgrp) {
        // words (theta slot 0, theta slot 1, phi slot 0, phi slot 1): one
        // 32-byte sector per row, one 256-bit load when the records are aligned
        double nn[4], ss[4] = {0.0, 0.0, 0.0, 0.0};
        if (pre && th == th2) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            nn[c] = pn2[c];
            ss[c] = ps2[c];
          }
        } else if (v4) {
          ld_global_v4(pn, nn[0], nn[1], nn[2], nn[3]);
          if (hasS) ld_global_v4(ps, ss[0], ss[1], ss[2], ss[3]);
        } else {
          const double2 n01 = __ldg(reinterpret_cast<const double2*>(pn));
          const double2 n23 = __ldg(reinterpret_cast<const double2*>(pn + 2));
          nn[0] = n01.x; nn[1] = n01.y; nn[2] = n23.x; nn[3] = n23.y;
          if (hasS) {
            const double2 s01 = __ldg(reinterpret_cast<const double2*>(ps));
            const double2 s23 = __ldg(reinterpret_cast<const double2*>(ps + 2));
            ss[0] = s01.x; ss[1] = s01.y; ss[2] = s23.x; ss[3] = s23.y;
          }
        }
        double sy[4], as[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          sy[c] = (nn[c] + ss[c]) * w;
          as[c] = hasS ? (nn[c] - ss[c]) * w : 0.0;
        }
        const double ai = __ldg(P.asin_t + th);
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          // type 6 + p: dP part takes (N + S) for p = 1, the m P part (N + S) / sin for p = 0
          const double* A0 = p ? sy : as;
          const double* A1 = p ? as : sy;
          const TypeGeo& g = p ? gb : ga;
          const double s0 = p ? sb : sa;
          double* x = X + (4 * p) * kst;
          x[0 * kst + th] = A0[0] * s0;
          x[1 * kst + th] = A0[1] * s0;
          x[2 * kst + th] = -A0[2] * s0;
          x[3 * kst + th] = -A0[3] * s0;
          if (m > 0) {
            const int k1 = g.kpart0 + th;
            const double s1 = pow2(-__ldg((p ? dxb : dxa) + k1)) * ai;
            x[0 * kst + k1] = -A1[3] * s1;
            x[1 * kst + k1] = A1[2] * s1;
            x[2 * kst + k1] = -A1[1] * s1;
            x[3 * kst + k1] = A1[0] * s1;
          }
        }
      } else {
        for (int f = 0; f < nF; ++f) {
          double2 nn, ss = make_double2(0.0, 0.0);
          if (v4 && f + 1 < nF && !(f & 1)) {
            // fields f, f + 1 in one 32-byte sector
            double4 a, b = make_double4(0.0, 0.0, 0.0, 0.0);
            if (pre && th == th2 && f == 0) {
              a = make_double4(pn2[0], pn2[1], pn2[2], pn2[3]);
              b = make_double4(ps2[0], ps2[1], ps2[2], ps2[3]);
            } else {
              ld_global_v4(pn + 2 * f, a.x, a.y, a.z, a.w);
              if (hasS) ld_global_v4(ps + 2 * f, b.x, b.y, b.z, b.w);
            }
            nn = make_double2(a.x, a.y);
            ss = make_double2(b.x, b.y);
            nxt = make_double2(a.z, a.w);
            sxt = make_double2(b.z, b.w);
          } else if (v4 && (f & 1)) {
            nn = nxt;
            ss = sxt;
          } else {
            nn = __ldg(reinterpret_cast<const double2*>(pn + 2 * f));
            if (hasS) ss = __ldg(reinterpret_cast<const double2*>(ps + 2 * f));
          }
          X[(4 * f + 0) * kst + th] = (nn.x + ss.x) * w * sa;
          X[(4 * f + 2) * kst + th] = hasS ? (nn.x - ss.x) * w * sb : 0.0;
          if (m > 0) {
            X[(4 * f + 1) * kst + th] = (nn.y + ss.y) * w * sa;
            X[(4 * f + 3) * kst + th] = hasS ? (nn.y - ss.y) * w * sb : 0.0;
          }
        }
      }
    }
  } else {
    for (int kl = threadIdx.x; kl < Kall; kl += blockDim.x) {
      const int l = m + kl, p = kl & 1, kk = kl >> 1;
      const int j0 = __ldg(P.jmap + (long long)m * 2 * (L + 1) + l);
      const int j1 = m > 0 ? __ldg(P.jmap + ((long long)m * 2 + 1) * (L + 1) + l) : 0;
      const double* dr = d_rj + P.J * (long long)r;
      if (vgrp) {
        // x[c][slot], c = 0: dS/dr column (theta/phi source 1), c = 1: toroidal (source 2)
        const double* d1 = dr + ld * (cols[v] + 1);
        const double* d2 = dr + ld * (cols[v] + 2);
        const double x10 = __ldg(d1 + j0) * ar, x20 = __ldg(d2 + j0) * ar;
        const double x11 = m > 0 ? __ldg(d1 + j1) * ar : 0.0, x21 = m > 0 ? __ldg(d2 + j1) * ar : 0.0;
        // type 0 takes odd l - m into part 0 (dP) and even into part 1 (m P); type 1 the reverse
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const bool part1 = (t == 0) ? (p == 0) : (p == 1);
          const TypeGeo& g = t ? gb : ga;
          const int k = (part1 ? g.kpart0 : 0) + kk;
          const double sc = pow2(-__ldg((t ? dxb : dxa) + k));
          double* x = X + (4 * t) * kst + k;
          if (!part1) {
            x[0 * kst] = x10 * sc;
            x[1 * kst] = x11 * sc;
            x[2 * kst] = -x20 * sc;
            x[3 * kst] = -x21 * sc;
          } else {
            x[0 * kst] = x21 * sc;
            x[1 * kst] = -x20 * sc;
            x[2 * kst] = x11 * sc;
            x[3 * kst] = -x10 * sc;
          }
        }
      } else {
        const int t = p;  // type 2 (even l - m) or 3 (odd)
        const double sc = pow2(-__ldg((t ? dxb : dxa) + kk));
        const double fr = ar * ar * g3_of(l);
        for (int f = 0; f < nF; ++f) {
          const double* d = dr + ld * cols[f];
          const double fac = (f < nv ? fr : 1.0) * sc;
          X[(4 * f + 2 * t) * kst + kk] = __ldg(d + j0) * fac;
          if (m > 0) X[(4 * f + 2 * t + 1) * kst + kk] = __ldg(d + j1) * fac;
        }
      }
    }
  }
  __syncthreads();

  double* colmax = X + ((nx + 1) & ~1);
  int* colexp = reinterpret_cast<int*>(colmax + kGrpCols);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  // ---- pass 2: column maxima
  for (int c = warp; c < ncolg; c += nw) {
    const int t = ctype(c);
    const int kp = (t == t0) ? ga.kpad : gb.kpad;
    double mx = 0.0;
    for (int k = 2 * lane; k < kp; k += 64) {
      const double2 x2 = *reinterpret_cast<const double2*>(X + c * kst + k);
      mx = fmax(mx, fmax(fabs(x2.x), fabs(x2.y)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      const int e = mx > 0.0 ? exp_above(mx) : 0;
      colmax[c] = mx;
      colexp[c] = e;
      const ColRef cr = FWD ? colref_fwd(P, S, r, i0 + c) : colref_bwd(P, S, r, i0 + c);
      S.bexp[S.beoff[m * kNT + t] + cr.col] = e - (8 * NS - 2);
    }
  }
  __syncthreads();
  // ---- pass 3: digits.  Work item = (column group, 32-wide K chunk).  A
  // column group is the set of columns that share one 256-byte block of a
  // core-matrix tile: 8 rows (one radius of types 2..5) or 4 rows (one radius
  // and vector of types 0/1/6/7).  Lane l cuts 4 consecutive k (4 (l % 8) ..)
  // of block row l / 8 (and l / 8 + 4 in 8-row groups) into one word per
  // slice; the k half h = k / 16 of row rr sits at byte h 128 + rr 16 of the
  // block.  Backward, each lane stores its words in place (one warp-wide
  // store covers two or four whole 32-byte sectors of each slice).  Forward,
  // the warp assembles the block's NS slices in shared memory (k halves 192
  // bytes apart, so the word stores hit 32 distinct banks) and writes them
  // with 16-byte stores: at L = 511 the forward slicer takes 14.6 ms this way
  // and 16.0 ms with in-place word stores, the backward 6.2 and 4.8 ms (the
  // staging blocks cost the backward CTAs one resident CTA per SM).
  unsigned char* wb = nullptr;
  if constexpr (FWD)
    wb = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(colexp + kGrpCols) + 15) &
                                          ~static_cast<uintptr_t>(15)) +
         warp * (NS * kSlab);
  int item0 = 0;
  const int q4 = lane >> 3, kq = 4 * (lane & 7);
  const int nfg = vgrp ? 1 : rs_groups(nF);  // 8-row blocks: one per group of four fields
  for (int gi = 0; gi < 2 * nfg; ++gi) {
    const int t = t0 + (gi & 1), fg = gi >> 1;
    const bool eight = !vgrp;  // 8-row groups: radius blocks of types 2..5
    const int gcol = eight ? (fg * S.nrR + r) * 8 : (v * S.nrT + r) * 4;
    const TypeGeo& geo = (t == t0) ? ga : gb;
    const int nkc = geo.kpad / kTK;
    const int nt = gcol / kTN, blk = (gcol % kTN) >> 3, rbase = gcol & 7;
    signed char* base = S.B + S.boff[m * kNT + t];
    unsigned char* live = nullptr;  // forward: the tile's live-chunk flags
    if constexpr (FWD) live = S.bnz + 64 * (S.foff[m * kNT + t] + nt);
    for (int kc = ((warp - item0) % nw + nw) % nw; kc < nkc; kc += nw) {
      const int k = kc * kTK + kq;
      signed char* dst0 = base + (long long)(nt * nkc + kc) * NS * (kTN * kTK) + blk * 256;
      uint32_t anynz = 0u;  // forward: OR of this lane's digit words
      for (int q = q4; q < (eight ? 8 : 4); q += 4) {
        // local column of block row rbase + q
        int c = -1;
        if (!eight) c = 4 * (t - t0) + q;
        else if (4 * fg + (q >> 1) < nF) c = 4 * (4 * fg + (q >> 1)) + 2 * (t - t0) + (q & 1);
        uint32_t wd[NS];
        if (c >= 0 && colmax[c] > 0.0) {
          const double sc = pow2((8 * NS - 2) - colexp[c]);
          const double2 x01 = *reinterpret_cast<const double2*>(X + c * kst + k);
          const double2 x23 = *reinterpret_cast<const double2*>(X + c * kst + k + 2);
          const double xv[4] = {x01.x * sc, x01.y * sc, x23.x * sc, x23.y * sc};
          digits4<NS>(xv, wd);
        } else {
#pragma unroll
          for (int s2 = 0; s2 < NS; ++s2) wd[s2] = 0u;
        }
        if constexpr (FWD) {
#pragma unroll
          for (int s2 = 0; s2 < NS; ++s2) anynz |= wd[s2];
          const int o = (kq >> 4) * 192 + (rbase + q) * 16 + (kq & 15);
#pragma unroll
          for (int s2 = 0; s2 < NS; ++s2) *reinterpret_cast<uint32_t*>(wb + s2 * kSlab + o) = wd[s2];
        } else {
          signed char* dst = dst0 + (kq >> 4) * 128 + (rbase + q) * 16 + (kq & 15);
#pragma unroll
          for (int s2 = 0; s2 < NS; ++s2) *reinterpret_cast<uint32_t*>(dst + s2 * (kTN * kTK)) = wd[s2];
        }
      }
      if constexpr (FWD) {
        // live-chunk flag of the tile: every writer stores the same 1
        if (__any_sync(0xffffffffu, anynz != 0u) && lane == 0 && kc < 64) live[kc] = 1;
        __syncwarp();
        if (eight) {
          for (int u = lane; u < NS * 16; u += 32) {
            const int s2 = u >> 4, h = (u >> 3) & 1, rr = u & 7;
            *reinterpret_cast<uint4*>(dst0 + s2 * (kTN * kTK) + h * 128 + rr * 16) =
                *reinterpret_cast<const uint4*>(wb + s2 * kSlab + h * 192 + rr * 16);
          }
        } else {
          for (int u = lane; u < NS * 8; u += 32) {
            const int s2 = u >> 3, h = (u >> 2) & 1, rr = rbase + (u & 3);
            *reinterpret_cast<uint4*>(dst0 + s2 * (kTN * kTK) + h * 128 + rr * 16) =
                *reinterpret_cast<const uint4*>(wb + s2 * kSlab + h * 192 + rr * 16);
          }
        }
        __syncwarp();
      }
    }
    item0 += nkc;
  }
}

// ---------------------------------------------------------------------------
// The split GEMM: persistent, warp-specialised.
//   warp 0 (one lane): issues the tcgen05.mma slice products into TMEM
//   warp 1 (one lane): streams pre-laid-out slice tiles with bulk copies into a
//                      stage ring, running ahead across tiles
//   warps 2..17:       epilogue (TMEM -> FP64 recombination -> output), four per TMEM lane quadrant
// One tile = (m, type, m-tile, n-tile).  The work lists pair the two parity
// tiles (types 0/1, 2/3, 4/5 or 6/7) of one output tile; one CTA runs them back
// to back and keeps the first in shared memory.  Backward it then emits the
// north row (first + second) and the south row (first - second) of the rtm
// records; forward it scatters both degrees l and l + 1 of each row.
struct Work {
  int m, t, mt, nt;
};

struct GemmArgs {
  Plan P;
  SliceTabs S;
  const Work* work;
  int nwork;
  int pair;        // 1: backward (rtm records out), 0: forward (d_rj out)
  double* d_rj;    // forward output
  long long ld;
  const int* cols;
  int* err;        // device error word
};

constexpr int kEpiWarps = 16;                // four per TMEM lane quadrant
constexpr int kGemmWarps = 2 + kEpiWarps;    // MMA issuer, bulk-copy producer, epilogue
constexpr int kCols = kTN * 4 / kEpiWarps;   // columns recombined by one epilogue warp
constexpr int kLd = 8;                       // columns per TMEM load
constexpr int kRing = 4;           // stage ring depth
constexpr int kXS = kTN + 2;       // stash row stride (doubles): 16-byte rows, conflict-free v2 accesses

__host__ __device__ constexpr unsigned make_idesc(int n) {
  // kind::i8: D s32 (2 << 4), A s8 (1 << 7), B s8 (1 << 10), K-major A/B, N = n, M = 128
  return (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(kTM >> 4) << 24);
}

// MMA schedule of one K chunk.  The B slices of a stage are consecutive 64-row
// core-matrix tiles (stride 256 B per 8 rows), so slices b .. b+nb-1 form one
// N = 64·nb operand, and the product A_a·[B_b .. B_b+nb-1] lands in the
// consecutive TMEM groups a+b .. a+b+nb-1.  This issues the 26 (10) slice
// products of tier split (fp32acc) as 9 (4) MMAs of N up to 256.  In the first
// chunk of a tile the entries flagged `init` run first without accumulation:
// together they cover every group exactly once and touch no group written
// before them.  Group g >= NS is first written by the single product
// (g - NS + 2, NS - 2), which the a-row runs then skip.
template <int NS, int TG>
struct MmaSched {
  int n = 0;
  int a[24] = {}, b[24] = {}, nb[24] = {}, init[24] = {};
  constexpr void push(int aa, int bb, int nn, int ii) {
    a[n] = aa; b[n] = bb; nb[n] = nn; init[n] = ii; ++n;
  }
  static constexpr bool is_single(int aa, int bb) { return bb == NS - 2 && aa >= 2 && aa <= TG - NS + 2; }
  constexpr MmaSched() {
    const int top0 = (NS - 1 < TG) ? NS - 1 : TG;
    for (int b0 = 0; b0 <= top0; b0 += 4) push(0, b0, (top0 - b0 + 1 < 4) ? top0 - b0 + 1 : 4, 1);
    for (int g = NS; g <= TG; ++g) push(g - NS + 2, NS - 2, 1, 1);
    for (int aa = 1; aa < NS; ++aa) {
      const int top = (NS - 1 < TG - aa) ? NS - 1 : TG - aa;
      int b0 = 0;
      while (b0 <= top) {
        int b1 = b0;  // run [b0, b1) avoiding the init singles
        while (b1 <= top && b1 - b0 < 4 && !is_single(aa, b1)) ++b1;
        if (b1 > b0) push(aa, b0, b1 - b0, 0);
        b0 = (b1 > b0) ? b1 : b0 + 1;
      }
    }
  }
};

// d = a * b + c with a 32 x 32 -> 64-bit signed product (one wide integer multiply-add)
__device__ __forceinline__ long long mad_wide(int a, int b, long long c) {
  long long d;
  asm("mad.wide.s32 %0, %1, %2, %3;\n" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}
// Integers x with |x| < 2^51 are carried as the bit pattern of the double
// 1.5 2^52 + x (that double's mantissa is 2^51 + x, its ulp 1): kBias + x read
// as a double, minus 1.5 2^52, is x exactly.
constexpr long long kBias = 0x4338000000000000LL;
constexpr double kBiasD = 6755399441055744.0;  // 1.5 2^52
template <int NS>
__host__ __device__ constexpr size_t gemm_stage_bytes() { return (size_t)NS * (kTM + kTN) * kTK; }

// 32-byte global store (sm_100 256-bit st.global); p must be 32-byte aligned
__device__ __forceinline__ void st_global_v4(double* p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};\n" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

// Launch parameters: one instance (a), or a group of instances of one tier
// whose pair units run in one persistent launch (GROUPED: unit u is pair
// gunit[u].y of instance gunit[u].x, with that instance's arguments inst[.]).
struct GemmLaunch {
  GemmArgs a;  // grouped: only pair and err are used
  const GemmArgs* inst;
  const int2* gunit;
  int gunits;
};

// Live K chunks of a work tile: forward tiles of at most 64 chunks read the
// forward slicer's bits, every other tile takes all chunks.
__device__ __forceinline__ unsigned long long chunk_mask(const SliceTabs& S, const Work& w, int nk, bool bwd) {
  if (bwd || nk <= 0 || nk > 64) return ~0ull;
  const uint4* f = reinterpret_cast<const uint4*>(S.bnz + 64 * (S.foff[w.m * kNT + w.t] + w.nt));
  unsigned long long mk = 0ull;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (16 * i >= nk) break;
    const uint4 q = __ldg(f + i);
    const unsigned x[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      // flag bytes (0 or 1) of chunks 16 i + 4 j .. + 3 -> four bits
      const unsigned b = (x[j] & 1u) | ((x[j] >> 7) & 2u) | ((x[j] >> 14) & 4u) | ((x[j] >> 21) & 8u);
      mk |= (unsigned long long)b << (16 * i + 4 * j);
    }
  }
  return mk;
}

template <int NS, int TG, bool GROUPED>
__global__ void __launch_bounds__(kGemmWarps * 32, 1) k_split_gemm(const __grid_constant__ GemmLaunch L) {
  extern __shared__ __align__(1024) unsigned char sm[];
  constexpr int A_BYTES = NS * kTM * kTK, B_BYTES = NS * kTN * kTK;
  constexpr int STAGE = A_BYTES + B_BYTES;
  double* stash = reinterpret_cast<double*>(sm + kRing * STAGE);  // [kTM][kXS]: first tile of a pair
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(stash + kTM * kXS);
  unsigned long long* full = bars;              // [kRing]
  unsigned long long* empty = bars + kRing;     // [kRing]
  unsigned long long* done = bars + 2 * kRing;  // accumulators ready
  unsigned long long* tfree = done + 1;         // TMEM drained by the epilogue
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(tfree + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // units are (even, odd) parity tile pairs run back to back by one CTA
  const bool bwd = L.a.pair != 0;
  const int per = 2;
  const int nunits = GROUPED ? L.gunits : L.a.nwork / per;
  // arguments of unit u and the index of its first work item
  auto unit = [&](int u, int& base) -> const GemmArgs& {
    if constexpr (GROUPED) {
      const int2 g = L.gunit[u];
      base = per * g.y;
      return L.inst[g.x];
    } else {
      base = per * u;
      return L.a;
    }
  };

  if (threadIdx.x == 0) {
    for (int q = 0; q < kRing; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], 1);
    }
    mbar_init(done, 1);
    mbar_init(tfree, kEpiWarps);
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

  auto nk_of = [&](const Plan& P, const Work& w) -> int {
    const TypeGeo g = type_geo(w.t, P.L, w.m, P.nh);
    return (g.rows > 0 && w.mt * kTM < g.rpad) ? g.kpad / kTK : 0;
  };

  if (warp == 1) {
    if (lane == 0) {
      // ---- producer
      long long gc = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        int base;
        const GemmArgs& A = unit(u, base);
        const SliceTabs& S = A.S;
        for (int h = 0; h < per && ok; ++h) {
          const Work w = A.work[base + h];
          const int nk = nk_of(A.P, w);
          const signed char* Ag = S.A + S.aoff[w.m * kNT + w.t] + (long long)w.mt * nk * A_BYTES;
          const signed char* Bg = S.B + S.boff[w.m * kNT + w.t] + (long long)w.nt * nk * B_BYTES;
          const unsigned long long live = chunk_mask(S, w, nk, bwd);
          for (int kc = 0; kc < nk; ++kc) {
            if (!((live >> (kc & 63)) & 1ull)) continue;  // all-zero B digits: nothing to add
            const int st = (int)(gc % kRing);
            if (gc >= kRing && !mbar_wait(&empty[st], (unsigned)(((gc / kRing) - 1) & 1))) { ok = false; break; }
            mbar_expect_tx(&full[st], STAGE);
            bulk_g2s(sm + st * STAGE, Ag + (long long)kc * A_BYTES, A_BYTES, &full[st]);
            bulk_g2s(sm + st * STAGE + A_BYTES, Bg + (long long)kc * B_BYTES, B_BYTES, &full[st]);
            ++gc;
          }
        }
      }
      if (!ok) atomicExch(L.a.err, KMHD_ERR_TIMEOUT);
    }
  } else if (warp == 0) {
    if (lane == 0) {
      // ---- MMA issuer
      constexpr MmaSched<NS, TG> sch{};
      long long gc = 0;
      int it = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        int base;
        const GemmArgs& A = unit(u, base);
        for (int h = 0; h < per; ++h, ++it) {
          const Work w = A.work[base + h];
          const int nk = nk_of(A.P, w);
          const unsigned long long live = chunk_mask(A.S, w, nk, bwd);
          if (it > 0 && ok && !mbar_wait(tfree, (unsigned)((it - 1) & 1))) ok = false;
          tc_fence_after();
          int issued = 0;  // the first issued chunk initialises the accumulators
          for (int kc = 0; kc < nk && ok; ++kc) {
            if (!((live >> (kc & 63)) & 1ull)) continue;
            const int st = (int)(gc % kRing);
            if (!mbar_wait(&full[st], (unsigned)((gc / kRing) & 1))) { ok = false; break; }
            tc_fence_after();
            // descriptors of slice 0; slice s starts s tiles further (start address field, 16-byte units)
            const uint64_t a0 = smem_desc(sm + st * STAGE, 128, 256);
            const uint64_t b0 = smem_desc(sm + st * STAGE + A_BYTES, 128, 256);
#pragma unroll
            for (int q = 0; q < sch.n; ++q) {
              const unsigned acc = (issued > 0 || !sch.init[q]) ? 1u : 0u;
              mma_i8(tmem + (unsigned)((sch.a[q] + sch.b[q]) * kTN), a0 + (uint64_t)(sch.a[q] * (kTM * kTK / 16)),
                     b0 + (uint64_t)(sch.b[q] * (kTN * kTK / 16)), make_idesc(kTN * sch.nb[q]), acc);
            }
            mma_commit(&empty[st]);
            ++gc;
            ++issued;
          }
          mma_commit(done);
        }
      }
      if (!ok) atomicExch(L.a.err, KMHD_ERR_TIMEOUT);
    }
  } else {
    // ---- epilogue warps 2..17: TMEM lane quadrant = warp % 4, four warps per
    // quadrant, each recombining one 16-column quarter of the tile
    const int quad = warp & 3;
    const int part = (warp - 2) >> 2;
    const int cbase = kCols * part;
    const int row = quad * 32 + lane;
    constexpr int kW = 8 * (2 * NS - 2 - TG);  // weight exponent of the lowest kept group
    int it = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
      int base;
      const GemmArgs& A = unit(u, base);
      const Plan& P = A.P;
      const SliceTabs& S = A.S;
      // 32-byte stores into the rtm records need 32-byte aligned records
      const bool v4ok = ((reinterpret_cast<uintptr_t>(P.rtm_b) | (uintptr_t)(P.ncb * 16)) & 31) == 0;
      for (int h = 0; h < per; ++h, ++it) {
        const Work w = A.work[base + h];
        const int nk = nk_of(P, w);
        const TypeGeo g = type_geo(w.t, P.L, w.m, P.nh);
        const int grow = w.mt * kTM + row;
        const int eA = (grow < g.rows) ? S.aexp[S.aeoff[w.m * kNT + w.t] + grow] : 0;
        // column exponents: lane i holds column cbase + i, broadcast by shuffles
        const int eBl = lane < kCols ? __ldg(S.bexp + S.beoff[w.m * kNT + w.t] + w.nt * kTN + cbase + lane) : 0;
        const bool anylive = chunk_mask(S, w, nk, bwd) != 0ull;  // else no MMA wrote the accumulators
        // value scale 2^(ea + eB): built from its exponent bits when every
        // exponent of this warp's block is in the normal range (warp-uniform test)
        const int ea = eA + kW;
        const bool fast = __reduce_min_sync(0xffffffffu, ea) + __reduce_min_sync(0xffffffffu, lane < kCols ? eBl : 0x3fffffff) >= -1022 &&
                          __reduce_max_sync(0xffffffffu, ea) + __reduce_max_sync(0xffffffffu, lane < kCols ? eBl : -0x3fffffff) <= 1023;
        if (ok && !mbar_wait(done, (unsigned)(it & 1))) ok = false;
        ok = __all_sync(0xffffffffu, ok);
        tc_fence_after();
        double val[kCols];  // columns cbase .. cbase + kCols - 1
        if (nk > 0 && ok && anylive) {
          auto drain = [&](auto fastc) {
            constexpr bool F = decltype(fastc)::value;
#pragma unroll
            for (int cb = 0; cb < kCols / kLd; ++cb) {
              int acc[TG + 1][kLd];
#pragma unroll
              for (int gi = 0; gi <= TG; ++gi)
                tmem_ld8(tmem + ((unsigned)(quad * 32) << 16) + (unsigned)(gi * kTN + cbase + cb * kLd), acc[gi]);
              tmem_wait_ld();
#pragma unroll
              for (int c = 0; c < kLd; ++c) {
                // sum_g acc[g] 256^(TG-g): the (up to) four lowest groups combine
                // exactly in int64 (|lo| < 2^51), the higher ones likewise
                // (|hi| < 2^43), both by wide multiply-adds onto the bias; one
                // rounding where hi 256^(TG-G0+1) + lo is formed
                constexpr int G0 = TG >= 3 ? TG - 3 : 0;
                long long lo = mad_wide(acc[TG][c], 1, kBias);
#pragma unroll
                for (int gi = TG - 1; gi >= G0; --gi) lo = mad_wide(acc[gi][c], 1 << (8 * (TG - gi)), lo);
                double v = __longlong_as_double(lo) - kBiasD;
                if constexpr (G0 > 0) {
                  long long hi = mad_wide(acc[G0 - 1][c], 1, kBias);
#pragma unroll
                  for (int gi = G0 - 2; gi >= 0; --gi) hi = mad_wide(acc[gi][c], 1 << (8 * (G0 - 1 - gi)), hi);
                  v = fma(__longlong_as_double(hi) - kBiasD, pow2(8 * (TG - G0 + 1)), v);
                }
                const int eB = __shfl_sync(0xffffffffu, eBl, cb * kLd + c);
                const double sc = F ? __longlong_as_double((long long)(ea + eB + 1023) << 52) : pow2(ea + eB);
                val[cb * kLd + c] = v * sc;
              }
            }
          };
          if (fast) drain(std::true_type{});
          else drain(std::false_type{});
        } else {
#pragma unroll
          for (int c = 0; c < kCols; ++c) val[c] = 0.0;
        }
        // TMEM drained: one arrival per warp, after every lane's loads completed
        tc_fence_before();
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(sptr(tfree)) : "memory");

        if (h == 0) {
          // first tile of the pair: keep this thread's half row in shared memory
          double* sr = stash + row * kXS + cbase;
#pragma unroll
          for (int c = 0; c < kCols; c += 2) *reinterpret_cast<double2*>(sr + c) = make_double2(val[c], val[c + 1]);
        } else if (!bwd) {
          // forward pair: row i carries degree l0 = m + 2 (128 mt + i) in the even
          // tile (stash) and l0 + 1 in the odd tile (val).  Scatter both into d_rj
          // with the r, r^2, g7, g6 factors; neighbouring lanes write neighbouring
          // j, so every 32-byte sector is completed by this warp.  The column
          // parameters (radius, field column) are warp-uniform.
          const double* sr = stash + row * kXS + cbase;
          const TypeGeo ge = type_geo(w.t - 1, P.L, w.m, P.nh);
          const int l0 = w.m + 2 * grow, l1 = l0 + 1;
          const bool ok0 = grow < ge.rows && l0 <= P.L, ok1 = grow < g.rows && l1 <= P.L;
          const bool s1 = w.m > 0;
          const long long jm = (long long)w.m * 2 * (P.L + 1);
          const long long j00 = ok0 ? P.jmap[jm + l0] : 0, j01 = (ok0 && s1) ? P.jmap[jm + P.L + 1 + l0] : 0;
          const long long j10 = ok1 ? P.jmap[jm + l1] : 0, j11 = (ok1 && s1) ? P.jmap[jm + P.L + 1 + l1] : 0;
          const double g70 = g7_of(l0, w.m), g71 = g7_of(l1, w.m);
          if (w.t == 5) {
            // column c = 8 (block - 8 nt) + 2 (f % 4) + slot, block = (f / 4) nrR + r
            const double g60 = g6_of(l0, w.m), g61 = g6_of(l1, w.m);
            // nrR is a multiple of 8, so the tile's 8-column blocks share one field group
            const int rg0 = w.nt * (kTN / 8) + cbase / 8;
            const int fg = rg0 / S.nrR, r0 = rg0 - fg * S.nrR;
#pragma unroll
            for (int rr = 0; rr < kCols / 8; ++rr) {
              const int r = r0 + rr;
              if (r >= P.nr) continue;
              const double r1 = P.radius[r];
              const long long jr = P.J * (long long)r;
#pragma unroll
              for (int f4 = 0; f4 < 4; ++f4) {
                const int f = 4 * fg + f4;
                if (f >= P.nvf + P.nsf) break;
                const bool vec = f < P.nvf;
                const double fac0 = vec ? r1 * r1 * g70 : g60, fac1 = vec ? r1 * r1 * g71 : g61;
                double* dst = A.d_rj + jr + A.ld * A.cols[f];
                const int c = 8 * rr + 2 * f4;
                if (ok0) {
                  dst[j00] = sr[c] * fac0;
                  if (s1) dst[j01] = sr[c + 1] * fac0;
                }
                if (ok1) {
                  dst[j10] = val[c] * fac1;
                  if (s1) dst[j11] = val[c + 1] * fac1;
                }
              }
            }
          } else {
            // column c = 4 (r + nrT v) + q, q = 2 (component - 1) + slot; nrT is a
            // multiple of 16, so the tile's columns belong to one vector
            const int rv0 = w.nt * (kTN / 4) + cbase / 4;
            const int v = rv0 / S.nrT, r0 = rv0 - v * S.nrT;
#pragma unroll
            for (int c4 = 0; c4 < kCols / 4; ++c4) {
              const int r = r0 + c4;
              if (v >= P.nvf) break;
              if (r >= P.nr) continue;
              const double rr1 = P.radius[r];
              const double fac0 = rr1 * g70, fac1 = rr1 * g71;
              double* dst = A.d_rj + P.J * (long long)r + A.ld * (A.cols[v] + 1);
              const int c = 4 * c4;
              if (ok0) {
                dst[j00] = sr[c] * fac0;
                dst[j00 + A.ld] = sr[c + 2] * fac0;
                if (s1) {
                  dst[j01] = sr[c + 1] * fac0;
                  dst[j01 + A.ld] = sr[c + 3] * fac0;
                }
              }
              if (ok1) {
                dst[j10] = val[c] * fac1;
                dst[j10 + A.ld] = val[c + 2] * fac1;
                if (s1) {
                  dst[j11] = val[c + 1] * fac1;
                  dst[j11 + A.ld] = val[c + 3] * fac1;
                }
              }
            }
          }
        } else {
          // second backward tile: north row th gets first + second, south row
          // nth-1-th first - second; an odd-Ntheta equator row gets the first alone
          const int th = grow;
          if (th < P.nh && ok) {
            const bool pairrow = th < P.nth / 2;
            const double* sr = stash + row * kXS + cbase;
            const long long rec = (long long)P.nth * P.ncb * 2;  // radius stride of the rtm records
            double* baseN = P.rtm_b + rtm_off(P, w.m, th, 0, P.ncb);
            double* baseS = P.rtm_b + rtm_off(P, w.m, P.nth - 1 - th, 0, P.ncb);
            if (w.t <= 1) {
              // column c = 4 (r + nrT v) + q: one vector's (theta c, theta s, phi c, phi s);
              // nrT is a multiple of 16, so the tile's columns belong to one vector
              const int g0 = (w.nt * kTN + cbase) >> 2;
              const int vv = g0 / S.nrT, r0 = g0 - vv * S.nrT;
#pragma unroll
              for (int c = 0; c < kCols; c += 4) {
                const int r = r0 + (c >> 2);
                if (vv >= P.nvb || r >= P.nr) continue;
                const double2 a01 = *reinterpret_cast<const double2*>(sr + c);
                const double2 a23 = *reinterpret_cast<const double2*>(sr + c + 2);
                double n[4], s_[4];
                const double a[4] = {a01.x, a01.y, a23.x, a23.y};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  n[q] = pairrow ? a[q] + val[c + q] : a[q];
                  s_[q] = a[q] - val[c + q];
                }
                double* dN = baseN + (long long)r * rec + 4 * vv;
                double* dS = baseS + (long long)r * rec + 4 * vv;
                if (v4ok) {
                  st_global_v4(dN, n[0], n[1], n[2], n[3]);
                  if (pairrow) st_global_v4(dS, s_[0], s_[1], s_[2], s_[3]);
                } else {
                  reinterpret_cast<double2*>(dN)[0] = make_double2(n[0], n[1]);
                  reinterpret_cast<double2*>(dN)[1] = make_double2(n[2], n[3]);
                  if (pairrow) {
                    reinterpret_cast<double2*>(dS)[0] = make_double2(s_[0], s_[1]);
                    reinterpret_cast<double2*>(dS)[1] = make_double2(s_[2], s_[3]);
                  }
                }
              }
            } else {
              // column c = 8 (block - 8 nt) + 2 (f % 4) + slot, block = (f / 4) nrR + r:
              // radial components and scalars, record words 4 nvb + 2 f
              const int nF = P.nvb + P.nsb;
              // nrR is a multiple of 8, so the tile's 8-column blocks share one field group
              const int rg0 = w.nt * (kTN / 8) + cbase / 8;
              const int fg = rg0 / S.nrR, r0 = rg0 - fg * S.nrR;
#pragma unroll
              for (int rr = 0; rr < kCols / 8; ++rr) {
                const int r = r0 + rr;
                if (r >= P.nr || 4 * fg >= nF) continue;
                double* dN = baseN + (long long)r * rec + 4 * P.nvb + 8 * fg;
                double* dS = baseS + (long long)r * rec + 4 * P.nvb + 8 * fg;
                const int nFg = nF - 4 * fg;  // fields of this group (at most 4 used)
#pragma unroll
                for (int fp = 0; fp < 2; ++fp) {
                  const int c = 8 * rr + 4 * fp;
                  if (2 * fp >= nFg) break;
                  const double2 a01 = *reinterpret_cast<const double2*>(sr + c);
                  const double2 a23 = *reinterpret_cast<const double2*>(sr + c + 2);
                  const double a[4] = {a01.x, a01.y, a23.x, a23.y};
                  double n[4], s_[4];
#pragma unroll
                  for (int q = 0; q < 4; ++q) {
                    n[q] = pairrow ? a[q] + val[c + q] : a[q];
                    s_[q] = a[q] - val[c + q];
                  }
                  if (v4ok && 2 * fp + 1 < nFg) {
                    st_global_v4(dN + 4 * fp, n[0], n[1], n[2], n[3]);
                    if (pairrow) st_global_v4(dS + 4 * fp, s_[0], s_[1], s_[2], s_[3]);
                  } else {
                    reinterpret_cast<double2*>(dN + 4 * fp)[0] = make_double2(n[0], n[1]);
                    if (pairrow) reinterpret_cast<double2*>(dS + 4 * fp)[0] = make_double2(s_[0], s_[1]);
                    if (2 * fp + 1 < nFg) {
                      reinterpret_cast<double2*>(dN + 4 * fp)[1] = make_double2(n[2], n[3]);
                      if (pairrow) reinterpret_cast<double2*>(dS + 4 * fp)[1] = make_double2(s_[2], s_[3]);
                    }
                  }
                }
              }
            }
          }
        }
      }
    }
    if (!ok) atomicExch(L.a.err, KMHD_ERR_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
}

}  // namespace

// ---------------------------------------------------------------------------
struct SplitState {
  int tier, ns, T;
  SliceTabs S;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  std::vector<long long> aoff, aeoff, deoff, boff, beoff, foff;
  long long nbnz = 0;  // 64-byte tile blocks of S.bnz
  Work* work_b = nullptr;  // backward work (parity tile pairs)
  Work* work_f = nullptr;  // forward work
  int nwork_b = 0, nwork_f = 0;
  std::vector<Work> wb_h, wf_h;  // host copies of the work lists
  // radial chunks: bounds [chunk_lo[c], chunk_lo[c + 1]) and each chunk's
  // slice of the chunk-ordered work lists work_bc / work_fc
  std::vector<int> chunk_lo, cb_off, cf_off;
  Work* work_bc = nullptr;
  Work* work_fc = nullptr;
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
  const size_t stage = (size_t)ns * (kTM + kTN) * kTK;
  return kRing * stage + sizeof(double) * kTM * kXS + (2 * kRing + 6) * 8 + 64;
}

template <int NS, int TG, bool GROUPED>
cudaError_t launch_gemm(const GemmLaunch& l, int units, cudaStream_t st) {
  auto kern = k_split_gemm<NS, TG, GROUPED>;
  const size_t smem = gemm_smem(NS);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::min(units, nsm);
  if (grid <= 0) return cudaSuccess;
  kern<<<grid, kGemmWarps * 32, smem, st>>>(l);
  return cudaGetLastError();
}

template <int NS, int TG>
cudaError_t launch_gemm(const GemmArgs& a, cudaStream_t st) {
  GemmLaunch l;
  l.a = a;
  l.inst = nullptr;
  l.gunit = nullptr;
  l.gunits = 0;
  return launch_gemm<NS, TG, false>(l, a.nwork / 2, st);
}

// Instantiations: the split tier keeps the digit pairs a + b <= 6 (26
// products) or <= 5 (21), the fp32acc tier a + b <= 3 (10) or <= 2 (6).
cudaError_t run_gemm(const SplitState* s, const GemmArgs& a, cudaStream_t st) {
  if (s->ns == 6) return s->T == 6 ? launch_gemm<6, 6>(a, st) : launch_gemm<6, 5>(a, st);
  return s->T == 3 ? launch_gemm<4, 3>(a, st) : launch_gemm<4, 2>(a, st);
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
  if (4 * (p.nvb + p.nsb) > kGrpCols || 4 * (p.nvf + p.nsf) > kGrpCols) return KMHD_ERR_SIZE;
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
    else if (t <= 3) n = 8 * S.nrR * rs_groups(p.nvb + p.nsb);
    else if (t <= 5) n = 8 * S.nrR * rs_groups(p.nvf + p.nsf);
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
  s->foff.resize((L + 1) * kNT);
  long long ao = 0, aeo = 0, deo = 0, bo = 0, beo = 0, fo = 0;
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
      s->foff[i] = fo;
      if (t >= 4) fo += S.npadT[t] / kTN;
      ao += (long long)g.rpad * g.kpad * s->ns;
      aeo += g.rpad;
      deo += g.kpad;
      bo += (long long)S.npadT[t] * g.kpad * s->ns;
      beo += S.npadT[t];
    }
  // work lists: parity pairs (0,1), (2,3) backward and (4,5), (6,7) forward per
  // (m, n-tile, m-tile), m-tile fastest: the units that read the same B panel
  // are adjacent in the list, start together on neighbouring CTAs and share
  // its chunks in L2.  A forward pair whose odd-parity type has one m-tile
  // fewer keeps that tile as an empty partner (no K chunks).
  for (int m = 0; m <= L; ++m) {
    for (int tp = 0; tp < 4; tp += 2) {
      if ((tp == 0 && p.nvb == 0)) continue;
      const TypeGeo g = type_geo(tp, L, m, p.nh);
      const int nn = S.npadT[tp] / kTN;
      for (int nt = 0; nt < nn; ++nt)
        for (int mt = 0; mt < g.rpad / kTM; ++mt) {
          wb.push_back({m, tp, mt, nt});
          wb.push_back({m, tp + 1, mt, nt});
        }
    }
    for (int tp = 4; tp < 8; tp += 2) {
      if (tp == 6 && p.nvf == 0) continue;
      const TypeGeo g = type_geo(tp, L, m, p.nh);  // even parity: at least as many rows as odd
      if (g.rows <= 0) continue;
      const int nn = S.npadT[tp] / kTN;
      for (int nt = 0; nt < nn; ++nt)
        for (int mt = 0; mt < g.rpad / kTM; ++mt) {
          wf.push_back({m, tp, mt, nt});
          wf.push_back({m, tp + 1, mt, nt});
        }
    }
  }
  int st_ = KMHD_OK;
  long long *aoff_d, *aeoff_d, *deoff_d, *boff_d, *beoff_d, *foff_d;
  s->nbnz = fo;
  if (p.err) s->err = p.err;  // the instance's error word
  if ((st_ = salloc(s, &S.A, (size_t)ao)) || (st_ = salloc(s, &S.aexp, (size_t)aeo)) ||
      (st_ = salloc(s, &S.dexp, (size_t)deo)) || (st_ = salloc(s, &S.B, (size_t)bo)) ||
      (st_ = salloc(s, &S.bexp, (size_t)beo)) || (st_ = salloc(s, &aoff_d, s->aoff.size())) ||
      (st_ = salloc(s, &aeoff_d, s->aeoff.size())) || (st_ = salloc(s, &deoff_d, s->deoff.size())) ||
      (st_ = salloc(s, &boff_d, s->boff.size())) || (st_ = salloc(s, &beoff_d, s->beoff.size())) ||
      (st_ = salloc(s, &foff_d, s->foff.size())) || (st_ = salloc(s, &S.bnz, (size_t)fo * 64)) ||
      (st_ = salloc(s, &s->work_b, wb.size())) || (st_ = salloc(s, &s->work_f, wf.size())) ||
      (!p.err && (st_ = salloc(s, &s->err, 1)))) {
    split_destroy(s);
    return st_;
  }
  S.aoff = aoff_d;
  S.aeoff = aeoff_d;
  S.deoff = deoff_d;
  S.boff = boff_d;
  S.beoff = beoff_d;
  S.foff = foff_d;
  s->nwork_b = (int)wb.size();
  s->nwork_f = (int)wf.size();
  s->wb_h = wb;
  s->wf_h = wf;
  auto up = [&](void* d, const void* h, size_t b) { return cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, st); };
  if (up(aoff_d, s->aoff.data(), sizeof(long long) * s->aoff.size()) ||
      up(aeoff_d, s->aeoff.data(), sizeof(long long) * s->aeoff.size()) ||
      up(deoff_d, s->deoff.data(), sizeof(long long) * s->deoff.size()) ||
      up(boff_d, s->boff.data(), sizeof(long long) * s->boff.size()) ||
      up(beoff_d, s->beoff.data(), sizeof(long long) * s->beoff.size()) ||
      up(foff_d, s->foff.data(), sizeof(long long) * s->foff.size()) ||
      cudaMemsetAsync(S.bnz, 0, 64 * (size_t)(fo > 0 ? fo : 1), st) ||
      (wb.size() && up(s->work_b, wb.data(), sizeof(Work) * wb.size())) ||
      (wf.size() && up(s->work_f, wf.data(), sizeof(Work) * wf.size())) ||
      cudaMemsetAsync(s->err, 0, sizeof(int), st) || cudaMemsetAsync(S.B, 0, (size_t)bo, st) ||
      cudaMemsetAsync(S.bexp, 0, sizeof(int) * (size_t)beo, st)) {
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

// First radius of a work tile's columns: vector types (0, 1, 6, 7) hold
// columns (v nrT + r) 4 + q, 16 radii per 64-column tile; radial/scalar types
// (2..5) hold ((f / 4) nrR + r) 8 + 2 (f % 4) + slot, 8 radii per tile (nrR is
// a multiple of 8, so no tile spans two field groups).
static int tile_r0(const SliceTabs& S, const Work& w) {
  if (w.t <= 1 || w.t >= 6) return (16 * w.nt) % S.nrT;
  return (8 * w.nt) % S.nrR;
}

int split_set_chunks(SplitState* s, const Plan& p, const std::vector<int>& bounds, cudaStream_t st) {
  const int nc = (int)bounds.size() - 1;
  if (nc < 1 || bounds.front() != 0 || bounds.back() != p.nr) return KMHD_ERR_ARG;
  for (int c = 0; c < nc; ++c)
    if (bounds[c + 1] <= bounds[c] || bounds[c] % 16 != 0) return KMHD_ERR_ARG;
  auto chunk_of = [&](int r0) {
    int c = 0;
    while (c + 1 < nc && r0 >= bounds[c + 1]) ++c;
    return c;
  };
  // stable per-chunk filtering keeps each parity pair together and the
  // m-tile-fastest order inside a chunk
  auto split_list = [&](const std::vector<Work>& w, std::vector<Work>& out, std::vector<int>& off) {
    out.clear();
    off.assign(nc + 1, 0);
    for (int c = 0; c < nc; ++c) {
      off[c] = (int)out.size();
      for (size_t i = 0; i < w.size(); ++i)
        if (chunk_of(tile_r0(s->S, w[i])) == c) out.push_back(w[i]);
    }
    off[nc] = (int)out.size();
  };
  std::vector<Work> bc, fc;
  split_list(s->wb_h, bc, s->cb_off);
  split_list(s->wf_h, fc, s->cf_off);
  if (bc.size() != s->wb_h.size() || fc.size() != s->wf_h.size()) return KMHD_ERR_ARG;
  int e;
  if (!s->work_bc && (e = salloc(s, &s->work_bc, bc.size()))) return e;
  if (!s->work_fc && (e = salloc(s, &s->work_fc, fc.size()))) return e;
  if ((bc.size() && cudaMemcpyAsync(s->work_bc, bc.data(), sizeof(Work) * bc.size(), cudaMemcpyHostToDevice, st)) ||
      (fc.size() && cudaMemcpyAsync(s->work_fc, fc.data(), sizeof(Work) * fc.size(), cudaMemcpyHostToDevice, st)))
    return KMHD_ERR_CUDA;
  s->chunk_lo = bounds;
  return cudaStreamSynchronize(st) == cudaSuccess ? KMHD_OK : KMHD_ERR_CUDA;
}

// Work list of the plan's radial window: the whole list, or one chunk's slice.
static int select_work(const SplitState* s, const Plan& p, bool fwd, const Work** w, int* n) {
  if (p.r_lo == 0 && p.r_hi == p.nr) {
    *w = fwd ? s->work_f : s->work_b;
    *n = fwd ? s->nwork_f : s->nwork_b;
    return KMHD_OK;
  }
  for (size_t c = 0; c + 1 < s->chunk_lo.size(); ++c)
    if (s->chunk_lo[c] == p.r_lo && s->chunk_lo[c + 1] == p.r_hi) {
      const std::vector<int>& off = fwd ? s->cf_off : s->cb_off;
      *w = (fwd ? s->work_fc : s->work_bc) + off[c];
      *n = off[c + 1] - off[c];
      return KMHD_OK;
    }
  return KMHD_ERR_ARG;
}

// dynamic shared memory of one slicer CTA (largest field group): the derived
// columns X[col][k] (k up to the padded K of the group's types), the column
// maxima and exponents, and (forward) eight per-warp slice staging blocks
size_t slice_smem(const Plan& p, bool fwd, int ns) {
  // K shrinks with m for the backward types and is m-independent forward: m = 0 is the largest
  const int nF = fwd ? p.nvf + p.nsf : p.nvb + p.nsb;
  const int tv = fwd ? 6 : 0, tr = fwd ? 4 : 2;
  const size_t kv = std::max(type_geo(tv, p.L, 0, p.nh).kpad, type_geo(tv + 1, p.L, 0, p.nh).kpad);
  const size_t kr = std::max(type_geo(tr, p.L, 0, p.nh).kpad, type_geo(tr + 1, p.L, 0, p.nh).kpad);
  const size_t nx = std::max(8 * kv, 4 * (size_t)nF * kr);
  const size_t stage = fwd ? (kSliceThreads / 32) * (size_t)ns * kSlab + 16 : 0;
  return sizeof(double) * (nx + 1 + kGrpCols) + kGrpCols * sizeof(int) + stage;
}

int split_slicer(SplitState* s, const Plan& p, bool fwd, const double* d_rj, long long ld, const int* cols,
                 cudaStream_t st) {
  const SliceTabs& S = s->S;
  const size_t smem = slice_smem(p, fwd, s->ns);
  auto kern = fwd ? (s->ns == 6 ? k_slice_mr<true, 6> : k_slice_mr<true, 4>)
                  : (s->ns == 6 ? k_slice_mr<false, 6> : k_slice_mr<false, 4>);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return KMHD_ERR_CUDA;
  // the forward slicer sets the live-chunk bits of the tiles it cuts
  if (fwd && p.r_hi > p.r_lo && s->nbnz > 0 &&
      cudaMemsetAsync(S.bnz, 0, 64 * (size_t)s->nbnz, st) != cudaSuccess)
    return KMHD_ERR_CUDA;
  if (p.r_hi > p.r_lo)
    kern<<<dim3((fwd ? p.nvf : p.nvb) + 1, p.r_hi - p.r_lo, p.L + 1), kSliceThreads, smem, st>>>(p, S, d_rj, ld, cols);
  return cudaGetLastError() == cudaSuccess ? KMHD_OK : KMHD_ERR_CUDA;
}

// Arguments of one instance's GEMM in direction fwd over the plan's window.
static int gemm_args(const SplitState* s, const Plan& p, bool fwd, double* d_rj, long long ld, const int* cols,
                     GemmArgs* a) {
  a->P = p;
  a->S = s->S;
  const int e = select_work(s, p, fwd, &a->work, &a->nwork);
  if (e != KMHD_OK) return e;
  a->pair = fwd ? 0 : 1;
  a->d_rj = fwd ? d_rj : nullptr;
  a->ld = fwd ? ld : 0;
  a->cols = fwd ? cols : nullptr;
  a->err = s->err;
  return KMHD_OK;
}

int split_bwd(SplitState* s, const Plan& p, int, const double* d_rj, long long ld, const int* cols, cudaStream_t st,
              cudaEvent_t mid) {
  int e = split_slicer(s, p, false, d_rj, ld, cols, st);
  if (e != KMHD_OK) return e;
  if (mid && cudaEventRecord(mid, st) != cudaSuccess) return KMHD_ERR_CUDA;
  GemmArgs a;
  if ((e = gemm_args(s, p, false, nullptr, 0, nullptr, &a)) != KMHD_OK) return e;
  if (a.nwork > 0 && run_gemm(s, a, st) != cudaSuccess) return KMHD_ERR_CUDA;
  return KMHD_OK;
}

int split_fwd(SplitState* s, const Plan& p, double* d_rj, long long ld, const int* cols, cudaStream_t st,
              cudaEvent_t mid) {
  int e = split_slicer(s, p, true, nullptr, 0, nullptr, st);
  if (e != KMHD_OK) return e;
  if (mid && cudaEventRecord(mid, st) != cudaSuccess) return KMHD_ERR_CUDA;
  GemmArgs a;
  if ((e = gemm_args(s, p, true, d_rj, ld, cols, &a)) != KMHD_OK) return e;
  if (a.nwork > 0 && run_gemm(s, a, st) != cudaSuccess) return KMHD_ERR_CUDA;
  return KMHD_OK;
}

int split_ns(const SplitState* s) { return s ? s->ns : 0; }
int split_terms(const SplitState* s) { return s ? s->T : 0; }

int split_products(int ns, int T) {
  int n = 0;
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b) n += a + b <= T;
  return n;
}

int split_set_terms(SplitState* s, int T) {
  if (!s) return KMHD_ERR_ARG;
  const int full = s->ns == 6 ? 6 : 3;
  if (T != full && T != full - 1) return KMHD_ERR_ARG;
  s->T = T;
  s->S.T = T;
  return KMHD_OK;
}

// ---------------------------------------------------------------------------
// Grouped GEMM of several instances of one tier: per direction one device
// array of the instances' arguments and one list of (instance, pair unit),
// largest instance first; one persistent launch runs them all.
struct SplitGroup {
  int ns = 0, T = 0, n = 0;
  GemmArgs* inst[2] = {nullptr, nullptr};  // [bwd, fwd]
  int2* unit[2] = {nullptr, nullptr};
  int nunit[2] = {0, 0};
  int* err = nullptr;
};

void split_group_destroy(SplitGroup* g) {
  if (!g) return;
  for (int d = 0; d < 2; ++d) {
    cudaFree(g->inst[d]);
    cudaFree(g->unit[d]);
  }
  delete g;
}

int split_group_create(SplitGroup** out, SplitState* const* ss, const Plan* plans, int n, double* const* d_rj_out,
                       const long long* ld_out, const int* const* cols_f, cudaStream_t st) {
  *out = nullptr;
  if (n < 1) return KMHD_ERR_ARG;
  SplitGroup* g = new SplitGroup();
  g->ns = ss[0]->ns;
  g->T = ss[0]->T;
  g->n = n;
  g->err = ss[0]->err;
  for (int d = 0; d < 2; ++d) {
    const bool fwd = d == 1;
    std::vector<GemmArgs> args(n);
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) {
      if (ss[i]->ns != g->ns || ss[i]->T != g->T) { split_group_destroy(g); return KMHD_ERR_ARG; }
      Plan p = plans[i];
      p.r_lo = 0;
      p.r_hi = p.nr;
      const int e = gemm_args(ss[i], p, fwd, d_rj_out[i], ld_out[i], cols_f[i], &args[i]);
      if (e != KMHD_OK) { split_group_destroy(g); return e; }
      order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return args[a].nwork > args[b].nwork; });
    std::vector<int2> units;
    for (int i : order)
      for (int u = 0; u < args[i].nwork / 2; ++u) units.push_back(make_int2(i, u));
    g->nunit[d] = (int)units.size();
    if (cudaMalloc(&g->inst[d], sizeof(GemmArgs) * n) != cudaSuccess ||
        cudaMalloc(&g->unit[d], sizeof(int2) * std::max<size_t>(units.size(), 1)) != cudaSuccess) {
      split_group_destroy(g);
      return KMHD_ERR_NOMEM;
    }
    if (cudaMemcpyAsync(g->inst[d], args.data(), sizeof(GemmArgs) * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (units.size() && cudaMemcpyAsync(g->unit[d], units.data(), sizeof(int2) * units.size(),
                                         cudaMemcpyHostToDevice, st) != cudaSuccess) ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      split_group_destroy(g);
      return KMHD_ERR_CUDA;
    }
  }
  *out = g;
  return KMHD_OK;
}

int split_group_gemm(SplitGroup* g, bool fwd, cudaStream_t st) {
  const int d = fwd ? 1 : 0;
  GemmLaunch l;
  std::memset(&l.a, 0, sizeof(l.a));
  l.a.pair = fwd ? 0 : 1;
  l.a.err = g->err;
  l.inst = g->inst[d];
  l.gunit = g->unit[d];
  l.gunits = g->nunit[d];
  cudaError_t e;
  if (g->ns == 6) e = g->T == 6 ? launch_gemm<6, 6, true>(l, l.gunits, st) : launch_gemm<6, 5, true>(l, l.gunits, st);
  else e = g->T == 3 ? launch_gemm<4, 3, true>(l, l.gunits, st) : launch_gemm<4, 2, true>(l, l.gunits, st);
  return e == cudaSuccess ? KMHD_OK : KMHD_ERR_CUDA;
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
    mma_i8(tmem, smem_desc(sa, lbo, sbo), smem_desc(sb, lbo, sbo), make_idesc(kTN), 0u);
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

namespace kmhd {
namespace {
// Failure-path self-test: the tcgen05 pipeline's bounded mbarrier wait on a
// barrier that nothing arrives on runs out and records KMHD_ERR_TIMEOUT.
__global__ void k_selftest_pipe_wait(int* err) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0, kSelfTestSpinCap)) atomicExch(err, KMHD_ERR_TIMEOUT);
}
}  // namespace
}  // namespace kmhd

extern "C" int kmhd_selftest_wait_timeout(int device, int which) {
  using namespace kmhd;
  if (which != 0 && which != 1) return KMHD_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return KMHD_ERR_DEVICE;
  int* err = nullptr;
  if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return KMHD_ERR_NOMEM;
  int st = KMHD_OK;
  if (cudaMemset(err, 0, sizeof(int)) != cudaSuccess) st = KMHD_ERR_CUDA;
  if (!st) {
    if (which == 0) k_selftest_pipe_wait<<<1, 32>>>(err);
    else if (launch_selftest_fft_wait(err, nullptr) != cudaSuccess) st = KMHD_ERR_CUDA;
  }
  // the kernel ends by itself (bounded wait) and leaves the context usable
  if (!st && cudaDeviceSynchronize() != cudaSuccess) st = KMHD_ERR_CUDA;
  int h = 0;
  if (!st && cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) st = KMHD_ERR_CUDA;
  cudaFree(err);
  return st ? st : h;
}

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


