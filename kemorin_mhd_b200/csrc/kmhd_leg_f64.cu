// kmhd_leg_f64.cu -- FP64 equator-symmetric Legendre transforms on the FP64
// tensor pipe (mma.sync m8n8k4 f64, DMMA).
//
// Backward (reference: leg_b_trans_vec_sym_dgemm / leg_b_trans_scl_sym_dgemm,
// PARALLEL_src/SPH_SHELL_src/legendre_bwd_sym_matmul.f90:301-500, with the
// pack of set_sp_rlm_for_leg_matmul.f90:153-276 and the unpack of
// cal_vr_rtm_by_matmul.f90:163-352).  Per order m >= 0, per parity p of l-m:
//   V(theta, col) = sum_k Ptab[m][p][k][theta] * SB[m][p][k][col]
// for P and dP, then the N/S (sym +/- asym) recombination and the +-m cross
// terms are applied in registers and the grid spectra are written to
// rtm_b[m][theta][r][comp][cos,sin].
//
// Forward (leg_f_trans_vec_sym_dgemm, legendre_fwd_sym_matmul.f90:315-452,
// pack set_vr_rtm_for_leg_matmul.f90:170-364, unpack cal_sp_rlm_by_matmul.f90:172-360):
//   S(k, col) = sum_theta Ptab[m][p][k][theta] * X[m][p][theta][col]
// where X = (N +- S) * w (* 1/sin theta) is formed while staging rtm_f into
// shared memory, and the r, r^2, g7, g6, m factors are applied in the epilogue
// before the scatter into d_rj.
//
// Column blocks hold kRB = 4 radii of every field ("quads"): a vector quad has
// three 8-column tiles X = (b+, b-), Y = (c+, c-), Z = (a+, a-) per radius in the
// backward direction (a = S g3 / r^2, b = dS/dr / r, c = T / r), so the m8n8
// accumulator fragment of a thread (row g, columns 2t, 2t+1) holds the cos and
// sin slots of one radius.
#include <type_traits>

#include "kmhd_internal.cuh"

namespace kmhd {
namespace {

template <int NV, int NS>
struct BwdGeo {
  static constexpr int CB = 24 * NV + 8 * NS;                       // columns per r-block
  // row strides = 32 B mod 128 B: a half warp (4 fragment rows x 32 B) spans all banks
  static constexpr int CBp = CB + ((4 - CB % 16) + 16) % 16;
  static constexpr int AS = kThBlk + 4;                              // A row stride (doubles)
  static constexpr int A_STAGE = 2 * kKC * AS;                       // P and dP
  static constexpr int B_STAGE = kKC * CBp;
  static constexpr size_t SMEM = sizeof(double) * 2 * (A_STAGE + B_STAGE);
  // both parities per stage, and two chunk pairs' recurrence coefficients
  static constexpr size_t SMEM_OTF = sizeof(double) * 4 * (A_STAGE + B_STAGE) + sizeof(double2) * 16 * kKC;
};

// ---------------------------------------------------------------------------
// d_rj -> SB packing.  CTA = (m, 32-wide l chunk, r block); both parities.
__global__ void k_pack_b(Plan p, const double* __restrict__ d_rj, long long ld,
                         const int* __restrict__ cols, int nv, int ns, int CB) {
  extern __shared__ double sm[];
  const int m = blockIdx.y;
  const int nlc = p.kpad[2 * m] / kKC;  // chunks of 32 l (16 k per parity)
  const int nrbw = win_nrb(p);
  const int lc = blockIdx.x / nrbw;
  const int rb = win_rb0(p) + blockIdx.x % nrbw;
  if (lc >= nlc) return;
  const int nc = 3 * nv + ns;
  const int L = p.L;
  // smem tile [slot][u][q][32]
  const int nitems = 2 * kRB * nc * 32;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    const int lo = it & 31;
    int rest = it >> 5;
    const int q = rest % nc;
    rest /= nc;
    const int u = rest % kRB;
    const int slot = rest / kRB;
    const int l = m + 32 * lc + lo;
    const int r = kRB * rb + u;
    double v = 0.0;
    if (l <= L && r < p.nr && (slot == 0 || m > 0)) {
      const int j = p.jmap[((long long)m * 2 + slot) * (L + 1) + l];
      const int col = q < 3 * nv ? cols[q / 3] + q % 3 : cols[nv + (q - 3 * nv)];
      v = d_rj[(long long)j + p.J * r + ld * col];
    }
    sm[it] = v;
  }
  __syncthreads();
  const int nout = 2 * kKC * CB;
  for (int it = threadIdx.x; it < nout; it += blockDim.x) {
    const int c = it % CB;
    const int rest = it / CB;
    const int kk = rest % kKC;
    const int par = rest / kKC;
    const int k = kKC * lc + kk;
    if (k >= p.kpad[2 * m + par]) continue;
    const int lo = 2 * kk + par;
    const int l = m + 32 * lc + lo;
    double v;
    int u, slot;
    if (c < 24 * nv) {
      const int vv = c / 24, t = c % 24, tile = t / 8, w = t % 8;
      u = w >> 1;
      slot = w & 1;
      const int r = kRB * rb + u;
      const double ar = r < p.nr ? 1.0 / p.radius[r] : 0.0;
      const double* s = sm + ((slot * kRB + u) * nc) * 32;
      if (tile == 0) v = s[(3 * vv + 1) * 32 + lo] * ar;                   // dpoldt = dS/dr / r
      else if (tile == 1) v = s[(3 * vv + 2) * 32 + lo] * ar;              // dtordt = T / r
      else v = s[(3 * vv + 0) * 32 + lo] * (ar * ar) * g3_of(l);            // pol = S / r^2 * g3
    } else {
      const int cc = c - 24 * nv, ss = cc / 8, w = cc % 8;
      u = w >> 1;
      slot = w & 1;
      v = sm[((slot * kRB + u) * nc + 3 * nv + ss) * 32 + lo];
    }
    p.SB[p.sboff[2 * m + par] + (long long)k * (p.nrb * CB) + rb * CB + c] = v;
  }
}

// ---------------------------------------------------------------------------
constexpr int kGenThreadsB = 64;  // generator warps of the on-the-fly backward kernel (one per latitude)

// OTF: P / dP of the CTA's 64 latitudes come from two generator warps that run
// the recurrence one chunk pair ahead of the tensor warps (chunk pair c = the
// parity-0 and parity-1 chunks c, i.e. l = m + 32c .. m + 32c + 31); each
// parity still accumulates its chunks in order, so only P's last bits differ
// from the stored-table kernel.
template <int NV, int NS, bool OTF>
__global__ void __launch_bounds__(kThreads + (OTF ? kGenThreadsB : 0), 1) k_leg_bwd_f64(Plan p) {
  using G = BwdGeo<NV, NS>;
  extern __shared__ double sm[];
  double* sA = sm;                                   // [2 stages][(OTF: 2 parities)][2][kKC][AS]
  double* sB = sm + (OTF ? 4 : 2) * G::A_STAGE;      // [2 stages][(OTF: 2 parities)][kKC][CBp]
  const int nthb = p.nh_pad / kThBlk;
  int b = blockIdx.x;
  const int nrbw = win_nrb(p);
  const int rb = win_rb0(p) + b % nrbw;
  b /= nrbw;
  const int thb = b % nthb;
  const int m = b / nthb;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int th0 = thb * kThBlk;
  const int n0 = p.kpad[2 * m] / kKC, n1 = p.kpad[2 * m + 1] / kKC;
  const int total = n0 + n1;
  const long long rowB = (long long)p.nrb * G::CB;

  auto loadB = [&](double* bs, int par, int ch) {
    const double* Bg = p.SB + p.sboff[2 * m + par] + (long long)(ch * kKC) * rowB + rb * G::CB;
    for (int it = tid; it < kKC * (G::CB / 2); it += kThreads) {
      const int row = it / (G::CB / 2), c2 = it % (G::CB / 2);
      cp_async16(bs + row * G::CBp + 2 * c2, Bg + (long long)row * rowB + 2 * c2);
    }
  };
  auto load = [&](int stage, int step) {
    const int par = step < n0 ? 0 : 1;
    const int ch = step < n0 ? step : step - n0;
    const double* Pg = p.P + p.poff[2 * m + par] + (long long)(ch * kKC) * p.nh_pad + th0;
    const double* dPg = p.dP + p.poff[2 * m + par] + (long long)(ch * kKC) * p.nh_pad + th0;
    double* a = sA + stage * G::A_STAGE;
    // 2 tables x 16 rows x 64 doubles = 2 x 16 x 32 chunks of 16 B
    for (int it = tid; it < 2 * kKC * (kThBlk / 2); it += kThreads) {
      const int tb = it / (kKC * (kThBlk / 2));
      const int rem = it % (kKC * (kThBlk / 2));
      const int row = rem / (kThBlk / 2), c2 = rem % (kThBlk / 2);
      const double* src = (tb ? dPg : Pg) + (long long)row * p.nh_pad + 2 * c2;
      cp_async16(a + tb * kKC * G::AS + row * G::AS + 2 * c2, src);
    }
    loadB(sB + stage * G::B_STAGE, par, ch);
  };

  // accumulators: [field][tile][parity][2]; tiles XP, XdP, YP, YdP, ZP
  double acc[NV > 0 ? NV : 1][5][2][2];
  double accS[NS > 0 ? NS : 1][2][2];
#pragma unroll
  for (int v = 0; v < (NV > 0 ? NV : 1); ++v)
#pragma unroll
    for (int q = 0; q < 5; ++q)
#pragma unroll
      for (int s = 0; s < 2; ++s) acc[v][q][s][0] = acc[v][q][s][1] = 0.0;
#pragma unroll
  for (int v = 0; v < (NS > 0 ? NS : 1); ++v)
#pragma unroll
    for (int s = 0; s < 2; ++s) accS[v][s][0] = accS[v][s][1] = 0.0;

  auto compute = [&](const double* a, const double* bs, auto parc) {
    constexpr int par = decltype(parc)::value;
#pragma unroll
    for (int kk = 0; kk < kKC / 4; ++kk) {
      const int kr = 4 * kk + t;
      const double aP = a[kr * G::AS + warp * 8 + g];
      const double adP = a[kKC * G::AS + kr * G::AS + warp * 8 + g];
      const double* brow = bs + kr * G::CBp + g;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double bX = brow[24 * v + 0], bY = brow[24 * v + 8], bZ = brow[24 * v + 16];
        dmma(acc[v][0][par][0], acc[v][0][par][1], aP, bX);
        dmma(acc[v][1][par][0], acc[v][1][par][1], adP, bX);
        dmma(acc[v][2][par][0], acc[v][2][par][1], aP, bY);
        dmma(acc[v][3][par][0], acc[v][3][par][1], adP, bY);
        dmma(acc[v][4][par][0], acc[v][4][par][1], aP, bZ);
      }
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double bS = brow[24 * NV + 8 * s];
        dmma(accS[s][par][0], accS[s][par][1], aP, bS);
      }
    }
  };

  if constexpr (!OTF) {
    if (total > 0) {
      load(0, 0);
      cp_async_commit();
    }
    for (int step = 0; step < total; ++step) {
      if (step + 1 < total) {
        load((step + 1) & 1, step + 1);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      const double* a = sA + (step & 1) * G::A_STAGE;
      const double* bs = sB + (step & 1) * G::B_STAGE;
      if (step < n0) compute(a, bs, std::integral_constant<int, 0>());
      else compute(a, bs, std::integral_constant<int, 1>());
      __syncthreads();
    }
  } else {
    const bool gen = warp >= kWarps;
    const int gi = tid - kThreads, ig = th0 + gi;  // generator thread: latitude ig
    double st6[6];
    double ct = 0.0;
    if (gen) {
      const double* sd = p.pseed + p.pseed_off[m] * 6 * p.nh_pad + ig;  // block 0: before l = m
#pragma unroll
      for (int q = 0; q < 6; ++q) st6[q] = sd[(long long)q * p.nh_pad];
      if (ig < p.nh) ct = p.cos_t[ig];
    }
    // recurrence coefficients of a chunk pair's 32 degrees, [2 buffers][j][4];
    // each call prefetches the next pair's into registers while it steps
    double2* cb = reinterpret_cast<double2*>(sm + 4 * (G::A_STAGE + G::B_STAGE));
    constexpr int kCE = 8 * kKC;  // coefficient pairs of one chunk pair
    if (gen)
      for (int e = gi; e < kCE; e += kGenThreadsB) cb[e] = pgen_coef(p, m, m + (e >> 2), e & 3);
    auto genA = [&](int stage, int c) {
      double* a = sA + stage * 2 * G::A_STAGE;
      asm volatile("bar.sync 1, %0;\n" ::"n"(kGenThreadsB));  // cb[c & 1] complete
      double2 nx[kCE / kGenThreadsB];
#pragma unroll
      for (int q = 0; q < kCE / kGenThreadsB; ++q) {
        const int e = gi + q * kGenThreadsB;
        nx[q] = c + 1 < n0 ? pgen_coef(p, m, m + 2 * kKC * (c + 1) + (e >> 2), e & 3) : make_double2(0.0, 0.0);
      }
      const double2* cc = cb + (c & 1) * kCE;
      const int l0 = m + 2 * kKC * c;
      const int nj = min(2 * kKC, p.L - l0 + 1);
      if (l0 >= m + 3 && ig < p.nh) {
#pragma unroll 4
        for (int j = 0; j < 2 * kKC; ++j) {
          double pv = 0.0, dpv = 0.0;
          if (j < nj) pgen_step_fast(st6, ct, cc + 4 * j, pv, dpv);
          double* ap = a + (j & 1) * G::A_STAGE + (j >> 1) * G::AS + gi;
          ap[0] = pv;
          ap[kKC * G::AS] = dpv;
        }
      } else {
        for (int j = 0; j < 2 * kKC; ++j) {
          double pv = 0.0, dpv = 0.0;
          if (j < nj && ig < p.nh) pgen_step(st6, p, m, l0 + j, ct, ig, cc + 4 * j, pv, dpv);
          double* ap = a + (j & 1) * G::A_STAGE + (j >> 1) * G::AS + gi;
          ap[0] = pv;
          ap[kKC * G::AS] = dpv;
        }
      }
      double2* cn = cb + ((c + 1) & 1) * kCE;
#pragma unroll
      for (int q = 0; q < kCE / kGenThreadsB; ++q) cn[gi + q * kGenThreadsB] = nx[q];
    };
    auto loadB2 = [&](int stage, int c) {
      loadB(sB + (2 * stage) * G::B_STAGE, 0, c);
      if (c < n1) loadB(sB + (2 * stage + 1) * G::B_STAGE, 1, c);
    };
    // separate loops (same __syncthreads count), so the generator state is
    // not live in the tensor warps
    if (gen) {
      genA(0, 0);
      for (int c = 0; c < n0; ++c) {
        __syncthreads();
        if (c + 1 < n0) genA((c + 1) & 1, c + 1);
      }
      return;  // the generator warps take no part in the epilogue
    }
    loadB2(0, 0);
    cp_async_commit();
    for (int c = 0; c < n0; ++c) {
      cp_async_wait<0>();
      __syncthreads();
      if (c + 1 < n0) {
        loadB2((c + 1) & 1, c + 1);
        cp_async_commit();
      }
      const double* a = sA + (c & 1) * 2 * G::A_STAGE;
      const double* bs = sB + (c & 1) * 2 * G::B_STAGE;
      compute(a, bs, std::integral_constant<int, 0>());
      if (c < n1) compute(a + G::A_STAGE, bs + G::B_STAGE, std::integral_constant<int, 1>());
    }
  }

  // ---- epilogue: N/S recombination and +-m cross terms
  const int i = th0 + warp * 8 + g;
  const int r = kRB * rb + t;
  if (i >= p.nh || r >= p.nr) return;
  const bool pair = i < p.nth / 2;
  const double ms = (double)m * p.asin_t[i];
  const int nc = p.ncb;
  double* outN = p.rtm_b + rtm_off(p, m, i, r, nc);
  double* outS = p.rtm_b + rtm_off(p, m, p.nth - 1 - i, r, nc);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double sym[6], asym[6];  // r cos, r sin, th cos, th sin, ph cos, ph sin
    // r component
    sym[0] = acc[v][4][0][0];
    asym[0] = acc[v][4][1][0];
    sym[1] = acc[v][4][0][1];
    asym[1] = acc[v][4][1][1];
    // theta: own slot dP*b, mirror slot -/+ m/sin * P*c
    sym[2] = acc[v][1][1][0] + ms * acc[v][2][0][1];
    asym[2] = acc[v][1][0][0] + ms * acc[v][2][1][1];
    sym[3] = acc[v][1][1][1] - ms * acc[v][2][0][0];
    asym[3] = acc[v][1][0][1] - ms * acc[v][2][1][0];
    // phi: own slot -dP*c, mirror slot +/- m/sin * P*b
    sym[4] = -acc[v][3][1][0] + ms * acc[v][0][0][1];
    asym[4] = -acc[v][3][0][0] + ms * acc[v][0][1][1];
    sym[5] = -acc[v][3][1][1] - ms * acc[v][0][0][0];
    asym[5] = -acc[v][3][0][1] - ms * acc[v][0][1][0];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double2 n, s;
      if (pair) {
        n.x = sym[2 * c] + asym[2 * c];
        n.y = sym[2 * c + 1] + asym[2 * c + 1];
        s.x = sym[2 * c] - asym[2 * c];
        s.y = sym[2 * c + 1] - asym[2 * c + 1];
        *reinterpret_cast<double2*>(outS + rec_off(3 * v + c, NV)) = s;
      } else {
        n.x = sym[2 * c];
        n.y = sym[2 * c + 1];
      }
      *reinterpret_cast<double2*>(outN + rec_off(3 * v + c, NV)) = n;
    }
  }
#pragma unroll
  for (int s2 = 0; s2 < NS; ++s2) {
    const double sc = accS[s2][0][0], ss = accS[s2][0][1];
    const double ac = accS[s2][1][0], as = accS[s2][1][1];
    double2 n, s;
    const int c = 3 * NV + s2;
    if (pair) {
      n.x = sc + ac; n.y = ss + as;
      s.x = sc - ac; s.y = ss - as;
      *reinterpret_cast<double2*>(outS + rec_off(c, NV)) = s;
    } else {
      n.x = sc; n.y = ss;
    }
    *reinterpret_cast<double2*>(outN + rec_off(c, NV)) = n;
  }
}

// ---------------------------------------------------------------------------
template <int NV, int NS>
struct FwdGeo {
  static constexpr int CF = 40 * NV + 8 * NS;
  static constexpr int CFp = CF + ((4 - CF % 16) + 16) % 16;
  static constexpr int AS = kKC + 4;                      // 160 B rows
  static constexpr int A_TILE = kLBlk * AS;
  static constexpr int B_TILE = kKC * CFp;
  static constexpr size_t SMEM = sizeof(double) * (4 * A_TILE + 2 * B_TILE);
  // A double-buffered, the block's recurrence coefficients and two chunks' seeds
  static constexpr size_t SMEM_OTF =
      sizeof(double) * (8 * A_TILE + 2 * B_TILE) + sizeof(double2) * 8 * kLBlk + sizeof(double) * 2 * 2 * 6 * kKC;
};

// OTF: the A tiles (P / dP of the block's 64 degrees at 16 latitudes) are
// generated by warp 0 one latitude chunk ahead, each latitude's recurrence
// starting from the seeds at the block's two 32-degree halves.
// Two CTAs per SM while the accumulators fit in 128 registers (up to ten
// components); one CTA with the whole register file for more (four or five
// vectors: 42-52 accumulators per lane), which would otherwise spill.
template <int NV, int NS, bool OTF>
__global__ void __launch_bounds__(kThreads, 3 * NV + NS > 10 ? 1 : 2)
k_leg_fwd_f64(Plan p, double* __restrict__ d_rj, long long ld, const int* __restrict__ cols) {
  using G = FwdGeo<NV, NS>;
  extern __shared__ double sm[];
  double* sA = sm;                              // [(OTF: 2 stages)][P_e, P_o, dP_e, dP_o][kLBlk][AS]
  double* sB = sm + (OTF ? 8 : 4) * G::A_TILE;  // [par][kKC][CFp]
  const int m = blockIdx.y;
  const int nrbw = win_nrb(p);
  const int kb = blockIdx.x / nrbw;
  const int rb = win_rb0(p) + blockIdx.x % nrbw;
  const int K0 = kcount(p.L, m, 0);
  if (kb * kLBlk >= K0) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int par = warp & 1, rgi = warp >> 1;
  const int nc = p.ncf;
  const int nchunk = p.nh_pad / kKC;

  double acc[NV > 0 ? NV : 1][5][2];
  double accS[NS > 0 ? NS : 1][2];
#pragma unroll
  for (int v = 0; v < (NV > 0 ? NV : 1); ++v)
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[v][q][0] = acc[v][q][1] = 0.0;
#pragma unroll
  for (int s = 0; s < (NS > 0 ? NS : 1); ++s) accS[s][0] = accS[s][1] = 0.0;

  constexpr int kItems = (kKC * kRB * (3 * NV + NS) + kThreads - 1) / kThreads;
  double2 pfN[kItems], pfS[kItems];
  // item it = tid + q kThreads of a chunk is (latitude row, radius u, component
  // c), the same in every chunk: decomposed once (nc is not a compile-time
  // constant, so the divisions stay out of the chunk loop), packed as
  // c | u << 8 | row << 12, or -1 past the chunk's items
  int item[kItems];
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    const int it = tid + q * kThreads;
    const int rest = it / nc;
    item[q] = it < kKC * kRB * nc ? (it - rest * nc) | (rest % kRB) << 8 | (rest / kRB) << 12 : -1;
  }
  // global loads of one chunk's rtm_f values into registers (overlaps the MMAs)
  auto prefetch = [&](int ch) {
    const int th0 = ch * kKC;
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
      pfN[q] = make_double2(0.0, 0.0);
      pfS[q] = make_double2(0.0, 0.0);
      if (item[q] >= 0) {
        const int i = th0 + (item[q] >> 12), r = kRB * rb + ((item[q] >> 8) & 15);
        if (i < p.nh && r < p.nr) {
          const int ro = rec_off(item[q] & 255, NV);
          pfN[q] = *reinterpret_cast<const double2*>(p.rtm_f + rtm_off(p, m, i, r, nc) + ro);
          if (i < p.nth / 2)
            pfS[q] = *reinterpret_cast<const double2*>(p.rtm_f + rtm_off(p, m, p.nth - 1 - i, r, nc) + ro);
        }
      }
    }
  };
  // OTF: warp 0 generates the next chunk's A tile (before its share of the
  // current chunk's MMAs).  Recurrence coefficients of the block's 64 degrees
  // [j][4] are loaded once; the seeds of the next chunk's 16 latitudes and two
  // 32-degree halves, [stage][half][6][kKC], arrive by cp.async a chunk ahead.
  double2* cb = reinterpret_cast<double2*>(sB + 2 * G::B_TILE);
  double* sS = reinterpret_cast<double*>(cb + 8 * kLBlk);
  const int nsd = (p.L - m + kSeedL) / kSeedL;  // seeds of order m
  auto seeds_async = [&](int stage, int ch) {
    for (int e = lane; e < 2 * 6 * (kKC / 2); e += 32) {
      const int h = e / (6 * (kKC / 2)), rem = e % (6 * (kKC / 2)), q = rem / (kKC / 2), c2 = rem % (kKC / 2);
      const int sdi = 2 * kb + h;
      if (sdi < nsd)
        cp_async16(sS + ((stage * 2 + h) * 6 + q) * kKC + 2 * c2,
                   p.pseed + ((p.pseed_off[m] + sdi) * 6 + q) * p.nh_pad + ch * kKC + 2 * c2);
    }
    cp_async_commit();
  };
  // lane: latitude ch * kKC + (lane & 15), degrees lh .. lh + 31 with
  // lh = l0 + 32 h (h = lane >> 4); block row j (l = l0 + j) is parity j & 1,
  // A row j >> 1
  auto genA = [&](int stage, int ch) {
    const int h = lane >> 4, tl = lane & 15;
    const int ig = ch * kKC + tl;
    double* a = sA + stage * 4 * G::A_TILE + tl;
    const int l0 = m + 2 * kLBlk * kb, lh = l0 + kSeedL * h;
    const int nj = min(kSeedL, p.L - lh + 1);
    const bool ok = ig < p.nh && nj > 0;
    double st6[6];
    const double* sd = sS + ((stage * 2 + h) * 6) * kKC + tl;
#pragma unroll
    for (int q = 0; q < 6; ++q) st6[q] = ok ? sd[q * kKC] : 0.0;
    const double ct = ok ? p.cos_t[ig] : 0.0;
    const double2* cc = cb + 4 * kSeedL * h;
    if (lh >= m + 3) {
#pragma unroll 4
      for (int jj = 0; jj < kSeedL; ++jj) {
        const int j = kSeedL * h + jj;
        double pv = 0.0, dpv = 0.0;
        if (ok && jj < nj) pgen_step_fast(st6, ct, cc + 4 * jj, pv, dpv);
        a[(j & 1) * G::A_TILE + (j >> 1) * G::AS] = pv;
        a[(2 + (j & 1)) * G::A_TILE + (j >> 1) * G::AS] = dpv;
      }
    } else {
      for (int jj = 0; jj < kSeedL; ++jj) {
        const int j = kSeedL * h + jj;
        double pv = 0.0, dpv = 0.0;
        if (ok && jj < nj) pgen_step(st6, p, m, lh + jj, ct, ig, cc + 4 * jj, pv, dpv);
        a[(j & 1) * G::A_TILE + (j >> 1) * G::AS] = pv;
        a[(2 + (j & 1)) * G::A_TILE + (j >> 1) * G::AS] = dpv;
      }
    }
  };
  if (OTF && warp == 0) {
    for (int e = lane; e < 8 * kLBlk; e += 32) cb[e] = pgen_coef(p, m, m + 2 * kLBlk * kb + (e >> 2), e & 3);
    seeds_async(0, 0);
    cp_async_wait<0>();
    __syncwarp();
    genA(0, 0);
    if (nchunk > 1) seeds_async(1, 1);
  }
  prefetch(0);
  for (int ch = 0; ch < nchunk; ++ch) {
    const int th0 = ch * kKC;
    // A: 4 tables x 32 k-rows x 16 theta
    for (int it = tid; !OTF && it < 4 * kLBlk * (kKC / 2); it += kThreads) {
      const int tb = it / (kLBlk * (kKC / 2));   // 0 P_e, 1 P_o, 2 dP_e, 3 dP_o
      const int rem = it % (kLBlk * (kKC / 2));
      const int row = rem / (kKC / 2), c2 = rem % (kKC / 2);
      const int pp = tb & 1;
      const int k = kb * kLBlk + row;
      double* dst = sA + tb * G::A_TILE + row * G::AS + 2 * c2;
      if (k < p.kpad[2 * m + pp]) {
        const double* src = (tb < 2 ? p.P : p.dP) + p.poff[2 * m + pp] + (long long)k * p.nh_pad + th0 + 2 * c2;
        cp_async16(dst, src);
      } else {
        dst[0] = 0.0;
        dst[1] = 0.0;
      }
    }
    cp_async_commit();
    // B: sym/asym with weights from the prefetched registers
#pragma unroll
    for (int q = 0; q < kItems; ++q) {
      if (item[q] < 0) continue;
      const int c = item[q] & 255, u = (item[q] >> 8) & 15, row = item[q] >> 12;
      const int i = th0 + row;
      const int r = kRB * rb + u;
      double2 sy = make_double2(0.0, 0.0), as = sy, syn = sy, asn = sy;
      if (i < p.nh && r < p.nr) {
        const double wp = p.weight[i], ai = p.asin_t[i];
        const double2 nv = pfN[q];
        if (i < p.nth / 2) {
          const double2 sv = pfS[q];
          sy = make_double2((nv.x + sv.x) * wp, (nv.y + sv.y) * wp);
          as = make_double2((nv.x - sv.x) * wp, (nv.y - sv.y) * wp);
          syn = make_double2((nv.x + sv.x) * wp * ai, (nv.y + sv.y) * wp * ai);
          asn = make_double2((nv.x - sv.x) * wp * ai, (nv.y - sv.y) * wp * ai);
        } else {  // equator row
          sy = make_double2(nv.x * wp, nv.y * wp);
          syn = make_double2(nv.x * wp * ai, nv.y * wp * ai);
        }
      }
      double* b0 = sB + row * G::CFp;               // parity 0
      double* b1 = sB + G::B_TILE + row * G::CFp;   // parity 1
      if (c < 3 * NV) {
        const int v = c / 3, qq = c % 3;
        const int base = 40 * v + 2 * u;
        if (qq == 0) {            // r: Zr tile (P)
          *reinterpret_cast<double2*>(b0 + base + 0) = sy;
          *reinterpret_cast<double2*>(b1 + base + 0) = as;
        } else if (qq == 1) {     // theta: U' tile (P, /sin), W tile (dP)
          *reinterpret_cast<double2*>(b0 + base + 16) = syn;
          *reinterpret_cast<double2*>(b1 + base + 16) = asn;
          *reinterpret_cast<double2*>(b0 + base + 24) = as;
          *reinterpret_cast<double2*>(b1 + base + 24) = sy;
        } else {                  // phi: U tile (P, /sin), W' tile (dP)
          *reinterpret_cast<double2*>(b0 + base + 8) = syn;
          *reinterpret_cast<double2*>(b1 + base + 8) = asn;
          *reinterpret_cast<double2*>(b0 + base + 32) = as;
          *reinterpret_cast<double2*>(b1 + base + 32) = sy;
        }
      } else {
        const int sc = c - 3 * NV;
        const int base = 40 * NV + 8 * sc + 2 * u;
        *reinterpret_cast<double2*>(b0 + base) = sy;
        *reinterpret_cast<double2*>(b1 + base) = as;
      }
    }
    if (ch + 1 < nchunk) prefetch(ch + 1);
    if (!OTF) cp_async_wait<0>();
    __syncthreads();
    if (OTF && warp == 0 && ch + 1 < nchunk) {
      cp_async_wait<0>();  // seeds of chunk ch + 1
      __syncwarp();
      if (ch + 2 < nchunk) seeds_async(ch & 1, ch + 2);
      genA((ch + 1) & 1, ch + 1);
    }
    const double* sAc = sA + (OTF ? (ch & 1) * 4 * G::A_TILE : 0);
    const double* aP = sAc + par * G::A_TILE + (rgi * 8 + g) * G::AS;
    const double* adP = sAc + (2 + par) * G::A_TILE + (rgi * 8 + g) * G::AS;
    const double* bb = sB + par * G::B_TILE;
#pragma unroll
    for (int kk = 0; kk < kKC / 4; ++kk) {
      const double a = aP[4 * kk + t], ad = adP[4 * kk + t];
      const double* brow = bb + (4 * kk + t) * G::CFp + g;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        dmma(acc[v][0][0], acc[v][0][1], a, brow[40 * v + 0]);    // Zr
        dmma(acc[v][1][0], acc[v][1][1], a, brow[40 * v + 8]);    // U
        dmma(acc[v][2][0], acc[v][2][1], a, brow[40 * v + 16]);   // U'
        dmma(acc[v][3][0], acc[v][3][1], ad, brow[40 * v + 24]);  // W
        dmma(acc[v][4][0], acc[v][4][1], ad, brow[40 * v + 32]);  // W'
      }
#pragma unroll
      for (int s = 0; s < NS; ++s) dmma(accS[s][0], accS[s][1], a, brow[40 * NV + 8 * s]);
    }
    __syncthreads();
  }

  // ---- epilogue (cal_sp_rlm_vector_sym_matmul / _scalar_)
  const int k = kb * kLBlk + rgi * 8 + g;
  const int l = m + 2 * k + par;
  const int r = kRB * rb + t;
  if (l > p.L || r >= p.nr) return;
  const double r1 = p.radius[r], r2 = r1 * r1;
  const double g7 = g7_of(l, m), gm = (double)m;
  const long long jp = p.jmap[((long long)m * 2 + 0) * (p.L + 1) + l] + p.J * r;
  const long long jn = m > 0 ? p.jmap[((long long)m * 2 + 1) * (p.L + 1) + l] + p.J * r : -1;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double* o = d_rj + ld * cols[v];
    // + slot (cos), gm = +m
    o[jp] = acc[v][0][0] * r2 * g7;
    o[jp + ld] = acc[v][3][0] * r1 * g7 - acc[v][1][1] * r1 * g7 * gm;
    o[jp + 2 * ld] = -(acc[v][2][1] * r1 * g7 * gm) - acc[v][4][0] * r1 * g7;
    if (jn >= 0) {  // - slot (sin), gm = -m
      o[jn] = acc[v][0][1] * r2 * g7;
      o[jn + ld] = acc[v][3][1] * r1 * g7 - acc[v][1][0] * r1 * g7 * (-gm);
      o[jn + 2 * ld] = -(acc[v][2][0] * r1 * g7 * (-gm)) - acc[v][4][1] * r1 * g7;
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double* o = d_rj + ld * cols[NV + s];
    const double g6 = g6_of(l, m);
    o[jp] = accS[s][0] * g6;
    if (jn >= 0) o[jn] = accS[s][1] * g6;
  }
}

template <int NV, int NS, bool OTF>
cudaError_t run_bwd_t(const Plan& p, cudaStream_t s) {
  using G = BwdGeo<NV, NS>;
  auto kern = k_leg_bwd_f64<NV, NS, OTF>;
  const size_t smem = OTF ? G::SMEM_OTF : G::SMEM;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const long long nblk = (long long)(p.L + 1) * (p.nh_pad / kThBlk) * win_nrb(p);
  if (nblk <= 0) return cudaSuccess;
  kern<<<(unsigned)nblk, kThreads + (OTF ? kGenThreadsB : 0), smem, s>>>(p);
  return cudaGetLastError();
}
template <int NV, int NS>
cudaError_t run_bwd(const Plan& p, cudaStream_t s) {
  return p.otf ? run_bwd_t<NV, NS, true>(p, s) : run_bwd_t<NV, NS, false>(p, s);
}

template <int NV, int NS, bool OTF>
cudaError_t run_fwd_t(const Plan& p, double* d_rj, long long ld, const int* cols, cudaStream_t s, int m_count) {
  using G = FwdGeo<NV, NS>;
  auto kern = k_leg_fwd_f64<NV, NS, OTF>;
  const size_t smem = OTF ? G::SMEM_OTF : G::SMEM;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int nkb = (kcount(p.L, 0, 0) + kLBlk - 1) / kLBlk;
  if (win_nrb(p) <= 0) return cudaSuccess;
  dim3 grid(nkb * win_nrb(p), m_count);
  kern<<<grid, kThreads, smem, s>>>(p, d_rj, ld, cols);
  return cudaGetLastError();
}
template <int NV, int NS>
cudaError_t run_fwd(const Plan& p, double* d_rj, long long ld, const int* cols, cudaStream_t s, int m_count) {
  return p.otf ? run_fwd_t<NV, NS, true>(p, d_rj, ld, cols, s, m_count)
               : run_fwd_t<NV, NS, false>(p, d_rj, ld, cols, s, m_count);
}

#define KMHD_DISPATCH(NVv, NSv, FN, ...)                                   \
  switch (NVv * 3 + NSv) {                                                 \
    case 1: return FN<0, 1>(__VA_ARGS__);                                  \
    case 2: return FN<0, 2>(__VA_ARGS__);                                  \
    case 3: return FN<1, 0>(__VA_ARGS__);                                  \
    case 4: return FN<1, 1>(__VA_ARGS__);                                  \
    case 5: return FN<1, 2>(__VA_ARGS__);                                  \
    case 6: return FN<2, 0>(__VA_ARGS__);                                  \
    case 7: return FN<2, 1>(__VA_ARGS__);                                  \
    case 8: return FN<2, 2>(__VA_ARGS__);                                  \
    case 9: return FN<3, 0>(__VA_ARGS__);                                  \
    case 10: return FN<3, 1>(__VA_ARGS__);                                 \
    case 11: return FN<3, 2>(__VA_ARGS__);                                 \
    case 12: return FN<4, 0>(__VA_ARGS__);                                 \
    case 13: return FN<4, 1>(__VA_ARGS__);                                 \
    case 14: return FN<4, 2>(__VA_ARGS__);                                 \
    case 15: return FN<5, 0>(__VA_ARGS__);                                 \
    case 16: return FN<5, 1>(__VA_ARGS__);                                 \
    case 17: return FN<5, 2>(__VA_ARGS__);                                 \
    default: return cudaErrorInvalidValue;                                 \
  }

}  // namespace

cudaError_t launch_pack_b(const Plan& p, int nlc_max, const double* d_rj, long long ld,
                               const int* cols, int nv, int ns, cudaStream_t s) {
  const int nc = 3 * nv + ns;
  const int CB = 24 * nv + 8 * ns;
  const size_t smem = sizeof(double) * 2 * kRB * nc * 32;
  cudaFuncSetAttribute(k_pack_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (win_nrb(p) <= 0) return cudaSuccess;
  dim3 grid(nlc_max * win_nrb(p), p.L + 1);
  k_pack_b<<<grid, kThreads, smem, s>>>(p, d_rj, ld, cols, nv, ns, CB);
  return cudaGetLastError();
}

cudaError_t launch_leg_bwd_f64(const Plan& p, cudaStream_t s) {
  KMHD_DISPATCH(p.nvb, p.nsb, run_bwd, p, s);
}

cudaError_t launch_leg_fwd_f64(const Plan& p, double* d_rj, long long ld, const int* cols,
                               cudaStream_t s, int m_count) {
  if (m_count <= 0 || m_count > p.L + 1) m_count = p.L + 1;
  KMHD_DISPATCH(p.nvf, p.nsf, run_fwd, p, d_rj, ld, cols, s, m_count);
}

size_t bwd_smem_bytes(int nv, int ns) {
  const int CB = 24 * nv + 8 * ns;
  const int CBp = CB + ((4 - CB % 16) + 16) % 16;
  return sizeof(double) * 2 * (2 * kKC * (kThBlk + 4) + kKC * CBp);
}

}  // namespace kmhd
