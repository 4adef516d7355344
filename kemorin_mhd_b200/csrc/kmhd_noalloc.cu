// kmhd_noalloc.cu -- kmhd_sph_cycle_noalloc: the FP64 transform cycle for small
// problems, with every device work buffer (Gauss/Schmidt tables, index maps,
// FFT twiddles, packed spectra, rtm records) carved out of one file-scope
// static device array instead of cudaMalloc'd memory.
//
// Why: some callers of this library cannot allocate device memory on their
// own -- a solver embedded in a host framework that owns the whole device
// pool and forbids other allocators, or a code path that must not call
// cudaMalloc/cudaFree between set-up and shutdown (the runtime may
// synchronise the device there).  The handle-based API allocates in
// kmhd_sph_create, so those callers get this entry point instead.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "kmhd_internal.cuh"

using namespace kmhd;

namespace {

// The fixed work area.  Every device that loads the library holds it until
// the process exits.  Its contents persist from call to call.
constexpr size_t kNoAllocBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_ws[kNoAllocBytes];

// Device address of g_noalloc_ws in the current device's context (host code
// only sees a host-side stand-in under that name).  Looked up on every call,
// with that device current: a cudaDeviceReset by the caller loads the module
// again, possibly at another address, so no address is kept between calls.
cudaError_t noalloc_base(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_ws);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned char*>(p);
  return cudaSuccess;
}

// Makes `dev` current for the scope and restores the caller's device after.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) return;
    ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Bump allocator over the work area: offsets are 256-byte aligned.  With a
// null base it only measures.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t n) {
    off = (off + 255) / 256 * 256;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += sizeof(T) * (n > 0 ? n : 1);
    return p;
  }
};

bool na_factor(int n, std::vector<int>& f) {
  f.clear();
  int r = n;
  while (r % 8 == 0) { f.push_back(8); r /= 8; }
  while (r % 4 == 0) { f.push_back(4); r /= 4; }
  while (r % 2 == 0) { f.push_back(2); r /= 2; }
  while (r % 3 == 0) { f.push_back(3); r /= 3; }
  while (r % 5 == 0) { f.push_back(5); r /= 5; }
  return r == 1 && (int)f.size() <= kMaxFftFactors;
}

// Same acceptance rules as kmhd_sph_create for the FP64 tier.
int na_validate(const kmhd_sph_desc* d) {
  if (!d) return KMHD_ERR_ARG;
  if (d->tier != KMHD_TIER_FP64) return KMHD_ERR_ARG;
  if (d->flags != 0) return KMHD_ERR_ARG;  // no autotuning, no on-the-fly tables here
  if (d->ltr < 1 || d->nth < 2 || d->nr < 1 || d->nph < 4) return KMHD_ERR_SIZE;
  if (d->nph <= 2 * d->ltr + 1) return KMHD_ERR_SIZE;
  if (!d->radius) return KMHD_ERR_ARG;
  if (d->nvector_b < 0 || d->nscalar_b < 0 || d->nvector_f < 0 || d->nscalar_f < 0) return KMHD_ERR_ARG;
  if (d->nvector_b > kMaxVec || d->nscalar_b > kMaxScl || d->nvector_f > kMaxVec || d->nscalar_f > kMaxScl)
    return KMHD_ERR_SIZE;
  if (d->nvector_b + d->nscalar_b == 0 || d->nvector_f + d->nscalar_f == 0) return KMHD_ERR_ARG;
  if (d->nproduct < 1 || d->nproduct > kMaxProd) return d->nproduct < 1 ? KMHD_ERR_ARG : KMHD_ERR_SIZE;
  if (!d->products) return KMHD_ERR_ARG;
  int nv = 0, ns = 0;
  for (int i = 0; i < d->nproduct; ++i) {
    const kmhd_product& p = d->products[i];
    switch (p.kind) {
      case KMHD_PROD_CROSS:
      case KMHD_PROD_DOT:
        if (p.a < 0 || p.a >= d->nvector_b || p.b < 0 || p.b >= d->nvector_b) return KMHD_ERR_ARG;
        break;
      case KMHD_PROD_VEC_SCALAR:
        if (p.a < 0 || p.a >= d->nvector_b || p.b < 0 || p.b >= d->nscalar_b) return KMHD_ERR_ARG;
        break;
      case KMHD_PROD_SCALAR:
        if (p.a < 0 || p.a >= d->nscalar_b || p.b < 0 || p.b >= d->nscalar_b) return KMHD_ERR_ARG;
        break;
      default:
        return KMHD_ERR_ARG;
    }
    if (p.kind == KMHD_PROD_CROSS || p.kind == KMHD_PROD_VEC_SCALAR) ++nv; else ++ns;
  }
  if (nv != d->nvector_f || ns != d->nscalar_f) return KMHD_ERR_ARG;
  std::vector<int> f;
  if (!na_factor(d->nph, f)) return KMHD_ERR_SIZE;
  const int ncb = 3 * d->nvector_b + d->nscalar_b, ncf = 3 * d->nvector_f + d->nscalar_f;
  const int npair = (std::max(ncb, ncf) + 1) / 2;
  if (sizeof(double2) * (size_t)npair * d->nph + sizeof(double) * 2 * (size_t)(d->ltr + 1) * ncb > 227 * 1024)
    return KMHD_ERR_SIZE;
  return KMHD_OK;
}

// Plan sizes and the host index tables (same construction as kmhd_sph_create).
struct NaHost {
  std::vector<int> kpad;
  std::vector<long long> poff, sboff;
  std::vector<int> jmap;
  std::vector<double2> tw;
  std::vector<int> rev;
  size_t nP = 0, nSB = 0, nrtm_b = 0, nrtm_f = 0;
};

int na_plan(const kmhd_sph_desc* d, Plan& p, NaHost& H) {
  std::memset(&p, 0, sizeof(p));
  p.L = d->ltr;
  p.nth = d->nth;
  p.nph = d->nph;
  p.nr = d->nr;
  p.nh = (d->nth + 1) / 2;
  p.nh_pad = (p.nh + kThBlk - 1) / kThBlk * kThBlk;
  p.nr4 = (d->nr + kRB - 1) / kRB * kRB;
  p.nrb = p.nr4 / kRB;
  p.r_lo = 0;
  p.r_hi = p.nr;
  p.J = (long long)(p.L + 1) * (p.L + 1);
  p.nvb = d->nvector_b;
  p.nsb = d->nscalar_b;
  p.nvf = d->nvector_f;
  p.nsf = d->nscalar_f;
  p.ncb = 3 * p.nvb + p.nsb;
  p.ncf = 3 * p.nvf + p.nsf;
  const int L = p.L;
  H.kpad.resize(2 * (L + 1));
  H.poff.resize(2 * (L + 1));
  H.sboff.resize(2 * (L + 1));
  const int CB = 24 * p.nvb + 8 * p.nsb;
  long long po = 0, so = 0;
  for (int m = 0; m <= L; ++m)
    for (int q = 0; q < 2; ++q) {
      const int K = kcount(L, m, q);
      const int kp = (K + kKC - 1) / kKC * kKC;
      H.kpad[2 * m + q] = kp;
      H.poff[2 * m + q] = po;
      H.sboff[2 * m + q] = so;
      po += (long long)kp * p.nh_pad;
      so += (long long)kp * p.nrb * CB;
    }
  H.nP = (size_t)po;
  H.nSB = (size_t)so;
  H.nrtm_b = (size_t)(L + 1) * p.nth * p.nr * p.ncb * 2;
  H.nrtm_f = (size_t)(L + 1) * p.nth * p.nr * p.ncf * 2;
  std::vector<int> fac;
  na_factor(p.nph, fac);
  p.nfac = (int)fac.size();
  for (int i = 0; i < p.nfac; ++i) p.fac[i] = fac[i];
  p.nprod = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int i = 0; i < d->nproduct; ++i) {
      const kmhd_product& q = d->products[i];
      const bool vec = q.kind == KMHD_PROD_CROSS || q.kind == KMHD_PROD_VEC_SCALAR;
      if (vec != (pass == 0)) continue;
      p.pkind[p.nprod] = q.kind;
      p.pa[p.nprod] = q.a;
      p.pb[p.nprod] = q.b;
      p.pcoef[p.nprod] = q.coef;
      ++p.nprod;
    }
  return KMHD_OK;
}

int na_tables(const kmhd_sph_desc* d, const Plan& p, NaHost& H) {
  const int L = p.L;
  H.jmap.assign((size_t)(L + 1) * 2 * (L + 1), -1);
  const long long J = p.J;
  std::vector<int> lm(2 * J);
  if (d->idx_rj_lm) {
    std::memcpy(lm.data(), d->idx_rj_lm, sizeof(int) * 2 * J);
  } else {
    long long j = 0;
    for (int m = -L; m <= L; ++m)
      for (int l = std::abs(m); l <= L; ++l) {
        lm[2 * j] = l;
        lm[2 * j + 1] = m;
        ++j;
      }
  }
  for (long long j = 0; j < J; ++j) {
    const int l = lm[2 * j], m = lm[2 * j + 1];
    if (l < 0 || l > L || std::abs(m) > l) return KMHD_ERR_ARG;
    int& e = H.jmap[((size_t)std::abs(m) * 2 + (m < 0 ? 1 : 0)) * (L + 1) + l];
    if (e != -1) return KMHD_ERR_ARG;
    e = (int)j;
  }
  H.tw.resize(p.nph);
  for (int k = 0; k < p.nph; ++k) {
    const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)p.nph;
    H.tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  H.rev.resize(p.nph);
  std::vector<int> strides(p.nfac);
  int s = p.nph;
  for (int i = 0; i < p.nfac; ++i) { s /= p.fac[i]; strides[i] = s; }
  for (int pos = 0; pos < p.nph; ++pos) {
    int rem = pos, k = 0, mul = 1;
    for (int i = 0; i < p.nfac; ++i) {
      const int q = rem / strides[i];
      rem %= strides[i];
      k += q * mul;
      mul *= p.fac[i];
    }
    H.rev[pos] = k;
  }
  return KMHD_OK;
}

// Lays the work buffers out over `base` (null: measure only); returns the bytes used.
struct NaBufs {
  double *radius, *colat, *weight, *asin_t, *P, *dP, *SB, *rtm_b, *rtm_f;
  long long *poff, *sboff;
  int *kpad, *jmap, *digrev, *cols_b, *cols_f, *err;
  double2* twid;
};

size_t na_layout(const Plan& p, const NaHost& H, unsigned char* base, NaBufs& b) {
  Carve c{base};
  const int L = p.L;
  b.radius = c.take<double>(p.nr);
  b.colat = c.take<double>(p.nth);
  b.weight = c.take<double>(p.nth);
  b.asin_t = c.take<double>(p.nth);
  b.poff = c.take<long long>(2 * (L + 1));
  b.sboff = c.take<long long>(2 * (L + 1));
  b.kpad = c.take<int>(2 * (L + 1));
  b.jmap = c.take<int>((size_t)(L + 1) * 2 * (L + 1));
  b.twid = c.take<double2>(p.nph);
  b.digrev = c.take<int>(p.nph);
  b.cols_b = c.take<int>(kMaxVec + kMaxScl);
  b.cols_f = c.take<int>(kMaxVec + kMaxScl);
  b.err = c.take<int>(1);
  b.P = c.take<double>(H.nP);
  b.dP = c.take<double>(H.nP);
  b.SB = c.take<double>(H.nSB);
  b.rtm_b = c.take<double>(H.nrtm_b);
  b.rtm_f = c.take<double>(H.nrtm_f);
  return c.off;
}

}  // namespace

extern "C" int kmhd_sph_cycle_noalloc(const kmhd_sph_desc* desc, const double* d_rj_in, int64_t ld_in,
                                      const int32_t* cols_b, double* d_rj_out, int64_t ld_out,
                                      const int32_t* cols_f, void* stream) {
  int st = na_validate(desc);
  if (st != KMHD_OK) return st;
  if (!d_rj_in || !d_rj_out || !cols_b || !cols_f) return KMHD_ERR_ARG;
  Plan p;
  NaHost H;
  na_plan(desc, p, H);
  if (ld_in < p.J * (long long)p.nr || ld_out < p.J * (long long)p.nr) return KMHD_ERR_ARG;
  for (int f = 0; f < p.nvb + p.nsb; ++f)
    if (cols_b[f] < 0) return KMHD_ERR_ARG;
  for (int f = 0; f < p.nvf + p.nsf; ++f)
    if (cols_f[f] < 0) return KMHD_ERR_ARG;
  NaBufs b;
  if (na_layout(p, H, nullptr, b) > kNoAllocBytes) return KMHD_ERR_SIZE;  // work area too small
  if ((st = na_tables(desc, p, H)) != KMHD_OK) return st;

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || desc->device < 0 || desc->device >= ndev)
    return KMHD_ERR_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, desc->device) != cudaSuccess) return KMHD_ERR_CUDA;
  if (prop.major != 10) return KMHD_ERR_DEVICE;
  const DeviceScope scope(desc->device);  // the caller's device is current again on return
  if (!scope.ok) return KMHD_ERR_CUDA;
  unsigned char* base = nullptr;
  if (noalloc_base(&base) != cudaSuccess) return KMHD_ERR_CUDA;
  na_layout(p, H, base, b);

  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int L = p.L;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess;
  };
  // The table kernel writes only the valid (l, theta) entries of P and dP:
  // the padding must be zero, and the previous call may have left data there.
  if (up(b.radius, desc->radius, sizeof(double) * p.nr) ||
      up(b.poff, H.poff.data(), sizeof(long long) * 2 * (L + 1)) ||
      up(b.sboff, H.sboff.data(), sizeof(long long) * 2 * (L + 1)) ||
      up(b.kpad, H.kpad.data(), sizeof(int) * 2 * (L + 1)) ||
      up(b.jmap, H.jmap.data(), sizeof(int) * H.jmap.size()) ||
      up(b.twid, H.tw.data(), sizeof(double2) * p.nph) || up(b.digrev, H.rev.data(), sizeof(int) * p.nph) ||
      up(b.cols_b, cols_b, sizeof(int) * (p.nvb + p.nsb)) ||
      up(b.cols_f, cols_f, sizeof(int) * (p.nvf + p.nsf)) ||
      cudaMemsetAsync(b.P, 0, sizeof(double) * H.nP, s) != cudaSuccess ||
      cudaMemsetAsync(b.dP, 0, sizeof(double) * H.nP, s) != cudaSuccess ||
      cudaMemsetAsync(b.err, 0, sizeof(int), s) != cudaSuccess)
    return KMHD_ERR_CUDA;
  p.err = b.err;
  p.radius = b.radius;
  p.colat = b.colat;
  p.weight = b.weight;
  p.asin_t = b.asin_t;
  p.P = b.P;
  p.dP = b.dP;
  p.poff = b.poff;
  p.kpad = b.kpad;
  p.jmap = b.jmap;
  p.SB = b.SB;
  p.sboff = b.sboff;
  p.rtm_b = b.rtm_b;
  p.rtm_f = b.rtm_f;
  p.twid = b.twid;
  p.digrev = b.digrev;
  const int nlc_max = H.kpad[0] / kKC;
  if (launch_tables(p, b.colat, b.weight, b.asin_t, b.P, b.dP, s) != cudaSuccess ||
      launch_pack_b(p, nlc_max, d_rj_in, ld_in, b.cols_b, p.nvb, p.nsb, s) != cudaSuccess ||
      launch_leg_bwd_f64(p, s) != cudaSuccess || launch_fft_cycle(p, s) != cudaSuccess ||
      launch_leg_fwd_f64(p, d_rj_out, ld_out, b.cols_f, s) != cudaSuccess)
    return KMHD_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return KMHD_ERR_CUDA;
  int herr = 0;  // a bounded device wait that expired
  if (cudaMemcpy(&herr, b.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return KMHD_ERR_CUDA;
  return herr ? herr : KMHD_OK;
}
