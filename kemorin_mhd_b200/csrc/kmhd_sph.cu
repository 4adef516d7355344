// kmhd_sph.cu -- C-ABI of the B200 spherical-transform cycle (include/kmhd_sph.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kmhd_internal.cuh"
#include "kmhd_split.cuh"

namespace kmhd {
size_t bwd_smem_bytes(int nv, int ns);
size_t fft_smem_bytes(const Plan& p, int npair);
}  // namespace kmhd

using namespace kmhd;

struct BatchGraph {
  std::vector<const void*> sig;  // per instance: handle, in, out, lds, path
  std::vector<int64_t> sig_ld;
  cudaStream_t s0 = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  // split-path instances of one tier (6 or 4 slices) share one grouped GEMM
  // launch per direction, on the group's stream
  // kinds: (6 slices, 26 products), (6, 21), (4, 10), (4, 6)
  SplitGroup* group[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaStream_t gs[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> ev;  // phase events of the grouped instances
};

struct kmhd_sph {
  kmhd_sph_desc desc;
  Plan plan;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<kmhd_product> products;
  std::vector<int> kpad_h;
  std::vector<long long> poff_h, sboff_h;
  std::vector<int> jmap_h;
  int nlc_max = 0;
  // device allocations
  std::vector<void*> allocs;
  int64_t bytes = 0;
  double *radius = nullptr, *colat = nullptr, *weight = nullptr, *asin_t = nullptr;
  double *P = nullptr, *dP = nullptr, *SB = nullptr, *rtm_b = nullptr, *rtm_f = nullptr;
  // on-the-fly P (KMHD_FLAG_P_ON_THE_FLY)
  double *cos_t = nullptr, *pseed = nullptr;
  double2 *pco = nullptr, *dco = nullptr, *pst = nullptr;
  long long* pseed_off = nullptr;
  long long *poff = nullptr, *sboff = nullptr;
  int *kpad = nullptr, *jmap = nullptr, *digrev = nullptr;
  double2* twid = nullptr;
  int *cols_b_d = nullptr, *cols_f_d = nullptr;
  int* err = nullptr;  // device error word (bounded waits of the FFT and tcgen05 kernels)
  // divergence post-processing: FDM / normalisation coefficients, host-pointer staging
  double *div_coef = nullptr, *div_stage = nullptr, *rot_stage = nullptr;
  // Coriolis curl: coupled modes (4 per j), coefficients (12 per j), staging
  int* cor_idx = nullptr;
  double *cor_cf = nullptr, *cor_stage = nullptr;
  // Coriolis curl inside the cycle (kmhd_sph_set_coriolis): backward vector
  // indices of velocity and vorticity, output column, coefficient
  int cor_on = 0, cor_iv_velo = 0, cor_iv_vort = 0, cor_col = 0;
  double cor_coef = 0.0;
  double* cor_cyc = nullptr;  // 2 J*Nr staging columns for host-pointer cycles
  int cor_pending = 0;        // kmhd_sph_b_trans left a Coriolis curl in cor_cyc for kmhd_sph_f_trans
  double* pole_out = nullptr;  // (2 Nr) x ncb pole values for host-pointer calls
  std::vector<double> radius_h;
  std::vector<int> cols_b_cache, cols_f_cache;
  // host-pointer staging
  double *stage_in = nullptr, *stage_out = nullptr, *stage_grid = nullptr;
  // split-precision state
  SplitState* split = nullptr;
  bool use_split = true;   // split tiers: run the split path (false: the FP64 DMMA path)
  bool autotune = false;   // choose the Legendre path (and product count) on the first batch call
  bool tuned = false;
  // autotuner record: times (ms) and errors against the FP64 path of the
  // candidates FP64, split with the full product count, split with one group fewer
  float tune_ms[3] = {0, 0, 0};
  double tune_err[3] = {0, 0, 0};
  // batched cycles whose first handle this is: captured graph and its signature
  struct BatchGraph* batch = nullptr;
  // host-pointer cycles: radial chunks (bounds, empty = no chunking) whose
  // copies in and out run on their own streams beside the chunk kernels
  std::vector<int> chunks;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_out;
  // timing
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_mid[2] = {nullptr, nullptr};  // after the bwd pack/slicer, after the fwd slicer
  double last_ms[4] = {0, 0, 0, 0};
  double last_kernel_ms[5] = {0, 0, 0, 0, 0};
  bool kernel_timed = false;
};

namespace {

const char* kMsg[] = {"ok",
                      "invalid argument",
                      "unsupported size",
                      "CUDA runtime error",
                      "device allocation failed",
                      "no sm_100 device",
                      "bounded device wait expired",
                      "invalid call order or handle state"};

thread_local std::string g_last_cuda;

#define KCHECK(call)                                                    \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) {                                            \
      g_last_cuda = cudaGetErrorString(e_);                             \
      return e_ == cudaErrorMemoryAllocation ? KMHD_ERR_NOMEM : KMHD_ERR_CUDA; \
    }                                                                   \
  } while (0)

template <typename T>
int dalloc(kmhd_sph* h, T** p, size_t n) {
  void* q = nullptr;
  const size_t bytes = sizeof(T) * (n > 0 ? n : 1);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    g_last_cuda = cudaGetErrorString(e);
    return KMHD_ERR_NOMEM;
  }
  h->allocs.push_back(q);
  h->bytes += (int64_t)bytes;
  *p = (T*)q;
  return KMHD_OK;
}

bool factor_fft(int n, std::vector<int>& f) {
  f.clear();
  int r = n;
  while (r % 8 == 0 && r / 8 >= 1) { f.push_back(8); r /= 8; }
  while (r % 4 == 0) { f.push_back(4); r /= 4; }
  while (r % 2 == 0) { f.push_back(2); r /= 2; }
  while (r % 3 == 0) { f.push_back(3); r /= 3; }
  while (r % 5 == 0) { f.push_back(5); r /= 5; }
  return r == 1 && (int)f.size() <= kMaxFftFactors;
}

int validate(const kmhd_sph_desc* d) {
  if (!d) return KMHD_ERR_ARG;
  if (d->ltr < 1 || d->nth < 2 || d->nr < 1 || d->nph < 4) return KMHD_ERR_SIZE;
  if (d->nph <= 2 * d->ltr + 1) return KMHD_ERR_SIZE;  // m <= L must stay below Nyquist
  if (!d->radius) return KMHD_ERR_ARG;
  if (d->nvector_b < 0 || d->nscalar_b < 0 || d->nvector_f < 0 || d->nscalar_f < 0)
    return KMHD_ERR_ARG;
  if (d->nvector_b > kMaxVec || d->nscalar_b > kMaxScl || d->nvector_f > kMaxVec ||
      d->nscalar_f > kMaxScl)
    return KMHD_ERR_SIZE;
  if (d->nvector_b + d->nscalar_b == 0) return KMHD_ERR_ARG;
  if (d->tier < KMHD_TIER_FP64 || d->tier > KMHD_TIER_FP32ACC) return KMHD_ERR_ARG;
  if ((d->flags & KMHD_FLAG_P_ON_THE_FLY) && d->tier != KMHD_TIER_FP64) return KMHD_ERR_ARG;
  if (d->flags & ~(KMHD_FLAG_AUTOTUNE | KMHD_FLAG_P_ON_THE_FLY)) return KMHD_ERR_ARG;
  if (d->nproduct < 0 || d->nproduct > kMaxProd) return KMHD_ERR_SIZE;
  if (d->nproduct > 0 && !d->products) return KMHD_ERR_ARG;
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
  if (d->nproduct > 0 && (nv != d->nvector_f || ns != d->nscalar_f)) return KMHD_ERR_ARG;
  std::vector<int> f;
  if (!factor_fft(d->nph, f)) return KMHD_ERR_SIZE;
  // one (r, theta) line of one component pair plus the staged spectra of the
  // line must fit in shared memory (wide lines go through the FFT pair by pair)
  const int ncb = 3 * d->nvector_b + d->nscalar_b;
  if (sizeof(double2) * (size_t)d->nph + sizeof(double) * 2 * (size_t)(d->ltr + 1) * ncb > 227 * 1024)
    return KMHD_ERR_SIZE;
  return KMHD_OK;
}

int sync_cols(kmhd_sph* h, const int32_t* cols, int n, std::vector<int>& cache, int* dev) {
  if (!cols) return KMHD_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (cols[i] < 0) return KMHD_ERR_ARG;
  if ((int)cache.size() == n && std::memcmp(cache.data(), cols, sizeof(int) * n) == 0) return KMHD_OK;
  cache.assign(cols, cols + n);
  KCHECK(cudaMemcpyAsync(dev, cols, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

int check_ld(const kmhd_sph* h, int64_t ld) {
  return ld >= h->plan.J * (long long)h->plan.nr ? KMHD_OK : KMHD_ERR_ARG;
}

}  // namespace

extern "C" {

const char* kmhd_strerror(int status) {
  if (status < 0 || status > KMHD_ERR_STATE) return "unknown status";
  if (status == KMHD_ERR_CUDA && !g_last_cuda.empty()) return g_last_cuda.c_str();
  return kMsg[status];
}

int64_t kmhd_sph_device_bytes(const kmhd_sph* h) { return h ? h->bytes : 0; }

int kmhd_sph_get_path(const kmhd_sph* h, int32_t* path) {
  if (!h || !path) return KMHD_ERR_ARG;
  *path = (h->split && h->use_split) ? 1 : 0;
  return KMHD_OK;
}

int kmhd_sph_get_tuning(const kmhd_sph* h, int32_t* path, int32_t* products, float* ms3, double* err3) {
  if (!h) return KMHD_ERR_ARG;
  if (path) *path = (h->split && h->use_split) ? 1 : 0;
  if (products) *products = h->split ? split_products(split_ns(h->split), split_terms(h->split)) : 0;
  for (int c = 0; c < 3; ++c) {
    if (ms3) ms3[c] = h->tuned ? h->tune_ms[c] : 0.0f;
    if (err3) err3[c] = h->tuned ? h->tune_err[c] : 0.0;
  }
  return KMHD_OK;
}

int kmhd_sph_set_products(kmhd_sph* h, int32_t products) {
  if (!h || !h->split) return KMHD_ERR_ARG;
  const int ns = split_ns(h->split), full = ns == 6 ? 6 : 3;
  for (int T = full - 1; T <= full; ++T)
    if (split_products(ns, T) == products) return split_set_terms(h->split, T);
  return KMHD_ERR_ARG;
}

int kmhd_sph_destroy(kmhd_sph* h) {
  if (!h) return KMHD_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->split) split_destroy(h->split);
  if (h->batch) {
    if (h->batch->exec) cudaGraphExecDestroy(h->batch->exec);
    if (h->batch->fork) cudaEventDestroy(h->batch->fork);
    for (cudaEvent_t e : h->batch->join) cudaEventDestroy(e);
    for (cudaEvent_t e : h->batch->ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) {
      split_group_destroy(h->batch->group[k]);
      if (h->batch->gs[k]) cudaStreamDestroy(h->batch->gs[k]);
    }
    if (h->batch->s0) cudaStreamDestroy(h->batch->s0);
    delete h->batch;
  }
  for (void* p : h->allocs) cudaFree(p);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : h->ev_mid)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : h->ev_out) cudaEventDestroy(e);
  if (h->s_in) cudaStreamDestroy(h->s_in);
  if (h->s_out) cudaStreamDestroy(h->s_out);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return KMHD_OK;
}

int kmhd_sph_create(const kmhd_sph_desc* d, kmhd_sph** out) {
  if (!out) return KMHD_ERR_ARG;
  *out = nullptr;
  int st = validate(d);
  if (st != KMHD_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || d->device < 0 || d->device >= ndev)
    return KMHD_ERR_DEVICE;
  cudaDeviceProp prop;
  KCHECK(cudaGetDeviceProperties(&prop, d->device));
  if (prop.major != 10) return KMHD_ERR_DEVICE;
  KCHECK(cudaSetDevice(d->device));

  kmhd_sph* h = new kmhd_sph();
  h->desc = *d;
  h->device = d->device;
  if (d->nproduct > 0) h->products.assign(d->products, d->products + d->nproduct);
  h->desc.products = nullptr;
  h->desc.radius = nullptr;
  h->desc.idx_rj_lm = nullptr;
  auto fail = [&](int code) { kmhd_sph_destroy(h); return code; };
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(KMHD_ERR_CUDA);
  h->stream = h->own_stream;
  for (auto& e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(KMHD_ERR_CUDA);
  for (auto& e : h->ev_mid)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(KMHD_ERR_CUDA);

  Plan& p = h->plan;
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

  // ---- index tables (host)
  h->kpad_h.resize(2 * (L + 1));
  h->poff_h.resize(2 * (L + 1));
  h->sboff_h.resize(2 * (L + 1));
  const int CB = 24 * p.nvb + 8 * p.nsb;
  long long po = 0, so = 0;
  for (int m = 0; m <= L; ++m)
    for (int q = 0; q < 2; ++q) {
      const int K = kcount(L, m, q);
      const int kp = (K + kKC - 1) / kKC * kKC;
      h->kpad_h[2 * m + q] = kp;
      h->poff_h[2 * m + q] = po;
      h->sboff_h[2 * m + q] = so;
      po += (long long)kp * p.nh_pad;
      so += (long long)kp * p.nrb * CB;
    }
  h->nlc_max = h->kpad_h[0] / kKC;
  // rj map: default order m = -L..L, l = |m|..L
  h->jmap_h.assign((size_t)(L + 1) * 2 * (L + 1), -1);
  {
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
      if (l < 0 || l > L || std::abs(m) > l) return fail(KMHD_ERR_ARG);
      const int am = std::abs(m), slot = m < 0 ? 1 : 0;
      int& e = h->jmap_h[((size_t)am * 2 + slot) * (L + 1) + l];
      if (e != -1) return fail(KMHD_ERR_ARG);  // duplicate mode
      e = (int)j;
    }
  }
  // FFT factors, twiddles e^{+2 pi i k/N}, digit reversal of the DIF output
  std::vector<int> fac;
  factor_fft(p.nph, fac);
  p.nfac = (int)fac.size();
  for (int i = 0; i < p.nfac; ++i) p.fac[i] = fac[i];
  std::vector<double2> tw(p.nph);
  for (int k = 0; k < p.nph; ++k) {
    const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)p.nph;
    tw[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  std::vector<int> rev(p.nph);
  {
    std::vector<int> strides(p.nfac);
    int s = p.nph;
    for (int i = 0; i < p.nfac; ++i) { s /= fac[i]; strides[i] = s; }
    for (int pos = 0; pos < p.nph; ++pos) {
      int rem = pos, k = 0, mul = 1;
      for (int i = 0; i < p.nfac; ++i) {
        const int q = rem / strides[i];
        rem %= strides[i];
        k += q * mul;
        mul *= fac[i];
      }
      rev[pos] = k;
    }
  }
  // products: vector-valued first, then scalar-valued, each in list order (the
  // forward field order); the grid kernel relies on this ordering
  p.nprod = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (const kmhd_product& q : h->products) {
      const bool vec = q.kind == KMHD_PROD_CROSS || q.kind == KMHD_PROD_VEC_SCALAR;
      if (vec != (pass == 0)) continue;
      p.pkind[p.nprod] = q.kind;
      p.pa[p.nprod] = q.a;
      p.pb[p.nprod] = q.b;
      p.pcoef[p.nprod] = q.coef;
      ++p.nprod;
    }

  // ---- device allocations
  const size_t nP = (size_t)po, nSB = (size_t)so;
  const bool otf = (d->flags & KMHD_FLAG_P_ON_THE_FLY) != 0;
  const size_t nrtm_b = (size_t)(L + 1) * p.nth * p.nr * p.ncb * 2;
  const size_t nrtm_f = (size_t)(L + 1) * p.nth * p.nr * std::max(p.ncf, 1) * 2;
  const size_t nrj = (size_t)p.J * p.nr;
  const size_t nnod = (size_t)p.nr * p.nth * p.nph;
  if ((st = dalloc(h, &h->radius, p.nr)) || (st = dalloc(h, &h->colat, p.nth)) ||
      (st = dalloc(h, &h->weight, p.nth)) || (st = dalloc(h, &h->asin_t, p.nth)) ||
      (!otf && ((st = dalloc(h, &h->P, nP)) || (st = dalloc(h, &h->dP, nP)))) ||
      (st = dalloc(h, &h->poff, 2 * (L + 1))) || (st = dalloc(h, &h->sboff, 2 * (L + 1))) ||
      (st = dalloc(h, &h->kpad, 2 * (L + 1))) || (st = dalloc(h, &h->jmap, h->jmap_h.size())) ||
      (st = dalloc(h, &h->twid, p.nph)) || (st = dalloc(h, &h->digrev, p.nph)) ||
      (st = dalloc(h, &h->cols_b_d, 16)) || (st = dalloc(h, &h->cols_f_d, 16)) || (st = dalloc(h, &h->err, 1)) ||
      (st = dalloc(h, &h->SB, nSB)) || (st = dalloc(h, &h->rtm_b, nrtm_b)) ||
      (st = dalloc(h, &h->rtm_f, nrtm_f)))
    return fail(st);
  (void)nrj;
  (void)nnod;
  cudaStream_t s = h->stream;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  };
  h->radius_h.assign(d->radius, d->radius + p.nr);
  if (up(h->radius, d->radius, sizeof(double) * p.nr) || up(h->poff, h->poff_h.data(), sizeof(long long) * 2 * (L + 1)) ||
      up(h->sboff, h->sboff_h.data(), sizeof(long long) * 2 * (L + 1)) ||
      up(h->kpad, h->kpad_h.data(), sizeof(int) * 2 * (L + 1)) ||
      up(h->jmap, h->jmap_h.data(), sizeof(int) * h->jmap_h.size()) ||
      up(h->twid, tw.data(), sizeof(double2) * p.nph) || up(h->digrev, rev.data(), sizeof(int) * p.nph) ||
      (!otf && (cudaMemsetAsync(h->P, 0, sizeof(double) * nP, s) || cudaMemsetAsync(h->dP, 0, sizeof(double) * nP, s))) ||
      cudaMemsetAsync(h->err, 0, sizeof(int), s))
    return fail(KMHD_ERR_CUDA);
  p.err = h->err;
  p.radius = h->radius;
  p.colat = h->colat;
  p.weight = h->weight;
  p.asin_t = h->asin_t;
  p.P = h->P;
  p.dP = h->dP;
  p.poff = h->poff;
  p.kpad = h->kpad;
  p.jmap = h->jmap;
  p.SB = h->SB;
  p.sboff = h->sboff;
  p.rtm_b = h->rtm_b;
  p.rtm_f = h->rtm_f;
  p.twid = h->twid;
  p.digrev = h->digrev;
  if (!fft_line_fits(p)) {
    // wide lines: per-CTA grid scratch of the pair-by-pair FFT cycle
    // (kWideCtasPerSm CTAs per SM; 72 MB at Nphi = 3072, L2-resident)
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device);
    const int npm = (std::max(p.ncb, p.ncf) + 1) / 2;
    const int nctas = kWideCtasPerSm * nsm;
    double2* sc = nullptr;
    if ((st = dalloc(h, &sc, (size_t)nctas * npm * p.nph))) return fail(st);
    p.fft_scratch = sc;
    p.fft_scratch_ctas = nctas;
  }
  if (launch_tables(p, h->colat, h->weight, h->asin_t, h->P, h->dP, s) != cudaSuccess)
    return fail(KMHD_ERR_CUDA);
  if (otf) {
    // recurrence coefficients, start values and the forward block seeds
    std::vector<long long> soff(L + 1);
    long long nseed = 0;
    for (int m = 0; m <= L; ++m) {
      soff[m] = nseed;
      nseed += (L - m + kSeedL) / kSeedL;
    }
    if ((st = dalloc(h, &h->cos_t, p.nh_pad)) || (st = dalloc(h, &h->pco, (size_t)(L + 2) * (L + 1))) ||
        (st = dalloc(h, &h->dco, (size_t)(L + 1) * (L + 1))) || (st = dalloc(h, &h->pst, (size_t)(L + 2) * p.nh_pad)) ||
        (st = dalloc(h, &h->pseed, (size_t)nseed * 6 * p.nh_pad)) || (st = dalloc(h, &h->pseed_off, (size_t)(L + 1))))
      return fail(st);
    if (up(h->pseed_off, soff.data(), sizeof(long long) * (L + 1)) ||
        cudaMemsetAsync(h->cos_t, 0, sizeof(double) * p.nh_pad, s))
      return fail(KMHD_ERR_CUDA);
    p.otf = 1;
    p.cos_t = h->cos_t;
    p.pco = h->pco;
    p.dco = h->dco;
    p.pst = h->pst;
    p.pseed = h->pseed;
    p.pseed_off = h->pseed_off;
    if (launch_otf_tables(p, h->cos_t, h->pco, h->dco, h->pst, h->pseed, h->pseed_off, s) != cudaSuccess)
      return fail(KMHD_ERR_CUDA);
  }
  h->autotune = (d->flags & KMHD_FLAG_AUTOTUNE) != 0 && d->tier != KMHD_TIER_FP64;
  if (d->tier != KMHD_TIER_FP64) {
    st = split_create(&h->split, p, d->tier, d->nslice, s);
    if (st != KMHD_OK) return fail(st);
    h->bytes += split_bytes(h->split);
  }
  // Radial chunks of host-pointer cycles: about sixteen chunks of a multiple
  // of 16 radii when the copies are large enough to be worth overlapping (the
  // first chunk's copy in and the last chunk's kernels and copy out are not
  // overlapped, so more chunks shorten the pipeline's fill and drain).
  {
    const double copy_bytes = 8.0 * (double)nrj * (p.ncb + p.ncf);
    const int step = 16 * std::max(1, (int)std::lround(p.nr / 256.0));
    if (copy_bytes >= 64.0 * (1 << 20) && p.nr >= 2 * step) {
      for (int r = 0; r + step < p.nr || r == 0; r += step) h->chunks.push_back(r);
      if (p.nr - h->chunks.back() < step / 2 && h->chunks.size() > 1) h->chunks.pop_back();
      h->chunks.push_back(p.nr);
      if (h->split && (st = split_set_chunks(h->split, p, h->chunks, s)) != KMHD_OK) return fail(st);
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(KMHD_ERR_CUDA);
  *out = h;
  return KMHD_OK;
}

int kmhd_sph_set_stream(kmhd_sph* h, void* stream) {
  if (!h) return KMHD_ERR_ARG;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return KMHD_OK;
}

int kmhd_sph_last_timing(kmhd_sph* h, double* ms4) {
  if (!h || !ms4) return KMHD_ERR_ARG;
  std::memcpy(ms4, h->last_ms, sizeof(h->last_ms));
  return KMHD_OK;
}

}  // extern "C"

namespace {

// Stage a host d_rj (selected columns) into a compact device buffer.
int stage_host_in(kmhd_sph* h, const double* d_rj, int64_t ld, const int32_t* cols, int nv, int ns,
                  const double** dev, int64_t* dev_ld, std::vector<int>& cols_c) {
  const Plan& p = h->plan;
  const size_t nrj = (size_t)p.J * p.nr;
  const int nc = 3 * nv + ns;
  if (!h->stage_in) {
    int st = dalloc(h, &h->stage_in, nrj * std::max(p.ncb, p.ncf));
    if (st) return st;
  }
  cols_c.resize(nv + ns);
  for (int f = 0; f < nv + ns; ++f) {
    const int ncomp = f < nv ? 3 : 1;
    const int c0 = f < nv ? 3 * f : 3 * nv + (f - nv);
    cols_c[f] = c0;
    for (int q = 0; q < ncomp; ++q)
      KCHECK(cudaMemcpyAsync(h->stage_in + nrj * (c0 + q), d_rj + ld * (cols[f] + q), sizeof(double) * nrj,
                             cudaMemcpyHostToDevice, h->stream));
  }
  (void)nc;
  *dev = h->stage_in;
  *dev_ld = (int64_t)nrj;
  return KMHD_OK;
}

int timed_begin(kmhd_sph* h) {
  KCHECK(cudaEventRecord(h->ev[0], h->stream));
  return KMHD_OK;
}

// `win` (optional): a copy of the plan restricted to one radial chunk.
int run_bwd_spectral(kmhd_sph* h, const double* d_rj, int64_t ld, bool timed = true, const Plan* win = nullptr) {
  const Plan& p = win ? *win : h->plan;
  if (h->split && h->use_split) {
    int st = split_bwd(h->split, p, h->nlc_max, d_rj, ld, h->cols_b_d, h->stream, timed ? h->ev_mid[0] : nullptr);
    return st;
  }
  KCHECK(launch_pack_b(p, h->nlc_max, d_rj, ld, h->cols_b_d, p.nvb, p.nsb, h->stream));
  if (timed) KCHECK(cudaEventRecord(h->ev_mid[0], h->stream));
  KCHECK(launch_leg_bwd_f64(p, h->stream));
  return KMHD_OK;
}

int run_fwd_spectral(kmhd_sph* h, double* d_rj, int64_t ld, bool timed = true, const Plan* win = nullptr) {
  const Plan& p = win ? *win : h->plan;
  if (h->split && h->use_split) {
    // split tiers: slicer + INT8 GEMM for every mode, then the dipole (l <= 2)
    // modes are accumulated again in FP64 by the DMMA kernel over orders m <= 2
    const int st = split_fwd(h->split, p, d_rj, ld, h->cols_f_d, h->stream, timed ? h->ev_mid[1] : nullptr);
    if (st != KMHD_OK) return st;
    KCHECK(launch_leg_fwd_f64(p, d_rj, ld, h->cols_f_d, h->stream, std::min(3, p.L + 1)));
    return KMHD_OK;
  }
  if (timed) KCHECK(cudaEventRecord(h->ev_mid[1], h->stream));  // the FP64 forward GEMM packs its operands itself
  KCHECK(launch_leg_fwd_f64(p, d_rj, ld, h->cols_f_d, h->stream));
  return KMHD_OK;
}

// One cycle with device pointers on the handle's stream, columns already on
// the device; no host synchronisation (safe inside stream capture).
int enqueue_cycle(kmhd_sph* h, const double* in, int64_t ld_in, double* out, int64_t ld_out) {
  int st;
  if ((st = run_bwd_spectral(h, in, ld_in, false))) return st;
  KCHECK(launch_fft_cycle(h->plan, h->stream));
  return run_fwd_spectral(h, out, ld_out, false);
}

// The instance's device error word (KMHD_ERR_TIMEOUT from a bounded wait of
// the FFT or tcgen05 kernels); synchronises the handle's stream.
int check_dev_err(kmhd_sph* h) {
  int v = 0;
  KCHECK(cudaMemcpyAsync(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return v;
}

// The registered Coriolis curl of radii [r0, r1): vel / vort point at the S
// columns of the velocity and vorticity triples (column stride ld), pol / tor
// at the two output columns; every pointer is the full-radius column base.
int enqueue_coriolis(kmhd_sph* h, const double* vel, const double* vort, int64_t ld, double* pol, double* tor,
                     int r0, int r1, cudaStream_t s) {
  const long long o = h->plan.J * (long long)r0;
  KCHECK(launch_rot_coriolis(h->plan.J, r1 - r0, vel + o, vort + o, ld, pol + o, tor + o, h->cor_idx, h->cor_cf,
                             h->radius + r0, h->cor_coef, s));
  return KMHD_OK;
}

// The registered Coriolis curl of a device-pointer cycle (all radii).
int enqueue_coriolis_dev(kmhd_sph* h, const double* in, int64_t ld_in, const int32_t* cols_b, double* out,
                         int64_t ld_out) {
  if (!h->cor_on) return KMHD_OK;
  return enqueue_coriolis(h, in + ld_in * cols_b[h->cor_iv_velo], in + ld_in * cols_b[h->cor_iv_vort], ld_in,
                          out + ld_out * h->cor_col, out + ld_out * (h->cor_col + 2), 0, h->plan.nr, h->stream);
}

// Column checks of a cycle with the Coriolis curl registered: its two output
// columns may not be written by the forward fields, nor be input columns of
// the cycle when input and output are one array.
int check_coriolis_cols(const kmhd_sph* h, const double* in, int64_t ld_in, const int32_t* cols_b, const double* out,
                        int64_t ld_out, const int32_t* cols_f) {
  const Plan& p = h->plan;
  for (int q = 0; q < 3; q += 2) {
    const int c = h->cor_col + q;
    for (int f = 0; f < p.nvf + p.nsf; ++f)
      if (c >= cols_f[f] && c < cols_f[f] + (f < p.nvf ? 3 : 1)) return KMHD_ERR_ARG;
    if (in == out && ld_in == ld_out)
      for (int f = 0; f < p.nvb + p.nsb; ++f)
        if (c >= cols_b[f] && c < cols_b[f] + (f < p.nvb ? 3 : 1)) return KMHD_ERR_ARG;
  }
  return KMHD_OK;
}

// Host-pointer cycle over the radial chunks.  Every stage is independent per
// radius, so chunk c's kernels run on the handle's stream while chunk c + 1's
// spectra come in on s_in and chunk c - 1's results go out on s_out.  The
// staging buffers hold every radius, so no chunk waits for a buffer to free.
int cycle_host_chunked(kmhd_sph* h, const double* d_rj_in, int64_t ld_in, const int32_t* cols_b,
                       double* d_rj_out, int64_t ld_out, const int32_t* cols_f) {
  const Plan& p = h->plan;
  const size_t nrj = (size_t)p.J * p.nr;
  const int nc = (int)h->chunks.size() - 1;
  if (!h->s_in) KCHECK(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
  if (!h->s_out) KCHECK(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
  while ((int)h->ev_in.size() < nc) {
    cudaEvent_t a = nullptr, b = nullptr;
    KCHECK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    h->ev_in.push_back(a);
    KCHECK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    h->ev_out.push_back(b);
  }
  int st;
  if (!h->stage_in && (st = dalloc(h, &h->stage_in, nrj * std::max(p.ncb, p.ncf)))) return st;
  if (!h->stage_out && (st = dalloc(h, &h->stage_out, nrj * std::max(p.ncf, 1)))) return st;
  if (h->cor_on && !h->cor_cyc && (st = dalloc(h, &h->cor_cyc, 2 * nrj))) return st;
  std::vector<int> cb(p.nvb + p.nsb), cf(p.nvf + p.nsf);
  for (int f = 0; f < p.nvb + p.nsb; ++f) cb[f] = f < p.nvb ? 3 * f : 3 * p.nvb + (f - p.nvb);
  for (int f = 0; f < p.nvf + p.nsf; ++f) cf[f] = f < p.nvf ? 3 * f : 3 * p.nvf + (f - p.nvf);
  if ((st = sync_cols(h, cb.data(), p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
  if ((st = sync_cols(h, cf.data(), p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) return st;
  // copies start after the work already queued on the handle's stream
  KCHECK(cudaEventRecord(h->ev[0], h->stream));
  KCHECK(cudaStreamWaitEvent(h->s_in, h->ev[0], 0));
  for (int c = 0; c < nc; ++c) {
    const long long o = p.J * (long long)h->chunks[c];
    const size_t bytes = sizeof(double) * (size_t)(p.J * (long long)(h->chunks[c + 1] - h->chunks[c]));
    for (int f = 0; f < p.nvb + p.nsb; ++f)
      for (int q = 0; q < (f < p.nvb ? 3 : 1); ++q)
        KCHECK(cudaMemcpyAsync(h->stage_in + nrj * (cb[f] + q) + o, d_rj_in + ld_in * (cols_b[f] + q) + o, bytes,
                               cudaMemcpyHostToDevice, h->s_in));
    KCHECK(cudaEventRecord(h->ev_in[c], h->s_in));
  }
  for (int c = 0; c < nc; ++c) {
    Plan w = p;
    w.r_lo = h->chunks[c];
    w.r_hi = h->chunks[c + 1];
    KCHECK(cudaStreamWaitEvent(h->stream, h->ev_in[c], 0));
    if (h->cor_on &&
        (st = enqueue_coriolis(h, h->stage_in + nrj * cb[h->cor_iv_velo], h->stage_in + nrj * cb[h->cor_iv_vort],
                               (int64_t)nrj, h->cor_cyc, h->cor_cyc + nrj, w.r_lo, w.r_hi, h->stream)))
      return st;
    if ((st = run_bwd_spectral(h, h->stage_in, (int64_t)nrj, false, &w))) return st;
    KCHECK(launch_fft_cycle(w, h->stream));
    if ((st = run_fwd_spectral(h, h->stage_out, (int64_t)nrj, false, &w))) return st;
    KCHECK(cudaEventRecord(h->ev_out[c], h->stream));
    KCHECK(cudaStreamWaitEvent(h->s_out, h->ev_out[c], 0));
    const long long o = p.J * (long long)w.r_lo;
    const size_t bytes = sizeof(double) * (size_t)(p.J * (long long)(w.r_hi - w.r_lo));
    for (int f = 0; f < p.nvf + p.nsf; ++f)
      for (int q = 0; q < (f < p.nvf ? 3 : 1); ++q)
        KCHECK(cudaMemcpyAsync(d_rj_out + ld_out * (cols_f[f] + q) + o, h->stage_out + nrj * (cf[f] + q) + o, bytes,
                               cudaMemcpyDeviceToHost, h->s_out));
    if (h->cor_on)
      for (int q = 0; q < 2; ++q)
        KCHECK(cudaMemcpyAsync(d_rj_out + ld_out * (h->cor_col + 2 * q) + o, h->cor_cyc + nrj * q + o, bytes,
                               cudaMemcpyDeviceToHost, h->s_out));
  }
  KCHECK(cudaEventRecord(h->ev[1], h->s_out));
  KCHECK(cudaStreamWaitEvent(h->stream, h->ev[1], 0));
  KCHECK(cudaEventRecord(h->ev[3], h->stream));
  KCHECK(cudaEventSynchronize(h->ev[3]));
  {
    const int e = check_dev_err(h);
    if (e != KMHD_OK) return e;
  }
  // the stages overlap: only the whole call is timed
  float t = 0;
  KCHECK(cudaEventElapsedTime(&t, h->ev[0], h->ev[3]));
  h->last_ms[0] = h->last_ms[1] = h->last_ms[2] = 0.0;
  h->last_ms[3] = t;
  h->kernel_timed = false;
  return KMHD_OK;
}

int finish_timing(kmhd_sph* h) {
  KCHECK(cudaEventSynchronize(h->ev[3]));
  {
    const int e = check_dev_err(h);
    if (e != KMHD_OK) return e;
  }
  float a = 0, b = 0, c = 0, t = 0;
  KCHECK(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
  KCHECK(cudaEventElapsedTime(&b, h->ev[1], h->ev[2]));
  KCHECK(cudaEventElapsedTime(&c, h->ev[2], h->ev[3]));
  KCHECK(cudaEventElapsedTime(&t, h->ev[0], h->ev[3]));
  h->last_ms[0] = a;
  h->last_ms[1] = b;
  h->last_ms[2] = c;
  h->last_ms[3] = t;
  h->kernel_timed = false;
  return KMHD_OK;
}

// Per-launch times of a full cycle: bwd pack/slicer, bwd GEMM, FFT + products,
// fwd slicer (0 for the FP64 tier), fwd GEMM.
int finish_kernel_timing(kmhd_sph* h) {
  float k[5] = {0, 0, 0, 0, 0};
  KCHECK(cudaEventElapsedTime(&k[0], h->ev[0], h->ev_mid[0]));
  KCHECK(cudaEventElapsedTime(&k[1], h->ev_mid[0], h->ev[1]));
  KCHECK(cudaEventElapsedTime(&k[2], h->ev[1], h->ev[2]));
  KCHECK(cudaEventElapsedTime(&k[3], h->ev[2], h->ev_mid[1]));
  KCHECK(cudaEventElapsedTime(&k[4], h->ev_mid[1], h->ev[3]));
  for (int i = 0; i < 5; ++i) h->last_kernel_ms[i] = k[i];
  h->kernel_timed = true;
  return KMHD_OK;
}

}  // namespace

extern "C" {

int kmhd_sph_b_trans(kmhd_sph* h, const double* d_rj, int64_t ld, const int32_t* cols_b,
                     double* fld_rtp, int32_t ptr_kind) {
  if (!h || !d_rj || !fld_rtp) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  KCHECK(cudaSetDevice(h->device));
  const Plan& p = h->plan;
  const double* src = d_rj;
  int64_t sld = ld;
  std::vector<int> cc;
  int st;
  if (ptr_kind == KMHD_PTR_HOST) {
    if ((st = stage_host_in(h, d_rj, ld, cols_b, p.nvb, p.nsb, &src, &sld, cc))) return st;
    if ((st = sync_cols(h, cc.data(), p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
  } else if ((st = sync_cols(h, cols_b, p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) {
    return st;
  }
  const size_t nnod = (size_t)p.nr * p.nth * p.nph;
  double* grid = fld_rtp;
  if (ptr_kind == KMHD_PTR_HOST) {
    if (!h->stage_grid && (st = dalloc(h, &h->stage_grid, nnod * std::max(p.ncb, p.ncf)))) return st;
    grid = h->stage_grid;
  }
  if ((st = timed_begin(h))) return st;
  if (h->cor_on) {
    // sph_b_trans_w_coriolis: the Coriolis curl of the received spectra, kept
    // for the next kmhd_sph_f_trans (copy_coriolis_terms_rlm)
    const size_t nrj = (size_t)p.J * p.nr;
    if (!h->cor_cyc && (st = dalloc(h, &h->cor_cyc, 2 * nrj))) return st;
    const int iv = ptr_kind == KMHD_PTR_HOST ? cc[h->cor_iv_velo] : cols_b[h->cor_iv_velo];
    const int iw = ptr_kind == KMHD_PTR_HOST ? cc[h->cor_iv_vort] : cols_b[h->cor_iv_vort];
    if ((st = enqueue_coriolis(h, src + sld * iv, src + sld * iw, sld, h->cor_cyc, h->cor_cyc + nrj, 0, p.nr,
                               h->stream)))
      return st;
    h->cor_pending = 1;
  }
  if ((st = run_bwd_spectral(h, src, sld))) return st;
  KCHECK(cudaEventRecord(h->ev[1], h->stream));
  KCHECK(launch_fft_bwd_grid(p, grid, h->stream));
  KCHECK(cudaEventRecord(h->ev[2], h->stream));
  KCHECK(cudaEventRecord(h->ev[3], h->stream));
  if (ptr_kind == KMHD_PTR_HOST)
    KCHECK(cudaMemcpyAsync(fld_rtp, grid, sizeof(double) * nnod * p.ncb, cudaMemcpyDeviceToHost, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return finish_timing(h);
}

int kmhd_sph_f_trans(kmhd_sph* h, const double* frc_rtp, double* d_rj, int64_t ld,
                     const int32_t* cols_f, int32_t ptr_kind) {
  if (!h || !d_rj || !frc_rtp) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.ncf == 0) return KMHD_ERR_STATE;
  if (h->cor_on && h->cor_pending)
    for (int q = 0; q < 3; q += 2)
      for (int f = 0; f < p.nvf + p.nsf; ++f)
        if (h->cor_col + q >= cols_f[f] && h->cor_col + q < cols_f[f] + (f < p.nvf ? 3 : 1)) return KMHD_ERR_ARG;
  KCHECK(cudaSetDevice(h->device));
  const size_t nnod = (size_t)p.nr * p.nth * p.nph;
  const size_t nrj = (size_t)p.J * p.nr;
  int st;
  const double* grid = frc_rtp;
  double* out = d_rj;
  int64_t old = ld;
  std::vector<int> cc(p.nvf + p.nsf);
  if (ptr_kind == KMHD_PTR_HOST) {
    if (!h->stage_grid && (st = dalloc(h, &h->stage_grid, nnod * std::max(p.ncb, p.ncf)))) return st;
    if (!h->stage_out && (st = dalloc(h, &h->stage_out, nrj * std::max(p.ncf, 1)))) return st;
    KCHECK(cudaMemcpyAsync(h->stage_grid, frc_rtp, sizeof(double) * nnod * p.ncf, cudaMemcpyHostToDevice, h->stream));
    grid = h->stage_grid;
    out = h->stage_out;
    old = (int64_t)nrj;
    for (int f = 0; f < p.nvf + p.nsf; ++f) cc[f] = f < p.nvf ? 3 * f : 3 * p.nvf + (f - p.nvf);
    if ((st = sync_cols(h, cc.data(), p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) return st;
  } else if ((st = sync_cols(h, cols_f, p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) {
    return st;
  }
  if ((st = timed_begin(h))) return st;
  KCHECK(cudaEventRecord(h->ev[1], h->stream));
  KCHECK(launch_fft_fwd_grid(p, grid, h->stream));
  KCHECK(cudaEventRecord(h->ev[2], h->stream));
  if ((st = run_fwd_spectral(h, out, old))) return st;
  KCHECK(cudaEventRecord(h->ev[3], h->stream));
  if (ptr_kind == KMHD_PTR_HOST) {
    for (int f = 0; f < p.nvf + p.nsf; ++f) {
      const int ncomp = f < p.nvf ? 3 : 1;
      for (int q = 0; q < ncomp; ++q)
        KCHECK(cudaMemcpyAsync(d_rj + ld * (cols_f[f] + q), out + nrj * (cc[f] + q), sizeof(double) * nrj,
                               cudaMemcpyDeviceToHost, h->stream));
    }
  }
  if (h->cor_on && h->cor_pending) {
    // sph_f_trans_w_coriolis: copy_coriolis_terms_rlm into the forward output
    const cudaMemcpyKind kind = ptr_kind == KMHD_PTR_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    for (int q = 0; q < 2; ++q)
      KCHECK(cudaMemcpyAsync(d_rj + ld * (h->cor_col + 2 * q), h->cor_cyc + nrj * q, sizeof(double) * nrj, kind,
                             h->stream));
    h->cor_pending = 0;
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  return finish_timing(h);
}

int kmhd_sph_cycle(kmhd_sph* h, const double* d_rj_in, int64_t ld_in, const int32_t* cols_b,
                   double* d_rj_out, int64_t ld_out, const int32_t* cols_f, int32_t ptr_kind) {
  if (!h || !d_rj_in || !d_rj_out) return KMHD_ERR_ARG;
  if (check_ld(h, ld_in) || check_ld(h, ld_out)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.ncf == 0 || p.nprod == 0) return KMHD_ERR_STATE;
  KCHECK(cudaSetDevice(h->device));
  const size_t nrj = (size_t)p.J * p.nr;
  const double* src = d_rj_in;
  int64_t sld = ld_in;
  double* out = d_rj_out;
  int64_t old = ld_out;
  std::vector<int> cb, cf(p.nvf + p.nsf);
  int st;
  if (h->cor_on && (st = check_coriolis_cols(h, d_rj_in, ld_in, cols_b, d_rj_out, ld_out, cols_f))) return st;
  if (ptr_kind == KMHD_PTR_HOST && h->chunks.size() > 2)
    return cycle_host_chunked(h, d_rj_in, ld_in, cols_b, d_rj_out, ld_out, cols_f);
  if (ptr_kind == KMHD_PTR_HOST) {
    if ((st = stage_host_in(h, d_rj_in, ld_in, cols_b, p.nvb, p.nsb, &src, &sld, cb))) return st;
    if ((st = sync_cols(h, cb.data(), p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
    if (!h->stage_out && (st = dalloc(h, &h->stage_out, nrj * std::max(p.ncf, 1)))) return st;
    out = h->stage_out;
    old = (int64_t)nrj;
    for (int f = 0; f < p.nvf + p.nsf; ++f) cf[f] = f < p.nvf ? 3 * f : 3 * p.nvf + (f - p.nvf);
    if ((st = sync_cols(h, cf.data(), p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) return st;
  } else {
    if ((st = sync_cols(h, cols_b, p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
    if ((st = sync_cols(h, cols_f, p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) return st;
  }
  double *cor_pol = nullptr, *cor_tor = nullptr;
  if (h->cor_on) {
    if (ptr_kind == KMHD_PTR_HOST) {
      if (!h->cor_cyc && (st = dalloc(h, &h->cor_cyc, 2 * nrj))) return st;
      cor_pol = h->cor_cyc;
      cor_tor = h->cor_cyc + nrj;
    } else {
      cor_pol = d_rj_out + ld_out * h->cor_col;
      cor_tor = d_rj_out + ld_out * (h->cor_col + 2);
    }
  }
  if ((st = timed_begin(h))) return st;
  // the Coriolis curl reads only the inputs: it runs before the forward
  // stage can write output columns that share the input array
  if (h->cor_on) {
    const int iv = ptr_kind == KMHD_PTR_HOST ? cb[h->cor_iv_velo] : cols_b[h->cor_iv_velo];
    const int iw = ptr_kind == KMHD_PTR_HOST ? cb[h->cor_iv_vort] : cols_b[h->cor_iv_vort];
    if ((st = enqueue_coriolis(h, src + sld * iv, src + sld * iw, sld, cor_pol, cor_tor, 0, p.nr, h->stream)))
      return st;
  }
  if ((st = run_bwd_spectral(h, src, sld))) return st;
  KCHECK(cudaEventRecord(h->ev[1], h->stream));
  KCHECK(launch_fft_cycle(p, h->stream));
  KCHECK(cudaEventRecord(h->ev[2], h->stream));
  if ((st = run_fwd_spectral(h, out, old))) return st;
  KCHECK(cudaEventRecord(h->ev[3], h->stream));
  if (ptr_kind == KMHD_PTR_HOST) {
    for (int f = 0; f < p.nvf + p.nsf; ++f) {
      const int ncomp = f < p.nvf ? 3 : 1;
      for (int q = 0; q < ncomp; ++q)
        KCHECK(cudaMemcpyAsync(d_rj_out + ld_out * (cols_f[f] + q), out + nrj * (cf[f] + q),
                               sizeof(double) * nrj, cudaMemcpyDeviceToHost, h->stream));
    }
    if (h->cor_on)
      for (int q = 0; q < 2; ++q)
        KCHECK(cudaMemcpyAsync(d_rj_out + ld_out * (h->cor_col + 2 * q), h->cor_cyc + nrj * q,
                               sizeof(double) * nrj, cudaMemcpyDeviceToHost, h->stream));
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  if ((st = finish_timing(h))) return st;
  return finish_kernel_timing(h);
}

}  // extern "C"

namespace {

// 3x3 inverse by cofactors, as cal_inverse_33_matrix / cal_det_33_matrix
// (CORE_src/BASE/cal_inverse_small_matrix.f90:57-80, 176-215).
double det22(double a00, double a01, double a10, double a11) { return a00 * a11 - a10 * a01; }
void inverse33(const double a[3][3], double inv[3][3]) {
  double det = 0.0;
  for (int k = 0; k < 3; ++k) {
    int c[2], n = 0;
    for (int q = 0; q < 3; ++q)
      if (q != k) c[n++] = q;
    det = det + ((k % 2) ? -1.0 : 1.0) * det22(a[1][c[0]], a[1][c[1]], a[2][c[0]], a[2][c[1]]) * a[0][k];
  }
  const double adet = 1.0 / det;
  for (int kj = 0; kj < 3; ++kj)
    for (int ki = 0; ki < 3; ++ki) {
      int rr[2], cc[2], nr = 0, nc = 0;
      for (int q = 0; q < 3; ++q) {
        if (q != ki) rr[nr++] = q;
        if (q != kj) cc[nc++] = q;
      }
      inv[kj][ki] = (((ki + kj) % 2) ? -1.0 : 1.0) * det22(a[rr[0]][cc[0]], a[rr[0]][cc[1]], a[rr[1]][cc[0]], a[rr[1]][cc[1]]) * adet;
    }
}

// Divergence coefficients on the device: d1[3 nr] (interior 3-point first
// derivative, nod_r_2nd_fdm_coef_noequi + copy_fdm2_nod_coefs_from_mat,
// CORE_src/SPH_SPECTR_src/set_radius_func_noequi.f90:193-260, t_fdm_coefs.f90:146-163),
// bnd[6] (fixed-field one-sided rows, cal_fdm2_coef_fix_fld_ICB / _CMB,
// MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90:155-190, 256-290), ar2[nr] =
// (1/r)^2 (set_radius_4_sph_dynamo.f90:105), g3[J] = max(l(l+1), 1/2).
int build_div_coef(kmhd_sph* h) {
  const Plan& p = h->plan;
  const int nr = p.nr, L = p.L;
  const std::vector<double>& r = h->radius_h;
  std::vector<double> c(3 * (size_t)nr + 6 + nr + (size_t)p.J + nr + (size_t)p.J + 3 * (size_t)nr, 0.0);
  double* d2c = c.data() + 3 * (size_t)nr + 6 + nr + (size_t)p.J + nr + (size_t)p.J;
  for (int k = 1; k < nr - 1; ++k) {
    const double dp = r[k + 1] - r[k], dn = r[k] - r[k - 1];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {1.0, dp, 0.5 * dp * dp}, {1.0, -dn, 0.5 * dn * dn}};
    double inv[3][3];
    inverse33(t, inv);
    c[3 * k + 0] = inv[1][2];
    c[3 * k + 1] = inv[1][0];
    c[3 * k + 2] = inv[1][1];
    // second derivative (fdm(2) of copy_fdm2_nod_coefs_from_mat, t_fdm_coefs.f90:146-163)
    d2c[3 * k + 0] = inv[2][2];
    d2c[3 * k + 1] = inv[2][0];
    d2c[3 * k + 2] = inv[2][1];
  }
  {
    const double d1 = r[1] - r[0], d2 = r[2] - r[0];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {1.0, d1, d1 * d1 / 2.0}, {1.0, d2, d2 * d2 / 2.0}};
    double inv[3][3];
    inverse33(t, inv);
    for (int q = 0; q < 3; ++q) c[3 * nr + q] = inv[1][q];
  }
  {
    const double d1 = r[nr - 1] - r[nr - 2], d2 = r[nr - 1] - r[nr - 3];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {1.0, -d1, d1 * d1 / 2.0}, {1.0, -d2, d2 * d2 / 2.0}};
    double inv[3][3];
    inverse33(t, inv);
    for (int q = 0; q < 3; ++q) c[3 * nr + 3 + q] = inv[1][q];
  }
  for (int k = 0; k < nr; ++k) {
    const double a1 = 1.0 / r[k];
    c[3 * nr + 6 + k] = a1 * a1;
  }
  double* g3 = c.data() + 4 * nr + 6;
  double* ar1 = g3 + p.J;  // 1/r (ar_1d_rj(k,1)) and l (g_sph_rj(j,1)) for the curl's boundary rows
  double* gl = ar1 + nr;
  for (int k = 0; k < nr; ++k) ar1[k] = 1.0 / r[k];
  for (int m = 0; m <= L; ++m)
    for (int slot = 0; slot < 2; ++slot)
      for (int l = m; l <= L; ++l) {
        const int j = h->jmap_h[((size_t)m * 2 + slot) * (L + 1) + l];
        if (j >= 0) {
          g3[j] = std::max(g3_of(l), 0.5);
          gl[j] = (double)l;
        }
      }
  int st;
  if ((st = dalloc(h, &h->div_coef, c.size()))) return st;
  KCHECK(cudaMemcpyAsync(h->div_coef, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

// Coriolis curl tables (per mode j of the rj order): the coupled modes and
// the sw / tw coefficients of interact_rot_coriolis_rlm
// (MHD_src/sph_MHD/interact_coriolis_rlm.f90), from the integrals of
// cal_gaunt_coriolis_rlm (same file) in closed form for the rotation's degree
// 1, order 0:
//   K(1,0; l-1,m; l,m) = 4 sqrt(l^2 - m^2) / ((2l-1)(2l+1))        (l >= 2, |m| <= l-1),
//   K(1,0; l+1,m; l,m) = 4 sqrt((l+1)^2 - m^2) / ((2l+1)(2l+3))    (l+1 <= L),
//   L(1,0; l,-m; l,m)  = -4 m / (2l+1)                              (l >= 1),
// with the mode itself (zero integral) where the partner does not exist and
// every integral of l = 0 zero.  These equal the reference's prime-factor
// evaluations (leadki / leadli, cal_gaunt_itgs.f90) to rounding; g3, g4, g5,
// g17 are g_sph_rlm's l(l+1) (1/2 at l = 0), (l-1)l, (l+1)(l+2),
// (2l+1)/(4l(l+1)) (0 at l = 0) (spherical_harmonics.f90:91-140).
int build_coriolis(kmhd_sph* h) {
  const Plan& p = h->plan;
  const int L = p.L;
  const long long J = p.J;
  auto jof = [&](int l, int m) { return h->jmap_h[((size_t)std::abs(m) * 2 + (m < 0 ? 1 : 0)) * (L + 1) + l]; };
  std::vector<int> idx(4 * (size_t)J, 0);
  std::vector<double> cf(12 * (size_t)J, 0.0);
  for (int am = 0; am <= L; ++am)
    for (int slot = 0; slot < 2; ++slot) {
      if (am == 0 && slot == 1) continue;
      const int m = slot ? -am : am;
      for (int l = am; l <= L; ++l) {
        const int j = jof(l, m);
        int k1 = j, k2 = j, ke = jof(0, 0);
        double gi1 = 0.0, gi2 = 0.0, ei = 0.0;
        const double dl = (double)l, dm = (double)m;
        if (l >= 2 && am <= l - 1) {
          gi1 = 4.0 * std::sqrt(dl * dl - dm * dm) / ((2.0 * dl - 1.0) * (2.0 * dl + 1.0));
          k1 = jof(l - 1, m);
        }
        if (l + 1 <= L) {
          gi2 = 4.0 * std::sqrt((dl + 1.0) * (dl + 1.0) - dm * dm) / ((2.0 * dl + 1.0) * (2.0 * dl + 3.0));
          k2 = jof(l + 1, m);
        }
        if (l >= 1) {
          ei = -4.0 * dm / (2.0 * dl + 1.0);
          ke = jof(l, -m);
        }
        if (l == 0) {
          k1 = k2 = ke = j;
          gi2 = ei = 0.0;
        }
        const double g3 = l == 0 ? 0.5 : dl * (dl + 1.0);
        const double g4 = (dl - 1.0) * dl, g5 = (dl + 1.0) * (dl + 2.0);
        const double g17 = l == 0 ? 0.0 : (2.0 * dl + 1.0) / (4.0 * dl * (dl + 1.0));
        int* q = idx.data() + 4 * (size_t)j;
        q[0] = k1;
        q[1] = k2;
        q[2] = ke;
        double* c = cf.data() + 12 * (size_t)j;
        c[0] = (2.0 - g4 - g3) * gi1 * g17;                                         // sw(1,1)
        c[1] = (2.0 - g5 - g3) * gi2 * g17;                                         // sw(2,1)
        c[2] = 2.0 * ei * g17;                                                      // sw(1,3)
        c[3] = g4 * (2.0 - g4 + g3) * gi1 * g17 * 0.5;                              // sw(1,2)
        c[4] = g5 * (2.0 - g5 + g3) * gi2 * g17 * 0.5;                              // sw(2,2)
        c[5] = -2.0 * ei * g17;                                                     // tw(1,1)
        c[6] = -g3 * ei * g17;                                                      // tw(1,2)
        c[7] = -(g3 * (2.0 + g4 - g3) + 2.0 * (-2.0 + g4 + g3)) * gi1 * g17 * 0.5;  // tw(1,3)
        c[8] = -(g3 * (2.0 + g5 - g3) + 2.0 * (-2.0 + g5 + g3)) * gi2 * g17 * 0.5;  // tw(2,3)
        c[9] = -(-2.0 + g4 + g3) * gi1 * g17;                                       // tw(1,4)
        c[10] = -(-2.0 + g5 + g3) * gi2 * g17;                                      // tw(2,4)
        c[11] = g3;
      }
    }
  int st;
  if ((st = dalloc(h, &h->cor_idx, idx.size())) || (st = dalloc(h, &h->cor_cf, cf.size()))) return st;
  KCHECK(cudaMemcpyAsync(h->cor_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, h->stream));
  KCHECK(cudaMemcpyAsync(h->cor_cf, cf.data(), sizeof(double) * cf.size(), cudaMemcpyHostToDevice, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

// Divergence of the vector in columns col_flux, col_flux + 1 into col_div;
// own_bnd = 1 puts each boundary node's own S into the one-sided rows (the
// force divergence), else fix_in / fix_out (NULL = zero).
int div_vec(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_flux, int32_t col_div, const double* fix_in,
            const double* fix_out, int own_bnd, int32_t ptr_kind, int flux_in = 0, int flux_out = 0) {
  if (!h || !d_rj) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  if (col_flux < 0 || col_div < 0 || col_div == col_flux || col_div == col_flux + 1) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.nr < 3) return KMHD_ERR_SIZE;
  KCHECK(cudaSetDevice(h->device));
  int st;
  if (!h->div_coef && (st = build_div_coef(h))) return st;
  const size_t nrj = (size_t)p.J * p.nr, last = (size_t)p.J * (p.nr - 1);
  const double *S = d_rj + ld * col_flux, *dS = d_rj + ld * (col_flux + 1), *fin = fix_in, *fout = fix_out;
  double* out = d_rj + ld * col_div;
  if (ptr_kind == KMHD_PTR_HOST) {
    // columns S, dS, div and the two boundary rows
    if (!h->div_stage && (st = dalloc(h, &h->div_stage, 3 * nrj + 2 * (size_t)p.J))) return st;
    double* s0 = h->div_stage;
    KCHECK(cudaMemcpyAsync(s0, S, sizeof(double) * nrj, cudaMemcpyHostToDevice, h->stream));
    KCHECK(cudaMemcpyAsync(s0 + nrj, dS, sizeof(double) * nrj, cudaMemcpyHostToDevice, h->stream));
    if (own_bnd) {
      fin = s0;
      fout = s0 + last;
    } else {
      if (fix_in) {
        KCHECK(cudaMemcpyAsync(s0 + 3 * nrj, fix_in, sizeof(double) * p.J, cudaMemcpyHostToDevice, h->stream));
        fin = s0 + 3 * nrj;
      }
      if (fix_out) {
        KCHECK(cudaMemcpyAsync(s0 + 3 * nrj + p.J, fix_out, sizeof(double) * p.J, cudaMemcpyHostToDevice, h->stream));
        fout = s0 + 3 * nrj + p.J;
      }
    }
    KCHECK(launch_div_flux(p.J, p.nr, s0, s0 + nrj, s0 + 2 * nrj, h->div_coef, fin, fout, h->stream, flux_in,
                           flux_out));
    KCHECK(cudaMemcpyAsync(out, s0 + 2 * nrj, sizeof(double) * nrj, cudaMemcpyDeviceToHost, h->stream));
  } else {
    if (own_bnd) {
      fin = S;
      fout = S + last;
    }
    KCHECK(launch_div_flux(p.J, p.nr, S, dS, out, h->div_coef, fin, fout, h->stream, flux_in, flux_out));
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

// Curl of the vector in columns col_fld .. col_fld + 2 into col_rot .. col_rot + 2.
int rot_vec(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_fld, int32_t col_rot, const RotBnd& b,
            int32_t ptr_kind) {
  if (!h || !d_rj) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  if (col_fld < 0 || col_rot < 0 || (col_rot < col_fld + 3 && col_fld < col_rot + 3)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.nr < 3) return KMHD_ERR_SIZE;
  KCHECK(cudaSetDevice(h->device));
  int st;
  if (!h->div_coef && (st = build_div_coef(h))) return st;
  const size_t nrj = (size_t)p.J * p.nr;
  if (ptr_kind == KMHD_PTR_HOST) {
    if (!h->rot_stage && (st = dalloc(h, &h->rot_stage, 6 * nrj))) return st;
    double* s0 = h->rot_stage;
    for (int q = 0; q < 3; ++q)
      KCHECK(cudaMemcpyAsync(s0 + q * nrj, d_rj + ld * (col_fld + q), sizeof(double) * nrj, cudaMemcpyHostToDevice,
                             h->stream));
    KCHECK(launch_rot_vec(p.J, p.nr, s0, s0 + nrj, s0 + 2 * nrj, s0 + 3 * nrj, s0 + 4 * nrj, s0 + 5 * nrj,
                          h->div_coef, b, h->stream));
    for (int q = 0; q < 3; ++q)
      KCHECK(cudaMemcpyAsync(d_rj + ld * (col_rot + q), s0 + (3 + q) * nrj, sizeof(double) * nrj,
                             cudaMemcpyDeviceToHost, h->stream));
  } else {
    const double* in = d_rj + ld * col_fld;
    double* out = d_rj + ld * col_rot;
    KCHECK(launch_rot_vec(p.J, p.nr, in, in + ld, in + 2 * ld, out, out + ld, out + 2 * ld, h->div_coef, b,
                          h->stream));
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

// Boundary rows of the curl of a force for the velocity conditions, built as
// the reference builds them (cofactor inverses of 3x3 Taylor matrices):
// non-slip d2S/dr2 from cal_fdm2_coef_fix_df_ICB / _CMB
// (MHD_src/sph_MHD/cal_fdm_coefs_4_boundaries.f90:195-231, 297-334), whose
// unknowns are ordered (dS/dr, S, d2S/dr2) at the inner and (S, dS/dr,
// d2S/dr2) at the outer boundary; dT/dr from the fixed-field one-sided rows;
// free slip from cal_fdm2_ICB_free_vp / _vt and cal_fdm2_CMB_free_vp / _vt
// (coef_fdm2_free_ICB.f90, coef_fdm2_free_CMB.f90).
RotBnd velocity_bnd(const std::vector<double>& r, int bc_icb, int bc_cmb) {
  const int nr = (int)r.size();
  RotBnd b{};
  double inv[3][3];
  if (bc_icb == KMHD_BC_NON_SLIP) {
    const double dr = r[1] - r[0];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {dr, 1.0, dr * dr / 2.0}};
    inverse33(t, inv);
    b.s_in[0] = inv[2][1];
    b.s_in[1] = inv[2][2];
    const double d1 = r[1] - r[0], d2 = r[2] - r[0];
    const double f[3][3] = {{1.0, 0.0, 0.0}, {1.0, d1, d1 * d1 / 2.0}, {1.0, d2, d2 * d2 / 2.0}};
    inverse33(f, inv);
    for (int q = 0; q < 3; ++q) b.t_in[q] = inv[1][q];
  } else {
    const double dr = r[1] - r[0], r0 = r[0];
    const double vp[3][3] = {{1.0, 0.0, 0.0}, {1.0, -r0, 0.5 * r0 * r0}, {1.0, dr, 0.5 * dr * dr}};
    inverse33(vp, inv);
    b.s_in[0] = inv[2][0];
    b.s_in[1] = inv[2][2];
    const double vt[3][3] = {{1.0, 0.0, 0.0}, {2.0, -r0, 0.0}, {1.0, dr, 0.5 * dr * dr}};
    inverse33(vt, inv);
    b.t_in[0] = inv[1][0];
  }
  if (bc_cmb == KMHD_BC_NON_SLIP) {
    const double dn = r[nr - 1] - r[nr - 2];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {1.0, -dn, dn * dn / 2.0}};
    inverse33(t, inv);
    b.s_out[0] = inv[2][0];
    b.s_out[1] = inv[2][2];
    const double d1 = r[nr - 1] - r[nr - 2], d2 = r[nr - 1] - r[nr - 3];
    const double f[3][3] = {{1.0, 0.0, 0.0}, {1.0, -d1, d1 * d1 / 2.0}, {1.0, -d2, d2 * d2 / 2.0}};
    inverse33(f, inv);
    for (int q = 0; q < 3; ++q) b.t_out[q] = inv[1][q];
  } else {
    const double dn = r[nr - 1] - r[nr - 2], r0 = r[nr - 1];
    const double vp[3][3] = {{1.0, 0.0, 0.0}, {1.0, -r0, 0.5 * r0 * r0}, {1.0, -dn, 0.5 * dn * dn}};
    inverse33(vp, inv);
    b.s_out[0] = inv[2][0];
    b.s_out[1] = inv[2][2];
    const double vt[3][3] = {{1.0, 0.0, 0.0}, {2.0, -r0, 0.0}, {1.0, -dn, 0.5 * dn * dn}};
    inverse33(vt, inv);
    b.t_out[0] = inv[1][0];
  }
  return b;
}

}  // namespace

extern "C" {

int kmhd_sph_div_flux(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_flux, int32_t col_div,
                      const double* fix_in, const double* fix_out, int32_t ptr_kind) {
  return div_vec(h, d_rj, ld, col_flux, col_div, fix_in, fix_out, 0, ptr_kind);
}

int kmhd_sph_rot_induction(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_fld, int32_t col_rot,
                           int32_t ptr_kind) {
  RotBnd b{};
  b.insulating_in = b.insulating_out = 1;
  return rot_vec(h, d_rj, ld, col_fld, col_rot, b, ptr_kind);
}

int kmhd_sph_div_flux_bc(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_flux, int32_t col_div, int32_t bc_icb,
                         int32_t bc_cmb, const double* val_in, const double* val_out, int32_t ptr_kind) {
  const int ok_in = bc_icb == KMHD_BC_FIXED_FIELD || bc_icb == KMHD_BC_FIXED_FLUX;
  const int ok_out = bc_cmb == KMHD_BC_FIXED_FIELD || bc_cmb == KMHD_BC_FIXED_FLUX;
  if (!ok_in || !ok_out) return KMHD_ERR_ARG;
  return div_vec(h, d_rj, ld, col_flux, col_div, val_in, val_out, 0, ptr_kind, bc_icb == KMHD_BC_FIXED_FLUX,
                 bc_cmb == KMHD_BC_FIXED_FLUX);
}

int kmhd_sph_rot_induction_bc(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_fld, int32_t col_rot,
                              int32_t bc_icb, int32_t bc_cmb, int32_t ptr_kind) {
  const int ok_in = bc_icb == KMHD_BC_INSULATOR || bc_icb == KMHD_BC_PSEUDO_VACUUM;
  const int ok_out = bc_cmb == KMHD_BC_INSULATOR || bc_cmb == KMHD_BC_PSEUDO_VACUUM;
  if (!ok_in || !ok_out) return KMHD_ERR_ARG;
  RotBnd b{};
  b.insulating_in = b.insulating_out = 1;
  b.qvac_in = bc_icb == KMHD_BC_PSEUDO_VACUUM;
  b.qvac_out = bc_cmb == KMHD_BC_PSEUDO_VACUUM;
  return rot_vec(h, d_rj, ld, col_fld, col_rot, b, ptr_kind);
}

int kmhd_sph_rot_force(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_fld, int32_t col_rot, int32_t bc_icb,
                       int32_t bc_cmb, int32_t ptr_kind) {
  if (!h) return KMHD_ERR_ARG;
  const int ok_in = bc_icb == KMHD_BC_NON_SLIP || bc_icb == KMHD_BC_FREE_SLIP;
  const int ok_out = bc_cmb == KMHD_BC_NON_SLIP || bc_cmb == KMHD_BC_FREE_SLIP;
  if (!ok_in || !ok_out) return KMHD_ERR_ARG;
  if (h->plan.nr < 3) return KMHD_ERR_SIZE;
  return rot_vec(h, d_rj, ld, col_fld, col_rot, velocity_bnd(h->radius_h, bc_icb, bc_cmb), ptr_kind);
}

int kmhd_sph_vorticity(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_velo, int32_t col_vort, int32_t bc_icb,
                       int32_t bc_cmb, int32_t ptr_kind) {
  if (!h) return KMHD_ERR_ARG;
  const int ok_in = bc_icb == KMHD_BC_NON_SLIP || bc_icb == KMHD_BC_FREE_SLIP;
  const int ok_out = bc_cmb == KMHD_BC_NON_SLIP || bc_cmb == KMHD_BC_FREE_SLIP;
  if (!ok_in || !ok_out) return KMHD_ERR_ARG;
  if (h->plan.nr < 3) return KMHD_ERR_SIZE;
  RotBnd b = velocity_bnd(h->radius_h, bc_icb, bc_cmb);
  b.d2_interior = 1;
  return rot_vec(h, d_rj, ld, col_velo, col_vort, b, ptr_kind);
}

int kmhd_sph_current(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_magne, int32_t col_current, int32_t bc_icb,
                     int32_t bc_cmb, int32_t ptr_kind) {
  if (!h) return KMHD_ERR_ARG;
  const int ok_in = bc_icb == KMHD_BC_INSULATOR || bc_icb == KMHD_BC_PSEUDO_VACUUM;
  const int ok_out = bc_cmb == KMHD_BC_INSULATOR || bc_cmb == KMHD_BC_PSEUDO_VACUUM;
  if (!ok_in || !ok_out) return KMHD_ERR_ARG;
  if (h->plan.nr < 3) return KMHD_ERR_SIZE;
  // the non-slip coefficient rows (fixed dS/dr): pseudo-vacuum takes dS/dr = 0,
  // an insulator the potential field's dS/dr, through the coefficient of the
  // fixed derivative (cal_sph_nod_icb_ins_rot2 / cal_sph_nod_cmb_ins_rot2,
  // cal_sph_exp_nod_icb_ins.f90, cal_sph_exp_nod_cmb_ins.f90;
  // cal_sph_nod_icb_qvc_rot2 / cal_sph_nod_cmb_qvc_rot2)
  RotBnd b = velocity_bnd(h->radius_h, KMHD_BC_NON_SLIP, KMHD_BC_NON_SLIP);
  b.d2_interior = 1;
  const std::vector<double>& r = h->radius_h;
  const int nr = (int)r.size();
  double inv[3][3];
  {
    const double dr = r[1] - r[0];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {dr, 1.0, dr * dr / 2.0}};
    inverse33(t, inv);
    b.cdr_in = inv[2][0];  // fdm2_fix_dr_ICB(-1,3): the fixed derivative's coefficient
  }
  {
    const double dn = r[nr - 1] - r[nr - 2];
    const double t[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {1.0, -dn, dn * dn / 2.0}};
    inverse33(t, inv);
    b.cdr_out = inv[2][1];  // fdm2_fix_dr_CMB(1,3)
  }
  b.ins_s_in = bc_icb == KMHD_BC_INSULATOR;
  b.ins_s_out = bc_cmb == KMHD_BC_INSULATOR;
  return rot_vec(h, d_rj, ld, col_magne, col_current, b, ptr_kind);
}

int kmhd_sph_div_force(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_fld, int32_t col_div, int32_t ptr_kind) {
  return div_vec(h, d_rj, ld, col_fld, col_div, nullptr, nullptr, 1, ptr_kind);
}

int kmhd_sph_rot_coriolis(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_velo, int32_t col_vort,
                          int32_t col_out, double coef_cor, int32_t ptr_kind) {
  if (!h || !d_rj) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  if (col_velo < 0 || col_vort < 0 || col_out < 0) return KMHD_ERR_ARG;
  for (int q = 0; q < 3; q += 2) {  // the two written columns may not be inputs
    const int c = col_out + q;
    if ((c >= col_velo && c < col_velo + 3) || (c >= col_vort && c < col_vort + 3)) return KMHD_ERR_ARG;
  }
  const Plan& p = h->plan;
  KCHECK(cudaSetDevice(h->device));
  int st;
  if (!h->cor_idx && (st = build_coriolis(h))) return st;
  const size_t nrj = (size_t)p.J * p.nr;
  if (ptr_kind == KMHD_PTR_HOST) {
    if (!h->cor_stage && (st = dalloc(h, &h->cor_stage, 8 * nrj))) return st;
    double* s0 = h->cor_stage;
    for (int q = 0; q < 3; ++q) {
      KCHECK(cudaMemcpyAsync(s0 + q * nrj, d_rj + ld * (col_velo + q), sizeof(double) * nrj, cudaMemcpyHostToDevice,
                             h->stream));
      KCHECK(cudaMemcpyAsync(s0 + (3 + q) * nrj, d_rj + ld * (col_vort + q), sizeof(double) * nrj,
                             cudaMemcpyHostToDevice, h->stream));
    }
    KCHECK(launch_rot_coriolis(p.J, p.nr, s0, s0 + 3 * nrj, (long long)nrj, s0 + 6 * nrj, s0 + 7 * nrj, h->cor_idx,
                               h->cor_cf, h->radius, coef_cor, h->stream));
    KCHECK(cudaMemcpyAsync(d_rj + ld * col_out, s0 + 6 * nrj, sizeof(double) * nrj, cudaMemcpyDeviceToHost, h->stream));
    KCHECK(cudaMemcpyAsync(d_rj + ld * (col_out + 2), s0 + 7 * nrj, sizeof(double) * nrj, cudaMemcpyDeviceToHost,
                           h->stream));
  } else {
    KCHECK(launch_rot_coriolis(p.J, p.nr, d_rj + ld * col_velo, d_rj + ld * col_vort, ld, d_rj + ld * col_out,
                               d_rj + ld * (col_out + 2), h->cor_idx, h->cor_cf, h->radius, coef_cor, h->stream));
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

int kmhd_sph_set_coriolis(kmhd_sph* h, double coef_cor, int32_t iv_velo, int32_t iv_vort, int32_t col_out) {
  if (!h) return KMHD_ERR_ARG;
  if (iv_velo < 0) {
    h->cor_on = 0;
    return KMHD_OK;
  }
  const Plan& p = h->plan;
  if (iv_velo >= p.nvb || iv_vort < 0 || iv_vort >= p.nvb || iv_vort == iv_velo || col_out < 0) return KMHD_ERR_ARG;
  KCHECK(cudaSetDevice(h->device));
  int st;
  if (!h->cor_idx && (st = build_coriolis(h))) return st;
  h->cor_iv_velo = iv_velo;
  h->cor_iv_vort = iv_vort;
  h->cor_col = col_out;
  h->cor_coef = coef_cor;
  h->cor_on = 1;
  return KMHD_OK;
}

int kmhd_sph_b_trans_pole(kmhd_sph* h, const double* d_rj, int64_t ld, const int32_t* cols_b, double* v_pole,
                          int32_t ptr_kind) {
  if (!h || !d_rj || !v_pole || !cols_b) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.nvb + p.nsb == 0) return KMHD_ERR_STATE;
  KCHECK(cudaSetDevice(h->device));
  int st;
  const double* src = d_rj;
  int64_t sld = ld;
  std::vector<int> cc;
  double* out = v_pole;
  const size_t nout = 2 * (size_t)p.nr * p.ncb;
  if (ptr_kind == KMHD_PTR_HOST) {
    if ((st = stage_host_in(h, d_rj, ld, cols_b, p.nvb, p.nsb, &src, &sld, cc))) return st;
    if ((st = sync_cols(h, cc.data(), p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
    if (!h->pole_out && (st = dalloc(h, &h->pole_out, nout))) return st;
    out = h->pole_out;
  } else if ((st = sync_cols(h, cols_b, p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) {
    return st;
  }
  KCHECK(launch_b_trans_pole(p, src, sld, h->cols_b_d, out, 2LL * p.nr, h->stream));
  if (ptr_kind == KMHD_PTR_HOST)
    KCHECK(cudaMemcpyAsync(v_pole, out, sizeof(double) * nout, cudaMemcpyDeviceToHost, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

int kmhd_sph_b_trans_center(kmhd_sph* h, const double* d_rj, int64_t ld, const int32_t* cols_b, double* v_center,
                            int32_t ptr_kind) {
  if (!h || !d_rj || !v_center || !cols_b) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (p.nvb + p.nsb == 0) return KMHD_ERR_STATE;
  if (p.nvb == 0) return KMHD_OK;  // scalars are left as they are
  KCHECK(cudaSetDevice(h->device));
  int st;
  const double* src = d_rj;
  int64_t sld = ld;
  std::vector<int> cc;
  double* out = v_center;
  if (ptr_kind == KMHD_PTR_HOST) {
    if ((st = stage_host_in(h, d_rj, ld, cols_b, p.nvb, p.nsb, &src, &sld, cc))) return st;
    if ((st = sync_cols(h, cc.data(), p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
    if (!h->pole_out && (st = dalloc(h, &h->pole_out, 2 * (size_t)p.nr * p.ncb))) return st;
    out = h->pole_out;
  } else if ((st = sync_cols(h, cols_b, p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) {
    return st;
  }
  KCHECK(launch_b_trans_center(p, src, sld, h->cols_b_d, out, h->stream));
  if (ptr_kind == KMHD_PTR_HOST)
    KCHECK(cudaMemcpyAsync(v_center, out, sizeof(double) * 3 * p.nvb, cudaMemcpyDeviceToHost, h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

int kmhd_sph_rot_buoyancy(kmhd_sph* h, double* d_rj, int64_t ld, int32_t col_t, double coef_t, int32_t col_c,
                          double coef_c, int32_t col_out, int32_t ptr_kind) {
  if (!h || !d_rj) return KMHD_ERR_ARG;
  if (check_ld(h, ld)) return KMHD_ERR_ARG;
  if (col_t < 0 || col_out < 0 || col_out == col_t || (col_c >= 0 && col_out == col_c)) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  KCHECK(cudaSetDevice(h->device));
  const size_t nrj = (size_t)p.J * p.nr;
  int st;
  if (ptr_kind == KMHD_PTR_HOST) {
    // T, C and the result in the divergence staging (3 columns)
    if (!h->div_stage && (st = dalloc(h, &h->div_stage, 3 * nrj + 2 * (size_t)p.J))) return st;
    double* s0 = h->div_stage;
    KCHECK(cudaMemcpyAsync(s0, d_rj + ld * col_t, sizeof(double) * nrj, cudaMemcpyHostToDevice, h->stream));
    if (col_c >= 0)
      KCHECK(cudaMemcpyAsync(s0 + nrj, d_rj + ld * col_c, sizeof(double) * nrj, cudaMemcpyHostToDevice, h->stream));
    KCHECK(launch_rot_buoyancy(p.J, p.nr, s0, coef_t, col_c >= 0 ? s0 + nrj : nullptr, coef_c, s0 + 2 * nrj, h->radius,
                               h->stream));
    KCHECK(cudaMemcpyAsync(d_rj + ld * col_out, s0 + 2 * nrj, sizeof(double) * nrj, cudaMemcpyDeviceToHost, h->stream));
  } else {
    KCHECK(launch_rot_buoyancy(p.J, p.nr, d_rj + ld * col_t, coef_t, col_c >= 0 ? d_rj + ld * col_c : nullptr, coef_c,
                               d_rj + ld * col_out, h->radius, h->stream));
  }
  KCHECK(cudaStreamSynchronize(h->stream));
  return KMHD_OK;
}

int kmhd_sph_last_kernel_timing(kmhd_sph* h, double* ms5) {
  if (!h || !ms5) return KMHD_ERR_ARG;
  if (!h->kernel_timed) return KMHD_ERR_STATE;
  std::memcpy(ms5, h->last_kernel_ms, sizeof(h->last_kernel_ms));
  return KMHD_OK;
}

int kmhd_sph_get_tables(kmhd_sph* h, int32_t m, double* colat, double* weight, double* P, double* dP) {
  if (!h) return KMHD_ERR_ARG;
  const Plan& p = h->plan;
  if (m < 0 || m > p.L) return KMHD_ERR_ARG;
  KCHECK(cudaSetDevice(h->device));
  KCHECK(cudaStreamSynchronize(h->stream));
  if (colat) KCHECK(cudaMemcpy(colat, h->colat, sizeof(double) * p.nth, cudaMemcpyDeviceToHost));
  if (weight) KCHECK(cudaMemcpy(weight, h->weight, sizeof(double) * p.nth, cudaMemcpyDeviceToHost));
  const int nl = p.L - m + 1;
  if (p.otf) {
    if (!P && !dP) return KMHD_OK;
    double *gP = nullptr, *gdP = nullptr;
    KCHECK(cudaMalloc(&gP, sizeof(double) * 2 * (size_t)nl * p.nh));
    gdP = gP + (size_t)nl * p.nh;
    cudaError_t e = launch_otf_order(p, m, gP, gdP, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess && P) e = cudaMemcpy(P, gP, sizeof(double) * (size_t)nl * p.nh, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && dP) e = cudaMemcpy(dP, gdP, sizeof(double) * (size_t)nl * p.nh, cudaMemcpyDeviceToHost);
    cudaFree(gP);
    KCHECK(e);
    return KMHD_OK;
  }
  for (int which = 0; which < 2; ++which) {
    double* dst = which ? dP : P;
    if (!dst) continue;
    const double* tab = which ? h->dP : h->P;
    for (int q = 0; q < 2; ++q) {
      const int K = kcount(p.L, m, q);
      std::vector<double> buf((size_t)K * p.nh_pad);
      KCHECK(cudaMemcpy(buf.data(), tab + h->poff_h[2 * m + q], sizeof(double) * buf.size(), cudaMemcpyDeviceToHost));
      for (int k = 0; k < K; ++k) {
        const int li = 2 * k + q;  // l - m
        for (int i = 0; i < p.nh; ++i) dst[(size_t)li * p.nh + i] = buf[(size_t)k * p.nh_pad + i];
      }
    }
    (void)nl;
  }
  return KMHD_OK;
}

int kmhd_sph_batch_cycle(kmhd_sph** hs, int32_t n, const double* const* d_rj_in, const int64_t* ld_in,
                         const int32_t* const* cols_b, double* const* d_rj_out, const int64_t* ld_out,
                         const int32_t* const* cols_f) {
  return batch_cycle_impl(hs, n, d_rj_in, ld_in, cols_b, d_rj_out, ld_out, cols_f);
}

}  // extern "C"

// Batched instances.  Every instance runs on its own handle's stream; one
// captured CUDA graph forks them all from an internal stream and joins them,
// so small instances fill the GPU together.  The graph is kept in the first
// handle and replayed while the batch (handles, pointers, leading dimensions,
// paths) stays the same.  Handles created with KMHD_FLAG_AUTOTUNE first time
// the FP64 DMMA path and their split path on the call's own data and keep the
// faster one (both meet the tier's error bound).
namespace {

// Per output column c: bits of max |out - ref| and max |ref| (non-negative
// doubles order like their bit patterns).
__global__ void k_col_err(const double* __restrict__ out, long long ld, const int* __restrict__ col,
                          const double* __restrict__ ref, long long rows, unsigned long long* res) {
  const int c = blockIdx.y;
  const double* o = out + ld * col[c];
  const double* f = ref + rows * c;
  double d = 0.0, a = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows; i += (long long)gridDim.x * blockDim.x) {
    d = fmax(d, fabs(o[i] - f[i]));
    a = fmax(a, fabs(f[i]));
  }
  for (int k = 16; k > 0; k >>= 1) {
    d = fmax(d, __shfl_xor_sync(0xffffffffu, d, k));
    a = fmax(a, __shfl_xor_sync(0xffffffffu, a, k));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(res + 2 * c, (unsigned long long)__double_as_longlong(d));
    atomicMax(res + 2 * c + 1, (unsigned long long)__double_as_longlong(a));
  }
}

// Candidates of a split-tier handle: 0 the FP64 DMMA path, 1 the split path
// with the tier's full slice-product count (26 / 10), 2 with the highest
// digit-pair group dropped (21 / 6).  Each runs twice on the call's own data
// (the first round warms up); the split candidates' outputs are compared with
// the FP64 path's (max-norm relative error per output column, the measure of
// the tier's bound), and the fastest candidate whose error stays within a
// quarter of the tier's bound (1e-12 split, 1e-6 fp32acc) is kept.  The
// reference times its Legendre variants at start-up the same way, without the
// error check (select_legendre_transform,
// MHD_src/sph_MHD/init_sphrical_transform_MHD.f90:201-345).
int autotune_path(kmhd_sph* h, const double* in, int64_t ld_in, double* out, int64_t ld_out) {
  const Plan& p = h->plan;
  const int full = split_ns(h->split) == 6 ? 6 : 3;
  const double bound = 0.25 * (h->desc.tier == KMHD_TIER_SPLIT_I8 ? 1e-12 : 1e-6);
  // written output columns: three per forward vector, one per scalar
  std::vector<int> cols;
  for (int f = 0; f < p.nvf + p.nsf; ++f)
    for (int q = 0; q < (f < p.nvf ? 3 : 1); ++q) cols.push_back(h->cols_f_cache[f] + q);
  const int nc = (int)cols.size();
  const long long rows = p.J * (long long)p.nr;
  double* ref = nullptr;
  int* col_d = nullptr;
  unsigned long long* res = nullptr;
  int st = KMHD_OK;
  auto fail = [&](int e) {
    cudaFree(ref);
    cudaFree(col_d);
    cudaFree(res);
    h->use_split = true;
    split_set_terms(h->split, full);
    return e;
  };
  if (cudaMalloc(&ref, sizeof(double) * rows * nc) != cudaSuccess || cudaMalloc(&col_d, sizeof(int) * nc) != cudaSuccess ||
      cudaMalloc(&res, sizeof(unsigned long long) * 2 * nc) != cudaSuccess)
    return fail(KMHD_ERR_NOMEM);
  if (cudaMemcpyAsync(col_d, cols.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
    return fail(KMHD_ERR_CUDA);
  float ms[3] = {0, 0, 0};
  double err[3] = {0, 0, 0};
  for (int rep = 0; rep < 2; ++rep) {
    for (int c = 0; c < 3; ++c) {
      h->use_split = c > 0;
      split_set_terms(h->split, c == 2 ? full - 1 : full);
      if (cudaEventRecord(h->ev[0], h->stream) != cudaSuccess) return fail(KMHD_ERR_CUDA);
      if ((st = enqueue_cycle(h, in, ld_in, out, ld_out))) return fail(st);
      if (cudaEventRecord(h->ev[3], h->stream) != cudaSuccess || cudaEventSynchronize(h->ev[3]) != cudaSuccess ||
          cudaEventElapsedTime(&ms[c], h->ev[0], h->ev[3]) != cudaSuccess)
        return fail(KMHD_ERR_CUDA);
      if ((st = check_dev_err(h))) return fail(st);
      if (rep == 0) continue;
      if (c == 0) {
        for (int k = 0; k < nc; ++k)
          if (cudaMemcpyAsync(ref + rows * k, out + ld_out * cols[k], sizeof(double) * rows, cudaMemcpyDeviceToDevice,
                              h->stream) != cudaSuccess)
            return fail(KMHD_ERR_CUDA);
        continue;
      }
      std::vector<unsigned long long> r(2 * nc);
      if (cudaMemsetAsync(res, 0, sizeof(unsigned long long) * 2 * nc, h->stream) != cudaSuccess) return fail(KMHD_ERR_CUDA);
      k_col_err<<<dim3(64, nc), 256, 0, h->stream>>>(out, ld_out, col_d, ref, rows, res);
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(r.data(), res, sizeof(unsigned long long) * 2 * nc, cudaMemcpyDeviceToHost, h->stream) !=
              cudaSuccess ||
          cudaStreamSynchronize(h->stream) != cudaSuccess)
        return fail(KMHD_ERR_CUDA);
      for (int k = 0; k < nc; ++k) {
        double d, a;
        std::memcpy(&d, &r[2 * k], sizeof(d));
        std::memcpy(&a, &r[2 * k + 1], sizeof(a));
        if (a > 0.0) err[c] = std::max(err[c], d / a);
      }
    }
  }
  int best = 0;
  for (int c = 1; c < 3; ++c)
    if (err[c] <= bound && ms[c] < ms[best]) best = c;
  h->use_split = best > 0;
  split_set_terms(h->split, best == 2 ? full - 1 : full);
  for (int c = 0; c < 3; ++c) {
    h->tune_ms[c] = ms[c];
    h->tune_err[c] = err[c];
  }
  h->tuned = true;
  cudaFree(ref);
  cudaFree(col_d);
  cudaFree(res);
  return KMHD_OK;
}

int batch_direct(kmhd_sph** hs, int32_t n, const double* const* in, const int64_t* ld_in,
                 const int32_t* const* cols_b, double* const* out, const int64_t* ld_out) {
  for (int i = 0; i < n; ++i) {
    int st = enqueue_coriolis_dev(hs[i], in[i], ld_in[i], cols_b[i], out[i], ld_out[i]);
    if (!st) st = enqueue_cycle(hs[i], in[i], ld_in[i], out[i], ld_out[i]);
    if (st) return st;
  }
  for (int i = 0; i < n; ++i) KCHECK(cudaStreamSynchronize(hs[i]->stream));
  return KMHD_OK;
}

}  // namespace

int batch_cycle_impl(kmhd_sph** hs, int32_t n, const double* const* d_rj_in, const int64_t* ld_in,
                     const int32_t* const* cols_b, double* const* d_rj_out, const int64_t* ld_out,
                     const int32_t* const* cols_f) {
  if (!hs || n <= 0 || !d_rj_in || !ld_in || !cols_b || !d_rj_out || !ld_out || !cols_f)
    return KMHD_ERR_ARG;
  int st;
  for (int i = 0; i < n; ++i) {
    kmhd_sph* h = hs[i];
    if (!h || !d_rj_in[i] || !d_rj_out[i]) return KMHD_ERR_ARG;
    if (h->device != hs[0]->device) return KMHD_ERR_ARG;
    if (check_ld(h, ld_in[i]) || check_ld(h, ld_out[i])) return KMHD_ERR_ARG;
    if (h->plan.ncf == 0 || h->plan.nprod == 0) return KMHD_ERR_STATE;
    if (h->cor_on && (st = check_coriolis_cols(h, d_rj_in[i], ld_in[i], cols_b[i], d_rj_out[i], ld_out[i], cols_f[i])))
      return st;
  }
  KCHECK(cudaSetDevice(hs[0]->device));
  // column tables to the device (may synchronise: before any capture)
  for (int i = 0; i < n; ++i) {
    kmhd_sph* h = hs[i];
    const Plan& p = h->plan;
    if ((st = sync_cols(h, cols_b[i], p.nvb + p.nsb, h->cols_b_cache, h->cols_b_d))) return st;
    if ((st = sync_cols(h, cols_f[i], p.nvf + p.nsf, h->cols_f_cache, h->cols_f_d))) return st;
  }
  for (int i = 0; i < n; ++i)
    if (hs[i]->autotune && !hs[i]->tuned && (st = autotune_path(hs[i], d_rj_in[i], ld_in[i], d_rj_out[i], ld_out[i])))
      return st;
  for (int i = 0; i < n; ++i) hs[i]->kernel_timed = false;
  // graph capture needs every instance on a capturable (non-legacy) stream
  bool capturable = true;
  for (int i = 0; i < n; ++i)
    if (hs[i]->stream == nullptr || hs[i]->stream == cudaStreamLegacy) capturable = false;
  if (!capturable) {
    if ((st = batch_direct(hs, n, d_rj_in, ld_in, cols_b, d_rj_out, ld_out))) return st;
  } else {
    std::vector<const void*> sig;
    std::vector<int64_t> sig_ld;
    for (int i = 0; i < n; ++i) {
      sig.push_back(hs[i]);
      sig.push_back(d_rj_in[i]);
      sig.push_back(d_rj_out[i]);
      sig.push_back(hs[i]->use_split ? hs[i] : nullptr);
      sig.push_back(reinterpret_cast<const void*>((intptr_t)(hs[i]->split ? split_terms(hs[i]->split) : 0)));
      sig.push_back(hs[i]->stream);
      sig_ld.push_back(ld_in[i]);
      sig_ld.push_back(ld_out[i]);
      // the Coriolis launch's arguments are captured too
      int64_t cbits = 0;
      std::memcpy(&cbits, &hs[i]->cor_coef, sizeof(cbits));
      sig_ld.push_back(hs[i]->cor_on ? cbits : 0);
      sig_ld.push_back(hs[i]->cor_on ? (int64_t)hs[i]->cor_col * 4096 + hs[i]->cor_iv_velo * 64 + hs[i]->cor_iv_vort + 1
                                     : 0);
      sig_ld.push_back(hs[i]->cor_on ? cols_b[i][hs[i]->cor_iv_velo] * 65536LL + cols_b[i][hs[i]->cor_iv_vort] : 0);
    }
    kmhd_sph* h0 = hs[0];
    if (!h0->batch) h0->batch = new BatchGraph();
    BatchGraph* bg = h0->batch;
    if (!bg->exec || bg->sig != sig || bg->sig_ld != sig_ld) {
      if (bg->exec) {
        cudaGraphExecDestroy(bg->exec);
        bg->exec = nullptr;
      }
      if (!bg->s0) KCHECK(cudaStreamCreateWithFlags(&bg->s0, cudaStreamNonBlocking));
      if (!bg->fork) KCHECK(cudaEventCreateWithFlags(&bg->fork, cudaEventDisableTiming));
      while ((int)bg->join.size() < n) {
        cudaEvent_t e;
        KCHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        bg->join.push_back(e);
      }
      // split-path instances by tier and product count: grouped GEMMs (built
      // before the capture); kind 0/1: 6 slices, 26/21 products, 2/3: 4 slices, 10/6
      std::vector<int> grp[4];
      for (int i = 0; i < n; ++i)
        if (hs[i]->split && hs[i]->use_split) {
          const bool six = split_ns(hs[i]->split) == 6;
          const int full = six ? 6 : 3;
          grp[(six ? 0 : 2) + (split_terms(hs[i]->split) == full ? 0 : 1)].push_back(i);
        }
      for (int k = 0; k < 4; ++k) {
        split_group_destroy(bg->group[k]);
        bg->group[k] = nullptr;
        if (grp[k].size() < 2) {
          grp[k].clear();  // a lone instance runs its own cycle
          continue;
        }
        std::vector<SplitState*> ss;
        std::vector<Plan> pl;
        std::vector<double*> outs;
        std::vector<long long> lds;
        std::vector<const int*> cfs;
        for (int i : grp[k]) {
          ss.push_back(hs[i]->split);
          pl.push_back(hs[i]->plan);
          outs.push_back(d_rj_out[i]);
          lds.push_back(ld_out[i]);
          cfs.push_back(hs[i]->cols_f_d);
        }
        if ((st = split_group_create(&bg->group[k], ss.data(), pl.data(), (int)ss.size(), outs.data(), lds.data(),
                                     cfs.data(), bg->s0)))
          return st;
        if (!bg->gs[k]) KCHECK(cudaStreamCreateWithFlags(&bg->gs[k], cudaStreamNonBlocking));
      }
      std::vector<char> grouped(n, 0);
      for (int k = 0; k < 4; ++k)
        for (int i : grp[k]) grouped[i] = 1;
      while (bg->ev.size() < (size_t)(2 * n + 8)) {
        cudaEvent_t e;
        KCHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        bg->ev.push_back(e);
      }
      cudaGraph_t graph = nullptr;
      KCHECK(cudaStreamBeginCapture(bg->s0, cudaStreamCaptureModeRelaxed));
      int cst = KMHD_OK;
      auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && cst == KMHD_OK) cst = KMHD_ERR_CUDA;
      };
      ck(cudaEventRecord(bg->fork, bg->s0));
      // ungrouped instances: the whole cycle on the instance's stream
      for (int i = 0; i < n && cst == KMHD_OK; ++i) {
        if (grouped[i]) continue;
        ck(cudaStreamWaitEvent(hs[i]->stream, bg->fork, 0));
        if (cst == KMHD_OK) cst = enqueue_coriolis_dev(hs[i], d_rj_in[i], ld_in[i], cols_b[i], d_rj_out[i], ld_out[i]);
        if (cst == KMHD_OK) cst = enqueue_cycle(hs[i], d_rj_in[i], ld_in[i], d_rj_out[i], ld_out[i]);
        ck(cudaEventRecord(bg->join[i], hs[i]->stream));
        ck(cudaStreamWaitEvent(bg->s0, bg->join[i], 0));
      }
      // grouped instances: slicers, FFT and the FP64 dipole modes on the
      // instance streams, one grouped GEMM per direction on the group stream
      for (int k = 0; k < 4 && cst == KMHD_OK; ++k) {
        if (grp[k].empty()) continue;
        cudaStream_t g = bg->gs[k];
        cudaEvent_t eg0 = bg->ev[2 * n + 2 * k], eg1 = bg->ev[2 * n + 2 * k + 1];
        ck(cudaStreamWaitEvent(g, bg->fork, 0));
        for (int i : grp[k]) {
          kmhd_sph* h = hs[i];
          ck(cudaStreamWaitEvent(h->stream, bg->fork, 0));
          if (cst == KMHD_OK) cst = enqueue_coriolis_dev(h, d_rj_in[i], ld_in[i], cols_b[i], d_rj_out[i], ld_out[i]);
          if (cst == KMHD_OK) cst = split_slicer(h->split, h->plan, false, d_rj_in[i], ld_in[i], h->cols_b_d, h->stream);
          ck(cudaEventRecord(bg->ev[2 * i], h->stream));
          ck(cudaStreamWaitEvent(g, bg->ev[2 * i], 0));
        }
        if (cst == KMHD_OK) cst = split_group_gemm(bg->group[k], false, g);
        ck(cudaEventRecord(eg0, g));
        for (int i : grp[k]) {
          kmhd_sph* h = hs[i];
          ck(cudaStreamWaitEvent(h->stream, eg0, 0));
          ck(launch_fft_cycle(h->plan, h->stream));
          if (cst == KMHD_OK) cst = split_slicer(h->split, h->plan, true, nullptr, 0, nullptr, h->stream);
          ck(cudaEventRecord(bg->ev[2 * i + 1], h->stream));
          ck(cudaStreamWaitEvent(g, bg->ev[2 * i + 1], 0));
        }
        if (cst == KMHD_OK) cst = split_group_gemm(bg->group[k], true, g);
        ck(cudaEventRecord(eg1, g));
        for (int i : grp[k]) {
          kmhd_sph* h = hs[i];
          ck(cudaStreamWaitEvent(h->stream, eg1, 0));
          // the dipole (l <= 2) modes again in FP64, as in the single cycle
          ck(launch_leg_fwd_f64(h->plan, d_rj_out[i], ld_out[i], h->cols_f_d, h->stream, std::min(3, h->plan.L + 1)));
          ck(cudaEventRecord(bg->join[i], h->stream));
          ck(cudaStreamWaitEvent(bg->s0, bg->join[i], 0));
        }
      }
      const cudaError_t ec = cudaStreamEndCapture(bg->s0, &graph);
      if (cst == KMHD_OK && ec == cudaSuccess && graph) {
        if (cudaGraphInstantiate(&bg->exec, graph, 0) != cudaSuccess) bg->exec = nullptr;
      }
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();  // clear a failed capture's error state
      bg->sig = sig;
      bg->sig_ld = sig_ld;
      if (!bg->exec) bg->sig.clear();
    }
    if (bg->exec) {
      KCHECK(cudaGraphLaunch(bg->exec, bg->s0));
      KCHECK(cudaStreamSynchronize(bg->s0));
    } else if ((st = batch_direct(hs, n, d_rj_in, ld_in, cols_b, d_rj_out, ld_out))) {
      return st;
    }
  }
  for (int i = 0; i < n; ++i) {
    const int e = check_dev_err(hs[i]);
    if (e != KMHD_OK) return e;
  }
  return KMHD_OK;
}
