// kmhd_split.cuh -- split-precision (Ozaki-style INT8 slice) Legendre tiers on tcgen05.
#pragma once
#include <vector>

#include "kmhd_internal.cuh"

namespace kmhd {

struct SplitState;

int split_create(SplitState** s, const Plan& p, int tier, int nslice, cudaStream_t st);
void split_destroy(SplitState* s);
int64_t split_bytes(const SplitState* s);
// `mid` (optional) is recorded on st between the slicer and the GEMM launch.
int split_bwd(SplitState* s, const Plan& p, int nlc_max, const double* d_rj, long long ld,
              const int* cols, cudaStream_t st, cudaEvent_t mid = nullptr);
int split_fwd(SplitState* s, const Plan& p, double* d_rj, long long ld, const int* cols,
              cudaStream_t st, cudaEvent_t mid = nullptr);
// The two halves of split_bwd / split_fwd: the slicer alone.
int split_slicer(SplitState* s, const Plan& p, bool fwd, const double* d_rj, long long ld, const int* cols,
                 cudaStream_t st);
int split_ns(const SplitState* s);
// Highest digit-pair group T kept by the GEMMs (slice products a + b <= T of
// the ns x ns digit pairs): the tier's full T (6 split, 3 fp32acc) or one less.
int split_terms(const SplitState* s);
int split_set_terms(SplitState* s, int T);
int split_products(int ns, int T);
// Grouped GEMM over n instances of one split tier (one persistent launch per
// direction over every instance's pair units; d_rj_out / ld_out / cols_f are
// the forward outputs, device pointers).  The arguments are copied to the
// device at creation, so the group is tied to those pointers.
struct SplitGroup;
int split_group_create(SplitGroup** g, SplitState* const* ss, const Plan* plans, int n, double* const* d_rj_out,
                       const long long* ld_out, const int* const* cols_f, cudaStream_t st);
int split_group_gemm(SplitGroup* g, bool fwd, cudaStream_t st);
void split_group_destroy(SplitGroup* g);
// Radial chunks for windowed launches: bounds[0] = 0 < bounds[1] < ... =
// p.nr, every bound but the last a multiple of 16.  split_bwd / split_fwd on a
// plan whose window [r_lo, r_hi) is one chunk run only that chunk's tiles.
int split_set_chunks(SplitState* s, const Plan& p, const std::vector<int>& bounds, cudaStream_t st);
// Reads and returns the device error word (KMHD_OK or KMHD_ERR_TIMEOUT); synchronises st.
int split_check_error(SplitState* s, cudaStream_t st);

}  // namespace kmhd

int batch_cycle_impl(kmhd_sph** hs, int32_t n, const double* const* d_rj_in, const int64_t* ld_in,
                     const int32_t* const* cols_b, double* const* d_rj_out, const int64_t* ld_out,
                     const int32_t* const* cols_f);
