// kmhd_split.cu -- split-precision tiers (placeholder until the tcgen05 kernels land).
#include "kmhd_split.cuh"

namespace kmhd {
struct SplitState { int tier; };
int split_create(SplitState** s, const Plan&, int, int, cudaStream_t) { *s = nullptr; return KMHD_ERR_SIZE; }
void split_destroy(SplitState* s) { delete s; }
int64_t split_bytes(const SplitState*) { return 0; }
int split_bwd(SplitState*, const Plan&, int, const double*, long long, const int*, cudaStream_t) { return KMHD_ERR_STATE; }
int split_fwd(SplitState*, const Plan&, double*, long long, const int*, cudaStream_t) { return KMHD_ERR_STATE; }
}  // namespace kmhd
