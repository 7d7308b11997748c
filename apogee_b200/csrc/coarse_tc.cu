// Tensor-core coarse pass: placeholder until the tcgen05 contraction lands.
#include "hier_kernels.cuh"
namespace mfb {
struct TcCoarse { int m; };
static const char *g_tc_err = "tensor-core coarse pass not built";
int tc_coarse_create(TcCoarse **out, int, int, int, int) { *out = nullptr; return -1; }
void tc_coarse_destroy(TcCoarse *) {}
int tc_coarse_pack_templates(TcCoarse *, const float2 *, int, int, cudaStream_t) { return -1; }
int tc_coarse_run(TcCoarse *, const TcRunArgs &, cudaStream_t) { return -1; }
const char *tc_coarse_error() { return g_tc_err; }
}  // namespace mfb
