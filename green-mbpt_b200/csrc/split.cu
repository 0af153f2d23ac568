// Split-precision contractions (filled in by the Ozaki INT8 engine).
#include "split.cuh"

namespace gb200 {

struct SplitEngine {};

SplitEngine* split_engine(Context&) { throw Error(GB200_ERR_INVALID, "split precision not built"); }
void split_prepare_integrals(Context&, SplitEngine&, cudaStream_t) {}
void split_gemm(Context&, SplitEngine&, const ZGemm&, cudaStream_t) {
  throw Error(GB200_ERR_INVALID, "split precision not built");
}
void split_invalidate(Context&) {}
void split_release(Context&) {}

}  // namespace gb200
