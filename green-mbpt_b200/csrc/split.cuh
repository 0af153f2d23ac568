// Split-precision (Ozaki-sliced INT8 tensor-core) contractions.
#pragma once

#include <vector>

#include "context.cuh"

namespace gb200 {

struct SplitEngine;

// The engine of a context (created on first use).
SplitEngine* split_engine(Context& c);
// C = alpha op(A) op(B) + beta C with both operands sliced into INT8 pieces,
// products on the tensor cores with exact INT32 accumulation, FP64 recombination;
// `slices` pieces per operand (0: the context's count).
void split_gemm(Context& c, SplitEngine& se, const ZGemm& g, cudaStream_t st, int slices = 0);
// The same for one contraction of each of several contexts (distinct contexts, all in split
// precision with `slices` pieces): every context slices its operands into its own buffers and one
// persistent tensor-core launch per K chunk walks the tiles of all of them.
void split_gemm_group(const std::vector<Context*>& cs, const std::vector<ZGemm>& gs, cudaStream_t st, int slices);
void split_release(Context& c);
// Longest K range one split launch takes without chunking (a contraction with an exponent sink
// must fit it).
int64_t split_max_chunk(int slices);
// Non-zero if a split kernel hit a bounded-wait timeout since the last check (flag is cleared).
int split_check_error(Context& c, cudaStream_t st);

}  // namespace gb200
