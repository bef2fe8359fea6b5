// Chunked line-solve launch interface (linesolve_chunk.cu).
#pragma once

#include "x3d_internal.h"

namespace x3d {

constexpr int kMaxChunkOps = 6;

// Up to six operators applied to the same input field along one direction:
// one staged read of the field, one write per operator.
template <typename T>
struct ChunkOps {
    LineOp<T> op[kMaxChunkOps];
    T *out[kMaxChunkOps];
    int kind[kMaxChunkOps];
    int nops;
};

// Number of (lines per CTA, chunk length) configurations launch_chunk knows.
constexpr int kChunkConfigs = 4;

// Launches the chunked kernel with configuration cfg in [0, kChunkConfigs).
// Returns X3D_EUNSUPPORTED (nothing launched) when the shape, alignment or
// shared-memory budget rules that configuration out.
template <typename T>
int launch_chunk(x3d_ctx_s *ctx, const ChunkOps<T> &ops, int dir, const T *in, int nx, int ny,
                 int nz, int cfg);

}  // namespace x3d
