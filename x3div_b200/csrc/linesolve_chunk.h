// Chunked line-solve stage kernels (linesolve_chunk.cu).
#pragma once

#include <cuda.h>

#include "x3d_internal.h"

namespace x3d {

constexpr int kMaxStageOps = 6;
constexpr int kMaxStageTiles = 3;

// One operator application inside a stage.  Its input is staged tile src_a,
// or the pointwise product of tiles src_a and src_b.  The solved values x
// update a register accumulator: acc = m x (accumulate = 0) or acc += m x,
// with m = 1 or m = tile[mul_tile] at the same point.  With flush set the
// accumulator is written out:  out = base + sign * acc  (base may be null,
// and may alias out), then optionally  out2 = base2 + scale2 * out.
template <typename T>
struct StageOp {
    LineOp<T> op;
    void *out;
    const void *base;
    void *out2;
    const void *base2;
    double sign, scale2;
    int kind;
    short src_a, src_b;
    short mul_tile;
    short accumulate;
    short flush;
    short out_f64;  // out, base, out2, base2 hold double rather than T
    // Set by launch_stage: base2 is staged input tile base2_tile (-1: read
    // from global memory); prefetch_base: base (or, without one, a base2
    // read from global memory) is prefetched into L2 when
    // the tile's inputs are requested.
    short base2_tile;
    short prefetch_base;
    // Set by launch_stage: the response entries the fixes of a full chunk
    // use (see chunk_solve_resp).
    int keep;
    // Responses of a chunk's solved values to its carries, for the launch's
    // chunk length L (set by launch_stage): y_j = y_j(local) + F resp[0][j]
    // + B resp[1][j] for a full chunk, resp[2], resp[3] for a short last
    // chunk, F and B the forward and backward carries (see chunk_solve_resp).
    T resp[4][kChunkLong<T>];
};

// Up to six operators along one direction over up to three staged inputs of
// one (nx, ny, nz) grid: one read of each input, the writes the flushes ask for.
template <typename T>
struct StageProgram {
    StageOp<T> ops[kMaxStageOps];
    const T *in[kMaxStageTiles];
    int nops, ntiles;
    int prefetch_mask;  // bit k: operator k's base is prefetched (set by launch_stage)
    int in_f64;         // T = float: in[] hold FP64 fields (y/z plain programs only)
};

// Number of (lines per CTA, chunk length, persistence, lines per thread)
// configurations launch_stage knows in 0 .. 15; 16 is the one-thread-per-line
// kernel (not a launch_stage configuration); 17, 18, 19 and 20 are
// configurations 6, 9, 3 and 0 compiled for three CTAs per SM (plain
// programs).
// kAllConfigs counts every configuration the
// dispatch tries.
constexpr int kChunkConfigs = 16;
constexpr int kAllConfigs = 21;
inline bool is_stage_cfg(int cfg) { return cfg >= 0 && cfg < kAllConfigs && cfg != kChunkConfigs; }

// Launches the chunked stage kernel with configuration cfg (is_stage_cfg).  Returns X3D_EUNSUPPORTED, launching nothing, when the
// shape, alignment or shared-memory budget rules that configuration out.
template <typename T>
int launch_stage(x3d_ctx_s *ctx, const StageProgram<T> &prog, int dir, int nx, int ny, int nz,
                 int cfg);

// One job of a box batch: up to six operators applied along one direction to
// one field of one box.  Filled on the host, read by the persistent batch
// kernel from device memory (the tensor map first, for its 64-byte alignment).
constexpr int kBatchThreads = 256;

template <typename T>
struct BatchJob {
    CUtensorMap tmap;  // y/z input map
    const T *in;
    T *out[kMaxStageOps];
    LineOp<T> op[kMaxStageOps];
    int kind[kMaxStageOps];
    int nops, dir, n, nx, ny, nz;
    int L;       // chunk length (kChunkLong or kChunkShort of T)
    int rclass;  // jobs with equal rclass have equal responses (same operators, line length and L)
    int xstage;  // x jobs: outputs staged in shared-memory rows, bulk row copies
    int W, C, box_n, nbox, pitch;
    int halo;    // y/z: staged rows in front of the line (periodic halo + alignment)
    long span;   // x: number of lines; y/z: tiles across x
    long tile0;  // first work item of the job
    long ntiles;
    // the entries of each operator's responses the fixes use (as
    // StageOp::keep; set by plan_batch_job)
    int keep[kMaxStageOps];
    // carry responses of each operator for the job's chunk length (as
    // StageOp::resp).  Everything before them is the job's header, which the
    // kernel copies to shared memory once per work item.
    T resp[kMaxStageOps][4][kChunkLong<T>];
};

// Chooses tiling for the job (chunk length L, kChunkLong or kChunkShort of
// T; at most w_req lines per tile when w_req > 0, else as many as the
// threads allow; x outputs staged in shared memory when xstage) and encodes
// its tensor map; false when the batch kernel cannot take the job.
template <typename T>
bool plan_batch_job(BatchJob<T> &J, int L, int w_req, int xstage, size_t *tile_bytes);

// Variants of the batch kernel: every job on the long chunk with x outputs
// straight out; each job's own chunk length; and x outputs staged in shared
// memory where a job sets xstage.  batch_variant picks the narrowest one a
// host job list needs.
enum BatchVariant { kBatchLong = 0, kBatchMixed = 1, kBatchStaged = 2 };
template <typename T>
int batch_variant(const BatchJob<T> *jobs, int njobs);

// Sets the shared-memory attribute of the batch kernel's variant for tiles
// up to tile_cap bytes and returns the persistent grid (SMs x resident CTAs
// per SM).
template <typename T>
int prepare_batch(size_t tile_cap, int variant, size_t smem_optin, int num_sms, int *grid);

// One persistent launch over every tile of every job (jobs and counter in
// device memory; the counter is reset by the launch itself, so the pair of
// operations can be captured in a CUDA graph and replayed).
template <typename T>
int launch_batch(cudaStream_t st, int grid, const BatchJob<T> *d_jobs, int njobs, long total,
                 unsigned long long *d_counter, size_t tile_cap, int variant, int *d_err);

// A plain program: operator k reads input 0 and writes out[k].
template <typename T>
StageProgram<T> plain_program(const T *in, const LineOp<T> *const *ops, const int *kinds,
                              void *const *outs, int nops);

}  // namespace x3d
