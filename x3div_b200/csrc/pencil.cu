// Block copies between strided 3-D arrays: the packing and unpacking of the
// pencil transposes over a p_row x p_col process grid (2decomp's
// transpose_x_to_y / y_to_x / y_to_z / z_to_y, called by
// src/x3d_transpose.f90:16-130).  A transpose sends each member of its row
// or column group one block of the rank's pencil, packed back to back into
// the send buffer, and places the blocks it receives into its new pencil:
// both steps are one launch over a list of blocks.
//
// Each block is a box of nz planes x ny rows x nx elements with its own
// offsets and y/z strides in the source and the destination.  The copy runs
// in 16-byte units where every offset, stride and row of the launch allows
// it (FP32 rows of a multiple of 4 elements, FP64 of 2, complex FP64
// always), else in 4-byte words; consecutive threads take consecutive units
// of a row, so both sides are coalesced along x.
#include <cstring>

#include "x3d_internal.h"

namespace x3d {

constexpr int kCopyBlocksPerLaunch = 32;

struct CopyUnitBlock {
    long long src, dst;       // offsets in units
    long long ssy, ssz;       // source strides in units
    long long dsy, dsz;       // destination strides in units
    long long row_units;      // units per row
    long long rows;           // ny * nz
    int ny;
};

struct CopyLaunch {
    CopyUnitBlock b[kCopyBlocksPerLaunch];
};

template <typename U>
__global__ void __launch_bounds__(256) k_copy_blocks(const __grid_constant__ CopyLaunch p, U *dst, const U *src)
{
    const CopyUnitBlock &b = p.b[blockIdx.y];
    const long long total = b.row_units * b.rows;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += step) {
        const long long row = i / b.row_units, x = i - row * b.row_units;
        const long long z = row / b.ny, y = row - z * b.ny;
        dst[b.dst + z * b.dsz + y * b.dsy + x] = src[b.src + z * b.ssz + y * b.ssy + x];
    }
}

int copy_blocks(x3d_ctx_s *ctx, void *dst, const void *src, int elem_bytes, const x3d_block *blocks, int count)
{
    if (count == 0) return X3D_OK;
    bool vec = (reinterpret_cast<uintptr_t>(dst) % 16 == 0) && (reinterpret_cast<uintptr_t>(src) % 16 == 0);
    for (int i = 0; i < count && vec; ++i) {
        const x3d_block &b = blocks[i];
        const long long eb = elem_bytes;
        for (long long v : {b.src_offset, b.dst_offset, (long long)b.nx, b.src_ystride, b.src_zstride, b.dst_ystride,
                            b.dst_zstride})
            if ((v * eb) % 16) vec = false;
    }
    const int ub = vec ? 16 : 4;  // elem_bytes is 4, 8 or 16; with vec every byte count divides by 16
    auto units = [&](long long elems) { return elems * elem_bytes / ub; };
    for (int first = 0; first < count; first += kCopyBlocksPerLaunch) {
        const int n = std::min(kCopyBlocksPerLaunch, count - first);
        CopyLaunch p;
        std::memset(&p, 0, sizeof(p));
        long long most = 0;
        for (int i = 0; i < n; ++i) {
            const x3d_block &b = blocks[first + i];
            CopyUnitBlock &u = p.b[i];
            u.src = units(b.src_offset);
            u.dst = units(b.dst_offset);
            u.ssy = units(b.src_ystride);
            u.ssz = units(b.src_zstride);
            u.dsy = units(b.dst_ystride);
            u.dsz = units(b.dst_zstride);
            u.row_units = units(b.nx);
            u.rows = (long long)b.ny * b.nz;
            u.ny = b.ny;
            most = std::max(most, u.row_units * u.rows);
        }
        // enough CTAs for the largest block, at most 8 per SM over the launch
        long long gx = (most + 255) / 256;
        const long long cap = std::max<long long>(1, (long long)ctx->num_sms * 8 / n);
        gx = std::max<long long>(1, std::min(gx, cap));
        const dim3 grid((unsigned)gx, (unsigned)n);
        ++ctx->launches;
        if (vec)
            k_copy_blocks<uint4><<<grid, 256, 0, ctx->stream>>>(p, static_cast<uint4 *>(dst),
                                                                static_cast<const uint4 *>(src));
        else
            k_copy_blocks<unsigned><<<grid, 256, 0, ctx->stream>>>(p, static_cast<unsigned *>(dst),
                                                                   static_cast<const unsigned *>(src));
        const int rc = cuda_check(ctx, cudaGetLastError(), "k_copy_blocks launch");
        if (rc) return rc;
    }
    return X3D_OK;
}

}  // namespace x3d
