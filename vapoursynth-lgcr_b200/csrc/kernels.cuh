// Kernel declarations of the Recon path. Every kernel takes
// (jobs, tileStart, njobs): FrameJob array, per-stage block prefix table,
// number of frames in the launch.
#pragma once

#include "recon.cuh"

namespace lgcr_b200 {

#define LGCR_STAGE_ARGS const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs

// k_plain: output rows per block (32 columns wide, 32x8 threads) and the
// most horizontal-table rows one block stages in shared memory.
constexpr int kPlainRows = 64;          // tallest blocks (frames whose windows fit)
constexpr int kPlainRowsShort = 32;     // other frames
constexpr int kPlainStagedRows = 40;
// k_plain's staged rows (float sums, hull float4, luma extrema float2 per
// row and column: 32 B) in dynamic shared memory; with the static row
// tables a block stays under 48 KB, so four blocks per SM keep 60 KB of L1.
constexpr size_t kPlainDynSmem = size_t(kPlainStagedRows) * 32 * (8 + 16 + 8);
// k_detail_map: most horizontal-table rows one block stages.
constexpr int kDetailStagedRows = 40;

// k_convert: samples per warp (one row segment: luma, chroma) and warps per
// block; the luma blocks of a frame come first, then the chroma blocks.
constexpr int kConvertLumaSpan = 512;
constexpr int kConvertSpan = 256;
constexpr int kConvertWarps = 8;
__host__ __device__ __forceinline__ int convertBlocks(int w, int h, int span = kConvertSpan) {
    return (h * ((w + span - 1) / span) + kConvertWarps - 1) / kConvertWarps;
}
__host__ __device__ __forceinline__ int convertLumaBlocks(int sw, int sh) {
    return convertBlocks(sw, sh, kConvertLumaSpan);
}

// k_tensor: columns each warp emits, warps per block (side by side), rows
// per strip.
constexpr int kTensorCols = 28;
constexpr int kTensorWarps = 8;
constexpr int kTensorRows = 32;

// k_dilate_h: widest row in mask words and the zero words on either side
// (the dilation radius must stay below 32 * kDilPadWords).
constexpr int kDilMaxWords = 2048;
constexpr int kDilPadWords = 8;

// k_count: chroma mask bytes per block.
constexpr int kCountChunk = 16384;

// k_mark_chroma: output rows per group of an upscaling frame's guided work
// list. Mask words are taken group by group, and within a group word column
// by word column, the group's rows in turn: consecutive list entries cover a
// few rows of one 32-pixel strip, so the pixels one guided block takes share
// chroma rows (8, 16 and 32 rows measured alike on 1080p -> 4K frames).
constexpr int kListRowGroup = 8;

// k_gate: chroma rows per block (32 columns wide, 32x8 threads, each thread
// takes every eighth row).
constexpr int kGateRows = 16;

__global__ void k_convert(LGCR_STAGE_ARGS);
__global__ void k_tensor(LGCR_STAGE_ARGS);
__global__ void k_dilate_h(LGCR_STAGE_ARGS);
__global__ void k_dilate_v(LGCR_STAGE_ARGS);
__global__ void k_mark_chroma(LGCR_STAGE_ARGS);
__global__ void k_count(LGCR_STAGE_ARGS);
__global__ void k_gate(LGCR_STAGE_ARGS);
__global__ void k_hpass(LGCR_STAGE_ARGS);
__global__ void k_plain(LGCR_STAGE_ARGS);
__global__ void k_plain_all(LGCR_STAGE_ARGS);
__global__ void k_guided(LGCR_STAGE_ARGS);
__global__ void k_guided3(LGCR_STAGE_ARGS);
__global__ void k_guided_staged(LGCR_STAGE_ARGS);
__global__ void k_guided_r(LGCR_STAGE_ARGS);
__global__ void k_guided3_r(LGCR_STAGE_ARGS);
__global__ void k_guided_staged_r(LGCR_STAGE_ARGS);
__global__ void k_guided_o(LGCR_STAGE_ARGS);
__global__ void k_guided3_o(LGCR_STAGE_ARGS);
__global__ void k_guided_staged_o(LGCR_STAGE_ARGS);
// dynamic shared memory of k_guided_staged: 8 warps x 8 x 40 samples of
// lc (4 B) and the (u, v) pair (16 B)
constexpr size_t kGuidedStageBytes = size_t(8) * 8 * 40 * (4 + 16);
__global__ void k_luma_h(LGCR_STAGE_ARGS);
__global__ void k_luma_v(LGCR_STAGE_ARGS);
__global__ void k_luma_radial(LGCR_STAGE_ARGS);
__global__ void k_store_chroma(LGCR_STAGE_ARGS);
// algo 6
__global__ void k_yc_h(LGCR_STAGE_ARGS);
// k_yc_tiled: chroma samples per block side and the most luma rows one
// block reads per candidate.
constexpr int kYcTile = 32;
constexpr int kYcRows = 80;
__global__ void k_yc_tiled(LGCR_STAGE_ARGS);
__global__ void k_affine(LGCR_STAGE_ARGS);
__global__ void k_detail_hpass(LGCR_STAGE_ARGS);
__global__ void k_detail_plain(LGCR_STAGE_ARGS);
__global__ void k_detail_nyq(LGCR_STAGE_ARGS, int pass);
// k_detail_map: output columns per block (32 computed with the halo) and
// output rows per block: tall when the tile's chroma rows fit, else short.
constexpr int kDetailTile = 30;
constexpr int kDetailRowsTall = 62;
__global__ void k_detail_map(LGCR_STAGE_ARGS);
__global__ void k_detail_resize_h(LGCR_STAGE_ARGS);
__global__ void k_detail_resize_v(LGCR_STAGE_ARGS);
__global__ void k_detail_resize_radial(LGCR_STAGE_ARGS);
__global__ void k_detail_transfer(LGCR_STAGE_ARGS);
__global__ void k_detail_transfer_list(LGCR_STAGE_ARGS);
__global__ void k_affine_list(LGCR_STAGE_ARGS);
// algo 4
__global__ void k_lgf(LGCR_STAGE_ARGS);
__global__ void k_roi(LGCR_STAGE_ARGS);
__global__ void k_blend(LGCR_STAGE_ARGS);
// bm / bp
__global__ void k_bm_guide(LGCR_STAGE_ARGS);
__global__ void k_bm_group(LGCR_STAGE_ARGS);
__global__ void k_bm_aggregate(LGCR_STAGE_ARGS);
__global__ void k_backproject(LGCR_STAGE_ARGS);

// Tile helper of the per-pixel stages: the block shape (chosen by the
// autotuner for the tunable stages) is the tile shape.
__device__ __forceinline__ void tile32x8(int tile, int width, int &x, int &y) {
    const int tilesX = (width + blockDim.x - 1) / blockDim.x;
    x = (tile % tilesX) * blockDim.x + threadIdx.x;
    y = (tile / tilesX) * blockDim.y + threadIdx.y;
}

} // namespace lgcr_b200
