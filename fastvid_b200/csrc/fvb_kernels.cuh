// fvb_kernels.cuh -- launch shapes and kernel declarations shared by the
// kernel files and the host orchestration (fvb_api.cu).
#pragma once

#include "fvb_common.cuh"

namespace fvb {

constexpr int kWarpsPerCta = 4;    // warps per CTA of the warp-per-item kernels
constexpr int kSrcStride = 66;     // u16 ring row stride: 64 columns + 2 (33 words: conflict-free)
constexpr int kFoldStride = 65;    // u32 ring row stride: 64 columns + 1 (conflict-free)
constexpr int kFastMaxW = 512;     // widest tile of the register-wavefront path
constexpr int kDefaultWavefrontBlock = 8;  // steps of a 32-step wavefront block unrolled (4, 8, 16, 32)
constexpr int kDefaultTileWarps = 1;       // warps per tile of the wavefront kernels (1 or 2)

// Whether a warp pair splits a tile's bands (the predictor and the
// reconstruction alike): at least two bands, and at least four wavefront
// blocks per band -- the second warp runs two blocks behind the first, and
// the band below needs the band above's last row up to one block ahead of
// it, which the schedule provides once a band has four blocks.
__host__ __device__ inline bool pair_splits(int w, int h) { return ((h + 31) >> 5) >= 2 && ((w + 62) >> 5) >= 4; }

// encoder (counts of pass `pass` from dims)
__global__ void enc_init_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims);
// enc_predict with a wavefront block of `unroll` steps (4, 8, 16, 32)
// and `tile_warps` (1, or 2: a warp pair splits each tile's bands)
void enc_predict_launch(int unroll, int tile_warps, int grid, cudaStream_t stream, const FrameDesc* frames,
                        FrameState* state, const BatchDims* dims, int pass, ShardInfo* shards, uint32_t* folded,
                        int* queue);
cudaError_t enc_predict_set_smem();
__global__ void enc_predict_wide_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                                        uint32_t* folded, uint16_t* recon);
__global__ void enc_analyze_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                                   ShardInfo* shards, const uint32_t* folded, uint8_t* rans_scratch);
// enc_rans with one-stage loads (pipe 0) or a software pipeline over blocks
// of `pipe` (8 or 16) steps
void enc_rans_launch(int pipe, int grid, cudaStream_t stream, const FrameState* state, const BatchDims* dims,
                     int pass, ShardInfo* shards, const uint32_t* folded, uint8_t* rans_scratch);
__global__ void enc_scan_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                                ShardInfo* shards, uint8_t* prefix);
__global__ void enc_emit_kernel(const FrameDesc* frames, int nframes, const ShardInfo* shards,
                                int64_t total_shards, const uint32_t* folded, const uint8_t* rans_scratch,
                                uint8_t* const* outs);
__global__ void enc_prefix_kernel(const FrameDesc* frames, int nframes, const uint8_t* prefix,
                                  uint8_t* const* outs);

// decoder: shards binned by mode (0 rANS, 1 Rice, 2 zero-run, 3 block pack);
// counts from dims (entry 0)
struct DecodeLists {
  int32_t count[4];
  int32_t next_group;       // dec_other work counter
  int32_t next_group_rans;  // dec_rans work counter
  int32_t pad[2];
};
struct RansTable;
__global__ void dec_parse_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims,
                                 ShardInfo* shards, DecodeLists* lists, int32_t* list_items);
__global__ void dec_rans_tables_kernel(const FrameDesc* frames, FrameState* state, const ShardInfo* shards,
                                       const DecodeLists* lists, const int32_t* list_items, RansTable* tables);
__global__ void dec_rans_kernel(const FrameDesc* frames, FrameState* state, const ShardInfo* shards,
                                DecodeLists* lists, const int32_t* list_items, const RansTable* tables,
                                uint32_t* folded);
__global__ void dec_other_kernel(const FrameDesc* frames, FrameState* state, const ShardInfo* shards,
                                 const BatchDims* dims, DecodeLists* lists, const int32_t* list_items,
                                 uint32_t* folded);
void dec_reconstruct_launch(int unroll, int tile_warps, int grid, cudaStream_t stream, const FrameDesc* frames,
                            const FrameState* state, const BatchDims* dims, const uint32_t* folded, int* queue);
cudaError_t dec_reconstruct_set_smem();
__global__ void dec_reconstruct_wide_kernel(const FrameDesc* frames, const FrameState* state, const BatchDims* dims,
                                            const uint32_t* folded);
__global__ void dec_reconstruct_serial_kernel(const FrameDesc* frames, const FrameState* state,
                                              const BatchDims* dims, const uint32_t* folded);

size_t enc_predict_smem();
size_t enc_emit_smem();
size_t dec_reconstruct_smem();
size_t dec_rans_smem();
size_t dec_rans_table_bytes();

}  // namespace fvb
