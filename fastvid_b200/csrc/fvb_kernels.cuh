// fvb_kernels.cuh -- launch shapes and kernel declarations shared by the
// kernel files and the host orchestration (fvb_api.cu).
#pragma once

#include <type_traits>

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

// ---------------------------------------------------------------------------
// The folded-symbol intermediate (predictor residuals, zigzag-folded, in
// tile-raster order) is held as u32, or as u16 when every frame of a batch
// has a bit depth below 16 or a quality below 100 (fold16).  Then the
// encoder's symbols are below 2^16: at depth <= 15 |q| <= 2^15 - 1, and a
// 16-bit frame below quality 100 has a step of at least 12.  The decoder
// accepts symbols up to 2 * max_sample (decode.cu bounds), which at depth 16
// can exceed 16 bits in a valid stream; such a symbol is stored as 65534 or
// 65535 by parity (fold_store), i.e. a residual of +32767 or -32768 steps,
// which clamps to the same sample as the original since the step is >= 12.
template <typename T>
constexpr int fold_stride() {
  return sizeof(T) == 2 ? kSrcStride : kFoldStride;
}
template <typename T>
using FoldPiece = std::conditional_t<sizeof(T) == 2, uint2, uint4>;  // four symbols

template <typename T>
__device__ __forceinline__ uint32_t ldf(const T* p) {
  return static_cast<uint32_t>(__ldg(p));
}
template <typename T>
__device__ __forceinline__ T fold_store(uint32_t v) {
  if constexpr (sizeof(T) == 2) return static_cast<T>(min(v, 65534u | (v & 1u)));
  else return v;
}
__device__ __forceinline__ uint32_t fold_at(const void* folded, int fold16, int64_t i) {
  return fold16 ? static_cast<uint32_t>(static_cast<const uint16_t*>(folded)[i])
                : static_cast<const uint32_t*>(folded)[i];
}
__device__ __forceinline__ void unpack_piece(const uint4& p, uint32_t (&x)[4]) {
  x[0] = p.x;
  x[1] = p.y;
  x[2] = p.z;
  x[3] = p.w;
}
__device__ __forceinline__ void unpack_piece(const uint2& p, uint32_t (&x)[4]) {
  x[0] = p.x & 0xffffu;
  x[1] = p.x >> 16;
  x[2] = p.y & 0xffffu;
  x[3] = p.y >> 16;
}
__device__ __forceinline__ void cp_async_piece(uint4* smem, const uint4* gmem) { cp_async16(smem, gmem); }
__device__ __forceinline__ void cp_async_piece(uint2* smem, const uint2* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// encoder (counts of pass `pass` from dims); `folded` is u16 when fold16
__global__ void enc_init_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims);
// enc_predict with a wavefront block of `unroll` steps (4, 8, 16, 32)
// and `tile_warps` (1, or 2: a warp pair splits each tile's bands)
void enc_predict_launch(int unroll, int tile_warps, bool fold16, int grid, cudaStream_t stream,
                        const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                        ShardInfo* shards, void* folded, int* queue);
cudaError_t enc_predict_set_smem();
__global__ void enc_predict_wide_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                                        void* folded, uint16_t* recon, int fold16);
void enc_analyze_launch(bool fold16, int grid, cudaStream_t stream, const FrameDesc* frames, FrameState* state,
                        const BatchDims* dims, int pass, ShardInfo* shards, const void* folded,
                        uint8_t* rans_scratch);
// enc_rans with one-stage loads (pipe 0) or a software pipeline over blocks
// of `pipe` (8 or 16) steps
void enc_rans_launch(int pipe, bool fold16, int grid, cudaStream_t stream, const FrameState* state,
                     const BatchDims* dims, int pass, ShardInfo* shards, const void* folded, uint8_t* rans_scratch);
__global__ void enc_scan_kernel(const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                                ShardInfo* shards, uint8_t* prefix);
// Records of one encoder region: pass 0's, or the later pass's (region b,
// indexed like pass 0's for the frames that took part in it).
struct EmitRegion {
  const ShardInfo* shards;
  const void* folded;
  const uint8_t* rans_scratch;
  int64_t count;  // shards 0 .. count-1 have records in this region
};
void enc_emit_launch(bool fold16, int grid, size_t smem, cudaStream_t stream, const FrameState* state,
                     EmitRegion a, EmitRegion b, int64_t total_shards, uint8_t* const* outs);
cudaError_t enc_emit_set_smem(int bytes);
__global__ void enc_prefix_kernel(const FrameDesc* frames, const FrameState* state, int nframes, const uint8_t* prefix,
                                  const uint8_t* prefix_b, uint8_t* const* outs);

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
void dec_rans_launch(bool fold16, int grid, size_t smem, cudaStream_t stream, const FrameDesc* frames,
                     FrameState* state, const ShardInfo* shards, DecodeLists* lists, const int32_t* list_items,
                     const RansTable* tables, void* folded);
cudaError_t dec_rans_set_attr(cudaFuncAttribute attr, int value);
void dec_other_launch(bool fold16, int grid, cudaStream_t stream, const FrameDesc* frames, FrameState* state,
                      const ShardInfo* shards, const BatchDims* dims, DecodeLists* lists, const int32_t* list_items,
                      void* folded);
void dec_reconstruct_launch(int unroll, int tile_warps, bool fold16, int grid, cudaStream_t stream,
                            const FrameDesc* frames, const FrameState* state, const BatchDims* dims,
                            const void* folded, int* queue);
cudaError_t dec_reconstruct_set_smem();
__global__ void dec_reconstruct_wide_kernel(const FrameDesc* frames, const FrameState* state, const BatchDims* dims,
                                            const void* folded, int fold16);
__global__ void dec_reconstruct_serial_kernel(const FrameDesc* frames, const FrameState* state,
                                              const BatchDims* dims, const void* folded, int fold16);

size_t enc_predict_smem(bool fold16);
size_t enc_emit_smem();
size_t dec_reconstruct_smem(bool fold16);
size_t dec_rans_smem();
size_t dec_rans_table_bytes();

}  // namespace fvb
