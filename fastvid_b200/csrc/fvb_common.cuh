// fvb_common.cuh -- shared constants, frame geometry and helpers for the
// sm_100a fastvid kernels.
//
// Bitstream constants follow the reference format (cuda/csrc/encode.cu:14-28,
// cuda/csrc/decode.cu:12-21): 32-byte header, 32-byte directory entry per tile,
// 4096-symbol shards, 128-symbol pack blocks, Rice k <= 16, order-0 rANS with
// 12-bit tables and 2^23 lower bound.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fvb {

constexpr int kHeaderBytes = 32;
constexpr int kDirBytes = 32;
constexpr int kShardSymbols = 4096;
constexpr int kBlockSymbols = 128;
constexpr int kMaxRice = 16;
constexpr int kModeZeroRun = 0;
constexpr int kModeRiceBase = 1;
constexpr int kModeBlockPack = 18;
constexpr int kModeOrder0 = 19;  // also the directory's entropy tag
constexpr int kRansAlphabet = 511;
constexpr int kRansTableLog = 12;
constexpr uint32_t kRansL = 1u << 23;
constexpr int kPredictTag = 6;
constexpr int kMaxTiles = 1 << 20;

// Largest shard record: the competition never picks a body above the block
// pack cost (<= 32 width bytes + 4096*17/8), forced rANS stays below that too.
constexpr int kMaxRecordBytes = 3 + 32 + (kShardSymbols * 17 + 7) / 8;

// rANS scratch per shard (encoder): symbol table for the 511 symbols (two
// words each: freq<<16|cum and floor(2^32/freq)), the serialised table, and
// four byte lanes written back to front.
constexpr int kRansTableWords = 1024;
constexpr int kRansSerialBytes = 1024;
constexpr int kRansLaneBytes = 1792;  // >= 1024 symbols * 12 bits / 8 + 1
constexpr int kRansScratchBytes = kRansTableWords * 4 + kRansSerialBytes + 4 * kRansLaneBytes;

// Status codes: the reference's device codes are kept (encode.cu:124-126,
// decode.cu:127-129): encoder 1 = sample above max, 2 = body > 65535;
// decoder 1 zero-run, 2 Rice, 3 block pack, 4 unknown mode, 5 rANS,
// 10 directory, 11 shard header.  Codes >= 100 are internal consistency
// failures of this implementation (never expected).
constexpr int kStatusInternal = 100;

// ---------------------------------------------------------------------------
// Frame description shared by host and device.  All tile/shard/sample indices
// are frame-local; *_base fields place the frame inside a batch.
struct FrameDesc {
  int32_t layout, bit_depth, quality, planes;
  int32_t width, height, tile_w, tile_h;
  int32_t plane_w[3];   // plane widths (chroma halved for yuv422)
  int32_t ptile_w[3];   // nominal tile width in each plane
  int32_t tiles_x[3];   // tiles per tile row in each plane
  int32_t tiles_y;      // tile rows
  int32_t last_h;       // height of the last tile row
  int32_t max_sample;   // 2^depth - 1
  int32_t step0;        // quality step before any frame policy
  int32_t force_order0; // rgb444 && (depth != 10 || width < 3840)
  int32_t use_med0;     // predictor of the first encode pass / of the decode
  int64_t tile0[4];     // first tile of each plane; tile0[planes] = ntiles
  int64_t shard0[4];    // first shard of each plane
  int64_t sample0[4];   // first sample of each plane
  int64_t shards_row[3];      // shards in one full-height tile row
  int32_t shards_int[3][2];   // shards of an interior tile [plane][last row?]
  int32_t shards_last[3][2];  // shards of a last-column tile
  int64_t ntiles, nshards, nsamples;
  int64_t tile_base, shard_base, sample_base;  // placement in the batch arrays
  int64_t prefix_base;   // byte offset of this frame's header+directory in prefix scratch
  int64_t prefix_bytes;  // 32 + 32 * ntiles
  int32_t slot;          // the frame's index in the caller's batch (results, outputs)
  int32_t pad_slot;
  // I/O
  const uint16_t* src[3];
  int64_t src_pitch[3];  // elements
  uint16_t* dst[3];
  int64_t dst_pitch[3];
  const uint8_t* stream;
  int64_t stream_len;
  uint32_t fps_num, fps_den;
};

// Counts of the work of one batch, read by the kernels from device memory
// (written with the frame table), so that a launch sequence captured for a
// bucket of batch sizes -- grids sized for the bucket's capacity -- serves
// any batch that fits it.  frames_p / tiles_p / shards_p: the frames, tiles
// and shards that take part in encoder pass p (the batch is laid out with
// frames of more passes first, so these are prefixes); entry 0 counts the
// whole batch (decode uses entry 0 only).
struct BatchDims {
  int32_t frames_p[3];
  int32_t passes;
  int64_t tiles_p[3];
  int64_t shards_p[3];
  int64_t samples;
};

// Per-frame mutable state (device), one per frame of a batch.
struct FrameState {
  int32_t step;        // step of the current pass
  int32_t use_med;     // predictor of the current pass
  int32_t active;      // current pass runs for this frame
  int32_t gray_med;    // header flag 0x40
  int32_t refined;     // header flag 0x80
  int32_t status;      // first error code
  int32_t pass;        // policy stage
  int32_t final_b;     // the frame's records are those of the later pass (region b)
  int64_t payload;     // sum of record bytes of the last completed pass
  int64_t baseline_payload;
  int64_t stream_len;  // header + directory + records
};

// Per-shard record shared by the encode and decode kernels.
struct ShardInfo {
  int64_t sample_base;   // global folded index of the first symbol
  int64_t offset;        // encode: byte offset of the record in the stream; decode: body offset
  int32_t count;         // symbols
  int32_t frame;         // frame index in the batch
  int32_t mode;          // chosen mode (encode) / parsed mode (decode)
  int32_t param;         // Rice k
  int32_t body;          // body bytes
  int32_t comp_mode;     // encode: competition winner
  int32_t comp_k;
  int32_t comp_body;
  int32_t comp_lane[4];  // encode: Rice lane bytes of the competition winner
  int32_t rans_ok;       // encode: shard is rANS eligible
  int32_t rans_table;    // encode: serialised table bytes
  int32_t rans_lane[4];  // encode: rANS lane bytes
  uint32_t rans_state[4];
};

// Tile placement computed arithmetically from the frame geometry, so no tile
// table ever has to be uploaded (the reference uploads tile_meta per call,
// encode.cu:739-767).
struct TileGeo {
  int32_t plane, x, y, w, h;
  int64_t sample_base;   // frame-local folded index of the tile's first sample
  int64_t first_shard;   // frame-local
  int32_t shard_count;
};

__host__ __device__ inline TileGeo tile_geo(const FrameDesc& f, int64_t t) {
  TileGeo g;
  int p = 0;
  if (f.planes == 3) p = (t >= f.tile0[1]) + (t >= f.tile0[2]);
  const int64_t lt = t - f.tile0[p];
  const int32_t ty = static_cast<int32_t>(lt / f.tiles_x[p]);
  const int32_t tx = static_cast<int32_t>(lt - static_cast<int64_t>(ty) * f.tiles_x[p]);
  const int last_row = ty == f.tiles_y - 1;
  const int last_col = tx == f.tiles_x[p] - 1;
  g.plane = p;
  g.x = tx * f.ptile_w[p];
  g.y = ty * f.tile_h;
  g.w = last_col ? f.plane_w[p] - g.x : f.ptile_w[p];
  g.h = last_row ? f.last_h : f.tile_h;
  g.sample_base = f.sample0[p] + static_cast<int64_t>(ty) * f.tile_h * f.plane_w[p] +
                  static_cast<int64_t>(tx) * f.ptile_w[p] * g.h;
  g.first_shard = f.shard0[p] + static_cast<int64_t>(ty) * f.shards_row[p] +
                  static_cast<int64_t>(tx) * f.shards_int[p][last_row];
  g.shard_count = last_col ? f.shards_last[p][last_row] : f.shards_int[p][last_row];
  return g;
}

// Locate the frame of a global index (frames sorted by base); n is small.
__device__ inline int find_frame(const int64_t* bases, int n, int64_t idx) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bases[mid] <= idx) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ inline void set_status(int32_t* status, int32_t code) { atomicCAS(status, 0, code); }

// Asynchronous global -> shared copies (cp.async, sm_80+), completed per
// thread with commit/wait groups.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ int varint_len(uint32_t v) {
  return v < (1u << 7) ? 1 : v < (1u << 14) ? 2 : v < (1u << 21) ? 3 : v < (1u << 28) ? 4 : 5;
}

__device__ __forceinline__ uint32_t zigzag(int32_t v) {
  return (static_cast<uint32_t>(v) << 1) ^ static_cast<uint32_t>(v >> 31);
}

__device__ __forceinline__ int32_t unzigzag(uint32_t v) {
  return static_cast<int32_t>(v >> 1) ^ -static_cast<int32_t>(v & 1);
}

// Median edge detector written as a median of three: min(L,A) <= MED <= max(L,A)
// and MED = L + A - UL when UL lies between them (encode.cu:169-177).
__device__ __forceinline__ int32_t predict_med(int32_t l, int32_t a, int32_t ul) {
  const int32_t mn = min(l, a), mx = max(l, a);
  return max(mn, min(mx, l + a - ul));
}

__device__ __forceinline__ int32_t predict_grad(int32_t l, int32_t a, int32_t ul, int32_t max_sample) {
  return max(0, min(max_sample, l + a - ul));
}

}  // namespace fvb
