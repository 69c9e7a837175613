// fvb_encode.cu -- sm_100a encoder kernels for the fastvid intra codec.
//
// Pipeline (one launch each, all frames of a batch at once):
//   enc_predict  : warp-per-tile register wavefront: predictor + quantizer +
//                  reconstruction + zigzag (reference encode.cu:128-193)
//   enc_analyze  : warp-per-shard cost model: Rice k search, zero-run, block
//                  pack, rANS histogram + 12-bit normalisation + table bytes
//                  (encode.cu:195-317, 319-392)
//   enc_rans     : thread-per-lane interleaved rANS (encode.cu:398-418)
//   enc_scan     : CTA-per-frame mode choice, record offsets, directory,
//                  header and the gray10/gray16 frame policy
//                  (encode.cu:420-430, 812-904)
//   enc_emit     : warp-per-shard record assembly in shared memory and one
//                  aligned copy-out (encode.cu:488-682)
// Nothing here traps; every failure is a status word.
#include "fvb_common.cuh"
#include "fvb_kernels.cuh"

namespace fvb {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int frame_of_tile(const FrameDesc* frames, int nframes, int64_t t) {
  int lo = 0, hi = nframes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (frames[mid].tile_base <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Division of n < 2^17 by a quantizer step 2..8191 with one multiply-high:
// m = ceil(2^32 / step) (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994).  With e = m*step - 2^32 < step,
// floor(n*m / 2^32) = floor(n / step) whenever n*e < 2^32, which holds for
// n < 2^17 and step < 2^13.  The host computes m (fvb_api.cu).
__device__ __forceinline__ int32_t div_step(uint32_t n, uint32_t magic) {
  return static_cast<int32_t>(__umulhi(n, magic));
}

// ---------------------------------------------------------------------------
// enc_predict

// Warp-per-tile register wavefront over 32-row bands.  Lane i holds row i of
// the band and processes column c = t - i at step t, so its left and
// upper-left neighbours are its own previous values and its upper neighbour
// is lane i-1's previous reconstruction (one shuffle); lane 0 reads the row
// above the band from the carry row written by lane 31 of the previous band.
// Source and output stream through two 64-column shared-memory rings in a
// skewed layout -- row r keeps column c at position (c + r) & 63 -- so at
// step t every lane touches position t & 63: one uniform offset, folded into
// the instruction's immediate inside each unrolled 32-step block.  Blocks in
// which every lane's column lies inside the tile run without predicates.

template <typename FoldT>
struct EncWarpSmem {
  static constexpr int kFS = fold_stride<FoldT>();
  uint16_t src[32 * kSrcStride];    // source ring (u16, skewed)
  FoldT fold[32 * kFS];             // folded-residual ring (skewed)
  uint16_t carry[kFastMaxW + 128];  // row above the band, column c at index c + 32
};

template <bool MED, bool STEP1, bool EDGE, int UNROLL, bool SPLIT, typename FoldT>
__device__ __forceinline__ void enc_block(EncWarpSmem<FoldT>& sm, const uint16_t* carry_in, uint16_t* carry_out, int lane,
                                          int t0, int W, int32_t maxs, int32_t step, int32_t half, uint32_t magic,
                                          bool band0, int32_t& rec, int32_t& a_prev) {
  const uint16_t* srow = sm.src + lane * kSrcStride + (t0 & 32);
  FoldT* frow = sm.fold + lane * EncWarpSmem<FoldT>::kFS + (t0 & 32);
  const uint16_t* crow_in = carry_in + 32 - lane + t0;  // lane 0: column t0 + u
  // one warp per tile reads and writes the same row: one pointer
  uint16_t* crow_out = SPLIT ? carry_out + 32 - lane + t0 : const_cast<uint16_t*>(crow_in);      // lane 31: column t0 + u - 31 (index (t - lane) + 32)
#pragma unroll UNROLL
  for (int u = 0; u < 32; ++u) {
    const int32_t s = srow[u];
    int32_t a = __shfl_up_sync(0xffffffffu, rec, 1);
    const int32_t above0 = crow_in[u];
    if (lane == 0) a = band0 ? 0 : above0;
    const int32_t pred = MED ? predict_med(rec, a, a_prev) : predict_grad(rec, a, a_prev, maxs);
    const int32_t res = s - pred;
    int32_t q, rn;
    if (STEP1) {
      q = res;
      rn = min(s, maxs);
    } else {
      const int32_t mag = static_cast<int32_t>(__umulhi(static_cast<uint32_t>(abs(res) + half), magic));
      q = res < 0 ? -mag : mag;
      rn = max(0, min(maxs, pred + q * step));
    }
    if (EDGE) {
      const int c = t0 + u - lane;
      if (c < 0) rn = 0;  // left of the tile: zero left/upper-left for column 0
      if (lane == 31 && c >= 0 && c < W) crow_out[u] = static_cast<uint16_t>(rn);
    } else {
      if (lane == 31) crow_out[u] = static_cast<uint16_t>(rn);
    }
    frow[u] = static_cast<FoldT>(zigzag(q));
    a_prev = a;
    rec = rn;
  }
}

// One warp's sweep of one 32-row band of a tile, block by block (the
// encoder's mirror of the decoder's RecBand): begin() stages the first
// source chunks, block(k) runs wavefront block k (staging the chunk ahead
// and flushing the folded residuals two chunks behind), end() flushes the
// rest.  vmax tracks the largest source sample read (the depth check).
template <bool MED, bool STEP1, int UNROLL, bool SPLIT, typename FoldT>
struct EncBand {
  static constexpr int kFS = EncWarpSmem<FoldT>::kFS;
  EncWarpSmem<FoldT>& sm;
  int lane;
  const uint16_t* __restrict__ plane;
  int64_t pitch;
  int W, H, x0, y0;
  int32_t maxs, step, half;
  uint32_t magic;
  int nchunks, nblocks;
  FoldT* __restrict__ ftile;
  uint32_t vmax = 0;
  int band_rows;
  bool band0;
  const uint16_t* __restrict__ rows;
  FoldT* __restrict__ frows;
  const uint16_t* carry_in;
  uint16_t* carry_out;
  int32_t rec, a_prev;
  uint32_t pf[32];

  __device__ EncBand(const FrameDesc& f, const TileGeo& g, int32_t step_, uint32_t magic_, FoldT* ftile_,
                     EncWarpSmem<FoldT>& sm_, int lane_)
      : sm(sm_), lane(lane_), plane(f.src[g.plane]), pitch(f.src_pitch[g.plane]), W(g.w), H(g.h), x0(g.x), y0(g.y),
        maxs(f.max_sample), step(step_), half(step_ >> 1), magic(magic_), nchunks((g.w + 31) >> 5),
        nblocks((g.w + 31 + 31) >> 5), ftile(ftile_) {}

  __device__ void load_chunk(int k) {
    const int col = k * 32 + lane;
    const uint16_t* __restrict__ p = rows + col;
    if (band_rows == 32 && col < W) {
#pragma unroll
      for (int r = 0; r < 32; ++r) pf[r] = __ldg(p + static_cast<int64_t>(r) * pitch);
    } else {
#pragma unroll
      for (int r = 0; r < 32; ++r) pf[r] = (r < band_rows && col < W) ? __ldg(p + static_cast<int64_t>(r) * pitch) : 0u;
    }
  }
  // Every loaded chunk is stored once, a wavefront block after its load was
  // issued; the depth check's maximum is taken here, where the loads have
  // landed, not right after they are issued.
  __device__ void store_chunk(int k) {
    const int pj = k * 32 + lane;
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      vmax = max(vmax, pf[r]);
      sm.src[r * kSrcStride + ((pj + r) & 63)] = static_cast<uint16_t>(pf[r]);
    }
  }
  __device__ void flush_chunk(int k) {
    const int col = k * 32 + lane;
    if (col < W) {
      FoldT* __restrict__ q = frows + col;
      if (band_rows == 32) {
#pragma unroll
        for (int r = 0; r < 32; ++r) q[static_cast<int64_t>(r) * W] = sm.fold[r * kFS + ((col + r) & 63)];
      } else {
        for (int r = 0; r < band_rows; ++r) q[static_cast<int64_t>(r) * W] = sm.fold[r * kFS + ((col + r) & 63)];
      }
    }
  }
  __device__ void begin(int band, const uint16_t* cin, uint16_t* cout) {
    band_rows = min(32, H - band * 32);
    band0 = band == 0;
    rows = plane + static_cast<int64_t>(y0 + band * 32) * pitch + x0;
    frows = ftile + static_cast<int64_t>(band * 32) * W;
    carry_in = cin;
    carry_out = cout;
    load_chunk(0);
    store_chunk(0);
    if (nchunks > 1) load_chunk(1);
    __syncwarp();
    rec = 0;
    a_prev = 0;
  }
  __device__ void block(int blk) {
    if (blk > 0) {
      if (blk < nchunks) store_chunk(blk);
      __syncwarp();
      if (blk >= 2 && blk - 2 < nchunks) flush_chunk(blk - 2);
      if (blk + 1 < nchunks) load_chunk(blk + 1);
    }
    const int t0 = blk * 32;
    if (t0 < 31 || t0 + 31 >= W)
      enc_block<MED, STEP1, true, UNROLL, SPLIT, FoldT>(sm, carry_in, carry_out, lane, t0, W, maxs, step, half, magic, band0, rec,
                                          a_prev);
    else
      enc_block<MED, STEP1, false, UNROLL, SPLIT, FoldT>(sm, carry_in, carry_out, lane, t0, W, maxs, step, half, magic, band0, rec,
                                           a_prev);
  }
  __device__ void end() {
    __syncwarp();
    for (int j = max(0, nblocks - 2); j < nchunks; ++j) flush_chunk(j);
    __syncwarp();
  }
};

// A tile by one warp: bands in order, one carry row (read by lane 0 before
// lane 31 overwrites it).  Kept apart from EncBand: written as one loop nest
// it needs no register spills.
template <bool MED, bool STEP1, int UNROLL, typename FoldT>
__device__ void enc_tile_fast(const FrameDesc& f, const TileGeo& g, int32_t step, uint32_t magic,
                              FoldT* __restrict__ folded_tile, EncWarpSmem<FoldT>& sm, int lane, int32_t& bad) {
  constexpr int kFS = EncWarpSmem<FoldT>::kFS;
  const uint16_t* __restrict__ plane = f.src[g.plane];
  const int64_t pitch = f.src_pitch[g.plane];
  const int W = g.w, H = g.h;
  const int32_t maxs = f.max_sample;
  const int32_t half = step >> 1;
  const int nchunks = (W + 31) >> 5;
  const int nblocks = (W + 31 + 31) >> 5;
  uint32_t vmax = 0;
  for (int band = 0; band * 32 < H; ++band) {
    const int band_rows = min(32, H - band * 32);
    const uint16_t* __restrict__ rows = plane + static_cast<int64_t>(g.y + band * 32) * pitch + g.x;
    FoldT* __restrict__ frows = folded_tile + static_cast<int64_t>(band * 32) * W;
    uint32_t pf[32];
    auto load_chunk = [&](int k) {
      const int col = k * 32 + lane;
      const uint16_t* __restrict__ p = rows + col;
      if (band_rows == 32 && col < W) {
#pragma unroll
        for (int r = 0; r < 32; ++r) pf[r] = __ldg(p + static_cast<int64_t>(r) * pitch);
      } else {
#pragma unroll
        for (int r = 0; r < 32; ++r) pf[r] = (r < band_rows && col < W) ? __ldg(p + static_cast<int64_t>(r) * pitch) : 0u;
      }
    };
    // the depth check's maximum where the loads have landed (each loaded
    // chunk is stored once, a wavefront block after its loads were issued)
    auto store_chunk = [&](int k) {
      const int pj = k * 32 + lane;
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        vmax = max(vmax, pf[r]);
        sm.src[r * kSrcStride + ((pj + r) & 63)] = static_cast<uint16_t>(pf[r]);
      }
    };
    auto flush_chunk = [&](int k) {
      const int col = k * 32 + lane;
      if (col < W) {
        FoldT* __restrict__ q = frows + col;
        if (band_rows == 32) {
#pragma unroll
          for (int r = 0; r < 32; ++r) q[static_cast<int64_t>(r) * W] = sm.fold[r * kFS + ((col + r) & 63)];
        } else {
          for (int r = 0; r < band_rows; ++r) q[static_cast<int64_t>(r) * W] = sm.fold[r * kFS + ((col + r) & 63)];
        }
      }
    };
    load_chunk(0);
    store_chunk(0);
    if (nchunks > 1) load_chunk(1);
    __syncwarp();
    int32_t rec = 0, a_prev = 0;
    const bool band0 = band == 0;
    for (int blk = 0; blk < nblocks; ++blk) {
      if (blk > 0) {
        if (blk < nchunks) store_chunk(blk);
        __syncwarp();
        if (blk >= 2 && blk - 2 < nchunks) flush_chunk(blk - 2);
        if (blk + 1 < nchunks) load_chunk(blk + 1);
      }
      const int t0 = blk * 32;
      const bool edge = t0 < 31 || t0 + 31 >= W;
      if (edge)
        enc_block<MED, STEP1, true, UNROLL, false, FoldT>(sm, sm.carry, sm.carry, lane, t0, W, maxs, step, half, magic, band0,
                                                   rec, a_prev);
      else
        enc_block<MED, STEP1, false, UNROLL, false, FoldT>(sm, sm.carry, sm.carry, lane, t0, W, maxs, step, half, magic,
                                                    band0, rec, a_prev);
    }
    __syncwarp();
    for (int j = max(0, nblocks - 2); j < nchunks; ++j) flush_chunk(j);
    __syncwarp();
  }
  if (vmax > static_cast<uint32_t>(maxs)) bad = 1;
}

// The two warps of pair p meet at named barrier 1 + p (64 threads).
__device__ __forceinline__ void enc_pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
}

template <bool MED, bool STEP1, int UNROLL, bool PAIRS, typename FoldT>
__device__ void enc_tile(const FrameDesc& f, const TileGeo& g, int32_t step, uint32_t magic,
                         FoldT* __restrict__ folded_tile, EncWarpSmem<FoldT>* smw, int warp, int lane,
                         int32_t& bad) {
  if constexpr (PAIRS) {
    if (pair_splits(g.w, g.h)) {
      // warp pair: even bands on the first warp, odd bands on the second two
      // blocks behind, in lock-step at the pair barrier after every slot (the
      // schedule of dec_reconstruct)
      const int pw = warp & 1;
      EncWarpSmem<FoldT>& sm = smw[warp];
      EncBand<MED, STEP1, UNROLL, true, FoldT> eb(f, g, step, magic, folded_tile, sm, lane);
      const int n = eb.nblocks, nbands = (g.h + 31) >> 5;
      const int own = pw ? (nbands / 2) * n : ((nbands + 1) / 2) * n;
      const int slots = max(((nbands + 1) / 2) * n, (nbands / 2) * n + 2);
      for (int gs = 0; gs < slots; ++gs) {
        const int sl = gs - 2 * pw;
        if (sl >= 0 && sl < own) {
          const int q = sl / n, blk = sl - q * n;
          if (blk == 0) eb.begin(2 * q + pw, smw[warp ^ 1].carry, sm.carry);
          eb.block(blk);
          if (blk == n - 1) eb.end();
        }
        enc_pair_sync(warp >> 1);
      }
      if (eb.vmax > static_cast<uint32_t>(f.max_sample)) bad = 1;
      return;
    }
    if (warp & 1) return;  // too small to split: the pair's first warp alone
  }
  enc_tile_fast<MED, STEP1, UNROLL, FoldT>(f, g, step, magic, folded_tile, smw[warp], lane, bad);
}

// Tiles come from a queue; with warp pairs the pair's first warp claims a
// tile and both read it after the pair barrier (two alternating slots), and
// both make the same decisions from it, so they meet at every barrier.
template <int UNROLL, bool PAIRS, typename FoldT>
__global__ void __launch_bounds__(kWarpsPerCta * 32, PAIRS ? 3 : 4)
enc_predict_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                   const BatchDims* __restrict__ dims, int pass, ShardInfo* __restrict__ shards,
                   FoldT* __restrict__ folded, int* __restrict__ queue) {
  static_assert(kWarpsPerCta % 2 == 0, "warp pairs");
  constexpr bool pairs = PAIRS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int64_t claimed[kWarpsPerCta / 2][2];
  const int nframes = dims->frames_p[pass];
  const int64_t total_tiles = dims->tiles_p[pass];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  EncWarpSmem<FoldT>* smw = reinterpret_cast<EncWarpSmem<FoldT>*>(smem_raw);
  for (int it = 0;; ++it) {
    int64_t t = 0;
    if (pairs) {
      if ((warp & 1) == 0 && lane == 0) claimed[warp >> 1][it & 1] = atomicAdd(queue, 1);
      enc_pair_sync(warp >> 1);
      t = claimed[warp >> 1][it & 1];
    } else {
      if (lane == 0) t = atomicAdd(queue, 1);
      t = __shfl_sync(kFull, t, 0);
    }
    if (t >= total_tiles) break;
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    FrameState& st = state[fi];
    const TileGeo g = tile_geo(f, t - f.tile_base);
    // shard records of this tile (encode.cu:753-759), written for every
    // frame of the pass, active or not: the later passes write a region of
    // their own, and the analysis kernels read every record of the pass
    // (frame index first) before they skip inactive frames; with pairs the
    // first warp writes them
    if (!pairs || (warp & 1) == 0) {
      for (int j = lane; j < g.shard_count; j += 32) {
        ShardInfo& si = shards[f.shard_base + g.first_shard + j];
        const int64_t local = static_cast<int64_t>(j) * kShardSymbols;
        si.sample_base = f.sample_base + g.sample_base + local;
        si.count = static_cast<int32_t>(min(static_cast<int64_t>(kShardSymbols), static_cast<int64_t>(g.w) * g.h - local));
        si.frame = fi;
      }
    }
    if (!st.active) continue;
    if (g.w > kFastMaxW) continue;  // wide tiles go through enc_predict_wide_kernel
    const int32_t step = st.step;
    const uint32_t magic = step > 1 ? static_cast<uint32_t>((0x100000000ull + step - 1) / step) : 0u;
    FoldT* ftile = folded + f.sample_base + g.sample_base;
    int32_t bad = 0;
    const bool med = st.use_med != 0;
    if (med) {
      if (step == 1) enc_tile<true, true, UNROLL, PAIRS, FoldT>(f, g, step, magic, ftile, smw, warp, lane, bad);
      else enc_tile<true, false, UNROLL, PAIRS, FoldT>(f, g, step, magic, ftile, smw, warp, lane, bad);
    } else {
      if (step == 1) enc_tile<false, true, UNROLL, PAIRS, FoldT>(f, g, step, magic, ftile, smw, warp, lane, bad);
      else enc_tile<false, false, UNROLL, PAIRS, FoldT>(f, g, step, magic, ftile, smw, warp, lane, bad);
    }
    if (__any_sync(kFull, bad) && lane == 0) set_status(&st.status, 1);
  }
}

// The wavefront block of enc_predict -- steps of each 32-step block unrolled
// -- is a launch-time choice (4, 8, 16 or 32; the autotuner's knob): every
// choice computes the same bytes.
cudaError_t enc_predict_set_smem() {
  const int b32 = static_cast<int>(enc_predict_smem(false)), b16 = static_cast<int>(enc_predict_smem(true));
  for (auto k : {enc_predict_kernel<4, false, uint32_t>, enc_predict_kernel<8, false, uint32_t>,
                 enc_predict_kernel<16, false, uint32_t>, enc_predict_kernel<32, false, uint32_t>,
                 enc_predict_kernel<8, true, uint32_t>}) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b32);
    if (e != cudaSuccess) return e;
  }
  for (auto k : {enc_predict_kernel<4, false, uint16_t>, enc_predict_kernel<8, false, uint16_t>,
                 enc_predict_kernel<16, false, uint16_t>, enc_predict_kernel<32, false, uint16_t>,
                 enc_predict_kernel<8, true, uint16_t>}) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b16);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename FoldT>
void enc_predict_launch_t(int unroll, int tile_warps, int grid, cudaStream_t stream, const FrameDesc* frames,
                          FrameState* state, const BatchDims* dims, int pass, ShardInfo* shards, void* folded,
                          int* queue) {
  // warp pairs run with the default wavefront block
  auto k = tile_warps == 2 ? enc_predict_kernel<8, true, FoldT>
           : unroll == 4   ? enc_predict_kernel<4, false, FoldT>
           : unroll == 16  ? enc_predict_kernel<16, false, FoldT>
           : unroll == 32  ? enc_predict_kernel<32, false, FoldT>
                           : enc_predict_kernel<8, false, FoldT>;
  k<<<grid, kWarpsPerCta * 32, enc_predict_smem(sizeof(FoldT) == 2), stream>>>(
      frames, state, dims, pass, shards, static_cast<FoldT*>(folded), queue);
}

void enc_predict_launch(int unroll, int tile_warps, bool fold16, int grid, cudaStream_t stream,
                        const FrameDesc* frames, FrameState* state, const BatchDims* dims, int pass,
                        ShardInfo* shards, void* folded, int* queue) {
  if (fold16)
    enc_predict_launch_t<uint16_t>(unroll, tile_warps, grid, stream, frames, state, dims, pass, shards, folded, queue);
  else
    enc_predict_launch_t<uint32_t>(unroll, tile_warps, grid, stream, frames, state, dims, pass, shards, folded, queue);
}

// Tiles wider than kFastMaxW: one CTA per tile walks the antidiagonals with
// the reconstruction kept in global scratch (same order as the reference,
// encode.cu:150-192).  Only used for unusually wide tile sizes.
__global__ void enc_predict_wide_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                                        const BatchDims* __restrict__ dims, int pass, void* __restrict__ folded_raw,
                                        uint16_t* __restrict__ recon, int fold16) {
  const int nframes = dims->frames_p[pass];
  const int64_t total_tiles = dims->tiles_p[pass];
  for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    FrameState& st = state[fi];
    if (!st.active) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    if (g.w <= kFastMaxW) continue;
    const int32_t step = st.step, maxs = f.max_sample;
    const bool med = st.use_med != 0;
    const uint16_t* plane = f.src[g.plane];
    const int64_t pitch = f.src_pitch[g.plane];
    uint16_t* rtile = recon + f.sample_base + g.sample_base;  // tile-raster scratch
    const int64_t fbase = f.sample_base + g.sample_base;
    int bad = 0;
    for (int d = 0; d < g.w + g.h - 1; ++d) {
      const int y0 = max(0, d - g.w + 1), y1 = min(d, g.h - 1);
      for (int y = y0 + threadIdx.x; y <= y1; y += blockDim.x) {
        const int x = d - y;
        const int32_t s = plane[static_cast<int64_t>(g.y + y) * pitch + g.x + x];
        if (s > maxs) bad = 1;
        const int64_t i = static_cast<int64_t>(y) * g.w + x;
        const int32_t l = x > 0 ? rtile[i - 1] : 0;
        const int32_t a = y > 0 ? rtile[i - g.w] : 0;
        const int32_t ul = (x > 0 && y > 0) ? rtile[i - g.w - 1] : 0;
        const int32_t pred = med ? predict_med(l, a, ul) : predict_grad(l, a, ul, maxs);
        const int32_t res = s - pred;
        const int32_t mag = (abs(res) + step / 2) / step;
        const int32_t q = res < 0 ? -mag : mag;
        rtile[i] = static_cast<uint16_t>(max(0, min(maxs, pred + q * step)));
        if (fold16) static_cast<uint16_t*>(folded_raw)[fbase + i] = static_cast<uint16_t>(zigzag(q));
        else static_cast<uint32_t*>(folded_raw)[fbase + i] = zigzag(q);
      }
      __syncthreads();
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_status(&st.status, 1);
  }
}

// ---------------------------------------------------------------------------
// enc_analyze: one warp per shard, one 128-symbol pack block per step.  Lane
// l holds symbols 4l..4l+3 of the block, so component j of every lane is
// Rice lane j (symbol i -> lane i % 4; shards of fewer than four symbols use
// lane i as well).
//
// Pass 1 gathers per shard:
//  * the class histograms (class = Rice lane) -- values below 8, nearly all
//    symbols of a predicted frame, in per-lane nibble counters, larger values
//    below 511 with shared-memory atomics;
//  * the block-pack widths (encode.cu:249-259) and the shard maximum.
// The Rice sums sum_i (v_i >> k), the zero-run value bytes and the order-0
// rANS table then come from the histograms; shards holding a value of 511 or
// more take a second per-sample pass for the Rice sums instead.  The
// zero-run run tokens are counted (in one more pass) only for shards whose
// value tokens alone do not already lose to block packing or Rice coding.

__device__ __forceinline__ int bitlen(uint32_t v) { return 32 - __clz(v); }
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(kFull, v); }

// 1 << s for s < 32 and 0 for larger s (PTX shl clamps the shift amount)
__device__ __forceinline__ uint32_t bit_or_zero(uint32_t s) {
  uint32_t r;
  asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(1u), "r"(s));
  return r;
}

// rANS encoding of a symbol with frequency f and start cum maps the state x
// (below f * 2^19 after renormalisation, so below 2^31) to
// (x / f) * 4096 + x % f + cum = x + cum + (x / f) * (4096 - f).  The quotient
// comes from a multiply-high and a shift by an exact reciprocal (Alverson,
// "Integer division using reciprocals", ARITH 1991): with s = ceil(log2 f)
// and m = ceil(2^(31+s) / f) < 2^32, floor(x * m / 2^(31+s)) = floor(x / f)
// for every x < 2^31, because m exceeds 2^(31+s)/f by less than one, which
// moves x * m / 2^(31+s) by less than x / 2^(31+s) < 2^-s <= 1/f.  For f = 1
// the multiplier 2^32-1 yields x - 1, and the bias carries the missing 4095.
// Table entry: the multiplier, then bias | (4096 - f) << 13 | (s - 1) << 25.
__device__ __forceinline__ uint32_t rans_multiplier(uint32_t f) {
  if (f < 2) return 0xffffffffu;
  const uint32_t s = 32 - __clz(f - 1);
  // m = floor((2^(31+s) - 1) / f) + 1 by long division in 16-bit digits:
  // 2^(31+s) - 1 = (2^(s-1) - 1) * 2^32 + 0xffffffff, and 2^(s-1) - 1 < f
  const uint32_t t1 = (((1u << (s - 1)) - 1u) << 16) | 0xffffu;
  const uint32_t q1 = t1 / f;
  const uint32_t t2 = ((t1 - q1 * f) << 16) | 0xffffu;
  return ((q1 << 16) | (t2 / f)) + 1u;
}
__device__ __forceinline__ uint32_t rans_packed(uint32_t f, uint32_t cum) {
  const uint32_t bias = f < 2 ? cum + 4095u : cum;
  const uint32_t sh = f < 2 ? 0u : 31u - __clz(f - 1);  // s - 1
  return bias | ((4096u - f) << 13) | (sh << 25);
}

// Zero-run token statistics of one 128-symbol block (encode.cu:232-240): a
// run of zeros costs varint(2(run-1)), one byte up to 64 zeros and two beyond
// (a shard holds at most 4096 symbols).  zm: this lane's zero components at
// positions p0..p0+3; positions past the shard end count as nonzero.
struct RunStats {
  int32_t carry = -1;      // last nonzero position of the blocks so far
  uint32_t runs = 0;       // runs started (per lane)
  uint32_t long_runs = 0;  // runs that reached 65 zeros (per lane)
};

__device__ __forceinline__ void run_block(RunStats& r, uint32_t zm, int32_t p0, int lane) {
  const uint32_t nzm = ~zm & 0xfu;
  int32_t last = nzm ? p0 + 31 - __clz(nzm) : -1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) last = max(last, __shfl_up_sync(kFull, last, o));
  const int32_t up = __shfl_up_sync(kFull, last, 1);
  const int32_t before = lane ? max(up, r.carry) : r.carry;  // last nonzero before p0
  r.carry = max(r.carry, __shfl_sync(kFull, last, 31));
  // a zero starts a run when its predecessor is nonzero (or the shard start)
  r.runs += __popc(zm & ((nzm << 1) | (before == p0 - 1 ? 1u : 0u)));
  // the run through p0 has p0-1-before zeros ahead of it; it reaches 65
  // zeros at component 64-(p0-1-before) if the zeros last that far
  const uint32_t jh = static_cast<uint32_t>(64 - (p0 - 1 - before));
  if (jh < 4u) {
    const uint32_t need = (2u << jh) - 1u;
    r.long_runs += (zm & need) == need;
  }
}

template <typename FoldT>
__global__ void __launch_bounds__(kWarpsPerCta * 32, 6)
enc_analyze_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                   const BatchDims* __restrict__ dims, int pass, ShardInfo* __restrict__ shards,
                   const FoldT* __restrict__ folded, uint8_t* __restrict__ rans_scratch) {
  // a lane's four symbols of a pack block: one 16-byte piece (u32 symbols)
  // or one 8-byte piece (u16 symbols)
  using Piece = FoldPiece<FoldT>;
  const int nframes = dims->frames_p[pass];
  const int64_t total_shards = dims->shards_p[pass];
  // Class counts: two classes share a 32-bit word (16-bit counts: a class
  // holds at most 1024 symbols); the words of classes (0,1) and (2,3) of a
  // value sit 520 words apart, in different banks.  list: the present values
  // in increasing order, value | total count << 16.  ring: each lane's next
  // kRing 16-byte pieces of the warp's block stream.
  constexpr int kRing = 6;  // measured on the 96-frame mix: 6 pieces ahead beats 8
  __shared__ __align__(16) uint32_t hcls_all[kWarpsPerCta][2][520];
  __shared__ uint32_t list_all[kWarpsPerCta][512];
  __shared__ __align__(16) Piece ring_all[kWarpsPerCta][kRing * 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t (*hcls)[520] = hcls_all[warp];
  uint32_t* list = list_all[warp];
  Piece* ring = ring_all[warp];
  const uint32_t lanes_below = (1u << lane) - 1u;
  for (int i = lane; i < 2 * 520 / 4; i += 32) reinterpret_cast<uint4*>(hcls[0])[i] = make_uint4(0, 0, 0, 0);
  __syncwarp();
  // frames of this pass (bit per frame, the first kMaskFrames frames; later
  // frames are treated as active until their own flag is read)
  constexpr int kMaskFrames = 4096;
  __shared__ uint32_t active_mask[kMaskFrames / 32];
  const int mask_words = min((nframes + 31) / 32, kMaskFrames / 32);
  for (int w = warp; w < mask_words; w += kWarpsPerCta) {
    const int i = w * 32 + lane;
    const uint32_t m = __ballot_sync(kFull, i < nframes && state[i].active);
    if (lane == 0) active_mask[w] = m;
  }
  __syncthreads();
  auto streamed = [&](int32_t frame) {
    return frame >= kMaskFrames || ((active_mask[frame >> 5] >> (frame & 31)) & 1u);
  };
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  const int64_t s0 = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp;
  // Whole blocks of a shard that starts piece-aligned are read through the
  // ring; the ragged last block and unaligned shards use direct loads.
  // Shards of frames that sit this pass out are skipped by both sides.
  auto whole_blocks = [&](int32_t count, int64_t base, int32_t frame) {
    return streamed(frame) && (reinterpret_cast<uintptr_t>(folded + base) & (sizeof(Piece) - 1)) == 0
               ? count / kBlockSymbols
               : 0;
  };
  // Producer: the warp's whole blocks in shard order, kRing pieces ahead of
  // the consumer and across shard boundaries, one commit group per piece
  // (empty past the end), so piece i sits in slot i % kRing and its group is
  // complete once at most kRing - 1 newer groups are pending.
  int64_t pt = s0;      // shard being fetched
  int pc = 0, pnf = 0;  // next block and whole blocks of pt
  const Piece* pp = nullptr;
  int32_t q_count = 0, q_frame = 0;  // shard pt + warps_total, loaded one shard early
  int64_t q_base = 0;
  int pslot = 0;
  if (pt < total_shards) {
    pnf = whole_blocks(shards[pt].count, shards[pt].sample_base, shards[pt].frame);
    pp = reinterpret_cast<const Piece*>(folded + shards[pt].sample_base);
    if (pt + warps_total < total_shards) {
      q_count = shards[pt + warps_total].count;
      q_frame = shards[pt + warps_total].frame;
      q_base = shards[pt + warps_total].sample_base;
    }
  }
  auto issue = [&]() {
    while (pc >= pnf && pt < total_shards) {
      pt += warps_total;
      pc = 0;
      if (pt < total_shards) {
        pnf = whole_blocks(q_count, q_base, q_frame);
        pp = reinterpret_cast<const Piece*>(folded + q_base);
        if (pt + warps_total < total_shards) {
          q_count = shards[pt + warps_total].count;
          q_frame = shards[pt + warps_total].frame;
          q_base = shards[pt + warps_total].sample_base;
        }
      }
    }
    if (pt < total_shards) {
      cp_async_piece(ring + pslot * 32 + lane, pp + pc * 32 + lane);
      ++pc;
    }
    cp_async_commit();
    pslot = pslot + 1 == kRing ? 0 : pslot + 1;
  };
  for (int i = 0; i < kRing; ++i) issue();
  int cslot = 0;
  // consumer: the next shard's descriptor is loaded while this one runs
  int32_t h_count = 0, h_frame = 0;
  int64_t h_base = 0;
  if (s0 < total_shards) {
    h_count = shards[s0].count;
    h_frame = shards[s0].frame;
    h_base = shards[s0].sample_base;
  }
  for (int64_t s = s0; s < total_shards; s += warps_total) {
    ShardInfo& si = shards[s];
    const int n = h_count;
    const int64_t base = h_base;
    const int32_t frame = h_frame;
    if (s + warps_total < total_shards) {
      h_count = shards[s + warps_total].count;
      h_frame = shards[s + warps_total].frame;
      h_base = shards[s + warps_total].sample_base;
    }
    if (!streamed(frame)) continue;
    FrameState& st = state[frame];
    const int32_t active = st.active;  // first needed after pass 1
    const FoldT* __restrict__ f = folded + base;
    const int lane_count = min(4, n);

    // ---- pass 1 ----
    uint32_t nib[4] = {0, 0, 0, 0};    // class j: 4-bit counts of values 0..7
    uint32_t acc_e[4] = {0, 0, 0, 0};  // class j: 8-bit counts of values 0, 2, 4, 6
    uint32_t acc_o[4] = {0, 0, 0, 0};  // class j: 8-bit counts of values 1, 3, 5, 7
    uint32_t shard_max = 0, clz_sum = 0, tail_bytes = 0;  // warp-uniform
    auto flush = [&]() {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc_e[j] += nib[j] & 0x0f0f0f0fu;
        acc_o[j] += (nib[j] >> 4) & 0x0f0f0f0fu;
        nib[j] = 0;
      }
    };
    auto count_big = [&](const uint32_t (&x)[4], uint32_t valid) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (((valid >> j) & 1u) && x[j] >= 8u && x[j] < static_cast<uint32_t>(kRansAlphabet))
          atomicAdd(&hcls[j >> 1][x[j]], 1u << (16 * (j & 1)));
    };
    const int nblk = (n + kBlockSymbols - 1) / kBlockSymbols;
    const int nfull = whole_blocks(n, base, frame);
    // whole blocks from the ring; the nibble counters take at most 8 blocks
    // between flushes
    for (int g = 0; g < nfull; g += 8) {
      const int ge = min(g + 8, nfull);
      for (int b = g; b < ge; ++b) {
        cp_async_wait<kRing - 1>();
        uint32_t x[4];
        unpack_piece(ring[cslot * 32 + lane], x);
#pragma unroll
        for (int j = 0; j < 4; ++j) nib[j] += bit_or_zero(x[j] << 2);  // values >= 8 add nothing
        const uint32_t bm = __reduce_max_sync(kFull, max(max(x[0], x[1]), max(x[2], x[3])));
        issue();  // refills the slot just read
        cslot = cslot + 1 == kRing ? 0 : cslot + 1;
        shard_max = max(shard_max, bm);
        clz_sum += __clz(bm);  // block bytes 1 + 128 * bitlen / 8
        if (bm >= 8u) count_big(x, 0xfu);
      }
      flush();
    }
    for (int b = nfull; b < nblk; ++b) {
      // the ragged last block, or every block of an unaligned shard
      const int p0 = b * kBlockSymbols + 4 * lane;
      uint32_t x[4];
      uint32_t valid = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const bool ok = p0 + j < n;
        x[j] = ok ? ldf(f + p0 + j) : 0u;
        valid |= ok ? 1u << j : 0u;
        nib[j] += ok ? bit_or_zero(x[j] << 2) : 0u;
      }
      const uint32_t bm = __reduce_max_sync(kFull, max(max(x[0], x[1]), max(x[2], x[3])));
      shard_max = max(shard_max, bm);
      tail_bytes += 1 + (min(kBlockSymbols, n - b * kBlockSymbols) * bitlen(bm) + 7) / 8;
      if (bm >= 8u) count_big(x, valid);
      if ((b & 7) == 7) flush();
    }
    flush();
    const uint32_t block_bytes = static_cast<uint32_t>(nfull) * 513u - 16u * clz_sum + tail_bytes;
    // clear the histogram bins the atomics of this shard may have touched
    auto clear_bins = [&]() {
      __syncwarp();
      const int used = static_cast<int>(min(shard_max, static_cast<uint32_t>(kRansAlphabet - 1)) >> 5) + 1;
      for (int it = 0; it < used; ++it) {
        hcls[0][it * 32 + lane] = 0;
        hcls[1][it * 32 + lane] = 0;
      }
      __syncwarp();
    };
    if (!active) {  // a frame past the active mask that sits this pass out: nothing written
      clear_bins();
      continue;
    }
    // warp totals of the small-value counts, as class-pair words; their
    // Rice sums for k = 0..2 (values below 8 have v >> 3 == 0)
    uint32_t small01[3] = {0, 0, 0}, small23[3] = {0, 0, 0};
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      // byte v/2 of classes (0,1) resp. (2,3) into the two 16-bit halves
      const uint32_t sel = static_cast<uint32_t>(v >> 1) | ((4u + static_cast<uint32_t>(v >> 1)) << 8);
      const uint32_t w01 =
          warp_sum(__byte_perm((v & 1) ? acc_o[0] : acc_e[0], (v & 1) ? acc_o[1] : acc_e[1], sel) & 0x00ff00ffu);
      const uint32_t w23 =
          warp_sum(__byte_perm((v & 1) ? acc_o[2] : acc_e[2], (v & 1) ? acc_o[3] : acc_e[3], sel) & 0x00ff00ffu);
      if (lane == v) {
        hcls[0][v] = w01;
        hcls[1][v] = w23;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        small01[k] += w01 * static_cast<uint32_t>(v >> k);
        small23[k] += w23 * static_cast<uint32_t>(v >> k);
      }
    }
    __syncwarp();

    uint32_t sk[kMaxRice + 1];
#pragma unroll
    for (int k = 0; k <= kMaxRice; ++k) sk[k] = 0;
    uint32_t nz_cost = 0;  // varint bytes of the nonzero value tokens
    int distinct = 0;
    if (shard_max < static_cast<uint32_t>(kRansAlphabet)) {
      // the list of present values and the value-token bytes: varint(2v-1)
      // is one byte up to v = 64 and two below 511
      int small_present = 0;
      uint32_t nzc = 0;
      const int iters = static_cast<int>(shard_max >> 5) + 1;
      for (int it = 0; it < iters; ++it) {
        const int v = it * 32 + lane;
        const uint32_t w01 = hcls[0][v], w23 = hcls[1][v];
        const uint32_t h = (w01 & 0xffffu) + (w01 >> 16) + (w23 & 0xffffu) + (w23 >> 16);
        const uint32_t pres = __ballot_sync(kFull, h != 0);
        if (h) list[distinct + __popc(pres & lanes_below)] = static_cast<uint32_t>(v) | (h << 16);
        if (it == 0) small_present = __popc(pres & 0xffu);
        distinct += __popc(pres);
        nzc += v ? h * (1u + (v > 64)) : 0u;
      }
      nz_cost = warp_sum(nzc);
      __syncwarp();
      // Rice sums, class l in lane l: the small values' part plus, one class
      // at a time, the values from 8 up
      const int cl = lane & 3;
      const uint32_t sel = lane < 4 ? 0xffffffffu : 0u;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint32_t w = (cl >> 1) ? small23[k] : small01[k];
        sk[k] = ((w >> (16 * (cl & 1))) & 0xffffu) & sel;
      }
      if (distinct > small_present) {
#pragma unroll 1
        for (int l = 0; l < 4; ++l) {
          uint32_t S[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) S[k] = 0;
          for (int e = small_present + lane; e < distinct; e += 32) {
            const uint32_t v = list[e] & 0xffffu;
            const uint32_t c = (hcls[l >> 1][v] >> (16 * (l & 1))) & 0xffffu;
#pragma unroll
            for (int k = 0; k < 9; ++k) S[k] += c * (v >> k);
          }
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            const uint32_t t = warp_sum(S[k]);
            if (lane == l) sk[k] += t;
          }
        }
      }
    } else {
      // pass 2: per-sample Rice sums and value costs, lane i % 32 of each
      // 32-symbol chunk (Rice lane i % 4 = lane % 4)
      const int nchunk = (n + 31) >> 5;
      for (int m = 0; m < nchunk; ++m) {
        const int idx = m * 32 + lane;
        const uint32_t v = idx < n ? ldf(f + idx) : 0u;
        const int kb = bitlen(__reduce_max_sync(kFull, v));
#pragma unroll
        for (int k = 0; k < 4; ++k) sk[k] += v >> k;
        if (kb > 4) {
#pragma unroll
          for (int k = 4; k < 8; ++k) sk[k] += v >> k;
        }
        if (kb > 8) {
#pragma unroll
          for (int k = 8; k < 12; ++k) sk[k] += v >> k;
        }
        if (kb > 12) {
#pragma unroll
          for (int k = 12; k <= kMaxRice; ++k) sk[k] += v >> k;
        }
        nz_cost += v != 0 ? 1u + (v > 64u) + (v > 8192u) + (v > (1u << 20)) : 0u;
      }
      nz_cost = warp_sum(nz_cost);
#pragma unroll
      for (int k = 0; k <= kMaxRice; ++k) {
        uint32_t v = sk[k];
        v += __shfl_xor_sync(kFull, v, 4);
        v += __shfl_xor_sync(kFull, v, 8);
        v += __shfl_xor_sync(kFull, v, 16);
        sk[k] = lane < 4 ? v : 0u;
      }
    }
    // Rice: lane l < lane_count holds the sums of Rice lane l
    int64_t best_bytes = INT64_MAX;
    int best_k = 0;
    uint32_t lane_bytes_best = 0;
    const int rl = lane & 3;
    const int nsym = rl < lane_count ? (n - rl + lane_count - 1) / lane_count : 0;
    // sums vanish beyond the shard's bit length, where the cost only grows
    const int kstop = min(kMaxRice, bitlen(shard_max));
#pragma unroll
    for (int k = 0; k <= kMaxRice; ++k) {
      if (k > kstop) break;
      const uint32_t v = __shfl_sync(kFull, sk[k], rl);
      const uint32_t bits = v + static_cast<uint32_t>(nsym) * (1u + k);
      const uint32_t lb = rl < lane_count ? (bits + 7) / 8 : 0u;
      uint32_t tot = lb + __shfl_xor_sync(kFull, lb, 1);
      tot += __shfl_xor_sync(kFull, tot, 2);
      if (static_cast<int64_t>(tot) < best_bytes) {
        best_bytes = tot;
        best_k = k;
        lane_bytes_best = lb;
      }
    }
    const int64_t rice_body = static_cast<int64_t>(lane_count - 1) * 4 + best_bytes;
    // zero-run coding wins only if its bytes are at most both others'; the
    // value tokens alone bound them from below
    int64_t zero_bytes = INT64_MAX;
    if (static_cast<int64_t>(nz_cost) <= min(static_cast<int64_t>(block_bytes), rice_body)) {
      RunStats rs;
      for (int b = 0; b < nblk; ++b) {
        const int p0 = b * kBlockSymbols + 4 * lane;
        uint32_t zm = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (p0 + j < n && __ldg(f + p0 + j) == 0u) zm |= 1u << j;
        run_block(rs, zm, p0, lane);
      }
      zero_bytes = static_cast<int64_t>(nz_cost) + warp_sum(rs.runs) + warp_sum(rs.long_runs);
    }
    int mode;
    int64_t body;
    if (static_cast<int64_t>(block_bytes) < zero_bytes && static_cast<int64_t>(block_bytes) < rice_body) {
      mode = kModeBlockPack;
      body = block_bytes;
    } else if (zero_bytes <= rice_body) {
      mode = kModeZeroRun;
      body = zero_bytes;
    } else {
      mode = kModeRiceBase + best_k;
      body = rice_body;
    }
    if (lane == 0) {
      si.comp_mode = mode;
      si.comp_k = best_k;
      si.comp_body = static_cast<int32_t>(body);
      // encode.cu:305-307; unreachable in practice (the block-pack bound is
      // 8736 bytes) but kept as the reference's guard.
      if (body > 65535) set_status(&st.status, 2);
    }
    if (lane < 4) si.comp_lane[lane] = lane < lane_count ? static_cast<int32_t>(lane_bytes_best) : 0;

    // order-0 rANS table (encode.cu:337-392), eligible when max < 511 and
    // at most 255 distinct symbols; one list entry per lane.
    const int rans_ok = shard_max < static_cast<uint32_t>(kRansAlphabet) && distinct <= 255;
    bool rans_keep = false;
    if (rans_ok) {
      // Normalisation as a prefix maximum: for the i-th present symbol,
      // end_i = i + min(max(1, max_{j<=i}(f_j - j)), 4097 - D) with
      // f_j = floor(P_j * 4096 / n), P_j the count of symbols up to the j-th;
      // the last symbol ends at 4096.  This equals the reference's clamp loop
      // (encode.cu:370-390): writing u_i = end_i - i turns
      // end_i = min(max(f_i, end_{i-1}+1), 4097-D+i) into
      // u_i = min(max(f_i - i, u_{i-1}), 4097-D) with u_{-1} = 1.
      const int D = distinct;
      const int32_t G = 4097 - D;
      // floor(x / n) for x <= 2^24 by a multiply-high with floor((2^32-1)/n)
      // and one correction (the estimate is exact or one low)
      const uint32_t un = static_cast<uint32_t>(n);
      const uint32_t ninv = 0xffffffffu / un;
      uint32_t* tab = reinterpret_cast<uint32_t*>(rans_scratch + s * static_cast<int64_t>(kRansScratchBytes));
      uint8_t* ser = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes) + kRansTableWords * 4;
      const int head = 1 + varint_len(static_cast<uint32_t>(D));
      uint32_t c_count = 0, c_cursor = static_cast<uint32_t>(head);
      int32_t c_u = 1, c_end = 0, c_v = 0;
      double info = 0.0;  // sum over the shard's symbols of log2(4096 / freq), this lane's entries
      for (int e0 = 0; e0 < D; e0 += 32) {
        const int e = e0 + lane;
        const bool ok = e < D;
        const uint32_t ent = ok ? list[e] : 0u;
        const int32_t v = static_cast<int32_t>(ent & 0xffffu);
        uint32_t P = ent >> 16;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(kFull, P, o);
          if (lane >= o) P += t;
        }
        P += c_count;
        const uint32_t x = P << kRansTableLog;
        uint32_t q = __umulhi(x, ninv);
        if (x - q * un >= un) ++q;
        int32_t u = ok ? static_cast<int32_t>(q) - e : INT32_MIN;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) u = max(u, __shfl_up_sync(kFull, u, o));
        u = max(u, c_u);
        const int32_t end = e == D - 1 ? (1 << kRansTableLog) : e + min(u, G);
        int32_t pe = __shfl_up_sync(kFull, end, 1), pv = __shfl_up_sync(kFull, v, 1);
        if (lane == 0) {
          pe = c_end;
          pv = c_v;
        }
        const uint32_t fr = static_cast<uint32_t>(end - pe);
        const uint32_t dv = static_cast<uint32_t>(v - pv);
        const uint32_t bytes = ok ? varint_len(dv) + (e != D - 1 ? varint_len(fr) : 0) : 0u;
        uint32_t binc = bytes;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(kFull, binc, o);
          if (lane >= o) binc += t;
        }
        if (ok) {
          info += static_cast<double>(ent >> 16) * (static_cast<double>(kRansTableLog) - log2(static_cast<double>(fr)));
          tab[2 * v] = rans_multiplier(fr);
          tab[2 * v + 1] = rans_packed(fr, static_cast<uint32_t>(pe));
          uint32_t cursor = c_cursor + binc - bytes;
          uint32_t d = dv;
          do {
            uint8_t byte = d & 0x7f;
            d >>= 7;
            if (d) byte |= 0x80;
            ser[cursor++] = byte;
          } while (d);
          if (e != D - 1) {
            uint32_t w = fr;
            do {
              uint8_t byte = w & 0x7f;
              w >>= 7;
              if (w) byte |= 0x80;
              ser[cursor++] = byte;
            } while (w);
          }
        }
        c_count = __shfl_sync(kFull, P, 31);
        c_u = __shfl_sync(kFull, u, 31);
        c_end = __shfl_sync(kFull, end, 31);
        c_v = __shfl_sync(kFull, v, 31);
        c_cursor += __shfl_sync(kFull, binc, 31);
      }
      if (lane == 0) {
        ser[0] = kRansTableLog;
        uint32_t d = static_cast<uint32_t>(D);
        int c = 1;
        do {
          uint8_t byte = d & 0x7f;
          d >>= 7;
          if (d) byte |= 0x80;
          ser[c++] = byte;
        } while (d);
        si.rans_table = static_cast<int32_t>(c_cursor);
      }
      // Skip the trial encoding when it cannot win.  Each rANS step takes a
      // state x in [f 2^11, f 2^19) after renormalisation to one at least
      // (x 4096 / f)(1 - 2^-11), and renormalising by b bytes keeps at least
      // (x / 2^8b)(1 - 2^-11) of it; a lane starts at 2^23 and ends below
      // 2^31.  So the bytes of the four lanes are at least
      // (I - 4 * 8 - 2 n log2(1/(1 - 2^-11))) / 8 >= (I - 38) / 8 for
      // I = sum log2(4096 / f) over the shard's n <= 4096 symbols, and with
      // a 64-bit margin for rounding, table + 28 + floor((I - 64) / 8) is a
      // lower bound of the rANS body.  When it reaches the best other body,
      // rANS cannot be chosen (encode.cu:420-430 takes it only when smaller,
      // or when the frame forces it) -- the bytes are the same without it.
      for (int o = 16; o > 0; o >>= 1) info += __shfl_xor_sync(kFull, info, o);
      const double bound = static_cast<double>(c_cursor) + 28.0 + floor((info - 64.0) / 8.0);
      rans_keep = frames[frame].force_order0 || bound < static_cast<double>(body);
    }
    if (lane == 0) si.rans_ok = rans_ok && rans_keep;
    clear_bins();
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// enc_rans: four interleaved lanes per shard, one thread per lane, eight
// shards per warp.  Lane bytes are written back to front so they end up in
// stream order (the reference reverses them at emission, encode.cu:609).

template <int PIPE, typename FoldT>
__global__ void __launch_bounds__(128)
enc_rans_kernel(const FrameState* __restrict__ state, const BatchDims* __restrict__ dims, int pass,
                ShardInfo* __restrict__ shards, const FoldT* __restrict__ folded,
                uint8_t* __restrict__ rans_scratch) {
  const int64_t total_shards = dims->shards_p[pass];
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t s = gid >> 2;
  const int lane = static_cast<int>(gid & 3);
  if (s >= total_shards) return;
  ShardInfo& si = shards[s];
  if (!state[si.frame].active || !si.rans_ok) return;
  const int n = si.count;
  const FoldT* __restrict__ f = folded + si.sample_base;
  uint8_t* base = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes);
  const uint2* __restrict__ tab = reinterpret_cast<const uint2*>(base);
  uint32_t* out_end = reinterpret_cast<uint32_t*>(base + kRansTableWords * 4 + kRansSerialBytes +
                                                  (lane + 1) * kRansLaneBytes);
  uint32_t x = kRansL;
  // pending bytes, earliest emitted in the highest position, as a 64-bit
  // value in two words (ahi:alo) moved by funnel shifts: a 64-bit variable
  // shift costs several instructions per step
  uint32_t ahi = 0, alo = 0;
  int nacc = 0, nwords = 0;
  const int first = n - 1 - ((n - 1 - lane) & 3);
  const int steps = first >= 0 ? first / 4 + 1 : 0;  // symbols first, first-4, ..., >= 0
  // one encoding step (encode.cu:401-418): renormalise -- at most two bytes,
  // since x < 2^31 and the threshold f * 2^19 >= 2^19 -- then the state map.
  // Pending bytes are written out a word at a time by flush(): after a pair
  // of steps (at most 3 + 4 = 7 pending, one word written leaves at most 3),
  // or after every step of an odd tail.
  auto step = [&](uint2 e) {
    const uint32_t cmpl = (e.y >> 13) & 0xfffu;
    const uint32_t thr = (4096u - cmpl) << 19;  // ((L >> 12) << 8) * f
    const uint32_t b1 = x >= thr, b2 = (x >> 8) >= thr;
    const int nb = static_cast<int>(b1 + b2);
    const uint32_t bytes = b2 ? __byte_perm(x, 0, 0x4401) : (x & 0xffu);  // first byte on top
    const uint32_t sh = 8u * static_cast<uint32_t>(nb);  // 0, 8 or 16
    ahi = __funnelshift_l(alo, ahi, sh);
    alo = (alo << sh) | (nb ? bytes : 0u);
    nacc += nb;
    x >>= sh;
    const uint32_t q = __umulhi(x, e.x) >> (e.y >> 25);
    x += (e.y & 0x1fffu) + q * cmpl;
  };
  auto flush = [&]() {
    if (nacc >= 4) {
      nacc -= 4;
      out_end[-(++nwords)] = __funnelshift_r(alo, ahi, 8 * nacc);  // (ahi:alo) >> 8 nacc, nacc 0..3
    }
  };
  int c = 0;
  if (PIPE == 0) {
    // symbols and table entries are loaded 16 steps ahead of the state chain
    constexpr int kAhead = 16;
    for (; c + kAhead <= steps; c += kAhead) {
      uint32_t v[kAhead];
      uint2 e[kAhead];
#pragma unroll
      for (int j = 0; j < kAhead; ++j) v[j] = ldf(f + first - 4 * (c + j));
#pragma unroll
      for (int j = 0; j < kAhead; ++j) e[j] = tab[v[j]];
#pragma unroll
      for (int j = 0; j < kAhead; j += 2) {
        step(e[j]);
        step(e[j + 1]);
        flush();
      }
    }
  } else {
    // Software pipeline over blocks of PIPE steps: while block b runs, the
    // table entries of block b+1 (whose symbols arrived a block earlier) and
    // the symbols of block b+2 are in flight, so neither the symbol load nor
    // the dependent table load sits on the state chain.
    constexpr int kB = PIPE > 0 ? PIPE : 2;  // even: steps go in pairs
    const int nblk = steps / kB;
    uint32_t vn[kB];      // symbols of block b+2
    uint2 en[kB], ec[kB];  // table entries of blocks b+1 and b
    auto load_v = [&](int b, uint32_t (&v)[kB]) {
#pragma unroll
      for (int j = 0; j < kB; ++j) v[j] = ldf(f + first - 4 * (b * kB + j));
    };
    if (nblk > 0) {
      load_v(0, vn);
#pragma unroll
      for (int j = 0; j < kB; ++j) ec[j] = tab[vn[j]];
    }
    if (nblk > 1) {
      load_v(1, vn);
#pragma unroll
      for (int j = 0; j < kB; ++j) en[j] = tab[vn[j]];
    }
    if (nblk > 2) load_v(2, vn);
    for (int b = 0; b < nblk; ++b) {
      uint2 cur[kB];
#pragma unroll
      for (int j = 0; j < kB; ++j) {
        cur[j] = ec[j];
        ec[j] = en[j];
      }
      if (b + 2 < nblk) {
#pragma unroll
        for (int j = 0; j < kB; ++j) en[j] = tab[vn[j]];
      }
      if (b + 3 < nblk) load_v(b + 3, vn);
#pragma unroll
      for (int j = 0; j < kB; j += 2) {
        step(cur[j]);
        step(cur[j + 1]);
        flush();
      }
    }
    c = nblk * kB;
  }
  for (; c < steps; ++c) {
    step(tab[ldf(f + first - 4 * c)]);
    flush();
  }
  if (nacc) out_end[-(nwords + 1)] = alo << (8 * (4 - nacc));  // low bytes unused
  si.rans_lane[lane] = 4 * nwords + nacc;
  si.rans_state[lane] = x;
}

// enc_rans with its loads either 16 steps ahead in one stage (PIPE 0) or
// pipelined over blocks of 8 or 16 steps (the autotuner's knob; identical
// bytes).
template <typename FoldT>
static void enc_rans_launch_t(int pipe, int grid, cudaStream_t stream, const FrameState* state,
                              const BatchDims* dims, int pass, ShardInfo* shards, const void* folded,
                              uint8_t* rans_scratch) {
  auto k = pipe == 8    ? enc_rans_kernel<8, FoldT>
           : pipe == 16 ? enc_rans_kernel<16, FoldT>
                        : enc_rans_kernel<0, FoldT>;
  k<<<grid, 128, 0, stream>>>(state, dims, pass, shards, static_cast<const FoldT*>(folded), rans_scratch);
}

void enc_rans_launch(int pipe, bool fold16, int grid, cudaStream_t stream, const FrameState* state,
                     const BatchDims* dims, int pass, ShardInfo* shards, const void* folded, uint8_t* rans_scratch) {
  if (fold16) enc_rans_launch_t<uint16_t>(pipe, grid, stream, state, dims, pass, shards, folded, rans_scratch);
  else enc_rans_launch_t<uint32_t>(pipe, grid, stream, state, dims, pass, shards, folded, rans_scratch);
}

void enc_analyze_launch(bool fold16, int grid, cudaStream_t stream, const FrameDesc* frames, FrameState* state,
                        const BatchDims* dims, int pass, ShardInfo* shards, const void* folded,
                        uint8_t* rans_scratch) {
  if (fold16)
    enc_analyze_kernel<uint16_t><<<grid, kWarpsPerCta * 32, 0, stream>>>(
        frames, state, dims, pass, shards, static_cast<const uint16_t*>(folded), rans_scratch);
  else
    enc_analyze_kernel<uint32_t><<<grid, kWarpsPerCta * 32, 0, stream>>>(
        frames, state, dims, pass, shards, static_cast<const uint32_t*>(folded), rans_scratch);
}

// ---------------------------------------------------------------------------
// enc_scan: one CTA per frame.  Final mode choice (encode.cu:420-430 and the
// kernel order at :789-805), exclusive scan of record sizes in shard order
// (:858-867), directory and header bytes (:871-904), frame policy (:812-847).

__device__ __forceinline__ void put32(uint8_t* p, uint32_t v) {
  p[0] = static_cast<uint8_t>(v);
  p[1] = static_cast<uint8_t>(v >> 8);
  p[2] = static_cast<uint8_t>(v >> 16);
  p[3] = static_cast<uint8_t>(v >> 24);
}

__global__ void __launch_bounds__(1024)
enc_scan_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                const BatchDims* __restrict__ dims, int pass, ShardInfo* __restrict__ shards,
                uint8_t* __restrict__ prefix) {
  const int nframes = dims->frames_p[pass];
  __shared__ int64_t warp_tot[32];
  __shared__ int64_t carry_s;
  const int fi = blockIdx.x;
  if (fi >= nframes) return;
  const FrameDesc& f = frames[fi];
  FrameState& st = state[fi];
  if (!st.active) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  ShardInfo* fs = shards + f.shard_base;
  for (int64_t base = 0; base < f.nshards; base += blockDim.x) {
    const int64_t s = base + threadIdx.x;
    int64_t rec = 0;
    if (s < f.nshards) {
      ShardInfo& si = fs[s];
      int mode = si.comp_mode, k = si.comp_k, body = si.comp_body;
      int lanes[4] = {si.comp_lane[0], si.comp_lane[1], si.comp_lane[2], si.comp_lane[3]};
      if (si.rans_ok) {
        const int rb = si.rans_table + 28 + si.rans_lane[0] + si.rans_lane[1] + si.rans_lane[2] + si.rans_lane[3];
        if (f.force_order0 || rb < body) {
          mode = kModeOrder0;
          k = kRansTableLog;
          body = rb;
          lanes[0] = si.rans_lane[0];
          lanes[1] = si.rans_lane[1];
          lanes[2] = si.rans_lane[2];
          lanes[3] = si.rans_lane[3];
        }
      }
      si.mode = mode;
      si.param = k;
      si.body = body;
      si.comp_lane[0] = lanes[0];
      si.comp_lane[1] = lanes[1];
      si.comp_lane[2] = lanes[2];
      si.comp_lane[3] = lanes[3];
      rec = body + 3;
    }
    // block exclusive scan
    int64_t inc = rec;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t v = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += v;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      int64_t w = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t v = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += v;
      }
      if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    const int64_t before = carry_s + (warp ? warp_tot[warp - 1] : 0) + inc - rec;
    if (s < f.nshards) fs[s].offset = f.prefix_bytes + before;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry_s = before + rec;
    __syncthreads();
  }
  const int64_t payload = carry_s;
  // directory (encode.cu:886-902)
  uint8_t* pre = prefix + f.prefix_base;
  for (int64_t t = threadIdx.x; t < f.ntiles; t += blockDim.x) {
    const TileGeo g = tile_geo(f, t);
    const int64_t off = fs[g.first_shard].offset;
    const int64_t end = (g.first_shard + g.shard_count < f.nshards) ? fs[g.first_shard + g.shard_count].offset
                                                                     : f.prefix_bytes + payload;
    uint8_t* e = pre + kHeaderBytes + t * kDirBytes;
    e[0] = static_cast<uint8_t>(g.plane);
    e[1] = kModeOrder0;
    e[2] = kPredictTag;
    e[3] = 0;
    put32(e + 4, g.x);
    put32(e + 8, g.y);
    put32(e + 12, g.w);
    put32(e + 16, g.h);
    put32(e + 20, static_cast<uint32_t>(off));
    put32(e + 24, static_cast<uint32_t>(static_cast<uint64_t>(off) >> 32));
    put32(e + 28, static_cast<uint32_t>(end - off));
    if (end - off > 0xffffffffll) set_status(&st.status, kStatusInternal + 1);  // "tile payload is too large"
  }
  if (threadIdx.x == 0) {
    // frame policy
    const int64_t N = f.nsamples;
    int next = 0;  // 0 done, 1 run again
    bool keep_a = false;  // the later pass lost: pass 0's records stand
    if (st.pass == 0) {
      st.baseline_payload = payload;
      if (f.layout == 0 && f.bit_depth == 10 && st.step > 1 && payload * 10 > N * 3) {
        st.gray_med = 1;
        st.use_med = 1;
        st.pass = 3;  // final pass with MED
        next = 1;
      } else if (f.layout == 0 && f.bit_depth == 16 && st.step > 1) {
        const bool direct = payload < N / 10 || payload > N / 2;
        const bool probe = !direct && payload < N / 5;
        if (direct || probe) {
          st.step = 1 + ((100 - f.quality) * 256 + 7) / 8;
          st.use_med = 0;
          st.pass = 1;
          next = 1;
        }
      }
    } else if (st.pass == 1) {
      // gray16 refined-step trial (its records are in region b)
      const int64_t b = st.baseline_payload;
      const bool direct = b < N / 10 || b > N / 2;
      if (direct || payload < N / 10) {
        st.refined = 1;
        st.final_b = 1;
      } else {
        // the reference re-encodes with the baseline step (encode.cu:840-845);
        // pass 0's records in region a are exactly that encoding
        st.step = f.step0;
        keep_a = true;
      }
    } else if (st.pass == 3) {
      st.final_b = 1;  // gray10 MED re-run: always final
    }
    st.payload = keep_a ? st.baseline_payload : payload;
    st.stream_len = f.prefix_bytes + st.payload;
    // header (encode.cu:871-885) -- written every pass, the last one stands
    pre[0] = 'F';
    pre[1] = 'V';
    pre[2] = 'I';
    pre[3] = 'D';
    pre[4] = 1;
    pre[5] = static_cast<uint8_t>(f.layout);
    pre[6] = static_cast<uint8_t>(f.quality);
    pre[7] = static_cast<uint8_t>((f.bit_depth - 8) | (st.gray_med ? 0x40 : 0) | (st.refined ? 0x80 : 0));
    put32(pre + 8, f.width);
    put32(pre + 12, f.height);
    pre[16] = static_cast<uint8_t>(f.tile_w);
    pre[17] = static_cast<uint8_t>(f.tile_w >> 8);
    pre[18] = static_cast<uint8_t>(f.tile_h);
    pre[19] = static_cast<uint8_t>(f.tile_h >> 8);
    put32(pre + 20, f.fps_num);
    put32(pre + 24, f.fps_den);
    put32(pre + 28, static_cast<uint32_t>(f.ntiles));
    // A failed pass stops the frame; otherwise the next pass runs only if the
    // policy asked for it.
    if (st.status != 0) next = 0;
    st.active = next;
  }
}

// Reset per-pass state before the first pass (device side, so batches need
// no host writes).
__global__ void enc_init_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                                const BatchDims* __restrict__ dims) {
  const int nframes = dims->frames_p[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nframes) return;
  FrameState s{};
  s.step = frames[i].step0;
  s.use_med = frames[i].use_med0;
  s.active = 1;
  state[i] = s;
}

// Before each re-run pass: reset the tile queue.  (Frames whose policy is
// finished keep active = 0 and are skipped by every kernel.)

// ---------------------------------------------------------------------------
// enc_emit: one warp per shard.  The record (mode byte, u16 body length,
// body) is assembled in shared memory -- bit codes merged with shared
// atomics, so no global atomics and no pre-zeroed output -- and copied out
// with aligned 32-bit stores plus byte stores at the two ragged ends.

// record buffer words: the largest record plus slack, rounded up to whole
// 16-byte vectors (so every warp's buffer is 16-byte aligned and is cleared
// with vector stores)
constexpr int kEmitWords = ((kMaxRecordBytes + 8 + 3) / 4 + 3) & ~3;

struct EmitWarpSmem {
  uint32_t buf[kEmitWords];
};
static_assert(sizeof(EmitWarpSmem) % 16 == 0, "record buffers must stay 16-byte aligned");

size_t enc_predict_smem(bool fold16) {
  return (fold16 ? sizeof(EncWarpSmem<uint16_t>) : sizeof(EncWarpSmem<uint32_t>)) * kWarpsPerCta;
}
size_t enc_emit_smem() { return sizeof(EmitWarpSmem) * kWarpsPerCta; }

// Every write into the record buffer is bounds-checked: a record can never
// outgrow kMaxRecordBytes, and a write past it is dropped rather than
// touching another warp's buffer.
__device__ __forceinline__ void or_bits(uint32_t* buf, int64_t bitpos, uint32_t bits, int nbits) {
  const int64_t w = bitpos >> 5;
  if (bitpos < 0 || w + 1 >= kEmitWords) return;
  const int sh = static_cast<int>(bitpos & 31);
  atomicOr(&buf[w], bits << sh);
  if (sh + nbits > 32) atomicOr(&buf[w + 1], bits >> (32 - sh));
}

__device__ __forceinline__ void put_byte(uint32_t* buf, int pos, uint32_t byte) {
  if (pos < 0 || (pos >> 2) >= kEmitWords) return;
  atomicOr(&buf[pos >> 2], (byte & 0xffu) << ((pos & 3) * 8));
}

// Record bytes [pos, pos+len) <- src[0, len) (global, any alignment).  Record
// word d (bytes 4d .. 4d+3) takes source bytes 4d-pos .. 4d-pos+3: the funnel
// shift of the two aligned source words that hold them, by the same amount
// for every d.  Each lane loads one source word; the word above it comes from
// the next lane (lane 31 loads its own), and the loads of two rounds of 32
// words are issued before either round is merged.  Words wholly inside the
// piece are plain stores; the two end words, which neighbouring pieces share,
// are merged with a shared atomic.  Only source words holding a byte of the
// piece are read.
__device__ __forceinline__ void put_bytes(uint32_t* buf, int pos, const uint8_t* __restrict__ src, int len, int lane) {
  if (len <= 0) return;
  const uintptr_t sa = reinterpret_cast<uintptr_t>(src);
  const uint32_t* __restrict__ sw = reinterpret_cast<const uint32_t*>(sa & ~static_cast<uintptr_t>(3));
  const int h = static_cast<int>(sa & 3);
  const int last_w = (h + len - 1) >> 2;  // last source word holding a piece byte
  const int qb = h - pos;                 // source byte index of record byte 4d is qb + 4d (>= -3)
  const int sh = 8 * (qb & 3);
  const int d0 = pos >> 2;
  const int d1 = min((pos + len - 1) >> 2, kEmitWords - 1);
  auto word = [&](int wi) { return (wi >= 0 && wi <= last_w) ? __ldg(sw + wi) : 0u; };
  for (int dd = d0; dd <= d1; dd += 64) {
    const int da = dd + lane, db = dd + 32 + lane;
    const int wa = (qb + 4 * da) >> 2, wb = (qb + 4 * db) >> 2;  // floor
    const uint32_t la = word(wa);
    const uint32_t lb = dd + 32 <= d1 ? word(wb) : 0u;
    const uint32_t ta = lane == 31 ? word(wa + 1) : 0u;
    const uint32_t tb = (lane == 31 && dd + 32 <= d1) ? word(wb + 1) : 0u;
    uint32_t ha = __shfl_down_sync(0xffffffffu, la, 1);
    uint32_t hb = __shfl_down_sync(0xffffffffu, lb, 1);
    if (lane == 31) {
      ha = ta;
      hb = tb;
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int d = r ? db : da;
      if (d > d1) continue;
      const uint32_t v = __funnelshift_r(r ? lb : la, r ? hb : ha, sh);
      const int s0 = 4 * d - pos;  // piece offset of record byte 4d (>= -3)
      if (s0 >= 0 && s0 + 3 < len) {
        buf[d] = v;
      } else {
        const int k0 = max(0, -s0), k1 = min(3, len - 1 - s0);
        const uint32_t mask = (0xffffffffu >> (8 * (3 - k1))) & (0xffffffffu << (8 * k0));
        atomicOr(&buf[d], v & mask);
      }
    }
  }
}

// put_bytes over the five pieces of an order-0 record held in memory (the
// serialised table, then the four lanes), with the loads of every piece's
// next 64 words issued before any is merged: the record then costs as many
// load latencies as its longest piece has rounds, not their sum.
__device__ __forceinline__ void put_pieces(uint32_t* buf, const uint8_t* const (&src)[5], const int (&pos)[5],
                                           const int (&len)[5], int lane) {
  int span = 0;  // destination words of the longest piece
#pragma unroll
  for (int i = 0; i < 5; ++i)
    if (len[i] > 0) span = max(span, ((pos[i] + len[i] - 1) >> 2) - (pos[i] >> 2) + 1);
  for (int off = 0; off < span; off += 64) {
    uint32_t la[5], lb[5], ta[5], tb[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const uintptr_t sa = reinterpret_cast<uintptr_t>(src[i]);
      const uint32_t* __restrict__ sw = reinterpret_cast<const uint32_t*>(sa & ~static_cast<uintptr_t>(3));
      const int h = static_cast<int>(sa & 3);
      const int last_w = len[i] > 0 ? (h + len[i] - 1) >> 2 : -1;
      const int qb = h - pos[i];
      const int d1 = len[i] > 0 ? min((pos[i] + len[i] - 1) >> 2, kEmitWords - 1) : -1;
      const int dd = (pos[i] >> 2) + off;
      auto word = [&](int wi) { return (wi >= 0 && wi <= last_w) ? __ldg(sw + wi) : 0u; };
      const int wa = (qb + 4 * (dd + lane)) >> 2, wb = (qb + 4 * (dd + 32 + lane)) >> 2;  // floor
      la[i] = dd <= d1 ? word(wa) : 0u;
      lb[i] = dd + 32 <= d1 ? word(wb) : 0u;
      ta[i] = (lane == 31 && dd <= d1) ? word(wa + 1) : 0u;
      tb[i] = (lane == 31 && dd + 32 <= d1) ? word(wb + 1) : 0u;
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int h = static_cast<int>(reinterpret_cast<uintptr_t>(src[i]) & 3);
      const int qb = h - pos[i];
      const int sh = 8 * (qb & 3);
      const int d1 = len[i] > 0 ? min((pos[i] + len[i] - 1) >> 2, kEmitWords - 1) : -1;
      const int dd = (pos[i] >> 2) + off;
      uint32_t ha = __shfl_down_sync(kFull, la[i], 1);
      uint32_t hb = __shfl_down_sync(kFull, lb[i], 1);
      if (lane == 31) {
        ha = ta[i];
        hb = tb[i];
      }
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int d = dd + 32 * r + lane;
        if (d > d1) continue;
        const uint32_t v = __funnelshift_r(r ? lb[i] : la[i], r ? hb : ha, sh);
        const int s0 = 4 * d - pos[i];  // piece offset of record byte 4d (>= -3)
        if (s0 >= 0 && s0 + 3 < len[i]) {
          buf[d] = v;
        } else {
          const int k0 = max(0, -s0), k1 = min(3, len[i] - 1 - s0);
          const uint32_t mask = (0xffffffffu >> (8 * (3 - k1))) & (0xffffffffu << (8 * k0));
          atomicOr(&buf[d], v & mask);
        }
      }
    }
  }
}

// Record bytes [pos, pos + 4n) <- the 32-bit little-endian values v held by
// lanes 0..n-1 (lane i's value at pos + 4i), merged with shared atomics.
__device__ __forceinline__ void put_words(uint32_t* buf, int pos, uint32_t v, int n, int lane) {
  if (lane >= n) return;
  const int p = pos + 4 * lane;
  const int w = p >> 2, sh = 8 * (p & 3);
  if (w < kEmitWords) atomicOr(&buf[w], v << sh);
  if (sh && w + 1 < kEmitWords) atomicOr(&buf[w + 1], v >> (32 - sh));
}

template <typename FoldT>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
enc_emit_kernel(const FrameState* __restrict__ state, EmitRegion ra, EmitRegion rb, int64_t total_shards,
                uint8_t* const* __restrict__ outs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* buf = reinterpret_cast<EmitWarpSmem*>(smem_raw)[warp].buf;
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp; s < total_shards; s += warps_total) {
    // the frame's records: pass 0's, or its later pass's (the shard record
    // of pass 0 names the frame either way).  Frames with a later pass come
    // first, so shards past region b's count skip the frame lookup.
    const bool from_b = s < rb.count && state[ra.shards[s].frame].final_b != 0;
    const ShardInfo& si = (from_b ? rb.shards : ra.shards)[s];
    {  // the next shard's record into L1 while this one is assembled
      const int64_t sn = s + warps_total;
      if (lane < 2 && sn < total_shards)  // its first and last byte: the record spans at most two lines
        asm volatile("prefetch.global.L1 [%0];" ::"l"(reinterpret_cast<const char*>(ra.shards + sn) +
                                                      (lane ? sizeof(ShardInfo) - 1 : 0)));
    }
    const FoldT* __restrict__ folded = static_cast<const FoldT*>(from_b ? rb.folded : ra.folded);
    const uint8_t* __restrict__ rans_scratch = from_b ? rb.rans_scratch : ra.rans_scratch;
    const int mode = si.mode, k = si.param, body = si.body, n = si.count;
    uint8_t* const dst_base = outs[si.frame];  // loaded now, used at the copy-out
    const int rec_len = min(body + 3, kMaxRecordBytes);
    const int nwords = (rec_len + 3) >> 2;
    // clear words 0 .. nwords (one past the record: the copy-out reads it)
    for (int i = lane; 4 * i <= nwords; i += 32) reinterpret_cast<uint4*>(buf)[i] = make_uint4(0, 0, 0, 0);
    __syncwarp();
    if (lane == 0) atomicOr(&buf[0], static_cast<uint32_t>(mode) | (static_cast<uint32_t>(body & 0xffff) << 8));
    const FoldT* __restrict__ f = folded + si.sample_base;
    if (mode == kModeZeroRun) {
      // Tokens in symbol order (encode.cu:514-536): a zero run of length L is
      // varint(2(L-1)), a value v is varint(2v-1).  A run's token is written
      // just before the value that ends it, or at the last symbol.  The warp
      // takes 128 symbols at a time, lane j holding symbols 4j..4j+3: the
      // zero run reaching a lane starts after the last nonzero symbol of the
      // lanes below (a ballot and one shuffle), the lane walks its four
      // symbols twice (token lengths, then bytes), and one warp scan of the
      // lengths places every lane's tokens.  The next 128 symbols are loaded
      // while these are placed.
      int cursor = 3;
      int run_start = 0;  // first index of the zero run reaching the chunk start
      const int nch = (n + 127) >> 7;
      uint32_t nx[4];
      auto load = [&](int m) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int idx = m * 128 + 4 * lane + c;
          nx[c] = idx < n ? ldf(f + idx) : 0u;
        }
      };
      load(0);
      for (int m = 0; m < nch; ++m) {
        const uint32_t v[4] = {nx[0], nx[1], nx[2], nx[3]};
        if (m + 1 < nch) load(m + 1);
        const int i0 = m * 128 + 4 * lane;
        int last_nz = -1;  // this lane's last nonzero symbol
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (v[c] != 0) last_nz = i0 + c;  // symbols past the end load as zero
        const uint32_t lanes_nz = __ballot_sync(kFull, last_nz >= 0);
        const uint32_t below = lanes_nz & ((1u << lane) - 1u);
        const int prev_nz = __shfl_sync(kFull, last_nz, below ? 31 - __clz(below) : 0);
        const int start = below ? prev_nz + 1 : run_start;
        // walk the lane's symbols: emit(t) is called for every token in order
        auto walk = [&](auto emit) {
          int st = start;
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int idx = i0 + c;
            if (idx >= n) break;
            if (v[c] != 0) {
              if (st < idx) emit(static_cast<uint32_t>(idx - st - 1) * 2);
              emit(v[c] * 2 - 1);
              st = idx + 1;
            } else if (idx == n - 1) {
              emit(static_cast<uint32_t>(idx - st) * 2);
            }
          }
        };
        int tlen = 0;
        walk([&](uint32_t t) { tlen += varint_len(t); });
        int inc = tlen;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int x = __shfl_up_sync(kFull, inc, o);
          if (lane >= o) inc += x;
        }
        int pos = cursor + inc - tlen;
        walk([&](uint32_t t) {
          do {
            uint32_t byte = t & 0x7f;
            t >>= 7;
            if (t) byte |= 0x80;
            put_byte(buf, pos++, byte);
          } while (t);
        });
        cursor += __shfl_sync(kFull, inc, 31);
        if (lanes_nz) run_start = __shfl_sync(kFull, last_nz, 31 - __clz(lanes_nz)) + 1;
      }
    } else if (mode >= kModeRiceBase && mode <= kModeRiceBase + kMaxRice) {
      // Rice lane c holds symbols c, c+4, ... (encode.cu:556-597; a shard of
      // n < 4 symbols has n lanes of one symbol).  The warp takes 256 symbols
      // at a time as two halves of 128, lane j holding symbols 4j..4j+3 of
      // each: component c of a half is then 32 consecutive codes of Rice
      // lane c, placed by one warp scan of their lengths; the eight scans of
      // a step are independent and run interleaved, and the second half's
      // codes follow the first's.  The next 256 symbols are loaded while
      // these are placed.
      const int lane_count = min(4, n);
      put_words(buf, 3, lane < lane_count - 1 ? static_cast<uint32_t>(si.comp_lane[lane]) : 0u, lane_count - 1,
                lane);
      int64_t bb[4];  // bit cursor of each Rice lane
      {
        int off = 3 + 4 * (lane_count - 1);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          bb[c] = 8 * static_cast<int64_t>(off);
          if (c < lane_count) off += si.comp_lane[c];
        }
      }
      const uint32_t rmask = k == 0 ? 0u : (1u << k) - 1u;
      const int nch = (n + 255) >> 8;
      uint32_t nx[8];  // element 4h + c: symbol 128h + 4 lane + c of the step
      auto load = [&](int m) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int idx = m * 256 + 128 * (i >> 2) + 4 * lane + (i & 3);
          nx[i] = idx < n ? ldf(f + idx) : 0u;
        }
      };
      load(0);
      for (int m = 0; m < nch; ++m) {
        uint32_t x[8], len[8], inc[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = nx[i];
        if (m + 1 < nch) load(m + 1);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const bool valid = m * 256 + 128 * (i >> 2) + 4 * lane + (i & 3) < n;
          len[i] = valid ? (x[i] >> k) + 1 + k : 0u;
          inc[i] = len[i];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const uint32_t t2 = __shfl_up_sync(kFull, inc[i], o);
            if (lane >= o) inc[i] += t2;
          }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t tot0 = __shfl_sync(kFull, inc[c], 31);
          const uint32_t tot1 = __shfl_sync(kFull, inc[4 + c], 31);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int i = 4 * h + c;
            if (len[i]) {
              const uint32_t v = x[i];
              const int64_t at = bb[c] + (h ? tot0 : 0u) + inc[i] - len[i] + (v >> k);
              or_bits(buf, at, 1u | ((v & rmask) << 1), k + 1);
            }
          }
          bb[c] += tot0 + tot1;
        }
      }
    } else if (mode == kModeBlockPack) {
      // widths and byte sizes of the (<= 32) blocks, one per lane
      const int nblk = (n + kBlockSymbols - 1) / kBlockSymbols;
      uint32_t my_w = 0;
      for (int b0 = 0; b0 < nblk; b0 += 4) {
        uint32_t mx[4] = {0, 0, 0, 0};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int i = 0; i < kBlockSymbols; i += 32) {
            const int idx = (b0 + u) * kBlockSymbols + i + lane;
            if (idx < n) mx[u] = max(mx[u], ldf(f + idx));
          }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint32_t m = __reduce_max_sync(kFull, mx[u]);
          if (lane == b0 + u) my_w = bitlen(m);
        }
      }
      const int my_n = lane < nblk ? min(kBlockSymbols, n - lane * kBlockSymbols) : 0;
      const uint32_t my_bytes = lane < nblk ? 1 + (my_n * my_w + 7) / 8 : 0;
      uint32_t inc = my_bytes;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t2 = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t2;
      }
      const uint32_t my_off = 3 + inc - my_bytes;
      if (lane < nblk) put_byte(buf, my_off, my_w);
      __syncwarp();
      for (int b = 0; b < nblk; ++b) {
        const uint32_t w = __shfl_sync(kFull, my_w, b);
        const uint32_t off = __shfl_sync(kFull, my_off, b);
        const int nb = min(kBlockSymbols, n - b * kBlockSymbols);
        if (w == 0) continue;
        for (int i = lane; i < nb; i += 32) {
          const uint32_t v = f[b * kBlockSymbols + i];  // FoldT widened
          or_bits(buf, static_cast<int64_t>(off + 1) * 8 + static_cast<int64_t>(i) * w, v, w);
        }
      }
    } else if (mode == kModeOrder0) {
      const uint8_t* base = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes);
      const uint8_t* ser = base + kRansTableWords * 4;
      const int tb = body - 28 - si.comp_lane[0] - si.comp_lane[1] - si.comp_lane[2] - si.comp_lane[3];
      // three lane lengths, then four final states: seven words from lanes 0..6
      const uint32_t lw = lane < 3 ? static_cast<uint32_t>(si.comp_lane[lane])
                                   : (lane < 7 ? si.rans_state[lane - 3] : 0u);
      put_words(buf, 3 + tb, lw, 7, lane);
      // the table at byte 3, the lanes after the 28 bytes of lengths and states
      const uint8_t* src[5];
      int pos[5], len[5];
      src[0] = ser;
      pos[0] = 3;
      len[0] = tb;
      int p = 31 + tb;
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        len[l + 1] = si.comp_lane[l];
        src[l + 1] = base + kRansTableWords * 4 + kRansSerialBytes + (l + 1) * kRansLaneBytes - len[l + 1];
        pos[l + 1] = p;
        p += len[l + 1];
      }
      put_pieces(buf, src, pos, len, lane);
    }
    __syncwarp();
    // copy out: record bytes [0, rec_len) -> out + offset; byte stores up to
    // the first 16-byte boundary of the destination, then one 16-byte store
    // per lane (five record words funnel-shifted), then the ragged tail
    uint8_t* dst = dst_base + si.offset;
    const uint8_t* bytes = reinterpret_cast<const uint8_t*>(buf);
    const int head = static_cast<int>((16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15);
    const int hb = min(head, rec_len);
    if (lane < hb) dst[lane] = bytes[lane];
    const int nvec = (rec_len - hb) >> 4;
    uint4* dv = reinterpret_cast<uint4*>(dst + hb);
    const int sh = 8 * (hb & 3);
    const int w0 = hb >> 2;
    for (int j = lane; j < nvec; j += 32) {
      const uint32_t* b = buf + w0 + 4 * j;  // words up to w0 + 4 nvec <= nwords
      const uint32_t a0 = b[0], a1 = b[1], a2 = b[2], a3 = b[3], a4 = b[4];
      dv[j] = make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh), __funnelshift_r(a2, a3, sh),
                         __funnelshift_r(a3, a4, sh));
    }
    const int tail_start = hb + nvec * 16;
    if (lane < rec_len - tail_start) dst[tail_start + lane] = bytes[tail_start + lane];
    __syncwarp();
  }
}

// Header + directory bytes of every frame into its output buffer (from the
// region whose records the frame emits).
__global__ void enc_prefix_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                  int nframes, const uint8_t* __restrict__ prefix, const uint8_t* __restrict__ prefix_b,
                                  uint8_t* const* __restrict__ outs) {
  const int fi = blockIdx.y;
  if (fi >= nframes) return;
  const FrameDesc& f = frames[fi];
  const uint8_t* src = (state[fi].final_b ? prefix_b : prefix) + f.prefix_base;
  uint8_t* dst = outs[fi];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < f.prefix_bytes;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

}  // namespace fvb

namespace fvb {
void enc_emit_launch(bool fold16, int grid, size_t smem, cudaStream_t stream, const FrameState* state,
                     EmitRegion a, EmitRegion b, int64_t total_shards, uint8_t* const* outs) {
  if (fold16)
    enc_emit_kernel<uint16_t><<<grid, kWarpsPerCta * 32, smem, stream>>>(state, a, b, total_shards, outs);
  else
    enc_emit_kernel<uint32_t><<<grid, kWarpsPerCta * 32, smem, stream>>>(state, a, b, total_shards, outs);
}

cudaError_t enc_emit_set_smem(int bytes) {
  cudaError_t e = cudaFuncSetAttribute(enc_emit_kernel<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(enc_emit_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
}  // namespace fvb
