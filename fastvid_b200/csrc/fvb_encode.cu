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

struct EncWarpSmem {
  uint16_t src[32 * kSrcStride];    // source ring (u16, skewed)
  uint32_t fold[32 * kFoldStride];  // folded-residual ring (u32, skewed)
  uint16_t carry[kFastMaxW + 128];  // row above the band, column c at index c + 32
};

template <bool MED, bool STEP1, bool EDGE>
__device__ __forceinline__ void enc_block(EncWarpSmem& sm, int lane, int t0, int W,
                                          int32_t maxs, int32_t step, int32_t half, uint32_t magic, bool band0,
                                          int32_t& rec, int32_t& a_prev) {
  const uint16_t* srow = sm.src + lane * kSrcStride + (t0 & 32);
  uint32_t* frow = sm.fold + lane * kFoldStride + (t0 & 32);
  uint16_t* crow = sm.carry + 32 - lane + t0;  // carry index (t - lane) + 32
#pragma unroll
  for (int u = 0; u < 32; ++u) {
    const int32_t s = srow[u];
    int32_t a = __shfl_up_sync(0xffffffffu, rec, 1);
    const int32_t above0 = crow[u];
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
      if (lane == 31 && c >= 0 && c < W) crow[u] = static_cast<uint16_t>(rn);
    } else {
      if (lane == 31) crow[u] = static_cast<uint16_t>(rn);
    }
    frow[u] = zigzag(q);
    a_prev = a;
    rec = rn;
  }
}

template <bool MED, bool STEP1>
__device__ void enc_tile_fast(const FrameDesc& f, const TileGeo& g, int32_t step, uint32_t magic,
                              uint32_t* __restrict__ folded_tile, EncWarpSmem& sm, int lane, int32_t& bad) {
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
    uint32_t* __restrict__ frows = folded_tile + static_cast<int64_t>(band * 32) * W;
    uint32_t pf[32];
    auto load_chunk = [&](int k) {
      const int col = k * 32 + lane;
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        pf[r] = (r < band_rows && col < W) ? rows[static_cast<int64_t>(r) * pitch + col] : 0u;
        vmax = max(vmax, pf[r]);
      }
    };
    auto store_chunk = [&](int k) {
      const int pj = k * 32 + lane;
#pragma unroll
      for (int r = 0; r < 32; ++r) sm.src[r * kSrcStride + ((pj + r) & 63)] = static_cast<uint16_t>(pf[r]);
    };
    auto flush_chunk = [&](int k) {
      const int col = k * 32 + lane;
      if (col < W) {
        for (int r = 0; r < band_rows; ++r)
          frows[static_cast<int64_t>(r) * W + col] = sm.fold[r * kFoldStride + ((col + r) & 63)];
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
      if (edge) enc_block<MED, STEP1, true>(sm, lane, t0, W, maxs, step, half, magic, band0, rec, a_prev);
      else enc_block<MED, STEP1, false>(sm, lane, t0, W, maxs, step, half, magic, band0, rec, a_prev);
    }
    __syncwarp();
    for (int j = max(0, nblocks - 2); j < nchunks; ++j) flush_chunk(j);
    __syncwarp();
  }
  if (vmax > static_cast<uint32_t>(maxs)) bad = 1;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32, 4)
enc_predict_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state, int nframes,
                   int64_t total_tiles, ShardInfo* __restrict__ shards, uint32_t* __restrict__ folded,
                   int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  EncWarpSmem& sm = reinterpret_cast<EncWarpSmem*>(smem_raw)[warp];
  for (;;) {
    int64_t t = 0;
    if (lane == 0) t = atomicAdd(queue, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= total_tiles) break;
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    FrameState& st = state[fi];
    if (!st.active) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    // shard records of this tile (encode.cu:753-759)
    for (int j = lane; j < g.shard_count; j += 32) {
      ShardInfo& si = shards[f.shard_base + g.first_shard + j];
      const int64_t local = static_cast<int64_t>(j) * kShardSymbols;
      si.sample_base = f.sample_base + g.sample_base + local;
      si.count = static_cast<int32_t>(min(static_cast<int64_t>(kShardSymbols), static_cast<int64_t>(g.w) * g.h - local));
      si.frame = fi;
    }
    if (g.w > kFastMaxW) continue;  // wide tiles go through enc_predict_wide_kernel
    const int32_t step = st.step;
    const uint32_t magic = step > 1 ? static_cast<uint32_t>((0x100000000ull + step - 1) / step) : 0u;
    uint32_t* ftile = folded + f.sample_base + g.sample_base;
    int32_t bad = 0;
    const bool med = st.use_med != 0;
    if (med) {
      if (step == 1) enc_tile_fast<true, true>(f, g, step, magic, ftile, sm, lane, bad);
      else enc_tile_fast<true, false>(f, g, step, magic, ftile, sm, lane, bad);
    } else {
      if (step == 1) enc_tile_fast<false, true>(f, g, step, magic, ftile, sm, lane, bad);
      else enc_tile_fast<false, false>(f, g, step, magic, ftile, sm, lane, bad);
    }
    if (__any_sync(kFull, bad) && lane == 0) set_status(&st.status, 1);
  }
}

// Tiles wider than kFastMaxW: one CTA per tile walks the antidiagonals with
// the reconstruction kept in global scratch (same order as the reference,
// encode.cu:150-192).  Only used for unusually wide tile sizes.
__global__ void enc_predict_wide_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                                        int nframes, int64_t total_tiles, uint32_t* __restrict__ folded,
                                        uint16_t* __restrict__ recon) {
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
    uint32_t* ftile = folded + f.sample_base + g.sample_base;
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
        ftile[i] = zigzag(q);
      }
      __syncthreads();
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_status(&st.status, 1);
  }
}

// ---------------------------------------------------------------------------
// enc_analyze: one warp per shard.  Lane l of chunk m holds symbol 32m+l, so
// its Rice lane is l % lane_count for every chunk.

__device__ __forceinline__ int bitlen(uint32_t v) { return 32 - __clz(v); }

__device__ __forceinline__ uint32_t warp_sum(uint32_t v) { return __reduce_add_sync(kFull, v); }

__global__ void __launch_bounds__(kWarpsPerCta * 32)
enc_analyze_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state, int nframes,
                   ShardInfo* __restrict__ shards, int64_t total_shards,
                   const uint32_t* __restrict__ folded, uint8_t* __restrict__ rans_scratch) {
  // Per warp: one histogram per Rice lane class (symbol i -> class i % 4) and
  // their total.  For shards whose values are all below 511 -- nearly every
  // shard -- the 17 Rice sums and the zero-run value cost come from the
  // histograms over the distinct values; only other shards take a second
  // per-sample pass.
  // class rows padded by 8 words: equal values of different classes fall in
  // different banks
  __shared__ uint32_t hcls_all[kWarpsPerCta][4][520];
  __shared__ uint32_t hist_all[kWarpsPerCta][512];
  __shared__ uint16_t list_all[kWarpsPerCta][512];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t (*hcls)[520] = hcls_all[warp];
  uint32_t* hist = hist_all[warp];
  uint16_t* list = list_all[warp];
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp; s < total_shards; s += warps_total) {
    ShardInfo& si = shards[s];
    const int fi = si.frame;
    FrameState& st = state[fi];
    if (!st.active) continue;
    const int n = si.count;
    const uint32_t* __restrict__ f = folded + si.sample_base;
    const int lane_count = min(4, n);
    for (int i = lane; i < 4 * 520; i += 32) hcls[0][i] = 0;
    __syncwarp();
    uint32_t sk[kMaxRice + 1];
#pragma unroll
    for (int k = 0; k <= kMaxRice; ++k) sk[k] = 0;
    uint32_t nz_cost = 0;           // per lane: varint bytes of nonzero values
    uint32_t runs = 0, long_runs = 0, cur_run = 0;  // warp-uniform
    uint32_t block_bytes = 0, bmax = 0, shard_max = 0, zc = 0;
    const int nchunk = (n + 31) >> 5;
    const uint32_t cls = static_cast<uint32_t>(lane & 3);
    // pass 1: zero runs, block widths, histograms; four chunks (one 128-symbol
    // pack block) per iteration, loads issued first
    for (int m0 = 0; m0 < nchunk; m0 += 4) {
     uint32_t vv[4];
#pragma unroll
     for (int j = 0; j < 4; ++j) {
       const int idx = (m0 + j) * 32 + lane;
       vv[j] = idx < n ? __ldg(f + idx) : 0u;
     }
#pragma unroll
     for (int j = 0; j < 4; ++j) {
      const int m = m0 + j;
      if (m >= nchunk) break;
      const int idx = m * 32 + lane;
      const bool valid = idx < n;
      const uint32_t v = vv[j];
      zc += valid && v == 0;
      // zero-run tokens (encode.cu:232-240): runs of zeros cost varint(2(run-1))
      const uint32_t z = __ballot_sync(kFull, valid && v == 0);
      const uint32_t vm = __ballot_sync(kFull, valid);
      const uint32_t starts = z & ~((z << 1) | (cur_run ? 1u : 0u));
      runs += __popc(starts);
      if (z == vm && vm == kFull) {
        if (cur_run <= 64 && cur_run + 32 > 64) ++long_runs;
        cur_run += 32;
      } else {
        const uint32_t lead = __ffs(~z) - 1;  // zeros continuing the carried run
        if (cur_run <= 64 && cur_run + lead > 64) ++long_runs;
        // trailing zeros up to the last valid symbol start (or extend) the carry
        const int top = 31 - __clz(vm);       // last valid lane
        const uint32_t zz = z << (31 - top);  // align last valid lane to bit 31
        cur_run = __clz(~zz);
      }
      // block pack: 4 chunks per 128-symbol block (encode.cu:249-259)
      bmax = max(bmax, v);
      if ((m & 3) == 3 || m == nchunk - 1) {
        const uint32_t bm = __reduce_max_sync(kFull, bmax);
        const int nb = min(kBlockSymbols, n - (m & ~3) * 32);
        block_bytes += 1 + (nb * bitlen(bm) + 7) / 8;
        shard_max = max(shard_max, bm);
        bmax = 0;
      }
      if (valid && v != 0 && v < kRansAlphabet) atomicAdd(&hcls[cls][v], 1u);
     }
    }
    // zeros per class (lanes with equal lane & 3 hold the same class)
    zc += __shfl_xor_sync(kFull, zc, 4);
    zc += __shfl_xor_sync(kFull, zc, 8);
    zc += __shfl_xor_sync(kFull, zc, 16);
    if (lane < 4) hcls[lane][0] = zc;
    __syncwarp();
    int distinct = 0;
    uint32_t present = 0;  // bit b: value 16*lane+b present
    uint32_t cnt_sum = 0;
    if (shard_max < kRansAlphabet) {
      // totals and the compact list of present values
#pragma unroll
      for (int b = 0; b < 16; ++b) {
        const int v = lane * 16 + b;
        const uint32_t h = hcls[0][v] + hcls[1][v] + hcls[2][v] + hcls[3][v];
        hist[v] = h;
        present |= (h != 0 ? 1u : 0u) << b;
        cnt_sum += h;
      }
      int rinc = __popc(present);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int r2 = __shfl_up_sync(kFull, rinc, o);
        if (lane >= o) rinc += r2;
      }
      int r = rinc - __popc(present);
      for (uint32_t pm = present; pm; pm &= pm - 1) list[r++] = static_cast<uint16_t>(lane * 16 + __ffs(pm) - 1);
      distinct = __shfl_sync(kFull, rinc, 31);
      __syncwarp();
      // Rice sums sum_i (v_i >> k) per class; v < 511 so only k <= 8 count
      uint32_t S[4][9];
#pragma unroll
      for (int l = 0; l < 4; ++l)
#pragma unroll
        for (int k = 0; k < 9; ++k) S[l][k] = 0;
      uint32_t nzc = 0;
      for (int e = lane; e < distinct; e += 32) {
        const uint32_t v = list[e];
        uint32_t tot = 0;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const uint32_t c = hcls[l][v];
          tot += c;
#pragma unroll
          for (int k = 0; k < 9; ++k) S[l][k] += c * (v >> k);
        }
        // value tokens varint(2v-1): one byte up to v = 64, two below 511
        nzc += v ? tot * (1u + (v > 64u)) : 0u;
      }
      const uint32_t nz_total = warp_sum(nzc);
      nz_cost = lane == 0 ? nz_total : 0u;
#pragma unroll
      for (int l = 0; l < 4; ++l)
#pragma unroll
        for (int k = 0; k < 9; ++k) {
          const uint32_t t = warp_sum(S[l][k]);
          if (lane == l) sk[k] = t;
        }
    } else {
      // pass 2: per-sample Rice sums and value costs
      for (int m = 0; m < nchunk; ++m) {
        const int idx = m * 32 + lane;
        const uint32_t v = idx < n ? __ldg(f + idx) : 0u;
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
    }
    const uint32_t zero_bytes = warp_sum(nz_cost) + runs + long_runs;
    // Rice: reduce the per-lane sums into the four lanes (symbol i -> lane i%4)
    int64_t best_bytes = INT64_MAX;
    int best_k = 0;
    uint32_t lane_bytes_best = 0;
    const int rl = lane & 3;
    const int nsym = rl < lane_count ? (n - rl + lane_count - 1) / lane_count : 0;
#pragma unroll
    for (int k = 0; k <= kMaxRice; ++k) {
      uint32_t v = sk[k];
      v += __shfl_xor_sync(kFull, v, 4);
      v += __shfl_xor_sync(kFull, v, 8);
      v += __shfl_xor_sync(kFull, v, 16);
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
    int mode;
    int64_t body;
    if (static_cast<int64_t>(block_bytes) < zero_bytes && static_cast<int64_t>(block_bytes) < rice_body) {
      mode = kModeBlockPack;
      body = block_bytes;
    } else if (static_cast<int64_t>(zero_bytes) <= rice_body) {
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
    // at most 255 distinct symbols.
    __syncwarp();
    int rans_ok = shard_max < kRansAlphabet;
    if (rans_ok) {
      if (distinct > 255) rans_ok = 0;
      if (rans_ok) {
        const int D = distinct;
        // exclusive prefix of counts and ranks over lanes
        uint32_t cinc = cnt_sum, rinc = __popc(present);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t c2 = __shfl_up_sync(kFull, cinc, o), r2 = __shfl_up_sync(kFull, rinc, o);
          if (lane >= o) {
            cinc += c2;
            rinc += r2;
          }
        }
        uint32_t P = cinc - cnt_sum;
        int rank = static_cast<int>(rinc) - __popc(present);
        // normalisation as a prefix maximum: for the i-th present symbol,
        // end_i = i + min(max(1, max_{j<=i}(f_j - j)), 4097 - D) with
        // f_j = floor(P_j * 4096 / n); the last symbol ends at 4096.  This
        // equals the reference's clamp loop (encode.cu:370-390): writing
        // u_i = end_i - i turns end_i = min(max(f_i, end_{i-1}+1), 4097-D+i)
        // into u_i = min(max(f_i - i, u_{i-1}), 4097-D) with u_{-1} = 1.
        int32_t dmax = INT32_MIN;
        {
          uint32_t p = P;
          int r = rank;
#pragma unroll
          for (int b = 0; b < 16; ++b) {
            const uint32_t h = hist[lane * 16 + b];
            if (h) {
              p += h;
              const int32_t fj = static_cast<int32_t>((p << kRansTableLog) / static_cast<uint32_t>(n));
              dmax = max(dmax, fj - r);
              ++r;
            }
          }
        }
        int32_t dinc = dmax;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t d2 = __shfl_up_sync(kFull, dinc, o);
          if (lane >= o) dinc = max(dinc, d2);
        }
        int32_t dpre = __shfl_up_sync(kFull, dinc, 1);
        if (lane == 0) dpre = INT32_MIN;
        // ends, cumulative starts and serialised table lengths
        uint32_t* tab = reinterpret_cast<uint32_t*>(rans_scratch + s * static_cast<int64_t>(kRansScratchBytes));
        const int G = 4097 - D;
        int32_t ends[16];
        int32_t run_max = dpre;
        uint32_t p = P;
        int r = rank;
        int32_t last_end_lane = 0;
#pragma unroll
        for (int b = 0; b < 16; ++b) {
          const uint32_t h = hist[lane * 16 + b];
          ends[b] = -1;
          if (h) {
            p += h;
            const int32_t fj = static_cast<int32_t>((p << kRansTableLog) / static_cast<uint32_t>(n));
            run_max = max(run_max, fj - r);
            ends[b] = (r == D - 1) ? (1 << kRansTableLog) : r + min(max(1, run_max), G);
            last_end_lane = ends[b];
            ++r;
          }
        }
        // previous end (cumulative) = exclusive prefix max of ends
        int32_t einc = last_end_lane;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t e2 = __shfl_up_sync(kFull, einc, o);
          if (lane >= o) einc = max(einc, e2);
        }
        int32_t prev_end = __shfl_up_sync(kFull, einc, 1);
        if (lane == 0) prev_end = 0;
        // previous present value (for table deltas): exclusive prefix max
        int32_t last_v = -1;
#pragma unroll
        for (int b = 0; b < 16; ++b)
          if (ends[b] >= 0) last_v = lane * 16 + b;
        int32_t vinc = last_v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t v2 = __shfl_up_sync(kFull, vinc, o);
          if (lane >= o) vinc = max(vinc, v2);
        }
        int32_t prev_v = __shfl_up_sync(kFull, vinc, 1);
        if (lane == 0 || prev_v < 0) prev_v = 0;
        // per-lane byte count of the serialised entries
        uint32_t my_bytes = 0;
        {
          int32_t pe = prev_end, pv = prev_v;
          int rr = rank;
#pragma unroll
          for (int b = 0; b < 16; ++b) {
            if (ends[b] >= 0) {
              const int v = lane * 16 + b;
              my_bytes += varint_len(static_cast<uint32_t>(v - pv));
              if (rr != D - 1) my_bytes += varint_len(static_cast<uint32_t>(ends[b] - pe));
              pe = ends[b];
              pv = v;
              ++rr;
            }
          }
        }
        uint32_t binc = my_bytes;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t b2 = __shfl_up_sync(kFull, binc, o);
          if (lane >= o) binc += b2;
        }
        const int head = 1 + varint_len(static_cast<uint32_t>(D));
        uint8_t* ser = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes) + kRansTableWords * 4;
        uint32_t cursor = head + binc - my_bytes;
        {
          int32_t pe = prev_end, pv = prev_v;
          int rr = rank;
#pragma unroll
          for (int b = 0; b < 16; ++b) {
            const int v = lane * 16 + b;
            if (ends[b] >= 0) {
              const uint32_t fr = static_cast<uint32_t>(ends[b] - pe);
              tab[2 * v] = (fr << 16) | static_cast<uint32_t>(pe);
              tab[2 * v + 1] = fr == 1 ? 0xffffffffu : static_cast<uint32_t>(0x100000000ull / fr);
              uint32_t d = static_cast<uint32_t>(v - pv);
              do {
                uint8_t byte = d & 0x7f;
                d >>= 7;
                if (d) byte |= 0x80;
                ser[cursor++] = byte;
              } while (d);
              if (rr != D - 1) {
                uint32_t e = fr;
                do {
                  uint8_t byte = e & 0x7f;
                  e >>= 7;
                  if (e) byte |= 0x80;
                  ser[cursor++] = byte;
                } while (e);
              }
              pe = ends[b];
              pv = v;
              ++rr;
            }
          }
        }
        if (lane == 31) {
          ser[0] = kRansTableLog;
          uint32_t d = static_cast<uint32_t>(D);
          int c = 1;
          do {
            uint8_t byte = d & 0x7f;
            d >>= 7;
            if (d) byte |= 0x80;
            ser[c++] = byte;
          } while (d);
          si.rans_table = head + static_cast<int32_t>(binc);
        }
      }
    }
    if (lane == 0) si.rans_ok = rans_ok;
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// enc_rans: four interleaved lanes per shard, one thread per lane, eight
// shards per warp.  Lane bytes are written back to front so they end up in
// stream order (the reference reverses them at emission, encode.cu:609).

// Division of a rANS state x < 2^31 by a frequency f <= 4096: q' = mulhi(x, m)
// with m = floor(2^32 / f) (m = 2^32 - 1 for f = 1) is floor(x / f) or one
// less, since x*m/2^32 > x/f - x/2^32 > x/f - 1; one compare fixes it and
// yields the remainder as well (reciprocal division with a correction step,
// Granlund & Montgomery, PLDI 1994).
__device__ __forceinline__ void div_freq(uint32_t x, uint32_t f, uint32_t m, uint32_t& q, uint32_t& r) {
  q = __umulhi(x, m);
  r = x - q * f;
  if (r >= f) {
    ++q;
    r -= f;
  }
}

__global__ void __launch_bounds__(128)
enc_rans_kernel(const FrameState* __restrict__ state, ShardInfo* __restrict__ shards, int64_t total_shards,
                const uint32_t* __restrict__ folded, uint8_t* __restrict__ rans_scratch) {
  const int64_t gid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t s = gid >> 2;
  const int lane = static_cast<int>(gid & 3);
  if (s >= total_shards) return;
  ShardInfo& si = shards[s];
  if (!state[si.frame].active || !si.rans_ok) return;
  const int n = si.count;
  const uint32_t* __restrict__ f = folded + si.sample_base;
  uint8_t* base = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes);
  const uint2* __restrict__ tab = reinterpret_cast<const uint2*>(base);
  uint32_t* out_end = reinterpret_cast<uint32_t*>(base + kRansTableWords * 4 + kRansSerialBytes +
                                                  (lane + 1) * kRansLaneBytes);
  uint32_t x = kRansL;
  uint64_t acc = 0;  // pending bytes, earliest emitted in the highest position
  int nacc = 0, nwords = 0;
  const int first = n - 1 - ((n - 1 - lane) & 3);
  const int steps = first >= 0 ? first / 4 + 1 : 0;  // symbols first, first-4, ..., >= 0
  constexpr int kAhead = 8;
  for (int c = 0; c < steps; c += kAhead) {
    uint32_t v[kAhead];
    uint2 e[kAhead];
#pragma unroll
    for (int j = 0; j < kAhead; ++j) v[j] = (c + j < steps) ? __ldg(f + first - 4 * (c + j)) : 0u;
#pragma unroll
    for (int j = 0; j < kAhead; ++j) e[j] = (c + j < steps) ? tab[v[j]] : make_uint2(1u << 16, 0u);
#pragma unroll
    for (int j = 0; j < kAhead; ++j) {
      if (c + j < steps) {
        const uint32_t fr = e[j].x >> 16, cum = e[j].x & 0xffffu;
        const uint32_t thr = fr << 19;  // ((L >> 12) << 8) * freq
        // renormalise: at most two bytes, since x < 2^31 and thr >= 2^19
        const uint32_t b1 = x >= thr, b2 = (x >> 8) >= thr;
        const int nb = static_cast<int>(b1 + b2);
        const uint64_t bytes = b2 ? (((x & 0xffu) << 8) | ((x >> 8) & 0xffu)) : (x & 0xffu);
        acc = (acc << (8 * nb)) | (nb ? bytes : 0u);
        nacc += nb;
        if (nacc >= 4) {
          nacc -= 4;
          out_end[-(++nwords)] = static_cast<uint32_t>(acc >> (8 * nacc));
        }
        x >>= 8 * nb;
        uint32_t q, r;
        div_freq(x, fr, e[j].y, q, r);
        x = (q << kRansTableLog) + r + cum;
      }
    }
  }
  if (nacc) out_end[-(nwords + 1)] = static_cast<uint32_t>(acc << (8 * (4 - nacc)));  // low bytes unused
  si.rans_lane[lane] = 4 * nwords + nacc;
  si.rans_state[lane] = x;
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
enc_scan_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state, int nframes,
                ShardInfo* __restrict__ shards, uint8_t* __restrict__ prefix) {
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
      const int64_t b = st.baseline_payload;
      const bool direct = b < N / 10 || b > N / 2;
      if (direct || payload < N / 10) {
        st.refined = 1;
      } else {
        st.step = f.step0;
        st.use_med = 0;
        st.pass = 2;
        next = 1;
      }
    }
    st.payload = payload;
    st.stream_len = f.prefix_bytes + payload;
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
__global__ void enc_init_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state, int nframes) {
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

struct EmitWarpSmem {
  uint32_t buf[(kMaxRecordBytes + 8 + 3) / 4];
};
static_assert(sizeof(EmitWarpSmem) % 16 == 0 || true, "");

size_t enc_predict_smem() { return sizeof(EncWarpSmem) * kWarpsPerCta; }
size_t enc_emit_smem() { return sizeof(EmitWarpSmem) * kWarpsPerCta; }

constexpr int kEmitWords = (kMaxRecordBytes + 8 + 3) / 4;

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

__global__ void __launch_bounds__(kWarpsPerCta * 32)
enc_emit_kernel(const FrameDesc* __restrict__ frames, int nframes, const ShardInfo* __restrict__ shards,
                int64_t total_shards, const uint32_t* __restrict__ folded,
                const uint8_t* __restrict__ rans_scratch, uint8_t* const* __restrict__ outs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* buf = reinterpret_cast<EmitWarpSmem*>(smem_raw)[warp].buf;
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp; s < total_shards; s += warps_total) {
    const ShardInfo& si = shards[s];
    const int mode = si.mode, k = si.param, body = si.body, n = si.count;
    const int rec_len = min(body + 3, kMaxRecordBytes);
    const int nwords = (rec_len + 3) >> 2;
    for (int i = lane; i <= nwords; i += 32) buf[i] = 0;
    __syncwarp();
    if (lane == 0) atomicOr(&buf[0], static_cast<uint32_t>(mode) | (static_cast<uint32_t>(body & 0xffff) << 8));
    const uint32_t* __restrict__ f = folded + si.sample_base;
    if (mode == kModeZeroRun) {
      // Tokens in symbol order (encode.cu:514-536): a zero run of length L is
      // varint(2(L-1)), a value v is varint(2v-1).  A run's token is written
      // just before the value that ends it, or at the last symbol.
      int cursor = 3;
      int run_start = 0;  // first index of the zero run reaching the chunk start
      const int nchunk = (n + 31) >> 5;
      for (int m = 0; m < nchunk; ++m) {
        const int idx = m * 32 + lane;
        const bool valid = idx < n;
        const uint32_t v = valid ? f[idx] : 1u;  // past the end acts as a terminator
        const uint32_t nzm = __ballot_sync(kFull, v != 0);
        const uint32_t below = nzm & ((1u << lane) - 1u);
        const int start = below ? m * 32 + (31 - __clz(below)) + 1 : run_start;
        uint32_t t1 = 0, t2 = 0;
        int l1 = 0, l2 = 0;
        if (valid && v != 0) {
          if (start < idx) {  // the preceding symbol was zero: close its run
            t1 = static_cast<uint32_t>(idx - start - 1) * 2;
            l1 = varint_len(t1);
          }
          t2 = v * 2 - 1;
          l2 = varint_len(t2);
        } else if (valid && idx == n - 1) {
          t1 = static_cast<uint32_t>(idx - start) * 2;
          l1 = varint_len(t1);
        }
        const int tlen = l1 + l2;
        int inc = tlen;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int x = __shfl_up_sync(kFull, inc, o);
          if (lane >= o) inc += x;
        }
        int pos = cursor + inc - tlen;
        for (int b = 0; b < l1; ++b) {
          uint32_t byte = t1 & 0x7f;
          t1 >>= 7;
          if (t1) byte |= 0x80;
          put_byte(buf, pos++, byte);
        }
        for (int b = 0; b < l2; ++b) {
          uint32_t byte = t2 & 0x7f;
          t2 >>= 7;
          if (t2) byte |= 0x80;
          put_byte(buf, pos++, byte);
        }
        cursor += __shfl_sync(kFull, inc, 31);
        run_start = nzm ? m * 32 + (31 - __clz(nzm)) + 1 : run_start;
      }
    } else if (mode >= kModeRiceBase && mode <= kModeRiceBase + kMaxRice) {
      const int lane_count = min(4, n);
      int64_t lane_off = 3 + static_cast<int64_t>(lane_count - 1) * 4;
      if (lane < lane_count - 1) {
        const uint32_t lb = static_cast<uint32_t>(si.comp_lane[lane]);
        for (int b = 0; b < 4; ++b) put_byte(buf, 3 + lane * 4 + b, lb >> (8 * b));
      }
      const uint32_t rmask = k == 0 ? 0u : (1u << k) - 1u;
      for (int l = 0; l < lane_count; ++l) {
        const int lsym = (n - l + lane_count - 1) / lane_count;
        int64_t bitbase = lane_off * 8;
        for (int g0 = 0; g0 < lsym; g0 += 32) {
          const int li = g0 + lane;
          const bool valid = li < lsym;
          const uint32_t v = valid ? f[l + li * lane_count] : 0u;
          const uint32_t q = v >> k;
          const uint32_t len = valid ? q + 1 + k : 0u;
          uint32_t inc = len;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t2 = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += t2;
          }
          if (valid) {
            const int64_t pos = bitbase + inc - len + q;
            or_bits(buf, pos, 1u | ((v & rmask) << 1), k + 1);
          }
          bitbase += __shfl_sync(kFull, inc, 31);
        }
        lane_off += si.comp_lane[l];
      }
    } else if (mode == kModeBlockPack) {
      // widths and byte sizes of the (<= 32) blocks, one per lane
      const int nblk = (n + kBlockSymbols - 1) / kBlockSymbols;
      uint32_t my_w = 0;
      for (int b = 0; b < nblk; ++b) {
        uint32_t mx = 0;
        for (int i = lane; i < kBlockSymbols && b * kBlockSymbols + i < n; i += 32) mx = max(mx, f[b * kBlockSymbols + i]);
        mx = __reduce_max_sync(kFull, mx);
        if (lane == b) my_w = bitlen(mx);
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
          const uint32_t v = f[b * kBlockSymbols + i];
          or_bits(buf, static_cast<int64_t>(off + 1) * 8 + static_cast<int64_t>(i) * w, v, w);
        }
      }
    } else if (mode == kModeOrder0) {
      const uint8_t* base = rans_scratch + s * static_cast<int64_t>(kRansScratchBytes);
      const uint8_t* ser = base + kRansTableWords * 4;
      const int tb = body - 28 - si.comp_lane[0] - si.comp_lane[1] - si.comp_lane[2] - si.comp_lane[3];
      for (int i = lane; i < tb; i += 32) put_byte(buf, 3 + i, ser[i]);
      int pos = 3 + tb;
      if (lane < 3) {
        for (int b = 0; b < 4; ++b) put_byte(buf, pos + lane * 4 + b, static_cast<uint32_t>(si.comp_lane[lane]) >> (8 * b));
      }
      pos += 12;
      if (lane < 4) {
        for (int b = 0; b < 4; ++b) put_byte(buf, pos + lane * 4 + b, si.rans_state[lane] >> (8 * b));
      }
      pos += 16;
      for (int l = 0; l < 4; ++l) {
        const int len = si.comp_lane[l];
        const uint8_t* lane_end = base + kRansTableWords * 4 + kRansSerialBytes + (l + 1) * kRansLaneBytes;
        for (int i = lane; i < len; i += 32) put_byte(buf, pos + i, lane_end[i - len]);
        pos += len;
      }
    }
    __syncwarp();
    // copy out: record bytes [0, rec_len) -> out + offset
    uint8_t* dst = outs[si.frame] + si.offset;
    const uint8_t* bytes = reinterpret_cast<const uint8_t*>(buf);
    const int head = static_cast<int>((4 - (reinterpret_cast<uintptr_t>(dst) & 3)) & 3);
    const int hb = min(head, rec_len);
    if (lane < hb) dst[lane] = bytes[lane];
    const int body_words = (rec_len - hb) >> 2;
    uint32_t* dw = reinterpret_cast<uint32_t*>(dst + hb);
    const int sh = hb * 8;
    for (int j = lane; j < body_words; j += 32) {
      const uint32_t lo = buf[j], hi = buf[j + 1];
      dw[j] = sh ? __funnelshift_r(lo, hi, sh) : lo;
    }
    const int tail_start = hb + body_words * 4;
    if (lane < rec_len - tail_start) dst[tail_start + lane] = bytes[tail_start + lane];
    __syncwarp();
  }
}

// Header + directory bytes of every frame into its output buffer.
__global__ void enc_prefix_kernel(const FrameDesc* __restrict__ frames, int nframes,
                                  const uint8_t* __restrict__ prefix, uint8_t* const* __restrict__ outs) {
  const int fi = blockIdx.y;
  if (fi >= nframes) return;
  const FrameDesc& f = frames[fi];
  const uint8_t* src = prefix + f.prefix_base;
  uint8_t* dst = outs[fi];
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < f.prefix_bytes;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

}  // namespace fvb
