// fvb_decode.cu -- sm_100a decoder kernels for the fastvid intra codec.
//
//   dec_parse        : thread-per-tile directory + shard-header walk
//                      (reference decode.cu:131-220)
//   dec_shards       : warp-per-shard entropy decode of every mode with every
//                      rejection rule of the reference (decode.cu:222-550)
//   dec_reconstruct  : warp-per-tile register wavefront, the mirror of
//                      enc_predict (decode.cu:552-606)
//   dec_reconstruct_serial : one thread per tile, raster order
//                      (decode.cu:608-656; the predictor="serial" diagnostic)
// A frame whose parse failed is skipped by the later kernels, so they never
// read shard records that were not written.
#include "fvb_common.cuh"
#include "fvb_kernels.cuh"

namespace fvb {

namespace {
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

__device__ __forceinline__ uint32_t rd16(const uint8_t* p) { return p[0] | (static_cast<uint32_t>(p[1]) << 8); }
__device__ __forceinline__ uint32_t rd32(const uint8_t* p) {
  return p[0] | (static_cast<uint32_t>(p[1]) << 8) | (static_cast<uint32_t>(p[2]) << 16) |
         (static_cast<uint32_t>(p[3]) << 24);
}
__device__ __forceinline__ uint64_t rd64(const uint8_t* p) {
  return rd32(p) | (static_cast<uint64_t>(rd32(p + 4)) << 32);
}
}  // namespace

// ---------------------------------------------------------------------------
// dec_parse: directory entry checks (status 10) and shard header walk
// (status 11), one thread per tile.

__global__ void dec_parse_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state, int nframes,
                                 int64_t total_tiles, ShardInfo* __restrict__ shards) {
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total_tiles;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    FrameState& st = state[fi];
    const int64_t lt = t - f.tile_base;
    const TileGeo g = tile_geo(f, lt);
    const uint8_t* enc = f.stream;
    const int64_t size = f.stream_len;
    const int64_t dir_end = kHeaderBytes + f.ntiles * kDirBytes;
    const uint8_t* e = enc + kHeaderBytes + lt * kDirBytes;
    if (e[0] != g.plane || e[1] != kModeOrder0 || e[2] != kPredictTag || e[3] != 0 ||
        rd32(e + 4) != static_cast<uint32_t>(g.x) || rd32(e + 8) != static_cast<uint32_t>(g.y) ||
        rd32(e + 12) != static_cast<uint32_t>(g.w) || rd32(e + 16) != static_cast<uint32_t>(g.h)) {
      set_status(&st.status, 10);
      continue;
    }
    const uint64_t off_u = rd64(e + 20);
    if (off_u > static_cast<uint64_t>(size)) {
      set_status(&st.status, 10);
      continue;
    }
    const int64_t off = static_cast<int64_t>(off_u);
    const int64_t plen = rd32(e + 28);
    if (plen > size - off) {
      set_status(&st.status, 10);
      continue;
    }
    if (lt == 0) {
      if (off != dir_end) {
        set_status(&st.status, 10);
        continue;
      }
    } else {
      const uint64_t poff = rd64(e - kDirBytes + 20);
      const uint64_t plen2 = rd32(e - kDirBytes + 28);
      if (poff > static_cast<uint64_t>(size) || plen2 > static_cast<uint64_t>(size) - poff || off_u != poff + plen2) {
        set_status(&st.status, 10);
        continue;
      }
    }
    if (lt + 1 == f.ntiles && off + plen != size) {
      set_status(&st.status, 10);
      continue;
    }
    const int64_t samples = static_cast<int64_t>(g.w) * g.h;
    const int64_t tile_end = off + plen;
    int64_t cursor = off, decoded = 0;
    bool ok = true;
    for (int j = 0; j < g.shard_count; ++j) {
      if (cursor > tile_end - 3) {
        ok = false;
        break;
      }
      const int mode = enc[cursor];
      const int64_t bl = rd16(enc + cursor + 1);
      const int64_t bo = cursor + 3;
      if (mode > 19 || bl > tile_end - bo) {
        ok = false;
        break;
      }
      const int64_t cnt = min(static_cast<int64_t>(kShardSymbols), samples - decoded);
      ShardInfo& si = shards[f.shard_base + g.first_shard + j];
      si.mode = mode;
      si.offset = bo;
      si.body = static_cast<int32_t>(bl);
      si.count = static_cast<int32_t>(cnt);
      si.sample_base = f.sample_base + g.sample_base + decoded;
      si.frame = fi;
      decoded += cnt;
      cursor = bo + bl;
    }
    if (!ok || decoded != samples || cursor != tile_end) set_status(&st.status, 11);
  }
}

// ---------------------------------------------------------------------------
// dec_shards: one warp per shard.

struct DecWarpSmem {
  uint8_t table[1 << kRansTableLog];
  uint16_t values[256], freq[256], cum[256];
  int32_t lane_start[4], lane_len[4];
  uint32_t states[4];
  int32_t nsym, valid;
  int32_t boff[32], bwidth[32];
};

// Rice lane reader with a 64-bit bit buffer (decode.cu:63-125 semantics).
struct RiceReader {
  const uint8_t* bytes;
  int64_t len, bp, pos;
  uint64_t buf;
  int nb;
  __device__ void refill() {
    while (nb <= 56 && bp < len) {
      buf |= static_cast<uint64_t>(bytes[bp++]) << nb;
      nb += 8;
    }
  }
  __device__ bool read(int k, uint32_t maxf, uint32_t* out) {
    uint32_t q = 0;
    for (;;) {
      if (nb == 0) {
        refill();
        if (nb == 0) return false;
      }
      if (buf == 0) {
        q += nb;
        pos += nb;
        nb = 0;
        if (q > maxf) return false;
        continue;
      }
      const int z = __ffsll(static_cast<long long>(buf)) - 1;
      q += z;
      const int used = z + 1;
      buf = used == 64 ? 0 : buf >> used;
      nb -= used;
      pos += used;
      if (q > maxf) return false;
      break;
    }
    if (nb < k) refill();
    if (nb < k) return false;
    const uint32_t r = k ? static_cast<uint32_t>(buf) & ((1u << k) - 1u) : 0u;
    buf >>= k;
    nb -= k;
    pos += k;
    const uint64_t v = (static_cast<uint64_t>(q) << k) + r;
    if (v > maxf) return false;
    *out = static_cast<uint32_t>(v);
    return true;
  }
};

__device__ bool read_varint_strict(const uint8_t* body, int64_t len, int64_t* cursor, uint32_t* value) {
  uint32_t result = 0;
  int shift = 0;
  for (int used = 0; used < 5; ++used) {
    if (*cursor >= len) return false;
    const uint8_t byte = body[(*cursor)++];
    if (used == 4 && byte > 0x0f) return false;
    result |= static_cast<uint32_t>(byte & 0x7f) << shift;
    if ((byte & 0x80) == 0) {
      if (varint_len(result) != used + 1) return false;
      *value = result;
      return true;
    }
    shift += 7;
  }
  return false;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32)
dec_shards_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                  const ShardInfo* __restrict__ shards, int64_t total_shards, uint32_t* __restrict__ folded) {
  __shared__ DecWarpSmem smem_all[kWarpsPerCta];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  DecWarpSmem& sm = smem_all[warp];
  const int64_t warps_total = static_cast<int64_t>(gridDim.x) * kWarpsPerCta;
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * kWarpsPerCta + warp; s < total_shards; s += warps_total) {
    const ShardInfo& si = shards[s];
    const int fi = si.frame;
    FrameState& st = state[fi];
    if (st.status != 0) continue;  // parse failed: shard records may be incomplete
    const FrameDesc& f = frames[fi];
    const uint32_t maxf = static_cast<uint32_t>(f.max_sample) * 2u;
    const int mode = si.mode;
    const int64_t blen = si.body;
    const int64_t n = si.count;
    const uint8_t* __restrict__ body = f.stream + si.offset;
    uint32_t* __restrict__ out = folded + si.sample_base;
    if (mode == 0) {
      // zero-run varints (decode.cu:237-295)
      if (lane == 0) {
        int64_t cursor = 0, produced = 0;
        int err = 0;
        while (produced < n && !err) {
          uint32_t token = 0;
          int shift = 0, used = 0;
          for (;;) {
            if (cursor >= blen || used == 5) {
              err = 1;
              break;
            }
            const uint8_t byte = body[cursor++];
            if (used == 4 && byte > 0x0f) {
              err = 1;
              break;
            }
            token |= static_cast<uint32_t>(byte & 0x7f) << shift;
            ++used;
            if ((byte & 0x80) == 0) break;
            shift += 7;
          }
          if (err) break;
          if (used != varint_len(token)) {
            err = 1;
            break;
          }
          if ((token & 1) == 0) {
            const int64_t run = static_cast<int64_t>(token / 2) + 1;
            if (run > n - produced) {
              err = 1;
              break;
            }
            for (int64_t i = 0; i < run; ++i) out[produced++] = 0;
          } else {
            const uint32_t value = (token + 1) / 2;
            if (value == 0 || value > maxf) {
              err = 1;
              break;
            }
            out[produced++] = value;
          }
        }
        if (err || cursor != blen) set_status(&st.status, 1);
      }
    } else if (mode >= 1 && mode <= 17) {
      // Rice lanes (decode.cu:297-340)
      const int lc = static_cast<int>(n < 4 ? n : 4);
      const int64_t table = static_cast<int64_t>(lc - 1) * 4;
      if (table > blen) {
        if (lane == 0) set_status(&st.status, 2);
      } else if (lane < lc) {
        int64_t loff = table;
        for (int i = 0; i < lane; ++i) loff += rd32(body + i * 4);
        const int64_t llen = lane + 1 < lc ? static_cast<int64_t>(rd32(body + lane * 4)) : blen - loff;
        bool ok = !(loff > blen || llen < 0 || llen > blen - loff);
        if (ok) {
          RiceReader rr{body + loff, llen, 0, 0, 0ull, 0};
          const int k = mode - 1;
          for (int64_t idx = lane; idx < n; idx += lc) {
            uint32_t v;
            if (!rr.read(k, maxf, &v)) {
              ok = false;
              break;
            }
            out[idx] = v;
          }
          if (ok) {
            const int64_t used = (rr.pos + 7) / 8;
            if (used != llen) ok = false;
            else if ((rr.pos & 7) != 0) {
              const uint8_t mask = static_cast<uint8_t>(~((1u << (rr.pos & 7)) - 1u));
              if (body[loff + used - 1] & mask) ok = false;
            }
          }
        }
        if (!ok) set_status(&st.status, 2);
      }
    } else if (mode == 18) {
      // block pack (decode.cu:342-396): walk the width bytes, then decode
      // the blocks warp-wide
      const int nblk = static_cast<int>((n + kBlockSymbols - 1) / kBlockSymbols);
      const int maxw = 32 - __clz(maxf);
      if (lane == 0) {
        int64_t cursor = 0;
        int ok = 1;
        for (int b = 0; b < nblk; ++b) {
          if (cursor >= blen) {
            ok = 0;
            break;
          }
          const int w = body[cursor++];
          if (w > maxw) {
            ok = 0;
            break;
          }
          const int64_t nb = min(static_cast<int64_t>(kBlockSymbols), n - static_cast<int64_t>(b) * kBlockSymbols);
          const int64_t pay = (nb * w + 7) / 8;
          if (pay > blen - cursor) {
            ok = 0;
            break;
          }
          sm.boff[b] = static_cast<int32_t>(cursor);
          sm.bwidth[b] = w;
          // padding bits of the block's last byte must be zero
          const int64_t bits = nb * w;
          if ((bits & 7) != 0) {
            const uint8_t mask = static_cast<uint8_t>(~((1u << (bits & 7)) - 1u));
            if (body[cursor + pay - 1] & mask) {
              ok = 0;
              break;
            }
          }
          cursor += pay;
        }
        if (ok && cursor != blen) ok = 0;
        sm.valid = ok;
        if (!ok) set_status(&st.status, 3);
      }
      __syncwarp();
      if (sm.valid) {
        int bad = 0;
        for (int b = 0; b < nblk; ++b) {
          const int w = sm.bwidth[b];
          const uint8_t* pay = body + sm.boff[b];
          const int nb = static_cast<int>(min(static_cast<int64_t>(kBlockSymbols), n - static_cast<int64_t>(b) * kBlockSymbols));
          for (int i = lane; i < nb; i += 32) {
            uint32_t v = 0;
            if (w) {
              const int64_t bit = static_cast<int64_t>(i) * w;
              const int64_t byte0 = bit >> 3;
              const int64_t last = (bit + w - 1) >> 3;
              uint64_t acc = 0;
              for (int64_t j = byte0; j <= last; ++j) acc |= static_cast<uint64_t>(pay[j]) << (8 * (j - byte0));
              v = static_cast<uint32_t>((acc >> (bit & 7)) & ((w == 32) ? 0xffffffffull : ((1ull << w) - 1)));
            }
            if (v > maxf) bad = 1;
            out[static_cast<int64_t>(b) * kBlockSymbols + i] = v;
          }
        }
        if (__any_sync(kFull, bad) && lane == 0) set_status(&st.status, 3);
      }
      __syncwarp();
    } else if (mode == kModeOrder0) {
      // order-0 rANS (decode.cu:428-550)
      if (lane == 0) {
        int valid = 1;
        int64_t cursor = 0;
        if (blen < 1 || body[cursor++] != kRansTableLog) valid = 0;
        uint32_t nsym = 0;
        if (valid && !read_varint_strict(body, blen, &cursor, &nsym)) valid = 0;
        if (nsym == 0 || nsym > 255) valid = 0;
        uint32_t prev = 0, assigned = 0;
        for (uint32_t i = 0; valid && i < nsym; ++i) {
          uint32_t delta = 0;
          if (!read_varint_strict(body, blen, &cursor, &delta) || (i != 0 && delta == 0) || prev + delta > maxf) {
            valid = 0;
            break;
          }
          const uint32_t value = prev + delta;
          uint32_t fr = (1u << kRansTableLog) - assigned;
          if (i + 1 != nsym && !read_varint_strict(body, blen, &cursor, &fr)) {
            valid = 0;
            break;
          }
          if (fr == 0 || assigned + fr > (1u << kRansTableLog) ||
              (i + 1 != nsym && assigned + fr == (1u << kRansTableLog))) {
            valid = 0;
            break;
          }
          sm.values[i] = static_cast<uint16_t>(value);
          sm.freq[i] = static_cast<uint16_t>(fr);
          sm.cum[i] = static_cast<uint16_t>(assigned);
          assigned += fr;
          prev = value;
        }
        if (assigned != (1u << kRansTableLog)) valid = 0;
        // lane lengths: the reference keeps them as int; any length >= 2^31
        // or a negative fourth length ends in status 5 there as well.
        int64_t total = 0;
        for (int l = 0; valid && l < 3; ++l) {
          if (cursor + 4 > blen) {
            valid = 0;
          } else {
            const int64_t ll = rd32(body + cursor);
            if (ll >= (1ll << 31)) valid = 0;
            sm.lane_len[l] = static_cast<int32_t>(ll);
            total += ll;
            cursor += 4;
          }
        }
        if (valid && cursor + 16 > blen) valid = 0;
        for (int l = 0; valid && l < 4; ++l) {
          sm.states[l] = rd32(body + cursor + l * 4);
          if (sm.states[l] < kRansL) valid = 0;
        }
        if (valid) {
          cursor += 16;
          const int64_t l3 = blen - cursor - total;
          if (l3 < 0) valid = 0;
          sm.lane_len[3] = static_cast<int32_t>(l3);
          for (int l = 0; valid && l < 4; ++l) {
            sm.lane_start[l] = static_cast<int32_t>(cursor);
            cursor += sm.lane_len[l];
          }
          if (valid && cursor != blen) valid = 0;
        }
        sm.nsym = static_cast<int32_t>(nsym);
        sm.valid = valid;
        if (!valid) set_status(&st.status, 5);
      }
      __syncwarp();
      if (sm.valid) {
        for (int sym = 0; sym < sm.nsym; ++sym) {
          const int b = sm.cum[sym], e = b + sm.freq[sym];
          for (int slot = b + lane; slot < e; slot += 32) sm.table[slot] = static_cast<uint8_t>(sym);
        }
        __syncwarp();
        if (lane < 4) {
          uint32_t x = sm.states[lane];
          const uint8_t* lb = body + sm.lane_start[lane];
          const int llen = sm.lane_len[lane];
          int cur = 0;
          bool ok = true;
          for (int64_t idx = lane; idx < n; idx += 4) {
            const uint32_t slot = x & ((1u << kRansTableLog) - 1u);
            const int sym = sm.table[slot];
            out[idx] = sm.values[sym];
            x = static_cast<uint32_t>(sm.freq[sym]) * (x >> kRansTableLog) + slot - sm.cum[sym];
            while (x < kRansL) {
              if (cur >= llen) {
                ok = false;
                break;
              }
              x = (x << 8) | lb[cur++];
            }
            if (!ok) break;
          }
          if (!ok || cur != llen || x != kRansL) set_status(&st.status, 5);
        }
      }
      __syncwarp();
    } else {
      if (lane == 0) set_status(&st.status, 4);
    }
  }
}

// ---------------------------------------------------------------------------
// dec_reconstruct: warp per tile, lane = row of a 32-row band, column c of
// row i at step c + i; the folded tile streams through a 64-column ring and
// the reconstruction is flushed to the output plane 32 columns at a time.

struct RecWarpSmem {
  uint32_t fold[32 * kFoldStride];
  uint16_t out[32 * kSrcStride];
  uint16_t carry[kFastMaxW];
};

size_t dec_reconstruct_smem() { return sizeof(RecWarpSmem) * kWarpsPerCta; }

template <bool MED>
__device__ void rec_tile_fast(const FrameDesc& f, const TileGeo& g, int32_t step,
                              const uint32_t* __restrict__ ftile, RecWarpSmem& sm, int lane) {
  uint16_t* __restrict__ plane = f.dst[g.plane];
  const int64_t pitch = f.dst_pitch[g.plane];
  const int W = g.w, H = g.h;
  const int32_t maxs = f.max_sample;
  const int nchunks = (W + 31) >> 5;
  const int nsteps = W + 31;
  const int nblocks = (nsteps + 31) >> 5;
  for (int band = 0; band * 32 < H; ++band) {
    const int band_rows = min(32, H - band * 32);
    uint16_t* __restrict__ orow = plane + static_cast<int64_t>(g.y + band * 32) * pitch + g.x;
    const uint32_t* __restrict__ frow = ftile + static_cast<int64_t>(band * 32) * W;
    uint32_t pf[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) pf[r] = (r < band_rows && lane < W) ? frow[static_cast<int64_t>(r) * W + lane] : 0u;
#pragma unroll
    for (int r = 0; r < 32; ++r) sm.fold[r * kFoldStride + lane] = pf[r];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      const int col = 32 + lane;
      pf[r] = (r < band_rows && col < W) ? frow[static_cast<int64_t>(r) * W + col] : 0u;
    }
    __syncwarp();
    int32_t rec = 0, a_prev = 0;
    for (int blk = 0; blk < nblocks; ++blk) {
      if (blk > 0) {
        if (blk < nchunks) {
          const int slot = (blk & 1) * 32;
#pragma unroll
          for (int r = 0; r < 32; ++r) sm.fold[r * kFoldStride + slot + lane] = pf[r];
        }
        __syncwarp();
        if (blk >= 2 && blk - 2 < nchunks) {
          const int j = blk - 2;
          const int col = j * 32 + lane;
          const int slot = (j & 1) * 32;
          if (col < W) {
            for (int r = 0; r < band_rows; ++r) orow[static_cast<int64_t>(r) * pitch + col] = sm.out[r * kSrcStride + slot + lane];
          }
        }
        if (blk + 1 < nchunks) {
          const int col = (blk + 1) * 32 + lane;
#pragma unroll
          for (int r = 0; r < 32; ++r)
            pf[r] = (r < band_rows && col < W) ? frow[static_cast<int64_t>(r) * W + col] : 0u;
        }
      }
      const int t0 = blk * 32;
#pragma unroll 4
      for (int u = 0; u < 32; ++u) {
        const int c = t0 + u - lane;
        const bool in = (c >= 0) && (c < W);
        const int cc = c & 63;
        const uint32_t fv = sm.fold[lane * kFoldStride + cc];
        int32_t a = __shfl_up_sync(kFull, rec, 1);
        if (lane == 0) a = (band > 0 && in) ? static_cast<int32_t>(sm.carry[c]) : 0;
        const int32_t pred = MED ? predict_med(rec, a, a_prev) : predict_grad(rec, a, a_prev, maxs);
        int32_t rn = max(0, min(maxs, pred + unzigzag(fv) * step));
        if (c < 0) rn = 0;
        if (in) {
          sm.out[lane * kSrcStride + cc] = static_cast<uint16_t>(rn);
          if (lane == 31) sm.carry[c] = static_cast<uint16_t>(rn);
        }
        a_prev = a;
        rec = rn;
      }
    }
    __syncwarp();
    for (int j = max(0, nblocks - 2); j < nchunks; ++j) {
      const int col = j * 32 + lane;
      const int slot = (j & 1) * 32;
      if (col < W) {
        for (int r = 0; r < band_rows; ++r) orow[static_cast<int64_t>(r) * pitch + col] = sm.out[r * kSrcStride + slot + lane];
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kWarpsPerCta * 32)
dec_reconstruct_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state, int nframes,
                       int64_t total_tiles, const uint32_t* __restrict__ folded, int* __restrict__ queue) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RecWarpSmem& sm = reinterpret_cast<RecWarpSmem*>(smem_raw)[warp];
  for (;;) {
    int64_t t = 0;
    if (lane == 0) t = atomicAdd(queue, 1);
    t = __shfl_sync(kFull, t, 0);
    if (t >= total_tiles) break;
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    if (state[fi].status != 0) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    if (g.w > kFastMaxW) continue;
    const uint32_t* ftile = folded + f.sample_base + g.sample_base;
    if (f.use_med0) rec_tile_fast<true>(f, g, f.step0, ftile, sm, lane);
    else rec_tile_fast<false>(f, g, f.step0, ftile, sm, lane);
  }
}

// Wide tiles: antidiagonal order with neighbours read back from the output
// plane (decode.cu:572-605).
__global__ void dec_reconstruct_wide_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                            int nframes, int64_t total_tiles, const uint32_t* __restrict__ folded) {
  for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    if (state[fi].status != 0) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    if (g.w <= kFastMaxW) continue;
    uint16_t* plane = f.dst[g.plane];
    const int64_t pitch = f.dst_pitch[g.plane];
    const uint32_t* ftile = folded + f.sample_base + g.sample_base;
    const int32_t maxs = f.max_sample, step = f.step0;
    for (int d = 0; d < g.w + g.h - 1; ++d) {
      const int y0 = max(0, d - g.w + 1), y1 = min(d, g.h - 1);
      for (int y = y0 + threadIdx.x; y <= y1; y += blockDim.x) {
        const int x = d - y;
        uint16_t* o = plane + static_cast<int64_t>(g.y + y) * pitch + g.x + x;
        const int32_t l = x > 0 ? o[-1] : 0;
        const int32_t a = y > 0 ? o[-pitch] : 0;
        const int32_t ul = (x > 0 && y > 0) ? o[-pitch - 1] : 0;
        const int32_t pred = f.use_med0 ? predict_med(l, a, ul) : predict_grad(l, a, ul, maxs);
        *o = static_cast<uint16_t>(max(0, min(maxs, pred + unzigzag(ftile[static_cast<int64_t>(y) * g.w + x]) * step)));
      }
      __syncthreads();
    }
  }
}

// predictor="serial": one thread per tile in raster order (decode.cu:608-656).
__global__ void dec_reconstruct_serial_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                              int nframes, int64_t total_tiles, const uint32_t* __restrict__ folded) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total_tiles) return;
  const int fi = frame_of_tile(frames, nframes, t);
  const FrameDesc& f = frames[fi];
  if (state[fi].status != 0) return;
  const TileGeo g = tile_geo(f, t - f.tile_base);
  uint16_t* plane = f.dst[g.plane];
  const int64_t pitch = f.dst_pitch[g.plane];
  const uint32_t* ftile = folded + f.sample_base + g.sample_base;
  const int32_t maxs = f.max_sample, step = f.step0;
  const bool med = f.use_med0 != 0;
  for (int y = 0; y < g.h; ++y) {
    int32_t left = 0, ul = 0;
    uint16_t* orow = plane + static_cast<int64_t>(g.y + y) * pitch + g.x;
    const uint32_t* frow = ftile + static_cast<int64_t>(y) * g.w;
    for (int x = 0; x < g.w; ++x) {
      const int32_t a = y > 0 ? orow[x - pitch] : 0;
      const int32_t pred = med ? predict_med(left, a, ul) : predict_grad(left, a, ul, maxs);
      const int32_t r = max(0, min(maxs, pred + unzigzag(frow[x]) * step));
      orow[x] = static_cast<uint16_t>(r);
      ul = a;
      left = r;
    }
  }
}

}  // namespace fvb
