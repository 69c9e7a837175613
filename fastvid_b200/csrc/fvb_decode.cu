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
__device__ __forceinline__ int list_of_mode(int mode) {
  return mode == kModeOrder0 ? 0 : (mode >= 1 && mode <= 17) ? 1 : mode == 0 ? 2 : 3;
}
}  // namespace

// ---------------------------------------------------------------------------
// dec_parse: directory entry checks (status 10) and shard header walk
// (status 11), one thread per tile.

__global__ void dec_parse_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                                 const BatchDims* __restrict__ dims, ShardInfo* __restrict__ shards,
                                 DecodeLists* __restrict__ lists, int32_t* __restrict__ list_items) {
  const int nframes = dims->frames_p[0];
  const int64_t total_tiles = dims->tiles_p[0], total_shards = dims->shards_p[0];
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
    if (!ok || decoded != samples || cursor != tile_end) {
      set_status(&st.status, 11);
      continue;
    }
    // bin the tile's shards by entropy mode for dec_shards; the lanes that
    // bin into the same list together take their slots with one atomic
    // (every shard of a batch lands on one of four counters)
    const int lane = static_cast<int>(threadIdx.x & 31);
    for (int j = 0; j < g.shard_count; ++j) {
      const int64_t s = f.shard_base + g.first_shard + j;
      const int list = list_of_mode(shards[s].mode);
      const unsigned active = __activemask();
      const unsigned peers = __match_any_sync(active, list);
      const int leader = __ffs(peers) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&lists->count[list], __popc(peers));
      base = __shfl_sync(peers, base, leader);
      const int pos = base + __popc(peers & ((1u << lane) - 1u));
      list_items[static_cast<int64_t>(list) * total_shards + pos] = static_cast<int32_t>(s);
    }
  }
}

// ---------------------------------------------------------------------------
// Entropy decode (decode.cu:222-550).  dec_parse bins shards by mode; then
//   dec_rans_tables  one thread per rANS shard parses its order-0 table
//                    serially (decode.cu:456-517) into a table record
//   dec_rans         a 4-lane group streams rANS shards: it copies a shard's
//                    table into shared memory, builds a bucket table of
//                    symbol starts, and lane l decodes lane l of the shard
//                    (decode.cu:530-549)
//   dec_other        a warp takes eight Rice, zero-run or block shards: Rice
//                    lane l of shard g on lane 4g+l (decode.cu:297-340),
//                    zero-run shard g on lane 4g (decode.cu:237-295), block
//                    shards one after another warp-wide (decode.cu:342-396)

constexpr int kGroup = 8;         // shards per warp
constexpr int kBucketShift = 4;   // a bucket covers 16 slots
constexpr int kBuckets = (1 << kRansTableLog) >> kBucketShift;

// One parsed order-0 table (decode.cu:456-517).  Symbol i covers slots
// cum_i .. cum_i + freq_i - 1 of the 4096-slot ring.
struct RansTable {
  int32_t lane_start[4], lane_len[4];
  uint32_t state[4];
  int32_t nsym, valid;
  int32_t pad[2];
  uint32_t freqcum[256];  // cum | freq << 12 (freq up to 4096: 13 bits)
  uint32_t value[256];    // the symbol's value as u16 (decode.cu:484)
};

size_t dec_rans_table_bytes() { return sizeof(RansTable); }

// Sequential reader of a byte range through aligned 32-bit loads.  Only words
// holding at least one byte of the range are loaded; four are kept in flight
// ahead of the bit buffer.  Bytes past the range read as zero.
struct ByteWindow {
  const uint32_t* words;
  int64_t next, last;
  int tail_bytes;
  uint64_t bits;
  int nbits;
  uint32_t q0, q1, q2, q3;
  int c0, c1, c2, c3;

  // Issues the load of the next word and returns it unmasked; nothing here
  // waits for the data (bytes past the range are masked off when merged).
  __device__ uint32_t load_word(int* nb) {
    const int64_t at = next < last ? next : (last > 0 ? last : 0);
    const int valid = next < last ? 4 : (next == last ? tail_bytes : 0);
    const uint32_t w = last >= 0 ? __ldg(words + at) : 0u;
    ++next;
    *nb = 8 * valid;
    return w;
  }
  __device__ void init(const uint8_t* p, int64_t len) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const int head = static_cast<int>(a & 3);
    words = reinterpret_cast<const uint32_t*>(a - head);
    next = 0;
    last = len > 0 ? (head + len - 1) >> 2 : -1;
    tail_bytes = len > 0 ? static_cast<int>((head + len - 1) & 3) + 1 : 0;
    int nb;
    const uint32_t w = load_word(&nb);
    q0 = load_word(&c0);
    q1 = load_word(&c1);
    q2 = load_word(&c2);
    q3 = load_word(&c3);
    const uint32_t w0 = nb >= 32 ? w : (w & ((1u << nb) - 1u));
    bits = nb ? (w0 >> (8 * head)) : 0u;
    nbits = nb ? nb - 8 * head : 0;
    refill();
  }
  __device__ void shift_in() {
    const uint32_t m0 = c0 >= 32 ? q0 : (q0 & ((1u << c0) - 1u));
    bits |= static_cast<uint64_t>(m0) << nbits;
    nbits += c0;
    q0 = q1;
    c0 = c1;
    q1 = q2;
    c1 = c2;
    q2 = q3;
    c2 = c3;
    q3 = load_word(&c3);
  }
  __device__ void refill_once() {
    if (nbits <= 32) shift_in();
  }
  __device__ void refill() {
    while (nbits <= 32 && c0) shift_in();
  }
  __device__ uint32_t byte() {  // next byte (zero past the range)
    if (nbits < 8) refill();
    const uint32_t b = static_cast<uint32_t>(bits) & 0xffu;
    bits >>= 8;
    nbits -= 8;
    return b;
  }
};


// A lane's byte stream through a private ring of 16 words in shared memory,
// fed by cp.async: 12 words before the first read, then two words with every
// eight-byte read -- as many as four decoding steps can consume -- so the
// ring stays at least 12 words ahead of the read position (the gap shrinks by
// at most the two words a read consumes and grows by the two it issues, up
// to the ring size).  A read may leave the newest four copy groups in flight;
// the words it touches (w .. w+2, at most ten words below the copy front,
// which advances at most two words per read) were issued five or more reads
// earlier, so their groups are complete.  There is no refill branch: every
// read issues its two copies under predicates.  Word w of the aligned range
// lives in slot w % 16; slot s of lane l is word s * 32 + l of the warp's ring
// block, so every lane reads and fills its own bank whatever its position.
// Only words holding a byte of the lane are copied (others keep stale bytes,
// and reading them is an overrun that the byte count check reports).  A
// 16-word ring (2 KB per warp, 32 before) lets four dec_rans CTAs share an
// SM.
struct LaneRing {
  static constexpr int kWords = 16;    // slots per lane
  static constexpr int kFill = 12;     // words copied before the first read
  static constexpr int kInFlight = 4;  // copy groups a read may leave pending
  static_assert(kFill >= 10 && kFill <= kWords, "read words must be five copy groups old");
  uint32_t* ring;          // slot 0 of this lane (slots 32 words apart)
  const uint32_t* words;   // aligned base of the lane's bytes
  int head;                // lane byte 0 = byte `head` of word 0
  int last;                // last word holding a lane byte (-1: none)
  int fetched;             // next word to copy

  // Copy word w into its slot if it holds a lane byte and its slot is free
  // (the word 32 below it is behind the read position `low`).
  __device__ void issue(int w, int low) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(ring + (w & (kWords - 1)) * 32));
    const int ok = (w <= last) & (w <= low + kWords - 1);
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %2, 0;\n @p cp.async.ca.shared.global [%0], [%1], 4;\n}\n" ::"r"(s),
        "l"(words + w), "r"(ok)
        : "memory");
  }
  __device__ void init(uint32_t* ring_smem, const uint8_t* p, int len) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    head = static_cast<int>(a & 3);
    words = reinterpret_cast<const uint32_t*>(a - head);
    ring = ring_smem;
    last = len > 0 ? (head + len - 1) >> 2 : -1;
#pragma unroll
    for (int i = 0; i < kFill; ++i) issue(i, 0);
    fetched = kFill;
    cp_async_commit();
  }
  __device__ void ready() { cp_async_wait<0>(); }
  // The eight bytes at lane positions cur..cur+7, first byte in the top
  // bits of hi, the next four in lo; cur advances by at most eight between
  // calls.
  __device__ void window(int cur, uint32_t& hi_out, uint32_t& lo_out) {
    const int pos = head + cur;
    const int w = pos >> 2;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      issue(fetched, w);
      fetched += fetched <= w + kWords - 1;
    }
    cp_async_commit();
    cp_async_wait<kInFlight>();
    const uint32_t a = ring[(w & (kWords - 1)) * 32], b = ring[((w + 1) & (kWords - 1)) * 32],
                   c = ring[((w + 2) & (kWords - 1)) * 32];
    const int sh = 8 * (pos & 3);
    hi_out = __byte_perm(__funnelshift_r(a, b, sh), 0, 0x0123);
    lo_out = __byte_perm(__funnelshift_r(b, c, sh), 0, 0x0123);
  }
};

// Order-0 table of one shard, parsed by one thread (decode.cu:456-517).
__device__ bool rans_parse_serial(const uint8_t* __restrict__ body, int64_t blen, uint32_t maxf,
                                  RansTable& t) {
  ByteWindow r;
  r.init(body, blen);
  int64_t cursor = 0;
  auto varint = [&](uint32_t* value) -> bool {
    uint32_t result = 0;
    int shift = 0;
    for (int used = 0; used < 5; ++used) {
      if (cursor >= blen) return false;
      const uint32_t b = r.byte();
      ++cursor;
      if (used == 4 && b > 0x0f) return false;
      result |= (b & 0x7f) << shift;
      if ((b & 0x80) == 0) {
        if (varint_len(result) != used + 1) return false;
        *value = result;
        return true;
      }
      shift += 7;
    }
    return false;
  };
  if (blen < 1) return false;
  ++cursor;
  if (r.byte() != kRansTableLog) return false;
  uint32_t n = 0;
  if (!varint(&n) || n == 0 || n > 255) return false;
  uint32_t prev = 0, assigned = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t delta = 0;
    if (!varint(&delta) || (i != 0 && delta == 0) || prev + delta > maxf) return false;
    const uint32_t value = prev + delta;
    uint32_t fr = (1u << kRansTableLog) - assigned;
    if (i + 1 != n && !varint(&fr)) return false;
    // no 32-bit wrap-around: a frequency above 4096 - assigned is rejected
    // (decode.cu:479-480 would wrap and then overrun its slot table)
    if (fr == 0 || fr > (1u << kRansTableLog) - assigned ||
        (i + 1 != n && fr == (1u << kRansTableLog) - assigned))
      return false;
    t.freqcum[i] = assigned | (fr << 12);
    t.value[i] = value & 0xffffu;
    assigned += fr;
    prev = value;
  }
  if (assigned != (1u << kRansTableLog)) return false;
  // three lane lengths (int in the reference: >= 2^31 ends in status 5
  // there too), four states, the fourth length implied
  int64_t total = 0;
  for (int l = 0; l < 3; ++l) {
    if (cursor + 4 > blen) return false;
    uint32_t v = r.byte();
    v |= r.byte() << 8;
    v |= r.byte() << 16;
    v |= r.byte() << 24;
    cursor += 4;
    if (v >= (1u << 31)) return false;
    t.lane_len[l] = static_cast<int32_t>(v);
    total += v;
  }
  if (cursor + 16 > blen) return false;
  for (int l = 0; l < 4; ++l) {
    uint32_t v = r.byte();
    v |= r.byte() << 8;
    v |= r.byte() << 16;
    v |= r.byte() << 24;
    if (v < kRansL) return false;
    t.state[l] = v;
  }
  cursor += 16;
  const int64_t l3 = blen - cursor - total;
  if (l3 < 0) return false;
  t.lane_len[3] = static_cast<int32_t>(l3);
  for (int l = 0; l < 4; ++l) {
    t.lane_start[l] = static_cast<int32_t>(cursor);
    cursor += t.lane_len[l];
  }
  t.nsym = static_cast<int32_t>(n);
  return cursor == blen;
}

__global__ void __launch_bounds__(128)
dec_rans_tables_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                       const ShardInfo* __restrict__ shards, const DecodeLists* __restrict__ lists,
                       const int32_t* __restrict__ list_items, RansTable* __restrict__ tables) {
  const int count = lists->count[0];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const ShardInfo& si = shards[list_items[p]];
    FrameState& st = state[si.frame];
    RansTable& t = tables[p];
    bool ok = false;
    if (st.status == 0) {  // a failed parse may have left shard records unwritten
      const FrameDesc& f = frames[si.frame];
      ok = rans_parse_serial(f.stream + si.offset, si.body, static_cast<uint32_t>(f.max_sample) * 2u, t);
      if (!ok) set_status(&st.status, 5);
    }
    t.valid = ok;
  }
}

// Shared memory of one dec_rans warp: one column per 4-lane group, the
// columns interleaved word by word (word k of group j at pool[k * 8 + j]) so
// that the groups' lookups fall in different banks; and the lanes' byte
// rings.  A column holds the shard's bucket table and, for tables of up to
// 64 symbols (a predicted shard holds a few dozen), its freq|cum and value
// words; larger tables are read from global memory.
constexpr int kColumns = 8;  // 4-lane groups per warp
constexpr int kColumnSymbols = 64;
constexpr int kColumnWords = kBuckets + 2 * kColumnSymbols;

struct RansWarpSm {
  uint32_t pool[kColumns * kColumnWords];
  // per-lane byte rings, slot-major: rings[s][lane]
  uint32_t rings[LaneRing::kWords][32];
};

size_t dec_rans_smem() { return sizeof(RansWarpSm) * kWarpsPerCta; }

// Bucket table of one shard: word u = (symbol holding slot 16u) << 16, with
// bit i set for every symbol whose range starts at slot 16u + i (i = 1..15).
// The symbol holding slot s is then the bucket's first symbol plus the
// starts at or below s inside the bucket -- one shared load and a population
// count, no search.  `fc` is the freq|cum list at a stride of 2^fc_shift
// words; lane l of the group writes buckets 64l .. 64l + 63.
__device__ __forceinline__ void build_buckets(uint32_t* bcol, const uint32_t* fc, int fc_shift, int nsym,
                                              int my_l) {
  constexpr uint32_t kSlots = 1u << kRansTableLog;
  auto start = [&](int i) { return i < nsym ? (fc[i << fc_shift] & (kSlots - 1u)) : kSlots; };
  int s = 0;
  uint32_t next = start(1);  // first slot of symbol s + 1
  for (int k = 0; k < kBuckets / 4; ++k) {
    const uint32_t u = static_cast<uint32_t>(my_l * (kBuckets / 4) + k);
    const uint32_t lo = u << kBucketShift;
    while (next <= lo) next = start(++s + 1);
    uint32_t w = static_cast<uint32_t>(s) << 16;
    for (int i = s + 1; next < lo + (1u << kBucketShift);) {
      w |= 1u << (next - lo);
      next = start(++i);
    }
    next = start(s + 1);
    bcol[u * kColumns] = w;
  }
}

// Decode lane `my_l` of one shard: n symbols from this lane's byte ring,
// initial state x; the bucket table at a stride of 8 words,
// the freq|cum and value words at a stride of 2^LOG_S.  Returns the bytes
// consumed and the final state.
template <int LOG_S, typename FoldT>
__device__ __forceinline__ void rans_decode_lane(const uint32_t* __restrict__ bcol, const uint32_t* __restrict__ fc_col,
                                                 const uint32_t* __restrict__ val_col, LaneRing& ring,
                                                 FoldT* __restrict__ out, int n, int my_l, uint32_t& x, int& cur) {
  cur = 0;
  ring.ready();
  // Branch-free step: after x = freq*(x>>12) + slot - cum, x >= 2^11, so
  // renormalisation shifts in one byte when x < 2^23 and a second when
  // x < 2^15 (decode.cu:540-545), taken from the top of an eight-byte window
  // read ahead of the state chain; four steps use at most eight bytes.
  // Reading past the lane is an error, found by the byte count.  The window
  // is two 32-bit words (whi, wlo), shifted by funnel shifts: a 64-bit
  // variable shift costs several instructions on the state chain.
  auto step = [&](uint32_t& whi, uint32_t& wlo, int idx) {
    const uint32_t slot = x & ((1u << kRansTableLog) - 1u);
    const uint32_t bw = bcol[(slot >> kBucketShift) * kColumns];
    // starts at offsets 1..r of the bucket survive the shift by 31 - r
    const uint32_t sym = (bw >> 16) + __popc(bw << ((slot & ((1u << kBucketShift) - 1u)) ^ 31u));
    const uint32_t fc = fc_col[sym << LOG_S];
    out[idx] = static_cast<FoldT>(val_col[sym << LOG_S]);  // symbols below 511
    x = (fc >> 12) * (x >> kRansTableLog) + slot - (fc & ((1u << kRansTableLog) - 1u));
    const int nb = (x < kRansL) + (x < (kRansL >> 8));
    const uint32_t sh = 8u * static_cast<uint32_t>(nb);  // 0, 8 or 16
    x = __funnelshift_l(whi, x, sh);
    whi = __funnelshift_l(wlo, whi, sh);
    wlo <<= sh;
    cur += nb;
  };
  int idx = my_l;
  for (; idx + 12 < n; idx += 16) {
    uint32_t whi, wlo;
    ring.window(cur, whi, wlo);
    step(whi, wlo, idx);
    step(whi, wlo, idx + 4);
    step(whi, wlo, idx + 8);
    step(whi, wlo, idx + 12);
  }
  if (idx < n) {
    uint32_t whi, wlo;
    ring.window(cur, whi, wlo);
    for (; idx < n; idx += 4) step(whi, wlo, idx);  // at most three steps
  }
  cp_async_wait<0>();
}

// Each 4-lane group streams rANS shards: it claims the next shard from the
// list, builds the shard's tables in its column and decodes its four lanes,
// then claims another -- so every lane stays busy until the list is done,
// whatever the mix of shards.
template <typename FoldT>
__global__ void __launch_bounds__(kWarpsPerCta * 32)
dec_rans_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                const ShardInfo* __restrict__ shards, DecodeLists* __restrict__ lists,
                const int32_t* __restrict__ list_items, const RansTable* __restrict__ tables,
                FoldT* __restrict__ folded) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RansWarpSm& sm = reinterpret_cast<RansWarpSm*>(smem_raw)[warp];
  const int j = lane >> 2, my_l = lane & 3;
  const unsigned group = 0xfu << (4 * j);
  const int count = lists->count[0];
  uint32_t* bcol = sm.pool + j;
  uint32_t* fc_col = sm.pool + kBuckets * kColumns + j;
  uint32_t* val_col = sm.pool + (kBuckets + kColumnSymbols) * kColumns + j;
  for (;;) {
    int p = 0;
    if (my_l == 0) p = atomicAdd(&lists->next_group_rans, 1);
    p = __shfl_sync(group, p, 4 * j);
    if (p >= count) break;
    const RansTable& t = tables[p];
    if (!t.valid) continue;
    const ShardInfo& si = shards[list_items[p]];
    const FrameDesc& f = frames[si.frame];
    const uint8_t* body = f.stream + si.offset;
    FoldT* out = folded + si.sample_base;
    uint32_t x = t.state[my_l];
    const int llen = t.lane_len[my_l];
    const uint8_t* lb = body + t.lane_start[my_l];
    const int nsym = t.nsym;
    const bool local = nsym <= kColumnSymbols;
    int cur = 0;
    LaneRing ring;
    ring.init(&sm.rings[0][lane], lb, llen);  // the first copies land while the tables are built
    __syncwarp(group);  // the group's previous shard is decoded
    if (local) {
      for (int i = my_l; i < nsym; i += 4) {
        fc_col[i * kColumns] = t.freqcum[i];
        val_col[i * kColumns] = t.value[i];
      }
      __syncwarp(group);
      build_buckets(bcol, fc_col, 3, nsym, my_l);
    } else {
      build_buckets(bcol, t.freqcum, 0, nsym, my_l);
    }
    __syncwarp(group);
    if (local)
      rans_decode_lane<3>(bcol, fc_col, val_col, ring, out, si.count, my_l, x, cur);
    else
      rans_decode_lane<0>(bcol, t.freqcum, t.value, ring, out, si.count, my_l, x, cur);
    if (cur != llen || x != kRansL) set_status(&state[si.frame].status, 5);
  }
}

// A Rice lane's bits, first bit lowest, through a private ring of 16 words
// in shared memory fed by cp.async (the LaneRing scheme): 12 words are copied
// before the first code; take() moves the next word into the 64-bit buffer
// whenever the buffer holds 32 bits or fewer -- branch-free, once per refill
// (the decoder then takes every code the buffer holds) -- and copies one more
// word for each word it takes, so the copies stay at least 11 words ahead of
// the word taken (10 ahead of the one read early).  (Loading words straight into a queue of
// registers made every refill wait for a load: moving a register whose load
// is in flight waits for it, and the four lanes of a shard refill at
// different codes, so a warp met a load latency at nearly every code.)  Words
// past the lane's last byte are not copied; bits read there are garbage, and
// every position is checked against the lane's bit count instead.
struct RiceRing {
  static constexpr int kWords = 16;
  static constexpr int kFill = 12;
  static constexpr int kInFlight = 10;  // a word is read at least 10 copy groups after its copy
  uint32_t* ring;         // slot 0 of this lane (slots 32 words apart)
  const uint32_t* words;  // aligned base of the lane's bytes
  int last;               // last word holding a lane byte (-1: none)
  int fetched;            // next word to copy
  int next;               // next word to take into the buffer
  uint64_t bits;          // buffered bits, next bit lowest (zeros above nbits)
  int nbits;
  uint32_t ahead;         // word `next`, read one take early so no code waits on the ring load

  __device__ void issue(int w) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(ring + (w & (kWords - 1)) * 32));
    const int ok = w <= last;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %2, 0;\n @p cp.async.ca.shared.global [%0], [%1], 4;\n}\n" ::"r"(sa),
        "l"(words + w), "r"(ok)
        : "memory");
  }
  __device__ void init(uint32_t* ring_smem, const uint8_t* p, int64_t len) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const int head = static_cast<int>(a & 3);
    words = reinterpret_cast<const uint32_t*>(a - head);
    ring = ring_smem;
    last = len > 0 ? static_cast<int>((head + len - 1) >> 2) : -1;
#pragma unroll
    for (int i = 0; i < kFill; ++i) issue(i);
    fetched = kFill;
    cp_async_commit();
    cp_async_wait<0>();
    bits = ring[0] >> (8 * head);  // the first word's bytes before the lane are dropped
    nbits = 32 - 8 * head;
    next = 1;
    ahead = ring[32];
  }
  // Takes the next word when 32 bits or fewer are buffered (afterwards at
  // least 33 are, or the buffer was already fuller).
  // The word taken was read from the ring by the take before (or by init);
  // the next one is read here, after the wait, for the take after: word w
  // is copied by the take that takes word w - 11 and read by the one that
  // takes word w - 1, ten copy groups later, so a wait leaving ten groups
  // pending covers it.
  __device__ void take() {
    const bool need = nbits <= 32;
    bits |= need ? static_cast<uint64_t>(ahead) << nbits : 0ull;
    nbits += need ? 32 : 0;
    next += need;
    if (need) issue(fetched);
    fetched += need;
    cp_async_commit();
    cp_async_wait<kInFlight>();
    const uint32_t w = ring[(next & (kWords - 1)) * 32];
    ahead = need ? w : ahead;
  }
};

// cnt zero symbols from p: element stores up to a 16-byte boundary, then
// 16-byte stores, then the tail (a zero run of a shard is up to 4,096
// symbols, written by one thread).
template <typename FoldT>
__device__ __forceinline__ void zero_fill(FoldT* p, int64_t cnt) {
  constexpr int kPer = 16 / sizeof(FoldT);
  int64_t i = 0;
  const int head = static_cast<int>(((16 - (reinterpret_cast<uintptr_t>(p) & 15)) & 15) / sizeof(FoldT));
  for (; i < head && i < cnt; ++i) p[i] = 0;
  uint4* v = reinterpret_cast<uint4*>(p + i);
  const int64_t nv = (cnt - i) / kPer;
  for (int64_t j = 0; j < nv; ++j) v[j] = make_uint4(0, 0, 0, 0);
  for (i += nv * kPer; i < cnt; ++i) p[i] = 0;
}

// A zero-run shard (decode.cu:237-295) decoded by the whole warp, 32 body
// bytes per step, one per lane.  A byte without the 0x80 bit ends a token
// (ballot); the lane holding a token's last byte gathers the token's bytes
// from the lanes before it by shuffles, with the bytes of a token begun in an
// earlier step carried over; the symbols of the step's tokens are placed by
// a warp prefix sum.  Every check of the serial parser is made -- at most
// five bytes, the fifth at most 0x0f, canonical length, a run no longer than
// the symbols left, a value in 1..maxf, no token after the last symbol, no
// partial token and no missing symbol at the end -- so a stream is accepted
// exactly when the serial parser accepts it.  The shard's symbols are zeroed
// first; value tokens then write theirs.  Warp-collective: every lane calls
// it with the same arguments.  Returns whether the shard is valid.
template <typename FoldT>
__device__ bool zero_run_warp(const uint8_t* __restrict__ body, int64_t blen, int n, uint32_t maxf,
                              FoldT* __restrict__ out, int lane) {
  for (int i = lane; i < n; i += 32) out[i] = 0;
  __syncwarp();
  int produced = 0;        // symbols of the steps so far (warp-uniform)
  uint32_t pend_val = 0;   // value bits of a token begun in an earlier step
  int pend_used = 0;       // its bytes so far (capped at 6)
  bool pend_bad = false;   // its fifth byte was above 0x0f, or it is too long
  bool bad = false;
  for (int64_t base = 0; base < blen && !bad; base += 32) {
    const bool vld = base + lane < blen;
    const uint32_t byte = vld ? body[base + lane] : 0u;
    const uint32_t endm = __ballot_sync(kFull, vld && !(byte & 0x80u));
    const int nvalid = static_cast<int>(min(static_cast<int64_t>(32), blen - base));
    const bool is_end = (endm >> lane) & 1u;
    const uint32_t below = endm & ((1u << lane) - 1u);
    const int prev = below ? 31 - __clz(below) : -1;  // the previous token's end in this step
    const bool carried = prev < 0;                    // the token began in an earlier step
    const int here = lane - prev;                     // its bytes in this step
    const int cu = carried ? pend_used : 0;
    uint32_t tok = carried ? pend_val : 0u;
    bool tb = carried && pend_bad;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
      const uint32_t bt = __shfl_sync(kFull, byte, max(lane - t, 0));
      const int p = cu + here - 1 - t;  // position of byte lane - t in the token
      if (t < here && p < 5) {
        tok |= (bt & 0x7fu) << (7 * p);
        if (p == 4 && bt > 0x0fu) tb = true;
      }
    }
    if (cu + here > 5) tb = true;
    if (!tb && cu + here != varint_len(tok)) tb = true;
    uint32_t cnt = 0;
    if (is_end) {
      if (tok & 1u) {
        const uint32_t value = (tok + 1u) >> 1;  // u32 arithmetic as in the reference
        if (value == 0u || value > maxf) tb = true;
        cnt = 1;
      } else {
        cnt = min((tok >> 1) + 1u, static_cast<uint32_t>(n) + 1u);  // a run; longer than n fails below
      }
    }
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += v;
    }
    const uint32_t start = static_cast<uint32_t>(produced) + inc - cnt;
    if (is_end) {
      if (start + cnt > static_cast<uint32_t>(n)) tb = true;  // a run past the end, or a token after it
      if (!tb && (tok & 1u)) out[start] = fold_store<FoldT>((tok + 1u) >> 1);
    }
    bad = __any_sync(kFull, is_end && tb);
    produced += static_cast<int>(__shfl_sync(kFull, inc, 31));
    // bytes after the step's last token end begin (or continue) a token
    const int last_end = endm ? 31 - __clz(endm) : -1;
    const int tail = nvalid - 1 - last_end;
    if (tail > 0) {
      const int c0 = endm ? 0 : pend_used;
      uint32_t v = endm ? 0u : pend_val;
      bool pb = endm ? false : pend_bad;
#pragma unroll
      for (int t = 0; t < 5; ++t) {
        const uint32_t bt = __shfl_sync(kFull, byte, min(last_end + 1 + t, 31));
        const int p = c0 + t;
        if (t < tail && p < 5) {
          v |= (bt & 0x7fu) << (7 * p);
          if (p == 4 && bt > 0x0fu) pb = true;
        }
      }
      pend_val = v;
      pend_used = min(c0 + tail, 6);
      pend_bad = pb || c0 + tail > 5;
    } else {
      pend_val = 0;
      pend_used = 0;
      pend_bad = false;
    }
  }
  return !bad && pend_used == 0 && produced == n;
}

struct OtherGroupSm {
  int32_t boff[32], bwidth[32];
  int32_t valid;
};

template <typename FoldT>
__global__ void __launch_bounds__(128)
dec_other_kernel(const FrameDesc* __restrict__ frames, FrameState* __restrict__ state,
                 const ShardInfo* __restrict__ shards, const BatchDims* __restrict__ dims,
                 DecodeLists* __restrict__ lists, const int32_t* __restrict__ list_items,
                 FoldT* __restrict__ folded) {
  const int64_t total_shards = dims->shards_p[0];
  __shared__ OtherGroupSm sm_all[4];
  __shared__ uint32_t rice_rings[4][RiceRing::kWords * 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  OtherGroupSm& sm = sm_all[warp];
  const int my_g = lane >> 2, my_l = lane & 3;
  int ngroups[3], total_groups = 0;
  for (int l = 0; l < 3; ++l) {
    ngroups[l] = (lists->count[l + 1] + kGroup - 1) / kGroup;
    total_groups += ngroups[l];
  }
  for (;;) {
    int g = 0;
    if (lane == 0) g = atomicAdd(&lists->next_group, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= total_groups) break;
    int list = 0;
    while (g >= ngroups[list]) {
      g -= ngroups[list];
      ++list;
    }
    ++list;  // 1 Rice, 2 zero-run, 3 block pack
    const int first = g * kGroup;
    const int count = lists->count[list];
    const int32_t* items = list_items + static_cast<int64_t>(list) * total_shards;
    const int64_t s_mine = (first + my_g < count) ? items[first + my_g] : -1;
    bool live = false;
    int fi = 0, mode = 0, n = 0;
    int64_t blen = 0;
    const uint8_t* body = nullptr;
    FoldT* out = nullptr;
    uint32_t maxf = 0;
    if (s_mine >= 0) {
      const ShardInfo& si = shards[s_mine];
      fi = si.frame;
      live = state[fi].status == 0;  // a failed parse may have left shard records unwritten
      mode = si.mode;
      n = si.count;
      blen = si.body;
      body = frames[fi].stream + si.offset;
      out = folded + si.sample_base;
      maxf = static_cast<uint32_t>(frames[fi].max_sample) * 2u;
    }
    if (list == 1) {
      // ---- Rice ---------------------------------------------------------------
      if (s_mine >= 0 && live) {
        const int lc = n < 4 ? n : 4;
        const int64_t table = static_cast<int64_t>(lc - 1) * 4;
        if (table > blen) {
          if (my_l == 0) set_status(&state[fi].status, 2);
        } else if (my_l < lc) {
          int64_t loff = table;
          for (int i = 0; i < my_l; ++i) loff += rd32(body + i * 4);
          const int64_t llen = my_l + 1 < lc ? static_cast<int64_t>(rd32(body + my_l * 4)) : blen - loff;
          bool ok = !(loff > blen || llen < 0 || llen > blen - loff);
          if (ok) {
            const int k = mode - 1;
            const uint32_t rmask = k ? (1u << k) - 1u : 0u;
            const int64_t total = 8 * llen;  // bits of this lane
            RiceRing rr;
            rr.init(&rice_rings[warp][lane], body + loff, llen);
            int64_t pos = 0;
            int idx = my_l;
            while (idx < n && ok) {
              // unary quotient: zeros up to the next one bit, then k
              // remainder bits (decode.cu:63-125)
              rr.take();
              uint32_t lo = static_cast<uint32_t>(rr.bits);
              int z0 = __ffs(lo) - 1;  // -1: no one bit in the low word
              if (z0 >= 0 && z0 + 1 + k <= rr.nbits) {
                // codes wholly buffered, each with a quotient below 32: one
                // pass over each, as many as the buffer holds
                do {
                  const int tot = z0 + 1 + k;  // at most 48
                  const uint32_t r = __funnelshift_rc(lo, static_cast<uint32_t>(rr.bits >> 32), z0 + 1) & rmask;
                  rr.bits >>= tot;
                  rr.nbits -= tot;
                  pos += tot;
                  const uint64_t v = (static_cast<uint64_t>(z0) << k) + r;
                  if (pos > total || v > maxf) {  // the code runs past the lane, or its value is too large
                    ok = false;
                    break;
                  }
                  out[idx] = fold_store<FoldT>(static_cast<uint32_t>(v));
                  idx += lc;
                  lo = static_cast<uint32_t>(rr.bits);
                  z0 = __ffs(lo) - 1;
                } while (idx < n && z0 >= 0 && z0 + 1 + k <= rr.nbits);
                continue;
              }
              uint64_t v;
              {
                uint32_t q = 0;
                while (rr.bits == 0) {  // every buffered bit is zero: a long quotient
                  q += rr.nbits;
                  pos += rr.nbits;
                  rr.nbits = 0;
                  if (pos >= total || q > maxf) {
                    ok = false;
                    break;
                  }
                  rr.take();
                }
                if (!ok) break;
                const int z = __ffsll(static_cast<long long>(rr.bits)) - 1;
                q += z;
                rr.bits = z == 63 ? 0ull : rr.bits >> (z + 1);
                rr.nbits -= z + 1;
                pos += z + 1;
                if (pos > total || q > maxf) {  // the one bit lies past the lane, or the quotient is too large
                  ok = false;
                  break;
                }
                if (rr.nbits < k) rr.take();
                const uint32_t r = static_cast<uint32_t>(rr.bits) & rmask;
                rr.bits >>= k;
                rr.nbits -= k;
                pos += k;
                v = (static_cast<uint64_t>(q) << k) + r;
                if (pos > total) {
                  ok = false;
                  break;
                }
              }
              if (v > maxf) {
                ok = false;
                break;
              }
              out[idx] = fold_store<FoldT>(static_cast<uint32_t>(v));
              idx += lc;
            }
            cp_async_wait<0>();  // no copy into the ring outlives the lane
            if (ok) {
              const int64_t used = (pos + 7) / 8;
              if (used != llen) ok = false;
              else if ((pos & 7) != 0) {
                const uint8_t mask = static_cast<uint8_t>(~((1u << (pos & 7)) - 1u));
                if (body[loff + used - 1] & mask) ok = false;
              }
            }
          }
          if (!ok) set_status(&state[fi].status, 2);
        }
      }
    } else if (list == 2) {
      // ---- zero-run: the warp takes the shards one after another --------------
      for (int k = 0; k < kGroup; ++k) {
        const int64_t sk = __shfl_sync(kFull, s_mine, 4 * k);
        if (sk < 0) continue;
        const bool lk = __shfl_sync(kFull, live, 4 * k);
        if (!lk) continue;
        const int nk = __shfl_sync(kFull, n, 4 * k);
        const int64_t bk = __shfl_sync(kFull, blen, 4 * k);
        const int fk = __shfl_sync(kFull, fi, 4 * k);
        const uint32_t mk = __shfl_sync(kFull, maxf, 4 * k);
        const uint8_t* bodyk =
            reinterpret_cast<const uint8_t*>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(body), 4 * k));
        FoldT* outk = reinterpret_cast<FoldT*>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(out), 4 * k));
        if (!zero_run_warp(bodyk, bk, nk, mk, outk, lane) && lane == 0) set_status(&state[fk].status, 1);
      }
    } else {
      // ---- block pack: the warp takes the shards one after another ------------
      for (int k = 0; k < kGroup; ++k) {
        const int64_t sk = __shfl_sync(kFull, s_mine, 4 * k);
        if (sk < 0) continue;
        const bool lk = __shfl_sync(kFull, live, 4 * k);
        if (!lk) continue;
        const int nk = __shfl_sync(kFull, n, 4 * k);
        const int64_t bk = __shfl_sync(kFull, blen, 4 * k);
        const int fk = __shfl_sync(kFull, fi, 4 * k);
        const uint32_t mk = __shfl_sync(kFull, maxf, 4 * k);
        const uint8_t* bodyk = reinterpret_cast<const uint8_t*>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(body), 4 * k));
        FoldT* outk = reinterpret_cast<FoldT*>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(out), 4 * k));
        const int nblk = (nk + kBlockSymbols - 1) / kBlockSymbols;
        const int maxw = 32 - __clz(mk);
        if (lane == 0) {
          int64_t cursor = 0;
          int ok = 1;
          for (int b = 0; b < nblk; ++b) {
            if (cursor >= bk) {
              ok = 0;
              break;
            }
            const int w = bodyk[cursor++];
            if (w > maxw) {
              ok = 0;
              break;
            }
            const int64_t nb = min(static_cast<int64_t>(kBlockSymbols), static_cast<int64_t>(nk) - static_cast<int64_t>(b) * kBlockSymbols);
            const int64_t pay = (nb * w + 7) / 8;
            if (pay > bk - cursor) {
              ok = 0;
              break;
            }
            sm.boff[b] = static_cast<int32_t>(cursor);
            sm.bwidth[b] = w;
            const int64_t bits = nb * w;
            if ((bits & 7) != 0) {
              const uint8_t mask = static_cast<uint8_t>(~((1u << (bits & 7)) - 1u));
              if (bodyk[cursor + pay - 1] & mask) {
                ok = 0;
                break;
              }
            }
            cursor += pay;
          }
          if (ok && cursor != bk) ok = 0;
          sm.valid = ok;
          if (!ok) set_status(&state[fk].status, 3);
        }
        __syncwarp();
        if (sm.valid) {
          int bad = 0;
          for (int b = 0; b < nblk; ++b) {
            const int w = sm.bwidth[b];
            const uint8_t* pay = bodyk + sm.boff[b];
            const int nb = min(kBlockSymbols, nk - b * kBlockSymbols);
            for (int i = lane; i < nb; i += 32) {
              uint32_t v = 0;
              if (w) {
                const int64_t bit = static_cast<int64_t>(i) * w;
                const int64_t byte0 = bit >> 3;
                const int64_t lastb = (bit + w - 1) >> 3;
                uint64_t acc = 0;
                for (int64_t j = byte0; j <= lastb; ++j) acc |= static_cast<uint64_t>(pay[j]) << (8 * (j - byte0));
                v = static_cast<uint32_t>((acc >> (bit & 7)) & ((1ull << w) - 1));
              }
              if (v > mk) bad = 1;
              outk[static_cast<int64_t>(b) * kBlockSymbols + i] = fold_store<FoldT>(v);
            }
          }
          if (__any_sync(kFull, bad) && lane == 0) set_status(&state[fk].status, 3);
        }
        __syncwarp();
      }
    }
  }
}


// ---------------------------------------------------------------------------
// dec_reconstruct: warp per tile, lane = row of a 32-row band, column c of
// row i at step c + i; the folded tile streams through a 64-column ring and
// the reconstruction is flushed to the output plane 32 columns at a time.

// Mirror of enc_tile_fast: the folded residuals stream in through a skewed
// 64-column ring, the reconstruction goes out through another and is flushed
// to the output plane 32 columns at a time (decode.cu:552-606).

template <typename FoldT>
struct RecWarpSmem {
  static constexpr int kFS = fold_stride<FoldT>();
  FoldT fold[32 * kFS];             // folded-residual ring (skewed)
  uint16_t out[32 * kSrcStride];    // reconstruction ring (u16, skewed)
  uint16_t carry[kFastMaxW + 128];  // row above the band, column c at index c + 32
};

size_t dec_reconstruct_smem(bool fold16) {
  return (fold16 ? sizeof(RecWarpSmem<uint16_t>) : sizeof(RecWarpSmem<uint32_t>)) * kWarpsPerCta;
}

template <bool MED, bool STEP1, bool EDGE, int UNROLL, bool SPLIT, typename FoldT>
__device__ __forceinline__ void rec_block(RecWarpSmem<FoldT>& sm, const uint16_t* carry_in, uint16_t* carry_out, int lane,
                                          int t0, int W, int32_t maxs, int32_t step, bool band0, int32_t& rec,
                                          int32_t& a_prev) {
  const FoldT* frow = sm.fold + lane * RecWarpSmem<FoldT>::kFS + (t0 & 32);
  uint16_t* orow = sm.out + lane * kSrcStride + (t0 & 32);
  const uint16_t* crow_in = carry_in + 32 - lane + t0;  // lane 0: column t0 + u
  // one warp per tile reads and writes the same row: one pointer
  uint16_t* crow_out = SPLIT ? carry_out + 32 - lane + t0 : const_cast<uint16_t*>(crow_in);      // lane 31: column t0 + u - 31
#pragma unroll UNROLL
  for (int u = 0; u < 32; ++u) {
    const uint32_t fv = frow[u];
    int32_t a = __shfl_up_sync(0xffffffffu, rec, 1);
    const int32_t above0 = crow_in[u];
    if (lane == 0) a = band0 ? 0 : above0;
    const int32_t pred = MED ? predict_med(rec, a, a_prev) : predict_grad(rec, a, a_prev, maxs);
    const int32_t q = unzigzag(fv);
    int32_t rn = max(0, min(maxs, STEP1 ? pred + q : pred + q * step));
    if (EDGE) {
      const int c = t0 + u - lane;
      if (c < 0) rn = 0;
      if (lane == 31 && c >= 0 && c < W) crow_out[u] = static_cast<uint16_t>(rn);
    } else {
      if (lane == 31) crow_out[u] = static_cast<uint16_t>(rn);
    }
    orow[u] = static_cast<uint16_t>(rn);
    a_prev = a;
    rec = rn;
  }
}

// One warp's sweep of one 32-row band of a tile, block by block: begin()
// stages the first folded chunks, block(k) runs wavefront block k (staging
// the chunk ahead and flushing the reconstruction two chunks behind), end()
// flushes the rest.  Lane 0 reads the row above the band from carry_in;
// lane 31 writes the band's last row to carry_out (one warp per tile: the
// same row, read before it is overwritten).
template <bool MED, bool STEP1, int UNROLL, bool SPLIT, typename FoldT>
struct RecBand {
  static constexpr int kFS = RecWarpSmem<FoldT>::kFS;
  RecWarpSmem<FoldT>& sm;
  int lane;
  uint16_t* __restrict__ plane;
  int64_t pitch;
  int W, H, x0, y0;
  int32_t maxs, step;
  int nchunks, nblocks;
  const FoldT* __restrict__ ftile;
  int band_rows;
  bool band0;
  uint16_t* __restrict__ orows;
  const FoldT* __restrict__ frows;
  const uint16_t* carry_in;
  uint16_t* carry_out;
  int32_t rec, a_prev;
  uint32_t pf[32];

  __device__ RecBand(const FrameDesc& f, const TileGeo& g, int32_t step_, const FoldT* ftile_,
                     RecWarpSmem<FoldT>& sm_, int lane_)
      : sm(sm_), lane(lane_), plane(f.dst[g.plane]), pitch(f.dst_pitch[g.plane]), W(g.w), H(g.h), x0(g.x),
        y0(g.y), maxs(f.max_sample), step(step_), nchunks((g.w + 31) >> 5), nblocks((g.w + 31 + 31) >> 5),
        ftile(ftile_) {}

  __device__ void load_chunk(int k) {
    const int col = k * 32 + lane;
    const FoldT* __restrict__ p = frows + col;
    if (band_rows == 32 && col < W) {
#pragma unroll
      for (int r = 0; r < 32; ++r) pf[r] = ldf(p + static_cast<int64_t>(r) * W);
    } else {
#pragma unroll
      for (int r = 0; r < 32; ++r) pf[r] = (r < band_rows && col < W) ? ldf(p + static_cast<int64_t>(r) * W) : 0u;
    }
  }
  __device__ void store_chunk(int k) {
    const int pj = k * 32 + lane;
#pragma unroll
    for (int r = 0; r < 32; ++r) sm.fold[r * kFS + ((pj + r) & 63)] = static_cast<FoldT>(pf[r]);
  }
  __device__ void flush_chunk(int k) {
    const int col = k * 32 + lane;
    if (col < W) {
      uint16_t* __restrict__ q = orows + col;
      if (band_rows == 32) {
#pragma unroll
        for (int r = 0; r < 32; ++r) q[static_cast<int64_t>(r) * pitch] = sm.out[r * kSrcStride + ((col + r) & 63)];
      } else {
        for (int r = 0; r < band_rows; ++r) q[static_cast<int64_t>(r) * pitch] = sm.out[r * kSrcStride + ((col + r) & 63)];
      }
    }
  }
  __device__ void begin(int band, const uint16_t* cin, uint16_t* cout) {
    band_rows = min(32, H - band * 32);
    band0 = band == 0;
    orows = plane + static_cast<int64_t>(y0 + band * 32) * pitch + x0;
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
      rec_block<MED, STEP1, true, UNROLL, SPLIT, FoldT>(sm, carry_in, carry_out, lane, t0, W, maxs, step, band0, rec, a_prev);
    else
      rec_block<MED, STEP1, false, UNROLL, SPLIT, FoldT>(sm, carry_in, carry_out, lane, t0, W, maxs, step, band0, rec, a_prev);
  }
  __device__ void end() {
    __syncwarp();
    for (int j = max(0, nblocks - 2); j < nchunks; ++j) flush_chunk(j);
    __syncwarp();
  }
};

// The two warps of pair p meet at named barrier 1 + p (64 threads).
__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
}

template <bool MED, bool STEP1, int UNROLL, bool PAIRS, typename FoldT>
__device__ void rec_tile(const FrameDesc& f, const TileGeo& g, int32_t step, const FoldT* __restrict__ ftile,
                         RecWarpSmem<FoldT>* smw, int warp, int lane) {
  if constexpr (PAIRS) {
    if (pair_splits(g.w, g.h)) {
      // warp pair: even bands on the first warp, odd bands on the second two
      // blocks behind, in lock-step at the pair barrier after every slot; each
      // warp writes its bands' last rows to its own carry row and reads the
      // other's.  Both warps take the same number of slots (a function of the
      // tile's size only).
      const int pw = warp & 1;
      RecWarpSmem<FoldT>& sm = smw[warp];
      RecBand<MED, STEP1, UNROLL, true, FoldT> rb(f, g, step, ftile, sm, lane);
      const int n = rb.nblocks, nbands = (g.h + 31) >> 5;
      const int own = pw ? (nbands / 2) * n : ((nbands + 1) / 2) * n;
      const int slots = max(((nbands + 1) / 2) * n, (nbands / 2) * n + 2);
      for (int gs = 0; gs < slots; ++gs) {
        const int sl = gs - 2 * pw;
        if (sl >= 0 && sl < own) {
          const int q = sl / n, blk = sl - q * n;
          if (blk == 0) rb.begin(2 * q + pw, smw[warp ^ 1].carry, sm.carry);
          rb.block(blk);
          if (blk == n - 1) rb.end();
        }
        pair_sync(warp >> 1);
      }
      return;
    }
    if (warp & 1) return;  // too small to split: the pair's first warp alone
  }
  RecWarpSmem<FoldT>& sm = smw[warp];
  RecBand<MED, STEP1, UNROLL, false, FoldT> rb(f, g, step, ftile, sm, lane);
  for (int band = 0; band * 32 < g.h; ++band) {
    rb.begin(band, sm.carry, sm.carry);
    for (int blk = 0; blk < rb.nblocks; ++blk) rb.block(blk);
    rb.end();
  }
}

// Tiles come from a queue.  With warp pairs, the pair's first warp claims a
// tile and both read it after the pair barrier (two alternating slots, so a
// claim never overwrites a tile the other warp has yet to read); both then
// make the same decisions from the same tile, so they meet at every barrier.
template <int UNROLL, bool PAIRS, typename FoldT>
__global__ void __launch_bounds__(kWarpsPerCta * 32, PAIRS ? 3 : 4)
dec_reconstruct_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                       const BatchDims* __restrict__ dims, const FoldT* __restrict__ folded,
                       int* __restrict__ queue) {
  static_assert(kWarpsPerCta % 2 == 0, "warp pairs");
  constexpr bool pairs = PAIRS;
  const int nframes = dims->frames_p[0];
  const int64_t total_tiles = dims->tiles_p[0];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int64_t claimed[kWarpsPerCta / 2][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RecWarpSmem<FoldT>* smw = reinterpret_cast<RecWarpSmem<FoldT>*>(smem_raw);
  for (int it = 0;; ++it) {
    int64_t t = 0;
    if (pairs) {
      if ((warp & 1) == 0 && lane == 0) claimed[warp >> 1][it & 1] = atomicAdd(queue, 1);
      pair_sync(warp >> 1);
      t = claimed[warp >> 1][it & 1];
    } else {
      if (lane == 0) t = atomicAdd(queue, 1);
      t = __shfl_sync(kFull, t, 0);
    }
    if (t >= total_tiles) break;
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    if (state[fi].status != 0) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    if (g.w > kFastMaxW) continue;
    const FoldT* ftile = folded + f.sample_base + g.sample_base;
    if (f.use_med0) {
      if (f.step0 == 1) rec_tile<true, true, UNROLL, PAIRS, FoldT>(f, g, 1, ftile, smw, warp, lane);
      else rec_tile<true, false, UNROLL, PAIRS, FoldT>(f, g, f.step0, ftile, smw, warp, lane);
    } else {
      if (f.step0 == 1) rec_tile<false, true, UNROLL, PAIRS, FoldT>(f, g, 1, ftile, smw, warp, lane);
      else rec_tile<false, false, UNROLL, PAIRS, FoldT>(f, g, f.step0, ftile, smw, warp, lane);
    }
  }
}

// The wavefront block of dec_reconstruct is a launch-time choice, as for
// enc_predict (4, 8, 16 or 32 steps unrolled; identical planes).
cudaError_t dec_reconstruct_set_smem() {
  const int b32 = static_cast<int>(dec_reconstruct_smem(false)), b16 = static_cast<int>(dec_reconstruct_smem(true));
  for (auto k : {dec_reconstruct_kernel<4, false, uint32_t>, dec_reconstruct_kernel<8, false, uint32_t>,
                 dec_reconstruct_kernel<16, false, uint32_t>, dec_reconstruct_kernel<32, false, uint32_t>,
                 dec_reconstruct_kernel<8, true, uint32_t>}) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b32);
    if (e != cudaSuccess) return e;
  }
  for (auto k : {dec_reconstruct_kernel<4, false, uint16_t>, dec_reconstruct_kernel<8, false, uint16_t>,
                 dec_reconstruct_kernel<16, false, uint16_t>, dec_reconstruct_kernel<32, false, uint16_t>,
                 dec_reconstruct_kernel<8, true, uint16_t>}) {
    const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b16);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename FoldT>
static void dec_reconstruct_launch_t(int unroll, int tile_warps, int grid, cudaStream_t stream,
                                     const FrameDesc* frames, const FrameState* state, const BatchDims* dims,
                                     const void* folded, int* queue) {
  // warp pairs run with the default wavefront block
  auto k = tile_warps == 2 ? dec_reconstruct_kernel<8, true, FoldT>
           : unroll == 4   ? dec_reconstruct_kernel<4, false, FoldT>
           : unroll == 16  ? dec_reconstruct_kernel<16, false, FoldT>
           : unroll == 32  ? dec_reconstruct_kernel<32, false, FoldT>
                           : dec_reconstruct_kernel<8, false, FoldT>;
  k<<<grid, kWarpsPerCta * 32, dec_reconstruct_smem(sizeof(FoldT) == 2), stream>>>(
      frames, state, dims, static_cast<const FoldT*>(folded), queue);
}

void dec_reconstruct_launch(int unroll, int tile_warps, bool fold16, int grid, cudaStream_t stream,
                            const FrameDesc* frames, const FrameState* state, const BatchDims* dims,
                            const void* folded, int* queue) {
  if (fold16) dec_reconstruct_launch_t<uint16_t>(unroll, tile_warps, grid, stream, frames, state, dims, folded, queue);
  else dec_reconstruct_launch_t<uint32_t>(unroll, tile_warps, grid, stream, frames, state, dims, folded, queue);
}

void dec_rans_launch(bool fold16, int grid, size_t smem, cudaStream_t stream, const FrameDesc* frames,
                     FrameState* state, const ShardInfo* shards, DecodeLists* lists, const int32_t* list_items,
                     const RansTable* tables, void* folded) {
  if (fold16)
    dec_rans_kernel<uint16_t><<<grid, kWarpsPerCta * 32, smem, stream>>>(frames, state, shards, lists, list_items,
                                                                         tables, static_cast<uint16_t*>(folded));
  else
    dec_rans_kernel<uint32_t><<<grid, kWarpsPerCta * 32, smem, stream>>>(frames, state, shards, lists, list_items,
                                                                         tables, static_cast<uint32_t*>(folded));
}

cudaError_t dec_rans_set_attr(cudaFuncAttribute attr, int value) {
  const cudaError_t e = cudaFuncSetAttribute(dec_rans_kernel<uint16_t>, attr, value);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(dec_rans_kernel<uint32_t>, attr, value);
}

void dec_other_launch(bool fold16, int grid, cudaStream_t stream, const FrameDesc* frames, FrameState* state,
                      const ShardInfo* shards, const BatchDims* dims, DecodeLists* lists, const int32_t* list_items,
                      void* folded) {
  if (fold16)
    dec_other_kernel<uint16_t><<<grid, 128, 0, stream>>>(frames, state, shards, dims, lists, list_items,
                                                         static_cast<uint16_t*>(folded));
  else
    dec_other_kernel<uint32_t><<<grid, 128, 0, stream>>>(frames, state, shards, dims, lists, list_items,
                                                         static_cast<uint32_t*>(folded));
}

// Wide tiles: antidiagonal order with neighbours read back from the output
// plane (decode.cu:572-605).
__global__ void dec_reconstruct_wide_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                            const BatchDims* __restrict__ dims, const void* __restrict__ folded,
                                            int fold16) {
  const int nframes = dims->frames_p[0];
  const int64_t total_tiles = dims->tiles_p[0];
  for (int64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const int fi = frame_of_tile(frames, nframes, t);
    const FrameDesc& f = frames[fi];
    if (state[fi].status != 0) continue;
    const TileGeo g = tile_geo(f, t - f.tile_base);
    if (g.w <= kFastMaxW) continue;
    uint16_t* plane = f.dst[g.plane];
    const int64_t pitch = f.dst_pitch[g.plane];
    const int64_t fbase = f.sample_base + g.sample_base;
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
        const uint32_t fv = fold_at(folded, fold16, fbase + static_cast<int64_t>(y) * g.w + x);
        *o = static_cast<uint16_t>(max(0, min(maxs, pred + unzigzag(fv) * step)));
      }
      __syncthreads();
    }
  }
}

// predictor="serial": one thread per tile in raster order (decode.cu:608-656).
__global__ void dec_reconstruct_serial_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                              const BatchDims* __restrict__ dims, const void* __restrict__ folded,
                                              int fold16) {
  const int nframes = dims->frames_p[0];
  const int64_t total_tiles = dims->tiles_p[0];
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total_tiles) return;
  const int fi = frame_of_tile(frames, nframes, t);
  const FrameDesc& f = frames[fi];
  if (state[fi].status != 0) return;
  const TileGeo g = tile_geo(f, t - f.tile_base);
  uint16_t* plane = f.dst[g.plane];
  const int64_t pitch = f.dst_pitch[g.plane];
  const int64_t fbase = f.sample_base + g.sample_base;
  const int32_t maxs = f.max_sample, step = f.step0;
  const bool med = f.use_med0 != 0;
  for (int y = 0; y < g.h; ++y) {
    int32_t left = 0, ul = 0;
    uint16_t* orow = plane + static_cast<int64_t>(g.y + y) * pitch + g.x;
    const int64_t frow = fbase + static_cast<int64_t>(y) * g.w;
    for (int x = 0; x < g.w; ++x) {
      const int32_t a = y > 0 ? orow[x - pitch] : 0;
      const int32_t pred = med ? predict_med(left, a, ul) : predict_grad(left, a, ul, maxs);
      const int32_t r = max(0, min(maxs, pred + unzigzag(fold_at(folded, fold16, frow + x)) * step));
      orow[x] = static_cast<uint16_t>(r);
      ul = a;
      left = r;
    }
  }
}

}  // namespace fvb
