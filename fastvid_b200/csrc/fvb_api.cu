// fvb_api.cu -- the extern "C" boundary (include/fastvid_b200.h) and the host
// orchestration of the sm_100a kernels: argument and header validation with
// the reference's messages, geometry, workspace layout and launch sequences.
//
// Host synchronisation: an encode waits once (the frame's status and stream
// length, after every analysis pass including the device-side frame policy);
// a decode waits once for its status word.  The reference waits after every
// analysis pass (encode.cu:806-807) and at the end of decode (decode.cu:718).
#include <atomic>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fastvid_b200.h"
#include "fvb_common.cuh"
#include "fvb_kernels.cuh"

using namespace fvb;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  g_error = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
  return FVB_ERR_CUDA;
}

#define FVB_CUDA(call)                                    \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

#define FVB_LAUNCHED(name)                                \
  do {                                                    \
    cudaError_t e_ = cudaGetLastError();                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, name);    \
  } while (0)

// ---------------------------------------------------------------------------
// Launch accounting and optional per-kernel timing.  Every kernel launch of
// this library is counted; while profiling is on, each launch is bracketed
// by CUDA events on its own stream and the elapsed times are summed per
// kernel when profiling ends.
enum KernelId {
  K_ENC_INIT, K_ENC_PREDICT, K_ENC_PREDICT_WIDE, K_ENC_ANALYZE, K_ENC_RANS, K_ENC_SCAN, K_ENC_PREFIX,
  K_ENC_EMIT, K_DEC_PARSE, K_DEC_SHARDS, K_DEC_RECON, K_DEC_RECON_WIDE, K_DEC_RECON_SERIAL, K_RESULTS,
  K_DEC_RANS, K_DEC_OTHER, K_COUNT
};
const char* const kKernelNames[K_COUNT] = {
    "enc_init", "enc_predict", "enc_predict_wide", "enc_analyze", "enc_rans", "enc_scan", "enc_prefix",
    "enc_emit", "dec_parse", "dec_rans_tables", "dec_reconstruct", "dec_reconstruct_wide",
    "dec_reconstruct_serial", "results", "dec_rans", "dec_other"};
constexpr int kGroupShards = 8;

std::atomic<int64_t> g_launches{0};

struct ProfRecord {
  int kernel;
  cudaEvent_t a, b;
};
struct Profiler {
  bool on = false;
  std::vector<ProfRecord> records;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};
thread_local Profiler g_prof;

struct LaunchScope {
  int kernel;
  cudaStream_t stream;
  cudaEvent_t a = nullptr;
  LaunchScope(int k, cudaStream_t s) : kernel(k), stream(s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (g_prof.on) {
      a = g_prof.get();
      cudaEventRecord(a, stream);
    }
  }
  ~LaunchScope() {
    if (a) {
      cudaEvent_t b = g_prof.get();
      cudaEventRecord(b, stream);
      g_prof.records.push_back({kernel, a, b});
    }
  }
};

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }

int fill_decode_descs(const fvb_frame* frames, int n, const uint8_t* const* streams, const int64_t* stream_lens,
                      uint16_t* const* planes, const int64_t* pitches, FrameDesc* descs);

// quality -> step (encode.cu:71-85)
int32_t quantization_step(int64_t layout, int64_t depth, int64_t q) {
  if ((layout == 0 && depth == 8) || (layout == 1 && depth == 8)) return 1;
  int32_t den = 6;
  if (layout == 1 && depth == 10) den = 20;
  else if (layout == 1 && depth == 16) den = 24;
  else if (layout == 2 && depth == 10) den = 10;
  const int32_t scale = int32_t{1} << (depth - 8);
  return 1 + static_cast<int32_t>(((100 - q) * scale + den - 1) / den);
}

int32_t refined_gray16_step(int64_t q) { return 1 + static_cast<int32_t>(((100 - q) * 256 + 7) / 8); }

int64_t count_tiles(int64_t w, int64_t h, int64_t tw, int64_t th, int layout) {
  const int planes = layout == 0 ? 1 : 3;
  const int64_t rows = (h + th - 1) / th;
  int64_t n = 0;
  for (int p = 0; p < planes; ++p) {
    const bool sub = layout == 1 && p != 0;
    const int64_t pw = sub ? (w + 1) / 2 : w;
    const int64_t nw = sub ? (tw + 1) / 2 : tw;
    n += rows * ((pw + nw - 1) / nw);
  }
  return n;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Upper bound of one shard record: 3 header bytes plus the larger of the
// block-pack bound and the rANS bound (table <= 1023 bytes, 28 bytes of lane
// lengths and states, <= 12 bits per symbol plus 2 bytes per lane).
int64_t shard_record_bound(int64_t c) {
  const int64_t block = ceil_div(c, kBlockSymbols) + ceil_div(c * 17, 8);
  const int64_t rans = 1023 + 28 + 4 * (ceil_div(ceil_div(c, 4) * 12, 8) + 2);
  return 3 + (block > rans ? block : rans);
}

// Geometry of one frame into the device descriptor (tile order of
// encode.cu:41-69; the per-row shard counts let tile_geo() find any tile's
// first shard arithmetically).
void build_desc(const fvb_frame& fr, FrameDesc& d, int use_med) {
  std::memset(&d, 0, sizeof(d));
  d.layout = fr.layout;
  d.bit_depth = fr.bit_depth;
  d.quality = fr.quality;
  d.planes = fr.layout == 0 ? 1 : 3;
  d.width = static_cast<int32_t>(fr.width);
  d.height = static_cast<int32_t>(fr.height);
  d.tile_w = static_cast<int32_t>(fr.tile_w);
  d.tile_h = static_cast<int32_t>(fr.tile_h);
  d.tiles_y = static_cast<int32_t>(ceil_div(fr.height, fr.tile_h));
  d.last_h = static_cast<int32_t>(fr.height - static_cast<int64_t>(d.tiles_y - 1) * fr.tile_h);
  int64_t tile = 0, shard = 0, sample = 0;
  for (int p = 0; p < d.planes; ++p) {
    const bool sub = fr.layout == 1 && p != 0;
    const int64_t pw = sub ? (fr.width + 1) / 2 : fr.width;
    const int64_t ptw = sub ? (fr.tile_w + 1) / 2 : fr.tile_w;
    const int64_t txs = ceil_div(pw, ptw);
    d.plane_w[p] = static_cast<int32_t>(pw);
    d.ptile_w[p] = static_cast<int32_t>(ptw);
    d.tiles_x[p] = static_cast<int32_t>(txs);
    d.tile0[p] = tile;
    d.shard0[p] = shard;
    d.sample0[p] = sample;
    const int64_t wl = pw - (txs - 1) * ptw;
    for (int r = 0; r < 2; ++r) {
      const int64_t h = r ? d.last_h : fr.tile_h;
      d.shards_int[p][r] = static_cast<int32_t>(ceil_div(ptw * h, kShardSymbols));
      d.shards_last[p][r] = static_cast<int32_t>(ceil_div(wl * h, kShardSymbols));
    }
    d.shards_row[p] = (txs - 1) * d.shards_int[p][0] + d.shards_last[p][0];
    const int64_t plane_shards = (d.tiles_y - 1) * d.shards_row[p] + (txs - 1) * d.shards_int[p][1] + d.shards_last[p][1];
    tile += txs * d.tiles_y;
    shard += plane_shards;
    sample += pw * fr.height;
  }
  d.tile0[d.planes] = tile;
  d.shard0[d.planes] = shard;
  d.sample0[d.planes] = sample;
  d.ntiles = tile;
  d.nshards = shard;
  d.nsamples = sample;
  d.max_sample = (1 << fr.bit_depth) - 1;
  d.step0 = fr.step;
  d.force_order0 = fr.layout == 2 && (fr.bit_depth != 10 || fr.width < 3840);
  d.use_med0 = use_med;
  d.prefix_bytes = kHeaderBytes + kDirBytes * tile;
  d.fps_num = static_cast<uint32_t>(fr.fps_num);
  d.fps_den = static_cast<uint32_t>(fr.fps_den);
}

int fill_frame(fvb_frame* fr) {
  const int64_t tiles = count_tiles(fr->width, fr->height, fr->tile_w, fr->tile_h, fr->layout);
  if (tiles > kMaxTiles) return fail(FVB_ERR_ARGUMENT, "too many tiles");
  fr->planes = fr->layout == 0 ? 1 : 3;
  const int64_t sec = fr->layout == 1 ? (fr->width + 1) / 2 : fr->width;
  fr->plane_width[0] = fr->width;
  fr->plane_width[1] = fr->planes == 3 ? sec : 0;
  fr->plane_width[2] = fr->planes == 3 ? sec : 0;
  FrameDesc d;
  build_desc(*fr, d, 0);
  fr->tiles = d.ntiles;
  fr->shards = d.nshards;
  fr->samples = d.nsamples;
  fr->prefix_bytes = d.prefix_bytes;
  int64_t bound = d.prefix_bytes;
  for (int64_t t = 0; t < d.ntiles; ++t) {
    const TileGeo g = tile_geo(d, t);
    const int64_t s = static_cast<int64_t>(g.w) * g.h;
    const int64_t full = s / kShardSymbols, rem = s % kShardSymbols;
    bound += full * shard_record_bound(kShardSymbols) + (rem ? shard_record_bound(rem) : 0);
  }
  fr->max_stream_bytes = bound;
  return FVB_OK;
}

int device_sms() {
  static int sms[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!sms[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms[dev] = v > 0 ? v : 148;
  }
  return sms[dev];
}

// A side stream with fork/join events, one per host thread and device.
// dec_other (Rice, zero-run and block shards) depends on dec_parse only, so
// on large batches it runs on the side stream beside dec_rans and fills the
// threads and issue slots that the rANS decoder leaves free on every SM.
// Per thread, so concurrent callers never share an event.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

int side_stream(SideStream** out) {
  thread_local SideStream per_device[64];
  *out = nullptr;
  int dev = 0;
  FVB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return FVB_OK;
  SideStream& ss = per_device[dev];
  if (!ss.stream) {
    FVB_CUDA(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
    FVB_CUDA(cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming));
    FVB_CUDA(cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking));
  }
  *out = &ss;
  return FVB_OK;
}

// batches of at least this many shards (about 256 thousand samples: a 720p
// gray frame has 240) decode their non-rANS shards on the side stream, beside
// the rANS shards; both kernels are latency-bound for a single frame, so
// overlapping them shortens its decode
constexpr int64_t kSideStreamShards = 64;

int ensure_smem_attrs() {
  static bool done[64] = {false};
  int dev = 0;
  FVB_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done[dev]) return FVB_OK;
  FVB_CUDA(enc_predict_set_smem());
  FVB_CUDA(enc_emit_set_smem(static_cast<int>(enc_emit_smem())));
  FVB_CUDA(dec_reconstruct_set_smem());
  FVB_CUDA(dec_rans_set_attr(cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(dec_rans_smem())));
  // the whole unified L1/shared array as shared memory: four dec_rans CTAs
  // (56 KB each) per SM
  FVB_CUDA(dec_rans_set_attr(cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return FVB_OK;
}

// ---------------------------------------------------------------------------
// workspace layouts

// Encoder passes a frame may need: gray10 frames with a step above 1 may
// re-run with the MED predictor, gray16 frames with a step above 1 may try a
// refined step (encode.cu frame policy, :812-847; the device decides whether
// the second pass runs).  The reference re-encodes a gray16 frame a third
// time, with the baseline step, when the refined step loses; here the second
// pass writes its records to a region of its own, so the first pass's
// records are still there and are emitted instead (identical bytes, one
// pass fewer).
int frame_passes(const fvb_frame& f) {
  if (f.layout == 0 && (f.bit_depth == 10 || f.bit_depth == 16) && f.step > 1) return 2;
  return 1;
}
constexpr int kMaxPasses = 3;  // capacity of the per-pass arrays (two passes are used)

// Work of a batch, or the capacity of a bucket of batches (layouts and
// launch grids are sized by capacity; kernels read the actual counts from
// the BatchDims record in the workspace).
struct Totals {
  int frames = 0;
  int64_t tiles = 0, shards = 0, samples = 0, prefix = 0;
  bool wide = false;
  bool fold16 = true;  // folded symbols held as u16 (every frame below depth 16 or quality 100)
  int passes = 1;
  // frames, tiles and shards that take part in pass p; the encoder lays the
  // batch out with frames of more passes first, so these are prefixes
  int frames_p[kMaxPasses] = {0, 0, 0};
  int64_t tiles_p[kMaxPasses] = {0, 0, 0}, shards_p[kMaxPasses] = {0, 0, 0};
  int64_t samples_p[kMaxPasses] = {0, 0, 0}, prefix_p[kMaxPasses] = {0, 0, 0};
};

Totals totals_of(const fvb_frame* frames, int n) {
  Totals t;
  t.frames = n;
  for (int i = 0; i < n; ++i) {
    const fvb_frame& f = frames[i];
    t.tiles += f.tiles;
    t.shards += f.shards;
    t.samples += f.samples;
    t.prefix += f.prefix_bytes;
    const int64_t ptw0 = f.tile_w;
    if (ptw0 > kFastMaxW) t.wide = true;
    if (f.bit_depth >= 16 && f.quality >= 100) t.fold16 = false;
    const int passes = frame_passes(f);
    if (passes > t.passes) t.passes = passes;
    for (int p = 0; p < passes; ++p) {
      ++t.frames_p[p];
      t.tiles_p[p] += f.tiles;
      t.shards_p[p] += f.shards;
      t.samples_p[p] += f.samples;
      t.prefix_p[p] += f.prefix_bytes;
    }
  }
  return t;
}

// Encoder batch layout order: frames that may need a second pass first, then
// the rest, each group in the caller's order (the later passes run over a
// prefix of the batch).
std::vector<int> encode_order(const fvb_frame* frames, int n) {
  std::vector<int> order;
  order.reserve(n);
  for (int passes = kMaxPasses; passes >= 1; --passes)
    for (int i = 0; i < n; ++i)
      if (frame_passes(frames[i]) == passes) order.push_back(i);
  return order;
}

BatchDims dims_of(const Totals& t) {
  BatchDims d{};
  for (int p = 0; p < kMaxPasses; ++p) {
    d.frames_p[p] = t.frames_p[p];
    d.tiles_p[p] = t.tiles_p[p];
    d.shards_p[p] = t.shards_p[p];
  }
  d.frames_p[0] = t.frames;
  d.tiles_p[0] = t.tiles;
  d.shards_p[0] = t.shards;
  d.passes = t.passes;
  d.samples = t.samples;
  return d;
}

// A batch fits a capacity when every count is within it and the launch
// sequence is the same (encoder passes, wide-tile kernels); a u32 capacity
// also serves a batch whose symbols would fit u16.
bool fits(const Totals& a, const Totals& cap) {
  if (a.frames > cap.frames || a.tiles > cap.tiles || a.shards > cap.shards || a.samples > cap.samples ||
      a.prefix > cap.prefix || a.passes != cap.passes || a.wide != cap.wide || (cap.fold16 && !a.fold16))
    return false;
  for (int p = 0; p < kMaxPasses; ++p)
    if (a.frames_p[p] > cap.frames_p[p] || a.tiles_p[p] > cap.tiles_p[p] || a.shards_p[p] > cap.shards_p[p] ||
        a.samples_p[p] > cap.samples_p[p] || a.prefix_p[p] > cap.prefix_p[p])
      return false;
  return true;
}

// Bucket capacity: v rounded up to m * 2^e with m in 4..8 (the capacity is
// at most 25 percent above v), and at least `floor`.
int64_t bucket_round(int64_t v, int64_t floor) {
  if (v <= floor) return floor;
  int e = 0;
  while ((v >> e) > 7) ++e;                                  // v >> e in 4..7 once v >= 8
  const int64_t m = (v + (int64_t{1} << e) - 1) >> e;        // ceil(v / 2^e) in 4..8
  return m << e;
}

Totals bucket_of(const Totals& t) {
  Totals b = t;
  b.frames = static_cast<int>(bucket_round(t.frames, 1));
  b.tiles = bucket_round(t.tiles, 16);
  b.shards = bucket_round(t.shards, 16);
  b.samples = bucket_round(t.samples, 1 << 16);
  b.prefix = bucket_round(t.prefix, 1 << 12);
  for (int p = 0; p < kMaxPasses; ++p) {
    b.frames_p[p] = t.frames_p[p] ? static_cast<int>(bucket_round(t.frames_p[p], 1)) : 0;
    b.tiles_p[p] = t.tiles_p[p] ? bucket_round(t.tiles_p[p], 16) : 0;
    b.shards_p[p] = t.shards_p[p] ? bucket_round(t.shards_p[p], 16) : 0;
    b.samples_p[p] = t.samples_p[p] ? bucket_round(t.samples_p[p], 1 << 16) : 0;
    b.prefix_p[p] = t.prefix_p[p] ? bucket_round(t.prefix_p[p], 1 << 12) : 0;
  }
  return b;
}

void to_bucket(const Totals& t, fvb_bucket* b) {
  std::memset(b, 0, sizeof(*b));
  b->frames = t.frames;
  b->tiles = t.tiles;
  b->shards = t.shards;
  b->samples = t.samples;
  b->prefix = t.prefix;
  for (int p = 0; p < kMaxPasses; ++p) {
    b->frames_p[p] = t.frames_p[p];
    b->tiles_p[p] = t.tiles_p[p];
    b->shards_p[p] = t.shards_p[p];
    b->samples_p[p] = t.samples_p[p];
    b->prefix_p[p] = t.prefix_p[p];
  }
  b->passes = t.passes;
  b->wide = t.wide ? 1 : 0;
  b->fold16 = t.fold16 ? 1 : 0;
}

int from_bucket(const fvb_bucket* b, Totals* t) {
  if (!b || b->frames <= 0 || b->frames > (1 << 24) || b->tiles < 0 || b->shards < 0 || b->samples < 0 ||
      b->prefix < 0 || b->passes < 1 || b->passes > kMaxPasses)
    return fail(FVB_ERR_ARGUMENT, "invalid bucket");
  *t = Totals{};
  t->frames = static_cast<int>(b->frames);
  t->tiles = b->tiles;
  t->shards = b->shards;
  t->samples = b->samples;
  t->prefix = b->prefix;
  for (int p = 0; p < kMaxPasses; ++p) {
    if (b->frames_p[p] < 0 || b->frames_p[p] > b->frames || b->tiles_p[p] < 0 || b->shards_p[p] < 0 ||
        b->samples_p[p] < 0 || b->prefix_p[p] < 0)
      return fail(FVB_ERR_ARGUMENT, "invalid bucket");
    t->frames_p[p] = static_cast<int>(b->frames_p[p]);
    t->tiles_p[p] = b->tiles_p[p];
    t->shards_p[p] = b->shards_p[p];
    t->samples_p[p] = b->samples_p[p];
    t->prefix_p[p] = b->prefix_p[p];
  }
  t->passes = b->passes;
  t->wide = b->wide != 0;
  t->fold16 = b->fold16 != 0;
  return FVB_OK;
}

// Records of encoder pass 0 and of the later passes (region "b", sized for
// the frames that take part in pass 1: a prefix of the batch, so the same
// global shard and sample indices address both regions).
struct EncLayout {
  size_t dims, frames, state, outs, queue, results, shards, folded, rans, prefix, recon;
  size_t shards_b, folded_b, rans_b, prefix_b, total;
};

EncLayout enc_layout(const Totals& t) {
  EncLayout w;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes);
    return r;
  };
  const size_t n = static_cast<size_t>(t.frames);
  w.dims = take(sizeof(BatchDims));
  w.frames = take(sizeof(FrameDesc) * n);
  w.state = take(sizeof(FrameState) * n);
  w.outs = take(sizeof(uint8_t*) * n);
  w.queue = take(kAlign);
  w.results = take(16 * static_cast<size_t>(n));
  w.shards = take(sizeof(ShardInfo) * t.shards);
  w.folded = take((t.fold16 ? 2 : 4) * static_cast<size_t>(t.samples));
  w.rans = take(static_cast<size_t>(kRansScratchBytes) * t.shards);
  w.prefix = take(static_cast<size_t>(t.prefix));
  w.recon = take(t.wide ? 2 * static_cast<size_t>(t.samples) : 0);
  const bool later = t.passes > 1;
  w.shards_b = take(later ? sizeof(ShardInfo) * t.shards_p[1] : 0);
  w.folded_b = take(later ? (t.fold16 ? 2 : 4) * static_cast<size_t>(t.samples_p[1]) : 0);
  w.rans_b = take(later ? static_cast<size_t>(kRansScratchBytes) * t.shards_p[1] : 0);
  w.prefix_b = take(later ? static_cast<size_t>(t.prefix_p[1]) : 0);
  w.total = o;
  return w;
}

struct DecLayout {
  size_t dims, frames, state, queue, results, shards, lists, items, tables, folded, total;
};

DecLayout dec_layout(const Totals& t) {
  DecLayout w;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t r = o;
    o = align_up(o + bytes);
    return r;
  };
  const size_t n = static_cast<size_t>(t.frames);
  w.dims = take(sizeof(BatchDims));
  w.frames = take(sizeof(FrameDesc) * n);
  w.state = take(sizeof(FrameState) * n);
  w.queue = take(kAlign);
  w.results = take(16 * static_cast<size_t>(n));
  w.shards = take(sizeof(ShardInfo) * t.shards);
  w.lists = take(sizeof(DecodeLists));
  w.items = take(4 * 4 * static_cast<size_t>(t.shards));
  w.tables = take(dec_rans_table_bytes() * static_cast<size_t>(t.shards));
  w.folded = take((t.fold16 ? 2 : 4) * static_cast<size_t>(t.samples));
  w.total = o;
  return w;
}

__global__ void gather_headers_kernel(const uint8_t* const* __restrict__ streams, const int64_t* __restrict__ lens,
                                      int n, uint8_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kHeaderBytes) return;
  const int k = i / kHeaderBytes, b = i % kHeaderBytes;
  out[i] = b < lens[k] ? streams[k][b] : 0;
}

// The 32-byte header of every frame of an encoded batch, in the caller's
// order, from the records region the frame emits (its final pass).
__global__ void encode_headers_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                                      const BatchDims* __restrict__ dims, const uint8_t* __restrict__ prefix_a,
                                      const uint8_t* __restrict__ prefix_b, uint8_t* __restrict__ out) {
  const int n = dims->frames_p[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kHeaderBytes) return;
  const int k = i / kHeaderBytes, b = i % kHeaderBytes;
  const FrameDesc& f = frames[k];
  out[f.slot * kHeaderBytes + b] = (state[k].final_b ? prefix_b : prefix_a)[f.prefix_base + b];
}

__global__ void results_kernel(const FrameDesc* __restrict__ frames, const FrameState* __restrict__ state,
                               const BatchDims* __restrict__ dims, int64_t* __restrict__ out, int decode) {
  const int n = dims->frames_p[0];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = frames[i].slot;
  out[2 * slot] = state[i].status;
  out[2 * slot + 1] = decode ? 0 : state[i].stream_len;
}

// Restores the caller's current device when an entry point returns: the
// library launches on the device that owns the workspace and switches to it
// for the call only.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// The device that a kernel can read `p` on: device memory, or managed memory
// (its preferred device); -1 for host, pinned-host or unknown pointers, which
// a kernel of this library must never be given.
int device_of(const void* p) {
  if (!p) return -1;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (attr.type == cudaMemoryTypeDevice) return attr.device;
  if (attr.type == cudaMemoryTypeManaged) return attr.device >= 0 ? attr.device : 0;
  return -1;
}

// The device's view of page-locked host memory (every cudaMallocHost /
// cudaHostAlloc allocation is mapped under unified addressing), or nullptr
// for pageable memory.  Small results (status words, stream lengths,
// headers) are written there by a kernel instead of a device-to-host copy:
// copies in that direction run in issue order on the copy engine, so a
// small copy issued while a large download is in flight on another stream
// would wait for all of it (measured on B200: a 64-byte copy waited for a
// 512 MB one), whereas kernel stores to host memory do not queue there.
void* host_mapped(void* p) {
  if (!p) return nullptr;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return attr.type == cudaMemoryTypeHost ? attr.devicePointer : nullptr;
}

int check_ws(void* ws, int64_t ws_bytes, size_t need) {
  if (!ws || ws_bytes < static_cast<int64_t>(need))
    return fail(FVB_ERR_WORKSPACE, "workspace is smaller than planned");
  if (reinterpret_cast<uintptr_t>(ws) & (kAlign - 1)) return fail(FVB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  // launch on the device that owns the workspace (the entry point's
  // DeviceGuard puts the caller's device back)
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, ws) == cudaSuccess && attr.type == cudaMemoryTypeDevice) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != attr.device) FVB_CUDA(cudaSetDevice(attr.device));
  } else {
    cudaGetLastError();
    return fail(FVB_ERR_WORKSPACE, "workspace must be device memory");
  }
  return FVB_OK;
}

int grid_for(int64_t items, int per_cta, int ctas_per_sm) {
  const int64_t want = ceil_div(items > 0 ? items : 1, per_cta);
  const int64_t cap = static_cast<int64_t>(device_sms()) * ctas_per_sm;
  return static_cast<int>(want < cap ? want : cap);
}

// Launch geometry of the persistent kernels: the grid is capped at this
// many CTAs per SM (0: the kernel has no such knob).  Outputs never depend on
// it -- every such kernel takes its work from a queue or a grid-stride loop.
constexpr int kDefaultCtas[K_COUNT] = {
    /*enc_init*/ 0, /*enc_predict*/ 4, /*enc_predict_wide*/ 8, /*enc_analyze*/ 6, /*enc_rans*/ 0,
    /*enc_scan*/ 0, /*enc_prefix*/ 0, /*enc_emit*/ 8, /*dec_parse*/ 8, /*dec_rans_tables*/ 16,
    /*dec_reconstruct*/ 4, /*dec_reconstruct_wide*/ 8, /*dec_reconstruct_serial*/ 0, /*results*/ 0,
    /*dec_rans*/ 16, /*dec_other*/ 16};
std::atomic<int> g_ctas[K_COUNT];
std::atomic<int> g_wavefront_block{kDefaultWavefrontBlock};
std::atomic<int> g_decode_overlap{1};
// rANS encoder fetch scheme per pass: 0, 8, 16, or -1 (automatic: the
// software pipeline over blocks of 8 steps when the launch leaves the SMs
// short of warps -- a single frame, the frame policy's later passes -- where
// the state chain would otherwise wait on its loads; the one-stage fetch,
// which holds fewer registers, when the launch fills the GPU)
std::atomic<int> g_rans_pipeline{-1};
std::atomic<int> g_rans_pipeline_tail{-1};
constexpr int kRansAutoCtasPerSm = 4;

int rans_pipe_for(int knob, int grid) {
  if (knob >= 0) return knob;
  return grid <= device_sms() * kRansAutoCtasPerSm ? 8 : 0;
}
std::atomic<int> g_tile_warps{kDefaultTileWarps};

int ctas(int kernel) {
  const int v = g_ctas[kernel].load(std::memory_order_relaxed);
  return v > 0 ? v : kDefaultCtas[kernel];
}

// The single-frame entry points read the stream and write the planes from
// kernels, so each must be device (or managed) memory: a host pointer is
// rejected here instead of faulting on the GPU.
int check_decode_pointers(const fvb_frame* frame, const uint8_t* stream, uint16_t* const* planes) {
  if (device_of(stream) < 0) return fail(FVB_ERR_ARGUMENT, "encoded stream must be device memory");
  for (int p = 0; p < frame->planes; ++p)
    if (device_of(planes[p]) < 0) return fail(FVB_ERR_ARGUMENT, "output planes must be device memory");
  return FVB_OK;
}

int check_plane_pointers(const fvb_frame* frame, const uint16_t* const* planes) {
  for (int p = 0; p < frame->planes; ++p)
    if (device_of(planes[p]) < 0) return fail(FVB_ERR_ARGUMENT, "input planes must be device memory");
  return FVB_OK;
}

// Profiling records CUDA events (created on demand); the allocation-free
// decode switches it off for its own launches.  The profiler is per thread,
// so no other thread sees the switch.
struct ProfilePause {
  bool was;
  ProfilePause() : was(g_prof.on) { g_prof.on = false; }
  ~ProfilePause() { g_prof.on = was; }
};

std::string status_message_encode(int64_t st) {
  if (st == kStatusInternal + 1) return "tile payload is too large";
  char buf[96];
  std::snprintf(buf, sizeof(buf), "CUDA encoder analysis failed (status %lld)", static_cast<long long>(st));
  return buf;
}

}  // namespace

// ===========================================================================
extern "C" {

int fvb_abi_version(void) { return FVB_ABI_VERSION; }

int64_t fvb_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int fvb_kernel_count(void) { return K_COUNT; }

int fvb_set_launch_ctas(int kernel, int ctas_per_sm) {
  if (kernel < 0 || kernel >= K_COUNT || kDefaultCtas[kernel] == 0)
    return fail(FVB_ERR_ARGUMENT, "kernel has no launch-geometry knob");
  if (ctas_per_sm < 0 || ctas_per_sm > 64) return fail(FVB_ERR_ARGUMENT, "CTAs per SM must be in 0..64");
  g_ctas[kernel].store(ctas_per_sm, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_launch_ctas(int kernel) {
  if (kernel < 0 || kernel >= K_COUNT || kDefaultCtas[kernel] == 0) return -1;
  return ctas(kernel);
}

int fvb_set_wavefront_block(int steps) {
  if (steps == 0) steps = kDefaultWavefrontBlock;
  if (steps != 4 && steps != 8 && steps != 16 && steps != 32)
    return fail(FVB_ERR_ARGUMENT, "wavefront block must be 4, 8, 16 or 32 steps");
  g_wavefront_block.store(steps, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_wavefront_block(void) { return g_wavefront_block.load(std::memory_order_relaxed); }

int fvb_set_decode_overlap(int on) {
  if (on != 0 && on != 1) return fail(FVB_ERR_ARGUMENT, "decode overlap must be 0 or 1");
  g_decode_overlap.store(on, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_decode_overlap(void) { return g_decode_overlap.load(std::memory_order_relaxed); }

int fvb_set_rans_pipeline(int steps) {
  if (steps != -1 && steps != 0 && steps != 8 && steps != 16)
    return fail(FVB_ERR_ARGUMENT, "rANS pipeline must be -1, 0, 8 or 16");
  g_rans_pipeline.store(steps, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_rans_pipeline(void) { return g_rans_pipeline.load(std::memory_order_relaxed); }

int fvb_set_rans_pipeline_tail(int steps) {
  if (steps != -1 && steps != 0 && steps != 8 && steps != 16)
    return fail(FVB_ERR_ARGUMENT, "rANS pipeline must be -1, 0, 8 or 16");
  g_rans_pipeline_tail.store(steps, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_rans_pipeline_tail(void) { return g_rans_pipeline_tail.load(std::memory_order_relaxed); }

int fvb_set_tile_warps(int warps) {
  if (warps == 0) warps = kDefaultTileWarps;
  if (warps != 1 && warps != 2) return fail(FVB_ERR_ARGUMENT, "warps per tile must be 1 or 2");
  g_tile_warps.store(warps, std::memory_order_relaxed);
  return FVB_OK;
}

int fvb_get_tile_warps(void) { return g_tile_warps.load(std::memory_order_relaxed); }

const char* fvb_kernel_name(int kernel) { return kernel >= 0 && kernel < K_COUNT ? kKernelNames[kernel] : ""; }

int fvb_profile_begin(void) {
  for (auto& r : g_prof.records) {
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.records.clear();
  g_prof.on = true;
  return FVB_OK;
}

int fvb_profile_end(double* ms, int64_t* launches, int n) {
  g_prof.on = false;
  for (int i = 0; i < n; ++i) {
    if (ms) ms[i] = 0.0;
    if (launches) launches[i] = 0;
  }
  for (auto& r : g_prof.records) {
    FVB_CUDA(cudaEventSynchronize(r.b));
    float t = 0.f;
    FVB_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kernel < n) {
      if (ms) ms[r.kernel] += t;
      if (launches) launches[r.kernel] += 1;
    }
    g_prof.pool.push_back(r.a);
    g_prof.pool.push_back(r.b);
  }
  g_prof.records.clear();
  return FVB_OK;
}

const char* fvb_last_error(void) { return g_error.c_str(); }

int fvb_encode_plan(int64_t width, int64_t height, int layout, int bit_depth, int quality, int64_t fps_num,
                    int64_t fps_den, int64_t tile_w, int64_t tile_h, fvb_frame* frame, int64_t* workspace_bytes) {
  // argument checks in the order of encode.cu:695-716
  if (!(layout >= 0 && layout <= 2)) return fail(FVB_ERR_ARGUMENT, "layout must be gray, yuv422, or rgb444");
  if (!(bit_depth == 8 || bit_depth == 10 || bit_depth == 12 || bit_depth == 16))
    return fail(FVB_ERR_ARGUMENT, "bit_depth must be 8, 10, 12, or 16");
  if (!(quality >= 1 && quality <= 100)) return fail(FVB_ERR_ARGUMENT, "quality must be in 1..=100");
  if (!(fps_num > 0 && fps_num <= 0xffffffffll && fps_den > 0 && fps_den <= 0xffffffffll))
    return fail(FVB_ERR_ARGUMENT, "frame-rate components must be nonzero u32 values");
  if (!(tile_w > 0 && tile_w <= 65535 && tile_h > 0 && tile_h <= 65535))
    return fail(FVB_ERR_ARGUMENT, "tile dimensions must be nonzero u16 values");
  if (!(width > 0 && height > 0 && width <= 0xffffffffll && height <= 0xffffffffll))
    return fail(FVB_ERR_ARGUMENT, "frame dimensions must be nonzero u32 values");
  if (width > 0x7fffffffll || height > 0x7fffffffll || width * height > (1ll << 36))
    return fail(FVB_ERR_ARGUMENT, "frame is too large");
  if (!frame) return fail(FVB_ERR_ARGUMENT, "frame is null");
  std::memset(frame, 0, sizeof(*frame));
  frame->layout = layout;
  frame->bit_depth = bit_depth;
  frame->quality = quality;
  frame->width = width;
  frame->height = height;
  frame->tile_w = tile_w;
  frame->tile_h = tile_h;
  frame->fps_num = fps_num;
  frame->fps_den = fps_den;
  frame->step = quantization_step(layout, bit_depth, quality);
  const int rc = fill_frame(frame);
  if (rc) return rc;
  if (workspace_bytes) {
    *workspace_bytes = static_cast<int64_t>(enc_layout(totals_of(frame, 1)).total);
  }
  return FVB_OK;
}

int fvb_batch_encode_plan(const fvb_frame* frames, int n, int64_t* workspace_bytes) {
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  *workspace_bytes = static_cast<int64_t>(enc_layout(totals_of(frames, n)).total);
  return FVB_OK;
}

int fvb_batch_bucket(const fvb_frame* frames, int n, fvb_bucket* bucket) {
  if (n <= 0 || !frames || !bucket) return fail(FVB_ERR_ARGUMENT, "empty batch");
  to_bucket(bucket_of(totals_of(frames, n)), bucket);
  return FVB_OK;
}

int fvb_bucket_encode_plan(const fvb_bucket* bucket, int64_t* workspace_bytes) {
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  *workspace_bytes = static_cast<int64_t>(enc_layout(cap).total);
  return FVB_OK;
}

}  // extern "C"

namespace {

// ---- encoder batch internals: `cap` sizes the workspace layout and the
// launch grids; the actual counts go to the device in BatchDims ------------

int encode_prepare(const Totals& cap, const fvb_frame* frames, int n, const uint16_t* const* planes,
                   const int64_t* pitches, void* workspace, int64_t workspace_bytes, void* cuda_stream) {
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  const Totals t = totals_of(frames, n);
  if (!fits(t, cap)) return fail(FVB_ERR_ARGUMENT, "batch does not fit the bucket");
  const EncLayout L = enc_layout(cap);
  int rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  // one upload: the dims record, then the frame table
  std::vector<unsigned char> table(L.frames + sizeof(FrameDesc) * n);
  const BatchDims dims = dims_of(t);
  std::memcpy(table.data() + L.dims, &dims, sizeof(dims));
  FrameDesc* descs = reinterpret_cast<FrameDesc*>(table.data() + L.frames);
  const std::vector<int> order = encode_order(frames, n);
  int64_t tb = 0, sb = 0, nb = 0, pb = 0;
  for (int j = 0; j < n; ++j) {
    const int i = order[j];
    FrameDesc& d = descs[j];
    build_desc(frames[i], d, frames[i].layout != 0);
    d.slot = i;
    for (int p = 0; p < d.planes; ++p) {
      const uint16_t* ptr = planes[3 * i + p];
      if (!ptr) return fail(FVB_ERR_ARGUMENT, "null plane pointer");
      d.src[p] = ptr;
      d.src_pitch[p] = pitches[3 * i + p];
      if (d.src_pitch[p] < d.plane_w[p]) return fail(FVB_ERR_ARGUMENT, "plane pitch is smaller than the plane width");
    }
    d.tile_base = tb;
    d.shard_base = sb;
    d.sample_base = nb;
    d.prefix_base = pb;
    tb += d.ntiles;
    sb += d.nshards;
    nb += d.nsamples;
    pb += d.prefix_bytes;
  }
  char* ws = static_cast<char*>(workspace);
  FVB_CUDA(cudaMemcpyAsync(ws, table.data(), table.size(), cudaMemcpyHostToDevice, stream));
  return FVB_OK;
}

int encode_enqueue(const Totals& cap, void* workspace, int64_t workspace_bytes, int64_t* results, void* cuda_stream) {
  const EncLayout L = enc_layout(cap);
  int rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  rc = ensure_smem_attrs();
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  char* ws = static_cast<char*>(workspace);
  const BatchDims* dims = reinterpret_cast<const BatchDims*>(ws + L.dims);
  const FrameDesc* frames_d = reinterpret_cast<const FrameDesc*>(ws + L.frames);
  FrameState* state = reinterpret_cast<FrameState*>(ws + L.state);
  int* queue = reinterpret_cast<int*>(ws + L.queue);
  const bool f16 = cap.fold16;  // u16 or u32 folded symbols
  uint16_t* recon = reinterpret_cast<uint16_t*>(ws + L.recon);
  const int n = cap.frames;
  {
    LaunchScope scope_(K_ENC_INIT, stream);
    enc_init_kernel<<<(n + 127) / 128, 128, 0, stream>>>(frames_d, state, dims);
  }
  FVB_LAUNCHED("enc_init_kernel");
  // pass p covers the batch's first frames_p[p] frames (layout order); the
  // later passes write region b
  for (int pass = 0; pass < cap.passes; ++pass) {
    const int nf = cap.frames_p[pass];
    const int64_t tiles = cap.tiles_p[pass], nsh = cap.shards_p[pass];
    ShardInfo* shards = reinterpret_cast<ShardInfo*>(ws + (pass ? L.shards_b : L.shards));
    void* folded = ws + (pass ? L.folded_b : L.folded);
    uint8_t* rans = reinterpret_cast<uint8_t*>(ws + (pass ? L.rans_b : L.rans));
    uint8_t* prefix = reinterpret_cast<uint8_t*>(ws + (pass ? L.prefix_b : L.prefix));
    FVB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), stream));
    {
      LaunchScope scope_(K_ENC_PREDICT, stream);
      const int tw = g_tile_warps.load(std::memory_order_relaxed);
      enc_predict_launch(g_wavefront_block.load(std::memory_order_relaxed), tw, f16,
                         grid_for(tiles * tw, kWarpsPerCta, ctas(K_ENC_PREDICT)), stream, frames_d, state, dims, pass,
                         shards, folded, queue);
    }
    FVB_LAUNCHED("enc_predict_kernel");
    if (cap.wide) {
      {
        LaunchScope scope_(K_ENC_PREDICT_WIDE, stream);
        enc_predict_wide_kernel<<<grid_for(tiles, 1, ctas(K_ENC_PREDICT_WIDE)), 256, 0, stream>>>(
            frames_d, state, dims, pass, folded, recon, f16 ? 1 : 0);
      }
      FVB_LAUNCHED("enc_predict_wide_kernel");
    }
    {
      // resident CTAs only: each warp streams its shards through one ring
      LaunchScope scope_(K_ENC_ANALYZE, stream);
      enc_analyze_launch(f16, grid_for(nsh, kWarpsPerCta, ctas(K_ENC_ANALYZE)), stream, frames_d, state, dims, pass,
                         shards, folded, rans);
    }
    FVB_LAUNCHED("enc_analyze_kernel");
    {
      LaunchScope scope_(K_ENC_RANS, stream);
      const int grid = static_cast<int>(ceil_div(nsh * 4 > 0 ? nsh * 4 : 1, 128));
      enc_rans_launch(rans_pipe_for((pass == 0 ? g_rans_pipeline : g_rans_pipeline_tail).load(std::memory_order_relaxed),
                                    grid),
                      f16, grid, stream, state, dims, pass, shards, folded, rans);
    }
    FVB_LAUNCHED("enc_rans_kernel");
    {
      LaunchScope scope_(K_ENC_SCAN, stream);
      enc_scan_kernel<<<nf > 0 ? nf : 1, 1024, 0, stream>>>(frames_d, state, dims, pass, shards, prefix);
    }
    FVB_LAUNCHED("enc_scan_kernel");
  }
  int64_t* res_d = reinterpret_cast<int64_t*>(ws + L.results);
  int64_t* direct = static_cast<int64_t*>(host_mapped(results));  // pinned: written by the kernel
  {
    LaunchScope scope_(K_RESULTS, stream);
    results_kernel<<<(n + 127) / 128, 128, 0, stream>>>(frames_d, state, dims, direct ? direct : res_d, 0);
  }
  FVB_LAUNCHED("results_kernel");
  if (results && !direct)
    FVB_CUDA(cudaMemcpyAsync(results, res_d, 16 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream));
  return FVB_OK;
}

int encode_emit(const Totals& cap, const fvb_frame* frames, int n, void* workspace, int64_t workspace_bytes,
                uint8_t* const* outs, void* cuda_stream) {
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  const Totals t = totals_of(frames, n);
  if (!fits(t, cap)) return fail(FVB_ERR_ARGUMENT, "batch does not fit the bucket");
  const EncLayout L = enc_layout(cap);
  int rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  rc = ensure_smem_attrs();
  if (rc) return rc;
  for (int i = 0; i < n; ++i)
    if (!outs[i]) return fail(FVB_ERR_ARGUMENT, "null output pointer");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  char* ws = static_cast<char*>(workspace);
  uint8_t** outs_d = reinterpret_cast<uint8_t**>(ws + L.outs);
  std::vector<uint8_t*> outs_laid(n);  // in batch layout order
  const std::vector<int> order = encode_order(frames, n);
  for (int j = 0; j < n; ++j) outs_laid[j] = outs[order[j]];
  FVB_CUDA(cudaMemcpyAsync(outs_d, outs_laid.data(), sizeof(uint8_t*) * n, cudaMemcpyHostToDevice, stream));
  const FrameDesc* frames_d = reinterpret_cast<const FrameDesc*>(ws + L.frames);
  int64_t max_prefix = 0;
  for (int i = 0; i < n; ++i) max_prefix = frames[i].prefix_bytes > max_prefix ? frames[i].prefix_bytes : max_prefix;
  dim3 gp(static_cast<unsigned>(ceil_div(max_prefix, 256 * 4) > 64 ? 64 : ceil_div(max_prefix, 256 * 4)), n);
  const FrameState* state = reinterpret_cast<const FrameState*>(ws + L.state);
  {
    LaunchScope scope_(K_ENC_PREFIX, stream);
    enc_prefix_kernel<<<gp, 256, 0, stream>>>(frames_d, state, n, reinterpret_cast<const uint8_t*>(ws + L.prefix),
                                              reinterpret_cast<const uint8_t*>(ws + L.prefix_b), outs_d);
  }
  FVB_LAUNCHED("enc_prefix_kernel");
  {
    LaunchScope scope_(K_ENC_EMIT, stream);
    enc_emit_launch(cap.fold16, grid_for(t.shards, kWarpsPerCta, ctas(K_ENC_EMIT)), enc_emit_smem(), stream, state,
                    EmitRegion{reinterpret_cast<const ShardInfo*>(ws + L.shards), ws + L.folded,
                               reinterpret_cast<const uint8_t*>(ws + L.rans), t.shards},
                    EmitRegion{reinterpret_cast<const ShardInfo*>(ws + L.shards_b), ws + L.folded_b,
                               reinterpret_cast<const uint8_t*>(ws + L.rans_b), t.passes > 1 ? t.shards_p[1] : 0},
                    t.shards, outs_d);
  }
  FVB_LAUNCHED("enc_emit_kernel");
  return FVB_OK;
}

}  // namespace

extern "C" {

int fvb_batch_encode_prepare(const fvb_frame* frames, int n, const uint16_t* const* planes, const int64_t* pitches,
                             void* workspace, int64_t workspace_bytes, void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  return encode_prepare(totals_of(frames, n), frames, n, planes, pitches, workspace, workspace_bytes, cuda_stream);
}

int fvb_batch_encode_enqueue(const fvb_frame* frames, int n, void* workspace, int64_t workspace_bytes,
                             int64_t* results, void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  return encode_enqueue(totals_of(frames, n), workspace, workspace_bytes, results, cuda_stream);
}

int fvb_batch_encode_emit(const fvb_frame* frames, int n, void* workspace, int64_t workspace_bytes,
                          uint8_t* const* outs, void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  return encode_emit(totals_of(frames, n), frames, n, workspace, workspace_bytes, outs, cuda_stream);
}

int fvb_bucket_encode_prepare(const fvb_bucket* bucket, const fvb_frame* frames, int n, const uint16_t* const* planes,
                              const int64_t* pitches, void* workspace, int64_t workspace_bytes, void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  return encode_prepare(cap, frames, n, planes, pitches, workspace, workspace_bytes, cuda_stream);
}

int fvb_bucket_encode_enqueue(const fvb_bucket* bucket, void* workspace, int64_t workspace_bytes, int64_t* results,
                              void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  return encode_enqueue(cap, workspace, workspace_bytes, results, cuda_stream);
}

int fvb_bucket_encode_emit(const fvb_bucket* bucket, const fvb_frame* frames, int n, void* workspace,
                           int64_t workspace_bytes, uint8_t* const* outs, void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  return encode_emit(cap, frames, n, workspace, workspace_bytes, outs, cuda_stream);
}

int fvb_bucket_encode_headers(const fvb_bucket* bucket, void* workspace, int64_t workspace_bytes, uint8_t* headers,
                              void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  if (!headers) return fail(FVB_ERR_ARGUMENT, "null argument");
  const EncLayout L = enc_layout(cap);
  rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  char* ws = static_cast<char*>(workspace);
  uint8_t* direct = static_cast<uint8_t*>(host_mapped(headers));
  if (!direct) return fail(FVB_ERR_ARGUMENT, "headers must be page-locked host memory");
  {
    LaunchScope scope_(K_RESULTS, stream);
    encode_headers_kernel<<<static_cast<int>(ceil_div(cap.frames * kHeaderBytes, 256)), 256, 0, stream>>>(
        reinterpret_cast<const FrameDesc*>(ws + L.frames), reinterpret_cast<const FrameState*>(ws + L.state),
        reinterpret_cast<const BatchDims*>(ws + L.dims), reinterpret_cast<const uint8_t*>(ws + L.prefix),
        reinterpret_cast<const uint8_t*>(ws + L.prefix_b), direct);
  }
  FVB_LAUNCHED("encode_headers_kernel");
  return FVB_OK;
}

int fvb_encode_analyze(const fvb_frame* frame, const uint16_t* const* planes, const int64_t* pitches, void* workspace,
                       int64_t workspace_bytes, void* cuda_stream, int64_t* stream_len) {
  DeviceGuard guard_;
  if (!frame || !planes || !pitches) return fail(FVB_ERR_ARGUMENT, "null argument");
  int rc = check_plane_pointers(frame, planes);
  if (rc) return rc;
  const uint16_t* p3[3] = {planes[0], frame->planes == 3 ? planes[1] : nullptr, frame->planes == 3 ? planes[2] : nullptr};
  const int64_t q3[3] = {pitches[0], frame->planes == 3 ? pitches[1] : 0, frame->planes == 3 ? pitches[2] : 0};
  rc = fvb_batch_encode_prepare(frame, 1, p3, q3, workspace, workspace_bytes, cuda_stream);
  if (rc) return rc;
  int64_t res[2] = {0, 0};
  rc = fvb_batch_encode_enqueue(frame, 1, workspace, workspace_bytes, res, cuda_stream);
  if (rc) return rc;
  FVB_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(cuda_stream)));
  if (res[0] != 0) return fail(static_cast<int>(res[0] < kStatusInternal ? res[0] : FVB_ERR_INTERNAL),
                               status_message_encode(res[0]));
  if (stream_len) *stream_len = res[1];
  return FVB_OK;
}

int fvb_encode_emit(const fvb_frame* frame, void* workspace, int64_t workspace_bytes, uint8_t* out, int64_t out_len,
                    void* cuda_stream) {
  DeviceGuard guard_;
  if (!frame || !out) return fail(FVB_ERR_ARGUMENT, "null argument");
  (void)out_len;
  uint8_t* outs[1] = {out};
  return fvb_batch_encode_emit(frame, 1, workspace, workspace_bytes, outs, cuda_stream);
}

// ---------------------------------------------------------------------------
// decode

int fvb_decode_plan(const uint8_t* b, int64_t header_len, int64_t size, fvb_frame* frame, int64_t* workspace_bytes) {
  // fastvid_cuda.cpp:142-183, same order and messages
  if (size < kHeaderBytes || header_len < kHeaderBytes || !b) return fail(FVB_ERR_FORMAT, "truncated Fastvid header");
  if (std::memcmp(b, "FVID", 4) != 0) return fail(FVB_ERR_FORMAT, "bad Fastvid magic");
  if (b[4] != 1) return fail(FVB_ERR_FORMAT, "unsupported Fastvid bitstream version");
  if (b[5] > 2) return fail(FVB_ERR_FORMAT, "unknown pixel layout");
  const int layout = b[5];
  const bool gray = layout == 0;
  const int quality = b[6];
  if (quality < 1 || quality > 100) return fail(FVB_ERR_FORMAT, "quality is out of range");
  const bool refined = (b[7] & 0x80) != 0;
  const bool gray_med = (b[7] & 0x40) != 0;
  const int depth = (b[7] & 0x3f) + 8;
  if (!(depth == 8 || depth == 10 || depth == 12 || depth == 16)) return fail(FVB_ERR_FORMAT, "unsupported high-bit depth");
  if (refined && !(gray && depth == 16 && quality < 100)) return fail(FVB_ERR_FORMAT, "invalid gray16 refinement flag");
  if (gray_med && !(gray && depth == 10 && quality < 100)) return fail(FVB_ERR_FORMAT, "invalid gray MED flag");
  auto u32 = [&](int o) {
    return static_cast<uint32_t>(b[o]) | (static_cast<uint32_t>(b[o + 1]) << 8) | (static_cast<uint32_t>(b[o + 2]) << 16) |
           (static_cast<uint32_t>(b[o + 3]) << 24);
  };
  const int64_t width = u32(8), height = u32(12);
  const int64_t tw = b[16] | (b[17] << 8), th = b[18] | (b[19] << 8);
  if (!(width > 0 && height > 0 && tw > 0 && th > 0)) return fail(FVB_ERR_FORMAT, "zero dimension");
  if (u32(20) == 0 || u32(24) == 0) return fail(FVB_ERR_FORMAT, "zero frame-rate component");
  const int64_t tile_count = u32(28);
  const int64_t expected = count_tiles(width, height, tw, th, layout);
  if (tile_count != expected) return fail(FVB_ERR_FORMAT, "tile count does not match dimensions");
  if (tile_count > kMaxTiles) return fail(FVB_ERR_FORMAT, "too many tiles");
  if (kHeaderBytes + tile_count * kDirBytes > size) return fail(FVB_ERR_FORMAT, "truncated tile directory");
  if (width > 0x7fffffffll || height > 0x7fffffffll || width * height > (1ll << 36))
    return fail(FVB_ERR_FORMAT, "frame is too large");
  if (!frame) return fail(FVB_ERR_ARGUMENT, "frame is null");
  std::memset(frame, 0, sizeof(*frame));
  frame->layout = layout;
  frame->bit_depth = depth;
  frame->quality = quality;
  frame->flags = b[7] & 0xc0;
  frame->width = width;
  frame->height = height;
  frame->tile_w = tw;
  frame->tile_h = th;
  frame->fps_num = u32(20);
  frame->fps_den = u32(24);
  frame->step = refined ? refined_gray16_step(quality) : quantization_step(layout, depth, quality);
  int rc = fill_frame(frame);
  if (rc) return rc;
  if (workspace_bytes) *workspace_bytes = static_cast<int64_t>(dec_layout(totals_of(frame, 1)).total);
  return FVB_OK;
}

int fvb_gather_headers(const uint8_t* const* streams, const int64_t* stream_lens, int n, void* scratch,
                       int64_t scratch_bytes, uint8_t* headers, void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !streams || !headers) return fail(FVB_ERR_ARGUMENT, "empty batch");
  const size_t need = align_up(16 * static_cast<size_t>(n)) + kHeaderBytes * static_cast<size_t>(n);
  int rc = check_ws(scratch, scratch_bytes, need);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  char* ws = static_cast<char*>(scratch);
  std::vector<uint64_t> table(2 * static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) {
    table[i] = reinterpret_cast<uint64_t>(streams[i]);
    table[n + i] = static_cast<uint64_t>(stream_lens[i]);
  }
  FVB_CUDA(cudaMemcpyAsync(ws, table.data(), 16 * static_cast<size_t>(n), cudaMemcpyHostToDevice, stream));
  uint8_t* direct = static_cast<uint8_t*>(host_mapped(headers));  // pinned: written by the kernel
  uint8_t* out_d = direct ? direct : reinterpret_cast<uint8_t*>(ws + align_up(16 * static_cast<size_t>(n)));
  {
    LaunchScope scope_(K_RESULTS, stream);
    gather_headers_kernel<<<static_cast<int>(ceil_div(n * kHeaderBytes, 256)), 256, 0, stream>>>(
        reinterpret_cast<const uint8_t* const*>(ws), reinterpret_cast<const int64_t*>(ws + 8 * static_cast<size_t>(n)),
        n, out_d);
  }
  FVB_LAUNCHED("gather_headers_kernel");
  if (!direct)
    FVB_CUDA(cudaMemcpyAsync(headers, out_d, kHeaderBytes * static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream));
  FVB_CUDA(cudaStreamSynchronize(stream));
  return FVB_OK;
}

int fvb_batch_decode_plan(const fvb_frame* frames, int n, int64_t* workspace_bytes) {
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  *workspace_bytes = static_cast<int64_t>(dec_layout(totals_of(frames, n)).total);
  return FVB_OK;
}

int fvb_bucket_decode_plan(const fvb_bucket* bucket, int64_t* workspace_bytes) {
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  *workspace_bytes = static_cast<int64_t>(dec_layout(cap).total);
  return FVB_OK;
}

}  // extern "C"

namespace {

// Device descriptors of a decode batch into caller-provided storage.
int fill_decode_descs(const fvb_frame* frames, int n, const uint8_t* const* streams, const int64_t* stream_lens,
                      uint16_t* const* planes, const int64_t* pitches, FrameDesc* descs) {
  int64_t tb = 0, sb = 0, nb = 0;
  for (int i = 0; i < n; ++i) {
    FrameDesc& d = descs[i];
    const bool gray = frames[i].layout == 0;
    build_desc(frames[i], d, ((frames[i].flags & 0x40) != 0) || !gray);
    d.slot = i;
    if (!streams[i]) return fail(FVB_ERR_ARGUMENT, "null stream pointer");
    d.stream = streams[i];
    d.stream_len = stream_lens[i];
    for (int p = 0; p < d.planes; ++p) {
      if (!planes[3 * i + p]) return fail(FVB_ERR_ARGUMENT, "null plane pointer");
      d.dst[p] = planes[3 * i + p];
      d.dst_pitch[p] = pitches[3 * i + p];
      if (d.dst_pitch[p] < d.plane_w[p]) return fail(FVB_ERR_ARGUMENT, "plane pitch is smaller than the plane width");
    }
    d.tile_base = tb;
    d.shard_base = sb;
    d.sample_base = nb;
    tb += d.ntiles;
    sb += d.nshards;
    nb += d.nsamples;
  }
  return FVB_OK;
}


int decode_prepare(const Totals& cap, const fvb_frame* frames, int n, const uint8_t* const* streams,
                   const int64_t* stream_lens, uint16_t* const* planes, const int64_t* pitches, void* workspace,
                   int64_t workspace_bytes, void* cuda_stream) {
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  const Totals t = totals_of(frames, n);
  if (!fits(t, cap)) return fail(FVB_ERR_ARGUMENT, "batch does not fit the bucket");
  const DecLayout L = dec_layout(cap);
  int rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  // one upload: the dims record, then the frame table
  std::vector<unsigned char> table(L.frames + sizeof(FrameDesc) * n);
  const BatchDims dims = dims_of(t);
  std::memcpy(table.data() + L.dims, &dims, sizeof(dims));
  rc = fill_decode_descs(frames, n, streams, stream_lens, planes, pitches,
                         reinterpret_cast<FrameDesc*>(table.data() + L.frames));
  if (rc) return rc;
  FVB_CUDA(cudaMemcpyAsync(workspace, table.data(), table.size(), cudaMemcpyHostToDevice, stream));
  return FVB_OK;
}

// The decode launch sequence.  `side_ok`: large batches may run dec_other on
// the calling thread's side stream (created on first use); the
// allocation-free decode passes false, so it never creates a stream.
int decode_enqueue(const Totals& t, int wavefront, void* workspace, int64_t workspace_bytes, int64_t* results,
                   void* cuda_stream, bool side_ok) {
  const int n = t.frames;
  const DecLayout L = dec_layout(t);
  int rc = check_ws(workspace, workspace_bytes, L.total);
  if (rc) return rc;
  rc = ensure_smem_attrs();
  if (rc) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  char* ws = static_cast<char*>(workspace);
  const BatchDims* dims = reinterpret_cast<const BatchDims*>(ws + L.dims);
  const FrameDesc* frames_d = reinterpret_cast<const FrameDesc*>(ws + L.frames);
  FrameState* state = reinterpret_cast<FrameState*>(ws + L.state);
  int* queue = reinterpret_cast<int*>(ws + L.queue);
  ShardInfo* shards = reinterpret_cast<ShardInfo*>(ws + L.shards);
  void* folded = ws + L.folded;  // u16 or u32 symbols (t.fold16)
  const bool f16 = t.fold16;
  DecodeLists* lists = reinterpret_cast<DecodeLists*>(ws + L.lists);
  int32_t* items = reinterpret_cast<int32_t*>(ws + L.items);
  FVB_CUDA(cudaMemsetAsync(state, 0, sizeof(FrameState) * n, stream));
  FVB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), stream));
  FVB_CUDA(cudaMemsetAsync(lists, 0, sizeof(DecodeLists), stream));
  {
    LaunchScope scope_(K_DEC_PARSE, stream);
    dec_parse_kernel<<<grid_for(t.tiles, 128, ctas(K_DEC_PARSE)), 128, 0, stream>>>(frames_d, state, dims, shards, lists,
                                                                                      items);
  }
  FVB_LAUNCHED("dec_parse_kernel");
  RansTable* tables = reinterpret_cast<RansTable*>(ws + L.tables);
  {
    LaunchScope scope_(K_DEC_SHARDS, stream);
    dec_rans_tables_kernel<<<grid_for(t.shards, 128, ctas(K_DEC_SHARDS)), 128, 0, stream>>>(frames_d, state, shards, lists, items,
                                                                           tables);
  }
  FVB_LAUNCHED("dec_rans_tables_kernel");
  SideStream* side = nullptr;
  if (side_ok && t.shards >= kSideStreamShards && g_decode_overlap.load(std::memory_order_relaxed)) {
    rc = side_stream(&side);
    if (rc) return rc;
  }
  if (side) FVB_CUDA(cudaEventRecord(side->fork, stream));
  {
    LaunchScope scope_(K_DEC_RANS, stream);
    dec_rans_launch(f16, grid_for(ceil_div(t.shards, kGroupShards), kWarpsPerCta, ctas(K_DEC_RANS)), dec_rans_smem(),
                    stream, frames_d, state, shards, lists, items, tables, folded);
  }
  FVB_LAUNCHED("dec_rans_kernel");
  {
    // launched after dec_rans, so the rANS decoder's CTAs are placed first
    cudaStream_t other = side ? side->stream : stream;
    if (side) FVB_CUDA(cudaStreamWaitEvent(other, side->fork, 0));
    {
      LaunchScope scope_(K_DEC_OTHER, other);
      dec_other_launch(f16, grid_for(ceil_div(t.shards, kGroupShards), 4, ctas(K_DEC_OTHER)), other, frames_d, state,
                       shards, dims, lists, items, folded);
    }
    const cudaError_t launched = cudaGetLastError();
    if (side) {  // joined even when the launch failed, so a stream capture is never left forked
      FVB_CUDA(cudaEventRecord(side->join, other));
      FVB_CUDA(cudaStreamWaitEvent(stream, side->join, 0));
    }
    if (launched != cudaSuccess) return cuda_fail(launched, "dec_other_kernel");
  }
  if (wavefront) {
    {
      LaunchScope scope_(K_DEC_RECON, stream);
      const int tw = g_tile_warps.load(std::memory_order_relaxed);
      dec_reconstruct_launch(g_wavefront_block.load(std::memory_order_relaxed), tw, f16,
                             grid_for(t.tiles * tw, kWarpsPerCta, ctas(K_DEC_RECON)), stream, frames_d, state, dims,
                             folded, queue);
    }
    FVB_LAUNCHED("dec_reconstruct_kernel");
    if (t.wide) {
      {
        LaunchScope scope_(K_DEC_RECON_WIDE, stream);
        dec_reconstruct_wide_kernel<<<grid_for(t.tiles, 1, ctas(K_DEC_RECON_WIDE)), 256, 0, stream>>>(
            frames_d, state, dims, folded, f16 ? 1 : 0);
      }
      FVB_LAUNCHED("dec_reconstruct_wide_kernel");
    }
  } else {
    {
      LaunchScope scope_(K_DEC_RECON_SERIAL, stream);
      dec_reconstruct_serial_kernel<<<static_cast<int>(ceil_div(t.tiles, 128)), 128, 0, stream>>>(
          frames_d, state, dims, folded, f16 ? 1 : 0);
    }
    FVB_LAUNCHED("dec_reconstruct_serial_kernel");
  }
  int64_t* res_d = reinterpret_cast<int64_t*>(ws + L.results);
  int64_t* direct = static_cast<int64_t*>(host_mapped(results));  // pinned: written by the kernel
  {
    LaunchScope scope_(K_RESULTS, stream);
    results_kernel<<<(n + 127) / 128, 128, 0, stream>>>(frames_d, state, dims, direct ? direct : res_d, 1);
  }
  FVB_LAUNCHED("results_kernel");
  if (results && !direct)
    FVB_CUDA(cudaMemcpyAsync(results, res_d, 16 * static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream));
  return FVB_OK;
}


}  // namespace

extern "C" {

int fvb_batch_decode_prepare(const fvb_frame* frames, int n, const uint8_t* const* streams, const int64_t* stream_lens,
                             uint16_t* const* planes, const int64_t* pitches, void* workspace, int64_t workspace_bytes,
                             void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  return decode_prepare(totals_of(frames, n), frames, n, streams, stream_lens, planes, pitches, workspace,
                        workspace_bytes, cuda_stream);
}

int fvb_batch_decode_enqueue(const fvb_frame* frames, int n, int wavefront, void* workspace, int64_t workspace_bytes,
                             int64_t* results, void* cuda_stream) {
  DeviceGuard guard_;
  if (n <= 0 || !frames) return fail(FVB_ERR_ARGUMENT, "empty batch");
  return decode_enqueue(totals_of(frames, n), wavefront, workspace, workspace_bytes, results, cuda_stream, true);
}

int fvb_bucket_decode_prepare(const fvb_bucket* bucket, const fvb_frame* frames, int n, const uint8_t* const* streams,
                              const int64_t* stream_lens, uint16_t* const* planes, const int64_t* pitches,
                              void* workspace, int64_t workspace_bytes, void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  return decode_prepare(cap, frames, n, streams, stream_lens, planes, pitches, workspace, workspace_bytes,
                        cuda_stream);
}

int fvb_bucket_decode_enqueue(const fvb_bucket* bucket, int wavefront, void* workspace, int64_t workspace_bytes,
                              int64_t* results, void* cuda_stream) {
  DeviceGuard guard_;
  Totals cap;
  const int rc = from_bucket(bucket, &cap);
  if (rc) return rc;
  return decode_enqueue(cap, wavefront, workspace, workspace_bytes, results, cuda_stream, true);
}

int fvb_decode(const fvb_frame* frame, const uint8_t* stream, int64_t stream_len, uint16_t* const* planes,
               const int64_t* pitches, int wavefront, void* workspace, int64_t workspace_bytes, void* cuda_stream) {
  DeviceGuard guard_;
  if (!frame || !planes || !pitches) return fail(FVB_ERR_ARGUMENT, "null argument");
  int rc = check_decode_pointers(frame, stream, planes);
  if (rc) return rc;
  uint16_t* p3[3] = {planes[0], frame->planes == 3 ? planes[1] : nullptr, frame->planes == 3 ? planes[2] : nullptr};
  const int64_t q3[3] = {pitches[0], frame->planes == 3 ? pitches[1] : 0, frame->planes == 3 ? pitches[2] : 0};
  const uint8_t* s1[1] = {stream};
  const int64_t l1[1] = {stream_len};
  rc = fvb_batch_decode_prepare(frame, 1, s1, l1, p3, q3, workspace, workspace_bytes, cuda_stream);
  if (rc) return rc;
  int64_t res[2] = {0, 0};
  rc = fvb_batch_decode_enqueue(frame, 1, wavefront, workspace, workspace_bytes, res, cuda_stream);
  if (rc) return rc;
  FVB_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(cuda_stream)));
  if (res[0] != 0) {
    char buf[96];
    std::snprintf(buf, sizeof(buf), "malformed entropy payload (CUDA status %lld)", static_cast<long long>(res[0]));
    return fail(static_cast<int>(res[0]), buf);
  }
  return FVB_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free decode.
//
// Some callers cannot allocate device memory when they decode: plug-ins
// inside media frameworks that are handed pre-allocated frame buffers while
// the host application owns the device heap, real-time pipelines that forbid
// allocation after start-up (cudaMalloc and cudaFree can block and
// synchronise the device), and components that run under a device-memory
// budget enforced elsewhere.  fvb_decode_noalloc serves them: its scratch is
// one file-scope __device__ array of kNoAllocScratchBytes, so the call needs
// no workspace and allocates nothing.  The array exists on every GPU that
// loads this library, for the life of the process.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_address[64] = {nullptr};

// Device address of the scratch array on `device`.  Host code only holds a
// host-side stand-in for the array's name, so the address is looked up once
// per device, with that device current, and cached.
int noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= 64) return fail(FVB_ERR_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_address[device]) {
    int cur = -1;
    FVB_CUDA(cudaGetDevice(&cur));
    if (cur != device) FVB_CUDA(cudaSetDevice(device));
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    // the kernels' shared-memory limits are set here too, so that later calls
    // only launch
    const int attrs = e == cudaSuccess ? ensure_smem_attrs() : FVB_OK;
    if (cur != device) cudaSetDevice(cur);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    if (attrs) return attrs;
    g_noalloc_address[device] = ptr;
  }
  *out = g_noalloc_address[device];
  return FVB_OK;
}

}  // namespace

extern "C" {

int64_t fvb_decode_noalloc_capacity(void) { return static_cast<int64_t>(kNoAllocScratchBytes); }

int fvb_decode_noalloc(const fvb_frame* frame, const uint8_t* stream, int64_t stream_len, uint16_t* const* planes,
                       const int64_t* pitches, int wavefront, void* cuda_stream) {
  DeviceGuard guard_;
  if (!frame || !stream || !planes || !pitches) return fail(FVB_ERR_ARGUMENT, "null argument");
  const Totals t = totals_of(frame, 1);
  const DecLayout L = dec_layout(t);
  if (L.total > kNoAllocScratchBytes) {
    char buf[192];
    std::snprintf(buf, sizeof(buf),
                  "frame needs %zu bytes of decode scratch; the allocation-free decode has %zu "
                  "(frames up to about 7 million samples)",
                  L.total, kNoAllocScratchBytes);
    return fail(FVB_ERR_WORKSPACE, buf);
  }
  int rc = check_decode_pointers(frame, stream, planes);
  if (rc) return rc;
  // the device that holds the output planes does the work
  void* scratch = nullptr;
  rc = noalloc_scratch(device_of(planes[0]), &scratch);
  if (rc) return rc;
  const ProfilePause no_events;
  uint16_t* p3[3] = {planes[0], frame->planes == 3 ? planes[1] : nullptr, frame->planes == 3 ? planes[2] : nullptr};
  const int64_t q3[3] = {pitches[0], frame->planes == 3 ? pitches[1] : 0, frame->planes == 3 ? pitches[2] : 0};
  const uint8_t* s1[1] = {stream};
  const int64_t l1[1] = {stream_len};
  cudaStream_t cs = static_cast<cudaStream_t>(cuda_stream);
  int64_t res[2] = {0, 0};
  FrameDesc desc;
  rc = check_ws(scratch, static_cast<int64_t>(kNoAllocScratchBytes), L.total);
  if (rc) return rc;
  rc = fill_decode_descs(frame, 1, s1, l1, p3, q3, &desc);
  if (rc) return rc;
  const BatchDims dims = dims_of(t);
  FVB_CUDA(cudaMemcpyAsync(static_cast<char*>(scratch) + L.dims, &dims, sizeof(BatchDims), cudaMemcpyHostToDevice,
                           cs));
  FVB_CUDA(cudaMemcpyAsync(static_cast<char*>(scratch) + L.frames, &desc, sizeof(FrameDesc), cudaMemcpyHostToDevice,
                           cs));
  // no side stream: dec_other runs on the caller's stream, so nothing is created
  rc = decode_enqueue(t, wavefront, scratch, static_cast<int64_t>(kNoAllocScratchBytes), res, cuda_stream, false);
  if (rc) return rc;
  FVB_CUDA(cudaStreamSynchronize(cs));
  if (res[0] != 0) {
    char buf[96];
    std::snprintf(buf, sizeof(buf), "malformed entropy payload (CUDA status %lld)", static_cast<long long>(res[0]));
    return fail(static_cast<int>(res[0]), buf);
  }
  return FVB_OK;
}

}  // extern "C"
