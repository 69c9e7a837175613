/*
 * fastvid_oracle.c -- CPU restatement of the fastvid intra codec.
 *
 * TEST INFRASTRUCTURE ONLY (parity oracle and timed CPU baseline).  Nothing
 * in the fastvid_b200 product path links, loads or calls this file.
 *
 * It restates, step by step, the reference CUDA codec:
 *   cuda/csrc/encode.cu        predictor, quantizer, shard analysis, rANS,
 *                              emission, frame policy, header/directory
 *   cuda/csrc/decode.cu        shard parsers and every rejection rule,
 *                              reconstruction
 *   cuda/csrc/fastvid_cuda.cpp header validation and host directory parse
 * Scalar code, raster order inside a tile (the antidiagonal order of the
 * reference computes the same values because every sample depends only on
 * its left, upper and upper-left neighbours).  Tiles and shards are
 * independent, so an optional thread pool splits them across host cores.
 */
#include "fastvid_oracle.h"

#include <pthread.h>
#include <stdarg.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum {
  kHeaderBytes = 32,
  kDirectoryEntryBytes = 32,
  kShardSymbols = 4096,
  kBlockSymbols = 128,
  kMaxRice = 16,
  kModeZeroRun = 0,
  kModeRiceBase = 1,
  kModeBlockPack = 18,
  kModeOrder0 = 19,
  kRansAlphabet = 511,
  kRansTableLog = 12,
  kPredictTag = 6,
  kMaxTiles = 1 << 20,
};
#define kRansL (1u << 23)

/* ------------------------------------------------------------------ */
/* small helpers                                                       */

static void set_msg(char* msg, int msg_len, const char* fmt, ...) {
  if (!msg || msg_len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, (size_t)msg_len, fmt, ap);
  va_end(ap);
}

static int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
static int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }
static int32_t min32(int32_t a, int32_t b) { return a < b ? a : b; }

/* encode.cu:108-114 */
static int varint_length(uint32_t v) {
  return v < (1u << 7) ? 1 : v < (1u << 14) ? 2 : v < (1u << 21) ? 3 : v < (1u << 28) ? 4 : 5;
}

/* encode.cu:445-456 */
static int write_varint(uint8_t* out, uint32_t v) {
  int n = 0;
  do {
    uint8_t b = (uint8_t)(v & 0x7f);
    v >>= 7;
    if (v) b |= 0x80;
    out[n++] = b;
  } while (v);
  return n;
}

static int bit_length(uint32_t v) {
  int n = 0;
  while (v) {
    ++n;
    v >>= 1;
  }
  return n;
}

static void put_u16(uint8_t* p, uint16_t v) {
  p[0] = (uint8_t)v;
  p[1] = (uint8_t)(v >> 8);
}
static void put_u32(uint8_t* p, uint32_t v) {
  for (int i = 0; i < 4; ++i) p[i] = (uint8_t)(v >> (8 * i));
}
static void put_u64(uint8_t* p, uint64_t v) {
  for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i));
}
static uint16_t get_u16(const uint8_t* p) { return (uint16_t)(p[0] | (p[1] << 8)); }
static uint32_t get_u32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t get_u64(const uint8_t* p) {
  return (uint64_t)get_u32(p) | ((uint64_t)get_u32(p + 4) << 32);
}

/* ------------------------------------------------------------------ */
/* thread pool: dynamic chunks over [0, n)                             */

typedef void (*range_fn)(void* ctx, int64_t begin, int64_t end);

typedef struct {
  range_fn fn;
  void* ctx;
  int64_t n;
  int64_t chunk;
  _Atomic int64_t next;
} pool_job;

static void* pool_worker(void* arg) {
  pool_job* job = (pool_job*)arg;
  for (;;) {
    int64_t b = atomic_fetch_add(&job->next, job->chunk);
    if (b >= job->n) break;
    job->fn(job->ctx, b, min64(job->n, b + job->chunk));
  }
  return NULL;
}

static void parallel_for(int threads, int64_t n, int64_t chunk, range_fn fn, void* ctx) {
  if (n <= 0) return;
  if (threads <= 1 || n <= chunk) {
    fn(ctx, 0, n);
    return;
  }
  pool_job job;
  job.fn = fn;
  job.ctx = ctx;
  job.n = n;
  job.chunk = chunk < 1 ? 1 : chunk;
  atomic_init(&job.next, 0);
  if (threads > 256) threads = 256;
  pthread_t tids[256];
  int started = 0;
  for (int i = 1; i < threads; ++i) {
    if (pthread_create(&tids[started], NULL, pool_worker, &job) == 0) ++started;
  }
  pool_worker(&job);
  for (int i = 0; i < started; ++i) pthread_join(tids[i], NULL);
}

/* ------------------------------------------------------------------ */
/* geometry (encode.cu:30-69, fastvid_cuda.cpp:111-137)                */

typedef struct {
  int64_t plane, x, y, w, h;
  int64_t folded_base, first_shard, shard_count;
  int64_t plane_base, plane_width;
} tile_t;

typedef struct {
  int64_t width, height, tile_w, tile_h;
  int layout;
  int64_t ntiles, nshards, nsamples;
  int64_t y_samples, secondary_width, secondary_samples;
  tile_t* tiles;
} geom_t;

static int64_t count_tiles(int64_t width, int64_t height, int64_t tw, int64_t th, int layout) {
  const int planes = layout == 0 ? 1 : 3;
  int64_t n = 0;
  const int64_t rows = (height + th - 1) / th;
  for (int p = 0; p < planes; ++p) {
    const int sub = layout == 1 && p != 0;
    const int64_t pw = sub ? (width + 1) / 2 : width;
    const int64_t nw = sub ? (tw + 1) / 2 : tw;
    n += rows * ((pw + nw - 1) / nw);
  }
  return n;
}

/* Builds the tile list; returns 0, or -1 when there are more than 2^20 tiles
 * (the reference checks the same bound after enumeration, encode.cu:735). */
static int geom_build(geom_t* g, int64_t width, int64_t height, int64_t tw, int64_t th, int layout) {
  memset(g, 0, sizeof(*g));
  g->width = width;
  g->height = height;
  g->tile_w = tw;
  g->tile_h = th;
  g->layout = layout;
  g->secondary_width = layout == 1 ? (width + 1) / 2 : width;
  g->y_samples = width * height;
  g->secondary_samples = g->secondary_width * height;
  const int64_t n = count_tiles(width, height, tw, th, layout);
  if (n > kMaxTiles) return -1;
  g->tiles = (tile_t*)calloc((size_t)(n ? n : 1), sizeof(tile_t));
  const int64_t plane_bases[3] = {0, g->y_samples, g->y_samples + g->secondary_samples};
  const int planes = layout == 0 ? 1 : 3;
  int64_t t = 0, folded = 0, shard = 0;
  for (int p = 0; p < planes; ++p) {
    const int sub = layout == 1 && p != 0;
    const int64_t pw = sub ? g->secondary_width : width;
    const int64_t nw = sub ? (tw + 1) / 2 : tw;
    for (int64_t y = 0; y < height; y += th) {
      for (int64_t x = 0; x < pw; x += nw) {
        tile_t* tl = &g->tiles[t++];
        tl->plane = p;
        tl->x = x;
        tl->y = y;
        tl->w = min64(nw, pw - x);
        tl->h = min64(th, height - y);
        const int64_t samples = tl->w * tl->h;
        tl->folded_base = folded;
        tl->first_shard = shard;
        tl->shard_count = (samples + kShardSymbols - 1) / kShardSymbols;
        tl->plane_base = plane_bases[p];
        tl->plane_width = pw;
        folded += samples;
        shard += tl->shard_count;
      }
    }
  }
  g->ntiles = n;
  g->nshards = shard;
  g->nsamples = folded;
  return 0;
}

static void geom_free(geom_t* g) {
  free(g->tiles);
  g->tiles = NULL;
}

int fvo_geometry(int64_t width, int64_t height, int layout, int64_t tile_w, int64_t tile_h,
                 int64_t* tiles, int64_t* shards, int64_t* samples) {
  geom_t g;
  if (geom_build(&g, width, height, tile_w, tile_h, layout) != 0) return -1;
  *tiles = g.ntiles;
  *shards = g.nshards;
  *samples = g.nsamples;
  geom_free(&g);
  return 0;
}

/* ------------------------------------------------------------------ */
/* quality -> step (encode.cu:71-89)                                   */

int32_t fvo_quantization_step(int layout, int bit_depth, int quality) {
  if ((layout == 0 && bit_depth == 8) || (layout == 1 && bit_depth == 8)) return 1;
  int32_t den = 6;
  if (layout == 1 && bit_depth == 10) den = 20;
  else if (layout == 1 && bit_depth == 16) den = 24;
  else if (layout == 2 && bit_depth == 10) den = 10;
  const int32_t scale = (int32_t)1 << (bit_depth - 8);
  return 1 + ((100 - quality) * scale + den - 1) / den;
}

int32_t fvo_refined_gray16_step(int quality) { return 1 + ((100 - quality) * 256 + 7) / 8; }

/* ------------------------------------------------------------------ */
/* predictor (encode.cu:128-193; decode.cu:552-656)                    */

static int32_t predict(int use_med, int32_t left, int32_t above, int32_t ul, int32_t max_sample) {
  if (use_med) {
    const int32_t mx = left > above ? left : above;
    const int32_t mn = left < above ? left : above;
    if (ul >= mx) return mn;
    if (ul <= mn) return mx;
    return left + above - ul;
  }
  return max32(0, min32(max_sample, left + above - ul));
}

static uint32_t zigzag(int32_t v) {
  return v >= 0 ? (uint32_t)v * 2u : (uint32_t)(-v) * 2u - 1u;
}
static int32_t unzigzag(uint32_t v) {
  return (v & 1) == 0 ? (int32_t)(v / 2) : -(int32_t)(v / 2) - 1;
}

typedef struct {
  const geom_t* g;
  const uint16_t* src;
  int32_t step, max_sample;
  int use_med;
  uint32_t* folded;
  uint16_t* recon;
  _Atomic int status;
} predict_ctx;

static void predict_range(void* vctx, int64_t begin, int64_t end) {
  predict_ctx* c = (predict_ctx*)vctx;
  for (int64_t t = begin; t < end; ++t) {
    const tile_t* tl = &c->g->tiles[t];
    for (int64_t y = 0; y < tl->h; ++y) {
      for (int64_t x = 0; x < tl->w; ++x) {
        const int64_t idx = tl->plane_base + (tl->y + y) * tl->plane_width + tl->x + x;
        const uint16_t s = c->src[idx];
        if (s > c->max_sample) {
          int zero = 0;
          atomic_compare_exchange_strong(&c->status, &zero, 1);
        }
        const int32_t left = x > 0 ? c->recon[idx - 1] : 0;
        const int32_t above = y > 0 ? c->recon[idx - tl->plane_width] : 0;
        const int32_t ul = (x > 0 && y > 0) ? c->recon[idx - tl->plane_width - 1] : 0;
        const int32_t pred = predict(c->use_med, left, above, ul, c->max_sample);
        const int32_t r = (int32_t)s - pred;
        const int32_t mag = ((r < 0 ? -r : r) + c->step / 2) / c->step;
        const int32_t q = r < 0 ? -mag : mag;
        const int32_t rec = max32(0, min32(c->max_sample, pred + q * c->step));
        c->recon[idx] = (uint16_t)rec;
        c->folded[tl->folded_base + y * tl->w + x] = zigzag(q);
      }
    }
  }
}

static int run_predict(const geom_t* g, const uint16_t* src, int32_t step, int32_t max_sample,
                       int use_med, uint32_t* folded, uint16_t* recon, int threads) {
  predict_ctx c;
  c.g = g;
  c.src = src;
  c.step = step;
  c.max_sample = max_sample;
  c.use_med = use_med;
  c.folded = folded;
  c.recon = recon;
  atomic_init(&c.status, 0);
  parallel_for(threads, g->ntiles, 4, predict_range, &c);
  return atomic_load(&c.status);
}

/* ------------------------------------------------------------------ */
/* per-shard analysis                                                  */

typedef struct {
  int64_t a[8]; /* mode, parameter, body, record, lane_bytes[4] (encode.cu:308-315) */
  /* order-0 rANS products (encode.cu:357-418) */
  int rans_ok;
  int table_len;         /* serialized table bytes (without lanes/states) */
  uint8_t table[1100];
  int lane_len[4];
  uint8_t lane[4][2048]; /* bytes in emission order (reversed on output) */
  uint32_t state[4];
} shard_analysis;

/* analyze_shards_kernel (encode.cu:195-317): Rice k search, zero-run and
 * block-pack costs, mode choice with the reference's tie rules. */
static void competition(const uint32_t* f, int count, int64_t* out, int* status) {
  const int lane_count = count < 4 ? count : 4;
  uint64_t lane_bits[kMaxRice + 1][4];
  memset(lane_bits, 0, sizeof(lane_bits));
  int64_t zero_bytes = 0;
  for (int i = 0; i < count; ++i) {
    const uint32_t v = f[i];
    const int lane = i % lane_count;
    for (int k = 0; k <= kMaxRice; ++k) lane_bits[k][lane] += (uint64_t)(v >> k) + 1 + (uint64_t)k;
    if (v != 0) {
      zero_bytes += varint_length(v * 2 - 1);
    } else if (i == 0 || f[i - 1] != 0) {
      uint32_t run = 1;
      while (i + (int)run < count && f[i + run] == 0) ++run;
      zero_bytes += varint_length((run - 1) * 2);
    }
  }
  int best_k = 0;
  int64_t best_lane_bytes = INT64_MAX;
  for (int k = 0; k <= kMaxRice; ++k) {
    int64_t bytes = 0;
    for (int l = 0; l < lane_count; ++l) bytes += (int64_t)((lane_bits[k][l] + 7) / 8);
    if (bytes < best_lane_bytes) {
      best_lane_bytes = bytes;
      best_k = k;
    }
  }
  const int64_t rice_body = (int64_t)(lane_count - 1) * 4 + best_lane_bytes;
  int64_t block_bytes = 0;
  for (int start = 0; start < count; start += kBlockSymbols) {
    const int n = count - start < kBlockSymbols ? count - start : kBlockSymbols;
    uint32_t mx = 0;
    for (int i = 0; i < n; ++i) mx = f[start + i] > mx ? f[start + i] : mx;
    const int w = bit_length(mx);
    block_bytes += 1 + (n * w + 7) / 8;
  }
  int mode;
  int64_t body;
  if (block_bytes < zero_bytes && block_bytes < rice_body) {
    mode = kModeBlockPack;
    body = block_bytes;
  } else if (zero_bytes <= rice_body) {
    mode = kModeZeroRun;
    body = zero_bytes;
  } else {
    mode = kModeRiceBase + best_k;
    body = rice_body;
  }
  if (body > 65535 && *status == 0) *status = 2;
  out[0] = mode;
  out[1] = best_k;
  out[2] = body;
  out[3] = body + 3;
  for (int l = 0; l < 4; ++l) out[4 + l] = l < lane_count ? (int64_t)((lane_bits[best_k][l] + 7) / 8) : 0;
}

/* analyze_order0_shards_kernel (encode.cu:319-431): histogram, 12-bit
 * normalisation, table serialisation and four interleaved rANS lanes.
 * Returns 1 when the shard is eligible (all values < 511, <= 255 symbols). */
static int order0(const uint32_t* f, int count, shard_analysis* sa) {
  uint32_t hist[kRansAlphabet];
  uint16_t freq[kRansAlphabet], cum[kRansAlphabet];
  memset(hist, 0, sizeof(hist));
  memset(freq, 0, sizeof(freq));
  memset(cum, 0, sizeof(cum));
  for (int i = 0; i < count; ++i) {
    if (f[i] >= kRansAlphabet) return 0;
    hist[f[i]]++;
  }
  int distinct = 0;
  for (int v = 0; v < kRansAlphabet; ++v) distinct += hist[v] != 0;
  if (distinct > 255) return 0;
  int cursor = 0;
  sa->table[cursor++] = kRansTableLog;
  cursor += write_varint(sa->table + cursor, (uint32_t)distinct);
  uint32_t assigned = 0, prefix = 0;
  int remaining = distinct, previous = 0;
  for (int v = 0; v < kRansAlphabet; ++v) {
    if (hist[v] == 0) continue;
    --remaining;
    prefix += hist[v];
    uint32_t end;
    if (remaining == 0) {
      end = 1u << kRansTableLog;
    } else {
      end = (uint32_t)(((uint64_t)prefix << kRansTableLog) / (uint64_t)count);
      if (end < assigned + 1) end = assigned + 1;
      if (end > (1u << kRansTableLog) - (uint32_t)remaining) end = (1u << kRansTableLog) - (uint32_t)remaining;
    }
    freq[v] = (uint16_t)(end - assigned);
    cum[v] = (uint16_t)assigned;
    cursor += write_varint(sa->table + cursor, (uint32_t)(v - previous));
    if (remaining != 0) cursor += write_varint(sa->table + cursor, end - assigned);
    assigned = end;
    previous = v;
  }
  sa->table_len = cursor;
  for (int lane = 0; lane < 4; ++lane) {
    uint32_t state = kRansL;
    int bytes = 0;
    for (int idx = count - 1 - ((count - 1 - lane) & 3); idx >= 0; idx -= 4) {
      const uint32_t v = f[idx];
      const uint32_t fr = freq[v];
      const uint64_t threshold = ((uint64_t)(kRansL >> kRansTableLog) << 8) * fr;
      while (state >= threshold) {
        sa->lane[lane][bytes++] = (uint8_t)state;
        state >>= 8;
      }
      state = ((state / fr) << kRansTableLog) + state % fr + cum[v];
    }
    sa->lane_len[lane] = bytes;
    sa->state[lane] = state;
  }
  return 1;
}

typedef struct {
  const geom_t* g;
  const uint32_t* folded;
  int force_order0;
  shard_analysis* sa;
  _Atomic int status;
} analyze_ctx;

static void shard_span(const geom_t* g, int64_t shard, int64_t* base, int* count);

static void analyze_range(void* vctx, int64_t begin, int64_t end) {
  analyze_ctx* c = (analyze_ctx*)vctx;
  for (int64_t s = begin; s < end; ++s) {
    int64_t base;
    int count;
    shard_span(c->g, s, &base, &count);
    const uint32_t* f = c->folded + base;
    shard_analysis* sa = &c->sa[s];
    int st = 0;
    /* Launch order of encode.cu:789-805: with force_order0 the rANS pass
     * runs first and the competition only fills shards it could not code. */
    if (!c->force_order0) competition(f, count, sa->a, &st);
    sa->rans_ok = order0(f, count, sa);
    if (sa->rans_ok) {
      /* table bytes + 3 lane lengths + 4 states + lanes (encode.cu:365, 421) */
      const int64_t body = (int64_t)sa->table_len + 12 + 16 + sa->lane_len[0] + sa->lane_len[1] +
                           sa->lane_len[2] + sa->lane_len[3];
      if (c->force_order0 || body < sa->a[2]) {
        sa->a[0] = kModeOrder0;
        sa->a[1] = kRansTableLog;
        sa->a[2] = body;
        sa->a[3] = body + 3;
        for (int l = 0; l < 4; ++l) sa->a[4 + l] = sa->lane_len[l];
      } else {
        sa->rans_ok = 0;
      }
    }
    if (c->force_order0 && !sa->rans_ok) competition(f, count, sa->a, &st);
    if (st) {
      int zero = 0;
      atomic_compare_exchange_strong(&c->status, &zero, st);
    }
  }
}

/* shard s -> folded base and symbol count (shard_metadata, encode.cu:747-760) */
static void shard_span(const geom_t* g, int64_t shard, int64_t* base, int* count) {
  int64_t lo = 0, hi = g->ntiles - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) / 2;
    if (g->tiles[mid].first_shard <= shard) lo = mid;
    else hi = mid - 1;
  }
  const tile_t* tl = &g->tiles[lo];
  const int64_t local = (shard - tl->first_shard) * kShardSymbols;
  *base = tl->folded_base + local;
  *count = (int)min64(kShardSymbols, tl->w * tl->h - local);
}

static int run_analysis(const geom_t* g, const uint32_t* folded, int force_order0,
                        shard_analysis* sa, int threads) {
  analyze_ctx c;
  c.g = g;
  c.folded = folded;
  c.force_order0 = force_order0;
  c.sa = sa;
  atomic_init(&c.status, 0);
  parallel_for(threads, g->nshards, 16, analyze_range, &c);
  return atomic_load(&c.status);
}

int fvo_predict(const uint16_t* samples, int64_t width, int64_t height, int layout, int bit_depth,
                int64_t tile_w, int64_t tile_h, int32_t step, int use_med, uint32_t* folded,
                uint16_t* recon) {
  geom_t g;
  if (geom_build(&g, width, height, tile_w, tile_h, layout) != 0) return -1;
  memset(recon, 0, (size_t)g.nsamples * sizeof(uint16_t));
  const int st = run_predict(&g, samples, step, (1 << bit_depth) - 1, use_med, folded, recon, 1);
  geom_free(&g);
  return st;
}

int fvo_analyze(const uint32_t* folded, int64_t width, int64_t height, int layout, int64_t tile_w,
                int64_t tile_h, int force_order0, int64_t* analysis) {
  geom_t g;
  if (geom_build(&g, width, height, tile_w, tile_h, layout) != 0) return -1;
  shard_analysis* sa = (shard_analysis*)calloc((size_t)(g.nshards ? g.nshards : 1), sizeof(shard_analysis));
  const int st = run_analysis(&g, folded, force_order0, sa, 1);
  for (int64_t s = 0; s < g.nshards; ++s) memcpy(analysis + s * 8, sa[s].a, sizeof(sa[s].a));
  free(sa);
  geom_free(&g);
  return st;
}

/* ------------------------------------------------------------------ */
/* emission (encode.cu:488-682)                                        */

static void set_bit(uint8_t* out, int64_t pos) { out[pos >> 3] |= (uint8_t)(1u << (pos & 7)); }

typedef struct {
  const geom_t* g;
  const uint32_t* folded;
  const shard_analysis* sa;
  const int64_t* offsets;
  uint8_t* out;
} emit_ctx;

static void emit_range(void* vctx, int64_t begin, int64_t end) {
  emit_ctx* c = (emit_ctx*)vctx;
  for (int64_t s = begin; s < end; ++s) {
    int64_t base;
    int count;
    shard_span(c->g, s, &base, &count);
    const uint32_t* f = c->folded + base;
    const int64_t* a = c->sa[s].a;
    uint8_t* rec = c->out + c->offsets[s];
    const int mode = (int)a[0];
    const int body_bytes = (int)a[2];
    rec[0] = (uint8_t)mode;
    put_u16(rec + 1, (uint16_t)body_bytes);
    uint8_t* body = rec + 3;
    if (mode == kModeZeroRun) { /* encode.cu:514-536 */
      int cur = 0;
      uint32_t run = 0;
      for (int i = 0; i < count; ++i) {
        if (f[i] == 0) {
          ++run;
        } else {
          if (run) {
            cur += write_varint(body + cur, (run - 1) * 2);
            run = 0;
          }
          cur += write_varint(body + cur, f[i] * 2 - 1);
        }
      }
      if (run) write_varint(body + cur, (run - 1) * 2);
    } else if (mode >= kModeRiceBase && mode <= kModeRiceBase + kMaxRice) { /* :538-585 */
      const int k = (int)a[1];
      const int lane_count = count < 4 ? count : 4;
      int64_t lane_off = (int64_t)(lane_count - 1) * 4;
      for (int l = 0; l < lane_count; ++l) {
        if (l + 1 < lane_count) put_u32(body + l * 4, (uint32_t)a[4 + l]);
        uint8_t* lo = body + lane_off;
        int64_t pos = 0;
        for (int i = l; i < count; i += lane_count) {
          const uint32_t v = f[i];
          const uint32_t q = v >> k;
          pos += q;
          set_bit(lo, pos++);
          for (int b = 0; b < k; ++b) {
            if ((v >> b) & 1u) set_bit(lo, pos);
            ++pos;
          }
        }
        lane_off += a[4 + l];
      }
    } else if (mode == kModeBlockPack) { /* :614-682 */
      int64_t cur = 0;
      for (int start = 0; start < count; start += kBlockSymbols) {
        const int n = count - start < kBlockSymbols ? count - start : kBlockSymbols;
        uint32_t mx = 0;
        for (int i = 0; i < n; ++i) mx = f[start + i] > mx ? f[start + i] : mx;
        const int w = bit_length(mx);
        body[cur++] = (uint8_t)w;
        int64_t pos = 0;
        for (int i = 0; i < n; ++i)
          for (int b = 0; b < w; ++b, ++pos)
            if ((f[start + i] >> b) & 1u) set_bit(body + cur, pos);
        cur += (n * w + 7) / 8;
      }
    } else if (mode == kModeOrder0) { /* :587-611 */
      const shard_analysis* sa = &c->sa[s];
      int cur = sa->table_len;
      memcpy(body, sa->table, (size_t)sa->table_len);
      for (int l = 0; l < 3; ++l) put_u32(body + cur + 4 * l, (uint32_t)sa->lane_len[l]);
      cur += 12;
      for (int l = 0; l < 4; ++l) put_u32(body + cur + 4 * l, sa->state[l]);
      cur += 16;
      for (int l = 0; l < 4; ++l) {
        for (int i = 0; i < sa->lane_len[l]; ++i) body[cur + i] = sa->lane[l][sa->lane_len[l] - 1 - i];
        cur += sa->lane_len[l];
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* encoder (encode.cu:686-931)                                         */

static int64_t total_payload(const shard_analysis* sa, int64_t n) {
  int64_t p = 0;
  for (int64_t s = 0; s < n; ++s) p += sa[s].a[3];
  return p;
}

int fvo_encode(const uint16_t* samples, int64_t width, int64_t height, int layout, int bit_depth,
               int quality, int64_t fps_num, int64_t fps_den, int64_t tile_w, int64_t tile_h,
               int threads, uint8_t** out, int64_t* out_len, char* msg, int msg_len) {
  *out = NULL;
  *out_len = 0;
  /* argument checks, encode.cu:695-725 */
  if (layout < 0 || layout > 2) {
    set_msg(msg, msg_len, "layout must be gray, yuv422, or rgb444");
    return -1;
  }
  if (!(bit_depth == 8 || bit_depth == 10 || bit_depth == 12 || bit_depth == 16)) {
    set_msg(msg, msg_len, "bit_depth must be 8, 10, 12, or 16");
    return -1;
  }
  if (quality < 1 || quality > 100) {
    set_msg(msg, msg_len, "quality must be in 1..=100");
    return -1;
  }
  if (!(fps_num > 0 && fps_num <= 0xffffffffLL && fps_den > 0 && fps_den <= 0xffffffffLL)) {
    set_msg(msg, msg_len, "frame-rate components must be nonzero u32 values");
    return -1;
  }
  if (!(tile_w > 0 && tile_w <= 65535 && tile_h > 0 && tile_h <= 65535)) {
    set_msg(msg, msg_len, "tile dimensions must be nonzero u16 values");
    return -1;
  }
  if (!(width > 0 && height > 0 && width <= 0xffffffffLL && height <= 0xffffffffLL)) {
    set_msg(msg, msg_len, "frame dimensions must be nonzero u32 values");
    return -1;
  }
  geom_t g;
  if (geom_build(&g, width, height, tile_w, tile_h, layout) != 0) {
    set_msg(msg, msg_len, "too many tiles");
    return -1;
  }
  const int64_t S = g.nsamples;
  uint32_t* folded = (uint32_t*)malloc((size_t)(S ? S : 1) * sizeof(uint32_t));
  uint16_t* recon = (uint16_t*)calloc((size_t)(S ? S : 1), sizeof(uint16_t));
  shard_analysis* sa = (shard_analysis*)calloc((size_t)(g.nshards ? g.nshards : 1), sizeof(shard_analysis));
  int32_t step = fvo_quantization_step(layout, bit_depth, quality);
  const int32_t max_sample = (1 << bit_depth) - 1;
  const int force_order0 = layout == 2 && (bit_depth != 10 || width < 3840);
  int rc = 0;

#define RUN_ANALYSIS(STEP, MED)                                                        \
  do {                                                                                 \
    int st_ = run_predict(&g, samples, (STEP), max_sample, (MED), folded, recon, threads); \
    int st2_ = run_analysis(&g, folded, force_order0, sa, threads);                    \
    if (!st_) st_ = st2_;                                                              \
    if (st_) {                                                                         \
      set_msg(msg, msg_len, "CUDA encoder analysis failed (status %d)", st_);          \
      rc = st_;                                                                        \
      goto done;                                                                       \
    }                                                                                  \
  } while (0)

  RUN_ANALYSIS(step, layout != 0);
  const int64_t baseline_payload = total_payload(sa, g.nshards);
  /* encode.cu:818-847: gray10 MED and gray16 refinement policies */
  const int gray_med = layout == 0 && bit_depth == 10 && step > 1 && baseline_payload * 10 > S * 3;
  if (gray_med) RUN_ANALYSIS(step, 1);
  int refined = 0;
  if (layout == 0 && bit_depth == 16 && step > 1) {
    const int direct = baseline_payload < S / 10 || baseline_payload > S / 2;
    const int probe = !direct && baseline_payload < S / 5;
    if (direct || probe) {
      const int32_t baseline_step = step;
      step = fvo_refined_gray16_step(quality);
      RUN_ANALYSIS(step, 0);
      const int64_t refined_payload = total_payload(sa, g.nshards);
      refined = direct || refined_payload < S / 10;
      if (!refined) {
        step = baseline_step;
        RUN_ANALYSIS(step, 0);
      }
    }
  }
  {
    /* offsets, tile lengths, header and directory (encode.cu:848-904) */
    const int64_t payload_start = kHeaderBytes + g.ntiles * kDirectoryEntryBytes;
    int64_t* offsets = (int64_t*)malloc((size_t)(g.nshards ? g.nshards : 1) * sizeof(int64_t));
    int64_t len = payload_start;
    for (int64_t s = 0; s < g.nshards; ++s) {
      offsets[s] = len;
      len += sa[s].a[3];
    }
    uint8_t* stream = (uint8_t*)calloc((size_t)len + 8, 1);
    memcpy(stream, "FVID", 4);
    stream[4] = 1;
    stream[5] = (uint8_t)layout;
    stream[6] = (uint8_t)quality;
    stream[7] = (uint8_t)((bit_depth - 8) | (gray_med ? 0x40 : 0) | (refined ? 0x80 : 0));
    put_u32(stream + 8, (uint32_t)width);
    put_u32(stream + 12, (uint32_t)height);
    put_u16(stream + 16, (uint16_t)tile_w);
    put_u16(stream + 18, (uint16_t)tile_h);
    put_u32(stream + 20, (uint32_t)fps_num);
    put_u32(stream + 24, (uint32_t)fps_den);
    put_u32(stream + 28, (uint32_t)g.ntiles);
    int64_t tile_off = payload_start;
    for (int64_t t = 0; t < g.ntiles; ++t) {
      const tile_t* tl = &g.tiles[t];
      int64_t tlen = 0;
      for (int64_t s = 0; s < tl->shard_count; ++s) tlen += sa[tl->first_shard + s].a[3];
      uint8_t* e = stream + kHeaderBytes + t * kDirectoryEntryBytes;
      e[0] = (uint8_t)tl->plane;
      e[1] = kModeOrder0; /* kEntropyParallelShards == 19 */
      e[2] = kPredictTag;
      e[3] = 0;
      put_u32(e + 4, (uint32_t)tl->x);
      put_u32(e + 8, (uint32_t)tl->y);
      put_u32(e + 12, (uint32_t)tl->w);
      put_u32(e + 16, (uint32_t)tl->h);
      put_u64(e + 20, (uint64_t)tile_off);
      if (tlen > 0xffffffffLL) {
        set_msg(msg, msg_len, "tile payload is too large");
        free(offsets);
        free(stream);
        rc = -1;
        goto done;
      }
      put_u32(e + 28, (uint32_t)tlen);
      tile_off += tlen;
    }
    emit_ctx ec;
    ec.g = &g;
    ec.folded = folded;
    ec.sa = sa;
    ec.offsets = offsets;
    ec.out = stream;
    parallel_for(threads, g.nshards, 16, emit_range, &ec);
    free(offsets);
    *out = stream;
    *out_len = len;
  }
done:
#undef RUN_ANALYSIS
  free(folded);
  free(recon);
  free(sa);
  geom_free(&g);
  return rc;
}

/* ------------------------------------------------------------------ */
/* decoder                                                             */

typedef struct {
  int64_t mode, body_offset, body_length, count, folded_base;
} shard_meta;

/* zero-run shard (decode.cu:237-295) */
static int decode_zero_run(const uint8_t* body, int64_t body_length, int64_t count,
                           uint32_t max_folded, uint32_t* out) {
  int64_t cursor = 0, produced = 0;
  while (produced < count) {
    uint32_t token = 0;
    int shift = 0, used = 0;
    for (;;) {
      if (cursor >= body_length || used == 5) return 1;
      const uint8_t byte = body[cursor++];
      if (used == 4 && byte > 0x0f) return 1;
      token |= (uint32_t)(byte & 0x7f) << shift;
      ++used;
      if ((byte & 0x80) == 0) break;
      shift += 7;
    }
    if (used != varint_length(token)) return 1;
    if ((token & 1) == 0) {
      const int64_t run = (int64_t)(token / 2) + 1;
      if (run > count - produced) return 1;
      for (int64_t i = 0; i < run; ++i) out[produced++] = 0;
    } else {
      const uint32_t value = (token + 1) / 2; /* u32 arithmetic as in the reference */
      if (value == 0 || value > max_folded) return 1;
      out[produced++] = value;
    }
  }
  return cursor != body_length ? 1 : 0;
}

/* Rice shard (decode.cu:63-125, 297-340) */
static int decode_rice(const uint8_t* body, int64_t body_length, int64_t count, int k,
                       uint32_t max_folded, uint32_t* out) {
  const int lane_count = (int)(count < 4 ? count : 4);
  const int64_t table_bytes = (int64_t)(lane_count - 1) * 4;
  if (table_bytes > body_length) return 2;
  for (int lane = 0; lane < lane_count; ++lane) {
    int64_t lane_off = table_bytes;
    for (int i = 0; i < lane; ++i) lane_off += get_u32(body + i * 4);
    const int64_t lane_len = lane + 1 < lane_count ? (int64_t)get_u32(body + lane * 4) : body_length - lane_off;
    if (lane_off > body_length || lane_len < 0 || lane_len > body_length - lane_off) return 2;
    const uint8_t* bytes = body + lane_off;
    const int64_t nbits = lane_len * 8;
    int64_t pos = 0;
    for (int64_t idx = lane; idx < count; idx += lane_count) {
      uint32_t q = 0;
      for (;;) {
        if (pos >= nbits) return 2;
        const int bit = (bytes[pos >> 3] >> (pos & 7)) & 1;
        ++pos;
        if (bit) break;
        ++q;
      }
      if (q > max_folded) return 2;
      if (pos + k > nbits) return 2;
      uint32_t r = 0;
      for (int b = 0; b < k; ++b, ++pos) r |= (uint32_t)((bytes[pos >> 3] >> (pos & 7)) & 1) << b;
      const uint64_t v = ((uint64_t)q << k) + r;
      if (v > max_folded) return 2;
      out[idx] = (uint32_t)v;
    }
    const int64_t used = (pos + 7) / 8;
    if (used != lane_len) return 2;
    if ((pos & 7) != 0) {
      const uint8_t mask = (uint8_t)~((1u << (pos & 7)) - 1);
      if (bytes[used - 1] & mask) return 2;
    }
  }
  return 0;
}

/* block-pack shard (decode.cu:342-396), blocks walked in order */
static int decode_block(const uint8_t* body, int64_t body_length, int64_t count,
                        uint32_t max_folded, uint32_t* out) {
  const int64_t nblocks = (count + kBlockSymbols - 1) / kBlockSymbols;
  const int max_width = bit_length(max_folded);
  int64_t cursor = 0;
  for (int64_t b = 0; b < nblocks; ++b) {
    if (cursor >= body_length) return 3;
    const int width = body[cursor++];
    if (width > max_width) return 3;
    const int64_t n = min64(kBlockSymbols, count - b * kBlockSymbols);
    const int64_t payload = (n * width + 7) / 8;
    if (payload > body_length - cursor) return 3;
    int64_t pos = 0;
    for (int64_t i = 0; i < n; ++i) {
      uint32_t v = 0;
      for (int bit = 0; bit < width; ++bit, ++pos)
        v |= (uint32_t)((body[cursor + (pos >> 3)] >> (pos & 7)) & 1) << bit;
      if (v > max_folded) return 3;
      out[b * kBlockSymbols + i] = v;
    }
    if ((pos & 7) != 0) {
      const uint8_t mask = (uint8_t)~((1u << (pos & 7)) - 1);
      if (body[cursor + payload - 1] & mask) return 3;
    }
    cursor += payload;
  }
  return cursor != body_length ? 3 : 0;
}

/* decode.cu:407-426 */
static int read_varint_o0(const uint8_t* body, int64_t len, int64_t* cursor, uint32_t* value) {
  uint32_t result = 0;
  int shift = 0;
  for (int used = 0; used < 5; ++used) {
    if (*cursor >= len) return 0;
    const uint8_t byte = body[(*cursor)++];
    if (used == 4 && byte > 0x0f) return 0;
    result |= (uint32_t)(byte & 0x7f) << shift;
    if ((byte & 0x80) == 0) {
      if (varint_length(result) != used + 1) return 0;
      *value = result;
      return 1;
    }
    shift += 7;
  }
  return 0;
}

/* order-0 rANS shard (decode.cu:428-550) */
static int decode_rans(const uint8_t* body, int64_t body_length, int64_t count,
                       uint32_t max_folded, uint32_t* out) {
  uint16_t values[256], freq[256], cum[256];
  uint8_t table[1 << kRansTableLog];
  int64_t cursor = 0;
  if (body_length < 1 || body[cursor++] != kRansTableLog) return 5;
  uint32_t n = 0;
  if (!read_varint_o0(body, body_length, &cursor, &n)) return 5;
  if (n == 0 || n > 255) return 5;
  uint32_t previous = 0, assigned = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t delta = 0;
    if (!read_varint_o0(body, body_length, &cursor, &delta) || (i != 0 && delta == 0) ||
        previous + delta > max_folded)
      return 5;
    const uint32_t value = previous + delta;
    uint32_t fr = (1u << kRansTableLog) - assigned;
    if (i + 1 != n && !read_varint_o0(body, body_length, &cursor, &fr)) return 5;
    /* decode.cu:479-480, with the sum taken without 32-bit wrap-around: a
     * frequency above 4096 - assigned is rejected even when the reference's
     * u32 sum would wrap (there the slot-table fill would run past its 4096
     * entries). */
    if (fr == 0 || fr > (1u << kRansTableLog) - assigned ||
        (i + 1 != n && fr == (1u << kRansTableLog) - assigned))
      return 5;
    values[i] = (uint16_t)value;
    freq[i] = (uint16_t)fr;
    cum[i] = (uint16_t)assigned;
    assigned += fr;
    previous = value;
  }
  if (assigned != (1u << kRansTableLog)) return 5;
  /* Three u32 lane lengths, four states, then the lanes.  The reference
   * stores the lengths as int; every stream with a length >= 2^31 or a
   * negative fourth length ends in a status-5 rejection there, which is the
   * rule written here directly. */
  int64_t lane_len[4];
  int64_t total = 0;
  for (int l = 0; l < 3; ++l) {
    if (cursor + 4 > body_length) return 5;
    lane_len[l] = get_u32(body + cursor);
    if (lane_len[l] >= (1LL << 31)) return 5;
    total += lane_len[l];
    cursor += 4;
  }
  if (cursor + 16 > body_length) return 5;
  uint32_t state[4];
  for (int l = 0; l < 4; ++l) {
    state[l] = get_u32(body + cursor + 4 * l);
    if (state[l] < kRansL) return 5;
  }
  cursor += 16;
  lane_len[3] = body_length - cursor - total;
  if (lane_len[3] < 0) return 5;
  int64_t lane_start[4];
  for (int l = 0; l < 4; ++l) {
    lane_start[l] = cursor;
    cursor += lane_len[l];
  }
  if (cursor != body_length) return 5;
  for (uint32_t s = 0; s < n; ++s)
    for (int slot = cum[s]; slot < cum[s] + freq[s]; ++slot) table[slot] = (uint8_t)s;
  for (int l = 0; l < 4; ++l) {
    uint32_t st = state[l];
    int64_t cur = 0;
    for (int64_t idx = l; idx < count; idx += 4) {
      const uint32_t slot = st & ((1u << kRansTableLog) - 1);
      const int sym = table[slot];
      out[idx] = values[sym];
      st = (uint32_t)freq[sym] * (st >> kRansTableLog) + slot - cum[sym];
      while (st < kRansL) {
        if (cur >= lane_len[l]) return 5;
        st = (st << 8) | body[lane_start[l] + cur++];
      }
    }
    if (cur != lane_len[l] || st != kRansL) return 5;
  }
  return 0;
}

typedef struct {
  const uint8_t* stream;
  const shard_meta* meta;
  uint32_t max_folded;
  uint32_t* folded;
  uint8_t* shard_status;
} dec_ctx;

static void decode_range(void* vctx, int64_t begin, int64_t end) {
  dec_ctx* c = (dec_ctx*)vctx;
  for (int64_t s = begin; s < end; ++s) {
    const shard_meta* m = &c->meta[s];
    const uint8_t* body = c->stream + m->body_offset;
    uint32_t* out = c->folded + m->folded_base;
    int st;
    if (m->mode == 0) st = decode_zero_run(body, m->body_length, m->count, c->max_folded, out);
    else if (m->mode >= 1 && m->mode <= 17)
      st = decode_rice(body, m->body_length, m->count, (int)m->mode - 1, c->max_folded, out);
    else if (m->mode == 18) st = decode_block(body, m->body_length, m->count, c->max_folded, out);
    else if (m->mode == 19) st = decode_rans(body, m->body_length, m->count, c->max_folded, out);
    else st = 4;
    c->shard_status[s] = (uint8_t)st;
  }
}

typedef struct {
  const geom_t* g;
  const uint32_t* folded;
  int32_t step, max_sample;
  int use_med;
  uint16_t* out;
} recon_ctx;

static void recon_range(void* vctx, int64_t begin, int64_t end) {
  recon_ctx* c = (recon_ctx*)vctx;
  for (int64_t t = begin; t < end; ++t) {
    const tile_t* tl = &c->g->tiles[t];
    for (int64_t y = 0; y < tl->h; ++y) {
      for (int64_t x = 0; x < tl->w; ++x) {
        const int64_t idx = tl->plane_base + (tl->y + y) * tl->plane_width + tl->x + x;
        const int32_t left = x > 0 ? c->out[idx - 1] : 0;
        const int32_t above = y > 0 ? c->out[idx - tl->plane_width] : 0;
        const int32_t ul = (x > 0 && y > 0) ? c->out[idx - tl->plane_width - 1] : 0;
        const int32_t pred = predict(c->use_med, left, above, ul, c->max_sample);
        const int32_t rec = pred + unzigzag(c->folded[tl->folded_base + y * tl->w + x]) * c->step;
        c->out[idx] = (uint16_t)max32(0, min32(c->max_sample, rec));
      }
    }
  }
}

int fvo_decode(const uint8_t* bytes, int64_t size, int wavefront, int threads, uint16_t** out,
               int64_t* out_samples, int64_t* width_out, int64_t* height_out, int* layout_out,
               int* depth_out, char* msg, int msg_len) {
  (void)wavefront;
  *out = NULL;
  *out_samples = 0;
  /* header validation, fastvid_cuda.cpp:142-183 */
#define FAIL(...)                          \
  do {                                     \
    set_msg(msg, msg_len, __VA_ARGS__);    \
    return -1;                             \
  } while (0)
  if (size < kHeaderBytes) FAIL("truncated Fastvid header");
  if (memcmp(bytes, "FVID", 4) != 0) FAIL("bad Fastvid magic");
  if (bytes[4] != 1) FAIL("unsupported Fastvid bitstream version");
  if (bytes[5] > 2) FAIL("unknown pixel layout");
  const int layout = bytes[5];
  const int gray = layout == 0;
  const int quality = bytes[6];
  if (quality < 1 || quality > 100) FAIL("quality is out of range");
  const int refined = (bytes[7] & 0x80) != 0;
  const int gray_med = (bytes[7] & 0x40) != 0;
  const int depth = (bytes[7] & 0x3f) + 8;
  if (!(depth == 8 || depth == 10 || depth == 12 || depth == 16)) FAIL("unsupported high-bit depth");
  if (refined && !(gray && depth == 16 && quality < 100)) FAIL("invalid gray16 refinement flag");
  if (gray_med && !(gray && depth == 10 && quality < 100)) FAIL("invalid gray MED flag");
  const int64_t width = get_u32(bytes + 8), height = get_u32(bytes + 12);
  const int64_t tw = get_u16(bytes + 16), th = get_u16(bytes + 18);
  if (!(width > 0 && height > 0 && tw > 0 && th > 0)) FAIL("zero dimension");
  if (get_u32(bytes + 20) == 0 || get_u32(bytes + 24) == 0) FAIL("zero frame-rate component");
  const int64_t tile_count = get_u32(bytes + 28);
  const int64_t expected = count_tiles(width, height, tw, th, layout);
  if (tile_count != expected) FAIL("tile count does not match dimensions");
  if (tile_count > kMaxTiles) FAIL("too many tiles");
  const int64_t directory_end = kHeaderBytes + tile_count * kDirectoryEntryBytes;
  if (directory_end > size) FAIL("truncated tile directory");
  geom_t g;
  if (geom_build(&g, width, height, tw, th, layout) != 0) FAIL("too many tiles");
#undef FAIL
#define GFAIL(...)                         \
  do {                                     \
    set_msg(msg, msg_len, __VA_ARGS__);    \
    free(meta);                            \
    geom_free(&g);                         \
    return -1;                             \
  } while (0)
  /* directory and shard headers, fastvid_cuda.cpp:255-333 */
  shard_meta* meta = (shard_meta*)calloc((size_t)(g.nshards ? g.nshards : 1), sizeof(shard_meta));
  int64_t next = directory_end;
  for (int64_t i = 0; i < tile_count; ++i) {
    const uint8_t* e = bytes + kHeaderBytes + i * kDirectoryEntryBytes;
    const tile_t* tl = &g.tiles[i];
    if (e[0] != tl->plane) GFAIL("non-canonical tile plane");
    if (e[1] != kModeOrder0) GFAIL("tile requires bounded-shard entropy");
    if (e[2] != kPredictTag) GFAIL("tile requires full-tile clamp-gradient prediction");
    if (e[3] != 0) GFAIL("nonzero reserved directory byte");
    if (!(get_u32(e + 4) == tl->x && get_u32(e + 8) == tl->y && get_u32(e + 12) == tl->w &&
          get_u32(e + 16) == tl->h))
      GFAIL("non-canonical tile directory");
    const uint64_t off = get_u64(e + 20);
    if (off > (uint64_t)INT64_MAX) GFAIL("payload offset is too large");
    const int64_t len = get_u32(e + 28);
    if ((int64_t)off != next) GFAIL("payloads are not contiguous");
    if (len > size - next) GFAIL("truncated tile payload");
    next += len;
  }
  if (next != size) GFAIL("trailing stream bytes");
  int64_t shard = 0;
  for (int64_t i = 0; i < tile_count; ++i) {
    const uint8_t* e = bytes + kHeaderBytes + i * kDirectoryEntryBytes;
    const tile_t* tl = &g.tiles[i];
    int64_t cursor = (int64_t)get_u64(e + 20);
    const int64_t tile_end = cursor + get_u32(e + 28);
    int64_t decoded = 0;
    while (decoded < tl->w * tl->h) {
      if (cursor + 3 > tile_end) GFAIL("truncated entropy shard header");
      const int64_t mode = bytes[cursor];
      const int64_t body_length = get_u16(bytes + cursor + 1);
      const int64_t body_offset = cursor + 3;
      if (mode > 19) GFAIL("unknown entropy shard mode");
      if (body_length > tile_end - body_offset) GFAIL("truncated entropy shard body");
      const int64_t n = min64(kShardSymbols, tl->w * tl->h - decoded);
      meta[shard].mode = mode;
      meta[shard].body_offset = body_offset;
      meta[shard].body_length = body_length;
      meta[shard].count = n;
      meta[shard].folded_base = tl->folded_base + decoded;
      ++shard;
      decoded += n;
      cursor = body_offset + body_length;
    }
    if (cursor != tile_end) GFAIL("trailing bounded-shard tile bytes");
  }
  const int32_t step = refined ? fvo_refined_gray16_step(quality) : fvo_quantization_step(layout, depth, quality);
  const int32_t max_sample = (1 << depth) - 1;
  uint32_t* folded = (uint32_t*)calloc((size_t)(g.nsamples ? g.nsamples : 1), sizeof(uint32_t));
  dec_ctx dc;
  dc.stream = bytes;
  dc.meta = meta;
  dc.max_folded = (uint32_t)(max_sample * 2);
  dc.folded = folded;
  dc.shard_status = (uint8_t*)calloc((size_t)(g.nshards ? g.nshards : 1), 1);
  parallel_for(threads, g.nshards, 8, decode_range, &dc);
  /* report the lowest failing shard, so the code does not depend on timing */
  int st = 0;
  for (int64_t s = 0; s < g.nshards && !st; ++s) st = dc.shard_status[s];
  free(dc.shard_status);
  if (st) {
    free(folded);
    GFAIL("malformed entropy payload (CUDA status %d)", st);
  }
  uint16_t* planes = (uint16_t*)malloc((size_t)(g.nsamples ? g.nsamples : 1) * sizeof(uint16_t));
  recon_ctx rc;
  rc.g = &g;
  rc.folded = folded;
  rc.step = step;
  rc.max_sample = max_sample;
  rc.use_med = gray_med || !gray;
  rc.out = planes;
  parallel_for(threads, g.ntiles, 4, recon_range, &rc);
  free(folded);
  free(meta);
  *out = planes;
  *out_samples = g.nsamples;
  *width_out = width;
  *height_out = height;
  *layout_out = layout;
  *depth_out = depth;
  geom_free(&g);
  return 0;
#undef GFAIL
}

void fvo_free(void* p) { free(p); }
