/*
 * fastvid_b200.h -- C ABI of the B200 (sm_100a) fastvid intra codec.
 *
 * Plain C types only: device pointers, sizes, an opaque CUDA stream handle
 * (a cudaStream_t passed as void*), and int status codes.  The caller owns
 * every buffer (workspace, inputs, outputs); the library allocates no device
 * memory.  Work runs on the device that owns the workspace; every entry point
 * returns with the caller's current device unchanged.  Streams are
 * byte-identical to the reference encoder (generative-workflows/fastvid
 * cuda/csrc/encode.cu) and decodes are bit-exact.
 *
 * Status codes: 0 is success.  Positive codes are the reference's device
 * status codes, unchanged: encoder 1 = a sample above 2^bit_depth-1,
 * 2 = a shard body above 65535 bytes; decoder 1 zero-run, 2 Rice, 3 block pack,
 * 4 unknown mode, 5 rANS, 10 tile directory, 11 shard header.  Negative codes
 * are host-side rejections (below).  fvb_last_error() returns the message of
 * the calling thread's last failure; the messages of argument and header
 * checks are the reference's own (cuda/csrc/encode.cu:695-735,
 * cuda/csrc/fastvid_cuda.cpp:142-183).
 */
#ifndef FASTVID_B200_H
#define FASTVID_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVB_ABI_VERSION 2

enum {
  FVB_OK = 0,
  FVB_ERR_ARGUMENT = -1,  /* invalid argument */
  FVB_ERR_FORMAT = -2,    /* stream header rejected on the host */
  FVB_ERR_WORKSPACE = -3, /* workspace or output smaller than required */
  FVB_ERR_CUDA = -4,      /* CUDA runtime failure */
  FVB_ERR_INTERNAL = -5   /* consistency check of this library failed */
};

/* One frame's parameters and derived geometry.  Filled by fvb_encode_plan or
 * fvb_decode_plan; the caller treats it as read-only. */
typedef struct fvb_frame {
  int32_t layout;     /* 0 gray, 1 yuv422, 2 rgb444 */
  int32_t bit_depth;  /* 8, 10, 12, 16 */
  int32_t quality;    /* 1..100 */
  int32_t flags;      /* decode: header byte 7 high bits (0x40 gray MED, 0x80 refined gray16) */
  int64_t width, height, tile_w, tile_h;
  int64_t fps_num, fps_den;
  int64_t tiles, shards, samples; /* geometry (reference encode.cu:41-69) */
  int64_t plane_width[3];
  int32_t planes;
  int32_t step;       /* quantizer step before the frame policy (encode) / of the stream (decode) */
  int64_t prefix_bytes;     /* 32 + 32 * tiles */
  int64_t max_stream_bytes; /* upper bound of the encoded size */
} fvb_frame;

int fvb_abi_version(void);
const char* fvb_last_error(void);

/* ---- instrumentation (no reference counterpart; the reference profiles
 * with torch.profiler around whole calls, cuda/benchmarks/profile_*.py) ---- */

/* Number of kernel launches this library has issued in the process. */
int64_t fvb_launch_count(void);
/* Kernel identifiers 0..fvb_kernel_count()-1 and their names. */
int fvb_kernel_count(void);
const char* fvb_kernel_name(int kernel);

/* Launch geometry of a persistent kernel (no counterpart in the reference;
 * the knob the autotuner sets): its grid is capped at `ctas_per_sm` CTAs per
 * SM, 0 restoring the built-in default.  Process-wide, read at each launch;
 * no output depends on it.  FVB_ERR_ARGUMENT for a kernel without the knob
 * or a value outside 0..64. */
int fvb_set_launch_ctas(int kernel, int ctas_per_sm);
/* The cap in effect, or -1 for a kernel without the knob. */
int fvb_get_launch_ctas(int kernel);
/* Wavefront block of the predictor and reconstruction kernels (no
 * counterpart in the reference, whose predictor walks antidiagonals with a
 * barrier per step, cuda/csrc/encode.cu:150-192): each warp sweeps 32-row
 * bands in blocks of 32 steps, `steps` (4, 8, 16 or 32) of them unrolled;
 * 0 restores the default (8).  Process-wide, read at each launch; no output
 * depends on it (the autotuner's knob). */
int fvb_set_wavefront_block(int steps);
int fvb_get_wavefront_block(void);
/* Warps per tile of the predictor and reconstruction kernels (no reference
 * counterpart; the autotuner's knob): 1, or 2 -- a warp pair sweeps a tile's
 * even and odd 32-row bands in lock-step, the second warp two blocks behind,
 * handing each band's last row over in shared memory (tiles of one band or
 * under 66 columns stay on one warp).  0 restores the default (1).
 * Process-wide, read at each launch; no output depends on it. */
int fvb_set_tile_warps(int warps);
int fvb_get_tile_warps(void);
/* Whether decode batches of 64 shards or more run dec_other (Rice,
 * zero-run and block-pack shards) on a side stream beside dec_rans (1, the
 * default) or after it on the caller's stream (0).  No reference
 * counterpart; process-wide, read at each launch; no output depends on it
 * (the autotuner's knob). */
int fvb_set_decode_overlap(int on);
int fvb_get_decode_overlap(void);
/* How the rANS encoder fetches ahead of its state chain (no reference
 * counterpart, whose lanes load as they go, cuda/csrc/encode.cu:398-418): 0
 * loads 16 symbols and then their table entries before each 16 steps; 8 or
 * 16 runs a software pipeline over blocks of that many steps, the symbols
 * two blocks and the table entries one block ahead; -1 (the default) picks
 * per launch: the 8-step pipeline when the launch has at most 4 CTAs per SM
 * (a single frame: its lanes' load latency is exposed), the one-stage fetch
 * otherwise (it holds fewer registers).  Process-wide, read at each launch;
 * no output depends on it (the autotuner's knob). */
int fvb_set_rans_pipeline(int steps);
int fvb_get_rans_pipeline(void);
/* The same choice for the encoder passes after the first, which re-encode
 * only the frames the frame policy retries (gray10 MED, gray16 step
 * refinement): few shards, so the pass is one lane's chain of dependent
 * steps long whatever the load, and fetching further ahead pays. */
int fvb_set_rans_pipeline_tail(int steps);
int fvb_get_rans_pipeline_tail(void);
/* While profiling is on (per calling thread), every launch is bracketed by
 * CUDA events on its stream; fvb_profile_end waits for them and writes, per
 * kernel id, the summed milliseconds and the number of launches. */
int fvb_profile_begin(void);
int fvb_profile_end(double* ms, int64_t* launches, int n);

/* ---- single frame (the drop-in path) -------------------------------------
 *
 * Encode = fvb_encode_plan + fvb_encode_analyze + fvb_encode_emit, which
 * together replace fastvid_encode_cuda (reference cuda/csrc/encode.cu:686-931,
 * bound as _C.encode at cuda/csrc/fastvid_cuda.cpp:366-377).
 */

/* Validates the arguments exactly as encode.cu:695-716 does and computes the
 * geometry and the workspace size (bytes, device memory). */
int fvb_encode_plan(int64_t width, int64_t height, int layout, int bit_depth, int quality,
                    int64_t fps_num, int64_t fps_den, int64_t tile_w, int64_t tile_h,
                    fvb_frame* frame, int64_t* workspace_bytes);

/* Predicts, analyses and lays out the stream on `cuda_stream` (the frame
 * policy of encode.cu:812-847 runs on the device), then waits for the one
 * 96-byte result read and returns the exact stream length.  planes[p] are
 * device pointers to uint16 planes with row pitch pitches[p] (elements);
 * host pointers return FVB_ERR_ARGUMENT before anything is launched.
 * Replaces encode.cu:727-870. */
int fvb_encode_analyze(const fvb_frame* frame, const uint16_t* const* planes, const int64_t* pitches,
                       void* workspace, int64_t workspace_bytes, void* cuda_stream, int64_t* stream_len);

/* Writes the stream (header, directory, shard records) into device buffer
 * `out` of out_len >= stream_len bytes; asynchronous on `cuda_stream`.
 * Replaces encode.cu:871-931. */
int fvb_encode_emit(const fvb_frame* frame, void* workspace, int64_t workspace_bytes, uint8_t* out,
                    int64_t out_len, void* cuda_stream);

/* Validates the 32-byte header (host memory) against the stream length,
 * exactly as fastvid_cuda.cpp:142-183, and computes geometry and workspace.
 * Replaces the host half of the binding's decode (fastvid_cuda.cpp:141-236). */
int fvb_decode_plan(const uint8_t* header, int64_t header_len, int64_t stream_len, fvb_frame* frame,
                    int64_t* workspace_bytes);

/* Decodes a device-resident stream into device planes (planes[p] with row
 * pitch pitches[p] elements), wavefront (1) or serial (0) reconstruction;
 * waits for the status word.  Replaces fastvid_decode_cuda
 * (cuda/csrc/decode.cu:660-730) including the device metadata parse.
 * The stream and the planes must be device (or managed) memory: a host
 * pointer returns FVB_ERR_ARGUMENT before anything is launched. */
int fvb_decode(const fvb_frame* frame, const uint8_t* stream, int64_t stream_len, uint16_t* const* planes,
               const int64_t* pitches, int wavefront, void* workspace, int64_t workspace_bytes,
               void* cuda_stream);

/* ---- batches (no reference counterpart: the reference batches with a Python
 * loop over the single-frame path, fastvid/__init__.py:44-53,63) ------------
 *
 * All frames share one launch of each kernel; per-frame bytes are identical
 * to the single-frame path. */

int fvb_batch_encode_plan(const fvb_frame* frames, int n, int64_t* workspace_bytes);

/* Uploads the frame table (planes: 3 pointers per frame, pitches likewise). */
int fvb_batch_encode_prepare(const fvb_frame* frames, int n, const uint16_t* const* planes,
                             const int64_t* pitches, void* workspace, int64_t workspace_bytes,
                             void* cuda_stream);

/* Enqueues every analysis pass; no host synchronisation, so it can be
 * captured into a CUDA graph.  Writes n result records (status, stream
 * length) into `results` (host memory, 2 int64 per frame).  Page-locked
 * `results` (cudaMallocHost / cudaHostAlloc) is written by a kernel
 * directly; other host memory gets a device-to-host copy, which queues
 * behind any larger download in flight on another stream. */
int fvb_batch_encode_enqueue(const fvb_frame* frames, int n, void* workspace, int64_t workspace_bytes,
                             int64_t* results, void* cuda_stream);

/* After the results are visible: writes frame i's stream at outs[i]
 * (host array of device pointers, one per frame; uploaded from pageable
 * memory, so this call is not capturable).  Asynchronous. */
int fvb_batch_encode_emit(const fvb_frame* frames, int n, void* workspace, int64_t workspace_bytes,
                          uint8_t* const* outs, void* cuda_stream);

/* Copies the 32-byte header of each device stream into host `headers`
 * (32 * n bytes) with one gather kernel (which writes page-locked
 * `headers` directly, other memory through one copy), and waits for it.
 * `scratch` is device memory of at least 16*n rounded up to 256, plus 32*n
 * bytes. */
int fvb_gather_headers(const uint8_t* const* streams, const int64_t* stream_lens, int n, void* scratch,
                       int64_t scratch_bytes, uint8_t* headers, void* cuda_stream);

int fvb_batch_decode_plan(const fvb_frame* frames, int n, int64_t* workspace_bytes);

/* streams[i]/stream_lens[i]: device streams; planes: 3 device pointers per
 * frame, pitches likewise.  Uploads the frame table. */
int fvb_batch_decode_prepare(const fvb_frame* frames, int n, const uint8_t* const* streams,
                             const int64_t* stream_lens, uint16_t* const* planes, const int64_t* pitches,
                             void* workspace, int64_t workspace_bytes, void* cuda_stream);

/* Enqueues parse, entropy decode and reconstruction for every frame (graph
 * capturable) and writes one record per frame (status, 0) into `results`,
 * as fvb_batch_encode_enqueue does. */
int fvb_batch_decode_enqueue(const fvb_frame* frames, int n, int wavefront, void* workspace,
                             int64_t workspace_bytes, int64_t* results, void* cuda_stream);

/* ---- shape buckets (no reference counterpart) -----------------------------
 *
 * A bucket is a capacity: frames, tiles, shards, samples and header bytes of a
 * batch (in total and per encoder pass), each rounded up to m * 2^e with m in
 * 4..8 (at most 25 percent above the batch's), plus the exact pass count and
 * wide-tile flag.  Workspace layout and launch grids follow the capacity and
 * the kernels read the batch's actual counts from the workspace, so one
 * enqueue -- and one CUDA graph captured from it -- serves every batch that
 * fits the bucket, whatever its mix of frames.  The fvb_batch_* calls above
 * are the same sequence with the batch's own totals as the capacity. */
typedef struct fvb_bucket {
  int64_t frames, tiles, shards, samples, prefix;
  int64_t frames_p[3], tiles_p[3], shards_p[3]; /* per encoder pass */
  int64_t samples_p[3], prefix_p[3];            /* per encoder pass */
  int32_t passes, wide;
  int32_t fold16, pad; /* 1: folded symbols held as u16 (every frame below depth 16 or quality 100) */
} fvb_bucket;

/* The bucket of a batch. */
int fvb_batch_bucket(const fvb_frame* frames, int n, fvb_bucket* bucket);
int fvb_bucket_encode_plan(const fvb_bucket* bucket, int64_t* workspace_bytes);
int fvb_bucket_decode_plan(const fvb_bucket* bucket, int64_t* workspace_bytes);
/* As the fvb_batch_* calls; the batch must fit the bucket (FVB_ERR_ARGUMENT
 * otherwise).  Enqueue needs no frame list: everything it launches is sized
 * by the bucket and reads the batch from the workspace.  `results` receives
 * bucket->frames records (the batch's first). */
int fvb_bucket_encode_prepare(const fvb_bucket* bucket, const fvb_frame* frames, int n,
                              const uint16_t* const* planes, const int64_t* pitches, void* workspace,
                              int64_t workspace_bytes, void* cuda_stream);
int fvb_bucket_encode_enqueue(const fvb_bucket* bucket, void* workspace, int64_t workspace_bytes, int64_t* results,
                              void* cuda_stream);
/* After fvb_bucket_encode_enqueue, on the same stream: writes the 32-byte
 * header of every frame (32 * n bytes, the caller's order) into page-locked
 * host memory `headers` by a kernel, so a caller that decodes the streams
 * next has them with the results -- no read of the streams' first bytes,
 * no extra wait.  Graph capturable. */
int fvb_bucket_encode_headers(const fvb_bucket* bucket, void* workspace, int64_t workspace_bytes, uint8_t* headers,
                              void* cuda_stream);
int fvb_bucket_encode_emit(const fvb_bucket* bucket, const fvb_frame* frames, int n, void* workspace,
                           int64_t workspace_bytes, uint8_t* const* outs, void* cuda_stream);
int fvb_bucket_decode_prepare(const fvb_bucket* bucket, const fvb_frame* frames, int n,
                              const uint8_t* const* streams, const int64_t* stream_lens, uint16_t* const* planes,
                              const int64_t* pitches, void* workspace, int64_t workspace_bytes, void* cuda_stream);
int fvb_bucket_decode_enqueue(const fvb_bucket* bucket, int wavefront, void* workspace, int64_t workspace_bytes,
                              int64_t* results, void* cuda_stream);

/* ---- allocation-free decode (no reference counterpart) --------------------
 *
 * For callers that cannot allocate device memory at decode time -- plug-ins
 * handed pre-allocated frames by a host application that owns the device
 * heap, real-time pipelines that forbid allocation after start-up (cudaMalloc
 * and cudaFree can block and synchronise the device), components held to a
 * device-memory budget enforced elsewhere.  Same contract as fvb_decode, but
 * the scratch is a fixed 32 MiB array inside the library
 * (fvb_decode_noalloc_capacity() bytes, frames up to about 13 million samples,
 * 7 million for lossless 16-bit frames; larger frames return FVB_ERR_WORKSPACE), so no workspace is passed and
 * nothing is allocated: no device memory, no streams, no events (dec_other
 * runs on the caller's stream).  Every GPU that loads the library holds the
 * array until the process exits.  The first call on a device does the
 * set-up: it looks up the array's device address (cudaGetSymbolAddress) and
 * sets the kernels' shared-memory limits.  The call is synchronous -- it
 * waits for its result before returning -- so it cannot be captured into a
 * CUDA graph: never call it on a stream that is being captured.  The stream
 * and the planes must be device (or managed) memory.  All calls share the
 * one array, which keeps the last call's contents (every decode rewrites
 * what it reads): calls whose work overlaps on the GPU (other threads, other
 * streams) race and must be serialised by the caller. */
int64_t fvb_decode_noalloc_capacity(void);
int fvb_decode_noalloc(const fvb_frame* frame, const uint8_t* stream, int64_t stream_len, uint16_t* const* planes,
                       const int64_t* pitches, int wavefront, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* FASTVID_B200_H */
