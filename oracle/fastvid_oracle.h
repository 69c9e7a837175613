/*
 * fastvid_oracle.h -- CPU restatement of the fastvid intra codec.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the CUDA path in
 * fastvid_b200: tests, the smoke check and the CPU-baseline leg of bench.py
 * call it as the checker.  The product path never links or calls it.
 *
 * Every function restates the reference algorithm in plain C; the comments in
 * fastvid_oracle.c cite the reference file:line each step follows
 * (cuda/csrc/encode.cu, cuda/csrc/decode.cu, cuda/csrc/fastvid_cuda.cpp).
 */
#ifndef FASTVID_ORACLE_H
#define FASTVID_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Quality -> quantizer step (encode.cu:71-89). */
int32_t fvo_quantization_step(int layout, int bit_depth, int quality);
int32_t fvo_refined_gray16_step(int quality);

/* Encode one frame.  `samples` holds the planes back to back (Y then Cb then
 * Cr), each plane row-major and contiguous, plane widths as the layout
 * dictates.  On success *out is a malloc'd stream of *out_len bytes (free with
 * fvo_free) and 0 is returned; otherwise a nonzero code and a message. */
int fvo_encode(const uint16_t* samples, int64_t width, int64_t height, int layout,
               int bit_depth, int quality, int64_t fps_num, int64_t fps_den,
               int64_t tile_w, int64_t tile_h, int threads, uint8_t** out,
               int64_t* out_len, char* msg, int msg_len);

/* Decode one stream.  On success *out is a malloc'd buffer of
 * *out_samples uint16 values (planes back to back) and the frame description
 * is returned through the pointers.  `wavefront` selects nothing on the CPU
 * (both reference reconstruction orders give the same values) but is kept so
 * the call mirrors the reference binding. */
int fvo_decode(const uint8_t* stream, int64_t len, int wavefront, int threads,
               uint16_t** out, int64_t* out_samples, int64_t* width, int64_t* height,
               int* layout, int* bit_depth, char* msg, int msg_len);

/* Stage-level entry points used by the kernel parity tests.
 * fvo_predict: predictor + quantizer + reconstruction + zigzag over every
 *   tile (encode.cu:128-193); writes folded[total] in tile-raster order and
 *   the reconstructed planes recon[total] in plane layout.
 * fvo_analyze: the per-shard mode competition and rANS override
 *   (encode.cu:195-431, order as in encode.cu:789-805); writes
 *   analysis[shards*8] = mode, parameter, body, record, lane_bytes[4]. */
int fvo_predict(const uint16_t* samples, int64_t width, int64_t height, int layout,
                int bit_depth, int64_t tile_w, int64_t tile_h, int32_t step, int use_med,
                uint32_t* folded, uint16_t* recon);
int fvo_analyze(const uint32_t* folded, int64_t width, int64_t height, int layout,
                int64_t tile_w, int64_t tile_h, int force_order0, int64_t* analysis);

/* Frame geometry: number of tiles, shards and samples. */
int fvo_geometry(int64_t width, int64_t height, int layout, int64_t tile_w, int64_t tile_h,
                 int64_t* tiles, int64_t* shards, int64_t* samples);

void fvo_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
