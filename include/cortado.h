/*
 * cortado.h -- C ABI of the B200 implementation of Cortado's encode/decode
 * path (a progressive, error-bounded float32 compressor).
 *
 * Each entry point replaces one host wrapper of the reference (cited below by
 * file:line within the reference project).  Differences from those wrappers:
 *   - work is enqueued on the caller's CUDA stream and nothing allocates or
 *     synchronizes on the hot path (the reference allocates and frees its
 *     carry array inside every call, include/d_server_encode.h:160-165);
 *   - errors are status codes: argument and error-bound problems are returned
 *     at once, problems the device detects (corrupt stream, size mismatch,
 *     a bounded wait that timed out) are latched in the context and returned
 *     by cortado_sync() -- the reference throws or calls __trap();
 *   - a context holds all scratch state; one context serves one stream at a
 *     time (use one context per concurrently used stream);
 *   - every device buffer must be 16-byte aligned (cudaMalloc's are) and
 *     every original size a multiple of 4 bytes.
 * Streams, .stor.meta files and decoded floats are byte-identical to the
 * reference's, except header bytes 12..15, which the reference leaves
 * unwritten and which are written as 0 here.
 *
 * Sizes are in bytes.  "d_" pointers are device pointers, "h_" host pointers.
 */
#ifndef CORTADO_H
#define CORTADO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* cortado_stream_t; /* same type as cudaStream_t */
typedef struct cortado_ctx cortado_ctx;

typedef enum {
  CORTADO_OK = 0,
  CORTADO_ERR_EB_TOO_SMALL = 1,   /* bound below FLT_MIN after the reference's adjustments */
  CORTADO_ERR_EB_TOO_LARGE = 2,   /* bound exponent + 24 reaches the float exponent limit */
  CORTADO_ERR_CORRUPT_STREAM = 3, /* malformed header, size table or chunk */
  CORTADO_ERR_SIZE_MISMATCH = 4,  /* stream size differs from the given original size */
  CORTADO_ERR_TIMEOUT = 5,        /* a bounded device wait gave up */
  CORTADO_ERR_OOM = 6,
  CORTADO_ERR_INVALID_ARG = 7,
  CORTADO_ERR_CUDA = 8,
  CORTADO_ERR_ALIGNMENT = 9,
  CORTADO_ERR_CAPACITY = 10,      /* output buffer smaller than required */
  CORTADO_ERR_SCRATCH_LIMIT = 11  /* input exceeds cortado_store_encode_noalloc's fixed scratch */
} cortado_status;

/* Chunk size of the format (reference include/consts.h:43). */
#define CORTADO_CHUNK_BYTES 16384

const char* cortado_status_string(cortado_status s);

/* Worst-case stream size for n_bytes of input: 16 + 2*chunks + 16384*chunks
 * (reference src/cortado_store.cu:196-198). */
int64_t cortado_max_stream_bytes(int64_t n_bytes);

/* Validates an absolute error bound and returns its biased float exponent,
 * the only part of a bound that reaches a stream
 * (reference include/d_server_encode.h:150-158). */
cortado_status cortado_eb_exponent(float eb_abs, int* biased_exponent);

/* Context: scratch (lookback words, chunk queue, status word) on `device`. */
cortado_status cortado_create(cortado_ctx** ctx, int device);
void cortado_destroy(cortado_ctx* ctx);
/* Upper bound of every device-side wait (default 2 s). */
cortado_status cortado_set_timeout(cortado_ctx* ctx, uint64_t timeout_ns);
/* Waits for `stream`, then returns (and clears) the first error the device
 * latched since the previous call. */
cortado_status cortado_sync(cortado_ctx* ctx, cortado_stream_t stream);

/* store: encodes n_bytes of float32 at the absolute bound eb_abs (stored bins
 * use eb_abs/2).  Replaces d_server_encode, include/d_server_encode.h:146-166.
 * out_capacity >= cortado_max_stream_bytes(n_bytes); *d_outsize receives the
 * stream length. */
cortado_status cortado_store_encode(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float eb_abs,
                                    void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                    cortado_stream_t stream);

/* storage decode: stored stream -> floats.  Replaces d_server_decode,
 * include/d_server_encode.h:263-267.  stream_bytes bounds the reads;
 * *d_outsize receives the decoded length (from the stream header). */
cortado_status cortado_store_decode(cortado_ctx* ctx, const void* d_stream, int64_t stream_bytes, void* d_out,
                                    int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream);

/* init_send: requantizes a stored stream to request_eb_abs and encodes it.
 * Replaces d_s2c_encode, include/d_s2c.h:203-224.  n_bytes is the original
 * size (the stored stream's header value; the reference passes the chunk
 * count). */
cortado_status cortado_init_send(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                 float request_eb_abs, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                 cortado_stream_t stream);

/* init_recv: decodes an init stream to floats.  Replaces d_client_decode,
 * include/d_client_encode.h:262-266.  Chunks the encoder stored uncompressed
 * are copied out as stored, as the reference does. */
cortado_status cortado_init_recv(cortado_ctx* ctx, const void* d_init, int64_t init_bytes, void* d_out,
                                 int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream);

/* resi_send: residual between the client's current bound src_eb_abs and the
 * finer dst_eb_abs, from a stored stream.  Replaces d_residual_encode,
 * include/d_residual_encode.h:204-230. */
cortado_status cortado_resi_send(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                 float src_eb_abs, float dst_eb_abs, void* d_out, int64_t out_capacity,
                                 int64_t* d_outsize, cortado_stream_t stream);

/* resi_recv: applies a residual stream to the client's current floats.
 * Replaces d_residual_apply, include/d_residual_encode.h:350-354 (the size
 * check of :257 becomes CORTADO_ERR_SIZE_MISMATCH). */
cortado_status cortado_resi_recv(cortado_ctx* ctx, const void* d_src, int64_t n_bytes, const void* d_resi,
                                 int64_t resi_bytes, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                 cortado_stream_t stream);

/* init_send fused with the client's init_recv, for a server that holds the
 * client's reconstruction on the same device (a serving loop).  Writes the
 * init stream exactly as cortado_init_send() does and, in the same pass,
 * d_client (n_bytes of floats) exactly as cortado_init_recv() of that stream
 * would, without decoding it again.  No single counterpart in the reference:
 * it replaces d_s2c_encode (include/d_s2c.h:203-224) followed by
 * d_client_decode (include/d_client_encode.h:262-266). */
cortado_status cortado_init_send_apply(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                       float request_eb_abs, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                       void* d_client, cortado_stream_t stream);

/* resi_send fused with the client's resi_recv: writes the residual stream as
 * cortado_resi_send() does and updates d_client (the client's floats at the
 * source bound, n_bytes) in place to what cortado_resi_recv() of that stream
 * would produce.  Replaces d_residual_encode (include/d_residual_encode.h:204-230)
 * followed by d_residual_apply (include/d_residual_encode.h:350-354). */
cortado_status cortado_resi_send_apply(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                       float src_eb_abs, float dst_eb_abs, void* d_out, int64_t out_capacity,
                                       int64_t* d_outsize, void* d_client, cortado_stream_t stream);

/* NOA range: min and max of the floats (NaNs ignored), synchronous.
 * Replaces d_INOA_find_range, include/preprocessors/include/INOA_f32.h:52-61. */
cortado_status cortado_noa_range(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float* h_min, float* h_max,
                                 cortado_stream_t stream);

/* ---- NOA bounds on the device: nothing waits for the host ----
 * The reference's drivers scale a normalized (NOA) bound on the host,
 * eb_abs = (max - min) * eb, after copying the range to the host
 * (src/cortado_store.cu:206-227, include/preprocessors/include/INOA_f32.h:52-61),
 * so every NOA operation waits for the device.  These entry points keep the
 * range in device memory and scale the bounds in the kernels with the same
 * float arithmetic (one rounding for the difference, one for the product,
 * the store's bins at eb_abs / 2): streams are byte-identical to the
 * host-scaled calls with storage.noa_scale's bounds.  A whole NOA flow can
 * then be enqueued without waiting, or captured in a CUDA graph.  Bound
 * errors (EB_TOO_SMALL, EB_TOO_LARGE) are latched in the context and
 * returned by cortado_sync(); such a call writes nothing. */
/* Range of n_bytes of floats into d_minmax[0] (min) and d_minmax[1] (max),
 * device floats, NaNs ignored; asynchronous. */
cortado_status cortado_noa_range_device(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float* d_minmax,
                                        cortado_stream_t stream);
/* store at the NOA bound eb_noa of the range in d_minmax. */
cortado_status cortado_store_encode_noa(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, const float* d_minmax,
                                        float eb_noa, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                        cortado_stream_t stream);
/* init_send at the NOA request bound request_eb_noa. */
cortado_status cortado_init_send_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                     const float* d_minmax, float request_eb_noa, void* d_out, int64_t out_capacity,
                                     int64_t* d_outsize, cortado_stream_t stream);
/* resi_send between the NOA bounds src_eb_noa and dst_eb_noa. */
cortado_status cortado_resi_send_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                     const float* d_minmax, float src_eb_noa, float dst_eb_noa, void* d_out,
                                     int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream);

/* init_send / resi_send fused with the client's receive (as
 * cortado_init_send_apply / cortado_resi_send_apply) at NOA bounds of the
 * range in d_minmax: the stream and the client's reconstruction are
 * byte-identical to the host-scaled fused calls; on a latched bound error
 * neither is written. */
cortado_status cortado_init_send_apply_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                           const float* d_minmax, float request_eb_noa, void* d_out,
                                           int64_t out_capacity, int64_t* d_outsize, void* d_client,
                                           cortado_stream_t stream);
cortado_status cortado_resi_send_apply_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                           const float* d_minmax, float src_eb_noa, float dst_eb_noa, void* d_out,
                                           int64_t out_capacity, int64_t* d_outsize, void* d_client,
                                           cortado_stream_t stream);

/* Bound verifier: writes to *d_first_bad (device) the first index i at which
 * recon[i] violates |orig[i] - recon[i]| <= eb_abs under the reference's
 * MAXABS_f32 rules (include/verifiers/MAXABS_f32.h:40-72; NaN and Inf must
 * match), or UINT64_MAX if every value is within the bound.  Asynchronous,
 * so it can follow each step of a captured chain. */
cortado_status cortado_verify_bound(cortado_ctx* ctx, const void* d_orig, const void* d_recon, int64_t n_bytes,
                                    float eb_abs, unsigned long long* d_first_bad, cortado_stream_t stream);

/* ---- batched form: many streams in one persistent launch ----
 * No single counterpart in the reference (it launches one kernel per field
 * and bound).  All items of one call run the same operation; their chunks
 * form one work queue, so uneven sizes share the GPU without per-launch
 * tails, and each item gets its own header, size table and offsets (a
 * per-item lookback).  Every item needs its original size n_bytes (> 0). */
typedef enum {
  CORTADO_OP_STORE = 0,        /* d_in: floats (in_bytes == n_bytes), eb1: bound */
  CORTADO_OP_INIT_SEND = 1,    /* d_in: stored stream, eb1: request bound */
  CORTADO_OP_RESI_SEND = 2,    /* d_in: stored stream, eb1: source, eb2: destination bound */
  CORTADO_OP_STORE_DECODE = 3, /* d_in: stored stream */
  CORTADO_OP_INIT_RECV = 4,    /* d_in: init stream */
  CORTADO_OP_RESI_RECV = 5,    /* d_in: residual stream, d_src: the client's floats */
  CORTADO_OP_INIT_SEND_APPLY = 6, /* as INIT_SEND, and d_src: the client's floats, written (init_send_apply) */
  CORTADO_OP_RESI_SEND_APPLY = 7  /* as RESI_SEND, and d_src: the client's floats, updated (resi_send_apply) */
} cortado_op;

typedef struct {
  const void* d_in;
  int64_t in_bytes;
  int64_t n_bytes;
  float eb1, eb2;
  const void* d_src;
  void* d_out;
  int64_t out_capacity;
  int64_t* d_outsize;
} cortado_item;

/* Runs `op` on n_items items in one launch (replaces n_items calls of the
 * corresponding entry point above, e.g. d_server_encode at 4 bounds for each
 * of 64 fields).  Device-side errors are latched as for single calls. */
cortado_status cortado_batch(cortado_ctx* ctx, cortado_op op, const cortado_item* items, int n_items,
                             cortado_stream_t stream);

/* Failure-detection self-test: launches one thread that waits, through the
 * same bounded wait the decoders use for payload offsets, on a word that no
 * launch can publish.  After the context's timeout (cortado_set_timeout) the
 * wait gives up and latches CORTADO_ERR_TIMEOUT, which the next
 * cortado_sync() returns (and clears); the context stays usable.  No
 * counterpart in the reference (its waits are unbounded). */
cortado_status cortado_selftest_timeout(cortado_ctx* ctx, cortado_stream_t stream);

/* Sizes the context's scratch ahead of use: lookback and payload-offset words
 * for `chunks` chunks in one call (a batched call counts the chunks of all its
 * items), and batch item tables of `items` entries.  Calls that find their
 * scratch too small grow it themselves, but growing frees and allocates
 * device memory, which waits for the device.  A serving loop reserves its
 * largest batch once at start-up instead.  No counterpart in the reference
 * (its wrappers allocate per call).  Returns once the scratch is ready. */
cortado_status cortado_reserve(cortado_ctx* ctx, int64_t chunks, int items);

/* Launch shape of `op` on this context: the persistent grid holds
 * ctas_per_sm CTAs per SM (capped by the kernel's occupancy limit); 0 restores
 * the occupancy limit.  Chosen by the autotuner (cortado_b200/autotune.py);
 * it changes speed only, never output bytes. */
cortado_status cortado_set_launch_ctas(cortado_ctx* ctx, cortado_op op, int ctas_per_sm);

/* Whether launches of `op` on this context give a warp of their helper CTA
 * to resolving lookback prefixes ahead of the flushes (encoders; default 1).
 * With 0, each chunk's flush walks the lookback words itself.  Chosen by the
 * autotuner (cortado_b200/autotune.py); it changes speed only, never output
 * bytes.  No counterpart in the reference (its lookback is a per-chunk spin,
 * include/d_compression.h:120-160). */
cortado_status cortado_set_resolver(cortado_ctx* ctx, cortado_op op, int enabled);

/* store without allocating: for callers that cannot call cudaMalloc.
 *
 * No counterpart in the reference.  Some callers of this library cannot
 * allocate device memory when they encode: code running under a host
 * framework that owns the whole device memory pool (a caching allocator or a
 * serving process that reserved its memory up front), or code on a real-time
 * path where an allocation's implicit synchronization is not allowed.  The
 * context-based cortado_store_encode() allocates its scratch at creation and
 * grows it for larger inputs; this entry point instead uses a fixed scratch
 * array compiled into the library (CORTADO_NOALLOC_MAX_BYTES / 16384 lookback
 * words plus three counters, 512 KiB), which every GPU that loads the library
 * holds until the process exits.  It calls no cudaMalloc, cudaFree or
 * allocating library routine.  Inputs and outputs are as for
 * cortado_store_encode(), on the device current at the call.
 *   - inputs larger than CORTADO_NOALLOC_MAX_BYTES return
 *     CORTADO_ERR_SCRATCH_LIMIT;
 *   - the first call on a device looks up the scratch array's device address
 *     (cudaGetSymbolAddress) and the launch size; make that first call before
 *     any stream capture;
 *   - all calls share the one array, so calls that overlap on the GPU (other
 *     streams, other host threads) race and give wrong output: serialize them;
 *   - the set-up is repeated when the calling thread's CUDA context changes
 *     (for example after cudaDeviceReset);
 *   - every device-side wait gives up after a fixed 2 s;
 *   - there is no context to latch device-side errors in: a failed launch
 *     writes a negative status (-CORTADO_ERR_TIMEOUT) to *d_outsize. */
#define CORTADO_NOALLOC_MAX_BYTES (1LL << 30)
cortado_status cortado_store_encode_noalloc(const void* d_in, int64_t n_bytes, float eb_abs, void* d_out,
                                            int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CORTADO_H */
