// libcortado: the C-ABI drop-in for the reference's encode/decode path.
// Declarations and the reference entry point each function replaces are in
// include/cortado.h.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <float.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/cortado.h"
#include "kernels.cuh"

using namespace cortado;

// ================================================================== kernels
// Resident CTAs per SM each kernel is compiled for (register budget
// 65536 / (128 * n)); every kernel holds two 17 KiB buffers, so shared memory
// allows 6.  resi_recv runs 5 (a budget of 102 registers; it uses 96): at 80
// its client and residual words spill, and it measured 4.6% faster at 5;
// every other kernel measured slower at 5 (and the store 10% slower with a
// third buffer at 4).
#ifndef MINB_STORE
#define MINB_STORE 6
#endif
#ifndef MINB_REENC
#define MINB_REENC 6
#endif
#ifndef MINB_DEC
#define MINB_DEC 6
#endif
#ifndef MINB_RAPPLY
#define MINB_RAPPLY 5
#endif

namespace {

__device__ __forceinline__ Ctl& ctl_block() {
  extern __shared__ uint8_t smem_raw[];
  return *reinterpret_cast<Ctl*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
}

// The thread that issues every TMA load and store of a CTA (warp 3, lane 0):
// bulk-store completion is tracked per thread, so the thread that reuses a
// buffer after a TMA store must be the one that issued the store.
constexpr int TMA_TID = 96;

// Reads this launch's lookback epoch and sets up the stage barriers (every
// CTA, at start; the caller synchronizes).  A stage's barrier completes a
// phase per use: two arrivals by the prefetching lane (one before its loads
// are issued, one after the stage's metadata and hand-copied bytes are
// written) plus the TMA bytes, so waiting on it also publishes the metadata.
__device__ __forceinline__ void begin_launch(Ctl& sm, const Sync& sy) {
  if (threadIdx.x == 0) sm.epoch = *(volatile unsigned int*)sy.epoch;
  if (threadIdx.x == TMA_TID) {
    mbar_init(&sm.bar[0], 2);
    mbar_init(&sm.bar[1], 2);
    mbar_init(&sm.bar_src, 1);
    fence_mbar_init();
  }
}

// The last CTA out resets the chunk queue and advances the epoch for the next
// launch on this scratch; when the 16-bit epoch wraps it first clears the
// lookback words, so no word of an old launch can carry the new epoch.
// Returns the status word's value to the last CTA's thread 0 (else 0).
__device__ __forceinline__ unsigned int finish_launch(Ctl& sm, const Sync& sy, bool take_status = false) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    sm.is_last = atomicAdd(&sy.counter[1], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  unsigned int st = 0;
  if (sm.is_last) {
    const unsigned int e = sm.epoch;
    if (e == 65535u)
      for (long long i = threadIdx.x; i < sy.flags_cap; i += blockDim.x) {
        sy.flags[i] = 0;
        if (sy.offs) sy.offs[i] = 0;
      }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (take_status) st = atomicExch(sy.status, 0u);
      *sy.epoch = (e == 65535u) ? 0u : e + 1u;
      sy.counter[0] = 0;
      sy.counter[1] = 0;
      sy.counter[6] = 0;
      __threadfence();
    }
  }
  return st;
}

// Loads the float words of a chunk into a swizzled buffer (zero past nw).
__device__ __forceinline__ void load_plain_rows(uint32_t* buf, const uint8_t* src, long long c, int nw) {
  const uint32_t* g = reinterpret_cast<const uint32_t*>(src) + c * (long long)CW;
  for (int w = threadIdx.x; w < CW; w += NT) buf[swz(w)] = (w < nw) ? g[w] : 0u;
}

struct StreamHdr {
  long long n, chunks;
  int eb_e;
  bool ok;
};

__device__ __forceinline__ StreamHdr read_header(const uint8_t* s, long long bytes) {
  StreamHdr h;
  h.ok = bytes >= HDR;
  h.n = h.ok ? *reinterpret_cast<const long long*>(s) : 0;
  h.eb_e = h.ok ? *reinterpret_cast<const int*>(s + 8) : 1;
  h.ok = h.ok && h.n >= 0 && (h.n & 3) == 0 && h.eb_e >= 1 && h.eb_e <= 230;
  h.chunks = h.ok ? (h.n + CS - 1) / CS : 0;
  h.ok = h.ok && (HDR + 2 * h.chunks <= bytes);
  if (!h.ok) h.chunks = 0;
  return h;
}

// Writes a stream header (int64 N, int32 exponent, int32 0).
__device__ __forceinline__ void write_header(uint8_t* out, long long n, int eb_e) {
  *reinterpret_cast<long long*>(out) = n;
  reinterpret_cast<int*>(out)[2] = eb_e;
  reinterpret_cast<int*>(out)[3] = 0;
}

// ---- work sources: what a queue index means.
// One stream: the queue index is the chunk; arguments and tensor maps are the
// kernel's own parameters; a decoder's header was checked at kernel start.
struct SingleSrc {
  static constexpr bool batched = false;
  const OpArgs* a;
  const CUtensorMap* map_in;
  const CUtensorMap* map_out;
  long long total;
  StreamHdr h;
  Quant q1, q2;  // the bounds' quantizers (resolved on the device for NOA entry points)
  __device__ __forceinline__ void quant(int, Quant& x1, Quant& x2) const {
    x1 = q1;
    x2 = q2;
  }
  __device__ __forceinline__ int locate(long long g, int, long long& c) const {
    c = g;
    return 0;
  }
  __device__ __forceinline__ const OpArgs& args(int) const { return *a; }
  __device__ __forceinline__ const CUtensorMap* min(int) const { return map_in; }
  __device__ __forceinline__ const CUtensorMap* mout(int) const { return map_out; }
  __device__ __forceinline__ StreamHdr header(int) const { return h; }
  __device__ __forceinline__ int header_bad(int, const StreamHdr&) const { return 0; }
  // offset scanner over the stream's size table (one warp)
  __device__ __forceinline__ void scan(unsigned int epoch) const {
    if (total > 0) scan_offsets(a->sy.offs, epoch, reinterpret_cast<const uint16_t*>(a->in + HDR), h.chunks);
  }
};

// Many streams in one launch: the queue runs over the items' chunks back to
// back; each item has its own lookback words (Sync.flags offset by its chunk
// base), header and size.
struct __align__(64) BatchItem {
  CUtensorMap map_in;   // store: the floats; resi_recv: the client's floats
  CUtensorMap map_out;  // decoders: the output floats
  OpArgs a;             // a.sy.flags already offset to this item
  long long chunk_base; // first queue index of this item
  long long chunks;
};

template <int OP>
struct BatchSrc {
  static constexpr bool batched = true;
  const BatchItem* items;
  int n_items;
  long long total;
  // Item of queue index g, searched by the whole warp forward from `cur` (the
  // item of an earlier index of this CTA, or -1): 32 chunk bases per read.
  __device__ __forceinline__ int locate(long long g, int cur, long long& c) const {
    const int lane = threadIdx.x & 31;
    int lo = cur < 0 ? 0 : cur;
    while (true) {
      const int i = lo + lane;
      const bool le = i < n_items && items[i].chunk_base <= g;
      const int cnt = __popc(__ballot_sync(0xffffffffu, le));
      if (cnt < 32) {
        const int it = lo + cnt - 1;
        c = g - items[it].chunk_base;
        return it;
      }
      lo += 31;
    }
  }
  __device__ __forceinline__ const OpArgs& args(int i) const { return items[i].a; }
  __device__ __forceinline__ void quant(int i, Quant& x1, Quant& x2) const {
    x1 = items[i].a.q1;
    x2 = items[i].a.q2;
  }
  __device__ __forceinline__ const CUtensorMap* min(int i) const { return &items[i].map_in; }
  __device__ __forceinline__ const CUtensorMap* mout(int i) const { return &items[i].map_out; }
  __device__ __forceinline__ StreamHdr header(int i) const { return read_header(items[i].a.in, items[i].a.in_bytes); }
  // 0 = usable; 2 = size mismatch; 3 = corrupt header
  __device__ __forceinline__ int header_bad(int i, const StreamHdr& h) const {
    const OpArgs& a = items[i].a;
    if (!h.ok) return 3;
    const bool ok = h.n == a.n && (OP == OP_S2C || OP == OP_RESI || h.n <= a.out_cap);
    return ok ? 0 : 2;
  }
  // offset scanner over every usable item's size table, item after item
  __device__ __forceinline__ void scan(unsigned int epoch) const {
    for (int i = 0; i < n_items; i++) {
      const StreamHdr h = header(i);
      if (header_bad(i, h)) continue;
      scan_offsets(items[i].a.sy.offs, epoch, reinterpret_cast<const uint16_t*>(items[i].a.in + HDR), h.chunks);
    }
  }
};

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// ---- prefetchers (warp 3): resolve queue index g and start its loads into
// stage t.  Every TMA is issued by lane 0 (TMA_TID).
struct WalkState {
  int item;                 // item of the last prefetched index (-1: none)
};

template <class Src>
__device__ __forceinline__ void prefetch_floats(Ctl& sm, int t, long long g, const Src& src, WalkState& ws) {
  const int lane = threadIdx.x & 31;
  StageMeta& m = sm.st[t];
  if (g >= src.total) {
    if (lane == 0) {
      m.g = g;
      mbar_arrive(&sm.bar[t]);
      mbar_arrive(&sm.bar[t]);
    }
    return;
  }
  long long c;
  const int item = src.locate(g, ws.item, c);
  const bool fresh = item != ws.item;
  ws.item = item;
  if (lane == 0) {
    const OpArgs& A = src.args(item);
    const int nw = (int)min((long long)CW, (A.n - c * CS) / 4);
    const bool tma = nw == CW && A.has_map_in;
    if (tma) {
      if (Src::batched && fresh) tensormap_acquire(src.min(item));
      fence_proxy_async();
      mbar_expect_tx(&sm.bar[t], CS);
      tma_load_rows(stage_buf(sm, t), src.min(item), (int)(c * 128), &sm.bar[t]);
    } else {
      mbar_arrive(&sm.bar[t]);
    }
    m.g = g;
    m.c = c;
    m.item = item;
    m.nw = nw;
    m.tma = tma;
    m.n = A.n;
    m.chunks = (A.n + CS - 1) / CS;
    m.bad = 0;
    mbar_arrive(&sm.bar[t]);
  }
}

// Decoders: the payload offset comes from the launch's offset scanner (the
// prefix sum of the size table that the reference's decoders form per CTA,
// d_s2c.h:98-106).  One bulk copy brings the payload's 16-byte-aligned span;
// the lanes copy the ragged tail.
template <class Src>
__device__ __forceinline__ void prefetch_stream(Ctl& sm, int t, long long g, const Src& src, WalkState& ws) {
  const int lane = threadIdx.x & 31;
  StageMeta& m = sm.st[t];
  if (g >= src.total) {
    if (lane == 0) {
      m.g = g;
      mbar_arrive(&sm.bar[t]);
      mbar_arrive(&sm.bar[t]);
    }
    return;
  }
  long long c;
  const int item = src.locate(g, ws.item, c);
  const bool fresh = item != ws.item;
  ws.item = item;
  const OpArgs& A = src.args(item);
  const StreamHdr h = src.header(item);
  const int hb = src.header_bad(item, h);
  if (hb) {
    if (lane == 0) {
      m.g = g;
      m.c = c;
      m.item = item;
      m.nw = CW;
      m.tma = 0;
      m.bad = hb;
      m.csize = 0;
      m.d = 0;
      m.n = 0;
      m.chunks = 0;
      m.eb_e = 1;
      mbar_arrive(&sm.bar[t]);
      mbar_arrive(&sm.bar[t]);
    }
    return;
  }
  const long long chunks = h.chunks;
  const int nw = (int)min((long long)CW, (h.n - c * CS) / 4);
  const int osize = nw * 4;
  const uint16_t* table = reinterpret_cast<const uint16_t*>(A.in + HDR);
  const uint8_t* data = A.in + HDR + 2 * chunks;
  const long long data_bytes = A.in_bytes - HDR - 2 * chunks;
  unsigned long long off = 0;
  int cs = 0;
  if (lane == 0) {
    cs = table[c];  // in flight together with the offset read
    off = wait_offset(A.sy, sm.epoch, c);
  }
  off = __shfl_sync(0xffffffffu, off, 0);
  cs = __shfl_sync(0xffffffffu, cs, 0);
  const int bad = (cs > osize) || (cs < 2 && cs != osize) || ((long long)off + cs > data_bytes);
  const uintptr_t Aa = reinterpret_cast<uintptr_t>(data + off);
  const uintptr_t a0 = Aa & ~uintptr_t(15);
  uintptr_t a1 = (Aa + (bad ? 0 : cs)) & ~uintptr_t(15);
  if (a1 < a0) a1 = a0;
  // The copy may run into the next payload's bytes: it takes the ragged tail
  // too unless that would read past the stream's valid bytes.
  const uintptr_t a1_up = (Aa + (bad ? 0 : cs) + 15) & ~uintptr_t(15);
  if (!bad && a1_up <= reinterpret_cast<uintptr_t>(A.in + A.in_bytes)) a1 = a1_up;
  const int d = (int)(Aa - a0);
  const int tma_len = (int)(a1 - a0);
  uint8_t* dst = reinterpret_cast<uint8_t*>(stage_buf(sm, t));
  if (lane == 0) {
    bulk_wait_read();  // a TMA store of this buffer's previous chunk may still be reading it
    fence_proxy_async();
    if (tma_len) {
      if (Src::batched && fresh) tensormap_acquire(src.mout(item));
      mbar_expect_tx(&sm.bar[t], (uint32_t)tma_len);
      bulk_load(dst, reinterpret_cast<const void*>(a0), (uint32_t)tma_len, &sm.bar[t]);
    } else {
      if (Src::batched && fresh) tensormap_acquire(src.mout(item));
      mbar_arrive(&sm.bar[t]);
    }
    if (Src::batched && fresh) tensormap_acquire(src.min(item));
    m.g = g;
    m.c = c;
    m.item = item;
    m.nw = nw;
    m.tma = tma_len != 0;
    m.bad = bad;
    m.csize = bad ? 0 : cs;
    m.d = d;
    m.tma_len = tma_len;
    m.off = off;
    m.n = h.n;
    m.chunks = chunks;
    m.eb_e = h.eb_e;
  }
  __syncwarp();
  if (!bad) {
    const uint8_t* gsrc = data + off;
    const int from = tma_len - d;  // payload bytes [from, cs) are copied by the lanes
    for (int i = lane + (from > 0 ? from : 0); i < cs; i += 32) dst[d + i] = gsrc[i];
  }
  __syncwarp();
  if (lane == 0) mbar_arrive(&sm.bar[t]);
}

// ---- the three pipelined loops.  Each CTA dequeues chunk indices from the
// launch's queue; warp 3 resolves an index and starts its loads.  Decoders
// take their indices one iteration ahead and load the next chunk while the
// current one is decoded; encoders take an index when they start the chunk.
//
// Encoders publish a chunk's compressed size as soon as it is known and write
// its payload one iteration later (flush_chunk): by then every earlier chunk
// has published too, and the resolver CTA has usually turned the chunk's own
// lookback word into an inclusive prefix, so no CTA waits on its
// predecessors while it holds the SM.

// Resolves and writes out the chunk pending in slot t (if any): warp 0 finds
// its output offset, a barrier publishes it, every thread stores the payload
// from `staging`, or a raw chunk's words from raw_word(args, chunk, w).
// Called by every thread.
template <class Src, typename RawWord>
__device__ __forceinline__ void flush_pending(Ctl& sm, const Src& src, int t, const uint8_t* staging,
                                              RawWord raw_word) {
  Pend& pd = sm.pend[t];
  const bool valid = pd.valid;  // written before an earlier barrier
  if (valid && threadIdx.x < 32) {
    const unsigned long long X = lookback_resolve(src.args(pd.item).sy, sm.epoch, pd.c, pd.csize);
    if (threadIdx.x == 0) sm.payload_off = X;
  }
  __syncthreads();
  if (valid) {
    const OpArgs& Q = src.args(pd.item);
    const long long chunks = (Q.n + CS - 1) / CS;
    const long long c = pd.c;
    flush_chunk(sm, pd, reinterpret_cast<const uint32_t*>(staging), false,
                [&](int w) -> uint32_t { return raw_word(Q, c, w); }, Q.out + HDR + 2 * chunks,
                reinterpret_cast<uint16_t*>(Q.out + HDR), Q.out_size, chunks);
  }
}

// Requantization through floats (d_s2c.h:132-137, d_RESI_4.h:57-76): the
// stored bin (or, for a raw chunk, the float itself) -> float (iSQ) -> request
// bin (CQ), or residual = destination bin minus the request bin requantized
// to the destination bound.  For the words (bit k of m) that the shift form
// cannot take; the choice is per word, so one outlier no longer sends its
// warp's 1024 words down the slow path.  Out of line: such words are rare
// (lossless words, raw chunks), and inlining the integer forms 32 times over
// made the loop large enough to stall on instruction fetch.  The words are
// the calling thread's own row of a swizzled buffer (row_store before the
// call, row_load after): a pointer to the caller's register array would put
// that array in local memory for the whole loop.
template <int OP>
__device__ __noinline__ void requant_words(uint32_t* buf, uint32_t m, bool raw, Quant qs, Quant q1, Quant q2) {
  const uint32_t base = 32u * threadIdx.x;
  for (; m; m &= m - 1) {
    const uint32_t w = swz(base + __ffs(m) - 1);
    const uint32_t x = raw ? buf[w] : iq_dec(buf[w], qs);
    if (OP == OP_S2C) {
      buf[w] = cq_enc(x, q1);
    } else {
      const uint32_t src_req = cq_enc(iq_dec(cq_enc(x, q1), q1), q2);
      buf[w] = cq_enc(x, q2) - src_req;
    }
  }
}

// store (d_server_encode_kernel): floats -> SQ -> encode.  A chunk arrives in
// buffer 0, which becomes its plane buffer; its compacted payload goes to
// buffer 1 once the previous chunk's payload has been flushed from there (that
// flush runs as soon as this chunk's size is published).  The next chunk is
// loaded when the compaction has read buffer 0.
template <class Src>
__device__ __forceinline__ void store_loop(Ctl& sm, const Src& src, const Sync& sy) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  begin_launch(sm, sy);
  if (tid == 0) {
    sm.pend[0].valid = 0;
    sm.pend[1].valid = 0;
  }
  WalkState ws{-1};
  __syncthreads();
  uint32_t* A = stage_buf(sm, 0);
  uint8_t* B = reinterpret_cast<uint8_t*>(stage_buf(sm, 1));
  // a raw chunk stores the original floats, read again from global memory
  auto raw_word = [](const OpArgs& Q, long long c, int w) -> uint32_t {
    return reinterpret_cast<const uint32_t*>(Q.in)[c * (long long)CW + w];
  };
  auto take_next = [&]() {
    if (warp == 3) {
      long long g = 0;
      if (lane == 0) g = atomicAdd(&sy.counter[0], 1u);
      prefetch_floats(sm, 0, __shfl_sync(0xffffffffu, g, 0), src, ws);
    }
  };
  take_next();
  uint32_t phase = 0;
  int s = 0;  // pending-chunk slot of this iteration's chunk
  for (;; s ^= 1) {
    if (!mbar_wait(&sm.bar[0], phase & 1, sy.timeout_ns)) latch(sy.status, DST_TIMEOUT);
    phase ^= 1u;
    const StageMeta& m = sm.st[0];
    if (m.g >= src.total) break;
    const int item = m.item;
    const OpArgs& A_ = src.args(item);
    const long long c = m.c;
    const int nw = m.nw;
    if (!m.tma) {
      load_plain_rows(A, A_.in, c, nw);
      __syncthreads();
    }
    Quant q1, q2_unused;
    src.quant(item, q1, q2_unused);
    if (Src::batched && c == 0 && tid == 0) write_header(A_.out, A_.n, q1.eb_e);
    uint32_t v[32];
    row_load(A, tid, v);
    {
      // the float form; a warp that holds lossless words (inf, NaN included)
      // chooses per word
      const FastQ fq = make_fastq(q1.eb_e);
      uint32_t amax = 0;
#pragma unroll
      for (int k = 0; k < 32; k++) amax = max(amax, v[k] & 0x7fffffffu);
      if (!__any_sync(0xffffffffu, amax >= fq.thr_bits)) {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = sq_fast(v[k], fq);
      } else {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = sq_mixed(v[k], fq, q1);
      }
    }
    auto flush_prev = [&]() {
      flush_pending(sm, src, s ^ 1, B, raw_word);
      __syncthreads();  // buffer 1 has been read
    };
    if (nw == CW) {
      encode_stage<true>(sm, A_.sy, v, A, B, c, nw, item, sm.pend[s], flush_prev);
    } else {
      flush_prev();
      row_store(A, tid, v);
      encode_stage_partial(sm, A_.sy, A, B, c, nw, item, sm.pend[s]);
    }
    if (tid == 0) sm.pend[s ^ 1].valid = 0;
    __syncthreads();  // buffer 0 has been read
    take_next();
  }
  flush_pending(sm, src, s ^ 1, B, raw_word);
}

// The client side of a served request, fused into init_send / resi_send
// (cortado_*_send_apply): the words the re-encoder is about to encode (request
// bins, or residuals) are applied to the client's reconstruction directly,
// so the stream just written need not be decoded again.  The results equal
// init_recv / resi_recv of that stream bit for bit:
//   init: iCQ(bin) (d_client_encode.h:230-254); a chunk that the encoder
//         stores uncompressed is rewritten with its bins afterwards
//         (client_raw_bins), as init_recv copies raw chunks out as stored;
//   resi: iCQ(CQ(client, dst) + residual, dst) (d_RESI_4.h:79-94); the
//         residual ints are the same whether the chunk compresses or not.
// A full chunk goes through the stage buffer X, whose rows 32w .. 32w+31
// only warp w touches at this point of the loop (row tid is each thread's
// own): the warp moves its 4 KiB of the client's floats between global and
// those rows 512 contiguous bytes at a time, and each thread works on its own
// row.  The float forms apply when the whole warp allows them (no lossless
// client word, no lossless bin), else the per-word forms, as in the decoders.
// A partial chunk works word by word on the client's floats directly.
template <int OP>
__device__ __forceinline__ void client_apply(const OpArgs& A, long long c, int nw, const uint32_t (&v)[32], Quant q,
                                             uint32_t* X) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const FastQ fq = make_fastq(q.eb_e);
  if (nw == CW) {
    uint4* g4 = reinterpret_cast<uint4*>(A.client) + c * (long long)(CW / 4) + 256 * warp;
    uint4* X4 = reinterpret_cast<uint4*>(X);
    uint4* own = X4 + 8 * tid;
    // lane l's part of the warp's i-th 512 bytes: linear 16-byte unit
    // 256*warp + 32*i + l, i.e. row 32*warp + 4*i + l/8, unit l%8 of that row
    auto unit = [&](int i) -> uint4* {
      const int r = 32 * warp + 4 * i + (lane >> 3);
      return X4 + 8 * r + ((lane & 7) ^ (r & 7));
    };
    __syncwarp();  // the rows' earlier uses by this warp's threads are done
    uint32_t bmax = 0;
    if (OP == OP_S2C) {
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const uint32_t neg = (uint32_t)((int32_t)v[k] >> 31);
        bmax = max(bmax, (v[k] ^ neg) - neg);
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) async_copy16(unit(i), g4 + 32 * i + lane);  // all eight in flight, no registers
      async_wait_all();
      __syncwarp();
      uint32_t amax = 0;
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint4 w = own[u ^ (tid & 7)];
        amax = max(amax, max(max(w.x & 0x7fffffffu, w.y & 0x7fffffffu), max(w.z & 0x7fffffffu, w.w & 0x7fffffffu)));
      }
      // destination bins of the client's floats plus the residuals, into the row
      const bool fast_c = !__any_sync(0xffffffffu, amax >= fq.thr_bits);
      __syncwarp();  // the row is read again below, not held in registers beside v
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint4 w = own[u ^ (tid & 7)];
        uint4 b;
        if (fast_c) {
          b = make_uint4(cq_fast(w.x, fq) + v[4 * u], cq_fast(w.y, fq) + v[4 * u + 1], cq_fast(w.z, fq) + v[4 * u + 2],
                         cq_fast(w.w, fq) + v[4 * u + 3]);
        } else {
          b = make_uint4(cq_mixed(w.x, fq, q) + v[4 * u], cq_mixed(w.y, fq, q) + v[4 * u + 1],
                         cq_mixed(w.z, fq, q) + v[4 * u + 2], cq_mixed(w.w, fq, q) + v[4 * u + 3]);
        }
        own[u ^ (tid & 7)] = b;
        const uint32_t b4[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const uint32_t neg = (uint32_t)((int32_t)b4[j] >> 31);
          bmax = max(bmax, (b4[j] ^ neg) - neg);
        }
      }
    }
    const bool fast_i = __all_sync(0xffffffffu, bmax < 0x800000u);
    if (OP == OP_S2C) {  // the request bins into the row
#pragma unroll
      for (int u = 0; u < 8; u++) own[u ^ (tid & 7)] = make_uint4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
    }
    __syncwarp();  // the warp's rows hold its bins
    // dequantized on the way out, 512 contiguous bytes at a time
#pragma unroll 2
    for (int i = 0; i < 8; i++) {
      const uint4 b = *unit(i);
      g4[32 * i + lane] = fast_i ? make_uint4(iq_fast(b.x, fq), iq_fast(b.y, fq), iq_fast(b.z, fq), iq_fast(b.w, fq))
                                 : make_uint4(iq_mixed(b.x, fq, q), iq_mixed(b.y, fq, q), iq_mixed(b.z, fq, q),
                                              iq_mixed(b.w, fq, q));
    }
    __syncwarp();  // the rows are read before the encoder reuses the buffer
  } else {
    uint32_t* row = reinterpret_cast<uint32_t*>(A.client) + c * (long long)CW + 32 * tid;
#pragma unroll
    for (int k = 0; k < 32; k++) {
      if (32 * tid + k < nw) {
        row[k] = (OP == OP_S2C) ? iq_mixed(v[k], fq, q) : iq_mixed(cq_mixed(row[k], fq, q) + v[k], fq, q);
      }
    }
  }
}

// init_send with apply, for a chunk stored uncompressed: its bins (rebuilt
// into row tid of Yw by raw_rebuild) replace the dequantized words this
// thread wrote, as init_recv emits a raw chunk's bins unchanged.
__device__ __noinline__ void client_raw_bins(const OpArgs& A, long long c, int nw, const uint32_t* Yw) {
  const int tid = threadIdx.x;
  uint32_t* row = reinterpret_cast<uint32_t*>(A.client) + c * (long long)CW + 32 * tid;
  for (int k = 0; k < 32; k++)
    if (32 * tid + k < nw) row[k] = Yw[swz(32 * tid + k)];
}

// Rebuilds a raw chunk's requantized words from the plane buffer into the
// staging buffer (out of line: only chunks that do not compress take it, and
// the re-encoders' loop is large enough to stall on instruction fetch).
__device__ __noinline__ void raw_rebuild(Ctl& sm, const uint32_t* X, int nw, uint32_t* Yw) {
  uint32_t w[32];
  if (nw == CW) planes_to_words<true>(sm, X, nw, w);
  else planes_to_words<false>(sm, X, nw, w);
  row_store(Yw, threadIdx.x, w);
}

// init_send / resi_send (d_s2c_encode_kernel, d_residual_encode_kernel):
// decode the stored chunk, requantize or form the residual, encode.  The
// payload arrives in buffer 0 and is expanded in place; after the
// requantization the same buffer is the encoder's plane buffer.  The compacted
// payload goes to buffer 1 once the previous chunk has been flushed from there
// (as in store_loop).  A chunk that does not compress stores its requantized
// words, which are rebuilt from the plane buffer (planes_to_words) into
// buffer 1 -- rare enough not to keep a third buffer for them.
// APPLY: the fused send-and-apply forms (items with a client's floats); the
// plain forms are compiled without that code.
template <int OP, bool APPLY, class Src>
__device__ __forceinline__ void reencode_loop(Ctl& sm, const Src& src, const Sync& sy) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  begin_launch(sm, sy);
  if (tid == 0) {
    sm.pend[0].valid = 0;
    sm.pend[1].valid = 0;
  }
  WalkState ws{-1};
  __syncthreads();  // sm.epoch
  if (gridDim.x == 1 && warp == 1) src.scan(sm.epoch);
  __syncthreads();
  uint32_t* X = stage_buf(sm, 0);
  uint32_t* Yw = stage_buf(sm, 1);
  uint8_t* Y = reinterpret_cast<uint8_t*>(Yw);
  // a raw chunk's payload is its requantized words, kept swizzled in buffer 1
  auto raw_word = [Yw](const OpArgs&, long long, int w) -> uint32_t { return Yw[swz(w)]; };
  auto take_next = [&]() {
    if (warp == 3) {
      long long g = 0;
      if (lane == 0) g = atomicAdd(&sy.counter[0], 1u);
      prefetch_stream(sm, 0, __shfl_sync(0xffffffffu, g, 0), src, ws);
      if (OP == OP_RESI && APPLY && lane == 0) {
        // resi_send with apply reads the client's chunk: bring it into L2 now
        const StageMeta& mn = sm.st[0];
        if (mn.g < src.total && mn.bad == 0) {
          const OpArgs& An = src.args(mn.item);
          if (An.client && mn.nw == CW) prefetch_l2(An.client + mn.c * (long long)CS, CS);
        }
      }
    }
  };
  take_next();
  uint32_t phase = 0;
  int s = 0;  // pending-chunk slot of this iteration's chunk
  for (;; s ^= 1) {
    if (!mbar_wait(&sm.bar[0], phase & 1, sy.timeout_ns)) latch(sy.status, DST_TIMEOUT);
    phase ^= 1u;
    const StageMeta& m = sm.st[0];
    if (m.g >= src.total) break;
    const int item = m.item;
    const OpArgs& A = src.args(item);
    const long long c = m.c;
    const int nw = m.nw;
    auto flush_prev = [&]() {
      flush_pending(sm, src, s ^ 1, Y, raw_word);
      __syncthreads();  // buffer 1 has been read
    };
    uint32_t v[32];
    bool raw;
    if (nw == CW) {
      decode_core<true>(sm, A.sy, m, X, X, v, raw, NoHook{});
    } else {
      raw = decode_core_partial(sm, A.sy, m, X, X, NoHook{});
      row_load(X, tid, v);
    }
    if (m.bad >= 2) {  // unusable stream header (batched): nothing to write
      if (tid == 0) sm.pend[s].valid = 0;
      flush_prev();
    } else {
      // stored bins -> floats (iSQ, skipped for chunks stored as floats) ->
      // request bins (CQ, d_s2c.h:132-137) or residuals (d_RESI_4.h:57-76)
      const Quant qs = make_quant(m.eb_e);
      Quant q1, q2;
      src.quant(item, q1, q2);
      // Shift form, when every word of the warp allows it: a lossy stored bin
      // a (|a| < 2^23) is the float a * 2^(e_s - 126), so its request bin is
      // a / 2^k1 rounded half away from zero (k1 = e_1 - e_s >= 0), and the
      // residual is a / 2^k2 (rounded) minus that request bin moved to the
      // destination's bins, (a / 2^k1 rounded) << (e_1 - e_2), exact while the
      // latter stays a lossy destination bin (magnitudes below `amax`).
      const int k1 = q1.eb_e - qs.eb_e;
      const int k2 = (OP == OP_RESI) ? q2.eb_e - qs.eb_e : 0;
      const int dd = (OP == OP_RESI) ? q1.eb_e - q2.eb_e : 0;
      // Words the shift form cannot take (lossless stored words, magnitudes
      // at or above amax, every word of a chunk stored raw or of a bound
      // order it does not cover) go through the float path out of line.
      // (amax = 0 when the shift form does not apply: no word qualifies and
      // every word keeps its stored bin for the float path.)
      const bool shift_ok = !raw && k1 >= 0 && k2 >= 0 && dd >= 0;
      const uint32_t amax = !shift_ok ? 0u
                            : (OP == OP_RESI && k2 == 0 && k1 >= 1 && k1 <= 23) ? 0x800000u - (1u << (k1 - 1))
                                                                                 : 0x800000u;
      const uint32_t h1 = shl_clamp(1u, (uint32_t)(k1 - 1)), h2 = shl_clamp(1u, (uint32_t)(k2 - 1));
      uint32_t slow = 0;
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const uint32_t neg = (uint32_t)((int32_t)v[k] >> 31);
        const uint32_t a = (v[k] ^ neg) - neg;
        const uint32_t m1 = shr_clamp(a + h1, (uint32_t)k1);
        const uint32_t r = (OP == OP_S2C) ? m1 : shr_clamp(a + h2, (uint32_t)k2) - shl_clamp(m1, (uint32_t)dd);
        const bool ok = a < amax;
        slow |= (ok ? 0u : 1u) << k;
        v[k] = ok ? (r ^ neg) - neg : v[k];
      }
      if (slow) {  // after the decoder's last barrier row tid of X is this thread's own
        row_store(X, tid, v);
        requant_words<OP>(X, slow, raw, qs, q1, q2);
        row_load(X, tid, v);
      }
      if (Src::batched && c == 0 && tid == 0) write_header(A.out, m.n, (OP == OP_S2C) ? q1.eb_e : q2.eb_e);
      if (APPLY && A.client) client_apply<OP>(A, c, nw, v, OP == OP_S2C ? q1 : q2, X);
      if (nw == CW) {
        encode_stage<true>(sm, A.sy, v, X, Y, c, nw, item, sm.pend[s], flush_prev);
      } else {
        flush_prev();
        row_store(X, tid, v);
        encode_stage_partial(sm, A.sy, X, Y, c, nw, item, sm.pend[s]);
        __syncthreads();  // sm.pend[s]
      }
      if (sm.pend[s].raw) {
        // the requantized words, rebuilt from the plane buffer, are the payload
        raw_rebuild(sm, X, nw, Yw);
        if (OP == OP_S2C && APPLY && A.client) client_raw_bins(A, c, nw, Yw);
      }
    }
    if (tid == 0) sm.pend[s ^ 1].valid = 0;
    __syncthreads();  // buffer 0 has been read; buffer 1 holds this chunk's payload
    take_next();
  }
  flush_pending(sm, src, s ^ 1, Y, raw_word);
}

// storage decode / init_recv / resi_recv (d_server_decode_kernel,
// d_client_decode_kernel, d_residual_apply_kernel).  The payload is expanded
// in place in its stage buffer, which then stages the output floats for one
// TMA store.  resi_recv's client chunk is loaded behind the next payload in
// the other stage buffer when that payload is small, else into this stage's
// buffer after the decode.
template <int OP, class Src>
__device__ __forceinline__ void decode_loop(Ctl& sm, const Src& src, const Sync& sy) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  begin_launch(sm, sy);
  __syncthreads();
  if (gridDim.x == 1 && warp == 1) src.scan(sm.epoch);
  __syncthreads();
  WalkState ws{-1};
  long long pending = 0;
  if (warp == 3) {
    long long g0 = 0;
    if (lane == 0) g0 = atomicAdd(&sy.counter[0], 1u);
    g0 = __shfl_sync(0xffffffffu, g0, 0);
    prefetch_stream(sm, 0, g0, src, ws);
    if (lane == 0) pending = atomicAdd(&sy.counter[0], 1u);
  }
  __syncthreads();
  uint32_t phase = 0;  // bits 0, 1: stages; bit 2: client chunk
  for (int s = 0;; s ^= 1) {
    const StageMeta& m = sm.st[s];
    if (m.g >= src.total) break;
    const int item = m.item;
    const OpArgs& A = src.args(item);
    const long long c = m.c;
    const int nw = m.nw;
    const bool full = nw == CW;
    uint32_t* P = stage_buf(sm, s);
    if (Src::batched && c == 0 && tid == 0 && m.bad < 2) *A.out_size = m.n;
    if (!mbar_wait(&sm.bar[s], (phase >> s) & 1, sy.timeout_ns)) latch(sy.status, DST_TIMEOUT);
    phase ^= 1u << s;
    auto next = [&]() {
      if (warp == 3) {
        const long long gp = __shfl_sync(0xffffffffu, pending, 0);
        if (lane == 0) pending = atomicAdd(&sy.counter[0], 1u);
        prefetch_stream(sm, s ^ 1, gp, src, ws);
        if (OP == OP_RAPPLY && lane == 0) {
          // When the next payload fills at most the first KiB of the other
          // stage buffer, this chunk's client floats are loaded behind it
          // (1024-byte aligned) now, overlapping the decode, instead of into
          // this stage's buffer once the decode has read it back.  A next
          // chunk that is present and usable means prefetch_stream has waited
          // for that buffer's previous TMA store and fenced the proxies.
          const StageMeta& mn = sm.st[s ^ 1];
          const bool side = full && A.has_map_in && m.bad == 0 && mn.g < src.total && mn.bad == 0 &&
                            mn.tma_len <= 1024 && mn.d + mn.csize <= 1024;
          sm.src_side = side ? 1u : 0u;
          if (side) {
            mbar_expect_tx(&sm.bar_src, CS);
            tma_load_rows(stage_buf(sm, s ^ 1) + 256, src.min(item), (int)(c * 128), &sm.bar_src);
          }
        }
      }
    };
    uint32_t v[32];
    bool raw;
    if (full) {
      decode_core<true>(sm, A.sy, m, P, P, v, raw, next);
    } else {
      next();
      raw = decode_core_partial(sm, A.sy, m, P, P, NoHook{});
      row_load(P, tid, v);
    }
    if (m.bad >= 2) {  // unusable stream header (batched): nothing to write
      __syncthreads();
      continue;
    }
    const Quant q = make_quant(m.eb_e);
    if (OP == OP_RAPPLY) {
      // d_iRESI_4 (d_RESI_4.h:79-94): requantize the client's floats to the
      // destination bound, add the residual, dequantize.  The client's chunk
      // is behind the next payload (sm.src_side) or comes into this stage's
      // buffer once the decoder has read it back.
      __syncthreads();  // sm.src_side
      const bool src_tma = full && A.has_map_in;
      const uint32_t* S = P;  // where the client's chunk is
      if (src_tma) {
        if (sm.src_side) {
          S = stage_buf(sm, s ^ 1) + 256;
        } else if (tid == TMA_TID) {
          fence_proxy_async();
          mbar_expect_tx(&sm.bar_src, CS);
          tma_load_rows(P, src.min(item), (int)(c * 128), &sm.bar_src);
        }
        if (!mbar_wait(&sm.bar_src, (phase >> 2) & 1, sy.timeout_ns)) latch(sy.status, DST_TIMEOUT);
        phase ^= 4u;
      } else {
        load_plain_rows(P, A.src, c, nw);
        __syncthreads();
      }
      // The client's words are read from shared memory 16 bytes at a time
      // and folded into v in place (client bin + residual), so only one
      // 32-word array is live.  The float forms, chosen per word in a warp
      // that holds lossless client words or bins.
      const uint4* Srow = reinterpret_cast<const uint4*>(S + 32 * tid);
      const FastQ fq = make_fastq(m.eb_e);
      uint32_t amax = 0;
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint4 w = Srow[u ^ (tid & 7)];
        amax = max(amax, max(max(w.x & 0x7fffffffu, w.y & 0x7fffffffu), max(w.z & 0x7fffffffu, w.w & 0x7fffffffu)));
      }
      if (!__any_sync(0xffffffffu, amax >= fq.thr_bits)) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const uint4 w = Srow[u ^ (tid & 7)];
          v[4 * u] += cq_fast(w.x, fq);
          v[4 * u + 1] += cq_fast(w.y, fq);
          v[4 * u + 2] += cq_fast(w.z, fq);
          v[4 * u + 3] += cq_fast(w.w, fq);
        }
      } else {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const uint4 w = Srow[u ^ (tid & 7)];
          v[4 * u] += cq_mixed(w.x, fq, q);
          v[4 * u + 1] += cq_mixed(w.y, fq, q);
          v[4 * u + 2] += cq_mixed(w.z, fq, q);
          v[4 * u + 3] += cq_mixed(w.w, fq, q);
        }
      }
      uint32_t bmax = 0;
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const uint32_t neg = (uint32_t)((int32_t)v[k] >> 31);
        bmax = max(bmax, (v[k] ^ neg) - neg);
      }
      if (__all_sync(0xffffffffu, bmax < 0x800000u)) {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = iq_fast(v[k], fq);
      } else {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = iq_mixed(v[k], fq, q);
      }
    } else if (!raw) {
      // chunks stored uncompressed are copied out as stored: original floats
      // for storage decode (d_server_encode.h:234-249), request bins for
      // init_recv (d_client_encode.h:230-254, the reference's behaviour).
      // The float dequantizer, chosen per word in a warp that holds lossless
      // bins.
      const FastQ fq = make_fastq(m.eb_e);
      uint32_t bmax = 0;
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const uint32_t neg = (uint32_t)((int32_t)v[k] >> 31);
        bmax = max(bmax, (v[k] ^ neg) - neg);
      }
      if (__all_sync(0xffffffffu, bmax < 0x800000u)) {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = iq_fast(v[k], fq);
      } else {
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = iq_mixed(v[k], fq, q);
      }
    }
    row_store(P, tid, v);  // every plane read finished before the decoder's last barrier
    const bool tma_out = full && A.has_map_out;
    if (tma_out) fence_proxy_async();
    __syncthreads();
    if (tma_out) {
      if (tid == TMA_TID) {
        tma_store_rows(src.mout(item), (int)(c * 128), P);
        bulk_commit();
      }
    } else {
      uint32_t* g = reinterpret_cast<uint32_t*>(A.out) + c * (long long)CW;
      for (int w = tid; w < nw; w += NT) g[w] = P[swz(w)];
      __syncthreads();
    }
  }
  if (tid == TMA_TID) bulk_wait_read();
}

// ---- the helper CTA of a launch (the first CTA to start, when there are at
// least two): warp 0 runs the lookback resolver (encoders), warp 1 the offset
// scanner (stream inputs).  Being the first to start, it is resident even
// when other kernels share the GPU and not every CTA of the launch fits at
// once, so the CTAs that wait for its offsets cannot wait for a CTA that
// waits for them.  A one-CTA launch scans its offsets itself first.
__device__ __forceinline__ bool helper_cta(Ctl& sm, const Sync& sy) {
  if (gridDim.x < 2) return false;
  if (threadIdx.x == 0) sm.is_last = atomicAdd(&sy.counter[6], 1u) == 0;
  __syncthreads();
  const bool h = sm.is_last;
  __syncthreads();
  return h;
}

template <bool RESOLVE, bool SCAN, class Src>
__device__ __forceinline__ void run_helper(Ctl& sm, const Src& src, const Sync& sy) {
  begin_launch(sm, sy);
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  if (RESOLVE && sy.resolver && warp == 0) resolve_loop(sy, sm.epoch, src.total);
  if (SCAN && warp == 1) src.scan(sm.epoch);
}

// ---- single-stream kernels
__global__ void __launch_bounds__(NT, MINB_STORE) k_store(const __grid_constant__ OpArgs a, const __grid_constant__ CUtensorMap map_in) {
  Ctl& sm = ctl_block();
  Quant q1, q2;
  const unsigned int noa_err = resolve_noa(a, q1, q2);  // every thread, the same result
  const long long chunks = noa_err ? 0 : (a.n + CS - 1) / CS;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (noa_err) {
      latch(a.sy.status, noa_err);  // nothing is written, as the host path writes nothing
    } else {
      write_header(a.out, a.n, q1.eb_e);
      if (chunks == 0) *a.out_size = HDR;
    }
  }
  const SingleSrc src{&a, &map_in, nullptr, chunks, StreamHdr{}, q1, q2};
  if (helper_cta(sm, a.sy)) run_helper<true, false>(sm, src, a.sy);
  else store_loop(sm, src, a.sy);
  finish_launch(sm, a.sy);
}

template <int OP, bool APPLY>
__global__ void __launch_bounds__(NT, MINB_REENC) k_reencode(const __grid_constant__ OpArgs a) {
  Ctl& sm = ctl_block();
  StreamHdr h = read_header(a.in, a.in_bytes);
  const bool hdr_ok = h.ok && h.n == a.n;
  if (!hdr_ok) h.chunks = 0;
  Quant q1, q2;
  const unsigned int noa_err = resolve_noa(a, q1, q2);  // every thread, the same result
  if (noa_err) h.chunks = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (noa_err) {
      latch(a.sy.status, noa_err);  // nothing is written, as the host path writes nothing
    } else {
      if (!hdr_ok) latch(a.sy.status, h.ok ? DST_SIZE_MISMATCH : DST_CORRUPT);
      write_header(a.out, hdr_ok ? h.n : 0, (OP == OP_S2C) ? q1.eb_e : q2.eb_e);
      if (h.chunks == 0) *a.out_size = HDR;
    }
  }
  const SingleSrc src{&a, nullptr, nullptr, h.chunks, h, q1, q2};
  if (helper_cta(sm, a.sy)) run_helper<true, true>(sm, src, a.sy);
  else reencode_loop<OP, APPLY>(sm, src, a.sy);
  finish_launch(sm, a.sy);
}

template <int OP>
__global__ void __launch_bounds__(NT, OP == OP_RAPPLY ? MINB_RAPPLY : MINB_DEC) k_decode(const __grid_constant__ OpArgs a, const __grid_constant__ CUtensorMap map_src,
                                               const __grid_constant__ CUtensorMap map_out) {
  Ctl& sm = ctl_block();
  StreamHdr h = read_header(a.in, a.in_bytes);
  bool hdr_ok = h.ok && h.n <= a.out_cap;
  if (OP == OP_RAPPLY) hdr_ok = hdr_ok && h.n == a.n;
  if (!hdr_ok) h.chunks = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (!hdr_ok) latch(a.sy.status, !h.ok ? DST_CORRUPT : (OP == OP_RAPPLY && h.n != a.n) ? DST_SIZE_MISMATCH : DST_CAPACITY);
    *a.out_size = hdr_ok ? h.n : 0;
  }
  const SingleSrc src{&a, &map_src, &map_out, h.chunks, h, a.q1, a.q2};
  if (helper_cta(sm, a.sy)) run_helper<false, true>(sm, src, a.sy);
  else decode_loop<OP>(sm, src, a.sy);
  finish_launch(sm, a.sy);
}

// ---- batched kernels: one persistent launch over many streams.
template <int OP, bool APPLY = false>
__global__ void __launch_bounds__(NT, OP == OP_STORE ? MINB_STORE : (OP == OP_RAPPLY ? MINB_RAPPLY : (OP == OP_S2C || OP == OP_RESI) ? MINB_REENC : MINB_DEC))
k_batch(const BatchItem* __restrict__ items, int n_items, long long total_chunks, const __grid_constant__ Sync sy) {
  Ctl& sm = ctl_block();
  const BatchSrc<OP> src{items, n_items, total_chunks};
  constexpr bool encoder = OP == OP_STORE || OP == OP_S2C || OP == OP_RESI;
  if (helper_cta(sm, sy)) run_helper<encoder, OP != OP_STORE>(sm, src, sy);
  else if (OP == OP_STORE) store_loop(sm, src, sy);
  else if (encoder) reencode_loop<OP, APPLY>(sm, src, sy);
  else decode_loop<OP>(sm, src, sy);
  finish_launch(sm, sy);
}

// ---- store without allocation (cortado_store_encode_noalloc)
// Fixed scratch for callers that cannot allocate device memory: one
// lookback word per chunk for up to CORTADO_NOALLOC_MAX_BYTES of input, then
// the chunk queue, the finished-CTA count, the status word, the epoch and the
// helper ticket (32-bit words 0, 1, 2, 3 and 6 of the last 4 entries).  Every GPU that
// loads the library holds this array until the process exits.
constexpr long long NOALLOC_CHUNKS = CORTADO_NOALLOC_MAX_BYTES / CS;
__device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_CHUNKS + 4];

// Same chunk loop as k_store; the last CTA out also reports a device-side
// error as a negative *out_size (there is no context to read it from) and
// clears the status word for the next call (finish_launch).
__global__ void __launch_bounds__(NT, MINB_STORE) k_store_noalloc(const __grid_constant__ OpArgs a,
                                                                  const __grid_constant__ CUtensorMap map_in) {
  Ctl& sm = ctl_block();
  const long long chunks = (a.n + CS - 1) / CS;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    write_header(a.out, a.n, a.q1.eb_e);
    if (chunks == 0) *a.out_size = HDR;
  }
  const SingleSrc src{&a, &map_in, nullptr, chunks, StreamHdr{}, a.q1, a.q2};
  if (helper_cta(sm, a.sy)) run_helper<true, false>(sm, src, a.sy);
  else store_loop(sm, src, a.sy);
  const unsigned int st = finish_launch(sm, a.sy, true);
  if (st) *a.out_size = -(long long)st;
}

// ---- bound verifier (MAXABS_f32, include/verifiers/MAXABS_f32.h:40-72): the
// first index whose reconstruction violates the absolute bound (NaN/Inf must
// match: unequal unless both are NaN), or n if none.
__device__ __forceinline__ bool maxabs_bad(float o, float r, float eb) {
  if (!isfinite(o) || !isfinite(r)) return (r != o) && (!isnan(o) || !isnan(r));
  const float lower = __fsub_rn(o, eb), upper = __fadd_rn(o, eb);
  return (r < lower) || (r > upper) || (fabsf(__fsub_rn(o, r)) > eb);
}

__global__ void k_verify(const float* __restrict__ orig, const float* __restrict__ recon, long long nw, float eb,
                         unsigned long long* first_bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw; i += stride) {
    if (maxabs_bad(orig[i], recon[i], eb)) {
      atomicMin(first_bad, (unsigned long long)i);
      return;
    }
  }
}

// ---- NOA range: min/max over the floats, NaNs ignored (fminf/fmaxf skip
// NaN operands).  Each thread keeps four 16-byte loads in flight per pass.
__device__ __forceinline__ unsigned int ordered(float f) {
  const unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void __launch_bounds__(256) k_minmax(const float* x, long long nw, unsigned int* out /* [2]: ordered-int min, max */) {
  float mn = INFINITY, mx = -INFINITY;
  const long long nv = nw / 4;
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long i = t;
  for (; i + 3 * nthr < nv; i += 4 * nthr) {
    float4 v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = __ldcs(x4 + i + j * nthr);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      mn = fminf(fminf(mn, v[j].x), fminf(v[j].y, fminf(v[j].z, v[j].w)));
      mx = fmaxf(fmaxf(mx, v[j].x), fmaxf(v[j].y, fmaxf(v[j].z, v[j].w)));
    }
  }
  for (; i < nv; i += nthr) {
    const float4 v = x4[i];
    mn = fminf(fminf(mn, v.x), fminf(v.y, fminf(v.z, v.w)));
    mx = fmaxf(fmaxf(mx, v.x), fmaxf(v.y, fmaxf(v.z, v.w)));
  }
  for (long long k = 4 * nv + t; k < nw; k += nthr) {
    mn = fminf(mn, x[k]);
    mx = fmaxf(mx, x[k]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&out[0], ordered(mn));
    atomicMax(&out[1], ordered(mx));
  }
}

// Hands the range to the host through mapped pinned memory (a plain store,
// no copy engine, so it is not queued behind bulk copies on other streams)
// and resets the device words for the next call.
__global__ void k_range_publish(unsigned int* words, volatile unsigned int* host) {
  host[0] = words[0];
  host[1] = words[1];
  words[0] = 0xffffffffu;
  words[1] = 0u;
  __threadfence_system();
}

// The range for the device-side NOA entry points: min and max as floats into
// device memory (no host hand-over), and the reduction words reset.
__global__ void k_range_to_device(unsigned int* words, float* out) {
  auto unord = [](unsigned int o) { return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o); };
  out[0] = unord(words[0]);
  out[1] = unord(words[1]);
  words[0] = 0xffffffffu;
  words[1] = 0u;
}

// Failure-detection self-test: one thread waits, through the decoders' own
// bounded wait, for a payload offset tagged with epoch 0x10000.  Lookback and
// offset words carry a 16-bit epoch, so no launch can ever publish it; the
// wait runs out after the context's timeout, latches DST_TIMEOUT and returns.
__global__ void k_wait_selftest(Sync sy) {
  if (threadIdx.x == 0) (void)wait_offset(sy, 0x10000u, 0);
}

}  // namespace

// ================================================================== host side
struct cortado_ctx {
  int device = 0;
  int sms = 0;
  int grid_store = 0, grid_reenc = 0, grid_dec = 0, grid_rapply = 0;
  unsigned long long* flags = nullptr;
  long long flags_cap = 0;
  unsigned int* words = nullptr;  // [0] queue, [1] finished, [2] status, [3..4] minmax, [5] epoch, [6] helper ticket
  int grid_batch[6] = {0, 0, 0, 0, 0, 0};
  int ctas_override[6] = {0, 0, 0, 0, 0, 0};  // per op: resident CTAs per SM (0 = occupancy limit)
  int resolver[6] = {1, 1, 1, 1, 1, 1};        // per op: lookback resolver warp on (encoders)
  // Item tables of the batched launch: a ring of ITEM_SLOTS slots, each with
  // items_cap entries in pinned host staging and in device memory, and an
  // event recorded after the launch that read it.  A call waits only for the
  // launch ITEM_SLOTS calls back, so the host keeps running ahead of the GPU.
  static constexpr int ITEM_SLOTS = 8;
  BatchItem* d_items = nullptr;
  BatchItem* h_items = nullptr;
  int items_cap = 0;
  int items_slot = 0;
  cudaEvent_t items_done[ITEM_SLOTS] = {};
  unsigned int* h_range = nullptr;  // mapped pinned host words: the last NOA range
  unsigned long long timeout_ns = 2000000000ull;
};

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// A float array viewed as rows of 128 bytes, loaded/stored one chunk (128 rows)
// at a time with the 128-byte swizzle.
bool make_rows_map(CUtensorMap* m, const void* base, long long n_bytes) {
  memset(m, 0, sizeof(*m));
  const long long rows = n_bytes / 128;
  if (rows < 128) return false;
  auto fn = tmap_encoder();
  if (!fn) return false;
  cuuint64_t dims[2] = {32, (cuuint64_t)rows};
  cuuint64_t strides[1] = {128};
  cuuint32_t box[2] = {32, 128};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cortado_status from_cuda(cudaError_t e) { return e == cudaSuccess ? CORTADO_OK : (e == cudaErrorMemoryAllocation ? CORTADO_ERR_OOM : CORTADO_ERR_CUDA); }

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int64_t chunks_of(int64_t n) { return (n + CS - 1) / CS; }

cortado_status eb_exponent(float eb, int* e) {
  if (!(eb >= FLT_MIN)) return (eb != eb) ? CORTADO_ERR_EB_TOO_LARGE : CORTADO_ERR_EB_TOO_SMALL;
  uint32_t bits;
  memcpy(&bits, &eb, 4);
  const int be = (int)((bits >> 23) & 0xff);
  if (be + 24 >= 255) return CORTADO_ERR_EB_TOO_LARGE;
  *e = be;
  return CORTADO_OK;
}

cortado_status ensure_flags(cortado_ctx* ctx, int64_t chunks, cudaStream_t st) {
  if (chunks <= ctx->flags_cap) return CORTADO_OK;
  long long cap = 1024;
  while (cap < chunks) cap *= 2;
  if (ctx->flags) {
    cudaStreamSynchronize(st);
    cudaFree(ctx->flags);
    ctx->flags = nullptr;
    ctx->flags_cap = 0;
  }
  // lookback words, then the input payload offsets
  cudaError_t e = cudaMalloc(&ctx->flags, (size_t)cap * 16);
  if (e != cudaSuccess) return from_cuda(e);
  e = cudaMemsetAsync(ctx->flags, 0, (size_t)cap * 16, st);
  if (e != cudaSuccess) return from_cuda(e);
  ctx->flags_cap = cap;
  return CORTADO_OK;
}

// Batch item tables: ITEM_SLOTS tables of at least n_items entries each.
// Growing waits for every launch that reads a table.
cortado_status ensure_items(cortado_ctx* ctx, int n_items) {
  constexpr int SLOTS = cortado_ctx::ITEM_SLOTS;
  if (n_items <= ctx->items_cap) return CORTADO_OK;
  for (cudaEvent_t ev : ctx->items_done) cudaEventSynchronize(ev);  // every table is free
  cudaFree(ctx->d_items);
  cudaFreeHost(ctx->h_items);
  ctx->d_items = nullptr;
  ctx->h_items = nullptr;
  int cap = 64;
  while (cap < n_items) cap *= 2;
  cudaError_t e = cudaMalloc(&ctx->d_items, sizeof(BatchItem) * cap * SLOTS);
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_items, sizeof(BatchItem) * cap * SLOTS);
  if (e != cudaSuccess) {
    ctx->items_cap = 0;
    return from_cuda(e);
  }
  ctx->items_cap = cap;
  return CORTADO_OK;
}

Sync next_sync(cortado_ctx* ctx, cudaStream_t, int op = 0) {
  Sync s;
  s.flags = ctx->flags;
  s.offs = ctx->flags + ctx->flags_cap;
  s.flags_cap = ctx->flags_cap;
  s.counter = ctx->words;
  s.status = ctx->words + 2;
  s.epoch = ctx->words + 5;
  s.timeout_ns = ctx->timeout_ns;
  s.resolver = ctx->resolver[op];
  return s;
}

int grid_for(int per_sm_grid, int64_t chunks) {
  long long g = chunks < 1 ? 1 : chunks;
  return (int)(g < per_sm_grid ? g : per_sm_grid);
}

// Grid of an op: the tuned CTAs per SM if set (never above the occupancy
// limit, which `occupancy` holds as a whole-GPU CTA count), else the limit.
int tuned_grid(const cortado_ctx* ctx, int op, int occupancy) {
  const int o = ctx->ctas_override[op];
  if (o <= 0) return occupancy;
  const long long g = (long long)o * ctx->sms;
  return (int)(g < occupancy ? g : occupancy);
}

template <typename K>
int occupancy_grid(K kernel, size_t smem, int sms) {
  int per = 0;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, NT, smem);
  if (per < 1) per = 1;
  return per * sms;
}

constexpr size_t SMEM_STD = smem_bytes(2);  // every encode / decode kernel

cortado_status launch_status(cudaError_t e) { return from_cuda(e == cudaSuccess ? cudaGetLastError() : e); }

}  // namespace

extern "C" {

const char* cortado_status_string(cortado_status s) {
  switch (s) {
    case CORTADO_OK: return "ok";
    case CORTADO_ERR_EB_TOO_SMALL: return "error bound too small";
    case CORTADO_ERR_EB_TOO_LARGE: return "error bound too large";
    case CORTADO_ERR_CORRUPT_STREAM: return "corrupt stream";
    case CORTADO_ERR_SIZE_MISMATCH: return "size mismatch";
    case CORTADO_ERR_TIMEOUT: return "device wait timed out";
    case CORTADO_ERR_OOM: return "out of device memory";
    case CORTADO_ERR_INVALID_ARG: return "invalid argument";
    case CORTADO_ERR_CUDA: return "CUDA error";
    case CORTADO_ERR_ALIGNMENT: return "buffer not 16-byte aligned";
    case CORTADO_ERR_CAPACITY: return "output buffer too small";
    case CORTADO_ERR_SCRATCH_LIMIT: return "input larger than the fixed scratch of the no-allocation entry point";
  }
  return "unknown status";
}

int64_t cortado_max_stream_bytes(int64_t n_bytes) {
  if (n_bytes < 0) return -1;
  const int64_t c = chunks_of(n_bytes);
  return HDR + 2 * c + c * (int64_t)CS;
}

cortado_status cortado_eb_exponent(float eb, int* biased_exponent) {
  int e = 0;
  const cortado_status s = eb_exponent(eb, &e);
  if (s == CORTADO_OK && biased_exponent) *biased_exponent = e;
  return s;
}

cortado_status cortado_create(cortado_ctx** out, int device) {
  if (!out) return CORTADO_ERR_INVALID_ARG;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return from_cuda(e);
  cortado_ctx* ctx = new cortado_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  e = cudaMalloc(&ctx->words, 64);
  if (e != cudaSuccess) { delete ctx; return from_cuda(e); }
  cudaMemset(ctx->words, 0, 64);
  cudaMemset(ctx->words + 3, 0xff, 4);  // NOA range words: min = all ones, max = 0
  e = cudaHostAlloc((void**)&ctx->h_range, 8, cudaHostAllocMapped);
  if (e != cudaSuccess) { cudaFree(ctx->words); delete ctx; return from_cuda(e); }
  ctx->grid_store = occupancy_grid(k_store, SMEM_STD, ctx->sms);
  ctx->grid_reenc = occupancy_grid(k_reencode<OP_S2C, false>, SMEM_STD, ctx->sms);
  occupancy_grid(k_reencode<OP_RESI, false>, SMEM_STD, ctx->sms);
  occupancy_grid(k_reencode<OP_S2C, true>, SMEM_STD, ctx->sms);  // the fused forms
  occupancy_grid(k_reencode<OP_RESI, true>, SMEM_STD, ctx->sms);
  ctx->grid_dec = occupancy_grid(k_decode<OP_SDEC>, SMEM_STD, ctx->sms);
  occupancy_grid(k_decode<OP_CDEC>, SMEM_STD, ctx->sms);
  ctx->grid_rapply = occupancy_grid(k_decode<OP_RAPPLY>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_STORE] = occupancy_grid(k_batch<OP_STORE>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_S2C] = occupancy_grid(k_batch<OP_S2C>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_RESI] = occupancy_grid(k_batch<OP_RESI>, SMEM_STD, ctx->sms);
  occupancy_grid(k_batch<OP_S2C, true>, SMEM_STD, ctx->sms);  // the fused forms: same shape, attributes set
  occupancy_grid(k_batch<OP_RESI, true>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_SDEC] = occupancy_grid(k_batch<OP_SDEC>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_CDEC] = occupancy_grid(k_batch<OP_CDEC>, SMEM_STD, ctx->sms);
  ctx->grid_batch[OP_RAPPLY] = occupancy_grid(k_batch<OP_RAPPLY>, SMEM_STD, ctx->sms);
  for (cudaEvent_t& ev : ctx->items_done) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cortado_status s = ensure_flags(ctx, 1024, 0);
  cudaDeviceSynchronize();
  if (s != CORTADO_OK) { cortado_destroy(ctx); return s; }
  *out = ctx;
  return from_cuda(cudaGetLastError());
}

void cortado_destroy(cortado_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  cudaFree(ctx->flags);
  cudaFree(ctx->words);
  cudaFree(ctx->d_items);
  cudaFreeHost(ctx->h_items);
  cudaFreeHost(ctx->h_range);
  for (cudaEvent_t ev : ctx->items_done)
    if (ev) cudaEventDestroy(ev);
  delete ctx;
}

cortado_status cortado_set_timeout(cortado_ctx* ctx, uint64_t timeout_ns) {
  if (!ctx || timeout_ns == 0) return CORTADO_ERR_INVALID_ARG;
  ctx->timeout_ns = timeout_ns;
  return CORTADO_OK;
}

cortado_status cortado_reserve(cortado_ctx* ctx, int64_t chunks, int items) {
  if (!ctx || chunks < 0 || items < 0) return CORTADO_ERR_INVALID_ARG;
  cortado_status s = ensure_flags(ctx, chunks, 0);
  if (s) return s;
  if ((s = ensure_items(ctx, items))) return s;
  return from_cuda(cudaStreamSynchronize(0));
}

cortado_status cortado_set_launch_ctas(cortado_ctx* ctx, cortado_op op, int ctas_per_sm) {
  if (!ctx || op < CORTADO_OP_STORE || op > CORTADO_OP_RESI_RECV || ctas_per_sm < 0 || ctas_per_sm > 64)
    return CORTADO_ERR_INVALID_ARG;
  ctx->ctas_override[op] = ctas_per_sm;
  return CORTADO_OK;
}

cortado_status cortado_set_resolver(cortado_ctx* ctx, cortado_op op, int enabled) {
  if (!ctx || op < CORTADO_OP_STORE || op > CORTADO_OP_RESI_RECV) return CORTADO_ERR_INVALID_ARG;
  ctx->resolver[op] = enabled ? 1 : 0;
  return CORTADO_OK;
}

cortado_status cortado_selftest_timeout(cortado_ctx* ctx, cortado_stream_t stream) {
  if (!ctx) return CORTADO_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const Sync sy = next_sync(ctx, st);  // offs holds at least 1024 words from creation
  k_wait_selftest<<<1, 32, 0, st>>>(sy);
  return from_cuda(cudaGetLastError());
}

cortado_status cortado_sync(cortado_ctx* ctx, cortado_stream_t stream) {
  if (!ctx) return CORTADO_ERR_INVALID_ARG;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return from_cuda(e);
  unsigned int st = 0;
  e = cudaMemcpy(&st, ctx->words + 2, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return from_cuda(e);
  if (st) cudaMemset(ctx->words + 2, 0, 4);
  return (cortado_status)st;
}

cortado_status cortado_store_encode(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float eb_abs, void* d_out,
                                    int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream) {
  if (!ctx || (!d_in && n_bytes) || !d_out || !d_outsize || n_bytes < 0 || (n_bytes & 3)) return CORTADO_ERR_INVALID_ARG;
  if (!aligned16(d_in) || !aligned16(d_out)) return CORTADO_ERR_ALIGNMENT;
  if (out_capacity < cortado_max_stream_bytes(n_bytes)) return CORTADO_ERR_CAPACITY;
  int e = 0;
  cortado_status s = eb_exponent(eb_abs / 2, &e);  // stored bins use half the bound
  if (s) return s;
  const int64_t chunks = chunks_of(n_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  if ((s = ensure_flags(ctx, chunks, st))) return s;
  OpArgs a{};
  a.in = (const uint8_t*)d_in;
  a.in_bytes = n_bytes;
  a.out = (uint8_t*)d_out;
  a.out_cap = out_capacity;
  a.out_size = (long long*)d_outsize;
  a.n = n_bytes;
  a.q1 = make_quant(e);
  a.sy = next_sync(ctx, st, OP_STORE);
  CUtensorMap map;
  a.has_map_in = make_rows_map(&map, d_in, n_bytes);
  k_store<<<grid_for(tuned_grid(ctx, OP_STORE, ctx->grid_store), chunks), NT, SMEM_STD, st>>>(a, map);
  return launch_status(cudaSuccess);
}

static cortado_status reencode(cortado_ctx* ctx, int op, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                               float eb1, float eb2, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                               cortado_stream_t stream, void* d_client = nullptr, const float* d_minmax = nullptr) {
  if (!ctx || !d_stored || !d_out || !d_outsize || n_bytes < 0 || (n_bytes & 3) || stored_bytes < HDR)
    return CORTADO_ERR_INVALID_ARG;
  if (!aligned16(d_stored) || !aligned16(d_out) || (d_client && !aligned16(d_client))) return CORTADO_ERR_ALIGNMENT;
  if (out_capacity < cortado_max_stream_bytes(n_bytes)) return CORTADO_ERR_CAPACITY;
  int e1 = 1, e2 = 1;
  cortado_status s = CORTADO_OK;
  if (!d_minmax) {  // NOA bounds are checked on the device
    if ((s = eb_exponent(eb1, &e1))) return s;
    if (op == OP_RESI && (s = eb_exponent(eb2, &e2))) return s;
  }
  const int64_t chunks = chunks_of(n_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  if ((s = ensure_flags(ctx, chunks, st))) return s;
  OpArgs a{};
  if (d_minmax) {
    a.noa = d_minmax;
    a.noa_eb1 = eb1;
    a.noa_eb2 = eb2;
    a.noa_mode = (op == OP_S2C) ? 2 : 3;
  }
  a.in = (const uint8_t*)d_stored;
  a.in_bytes = stored_bytes;
  a.out = (uint8_t*)d_out;
  a.out_cap = out_capacity;
  a.out_size = (long long*)d_outsize;
  a.n = n_bytes;
  a.q1 = make_quant(e1);
  a.q2 = make_quant(e2);
  a.client = (uint8_t*)d_client;
  a.sy = next_sync(ctx, st, op);
  const int grid = grid_for(tuned_grid(ctx, op, ctx->grid_reenc), chunks);
  if (op == OP_S2C && d_client) k_reencode<OP_S2C, true><<<grid, NT, SMEM_STD, st>>>(a);
  else if (op == OP_S2C) k_reencode<OP_S2C, false><<<grid, NT, SMEM_STD, st>>>(a);
  else if (d_client) k_reencode<OP_RESI, true><<<grid, NT, SMEM_STD, st>>>(a);
  else k_reencode<OP_RESI, false><<<grid, NT, SMEM_STD, st>>>(a);
  return launch_status(cudaSuccess);
}

cortado_status cortado_init_send(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                 float request_eb_abs, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                 cortado_stream_t stream) {
  return reencode(ctx, OP_S2C, d_stored, stored_bytes, n_bytes, request_eb_abs, 0.0f, d_out, out_capacity, d_outsize, stream);
}

cortado_status cortado_resi_send(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                 float src_eb_abs, float dst_eb_abs, void* d_out, int64_t out_capacity,
                                 int64_t* d_outsize, cortado_stream_t stream) {
  return reencode(ctx, OP_RESI, d_stored, stored_bytes, n_bytes, src_eb_abs, dst_eb_abs, d_out, out_capacity, d_outsize,
                  stream);
}

cortado_status cortado_init_send_apply(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                       float request_eb_abs, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                       void* d_client, cortado_stream_t stream) {
  if (!d_client && n_bytes) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_S2C, d_stored, stored_bytes, n_bytes, request_eb_abs, 0.0f, d_out, out_capacity, d_outsize,
                  stream, d_client);
}

cortado_status cortado_resi_send_apply(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                       float src_eb_abs, float dst_eb_abs, void* d_out, int64_t out_capacity,
                                       int64_t* d_outsize, void* d_client, cortado_stream_t stream) {
  if (!d_client && n_bytes) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_RESI, d_stored, stored_bytes, n_bytes, src_eb_abs, dst_eb_abs, d_out, out_capacity, d_outsize,
                  stream, d_client);
}

cortado_status cortado_noa_range_device(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float* d_minmax,
                                        cortado_stream_t stream) {
  if (!ctx || !d_in || !d_minmax || n_bytes <= 0 || (n_bytes & 3)) return CORTADO_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const long long nw = n_bytes / 4;
  long long blocks = (nw / 4 + 1023) / 1024;
  if (blocks > 8L * ctx->sms) blocks = 8L * ctx->sms;
  if (blocks < 1) blocks = 1;
  k_minmax<<<(int)blocks, 256, 0, st>>>((const float*)d_in, nw, ctx->words + 3);
  k_range_to_device<<<1, 1, 0, st>>>(ctx->words + 3, d_minmax);
  return launch_status(cudaSuccess);
}

cortado_status cortado_store_encode_noa(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, const float* d_minmax,
                                        float eb_noa, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                        cortado_stream_t stream) {
  if (!ctx || (!d_in && n_bytes) || !d_out || !d_outsize || !d_minmax || n_bytes < 0 || (n_bytes & 3))
    return CORTADO_ERR_INVALID_ARG;
  if (!aligned16(d_in) || !aligned16(d_out)) return CORTADO_ERR_ALIGNMENT;
  if (out_capacity < cortado_max_stream_bytes(n_bytes)) return CORTADO_ERR_CAPACITY;
  const int64_t chunks = chunks_of(n_bytes);
  cudaStream_t st = (cudaStream_t)stream;
  cortado_status s = ensure_flags(ctx, chunks, st);
  if (s) return s;
  OpArgs a{};
  a.in = (const uint8_t*)d_in;
  a.in_bytes = n_bytes;
  a.out = (uint8_t*)d_out;
  a.out_cap = out_capacity;
  a.out_size = (long long*)d_outsize;
  a.n = n_bytes;
  a.q1 = make_quant(1);
  a.noa = d_minmax;
  a.noa_eb1 = eb_noa;
  a.noa_mode = 1;
  a.sy = next_sync(ctx, st, OP_STORE);
  CUtensorMap map;
  a.has_map_in = make_rows_map(&map, d_in, n_bytes);
  k_store<<<grid_for(tuned_grid(ctx, OP_STORE, ctx->grid_store), chunks), NT, SMEM_STD, st>>>(a, map);
  return launch_status(cudaSuccess);
}

cortado_status cortado_init_send_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                     const float* d_minmax, float request_eb_noa, void* d_out, int64_t out_capacity,
                                     int64_t* d_outsize, cortado_stream_t stream) {
  if (!d_minmax) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_S2C, d_stored, stored_bytes, n_bytes, request_eb_noa, 0.0f, d_out, out_capacity, d_outsize,
                  stream, nullptr, d_minmax);
}

cortado_status cortado_resi_send_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                     const float* d_minmax, float src_eb_noa, float dst_eb_noa, void* d_out,
                                     int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream) {
  if (!d_minmax) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_RESI, d_stored, stored_bytes, n_bytes, src_eb_noa, dst_eb_noa, d_out, out_capacity,
                  d_outsize, stream, nullptr, d_minmax);
}

cortado_status cortado_init_send_apply_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                           const float* d_minmax, float request_eb_noa, void* d_out,
                                           int64_t out_capacity, int64_t* d_outsize, void* d_client,
                                           cortado_stream_t stream) {
  if (!d_minmax || (!d_client && n_bytes)) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_S2C, d_stored, stored_bytes, n_bytes, request_eb_noa, 0.0f, d_out, out_capacity, d_outsize,
                  stream, d_client, d_minmax);
}

cortado_status cortado_resi_send_apply_noa(cortado_ctx* ctx, const void* d_stored, int64_t stored_bytes, int64_t n_bytes,
                                           const float* d_minmax, float src_eb_noa, float dst_eb_noa, void* d_out,
                                           int64_t out_capacity, int64_t* d_outsize, void* d_client,
                                           cortado_stream_t stream) {
  if (!d_minmax || (!d_client && n_bytes)) return CORTADO_ERR_INVALID_ARG;
  return reencode(ctx, OP_RESI, d_stored, stored_bytes, n_bytes, src_eb_noa, dst_eb_noa, d_out, out_capacity,
                  d_outsize, stream, d_client, d_minmax);
}

static cortado_status decode(cortado_ctx* ctx, int op, const void* d_stream, int64_t stream_bytes, const void* d_src,
                             int64_t n_bytes, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                             cortado_stream_t stream) {
  if (!ctx || !d_stream || !d_out || !d_outsize || stream_bytes < HDR || out_capacity < 0) return CORTADO_ERR_INVALID_ARG;
  if (!aligned16(d_stream) || !aligned16(d_out) || (d_src && !aligned16(d_src))) return CORTADO_ERR_ALIGNMENT;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t chunk_bound = chunks_of(op == OP_RAPPLY ? n_bytes : out_capacity);
  cortado_status es = ensure_flags(ctx, chunk_bound, st);
  if (es) return es;
  OpArgs a{};
  a.in = (const uint8_t*)d_stream;
  a.in_bytes = stream_bytes;
  a.src = (const uint8_t*)d_src;
  a.out = (uint8_t*)d_out;
  a.out_cap = out_capacity;
  a.out_size = (long long*)d_outsize;
  a.n = n_bytes;
  a.sy = next_sync(ctx, st, op);
  CUtensorMap msrc, mout;
  memset(&msrc, 0, sizeof(msrc));
  // The output map needs the decoded size, which only the stream header holds:
  // cover the whole output capacity (TMA is only used for full chunks, which
  // the kernel checks lie inside the header's size).
  a.has_map_out = make_rows_map(&mout, d_out, op == OP_RAPPLY ? n_bytes : out_capacity);
  if (op == OP_RAPPLY) a.has_map_in = make_rows_map(&msrc, d_src, n_bytes);
  if (op == OP_SDEC) k_decode<OP_SDEC><<<grid_for(tuned_grid(ctx, op, ctx->grid_dec), chunk_bound), NT, SMEM_STD, st>>>(a, msrc, mout);
  else if (op == OP_CDEC) k_decode<OP_CDEC><<<grid_for(tuned_grid(ctx, op, ctx->grid_dec), chunk_bound), NT, SMEM_STD, st>>>(a, msrc, mout);
  else k_decode<OP_RAPPLY><<<grid_for(tuned_grid(ctx, op, ctx->grid_rapply), chunk_bound), NT, SMEM_STD, st>>>(a, msrc, mout);
  return launch_status(cudaSuccess);
}

cortado_status cortado_store_decode(cortado_ctx* ctx, const void* d_stream, int64_t stream_bytes, void* d_out,
                                    int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream) {
  return decode(ctx, OP_SDEC, d_stream, stream_bytes, nullptr, 0, d_out, out_capacity, d_outsize, stream);
}

cortado_status cortado_init_recv(cortado_ctx* ctx, const void* d_init, int64_t init_bytes, void* d_out,
                                 int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream) {
  return decode(ctx, OP_CDEC, d_init, init_bytes, nullptr, 0, d_out, out_capacity, d_outsize, stream);
}

cortado_status cortado_resi_recv(cortado_ctx* ctx, const void* d_src, int64_t n_bytes, const void* d_resi,
                                 int64_t resi_bytes, void* d_out, int64_t out_capacity, int64_t* d_outsize,
                                 cortado_stream_t stream) {
  if (!d_src && n_bytes) return CORTADO_ERR_INVALID_ARG;
  if (n_bytes < 0 || (n_bytes & 3) || out_capacity < n_bytes) return n_bytes < 0 || (n_bytes & 3) ? CORTADO_ERR_INVALID_ARG : CORTADO_ERR_CAPACITY;
  return decode(ctx, OP_RAPPLY, d_resi, resi_bytes, d_src, n_bytes, d_out, out_capacity, d_outsize, stream);
}

cortado_status cortado_verify_bound(cortado_ctx* ctx, const void* d_orig, const void* d_recon, int64_t n_bytes,
                                    float eb_abs, unsigned long long* d_first_bad, cortado_stream_t stream) {
  if (!ctx || !d_orig || !d_recon || !d_first_bad || n_bytes < 0 || (n_bytes & 3) || !(eb_abs > 0))
    return CORTADO_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const long long nw = n_bytes / 4;
  cudaError_t e = cudaMemsetAsync(d_first_bad, 0xff, 8, st);
  if (e != cudaSuccess) return from_cuda(e);
  long long blocks = (nw + 255) / 256;
  if (blocks > 8L * ctx->sms) blocks = 8L * ctx->sms;
  if (blocks < 1) blocks = 1;
  k_verify<<<(int)blocks, 256, 0, st>>>((const float*)d_orig, (const float*)d_recon, nw, eb_abs, d_first_bad);
  return launch_status(cudaSuccess);
}

cortado_status cortado_noa_range(cortado_ctx* ctx, const void* d_in, int64_t n_bytes, float* h_min, float* h_max,
                                 cortado_stream_t stream) {
  if (!ctx || !d_in || !h_min || !h_max || n_bytes <= 0 || (n_bytes & 3)) return CORTADO_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const long long nw = n_bytes / 4;
  long long blocks = (nw / 4 + 1023) / 1024;
  if (blocks > 8L * ctx->sms) blocks = 8L * ctx->sms;
  if (blocks < 1) blocks = 1;
  k_minmax<<<(int)blocks, 256, 0, st>>>((const float*)d_in, nw, ctx->words + 3);
  k_range_publish<<<1, 1, 0, st>>>(ctx->words + 3, ctx->h_range);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return from_cuda(e);
  const unsigned int r[2] = {((volatile unsigned int*)ctx->h_range)[0], ((volatile unsigned int*)ctx->h_range)[1]};
  auto unord = [](unsigned int o) -> float {
    const unsigned int u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    float f;
    memcpy(&f, &u, 4);
    return f;
  };
  *h_min = unord(r[0]);
  *h_max = unord(r[1]);
  return CORTADO_OK;
}

cortado_status cortado_batch(cortado_ctx* ctx, cortado_op op, const cortado_item* items, int n_items,
                             cortado_stream_t stream) {
  if (!ctx || !items || n_items <= 0 || op < CORTADO_OP_STORE || op > CORTADO_OP_RESI_SEND_APPLY) return CORTADO_ERR_INVALID_ARG;
  // the fused send-and-apply forms run the re-encoders with the client's floats
  const bool apply = op == CORTADO_OP_INIT_SEND_APPLY || op == CORTADO_OP_RESI_SEND_APPLY;
  if (apply) op = (op == CORTADO_OP_INIT_SEND_APPLY) ? CORTADO_OP_INIT_SEND : CORTADO_OP_RESI_SEND;
  static_assert((int)CORTADO_OP_STORE == OP_STORE && (int)CORTADO_OP_INIT_SEND == OP_S2C &&
                    (int)CORTADO_OP_RESI_SEND == OP_RESI && (int)CORTADO_OP_STORE_DECODE == OP_SDEC &&
                    (int)CORTADO_OP_INIT_RECV == OP_CDEC && (int)CORTADO_OP_RESI_RECV == OP_RAPPLY,
                "op numbering");
  cudaStream_t st = (cudaStream_t)stream;
  // per-item checks, as the single-stream entry points make them
  long long total = 0;
  for (int i = 0; i < n_items; i++) {
    const cortado_item& it = items[i];
    if (!it.d_in || !it.d_out || !it.d_outsize || it.n_bytes <= 0 || (it.n_bytes & 3)) return CORTADO_ERR_INVALID_ARG;
    if (!aligned16(it.d_in) || !aligned16(it.d_out) || (it.d_src && !aligned16(it.d_src))) return CORTADO_ERR_ALIGNMENT;
    int e = 0;
    cortado_status s;
    switch (op) {
      case CORTADO_OP_STORE:
        if (it.in_bytes != it.n_bytes) return CORTADO_ERR_INVALID_ARG;
        if (it.out_capacity < cortado_max_stream_bytes(it.n_bytes)) return CORTADO_ERR_CAPACITY;
        if ((s = eb_exponent(it.eb1 / 2, &e))) return s;
        break;
      case CORTADO_OP_INIT_SEND:
      case CORTADO_OP_RESI_SEND:
        if (it.in_bytes < HDR || (apply && !it.d_src)) return CORTADO_ERR_INVALID_ARG;
        if (it.out_capacity < cortado_max_stream_bytes(it.n_bytes)) return CORTADO_ERR_CAPACITY;
        if ((s = eb_exponent(it.eb1, &e))) return s;
        if (op == CORTADO_OP_RESI_SEND && (s = eb_exponent(it.eb2, &e))) return s;
        break;
      case CORTADO_OP_RESI_RECV:
        if (!it.d_src) return CORTADO_ERR_INVALID_ARG;
        // fall through
      default:
        if (it.in_bytes < HDR) return CORTADO_ERR_INVALID_ARG;
        if (it.out_capacity < it.n_bytes) return CORTADO_ERR_CAPACITY;
        break;
    }
    total += chunks_of(it.n_bytes);
  }
  cortado_status s = ensure_flags(ctx, total, st);
  if (s) return s;
  constexpr int SLOTS = cortado_ctx::ITEM_SLOTS;
  if ((s = ensure_items(ctx, n_items))) return s;
  const int slot = ctx->items_slot;
  ctx->items_slot = (slot + 1) % SLOTS;
  cudaEventSynchronize(ctx->items_done[slot]);  // the launch that last read this slot has ended
  BatchItem* h_tab = ctx->h_items + (size_t)slot * ctx->items_cap;
  BatchItem* d_tab = ctx->d_items + (size_t)slot * ctx->items_cap;
  const Sync sy = next_sync(ctx, st, op);
  long long base = 0;
  for (int i = 0; i < n_items; i++) {
    const cortado_item& it = items[i];
    BatchItem& b = h_tab[i];
    memset(&b, 0, sizeof(b));
    OpArgs& a = b.a;
    a.in = (const uint8_t*)it.d_in;
    a.in_bytes = it.in_bytes;
    a.src = (const uint8_t*)it.d_src;
    a.out = (uint8_t*)it.d_out;
    a.out_cap = it.out_capacity;
    a.out_size = (long long*)it.d_outsize;
    a.n = it.n_bytes;
    int e1 = 1, e2 = 1;
    eb_exponent(op == CORTADO_OP_STORE ? it.eb1 / 2 : it.eb1, &e1);
    eb_exponent(it.eb2, &e2);
    a.q1 = make_quant(e1);
    a.q2 = make_quant(e2);
    a.client = apply ? (uint8_t*)it.d_src : nullptr;
    a.sy = sy;
    a.sy.flags = sy.flags + base;
    a.sy.offs = sy.offs + base;
    if (op == CORTADO_OP_STORE) a.has_map_in = make_rows_map(&b.map_in, it.d_in, it.n_bytes);
    if (op == CORTADO_OP_RESI_RECV) a.has_map_in = make_rows_map(&b.map_in, it.d_src, it.n_bytes);
    if (op == CORTADO_OP_STORE_DECODE || op == CORTADO_OP_INIT_RECV || op == CORTADO_OP_RESI_RECV)
      a.has_map_out = make_rows_map(&b.map_out, it.d_out, it.n_bytes);
    b.chunk_base = base;
    b.chunks = chunks_of(it.n_bytes);
    base += b.chunks;
  }
  cudaError_t e = cudaMemcpyAsync(d_tab, h_tab, sizeof(BatchItem) * n_items, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return from_cuda(e);
  const int grid = grid_for(tuned_grid(ctx, op, ctx->grid_batch[op]), total);
  const size_t smem = (op == CORTADO_OP_RESI_RECV) ? SMEM_STD : SMEM_STD;
  switch (op) {
    case CORTADO_OP_STORE: k_batch<OP_STORE><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy); break;
    case CORTADO_OP_INIT_SEND:
      if (apply) k_batch<OP_S2C, true><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy);
      else k_batch<OP_S2C><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy);
      break;
    case CORTADO_OP_RESI_SEND:
      if (apply) k_batch<OP_RESI, true><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy);
      else k_batch<OP_RESI><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy);
      break;
    case CORTADO_OP_STORE_DECODE: k_batch<OP_SDEC><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy); break;
    case CORTADO_OP_INIT_RECV: k_batch<OP_CDEC><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy); break;
    case CORTADO_OP_RESI_RECV: k_batch<OP_RAPPLY><<<grid, NT, smem, st>>>(d_tab, n_items, total, sy); break;
  }
  cudaEventRecord(ctx->items_done[slot], st);
  return launch_status(cudaSuccess);
}

// Per-device set-up of the no-allocation entry point: the device address of
// g_noalloc_scratch and the persistent grid size, valid for the CUDA context
// that was current when they were looked up (a device reset or a new primary
// context gets a new address, so a change of context repeats the set-up).
struct NoallocDev {
  bool ready = false;
  CUcontext ctx = nullptr;
  unsigned long long* scratch = nullptr;
  int grid = 0;
};

// The calling thread's current CUDA context (driver entry point, as for the
// tensor-map encoder), or null when it cannot be queried.
static CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Fn>(p);
  });
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}
static NoallocDev g_noalloc_dev[64];
static std::mutex g_noalloc_mu;

cortado_status cortado_store_encode_noalloc(const void* d_in, int64_t n_bytes, float eb_abs, void* d_out,
                                            int64_t out_capacity, int64_t* d_outsize, cortado_stream_t stream) {
  if ((!d_in && n_bytes) || !d_out || !d_outsize || n_bytes < 0 || (n_bytes & 3)) return CORTADO_ERR_INVALID_ARG;
  if (n_bytes > CORTADO_NOALLOC_MAX_BYTES) return CORTADO_ERR_SCRATCH_LIMIT;
  if (!aligned16(d_in) || !aligned16(d_out)) return CORTADO_ERR_ALIGNMENT;
  if (out_capacity < cortado_max_stream_bytes(n_bytes)) return CORTADO_ERR_CAPACITY;
  int e = 0;
  cortado_status s = eb_exponent(eb_abs / 2, &e);
  if (s) return s;
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return from_cuda(ce);
  if (dev < 0 || dev >= 64) return CORTADO_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  NoallocDev& d = g_noalloc_dev[dev];
  const CUcontext cur = current_context();
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!d.ready || d.ctx != cur) {
      // device `dev` is current here
      void* p = nullptr;
      ce = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (ce != cudaSuccess) return from_cuda(ce);
      int sms = 0;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      d.grid = occupancy_grid(k_store_noalloc, SMEM_STD, sms);
      d.scratch = (unsigned long long*)p;
      d.ctx = cur;
      d.ready = true;
    }
  }
  OpArgs a{};
  a.in = (const uint8_t*)d_in;
  a.in_bytes = n_bytes;
  a.out = (uint8_t*)d_out;
  a.out_cap = out_capacity;
  a.out_size = (long long*)d_outsize;
  a.n = n_bytes;
  a.q1 = make_quant(e);
  a.sy.flags = d.scratch;
  a.sy.offs = nullptr;
  a.sy.flags_cap = NOALLOC_CHUNKS;
  a.sy.counter = reinterpret_cast<unsigned int*>(d.scratch + NOALLOC_CHUNKS);
  a.sy.status = a.sy.counter + 2;
  a.sy.epoch = a.sy.counter + 3;
  a.sy.timeout_ns = 2000000000ull;
  a.sy.resolver = 1;
  CUtensorMap map;
  a.has_map_in = make_rows_map(&map, d_in, n_bytes);
  k_store_noalloc<<<grid_for(d.grid, chunks_of(n_bytes)), NT, SMEM_STD, st>>>(a, map);
  return launch_status(cudaSuccess);
}

}  // extern "C"

