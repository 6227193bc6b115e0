// The fused per-chunk encode and decode stages and the shared-memory layout
// of the pipelined kernels built from them.  Reference counterparts:
//   store encode   include/d_server_encode.h:51-143
//   storage decode include/d_server_encode.h:174-260
//   init_send      include/d_s2c.h:51-200
//   init_recv      include/d_client_encode.h:173-259
//   resi_send      include/d_residual_encode.h:51-201
//   resi_recv      include/d_residual_encode.h:238-347
// Differences in mechanism (not in output bytes): output offsets from a
// bounded, epoch-tagged decoupled lookback, resolved one chunk later
// (encoders), and input offsets from a prefix sum of the size table computed
// once per launch (decoders, re-encoders); one 128-thread CTA per chunk with
// the data held in registers; TMA for float chunks and compressed payloads;
// errors latched in a status word instead of printf + __trap.
#pragma once
#include "device.cuh"

namespace cortado {

enum Op : int { OP_STORE = 0, OP_S2C = 1, OP_RESI = 2, OP_SDEC = 3, OP_CDEC = 4, OP_RAPPLY = 5 };

struct OpArgs {
  const uint8_t* in;        // store: floats; others: input stream
  long long in_bytes;       // store: N; others: valid bytes of the input stream
  const uint8_t* src;       // resi_recv: client floats
  uint8_t* out;             // output stream or floats
  long long out_cap;
  long long* out_size;      // device
  long long n;              // original bytes (host-known for encoders; 0 = read header)
  Quant q1, q2;             // store: server; init_send: request; resi_send: src, dst
  Sync sy;
  int has_map_in, has_map_out;
  uint8_t* client;          // init_send / resi_send with apply: the client's reconstruction (floats), or null
  // NOA bounds resolved on the device (cortado_*_noa): q1/q2 come from
  // noa_eb1/noa_eb2 times the range max - min of noa[0..1] (device floats)
  const float* noa;
  float noa_eb1, noa_eb2;
  int noa_mode;             // 0: q1/q2 as given; 1: store (half of eb1); 2: init (eb1); 3: residual (eb1, eb2)
};

// The NOA bounds of the drivers (src/cortado_store.cu:222-227,
// src/cortado_init.cu:294-296, src/cortado_resi.cu:329-332), evaluated on the
// device: eb_abs = float(max - min) * eb, each step rounded once, the store's
// bins at eb_abs / 2, then the checks and biased exponent of the host-side
// eb_exponent.  Returns 0 or the status to latch.
__device__ __forceinline__ unsigned int noa_exponent(float eb, int* e) {
  if (!(eb >= 1.17549435e-38f)) return (eb != eb) ? DST_EB_TOO_LARGE : DST_EB_TOO_SMALL;  // FLT_MIN
  const int be = (int)((__float_as_uint(eb) >> 23) & 0xffu);
  if (be + 24 >= 255) return DST_EB_TOO_LARGE;
  *e = be;
  return 0;
}
__device__ __forceinline__ unsigned int resolve_noa(const OpArgs& a, Quant& q1, Quant& q2) {
  q1 = a.q1;
  q2 = a.q2;
  if (!a.noa_mode) return 0;
  const float range = __fsub_rn(a.noa[1], a.noa[0]);
  float eb1 = __fmul_rn(range, a.noa_eb1);
  if (a.noa_mode == 1) eb1 = __fdiv_rn(eb1, 2.0f);  // stored bins use half the bound
  int e1 = 1, e2 = 1;
  unsigned int st = noa_exponent(eb1, &e1);
  if (!st && a.noa_mode == 3) st = noa_exponent(__fmul_rn(range, a.noa_eb2), &e2);
  if (st) return st;
  q1 = make_quant(e1);
  if (a.noa_mode == 3) q2 = make_quant(e2);
  return 0;
}

// ---------------------------------------------------------------- shared memory
// A CTA owns a 1 KiB control block followed by two chunk buffers of
// BUF_WORDS words (16 KiB + slack, a multiple of 1024 bytes so that every
// buffer keeps the 1024-byte alignment TMA's 128B swizzle needs).  How the
// loops use them is described at each loop (cortado.cu).
constexpr int BUF_WORDS = 4352;
constexpr int CTL_BYTES = 1024;

// What the prefetch of one queue entry found (written by warp 3, read by all
// threads in the iteration that processes it).
struct StageMeta {
  long long g;              // queue index (>= the queue length: no chunk)
  long long c;              // chunk within its stream
  long long n;              // stream's original bytes
  long long chunks;         // stream's chunks
  unsigned long long off;   // decoders: payload offset in the stream's data section
  int item;                 // batched launches: the stream
  int nw;                   // words in the chunk
  int tma;                  // the stage's loads complete on its mbarrier
  int bad;                  // 1: corrupt size entry; 2: unusable stream header
  int csize;                // decoders: payload bytes
  int d;                    // decoders: payload's byte offset in the stage buffer
  int tma_len;              // decoders: bytes brought by the bulk copy
  int eb_e;                 // decoders: the stream's exponent
};

// The chunk whose payload waits in a staging buffer for its output offset
// (written by thread 0 at the end of encode_stage, flushed one iteration later).
struct Pend {
  long long c;
  int item;
  int nw;
  int csize;
  int raw;
  int valid;
};

struct __align__(16) Ctl {
  uint16_t l2[NT];          // level-2 bitmap (2 bytes per segment thread)
  uint16_t rb[NT];          // decoder: RE1 rank base per segment thread
  uint32_t scan_a[4], scan_b[4], scan_c[4], xchg[4];
  uint64_t bar[2];          // per stage: its TMA loads
  uint64_t bar_src;         // resi_recv: the client chunk
  StageMeta st[2];
  Pend pend[2];             // encoders: the chunk of each stage, until it is flushed
  unsigned long long payload_off;
  unsigned int epoch, is_last;
  unsigned int src_side;    // resi_recv: this chunk's client floats are behind the next payload
  uint32_t info[8];
};
static_assert(sizeof(Ctl) <= CTL_BYTES, "control block");

__host__ __device__ constexpr size_t smem_bytes(int nbuf) { return CTL_BYTES + (size_t)nbuf * BUF_WORDS * 4 + 1024; }

__device__ __forceinline__ uint32_t* stage_buf(Ctl& sm, int k) {
  return reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(&sm) + CTL_BYTES + k * (BUF_WORDS * 4));
}

struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

// Writes `csize` payload bytes to global memory at dst (any alignment) with
// 16-byte stores for the aligned interior.  word(q) returns payload word q
// (bytes 4q..4q+3, little-endian).
template <typename WordFn>
__device__ __forceinline__ void store_payload(uint8_t* dst, int csize, WordFn word) {
  const int tid = threadIdx.x;
  const uintptr_t A = reinterpret_cast<uintptr_t>(dst);
  const uintptr_t a0 = (A + 15) & ~uintptr_t(15);
  const uintptr_t a1 = (A + csize) & ~uintptr_t(15);
  auto byte_at = [&](int i) -> uint8_t { return (uint8_t)(word(i >> 2) >> (8 * (i & 3))); };
  if (a1 > a0) {
    const int head = (int)(a0 - A);
    const int nblk = (int)((a1 - a0) >> 4);
    const int r = head & 3;
    for (int b = tid; b < nblk; b += NT) {
      const int o = head + 16 * b;
      const int q = o >> 2;
      uint32_t w0 = word(q), w1 = word(q + 1), w2 = word(q + 2), w3 = word(q + 3);
      if (r) {
        const uint32_t w4 = word(q + 4);
        w0 = __funnelshift_r(w0, w1, 8 * r);
        w1 = __funnelshift_r(w1, w2, 8 * r);
        w2 = __funnelshift_r(w2, w3, 8 * r);
        w3 = __funnelshift_r(w3, w4, 8 * r);
      }
      *reinterpret_cast<uint4*>(a0 + 16 * (uintptr_t)b) = make_uint4(w0, w1, w2, w3);
    }
    if (tid < head) dst[tid] = byte_at(tid);
    const int tail = (int)(A + csize - a1);
    if (tid < tail) dst[(a1 - A) + tid] = byte_at((int)(a1 - A) + tid);
  } else {
    for (int i = tid; i < csize; i += NT) dst[i] = byte_at(i);
  }
}

// Physical plane-buffer word offsets of linear word s*128 + tid for even and
// odd s (full chunk): the swizzle term depends on s only through its parity,
// so the 32 plane words of a thread sit at base + 128*s + (s odd ? o : e).
__device__ __forceinline__ void plane_offsets(int tid, uint32_t& e, uint32_t& o) {
  const uint32_t lane = tid & 31, warp = tid >> 5;
  e = 32 * warp + ((((lane >> 2) & 7u) ^ warp) << 2) + (lane & 3);
  o = 32 * warp + ((((lane >> 2) & 7u) ^ (warp + 4)) << 2) + (lane & 3);
}

// ---------------------------------------------------------------- rotated walks
// Zero elimination moves each thread's bytes to a contiguous region that
// starts wherever the previous thread's ended.  For dense data those regions
// are about 128 bytes apart, so threads that walk their 32 words in the same
// order store to the same shared-memory bank (a 32-way conflict).  The
// compaction of a dense warp therefore walks each thread's words starting at
// word `lane`: nibble j of the rotated mask (rot_nibbles) belongs to word
// (lane + j) % 32, and nibble_prefix gives the byte count before the starting
// word.

// Bytes before word k of a segment: the set bits of the 4-bit-per-word mask
// M (128 bits) below nibble k.
__device__ __forceinline__ uint32_t nibble_prefix(const uint32_t (&M)[4], int k) {
  const int nb = 4 * k;
  uint32_t c = 0;
#pragma unroll
  for (int w = 0; w < 4; w++) {
    const int lim = nb - 32 * w;
    const uint32_t mask = lim >= 32 ? 0xffffffffu : (lim <= 0 ? 0u : (1u << lim) - 1u);
    c += __popc(M[w] & mask);
  }
  return c;
}

// The 128-bit mask M rotated right by 4*r bits.
__device__ __forceinline__ void rot_nibbles(const uint32_t (&M)[4], int r, uint32_t (&R)[4]) {
  uint32_t a0 = M[0], a1 = M[1], a2 = M[2], a3 = M[3];
  if (r & 8) {
    const uint32_t t = a0;
    a0 = a1; a1 = a2; a2 = a3; a3 = t;
  }
  if (r & 16) {
    uint32_t t = a0; a0 = a2; a2 = t;
    t = a1; a1 = a3; a3 = t;
  }
  const uint32_t bs = 4 * (r & 7);
  R[0] = __funnelshift_r(a0, a1, bs);
  R[1] = __funnelshift_r(a1, a2, bs);
  R[2] = __funnelshift_r(a2, a3, bs);
  R[3] = __funnelshift_r(a3, a0, bs);
}

// ============================================================== encode stage
// Input: v[32] = the pre-DIFFMS words of group g = threadIdx.x (quantized bins
// or residuals; words at or beyond nw are 0).  `plane` is a swizzled 16 KiB
// buffer that may be overwritten once every thread has passed the first
// barrier; it becomes the plane buffer (d_DIFFMS_4 -> d_BIT_4 -> d_RZE_1, raw
// fallback).  The compacted payload goes to `staging` (linear bytes), which
// the caller may still be reading until after_publish() returns.  The chunk's
// size is published for the lookback; the payload is written out later by
// flush_chunk, once the size of every earlier chunk is known (a raw chunk's
// words are read back from wherever the caller keeps them).  The chunk is
// recorded in `pend`.  after_publish() runs on every thread once the size is
// published (it may hold barriers: the pipelined loops flush the previous
// chunk there, a whole iteration after that chunk's own publication).
// FULL: a whole 16 KiB chunk (nw == 4096), with compile-time addressing.
template <bool FULL, typename Hook>
__device__ __forceinline__ void encode_stage(Ctl& sm, const Sync& sy, uint32_t (&v)[32], uint32_t* plane,
                                             uint8_t* st, long long c, int nw_in, int item, Pend& pend,
                                             Hook after_publish) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nw = FULL ? CW : nw_in;
  const int osize = nw * 4;
  const int G = nw >> 5, rem = nw & 31;

  // DIFFMS (d_DIFFMS.h:44-66): word minus its predecessor, then zig-zag.
  if (lane == 31) sm.xchg[warp] = v[31];
  uint32_t vany = 0;
#pragma unroll
  for (int k = 0; k < 32; k++) vany |= v[k];
  const bool any_nz = __syncthreads_or(vany != 0);
  if (!any_nz) {
    // All words zero: DIFFMS, BIT_4 and zero elimination leave no byte, so
    // RZE_1 emits only its 2-byte trailer (the original chunk size).
    if (tid == 0) {
      lookback_publish(sy, sm.epoch, c, 2u);
      pend = Pend{c, item, nw, 2, 0, 1};
    }
    after_publish();
    if (tid == 0) {
      st[0] = (uint8_t)osize;
      st[1] = (uint8_t)(osize >> 8);
    }
    return;
  }
  uint32_t prev = __shfl_up_sync(0xffffffffu, v[31], 1);
  if (lane == 0) prev = warp ? sm.xchg[warp - 1] : 0u;
#pragma unroll
  for (int k = 0; k < 32; k++) {
    const uint32_t cur = v[k];
    const uint32_t d = cur - prev;
    prev = cur;
    v[k] = (d << 1) ^ (uint32_t)((int32_t)d >> 31);
  }
  if (!FULL && 32 * tid + 32 > nw) {
#pragma unroll
    for (int k = 0; k < 32; k++)
      if (32 * tid + k >= nw) v[k] = 0;
  }
  // BIT_4: full groups are transposed into the planes (plane s at linear
  // words s*G .. s*G+G-1); the trailing partial group is copied untransposed.
  if (FULL) {
    uint32_t any = 0;
#pragma unroll
    for (int k = 0; k < 32; k++) any |= v[k];
    if (any) transpose32(v);  // an all-zero group transposes to all-zero planes
    uint32_t pe, po;
    plane_offsets(tid, pe, po);
#pragma unroll
    for (int s = 0; s < 32; s++) plane[128 * s + ((s & 1) ? po : pe)] = v[s];
  } else if (tid < G) {
    transpose32(v);
#pragma unroll
    for (int s = 0; s < 32; s++) plane[swz(s * G + tid)] = v[s];
  } else if (tid == G && rem) {
#pragma unroll
    for (int k = 0; k < 32; k++)
      if (k < rem) plane[swz(32 * G + k)] = v[k];
  }
  __syncthreads();

  // Segment layout: thread t owns BIT-output words 32t..32t+31.
  uint32_t q[32];
  row_load(plane, tid, q);
  if (!FULL && 32 * tid + 32 > nw) {
#pragma unroll
    for (int k = 0; k < 32; k++)
      if (32 * tid + k >= nw) q[k] = 0;
  }
  // Zero-elimination bitmap (d_ZEencodebyteshort): bit i <-> byte i != 0.
  uint32_t M[4] = {0, 0, 0, 0};
  uint32_t qany = 0;
#pragma unroll
  for (int k = 0; k < 32; k++) qany |= q[k];
  if (qany) {
#pragma unroll
    for (int j = 0; j < 4; j++) {
      uint32_t m = 0;
#pragma unroll
      for (int i = 0; i < 8; i++) m |= nz_nibble(q[8 * j + i]) << (4 * i);
      M[j] = m;
    }
  }
  const uint32_t nz = __popc(M[0]) + __popc(M[1]) + __popc(M[2]) + __popc(M[3]);
  // Last bitmap byte of the previous segment (RE's predecessor of byte 0).
  uint32_t pb = 0;
  if (tid > 0) {
    const int w = 32 * tid - 2;
    const uint32_t x0 = (FULL || w < nw) ? plane[swz(w)] : 0u;
    const uint32_t x1 = (FULL || w + 1 < nw) ? plane[swz(w + 1)] : 0u;
    pb = nz_nibble(x0) | (nz_nibble(x1) << 4);
  }
  // Repetition elimination, level 1 (d_REencode4wordsperthread): keep bitmap
  // byte j iff it differs from byte j-1.
  uint32_t K = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const uint32_t sh = (M[j] << 8) | (j ? (M[j - 1] >> 24) : pb);
    K |= nz_nibble(M[j] ^ sh) << (4 * j);
  }
  const uint32_t c1 = __popc(K);
  sm.l2[tid] = (uint16_t)K;
  uint32_t tot;
  const uint32_t ex = block_scan_excl(nz | (c1 << 16), sm.scan_a, tot);
  const uint32_t NZ = tot & 0xffffu, C1 = tot >> 16;
  const uint32_t zoff = ex & 0xffffu, c1off = ex >> 16;
  // (barrier inside the scan: the plane buffer is now free -> staging)

  // Levels 2 and 3 and the top bitmap (d_REencode1wordperthread) from the
  // 256-byte level-2 bitmap; every warp derives the chunk size, so no barrier
  // is needed before the compaction; warp 0 writes the bytes.
  const uint2 b2 = reinterpret_cast<const uint2*>(sm.l2)[lane];
  const uint32_t pprev = __shfl_up_sync(0xffffffffu, b2.y >> 24, 1);
  const uint32_t p0 = lane ? pprev : 0u;
  const uint32_t k2 = nz_nibble(b2.x ^ ((b2.x << 8) | p0)) | (nz_nibble(b2.y ^ ((b2.y << 8) | (b2.x >> 24))) << 4);
  uint32_t C2;
  const uint32_t off2 = warp_scan_excl(__popc(k2), C2);
  const uint32_t p3 = __shfl_up_sync(0xffffffffu, k2, 1);
  const bool keep3 = k2 != (lane ? p3 : 0u);
  const uint32_t top = __ballot_sync(0xffffffffu, keep3);
  const uint32_t C3 = __popc(top);
  const uint32_t off3 = __popc(top & ((1u << lane) - 1u));
  const uint32_t T = NZ + C1 + C2 + C3;
  unsigned int csize = (NZ == 0) ? 2u : T + 6u;
  const bool raw = csize >= (unsigned)osize;
  if (raw) csize = osize;
  if (tid == 0) {
    lookback_publish(sy, sm.epoch, c, csize);
    pend = Pend{c, item, nw, (int)csize, (int)raw, 1};
  }
  after_publish();
  if (raw) return;
  if (warp == 0) {
    if (NZ == 0) {
      if (lane == 0) {
        st[0] = (uint8_t)osize;
        st[1] = (uint8_t)(osize >> 8);
      }
    } else {
      uint32_t p = NZ + C1 + off2;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if ((k2 >> j) & 1) st[p++] = (uint8_t)((j < 4 ? b2.x : b2.y) >> (8 * (j & 3)));
      if (keep3) st[NZ + C1 + C2 + off3] = (uint8_t)k2;
      if (lane < 4) st[T + lane] = (uint8_t)(top >> (8 * lane));
      if (lane == 4) st[T + 4] = (uint8_t)osize;
      if (lane == 5) st[T + 5] = (uint8_t)(osize >> 8);
    }
  }
  // Compaction of the zero-eliminated bytes and the kept level-1 bitmap bytes.
  // When many lanes of the warp hold data, the words are read back from the
  // plane buffer in the lane-rotated order (conflict-free stores); otherwise
  // they come from registers in order.
  const bool dense = __popc(__ballot_sync(0xffffffffu, nz > 16)) >= 2;
  if (nz && !dense) {
    // only the non-zero words, in order: bit k of wm <-> word k has a byte
    uint32_t wm = nz_nibbles8(M[0]) | (nz_nibbles8(M[1]) << 8) | (nz_nibbles8(M[2]) << 16) | (nz_nibbles8(M[3]) << 24);
    uint32_t p = zoff;
    const uint32_t rowbase = 32u * tid;
    while (wm) {
      const uint32_t k = __ffs(wm) - 1;
      wm &= wm - 1;
      const uint32_t m = nibble_at(M, k);
      const uint32_t w = plane[swz(rowbase + k)];
      if (m & 1u) st[p] = (uint8_t)w;
      if (m & 2u) st[p + (m & 1u)] = (uint8_t)(w >> 8);
      if (m & 4u) st[p + __popc(m & 3u)] = (uint8_t)(w >> 16);
      if (m & 8u) st[p + __popc(m & 7u)] = (uint8_t)(w >> 24);
      p += __popc(m);
    }
  } else if (nz) {
    uint32_t R[4];
    rot_nibbles(M, lane, R);
    uint32_t rel = nibble_prefix(M, lane);
    const uint32_t rowbase = 32u * tid;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const uint32_t k = (lane + j) & 31;
      if (k == 0) rel = 0;
      const uint32_t m = (R[j >> 3] >> (4 * (j & 7))) & 15u;
      if (m) {
        const uint32_t w = plane[swz(rowbase + k)];
        uint32_t p = zoff + rel;
        if (m == 15u) {
          st[p] = (uint8_t)w;
          st[p + 1] = (uint8_t)(w >> 8);
          st[p + 2] = (uint8_t)(w >> 16);
          st[p + 3] = (uint8_t)(w >> 24);
        } else {
#pragma unroll
          for (int b = 0; b < 4; b++)
            if ((m >> b) & 1) st[p++] = (uint8_t)(w >> (8 * b));
        }
        rel += __popc(m);
      }
    }
  }
  if (K) {
    uint32_t p = NZ + c1off;
#pragma unroll
    for (int j = 0; j < 16; j++)
      if ((K >> j) & 1) st[p++] = (uint8_t)(M[j >> 2] >> (8 * (j & 3)));
  }
}

// Writes out a pending chunk (p, output offset sm.payload_off, both visible
// after a barrier) from its staging buffer -- or, for a raw chunk without a
// staged copy, from raw_word(w) -- and its size-table entry; the stream's last
// chunk also sets the stream size.
template <typename RawWord>
__device__ __forceinline__ void flush_chunk(const Ctl& sm, const Pend& p, const uint32_t* staging, bool raw_staged,
                                            RawWord raw_word, uint8_t* data_out, uint16_t* table_out,
                                            long long* out_size, long long chunks) {
  const unsigned long long X = sm.payload_off;
  const int nw = p.nw;
  if (p.raw && !raw_staged) {
    store_payload(data_out + X, p.csize, [&](int w) -> uint32_t { return w < nw ? raw_word(w) : 0u; });
  } else {
    store_payload(data_out + X, p.csize, [&](int w) -> uint32_t { return staging[w]; });
  }
  if (threadIdx.x == 0) {
    table_out[p.c] = (uint16_t)p.csize;
    if (p.c == chunks - 1) *out_size = HDR + 2 * chunks + (long long)(X + p.csize);
  }
}

// Inverse of DIFFMS + BIT_4 for a chunk whose BIT_4 output sits in the
// swizzled plane buffer: gathers the plane words of group g = threadIdx.x,
// transposes them back, undoes the zig-zag and the differences (in-thread
// prefix sum plus a block scan of the group totals), and returns the group's
// words in v[32] (words at or beyond nw are 0).  Ends with a barrier (the
// scan's), after which the plane buffer may be reused.
template <bool FULL>
__device__ __forceinline__ void planes_to_words(Ctl& sm, const uint32_t* plane, int nw_in, uint32_t (&v)[32]) {
  const int tid = threadIdx.x;
  const int nw = FULL ? CW : nw_in;
  const int G = nw >> 5, rem = nw & 31;
  // ---- undo BIT_4 (d_iBIT_4): gather plane words of group g, transpose.
  if (FULL) {
    uint32_t pe, po;
    plane_offsets(tid, pe, po);
    uint32_t any = 0;
#pragma unroll
    for (int s = 0; s < 32; s++) {
      v[s] = plane[128 * s + ((s & 1) ? po : pe)];
      any |= v[s];
    }
    if (any) transpose32(v);
  } else if (tid < G) {
#pragma unroll
    for (int s = 0; s < 32; s++) v[s] = plane[swz(s * G + tid)];
    transpose32(v);
  } else {
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = (tid == G && k < rem) ? plane[swz(32 * G + k)] : 0u;
  }
  // ---- undo DIFFMS (d_iDIFFMS, d_DIFFMS.h:69-102): un-zig-zag, prefix sum.
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 32; k++) {
    const uint32_t z = v[k];
    acc += (z >> 1) ^ (0u - (z & 1u));
    v[k] = acc;
  }
  uint32_t dummy;
  const uint32_t carry = block_scan_excl(acc, sm.scan_c, dummy);  // (its barrier: every plane read is done)
#pragma unroll
  for (int k = 0; k < 32; k++) v[k] += carry;
  if (!FULL && 32 * tid + 32 > nw) {
#pragma unroll
    for (int k = 0; k < 32; k++)
      if (32 * tid + k >= nw) v[k] = 0;
  }
}

// ============================================================== decode stage
// Undoes RZE_1, BIT_4 and DIFFMS for the chunk whose payload the stage's
// loads brought into P (at byte offset m.d, m.csize bytes; see StageMeta) and
// returns the pre-pipeline words of group g = threadIdx.x in v[32] (words at
// or beyond nw are 0).  raw_out reports a chunk stored uncompressed (its words
// are returned as stored).  `plane` is the swizzled buffer for the BIT_4
// planes; when it is P itself the payload is expanded into registers first
// (one more barrier) and P ends up holding the planes.  side() runs on every
// thread before the first barrier: warp 3 prefetches the next chunk there
// while warp 0 decodes this chunk's bitmaps.
template <bool FULL, typename Side>
__device__ __forceinline__ void decode_core(Ctl& sm, const Sync& sy, const StageMeta& m, uint32_t* P,
                                            uint32_t* plane, uint32_t (&v)[32], bool& raw_out, Side side) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nw = FULL ? CW : m.nw;
  const int osize = nw * 4;
  const bool inplace = plane == P;
  const uint8_t* st = reinterpret_cast<const uint8_t*>(P);
  const int csize = m.csize;
  const int d = m.d;
  side();
  raw_out = false;
  if (m.bad) {  // corrupt size entry or stream header
    if (tid == 0) latch(sy.status, m.bad == 1 ? DST_CORRUPT : DST_SIZE_MISMATCH);
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = 0;
    __syncthreads();
    return;
  }
  if (csize == osize) {
    // Stored uncompressed: realign the payload words (thread t: words
    // t + 128j, conflict-free) into the swizzled plane buffer.
    raw_out = true;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int w = tid + NT * j;
      const int o = d + 4 * w;
      v[j] = (FULL || w < nw) ? __funnelshift_r(P[o >> 2], P[(o >> 2) + 1], 8 * (o & 3)) : 0u;
    }
    if (inplace) __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int w = tid + NT * j;
      if (FULL || w < nw) plane[swz(w)] = v[j];
    }
    __syncthreads();
    row_load(plane, tid, v);
    if (!FULL && 32 * tid + 32 > nw) {
#pragma unroll
      for (int k = 0; k < 32; k++)
        if (32 * tid + k >= nw) v[k] = 0;
    }
    return;
  }
  // ---- undo RZE_1 (d_iRZE, d_RZE.h:127-206)
  const int orig = st[d + csize - 2] | (st[d + csize - 1] << 8);
  bool ok = (orig == osize);
  if (csize == 2) {
    // Trailer only: the BIT_4 output was all zero, so every word decodes to 0.
    if (!ok && tid == 0) latch(sy.status, DST_CORRUPT);
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = 0;
    __syncthreads();  // the trailer was read from P, which the caller reuses
    return;
  }
  uint32_t M[4] = {0, 0, 0, 0};
  const int T = csize - 6;
  if (warp == 0) {
    bool wok = T >= 0;
    const int Tc = T < 0 ? 0 : T;
    const uint32_t top = (uint32_t)st[d + Tc] | ((uint32_t)st[d + Tc + 1] << 8) | ((uint32_t)st[d + Tc + 2] << 16) |
                         ((uint32_t)st[d + Tc + 3] << 24);
    const int c3 = __popc(top);
    wok = wok && (c3 <= T);
    const int b3 = Tc - c3;
    const int r3 = __popc(top & (0xffffffffu >> (31 - lane))) - 1;
    const uint32_t l3 = (r3 >= 0 && wok) ? st[d + b3 + r3] : 0u;
    uint32_t c2u;
    const uint32_t e2 = warp_scan_excl(__popc(l3), c2u);
    const int c2 = (int)c2u;
    wok = wok && (c3 + c2 <= T);
    const int b2 = b3 - c2;
    uint32_t l2lo = 0, l2hi = 0;
    uint8_t prevb = 0;
    if (wok && e2 > 0) prevb = st[d + b2 + e2 - 1];
    uint32_t rk = e2;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if ((l3 >> j) & 1) prevb = wok ? st[d + b2 + rk++] : 0;
      if (j < 4) l2lo |= (uint32_t)prevb << (8 * j);
      else l2hi |= (uint32_t)prevb << (8 * (j - 4));
    }
    reinterpret_cast<uint2*>(sm.l2)[lane] = make_uint2(l2lo, l2hi);
    // RE1 rank base for segment threads 4*lane .. 4*lane+3.
    const uint32_t p0 = __popc(l2lo & 0xffffu), p1 = __popc(l2lo >> 16), p2 = __popc(l2hi & 0xffffu);
    const uint32_t p3 = __popc(l2hi >> 16);
    uint32_t c1u;
    const uint32_t e1 = warp_scan_excl(p0 + p1 + p2 + p3, c1u);
    sm.rb[4 * lane] = (uint16_t)e1;
    sm.rb[4 * lane + 1] = (uint16_t)(e1 + p0);
    sm.rb[4 * lane + 2] = (uint16_t)(e1 + p0 + p1);
    sm.rb[4 * lane + 3] = (uint16_t)(e1 + p0 + p1 + p2);
    const int c1 = (int)c1u;
    wok = wok && (c3 + c2 + c1 <= T);
    if (lane == 0) {
      sm.info[5] = wok ? (uint32_t)(b2 - c1) : 0u;  // start of RE1 data = count of ZE bytes
      sm.info[6] = wok;
    }
  }
  __syncthreads();
  const bool wok = sm.info[6];
  ok = ok && wok;
  const uint32_t zbase = sm.info[5];
  if (wok) {
    const uint32_t Kb = sm.l2[tid];
    uint32_t rk = sm.rb[tid];
    uint8_t prevb = rk > 0 ? st[d + zbase + rk - 1] : 0;
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if ((Kb >> j) & 1) prevb = st[d + zbase + rk++];
      M[j >> 2] |= (uint32_t)prevb << (8 * (j & 3));
    }
  }
  // bitmap bits beyond the chunk must be clear
  if (!FULL && 32 * tid + 32 > nw) {
#pragma unroll
    for (int k = 0; k < 32; k++)
      if (32 * tid + k >= nw) {
        const uint32_t bm = 15u << (4 * (k & 7));
        if (M[k >> 3] & bm) ok = false;
        M[k >> 3] &= ~bm;
      }
  }
  const uint32_t nz = __popc(M[0]) + __popc(M[1]) + __popc(M[2]) + __popc(M[3]);
  uint32_t NZ;
  const uint32_t zoff = block_scan_excl(nz, sm.scan_b, NZ);
  if (NZ != zbase) ok = false;
  if (!ok) latch(sy.status, DST_CORRUPT);
  // ZE decode: scatter the non-zero bytes back into the 32 words.  A warp
  // whose threads each hold at most 4 non-zero words expands just those (kept
  // in registers until every payload byte has been read) into zero-filled
  // rows; a denser warp expands all 32 words.
  uint32_t wm = ok ? (nz_nibbles8(M[0]) | (nz_nibbles8(M[1]) << 8) | (nz_nibbles8(M[2]) << 16) |
                      (nz_nibbles8(M[3]) << 24))
                   : 0u;
  if (__all_sync(0xffffffffu, __popc(wm) <= 4)) {
    uint32_t kv[4], xv[4];
    uint32_t p = (uint32_t)d + zoff;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      kv[i] = 32;
      xv[i] = 0;
      if (wm) {
        const uint32_t k = __ffs(wm) - 1;
        wm &= wm - 1;
        const uint32_t mk = nibble_at(M, k);
        const uint32_t lo = P[p >> 2], hi = P[(p >> 2) + 1];
        xv[i] = __byte_perm(__funnelshift_r(lo, hi, 8 * (p & 3)), 0u, expand_sel(mk));
        kv[i] = k;
        p += __popc(mk);
      }
    }
    if (inplace) __syncthreads();  // every payload byte has been read
    uint4* row = reinterpret_cast<uint4*>(plane + 32 * tid);
#pragma unroll
    for (int u = 0; u < 8; u++) row[u ^ (tid & 7)] = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (kv[i] < 32) plane[swz(32 * tid + kv[i])] = xv[i];
    __syncthreads();
  } else {
  uint32_t q[32];
  if (!ok || (M[0] | M[1] | M[2] | M[3]) == 0) {
#pragma unroll
    for (int k = 0; k < 32; k++) q[k] = 0;
  } else {
    uint32_t p = (uint32_t)d + zoff;
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const uint32_t mk = (M[k >> 3] >> (4 * (k & 7))) & 15u;
      uint32_t x = 0;
      if (mk) {
        const uint32_t lo = P[p >> 2], hi = P[(p >> 2) + 1];
        x = __byte_perm(__funnelshift_r(lo, hi, 8 * (p & 3)), 0u, expand_sel(mk));
        p += __popc(mk);
      }
      q[k] = x;
    }
  }
  if (inplace) __syncthreads();  // every payload byte has been read
  row_store(plane, tid, q);
  __syncthreads();
  }
  planes_to_words<FULL>(sm, plane, nw, v);
}

// The partial last chunk of a stream (at most one per stream) runs out of
// line, so the full-chunk loop body stays small enough for the instruction
// caches.  Its words pass through the calling thread's own row of the plane
// buffer (row tid = linear words 32*tid .. 32*tid+31), never through a pointer
// to the caller's register array: taking that array's address would put it in
// local memory on the hot full-chunk path as well.
// encode_stage_partial: the caller has stored its group's words in row tid of
// `plane` (row_store).
__device__ __noinline__ void encode_stage_partial(Ctl& sm, const Sync& sy, uint32_t* plane, uint8_t* st, long long c,
                                                  int nw, int item, Pend& pend) {
  uint32_t w[32];
  row_load(plane, threadIdx.x, w);
  encode_stage<false>(sm, sy, w, plane, st, c, nw, item, pend, NoHook{});
}

// decode_core_partial: leaves the group's words in row tid of `plane` (the
// caller reads them back with row_load) and returns whether the chunk was
// stored uncompressed.  decode_core ends with a barrier after which no thread
// reads another thread's row, so each thread may overwrite its own.
template <typename Side>
__device__ __noinline__ bool decode_core_partial(Ctl& sm, const Sync& sy, const StageMeta& m, uint32_t* P,
                                                 uint32_t* plane, Side side) {
  uint32_t w[32];
  bool raw = false;
  decode_core<false>(sm, sy, m, P, plane, w, raw, side);
  row_store(plane, threadIdx.x, w);
  return raw;
}

}  // namespace cortado
